"""B200-native two-electron integral path of Quax."""
