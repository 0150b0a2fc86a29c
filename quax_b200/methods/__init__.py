"""Consumers of the integral path (RHF), mirroring quax/methods."""
