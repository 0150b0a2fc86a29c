"""Two-electron integral path: C-ABI binding, device engine, reference-shaped API.

Importing this package loads nothing on the GPU; ``libint_interface`` loads the
shared library on import (like the reference's module, quax/integrals/__init__.py).
"""
from .engine import EriEngine  # noqa: F401
