"""The reference's import name: ``import wtet`` runs the B200 library.

half-potato/wtet ships its Python API as package ``wtet`` with the compiled
module ``wtet._core`` (python/wtet/__init__.py:48-69, pyproject.toml:48-51).
This package re-exports the same names from wtet_b200, so code written
against the reference keeps working unchanged; the additions (batched and
device-resident calls, verification, canonical form) are re-exported too.
"""
from wtet_b200 import *  # noqa: F401,F403
from wtet_b200 import __all__, __version__  # noqa: F401

from . import _core  # noqa: F401
