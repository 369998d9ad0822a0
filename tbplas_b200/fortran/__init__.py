"""Drop-in replacement of the reference package `tbplas.fortran` (f2py module)."""
from . import f2py

__all__ = ["f2py"]
