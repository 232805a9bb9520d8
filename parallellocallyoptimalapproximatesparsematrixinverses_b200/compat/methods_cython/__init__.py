"""Drop-in for the reference's methods_cython package (methods_cython/__init__.py):
the same exported names, served by libspai_b200.so."""
from .methods import OutputResult, global_spai, inner_outer

__all__ = ['OutputResult', 'global_spai', 'inner_outer']
