"""methods_cython.backward_error (reference backward_error.pyx:45-144):
parallel_threads, matvec and pcg with the (history, status) contract, on the
device."""
from parallellocallyoptimalapproximatesparsematrixinverses_b200.backward_error import matvec, parallel_threads, pcg

__all__ = ['matvec', 'parallel_threads', 'pcg']
