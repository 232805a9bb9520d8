"""Import shims for callers of the reference's compiled modules.

Put this directory on sys.path (next to the repository root) and
`import methods_cython` resolves to the device library with the reference's
names: methods_cython.{global_spai, inner_outer, OutputResult} and
methods_cython.backward_error.{matvec, pcg, parallel_threads}
(reference methods_cython/__init__.py, methods.pyx, backward_error.pyx).
"""
