"""methods_cython.methods (reference methods.pyx:61-258): OutputResult,
GlobalSpaiMethods / InnerOuterMethods and their instances, with the same
arguments, defaults and errors, on the device."""
from parallellocallyoptimalapproximatesparsematrixinverses_b200.methods import (GlobalSpaiMethods, InnerOuterMethods,
                                                                                  OutputResult, global_spai,
                                                                                  inner_outer)

__all__ = ['GlobalSpaiMethods', 'InnerOuterMethods', 'OutputResult', 'global_spai', 'inner_outer']
