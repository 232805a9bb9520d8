"""B200-native Global SPAI / Inner-Outer sparse approximate inverses and the
PCG evaluator, behind the reference's C ABI (include/methods_c_api.h) and its
methods_cython Python surface.

    from parallellocallyoptimalapproximatesparsematrixinverses_b200 import global_spai, inner_outer, pcg
"""
from .backward_error import matvec, parallel_threads, pcg
from .methods import GlobalSpaiMethods, InnerOuterMethods, OutputResult, Session, global_spai, inner_outer

__all__ = [
    "GlobalSpaiMethods", "InnerOuterMethods", "OutputResult", "Session", "global_spai", "inner_outer",
    "matvec", "parallel_threads", "pcg",
]
