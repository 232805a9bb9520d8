#pragma once
// Minimum-norm least-squares solve of a symmetric-scaled 2x2 system
// (reference src/common/sparse_operations.cpp:58-73, which calls Eigen's
// completeOrthogonalDecomposition).  The decomposition is restated from its
// published algorithm: Householder QR with column pivoting (pivot = larger
// column norm, LAPACK-style norm downdating), rank = number of |R_ii| above
// 2 * eps * max|R_ii|, and for rank 1 a right Householder reflection that
// zeroes R_12 (complete orthogonal decomposition), then back substitution.
// Used on the host for the global LOMR step and on the device for the
// per-column Inner-Outer LOMR steps; both must round identically, so every
// operation is an explicit IEEE multiply/add/divide/sqrt.

#include <cmath>
#include <cstdint>

namespace spai {

#ifdef __CUDACC__
#define SPAI_HD __host__ __device__
#else
#define SPAI_HD
#endif

namespace cod_detail {

SPAI_HD inline double Mul(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dmul_rn(a, b);
#else
  return a * b;
#endif
}
SPAI_HD inline double Add(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dadd_rn(a, b);
#else
  return a + b;
#endif
}
SPAI_HD inline double Sub(double a, double b) {
#ifdef __CUDA_ARCH__
  return __dsub_rn(a, b);
#else
  return a - b;
#endif
}
SPAI_HD inline double Div(double a, double b) {
#ifdef __CUDA_ARCH__
  return __ddiv_rn(a, b);
#else
  return a / b;
#endif
}
SPAI_HD inline double Sqrt(double a) {
#ifdef __CUDA_ARCH__
  return __dsqrt_rn(a);
#else
  return std::sqrt(a);
#endif
}
SPAI_HD inline bool Finite(double v) {
#ifdef __CUDA_ARCH__
  return isfinite(v);
#else
  return std::isfinite(v);
#endif
}

constexpr double kEps = 2.220446049250313080847e-16;
constexpr double kMinNormal = 2.2250738585072014e-308;

struct Reflector {
  double tau;
  double beta;
  double essential;
};

// H = I - tau v v^T, v = (1, essential), maps (head, tail) to (beta, 0).
SPAI_HD inline Reflector Make(double head, double tail, bool has_tail) {
  Reflector h;
  const double tail_sq = has_tail ? Mul(tail, tail) : 0.0;
  if (tail_sq <= kMinNormal) {
    h.tau = 0.0;
    h.beta = head;
    h.essential = 0.0;
    return h;
  }
  double beta = Sqrt(Add(Mul(head, head), tail_sq));
  if (head >= 0.0) beta = -beta;
  h.beta = beta;
  h.essential = Div(tail, Sub(head, beta));
  h.tau = Div(Sub(beta, head), beta);
  return h;
}

SPAI_HD inline void Apply(const Reflector& h, double& u0, double& u1) {
  if (h.tau == 0.0) return;
  double t = Mul(h.essential, u1);
  t = Add(t, u0);
  u0 = Sub(u0, Mul(h.tau, t));
  u1 = Sub(u1, Mul(Mul(h.tau, h.essential), t));
}

SPAI_HD inline void Swap(double& a, double& b) {
  const double t = a;
  a = b;
  b = t;
}

// s: scaled matrix (row major), rhs: scaled right-hand side.
SPAI_HD inline void CodSolve(const double s[4], const double rhs[2], double out[2]) {
  double q00 = s[0], q01 = s[1], q10 = s[2], q11 = s[3];
  double direct0 = Sqrt(Add(Mul(q00, q00), Mul(q10, q10)));
  double direct1 = Sqrt(Add(Mul(q01, q01), Mul(q11, q11)));
  double upd0 = direct0;
  double upd1 = direct1;
  const double max_norm = upd1 > upd0 ? upd1 : upd0;
  const double scaled = Mul(max_norm, kEps);
  const double threshold_helper = Div(Mul(scaled, scaled), 2.0);
  const double downdate_threshold = Sqrt(kEps);
  int nonzero_pivots = 2;
  double max_pivot = 0.0;
  const bool pivot = upd1 > upd0;
  const double biggest = pivot ? upd1 : upd0;
  if (Mul(biggest, biggest) < Mul(threshold_helper, 2.0)) nonzero_pivots = 0;
  if (pivot) {
    Swap(q00, q01);
    Swap(q10, q11);
    Swap(upd0, upd1);
    Swap(direct0, direct1);
  }
  const Reflector h0 = Make(q00, q10, true);
  q00 = h0.beta;
  q10 = h0.essential;
  if (fabs(h0.beta) > max_pivot) max_pivot = fabs(h0.beta);
  Apply(h0, q01, q11);
  if (upd1 != 0.0) {
    double temp = Div(fabs(q01), upd1);
    temp = Mul(Add(1.0, temp), Sub(1.0, temp));
    temp = temp < 0.0 ? 0.0 : temp;
    const double ratio = Div(upd1, direct1);
    const double temp2 = Mul(temp, Mul(ratio, ratio));
    if (temp2 <= downdate_threshold) {
      direct1 = Sqrt(Mul(q11, q11));
      upd1 = direct1;
    } else {
      upd1 = Mul(upd1, Sqrt(temp));
    }
  }
  if (nonzero_pivots == 2 && Mul(upd1, upd1) < threshold_helper) nonzero_pivots = 1;
  if (fabs(q11) > max_pivot) max_pivot = fabs(q11);
  const double rank_threshold = Mul(fabs(max_pivot), Mul(kEps, 2.0));
  int rank = 0;
  if (nonzero_pivots > 0 && fabs(q00) > rank_threshold) ++rank;
  if (nonzero_pivots > 1 && fabs(q11) > rank_threshold) ++rank;
  if (rank == 0) {
    out[0] = 0.0;
    out[1] = 0.0;
    return;
  }
  Reflector zh{0.0, 0.0, 0.0};
  if (rank == 1) {
    zh = Make(q00, q01, true);
    q00 = zh.beta;
    q01 = zh.essential;
  }
  double c0 = rhs[0];
  double c1 = rhs[1];
  Apply(h0, c0, c1);
  double y0;
  double y1;
  if (rank == 2) {
    if (c1 != 0.0) {
      c1 = Div(c1, q11);
      c0 = Sub(c0, Mul(c1, q01));
    }
    if (c0 != 0.0) c0 = Div(c0, q00);
    y0 = c0;
    y1 = c1;
  } else {
    if (c0 != 0.0) c0 = Div(c0, q00);
    y0 = c0;
    y1 = 0.0;
    Apply(zh, y0, y1);
  }
  if (pivot) Swap(y0, y1);
  out[0] = y0;
  out[1] = y1;
}

}  // namespace cod_detail

// m: row-major 2x2, x: right-hand side; non-finite input or output gives 0.
SPAI_HD inline void SolveLeastSquares2x2(const double m[4], const double x[2], double out[2]) {
  using namespace cod_detail;
  out[0] = 0.0;
  out[1] = 0.0;
  if (!Finite(m[0]) || !Finite(m[1]) || !Finite(m[2]) || !Finite(m[3]) || !Finite(x[0]) || !Finite(x[1])) return;
  double scale[2];
  for (int i = 0; i < 2; ++i) {
    const double root = Sqrt(fabs(m[3 * i]));
    scale[i] = root > 0.0 ? Div(1.0, root) : 1.0;
  }
  const double s[4] = {Mul(Mul(scale[0], m[0]), scale[0]), Mul(Mul(scale[0], m[1]), scale[1]),
                       Mul(Mul(scale[1], m[2]), scale[0]), Mul(Mul(scale[1], m[3]), scale[1])};
  const double rhs[2] = {Mul(scale[0], x[0]), Mul(scale[1], x[1])};
  double y[2];
  CodSolve(s, rhs, y);
  out[0] = Mul(scale[0], y[0]);
  out[1] = Mul(scale[1], y[1]);
  if (!Finite(out[0]) || !Finite(out[1])) {
    out[0] = 0.0;
    out[1] = 0.0;
  }
}

}  // namespace spai
