// TEST INFRASTRUCTURE ONLY -- CPU restatement ("oracle") of the reference's SPAI
// (src/common, src/global_spai, src/inner_outer) and PCG
// (methods_cython/backward_error.pyx) hot path.  It is the checker for the CUDA
// library and the CPU baseline in bench.py; the product never links it.
//
// The reference computes on Eigen 3 (Debian libeigen3-dev 3.4.0 in its
// Dockerfile; Eigen is not vendored and not installed here).  The arithmetic
// this file restates from Eigen's published algorithms:
//   * sparse x sparse product: Gustavson column by column; each output entry is
//     the first product x*y, then += x*y in ascending k of the right operand's
//     column; no FMA; structural zeros from cancellation are kept;
//   * prune(ref, eps): keep an entry iff !(|v| <= |ref| * eps);
//   * sparse sum/cwiseProduct/squaredNorm/dot: sequential in storage order;
//   * sparse a + b: union; an entry present on one side only is v + 0.0 / 0.0 + v;
//   * completeOrthogonalDecomposition of a 2x2: column-pivoted Householder QR,
//     rank threshold eps * 2 * max pivot, right Householder for rank 1.
// Every function cites the reference lines it follows.

#include "spai_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <numeric>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <omp.h>

namespace {

// methods_common.hpp:32 -- relative threshold for pruning.
constexpr double kEps = std::numeric_limits<double>::epsilon();
// include/methods.hpp:15 -- smallest accepted max_density.
constexpr double kMinDensity = 1e-9;

// ---------------------------------------------------------------------------
// Compressed sparse column matrix with int64 indices (include/methods.hpp:17).
struct Csc {
  int64_t rows = 0;
  int64_t cols = 0;
  std::vector<int64_t> ptr;
  std::vector<int64_t> idx;
  std::vector<double> val;

  Csc() : ptr(1, 0) {}
  Csc(int64_t r, int64_t c) : rows(r), cols(c), ptr(c + 1, 0) {}
  int64_t nnz() const { return ptr.back(); }
};

inline bool IsNonZero(double v) { return !(std::fabs(v) <= 0.0); }

// Eigen prune(0.0): remove entries with |v| <= 0 (NaN survives).
void DropZeros(Csc& x) {
  int64_t out = 0;
  int64_t start = 0;
  for (int64_t j = 0; j < x.cols; ++j) {
    const int64_t end = x.ptr[j + 1];
    for (int64_t p = start; p < end; ++p) {
      if (IsNonZero(x.val[p])) {
        x.idx[out] = x.idx[p];
        x.val[out] = x.val[p];
        ++out;
      }
    }
    start = end;
    x.ptr[j + 1] = out;
  }
  x.idx.resize(out);
  x.val.resize(out);
}

template <class Keep>
void PruneIf(Csc& x, Keep keep) {
  int64_t out = 0;
  int64_t start = 0;
  for (int64_t j = 0; j < x.cols; ++j) {
    const int64_t end = x.ptr[j + 1];
    for (int64_t p = start; p < end; ++p) {
      if (keep(x.idx[p], j, x.val[p])) {
        x.idx[out] = x.idx[p];
        x.val[out] = x.val[p];
        ++out;
      }
    }
    start = end;
    x.ptr[j + 1] = out;
  }
  x.idx.resize(out);
  x.val.resize(out);
}

struct Work {
  std::vector<char> seen;
  std::vector<double> acc;
  std::vector<int64_t> rows;
  void Ensure(int64_t n) {
    if (static_cast<int64_t>(seen.size()) < n) {
      seen.assign(n, 0);
      acc.assign(n, 0.0);
    }
  }
};

// C = X * B, conservative Gustavson (state_manager.cpp:59; dropping.cpp:98).
Csc Product(const Csc& x, const Csc& b, Work& w) {
  w.Ensure(x.rows);
  Csc c(x.rows, b.cols);
  for (int64_t j = 0; j < b.cols; ++j) {
    w.rows.clear();
    for (int64_t pb = b.ptr[j]; pb < b.ptr[j + 1]; ++pb) {
      const int64_t k = b.idx[pb];
      const double y = b.val[pb];
      for (int64_t px = x.ptr[k]; px < x.ptr[k + 1]; ++px) {
        const int64_t i = x.idx[px];
        const double prod = x.val[px] * y;
        if (!w.seen[i]) {
          w.seen[i] = 1;
          w.acc[i] = prod;
          w.rows.push_back(i);
        } else {
          w.acc[i] += prod;
        }
      }
    }
    std::sort(w.rows.begin(), w.rows.end());
    for (const int64_t i : w.rows) {
      c.idx.push_back(i);
      c.val.push_back(w.acc[i]);
      w.seen[i] = 0;
    }
    c.ptr[j + 1] = static_cast<int64_t>(c.idx.size());
  }
  return c;
}

// R = I - A*M for the columns [first, first + M.cols) (dropping.cpp:97-104):
// the product is negated, 1.0 is added on the global diagonal (inserted when
// absent), then exact zeros are pruned.
Csc Residual(const Csc& a, const Csc& m, int64_t first, Work& w) {
  Csc am = Product(a, m, w);
  Csc r(am.rows, am.cols);
  r.idx.reserve(am.nnz() + am.cols);
  r.val.reserve(am.nnz() + am.cols);
  for (int64_t j = 0; j < am.cols; ++j) {
    const int64_t diag = first + j;
    bool placed = false;
    for (int64_t p = am.ptr[j]; p < am.ptr[j + 1]; ++p) {
      const int64_t i = am.idx[p];
      if (!placed && i > diag) {
        r.idx.push_back(diag);
        r.val.push_back(1.0);
        placed = true;
      }
      double v = -am.val[p];
      if (i == diag) {
        v = v + 1.0;
        placed = true;
      }
      r.idx.push_back(i);
      r.val.push_back(v);
    }
    if (!placed) {
      r.idx.push_back(diag);
      r.val.push_back(1.0);
    }
    r.ptr[j + 1] = static_cast<int64_t>(r.idx.size());
  }
  DropZeros(r);
  return r;
}

// Union combination out = ys*Y (+) xs*X with the Eigen conventions for
// one-sided entries.  scale_y == false means Y enters unscaled.
Csc Union(const Csc& y, bool scale_y, double ys, const Csc& x, double xs) {
  Csc out(y.rows, y.cols);
  out.idx.reserve(y.nnz() + x.nnz());
  out.val.reserve(y.nnz() + x.nnz());
  for (int64_t j = 0; j < y.cols; ++j) {
    int64_t p = y.ptr[j];
    int64_t q = x.ptr[j];
    const int64_t pe = y.ptr[j + 1];
    const int64_t qe = x.ptr[j + 1];
    while (p < pe || q < qe) {
      if (p < pe && q < qe && y.idx[p] == x.idx[q]) {
        const double yv = scale_y ? ys * y.val[p] : y.val[p];
        out.idx.push_back(y.idx[p]);
        out.val.push_back(yv + xs * x.val[q]);
        ++p;
        ++q;
      } else if (p < pe && (q >= qe || y.idx[p] < x.idx[q])) {
        const double yv = scale_y ? ys * y.val[p] : y.val[p];
        out.idx.push_back(y.idx[p]);
        out.val.push_back(yv + 0.0);
        ++p;
      } else {
        out.idx.push_back(x.idx[q]);
        out.val.push_back(0.0 + xs * x.val[q]);
        ++q;
      }
    }
    out.ptr[j + 1] = static_cast<int64_t>(out.idx.size());
  }
  return out;
}

// t <- t + c*d, then exact zeros pruned (sparse_operations.cpp:41-49).
void AddScaled(Csc& t, const Csc& d, double c) {
  if (c != 0.0) {
    t = Union(t, false, 1.0, d, c);
  }
  DropZeros(t);
}

// y <- b*y + a*x, then exact zeros pruned (sparse_operations.cpp:22-26).
void LinComb(const Csc& x, double a, Csc& y, double b) {
  y = Union(y, true, b, x, a);
  DropZeros(y);
}

// Column j scaled by a[j], then exact zeros pruned (sparse_operations.cpp:28-39).
void ScaleColumns(Csc& x, const std::vector<double>& a) {
  for (int64_t j = 0; j < x.cols; ++j) {
    for (int64_t p = x.ptr[j]; p < x.ptr[j + 1]; ++p) {
      x.val[p] *= a[j];
    }
  }
  DropZeros(x);
}

Csc Transpose(const Csc& x) {
  Csc t(x.cols, x.rows);
  std::vector<int64_t> count(x.rows + 1, 0);
  for (int64_t p = 0; p < x.nnz(); ++p) {
    ++count[x.idx[p] + 1];
  }
  for (int64_t i = 0; i < x.rows; ++i) {
    count[i + 1] += count[i];
  }
  t.ptr = count;
  t.idx.resize(x.nnz());
  t.val.resize(x.nnz());
  std::vector<int64_t> cursor(count.begin(), count.end() - 1);
  for (int64_t j = 0; j < x.cols; ++j) {
    for (int64_t p = x.ptr[j]; p < x.ptr[j + 1]; ++p) {
      const int64_t dst = cursor[x.idx[p]]++;
      t.idx[dst] = j;
      t.val[dst] = x.val[p];
    }
  }
  return t;
}

// Columns [first, first+width) of a matrix.
Csc Columns(const Csc& x, int64_t first, int64_t width) {
  Csc out(x.rows, width);
  const int64_t base = x.ptr[first];
  for (int64_t j = 0; j <= width; ++j) {
    out.ptr[j] = x.ptr[first + j] - base;
  }
  out.idx.assign(x.idx.begin() + base, x.idx.begin() + x.ptr[first + width]);
  out.val.assign(x.val.begin() + base, x.val.begin() + x.ptr[first + width]);
  return out;
}

// Sequential accumulations inside one column (Eigen storage-order sums).
inline void AccSquares(const Csc& x, int64_t j, double& s) {
  for (int64_t p = x.ptr[j]; p < x.ptr[j + 1]; ++p) {
    s += x.val[p] * x.val[p];
  }
}

inline void AccDot(const Csc& x, const Csc& y, int64_t j, double& s) {
  int64_t p = x.ptr[j];
  int64_t q = y.ptr[j];
  const int64_t pe = x.ptr[j + 1];
  const int64_t qe = y.ptr[j + 1];
  while (p < pe && q < qe) {
    if (x.idx[p] == y.idx[q]) {
      s += x.val[p] * y.val[q];
      ++p;
      ++q;
    } else if (x.idx[p] < y.idx[q]) {
      ++p;
    } else {
      ++q;
    }
  }
}

double ColumnDot(const Csc& x, const Csc& y, int64_t j) {
  double s = 0.0;
  AccDot(x, y, j, s);
  return s;
}

double ColumnSquares(const Csc& x, int64_t j) {
  double s = 0.0;
  AccSquares(x, j, s);
  return s;
}

// binary-search lookup; 0 when the entry is absent (Eigen coeff()).
double Coeff(const Csc& x, int64_t row, int64_t col) {
  const auto begin = x.idx.begin() + x.ptr[col];
  const auto end = x.idx.begin() + x.ptr[col + 1];
  const auto it = std::lower_bound(begin, end, row);
  if (it != end && *it == row) {
    return x.val[it - x.idx.begin()];
  }
  return 0.0;
}

// ---------------------------------------------------------------------------
// The fixed summation tree of the CUDA library: chunks of 4096 values, each
// folded by 256 lanes (lane t adds values t, t+256, ... in order) and a
// butterfly over the lanes with strides 128, 64, ..., 1; repeated over the
// chunk sums until one value is left.
double TreeSum(const double* values, int64_t count) {
  constexpr int64_t kLanes = 256;
  constexpr int64_t kChunk = 4096;
  if (count <= 0) {
    return 0.0;
  }
  std::vector<double> level(values, values + count);
  do {
    const int64_t chunks = (count + kChunk - 1) / kChunk;
    std::vector<double> next(chunks);
    double lane[kLanes];
    double tmp[kLanes];
    for (int64_t c = 0; c < chunks; ++c) {
      for (int64_t t = 0; t < kLanes; ++t) {
        double s = 0.0;
        for (int64_t m = 0; m < kChunk / kLanes; ++m) {
          const int64_t i = c * kChunk + t + kLanes * m;
          if (i < count) {
            s += level[i];
          }
        }
        lane[t] = s;
      }
      for (int64_t stride = kLanes / 2; stride >= 1; stride /= 2) {
        for (int64_t t = 0; t < kLanes; ++t) {
          tmp[t] = lane[t] + lane[t ^ stride];
        }
        std::memcpy(lane, tmp, sizeof(lane));
      }
      next[c] = lane[0];
    }
    level.swap(next);
    count = chunks;
  } while (count > 1);
  return level[0];
}

// ---------------------------------------------------------------------------
// 2x2 minimum-norm least squares (sparse_operations.cpp:58-73).
struct Reflector {
  double tau = 0.0;
  double beta = 0.0;
  double essential = 0.0;
};

// H = I - tau*v*v^T with v = (1, essential) maps (c0, tail) to (beta, 0).
Reflector MakeReflector(double c0, double tail, bool has_tail) {
  Reflector h;
  const double tail_sq = has_tail ? tail * tail : 0.0;
  if (tail_sq <= std::numeric_limits<double>::min()) {
    h.tau = 0.0;
    h.beta = c0;
    h.essential = 0.0;
    return h;
  }
  double beta = std::sqrt(c0 * c0 + tail_sq);
  if (c0 >= 0.0) {
    beta = -beta;
  }
  h.beta = beta;
  h.essential = tail / (c0 - beta);
  h.tau = (beta - c0) / beta;
  return h;
}

void ApplyReflector(const Reflector& h, double& u0, double& u1) {
  if (h.tau == 0.0) {
    return;
  }
  double t = h.essential * u1;
  t = t + u0;
  u0 = u0 - h.tau * t;
  u1 = u1 - (h.tau * h.essential) * t;
}

// Complete orthogonal decomposition solve of a 2x2 (already scaled) system.
void CodSolve2x2(const double s[2][2], const double rhs[2], double out[2]) {
  double q[2][2] = {{s[0][0], s[0][1]}, {s[1][0], s[1][1]}};
  double norm_direct[2];
  double norm_updated[2];
  for (int j = 0; j < 2; ++j) {
    norm_direct[j] = std::sqrt(q[0][j] * q[0][j] + q[1][j] * q[1][j]);
    norm_updated[j] = norm_direct[j];
  }
  const double max_norm = norm_updated[1] > norm_updated[0] ? norm_updated[1] : norm_updated[0];
  const double threshold_helper = (max_norm * kEps) * (max_norm * kEps) / 2.0;
  const double downdate_threshold = std::sqrt(kEps);
  int nonzero_pivots = 2;
  double max_pivot = 0.0;

  // pivot step 0
  const int pivot = norm_updated[1] > norm_updated[0] ? 1 : 0;
  const double biggest_sq = norm_updated[pivot] * norm_updated[pivot];
  if (nonzero_pivots == 2 && biggest_sq < threshold_helper * 2.0) {
    nonzero_pivots = 0;
  }
  if (pivot == 1) {
    std::swap(q[0][0], q[0][1]);
    std::swap(q[1][0], q[1][1]);
    std::swap(norm_updated[0], norm_updated[1]);
    std::swap(norm_direct[0], norm_direct[1]);
  }
  const Reflector h0 = MakeReflector(q[0][0], q[1][0], true);
  q[0][0] = h0.beta;
  q[1][0] = h0.essential;
  if (std::fabs(h0.beta) > max_pivot) {
    max_pivot = std::fabs(h0.beta);
  }
  ApplyReflector(h0, q[0][1], q[1][1]);
  if (norm_updated[1] != 0.0) {
    double temp = std::fabs(q[0][1]) / norm_updated[1];
    temp = (1.0 + temp) * (1.0 - temp);
    temp = temp < 0.0 ? 0.0 : temp;
    const double ratio = norm_updated[1] / norm_direct[1];
    const double temp2 = temp * (ratio * ratio);
    if (temp2 <= downdate_threshold) {
      norm_direct[1] = std::sqrt(q[1][1] * q[1][1]);
      norm_updated[1] = norm_direct[1];
    } else {
      norm_updated[1] *= std::sqrt(temp);
    }
  }
  // pivot step 1 (single remaining column, reflector of length 1 is identity)
  const double last_sq = norm_updated[1] * norm_updated[1];
  if (nonzero_pivots == 2 && last_sq < threshold_helper * 1.0) {
    nonzero_pivots = 1;
  }
  if (std::fabs(q[1][1]) > max_pivot) {
    max_pivot = std::fabs(q[1][1]);
  }

  const double rank_threshold = std::fabs(max_pivot) * (kEps * 2.0);
  int rank = 0;
  for (int i = 0; i < nonzero_pivots; ++i) {
    rank += std::fabs(q[i][i]) > rank_threshold ? 1 : 0;
  }
  if (rank == 0) {
    out[0] = 0.0;
    out[1] = 0.0;
    return;
  }
  Reflector zh;
  if (rank == 1) {
    zh = MakeReflector(q[0][0], q[0][1], true);
    q[0][0] = zh.beta;
    q[0][1] = zh.essential;
  }
  double c0 = rhs[0];
  double c1 = rhs[1];
  ApplyReflector(h0, c0, c1);
  double y0 = 0.0;
  double y1 = 0.0;
  if (rank == 2) {
    if (c1 != 0.0) {
      c1 /= q[1][1];
      c0 -= c1 * q[0][1];
    }
    if (c0 != 0.0) {
      c0 /= q[0][0];
    }
    y0 = c0;
    y1 = c1;
  } else {
    if (c0 != 0.0) {
      c0 /= q[0][0];
    }
    y0 = c0;
    y1 = 0.0;
    ApplyReflector(zh, y0, y1);
  }
  if (pivot == 1) {
    std::swap(y0, y1);
  }
  out[0] = y0;
  out[1] = y1;
}

void SolveLeastSquares2x2(const double m[2][2], const double x[2], double out[2]) {
  out[0] = 0.0;
  out[1] = 0.0;
  for (int i = 0; i < 2; ++i) {
    if (!std::isfinite(x[i]) || !std::isfinite(m[i][0]) || !std::isfinite(m[i][1])) {
      return;
    }
  }
  double scale[2];
  for (int i = 0; i < 2; ++i) {
    const double root = std::sqrt(std::fabs(m[i][i]));
    scale[i] = root > 0.0 ? 1.0 / root : 1.0;
  }
  double s[2][2];
  for (int i = 0; i < 2; ++i) {
    for (int j = 0; j < 2; ++j) {
      s[i][j] = (scale[i] * m[i][j]) * scale[j];
    }
  }
  const double rhs[2] = {scale[0] * x[0], scale[1] * x[1]};
  double y[2];
  CodSolve2x2(s, rhs, y);
  out[0] = scale[0] * y[0];
  out[1] = scale[1] * y[1];
  if (!std::isfinite(out[0]) || !std::isfinite(out[1])) {
    out[0] = 0.0;
    out[1] = 0.0;
  }
}

// sparse_operations.cpp:10-20
inline bool IsFiniteNonZero(double v) { return std::isfinite(v) && std::fabs(v) > 0.0; }

inline double SafeQuotient(double num, double den) {
  if (!IsFiniteNonZero(den)) {
    return 0.0;
  }
  const double q = num / den;
  return std::isfinite(q) ? q : 0.0;
}

// ---------------------------------------------------------------------------
enum class Mat { M, R, Z, P, AP, AZ, Tmp, Q };

struct Batch {
  int64_t first = 0;
  int64_t width = 0;
  Csc m, r, z, p, ap, az, tmp, q;

  Csc& Get(Mat t) {
    switch (t) {
      case Mat::M: return m;
      case Mat::R: return r;
      case Mat::Z: return z;
      case Mat::P: return p;
      case Mat::AP: return ap;
      case Mat::AZ: return az;
      case Mat::Tmp: return tmp;
      case Mat::Q: return q;
    }
    return tmp;
  }
  const Csc& Get(Mat t) const { return const_cast<Batch*>(this)->Get(t); }
};

struct Params {
  Csc a;
  Csc m0;
  Csc pr;
  bool has_m0 = false;
  bool has_pr = false;
  int64_t max_iterations = 100;
  double tolerance = 1e-9;
  double max_density = 0.03;
  bool dropping = true;
  int64_t num_threads = 1;
  int64_t inner_iterations = 2;
};

struct History {
  std::vector<SingleIterationData> rows;
  double initial_residual = 0.0;
  int64_t iterations = 0;
  bool converged = false;
};

class State {
 public:
  State(const Params& params, const OracleOptions& options, bool symmetric)
      : params_(params), symmetric_(symmetric), order_(options.order), topk_(options.topk_per_column) {
    Validate();
    n_ = params.a.cols;
    if (params.num_threads <= 0) {
      throw std::invalid_argument("Invalid threads count value");
    }
    int64_t batches = options.batch_count > 0 ? options.batch_count : params.num_threads;
    batches = std::min(batches, n_);
    threads_ = static_cast<int>(options.omp_threads > 0 ? options.omp_threads : std::min<int64_t>(batches, omp_get_max_threads()));
    threads_ = std::max(1, threads_);
    work_.resize(threads_);
    InitBatches(batches);
    if (params.dropping) {
      col_norm2_.assign(n_, 0.0);
      for (int64_t k = 0; k < n_; ++k) {
        col_norm2_[k] = ColumnSquares(params.a, k);
      }
    } else {
      col_norm2_.assign(n_, 0.0);
    }
    pr_ = params.has_pr ? params.pr : DiagonalInverse(params.a);
    if (params.dropping) {
      ApplyDroppingStrategy();
    } else {
      ForBatches([&](Batch& b, Work& w) { b.r = Residual(params_.a, b.m, b.first, w); });
    }
    history_.initial_residual = ResidualNorm();
  }

  // ---- glue used by the methods -------------------------------------------
  int64_t n() const { return n_; }
  const Params& params() const { return params_; }
  const Csc& a() const { return params_.a; }
  const Csc& pr() const { return pr_; }
  std::vector<Batch>& batches() { return batches_; }
  History& history() { return history_; }

  template <class F>
  void ForBatches(F f) {
    const int64_t count = static_cast<int64_t>(batches_.size());
    if (threads_ == 1) {
      for (int64_t b = 0; b < count; ++b) {
        f(batches_[b], work_[0]);
      }
      return;
    }
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads_)
    for (int64_t b = 0; b < count; ++b) {
      f(batches_[b], work_[omp_get_thread_num()]);
    }
  }

  // Global sum of per-entry terms: acc(batch, local column, running sum).
  template <class Acc>
  double GlobalSum(Acc acc) {
    if (order_ == 0) {
      std::vector<double> partial(batches_.size(), 0.0);
      for (size_t b = 0; b < batches_.size(); ++b) {
        double s = 0.0;
        for (int64_t j = 0; j < batches_[b].width; ++j) {
          acc(batches_[b], j, s);
        }
        partial[b] = s;
      }
      double total = 0.0;
      for (const double v : partial) {
        total += v;
      }
      return total;
    }
    std::vector<double> column(n_, 0.0);
    for (auto& b : batches_) {
      for (int64_t j = 0; j < b.width; ++j) {
        double s = 0.0;
        acc(b, j, s);
        column[b.first + j] = s;
      }
    }
    return TreeSum(column.data(), n_);
  }

  double Dot(Mat x, Mat y) {
    return GlobalSum([&](const Batch& b, int64_t j, double& s) { AccDot(b.Get(x), b.Get(y), j, s); });
  }

  double SquaredNorm(Mat x) {
    return GlobalSum([&](const Batch& b, int64_t j, double& s) { AccSquares(b.Get(x), j, s); });
  }

  double ResidualNorm() { return std::sqrt(SquaredNorm(Mat::R)); }

  // MultiplyBatches (state_manager.cpp:47-66): exact zeros are pruned only
  // when dropping is disabled.
  void Multiply(const Csc& left, Mat in, Mat out) {
    ForBatches([&](Batch& b, Work& w) {
      b.Get(out) = Product(left, b.Get(in), w);
      if (!params_.dropping) {
        DropZeros(b.Get(out));
      }
    });
  }

  void RecomputeResidual() {
    ForBatches([&](Batch& b, Work& w) { b.r = Residual(params_.a, b.m, b.first, w); });
  }

  int64_t CountNonZeros(Mat t) const {
    int64_t total = 0;
    for (const auto& b : batches_) {
      total += b.Get(t).nnz();
    }
    return total;
  }

  // state_manager.cpp:68-71
  int64_t MaxNonZeros() const {
    const double limit = params_.max_density * static_cast<double>(n_) * static_cast<double>(n_);
    return std::max(n_, static_cast<int64_t>(std::floor(limit)));
  }

  Csc AssembleM() const {
    Csc out(n_, n_);
    for (const auto& b : batches_) {
      const int64_t base = static_cast<int64_t>(out.idx.size());
      for (int64_t j = 0; j < b.width; ++j) {
        out.ptr[b.first + j + 1] = base + b.m.ptr[j + 1];
      }
      out.idx.insert(out.idx.end(), b.m.idx.begin(), b.m.idx.end());
      out.val.insert(out.val.end(), b.m.val.begin(), b.m.val.end());
    }
    return out;
  }

  // M := 0.5 * (M + M^T) (dropping.cpp:106-120).
  void EnsureSymmetry() {
    if (!symmetric_) {
      return;
    }
    const Csc full = AssembleM();
    const Csc trans = Transpose(full);
    ForBatches([&](Batch& b, Work&) {
      const Csc left = Columns(full, b.first, b.width);
      const Csc right = Columns(trans, b.first, b.width);
      Csc sum = Union(left, false, 1.0, right, 1.0);
      for (double& v : sum.val) {
        v = 0.5 * v;
      }
      b.m = std::move(sum);
    });
  }

  // dropping.cpp:122-175 (global budget) or the per-column top-k variant.
  void ApplyDroppingStrategy() {
    EnsureSymmetry();
    ForBatches([&](Batch& b, Work& w) {
      std::vector<double> threshold(b.width);
      for (int64_t j = 0; j < b.width; ++j) {
        threshold[j] = kEps * std::sqrt(ColumnSquares(b.m, j));
      }
      PruneIf(b.m, [&](int64_t row, int64_t col, double v) {
        return v != 0.0 && (row == b.first + col || std::fabs(v) >= threshold[col]);
      });
      if (topk_ > 0) {
        KeepTopKPerColumn(b.m, b.first, true);
      }
      b.r = Residual(params_.a, b.m, b.first, w);
    });
    if (topk_ > 0) {
      return;
    }
    const int64_t budget = MaxNonZeros();
    const int64_t nonzeros = CountNonZeros(Mat::M);
    if (nonzeros <= budget) {
      return;
    }
    // Tmp = A * R (dropping enabled, so nothing pruned)
    Multiply(params_.a, Mat::R, Mat::Tmp);
    std::vector<int64_t> offsets(batches_.size() + 1, 0);
    for (size_t bi = 0; bi < batches_.size(); ++bi) {
      const Batch& b = batches_[bi];
      int64_t count = 0;
      for (int64_t j = 0; j < b.width; ++j) {
        for (int64_t p = b.m.ptr[j]; p < b.m.ptr[j + 1]; ++p) {
          count += b.m.idx[p] != b.first + j ? 1 : 0;
        }
      }
      offsets[bi + 1] = offsets[bi] + count;
    }
    std::vector<Key> keys(offsets.back());
    for (size_t bi = 0; bi < batches_.size(); ++bi) {
      const Batch& b = batches_[bi];
      int64_t off = offsets[bi];
      for (int64_t j = 0; j < b.width; ++j) {
        for (int64_t p = b.m.ptr[j]; p < b.m.ptr[j + 1]; ++p) {
          if (b.m.idx[p] == b.first + j) {
            continue;
          }
          keys[off] = Key{Score(b, j, b.m.idx[p], b.m.val[p]), off};
          ++off;
        }
      }
    }
    const Key cutoff = Cutoff(keys, nonzeros - budget);
    for (size_t bi = 0; bi < batches_.size(); ++bi) {
      Batch& b = batches_[bi];
      int64_t off = offsets[bi];
      PruneIf(b.m, [&](int64_t row, int64_t col, double v) {
        if (row == b.first + col) {
          return true;
        }
        const Key key{Score(b, col, row, v), off};
        ++off;
        return Less(cutoff, key);
      });
    }
    RecomputeResidual();
  }

  // dropping.cpp:177-224 (global budget) or the per-column top-k variant.
  bool DropForMatrixType(Mat t) {
    if (!params_.dropping) {
      return false;
    }
    const int64_t original = CountNonZeros(t);
    if (order_ == 0) {
      ForBatches([&](Batch& b, Work&) {
        Csc& x = b.Get(t);
        double s = 0.0;
        for (int64_t j = 0; j < x.cols; ++j) {
          AccSquares(x, j, s);
        }
        const double limit = std::sqrt(s) * kEps;
        PruneIf(x, [&](int64_t, int64_t, double v) { return !(std::fabs(v) <= limit); });
      });
    } else {
      const double limit = std::sqrt(SquaredNorm(t)) * kEps;
      ForBatches([&](Batch& b, Work&) {
        PruneIf(b.Get(t), [&](int64_t, int64_t, double v) { return !(std::fabs(v) <= limit); });
      });
    }
    if (topk_ > 0) {
      ForBatches([&](Batch& b, Work&) { KeepTopKPerColumn(b.Get(t), b.first, false); });
      return CountNonZeros(t) != original;
    }
    const int64_t budget = MaxNonZeros();
    const int64_t nonzeros = CountNonZeros(t);
    if (nonzeros <= budget) {
      return nonzeros != original;
    }
    std::vector<Key> keys;
    keys.reserve(nonzeros);
    for (auto& b : batches_) {
      const Csc& x = b.Get(t);
      for (int64_t p = 0; p < x.nnz(); ++p) {
        keys.push_back(Key{std::fabs(x.val[p]), static_cast<int64_t>(keys.size())});
      }
    }
    const Key cutoff = Cutoff(keys, nonzeros - budget);
    int64_t off = 0;
    for (auto& b : batches_) {
      PruneIf(b.Get(t), [&](int64_t, int64_t, double v) {
        const Key key{std::fabs(v), off};
        ++off;
        return Less(cutoff, key);
      });
    }
    return true;
  }

  // StabilizeResiduals (state_manager.cpp:81-95)
  void StabilizeResiduals() {
    const double norm = ResidualNorm();
    const double floor = 64.0 * kEps * std::sqrt(static_cast<double>(n_));
    const double limit = std::max(10.0 * params_.tolerance, floor);
    if (std::isfinite(norm) && norm > limit) {
      return;
    }
    RecomputeResidual();
  }

  // UpdateResidualsAfterDropping (methods_common.hpp:83-93)
  template <class F>
  void UpdateResiduals(F callback, bool stabilize) {
    if (params_.dropping) {
      ApplyDroppingStrategy();
      return;
    }
    ForBatches([&](Batch& b, Work& w) { callback(b, w); });
    if (stabilize) {
      StabilizeResiduals();
    }
  }

  // OutputResult::AppendIteration (result_operations.cpp:53-67)
  bool AppendIteration(Mat direction) {
    const int64_t iter = static_cast<int64_t>(history_.rows.size());
    history_.iterations = iter;
    const double residual = history_.rows.empty() ? history_.initial_residual : ResidualNorm();
    const double entries = static_cast<double>(n_) * static_cast<double>(n_);
    SingleIterationData row;
    row.iteration = iter;
    row.residual_norm = residual;
    row.density_m = static_cast<double>(CountNonZeros(Mat::M)) / entries;
    row.density_direction = static_cast<double>(CountNonZeros(direction)) / entries;
    history_.rows.push_back(row);
    if (row.residual_norm < params_.tolerance) {
      history_.converged = true;
      return true;
    }
    return !params_.dropping && params_.max_density < 1.0 && row.density_m >= params_.max_density;
  }

 private:
  struct Key {
    double score = 0.0;
    int64_t offset = 0;
  };

  // dropping.cpp:31-33
  static bool Less(const Key& a, const Key& b) {
    return a.score < b.score || (a.score == b.score && a.offset < b.offset);
  }

  // dropping.cpp:86-93
  static Key Cutoff(std::vector<Key>& keys, int64_t drop) {
    if (drop <= 0 || drop > static_cast<int64_t>(keys.size())) {
      throw std::invalid_argument("Invalid global sparse dropping count");
    }
    auto nth = keys.begin() + drop - 1;
    std::nth_element(keys.begin(), nth, keys.end(), Less);
    return *nth;
  }

  // dropping.cpp:19-29: m^2 ||A e_k||^2 + 2 m (A R)_{k,l}; non-finite -> -inf.
  double Score(const Batch& b, int64_t col, int64_t row, double v) const {
    const double s = v * v * col_norm2_[row] + 2.0 * v * Coeff(b.tmp, row, col);
    return std::isfinite(s) ? s : -std::numeric_limits<double>::infinity();
  }

  // Per-column top-k by magnitude: drop the smallest (|v|, row) keys until K
  // remain; with protect_diagonal the diagonal is always kept and counts
  // toward K.
  void KeepTopKPerColumn(Csc& x, int64_t first, bool protect_diagonal) const {
    const int64_t k = topk_;
    std::vector<char> keep;
    std::vector<int64_t> order;
    PruneIf(x, [](int64_t, int64_t, double) { return true; });
    Csc out(x.rows, x.cols);
    for (int64_t j = 0; j < x.cols; ++j) {
      const int64_t begin = x.ptr[j];
      const int64_t end = x.ptr[j + 1];
      const int64_t count = end - begin;
      keep.assign(count, 1);
      if (count > k) {
        order.clear();
        int64_t diag_slots = 0;
        for (int64_t p = begin; p < end; ++p) {
          if (protect_diagonal && x.idx[p] == first + j) {
            diag_slots = 1;
            continue;
          }
          order.push_back(p);
        }
        const int64_t keep_off = std::max<int64_t>(0, k - diag_slots);
        const int64_t drop = static_cast<int64_t>(order.size()) - keep_off;
        if (drop > 0) {
          std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
            const double fa = std::fabs(x.val[a]);
            const double fb = std::fabs(x.val[b]);
            return fa < fb || (fa == fb && x.idx[a] < x.idx[b]);
          });
          for (int64_t i = 0; i < drop; ++i) {
            keep[order[i] - begin] = 0;
          }
        }
      }
      for (int64_t p = begin; p < end; ++p) {
        if (keep[p - begin]) {
          out.idx.push_back(x.idx[p]);
          out.val.push_back(x.val[p]);
        }
      }
      out.ptr[j + 1] = static_cast<int64_t>(out.idx.size());
    }
    x = std::move(out);
  }

  // ValidateProblem (methods_common.cpp:12-36)
  void Validate() const {
    const Csc& a = params_.a;
    if (a.rows != a.cols || a.rows == 0) {
      throw std::invalid_argument("A must be a non-empty square matrix");
    }
    if (params_.has_m0 && (params_.m0.rows != a.rows || params_.m0.cols != a.cols)) {
      throw std::invalid_argument("Initial preconditioner M0 must have the same shape as A");
    }
    if (params_.has_pr && (params_.pr.rows != a.rows || params_.pr.cols != a.cols)) {
      throw std::invalid_argument("Pr must have the same shape as A");
    }
    if (params_.max_iterations <= 0) {
      throw std::invalid_argument("max_iterations must be positive");
    }
    if (!std::isfinite(params_.tolerance) || params_.tolerance < 0.0) {
      throw std::invalid_argument("tolerance must be finite and non-negative");
    }
    if (!std::isfinite(params_.max_density) || params_.max_density <= kMinDensity || params_.max_density > 1.0) {
      throw std::invalid_argument("max_density must be finite and in the interval (0, 1]");
    }
    const double entries = params_.max_density * static_cast<double>(a.rows) * static_cast<double>(a.rows);
    if (params_.dropping && entries < static_cast<double>(a.rows)) {
      throw std::invalid_argument("max_density is too small to preserve the diagonal of M");
    }
  }

  // GetDiagonalInversePreconditioner (methods_common.cpp:50-63)
  static Csc DiagonalInverse(const Csc& a) {
    std::vector<double> diag(a.cols, 0.0);
    for (int64_t j = 0; j < a.cols; ++j) {
      diag[j] = Coeff(a, j, j);
    }
    for (const double d : diag) {
      if (!std::isfinite(d) || d <= 0.0) {
        throw std::invalid_argument("A has an invalid diagonal entry; provide Pr explicitly");
      }
    }
    Csc pr(a.rows, a.cols);
    for (int64_t j = 0; j < a.cols; ++j) {
      const double inv = 1.0 / diag[j];
      if (!std::isfinite(inv)) {
        throw std::invalid_argument("A diagonal cannot be inverted safely; provide Pr explicitly");
      }
      pr.idx.push_back(j);
      pr.val.push_back(inv);
      pr.ptr[j + 1] = j + 1;
    }
    return pr;
  }

  // InitializeBatches (methods_common.cpp:78-103)
  void InitBatches(int64_t count) {
    batches_.resize(count);
    Csc identity;
    if (!params_.has_m0) {
      identity = Csc(n_, n_);
      for (int64_t j = 0; j < n_; ++j) {
        identity.idx.push_back(j);
        identity.val.push_back(1.0);
        identity.ptr[j + 1] = j + 1;
      }
    }
    const Csc& start = params_.has_m0 ? params_.m0 : identity;
    for (int64_t i = 0; i < count; ++i) {
      Batch& b = batches_[i];
      b.first = n_ * i / count;
      b.width = n_ * (i + 1) / count - b.first;
      b.m = Columns(start, b.first, b.width);
      for (Csc* x : {&b.r, &b.z, &b.p, &b.ap, &b.az, &b.tmp, &b.q}) {
        *x = Csc(n_, b.width);
      }
    }
  }

  const Params& params_;
  bool symmetric_;
  int64_t order_;
  int64_t topk_;
  int64_t n_ = 0;
  int threads_ = 1;
  std::vector<Work> work_;
  std::vector<Batch> batches_;
  std::vector<double> col_norm2_;
  Csc pr_;
  History history_;
};

// ---------------------------------------------------------------------------
// Global SPAI CG (conjugate_gradient.cpp:15-83)
void RunCg(State& s) {
  const Params& prm = s.params();
  s.Multiply(s.pr(), Mat::R, Mat::Z);
  s.ForBatches([&](Batch& b, Work&) { b.p = b.z; });
  double r_z = s.Dot(Mat::R, Mat::Z);
  s.DropForMatrixType(Mat::P);
  if (s.AppendIteration(Mat::P)) {
    return;
  }
  s.Multiply(s.a(), Mat::P, Mat::AP);
  for (int64_t i = 1; i <= prm.max_iterations; ++i) {
    const double den = s.Dot(Mat::P, Mat::AP);
    if (!IsFiniteNonZero(r_z) || !IsFiniteNonZero(den)) {
      break;
    }
    const double alpha = r_z / den;
    if (!std::isfinite(alpha)) {
      break;
    }
    const double previous = r_z;
    s.ForBatches([&](Batch& b, Work&) { AddScaled(b.m, b.p, alpha); });
    s.UpdateResiduals([&](Batch& b, Work&) { AddScaled(b.r, b.ap, -alpha); }, false);
    if (s.AppendIteration(Mat::P)) {
      break;
    }
    s.Multiply(s.pr(), Mat::R, Mat::Z);
    r_z = s.Dot(Mat::R, Mat::Z);
    const double beta = r_z / previous;
    if (!std::isfinite(beta)) {
      break;
    }
    s.ForBatches([&](Batch& b, Work&) { LinComb(b.z, 1.0, b.p, beta); });
    s.DropForMatrixType(Mat::P);
    s.Multiply(s.a(), Mat::P, Mat::AP);
  }
}

// Global SPAI MR (minimal_residual.cpp:31-93)
void RunMr(State& s) {
  const Params& prm = s.params();
  s.Multiply(s.pr(), Mat::R, Mat::Z);
  if (s.AppendIteration(Mat::Z)) {
    return;
  }
  s.Multiply(s.a(), Mat::Z, Mat::AZ);
  s.Multiply(s.pr(), Mat::AZ, Mat::Tmp);
  double num = s.Dot(Mat::Z, Mat::Tmp);
  double den = s.SquaredNorm(Mat::Tmp);
  for (int64_t i = 1; i <= prm.max_iterations; ++i) {
    if (!IsFiniteNonZero(den)) {
      break;
    }
    const double alpha = num / den;
    if (!std::isfinite(alpha)) {
      break;
    }
    s.ForBatches([&](Batch& b, Work&) { AddScaled(b.m, b.z, alpha); });
    s.UpdateResiduals([&](Batch& b, Work& w) { b.r = Residual(s.a(), b.m, b.first, w); }, false);
    if (s.AppendIteration(Mat::Z)) {
      break;
    }
    s.Multiply(s.pr(), Mat::R, Mat::Z);
    s.Multiply(s.a(), Mat::Z, Mat::AZ);
    s.Multiply(s.pr(), Mat::AZ, Mat::Tmp);
    num = s.Dot(Mat::Z, Mat::Tmp);
    den = s.SquaredNorm(Mat::Tmp);
  }
}

// Global SPAI LOMR (locally_minimal_residual.cpp:36-118)
void RunLomr(State& s) {
  const Params& prm = s.params();
  s.Multiply(s.pr(), Mat::R, Mat::Z);
  if (s.AppendIteration(Mat::Z)) {
    return;
  }
  for (int64_t i = 1; i <= prm.max_iterations; ++i) {
    s.Multiply(s.a(), Mat::P, Mat::AP);
    s.Multiply(s.a(), Mat::Z, Mat::AZ);
    s.Multiply(s.pr(), Mat::AZ, Mat::Tmp);
    const double az_praz = s.Dot(Mat::AZ, Mat::Tmp);
    const double z_az = s.Dot(Mat::Z, Mat::AZ);
    double ap_prap = 0.0;
    double az_prap = 0.0;
    double z_ap = 0.0;
    if (i > 1) {
      s.Multiply(s.pr(), Mat::AP, Mat::Tmp);
      ap_prap = s.Dot(Mat::AP, Mat::Tmp);
      az_prap = s.Dot(Mat::AZ, Mat::Tmp);
      z_ap = s.Dot(Mat::Z, Mat::AP);
    }
    double delta = 0.0;
    double gamma = 0.0;
    if (i == 1) {
      if (!IsFiniteNonZero(az_praz)) {
        break;
      }
      delta = z_az / az_praz;
      gamma = 1.0;
    } else {
      const double gram[2][2] = {{az_praz, az_prap}, {az_prap, ap_prap}};
      const double rhs[2] = {z_az, z_ap};
      double coef[2];
      SolveLeastSquares2x2(gram, rhs, coef);
      delta = coef[0];
      gamma = coef[1];
    }
    if (!std::isfinite(delta) || !std::isfinite(gamma)) {
      break;
    }
    s.ForBatches([&](Batch& b, Work&) {
      AddScaled(b.m, b.z, delta);
      AddScaled(b.m, b.p, gamma);
    });
    s.UpdateResiduals([&](Batch& b, Work&) {
      AddScaled(b.r, b.az, -delta);
      AddScaled(b.r, b.ap, -gamma);
    }, false);
    const double ratio = delta != 0.0 ? gamma / delta : 0.0;
    const double restart = std::isfinite(ratio) ? ratio : 0.0;
    s.ForBatches([&](Batch& b, Work&) { LinComb(b.z, 1.0, b.p, restart); });
    s.DropForMatrixType(Mat::P);
    if (s.AppendIteration(Mat::P)) {
      break;
    }
    s.Multiply(s.pr(), Mat::R, Mat::Z);
  }
}

// Inner-Outer MR / LOMR (inner_outer_common.hpp:14-107)
void RunInnerOuter(State& s, bool locally_optimal) {
  const Params& prm = s.params();
  if (s.AppendIteration(Mat::P)) {
    return;
  }
  std::vector<std::vector<double>> normalization(s.batches().size());
  for (size_t bi = 0; bi < s.batches().size(); ++bi) {
    normalization[bi].assign(s.batches()[bi].width, 1.0);
  }
  std::vector<Batch>& batches = s.batches();
  for (int64_t iteration = 0; iteration < prm.max_iterations;) {
    const Csc outer = s.AssembleM();
    s.ForBatches([&](Batch& b, Work& w) {
      b.r = Residual(s.a(), b.m, b.first, w);
      b.q = Csc(s.n(), b.width);
    });
    const int64_t inner_count = std::min(prm.inner_iterations, prm.max_iterations - iteration);
    for (int64_t inner = 0; inner < inner_count; ++inner, ++iteration) {
      s.Multiply(outer, Mat::R, Mat::Z);
      s.Multiply(s.a(), Mat::Z, Mat::AZ);
      s.ForBatches([&](Batch& b, Work& w) {
        const size_t bi = static_cast<size_t>(&b - batches.data());
        std::vector<double> delta(b.width, 0.0);
        std::vector<double> gamma(b.width, 0.0);
        if (locally_optimal) {
          b.ap = Product(s.a(), b.q, w);
        }
        for (int64_t j = 0; j < b.width; ++j) {
          const double r_az = ColumnDot(b.r, b.az, j);
          const double az_az = ColumnSquares(b.az, j);
          if (!locally_optimal || inner == 0) {
            delta[j] = SafeQuotient(r_az, az_az);
            gamma[j] = locally_optimal ? 1.0 : 0.0;
          } else {
            const double coupling = ColumnDot(b.az, b.ap, j);
            const double gram[2][2] = {{az_az, coupling}, {coupling, ColumnSquares(b.ap, j)}};
            const double rhs[2] = {r_az, ColumnDot(b.r, b.ap, j)};
            double coef[2];
            SolveLeastSquares2x2(gram, rhs, coef);
            delta[j] = coef[0];
            gamma[j] = coef[1];
          }
          const double inverse = delta[j] != 0.0 ? 1.0 / delta[j] : 1.0;
          normalization[bi][j] = std::isfinite(inverse) ? inverse : 1.0;
        }
        b.p = b.z;
        ScaleColumns(b.p, delta);
        if (locally_optimal) {
          ScaleColumns(b.q, gamma);
          AddScaled(b.p, b.q, 1.0);
        }
      });
      const bool dropped = s.DropForMatrixType(Mat::P);
      s.Multiply(s.a(), Mat::P, Mat::AP);
      s.ForBatches([&](Batch& b, Work&) {
        const size_t bi = static_cast<size_t>(&b - batches.data());
        if (dropped) {
          std::vector<double> correction(b.width);
          for (int64_t j = 0; j < b.width; ++j) {
            correction[j] = SafeQuotient(ColumnDot(b.r, b.ap, j), ColumnSquares(b.ap, j));
          }
          ScaleColumns(b.p, correction);
          ScaleColumns(b.ap, correction);
        }
        AddScaled(b.m, b.p, 1.0);
        if (locally_optimal) {
          b.q = b.p;
          ScaleColumns(b.q, normalization[bi]);
        }
      });
      s.UpdateResiduals([](Batch& b, Work&) { AddScaled(b.r, b.ap, -1.0); }, true);
      if (s.AppendIteration(Mat::P)) {
        return;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// GetCompressedSparseMatrix (methods_c_api.cpp:16-40)
Csc ToCsc(const MatrixData& d) {
  if (d.rows <= 0 || d.cols <= 0 || d.nnz <= 0) {
    throw std::invalid_argument("Sparse matrix dimensions and nnz must be positive");
  }
  for (int64_t i = 0; i < d.cols; ++i) {
    if (d.col_offsets[i] > d.col_offsets[i + 1]) {
      throw std::invalid_argument("Sparse matrix column offsets must be non-decreasing");
    }
  }
  for (int64_t i = 0; i < d.nnz; ++i) {
    if (d.row_indices[i] < 0 || d.row_indices[i] >= d.rows) {
      throw std::invalid_argument("Sparse matrix row idx is out of range");
    }
  }
  Csc c(d.rows, d.cols);
  for (int64_t j = 0; j < d.cols; ++j) {
    for (int64_t p = d.col_offsets[j]; p < d.col_offsets[j + 1]; ++p) {
      c.idx.push_back(d.row_indices[p]);
      c.val.push_back(d.values[p]);
    }
    c.ptr[j + 1] = static_cast<int64_t>(c.idx.size());
  }
  return c;
}

Result ErrorResult(const std::string& message) {
  Result out{};
  out.error_message = new char[message.size() + 1];
  std::memcpy(out.error_message, message.c_str(), message.size() + 1);
  return out;
}

Result SuccessResult(const Csc& m, const History& h) {
  Result out{};
  out.rows = m.rows;
  out.cols = m.cols;
  out.nnz = m.nnz();
  out.iterations = h.iterations;
  out.converged = h.converged ? 1 : 0;
  out.history_size = static_cast<int64_t>(h.rows.size());
  out.col_offsets = new int64_t[m.cols + 1];
  out.row_indices = new int64_t[m.nnz()];
  out.values = new double[m.nnz()];
  out.history = new SingleIterationData[h.rows.size()];
  std::memcpy(out.col_offsets, m.ptr.data(), sizeof(int64_t) * (m.cols + 1));
  if (m.nnz() > 0) {
    std::memcpy(out.row_indices, m.idx.data(), sizeof(int64_t) * m.nnz());
    std::memcpy(out.values, m.val.data(), sizeof(double) * m.nnz());
  }
  for (size_t i = 0; i < h.rows.size(); ++i) {
    out.history[i] = h.rows[i];
  }
  return out;
}

inline double PcgDot(const double* x, const double* y, int64_t n, int64_t order, std::vector<double>& scratch) {
  if (order == 0) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) {
      s += x[i] * y[i];
    }
    return s;
  }
  for (int64_t i = 0; i < n; ++i) {
    scratch[i] = x[i] * y[i];
  }
  return TreeSum(scratch.data(), n);
}

// _multiply / _row_dot (backward_error.pyx:16-34): per row sequential.
inline void PcgSpmv(int64_t n, const double* v, const int64_t* idx, const int64_t* off, const double* x, double* out) {
  for (int64_t row = 0; row < n; ++row) {
    double s = 0.0;
    for (int64_t k = off[row]; k < off[row + 1]; ++k) {
      s += v[k] * x[idx[k]];
    }
    out[row] = s;
  }
}

}  // namespace

extern "C" {

Result oracle_run(int64_t method, MatrixData A, MatrixData M0, MatrixData Pr, MethodParams cparams,
                  OracleOptions options) {
  try {
    Params p;
    p.a = ToCsc(A);
    p.has_m0 = cparams.use_initial_m != 0;
    if (p.has_m0) {
      p.m0 = ToCsc(M0);
    }
    p.has_pr = cparams.use_preconditioner != 0;
    if (p.has_pr) {
      p.pr = ToCsc(Pr);
    }
    p.max_iterations = cparams.max_iterations;
    p.tolerance = cparams.tolerance;
    p.max_density = cparams.max_density;
    p.dropping = cparams.enable_dropping != 0;
    p.num_threads = cparams.num_threads;
    p.inner_iterations = cparams.inner_iterations;
    if (method < 0 || method > 4) {
      throw std::invalid_argument("unknown method id");
    }
    if (options.topk_per_column < 0) {
      throw std::invalid_argument("topk_per_column must be non-negative");
    }
    const bool inner_outer = method >= 3;
    if (inner_outer && p.inner_iterations <= 0) {
      throw std::invalid_argument("inner_iterations must be positive");
    }
    State state(p, options, !inner_outer);
    switch (method) {
      case 0: RunCg(state); break;
      case 1: RunMr(state); break;
      case 2: RunLomr(state); break;
      case 3: RunInnerOuter(state, false); break;
      case 4: RunInnerOuter(state, true); break;
    }
    return SuccessResult(state.AssembleM(), state.history());
  } catch (const std::exception& ex) {
    return ErrorResult(ex.what());
  } catch (...) {
    return ErrorResult("Unknown failure.");
  }
}

void oracle_free(Result* r) {
  if (r == nullptr) {
    return;
  }
  delete[] r->col_offsets;
  delete[] r->row_indices;
  delete[] r->values;
  delete[] r->history;
  delete[] r->error_message;
  r->col_offsets = nullptr;
  r->row_indices = nullptr;
  r->values = nullptr;
  r->history = nullptr;
  r->error_message = nullptr;
}

// backward_error.pyx:69-144
int64_t oracle_pcg(int64_t n, const double* av, const int64_t* ai, const int64_t* ao, const double* mv,
                   const int64_t* mi, const int64_t* mo, const double* b, int64_t max_iterations,
                   double tolerance, int64_t order, int64_t refresh_period, double* history,
                   int64_t* status_out, double* x_out) {
  std::vector<double> r(b, b + n), z(n), p(n), ap(n), x(n, 0.0), scratch(n);
  int64_t count = 1;
  int64_t status = 0;
  PcgSpmv(n, mv, mi, mo, r.data(), z.data());
  p = z;
  double r_r = PcgDot(r.data(), r.data(), n, order, scratch);
  const double b_norm = std::sqrt(r_r);
  double r_z = PcgDot(r.data(), z.data(), n, order, scratch);
  history[0] = 1.0;
  while (count < max_iterations && history[count - 1] > tolerance) {
    PcgSpmv(n, av, ai, ao, p.data(), ap.data());
    const double den = PcgDot(p.data(), ap.data(), n, order, scratch);
    if (!std::isfinite(r_z) || !std::isfinite(den) || r_z == 0.0 || den == 0.0) {
      status = 2;
      break;
    }
    const double alpha = r_z / den;
    if (!std::isfinite(alpha)) {
      status = 2;
      break;
    }
    double beta = r_z;
    for (int64_t i = 0; i < n; ++i) {
      x[i] += alpha * p[i];
      r[i] -= alpha * ap[i];
    }
    r_r = PcgDot(r.data(), r.data(), n, order, scratch);
    double error = std::sqrt(r_r) / b_norm;
    // The reference refreshes the true residual when the recursive one
    // reaches the tolerance and then restarts the direction (beta = 0).
    // refresh_period > 0 adds a periodic true-residual replacement that keeps
    // the direction.
    const bool converged_refresh = error <= tolerance;
    const bool periodic_refresh = refresh_period > 0 && count % refresh_period == 0;
    if (converged_refresh || periodic_refresh) {
      PcgSpmv(n, av, ai, ao, x.data(), ap.data());
      for (int64_t i = 0; i < n; ++i) {
        r[i] = b[i] - ap[i];
      }
      r_r = PcgDot(r.data(), r.data(), n, order, scratch);
      error = std::sqrt(r_r) / b_norm;
    }
    PcgSpmv(n, mv, mi, mo, r.data(), z.data());
    r_z = PcgDot(r.data(), z.data(), n, order, scratch);
    beta = converged_refresh ? 0.0 : r_z / beta;
    history[count] = error;
    ++count;
    if (!std::isfinite(error)) {
      status = 3;
      break;
    }
    if (!std::isfinite(beta)) {
      status = 2;
      break;
    }
    for (int64_t i = 0; i < n; ++i) {
      p[i] = z[i] + beta * p[i];
    }
  }
  PcgSpmv(n, av, ai, ao, x.data(), ap.data());
  for (int64_t i = 0; i < n; ++i) {
    r[i] = b[i] - ap[i];
  }
  history[count - 1] = std::sqrt(PcgDot(r.data(), r.data(), n, order, scratch)) / b_norm;
  if (!std::isfinite(history[count - 1])) {
    status = 3;
  } else if (history[count - 1] <= tolerance) {
    status = 1;
  }
  *status_out = status;
  if (x_out != nullptr) {
    std::memcpy(x_out, x.data(), sizeof(double) * n);
  }
  return count;
}

double oracle_tree_sum(const double* values, int64_t count) { return TreeSum(values, count); }

void oracle_solve_2x2(const double* m, const double* rhs, double* solution) {
  const double mm[2][2] = {{m[0], m[1]}, {m[2], m[3]}};
  const double x[2] = {rhs[0], rhs[1]};
  SolveLeastSquares2x2(mm, x, solution);
}

}  // extern "C"
