#pragma once
// C++ API of libspai_b200.so with the reference's names and signatures
// (reference include/methods.hpp:11-153): methods::common::InputParams,
// SingleIterationData, OutputResult, and the five Run* functions of
// methods::global_spai and methods::inner_outer.
//
// The reference declares these over Eigen::SparseMatrix<double, ColMajor,
// int64_t> (include/methods.hpp:17).  Eigen is not a dependency of this
// library, so methods::common::SparseMatrix here is a small column-compressed
// matrix of the same layout (int64 column offsets, int64 row indices, FP64
// values) with the subset of Eigen's interface that callers of this API use:
// construction from triplets, setIdentity, rows/cols/nonZeros/outerSize,
// isCompressed/makeCompressed, the raw index and value pointers, coeff,
// products, differences and the Frobenius norm.  Code written against the
// reference compiles unchanged when it names the matrix type through
// methods::common (mc::SparseMatrix) and builds triplets with
// methods::common::Triplet instead of Eigen::Triplet.
//
// Everything is header-only and inline: each Run* call converts its inputs
// to the C ABI of methods_c_api.h (the reference's own entry points,
// include/methods_c_api.h:48-56), so the C++ API inherits their behaviour --
// FP64, the reference's summation order over min(n, num_threads) column
// batches, and the reference's validation messages, which are rethrown here
// as std::runtime_error with the same what() text (the reference throws
// std::invalid_argument / std::runtime_error from ValidateProblem,
// src/common/methods_common.cpp:12-48).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "methods_c_api.h"

namespace methods {

namespace common {

inline constexpr double EPS = 1e-9;  // reference include/methods.hpp:15

// (row, col, value) entry for SparseMatrix::setFromTriplets (Eigen::Triplet's role).
template <class Scalar = double, class Index = int64_t>
class Triplet {
 public:
  Triplet(Index row = 0, Index col = 0, Scalar value = Scalar(0)) : row_(row), col_(col), value_(value) {}
  Index row() const { return row_; }
  Index col() const { return col_; }
  Scalar value() const { return value_; }

 private:
  Index row_;
  Index col_;
  Scalar value_;
};

// Column-compressed FP64 matrix with int64 indices, always compressed:
// offsets[cols + 1], rows[nnz] ascending inside each column, values[nnz].
class SparseMatrix {
 public:
  SparseMatrix() : offsets_(1, 0) {}
  SparseMatrix(int64_t rows, int64_t cols) : rows_(rows), cols_(cols), offsets_(static_cast<size_t>(cols) + 1, 0) {
    if (rows < 0 || cols < 0) throw std::invalid_argument("SparseMatrix: negative dimension");
  }
  // From compressed arrays (copied); rows must be sorted and unique per column.
  SparseMatrix(int64_t rows, int64_t cols, std::vector<int64_t> offsets, std::vector<int64_t> row_indices,
               std::vector<double> values)
      : rows_(rows), cols_(cols), offsets_(std::move(offsets)), rows_idx_(std::move(row_indices)),
        values_(std::move(values)) {
    if (offsets_.size() != static_cast<size_t>(cols) + 1 || offsets_.front() != 0 ||
        static_cast<size_t>(offsets_.back()) != rows_idx_.size() || rows_idx_.size() != values_.size()) {
      throw std::invalid_argument("SparseMatrix: inconsistent compressed arrays");
    }
  }

  int64_t rows() const { return rows_; }
  int64_t cols() const { return cols_; }
  int64_t size() const { return rows_ * cols_; }
  int64_t outerSize() const { return cols_; }
  int64_t nonZeros() const { return static_cast<int64_t>(values_.size()); }
  bool isCompressed() const { return true; }
  void makeCompressed() {}

  const int64_t* outerIndexPtr() const { return offsets_.data(); }
  const int64_t* innerIndexPtr() const { return rows_idx_.data(); }
  const double* valuePtr() const { return values_.data(); }

  // Entries are summed where (row, col) repeats, as Eigen's setFromTriplets does.
  template <class It>
  void setFromTriplets(It first, It last) {
    std::vector<std::pair<std::pair<int64_t, int64_t>, double>> entries;
    for (It it = first; it != last; ++it) {
      const int64_t r = static_cast<int64_t>(it->row());
      const int64_t c = static_cast<int64_t>(it->col());
      if (r < 0 || r >= rows_ || c < 0 || c >= cols_) throw std::out_of_range("setFromTriplets: index out of range");
      entries.push_back({{c, r}, static_cast<double>(it->value())});
    }
    std::stable_sort(entries.begin(), entries.end(),
                     [](const auto& a, const auto& b) { return a.first < b.first; });
    offsets_.assign(static_cast<size_t>(cols_) + 1, 0);
    rows_idx_.clear();
    values_.clear();
    for (size_t i = 0; i < entries.size(); ++i) {
      if (i > 0 && entries[i].first == entries[i - 1].first) {
        values_.back() += entries[i].second;
        continue;
      }
      rows_idx_.push_back(entries[i].first.second);
      values_.push_back(entries[i].second);
      ++offsets_[static_cast<size_t>(entries[i].first.first) + 1];
    }
    for (int64_t j = 0; j < cols_; ++j) offsets_[j + 1] += offsets_[j];
  }

  void setIdentity() {
    const int64_t d = std::min(rows_, cols_);
    offsets_.assign(static_cast<size_t>(cols_) + 1, 0);
    rows_idx_.clear();
    values_.clear();
    for (int64_t j = 0; j < cols_; ++j) {
      if (j < d) {
        rows_idx_.push_back(j);
        values_.push_back(1.0);
      }
      offsets_[j + 1] = static_cast<int64_t>(values_.size());
    }
  }

  double coeff(int64_t row, int64_t col) const {
    const auto b = rows_idx_.begin() + offsets_[col];
    const auto e = rows_idx_.begin() + offsets_[col + 1];
    const auto it = std::lower_bound(b, e, row);
    return (it != e && *it == row) ? values_[static_cast<size_t>(it - rows_idx_.begin())] : 0.0;
  }

  double squaredNorm() const {
    double s = 0.0;
    for (const double v : values_) s += v * v;
    return s;
  }
  double norm() const { return std::sqrt(squaredNorm()); }

  // this * other (column by column, dense accumulator per column)
  SparseMatrix operator*(const SparseMatrix& other) const {
    if (cols_ != other.rows_) throw std::invalid_argument("SparseMatrix product: inner dimensions differ");
    SparseMatrix out(rows_, other.cols_);
    std::vector<double> acc(static_cast<size_t>(rows_), 0.0);
    std::vector<char> hit(static_cast<size_t>(rows_), 0);
    std::vector<int64_t> touched;
    for (int64_t j = 0; j < other.cols_; ++j) {
      touched.clear();
      for (int64_t p = other.offsets_[j]; p < other.offsets_[j + 1]; ++p) {
        const int64_t k = other.rows_idx_[p];
        const double bv = other.values_[p];
        for (int64_t q = offsets_[k]; q < offsets_[k + 1]; ++q) {
          const int64_t i = rows_idx_[q];
          if (!hit[i]) {
            hit[i] = 1;
            acc[i] = 0.0;
            touched.push_back(i);
          }
          acc[i] += values_[q] * bv;
        }
      }
      std::sort(touched.begin(), touched.end());
      for (const int64_t i : touched) {
        out.rows_idx_.push_back(i);
        out.values_.push_back(acc[i]);
        hit[i] = 0;
      }
      out.offsets_[j + 1] = static_cast<int64_t>(out.values_.size());
    }
    return out;
  }

  SparseMatrix operator-(const SparseMatrix& other) const { return Combine(other, -1.0); }
  SparseMatrix operator+(const SparseMatrix& other) const { return Combine(other, 1.0); }

 private:
  SparseMatrix Combine(const SparseMatrix& other, double sign) const {
    if (rows_ != other.rows_ || cols_ != other.cols_) throw std::invalid_argument("SparseMatrix: shapes differ");
    SparseMatrix out(rows_, cols_);
    for (int64_t j = 0; j < cols_; ++j) {
      int64_t p = offsets_[j];
      int64_t q = other.offsets_[j];
      while (p < offsets_[j + 1] || q < other.offsets_[j + 1]) {
        const int64_t rp = p < offsets_[j + 1] ? rows_idx_[p] : std::numeric_limits<int64_t>::max();
        const int64_t rq = q < other.offsets_[j + 1] ? other.rows_idx_[q] : std::numeric_limits<int64_t>::max();
        if (rp == rq) {
          out.rows_idx_.push_back(rp);
          out.values_.push_back(values_[p++] + sign * other.values_[q++]);
        } else if (rp < rq) {
          out.rows_idx_.push_back(rp);
          out.values_.push_back(values_[p++]);
        } else {
          out.rows_idx_.push_back(rq);
          out.values_.push_back(sign * other.values_[q++]);
        }
      }
      out.offsets_[j + 1] = static_cast<int64_t>(out.values_.size());
    }
    return out;
  }

  int64_t rows_ = 0;
  int64_t cols_ = 0;
  std::vector<int64_t> offsets_;
  std::vector<int64_t> rows_idx_;
  std::vector<double> values_;
};

inline SparseMatrix EnsureCompressedSparseMatrix(SparseMatrix matrix = SparseMatrix()) {
  matrix.makeCompressed();
  return matrix;
}

// Reference include/methods.hpp:28-62: the problem and the run options; the
// budget max(n, floor(max_density * n^2)) is computed as there.
struct InputParams {
  SparseMatrix A;
  SparseMatrix M0;
  SparseMatrix Pr;

  int64_t max_iterations = 100;
  // Absolute Frobenius residual tolerance, with or without dropping.
  double tolerance = 1e-9;
  double max_density = 0.03;
  bool enable_dropping = true;
  int64_t max_non_zeros = -1;

  InputParams(SparseMatrix A = SparseMatrix(), SparseMatrix M0 = SparseMatrix(), SparseMatrix Pr = SparseMatrix(),
              const int64_t max_iterations = 100, const double tolerance = 1e-9, const double max_density = 0.03,
              const bool enable_dropping = true)
      : A(EnsureCompressedSparseMatrix(std::move(A))),
        M0(EnsureCompressedSparseMatrix(std::move(M0))),
        Pr(EnsureCompressedSparseMatrix(std::move(Pr))),
        max_iterations(max_iterations),
        tolerance(tolerance),
        max_density(max_density),
        enable_dropping(enable_dropping),
        max_non_zeros(std::max(this->A.rows(), static_cast<int64_t>(std::floor(
                                                   max_density * static_cast<double>(this->A.rows()) *
                                                   static_cast<double>(this->A.rows()))))) {}
};

// Reference include/methods.hpp:64-80.
struct SingleIterationData {
  int64_t iteration = 0;
  double residual_norm = 0.0;
  double density_m = 0.0;
  double density_direction = 0.0;

  SingleIterationData(int64_t iteration = 0, double residual_norm = 0.0, double density_m = 0.0,
                      double density_direction = 0.0)
      : iteration(iteration), residual_norm(residual_norm), density_m(density_m),
        density_direction(density_direction) {}
};

using IterationHistory = std::vector<SingleIterationData>;

// Reference include/methods.hpp:84-133 (its public members).
struct OutputResult {
  std::string method;
  SparseMatrix M;
  int64_t iterations = 0;
  bool converged = false;
  IterationHistory history;

  OutputResult() = default;
  explicit OutputResult(std::string method) : method(std::move(method)) {}
  OutputResult(SparseMatrix M, const int64_t iterations = 0, const bool converged = false, std::string method = "",
               IterationHistory history = IterationHistory())
      : method(std::move(method)), M(EnsureCompressedSparseMatrix(std::move(M))), iterations(iterations),
        converged(converged), history(std::move(history)) {}
};

namespace detail {

inline MatrixData View(const SparseMatrix& m) {
  MatrixData d;
  d.rows = m.rows();
  d.cols = m.cols();
  d.nnz = m.nonZeros();
  d.col_offsets = m.outerIndexPtr();
  d.row_indices = m.innerIndexPtr();
  d.values = m.valuePtr();
  return d;
}

// Calls one of the reference's C entry points and turns its Result into an
// OutputResult (the Result is always released with free_mem).
template <class Entry>
OutputResult Run(Entry entry, const char* method, const InputParams& params, int64_t num_threads,
                 int64_t inner_iterations) {
  MethodParams p;
  p.max_iterations = params.max_iterations;
  p.tolerance = params.tolerance;
  p.max_density = params.max_density;
  p.enable_dropping = params.enable_dropping ? 1 : 0;
  p.num_threads = num_threads;
  // the reference uses M0 and Pr when they are non-empty (methods_common.cpp:105-110)
  p.use_initial_m = params.M0.size() != 0 ? 1 : 0;
  p.use_preconditioner = params.Pr.size() != 0 ? 1 : 0;
  p.inner_iterations = inner_iterations;
  Result r = entry(View(params.A), View(params.M0), View(params.Pr), p);
  if (r.error_message != nullptr) {
    const std::string message(r.error_message);
    free_mem(&r);
    throw std::runtime_error(message);
  }
  OutputResult out;
  try {
    std::vector<int64_t> offsets(r.col_offsets, r.col_offsets + r.cols + 1);
    std::vector<int64_t> rows(r.row_indices, r.row_indices + r.nnz);
    std::vector<double> values(r.values, r.values + r.nnz);
    out.M = SparseMatrix(r.rows, r.cols, std::move(offsets), std::move(rows), std::move(values));
    out.method = method;
    out.iterations = r.iterations;
    out.converged = r.converged != 0;
    out.history.reserve(static_cast<size_t>(r.history_size));
    for (int64_t i = 0; i < r.history_size; ++i) {
      const auto& h = r.history[i];
      out.history.emplace_back(h.iteration, h.residual_norm, h.density_m, h.density_direction);
    }
  } catch (...) {
    free_mem(&r);
    throw;
  }
  free_mem(&r);
  return out;
}

}  // namespace detail

}  // namespace common

namespace global_spai {

// Reference include/methods.hpp:137-143.
inline common::OutputResult RunConjugateGradient(const common::InputParams& params, const int64_t num_threads = 1) {
  return common::detail::Run(spai_global_cg, "cg", params, num_threads, 2);
}

inline common::OutputResult RunMinimalResidual(const common::InputParams& params, const int64_t num_threads = 1) {
  return common::detail::Run(spai_global_mr, "mr", params, num_threads, 2);
}

inline common::OutputResult RunLocallyOptimalMinimalResidual(const common::InputParams& params,
                                                             const int64_t num_threads = 1) {
  return common::detail::Run(spai_global_lomr, "lomr", params, num_threads, 2);
}

}  // namespace global_spai

namespace inner_outer {

// Reference include/methods.hpp:147-151.
inline common::OutputResult RunMinimalResidual(const common::InputParams& params, const int64_t num_threads = 1,
                                               const int64_t inner_iterations = 2) {
  return common::detail::Run(inner_outer_mr, "inner_outer_mr", params, num_threads, inner_iterations);
}

inline common::OutputResult RunLocallyOptimalMinimalResidual(const common::InputParams& params,
                                                             const int64_t num_threads = 1,
                                                             const int64_t inner_iterations = 2) {
  return common::detail::Run(inner_outer_lomr, "inner_outer_lomr", params, num_threads, inner_iterations);
}

}  // namespace inner_outer

}  // namespace methods
