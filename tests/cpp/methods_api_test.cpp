// C++ caller of the drop-in API (include/methods.hpp over include/methods_c_api.h),
// linked against libspai_b200.so.  It checks the properties the reference's own
// C++ test checks (reference tests/test.cpp:107-179) on the same fixture --
// tridiag(-1, 2, -1) with n = 12, M0 = Pr = I -- and writes each result's
// history and M to stdout for the Python side to compare with the oracle.
//
//   methods_api_test            run every check, exit 0 when all hold
//   methods_api_test --dump     also print "name iterations residuals... | nnz values..." lines

#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <iostream>
#include <string>
#include <vector>

#include "methods.hpp"

namespace {

namespace mc = methods::common;
namespace mgs = methods::global_spai;
namespace mio = methods::inner_outer;

int failures = 0;
bool dump = false;

void Check(bool ok, const std::string& what) {
  if (!ok) {
    std::cout << "FAILED: " << what << "\n";
    ++failures;
  }
}

mc::SparseMatrix Tridiagonal(int64_t n) {
  std::vector<mc::Triplet<double, int64_t>> entries;
  for (int64_t i = 0; i < n; ++i) {
    entries.emplace_back(i, i, 2.0);
    if (i > 0) entries.emplace_back(i, i - 1, -1.0);
    if (i + 1 < n) entries.emplace_back(i, i + 1, -1.0);
  }
  mc::SparseMatrix a(n, n);
  a.setFromTriplets(entries.begin(), entries.end());
  return a;
}

mc::SparseMatrix Identity(int64_t n) {
  mc::SparseMatrix i(n, n);
  i.setIdentity();
  return i;
}

double ResidualNorm(const mc::SparseMatrix& a, const mc::SparseMatrix& m) {
  return (Identity(a.rows()) - a * m).norm();
}

void Dump(const std::string& name, const mc::OutputResult& r) {
  if (!dump) return;
  std::printf("%s %lld", name.c_str(), static_cast<long long>(r.iterations));
  for (const auto& h : r.history) std::printf(" %.17g", h.residual_norm);
  std::printf(" | %lld", static_cast<long long>(r.M.nonZeros()));
  for (int64_t k = 0; k < r.M.nonZeros(); ++k) std::printf(" %.17g", r.M.valuePtr()[k]);
  std::printf("\n");
}

using Method = std::function<mc::OutputResult(const mc::InputParams&, int64_t)>;

struct Named {
  const char* name;
  Method run;
};

}  // namespace

int main(int argc, char** argv) {
  dump = argc > 1 && std::strcmp(argv[1], "--dump") == 0;
  const int64_t n = 12;
  const mc::SparseMatrix a = Tridiagonal(n);
  Check(a.outerSize() == a.cols() && a.isCompressed() && a.nonZeros() == 3 * n - 2, "tridiagonal fixture");
  const mc::InputParams params(a, Identity(n), Identity(n), 8, 1e-14, 1.0);
  Check(params.max_non_zeros == n * n, "budget max(n, floor(density n^2))");
  const double initial = ResidualNorm(params.A, params.M0);
  const std::vector<Named> methods_list = {
      {"global_cg", [](const mc::InputParams& p, int64_t t) { return mgs::RunConjugateGradient(p, t); }},
      {"global_mr", [](const mc::InputParams& p, int64_t t) { return mgs::RunMinimalResidual(p, t); }},
      {"global_lomr", [](const mc::InputParams& p, int64_t t) { return mgs::RunLocallyOptimalMinimalResidual(p, t); }},
      {"inner_outer_mr", [](const mc::InputParams& p, int64_t t) { return mio::RunMinimalResidual(p, t); }},
      {"inner_outer_lomr",
       [](const mc::InputParams& p, int64_t t) { return mio::RunLocallyOptimalMinimalResidual(p, t); }},
  };

  // 1 and 2 column batches agree to 1e-10; history bookkeeping; the residual falls
  for (const Named& m : methods_list) {
    const mc::OutputResult one = m.run(params, 1);
    const mc::OutputResult two = m.run(params, 2);
    Dump(std::string(m.name) + "_p1", one);
    for (const mc::OutputResult* r : {&one, &two}) {
      Check(!r->history.empty() && static_cast<int64_t>(r->history.size()) == r->iterations + 1,
            std::string(m.name) + ": history length");
      Check(r->history.front().iteration == 0 && r->history.back().iteration == r->iterations,
            std::string(m.name) + ": iteration numbers");
      Check(r->history.back().residual_norm < initial, std::string(m.name) + ": residual decreases");
    }
    Check(one.iterations == two.iterations, std::string(m.name) + ": same iterations at 1 and 2 batches");
    Check((one.M - two.M).norm() < 1e-10, std::string(m.name) + ": same M at 1 and 2 batches");
    Check(std::fabs(one.history.back().residual_norm - two.history.back().residual_norm) < 1e-10,
          std::string(m.name) + ": same residual at 1 and 2 batches");
    Check(one.method.find(std::string(m.name).substr(std::string(m.name).find('_') + 1)) != std::string::npos,
          std::string(m.name) + ": method name");
  }

  // absolute stop (tests/test.cpp:129-139)
  mc::InputParams absolute = params;
  absolute.tolerance = 0.9 * initial;
  const mc::OutputResult stop = mgs::RunMinimalResidual(absolute, 2);
  Check(stop.converged && stop.iterations == 1 && stop.history.size() == 2 &&
            stop.history.back().residual_norm < absolute.tolerance,
        "absolute stopping criterion");

  // dropping keeps nnz(M) within the budget (tests/test.cpp:141-151)
  mc::InputParams sparse_params = params;
  sparse_params.max_iterations = 3;
  sparse_params.max_density = 0.12;
  sparse_params.tolerance = 0.0;
  const int64_t budget = std::max<int64_t>(n, static_cast<int64_t>(std::floor(0.12 * n * n)));
  for (const Named& m : methods_list) {
    const mc::OutputResult one = m.run(sparse_params, 1);
    const mc::OutputResult four = m.run(sparse_params, 4);
    Dump(std::string(m.name) + "_drop", one);
    Check(one.M.nonZeros() <= budget && four.M.nonZeros() <= budget, std::string(m.name) + ": budget");
    Check(one.iterations == 3 && four.iterations == 3, std::string(m.name) + ": three iterations");
    Check((one.M - four.M).norm() < 1e-10, std::string(m.name) + ": same M at 1 and 4 batches");
  }

  // without dropping the density limit stops the run (tests/test.cpp:153-165)
  mc::InputParams no_drop = params;
  no_drop.max_iterations = 8;
  no_drop.tolerance = 0.0;
  no_drop.max_density = 0.2;
  no_drop.enable_dropping = false;
  for (const Named& m : methods_list) {
    const mc::OutputResult r = m.run(no_drop, 1);
    Check(!r.converged && r.iterations > 0 && r.iterations < 8 && r.history.back().density_m >= 0.2,
          std::string(m.name) + ": density stop");
  }

  // the recorded residual is the true ||I - A M||_F (tests/test.cpp:167-178)
  mc::InputParams reliable = params;
  reliable.max_iterations = 20;
  reliable.tolerance = 1e-20;
  const mc::OutputResult r = mio::RunLocallyOptimalMinimalResidual(reliable, 2);
  Check(r.iterations == 20 && !r.converged, "twenty iterations without convergence");
  Check(std::fabs(r.history.back().residual_norm - ResidualNorm(a, r.M)) < 1e-9, "recorded residual is the true one");

  // the reference's validation messages come back as exceptions
  bool threw = false;
  try {
    mc::InputParams bad = params;
    bad.max_density = 1.5;
    mgs::RunMinimalResidual(bad, 1);
  } catch (const std::runtime_error& ex) {
    threw = std::string(ex.what()).find("density") != std::string::npos;
  }
  Check(threw, "invalid max_density is reported");
  threw = false;
  try {
    mgs::RunMinimalResidual(params, 0);
  } catch (const std::runtime_error& ex) {
    threw = std::string(ex.what()).find("threads") != std::string::npos;
  }
  Check(threw, "invalid thread count is reported");

  std::cout << (failures == 0 ? "all checks passed" : "checks failed") << "\n";
  return failures == 0 ? 0 : 1;
}
