// Matrix Market I/O on the host, for inputs too large to route through
// scipy.  The reference loads every matrix with
//   mmread(path).tocsc().astype(float64); sum_duplicates(); eliminate_zeros();
//   sort_indices()                                   (scripts/common.py:397-402)
// and saves preconditioners with mmwrite (scripts/common.py:494-500); the
// reader returns exactly that canonical CSC and the writer emits a file both
// readers parse back to the same bits.
//
// Reading: the file is mapped into memory, the entry lines are split
// into one slice per thread at line boundaries, every thread parses its
// slice in place (integers by hand, values with std::from_chars, which rounds
// correctly); the entries are bucketed by column in file order (per-slice
// offsets, in parallel), each column is sorted by row (stably, so duplicates
// keep their file order), duplicates are summed and explicit zeros cleared.

#include <algorithm>
#include <charconv>
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

#include "../../include/methods_c_api.h"
#include "../../include/spai_b200.h"

namespace spai {
namespace {

enum class Field { kReal, kInteger, kPattern };
enum class Symmetry { kGeneral, kSymmetric, kSkew };

struct Header {
  bool coordinate = true;
  Field field = Field::kReal;
  Symmetry symmetry = Symmetry::kGeneral;
  int64_t rows = 0;
  int64_t cols = 0;
  int64_t entries = 0;  // coordinate: stored entries; array: values in the file
};

std::string Lower(std::string s) {
  for (char& c : s) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
  return s;
}

// The file mapped read-only into memory (no copy; pages are faulted in by
// the threads that parse them).
class FileView {
 public:
  explicit FileView(const char* path) {
    if (path == nullptr) throw std::invalid_argument("path must not be null");
    const int fd = ::open(path, O_RDONLY);
    if (fd < 0) throw std::runtime_error(std::string("cannot open ") + path + ": " + std::strerror(errno));
    struct stat st;
    if (::fstat(fd, &st) != 0) {
      ::close(fd);
      throw std::runtime_error(std::string("cannot read ") + path);
    }
    size_ = static_cast<size_t>(st.st_size);
    if (size_ > 0) {
      void* m = ::mmap(nullptr, size_, PROT_READ, MAP_PRIVATE, fd, 0);
      if (m == MAP_FAILED) {
        ::close(fd);
        throw std::runtime_error(std::string("cannot map ") + path + ": " + std::strerror(errno));
      }
      data_ = static_cast<const char*>(m);
    }
    ::close(fd);
  }
  ~FileView() {
    if (data_ != nullptr) ::munmap(const_cast<char*>(data_), size_);
  }
  FileView(const FileView&) = delete;
  FileView& operator=(const FileView&) = delete;
  const char* data() const { return data_; }
  size_t size() const { return size_; }
  char operator[](size_t i) const { return data_[i]; }

 private:
  const char* data_ = nullptr;
  size_t size_ = 0;
};

// Next line [begin, end) starting at `at`; returns false at the end of the data.
bool NextLine(const FileView& d, size_t& at, size_t& begin, size_t& end) {
  const size_t size = d.size();
  if (at >= size) return false;
  begin = at;
  while (at < size && d[at] != '\n') ++at;
  end = at;
  if (end > begin && d[end - 1] == '\r') --end;
  if (at < size) ++at;
  return true;
}

bool Blank(const FileView& d, size_t begin, size_t end) {
  for (size_t i = begin; i < end; ++i) {
    if (d[i] != ' ' && d[i] != '\t') return false;
  }
  return true;
}

// Header line, comments and the size line; `at` ends at the first entry line.
Header ParseHeader(const FileView& d, size_t& at) {
  size_t b;
  size_t e;
  if (!NextLine(d, at, b, e)) throw std::runtime_error("empty Matrix Market file");
  std::vector<std::string> tokens;
  {
    std::string line(d.data() + b, e - b);
    size_t i = 0;
    while (i < line.size()) {
      while (i < line.size() && (line[i] == ' ' || line[i] == '\t')) ++i;
      size_t j = i;
      while (j < line.size() && line[j] != ' ' && line[j] != '\t') ++j;
      if (j > i) tokens.push_back(Lower(line.substr(i, j - i)));
      i = j;
    }
  }
  if (tokens.size() < 5 || tokens[0] != "%%matrixmarket" || tokens[1] != "matrix") {
    throw std::runtime_error("not a Matrix Market matrix file (header '%%MatrixMarket matrix ...' expected)");
  }
  Header h;
  if (tokens[2] == "coordinate") {
    h.coordinate = true;
  } else if (tokens[2] == "array") {
    h.coordinate = false;
  } else {
    throw std::runtime_error("unknown Matrix Market format '" + tokens[2] + "'");
  }
  if (tokens[3] == "real" || tokens[3] == "double") {
    h.field = Field::kReal;
  } else if (tokens[3] == "integer") {
    h.field = Field::kInteger;
  } else if (tokens[3] == "pattern") {
    h.field = Field::kPattern;
  } else if (tokens[3] == "complex") {
    throw std::runtime_error("complex matrices are not supported");
  } else {
    throw std::runtime_error("unknown Matrix Market field '" + tokens[3] + "'");
  }
  if (tokens[4] == "general") {
    h.symmetry = Symmetry::kGeneral;
  } else if (tokens[4] == "symmetric") {
    h.symmetry = Symmetry::kSymmetric;
  } else if (tokens[4] == "skew-symmetric") {
    h.symmetry = Symmetry::kSkew;
  } else if (tokens[4] == "hermitian") {
    throw std::runtime_error("hermitian matrices are not supported");
  } else {
    throw std::runtime_error("unknown Matrix Market symmetry '" + tokens[4] + "'");
  }
  if (!h.coordinate && h.field == Field::kPattern) throw std::runtime_error("array format cannot be pattern");
  // comments and blank lines, then the size line
  while (true) {
    if (!NextLine(d, at, b, e)) throw std::runtime_error("missing size line");
    if (d[b] == '%' || Blank(d, b, e)) continue;
    break;
  }
  std::string size_line(d.data() + b, e - b);
  long long r = 0;
  long long c = 0;
  long long n = 0;
  const int got = std::sscanf(size_line.c_str(), "%lld %lld %lld", &r, &c, &n);
  if (h.coordinate ? got != 3 : got < 2) throw std::runtime_error("malformed size line '" + size_line + "'");
  if (r <= 0 || c <= 0 || (h.coordinate && n < 0)) throw std::runtime_error("invalid sizes '" + size_line + "'");
  if (h.symmetry != Symmetry::kGeneral && r != c) throw std::runtime_error("a symmetric matrix must be square");
  h.rows = r;
  h.cols = c;
  if (h.coordinate) {
    h.entries = n;
  } else {
    h.entries = h.symmetry == Symmetry::kGeneral ? r * c : (h.symmetry == Symmetry::kSymmetric ? r * (r + 1) / 2
                                                                                                 : r * (r - 1) / 2);
  }
  return h;
}

struct Triplets {
  std::vector<int64_t> row;
  std::vector<int64_t> col;
  std::vector<double> val;
  int64_t stored = 0;  // entry lines read (before symmetric mirroring)
};

const char* SkipSpace(const char* p, const char* end) {
  while (p < end && (*p == ' ' || *p == '\t')) ++p;
  return p;
}

const char* ParseIndex(const char* p, const char* end, int64_t& out) {
  p = SkipSpace(p, end);
  if (p == end || *p < '0' || *p > '9') throw std::runtime_error("malformed index in an entry line");
  int64_t v = 0;
  while (p < end && *p >= '0' && *p <= '9') {
    v = v * 10 + (*p - '0');
    if (v > (int64_t(1) << 62)) throw std::runtime_error("index out of range in an entry line");
    ++p;
  }
  out = v;
  return p;
}

// std::from_chars rounds correctly (as strtod and Python's float do) and
// ignores the locale; it takes no leading '+', which Matrix Market allows.
const char* ParseValue(const char* p, const char* end, double& out) {
  p = SkipSpace(p, end);
  const char* first = (p < end && *p == '+' && p + 1 < end && p[1] != '-' && p[1] != '+') ? p + 1 : p;
  const auto r = std::from_chars(first, end, out);
  if (r.ec == std::errc::invalid_argument || r.ptr == first) throw std::runtime_error("malformed value in an entry line");
  if (r.ec == std::errc::result_out_of_range) {
    // from_chars leaves `out` untouched on over- or underflow; strtod gives +-inf or the rounded subnormal/zero
    out = std::strtod(std::string(first, r.ptr).c_str(), nullptr);
  }
  return r.ptr;
}

// Parses the entry lines in [from, to) (whole lines).  Array files give the
// linear position of their first value in `position`.
void ParseSlice(const FileView& d, size_t from, size_t to, const Header& h, int64_t position,
                Triplets& out, std::string& error) {
  try {
    // array files: (i, j) of the slice's first value, then advanced value by value
    // (column-major; symmetric storage keeps the lower triangle, skew the strict one)
    const int64_t skip = h.symmetry == Symmetry::kSkew ? 1 : 0;
    int64_t ai = 0;
    int64_t aj = 0;
    if (!h.coordinate) {
      if (h.symmetry == Symmetry::kGeneral) {
        aj = position / h.rows;
        ai = position % h.rows;
      } else {
        int64_t k = position;
        while (aj < h.cols && k >= h.rows - aj - skip) {
          k -= h.rows - aj - skip;
          ++aj;
        }
        ai = aj + skip + k;
      }
    }
    const char* p = d.data() + from;
    const char* const stop = d.data() + to;
    // room for every line of the slice (twice for mirrored entries)
    const size_t lines = static_cast<size_t>(std::count(p, stop, '\n')) + 1;
    const size_t room = h.symmetry == Symmetry::kGeneral ? lines : 2 * lines;
    out.row.reserve(room);
    out.col.reserve(room);
    out.val.reserve(room);
    while (p < stop) {
      const char* newline = static_cast<const char*>(std::memchr(p, '\n', static_cast<size_t>(stop - p)));
      const char* next = newline != nullptr ? newline + 1 : stop;
      const char* end = newline != nullptr ? newline : stop;
      if (end > p && end[-1] == '\r') --end;
      const char* q = SkipSpace(p, end);
      if (q == end || *p == '%') {
        p = next;
        continue;
      }
      int64_t i;
      int64_t j;
      double v = 1.0;
      if (h.coordinate) {
        q = ParseIndex(q, end, i);
        q = ParseIndex(q, end, j);
        if (h.field != Field::kPattern) q = ParseValue(q, end, v);
        if (i < 1 || i > h.rows || j < 1 || j > h.cols) throw std::runtime_error("entry index out of range");
        --i;
        --j;
      } else {
        q = ParseValue(q, end, v);
        if (aj >= h.cols) throw std::runtime_error("more values than the array holds");
        i = ai;
        j = aj;
        if (++ai >= h.rows) {
          ++aj;
          ai = h.symmetry == Symmetry::kGeneral ? 0 : aj + skip;
        }
      }
      if (SkipSpace(q, end) != end) throw std::runtime_error("unexpected text after an entry");
      if (h.symmetry == Symmetry::kSkew && i == j) throw std::runtime_error("skew-symmetric diagonal entry");
      ++out.stored;
      out.row.push_back(i);
      out.col.push_back(j);
      out.val.push_back(v);
      if (h.symmetry != Symmetry::kGeneral && i != j) {
        out.row.push_back(j);
        out.col.push_back(i);
        out.val.push_back(h.symmetry == Symmetry::kSkew ? -v : v);
      }
      p = next;
    }
  } catch (const std::exception& ex) {
    error = ex.what();
  }
}

// Line starts of the entry region, split into `parts` slices of whole lines.
std::vector<size_t> SliceBounds(const FileView& d, size_t begin, int parts) {
  const size_t size = d.size();
  std::vector<size_t> bounds{begin};
  for (int k = 1; k < parts; ++k) {
    size_t at = begin + (size - begin) * static_cast<size_t>(k) / static_cast<size_t>(parts);
    at = std::max(at, bounds.back());
    while (at < size && at > begin && d[at - 1] != '\n') ++at;
    bounds.push_back(at);
  }
  bounds.push_back(size);
  return bounds;
}

// Array files: the number of value lines before each slice start (values are one per line).
int64_t CountValueLines(const FileView& d, size_t from, size_t to) {
  int64_t count = 0;
  size_t at = from;
  size_t b;
  size_t e;
  while (at < to && NextLine(d, at, b, e)) {
    if (d[b] == '%' || Blank(d, b, e)) continue;
    ++count;
  }
  return count;
}

// f(0) .. f(parts - 1), one thread each (inline when parts == 1).
template <class F>
void RunParallel(int parts, F f) {
  if (parts <= 1) {
    f(0);
    return;
  }
  std::vector<std::thread> pool;
  for (int k = 0; k < parts; ++k) pool.emplace_back(f, k);
  for (auto& t : pool) t.join();
}

// The result in the arrays the C ABI hands out (new[], released by free_mem).
struct CscOut {
  int64_t rows = 0;
  int64_t cols = 0;
  int64_t nnz = 0;
  std::unique_ptr<int64_t[]> ptr;
  std::unique_ptr<int64_t[]> idx;
  std::unique_ptr<double[]> val;
};

CscOut ReadMatrixMarket(const char* path, int threads) {
  const FileView d(path);
  size_t at = 0;
  const Header h = ParseHeader(d, at);
  if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
  const size_t region = d.size() - at;
  // one slice per MiB of entries, at most one per thread, and per-slice column
  // counts of at most 256 MiB in total
  size_t parts_cap = std::min<size_t>(static_cast<size_t>(threads), region / (1 << 20) + 1);
  parts_cap = std::min<size_t>(parts_cap, (size_t(256) << 20) / (8 * (static_cast<size_t>(h.cols) + 1)) + 1);
  const int parts = static_cast<int>(std::max<size_t>(1, parts_cap));
  const std::vector<size_t> bounds = SliceBounds(d, at, parts);
  std::vector<int64_t> first_position(static_cast<size_t>(parts), 0);
  if (!h.coordinate) {
    for (int k = 1; k < parts; ++k) first_position[k] = first_position[k - 1] + CountValueLines(d, bounds[k - 1], bounds[k]);
  }
  std::vector<Triplets> slices(static_cast<size_t>(parts));
  std::vector<std::string> errors(static_cast<size_t>(parts));
  RunParallel(parts, [&](int k) {
    ParseSlice(d, bounds[k], bounds[k + 1], h, first_position[k], slices[k], errors[k]);
  });
  for (const auto& e : errors) {
    if (!e.empty()) throw std::runtime_error(e);
  }
  // the file must hold exactly the announced number of entries
  int64_t stored = 0;
  for (const auto& sl : slices) stored += sl.stored;
  if (stored != h.entries) {
    throw std::runtime_error("expected " + std::to_string(h.entries) + " entries, found " + std::to_string(stored));
  }
  // Bucket by column: slice k's entries of column c go after those of the
  // slices before it, in file order (offsets from per-slice column counts).
  const size_t cols = static_cast<size_t>(h.cols);
  std::vector<std::vector<int64_t>> at_col(slices.size());
  RunParallel(parts, [&](int k) {
    at_col[k].assign(cols + 1, 0);
    for (const int64_t c : slices[k].col) ++at_col[k][c];
  });
  std::vector<int64_t> col_begin(cols + 1, 0);
  int64_t running = 0;
  for (size_t c = 0; c < cols; ++c) {
    col_begin[c] = running;
    for (int k = 0; k < parts; ++k) {
      const int64_t n = at_col[k][c];
      at_col[k][c] = running;
      running += n;
    }
  }
  col_begin[cols] = running;
  const int64_t total = running;
  std::vector<int64_t> rows(static_cast<size_t>(total));
  std::vector<double> vals(static_cast<size_t>(total));
  RunParallel(parts, [&](int k) {
    Triplets& sl = slices[k];
    std::vector<int64_t>& cursor = at_col[k];
    for (size_t q = 0; q < sl.col.size(); ++q) {
      const int64_t to = cursor[sl.col[q]]++;
      rows[to] = sl.row[q];
      vals[to] = sl.val[q];
    }
    sl = Triplets();
    cursor = std::vector<int64_t>();
  });
  // Per column: rows ascending (stable, so duplicates stay in file order),
  // duplicates summed, explicit zeros dropped; compacted in place.
  std::vector<int64_t> kept(cols, 0);
  const int64_t chunk = static_cast<int64_t>((cols + static_cast<size_t>(parts) - 1) / static_cast<size_t>(parts));
  RunParallel(parts, [&](int k) {
    std::vector<std::pair<int64_t, double>> scratch;
    const int64_t c_end = std::min<int64_t>(h.cols, (k + 1) * chunk);
    for (int64_t c = k * chunk; c < c_end; ++c) {
      const int64_t b = col_begin[c];
      const int64_t e = col_begin[c + 1];
      bool sorted = true;
      for (int64_t q = b + 1; q < e && sorted; ++q) sorted = rows[q - 1] <= rows[q];
      if (!sorted) {
        scratch.clear();
        for (int64_t q = b; q < e; ++q) scratch.emplace_back(rows[q], vals[q]);
        std::stable_sort(scratch.begin(), scratch.end(),
                         [](const auto& x, const auto& y) { return x.first < y.first; });
        for (int64_t q = b; q < e; ++q) {
          rows[q] = scratch[q - b].first;
          vals[q] = scratch[q - b].second;
        }
      }
      int64_t w = b;
      int64_t q = b;
      while (q < e) {
        const int64_t r = rows[q];
        double v = vals[q++];
        while (q < e && rows[q] == r) v += vals[q++];
        if (v != 0.0) {  // eliminate_zeros: explicit (and cancelled) zeros leave, NaN stays
          rows[w] = r;
          vals[w] = v;
          ++w;
        }
      }
      kept[c] = w - b;
    }
  });
  CscOut out;
  out.rows = h.rows;
  out.cols = h.cols;
  out.ptr.reset(new int64_t[cols + 1]);
  out.ptr[0] = 0;
  for (size_t c = 0; c < cols; ++c) out.ptr[c + 1] = out.ptr[c] + kept[c];
  out.nnz = out.ptr[cols];
  out.idx.reset(new int64_t[out.nnz > 0 ? out.nnz : 1]);
  out.val.reset(new double[out.nnz > 0 ? out.nnz : 1]);
  RunParallel(parts, [&](int k) {
    const int64_t c_end = std::min<int64_t>(h.cols, (k + 1) * chunk);
    for (int64_t c = k * chunk; c < c_end; ++c) {
      std::copy(rows.begin() + col_begin[c], rows.begin() + col_begin[c] + kept[c], out.idx.get() + out.ptr[c]);
      std::copy(vals.begin() + col_begin[c], vals.begin() + col_begin[c] + kept[c], out.val.get() + out.ptr[c]);
    }
  });
  return out;
}

void WriteMatrixMarket(const char* path, const MatrixData& m, bool symmetric) {
  if (path == nullptr) throw std::invalid_argument("path must not be null");
  if (m.rows <= 0 || m.cols <= 0 || m.nnz < 0) throw std::invalid_argument("matrix dimensions must be positive");
  if (symmetric && m.rows != m.cols) throw std::invalid_argument("a symmetric matrix must be square");
  if (m.col_offsets == nullptr || (m.nnz > 0 && (m.row_indices == nullptr || m.values == nullptr))) {
    throw std::invalid_argument("matrix arrays must not be null");
  }
  int64_t written = 0;
  for (int64_t c = 0; c < m.cols; ++c) {
    if (m.col_offsets[c + 1] < m.col_offsets[c]) throw std::invalid_argument("column offsets must be non-decreasing");
    for (int64_t p = m.col_offsets[c]; p < m.col_offsets[c + 1]; ++p) {
      const int64_t r = m.row_indices[p];
      if (r < 0 || r >= m.rows) throw std::invalid_argument("row index out of range");
      if (!symmetric || r >= c) ++written;
    }
  }
  FILE* f = std::fopen(path, "wb");
  if (f == nullptr) throw std::runtime_error(std::string("cannot create ") + path + ": " + std::strerror(errno));
  std::string text;
  text.reserve(1 << 20);
  text += symmetric ? "%%MatrixMarket matrix coordinate real symmetric\n" : "%%MatrixMarket matrix coordinate real general\n";
  text += std::to_string(m.rows) + " " + std::to_string(m.cols) + " " + std::to_string(written) + "\n";
  char line[96];
  bool failed = false;
  for (int64_t c = 0; c < m.cols && !failed; ++c) {
    for (int64_t p = m.col_offsets[c]; p < m.col_offsets[c + 1]; ++p) {
      const int64_t r = m.row_indices[p];
      if (symmetric && r < c) continue;
      // 17 significant digits: every double reads back to the same bits
      const int len = std::snprintf(line, sizeof(line), "%lld %lld %.17g\n", static_cast<long long>(r + 1),
                                    static_cast<long long>(c + 1), m.values[p]);
      text.append(line, static_cast<size_t>(len));
      if (text.size() > (1u << 20)) {
        failed |= std::fwrite(text.data(), 1, text.size(), f) != text.size();
        text.clear();
      }
    }
  }
  if (!failed && !text.empty()) failed = std::fwrite(text.data(), 1, text.size(), f) != text.size();
  failed |= std::fclose(f) != 0;
  if (failed) throw std::runtime_error(std::string("cannot write ") + path);
}

void CopyMessage(const std::string& message, char* out, int64_t capacity) {
  if (out == nullptr || capacity <= 0) return;
  const size_t n = std::min<size_t>(message.size(), static_cast<size_t>(capacity - 1));
  std::memcpy(out, message.data(), n);
  out[n] = '\0';
}

}  // namespace
}  // namespace spai

extern "C" {

Result spai_mtx_read(const char* path, int64_t threads) {
  Result out{};
  try {
    spai::CscOut m = spai::ReadMatrixMarket(path, static_cast<int>(threads));
    out.rows = m.rows;
    out.cols = m.cols;
    out.nnz = m.nnz;
    out.col_offsets = m.ptr.release();
    out.row_indices = m.idx.release();
    out.values = m.val.release();
  } catch (const std::exception& ex) {
    out = Result{};
    const std::string message = ex.what();
    out.error_message = new char[message.size() + 1];
    std::memcpy(out.error_message, message.c_str(), message.size() + 1);
  }
  return out;
}

int64_t spai_mtx_write(const char* path, MatrixData m, int64_t symmetric, char* error, int64_t error_capacity) {
  try {
    spai::WriteMatrixMarket(path, m, symmetric != 0);
    return 0;
  } catch (const std::exception& ex) {
    spai::CopyMessage(ex.what(), error, error_capacity);
    return -1;
  }
}

}  // extern "C"
