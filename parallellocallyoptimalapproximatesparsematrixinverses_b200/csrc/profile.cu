#include "profile.cuh"

#include <atomic>
#include <map>
#include <mutex>
#include <vector>

namespace spai {
namespace prof {

namespace {

struct Pending {
  std::string name;
  cudaEvent_t start;
  cudaEvent_t stop;
  double bytes;
};

struct Totals {
  double ms = 0.0;
  int64_t count = 0;
  double bytes = 0.0;
};

std::atomic<bool> g_enabled{false};
std::mutex g_mutex;
std::vector<Pending> g_pending;
std::map<std::string, Totals> g_totals;
std::vector<cudaEvent_t> g_free_events;  // recycled so a scope never creates events in steady state

cudaEvent_t TakeEvent() {
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_free_events.empty()) {
      cudaEvent_t e = g_free_events.back();
      g_free_events.pop_back();
      return e;
    }
  }
  cudaEvent_t e = nullptr;
  if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
  return e;
}

void Drain() {
  for (Pending& p : g_pending) {
    float ms = 0.0f;
    if (cudaEventSynchronize(p.stop) == cudaSuccess && cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
      Totals& t = g_totals[p.name];
      t.ms += ms;
      t.count += 1;
      t.bytes += p.bytes;
    }
    g_free_events.push_back(p.start);
    g_free_events.push_back(p.stop);
  }
  g_pending.clear();
}

}  // namespace

bool Enabled() { return g_enabled.load(std::memory_order_relaxed); }

void SetEnabled(bool on) { g_enabled.store(on); }

void Reset() {
  std::lock_guard<std::mutex> lock(g_mutex);
  Drain();
  g_totals.clear();
}

void AddBytes(const char* name, double bytes) {
  if (!Enabled()) return;
  std::lock_guard<std::mutex> lock(g_mutex);
  g_totals[name].bytes += bytes;
}

bool Read(const std::string& name, double* ms, int64_t* count, double* bytes) {
  std::lock_guard<std::mutex> lock(g_mutex);
  Drain();
  auto it = g_totals.find(name);
  if (it == g_totals.end()) {
    *ms = 0.0;
    *count = 0;
    *bytes = 0.0;
    return false;
  }
  *ms = it->second.ms;
  *count = it->second.count;
  *bytes = it->second.bytes;
  return true;
}

Scope::Scope(cudaStream_t stream, const char* name, double bytes) : stream_(stream), name_(name), bytes_(bytes) {
  if (!Enabled()) return;
  start_ = TakeEvent();
  if (start_ == nullptr) return;
  cudaEventRecord(start_, stream_);
  active_ = true;
}

Scope::~Scope() {
  if (!active_) return;
  cudaEvent_t stop = TakeEvent();
  if (stop == nullptr) return;
  cudaEventRecord(stop, stream_);
  std::lock_guard<std::mutex> lock(g_mutex);
  g_pending.push_back(Pending{name_, start_, stop, bytes_});
  // fold finished pairs into the totals without blocking, so events recycle
  if (g_pending.size() >= 256) {
    size_t done = 0;
    while (done < g_pending.size() && cudaEventQuery(g_pending[done].stop) == cudaSuccess) ++done;
    for (size_t i = 0; i < done; ++i) {
      Pending& p = g_pending[i];
      float ms = 0.0f;
      if (cudaEventElapsedTime(&ms, p.start, p.stop) == cudaSuccess) {
        Totals& t = g_totals[p.name];
        t.ms += ms;
        t.count += 1;
        t.bytes += p.bytes;
      }
      g_free_events.push_back(p.start);
      g_free_events.push_back(p.stop);
    }
    g_pending.erase(g_pending.begin(), g_pending.begin() + static_cast<std::ptrdiff_t>(done));
  }
}

}  // namespace prof
}  // namespace spai
