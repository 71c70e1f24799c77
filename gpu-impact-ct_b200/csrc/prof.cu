// prof.cu -- event-based per-kernel timing and launch counting (see prof.cuh).
#include <atomic>
#include <mutex>
#include <vector>

#include "../../include/impact_b200.h"
#include "prof.cuh"

namespace impact {
namespace prof {

namespace {
using Pending = Pair;
std::mutex mu;
bool on = false;
bool capturing = false;
std::vector<Pair> captured;
std::vector<cudaEvent_t> pool;
std::vector<Pending> pending;
std::vector<cudaEvent_t> open_start;  // token -> start event
long long launches[K_COUNT] = {};
double total_ms[K_COUNT] = {};
double total_bytes[K_COUNT] = {};
std::atomic<long long> g_count{0};

cudaEvent_t take() {
  if (!pool.empty()) {
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}
const char* kNames[K_COUNT] = {"jacobi_sweep", "jacobi_init2", "div_grad_dot", "x_update", "p_update",
                               "r_update", "nl_rhs", "project", "divergence2", "mg_sweep", "mg_init",
                               "mg_residual", "mg_transfer", "mg_pre_smooth", "mg_post_smooth", "mx_residual", "mx_apply",
                               "mg_coarse_tail", "kr_init"};
}  // namespace

bool enabled() { return on; }

int begin(cudaStream_t s) {
  if (!on) return -1;
  std::lock_guard<std::mutex> lk(mu);
  cudaEvent_t e = take();
  if (capturing)
    cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
  else
    cudaEventRecord(e, s);
  open_start.push_back(e);
  return (int)open_start.size() - 1;
}

void end(int token, int kid, double bytes, cudaStream_t s) {
  if (token < 0) return;
  std::lock_guard<std::mutex> lk(mu);
  cudaEvent_t e = take();
  if (capturing)
    cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
  else
    cudaEventRecord(e, s);
  (capturing ? captured : pending).push_back({kid, bytes, open_start[token], e});
  open_start[token] = nullptr;
  // compact the token table once every open pair is closed
  bool all_closed = true;
  for (cudaEvent_t x : open_start)
    if (x) {
      all_closed = false;
      break;
    }
  if (all_closed) open_start.clear();
}

void flush() {
  if (!on) return;
  std::lock_guard<std::mutex> lk(mu);
  std::vector<Pending> keep;
  for (Pending& p : pending) {
    if (cudaEventQuery(p.b) != cudaSuccess) {
      keep.push_back(p);
      continue;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    launches[p.kid] += 1;
    total_ms[p.kid] += ms;
    total_bytes[p.kid] += p.bytes;
    pool.push_back(p.a);
    pool.push_back(p.b);
  }
  pending.swap(keep);
}

void count(long long n) { g_count += n; }

void capture_begin() {
  std::lock_guard<std::mutex> lk(mu);
  capturing = true;
  captured.clear();
}

std::vector<Pair> capture_end() {
  std::lock_guard<std::mutex> lk(mu);
  capturing = false;
  std::vector<Pair> out;
  out.swap(captured);
  return out;
}

void graph_account(const std::vector<Pair>& pairs) {
  std::lock_guard<std::mutex> lk(mu);
  for (const Pair& p : pairs) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.a, p.b) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    launches[p.kid] += 1;
    total_ms[p.kid] += ms;
    total_bytes[p.kid] += p.bytes;
  }
}

void graph_release(std::vector<Pair>& pairs) {
  std::lock_guard<std::mutex> lk(mu);
  for (const Pair& p : pairs) {
    pool.push_back(p.a);
    pool.push_back(p.b);
  }
  pairs.clear();
}

}  // namespace prof
}  // namespace impact

using namespace impact::prof;

extern "C" void impact_b200_profile_enable(int enable) {
  std::lock_guard<std::mutex> lk(mu);
  on = enable != 0;
}
extern "C" void impact_b200_profile_reset(void) {
  std::lock_guard<std::mutex> lk(mu);
  for (int k = 0; k < K_COUNT; ++k) {
    launches[k] = 0;
    total_ms[k] = 0.0;
    total_bytes[k] = 0.0;
  }
}
extern "C" int impact_b200_profile_read(int kid, long long* n, double* ms, double* bytes, const char** name) {
  flush();
  if (kid < 0 || kid >= K_COUNT) return -1;
  std::lock_guard<std::mutex> lk(mu);
  if (n) *n = launches[kid];
  if (ms) *ms = total_ms[kid];
  if (bytes) *bytes = total_bytes[kid];
  if (name) *name = kNames[kid];
  return 0;
}
extern "C" long long impact_b200_launch_count(void) { return g_count.load(); }
