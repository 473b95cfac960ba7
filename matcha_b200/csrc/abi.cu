// Error reporting, version and launch timing of the matcha_b200 C ABI.
#include <stdio.h>
#include <string.h>
#include <atomic>
#include <mutex>
#include <vector>
#include "common.cuh"

namespace {
thread_local char g_last_error[512] = {0};

// Launch timing: a pool of event pairs, filled in launch order while recording is on.
struct ProfLaunch {
  const char* name;
  cudaEvent_t begin, end;
};
std::atomic<bool> g_prof_on{false};
std::mutex g_prof_mu;
std::vector<cudaEvent_t> g_prof_pool;    // 2 per launch
std::vector<ProfLaunch> g_prof_launches;  // recorded
size_t g_prof_cap = 0;
int g_prof_dropped = 0;
bool g_prof_open = false;  // a begin event is waiting for its end

void prof_clear() {
  for (cudaEvent_t e : g_prof_pool) cudaEventDestroy(e);
  g_prof_pool.clear();
  g_prof_launches.clear();
  g_prof_cap = 0;
  g_prof_dropped = 0;
  g_prof_open = false;
}
}  // namespace

void mtb_prof_begin(cudaStream_t st) {
  if (!g_prof_on.load(std::memory_order_relaxed)) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  const size_t n = g_prof_launches.size();
  if (n >= g_prof_cap) {
    ++g_prof_dropped;
    return;
  }
  if (cudaEventRecord(g_prof_pool[2 * n], st) == cudaSuccess) g_prof_open = true;
}

void mtb_prof_end(cudaStream_t st, const char* kernel) {
  if (!g_prof_on.load(std::memory_order_relaxed)) return;
  std::lock_guard<std::mutex> lk(g_prof_mu);
  if (!g_prof_open) return;
  g_prof_open = false;
  const size_t n = g_prof_launches.size();
  if (cudaEventRecord(g_prof_pool[2 * n + 1], st) == cudaSuccess)
    g_prof_launches.push_back({kernel, g_prof_pool[2 * n], g_prof_pool[2 * n + 1]});
}

extern "C" int mtb_profile_start(int max_launches) {
  MTB_ARG_CHECK(max_launches > 0 && max_launches <= (1 << 20), "max_launches must be in [1, 2^20]");
  g_prof_on.store(false);
  std::lock_guard<std::mutex> lk(g_prof_mu);
  prof_clear();
  g_prof_pool.assign((size_t)2 * max_launches, nullptr);
  for (cudaEvent_t& e : g_prof_pool) {
    cudaError_t err = cudaEventCreate(&e);
    if (err != cudaSuccess) {
      e = nullptr;
      prof_clear();
      mtb_set_last_error(cudaGetErrorString(err), __FILE__, __LINE__);
      return err == cudaErrorMemoryAllocation ? MTB_ERR_OOM : MTB_ERR_CUDA;
    }
  }
  g_prof_cap = (size_t)max_launches;
  g_prof_on.store(true);
  return MTB_OK;
}

extern "C" int mtb_profile_stop(void) {
  g_prof_on.store(false);
  return MTB_OK;
}

extern "C" int mtb_profile_read(int max_entries, char* names, float* ms, int* launches, int* n_entries,
                                int* dropped) {
  MTB_ARG_CHECK(max_entries > 0 && names && ms && launches && n_entries && dropped, "bad profile_read arguments");
  std::lock_guard<std::mutex> lk(g_prof_mu);
  int n = 0;
  for (const ProfLaunch& l : g_prof_launches) {
    MTB_CUDA_TRY(cudaEventSynchronize(l.end));
    float t = 0.f;
    MTB_CUDA_TRY(cudaEventElapsedTime(&t, l.begin, l.end));
    int k = 0;
    while (k < n && strncmp(names + (size_t)k * MTB_PROFILE_NAME_LEN, l.name, MTB_PROFILE_NAME_LEN - 1) != 0) ++k;
    if (k == n) {
      if (n == max_entries) continue;
      strncpy(names + (size_t)k * MTB_PROFILE_NAME_LEN, l.name, MTB_PROFILE_NAME_LEN - 1);
      names[(size_t)k * MTB_PROFILE_NAME_LEN + MTB_PROFILE_NAME_LEN - 1] = 0;
      ms[k] = 0.f;
      launches[k] = 0;
      ++n;
    }
    ms[k] += t;
    launches[k] += 1;
  }
  *n_entries = n;
  *dropped = g_prof_dropped;
  return MTB_OK;
}

void mtb_set_last_error(const char* msg, const char* file, int line) {
  const char* base = strrchr(file, '/');
  snprintf(g_last_error, sizeof(g_last_error), "%s (%s:%d)", msg, base ? base + 1 : file, line);
}

extern "C" int mtb_version(void) { return 100; }

extern "C" const char* mtb_last_error(void) { return g_last_error; }
