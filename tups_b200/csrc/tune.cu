// Tile-shape tuner (no counterpart in the reference).
//
// The BSE GEMM and the crossing kernel each come in several instantiations
// (tile sizes, warps, pipeline stages, column layouts).  The first call of a
// context on a new shape times every candidate on the call's own operands
// with CUDA events on the library's stream, keeps the fastest, and records
// the choice process-wide under a key naming the kernel and the shape, so
// later calls and later contexts of the same shape reuse it without timing.
//
// Only candidates that compute every output element with the same
// arithmetic in the same order are ever compared (they differ in how the
// elements are spread over CTAs and warps, not in the K order of any sum),
// so the tuner's choice never changes a result bit.  Nothing is tuned while
// a stream capture is active; the default candidate (index 0) runs then.
#include <cstdio>
#include <map>
#include <mutex>
#include <sstream>

#include "tups_device.cuh"

namespace tups {

namespace {
struct TuneEntry {
  int choice = 0;
  std::vector<std::string> names;
  std::vector<double> ms;
};
std::mutex g_tune_mu;
std::map<std::string, TuneEntry> g_tune;
// candidates fixed by name for every key that starts with a prefix
std::vector<std::pair<std::string, std::string>> g_force;
}  // namespace

int tune_forced(const std::string& key, const std::vector<std::string>& names) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  for (const auto& f : g_force)
    if (key.compare(0, f.first.size(), f.first) == 0)
      for (size_t c = 0; c < names.size(); c++)
        if (names[c] == f.second) return (int)c;
  return -1;
}

bool tune_get(const std::string& key, int* choice) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  auto it = g_tune.find(key);
  if (it == g_tune.end()) return false;
  *choice = it->second.choice;
  return true;
}

void tune_put(const std::string& key, int choice, const std::vector<std::string>& names,
              const std::vector<double>& ms) {
  std::lock_guard<std::mutex> lock(g_tune_mu);
  TuneEntry& e = g_tune[key];
  e.choice = choice;
  e.names = names;
  e.ms = ms;
}

bool tune_allowed(tups_ctx* ctx) {
  if (!ctx->autotune) return false;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(ctx->stream, &cs) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return cs == cudaStreamCaptureStatusNone;
}

int tune_pick(tups_ctx* ctx, const std::string& key, int n_cand, const std::vector<std::string>& names,
              const std::function<int(int)>& run, int reps, int* choice) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
    if (e0) cudaEventDestroy(e0);
    cudaGetLastError();
    return set_error(ctx, TUPS_ERR_CUDA, "tuner events");
  }
  std::vector<double> best(n_cand, -1.0);
  int rc = TUPS_OK;
  for (int rep = 0; rep < reps && rc == TUPS_OK; rep++)
    for (int c = 0; c < n_cand && rc == TUPS_OK; c++) {
      cudaEventRecord(e0, ctx->stream);
      rc = run(c);
      cudaEventRecord(e1, ctx->stream);
      if (rc) break;
      float ms = 0.0f;
      if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess) {
        cudaGetLastError();
        rc = set_error(ctx, TUPS_ERR_CUDA, "tuner timing");
        break;
      }
      if (best[c] < 0.0 || ms < best[c]) best[c] = ms;
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  int pick = 0;
  for (int c = 1; c < n_cand; c++)
    if (best[c] < best[pick]) pick = c;
  tune_put(key, pick, names, best);
  ctx->tile_tunings++;
  *choice = pick;
  return TUPS_OK;
}

}  // namespace tups

extern "C" int tups_set_autotune(tups_ctx* ctx, int enable) {
  if (!ctx) return TUPS_ERR_BADARG;
  ctx->autotune = enable != 0;
  return TUPS_OK;
}

extern "C" int tups_set_tuning(const char* key_prefix, const char* name) {
  std::lock_guard<std::mutex> lock(tups::g_tune_mu);
  if (!key_prefix) {
    tups::g_force.clear();
    return TUPS_OK;
  }
  const std::string k(key_prefix);
  for (size_t i = 0; i < tups::g_force.size(); i++)
    if (tups::g_force[i].first == k) {
      tups::g_force.erase(tups::g_force.begin() + i);
      break;
    }
  if (name) tups::g_force.emplace_back(k, std::string(name));
  return TUPS_OK;
}

extern "C" int tups_get_tuning(char* buf, size_t len) {
  std::ostringstream os;
  {
    std::lock_guard<std::mutex> lock(tups::g_tune_mu);
    for (const auto& kv : tups::g_tune) {
      os << kv.first << " | choice " << kv.second.names[kv.second.choice] << " |";
      for (size_t i = 0; i < kv.second.names.size(); i++) {
        char t[64];
        std::snprintf(t, sizeof t, " %s=%.4f", kv.second.names[i].c_str(), kv.second.ms[i]);
        os << t;
      }
      os << "\n";
    }
  }
  const std::string s = os.str();
  if (!buf || len == 0) return (int)s.size() + 1;
  const size_t n = std::min(len - 1, s.size());
  std::memcpy(buf, s.data(), n);
  buf[n] = '\0';
  return (int)s.size() + 1;
}
