// Per-phase device timing (the reference prints wall-clock seconds per phase,
// SRC/loop.f90:64-178) and stream event markers.
#include "tups_internal.h"

namespace tups {

static constexpr int kMaxPending = 256;

void phase_begin(tups_ctx* ctx, int p) {
  if (!ctx->timing) return;
  if (ctx->ev_used[p] >= kMaxPending) phase_collect(ctx);
  int i = ctx->ev_used[p];
  if ((int)ctx->ev_begin[p].size() <= i) {
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    ctx->ev_begin[p].push_back(a);
    ctx->ev_end[p].push_back(b);
  }
  cudaEventRecord(ctx->ev_begin[p][i], ctx->stream);
}

void phase_end(tups_ctx* ctx, int p) {
  if (!ctx->timing) return;
  int i = ctx->ev_used[p];
  cudaEventRecord(ctx->ev_end[p][i], ctx->stream);
  ctx->ev_used[p] = i + 1;
}

void phase_collect(tups_ctx* ctx) {
  cudaStreamSynchronize(ctx->stream);
  for (int p = 0; p < TUPS_NPHASE; p++) {
    for (int i = 0; i < ctx->ev_used[p]; i++) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, ctx->ev_begin[p][i], ctx->ev_end[p][i]) == cudaSuccess) {
        ctx->phase_ms[p] += ms;
        ctx->phase_count[p] += 1;
      }
    }
    ctx->ev_used[p] = 0;
  }
  cudaGetLastError();
}

void destroy_events(tups_ctx* ctx) {
  for (int p = 0; p < TUPS_NPHASE; p++) {
    for (auto e : ctx->ev_begin[p]) cudaEventDestroy(e);
    for (auto e : ctx->ev_end[p]) cudaEventDestroy(e);
    ctx->ev_begin[p].clear();
    ctx->ev_end[p].clear();
  }
  for (auto& m : ctx->marks)
    if (m) {
      cudaEventDestroy(m);
      m = nullptr;
    }
  for (auto& m : ctx->tune_ev)
    if (m) {
      cudaEventDestroy(m);
      m = nullptr;
    }
}

}  // namespace tups

extern "C" int tups_set_timing(tups_ctx* ctx, int enable) {
  if (!ctx) return TUPS_ERR_BADARG;
  if (ctx->timing) tups::phase_collect(ctx);
  ctx->timing = enable != 0;
  for (int p = 0; p < TUPS_NPHASE; p++) {
    ctx->phase_ms[p] = 0.0;
    ctx->phase_count[p] = 0;
    ctx->ev_used[p] = 0;
  }
  return TUPS_OK;
}

extern "C" int tups_get_phase_times(tups_ctx* ctx, double* ms, int* count) {
  if (!ctx) return TUPS_ERR_BADARG;
  tups::phase_collect(ctx);
  for (int p = 0; p < TUPS_NPHASE; p++) {
    if (ms) ms[p] = ctx->phase_ms[p];
    if (count) count[p] = ctx->phase_count[p];
  }
  return TUPS_OK;
}

extern "C" int tups_record_event(tups_ctx* ctx, int slot) {
  if (!ctx || slot < 0 || slot >= 8) return TUPS_ERR_BADARG;
  if (!ctx->marks[slot]) {
    cudaError_t e = cudaEventCreate(&ctx->marks[slot]);
    if (e != cudaSuccess) return tups::cuda_check(ctx, e, "cudaEventCreate");
  }
  return tups::cuda_check(ctx, cudaEventRecord(ctx->marks[slot], ctx->stream), "cudaEventRecord");
}

extern "C" int tups_event_elapsed(tups_ctx* ctx, int a, int b, double* ms) {
  if (!ctx || !ms || a < 0 || a >= 8 || b < 0 || b >= 8 || !ctx->marks[a] || !ctx->marks[b])
    return TUPS_ERR_BADARG;
  int rc = tups::cuda_check(ctx, cudaEventSynchronize(ctx->marks[b]), "cudaEventSynchronize");
  if (rc) return rc;
  float f = 0.f;
  rc = tups::cuda_check(ctx, cudaEventElapsedTime(&f, ctx->marks[a], ctx->marks[b]), "cudaEventElapsedTime");
  *ms = f;
  return rc;
}
