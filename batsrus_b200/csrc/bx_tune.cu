// bx_tune.cu -- the autotuner: the table of launch-shape knobs, the
// Krylov-kernel tuning, and the C ABI (bx_autotune, bx_tune_info,
// bx_tune_set).  No counterpart in the reference, whose launch shapes are
// fixed by its OpenACC directives.
#include <cuda_runtime.h>

#include <cstring>

#include "bx_core.h"
#include "bx_krylov.cuh"
#include "bx_tune.h"

namespace bx {

static const int g_default[kNumTune] = {2, 4, 2, 1, 192, 0, 3};
static TuneKnobInfo g_knobs[kNumTune] = {
    {"stage_ctas_per_sm", 4, {1, 2, 3, 4}, 2, 0, {}},
    {"krylov_ctas_per_sm", 4, {2, 4, 6, 8}, 4, 0, {}},
    {"krylov_unroll", 3, {1, 2, 4}, 2, 0, {}},
    {"heat_ilu_warps", 3, {1, 2, 4}, 1, 0, {}},
    // 0: 8 x the widest wavefront, one pass each; 128, 192, 256: several passes per
    // wavefront, more CTAs (grid blocks) per SM.  BF16 apply at 128^3: 0.65, 0.55, 0.50,
    // 0.60 ms
    {"bilu_threads", 4, {0, 128, 192, 256}, 192, 0, {}},
    {"stage_variant", 4, {0, 1, 2, 3}, 0, 0, {}},
    // changes the rounding of the Krylov coefficients: a setting, not timed
    {"krylov_gs_steps", 4, {1, 2, 3, 4}, 3, 0, {}},
};

TuneKnobInfo &tune_knob(int knob) { return g_knobs[knob]; }

// time `reps` calls of fn on stream st (after one untimed call)
template <class F>
static int time_ms(cudaStream_t st, int reps, F &&fn, float &ms) {
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return core_fail(BX_ERR_CUDA, "cudaEventCreate");
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return core_fail(BX_ERR_CUDA, "cudaEventCreate");
  }
  fn();
  cudaEventRecord(e0, st);
  for (int r = 0; r < reps; r++) fn();
  cudaEventRecord(e1, st);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return core_fail(BX_ERR_CUDA, "autotune timing: %s", cudaGetErrorString(e));
  ms = t / reps;
  return BX_OK;
}

// the middle MGS pass (w -= h V_q-1; w . V_q) on three scratch vectors of
// 2^24 doubles (larger than L2), for every pair of grid and unroll depth
int tune_krylov() {
  Core c = core();
  TuneKnobInfo &kc0 = g_knobs[kTuneKryCtas], &ku0 = g_knobs[kTuneKryUnroll];
  if (!c.ready || (kc0.tuned == 2 && ku0.tuned == 2)) return BX_OK;
  const long n = 1l << 24;
  double *buf = nullptr, *partial = nullptr;
  unsigned *cnt = nullptr;
  if (cudaMalloc(&buf, sizeof(double) * (3 * n + 8)) != cudaSuccess) return core_fail(BX_ERR_NOMEM, "autotune scratch");
  if (cudaMalloc(&partial, sizeof(double) * kKryMaxBlocks) != cudaSuccess ||
      cudaMalloc(&cnt, sizeof(unsigned)) != cudaSuccess) {
    cudaFree(buf);
    if (partial) cudaFree(partial);
    return core_fail(BX_ERR_NOMEM, "autotune scratch");
  }
  cudaMemsetAsync(buf, 0, sizeof(double) * (3 * n + 8), c.st);
  cudaMemsetAsync(cnt, 0, sizeof(unsigned), c.st);
  double *w = buf, *v0 = buf + n, *v1 = buf + 2 * n, *h = buf + 3 * n;
  TuneKnobInfo &kc = g_knobs[kTuneKryCtas], &ku = g_knobs[kTuneKryUnroll];
  const int c0 = kc.value, u0 = ku.value;  // kept when a timing fails
  float best = 1e30f;
  int bc = c0, bu = u0, r = BX_OK;
  const bool fixC = kc.tuned == 2, fixU = ku.tuned == 2;  // set by the caller: kept
  for (int j = 0; j < ku.nCand; j++) ku.ms[j] = 1e30f;
  for (int i = 0; i < kc.nCand && !r; i++) {
    kc.ms[i] = 1e30f;
    if (fixC && kc.cand[i] != c0) continue;
    for (int j = 0; j < ku.nCand && !r; j++) {
      if (fixU && ku.cand[j] != u0) continue;
      kc.value = kc.cand[i];
      ku.value = ku.cand[j];
      float ms = 0;
      r = time_ms(c.st, 5, [&] { kry_mgs(w, v0, h, v1, n, partial, cnt, h + 1, c.st); }, ms);
      // each knob records its best time over the other knob's candidates
      if (ms < kc.ms[i]) kc.ms[i] = ms;
      if (ms < ku.ms[j]) ku.ms[j] = ms;
      if (ms < best) { best = ms; bc = kc.cand[i]; bu = ku.cand[j]; }
    }
  }
  cudaFree(buf);
  cudaFree(partial);
  cudaFree(cnt);
  kc.value = bc;
  ku.value = bu;
  if (!r) {
    if (!fixC) kc.tuned = 1;
    if (!fixU) ku.tuned = 1;
  }
  return r;
}

}  // namespace bx

using namespace bx;

extern "C" {

int bx_autotune(void) {
  Core c = core();
  if (!c.ready) return core_fail(BX_ERR_STATE, "bx_init has not been called");
  int r = tune_stage();
  if (!r) r = tune_krylov();
  if (!r) r = tune_heat();
  if (!r) r = tune_bilu();
  return r;
}

int bx_tune_info(int iKnob, char *name, int nameLen, int *value, int *tuned, int *nCand, int *cand, float *ms) {
  if (iKnob < 0 || iKnob >= kNumTune) return core_fail(BX_ERR_ARG, "knob %d outside 0..%d", iKnob, kNumTune - 1);
  const TuneKnobInfo &k = g_knobs[iKnob];
  if (name && nameLen > 0) {
    std::strncpy(name, k.name, nameLen - 1);
    name[nameLen - 1] = 0;
  }
  if (value) *value = k.value;
  if (tuned) *tuned = k.tuned;
  if (nCand) *nCand = k.nCand;
  for (int i = 0; i < k.nCand; i++) {
    if (cand) cand[i] = k.cand[i];
    if (ms) ms[i] = k.ms[i];
  }
  return BX_OK;
}

int bx_tune_set(const char *name, int value) {
  if (!name) return core_fail(BX_ERR_ARG, "null argument");
  for (int i = 0; i < kNumTune; i++) {
    TuneKnobInfo &k = g_knobs[i];
    if (std::strcmp(k.name, name)) continue;
    for (int j = 0; j < k.nCand; j++)
      if (k.cand[j] == value) {
        k.value = value;
        k.tuned = 2;
        return BX_OK;
      }
    return core_fail(BX_ERR_ARG, "%d is not a candidate of %s", value, name);
  }
  return core_fail(BX_ERR_ARG, "no knob named %s", name);
}

int bx_tune_reset(void) {
  for (int i = 0; i < kNumTune; i++) {
    g_knobs[i].value = g_default[i];
    g_knobs[i].tuned = 0;
    for (float &m : g_knobs[i].ms) m = 0.0f;
  }
  return BX_OK;
}

}  // extern "C"
