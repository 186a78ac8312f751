// bx_tune.h -- launch-shape knobs of the kernels and their autotuned values.
//
// Each knob lists its candidate values; bx_autotune (bx_tune.cu) times every
// candidate of every knob whose context is ready with CUDA events on the
// live data and keeps the fastest.  Launchers read the current value with
// tune_value().  The candidates of a knob never change the arithmetic of a
// kernel except the Krylov reduction grid, which changes the summation order
// of the inner products (each order is deterministic).
#pragma once

namespace bx {

enum TuneKnob {
  kTuneStageGrid = 0,  // persistent stage kernel CTAs per SM (several fit for 4^3 blocks)
  kTuneKryCtas,        // Krylov vector kernels: CTAs per SM (256 threads each)
  kTuneKryUnroll,      // Krylov MGS step: independent 16-byte loads in flight per thread and vector
  kTuneHeatIluWarps,   // heat ILU sweeps: warps (groups of 32 blocks) per CTA
  kTuneBiluThreads,    // JFNK BILU sweeps: threads per block CTA (8 per cell of a wavefront)
  kTuneStageVariant,   // stage kernel, 8^3 blocks: 0 one face phase (FP64: 512 threads, 3: 576); one
                       // direction at a time with 1: one face per thread (576 threads), 2: two (288)
  kTuneKryGsSteps,     // Gram-Schmidt steps per pass over w (1 to 4); set, not timed
  kNumTune
};

struct TuneKnobInfo {
  const char *name;
  int nCand;
  int cand[8];
  int value;      // current value
  int tuned;      // 1 after bx_autotune chose it, 2 when set by the caller
  float ms[8];    // measured time of each candidate (last autotune)
};

TuneKnobInfo &tune_knob(int knob);
inline int tune_value(int knob) { return tune_knob(knob).value; }

// tuning procedures of the parts (each returns BX_OK, or skips silently when
// its context is not ready)
int tune_stage();   // bx_capi.cu
int tune_krylov();  // bx_tune.cu
int tune_heat();    // bx_heat.cu
int tune_bilu();    // bx_implicit.cu

}  // namespace bx
