// dg_k_wave.cu — instances of the wavefront step (one block per ticket, and the persistent form)
// for one shot and for 2 to 128 shots, plain and Kahan.
#include "dg_kernels.cuh"

namespace dg {

WaveFn kernel_wave(int S, bool kahan, bool persistent) {
#define DG_WV(SS, LAYOUT, KH)                                            \
  if (S == SS && kahan == KH)                                            \
    return persistent ? (WaveFn)k_step_wave_p<LAYOUT, KH> : (WaveFn)k_step_wave<LAYOUT, KH>;
#define DG_WV2(SS) DG_WV(SS, WaveTwoShots<SS>, false) DG_WV(SS, WaveTwoShots<SS>, true)
  DG_WV(1, WaveOneShot, false) DG_WV(1, WaveOneShot, true)
  DG_WV2(2) DG_WV2(4) DG_WV2(8) DG_WV2(16) DG_WV2(32) DG_WV2(64) DG_WV2(128)
#undef DG_WV2
#undef DG_WV
  return nullptr;
}

}  // namespace dg
