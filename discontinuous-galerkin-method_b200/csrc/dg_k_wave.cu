// dg_k_wave.cu — instances of the wavefront step (one block per ticket, and the persistent form)
// for one shot and for 2 to 128 shots, plain and Kahan.
#include "dg_kernels.cuh"

namespace dg {

WaveFn kernel_wave_async(int S, bool kahan) {
#define DG_WVA(SS, KH) \
  if (S == SS && kahan == KH) return (WaveFn)k_step_wave_p<WaveTwoShotsAsync<SS>, KH>;
  DG_WVA(16, false) DG_WVA(16, true) DG_WVA(32, false) DG_WVA(32, true) DG_WVA(64, false) DG_WVA(64, true)
  DG_WVA(128, false) DG_WVA(128, true)
#undef DG_WVA
  return nullptr;
}

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
