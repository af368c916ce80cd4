// Per-mode field counts of the staggered-grid step, shared by the tiled
// step kernels (step.cu) and the row-marching kernels (march.cu).
#pragma once
#include "seispie_b200.h"

namespace fwi {

template <int MODE>
struct Fields;
// NS stress fields (with halo), NV velocity/displacement components,
// NVP per-cell parameters of the velocity half, NIP of the stress half,
// NINJ injected components.
template <>
struct Fields<FWI_SH> {
    static constexpr int NS = 2, NV = 1, NVP = 2, NIP = 1, NINJ = 1;
};
template <>
struct Fields<FWI_PSV> {
    static constexpr int NS = 3, NV = 2, NVP = 2, NIP = 2, NINJ = 2;
};
template <>
struct Fields<FWI_SPIN> {
    static constexpr int NS = 6, NV = 3, NVP = 3, NIP = 4, NINJ = 2;
};

// Stress fields whose D_x^- is taken (SH: sxy; P-SV: sxx, sxz; spin also
// syx_c, syy_c) -- these get an x register window in step_kernel_rw.
__host__ __device__ constexpr bool takes_dxm(int mode, int f) {
    return mode == FWI_SH ? f == 0 : (f == 0 || f == 2 || (mode == FWI_SPIN && (f == 3 || f == 4)));
}

}  // namespace fwi
