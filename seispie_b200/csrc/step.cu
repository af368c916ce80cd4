// Fused staggered-grid time step for SH, P-SV and micropolar-spin waves.
//
// One launch advances every shot of a batch by one time step.  It replaces
// the per-step kernel sequence of the reference's run_forward / run_adjoint
// (seispie/solver/fd2d/solver.py:205-234, 309-314):
//   div_sy / div_sxz / div_sxyz_c  -> stress divergence          (velocity half)
//   stf_dsy / stf_dsxz             -> source scatter into it
//   add_vy / add_vxz               -> velocity and displacement update
//   div_vy / div_vxz               -> velocity gradient            (stress half)
//   add_sy / add_sxz / add_sy_c    -> stress update
//   save_obs                       -> receiver gather of displacement
// where the reference keeps every intermediate (dsx, dvxdx, ...) in HBM and
// launches 6 (SH), 8 (P-SV) or 15 (spin) kernels per step.
//
// Design.  A CTA owns a TX x TZ interior tile of one shot.  It stages in
// shared memory (cp.async, 16-byte chunks, zero-filled outside the grid):
//   stress  rows x0-3 .. x0+TX+2, columns z0-4 .. z0+TZ+3
//   velocity, dt/rho, sponge   rows x0-1 .. x0+TX+1, same columns
//   displacement and stiffness of the interior
// computes the new velocity on the interior plus the one-left / two-right
// halo the 4th-order D+ stencil needs (redundant with the neighbour tiles),
// then the new stress of the interior from that shared-memory velocity.
// HBM sees each state field read once and written once per step; the halo
// re-reads hit L2.  Velocity and stress are ping-ponged between two buffers
// because a neighbouring tile may still be reading the old halo.
//
// Two compute mappings share the staging:
//   step_kernel      any TX x TZ; each thread walks cells of the tile.
//   step_kernel_rw   TZ = 32: lane = z, each warp owns TX/8 consecutive x
//                    rows and keeps the x-derivative taps in a register
//                    window sliding down x, so a row of a field is read from
//                    shared memory once instead of four times.
// Both do the same arithmetic per cell, so their results are bit-identical.
//
// Derivative masks follow solver.py:22-51 exactly: D- is zero unless
// 2 <= i < n-2, D+ is zero unless 1 <= i < n-2 (same for j), so no value
// outside the grid or in row padding ever reaches a result.
#include <cstdio>

#include "common.cuh"

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

struct StepArgs {
    int nx, nz, pitch, nt, it, nrec;
    FastDiv divnz;
    float cx1, cx2, cz1, cz2;  // 9/(8dx), 1/(24dx), 9/(8dz), 1/(24dz)
    float dt, dt2;             // dt and 2*dt rounded to float
    const float *sig_in[6];
    float *sig_out[6];
    const float *vel_in[3];
    float *vel_out[3];
    float *disp[3];
    const float *vp[3];  // buo, bound, buo_j
    const float *ip[4];  // SH: mu | P-SV: lam, mu | spin: lam, mu, nu, mnc
    const int *inj_ptr, *inj_cell, *inj_row;
    const float *stf[2];  // injected components in slot order
    const int *rec_cell;
    float *obs[3];
    float *snap_u[3];  // already offset to the slot, or NULL
    float *snap_v[3];
    float *seg_v[3];   // per-step store of the new velocity (exact adjoint), slot-offset, or NULL
    float *seg_ds[3];  // per-step store of the stress divergence incl. sources, or NULL
};

template <int MODE, int TX, int TZ>
struct Tile {
    using F = Fields<MODE>;
    // stress region: rows x0-3 .. x0+TX+2 (D- of the velocity halo row
    // x0+TX+1 reaches x0+TX+2), columns z0-4 .. z0+TZ+3
    static constexpr int SX = TX + 6, SZ = TZ + 8;
    static constexpr int VX = TX + 3, RVZ = TZ + 3;  // velocity rows / computed columns
    // per-field strides padded to 128 bytes (TMA destinations must be aligned)
    static constexpr int FS = (SX * SZ + 31) / 32 * 32, FV = (VX * SZ + 31) / 32 * 32;
    static constexpr int S_SZ = F::NS * FS;
    static constexpr int V_SZ = F::NV * FV;
    static constexpr int P_SZ = F::NVP * FV;
    static constexpr int U_SZ = F::NV * TX * TZ;
    static constexpr int I_SZ = F::NIP * TX * TZ;
    static constexpr int J_SZ = F::NINJ * VX * RVZ;
    static constexpr int LIST = kThreads * (1 + F::NINJ) + 8;  // compacted injection entries + warp counts
    // mbarrier of the TMA variant after the list, 8-byte aligned
    static constexpr int BAR_OFF = (S_SZ + V_SZ + P_SZ + U_SZ + I_SZ + J_SZ + LIST + 1) / 2 * 2;
    static constexpr size_t bytes = sizeof(float) * (size_t)(BAR_OFF + 2);
    static_assert(TZ % 4 == 0, "TZ must be a multiple of 4");
};

// Shared-memory regions of one CTA.
template <int MODE, int TX, int TZ>
struct Smem {
    using T = Tile<MODE, TX, TZ>;
    float *S, *V, *P, *U, *I, *J, *val;
    int *loc, *warp;
    __device__ explicit Smem(float *base) {
        S = base;
        V = S + T::S_SZ;
        P = V + T::V_SZ;
        U = P + T::P_SZ;
        I = U + T::U_SZ;
        J = I + T::I_SZ;
        loc = reinterpret_cast<int *>(J + T::J_SZ);
        val = reinterpret_cast<float *>(loc + kThreads);
        warp = reinterpret_cast<int *>(val + Fields<MODE>::NINJ * kThreads);
    }
};

// Stage NF fields (shared-memory field stride FSTR floats) of a ROWS x COLS
// window starting at (gx0, gz0) with 16-byte cp.async copies; the chunk
// geometry is computed once for all fields.  Chunks outside the grid are
// zero-filled.
template <int NF, int ROWS, int COLS, int FSTR>
__device__ __forceinline__ void stage_strided(float *dst, const float *const *src, long long off, int gx0, int gz0,
                                              int nx, int pitch, int tid) {
    constexpr int C4 = COLS / 4, PER = ROWS * C4;
    for (int q = tid; q < PER; q += kThreads) {
        const int r = q / C4, c = q - r * C4;
        const int gx = gx0 + r, gz = gz0 + 4 * c;
        const bool ok = gx >= 0 && gx < nx && gz >= 0 && gz < pitch;
        const long long o = ok ? off + (long long)gx * pitch + gz : 0;
#pragma unroll
        for (int f = 0; f < NF; f++) cp_async16(dst + f * FSTR + r * COLS + 4 * c, src[f] + o, ok ? 16 : 0);
    }
}

// Entries of this shot at cells of the computed region, summed per cell in
// entry order into J (NINJ components, VX x RVZ cells): the source scatter
// stf_dsy / stf_dsxz (solver.py:78-93).  Returns whether any entry falls in
// the tile (J is written only then).  Block-wide: every thread must call it.
template <int NINJ, int VX, int RVZ>
__device__ __forceinline__ bool scatter_entries(const int *inj_ptr, const int *inj_cell, const int *inj_row,
                                                const float *const *val_src, int nt, int it, const FastDiv &divnz,
                                                int nz, int x0, int z0, int shot, float *J, int *sLoc, float *sVal,
                                                int *sWarp) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    bool has = false;
    if (!inj_ptr) return false;
    const int p0 = inj_ptr[shot], p1 = inj_ptr[shot + 1];
    for (int base = p0; base < p1; base += kThreads) {
        const int e = base + tid;
        int loc = -1;
        float val[NINJ];
        if (e < p1) {
            const int k = inj_cell[e];
            const int gx = fdiv(k, divnz), gz = k - gx * nz;
            const int rx = gx - (x0 - 1), rz = gz - (z0 - 1);
            if (rx >= 0 && rx < VX && rz >= 0 && rz < RVZ) {
                loc = rx * RVZ + rz;
                const long long src = (long long)inj_row[e] * nt + it;
#pragma unroll
                for (int c = 0; c < NINJ; c++) val[c] = val_src[c][src];
            }
        }
        const int n_in = __syncthreads_count(loc >= 0);
        if (n_in == 0) continue;
        if (!has) {
            for (int q = tid; q < NINJ * VX * RVZ; q += kThreads) J[q] = 0.f;
            has = true;
        }
        const unsigned ball = __ballot_sync(0xffffffffu, loc >= 0);
        if (lane == 0) sWarp[warp] = __popc(ball);
        __syncthreads();
        if (loc >= 0) {
            int pos = __popc(ball & ((1u << lane) - 1u));
            for (int w = 0; w < warp; w++) pos += sWarp[w];
            sLoc[pos] = loc;
#pragma unroll
            for (int c = 0; c < NINJ; c++) sVal[c * kThreads + pos] = val[c];
        }
        __syncthreads();
        if (tid == 0) {
            for (int q = 0; q < n_in; q++) {
#pragma unroll
                for (int c = 0; c < NINJ; c++) J[c * VX * RVZ + sLoc[q]] += sVal[c * kThreads + q];
            }
        }
        __syncthreads();
    }
    return has;
}

// ---------------------------------------------------------- TMA staging
// Tensor maps of one step: stress / velocity of the current half and the
// displacement as 3-D maps (z = pitch, x, shot), the model as 2-D maps.
struct TmaMaps {
    CUtensorMap sig[6];
    CUtensorMap vel[3];
    CUtensorMap disp[3];
    CUtensorMap vp[3];  // model fields read on the velocity region
    CUtensorMap ip[4];  // model fields read on the interior
};

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, int count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after ~2^22 polls (each poll may suspend the warp
// for a while), so a lost transaction ends the kernel instead of hanging it.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    for (int i = 0; i < (1 << 22); i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::
            "r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int c0, int c1, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];\n" ::"r"(
            smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(smem_u32(bar))
        : "memory");
}

// Device-side status of the TMA kernels (a wait that gave up), read and
// cleared by fwi_device_status.
__device__ int g_device_status = 0;

// Staging copies plus the source scatter (stf_dsy / stf_dsxz, solver.py:78-93):
// entries of this shot inside the computed velocity region are summed per
// cell into sm.J, in entry order, while the copies are in flight.  Returns
// whether the tile holds any entry (then sm.J is valid).  Ends with the
// staged data visible to the whole CTA.
template <int MODE, int TX, int TZ>
__device__ __forceinline__ bool prologue(const StepArgs &a, const Smem<MODE, TX, TZ> &sm, int x0, int z0, int shot) {
    using T = Tile<MODE, TX, TZ>;
    using F = Fields<MODE>;
    constexpr int SX = T::SX, SZ = T::SZ, VX = T::VX, RVZ = T::RVZ;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nx = a.nx, nz = a.nz, pitch = a.pitch;
    const long long soff = (long long)shot * nx * pitch;
    stage_strided<F::NS, SX, SZ, T::FS>(sm.S, a.sig_in, soff, x0 - 3, z0 - 4, nx, pitch, tid);
    stage_strided<F::NV, VX, SZ, T::FV>(sm.V, a.vel_in, soff, x0 - 1, z0 - 4, nx, pitch, tid);
    stage_strided<F::NVP, VX, SZ, T::FV>(sm.P, a.vp, 0, x0 - 1, z0 - 4, nx, pitch, tid);
    stage_strided<F::NV, TX, TZ, TX * TZ>(sm.U, a.disp, soff, x0, z0, nx, pitch, tid);
    stage_strided<F::NIP, TX, TZ, TX * TZ>(sm.I, a.ip, 0, x0, z0, nx, pitch, tid);
    cp_async_commit();
    const bool has_inj = scatter_entries<F::NINJ, VX, RVZ>(a.inj_ptr, a.inj_cell, a.inj_row, a.stf, a.nt, a.it,
                                                           a.divnz, nz, x0, z0, shot, sm.J, sm.loc, sm.val, sm.warp);
    (void)lane;
    (void)warp;
    cp_async_wait_all();
    __syncthreads();
    return has_inj;
}

// The same staging with TMA: one thread issues one tensor copy per field
// (zero fill outside the grid comes from the tensor maps), completion is
// counted on an mbarrier, and the source scatter overlaps the copies.  Returns
// -1 if the wait gave up (the kernel must then return), else has_inj.
template <int MODE, int TX, int TZ>
__device__ __forceinline__ int prologue_tma(const StepArgs &a, const TmaMaps &m, const Smem<MODE, TX, TZ> &sm,
                                            uint64_t *bar, int x0, int z0, int shot) {
    using T = Tile<MODE, TX, TZ>;
    using F = Fields<MODE>;
    constexpr int SX = T::SX, SZ = T::SZ, VX = T::VX, RVZ = T::RVZ;
    constexpr uint32_t bytes = 4u * (F::NS * SX * SZ + (F::NV + F::NVP) * VX * SZ + (F::NV + F::NIP) * TX * TZ);
    static_assert(bytes < (1u << 20), "mbarrier transaction count limit");
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        mbar_expect_tx(bar, bytes);
#pragma unroll
        for (int f = 0; f < F::NS; f++) tma_load_3d(sm.S + f * T::FS, &m.sig[f], z0 - 4, x0 - 3, shot, bar);
#pragma unroll
        for (int q = 0; q < F::NV; q++) tma_load_3d(sm.V + q * T::FV, &m.vel[q], z0 - 4, x0 - 1, shot, bar);
#pragma unroll
        for (int p = 0; p < F::NVP; p++) tma_load_2d(sm.P + p * T::FV, &m.vp[p], z0 - 4, x0 - 1, bar);
#pragma unroll
        for (int q = 0; q < F::NV; q++) tma_load_3d(sm.U + q * TX * TZ, &m.disp[q], z0, x0, shot, bar);
#pragma unroll
        for (int p = 0; p < F::NIP; p++) tma_load_2d(sm.I + p * TX * TZ, &m.ip[p], z0, x0, bar);
    }
    const bool has_inj = scatter_entries<F::NINJ, VX, RVZ>(a.inj_ptr, a.inj_cell, a.inj_row, a.stf, a.nt, a.it,
                                                           a.divnz, a.nz, x0, z0, shot, sm.J, sm.loc, sm.val, sm.warp);
    const bool ok = mbar_wait(bar, 0);
    if (__syncthreads_or(!ok)) {  // block-uniform decision
        if (threadIdx.x == 0) atomicExch(&g_device_status, 1);
        if (!ok) mbar_wait(bar, 0);  // one more bounded chance for the copies in flight to land
        return -1;
    }
    return has_inj ? 1 : 0;
}

// Velocity update of one cell from its stress divergence ds (all in shared
// memory): v = bound * (v + ds * dt/rho)  (add_vy / add_vxz, solver.py:95-109).
// (rx, rz): velocity-region row and computed column; writes sm.V in place.
template <int MODE, int TX, int TZ>
__device__ __forceinline__ void velocity_update(const Smem<MODE, TX, TZ> &sm, int rx, int rz, float (&ds)[3],
                                                bool has_inj, float (&vnew)[3]) {
    using T = Tile<MODE, TX, TZ>;
    using F = Fields<MODE>;
    constexpr int SZ = T::SZ, VX = T::VX, RVZ = T::RVZ;
    if (has_inj) {
#pragma unroll
        for (int c = 0; c < F::NINJ; c++) ds[c] += sm.J[c * VX * RVZ + rx * RVZ + rz];
    }
    const int vi = rx * SZ + rz + 3;
    const float buo = sm.P[vi], bnd = sm.P[T::FV + vi];
#pragma unroll
    for (int c = 0; c < F::NV; c++) {
        const float b = (MODE == FWI_SPIN && c == 2) ? sm.P[2 * T::FV + vi] : buo;
        const float v = bnd * (sm.V[c * T::FV + vi] + ds[c] * b);
        sm.V[c * T::FV + vi] = v;
        vnew[c] = v;
    }
}

// Stress divergence of one cell (div_sy / div_sxz / div_sxyz_c,
// solver.py:54-75) from D_x^- and D_z^- values supplied by the caller.
template <int MODE, class DXM, class DZM, class CEN>
__device__ __forceinline__ void divergence(DXM dxm, DZM dzm, CEN center, float (&ds)[3]) {
    if (MODE == FWI_SH) {
        ds[0] = dxm(0) + dzm(1);
    } else {
        ds[0] = dxm(0) + dzm(2);
        ds[1] = dxm(2) + dzm(1);
        if (MODE == FWI_SPIN) {
            ds[0] += dzm(4);
            ds[1] -= dxm(4);
            ds[2] = (dxm(3) + dzm(5)) + 2.f * center(4);
        }
    }
}

// Stress update of one interior cell (add_sy / add_sxz / add_sy_c,
// solver.py:128-149) from D+ of the new velocity; s0 points at the cell's
// old stress in shared memory, ip at its stiffness, g is its HBM offset.
template <int MODE, int TX, int TZ, class DXP, class DZP>
__device__ __forceinline__ void stress_update(const StepArgs &a, const float *s0, const float *ip, float vyc, long long g,
                                              DXP dxp, DZP dzp) {
    using T = Tile<MODE, TX, TZ>;
    constexpr int FS = T::FS, FI = TX * TZ;
    const float dt = a.dt;
    if (MODE == FWI_SH) {
        const float dm = dt * ip[0];
        a.sig_out[0][g] = s0[0] + dm * dxp(0);
        a.sig_out[1][g] = s0[FS] + dm * dzp(0);
    } else {
        const float lam = ip[0], mu = ip[FI];
        const float vxx = dxp(0), vxz = dzp(0), vzx = dxp(1), vzz = dzp(1);
        const float l2m = lam + 2.f * mu;
        a.sig_out[0][g] = s0[0] + dt * (l2m * vxx + lam * vzz);
        a.sig_out[1][g] = s0[FS] + dt * (l2m * vzz + lam * vxx);
        a.sig_out[2][g] = s0[2 * FS] + dt * (mu * (vxz + vzx));
        if (MODE == FWI_SPIN) {
            const float nu = ip[2 * FI], mnc = ip[3 * FI];
            a.sig_out[4][g] = s0[4 * FS] + a.dt2 * nu * (-vyc - 0.5f * (vzx - vxz));
            a.sig_out[3][g] = s0[3 * FS] + dt * mnc * dxp(2);
            a.sig_out[5][g] = s0[5 * FS] + dt * mnc * dzp(2);
        }
    }
}

// Interior bookkeeping after a velocity update: HBM writes of v and u,
// snapshots, u into shared memory for the receivers.
template <int MODE, int TX, int TZ>
__device__ __forceinline__ void store_interior(const StepArgs &a, const Smem<MODE, TX, TZ> &sm, int ci, long long g,
                                               const float (&v)[3], const float (&ds)[3]) {
#pragma unroll
    for (int q = 0; q < Fields<MODE>::NV; q++) {
        const float u = sm.U[q * TX * TZ + ci] + v[q] * a.dt;
        sm.U[q * TX * TZ + ci] = u;
        a.vel_out[q][g] = v[q];
        a.disp[q][g] = u;
        if (a.snap_u[q]) a.snap_u[q][g] = u;
        if (a.snap_v[q]) a.snap_v[q][g] = v[q];
        if (a.seg_v[q]) a.seg_v[q][g] = v[q];
        if (a.seg_ds[q]) a.seg_ds[q][g] = ds[q];
    }
}

// Receivers of this tile record the new displacement (save_obs).
template <int MODE, int TX, int TZ>
__device__ __forceinline__ void gather_receivers(const StepArgs &a, const Smem<MODE, TX, TZ> &sm, int x0, int z0,
                                                 int shot) {
    if (!a.rec_cell) return;
    for (int r = threadIdx.x; r < a.nrec; r += kThreads) {
        const int k = a.rec_cell[r];
        const int gx = fdiv(k, a.divnz), gz = k - gx * a.nz;
        const int ix = gx - x0, iz = gz - z0;
        if (ix >= 0 && ix < TX && iz >= 0 && iz < TZ) {
            const long long o = ((long long)shot * a.nrec + r) * a.nt + a.it;
#pragma unroll
            for (int q = 0; q < Fields<MODE>::NV; q++)
                if (a.obs[q]) a.obs[q][o] = sm.U[q * TX * TZ + ix * TZ + iz];
        }
    }
}

// Velocity of one cell of the computed region, generic path (all loads from
// shared memory).  Returns false for a cell outside the grid (v set to 0).
template <int MODE, int TX, int TZ>
__device__ __forceinline__ bool velocity_cell(const StepArgs &a, const Smem<MODE, TX, TZ> &sm, int x0, int z0, int rx,
                                              int rz, bool has_inj, float (&v)[3], float (&ds)[3]) {
    using T = Tile<MODE, TX, TZ>;
    constexpr int SX = T::SX, SZ = T::SZ, VX = T::VX;
    const int gx = x0 - 1 + rx, gz = z0 - 1 + rz;
    const int cz = rz + 3;
    if (gx < 0 || gx >= a.nx || gz < 0 || gz >= a.nz) {
#pragma unroll
        for (int c = 0; c < Fields<MODE>::NV; c++) sm.V[c * T::FV + rx * SZ + cz] = 0.f;
        return false;
    }
    const bool okx = gx >= 2 && gx < a.nx - 2, okz = gz >= 2 && gz < a.nz - 2;
    const float *s0 = sm.S + (rx + 2) * SZ + cz;
    const float cx1 = a.cx1, cx2 = a.cx2, cz1 = a.cz1, cz2 = a.cz2;
    auto dxm = [&](int f) -> float {
        if (!okx) return 0.f;
        const float *s = s0 + f * T::FS;
        return cx1 * (s[0] - s[-SZ]) - cx2 * (s[SZ] - s[-2 * SZ]);
    };
    auto dzm = [&](int f) -> float {
        if (!okz) return 0.f;
        const float *s = s0 + f * T::FS;
        return cz1 * (s[0] - s[-1]) - cz2 * (s[1] - s[-2]);
    };
    auto center = [&](int f) -> float { return s0[f * T::FS]; };
    divergence<MODE>(dxm, dzm, center, ds);
    velocity_update<MODE, TX, TZ>(sm, rx, rz, ds, has_inj, v);
    return true;
}

// Halo cells of the velocity region: rows x0-1, x0+TX, x0+TX+1 (all columns)
// and columns z0-1, z0+TZ, z0+TZ+1 of the interior rows.
template <int MODE, int TX, int TZ>
__device__ __forceinline__ void velocity_halo(const StepArgs &a, const Smem<MODE, TX, TZ> &sm, int x0, int z0,
                                              bool has_inj) {
    constexpr int RVZ = Tile<MODE, TX, TZ>::RVZ;
    constexpr int HROW = 3 * RVZ, HC = HROW + 3 * TX;
    for (int c = threadIdx.x; c < HC; c += kThreads) {
        int rx, rz;
        if (c < HROW) {
            const int r3 = c / RVZ;
            rx = r3 == 0 ? 0 : TX + r3;
            rz = c - r3 * RVZ;
        } else {
            const int c2 = c - HROW, k3 = c2 % 3;
            rx = 1 + c2 / 3;
            rz = k3 == 0 ? 0 : TZ + k3;
        }
        float v[3], ds[3];
        velocity_cell<MODE, TX, TZ>(a, sm, x0, z0, rx, rz, has_inj, v, ds);
    }
}

// ------------------------------------------------------- generic mapping

template <int MODE, int TX, int TZ>
__global__ void __launch_bounds__(kThreads, MODE == FWI_SPIN ? 1 : 2) step_kernel(const StepArgs a) {
    using T = Tile<MODE, TX, TZ>;
    constexpr int SX = T::SX, SZ = T::SZ, VX = T::VX;
    extern __shared__ __align__(128) float smem[];
    const Smem<MODE, TX, TZ> sm(smem);
    const int z0 = blockIdx.x * TZ, x0 = blockIdx.y * TX, shot = blockIdx.z;
    const int nx = a.nx, nz = a.nz, pitch = a.pitch;
    const long long soff = (long long)shot * nx * pitch;
    const bool has_inj = prologue<MODE, TX, TZ>(a, sm, x0, z0, shot);

    for (int c = threadIdx.x; c < TX * TZ; c += kThreads) {
        const int ix = c / TZ, iz = c - ix * TZ;
        float v[3], ds[3];
        if (velocity_cell<MODE, TX, TZ>(a, sm, x0, z0, ix + 1, iz + 1, has_inj, v, ds))
            store_interior<MODE, TX, TZ>(a, sm, c, soff + (long long)(x0 + ix) * pitch + (z0 + iz), v, ds);
    }
    velocity_halo<MODE, TX, TZ>(a, sm, x0, z0, has_inj);
    __syncthreads();
    gather_receivers<MODE, TX, TZ>(a, sm, x0, z0, shot);

    const float cx1 = a.cx1, cx2 = a.cx2, cz1 = a.cz1, cz2 = a.cz2;
    for (int c = threadIdx.x; c < TX * TZ; c += kThreads) {
        const int ix = c / TZ, iz = c - ix * TZ;
        const int gx = x0 + ix, gz = z0 + iz;
        if (gx >= nx || gz >= nz) continue;
        const bool okx = gx >= 1 && gx < nx - 2, okz = gz >= 1 && gz < nz - 2;
        const float *v0 = sm.V + (ix + 1) * SZ + (iz + 4);
        auto dxp = [&](int f) -> float {
            if (!okx) return 0.f;
            const float *v = v0 + f * T::FV;
            return cx1 * (v[SZ] - v[0]) - cx2 * (v[2 * SZ] - v[-SZ]);
        };
        auto dzp = [&](int f) -> float {
            if (!okz) return 0.f;
            const float *v = v0 + f * T::FV;
            return cz1 * (v[1] - v[0]) - cz2 * (v[2] - v[-1]);
        };
        const float vyc = MODE == FWI_SPIN ? v0[2 * T::FV] : 0.f;
        stress_update<MODE, TX, TZ>(a, sm.S + (ix + 3) * SZ + (iz + 4), sm.I + c, vyc,
                                    soff + (long long)gx * pitch + gz, dxp, dzp);
    }
    (void)SX;
}

// -------------------------------------------------- register-window mapping

template <int MODE, int TX, bool TMA>
__device__ __forceinline__ void rw_body(const StepArgs &a, const TmaMaps &maps, float *smem, int x0, int z0,
                                        int shot);

template <int MODE, int TX, bool TMA>
__global__ void __launch_bounds__(kThreads, MODE == FWI_SPIN ? 1 : 3)
    step_kernel_rw(const __grid_constant__ StepArgs a, const __grid_constant__ TmaMaps maps) {
    extern __shared__ __align__(128) float smem[];
    rw_body<MODE, TX, TMA>(a, maps, smem, blockIdx.y * TX, blockIdx.x * 32, blockIdx.z);
}

// Body of the register-window step for the tile (x0, z0) of `shot`.
template <int MODE, int TX, bool TMA>
__device__ __forceinline__ void rw_body(const StepArgs &a, const TmaMaps &maps, float *smem, int x0, int z0,
                                        int shot) {
    constexpr int TZ = 32, RPW = TX / (kThreads / 32);
    static_assert(RPW >= 1 && RPW * (kThreads / 32) == TX, "TX must be a multiple of the warp count");
    using T = Tile<MODE, TX, TZ>;
    using F = Fields<MODE>;
    constexpr int SX = T::SX, SZ = T::SZ, VX = T::VX;
    const Smem<MODE, TX, TZ> sm(smem);
    const int nx = a.nx, nz = a.nz, pitch = a.pitch;
    const long long soff = (long long)shot * nx * pitch;
    bool has_inj;
    if constexpr (TMA) {
        const int r = prologue_tma<MODE, TX, TZ>(a, maps, sm, reinterpret_cast<uint64_t *>(smem + T::BAR_OFF), x0,
                                                 z0, shot);
        if (r < 0) return;
        has_inj = r > 0;
    } else {
        has_inj = prologue<MODE, TX, TZ>(a, sm, x0, z0, shot);
    }

    const int lane = threadIdx.x & 31, ix0 = (threadIdx.x >> 5) * RPW;
    const int gz = z0 + lane, col = lane + 4;
    const bool zin = gz < nz;
    const float cx1 = a.cx1, cx2 = a.cx2, cz1 = a.cz1, cz2 = a.cz2;

    // ---- velocity on the warp's interior rows: S rows ix0+1 .. ix0+RPW+3 of
    // the D_x^- fields sit in registers (window index q <-> S row ix0+1+q)
    {
        const bool okz = gz >= 2 && gz < nz - 2;
        float w[F::NS][RPW + 3];
#pragma unroll
        for (int f = 0; f < F::NS; f++)
            if (takes_dxm(MODE, f)) {
#pragma unroll
                for (int r = 0; r < RPW + 3; r++) w[f][r] = sm.S[f * T::FS + (ix0 + 1 + r) * SZ + col];
            }
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            const int ix = ix0 + q, gx = x0 + ix;
            const int vi = (ix + 1) * SZ + col;
            if (!(zin && gx < nx)) {
#pragma unroll
                for (int c = 0; c < F::NV; c++) sm.V[c * T::FV + vi] = 0.f;
                continue;
            }
            const bool okx = gx >= 2 && gx < nx - 2;
            const float *srow = sm.S + (ix + 3) * SZ + col;
            auto dxm = [&](int f) -> float {
                return okx ? cx1 * (w[f][q + 2] - w[f][q + 1]) - cx2 * (w[f][q + 3] - w[f][q]) : 0.f;
            };
            auto center = [&](int f) -> float { return takes_dxm(MODE, f) ? w[f][q + 2] : srow[f * T::FS]; };
            auto dzm = [&](int f) -> float {
                if (!okz) return 0.f;
                const float *s = srow + f * T::FS;
                return cz1 * (center(f) - s[-1]) - cz2 * (s[1] - s[-2]);
            };
            float ds[3], v[3];
            divergence<MODE>(dxm, dzm, center, ds);
            velocity_update<MODE, TX, TZ>(sm, ix + 1, lane + 1, ds, has_inj, v);
            store_interior<MODE, TX, TZ>(a, sm, ix * TZ + lane, soff + (long long)gx * pitch + gz, v, ds);
        }
    }
    velocity_halo<MODE, TX, TZ>(a, sm, x0, z0, has_inj);
    __syncthreads();
    gather_receivers<MODE, TX, TZ>(a, sm, x0, z0, shot);

    // ---- stress on the same rows: V rows ix0 .. ix0+RPW+2 in registers
    // (window index q <-> V row ix0+q; the cell of row ix is V row ix+1)
    {
        const bool okz = gz >= 1 && gz < nz - 2;
        float w[F::NV][RPW + 3];
#pragma unroll
        for (int f = 0; f < F::NV; f++) {
#pragma unroll
            for (int r = 0; r < RPW + 3; r++) w[f][r] = sm.V[f * T::FV + (ix0 + r) * SZ + col];
        }
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            const int ix = ix0 + q, gx = x0 + ix;
            if (!(zin && gx < nx)) continue;
            const bool okx = gx >= 1 && gx < nx - 2;
            const float *vrow = sm.V + (ix + 1) * SZ + col;
            auto dxp = [&](int f) -> float {
                return okx ? cx1 * (w[f][q + 2] - w[f][q + 1]) - cx2 * (w[f][q + 3] - w[f][q]) : 0.f;
            };
            auto dzp = [&](int f) -> float {
                if (!okz) return 0.f;
                const float *v = vrow + f * T::FV;
                return cz1 * (v[1] - w[f][q + 1]) - cz2 * (v[2] - v[-1]);
            };
            const float vyc = MODE == FWI_SPIN ? w[F::NV - 1][q + 1] : 0.f;
            stress_update<MODE, TX, TZ>(a, sm.S + (ix + 3) * SZ + col, sm.I + ix * TZ + lane, vyc,
                                        soff + (long long)gx * pitch + gz, dxp, dzp);
        }
    }
}

// ------------------------------------------- uneven multi-instance batches
//
// Independent instances (each its own grid, model, shots, sources,
// receivers and nt) stepped together: one launch per step covers every tile
// of every shot of every instance still running.  Instances are ordered by
// nt, longest first, so the running ones are a prefix; block b finds its
// instance by binary search in the prefix sums of the per-instance block
// counts, copies that instance's step arguments into shared memory and runs
// the register-window step body on its tile.

struct MultiInst {
    StepArgs a[2];  // arguments with the ping-pong halves in order (cur = 0 / 1)
    int tiles_z, tiles_x, nshots, nt;
};

template <int MODE, int TX>
__global__ void __launch_bounds__(kThreads, MODE == FWI_SPIN ? 1 : 3)
    step_kernel_multi(const MultiInst *inst, const int *prefix, int nactive, int it, int cur) {
    extern __shared__ __align__(128) float smem[];
    __shared__ StepArgs sa;
    __shared__ int sinfo[4];
    if (threadIdx.x == 0) {
        const int b = blockIdx.x;
        int lo = 0, hi = nactive - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (prefix[mid] <= b) lo = mid;
            else hi = mid - 1;
        }
        const MultiInst &m = inst[lo];
        const int local = b - prefix[lo], per_shot = m.tiles_z * m.tiles_x;
        const int shot = local / per_shot, r = local - shot * per_shot;
        const int xt = r / m.tiles_z, zt = r - xt * m.tiles_z;
        sinfo[0] = lo;
        sinfo[1] = shot;
        sinfo[2] = xt * TX;
        sinfo[3] = zt * 32;
    }
    __syncthreads();
    const int *src = reinterpret_cast<const int *>(&inst[sinfo[0]].a[cur]);
    int *dst = reinterpret_cast<int *>(&sa);
    for (int w = threadIdx.x; w < (int)(sizeof(StepArgs) / 4); w += kThreads) dst[w] = src[w];
    __syncthreads();
    if (threadIdx.x == 0) sa.it = it;
    __syncthreads();
    const TmaMaps &unused = *reinterpret_cast<const TmaMaps *>(inst);  // the cp.async body never reads it
    rw_body<MODE, TX, false>(sa, unused, smem, sinfo[2], sinfo[3], sinfo[1]);
}

// ------------------------------------------------ exact discrete adjoint
//
// The forward step above is linear in the state.  For SH / P-SV it reads
//   d  = D- sig + f            (stress divergence plus sources)
//   v' = B (v + b d)           (b = dt/rho, B = sponge)
//   u' = u + dt v'
//   sig' = sig + dt S(D+ v')   (S: lam/mu stress-strain law)
// Its exact transpose, run backwards in time on the adjoint state
// (sig~, v~, u~), is one launch of adjoint_kernel per step:
//   u~  += P^T g               (g = dL/d(trace) of this step, at receivers)
//   a    = v~ + dt u~ + (D+)^T (dt S^T sig~)
//   v~'  = B a
//   sig~' = sig~ + (D-)^T (b v~')
// with (D+)^T and (D-)^T the transposes of the reference's masked stencils
// (solver.py:22-51) -- boundary masks included, so the adjoint is exact to
// rounding.  grad_kernel then adds this step's terms of
//   dL/dlam = sum dt (sxx~+szz~)(exx+ezz),
//   dL/dmu  = sum dt (2 sxx~ exx + 2 szz~ ezz + sxz~ (exz+ezx))  [SH: dt (sxy~ exy + szy~ ezy)]
//   dL/db   = sum v~' . d
// from the forward v' and d stored per step by a recomputed forward segment.

struct AdjArgs {
    int nx, nz, pitch, nt, it;
    FastDiv divnz;
    float cx1, cx2, cz1, cz2, dt;
    const float *sig_in[3];
    float *sig_out[3];
    const float *vel_in[2];
    float *vel_out[2];
    float *disp[2];
    const float *buo, *bound, *lam, *mu;
    const int *inj_ptr, *inj_cell, *inj_row;
    const float *g[2];  // trace gradients in forward time order, injected into u~
};

template <int MODE, int TX, int TZ>
struct AdjTile {
    using F = Fields<MODE>;
    static constexpr int SX = TX + 6, SZ = TZ + 8, VX = TX + 3, RVZ = TZ + 3;
    static constexpr int NL = MODE == FWI_SH ? 1 : 2;   // stiffness fields staged with halo
    static constexpr int NTT = MODE == FWI_SH ? 2 : 3;  // dt S^T sig~ fields
    static constexpr int FS = (SX * SZ + 3) / 4 * 4, FV = (VX * SZ + 3) / 4 * 4;
    static constexpr int S_SZ = (F::NS + NL + NTT) * FS;
    static constexpr int V_SZ = (2 * F::NV + 2) * FV;
    static constexpr int J_SZ = F::NINJ * VX * RVZ;
    static constexpr int LIST = kThreads * (1 + F::NINJ) + 8;
    static constexpr size_t bytes = sizeof(float) * (size_t)(S_SZ + V_SZ + J_SZ + LIST);
};

template <int MODE, int TX, int TZ>
__global__ void __launch_bounds__(kThreads, 2) adjoint_kernel(const AdjArgs a) {
    using T = AdjTile<MODE, TX, TZ>;
    using F = Fields<MODE>;
    constexpr int SX = T::SX, SZ = T::SZ, VX = T::VX, RVZ = T::RVZ, FS = T::FS, FV = T::FV;
    constexpr int NS = F::NS, NV = F::NV, NL = T::NL;
    extern __shared__ __align__(128) float smem[];
    float *sSig = smem, *sL = sSig + NS * FS, *sT = sL + NL * FS;
    float *sV = sT + T::NTT * FS, *sU = sV + NV * FV, *sB = sU + NV * FV;
    float *sJ = sB + 2 * FV;
    int *sLoc = reinterpret_cast<int *>(sJ + T::J_SZ);
    float *sVal = reinterpret_cast<float *>(sLoc + kThreads);
    int *sWarp = reinterpret_cast<int *>(sVal + F::NINJ * kThreads);

    const int tid = threadIdx.x;
    const int z0 = blockIdx.x * TZ, x0 = blockIdx.y * TX, shot = blockIdx.z;
    const int nx = a.nx, nz = a.nz, pitch = a.pitch;
    const long long soff = (long long)shot * nx * pitch;
    const float *lm[2] = {MODE == FWI_SH ? a.mu : a.lam, a.mu};
    const float *bb[2] = {a.buo, a.bound};
    stage_strided<NS, SX, SZ, FS>(sSig, a.sig_in, soff, x0 - 3, z0 - 4, nx, pitch, tid);
    stage_strided<NL, SX, SZ, FS>(sL, lm, 0, x0 - 3, z0 - 4, nx, pitch, tid);
    stage_strided<NV, VX, SZ, FV>(sV, a.vel_in, soff, x0 - 1, z0 - 4, nx, pitch, tid);
    stage_strided<NV, VX, SZ, FV>(sU, a.disp, soff, x0 - 1, z0 - 4, nx, pitch, tid);
    stage_strided<2, VX, SZ, FV>(sB, bb, 0, x0 - 1, z0 - 4, nx, pitch, tid);
    cp_async_commit();
    const bool has_inj = scatter_entries<F::NINJ, VX, RVZ>(a.inj_ptr, a.inj_cell, a.inj_row, a.g, a.nt, a.it,
                                                           a.divnz, nz, x0, z0, shot, sJ, sLoc, sVal, sWarp);
    cp_async_wait_all();
    __syncthreads();

    const float dt = a.dt, cx1 = a.cx1, cx2 = a.cx2, cz1 = a.cz1, cz2 = a.cz2;
    // t = dt S^T sig~ over the whole stress region (zero outside the grid)
    for (int c = tid; c < SX * SZ; c += kThreads) {
        if (MODE == FWI_SH) {
            const float m = sL[c];
            sT[c] = dt * (m * sSig[c]);
            sT[FS + c] = dt * (m * sSig[FS + c]);
        } else {
            const float l = sL[c], m = sL[FS + c], l2m = l + 2.f * m;
            const float sxx = sSig[c], szz = sSig[FS + c], sxz = sSig[2 * FS + c];
            sT[c] = dt * (l2m * sxx + l * szz);
            sT[FS + c] = dt * (l * sxx + l2m * szz);
            sT[2 * FS + c] = dt * (m * sxz);
        }
    }
    __syncthreads();

    // velocity-like half on the computed region (rows x0-1..x0+TX+1, columns z0-1..z0+TZ+1)
    auto mxp = [&](int k) -> float { return (k >= 1 && k < nx - 2) ? 1.f : 0.f; };
    auto mzp = [&](int k) -> float { return (k >= 1 && k < nz - 2) ? 1.f : 0.f; };
    for (int c = tid; c < VX * RVZ; c += kThreads) {
        const int rx = c / RVZ, rz = c - rx * RVZ;
        const int gx = x0 - 1 + rx, gz = z0 - 1 + rz;
        const int vi = rx * SZ + rz + 3, si = (rx + 2) * SZ + rz + 3;
        if (gx < 0 || gx >= nx || gz < 0 || gz >= nz) {
#pragma unroll
            for (int q = 0; q < NV; q++) sV[q * FV + vi] = 0.f;
            continue;
        }
        // (D+)^T along x and z of field f of t
        auto dxpT = [&](int f) -> float {
            const float *t = sT + f * FS + si;
            return cx1 * (t[-SZ] * mxp(gx - 1) - t[0] * mxp(gx)) - cx2 * (t[-2 * SZ] * mxp(gx - 2) - t[SZ] * mxp(gx + 1));
        };
        auto dzpT = [&](int f) -> float {
            const float *t = sT + f * FS + si;
            return cz1 * (t[-1] * mzp(gz - 1) - t[0] * mzp(gz)) - cz2 * (t[-2] * mzp(gz - 2) - t[1] * mzp(gz + 1));
        };
        float acc[2];
        if (MODE == FWI_SH) {
            acc[0] = dxpT(0) + dzpT(1);
        } else {
            acc[0] = dxpT(0) + dzpT(2);
            acc[1] = dxpT(2) + dzpT(1);
        }
        const bool interior = rx >= 1 && rx <= TX && rz >= 1 && rz <= TZ;
        const long long g = soff + (long long)gx * pitch + gz;
        const float bnd = sB[FV + vi], buo = sB[vi];
#pragma unroll
        for (int q = 0; q < NV; q++) {
            float uu = sU[q * FV + vi];
            if (has_inj) uu += sJ[q * VX * RVZ + rx * RVZ + rz];
            const float vn = bnd * ((sV[q * FV + vi] + dt * uu) + acc[q]);
            sV[q * FV + vi] = buo * vn;  // b v~' for the stress-like half
            if (interior) {
                a.vel_out[q][g] = vn;
                a.disp[q][g] = uu;
            }
        }
    }
    __syncthreads();

    // stress-like half on the interior: sig~' = sig~ + (D-)^T (b v~')
    auto mxm = [&](int k) -> float { return (k >= 2 && k < nx - 2) ? 1.f : 0.f; };
    auto mzm = [&](int k) -> float { return (k >= 2 && k < nz - 2) ? 1.f : 0.f; };
    for (int c = tid; c < TX * TZ; c += kThreads) {
        const int ix = c / TZ, iz = c - ix * TZ;
        const int gx = x0 + ix, gz = z0 + iz;
        if (gx >= nx || gz >= nz) continue;
        const int vi = (ix + 1) * SZ + iz + 4, si = (ix + 3) * SZ + iz + 4;
        auto dxmT = [&](int q) -> float {
            const float *w = sV + q * FV + vi;
            return cx1 * (w[0] * mxm(gx) - w[SZ] * mxm(gx + 1)) - cx2 * (w[-SZ] * mxm(gx - 1) - w[2 * SZ] * mxm(gx + 2));
        };
        auto dzmT = [&](int q) -> float {
            const float *w = sV + q * FV + vi;
            return cz1 * (w[0] * mzm(gz) - w[1] * mzm(gz + 1)) - cz2 * (w[-1] * mzm(gz - 1) - w[2] * mzm(gz + 2));
        };
        const long long g = soff + (long long)gx * pitch + gz;
        if (MODE == FWI_SH) {
            a.sig_out[0][g] = sSig[si] + dxmT(0);
            a.sig_out[1][g] = sSig[FS + si] + dzmT(0);
        } else {
            a.sig_out[0][g] = sSig[si] + dxmT(0);
            a.sig_out[1][g] = sSig[FS + si] + dzmT(1);
            a.sig_out[2][g] = sSig[2 * FS + si] + (dzmT(0) + dxmT(1));
        }
    }
}

// This step's gradient terms, all shots of the batch summed per cell in shot
// order into FP64 accumulators ([nx][pitch]).  sig_adj: sig~ before the
// transposed step (adjoint of sig(it+1)); vel_adj: v~ after it (= B a);
// vf: forward v(it+1); dsf: forward divergence of step it.
struct AdjPtrs {
    const float *sig_adj[3], *vel_adj[2], *vf[2], *dsf[2];
};

template <int MODE>
__global__ void grad_kernel(const AdjPtrs p, double *k_lam, double *k_mu, double *k_buo, int nx, int nz, int pitch,
                            int nshots, float cx1, float cx2, float cz1, float cz2, double dt) {
    const float *const *sig_adj = p.sig_adj;
    const float *const *vel_adj = p.vel_adj;
    const float *const *vf = p.vf;
    const float *const *dsf = p.dsf;
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= nz) return;
    const bool okx = i >= 1 && i < nx - 2, okz = j >= 1 && j < nz - 2;
    const long long o = (long long)i * pitch + j, field = (long long)nx * pitch;
    double al = 0.0, am = 0.0, ab = 0.0;
    for (int s = 0; s < nshots; s++) {
        const long long g = s * field + o;
        auto dxp = [&](const float *v) -> float {
            return okx ? cx1 * (v[g + pitch] - v[g]) - cx2 * (v[g + 2 * pitch] - v[g - pitch]) : 0.f;
        };
        auto dzp = [&](const float *v) -> float {
            return okz ? cz1 * (v[g + 1] - v[g]) - cz2 * (v[g + 2] - v[g - 1]) : 0.f;
        };
        if (MODE == FWI_SH) {
            am += ((double)sig_adj[0][g] * dxp(vf[0]) + (double)sig_adj[1][g] * dzp(vf[0])) * dt;
            ab += (double)vel_adj[0][g] * dsf[0][g];
        } else {
            const double exx = dxp(vf[0]), exz = dzp(vf[0]), ezx = dxp(vf[1]), ezz = dzp(vf[1]);
            const double sxx = sig_adj[0][g], szz = sig_adj[1][g], sxz = sig_adj[2][g];
            al += (sxx + szz) * (exx + ezz) * dt;
            am += (2.0 * (sxx * exx + szz * ezz) + sxz * (exz + ezx)) * dt;
            ab += (double)vel_adj[0][g] * dsf[0][g] + (double)vel_adj[1][g] * dsf[1][g];
        }
    }
    if (k_lam && MODE != FWI_SH) k_lam[o] += al;
    if (k_mu) k_mu[o] += am;
    if (k_buo) k_buo[o] += ab;
}

// One transposed step (forward step `it`, adjoint state it+1 -> it) and its
// gradient terms.
int launch_adjoint_step(const fwi_batch *b, int it, cudaStream_t st) {
    AdjArgs a;
    a.nx = b->nx;
    a.nz = b->nz;
    a.pitch = b->pitch;
    a.nt = b->nt;
    a.it = it;
    a.divnz = make_fastdiv(b->nz);
    a.cx1 = (float)(9.0 / (8.0 * (double)b->dx));
    a.cx2 = (float)(1.0 / (24.0 * (double)b->dx));
    a.cz1 = (float)(9.0 / (8.0 * (double)b->dz));
    a.cz2 = (float)(1.0 / (24.0 * (double)b->dz));
    a.dt = (float)b->dt;
    const int cur = b->cur, nxt = 1 - b->cur;
    const int ns = b->mode == FWI_SH ? 2 : 3, nv = b->mode == FWI_SH ? 1 : 2;
    for (int f = 0; f < 3; f++) {
        a.sig_in[f] = f < ns ? b->sig[cur][f] : nullptr;
        a.sig_out[f] = f < ns ? b->sig[nxt][f] : nullptr;
    }
    for (int q = 0; q < 2; q++) {
        a.vel_in[q] = q < nv ? b->vel[cur][q] : nullptr;
        a.vel_out[q] = q < nv ? b->vel[nxt][q] : nullptr;
        a.disp[q] = q < nv ? b->disp[q] : nullptr;
    }
    a.buo = b->buo;
    a.bound = b->bound;
    a.lam = b->lam;
    a.mu = b->mu;
    a.inj_ptr = b->inj_ptr;
    a.inj_cell = b->inj_cell;
    a.inj_row = b->inj_row;
    if (b->mode == FWI_SH) {
        a.g[0] = b->stf[1];
        a.g[1] = nullptr;
    } else {
        a.g[0] = b->stf[0];
        a.g[1] = b->stf[2];
    }
    constexpr int TX = 32, TZ = 32;
    dim3 grid((b->nz + TZ - 1) / TZ, (b->nx + TX - 1) / TX, b->nshots);
    if (b->mode == FWI_SH) {
        using T = AdjTile<FWI_SH, TX, TZ>;
        static bool set = false;
        if (!set) {
            cudaError_t e = cudaFuncSetAttribute(adjoint_kernel<FWI_SH, TX, TZ>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::bytes);
            if (e != cudaSuccess) return set_error(FWI_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
            set = true;
        }
        adjoint_kernel<FWI_SH, TX, TZ><<<grid, kThreads, T::bytes, st>>>(a);
    } else {
        using T = AdjTile<FWI_PSV, TX, TZ>;
        static bool set = false;
        if (!set) {
            cudaError_t e = cudaFuncSetAttribute(adjoint_kernel<FWI_PSV, TX, TZ>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::bytes);
            if (e != cudaSuccess) return set_error(FWI_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
            set = true;
        }
        adjoint_kernel<FWI_PSV, TX, TZ><<<grid, kThreads, T::bytes, st>>>(a);
    }
    int rc = check_launch("adjoint_kernel");
    if (rc) return rc;
    // gradient terms of this step
    const long long field = (long long)b->nshots * b->nx * b->pitch;
    const int slot = it - b->seg0;
    const float *sa[3] = {a.sig_in[0], a.sig_in[1], a.sig_in[2]};
    const float *va[2] = {a.vel_out[0], a.vel_out[1]};
    const int cx = b->mode == FWI_SH ? 1 : 0, czs = b->mode == FWI_SH ? 1 : 2;
    const float *vf[2] = {b->seg_v[cx] + slot * field, nv > 1 ? b->seg_v[czs] + slot * field : nullptr};
    const float *df[2] = {b->seg_ds[cx] + slot * field, nv > 1 ? b->seg_ds[czs] + slot * field : nullptr};
    dim3 g2((b->nz + 127) / 128, b->nx);
    AdjPtrs ptrs;
    for (int f = 0; f < 3; f++) ptrs.sig_adj[f] = sa[f];
    for (int q = 0; q < 2; q++) {
        ptrs.vel_adj[q] = va[q];
        ptrs.vf[q] = vf[q];
        ptrs.dsf[q] = df[q];
    }
    if (b->mode == FWI_SH)
        grad_kernel<FWI_SH><<<g2, 128, 0, st>>>(ptrs, nullptr, b->k_mu, b->k_rho, b->nx, b->nz, b->pitch, b->nshots,
                                               a.cx1, a.cx2, a.cz1, a.cz2, b->dt);
    else
        grad_kernel<FWI_PSV><<<g2, 128, 0, st>>>(ptrs, b->k_lam, b->k_mu, b->k_rho, b->nx, b->nz, b->pitch,
                                                b->nshots, a.cx1, a.cx2, a.cz1, a.cz2, b->dt);
    return check_launch("grad_kernel");
}

// ------------------------------------------------------------- launching

struct TileShape {
    int tx, tz, rw;
};
// Variants selectable through fwi_batch.tile; 0 is the default.
// rw: 0 generic mapping, 1 register window + cp.async, 2 register window + TMA
static const TileShape kTiles[] = {{32, 32, 2}, {32, 32, 0}, {16, 64, 0}, {16, 32, 0}, {64, 32, 0}, {8, 64, 0},
                                   {32, 32, 1}, {16, 32, 1}, {64, 32, 1}, {32, 32, 2}, {16, 32, 2}, {8, 32, 2}};
constexpr int kNumTiles = sizeof(kTiles) / sizeof(kTiles[0]);

// cuTensorMapEncodeTiled, fetched from the driver at run time.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// Tiled float32 map over a [nshots][nx][pitch] block (rank 3) or an
// [nx][pitch] model array (rank 2), box (bz, bx), zero fill outside.
static int encode_map(CUtensorMap *m, const float *base, int rank, int pitch, int nx, int nshots, int bz, int bx) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return set_error(FWI_ECUDA, "cuTensorMapEncodeTiled unavailable from the driver");
    cuuint64_t dims[3] = {(cuuint64_t)pitch, (cuuint64_t)nx, (cuuint64_t)(nshots < 1 ? 1 : nshots)};
    cuuint64_t strides[2] = {(cuuint64_t)pitch * 4, (cuuint64_t)pitch * (cuuint64_t)nx * 4};
    cuuint32_t box[3] = {(cuuint32_t)bz, (cuuint32_t)bx, 1};
    cuuint32_t es[3] = {1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, (cuuint32_t)rank, const_cast<float *>(base), dims, strides,
                    box, es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(FWI_ECUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return 0;
}

template <int MODE, int TX, int TZ>
static int build_maps(const StepArgs &a, int nshots, TmaMaps &m) {
    using T = Tile<MODE, TX, TZ>;
    using F = Fields<MODE>;
    int rc = 0;
    for (int f = 0; f < F::NS && !rc; f++) rc = encode_map(&m.sig[f], a.sig_in[f], 3, a.pitch, a.nx, nshots, T::SZ, T::SX);
    for (int q = 0; q < F::NV && !rc; q++) rc = encode_map(&m.vel[q], a.vel_in[q], 3, a.pitch, a.nx, nshots, T::SZ, T::VX);
    for (int q = 0; q < F::NV && !rc; q++) rc = encode_map(&m.disp[q], a.disp[q], 3, a.pitch, a.nx, nshots, TZ, TX);
    for (int p = 0; p < F::NVP && !rc; p++) rc = encode_map(&m.vp[p], a.vp[p], 2, a.pitch, a.nx, 1, T::SZ, T::VX);
    for (int p = 0; p < F::NIP && !rc; p++) rc = encode_map(&m.ip[p], a.ip[p], 2, a.pitch, a.nx, 1, TZ, TX);
    return rc;
}

// kind: 0 generic mapping, 1 register window (cp.async), 2 register window (TMA)
template <int MODE, int TX, int TZ, int KIND>
static int launch_tile(const StepArgs &a, int nshots, cudaStream_t st) {
    using T = Tile<MODE, TX, TZ>;
    static bool attr_set = false;
    static TmaMaps none;  // unused by the cp.async variants
    if constexpr (KIND == 0) {
        if (!attr_set) {
            cudaError_t e = cudaFuncSetAttribute(step_kernel<MODE, TX, TZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)T::bytes);
            if (e != cudaSuccess) return set_error(FWI_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
            attr_set = true;
        }
        dim3 grid((a.nz + TZ - 1) / TZ, (a.nx + TX - 1) / TX, nshots);
        step_kernel<MODE, TX, TZ><<<grid, kThreads, T::bytes, st>>>(a);
    } else {
        static_assert(TZ == 32, "the register-window mapping has one lane per z column");
        constexpr bool TMA = KIND == 2;
        if (!attr_set) {
            cudaError_t e = cudaFuncSetAttribute(step_kernel_rw<MODE, TX, TMA>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::bytes);
            if (e != cudaSuccess) return set_error(FWI_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
            attr_set = true;
        }
        const TmaMaps *maps = &none;
        TmaMaps built;
        if constexpr (TMA) {
            int rc = build_maps<MODE, TX, TZ>(a, nshots, built);
            if (rc) return rc;
            maps = &built;
        }
        dim3 grid((a.nz + TZ - 1) / TZ, (a.nx + TX - 1) / TX, nshots);
        step_kernel_rw<MODE, TX, TMA><<<grid, kThreads, T::bytes, st>>>(a, *maps);
    }
    return check_launch("step_kernel");
}

template <int MODE>
static int launch_mode(const StepArgs &a, int nshots, int tile, cudaStream_t st) {
    switch (tile) {
        case 0: return launch_tile<MODE, 32, 32, 2>(a, nshots, st);
        case 1: return launch_tile<MODE, 32, 32, 0>(a, nshots, st);
        case 2: return launch_tile<MODE, 16, 64, 0>(a, nshots, st);
        case 3: return launch_tile<MODE, 16, 32, 0>(a, nshots, st);
        case 4: return launch_tile<MODE, 64, 32, 0>(a, nshots, st);
        case 5: return launch_tile<MODE, 8, 64, 0>(a, nshots, st);
        case 6: return launch_tile<MODE, 32, 32, 1>(a, nshots, st);
        case 7: return launch_tile<MODE, 16, 32, 1>(a, nshots, st);
        case 8: return launch_tile<MODE, 64, 32, 1>(a, nshots, st);
        case 9: return launch_tile<MODE, 32, 32, 2>(a, nshots, st);
        case 10: return launch_tile<MODE, 16, 32, 2>(a, nshots, st);
        case 11: return launch_tile<MODE, 8, 32, 2>(a, nshots, st);
    }
    return set_error(FWI_EINVAL, "unknown tile variant %d", tile);
}

int tile_count() { return kNumTiles; }

bool tile_shape(int tile, int *tx, int *tz) {
    if (tile < 0 || tile >= kNumTiles) return false;
    *tx = kTiles[tile].tx;
    *tz = kTiles[tile].tz;
    return true;
}

int tile_kind(int tile) { return (tile < 0 || tile >= kNumTiles) ? -1 : kTiles[tile].rw; }

// Fill the per-step arguments shared by every step of a run.
static void base_args(const fwi_batch *b, StepArgs &a) {
    a.nx = b->nx;
    a.nz = b->nz;
    a.pitch = b->pitch;
    a.nt = b->nt;
    a.nrec = b->nrec;
    a.divnz = make_fastdiv(b->nz);
    a.cx1 = (float)(9.0 / (8.0 * (double)b->dx));
    a.cx2 = (float)(1.0 / (24.0 * (double)b->dx));
    a.cz1 = (float)(9.0 / (8.0 * (double)b->dz));
    a.cz2 = (float)(1.0 / (24.0 * (double)b->dz));
    a.dt = (float)b->dt;
    a.dt2 = (float)(2.0 * b->dt);
    a.vp[0] = b->buo;
    a.vp[1] = b->bound;
    a.vp[2] = b->buo_j;
    if (b->mode == FWI_SH) {
        a.ip[0] = b->mu;
        a.ip[1] = a.ip[2] = a.ip[3] = nullptr;
    } else {
        a.ip[0] = b->lam;
        a.ip[1] = b->mu;
        a.ip[2] = b->nu;
        a.ip[3] = b->mnc;
    }
    a.inj_ptr = b->inj_ptr;
    a.inj_cell = b->inj_cell;
    a.inj_row = b->inj_row;
    a.rec_cell = b->rec_cell;
}

static int nfields_sig(int mode) { return mode == FWI_SH ? 2 : mode == FWI_PSV ? 3 : 6; }
static int nfields_vel(int mode) { return mode == FWI_SH ? 1 : mode == FWI_PSV ? 2 : 3; }

// Component slot of the k-th velocity field in the user-facing x/y/z arrays
// (obs, stf, snapshots): SH {y}; P-SV {x, z}; spin {x, z, y}.
static int comp_slot(int mode, int q) {
    if (mode == FWI_SH) return 1;
    return q == 0 ? 0 : q == 1 ? 2 : 1;
}

int launch_step(const fwi_batch *b, int adjoint, int it, bool snap_u_next, int snap_u_slot, bool snap_v,
                int snap_v_slot, cudaStream_t st) {
    StepArgs a;
    base_args(b, a);
    a.it = it;
    const int cur = b->cur, nxt = 1 - b->cur;
    const int ns = nfields_sig(b->mode), nv = nfields_vel(b->mode);
    for (int f = 0; f < 6; f++) {
        a.sig_in[f] = f < ns ? b->sig[cur][f] : nullptr;
        a.sig_out[f] = f < ns ? b->sig[nxt][f] : nullptr;
    }
    const long long field = (long long)b->nshots * b->nx * b->pitch;
    for (int q = 0; q < 3; q++) {
        const bool on = q < nv;
        a.vel_in[q] = on ? b->vel[cur][q] : nullptr;
        a.vel_out[q] = on ? b->vel[nxt][q] : nullptr;
        a.disp[q] = on ? b->disp[q] : nullptr;
        const int slot = on ? comp_slot(b->mode, q) : 0;
        a.obs[q] = (on && !adjoint) ? b->obs[slot] : nullptr;
        a.snap_u[q] = (on && !adjoint && snap_u_next && b->snap_u[slot]) ? b->snap_u[slot] + snap_u_slot * field
                                                                          : nullptr;
        a.snap_v[q] = (on && !adjoint && snap_v && b->snap_v[slot]) ? b->snap_v[slot] + snap_v_slot * field
                                                                     : nullptr;
        const bool seg = on && !adjoint && it - b->seg0 >= 0 && it - b->seg0 < b->nseg;
        a.seg_v[q] = (seg && b->seg_v[slot]) ? b->seg_v[slot] + (long long)(it - b->seg0) * field : nullptr;
        a.seg_ds[q] = (seg && b->seg_ds[slot]) ? b->seg_ds[slot] + (long long)(it - b->seg0) * field : nullptr;
    }
    if (b->mode == FWI_SH) {
        a.stf[0] = b->stf[1];
        a.stf[1] = nullptr;
    } else {
        a.stf[0] = b->stf[0];
        a.stf[1] = b->stf[2];
    }
    if (adjoint) a.rec_cell = nullptr;  // the adjoint records nothing (solver.py:308-321)
    switch (b->mode) {
        case FWI_SH: return launch_mode<FWI_SH>(a, b->nshots, b->tile, st);
        case FWI_PSV: return launch_mode<FWI_PSV>(a, b->nshots, b->tile, st);
        case FWI_SPIN: return launch_mode<FWI_SPIN>(a, b->nshots, b->tile, st);
    }
    return set_error(FWI_EINVAL, "unknown mode %d", b->mode);
}

// ---------------------------------------------- multi-instance host side

// Forward step arguments of batch b for ping-pong half `cur` (no snapshots,
// no segment stores).
static void forward_args(const fwi_batch *b, int cur, StepArgs &a) {
    base_args(b, a);
    a.it = 0;
    const int ns = nfields_sig(b->mode), nv = nfields_vel(b->mode), nxt = 1 - cur;
    for (int f = 0; f < 6; f++) {
        a.sig_in[f] = f < ns ? b->sig[cur][f] : nullptr;
        a.sig_out[f] = f < ns ? b->sig[nxt][f] : nullptr;
    }
    for (int q = 0; q < 3; q++) {
        const bool on = q < nv;
        a.vel_in[q] = on ? b->vel[cur][q] : nullptr;
        a.vel_out[q] = on ? b->vel[nxt][q] : nullptr;
        a.disp[q] = on ? b->disp[q] : nullptr;
        a.obs[q] = on ? b->obs[comp_slot(b->mode, q)] : nullptr;
        a.snap_u[q] = a.snap_v[q] = a.seg_v[q] = a.seg_ds[q] = nullptr;
    }
    if (b->mode == FWI_SH) {
        a.stf[0] = b->stf[1];
        a.stf[1] = nullptr;
    } else {
        a.stf[0] = b->stf[0];
        a.stf[1] = b->stf[2];
    }
}

// Instances ordered by nt, longest first (stable), and the prefix sums of
// their block counts.
static void multi_plan(fwi_batch *const *bs, int n, int tx, int *order, long long *prefix) {
    for (int i = 0; i < n; i++) order[i] = i;
    for (int i = 1; i < n; i++)
        for (int j = i; j > 0 && bs[order[j]]->nt > bs[order[j - 1]]->nt; j--) {
            const int t = order[j];
            order[j] = order[j - 1];
            order[j - 1] = t;
        }
    prefix[0] = 0;
    for (int i = 0; i < n; i++) {
        const fwi_batch *b = bs[order[i]];
        prefix[i + 1] = prefix[i] + (long long)((b->nz + 31) / 32) * ((b->nx + tx - 1) / tx) * b->nshots;
    }
}

static int multi_tx(int tile) { return tile == 0 ? 32 : (tile_kind(tile) >= 1 && kTiles[tile].tz == 32 ? kTiles[tile].tx : -1); }

long long multi_workspace_bytes(int n) {
    return (long long)n * (long long)sizeof(MultiInst) + 4ll * (n + 1) + 256;
}

int multi_prepare(fwi_batch *const *bs, int n, void *ws, int (*check)(const fwi_batch *, int, int, int)) {
    if (n < 1 || n > 4096 || !bs || !ws) return set_error(FWI_EINVAL, "fwi_multi_prepare: 1 <= n <= 4096 batches");
    const int mode = bs[0]->mode, tx = multi_tx(bs[0]->tile);
    if (tx < 0) return set_error(FWI_EINVAL, "fwi_multi_prepare: tile %d is not a 32-column register-window variant",
                                 bs[0]->tile);
    for (int i = 0; i < n; i++) {
        int rc = check(bs[i], 0, 0, 0);
        if (rc) return rc;
        if (bs[i]->mode != mode || bs[i]->tile != bs[0]->tile)
            return set_error(FWI_EINVAL, "fwi_multi_prepare: all batches need the same mode and tile");
        if (bs[i]->cur != bs[0]->cur) return set_error(FWI_EINVAL, "fwi_multi_prepare: batches out of step (cur)");
    }
    int *order = new int[n];
    long long *prefix = new long long[n + 1];
    multi_plan(bs, n, tx, order, prefix);
    if (prefix[n] >= (1ll << 31)) {
        delete[] order;
        delete[] prefix;
        return set_error(FWI_ERANGE, "fwi_multi_prepare: %lld blocks per step exceed 2^31", prefix[n]);
    }
    MultiInst *h = new MultiInst[n];
    int *hp = new int[n + 1];
    for (int i = 0; i < n; i++) {
        const fwi_batch *b = bs[order[i]];
        forward_args(b, 0, h[i].a[0]);
        forward_args(b, 1, h[i].a[1]);
        h[i].tiles_z = (b->nz + 31) / 32;
        h[i].tiles_x = (b->nx + tx - 1) / tx;
        h[i].nshots = b->nshots;
        h[i].nt = b->nt;
    }
    for (int i = 0; i <= n; i++) hp[i] = (int)prefix[i];
    char *w = static_cast<char *>(ws);
    cudaError_t e = cudaMemcpy(w, h, sizeof(MultiInst) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(w + sizeof(MultiInst) * n, hp, 4 * (n + 1), cudaMemcpyHostToDevice);
    delete[] h;
    delete[] hp;
    delete[] order;
    delete[] prefix;
    (void)mode;
    if (e != cudaSuccess) return set_error(FWI_ECUDA, "fwi_multi_prepare: %s", cudaGetErrorString(e));
    return 0;
}

template <int MODE, int TX>
static int launch_multi(const MultiInst *inst, const int *prefix, int nactive, int blocks, int it, int cur,
                        cudaStream_t st) {
    using T = Tile<MODE, TX, 32>;
    static bool set = false;
    if (!set) {
        cudaError_t e = cudaFuncSetAttribute(step_kernel_multi<MODE, TX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)T::bytes);
        if (e != cudaSuccess) return set_error(FWI_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
        set = true;
    }
    step_kernel_multi<MODE, TX><<<blocks, kThreads, T::bytes, st>>>(inst, prefix, nactive, it, cur);
    return check_launch("step_kernel_multi");
}

int multi_run(fwi_batch *const *bs, int n, void *ws, int it0, int nsteps, cudaStream_t st) {
    if (n < 1 || !bs || !ws || nsteps < 0 || it0 < 0) return set_error(FWI_EINVAL, "fwi_multi_run: bad arguments");
    const int mode = bs[0]->mode, tx = multi_tx(bs[0]->tile);
    if (tx != 32 && tx != 16 && tx != 64) return set_error(FWI_EINVAL, "fwi_multi_run: unsupported tile");
    int *order = new int[n];
    long long *prefix = new long long[n + 1];
    multi_plan(bs, n, tx, order, prefix);
    const MultiInst *inst = static_cast<const MultiInst *>(ws);
    const int *pdev = reinterpret_cast<const int *>(static_cast<const char *>(ws) + sizeof(MultiInst) * n);
    int rc = 0;
    const int cur0 = bs[order[0]]->cur;
    for (int it = it0; it < it0 + nsteps && !rc; it++) {
        int nactive = 0;
        while (nactive < n && bs[order[nactive]]->nt > it) nactive++;
        if (!nactive) break;
        const int cur = (cur0 + (it - it0)) & 1;
        const int blocks = (int)prefix[nactive];
        if (mode == FWI_SH) {
            rc = tx == 32 ? launch_multi<FWI_SH, 32>(inst, pdev, nactive, blocks, it, cur, st)
                 : tx == 16 ? launch_multi<FWI_SH, 16>(inst, pdev, nactive, blocks, it, cur, st)
                            : launch_multi<FWI_SH, 64>(inst, pdev, nactive, blocks, it, cur, st);
        } else if (mode == FWI_PSV) {
            rc = tx == 32 ? launch_multi<FWI_PSV, 32>(inst, pdev, nactive, blocks, it, cur, st)
                 : tx == 16 ? launch_multi<FWI_PSV, 16>(inst, pdev, nactive, blocks, it, cur, st)
                            : launch_multi<FWI_PSV, 64>(inst, pdev, nactive, blocks, it, cur, st);
        } else {
            rc = launch_multi<FWI_SPIN, 32>(inst, pdev, nactive, blocks, it, cur, st);
        }
        for (int i = 0; i < nactive && !rc; i++) bs[order[i]]->cur ^= 1;
    }
    delete[] order;
    delete[] prefix;
    return rc;
}

}  // namespace fwi
