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
#include <cooperative_groups.h>

#include <type_traits>

#include <cstdio>

#include "common.cuh"
#include "stencil.cuh"

namespace cg = cooperative_groups;

namespace fwi {

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
    float *seg_e[6];   // per-step store of the stress-update terms of the new velocity (exact adjoint):
                       // SH exy, ezy | P-SV exx, ezz, exz+ezx | spin also -vyc-(ezx-exz)/2, Dx+vyc,
                       // Dz+vyc; slot-offset, or NULL
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

// Device-side status of the TMA kernels (a wait that gave up), read and
// cleared by fwi_device_status.
__device__ int g_device_status = 0;

int step_device_status(int clear, int *status) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_device_status, sizeof(int)) != cudaSuccess)
        return set_error(FWI_ECUDA, "fwi_device_status: reading the step kernels' status failed");
    if (clear && v) {
        const int z = 0;
        if (cudaMemcpyToSymbol(g_device_status, &z, sizeof(int)) != cudaSuccess)
            return set_error(FWI_ECUDA, "fwi_device_status: clearing the step kernels' status failed");
    }
    *status = v;
    return 0;
}

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
        const float dm = dt * ip[0], exy = dxp(0), ezy = dzp(0);
        a.sig_out[0][g] = s0[0] + dm * exy;
        a.sig_out[1][g] = s0[FS] + dm * ezy;
        if (a.seg_e[0]) {
            a.seg_e[0][g] = exy;
            a.seg_e[1][g] = ezy;
        }
    } else {
        const float lam = ip[0], mu = ip[FI];
        const float vxx = dxp(0), vxz = dzp(0), vzx = dxp(1), vzz = dzp(1);
        const float l2m = lam + 2.f * mu, shear = vxz + vzx;
        a.sig_out[0][g] = s0[0] + dt * (l2m * vxx + lam * vzz);
        a.sig_out[1][g] = s0[FS] + dt * (l2m * vzz + lam * vxx);
        a.sig_out[2][g] = s0[2 * FS] + dt * (mu * shear);
        if (MODE == FWI_PSV && a.seg_e[0]) {
            a.seg_e[0][g] = vxx;
            a.seg_e[1][g] = vzz;
            a.seg_e[2][g] = shear;
        }
        if (MODE == FWI_SPIN) {
            const float nu = ip[2 * FI], mnc = ip[3 * FI];
            const float rot = -vyc - 0.5f * (vzx - vxz), eyx = dxp(2), eyz = dzp(2);
            a.sig_out[4][g] = s0[4 * FS] + a.dt2 * nu * rot;
            a.sig_out[3][g] = s0[3 * FS] + dt * mnc * eyx;
            a.sig_out[5][g] = s0[5 * FS] + dt * mnc * eyz;
            if (a.seg_e[0]) {
                a.seg_e[0][g] = vxx;
                a.seg_e[1][g] = vzz;
                a.seg_e[2][g] = shear;
                a.seg_e[3][g] = rot;
                a.seg_e[4][g] = eyx;
                a.seg_e[5][g] = eyz;
            }
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
    constexpr int SZ = T::SZ;
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
    constexpr int SX = T::SX, SZ = T::SZ;
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
    constexpr int SZ = T::SZ;
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

// ------------------------------------------------------------- launching

struct TileShape {
    int tx, tz, rw;
};
// Variants selectable through fwi_batch.tile; 0 is the default.
// rw: 0 generic mapping, 1 register window + cp.async, 2 register window + TMA
static const TileShape kTiles[] = {{32, 32, 2}, {32, 32, 0}, {16, 64, 0}, {16, 32, 0}, {64, 32, 0}, {8, 64, 0},
                                   {32, 32, 1}, {16, 32, 1}, {64, 32, 1}, {32, 32, 2}, {16, 32, 2}, {8, 32, 2}};
constexpr int kNumTiles = sizeof(kTiles) / sizeof(kTiles[0]);

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
        a.seg_ds[q] = (seg && b->seg_ds[slot]) ? b->seg_ds[slot] + (long long)(it - b->seg0) * field : nullptr;
    }
    {
        const bool seg = !adjoint && it - b->seg0 >= 0 && it - b->seg0 < b->nseg;
        const int ne = b->mode == FWI_SH ? 2 : b->mode == FWI_PSV ? 3 : 6;
        for (int k = 0; k < 6; k++)
            a.seg_e[k] = (seg && k < ne && b->seg_e[k]) ? b->seg_e[k] + (long long)(it - b->seg0) * field : nullptr;
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
        a.snap_u[q] = a.snap_v[q] = a.seg_ds[q] = nullptr;
    }
    for (int k = 0; k < 6; k++) a.seg_e[k] = nullptr;
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
        if (!bs[i]->disp[0]) return set_error(FWI_EINVAL, "fwi_multi_prepare: batches need displacement fields");
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

// ------------------------------------------------ exact discrete adjoint
//
// The forward step above is linear in the state.  For SH / P-SV it reads
//   d  = D- sig + f            (stress divergence plus sources)
//   v' = B (v + b d)           (b = dt/rho, B = sponge)
//   u' = u + dt v'
//   sig' = sig + dt S(D+ v')   (S: lam/mu stress-strain law)
// Its exact transpose, run backwards in time on the adjoint state, is
//   a    = v~ + dt u~ + (D+)^T (dt S^T sig~)
//   v~'  = B a
//   sig~' = sig~ + (D-)^T (b v~')
// with (D+)^T and (D-)^T the transposes of the reference's masked stencils
// (solver.py:22-51), boundary masks included, so the adjoint is exact to
// rounding.  The displacement feeds nothing but the receivers, so its
// adjoint u~ is zero away from them and equals, at a receiver, the sum of
// dL/d(trace) over the steps still to come: the caller passes those suffix
// sums (fwi_trace_suffix_sum) as the injection values and u~ never exists
// as a field.  The same launch adds this step's gradient terms
//   dL/dlam = sum dt (sxx~+szz~)(exx+ezz),
//   dL/dmu  = sum dt (2 sxx~ exx + 2 szz~ ezz + sxz~ (exz+ezx))  [SH: dt (sxy~ exy + szy~ ezy)]
//   dL/db   = sum v~' . d
// (sig~ before the step; e = D+ of the forward v' and d are stored per step,
// pointwise, by a recomputed forward segment).
//
// Mapping.  A cluster of C <= 8 CTAs owns one 32 x 32 tile; CTA r of the
// cluster processes shots r, r+C, ... in turn, keeping the model tile
// (stiffness with halo, dt/rho, sponge) in shared memory across its shots
// and its gradient terms in registers.  Per shot it forms t = dt S^T sig~ in
// place over the staged sig~, computes v~' on the interior (lane = z, x taps
// in a register window, as step_kernel_rw) plus the halo, then sig~' and the
// gradient terms of the interior.  Staging is pipelined with TMA: the next
// shot's sig~ streams in as soon as t has been consumed, its v~ and strain
// once the stress half is done (the injection waits for v~ only after t has
// been formed, so that copy overlaps the t pass).  At the
// end the cluster sums its CTAs' terms through distributed shared memory in
// rank order and adds them once into the FP64 gradient arrays: one
// read-modify-write per cell and step for all shots, deterministic, no
// atomics.

struct AdjArgs {
    int nx, nz, pitch, nt, it, nshots;
    FastDiv divnz;
    float cx1, cx2, cz1, cz2, dt, dt2;
    float *sig_out[6];
    float *vel_out[3];
    const float *dsf[3];  // forward divergence of step it, per velocity component (NULL: no density terms)
    const float *ef[6];   // forward stress-update terms of v(it+1) (fwi_batch.seg_e)
    double *k[6];         // SH: dL/dmu, dL/dbuo | P-SV: dL/dlam, dL/dmu, dL/dbuo |
                          // spin: dL/dlam, dL/dmu, dL/dnu, dL/dmnc, dL/dbuo, dL/dbuo_j ([nx][pitch], NULL skips)
    const int *inj_ptr, *inj_cell, *inj_row;
    const float *g[2];    // u~ at the receivers per step (forward time order)
};

struct AdjMaps {
    CUtensorMap sig[6];  // sig~, stress region box
    CUtensorMap vel[3];  // v~, velocity region box
    CUtensorMap ef[6];   // forward stress-update terms, interior box
    CUtensorMap lm[4];   // SH: mu | P-SV: lam, mu | spin: lam, mu, nu, mnc; stress region box
    CUtensorMap vp[3];   // dt/rho, sponge (spin: dt/j); velocity region box
};

template <int MODE>
struct AdjTile {
    using F = Fields<MODE>;
    // spin holds twice the fields: 16 x 32 tiles keep two CTAs per SM
    static constexpr int TX = MODE == FWI_SPIN ? 16 : 32, TZ = 32;
    static constexpr int SX = TX + 6, SZ = TZ + 8, VX = TX + 3, RVZ = TZ + 3;
    static constexpr int FS = (SX * SZ + 31) / 32 * 32, FV = (VX * SZ + 31) / 32 * 32;
    static constexpr int NL = MODE == FWI_SH ? 1 : MODE == FWI_PSV ? 2 : 4;  // stiffness fields
    static constexpr int NK = MODE == FWI_SH ? 2 : MODE == FWI_PSV ? 3 : 6;  // gradient fields
    static constexpr int NE = MODE == FWI_SH ? 2 : MODE == FWI_PSV ? 3 : 6;  // forward stress-update terms
    static constexpr int NP = MODE == FWI_SPIN ? 3 : 2;                      // velocity-region model fields
    static constexpr int KB = MODE == FWI_SH ? 1 : MODE == FWI_PSV ? 2 : 4;  // gradient slot of dt/rho
    // sig~ (turned into t in place), v~, the forward strain of the interior,
    // the model tile, the injection list and three mbarriers (model, sig~,
    // v~ with strain)
    static constexpr int V_OFF = F::NS * FS, E_OFF = V_OFF + F::NV * FV;
    static constexpr int L_OFF = E_OFF + NE * TX * TZ, P_OFF = L_OFF + NL * FS;
    static constexpr int LIST_OFF = P_OFF + NP * FV;
    static constexpr int LIST = kThreads * (1 + F::NINJ) + 8;
    static constexpr int BAR_OFF = (LIST_OFF + LIST + 1) / 2 * 2;
    static constexpr size_t bytes = sizeof(float) * (size_t)(BAR_OFF + 8);
    static constexpr uint32_t sig_bytes = 4u * F::NS * SX * SZ;
    static constexpr uint32_t vel_bytes = 4u * (F::NV * VX * SZ + NE * TX * TZ);
    static constexpr uint32_t model_bytes = 4u * (NL * SX * SZ + NP * VX * SZ);
    static_assert(NK * TX * TZ <= L_OFF, "gradient terms overlay the per-shot buffers");
    static_assert(vel_bytes < (1u << 20) && model_bytes < (1u << 20), "mbarrier transaction count limit");
};

// Injection of u~ for one shot: entries whose cell lies in the computed
// velocity region add dt * u~ to the staged v~, summed per cell in entry
// order.  adj_collect compacts up to kThreads entries [base, p1) into the
// list (block-wide; the count it returns is block-uniform) and may run
// while the staging copies are in flight; adj_apply adds them once v~ has
// landed and the list is visible to thread 0.
// adj_fetch: this thread's entry base + tid (its shared-memory location in
// the staged v~, or -1, and its u~ values); no barrier, so it can be issued
// well before adj_compact needs it.
template <int MODE>
__device__ __forceinline__ void adj_fetch(const AdjArgs &a, int base, int p1, int x0, int z0, int &loc,
                                          float (&val)[Fields<MODE>::NINJ]) {
    using T = AdjTile<MODE>;
    const int e = base + (int)threadIdx.x;
    loc = -1;
#pragma unroll
    for (int c = 0; c < Fields<MODE>::NINJ; c++) val[c] = 0.f;
    if (e < p1) {
        const int k = a.inj_cell[e];
        const int gx = fdiv(k, a.divnz), gz = k - gx * a.nz;
        const int rx = gx - (x0 - 1), rz = gz - (z0 - 1);
        if (rx >= 0 && rx < T::VX && rz >= 0 && rz < T::RVZ) {
            loc = rx * T::SZ + rz + 3;
            const long long src = (long long)a.inj_row[e] * a.nt + a.it;
#pragma unroll
            for (int c = 0; c < Fields<MODE>::NINJ; c++) val[c] = a.g[c][src];
        }
    }
}

template <int MODE>
__device__ __forceinline__ int adj_compact(int loc, const float (&val)[Fields<MODE>::NINJ], int *sLoc, float *sVal,
                                           int *sWarp) {
    constexpr int NINJ = Fields<MODE>::NINJ;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned ball = __ballot_sync(0xffffffffu, loc >= 0);
    if (lane == 0) sWarp[warp] = __popc(ball);
    __syncthreads();
    int n = 0, pos = __popc(ball & ((1u << lane) - 1u));
    for (int w = 0; w < kThreads / 32; w++) {
        if (w < warp) pos += sWarp[w];
        n += sWarp[w];
    }
    if (loc >= 0) {
        sLoc[pos] = loc;
#pragma unroll
        for (int c = 0; c < NINJ; c++) sVal[c * kThreads + pos] = val[c];
    }
    return n;
}

template <int MODE>
__device__ __forceinline__ int adj_collect(const AdjArgs &a, int base, int p1, int x0, int z0, int *sLoc,
                                           float *sVal, int *sWarp) {
    int loc;
    float val[Fields<MODE>::NINJ];
    adj_fetch<MODE>(a, base, p1, x0, z0, loc, val);
    return adj_compact<MODE>(loc, val, sLoc, sVal, sWarp);
}

template <int MODE>
__device__ __forceinline__ void adj_apply(float *sV, int n, const int *sLoc, const float *sVal, float dt) {
    if (threadIdx.x != 0) return;
    for (int q = 0; q < n; q++) {
#pragma unroll
        for (int c = 0; c < Fields<MODE>::NINJ; c++)
            sV[c * AdjTile<MODE>::FV + sLoc[q]] += dt * sVal[c * kThreads + q];
    }
}

// The velocity-like terms of the transposed step, (C^T t) per component,
// from the transposed D+ of t (dxpT, dzpT) and, for spin, t4 at the cell:
//   SH    a_y = Dx+^T t0 + Dz+^T t1
//   P-SV  a_x = Dx+^T t0 + Dz+^T t2,  a_z = Dx+^T t2 + Dz+^T t1
//   spin  a_x += Dz+^T t4 / 2,  a_z -= Dx+^T t4 / 2,  a_yc = -t4 + Dx+^T t3 + Dz+^T t5
// (the transpose of stress_update's syy_c term dt2 nu (-vyc - (vzx - vxz)/2)).
template <int MODE, class DXP, class DZP>
__device__ __forceinline__ void adj_vel_terms(DXP dxpT, DZP dzpT, float t4c, float (&acc)[3]) {
    if (MODE == FWI_SH) {
        acc[0] = dxpT(0) + dzpT(1);
    } else {
        acc[0] = dxpT(0) + dzpT(2);
        acc[1] = dxpT(2) + dzpT(1);
        if (MODE == FWI_SPIN) {
            acc[0] += 0.5f * dzpT(4);
            acc[1] -= 0.5f * dxpT(4);
            acc[2] = (dxpT(3) + dzpT(5)) - t4c;
        }
    }
}

template <int MODE>
__global__ void __launch_bounds__(kThreads, MODE == FWI_SH ? 4 : MODE == FWI_PSV ? 3 : 2)
    adjoint_kernel(const __grid_constant__ AdjArgs a, const __grid_constant__ AdjMaps m) {
    using T = AdjTile<MODE>;
    using F = Fields<MODE>;
    constexpr int TX = T::TX, TZ = T::TZ, SX = T::SX, SZ = T::SZ, RVZ = T::RVZ, FS = T::FS, FV = T::FV;
    constexpr int NS = F::NS, NV = F::NV, NL = T::NL, NK = T::NK, NE = T::NE, RPW = TX / (kThreads / 32);
    extern __shared__ __align__(128) float smem[];
    float *sS = smem, *sV = smem + T::V_OFF, *sE = smem + T::E_OFF, *sL = smem + T::L_OFF, *sP = smem + T::P_OFF;
    int *sLoc = reinterpret_cast<int *>(smem + T::LIST_OFF);
    float *sVal = reinterpret_cast<float *>(sLoc + kThreads);
    int *sWarp = reinterpret_cast<int *>(sVal + F::NINJ * kThreads);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + T::BAR_OFF);  // model, sig~, v~ with strain
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank(), csize = (int)cluster.num_blocks();

    const int tid = threadIdx.x, lane = tid & 31, ix0 = (tid >> 5) * RPW;
    const int z0 = blockIdx.x * TZ, x0 = blockIdx.y * TX;
    const int nx = a.nx, nz = a.nz, pitch = a.pitch, nshots = a.nshots;
    const int gz = z0 + lane, col = lane + 4;
    const bool zin = gz < nz;
    const float dt = a.dt, cx1 = a.cx1, cx2 = a.cx2, cz1 = a.cz1, cz2 = a.cz2;
    // z masks of this lane: (D+)^T taps gz-2..gz+1, (D-)^T taps gz-1..gz+2;
    // all ones (and skipped) unless the tile reaches a z edge
    const bool zedge = !(z0 >= 3 && z0 + TZ + 4 <= nz);
    float pz[4], mz[4];
#pragma unroll
    for (int d = 0; d < 4; d++) {
        const int kp = gz - 2 + d, km = gz - 1 + d;
        pz[d] = (kp >= 1 && kp < nz - 2) ? 1.f : 0.f;
        mz[d] = (km >= 2 && km < nz - 2) ? 1.f : 0.f;
    }

    // copies issued by thread 0; each refill of a buffer is ordered after the
    // generic-proxy accesses that preceded it (the barrier before the call)
    auto issue_sig = [&](int shot) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&bar[1], T::sig_bytes);
#pragma unroll
        for (int f = 0; f < NS; f++) tma_load_3d(sS + f * FS, &m.sig[f], z0 - 4, x0 - 3, shot, &bar[1]);
    };
    auto issue_vel = [&](int shot) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&bar[2], T::vel_bytes);
#pragma unroll
        for (int q = 0; q < NV; q++) tma_load_3d(sV + q * FV, &m.vel[q], z0 - 4, x0 - 1, shot, &bar[2]);
#pragma unroll
        for (int k = 0; k < NE; k++) tma_load_3d(sE + k * TX * TZ, &m.ef[k], z0, x0, shot, &bar[2]);
    };
    if (tid == 0) {
#pragma unroll
        for (int b = 0; b < 3; b++) mbar_init(&bar[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        mbar_expect_tx(&bar[0], T::model_bytes);
#pragma unroll
        for (int f = 0; f < NL; f++) tma_load_2d(sL + f * FS, &m.lm[f], z0 - 4, x0 - 3, &bar[0]);
#pragma unroll
        for (int p = 0; p < T::NP; p++) tma_load_2d(sP + p * FV, &m.vp[p], z0 - 4, x0 - 1, &bar[0]);
        if (crank < nshots) {
            issue_sig(crank);
            issue_vel(crank);
        }
    }

    float gk[NK][RPW];
#pragma unroll
    for (int k = 0; k < NK; k++)
#pragma unroll
        for (int q = 0; q < RPW; q++) gk[k][q] = 0.f;

    // injection entries of the next shot, fetched a shot ahead (one entry
    // per thread; shots with more entries than threads are collected later)
    int nx_loc = -1;
    float nx_val[F::NINJ];
    auto prefetch_entries = [&](int shot) {
        const int q0 = a.inj_ptr ? a.inj_ptr[shot] : 0, q1 = a.inj_ptr ? a.inj_ptr[shot + 1] : 0;
        if (q1 - q0 <= kThreads) adj_fetch<MODE>(a, q0, q1, x0, z0, nx_loc, nx_val);
    };
    if (crank < nshots) prefetch_entries(crank);
    int i = 0;
    for (int shot = crank; shot < nshots; shot += csize, i++) {
        const long long soff = (long long)shot * nx * pitch;
        // forward divergence of the interior cells (read once: straight from HBM)
        float dsv[NV][RPW];
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            const int gx = x0 + ix0 + q;
            const bool in = zin && gx < nx;
#pragma unroll
            for (int c = 0; c < NV; c++) dsv[c][q] = (in && a.dsf[0]) ? a.dsf[c][soff + (long long)gx * pitch + gz] : 0.f;
        }
        const int p0 = a.inj_ptr ? a.inj_ptr[shot] : 0, p1 = a.inj_ptr ? a.inj_ptr[shot + 1] : 0;
        const bool single = p1 - p0 <= kThreads;
        int n_in = 0;
        if (single && p1 > p0) n_in = adj_compact<MODE>(nx_loc, nx_val, sLoc, sVal, sWarp);

        // sig~ of the interior cells into registers (t overwrites it)
        bool ok = mbar_wait(&bar[1], i & 1);
        if (i == 0) ok = mbar_wait(&bar[0], 0) && ok;
        float sg[NS][RPW];
#pragma unroll
        for (int f = 0; f < NS; f++)
#pragma unroll
            for (int q = 0; q < RPW; q++) sg[f][q] = sS[f * FS + (ix0 + q + 3) * SZ + col];
        if (__syncthreads_or(!ok)) {  // block-uniform decision
            if (tid == 0) atomicExch(&g_device_status, 1);
            // one more bounded chance for every copy in flight to land
            mbar_wait(&bar[1], i & 1);
            mbar_wait(&bar[2], i & 1);
            if (i == 0) mbar_wait(&bar[0], 0);
            break;
        }
        // t = dt S^T sig~ in place over the whole stress region, four cells
        // (one 16-byte vector) at a time
        for (int c = tid; c < SX * (SZ / 4); c += kThreads) {
            float4 *s4 = reinterpret_cast<float4 *>(sS) + c;
            const float4 *l4 = reinterpret_cast<const float4 *>(sL) + c;
            constexpr int F4 = FS / 4;
            if (MODE == FWI_SH) {
                const float4 mu = l4[0];
                float4 a0 = s4[0], a1 = s4[F4];
                a0.x = dt * (mu.x * a0.x); a0.y = dt * (mu.y * a0.y); a0.z = dt * (mu.z * a0.z); a0.w = dt * (mu.w * a0.w);
                a1.x = dt * (mu.x * a1.x); a1.y = dt * (mu.y * a1.y); a1.z = dt * (mu.z * a1.z); a1.w = dt * (mu.w * a1.w);
                s4[0] = a0;
                s4[F4] = a1;
            } else {
                const float4 l = l4[0], mu = l4[F4];
                float4 xx = s4[0], zz = s4[F4], xz = s4[2 * F4];
                auto t3 = [&](float lc, float mc, float &sxx, float &szz, float &sxz) {
                    const float l2m = lc + 2.f * mc, a = sxx, b = szz;
                    sxx = dt * (l2m * a + lc * b);
                    szz = dt * (lc * a + l2m * b);
                    sxz = dt * (mc * sxz);
                };
                t3(l.x, mu.x, xx.x, zz.x, xz.x);
                t3(l.y, mu.y, xx.y, zz.y, xz.y);
                t3(l.z, mu.z, xx.z, zz.z, xz.z);
                t3(l.w, mu.w, xx.w, zz.w, xz.w);
                s4[0] = xx;
                s4[F4] = zz;
                s4[2 * F4] = xz;
                if (MODE == FWI_SPIN) {
                    // t3 = dt mnc syx~, t4 = 2dt nu syy~, t5 = dt mnc syz~
                    const float4 nu = l4[2 * F4], mn = l4[3 * F4];
                    float4 a3 = s4[3 * F4], a4 = s4[4 * F4], a5 = s4[5 * F4];
                    const float d2 = a.dt2;
                    a3.x = dt * (mn.x * a3.x); a3.y = dt * (mn.y * a3.y); a3.z = dt * (mn.z * a3.z); a3.w = dt * (mn.w * a3.w);
                    a5.x = dt * (mn.x * a5.x); a5.y = dt * (mn.y * a5.y); a5.z = dt * (mn.z * a5.z); a5.w = dt * (mn.w * a5.w);
                    a4.x = d2 * (nu.x * a4.x); a4.y = d2 * (nu.y * a4.y); a4.z = d2 * (nu.z * a4.z); a4.w = d2 * (nu.w * a4.w);
                    s4[3 * F4] = a3;
                    s4[4 * F4] = a4;
                    s4[5 * F4] = a5;
                }
            }
        }
        // v~ and the forward strain of this shot; u~ enters v~ (thread 0)
        ok = mbar_wait(&bar[2], i & 1);
        if (single && ok) adj_apply<MODE>(sV, n_in, sLoc, sVal, dt);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(&g_device_status, 1);
            mbar_wait(&bar[2], i & 1);
            break;
        }
        if (!single) {
            for (int base = p0; base < p1; base += kThreads) {
                __syncthreads();
                const int n = adj_collect<MODE>(a, base, p1, x0, z0, sLoc, sVal, sWarp);
                __syncthreads();
                adj_apply<MODE>(sV, n, sLoc, sVal, dt);
            }
            __syncthreads();
        }

        // ---- v~' on the warp's interior rows; t rows x-2 .. x+1 of the
        // x-differentiated fields in a register window, pre-masked
        // (window index r <-> stress row ix0+1+r <-> grid row x0+ix0-2+r)
        auto vel_interior = [&](auto zm) {
            constexpr bool ZM = decltype(zm)::value;  // z masks needed (tile at a z edge)
            float w[NS][RPW + 3];
#pragma unroll
            for (int f = 0; f < NS; f++)
                if (takes_dxm(MODE, f)) {
#pragma unroll
                    for (int r = 0; r < RPW + 3; r++) {
                        const int gr = x0 + ix0 - 2 + r;
                        w[f][r] = (gr >= 1 && gr < nx - 2) ? sS[f * FS + (ix0 + 1 + r) * SZ + col] : 0.f;
                    }
                }
#pragma unroll
            for (int q = 0; q < RPW; q++) {
                const int ix = ix0 + q, gx = x0 + ix;
                const int vi = (ix + 1) * SZ + col;
                if (!(zin && gx < nx)) {
#pragma unroll
                    for (int c = 0; c < NV; c++) sV[c * FV + vi] = 0.f;
                    continue;
                }
                const float *trow = sS + (ix + 3) * SZ + col;
                auto dxpT = [&](int f) -> float {
                    return cx1 * (w[f][q + 1] - w[f][q + 2]) - cx2 * (w[f][q] - w[f][q + 3]);
                };
                auto dzpT = [&](int f) -> float {
                    const float *t = trow + f * FS;
                    if constexpr (ZM)
                        return cz1 * (t[-1] * pz[1] - t[0] * pz[2]) - cz2 * (t[-2] * pz[0] - t[1] * pz[3]);
                    else
                        return cz1 * (t[-1] - t[0]) - cz2 * (t[-2] - t[1]);
                };
                float acc[3];
                adj_vel_terms<MODE>(dxpT, dzpT, MODE == FWI_SPIN ? trow[4 * FS] : 0.f, acc);
                const float buo = sP[vi], bnd = sP[FV + vi];
                const long long g = soff + (long long)gx * pitch + gz;
                float gb = 0.f;
#pragma unroll
                for (int c = 0; c < NV; c++) {
                    const float vn = bnd * (sV[c * FV + vi] + acc[c]);
                    a.vel_out[c][g] = vn;
                    if (MODE == FWI_SPIN && c == 2) {
                        sV[c * FV + vi] = sP[2 * FV + vi] * vn;
                        gk[T::KB + 1][q] += vn * dsv[c][q];
                    } else {
                        sV[c * FV + vi] = buo * vn;
                        gb += vn * dsv[c][q];
                    }
                }
                gk[T::KB][q] += gb;
            }
        };
        if (zedge) vel_interior(std::true_type{});
        else vel_interior(std::false_type{});
        // ---- v~' on the halo rows x0-1, x0+TX, x0+TX+1 and columns z0-1,
        // z0+TZ, z0+TZ+1 (redundant with the neighbour tiles; masks per tap)
        {
            constexpr int HROW = 3 * RVZ, HC = HROW + 3 * TX;
            auto mxp = [&](int k) -> float { return (k >= 1 && k < nx - 2) ? 1.f : 0.f; };
            auto mzp = [&](int k) -> float { return (k >= 1 && k < nz - 2) ? 1.f : 0.f; };
            for (int c = tid; c < HC; c += kThreads) {
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
                const int hx = x0 - 1 + rx, hz = z0 - 1 + rz;
                const int vi = rx * SZ + rz + 3, si = (rx + 2) * SZ + rz + 3;
                if (hx < 0 || hx >= nx || hz < 0 || hz >= nz) {
#pragma unroll
                    for (int q = 0; q < NV; q++) sV[q * FV + vi] = 0.f;
                    continue;
                }
                auto dxpT = [&](int f) -> float {
                    const float *t = sS + f * FS + si;
                    return cx1 * (t[-SZ] * mxp(hx - 1) - t[0] * mxp(hx)) -
                           cx2 * (t[-2 * SZ] * mxp(hx - 2) - t[SZ] * mxp(hx + 1));
                };
                auto dzpT = [&](int f) -> float {
                    const float *t = sS + f * FS + si;
                    return cz1 * (t[-1] * mzp(hz - 1) - t[0] * mzp(hz)) - cz2 * (t[-2] * mzp(hz - 2) - t[1] * mzp(hz + 1));
                };
                float acc[3];
                adj_vel_terms<MODE>(dxpT, dzpT, MODE == FWI_SPIN ? sS[4 * FS + si] : 0.f, acc);
                const float bnd = sP[FV + vi];
#pragma unroll
                for (int q = 0; q < NV; q++) {
                    const float b = (MODE == FWI_SPIN && q == 2) ? sP[2 * FV + vi] : sP[vi];
                    sV[q * FV + vi] = b * (bnd * (sV[q * FV + vi] + acc[q]));
                }
            }
        }
        __syncthreads();
        // t has been consumed: the next shot's sig~ streams in during the stress half
        if (tid == 0 && shot + csize < nshots) issue_sig(shot + csize);
        if (shot + csize < nshots) prefetch_entries(shot + csize);

        // ---- sig~' and the stiffness gradient terms on the interior; b v~'
        // rows x-1 .. x+2 in a register window, pre-masked
        // (window index r <-> velocity row ix0+r <-> grid row x0+ix0-1+r)
        auto stress_interior = [&](auto zm) {
            constexpr bool ZM = decltype(zm)::value;
            float w[NV][RPW + 3];
#pragma unroll
            for (int c = 0; c < NV; c++) {
#pragma unroll
                for (int r = 0; r < RPW + 3; r++) {
                    const int gr = x0 + ix0 - 1 + r;
                    w[c][r] = (gr >= 2 && gr < nx - 2) ? sV[c * FV + (ix0 + r) * SZ + col] : 0.f;
                }
            }
#pragma unroll
            for (int q = 0; q < RPW; q++) {
                const int ix = ix0 + q, gx = x0 + ix;
                if (!(zin && gx < nx)) continue;
                const float *vrow = sV + (ix + 1) * SZ + col;
                const float *e = sE + ix * TZ + lane;
                auto dxmT = [&](int c) -> float {
                    return cx1 * (w[c][q + 1] - w[c][q + 2]) - cx2 * (w[c][q] - w[c][q + 3]);
                };
                auto dzmT = [&](int c) -> float {
                    const float *v = vrow + c * FV;
                    if constexpr (ZM)
                        return cz1 * (v[0] * mz[1] - v[1] * mz[2]) - cz2 * (v[-1] * mz[0] - v[2] * mz[3]);
                    else
                        return cz1 * (v[0] - v[1]) - cz2 * (v[-1] - v[2]);
                };
                const long long g = soff + (long long)gx * pitch + gz;
                if (MODE == FWI_SH) {
                    a.sig_out[0][g] = sg[0][q] + dxmT(0);
                    a.sig_out[1][g] = sg[1][q] + dzmT(0);
                    gk[0][q] += dt * (sg[0][q] * e[0] + sg[1][q] * e[TX * TZ]);
                } else {
                    a.sig_out[0][g] = sg[0][q] + dxmT(0);
                    a.sig_out[1][g] = sg[1][q] + dzmT(1);
                    a.sig_out[2][g] = sg[2][q] + (dzmT(0) + dxmT(1));
                    const float sxx = sg[0][q], szz = sg[1][q], sxz = sg[2][q];
                    const float exx = e[0], ezz = e[TX * TZ];
                    gk[0][q] += dt * ((sxx + szz) * (exx + ezz));
                    gk[1][q] += dt * (2.f * (sxx * exx + szz * ezz) + sxz * e[2 * TX * TZ]);
                    if (MODE == FWI_SPIN) {
                        // (A^T w): syx~ += (Dx-)^T w_y, syy~ += (Dz-)^T w_x - (Dx-)^T w_z + 2 w_y,
                        // syz~ += (Dz-)^T w_y
                        a.sig_out[3][g] = sg[3][q] + dxmT(2);
                        a.sig_out[4][g] = sg[4][q] + ((dzmT(0) - dxmT(1)) + 2.f * vrow[2 * FV]);
                        a.sig_out[5][g] = sg[5][q] + dzmT(2);
                        gk[2][q] += a.dt2 * (sg[4][q] * e[3 * TX * TZ]);
                        gk[3][q] += dt * (sg[3][q] * e[4 * TX * TZ] + sg[5][q] * e[5 * TX * TZ]);
                    }
                }
            }
        };
        if (zedge) stress_interior(std::true_type{});
        else stress_interior(std::false_type{});
        __syncthreads();
        // v~ and strain buffers are free: the next shot streams into them
        if (tid == 0 && shot + csize < nshots) issue_vel(shot + csize);
    }
    if (crank >= nshots) mbar_wait(&bar[0], 0);  // no shot: let the model copies land

    // ---- cluster sum of the gradient terms, in rank order, into FP64
    float *part = smem;
#pragma unroll
    for (int k = 0; k < NK; k++)
#pragma unroll
        for (int q = 0; q < RPW; q++) part[k * TX * TZ + (ix0 + q) * TZ + lane] = gk[k][q];
    cluster.sync();
    const int chunk = (TX * TZ + csize - 1) / csize, c0 = crank * chunk;
    for (int e = tid; e < NK * chunk; e += kThreads) {
        const int k = e / chunk, c = c0 + (e - k * chunk);
        if (c >= TX * TZ || !a.k[k]) continue;
        const int gx = x0 + c / TZ, gzc = z0 + c % TZ;
        if (gx >= nx || gzc >= nz) continue;
        double s = 0.0;
        for (int j = 0; j < csize; j++) s += (double)cluster.map_shared_rank(part, j)[k * TX * TZ + c];
        a.k[k][(long long)gx * pitch + gzc] += s;
    }
    cluster.sync();  // keep this CTA's shared memory alive until every rank has read it
}

// ------------------------------------------------ exact adjoint, wide P-SV tile
//
// The P-SV transposed step of adjoint_kernel with each lane owning two
// adjacent z columns (float2 loads and stores) of a 32 x 64 tile: half the
// address, mask and loop work per cell, a 14 % velocity halo instead of
// 20 %, and a stress region 1.34 times the interior instead of 1.48.  The
// forward strain and divergence are read straight from HBM (pointwise, once)
// instead of being staged, which keeps two CTAs per SM.  Same arithmetic per
// cell as adjoint_kernel<FWI_PSV> (the adjoint fields agree bit for bit);
// the gradient terms are summed over the cluster's CTAs in rank order as
// there.

struct WideTile {
    static constexpr int TX = 32, TZ = 64, SX = TX + 6, SZ = TZ + 8, VX = TX + 3, RVZ = TZ + 3;
    static constexpr int RPW = TX / (kThreads / 32);
    static constexpr int FS = (SX * SZ + 31) / 32 * 32, FV = (VX * SZ + 31) / 32 * 32;
    static constexpr int NS = 3, NV = 2, NK = 3, NINJ = 2;
    // sig~ (turned into t in place), v~ (turned into b v~'), lam and mu of
    // the stress region, dt/rho and sponge of the velocity region, the
    // injection list and three mbarriers (model, sig~, v~)
    static constexpr int V_OFF = NS * FS, L_OFF = V_OFF + NV * FV, P_OFF = L_OFF + 2 * FS;
    static constexpr int LIST_OFF = P_OFF + 2 * FV;
    static constexpr int LIST = kThreads * (1 + NINJ) + 8;
    static constexpr int BAR_OFF = (LIST_OFF + LIST + 1) / 2 * 2;
    static constexpr size_t bytes = sizeof(float) * (size_t)(BAR_OFF + 8);
    static constexpr uint32_t sig_bytes = 4u * NS * SX * SZ;
    static constexpr uint32_t vel_bytes = 4u * NV * VX * SZ;
    static constexpr uint32_t model_bytes = 4u * (2 * SX * SZ + 2 * VX * SZ);
    static_assert(RPW * (kThreads / 32) == TX && 2 * 32 == TZ, "a warp spans the tile's z extent, two columns a lane");
    static_assert(NK * TX * TZ <= L_OFF, "gradient terms overlay the per-shot buffers");
    static_assert(FS % 4 == 0 && FV % 4 == 0 && SZ % 4 == 0, "float4 / float2 alignment of the regions");
};

struct WideMaps {
    CUtensorMap sig[3];  // sig~, stress region box
    CUtensorMap vel[2];  // v~, velocity region box
    CUtensorMap lm[2];   // lam, mu; stress region box
    CUtensorMap vp[2];   // dt/rho, sponge; velocity region box
};

// One injection entry per thread: its location in the staged v~ (or -1)
// and its u~ values (adj_fetch for the wide tile).
__device__ __forceinline__ void wide_fetch(const AdjArgs &a, int base, int p1, int x0, int z0, int &loc,
                                           float (&val)[2]) {
    using T = WideTile;
    const int e = base + (int)threadIdx.x;
    loc = -1;
    val[0] = val[1] = 0.f;
    if (e < p1) {
        const int k = a.inj_cell[e];
        const int gx = fdiv(k, a.divnz), gz = k - gx * a.nz;
        const int rx = gx - (x0 - 1), rz = gz - (z0 - 1);
        if (rx >= 0 && rx < T::VX && rz >= 0 && rz < T::RVZ) {
            loc = rx * T::SZ + rz + 3;
            const long long src = (long long)a.inj_row[e] * a.nt + a.it;
            val[0] = a.g[0][src];
            val[1] = a.g[1][src];
        }
    }
}

__device__ __forceinline__ void wide_apply(float *sV, int n, const int *sLoc, const float *sVal, float dt) {
    if (threadIdx.x != 0) return;
    for (int q = 0; q < n; q++) {
        sV[sLoc[q]] += dt * sVal[q];
        sV[WideTile::FV + sLoc[q]] += dt * sVal[kThreads + q];
    }
}

__device__ __forceinline__ float2 ld2(const float *p) { return *reinterpret_cast<const float2 *>(p); }
__device__ __forceinline__ void st2(float *p, float x, float y) { *reinterpret_cast<float2 *>(p) = make_float2(x, y); }

__global__ void __launch_bounds__(kThreads, 2)
    adjoint_wide_kernel(const __grid_constant__ AdjArgs a, const __grid_constant__ WideMaps m) {
    using T = WideTile;
    constexpr int TX = T::TX, TZ = T::TZ, SX = T::SX, SZ = T::SZ, RVZ = T::RVZ, FS = T::FS, FV = T::FV;
    constexpr int RPW = T::RPW;
    extern __shared__ __align__(128) float smem[];
    float *sS = smem, *sV = smem + T::V_OFF, *sL = smem + T::L_OFF, *sP = smem + T::P_OFF;
    int *sLoc = reinterpret_cast<int *>(smem + T::LIST_OFF);
    float *sVal = reinterpret_cast<float *>(sLoc + kThreads);
    int *sWarp = reinterpret_cast<int *>(sVal + T::NINJ * kThreads);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + T::BAR_OFF);  // model, sig~, v~
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank(), csize = (int)cluster.num_blocks();

    const int tid = threadIdx.x, lane = tid & 31, ix0 = (tid >> 5) * RPW;
    const int z0 = blockIdx.x * TZ, x0 = blockIdx.y * TX;
    const int nx = a.nx, nz = a.nz, pitch = a.pitch, nshots = a.nshots;
    const int gz = z0 + 2 * lane, col = 2 * lane + 4;  // this lane's columns: gz and gz + 1
    const bool zin0 = gz < nz, zin1 = gz + 1 < nz;
    const float dt = a.dt, cx1 = a.cx1, cx2 = a.cx2, cz1 = a.cz1, cz2 = a.cz2;
    // z masks of the two columns: (D+)^T taps gz-2..gz+1, (D-)^T taps
    // gz-1..gz+2; all ones (and skipped) unless the tile reaches a z edge
    const bool zedge = !(z0 >= 3 && z0 + TZ + 4 <= nz);
    float pz[2][4], mz[2][4];
#pragma unroll
    for (int e = 0; e < 2; e++)
#pragma unroll
        for (int d = 0; d < 4; d++) {
            const int kp = gz + e - 2 + d, km = gz + e - 1 + d;
            pz[e][d] = (kp >= 1 && kp < nz - 2) ? 1.f : 0.f;
            mz[e][d] = (km >= 2 && km < nz - 2) ? 1.f : 0.f;
        }

    auto issue_sig = [&](int shot) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&bar[1], T::sig_bytes);
#pragma unroll
        for (int f = 0; f < T::NS; f++) tma_load_3d(sS + f * FS, &m.sig[f], z0 - 4, x0 - 3, shot, &bar[1]);
    };
    auto issue_vel = [&](int shot) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&bar[2], T::vel_bytes);
#pragma unroll
        for (int q = 0; q < T::NV; q++) tma_load_3d(sV + q * FV, &m.vel[q], z0 - 4, x0 - 1, shot, &bar[2]);
    };
    grid_dep_trigger();
    if (tid == 0) {
#pragma unroll
        for (int b = 0; b < 3; b++) mbar_init(&bar[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    if (tid == 0) {
        // the model tile (no step writes it) streams in while the previous
        // step may still be running
        mbar_expect_tx(&bar[0], T::model_bytes);
#pragma unroll
        for (int f = 0; f < 2; f++) tma_load_2d(sL + f * FS, &m.lm[f], z0 - 4, x0 - 3, &bar[0]);
#pragma unroll
        for (int p = 0; p < 2; p++) tma_load_2d(sP + p * FV, &m.vp[p], z0 - 4, x0 - 1, &bar[0]);
    }
    // the previous step (adjoint state, gradient sums) is complete from here on
    grid_dep_wait();
    if (tid == 0 && crank < nshots) {
        issue_sig(crank);
        issue_vel(crank);
    }

    float2 gk[T::NK][RPW];
#pragma unroll
    for (int k = 0; k < T::NK; k++)
#pragma unroll
        for (int q = 0; q < RPW; q++) gk[k][q] = make_float2(0.f, 0.f);

    // the next shot's injection range and (one per thread) entries, fetched a shot ahead
    int nx_loc = -1, np0 = 0, np1 = 0;
    float nx_val[2];
    auto prefetch_entries = [&](int shot) {
        np0 = a.inj_ptr ? a.inj_ptr[shot] : 0;
        np1 = a.inj_ptr ? a.inj_ptr[shot + 1] : 0;
        if (np1 - np0 <= kThreads) wide_fetch(a, np0, np1, x0, z0, nx_loc, nx_val);
    };
    if (crank < nshots) prefetch_entries(crank);
    int i = 0;
    for (int shot = crank; shot < nshots; shot += csize, i++) {
        const long long soff = (long long)shot * nx * pitch;
        const int p0 = np0, p1 = np1;
        // forward divergence of the interior cells (pointwise, straight from HBM)
        float2 dsv[2][RPW];
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            const int gx = x0 + ix0 + q;
            const bool in = zin0 && gx < nx;
            const long long g = soff + (long long)gx * pitch + gz;
#pragma unroll
            for (int c = 0; c < 2; c++) dsv[c][q] = (in && a.dsf[0]) ? ld2(a.dsf[c] + g) : make_float2(0.f, 0.f);
        }
        const bool single = p1 - p0 <= kThreads;
        int n_in = 0;
        if (single && p1 > p0) n_in = adj_compact<FWI_PSV>(nx_loc, nx_val, sLoc, sVal, sWarp);

        // sig~ of the interior cells into registers (t overwrites it)
        bool ok = mbar_wait(&bar[1], i & 1);
        if (i == 0) ok = mbar_wait(&bar[0], 0) && ok;
        float2 sg[3][RPW];
#pragma unroll
        for (int f = 0; f < 3; f++)
#pragma unroll
            for (int q = 0; q < RPW; q++) sg[f][q] = ld2(sS + f * FS + (ix0 + q + 3) * SZ + col);
        if (__syncthreads_or(!ok)) {  // block-uniform decision
            if (tid == 0) atomicExch(&g_device_status, 1);
            mbar_wait(&bar[1], i & 1);
            mbar_wait(&bar[2], i & 1);
            if (i == 0) mbar_wait(&bar[0], 0);
            break;
        }
        // t = dt S^T sig~ in place over the whole stress region, four cells at a time
        for (int c = tid; c < SX * (SZ / 4); c += kThreads) {
            float4 *s4 = reinterpret_cast<float4 *>(sS) + c;
            const float4 *l4 = reinterpret_cast<const float4 *>(sL) + c;
            constexpr int F4 = FS / 4;
            const float4 l = l4[0], mu = l4[F4];
            float4 xx = s4[0], zz = s4[F4], xz = s4[2 * F4];
            auto t3 = [&](float lc, float mc, float &sxx, float &szz, float &sxz) {
                const float l2m = lc + 2.f * mc, p = sxx, r = szz;
                sxx = dt * (l2m * p + lc * r);
                szz = dt * (lc * p + l2m * r);
                sxz = dt * (mc * sxz);
            };
            t3(l.x, mu.x, xx.x, zz.x, xz.x);
            t3(l.y, mu.y, xx.y, zz.y, xz.y);
            t3(l.z, mu.z, xx.z, zz.z, xz.z);
            t3(l.w, mu.w, xx.w, zz.w, xz.w);
            s4[0] = xx;
            s4[F4] = zz;
            s4[2 * F4] = xz;
        }
        // v~ of this shot; u~ enters v~ (thread 0)
        ok = mbar_wait(&bar[2], i & 1);
        if (single && ok) wide_apply(sV, n_in, sLoc, sVal, dt);
        if (__syncthreads_or(!ok)) {
            if (tid == 0) atomicExch(&g_device_status, 1);
            mbar_wait(&bar[2], i & 1);
            break;
        }
        if (!single) {
            for (int base = p0; base < p1; base += kThreads) {
                __syncthreads();
                int loc;
                float val[2];
                wide_fetch(a, base, p1, x0, z0, loc, val);
                const int n = adj_compact<FWI_PSV>(loc, val, sLoc, sVal, sWarp);
                __syncthreads();
                wide_apply(sV, n, sLoc, sVal, dt);
            }
            __syncthreads();
        }

        // ---- v~' on the warp's interior rows, two columns per lane; t rows
        // x-2 .. x+1 of t0 and t2 (the x-differentiated terms) in a register
        // window, pre-masked (window index r <-> stress row ix0+1+r <-> grid
        // row x0+ix0-2+r)
        auto vel_interior = [&](auto zm) {
            constexpr bool ZM = decltype(zm)::value;  // z masks needed (tile at a z edge)
            float2 w0[RPW + 3], w2[RPW + 3];
#pragma unroll
            for (int r = 0; r < RPW + 3; r++) {
                const int gr = x0 + ix0 - 2 + r;
                const bool on = gr >= 1 && gr < nx - 2;
                w0[r] = on ? ld2(sS + (ix0 + 1 + r) * SZ + col) : make_float2(0.f, 0.f);
                w2[r] = on ? ld2(sS + 2 * FS + (ix0 + 1 + r) * SZ + col) : make_float2(0.f, 0.f);
            }
            // (D+z)^T of t at the two columns from the taps t[-2] .. t[2+1]
            auto dzpT = [&](const float *t, float &d0, float &d1) {
                const float2 A = ld2(t - 2), B = ld2(t), C = ld2(t + 2);
                if constexpr (ZM) {
                    d0 = cz1 * (A.y * pz[0][1] - B.x * pz[0][2]) - cz2 * (A.x * pz[0][0] - B.y * pz[0][3]);
                    d1 = cz1 * (B.x * pz[1][1] - B.y * pz[1][2]) - cz2 * (A.y * pz[1][0] - C.x * pz[1][3]);
                } else {
                    d0 = cz1 * (A.y - B.x) - cz2 * (A.x - B.y);
                    d1 = cz1 * (B.x - B.y) - cz2 * (A.y - C.x);
                }
            };
#pragma unroll
            for (int q = 0; q < RPW; q++) {
                const int ix = ix0 + q, gx = x0 + ix;
                const int vi = (ix + 1) * SZ + col;
                if (!(zin0 && gx < nx)) {
                    st2(sV + vi, 0.f, 0.f);
                    st2(sV + FV + vi, 0.f, 0.f);
                    continue;
                }
                const float *trow = sS + (ix + 3) * SZ + col;
                const float dx0x = cx1 * (w0[q + 1].x - w0[q + 2].x) - cx2 * (w0[q].x - w0[q + 3].x);
                const float dx0y = cx1 * (w0[q + 1].y - w0[q + 2].y) - cx2 * (w0[q].y - w0[q + 3].y);
                const float dx2x = cx1 * (w2[q + 1].x - w2[q + 2].x) - cx2 * (w2[q].x - w2[q + 3].x);
                const float dx2y = cx1 * (w2[q + 1].y - w2[q + 2].y) - cx2 * (w2[q].y - w2[q + 3].y);
                float dz1x, dz1y, dz2x, dz2y;
                dzpT(trow + FS, dz1x, dz1y);
                dzpT(trow + 2 * FS, dz2x, dz2y);
                // a_x = Dx+^T t0 + Dz+^T t2,  a_z = Dx+^T t2 + Dz+^T t1
                const float2 buo = ld2(sP + vi), bnd = ld2(sP + FV + vi);
                const float2 v0 = ld2(sV + vi), v1 = ld2(sV + FV + vi);
                float vxx = bnd.x * (v0.x + (dx0x + dz2x)), vxy = bnd.y * (v0.y + (dx0y + dz2y));
                float vzx = bnd.x * (v1.x + (dx2x + dz1x)), vzy = bnd.y * (v1.y + (dx2y + dz1y));
                if (!zin1) vxy = vzy = 0.f;
                const long long g = soff + (long long)gx * pitch + gz;
                st2(a.vel_out[0] + g, vxx, vxy);
                st2(a.vel_out[1] + g, vzx, vzy);
                st2(sV + vi, buo.x * vxx, buo.y * vxy);
                st2(sV + FV + vi, buo.x * vzx, buo.y * vzy);
                float gbx = 0.f, gby = 0.f;
                gbx += vxx * dsv[0][q].x;
                gbx += vzx * dsv[1][q].x;
                gby += vxy * dsv[0][q].y;
                gby += vzy * dsv[1][q].y;
                gk[2][q].x += gbx;
                if (zin1) gk[2][q].y += gby;
            }
        };
        if (zedge) vel_interior(std::true_type{});
        else vel_interior(std::false_type{});
        // the forward strain of the interior for the stress half: loads in
        // flight during the halo and the barrier
        float2 ef[3][RPW];
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            const int gx = x0 + ix0 + q;
            const bool in = zin0 && gx < nx;
            const long long g = soff + (long long)gx * pitch + gz;
#pragma unroll
            for (int k = 0; k < 3; k++) ef[k][q] = in ? ld2(a.ef[k] + g) : make_float2(0.f, 0.f);
        }
        // ---- v~' on the halo rows x0-1, x0+TX, x0+TX+1 and columns z0-1,
        // z0+TZ, z0+TZ+1 (redundant with the neighbour tiles; masks per tap)
        {
            constexpr int HROW = 3 * RVZ, HC = HROW + 3 * TX;
            auto mxp = [&](int k) -> float { return (k >= 1 && k < nx - 2) ? 1.f : 0.f; };
            auto mzp = [&](int k) -> float { return (k >= 1 && k < nz - 2) ? 1.f : 0.f; };
            for (int c = tid; c < HC; c += kThreads) {
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
                const int hx = x0 - 1 + rx, hz = z0 - 1 + rz;
                const int vi = rx * SZ + rz + 3, si = (rx + 2) * SZ + rz + 3;
                if (hx < 0 || hx >= nx || hz < 0 || hz >= nz) {
                    sV[vi] = 0.f;
                    sV[FV + vi] = 0.f;
                    continue;
                }
                auto dxpT = [&](int f) -> float {
                    const float *t = sS + f * FS + si;
                    return cx1 * (t[-SZ] * mxp(hx - 1) - t[0] * mxp(hx)) -
                           cx2 * (t[-2 * SZ] * mxp(hx - 2) - t[SZ] * mxp(hx + 1));
                };
                auto dzpT1 = [&](int f) -> float {
                    const float *t = sS + f * FS + si;
                    return cz1 * (t[-1] * mzp(hz - 1) - t[0] * mzp(hz)) - cz2 * (t[-2] * mzp(hz - 2) - t[1] * mzp(hz + 1));
                };
                const float acc0 = dxpT(0) + dzpT1(2), acc1 = dxpT(2) + dzpT1(1);
                const float bnd = sP[FV + vi], b = sP[vi];
                sV[vi] = b * (bnd * (sV[vi] + acc0));
                sV[FV + vi] = b * (bnd * (sV[FV + vi] + acc1));
            }
        }
        __syncthreads();
        // t has been consumed: the next shot's sig~ streams in during the stress half
        if (tid == 0 && shot + csize < nshots) issue_sig(shot + csize);
        if (shot + csize < nshots) prefetch_entries(shot + csize);

        // ---- sig~' and the stiffness gradient terms on the interior; b v~'
        // rows x-1 .. x+2 in a register window, pre-masked (window index r
        // <-> velocity row ix0+r <-> grid row x0+ix0-1+r)
        auto stress_interior = [&](auto zm) {
            constexpr bool ZM = decltype(zm)::value;
            float2 w0[RPW + 3], w1[RPW + 3];
#pragma unroll
            for (int r = 0; r < RPW + 3; r++) {
                const int gr = x0 + ix0 - 1 + r;
                const bool on = gr >= 2 && gr < nx - 2;
                w0[r] = on ? ld2(sV + (ix0 + r) * SZ + col) : make_float2(0.f, 0.f);
                w1[r] = on ? ld2(sV + FV + (ix0 + r) * SZ + col) : make_float2(0.f, 0.f);
            }
            // (D-z)^T of b v~' at the two columns from the taps v[-1] .. v[2+1]
            auto dzmT = [&](const float *v, float &d0, float &d1) {
                const float2 A = ld2(v - 2), B = ld2(v), C = ld2(v + 2);
                if constexpr (ZM) {
                    d0 = cz1 * (B.x * mz[0][1] - B.y * mz[0][2]) - cz2 * (A.y * mz[0][0] - C.x * mz[0][3]);
                    d1 = cz1 * (B.y * mz[1][1] - C.x * mz[1][2]) - cz2 * (B.x * mz[1][0] - C.y * mz[1][3]);
                } else {
                    d0 = cz1 * (B.x - B.y) - cz2 * (A.y - C.x);
                    d1 = cz1 * (B.y - C.x) - cz2 * (B.x - C.y);
                }
            };
#pragma unroll
            for (int q = 0; q < RPW; q++) {
                const int ix = ix0 + q, gx = x0 + ix;
                if (!(zin0 && gx < nx)) continue;
                const float *vrow = sV + (ix + 1) * SZ + col;
                const float dx0x = cx1 * (w0[q + 1].x - w0[q + 2].x) - cx2 * (w0[q].x - w0[q + 3].x);
                const float dx0y = cx1 * (w0[q + 1].y - w0[q + 2].y) - cx2 * (w0[q].y - w0[q + 3].y);
                const float dx1x = cx1 * (w1[q + 1].x - w1[q + 2].x) - cx2 * (w1[q].x - w1[q + 3].x);
                const float dx1y = cx1 * (w1[q + 1].y - w1[q + 2].y) - cx2 * (w1[q].y - w1[q + 3].y);
                float dz0x, dz0y, dz1x, dz1y;
                dzmT(vrow, dz0x, dz0y);
                dzmT(vrow + FV, dz1x, dz1y);
                const long long g = soff + (long long)gx * pitch + gz;
                const float2 sxx = sg[0][q], szz = sg[1][q], sxz = sg[2][q];
                float o0y = sxx.y + dx0y, o1y = szz.y + dz1y, o2y = sxz.y + (dz0y + dx1y);
                if (!zin1) o0y = o1y = o2y = 0.f;
                st2(a.sig_out[0] + g, sxx.x + dx0x, o0y);
                st2(a.sig_out[1] + g, szz.x + dz1x, o1y);
                st2(a.sig_out[2] + g, sxz.x + (dz0x + dx1x), o2y);
                const float2 exx = ef[0][q], ezz = ef[1][q], exz = ef[2][q];
                gk[0][q].x += dt * ((sxx.x + szz.x) * (exx.x + ezz.x));
                gk[1][q].x += dt * (2.f * (sxx.x * exx.x + szz.x * ezz.x) + sxz.x * exz.x);
                if (zin1) {
                    gk[0][q].y += dt * ((sxx.y + szz.y) * (exx.y + ezz.y));
                    gk[1][q].y += dt * (2.f * (sxx.y * exx.y + szz.y * ezz.y) + sxz.y * exz.y);
                }
            }
        };
        if (zedge) stress_interior(std::true_type{});
        else stress_interior(std::false_type{});
        __syncthreads();
        // the v~ buffer is free: the next shot streams into it
        if (tid == 0 && shot + csize < nshots) issue_vel(shot + csize);
    }
    if (crank >= nshots) mbar_wait(&bar[0], 0);  // no shot: let the model copies land

    // ---- cluster sum of the gradient terms, in rank order, into FP64
    float *part = smem;
#pragma unroll
    for (int k = 0; k < T::NK; k++)
#pragma unroll
        for (int q = 0; q < RPW; q++) st2(part + k * TX * TZ + (ix0 + q) * TZ + 2 * lane, gk[k][q].x, gk[k][q].y);
    cluster.sync();
    // four cells per thread and pass: their FP64 gradient loads in flight together
    const int chunk = (TX * TZ + csize - 1) / csize, c0 = crank * chunk;
    for (int e0 = tid; e0 < T::NK * chunk; e0 += 4 * kThreads) {
        double kv[4];
        long long gi[4];
        int kk[4], ci[4];
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int e = e0 + u * kThreads;
            kk[u] = -1;
            if (e < T::NK * chunk) {
                const int k = e / chunk, c = c0 + (e - k * chunk);
                const int gx = x0 + c / TZ, gzc = z0 + c % TZ;
                if (c < TX * TZ && a.k[k] && gx < nx && gzc < nz) {
                    kk[u] = k;
                    ci[u] = k * TX * TZ + c;
                    gi[u] = (long long)gx * pitch + gzc;
                }
            }
            kv[u] = kk[u] >= 0 ? a.k[kk[u]][gi[u]] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < 4; u++) {
            if (kk[u] < 0) continue;
            double s = 0.0;
            for (int j = 0; j < csize; j++) s += (double)cluster.map_shared_rank(part, j)[ci[u]];
            a.k[kk[u]][gi[u]] = kv[u] + s;
        }
    }
    cluster.sync();  // keep this CTA's shared memory alive until every rank has read it
}

static int wide_maps(const fwi_batch *b, WideMaps &m) {
    using T = WideTile;
    const int cur = b->cur, nx = b->nx, pitch = b->pitch, ns = b->nshots;
    int rc = 0;
    for (int f = 0; f < 3 && !rc; f++) rc = encode_map(&m.sig[f], b->sig[cur][f], 3, pitch, nx, ns, T::SZ, T::SX);
    for (int q = 0; q < 2 && !rc; q++) rc = encode_map(&m.vel[q], b->vel[cur][q], 3, pitch, nx, ns, T::SZ, T::VX);
    const float *lm[2] = {b->lam, b->mu};
    for (int f = 0; f < 2 && !rc; f++) rc = encode_map(&m.lm[f], lm[f], 2, pitch, nx, 1, T::SZ, T::SX);
    const float *vp[2] = {b->buo, b->bound};
    for (int p = 0; p < 2 && !rc; p++) rc = encode_map(&m.vp[p], vp[p], 2, pitch, nx, 1, T::SZ, T::VX);
    return rc;
}

// Tensor maps of one transposed step.
template <int MODE>
static int adjoint_maps(const fwi_batch *b, const AdjArgs &a, AdjMaps &m) {
    using T = AdjTile<MODE>;
    using F = Fields<MODE>;
    const int cur = b->cur, nx = b->nx, pitch = b->pitch, ns = b->nshots;
    int rc = 0;
    for (int f = 0; f < F::NS && !rc; f++) rc = encode_map(&m.sig[f], b->sig[cur][f], 3, pitch, nx, ns, T::SZ, T::SX);
    for (int q = 0; q < F::NV && !rc; q++) rc = encode_map(&m.vel[q], b->vel[cur][q], 3, pitch, nx, ns, T::SZ, T::VX);
    for (int k = 0; k < T::NE && !rc; k++) rc = encode_map(&m.ef[k], a.ef[k], 3, pitch, nx, ns, T::TZ, T::TX);
    const float *lm[4] = {MODE == FWI_SH ? b->mu : b->lam, b->mu, b->nu, b->mnc};
    for (int f = 0; f < T::NL && !rc; f++) rc = encode_map(&m.lm[f], lm[f], 2, pitch, nx, 1, T::SZ, T::SX);
    const float *vp[3] = {b->buo, b->bound, b->buo_j};
    for (int p = 0; p < T::NP && !rc; p++) rc = encode_map(&m.vp[p], vp[p], 2, pitch, nx, 1, T::SZ, T::VX);
    return rc;
}

// Shots processed side by side per tile (the cluster size, portable limit
// 8): every CTA pays one cluster reduction, so the fewest CTAs that still
// give about 2.5 waves of the resident-CTA slots (measured on 512 x 512 x 32
// shots: 4 beats 2, 8 and 16).
static int adjoint_cluster(int nshots, long long tiles, int ctas_per_sm) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
            sms = 148;
    }
    int c = 8;
    while (c > 1 && tiles * c * 2 > 5ll * sms * ctas_per_sm) c /= 2;
    return c < nshots ? c : nshots;
}

template <int MODE>
static int launch_adjoint(const fwi_batch *b, const AdjArgs &a, cudaStream_t st) {
    using T = AdjTile<MODE>;
    static bool set = false;
    if (!set) {
        cudaError_t e = cudaFuncSetAttribute(adjoint_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)T::bytes);
        if (e != cudaSuccess) return set_error(FWI_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
        set = true;
    }
    AdjMaps m;
    int rc = adjoint_maps<MODE>(b, a, m);
    if (rc) return rc;
    const int C = adjoint_cluster(b->nshots, (long long)((b->nz + T::TZ - 1) / T::TZ) * ((b->nx + T::TX - 1) / T::TX),
                                  MODE == FWI_SH ? 4 : MODE == FWI_PSV ? 3 : 2);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((b->nz + T::TZ - 1) / T::TZ, (b->nx + T::TX - 1) / T::TX, C);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = T::bytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = C;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, adjoint_kernel<MODE>, a, m);
    if (e != cudaSuccess) return set_error(FWI_ECUDA, "adjoint_kernel launch: %s", cudaGetErrorString(e));
    return check_launch("adjoint_kernel");
}

static int launch_adjoint_wide(const fwi_batch *b, const AdjArgs &a, bool pdl, cudaStream_t st) {
    using T = WideTile;
    static bool set = false;
    if (!set) {
        cudaError_t e = cudaFuncSetAttribute(adjoint_wide_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)T::bytes);
        if (e != cudaSuccess) return set_error(FWI_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
        set = true;
    }
    WideMaps m;
    int rc = wide_maps(b, m);
    if (rc) return rc;
    const int tz = (b->nz + T::TZ - 1) / T::TZ, tx = (b->nx + T::TX - 1) / T::TX;
    const int C = adjoint_cluster(b->nshots, (long long)tz * tx, 2);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(tz, tx, C);
    cfg.blockDim = dim3(kThreads, 1, 1);
    cfg.dynamicSmemBytes = T::bytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = 1;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = C;
    set_pdl_attr(attr[1], true);
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 2 : 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, adjoint_wide_kernel, a, m);
    if (e != cudaSuccess) return set_error(FWI_ECUDA, "adjoint_wide_kernel launch: %s", cudaGetErrorString(e));
    return check_launch("adjoint_wide_kernel");
}

// One transposed step (forward step `it`, adjoint state it+1 -> it) with
// its gradient terms.
int launch_adjoint_step(const fwi_batch *b, int it, bool pdl, cudaStream_t st) {
    AdjArgs a;
    a.nx = b->nx;
    a.nz = b->nz;
    a.pitch = b->pitch;
    a.nt = b->nt;
    a.it = it;
    a.nshots = b->nshots;
    a.divnz = make_fastdiv(b->nz);
    a.cx1 = (float)(9.0 / (8.0 * (double)b->dx));
    a.cx2 = (float)(1.0 / (24.0 * (double)b->dx));
    a.cz1 = (float)(9.0 / (8.0 * (double)b->dz));
    a.cz2 = (float)(1.0 / (24.0 * (double)b->dz));
    a.dt = (float)b->dt;
    a.dt2 = (float)(2.0 * b->dt);
    const int mode = b->mode;
    const int nxt = 1 - b->cur, ns = nfields_sig(mode), nv = nfields_vel(mode);
    const int ne = mode == FWI_SH ? 2 : mode == FWI_PSV ? 3 : 6;
    for (int f = 0; f < 6; f++) a.sig_out[f] = f < ns ? b->sig[nxt][f] : nullptr;
    for (int q = 0; q < 3; q++) a.vel_out[q] = q < nv ? b->vel[nxt][q] : nullptr;
    const long long field = (long long)b->nshots * b->nx * b->pitch;
    const long long slot = it - b->seg0;
    for (int k = 0; k < 6; k++) a.ef[k] = k < ne ? b->seg_e[k] + slot * field : nullptr;
    // divergence stores (all components or none: without them the density terms are skipped)
    bool ds = true;
    for (int q = 0; q < nv; q++) ds = ds && b->seg_ds[comp_slot(mode, q)];
    for (int q = 0; q < 3; q++) a.dsf[q] = (ds && q < nv) ? b->seg_ds[comp_slot(mode, q)] + slot * field : nullptr;
    for (int k = 0; k < 6; k++) a.k[k] = nullptr;
    if (mode == FWI_SH) {
        a.k[0] = b->k_mu;
        a.k[1] = b->k_rho;
    } else {
        a.k[0] = b->k_lam;
        a.k[1] = b->k_mu;
        if (mode == FWI_PSV) {
            a.k[2] = b->k_rho;
        } else {
            a.k[2] = b->k_nu;
            a.k[3] = b->k_mnc;
            a.k[4] = b->k_rho;
            a.k[5] = b->k_buoj;
        }
    }
    a.inj_ptr = b->inj_ptr;
    a.inj_cell = b->inj_cell;
    a.inj_row = b->inj_row;
    a.g[0] = mode == FWI_SH ? b->stf[1] : b->stf[0];
    a.g[1] = mode == FWI_SH ? nullptr : b->stf[2];
    switch (mode) {
        case FWI_SH: return launch_adjoint<FWI_SH>(b, a, st);
        case FWI_PSV: return b->adj_tile == 1 ? launch_adjoint<FWI_PSV>(b, a, st) : launch_adjoint_wide(b, a, pdl, st);
        default: return launch_adjoint<FWI_SPIN>(b, a, st);
    }
}

}  // namespace fwi

cudaError_t fwi::step_set_wait_limit(int polls) { return fwi::set_wait_limit_here(polls); }
