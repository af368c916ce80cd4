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
};

template <int MODE, int TX, int TZ>
struct Tile {
    using F = Fields<MODE>;
    // stress region: rows x0-3 .. x0+TX+2 (D- of the velocity halo row
    // x0+TX+1 reaches x0+TX+2), columns z0-4 .. z0+TZ+3
    static constexpr int SX = TX + 6, SZ = TZ + 8;
    static constexpr int VX = TX + 3, RVZ = TZ + 3;  // velocity rows / computed columns
    static constexpr int S_SZ = F::NS * SX * SZ;
    static constexpr int V_SZ = F::NV * VX * SZ;
    static constexpr int P_SZ = F::NVP * VX * SZ;
    static constexpr int U_SZ = F::NV * TX * TZ;
    static constexpr int I_SZ = F::NIP * TX * TZ;
    static constexpr int J_SZ = F::NINJ * VX * RVZ;
    static constexpr int LIST = kThreads * (1 + F::NINJ) + 8;  // compacted injection entries + warp counts
    static constexpr size_t bytes = sizeof(float) * (size_t)(S_SZ + V_SZ + P_SZ + U_SZ + I_SZ + J_SZ + LIST);
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

// Stage NF fields of a ROWS x COLS window starting at (gx0, gz0) into dst.
template <int NF, int ROWS, int COLS>
__device__ __forceinline__ void stage(float *dst, const float *const *src, long long off, int gx0, int gz0,
                                      int nx, int pitch, int tid) {
    constexpr int C4 = COLS / 4;
    constexpr int PER = ROWS * C4;
#pragma unroll
    for (int f = 0; f < NF; f++) {
        const float *base = src[f] + off;
        for (int q = tid; q < PER; q += kThreads) {
            int r = q / C4, c = q - r * C4;
            int gx = gx0 + r, gz = gz0 + 4 * c;
            bool ok = gx >= 0 && gx < nx && gz >= 0 && gz < pitch;
            const float *g = ok ? base + (long long)gx * pitch + gz : base;
            cp_async16(dst + f * ROWS * COLS + r * COLS + 4 * c, g, ok ? 16 : 0);
        }
    }
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
    stage<F::NS, SX, SZ>(sm.S, a.sig_in, soff, x0 - 3, z0 - 4, nx, pitch, tid);
    stage<F::NV, VX, SZ>(sm.V, a.vel_in, soff, x0 - 1, z0 - 4, nx, pitch, tid);
    stage<F::NVP, VX, SZ>(sm.P, a.vp, 0, x0 - 1, z0 - 4, nx, pitch, tid);
    stage<F::NV, TX, TZ>(sm.U, a.disp, soff, x0, z0, nx, pitch, tid);
    stage<F::NIP, TX, TZ>(sm.I, a.ip, 0, x0, z0, nx, pitch, tid);
    cp_async_commit();

    bool has_inj = false;
    if (a.inj_ptr) {
        const int p0 = a.inj_ptr[shot], p1 = a.inj_ptr[shot + 1];
        for (int base = p0; base < p1; base += kThreads) {
            const int e = base + tid;
            int loc = -1;
            float val[F::NINJ];
            if (e < p1) {
                const int k = a.inj_cell[e];
                const int gx = fdiv(k, a.divnz), gz = k - gx * nz;
                const int rx = gx - (x0 - 1), rz = gz - (z0 - 1);
                if (rx >= 0 && rx < VX && rz >= 0 && rz < RVZ) {
                    loc = rx * RVZ + rz;
                    const long long src = (long long)a.inj_row[e] * a.nt + a.it;
#pragma unroll
                    for (int c = 0; c < F::NINJ; c++) val[c] = a.stf[c][src];
                }
            }
            const int n_in = __syncthreads_count(loc >= 0);
            if (n_in == 0) continue;
            if (!has_inj) {
                for (int q = tid; q < T::J_SZ; q += kThreads) sm.J[q] = 0.f;
                has_inj = true;
            }
            const unsigned ball = __ballot_sync(0xffffffffu, loc >= 0);
            if (lane == 0) sm.warp[warp] = __popc(ball);
            __syncthreads();
            if (loc >= 0) {
                int pos = __popc(ball & ((1u << lane) - 1u));
                for (int w = 0; w < warp; w++) pos += sm.warp[w];
                sm.loc[pos] = loc;
#pragma unroll
                for (int c = 0; c < F::NINJ; c++) sm.val[c * kThreads + pos] = val[c];
            }
            __syncthreads();
            if (tid == 0) {
                for (int q = 0; q < n_in; q++) {
#pragma unroll
                    for (int c = 0; c < F::NINJ; c++) sm.J[c * VX * RVZ + sm.loc[q]] += sm.val[c * kThreads + q];
                }
            }
            __syncthreads();
        }
    }
    cp_async_wait_all();
    __syncthreads();
    return has_inj;
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
    const float buo = sm.P[vi], bnd = sm.P[VX * SZ + vi];
#pragma unroll
    for (int c = 0; c < F::NV; c++) {
        const float b = (MODE == FWI_SPIN && c == 2) ? sm.P[2 * VX * SZ + vi] : buo;
        const float v = bnd * (sm.V[c * VX * SZ + vi] + ds[c] * b);
        sm.V[c * VX * SZ + vi] = v;
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
    constexpr int FS = T::SX * T::SZ, FI = TX * TZ;
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
                                               const float (&v)[3]) {
#pragma unroll
    for (int q = 0; q < Fields<MODE>::NV; q++) {
        const float u = sm.U[q * TX * TZ + ci] + v[q] * a.dt;
        sm.U[q * TX * TZ + ci] = u;
        a.vel_out[q][g] = v[q];
        a.disp[q][g] = u;
        if (a.snap_u[q]) a.snap_u[q][g] = u;
        if (a.snap_v[q]) a.snap_v[q][g] = v[q];
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
                                              int rz, bool has_inj, float (&v)[3]) {
    using T = Tile<MODE, TX, TZ>;
    constexpr int SX = T::SX, SZ = T::SZ, VX = T::VX;
    const int gx = x0 - 1 + rx, gz = z0 - 1 + rz;
    const int cz = rz + 3;
    if (gx < 0 || gx >= a.nx || gz < 0 || gz >= a.nz) {
#pragma unroll
        for (int c = 0; c < Fields<MODE>::NV; c++) sm.V[c * VX * SZ + rx * SZ + cz] = 0.f;
        return false;
    }
    const bool okx = gx >= 2 && gx < a.nx - 2, okz = gz >= 2 && gz < a.nz - 2;
    const float *s0 = sm.S + (rx + 2) * SZ + cz;
    const float cx1 = a.cx1, cx2 = a.cx2, cz1 = a.cz1, cz2 = a.cz2;
    auto dxm = [&](int f) -> float {
        if (!okx) return 0.f;
        const float *s = s0 + f * SX * SZ;
        return cx1 * (s[0] - s[-SZ]) - cx2 * (s[SZ] - s[-2 * SZ]);
    };
    auto dzm = [&](int f) -> float {
        if (!okz) return 0.f;
        const float *s = s0 + f * SX * SZ;
        return cz1 * (s[0] - s[-1]) - cz2 * (s[1] - s[-2]);
    };
    auto center = [&](int f) -> float { return s0[f * SX * SZ]; };
    float ds[3];
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
        float v[3];
        velocity_cell<MODE, TX, TZ>(a, sm, x0, z0, rx, rz, has_inj, v);
    }
}

// ------------------------------------------------------- generic mapping

template <int MODE, int TX, int TZ>
__global__ void __launch_bounds__(kThreads, MODE == FWI_SPIN ? 1 : 2) step_kernel(const StepArgs a) {
    using T = Tile<MODE, TX, TZ>;
    constexpr int SX = T::SX, SZ = T::SZ, VX = T::VX;
    extern __shared__ __align__(16) float smem[];
    const Smem<MODE, TX, TZ> sm(smem);
    const int z0 = blockIdx.x * TZ, x0 = blockIdx.y * TX, shot = blockIdx.z;
    const int nx = a.nx, nz = a.nz, pitch = a.pitch;
    const long long soff = (long long)shot * nx * pitch;
    const bool has_inj = prologue<MODE, TX, TZ>(a, sm, x0, z0, shot);

    for (int c = threadIdx.x; c < TX * TZ; c += kThreads) {
        const int ix = c / TZ, iz = c - ix * TZ;
        float v[3];
        if (velocity_cell<MODE, TX, TZ>(a, sm, x0, z0, ix + 1, iz + 1, has_inj, v))
            store_interior<MODE, TX, TZ>(a, sm, c, soff + (long long)(x0 + ix) * pitch + (z0 + iz), v);
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
            const float *v = v0 + f * VX * SZ;
            return cx1 * (v[SZ] - v[0]) - cx2 * (v[2 * SZ] - v[-SZ]);
        };
        auto dzp = [&](int f) -> float {
            if (!okz) return 0.f;
            const float *v = v0 + f * VX * SZ;
            return cz1 * (v[1] - v[0]) - cz2 * (v[2] - v[-1]);
        };
        const float vyc = MODE == FWI_SPIN ? v0[2 * VX * SZ] : 0.f;
        stress_update<MODE, TX, TZ>(a, sm.S + (ix + 3) * SZ + (iz + 4), sm.I + c, vyc,
                                    soff + (long long)gx * pitch + gz, dxp, dzp);
    }
    (void)SX;
}

// -------------------------------------------------- register-window mapping

template <int MODE, int TX>
__global__ void __launch_bounds__(kThreads, MODE == FWI_SPIN ? 1 : 3) step_kernel_rw(const StepArgs a) {
    constexpr int TZ = 32, RPW = TX / (kThreads / 32);
    static_assert(RPW >= 1 && RPW * (kThreads / 32) == TX, "TX must be a multiple of the warp count");
    using T = Tile<MODE, TX, TZ>;
    using F = Fields<MODE>;
    constexpr int SX = T::SX, SZ = T::SZ, VX = T::VX;
    extern __shared__ __align__(16) float smem[];
    const Smem<MODE, TX, TZ> sm(smem);
    const int z0 = blockIdx.x * TZ, x0 = blockIdx.y * TX, shot = blockIdx.z;
    const int nx = a.nx, nz = a.nz, pitch = a.pitch;
    const long long soff = (long long)shot * nx * pitch;
    const bool has_inj = prologue<MODE, TX, TZ>(a, sm, x0, z0, shot);

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
                for (int r = 0; r < RPW + 3; r++) w[f][r] = sm.S[f * SX * SZ + (ix0 + 1 + r) * SZ + col];
            }
#pragma unroll
        for (int q = 0; q < RPW; q++) {
            const int ix = ix0 + q, gx = x0 + ix;
            const int vi = (ix + 1) * SZ + col;
            if (!(zin && gx < nx)) {
#pragma unroll
                for (int c = 0; c < F::NV; c++) sm.V[c * VX * SZ + vi] = 0.f;
                continue;
            }
            const bool okx = gx >= 2 && gx < nx - 2;
            const float *srow = sm.S + (ix + 3) * SZ + col;
            auto dxm = [&](int f) -> float {
                return okx ? cx1 * (w[f][q + 2] - w[f][q + 1]) - cx2 * (w[f][q + 3] - w[f][q]) : 0.f;
            };
            auto center = [&](int f) -> float { return takes_dxm(MODE, f) ? w[f][q + 2] : srow[f * SX * SZ]; };
            auto dzm = [&](int f) -> float {
                if (!okz) return 0.f;
                const float *s = srow + f * SX * SZ;
                return cz1 * (center(f) - s[-1]) - cz2 * (s[1] - s[-2]);
            };
            float ds[3], v[3];
            divergence<MODE>(dxm, dzm, center, ds);
            velocity_update<MODE, TX, TZ>(sm, ix + 1, lane + 1, ds, has_inj, v);
            store_interior<MODE, TX, TZ>(a, sm, ix * TZ + lane, soff + (long long)gx * pitch + gz, v);
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
            for (int r = 0; r < RPW + 3; r++) w[f][r] = sm.V[f * VX * SZ + (ix0 + r) * SZ + col];
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
                const float *v = vrow + f * VX * SZ;
                return cz1 * (v[1] - w[f][q + 1]) - cz2 * (v[2] - v[-1]);
            };
            const float vyc = MODE == FWI_SPIN ? w[F::NV - 1][q + 1] : 0.f;
            stress_update<MODE, TX, TZ>(a, sm.S + (ix + 3) * SZ + col, sm.I + ix * TZ + lane, vyc,
                                        soff + (long long)gx * pitch + gz, dxp, dzp);
        }
    }
}

// ------------------------------------------------------------- launching

struct TileShape {
    int tx, tz, rw;
};
// Variants selectable through fwi_batch.tile; 0 is the default.
static const TileShape kTiles[] = {{32, 32, 1}, {32, 32, 0}, {16, 64, 0}, {16, 32, 0}, {64, 32, 0},
                                   {8, 64, 0},  {32, 32, 1}, {16, 32, 1}, {64, 32, 1}};
constexpr int kNumTiles = sizeof(kTiles) / sizeof(kTiles[0]);

template <int MODE, int TX, int TZ, bool RW>
static int launch_tile(const StepArgs &a, int nshots, cudaStream_t st) {
    using T = Tile<MODE, TX, TZ>;
    void (*kern)(const StepArgs);
    if constexpr (RW) {
        static_assert(TZ == 32, "the register-window mapping has one lane per z column");
        kern = step_kernel_rw<MODE, TX>;
    } else {
        kern = step_kernel<MODE, TX, TZ>;
    }
    static bool attr_set = false;
    if (!attr_set) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::bytes);
        if (e != cudaSuccess) return set_error(FWI_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
        attr_set = true;
    }
    dim3 grid((a.nz + TZ - 1) / TZ, (a.nx + TX - 1) / TX, nshots);
    kern<<<grid, kThreads, T::bytes, st>>>(a);
    return check_launch("step_kernel");
}

template <int MODE>
static int launch_mode(const StepArgs &a, int nshots, int tile, cudaStream_t st) {
    switch (tile) {
        case 0: return launch_tile<MODE, 32, 32, true>(a, nshots, st);
        case 1: return launch_tile<MODE, 32, 32, false>(a, nshots, st);
        case 2: return launch_tile<MODE, 16, 64, false>(a, nshots, st);
        case 3: return launch_tile<MODE, 16, 32, false>(a, nshots, st);
        case 4: return launch_tile<MODE, 64, 32, false>(a, nshots, st);
        case 5: return launch_tile<MODE, 8, 64, false>(a, nshots, st);
        case 6: return launch_tile<MODE, 32, 32, true>(a, nshots, st);
        case 7: return launch_tile<MODE, 16, 32, true>(a, nshots, st);
        case 8: return launch_tile<MODE, 64, 32, true>(a, nshots, st);
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

}  // namespace fwi
