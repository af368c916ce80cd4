// Row-marching forward step for displacement-free SH and P-SV batches.
//
// Same arithmetic per cell as the tiled step kernels of step.cu (and so as
// the reference's div_sy / div_sxz, stf_dsy / stf_dsxz, add_vy / add_vxz,
// div_vy / div_vxz, add_sy / add_sxz and save_obs, solver.py:54-156), with a
// layout that keeps the instruction count per cell low enough for the step to
// be bound by HBM rather than by issue:
//
//   * A CTA spans the whole z extent of the grid (thread j = column j, up to
//     1024 columns) and marches down a contiguous range of x rows of one
//     shot.  The 4th-order x derivatives come from register windows of four
//     rows, the z derivatives from the neighbouring columns of the current
//     row in shared memory, so every value is loaded from shared memory once
//     per row and there is no 2-D index arithmetic per cell.
//   * Rows of the state (stress, velocity) stream into a ring of row slots in
//     shared memory with untiled bulk copies (cp.async.bulk, one per field
//     and row, completion on an mbarrier per slot, bounded waits), issued by
//     one thread several rows ahead of the march.  The model, shared by the
//     shots and resident in L2, is read with ordinary loads one row ahead.
//   * The new velocity of row r goes to a four-row ring in shared memory;
//     the stress of row r-2 is updated in the same iteration from the
//     velocity window (D+x) and that ring (D+z).  One block barrier per row.
//   * The rows of all shots form one sequence, split evenly over a grid of
//     resident CTAs (one pass, no tail wave); a CTA whose range starts in
//     the middle of a shot recomputes the velocity of the row above its range
//     and of the two below it (the D+x stencil needs them).
//   * No displacement field: the displacement only feeds the receivers, so
//     the kernel records the new velocity at the receivers and
//     displacement_traces_kernel turns each trace into the running sum
//     u(it) = u(it-1) + v(it) dt afterwards -- the same float operations in
//     the same order as the displacement update of add_vy / add_vxz
//     (solver.py:95-109), so the traces are bit-identical.
//   * Sources and receivers are visited in cell order: the injection entries
//     of a shot must be sorted by cell (entries at one cell keep their order,
//     so the per-cell sums are unchanged) and rec_order lists the receivers
//     by cell.  Each CTA stages the points of its rows in shared-memory
//     windows and walks them with the march.
#include <cstdio>

#include "common.cuh"
#include "stencil.cuh"

namespace fwi {

// Status word of the row-marching kernels (a bounded wait gave up).
__device__ int g_march_status = 0;

int march_device_status(int clear, int *status) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_march_status, sizeof(int)) != cudaSuccess)
        return set_error(FWI_ECUDA, "fwi_device_status: reading the row-marching kernels' status failed");
    if (clear && v) {
        const int z = 0;
        if (cudaMemcpyToSymbol(g_march_status, &z, sizeof(int)) != cudaSuccess)
            return set_error(FWI_ECUDA, "fwi_device_status: clearing the row-marching kernels' status failed");
    }
    *status = v;
    return 0;
}

constexpr int kPts = 256;       // points (injection entries, receivers) staged per window
constexpr int kMaxCols = 1024;  // z extent a CTA can span (one thread per column)

struct MarchArgs {
    int nx, nz, pitch, nt, it, nrec;
    int rl, nslots;         // shared-memory row length (floats) and ring depth
    long long rows_total;   // nshots * nx
    float cx1, cx2, cz1, cz2, dt;
    const float *sig_in[3];
    float *sig_out[3];
    const float *vel_in[2];
    float *vel_out[2];
    const float *buo, *bound;
    const float *ip[2];     // SH: mu | P-SV: lam, mu
    const int *inj_ptr, *inj_cell, *inj_row;
    const float *stf[2];    // injected components in slot order
    const int *rec_cell, *rec_order;
    float *obs[2];          // per velocity component, NULL skips
    float *seg_e[3];        // per-step strain store of this step (slot-offset), or NULL
    float *seg_ds[2];       // per-step divergence store, or NULL
};

// Shared-memory layout, in floats: ring [nslots][NF][rl], velocity ring
// [4][NV][rl], injection window (cells, NINJ value rows), receiver window
// (cells, ids), two cursors, then the mbarriers (8-byte aligned).
struct MarchLayout {
    int vring, icell, ival, rcell, rid, cur, bar;
    size_t bytes;
};

__host__ __device__ inline MarchLayout march_layout(int nf, int nv, int ninj, int rl, int nslots) {
    MarchLayout L;
    L.vring = nslots * nf * rl;
    L.icell = L.vring + 4 * nv * rl;
    L.ival = L.icell + kPts;
    L.rcell = L.ival + ninj * kPts;
    L.rid = L.rcell + kPts;
    L.cur = L.rid + kPts;  // two cursors (8 ints)
    L.bar = (L.cur + 8 + 1) / 2 * 2;
    L.bytes = sizeof(float) * (size_t)L.bar + 8 * (size_t)nslots;
    return L;
}

// First index in [lo, hi) whose key is >= v (keys non-decreasing);
// key(i) = cell[perm ? perm[i] : i].
__device__ __forceinline__ int lower_bound_cells(const int *cell, const int *perm, int lo, int hi, int v) {
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const int c = cell[perm ? perm[mid] : mid];
        if (c < v) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// A window of consecutive points [w0, w0+wn) of the range [p, end) staged in
// shared memory; p is the next point to visit.  Kept in shared memory; the
// march holds only the cell of the next point in a register and reads the
// cursor on the rows that have points.  Every thread sees the same values,
// so branches on them are block-uniform.
struct Cursor {
    int p, end, w0, wn;
};
constexpr int kNone = 0x7fffffff;  // "no further point"

template <int MODE>
__global__ void __launch_bounds__(kMaxCols) march_kernel(const __grid_constant__ MarchArgs a) {
    using F = Fields<MODE>;
    constexpr int NS = F::NS, NV = F::NV, NF = NS + NV, NINJ = F::NINJ;
    extern __shared__ __align__(128) float smem[];
    const int RL = a.rl, N = a.nslots;
    const MarchLayout L = march_layout(NF, NV, NINJ, RL, N);
    int *const i_cell = reinterpret_cast<int *>(smem + L.icell);
    float *const i_val = smem + L.ival;
    int *const r_cell = reinterpret_cast<int *>(smem + L.rcell);
    int *const r_id = reinterpret_cast<int *>(smem + L.rid);
    Cursor *const cur_s = reinterpret_cast<Cursor *>(smem + L.cur);  // [0] injection, [1] receivers
    uint64_t *const full = reinterpret_cast<uint64_t *>(smem + L.bar);

    const int tid = threadIdx.x, j = tid;
    const int nx = a.nx, nz = a.nz, pitch = a.pitch, nt = a.nt, it = a.it;
    const bool jin = j < nz;
    const float cx1 = a.cx1, cx2 = a.cx2, cz1 = a.cz1, cz2 = a.cz2, dt = a.dt;
    const uint32_t row_bytes = 4u * (uint32_t)pitch;
    // row buffers start 4 floats into their slot so that columns -4 .. rl-5 are addressable
    auto ring_row = [&](int slot, int f) -> float * { return smem + (slot * NF + f) * RL + 4; };
    auto vel_row = [&](int k, int c) -> float * { return smem + L.vring + (k * NV + c) * RL + 4; };

    if (tid == 0) {
        for (int i = 0; i < N; i++) mbar_init(&full[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();

    // thread 0: stream row q of the shot at soff into the slot of sequence number sn
    auto issue = [&](long long soff, int q, int sn) {
        const int slot = sn % N;
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(&full[slot], NF * row_bytes);
        const long long o = soff + (long long)q * pitch;
#pragma unroll
        for (int f = 0; f < NS; f++) bulk_load(ring_row(slot, f), a.sig_in[f] + o, row_bytes, &full[slot]);
#pragma unroll
        for (int c = 0; c < NV; c++) bulk_load(ring_row(slot, NS + c), a.vel_in[c] + o, row_bytes, &full[slot]);
    };
    auto wait_seq = [&](int sn) -> bool { return mbar_wait(&full[sn % N], (uint32_t)((sn / N) & 1)); };

    const bool rec_on = a.rec_order && a.nrec > 0 && (a.obs[0] || (NV > 1 && a.obs[1]));
    const bool inj_on = a.inj_ptr != nullptr;
    const int R = (int)a.rows_total, G = gridDim.x;
    int Lrow = (int)((long long)R * blockIdx.x / G);
    const int Lend = (int)((long long)R * (blockIdx.x + 1) / G);
    int seq = 0;  // ring sequence number of the next row to issue (same in every thread)

    // stage the window of points starting at c.p (block-wide: every thread
    // calls it with the same cursor, which it updates in place)
    auto load_inj = [&](Cursor &c) {
        __syncthreads();
        const int n = min(kPts, c.end - c.p);
        for (int k = tid; k < n; k += blockDim.x) {
            const int e = c.p + k;
            i_cell[k] = a.inj_cell[e];
            const long long src = (long long)a.inj_row[e] * nt + it;
#pragma unroll
            for (int q = 0; q < NINJ; q++) i_val[q * kPts + k] = a.stf[q][src];
        }
        c.w0 = c.p;
        c.wn = n;
        __syncthreads();
    };
    auto load_rec = [&](Cursor &c) {
        __syncthreads();
        const int n = min(kPts, c.end - c.p);
        for (int k = tid; k < n; k += blockDim.x) {
            const int r = a.rec_order[c.p + k];
            r_id[k] = r;
            r_cell[k] = a.rec_cell[r];
        }
        c.w0 = c.p;
        c.wn = n;
        __syncthreads();
    };
    // after the points of a row: store the cursor back (block-wide) and
    // return the cell of the next point, or kNone
    auto park = [&](Cursor &c, int which, bool inj) -> int {
        if (c.p < c.end && c.p - c.w0 >= c.wn) {
            if (inj) load_inj(c);
            else load_rec(c);
        }
        const int nxt = c.p < c.end ? (inj ? i_cell : r_cell)[c.p - c.w0] : kNone;
        __syncthreads();
        if (tid == 0) cur_s[which] = c;
        __syncthreads();
        return nxt;
    };

    while (Lrow < Lend) {
        const int shot = Lrow / nx, a0 = Lrow - shot * nx;
        const int b0 = min(nx, a0 + (Lend - Lrow));
        Lrow += b0 - a0;
        const long long soff = (long long)shot * nx * pitch;
        const int va = max(a0 - 1, 0), vb = min(b0 + 2, nx);  // velocity rows computed
        const int qa = max(va - 2, 0), qb = min(vb + 1, nx);  // rows streamed through the ring
        const int sb = seq - qa;                               // ring sequence number of row q: sb + q
        seq += qb - qa;
        int nexti = min(qa + N, qb);
        if (tid == 0) {
            for (int q = qa; q < nexti; q++) issue(soff, q, sb + q);
            int p0 = 0, p1 = 0;
            if (inj_on) {
                p0 = a.inj_ptr[shot];
                p1 = a.inj_ptr[shot + 1];
            }
            const int i0 = inj_on ? lower_bound_cells(a.inj_cell, nullptr, p0, p1, va * nz) : 0;
            const int i1 = inj_on ? lower_bound_cells(a.inj_cell, nullptr, p0, p1, vb * nz) : 0;
            const int r0 = rec_on ? lower_bound_cells(a.rec_cell, a.rec_order, 0, a.nrec, a0 * nz) : 0;
            const int r1 = rec_on ? lower_bound_cells(a.rec_cell, a.rec_order, 0, a.nrec, b0 * nz) : 0;
            cur_s[0] = Cursor{i0, i1, i0, 0};
            cur_s[1] = Cursor{r0, r1, r0, 0};
        }
        __syncthreads();
        int inj_next, rec_next;  // cell of the next injection entry / receiver, or kNone
        {
            Cursor c = cur_s[0];
            inj_next = c.p < c.end ? park(c, 0, true) : kNone;
            c = cur_s[1];
            rec_next = c.p < c.end ? park(c, 1, false) : kNone;
        }

        bool ok = true;
        // register windows: stress rows r-2 .. r+1 (SH: sxy, szy; P-SV: sxx, szz, sxz),
        // new velocity rows r-3 .. r
        float ws[NS][4], wv[NV][4];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int q = va - 2 + k;
            if (q >= qa) {
                ok = wait_seq(sb + q) && ok;
                const int sl = (sb + q) % N;
#pragma unroll
                for (int f = 0; f < NS; f++) ws[f][k] = ring_row(sl, f)[j];
            } else {
#pragma unroll
                for (int f = 0; f < NS; f++) ws[f][k] = 0.f;
            }
        }
#pragma unroll
        for (int c = 0; c < NV; c++)
#pragma unroll
            for (int k = 0; k < 4; k++) wv[c][k] = 0.f;
        // model of the first row: dt/rho and sponge (row va), stiffness (row va-2)
        auto ld_model = [&](const float *p, int row) -> float {
            return (jin && row >= 0 && row < nx) ? __ldg(p + (long long)row * pitch + j) : 0.f;
        };
        float buo = ld_model(a.buo, va), bnd = ld_model(a.bound, va);
        float ip0 = ld_model(a.ip[0], va - 2), ip1 = MODE == FWI_PSV ? ld_model(a.ip[1], va - 2) : 0.f;
        if (__syncthreads_or(!ok)) goto bail;
        // rows above va are consumed: their slots take the next rows
        for (int q = qa; q < va; q++)
            if (nexti < qb) {
                if (tid == 0) issue(soff, nexti, sb + nexti);
                nexti++;
            }

        for (int r = va; r < b0 + 2; r++) {
            // next iteration's model values (one row ahead)
            const float buo_n = ld_model(a.buo, r + 1), bnd_n = ld_model(a.bound, r + 1);
            const float ip0_n = ld_model(a.ip[0], r - 1);
            const float ip1_n = MODE == FWI_PSV ? ld_model(a.ip[1], r - 1) : 0.f;
            float vn[NV];
            if (r < vb) {
                // ---- velocity of row r
                if (r + 1 < qb) {
                    ok = wait_seq(sb + r + 1) && ok;
                    const int sl = (sb + r + 1) % N;
#pragma unroll
                    for (int f = 0; f < NS; f++) ws[f][3] = ring_row(sl, f)[j];
                } else {
#pragma unroll
                    for (int f = 0; f < NS; f++) ws[f][3] = 0.f;
                }
                const int sr = (sb + r) % N;
                const bool okx = r >= 2 && r < nx - 2, okz = j >= 2 && j < nz - 2;
                auto dxm = [&](int f) -> float {
                    return okx ? cx1 * (ws[f][2] - ws[f][1]) - cx2 * (ws[f][3] - ws[f][0]) : 0.f;
                };
                auto dzm = [&](int f) -> float {
                    const float *s = ring_row(sr, f) + j;
                    return okz ? cz1 * (ws[f][2] - s[-1]) - cz2 * (s[1] - s[-2]) : 0.f;
                };
                float ds[NV];
                if constexpr (MODE == FWI_SH) {
                    ds[0] = dxm(0) + dzm(1);
                } else {
                    ds[0] = dxm(0) + dzm(2);
                    ds[1] = dxm(2) + dzm(1);
                }
                // sources of row r, summed per cell in entry order (stf_dsy / stf_dsxz, solver.py:78-93)
                if (inj_next < (r + 1) * nz) {
                    const int lo = r * nz, hi = lo + nz;
                    float acc[NINJ];
#pragma unroll
                    for (int q = 0; q < NINJ; q++) acc[q] = 0.f;
                    Cursor c = cur_s[0];
                    while (c.p < c.end) {
                        if (c.p - c.w0 >= c.wn) load_inj(c);
                        const int k = c.p - c.w0, cell = i_cell[k];
                        if (cell >= hi) break;
                        if (cell - lo == j) {
#pragma unroll
                            for (int q = 0; q < NINJ; q++) acc[q] += i_val[q * kPts + k];
                        }
                        c.p++;
                    }
                    inj_next = park(c, 0, true);
#pragma unroll
                    for (int q = 0; q < NV; q++) ds[q] += acc[q];
                }
                const long long g = soff + (long long)r * pitch + j;
                const bool own = r >= a0 && r < b0 && jin;
#pragma unroll
                for (int c = 0; c < NV; c++) {
                    const float vold = ring_row(sr, NS + c)[j];
                    vn[c] = bnd * (vold + ds[c] * buo);
                    vel_row(r & 3, c)[j] = vn[c];
                    if (own) {
                        a.vel_out[c][g] = vn[c];
                        if (a.seg_ds[c]) a.seg_ds[c][g] = ds[c];
                    }
                }
                // receivers of row r record the new velocity (save_obs, solver.py:151-156)
                if (rec_next < (r + 1) * nz) {
                    const int lo = r * nz, hi = lo + nz;
                    Cursor c = cur_s[1];
                    while (c.p < c.end) {
                        if (c.p - c.w0 >= c.wn) load_rec(c);
                        const int k = c.p - c.w0, cell = r_cell[k];
                        if (cell >= hi) break;
                        if (cell - lo == j) {
                            const long long o = ((long long)shot * a.nrec + r_id[k]) * nt + it;
#pragma unroll
                            for (int q = 0; q < NV; q++)
                                if (a.obs[q]) a.obs[q][o] = vn[q];
                        }
                        c.p++;
                    }
                    rec_next = park(c, 1, false);
                }
            } else {
#pragma unroll
                for (int c = 0; c < NV; c++) {
                    vn[c] = 0.f;
                    vel_row(r & 3, c)[j] = 0.f;
                }
            }
#pragma unroll
            for (int c = 0; c < NV; c++) {
                wv[c][0] = wv[c][1];
                wv[c][1] = wv[c][2];
                wv[c][2] = wv[c][3];
                wv[c][3] = vn[c];
            }
            if (__syncthreads_or(!ok)) goto bail;
            // row r is consumed: its slot takes row r + nslots
            if (nexti < qb) {
                if (tid == 0) issue(soff, nexti, sb + nexti);
                nexti++;
            }

            // ---- stress of row s = r - 2 (add_sy / add_sxz, solver.py:128-149)
            const int s = r - 2;
            if (s >= a0 && s < b0 && jin) {
                const bool okx = s >= 1 && s < nx - 2, okz = j >= 1 && j < nz - 2;
                auto dxp = [&](int c) -> float {
                    return okx ? cx1 * (wv[c][2] - wv[c][1]) - cx2 * (wv[c][3] - wv[c][0]) : 0.f;
                };
                auto dzp = [&](int c) -> float {
                    const float *v = vel_row(s & 3, c) + j;
                    return okz ? cz1 * (v[1] - wv[c][1]) - cz2 * (v[2] - v[-1]) : 0.f;
                };
                const long long g = soff + (long long)s * pitch + j;
                if constexpr (MODE == FWI_SH) {
                    const float dm = dt * ip0, exy = dxp(0), ezy = dzp(0);
                    a.sig_out[0][g] = ws[0][0] + dm * exy;
                    a.sig_out[1][g] = ws[1][0] + dm * ezy;
                    if (a.seg_e[0]) {
                        a.seg_e[0][g] = exy;
                        a.seg_e[1][g] = ezy;
                    }
                } else {
                    const float lam = ip0, mu = ip1;
                    const float vxx = dxp(0), vxz = dzp(0), vzx = dxp(1), vzz = dzp(1);
                    const float l2m = lam + 2.f * mu, shear = vxz + vzx;
                    a.sig_out[0][g] = ws[0][0] + dt * (l2m * vxx + lam * vzz);
                    a.sig_out[1][g] = ws[1][0] + dt * (l2m * vzz + lam * vxx);
                    a.sig_out[2][g] = ws[2][0] + dt * (mu * shear);
                    if (a.seg_e[0]) {
                        a.seg_e[0][g] = vxx;
                        a.seg_e[1][g] = vzz;
                        a.seg_e[2][g] = shear;
                    }
                }
            }
#pragma unroll
            for (int f = 0; f < NS; f++) {
                ws[f][0] = ws[f][1];
                ws[f][1] = ws[f][2];
                ws[f][2] = ws[f][3];
            }
            buo = buo_n;
            bnd = bnd_n;
            ip0 = ip0_n;
            ip1 = ip1_n;
        }
        continue;
    bail:
        // a wait gave up: let the copies still in flight land, then stop
        if (tid == 0) atomicExch(&g_march_status, 1);
        for (int q = max(qa, nexti - N); q < nexti; q++) wait_seq(sb + q);
        return;
    }
}

// Displacement traces from velocity traces: u(it) = u(it-1) + v(it) dt over
// steps [it0, it0+n) of every trace ([trace][nt]), u(it0-1) being the
// trace's value before it0 (0 at it0 = 0) -- the displacement update of
// add_vy / add_vxz (solver.py:95-109) in the same float operations.
__global__ void displacement_traces_kernel(float *obs, long long ntr, int nt, int it0, int n, float dt) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntr) return;
    float *p = obs + t * nt;
    float u = it0 > 0 ? p[it0 - 1] : 0.f;
    for (int i = it0; i < it0 + n; i++) {
        u = u + p[i] * dt;
        p[i] = u;
    }
}

// ------------------------------------------------------------- host side

static int comp_slot_of(int mode, int q) { return mode == FWI_SH ? 1 : (q == 0 ? 0 : 2); }

// Ring depth and bytes for a grid: as deep as 8 rows while two CTAs fit an
// SM, else one CTA per SM; fewer than three slots is an error.
static bool march_plan(int mode, int rl, int *nslots, size_t *bytes) {
    const int nf = mode == FWI_SH ? 3 : 5, nv = mode == FWI_SH ? 1 : 2, ninj = mode == FWI_SH ? 1 : 2;
    const size_t budgets[2] = {(size_t)110 * 1024, (size_t)224 * 1024};
    for (size_t budget : budgets) {
        for (int n = 8; n >= 3; n--) {
            const MarchLayout L = march_layout(nf, nv, ninj, rl, n);
            if (L.bytes <= budget) {
                *nslots = n;
                *bytes = L.bytes;
                return true;
            }
        }
    }
    return false;
}

bool march_supported(const fwi_batch *b) {
    return (b->mode == FWI_SH || b->mode == FWI_PSV) && b->nz <= kMaxCols;
}

template <int MODE>
static int launch_march_mode(const MarchArgs &a, int nthr, size_t bytes, cudaStream_t st) {
    static size_t attr_bytes = 0;
    static int sms = 0, occ = 0, occ_thr = 0;
    static size_t occ_bytes = 0;
    if (bytes > attr_bytes) {
        cudaError_t e = cudaFuncSetAttribute(march_kernel<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)bytes);
        if (e != cudaSuccess) return set_error(FWI_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
        attr_bytes = bytes;
    }
    if (!sms) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
            sms = 148;
    }
    if (occ_thr != nthr || occ_bytes != bytes) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, march_kernel<MODE>, nthr, bytes) != cudaSuccess ||
            occ < 1)
            return set_error(FWI_ECUDA, "march_kernel: %d threads with %zu bytes of shared memory do not fit an SM",
                             nthr, bytes);
        occ_thr = nthr;
        occ_bytes = bytes;
    }
    const long long grid = a.rows_total < (long long)sms * occ ? a.rows_total : (long long)sms * occ;
    march_kernel<MODE><<<(unsigned)grid, nthr, bytes, st>>>(a);
    return check_launch("march_kernel");
}

int launch_march(const fwi_batch *b, int it, cudaStream_t st) {
    MarchArgs a;
    const int mode = b->mode;
    a.nx = b->nx;
    a.nz = b->nz;
    a.pitch = b->pitch;
    a.nt = b->nt;
    a.it = it;
    a.nrec = b->nrec;
    a.rows_total = (long long)b->nshots * b->nx;
    if (a.rows_total >= (1ll << 31))
        return set_error(FWI_ERANGE, "row-marching step: nshots * nx = %lld rows exceed 2^31", a.rows_total);
    a.cx1 = (float)(9.0 / (8.0 * (double)b->dx));
    a.cx2 = (float)(1.0 / (24.0 * (double)b->dx));
    a.cz1 = (float)(9.0 / (8.0 * (double)b->dz));
    a.cz2 = (float)(1.0 / (24.0 * (double)b->dz));
    a.dt = (float)b->dt;
    const int cur = b->cur, nxt = 1 - cur;
    const int ns = mode == FWI_SH ? 2 : 3, nv = mode == FWI_SH ? 1 : 2, ne = ns == 2 ? 2 : 3;
    for (int f = 0; f < 3; f++) {
        a.sig_in[f] = f < ns ? b->sig[cur][f] : nullptr;
        a.sig_out[f] = f < ns ? b->sig[nxt][f] : nullptr;
    }
    const long long field = (long long)b->nshots * b->nx * b->pitch;
    const bool seg = it - b->seg0 >= 0 && it - b->seg0 < b->nseg;
    for (int q = 0; q < 2; q++) {
        const bool on = q < nv;
        const int slot = on ? comp_slot_of(mode, q) : 0;
        a.vel_in[q] = on ? b->vel[cur][q] : nullptr;
        a.vel_out[q] = on ? b->vel[nxt][q] : nullptr;
        a.obs[q] = on ? b->obs[slot] : nullptr;
        a.seg_ds[q] = (on && seg && b->seg_ds[slot]) ? b->seg_ds[slot] + (long long)(it - b->seg0) * field : nullptr;
    }
    for (int k = 0; k < 3; k++)
        a.seg_e[k] = (seg && k < ne && b->seg_e[k]) ? b->seg_e[k] + (long long)(it - b->seg0) * field : nullptr;
    a.buo = b->buo;
    a.bound = b->bound;
    a.ip[0] = mode == FWI_SH ? b->mu : b->lam;
    a.ip[1] = mode == FWI_SH ? nullptr : b->mu;
    a.inj_ptr = b->inj_ptr;
    a.inj_cell = b->inj_cell;
    a.inj_row = b->inj_row;
    a.stf[0] = mode == FWI_SH ? b->stf[1] : b->stf[0];
    a.stf[1] = mode == FWI_SH ? nullptr : b->stf[2];
    a.rec_cell = b->rec_cell;
    a.rec_order = b->rec_order;
    const int nthr = ((b->nz + 31) / 32) * 32 < 64 ? 64 : ((b->nz + 31) / 32) * 32;
    int rl = (b->pitch > nthr ? b->pitch : nthr) + 8;
    rl = (rl + 3) / 4 * 4;
    a.rl = rl;
    size_t bytes = 0;
    if (!march_plan(mode, rl, &a.nslots, &bytes))
        return set_error(FWI_ERANGE, "row-marching step: rows of %d columns do not fit shared memory", b->pitch);
    return mode == FWI_SH ? launch_march_mode<FWI_SH>(a, nthr, bytes, st)
                          : launch_march_mode<FWI_PSV>(a, nthr, bytes, st);
}

// Binary version (major*10 + minor) of the device code the library loaded.
int kernel_binary_version(int *v) {
    cudaFuncAttributes fa;
    const cudaError_t e = cudaFuncGetAttributes(&fa, displacement_traces_kernel);
    if (e != cudaSuccess) return set_error(FWI_ECUDA, "cudaFuncGetAttributes: %s", cudaGetErrorString(e));
    *v = fa.binaryVersion;
    return 0;
}

int launch_displacement_traces(float *obs, long long ntr, int nt, int it0, int n, double dt, cudaStream_t st) {
    if (ntr <= 0 || n <= 0) return 0;
    const int th = 128;
    displacement_traces_kernel<<<(unsigned)((ntr + th - 1) / th), th, 0, st>>>(obs, ntr, nt, it0, n, (float)dt);
    return check_launch("displacement_traces_kernel");
}

}  // namespace fwi
