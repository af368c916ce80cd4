// Row-marching forward step for displacement-free SH and P-SV batches.
//
// Same arithmetic per cell as the tiled step kernels of step.cu (and so as
// the reference's div_sy / div_sxz, stf_dsy / stf_dsxz, add_vy / add_vxz,
// div_vy / div_vxz, add_sy / add_sxz and save_obs, solver.py:54-156), with a
// layout that keeps the instruction count per cell low enough for the step to
// be bound by HBM rather than by issue:
//
//   * A CTA spans the whole z extent of the grid -- thread t owns the four
//     columns 4t .. 4t+3 (up to 1024 columns) -- and marches down a
//     contiguous range of x rows of one shot.  Every shared-memory access
//     and every store is a 16-byte vector for four cells; the z neighbours
//     come from one 8- and one 4-byte load beside it.  The 4th-order x
//     derivatives of the stress come from register windows of four rows.
//   * Rows of the state (stress, velocity) stream into a ring of N row slots
//     in shared memory with untiled bulk copies (cp.async.bulk, one per field
//     and row, completion on an mbarrier per slot, bounded waits), issued by
//     one thread N-1 rows ahead of the march.  The model, shared by the shots
//     and resident in L2, is read with 16-byte loads one row ahead.
//   * The new velocity of row r goes to an eight-row ring in shared memory;
//     the stress of row r-2 is updated in the same iteration from that ring
//     (rows r-3 .. r for D+x, row r-2's neighbours for D+z).  One block
//     barrier per row.
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
#include <type_traits>

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

constexpr int kPts = 128;        // points (injection entries, receivers) staged per window
constexpr int kMaxPitch = 1024;  // row length (floats) a CTA can span: 256 threads of 4 columns
constexpr int kVRing = 5;        // rows of the new-velocity ring (rows s-1 .. s+2 live, plus one for barrier slack)

struct MarchArgs {
    int nx, nz, pitch, nt, it, nrec;
    int rl;                 // shared-memory row length (floats)
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
// [kVRing][NV][rl], injection window (cells, NINJ value rows), receiver
// window (cells, ids), two double-buffered cursors, then the mbarriers
// (8-byte aligned).
struct MarchLayout {
    int vring, icell, ival, rcell, rid, cur, bar;
    size_t bytes;
};

__host__ __device__ inline MarchLayout march_layout(int nf, int nv, int ninj, int rl, int nslots) {
    MarchLayout L;
    L.vring = nslots * nf * rl;
    L.icell = L.vring + kVRing * nv * rl;
    L.ival = L.icell + kPts;
    L.rcell = L.ival + ninj * kPts;
    L.rid = L.rcell + kPts;
    L.cur = L.rid + kPts;  // two double-buffered cursors (16 ints)
    L.bar = (L.cur + 16 + 1) / 2 * 2;
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

__device__ __forceinline__ void ld4(float (&d)[4], const float *p) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
    d[3] = v.w;
}
__device__ __forceinline__ void st4(float *p, const float (&d)[4]) {
    *reinterpret_cast<float4 *>(p) = make_float4(d[0], d[1], d[2], d[3]);
}
__device__ __forceinline__ void ldg4(float (&d)[4], const float *p) {
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    d[0] = v.x;
    d[1] = v.y;
    d[2] = v.z;
    d[3] = v.w;
}

template <int MODE, int N>
__global__ void __launch_bounds__(kMaxPitch / 4, 2) march_kernel(const __grid_constant__ MarchArgs a) {
    using F = Fields<MODE>;
    constexpr int NS = F::NS, NV = F::NV, NF = NS + NV, NINJ = F::NINJ;
    // stress fields with an x register window (D-x) and the one without
    constexpr int FX0 = 0, FX1 = MODE == FWI_SH ? 0 : 2, FZ = 1;
    constexpr int NW = MODE == FWI_SH ? 1 : 2;
    extern __shared__ __align__(128) float smem[];
    const int RL = a.rl;
    const MarchLayout L = march_layout(NF, NV, NINJ, RL, N);
    int *const i_cell = reinterpret_cast<int *>(smem + L.icell);
    float *const i_val = smem + L.ival;
    int *const r_cell = reinterpret_cast<int *>(smem + L.rcell);
    int *const r_id = reinterpret_cast<int *>(smem + L.rid);
    // cursors [list][buffer]: list 0 injection, 1 receivers; the buffer in use flips at every store
    Cursor *const cur_s = reinterpret_cast<Cursor *>(smem + L.cur);
    uint64_t *const full = reinterpret_cast<uint64_t *>(smem + L.bar);

    const int tid = threadIdx.x, j0 = 4 * tid;
    const int nx = a.nx, nz = a.nz, pitch = a.pitch, nt = a.nt, it = a.it;
    const bool tin = j0 < pitch;  // this thread's four columns lie in the rows
    const float cx1 = a.cx1, cx2 = a.cx2, cz1 = a.cz1, cz2 = a.cz2, dt = a.dt;
    const uint32_t row_bytes = 4u * (uint32_t)pitch;
    // row buffers start 4 floats into their slot so that columns -4 .. rl-5 are addressable
    auto ring_row = [&](int slot, int f) -> float * { return smem + (slot * NF + f) * RL + 4; };


    grid_dep_trigger();
    if (tid == 0) {
        for (int i = 0; i < N; i++) mbar_init(&full[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    // the previous step (state rows, and the stress / velocity buffers this
    // step overwrites) is complete from here on
    grid_dep_wait();

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
    // Only warp 0 waits for rows (the others wait at the block barrier that
    // follows, without issuing); the barrier then makes the landed row
    // visible to every thread.
    const bool waiter = tid < 32;
    // per-column masks, fixed for the whole march: D-z (2 <= j < nz-2),
    // D+z (1 <= j < nz-2) and "inside the grid" (j < nz)
    bool zm[4], zp[4], zin[4];
#pragma unroll
    for (int e = 0; e < 4; e++) {
        const int c = j0 + e;
        zm[e] = c >= 2 && c < nz - 2;
        zp[e] = c >= 1 && c < nz - 2;
        zin[e] = c < nz;
    }
    // warps without a masked column (all but those at the z edges) skip the masks
    const bool zedge = __any_sync(0xffffffffu, !(j0 >= 2 && j0 + 3 < nz - 2));

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
    // after the points of a row: store the cursor into the other buffer of
    // its list (slow threads may still read the one in use; the row barrier
    // that follows orders the store before the next use) and return the cell
    // of the next point, or kNone.  Every thread holds the same cursor.
    auto park = [&](Cursor &c, int which, int &buf, bool inj) -> int {
        if (c.p < c.end && c.p - c.w0 >= c.wn) {
            if (inj) load_inj(c);
            else load_rec(c);
        }
        const int nxt = c.p < c.end ? (inj ? i_cell : r_cell)[c.p - c.w0] : kNone;
        buf ^= 1;
        if (tid == 0) cur_s[2 * which + buf] = c;
        return nxt;
    };
    // model row `row` at this thread's columns (zero outside the grid)
    auto ld_model = [&](float (&d)[4], const float *p, int row) {
        if (tin && row >= 0 && row < nx) {
            ldg4(d, p + (long long)row * pitch + j0);
        } else {
#pragma unroll
            for (int e = 0; e < 4; e++) d[e] = 0.f;
        }
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
            cur_s[2] = Cursor{r0, r1, r0, 0};
        }
        __syncthreads();
        int inj_next, rec_next;  // cell of the next injection entry / receiver, or kNone
        int ib = 0, rb = 0;      // cursor buffers in use
        {
            Cursor c = cur_s[0];
            inj_next = c.p < c.end ? park(c, 0, ib, true) : kNone;
            c = cur_s[2];
            rec_next = c.p < c.end ? park(c, 1, rb, false) : kNone;
        }

        bool ok = true;
        // register windows of four cells: the D-x stress fields at rows
        // r-2 .. r+1 (SH: sxy; P-SV: sxx, sxz), the other stress field at rows
        // r-2 .. r (SH: szy; P-SV: szz)
        float wx[NW][4][4], wz[3][4];
        // the window rows va-2 .. va must have landed before the first iteration
        if (waiter)
            for (int q = qa; q <= va; q++) ok = wait_seq(sb + q) && ok;
        if (__syncthreads_or(!ok)) goto bail;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const int q = va - 2 + k;
            if (q >= qa) {
                const int sl = (sb + q) % N;
                ld4(wx[0][k], ring_row(sl, FX0) + j0);
                if (NW > 1) ld4(wx[NW - 1][k], ring_row(sl, FX1) + j0);
                if (k < 2) ld4(wz[k + 1], ring_row(sl, FZ) + j0);  // rows va-2, va-1 -> wz[1], wz[2]
            } else {
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    wx[0][k][e] = wx[NW - 1][k][e] = 0.f;
                    if (k < 2) wz[k + 1][e] = 0.f;
                }
            }
        }
        // model of the first row: dt/rho and sponge (row va), stiffness (row va-2)
        float buo[4], bnd[4], ip0[4], ip1[4];
        ld_model(buo, a.buo, va);
        ld_model(bnd, a.bound, va);
        ld_model(ip0, a.ip[0], va - 2);
        if (MODE == FWI_PSV) ld_model(ip1, a.ip[1], va - 2);
        // rows above va are consumed once every thread has its window: their
        // slots take the next rows; then row va+1, which the first iteration
        // reads, has to land
        __syncthreads();
        for (int q = qa; q < va; q++)
            if (nexti < qb) {
                if (tid == 0) issue(soff, nexti, sb + nexti);
                nexti++;
            }
        if (waiter && va + 1 < qb) ok = wait_seq(sb + va + 1) && ok;
        if (__syncthreads_or(!ok)) goto bail;

        // vk: velocity-ring slot of row r
        for (int r = va, vk = va % kVRing; r < b0 + 2; r++, vk = vk == kVRing - 1 ? 0 : vk + 1) {
            // next iteration's model values (one row ahead): dt/rho and sponge of row r+1,
            // stiffness of row r-1
            float buo_n[4], bnd_n[4], ip0_n[4], ip1_n[4];
            {
                const long long m1 = (long long)(r + 1) * pitch + j0, m2 = m1 - 2ll * pitch;
                const bool ok1 = tin && r + 1 < nx, ok2 = tin && r >= 1 && r - 1 < nx;
#pragma unroll
                for (int e = 0; e < 4; e++) buo_n[e] = bnd_n[e] = ip0_n[e] = ip1_n[e] = 0.f;
                if (ok1) {
                    ldg4(buo_n, a.buo + m1);
                    ldg4(bnd_n, a.bound + m1);
                }
                if (ok2) {
                    ldg4(ip0_n, a.ip[0] + m2);
                    if (MODE == FWI_PSV) ldg4(ip1_n, a.ip[1] + m2);
                }
            }
            // velocity-ring slots of rows r-3 .. r (row r-3+k in slot vs[k])
            int vs[4];
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const int q = vk - 3 + k;
                vs[k] = q < 0 ? q + kVRing : q;
            }
            auto vrow = [&](int slot, int c) -> float * { return smem + L.vring + (slot * NV + c) * RL + 4 + j0; };
            // the z window shifts: wz[0..2] <- rows r-2, r-1, r
#pragma unroll
            for (int e = 0; e < 4; e++) {
                wz[0][e] = wz[1][e];
                wz[1][e] = wz[2][e];
            }
            float vn[NV][4];
            const long long grow = soff + (long long)r * pitch + j0;
            if (r < vb) {
                // ---- velocity of row r
                if (r + 1 < qb) {  // landed: waited for before the previous row's barrier
                    const int sl = (sb + r + 1) % N;
                    ld4(wx[0][3], ring_row(sl, FX0) + j0);
                    if (NW > 1) ld4(wx[NW - 1][3], ring_row(sl, FX1) + j0);
                } else {
#pragma unroll
                    for (int e = 0; e < 4; e++) wx[0][3][e] = wx[NW - 1][3][e] = 0.f;
                }
                const int sr = (sb + r) % N;
                ld4(wz[2], ring_row(sr, FZ) + j0);
                const bool okx = r >= 2 && r < nx - 2;
                // D-x of window field w, element e
                auto dxm = [&](int w, int e) -> float {
                    return okx ? cx1 * (wx[w][2][e] - wx[w][1][e]) - cx2 * (wx[w][3][e] - wx[w][0][e]) : 0.f;
                };
                float ds[NV][4];
                // the stress divergence; ZE: this warp holds columns near a z edge (per-column masks)
                auto divergence = [&](auto ze_t) {
                    constexpr bool ZE = decltype(ze_t)::value;
                    // D-z of stress field f at row r, element e, from columns j0-2 .. j0+4:
                    // x[i] = column j0-2+i, with the centre taken from `cen`
                    auto dzm_row = [&](int f, const float (&cen)[4], float (&out)[4]) {
                        const float *s = ring_row(sr, f) + j0;
                        const float2 l2 = *reinterpret_cast<const float2 *>(s - 2);
                        const float rr = s[4];
                        const float x[7] = {l2.x, l2.y, cen[0], cen[1], cen[2], cen[3], rr};
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const float d = cz1 * (x[e + 2] - x[e + 1]) - cz2 * (x[e + 3] - x[e]);
                            out[e] = (!ZE || zm[e]) ? d : 0.f;
                        }
                    };
                    if constexpr (MODE == FWI_SH) {
                        float zz[4];
                        dzm_row(1, wz[2], zz);
#pragma unroll
                        for (int e = 0; e < 4; e++) ds[0][e] = dxm(0, e) + zz[e];
                    } else {
                        float zxz[4], zzz[4];
                        dzm_row(2, wx[1][2], zxz);
                        dzm_row(1, wz[2], zzz);
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            ds[0][e] = dxm(0, e) + zxz[e];
                            ds[1][e] = dxm(1, e) + zzz[e];
                        }
                    }
                };
                if (zedge) divergence(std::true_type{});
                else divergence(std::false_type{});
                // sources of row r, summed per cell in entry order (stf_dsy / stf_dsxz, solver.py:78-93)
                if (inj_next < (r + 1) * nz) {
                    const int lo = r * nz, hi = lo + nz;
                    float acc[NINJ][4];
#pragma unroll
                    for (int q = 0; q < NINJ; q++)
#pragma unroll
                        for (int e = 0; e < 4; e++) acc[q][e] = 0.f;
                    Cursor c = cur_s[ib];
                    while (c.p < c.end) {
                        if (c.p - c.w0 >= c.wn) load_inj(c);
                        const int k = c.p - c.w0, cell = i_cell[k];
                        if (cell >= hi) break;
                        const int off = cell - lo - j0;
#pragma unroll
                        for (int e = 0; e < 4; e++)
                            if (off == e) {
#pragma unroll
                                for (int q = 0; q < NINJ; q++) acc[q][e] += i_val[q * kPts + k];
                            }
                        c.p++;
                    }
                    inj_next = park(c, 0, ib, true);
#pragma unroll
                    for (int q = 0; q < NV; q++)
#pragma unroll
                        for (int e = 0; e < 4; e++) ds[q][e] += acc[q][e];
                }
                const bool own = r >= a0 && r < b0 && tin;
                auto velocity = [&](auto ze_t) {
                    constexpr bool ZE = decltype(ze_t)::value;
#pragma unroll
                    for (int c = 0; c < NV; c++) {
                        float vold[4];
                        ld4(vold, ring_row(sr, NS + c) + j0);
#pragma unroll
                        for (int e = 0; e < 4; e++) {
                            const float v = bnd[e] * (vold[e] + ds[c][e] * buo[e]);
                            vn[c][e] = (!ZE || zin[e]) ? v : 0.f;  // padding columns stay zero
                            if (ZE && !zin[e]) ds[c][e] = 0.f;
                        }
                        st4(vrow(vs[3], c), vn[c]);
                        if (own) {
                            st4(a.vel_out[c] + grow, vn[c]);
                            if (a.seg_ds[c]) st4(a.seg_ds[c] + grow, ds[c]);
                        }
                    }
                };
                if (zedge) velocity(std::true_type{});
                else velocity(std::false_type{});
                // receivers of row r record the new velocity (save_obs, solver.py:151-156)
                if (rec_next < (r + 1) * nz) {
                    const int lo = r * nz, hi = lo + nz;
                    Cursor c = cur_s[2 + rb];
                    while (c.p < c.end) {
                        if (c.p - c.w0 >= c.wn) load_rec(c);
                        const int k = c.p - c.w0, cell = r_cell[k];
                        if (cell >= hi) break;
                        const int off = cell - lo - j0;
                        if (off >= 0 && off < 4) {
                            const long long o = ((long long)shot * a.nrec + r_id[k]) * nt + it;
#pragma unroll
                            for (int e = 0; e < 4; e++)
                                if (off == e) {
#pragma unroll
                                    for (int q = 0; q < NV; q++)
                                        if (a.obs[q]) a.obs[q][o] = vn[q][e];
                                }
                        }
                        c.p++;
                    }
                    rec_next = park(c, 1, rb, false);
                }
            } else {
#pragma unroll
                for (int c = 0; c < NV; c++) {
#pragma unroll
                    for (int e = 0; e < 4; e++) vn[c][e] = 0.f;
                    st4(vrow(vs[3], c), vn[c]);
                }
            }
            // the next iteration reads row r+2: warp 0 waits for it before the barrier
            if (waiter && r + 2 < qb && r + 2 < vb + 1) ok = wait_seq(sb + r + 2) && ok;
            if (__syncthreads_or(!ok)) goto bail;
            // row r is consumed: its slot takes row r + N
            if (nexti < qb) {
                if (tid == 0) issue(soff, nexti, sb + nexti);
                nexti++;
            }

            // ---- stress of row s = r - 2 (add_sy / add_sxz, solver.py:128-149)
            const int s = r - 2;
            auto stress = [&](auto ze_t) {
                constexpr bool ZE = decltype(ze_t)::value;
                const bool okx = s >= 1 && s < nx - 2;
                const long long gs = soff + (long long)s * pitch + j0;
                float ex[NV][4], ez[NV][4];
#pragma unroll
                for (int c = 0; c < NV; c++) {
                    // rows s-1 .. s+2 of the new velocity, and row s's z neighbours:
                    // y[i] = column j0-1+i of row s
                    float v0[4], v1[4], v2[4], v3[4];
                    ld4(v0, vrow(vs[0], c));
                    ld4(v1, vrow(vs[1], c));
                    ld4(v2, vrow(vs[2], c));
                    ld4(v3, vrow(vs[3], c));
                    const float *vsr = vrow(vs[1], c);
                    const float l1 = vsr[-1];
                    const float2 r2 = *reinterpret_cast<const float2 *>(vsr + 4);
                    const float y[7] = {l1, v1[0], v1[1], v1[2], v1[3], r2.x, r2.y};
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        ex[c][e] = okx ? cx1 * (v2[e] - v1[e]) - cx2 * (v3[e] - v0[e]) : 0.f;
                        const float d = cz1 * (y[e + 2] - y[e + 1]) - cz2 * (y[e + 3] - y[e]);
                        ez[c][e] = (!ZE || zp[e]) ? d : 0.f;
                    }
                }
                if constexpr (MODE == FWI_SH) {
                    float o0[4], o1[4];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const float dm = dt * ip0[e], exy = ex[0][e], ezy = ez[0][e];
                        const bool in = !ZE || zin[e];  // padding columns stay zero
                        o0[e] = in ? wx[0][0][e] + dm * exy : 0.f;
                        o1[e] = in ? wz[0][e] + dm * ezy : 0.f;
                    }
                    st4(a.sig_out[0] + gs, o0);
                    st4(a.sig_out[1] + gs, o1);
                    if (a.seg_e[0]) {
                        st4(a.seg_e[0] + gs, ex[0]);
                        st4(a.seg_e[1] + gs, ez[0]);
                    }
                } else {
                    float o0[4], o1[4], o2[4], sh[4];
#pragma unroll
                    for (int e = 0; e < 4; e++) {
                        const float lam = ip0[e], mu = ip1[e];
                        const float vxx = ex[0][e], vxz = ez[0][e], vzx = ex[1][e], vzz = ez[1][e];
                        const float l2m = lam + 2.f * mu, shear = vxz + vzx;
                        const bool in = !ZE || zin[e];  // padding columns stay zero
                        o0[e] = in ? wx[0][0][e] + dt * (l2m * vxx + lam * vzz) : 0.f;
                        o1[e] = in ? wz[0][e] + dt * (l2m * vzz + lam * vxx) : 0.f;
                        o2[e] = in ? wx[1][0][e] + dt * (mu * shear) : 0.f;
                        sh[e] = in ? shear : 0.f;
                    }
                    st4(a.sig_out[0] + gs, o0);
                    st4(a.sig_out[1] + gs, o1);
                    st4(a.sig_out[2] + gs, o2);
                    if (a.seg_e[0]) {
                        st4(a.seg_e[0] + gs, ex[0]);
                        st4(a.seg_e[1] + gs, ez[1]);
                        st4(a.seg_e[2] + gs, sh);
                    }
                }
            };
            if (s >= a0 && s < b0 && tin) {
                if (zedge) stress(std::true_type{});
                else stress(std::false_type{});
            }
#pragma unroll
            for (int w = 0; w < NW; w++)
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    wx[w][0][e] = wx[w][1][e];
                    wx[w][1][e] = wx[w][2][e];
                    wx[w][2][e] = wx[w][3][e];
                }
#pragma unroll
            for (int e = 0; e < 4; e++) {
                buo[e] = buo_n[e];
                bnd[e] = bnd_n[e];
                ip0[e] = ip0_n[e];
                if (MODE == FWI_PSV) ip1[e] = ip1_n[e];
            }
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

// Shared-memory bytes of a ring depth for a row length.
static size_t march_bytes(int mode, int rl, int n) {
    const int nf = mode == FWI_SH ? 3 : 5, nv = mode == FWI_SH ? 1 : 2, ninj = mode == FWI_SH ? 1 : 2;
    return march_layout(nf, nv, ninj, rl, n).bytes;
}

bool march_supported(const fwi_batch *b) {
    return (b->mode == FWI_SH || b->mode == FWI_PSV) && b->pitch <= kMaxPitch;
}

template <int MODE, int N>
static int march_occupancy(int nthr, size_t bytes, int *occ) {
    cudaError_t e = cudaFuncSetAttribute(march_kernel<MODE, N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(occ, march_kernel<MODE, N>, nthr, bytes);
    if (e != cudaSuccess) return set_error(FWI_ECUDA, "march_kernel occupancy: %s", cudaGetErrorString(e));
    return 0;
}

template <int MODE>
static int march_occupancy_n(int n, int nthr, size_t bytes, int *occ) {
    switch (n) {
        case 3: return march_occupancy<MODE, 3>(nthr, bytes, occ);
        case 4: return march_occupancy<MODE, 4>(nthr, bytes, occ);
        case 6: return march_occupancy<MODE, 6>(nthr, bytes, occ);
        default: return march_occupancy<MODE, 8>(nthr, bytes, occ);
    }
}

// Ring depth and resident CTAs per SM for a launch shape: the requested
// depth, or the one with the most resident CTAs (shared memory and
// registers both counted), the deepest among those.  Cached per shape.
template <int MODE>
static int march_choose(int nthr, int rl, int want, int *n_out, size_t *bytes_out, int *occ_out) {
    struct Entry {
        int nthr, rl, want, n, occ;
        size_t bytes;
    };
    static Entry cache[16];
    static int ncache = 0;
    for (int i = 0; i < ncache; i++)
        if (cache[i].nthr == nthr && cache[i].rl == rl && cache[i].want == want) {
            *n_out = cache[i].n;
            *bytes_out = cache[i].bytes;
            *occ_out = cache[i].occ;
            return 0;
        }
    int best = 0, best_occ = 0;
    size_t best_bytes = 0;
    for (int n : {3, 4, 6, 8}) {
        if (want && n != want) continue;
        const size_t b = march_bytes(MODE, rl, n);
        if (b > (size_t)227 * 1024) continue;
        int occ = 0;
        const int rc = march_occupancy_n<MODE>(n, nthr, b, &occ);
        if (rc) return rc;
        if (occ >= 1 && occ >= best_occ) {
            best = n;
            best_occ = occ;
            best_bytes = b;
        }
    }
    if (!best) return set_error(FWI_ERANGE, "row-marching step: rows of %d floats do not fit an SM", rl - 8);
    if (ncache < 16) cache[ncache++] = Entry{nthr, rl, want, best, best_occ, best_bytes};
    *n_out = best;
    *bytes_out = best_bytes;
    *occ_out = best_occ;
    return 0;
}

template <int MODE, int N>
static int launch_march_mode(const MarchArgs &a, int nthr, size_t bytes, int occ, bool pdl, cudaStream_t st) {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
            sms = 148;
    }
    const long long grid = a.rows_total < (long long)sms * occ ? a.rows_total : (long long)sms * occ;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)grid, 1, 1);
    cfg.blockDim = dim3(nthr, 1, 1);
    cfg.dynamicSmemBytes = bytes;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    set_pdl_attr(attr[0], true);
    cfg.attrs = attr;
    cfg.numAttrs = pdl ? 1 : 0;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, march_kernel<MODE, N>, a);
    if (e != cudaSuccess) return set_error(FWI_ECUDA, "march_kernel launch: %s", cudaGetErrorString(e));
    return check_launch("march_kernel");
}

int launch_march(const fwi_batch *b, int it, bool pdl, cudaStream_t st) {
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
    // four columns per thread, whole warps
    const int nthr = ((b->pitch / 4 + 31) / 32) * 32;
    a.rl = 4 * nthr + 8;
    size_t bytes = 0;
    int n = 0, occ = 0;
    int rc = mode == FWI_SH ? march_choose<FWI_SH>(nthr, a.rl, b->ring, &n, &bytes, &occ)
                            : march_choose<FWI_PSV>(nthr, a.rl, b->ring, &n, &bytes, &occ);
    if (rc) return rc;
    if (b->ctas_per_sm > 0 && b->ctas_per_sm < occ) occ = b->ctas_per_sm;
    if (mode == FWI_SH) {
        switch (n) {
            case 3: return launch_march_mode<FWI_SH, 3>(a, nthr, bytes, occ, pdl, st);
            case 4: return launch_march_mode<FWI_SH, 4>(a, nthr, bytes, occ, pdl, st);
            case 6: return launch_march_mode<FWI_SH, 6>(a, nthr, bytes, occ, pdl, st);
            default: return launch_march_mode<FWI_SH, 8>(a, nthr, bytes, occ, pdl, st);
        }
    }
    switch (n) {
        case 3: return launch_march_mode<FWI_PSV, 3>(a, nthr, bytes, occ, pdl, st);
        case 4: return launch_march_mode<FWI_PSV, 4>(a, nthr, bytes, occ, pdl, st);
        case 6: return launch_march_mode<FWI_PSV, 6>(a, nthr, bytes, occ, pdl, st);
        default: return launch_march_mode<FWI_PSV, 8>(a, nthr, bytes, occ, pdl, st);
    }
}

// A bounded wait on an mbarrier that nothing ever completes: the wait runs
// out after the current poll limit, the kernel records it in the status word
// like a step kernel whose copies were lost, and returns.  No copy is in
// flight, so giving up is harmless; used to test the failure path.
__global__ void wait_selftest_kernel() {
    __shared__ uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        if (!mbar_wait(&bar, 0)) atomicExch(&g_march_status, 1);
    }
}

int launch_wait_selftest(cudaStream_t st) {
    wait_selftest_kernel<<<1, 32, 0, st>>>();
    return check_launch("wait_selftest_kernel");
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

cudaError_t fwi::march_set_wait_limit(int polls) { return fwi::set_wait_limit_here(polls); }
