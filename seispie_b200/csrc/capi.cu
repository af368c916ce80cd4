// extern "C" entry points of libseispie_b200.so (declared in
// include/seispie_b200.h): argument checks, error reporting and the host
// time loop that enqueues the fused step kernels.
#include <cstdarg>
#include <cstdio>
#include <atomic>
#include <cstring>

#include "common.cuh"

namespace fwi {

static thread_local int g_code = 0;
static thread_local char g_msg[512] = "";

int set_error(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
    va_end(ap);
    g_code = code;
    return code;
}

static std::atomic<long long> g_launches{0};

int check_launch(const char *what) {
    g_launches.fetch_add(1, std::memory_order_relaxed);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(FWI_ECUDA, "%s: %s", what, cudaGetErrorString(e));
    return 0;
}

// defined in step.cu / aux.cu
int launch_step(const fwi_batch *b, int adjoint, int it, bool snap_u_next, int snap_u_slot, bool snap_v,
                int snap_v_slot, cudaStream_t st);
int launch_interaction(const fwi_batch *b, int isae, cudaStream_t st);
int launch_adjoint_step(const fwi_batch *b, int it, bool pdl, cudaStream_t st);
int launch_march(const fwi_batch *b, int it, bool pdl, cudaStream_t st);
bool march_supported(const fwi_batch *b);
int launch_displacement_traces(float *obs, long long ntr, int nt, int it0, int n, double dt, cudaStream_t st);
int kernel_binary_version(int *v);
int launch_wait_selftest(cudaStream_t st);
long long multi_workspace_bytes(int n);
int multi_prepare(fwi_batch *const *bs, int n, void *ws, int (*check)(const fwi_batch *, int, int, int));
int multi_run(fwi_batch *const *bs, int n, void *ws, int it0, int nsteps, cudaStream_t st);
int launch_misfit(const float *data, const float *syn, float *adstf, double *misfit, double *partial, int nshots,
                  int nrec, int nt, double dt, cudaStream_t st, bool grad);
long long misfit_partials(int nrec, int nt);
int launch_suffix_sum(const float *g, float *out, long long ntraces, int nt, cudaStream_t st);
int launch_energy(const float *f, int nshots, long long field, double *acc, cudaStream_t st);
int launch_smooth(const double *in, int in_pitch, float *out, int out_pitch, double *tmp, int nx, int nz, int sigma,
                  cudaStream_t st);
int launch_vps2lm(float *lam, float *mu, const float *rho, long long n, cudaStream_t st);
int launch_lm2vps(float *vp, float *vs, const float *rho, long long n, cudaStream_t st);
int launch_bound(float *bound, int nx, int nz, int pitch, int width, double alpha, int l, int r, int b, int t,
                 cudaStream_t st);
int launch_ricker(const double *par, int nsrc, int nt, double dt, float *sx, float *sy, float *sz, cudaStream_t st);
int launch_prepare(const float *rho, const float *jr, const float *muc, const float *nuc, double dt, long long n,
                   float *buo, float *buo_j, float *mnc, cudaStream_t st);
int tile_count();
bool tile_shape(int tile, int *tx, int *tz);
int tile_kind(int tile);

static bool aligned16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

#define REQUIRE(cond, ...)                                        \
    do {                                                          \
        if (!(cond)) return set_error(FWI_EINVAL, __VA_ARGS__);   \
    } while (0)

static int check_batch(const fwi_batch *b, int adjoint, int it0, int nsteps) {
    REQUIRE(b, "batch is NULL");
    REQUIRE(b->mode == FWI_SH || b->mode == FWI_PSV || b->mode == FWI_SPIN, "mode %d unknown", b->mode);
    REQUIRE(b->step_overlap == 0 || b->step_overlap == 1, "step_overlap must be 0 or 1 (got %d)", b->step_overlap);
    REQUIRE(b->nx >= 1 && b->nz >= 1, "grid %dx%d is empty", b->nx, b->nz);
    REQUIRE(b->pitch >= b->nz && b->pitch % 4 == 0, "pitch %d must be >= nz (%d) and a multiple of 4", b->pitch,
            b->nz);
    REQUIRE(b->nshots >= 1 && b->nshots <= 65535, "nshots %d out of range [1, 65535]", b->nshots);
    REQUIRE((long long)b->nx * b->nz < (1ll << 31), "grid of %lld cells exceeds 2^31", (long long)b->nx * b->nz);
    REQUIRE(b->cur == 0 || b->cur == 1, "cur must be 0 or 1");
    REQUIRE(b->tile >= 0 && b->tile < tile_count(), "tile variant %d unknown", b->tile);
    REQUIRE(b->nt >= 1, "nt must be >= 1");
    REQUIRE(it0 >= 0 && nsteps >= 0 && (long long)it0 + nsteps <= b->nt, "steps [%d, %d) outside [0, nt=%d)", it0,
            it0 + nsteps, b->nt);
    REQUIRE(b->dx > 0.f && b->dz > 0.f && b->dt > 0.0, "dx, dz and dt must be positive");
    const int ns = b->mode == FWI_SH ? 2 : b->mode == FWI_PSV ? 3 : 6;
    const int nv = b->mode == FWI_SH ? 1 : b->mode == FWI_PSV ? 2 : 3;
    for (int h = 0; h < 2; h++) {
        for (int f = 0; f < ns; f++)
            REQUIRE(b->sig[h][f] && aligned16(b->sig[h][f]), "sig[%d][%d] NULL or not 16-byte aligned", h, f);
        for (int q = 0; q < nv; q++)
            REQUIRE(b->vel[h][q] && aligned16(b->vel[h][q]), "vel[%d][%d] NULL or not 16-byte aligned", h, q);
    }
    const bool nodisp = !b->disp[0];
    for (int q = 0; q < nv; q++)
        REQUIRE(nodisp ? !b->disp[q] : (b->disp[q] && aligned16(b->disp[q])),
                "disp[] must be all NULL (displacement-free) or all set and 16-byte aligned (disp[%d])", q);
    REQUIRE(b->buo && b->bound && b->mu && aligned16(b->buo) && aligned16(b->bound) && aligned16(b->mu),
            "buo, bound and mu must be non-NULL and 16-byte aligned");
    if (b->mode != FWI_SH) REQUIRE(b->lam && aligned16(b->lam), "lam must be non-NULL and 16-byte aligned");
    if (b->mode == FWI_SPIN)
        REQUIRE(b->buo_j && b->nu && b->mnc && aligned16(b->buo_j) && aligned16(b->nu) && aligned16(b->mnc),
                "spin needs buo_j, nu and mnc (16-byte aligned)");
    if (b->inj_ptr) {
        REQUIRE(b->inj_cell && b->inj_row, "inj_cell and inj_row are required with inj_ptr");
        if (b->mode == FWI_SH) REQUIRE(b->stf[1], "SH injection needs stf[1]");
        else REQUIRE(b->stf[0] && b->stf[2], "P-SV injection needs stf[0] and stf[2]");
    }
    if (b->nrec > 0 && !adjoint) REQUIRE(b->rec_cell, "rec_cell is required when nrec > 0");
    if (nodisp && nsteps > 0) {
        REQUIRE(!adjoint, "the continuous adjoint (adjoint = 1) needs displacement fields");
        REQUIRE(march_supported(b), "displacement-free batches: SH or P-SV with nz <= 1024 (mode %d, nz %d)", b->mode,
                b->nz);
        for (int c = 0; c < 3; c++)
            REQUIRE(!b->snap_u[c] && !b->snap_v[c], "displacement-free batches take no snapshots");
        const bool rec = b->nrec > 0 && (b->obs[0] || b->obs[1] || b->obs[2]);
        REQUIRE(!rec || b->rec_order, "displacement-free batches that record traces need rec_order");
        REQUIRE(b->ring == 0 || b->ring == 3 || b->ring == 4 || b->ring == 6 || b->ring == 8,
                "ring must be 0, 3, 4, 6 or 8 (got %d)", b->ring);
        REQUIRE(b->ctas_per_sm >= 0, "ctas_per_sm must be >= 0 (got %d)", b->ctas_per_sm);
    }
    if (adjoint) {
        REQUIRE(b->sae >= 1, "the adjoint needs adjoint_interval >= 1");
        REQUIRE(b->nsa >= 1, "the adjoint needs nsa >= 1 snapshots");
        if (b->mode == FWI_SH) REQUIRE(b->snap_u[1], "SH adjoint needs snap_u[1]");
        else REQUIRE(b->snap_u[0] && b->snap_u[2], "P-SV adjoint needs snap_u[0] and snap_u[2]");
        REQUIRE(b->mode != FWI_SPIN, "the spin adjoint is not provided");
        // the correlation at step it reads slot it/sae (solver.py:315-318)
        const int last = it0 + nsteps - 1;
        if (nsteps > 0) {
            const int last_corr = last - last % b->sae;
            REQUIRE(last_corr < it0 || last_corr / b->sae < b->nsa,
                    "adjoint step %d needs snapshot %d but only %d exist (nt must not exceed nsa*sae)", last_corr,
                    last_corr / b->sae, b->nsa);
        }
    }
    return 0;
}

}  // namespace fwi

using namespace fwi;

extern "C" {

int fwi_abi_version(void) { return FWI_ABI_VERSION; }

long long fwi_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

int fwi_binary_version(void) {
    int v = 0;
    const int rc = kernel_binary_version(&v);
    return rc ? rc : v;
}

int fwi_device_status(int *status, int clear) {
    if (!status) return set_error(FWI_EINVAL, "fwi_device_status: NULL status");
    int a = 0, m = 0, b = 0;
    int rc = step_device_status(clear, &a);
    if (!rc) rc = march_device_status(clear, &m);
    if (!rc) rc = unet_device_status(clear, &b);
    if (rc) return rc;
    *status = (a || m ? 1 : 0) | (b ? 2 : 0);
    return 0;
}

int fwi_set_wait_limit(int polls) {
    REQUIRE(polls >= 0, "fwi_set_wait_limit: polls must be >= 0 (0 restores the default)");
    const int p = polls ? polls : kDefaultWaitPolls;
    cudaError_t e = step_set_wait_limit(p);
    if (e == cudaSuccess) e = march_set_wait_limit(p);
    if (e == cudaSuccess) e = unet_set_wait_limit(p);
    if (e != cudaSuccess) return set_error(FWI_ECUDA, "fwi_set_wait_limit: %s", cudaGetErrorString(e));
    return 0;
}

int fwi_wait_selftest(void *stream) { return launch_wait_selftest((cudaStream_t)stream); }

int fwi_last_error(char *buf, size_t len) {
    if (buf && len) {
        strncpy(buf, g_msg, len - 1);
        buf[len - 1] = '\0';
    }
    return g_code;
}

int fwi_tile_kind(int tile) {
    const int k = tile_kind(tile);
    return k < 0 ? set_error(FWI_EINVAL, "tile variant %d unknown", tile) : k;
}

int fwi_tile_shape(int tile, int *tx, int *tz) {
    int x = 0, z = 0;
    REQUIRE(tile_shape(tile, &x, &z), "tile variant %d unknown", tile);
    if (tx) *tx = x;
    if (tz) *tz = z;
    return 0;
}

int fwi_vps2lm(float *lam_io, float *mu_io, const float *rho, long long n, void *stream) {
    REQUIRE(lam_io && mu_io && rho && n >= 0, "fwi_vps2lm: NULL pointer or negative size");
    if (n == 0) return 0;
    return launch_vps2lm(lam_io, mu_io, rho, n, (cudaStream_t)stream);
}

int fwi_lm2vps(float *vp_io, float *vs_io, const float *rho, long long n, void *stream) {
    REQUIRE(vp_io && vs_io && rho && n >= 0, "fwi_lm2vps: NULL pointer or negative size");
    if (n == 0) return 0;
    return launch_lm2vps(vp_io, vs_io, rho, n, (cudaStream_t)stream);
}

int fwi_set_bound(float *bound, int nx, int nz, int pitch, int width, double alpha, int left, int right, int bottom,
                  int top, void *stream) {
    REQUIRE(bound && nx >= 1 && nz >= 1 && pitch >= nz, "fwi_set_bound: bad arguments");
    return launch_bound(bound, nx, nz, pitch, width, alpha, left, right, bottom, top, (cudaStream_t)stream);
}

int fwi_ricker(const double *params, int nsrc, int nt, double dt, float *stf_x, float *stf_y, float *stf_z,
               void *stream) {
    REQUIRE(params && nsrc >= 0 && nt >= 0 && nsrc <= 65535, "fwi_ricker: bad arguments");
    if (nsrc == 0 || nt == 0) return 0;
    return launch_ricker(params, nsrc, nt, dt, stf_x, stf_y, stf_z, (cudaStream_t)stream);
}

int fwi_prepare_model(const float *rho, const float *j, const float *mu_c, const float *nu_c, double dt, long long n,
                      float *buo, float *buo_j, float *mnc, void *stream) {
    REQUIRE(rho && buo && n >= 0, "fwi_prepare_model: rho and buo are required");
    REQUIRE(!buo_j || j, "fwi_prepare_model: buo_j needs j");
    REQUIRE(!mnc || (mu_c && nu_c), "fwi_prepare_model: mnc needs mu_c and nu_c");
    if (n == 0) return 0;
    return launch_prepare(rho, j, mu_c, nu_c, dt, n, buo, buo_j, mnc, (cudaStream_t)stream);
}

int fwi_run(fwi_batch *b, int adjoint, int it0, int nsteps, void *stream) {
    int rc = check_batch(b, adjoint, it0, nsteps);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    if (!b->disp[0]) {
        // displacement-free: row-marching steps recording velocity at the
        // receivers, then the traces' running sums over these steps
        // every launch after the first follows a row-marching step of this loop
        // directly in the stream, so it may overlap that step's tail
        const bool pdl = b->step_overlap != 0;
        for (int it = it0; it < it0 + nsteps; it++) {
            rc = launch_march(b, it, pdl && it > it0, st);
            if (rc) return rc;
            b->cur ^= 1;
        }
        const long long ntr = (long long)b->nshots * b->nrec;
        for (int c = 0; c < 3 && b->nrec > 0; c++) {
            if (!b->obs[c]) continue;
            rc = launch_displacement_traces(b->obs[c], ntr, b->nt, it0, nsteps, b->dt, st);
            if (rc) return rc;
        }
        return 0;
    }
    const long long field = (long long)b->nshots * b->nx * b->pitch;
    const int sae = b->sae, nsa = b->nsa;
    if (!adjoint && sae > 0 && nsteps > 0 && (it0 + 1) % sae == 0) {
        // snapshot of the state before step it0 (solver.py:194-203)
        const int slot = nsa - (it0 + 1) / sae;
        if (slot >= 0 && slot < nsa) {
            for (int c = 0; c < 3; c++) {
                const int q = b->mode == FWI_SH ? (c == 1 ? 0 : -1) : (c == 0 ? 0 : c == 2 ? 1 : 2);
                if (q < 0 || !b->snap_u[c] || (b->mode == FWI_PSV && c == 1)) continue;
                cudaError_t e = cudaMemcpyAsync(b->snap_u[c] + slot * field, b->disp[q], field * sizeof(float),
                                                cudaMemcpyDeviceToDevice, st);
                if (e != cudaSuccess) return set_error(FWI_ECUDA, "snapshot copy: %s", cudaGetErrorString(e));
            }
        }
    }
    for (int it = it0; it < it0 + nsteps; it++) {
        bool su = false, sv = false;
        int sus = 0, svs = 0;
        if (!adjoint && sae > 0) {
            if (it + 1 < it0 + nsteps && (it + 2) % sae == 0) {
                sus = nsa - (it + 2) / sae;
                su = sus >= 0 && sus < nsa;
            }
            if ((it + 1) % sae == 0) {
                svs = nsa - (it + 1) / sae;
                sv = svs >= 0 && svs < nsa;
            }
        }
        rc = launch_step(b, adjoint, it, su, sus, sv, svs, st);
        if (rc) return rc;
        b->cur ^= 1;
        if (adjoint && it % sae == 0) {
            rc = launch_interaction(b, it / sae, st);
            if (rc) return rc;
        }
    }
    return 0;
}

int fwi_run_transposed(fwi_batch *b, int it_hi, int nsteps, void *stream) {
    int rc = check_batch(b, 0, 0, 0);
    if (rc) return rc;
    REQUIRE(b->mode == FWI_SH || b->mode == FWI_PSV || b->mode == FWI_SPIN, "fwi_run_transposed: unknown mode");
    REQUIRE(nsteps >= 0 && it_hi - nsteps >= 0 && it_hi <= b->nt, "fwi_run_transposed: steps [%d, %d) outside [0, %d)",
            it_hi - nsteps, it_hi, b->nt);
    REQUIRE(it_hi - nsteps >= b->seg0 && it_hi <= b->seg0 + b->nseg,
            "fwi_run_transposed: steps [%d, %d) not stored in the segment [%d, %d)", it_hi - nsteps, it_hi, b->seg0,
            b->seg0 + b->nseg);
    const int cx = b->mode == FWI_SH ? 1 : 0;
    const int ne = b->mode == FWI_SH ? 2 : b->mode == FWI_PSV ? 3 : 6;
    // the divergence stores feed only the density terms (k_rho, spin also k_buoj)
    const bool ds = b->seg_ds[cx] && (b->mode == FWI_SH || b->seg_ds[2]) && (b->mode != FWI_SPIN || b->seg_ds[1]);
    bool stores = true;
    for (int k = 0; k < ne; k++) stores = stores && b->seg_e[k];
    REQUIRE(stores, "fwi_run_transposed: the segment stores seg_e are required");
    REQUIRE(ds || (!b->k_rho && !(b->mode == FWI_SPIN && b->k_buoj)),
            "fwi_run_transposed: the density kernels need the divergence stores seg_ds");
    REQUIRE(b->k_mu, "fwi_run_transposed: k_mu is required");
    REQUIRE(b->adj_tile == 0 || b->adj_tile == 1, "fwi_run_transposed: adj_tile must be 0 or 1 (got %d)", b->adj_tile);
    if (b->inj_ptr) {
        REQUIRE(b->inj_cell && b->inj_row, "inj_cell and inj_row are required with inj_ptr");
        REQUIRE(b->stf[cx] && (b->mode == FWI_SH || b->stf[2]), "fwi_run_transposed: trace gradients (stf) missing");
    }
    cudaStream_t st = (cudaStream_t)stream;
    // every launch after the first follows a transposed step of this loop directly
    const bool pdl = b->step_overlap != 0;
    for (int it = it_hi - 1; it >= it_hi - nsteps; it--) {
        rc = launch_adjoint_step(b, it, pdl && it < it_hi - 1, st);
        if (rc) return rc;
        b->cur ^= 1;
    }
    return 0;
}

long long fwi_multi_workspace_bytes(int n) { return multi_workspace_bytes(n); }

int fwi_multi_prepare(fwi_batch *const *batches, int n, void *workspace) {
    return multi_prepare(batches, n, workspace, check_batch);
}

int fwi_multi_run(fwi_batch *const *batches, int n, void *workspace, int it0, int nsteps, void *stream) {
    return multi_run(batches, n, workspace, it0, nsteps, (cudaStream_t)stream);
}

long long fwi_misfit_partials(int nrec, int nt) { return misfit_partials(nrec, nt); }

int fwi_misfit(const float *data, const float *syn, float *adstf, double *misfit, double *partial, int nshots,
               int nrec, int nt, double dt, void *stream) {
    REQUIRE(data && syn && adstf && misfit && partial, "fwi_misfit: NULL pointer");
    REQUIRE(nshots >= 1 && nshots <= 65535 && nrec >= 0 && nrec <= 65535 && nt >= 0,
            "fwi_misfit: nshots in [1, 65535], nrec in [0, 65535], nt >= 0");
    if (nrec == 0 || nt == 0) {
        cudaError_t e = cudaMemsetAsync(misfit, 0, sizeof(double) * nshots, (cudaStream_t)stream);
        return e == cudaSuccess ? 0 : set_error(FWI_ECUDA, "fwi_misfit: %s", cudaGetErrorString(e));
    }
    return launch_misfit(data, syn, adstf, misfit, partial, nshots, nrec, nt, dt, (cudaStream_t)stream, false);
}

int fwi_misfit_tracegrad(const float *data, const float *syn, float *grad, double *misfit, double *partial,
                         int nshots, int nrec, int nt, double dt, void *stream) {
    REQUIRE(data && syn && grad && misfit && partial, "fwi_misfit_tracegrad: NULL pointer");
    REQUIRE(nshots >= 1 && nshots <= 65535 && nrec >= 1 && nrec <= 65535 && nt >= 1,
            "fwi_misfit_tracegrad: nshots in [1, 65535], nrec in [1, 65535], nt >= 1");
    return launch_misfit(data, syn, grad, misfit, partial, nshots, nrec, nt, dt, (cudaStream_t)stream, true);
}

int fwi_trace_suffix_sum(const float *g, float *out, long long ntraces, int nt, void *stream) {
    REQUIRE(g && out, "fwi_trace_suffix_sum: NULL pointer");
    REQUIRE(ntraces >= 0 && ntraces <= 0x7fffffffll && nt >= 0, "fwi_trace_suffix_sum: ntraces in [0, 2^31), nt >= 0");
    if (ntraces == 0 || nt == 0) return 0;
    return launch_suffix_sum(g, out, ntraces, nt, (cudaStream_t)stream);
}

int fwi_energy_accumulate(const float *f, int nshots, long long field, double *acc, void *stream) {
    REQUIRE(f && acc, "fwi_energy_accumulate: NULL pointer");
    REQUIRE(nshots >= 0 && field >= 0, "fwi_energy_accumulate: negative size");
    if (!nshots || !field) return 0;
    return launch_energy(f, nshots, field, acc, (cudaStream_t)stream);
}

int fwi_smooth(const double *in, int in_pitch, float *out, int out_pitch, double *tmp, int nx, int nz, int sigma,
               void *stream) {
    REQUIRE(in && out && tmp, "fwi_smooth: NULL pointer");
    REQUIRE(nx >= 1 && nz >= 1 && in_pitch >= nz && out_pitch >= nz, "fwi_smooth: bad grid or pitch");
    REQUIRE(sigma >= 1, "fwi_smooth: sigma must be >= 1 (the reference divides by sigma)");
    REQUIRE(6ll * sigma < (1 << 20), "fwi_smooth: sigma too large");
    return launch_smooth(in, in_pitch, out, out_pitch, tmp, nx, nz, sigma, (cudaStream_t)stream);
}

}  // extern "C"
