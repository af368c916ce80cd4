/*
 * fd2d_oracle.c -- CPU restatement of seispie's fd2d solver path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA path in
 * seispie_b200 is compared against; it is never linked into, loaded by or
 * called from the product library.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg use it.
 *
 * It restates, step for step, the Numba kernels of the reference:
 *   seispie/solver/fd2d/solver.py:22-163   stencils, scatter, gather, interaction
 *   seispie/solver/fd2d/solver.py:166-329  forward / adjoint time loops
 *   seispie/solver/fd2d/fd2d.py:21-108     vps2lm, lm2vps, set_bound, smoothing
 *   seispie/solver/misfit/waveform.py:5-34 misfit and adjoint source
 * Every intermediate array of the reference (dsy, dvydx, ...) exists here too,
 * and the kernels run in the reference's launch order, so the arithmetic is
 * the same sequence of IEEE operations.
 *
 * The file is compiled twice (see oracle/Makefile):
 *   REAL=float   "as-reference" mode.  Under numpy 2 (NEP 50) the reference's
 *                simulator run does every operation in float32 with Python
 *                floats (dt, alpha, taper) rounded to float32 first; this mode
 *                repeats that, with -ffp-contract=off so no FMA is formed.
 *   REAL=double  FP64 oracle used to state the error of the FP32 GPU kernels.
 *
 * Grid layout is the reference's: k = i*nz + j, x index i, z index j
 * (fd2d/solver.py:14-19).  All loops over cells are independent, so the
 * OpenMP split does not change any result.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL float
#endif
typedef REAL real;

#define EXPORT __attribute__((visibility("default")))

/* ---------------------------------------------------------------- stencils */

/* diff_x: solver.py:22-27 (D_x^-) */
static inline real dxm(const real *v, int i, long k, real dx, int nx, int nz) {
    if (i >= 2 && i < nx - 2)
        return (real)9 * (v[k] - v[k - nz]) / ((real)8 * dx) - (v[k + nz] - v[k - 2 * nz]) / ((real)24 * dx);
    return 0;
}
/* diff_x1: solver.py:30-35 (D_x^+) */
static inline real dxp(const real *v, int i, long k, real dx, int nx, int nz) {
    if (i >= 1 && i < nx - 2)
        return (real)9 * (v[k + nz] - v[k]) / ((real)8 * dx) - (v[k + 2 * nz] - v[k - nz]) / ((real)24 * dx);
    return 0;
}
/* diff_z: solver.py:38-43 (D_z^-) */
static inline real dzm(const real *v, int j, long k, real dz, int nz) {
    if (j >= 2 && j < nz - 2)
        return (real)9 * (v[k] - v[k - 1]) / ((real)8 * dz) - (v[k + 1] - v[k - 2]) / ((real)24 * dz);
    return 0;
}
/* diff_z1: solver.py:46-51 (D_z^+) */
static inline real dzp(const real *v, int j, long k, real dz, int nz) {
    if (j >= 1 && j < nz - 2)
        return (real)9 * (v[k + 1] - v[k]) / ((real)8 * dz) - (v[k + 2] - v[k - 1]) / ((real)24 * dz);
    return 0;
}

#define FOR_CELLS(nx, nz)                                   \
    _Pragma("omp parallel for schedule(static)")            \
    for (int i = 0; i < (nx); i++)                          \
        for (int j = 0; j < (nz); j++)

/* div_sy: solver.py:54-58 */
static void div_sy(real *dsy, const real *sxy, const real *szy, real dx, real dz, int nx, int nz) {
    FOR_CELLS(nx, nz) {
        long k = (long)i * nz + j;
        dsy[k] = dxm(sxy, i, k, dx, nx, nz) + dzm(szy, j, k, dz, nz);
    }
}
/* div_sxz: solver.py:61-66 */
static void div_sxz(real *dsx, real *dsz, const real *sxx, const real *szz, const real *sxz,
                    real dx, real dz, int nx, int nz) {
    FOR_CELLS(nx, nz) {
        long k = (long)i * nz + j;
        dsx[k] = dxm(sxx, i, k, dx, nx, nz) + dzm(sxz, j, k, dz, nz);
        dsz[k] = dxm(sxz, i, k, dx, nx, nz) + dzm(szz, j, k, dz, nz);
    }
}
/* div_sxyz_c: solver.py:69-75 */
static void div_sxyz_c(real *dsx, real *dsz, real *dsy_c, const real *syy_c, real dx, real dz, int nx, int nz) {
    FOR_CELLS(nx, nz) {
        long k = (long)i * nz + j;
        dsx[k] += dzm(syy_c, j, k, dz, nz);
        dsz[k] -= dxm(syy_c, i, k, dx, nx, nz);
        dsy_c[k] += (real)2 * syy_c[k];
    }
}
/* stf_dsy / stf_dsxz: solver.py:78-93.  Blocks b = 0..n-1 in order; only
 * b == isrc when isrc >= 0.  ds may be NULL for an unused component. */
static void stf_add(real *ds, const real *stf, const int *ids, int n, int isrc, int it, int nt) {
    for (int b = 0; b < n; b++)
        if (isrc < 0 || isrc == b) ds[ids[b]] += stf[(long)b * nt + it];
}
/* add_vy: solver.py:95-100 (also the spin vy_c update with j in place of rho) */
static void add_vy(real *vy, real *uy, const real *dsy, const real *rho, const real *bound, real dt, long npt) {
#pragma omp parallel for schedule(static)
    for (long k = 0; k < npt; k++) {
        vy[k] = bound[k] * (vy[k] + dt * dsy[k] / rho[k]);
        uy[k] += vy[k] * dt;
    }
}
/* add_vxz: solver.py:102-109 */
static void add_vxz(real *vx, real *vz, real *ux, real *uz, const real *dsx, const real *dsz,
                    const real *rho, const real *bound, real dt, long npt) {
#pragma omp parallel for schedule(static)
    for (long k = 0; k < npt; k++) {
        vx[k] = bound[k] * (vx[k] + dt * dsx[k] / rho[k]);
        vz[k] = bound[k] * (vz[k] + dt * dsz[k] / rho[k]);
        ux[k] += vx[k] * dt;
        uz[k] += vz[k] * dt;
    }
}
/* div_vy: solver.py:112-117 */
static void div_vy(real *dvydx, real *dvydz, const real *vy, real dx, real dz, int nx, int nz) {
    FOR_CELLS(nx, nz) {
        long k = (long)i * nz + j;
        dvydx[k] = dxp(vy, i, k, dx, nx, nz);
        dvydz[k] = dzp(vy, j, k, dz, nz);
    }
}
/* div_vxz: solver.py:119-126 */
static void div_vxz(real *dvxdx, real *dvxdz, real *dvzdx, real *dvzdz, const real *vx, const real *vz,
                    real dx, real dz, int nx, int nz) {
    FOR_CELLS(nx, nz) {
        long k = (long)i * nz + j;
        dvxdx[k] = dxp(vx, i, k, dx, nx, nz);
        dvxdz[k] = dzp(vx, j, k, dz, nz);
        dvzdx[k] = dxp(vz, i, k, dx, nx, nz);
        dvzdz[k] = dzp(vz, j, k, dz, nz);
    }
}
/* add_sy: solver.py:128-133 */
static void add_sy(real *sxy, real *szy, const real *dvydx, const real *dvydz, const real *mu, real dt, long npt) {
#pragma omp parallel for schedule(static)
    for (long k = 0; k < npt; k++) {
        sxy[k] += dt * mu[k] * dvydx[k];
        szy[k] += dt * mu[k] * dvydz[k];
    }
}
/* add_sy_c: solver.py:135-141.  2*dt is a Python float product, exact in
 * both precisions; 0.5 is exact. */
static void add_sy_c(real *syx_c, real *syy_c, real *syz_c, const real *vy_c, const real *dvydx_c,
                     const real *dvydz_c, const real *dvxdz, const real *dvzdx, const real *nu,
                     const real *mu_c, const real *nu_c, real dt, real dt2, long npt) {
#pragma omp parallel for schedule(static)
    for (long k = 0; k < npt; k++) {
        syy_c[k] += dt2 * nu[k] * (-vy_c[k] - (real)0.5 * (dvzdx[k] - dvxdz[k]));
        syx_c[k] += dt * (mu_c[k] + nu_c[k]) * dvydx_c[k];
        syz_c[k] += dt * (mu_c[k] + nu_c[k]) * dvydz_c[k];
    }
}
/* add_sxz: solver.py:143-149 */
static void add_sxz(real *sxx, real *szz, real *sxz, const real *dvxdx, const real *dvxdz, const real *dvzdx,
                    const real *dvzdz, const real *lam, const real *mu, real dt, long npt) {
#pragma omp parallel for schedule(static)
    for (long k = 0; k < npt; k++) {
        sxx[k] += dt * ((lam[k] + (real)2 * mu[k]) * dvxdx[k] + lam[k] * dvzdz[k]);
        szz[k] += dt * ((lam[k] + (real)2 * mu[k]) * dvzdz[k] + lam[k] * dvxdx[k]);
        sxz[k] += dt * (mu[k] * (dvxdz[k] + dvzdx[k]));
    }
}
/* save_obs: solver.py:151-156 (receiver-major obs[b*nt + it]) */
static void save_obs(real *obs, const real *u, const int *rec_id, int nrec, int it, int nt) {
    for (int b = 0; b < nrec; b++) obs[(long)b * nt + it] = u[rec_id[b]];
}

/* ------------------------------------------------------------ model setup */

/* vps2lm: fd2d.py:21-33 (in place: lam holds vp, mu holds vs on entry) */
EXPORT void orc_vps2lm(real *lam, real *mu, const real *rho, long n) {
    for (long k = 0; k < n; k++) {
        real vp = lam[k], vs = mu[k];
        if (vp > vs) lam[k] = rho[k] * (vp * vp - (real)2 * vs * vs);
        else lam[k] = 0;
        mu[k] = rho[k] * vs * vs;
    }
}
/* lm2vps: fd2d.py:36-44 (in place: vp holds lambda, vs holds mu on entry) */
EXPORT void orc_lm2vps(real *vp, real *vs, const real *rho, long n) {
    for (long k = 0; k < n; k++) {
        real lam = vp[k], mu = vs[k];
        vp[k] = (real)sqrt((double)((lam + (real)2 * mu) / rho[k]));
        vs[k] = (real)sqrt((double)(mu / rho[k]));
    }
}
/* set_bound: fd2d.py:47-68.  aw and exp() are Python floats (double); each
 * factor is rounded to REAL before the multiply, as the simulator does. */
EXPORT void orc_set_bound(real *bound, int nx, int nz, int width, double alpha,
                          int left, int right, int bottom, int top) {
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < nz; j++) {
            long k = (long)i * nz + j;
            real b = 1;
            if (left && i + 1 < width) { double aw = alpha * (width - i - 1); b *= (real)exp(-aw * aw); }
            if (right && i > nx - width) { double aw = alpha * (width + i - nx); b *= (real)exp(-aw * aw); }
            if (bottom && j > nz - width) { double aw = alpha * (width + j - nz); b *= (real)exp(-aw * aw); }
            if (top && j + 1 < width) { double aw = alpha * (width - j - 1); b *= (real)exp(-aw * aw); }
            bound[k] = b;
        }
}

/* ----------------------------------------------------------- time loops */

/* Model parameter table, in this order (unused entries may be NULL):
 *   0 rho  1 lam  2 mu  3 bound  4 nu  5 j  6 mu_c  7 nu_c
 * State table (fields the caller owns; all npt long; zeroed here first as in
 * clear_wavefields, fd2d.py:318-341):
 *   0 vx 1 vz 2 ux 3 uz 4 sxx 5 szz 6 sxz 7 vy 8 uy 9 sxy 10 szy
 *   11 vy_c 12 uy_c 13 syx_c 14 syy_c 15 syz_c
 */
enum { P_RHO, P_LAM, P_MU, P_BOUND, P_NU, P_J, P_MUC, P_NUC };
enum { S_VX, S_VZ, S_UX, S_UZ, S_SXX, S_SZZ, S_SXZ, S_VY, S_UY, S_SXY, S_SZY,
       S_VYC, S_UYC, S_SYXC, S_SYYC, S_SYZC, S_COUNT };

typedef struct {
    real *dsx, *dsz, *dsy, *dsy_c;
    real *dvxdx, *dvxdz, *dvzdx, *dvzdz, *dvydx, *dvydz, *dvydx_c, *dvydz_c;
} scratch_t;

static void scratch_alloc(scratch_t *s, long npt) {
    real **p = (real **)s;
    for (size_t q = 0; q < sizeof(scratch_t) / sizeof(real *); q++) p[q] = (real *)calloc(npt, sizeof(real));
}
static void scratch_free(scratch_t *s) {
    real **p = (real **)s;
    for (size_t q = 0; q < sizeof(scratch_t) / sizeof(real *); q++) free(p[q]);
}

/* One time step of solver.py:205-234 (sh and/or psv[+spin]).  `ids`, `stf*`
 * and `isrc` describe the injected sources (forward: src_id/stf, isrc per
 * combine_sources; adjoint: rec_id/adstf, isrc=-1).  obs_* may be NULL (the
 * adjoint records nothing). */
static void one_step(int sh, int psv, int spin, int nx, int nz, real dx, real dz, real dt, real dt2,
                     real *const *p, real *const *s, scratch_t *w,
                     int ninj, const int *ids, const real *stf_x, const real *stf_y, const real *stf_z,
                     int isrc, int it, int nt, int nrec, const int *rec_id,
                     real *obs_x, real *obs_y, real *obs_z) {
    long npt = (long)nx * nz;
    if (sh) {
        div_sy(w->dsy, s[S_SXY], s[S_SZY], dx, dz, nx, nz);
        stf_add(w->dsy, stf_y, ids, ninj, isrc, it, nt);
        add_vy(s[S_VY], s[S_UY], w->dsy, p[P_RHO], p[P_BOUND], dt, npt);
        div_vy(w->dvydx, w->dvydz, s[S_VY], dx, dz, nx, nz);
        add_sy(s[S_SXY], s[S_SZY], w->dvydx, w->dvydz, p[P_MU], dt, npt);
        if (obs_y) save_obs(obs_y, s[S_UY], rec_id, nrec, it, nt);
    }
    if (psv) {
        div_sxz(w->dsx, w->dsz, s[S_SXX], s[S_SZZ], s[S_SXZ], dx, dz, nx, nz);
        if (spin) {
            div_sy(w->dsy_c, s[S_SYXC], s[S_SYZC], dx, dz, nx, nz);
            div_sxyz_c(w->dsx, w->dsz, w->dsy_c, s[S_SYYC], dx, dz, nx, nz);
        }
        /* stf_dsxz adds x then z for each block */
        for (int b = 0; b < ninj; b++)
            if (isrc < 0 || isrc == b) {
                w->dsx[ids[b]] += stf_x[(long)b * nt + it];
                w->dsz[ids[b]] += stf_z[(long)b * nt + it];
            }
        add_vxz(s[S_VX], s[S_VZ], s[S_UX], s[S_UZ], w->dsx, w->dsz, p[P_RHO], p[P_BOUND], dt, npt);
        div_vxz(w->dvxdx, w->dvxdz, w->dvzdx, w->dvzdz, s[S_VX], s[S_VZ], dx, dz, nx, nz);
        add_sxz(s[S_SXX], s[S_SZZ], s[S_SXZ], w->dvxdx, w->dvxdz, w->dvzdx, w->dvzdz, p[P_LAM], p[P_MU], dt, npt);
        if (spin) {
            add_vy(s[S_VYC], s[S_UYC], w->dsy_c, p[P_J], p[P_BOUND], dt, npt);
            div_vy(w->dvydx_c, w->dvydz_c, s[S_VYC], dx, dz, nx, nz);
            add_sy_c(s[S_SYXC], s[S_SYYC], s[S_SYZC], s[S_VYC], w->dvydx_c, w->dvydz_c, w->dvxdz, w->dvzdx,
                     p[P_NU], p[P_MUC], p[P_NUC], dt, dt2, npt);
        }
        if (obs_x) save_obs(obs_x, s[S_UX], rec_id, nrec, it, nt);
        if (obs_z) save_obs(obs_z, s[S_UZ], rec_id, nrec, it, nt);
        if (spin && obs_y) save_obs(obs_y, s[S_UYC], rec_id, nrec, it, nt);
    }
}

static void clear_state(real *const *s, long npt) {
    for (int q = 0; q < S_COUNT; q++)
        if (s[q]) memset(s[q], 0, npt * sizeof(real));
}

/* run_forward: solver.py:166-242.  Snapshot arrays snap_* are [nsa][npt]
 * (may be NULL).  The u snapshot of slot nsa-(it+1)/sae is taken before step
 * it whenever (it+1) % sae == 0; v snapshots are taken after that step, as the
 * reference does (solver.py:193-203, 236-242). */
EXPORT void orc_forward(int sh, int psv, int spin, int nx, int nz, double dx_, double dz_, double dt_, int nt,
                        real *const *p, real *const *s,
                        int nsrc, const int *src_id, const real *stf_x, const real *stf_y, const real *stf_z,
                        int isrc, int nrec, const int *rec_id, real *obs_x, real *obs_y, real *obs_z,
                        int sae, int nsa, real *snap_ux, real *snap_uz, real *snap_uy,
                        real *snap_vx, real *snap_vz, real *snap_vy) {
    real dx = (real)dx_, dz = (real)dz_, dt = (real)dt_, dt2 = (real)(2.0 * dt_);
    long npt = (long)nx * nz;
    scratch_t w;
    scratch_alloc(&w, npt);
    clear_state(s, npt);
    for (int it = 0; it < nt; it++) {
        int isa = -1;
        if (sae && (it + 1) % sae == 0) isa = nsa - (it + 1) / sae;
        if (isa >= 0) {
            if (sh && snap_uy) memcpy(snap_uy + (long)isa * npt, s[S_UY], npt * sizeof(real));
            if (psv && snap_ux) memcpy(snap_ux + (long)isa * npt, s[S_UX], npt * sizeof(real));
            if (psv && snap_uz) memcpy(snap_uz + (long)isa * npt, s[S_UZ], npt * sizeof(real));
        }
        one_step(sh, psv, spin, nx, nz, dx, dz, dt, dt2, p, s, &w, nsrc, src_id, stf_x, stf_y, stf_z,
                 isrc, it, nt, nrec, rec_id, obs_x, obs_y, obs_z);
        if (isa >= 0) {
            if (sh && snap_vy) memcpy(snap_vy + (long)isa * npt, s[S_VY], npt * sizeof(real));
            if (psv && snap_vx) memcpy(snap_vx + (long)isa * npt, s[S_VX], npt * sizeof(real));
            if (psv && snap_vz) memcpy(snap_vz + (long)isa * npt, s[S_VZ], npt * sizeof(real));
        }
    }
    scratch_free(&w);
}

/* run_adjoint, SH branch: solver.py:290-321.  The adjoint source adstf_y
 * [nrec*nt] is injected at rec_id for every receiver; every sae steps the
 * displacement gradients of the adjoint field and of snapshot uy_fwd[it/sae]
 * are correlated into k_mu (interaction_muy, solver.py:159-163) with
 * ndt = sae*dt. */
EXPORT void orc_adjoint_sh(int nx, int nz, double dx_, double dz_, double dt_, int nt,
                           real *const *p, real *const *s, int nrec, const int *rec_id, const real *adstf_y,
                           int sae, const real *uy_fwd, real *k_mu) {
    real dx = (real)dx_, dz = (real)dz_, dt = (real)dt_;
    real ndt = (real)(sae * dt_);
    long npt = (long)nx * nz;
    scratch_t w;
    scratch_alloc(&w, npt);
    real *fw_dx = (real *)calloc(npt, sizeof(real)), *fw_dz = (real *)calloc(npt, sizeof(real));
    clear_state(s, npt);
    for (int it = 0; it < nt; it++) {
        one_step(1, 0, 0, nx, nz, dx, dz, dt, dt, p, s, &w, nrec, rec_id, NULL, adstf_y, NULL,
                 -1, it, nt, 0, NULL, NULL, NULL, NULL);
        if ((it + sae) % sae == 0) {
            int isae = (it + sae) / sae - 1;
            const real *u = uy_fwd + (long)isae * npt;
            div_vy(w.dvydx, w.dvydz, s[S_UY], dx, dz, nx, nz);
            div_vy(fw_dx, fw_dz, u, dx, dz, nx, nz);
#pragma omp parallel for schedule(static)
            for (long k = 0; k < npt; k++)
                k_mu[k] += (w.dvydx[k] * fw_dx[k] + w.dvydz[k] * fw_dz[k]) * ndt;
        }
    }
    free(fw_dx);
    free(fw_dz);
    scratch_free(&w);
}

/* P-SV adjoint.  The reference's P-SV branch (solver.py:324-329) cannot run
 * (it names undefined isrc/rho/bound and re-injects the forward source), so
 * this is the definition the GPU kernel implements: the SH recipe carried to
 * P-SV.  The adjoint sources adstf_x / adstf_z are injected at rec_id and,
 * every sae steps, the displacement strains of the adjoint field and of
 * snapshot slot it/sae are correlated with ndt = sae*dt:
 *   k_lam += (exx' + ezz') (exx + ezz)
 *   k_mu  += 2 (exx' exx + ezz' ezz) + (exz') (exz)        exz = Dz+ux + Dx+uz
 *   k_rho += vx' vx + vz' vz                                (velocity snapshots)
 * with e.. = D+ of ux/uz as in div_vxz.  Accumulators are REAL. */
EXPORT void orc_adjoint_psv(int nx, int nz, double dx_, double dz_, double dt_, int nt,
                            real *const *p, real *const *s, int nrec, const int *rec_id,
                            const real *adstf_x, const real *adstf_z, int sae,
                            const real *ux_fwd, const real *uz_fwd, const real *vx_fwd, const real *vz_fwd,
                            real *k_lam, real *k_mu, real *k_rho) {
    real dx = (real)dx_, dz = (real)dz_, dt = (real)dt_;
    real ndt = (real)(sae * dt_);
    long npt = (long)nx * nz;
    scratch_t w, f;
    scratch_alloc(&w, npt);
    scratch_alloc(&f, npt);
    clear_state(s, npt);
    for (int it = 0; it < nt; it++) {
        one_step(0, 1, 0, nx, nz, dx, dz, dt, dt, p, s, &w, nrec, rec_id, adstf_x, NULL, adstf_z,
                 -1, it, nt, 0, NULL, NULL, NULL, NULL);
        if ((it + sae) % sae == 0) {
            int isae = (it + sae) / sae - 1;
            div_vxz(w.dvxdx, w.dvxdz, w.dvzdx, w.dvzdz, s[S_UX], s[S_UZ], dx, dz, nx, nz);
            div_vxz(f.dvxdx, f.dvxdz, f.dvzdx, f.dvzdz, ux_fwd + (long)isae * npt, uz_fwd + (long)isae * npt,
                    dx, dz, nx, nz);
            const real *fvx = vx_fwd ? vx_fwd + (long)isae * npt : NULL;
            const real *fvz = vz_fwd ? vz_fwd + (long)isae * npt : NULL;
#pragma omp parallel for schedule(static)
            for (long k = 0; k < npt; k++) {
                real ea = w.dvxdx[k] + w.dvzdz[k], eb = f.dvxdx[k] + f.dvzdz[k];
                real sa = w.dvxdz[k] + w.dvzdx[k], sb = f.dvxdz[k] + f.dvzdx[k];
                if (k_lam) k_lam[k] += ea * eb * ndt;
                if (k_mu) k_mu[k] += ((real)2 * (w.dvxdx[k] * f.dvxdx[k] + w.dvzdz[k] * f.dvzdz[k]) + sa * sb) * ndt;
                if (k_rho && fvx) k_rho[k] += (s[S_VX][k] * fvx[k] + s[S_VZ][k] * fvz[k]) * ndt;
            }
        }
    }
    scratch_free(&w);
    scratch_free(&f);
}

/* -------------------------------------------------------- misfit, smooth */

/* diff + waveform: waveform.py:5-34.  syn holds the observed data, obs the
 * current synthetic (the reference's naming).  The taper is a Python float
 * rounded to REAL before use.  Returns ||r||_2 accumulated in double. */
EXPORT double orc_misfit(const real *syn, const real *obs, real *adstf, real *resid, int nt, double dt, int nrec) {
    double t_end = (nt - 1) * dt, tw = t_end / 10, t_min = tw, t_max = t_end - tw;
    double acc = 0;
    for (int it = 0; it < nt; it++) {
        double t = it * dt, taper;
        if (t <= t_min) taper = 0.5 + 0.5 * cos(M_PI * (t_min - t) / tw);
        else if (t >= t_max) taper = 0.5 + 0.5 * cos(M_PI * (t_max - t) / tw);
        else taper = 1;
        real tp = (real)taper;
        for (int ir = 0; ir < nrec; ir++) {
            long kt = (long)ir * nt + it, akt = (long)ir * nt + nt - it - 1;
            real r = (syn[kt] - obs[kt]) * tp;
            if (resid) resid[kt] = r;
            adstf[akt] = r * tp * (real)2;
            acc += (double)r * (double)r;
        }
    }
    return sqrt(acc);
}

/* gaussian: fd2d.py:71-73 (Python float arithmetic) */
static double gaussian(double x, double sigma) {
    return (1 / (sqrt(2 * M_PI) * sigma)) * exp(-x * x / (2 * sigma * sigma));
}

/* init_gausian + apply_gauxxian_x/z: fd2d.py:76-108, smooth fd2d.py:349-352.
 * Full-width sums in the reference's order.  Each product of a Python-float
 * weight and a REAL sample is a REAL operation, and so is the running sum
 * (the simulator starts from int 0 and then carries numpy float32). */
EXPORT void orc_smooth(real *data, int nx, int nz, int sigma) {
    long npt = (long)nx * nz;
    real *gsum = (real *)malloc(npt * sizeof(real)), *gtmp = (real *)malloc(npt * sizeof(real));
    double s = sigma;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < nz; j++) {
            double sx = 0, sz = 0;
            for (int n = 0; n < nx; n++) sx += gaussian(i - n, s);
            for (int n = 0; n < nz; n++) sz += gaussian(j - n, s);
            gsum[(long)i * nz + j] = (real)(sx * sz);
        }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < nz; j++) {
            real acc = 0;
            for (int n = 0; n < nx; n++) acc = acc + (real)gaussian(i - n, s) * data[(long)n * nz + j];
            gtmp[(long)i * nz + j] = acc;
        }
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; i++)
        for (int j = 0; j < nz; j++) {
            real acc = 0;
            for (int n = 0; n < nz; n++) acc = acc + (real)gaussian(j - n, s) * gtmp[(long)i * nz + n];
            data[(long)i * nz + j] = acc / gsum[(long)i * nz + j];
        }
    free(gsum);
    free(gtmp);
}

EXPORT int orc_real_size(void) { return (int)sizeof(real); }
