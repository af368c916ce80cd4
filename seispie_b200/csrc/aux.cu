// Non-stencil kernels of the FWI path: model set-up, source-time functions,
// adjoint interaction (sensitivity kernels), misfit / adjoint source and
// Gaussian smoothing.  Each cites the reference code it replaces.
#include <cmath>

#include "common.cuh"

namespace fwi {

// ----------------------------------------------------------- model set-up

// vps2lm, fd2d.py:21-33.  Explicit _rn intrinsics keep the reference's
// float32 rounding sequence (no FMA contraction): lam = rho*(vp*vp - (2*vs)*vs).
__global__ void vps2lm_kernel(float *lam, float *mu, const float *rho, long long n) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const float vp = lam[k], vs = mu[k], r = rho[k];
        lam[k] = vp > vs ? __fmul_rn(r, __fsub_rn(__fmul_rn(vp, vp), __fmul_rn(__fmul_rn(2.f, vs), vs))) : 0.f;
        mu[k] = __fmul_rn(__fmul_rn(r, vs), vs);
    }
}

// lm2vps, fd2d.py:36-44
__global__ void lm2vps_kernel(float *vp, float *vs, const float *rho, long long n) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        const float lam = vp[k], mu = vs[k], r = rho[k];
        vp[k] = sqrtf(__fdiv_rn(__fadd_rn(lam, __fmul_rn(2.f, mu)), r));
        vs[k] = sqrtf(__fdiv_rn(mu, r));
    }
}

// set_bound, fd2d.py:47-68: each Gaussian factor is a double, rounded to
// float before the float multiply.
__global__ void bound_kernel(float *bound, int nx, int nz, int pitch, int width, double alpha, int left, int right,
                             int bottom, int top) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= pitch) return;
    float b = 1.f;
    if (j >= nz) {
        b = 0.f;  // row padding stays zero
    } else {
        if (left && i + 1 < width) {
            const double aw = alpha * (double)(width - i - 1);
            b = __fmul_rn(b, (float)exp(-aw * aw));
        }
        if (right && i > nx - width) {
            const double aw = alpha * (double)(width + i - nx);
            b = __fmul_rn(b, (float)exp(-aw * aw));
        }
        if (bottom && j > nz - width) {
            const double aw = alpha * (double)(width + j - nz);
            b = __fmul_rn(b, (float)exp(-aw * aw));
        }
        if (top && j + 1 < width) {
            const double aw = alpha * (double)(width - j - 1);
            b = __fmul_rn(b, (float)exp(-aw * aw));
        }
    }
    bound[(long long)i * pitch + j] = b;
}

// ricker, ricker.py:7-11, evaluated for t = it*dt as import_sources does
// (fd2d.py:136-138).  Products are kept unfused to follow numpy's rounding.
__global__ void ricker_kernel(const double *par, int nsrc, int nt, double dt, float *sx, float *sy, float *sz) {
    const int it = blockIdx.x * blockDim.x + threadIdx.x, s = blockIdx.y;
    if (it >= nt || s >= nsrc) return;
    const double f0 = par[4 * s], t0 = par[4 * s + 1], ang = par[4 * s + 2], amp = par[4 * s + 3];
    const double t = __dmul_rn((double)it, dt);
    const double pf = __dmul_rn(M_PI, f0);
    const double a = __dmul_rn(pf, pf);
    const double tt = __dsub_rn(t, t0);
    const double tt2 = __dmul_rn(tt, tt);
    const double poly = __dsub_rn(1.0, __dmul_rn(__dmul_rn(2.0, a), tt2));
    const double stf = __dmul_rn(__dmul_rn(-amp, poly), exp(__dmul_rn(-a, tt2)));
    const double rad = __dmul_rn(ang, M_PI / 180.0);
    const long long k = (long long)s * nt + it;
    if (sx) sx[k] = (float)__dmul_rn(stf, sin(rad));
    if (sy) sy[k] = (float)stf;
    if (sz) sz[k] = (float)__dmul_rn(-stf, cos(rad));
}

// Derived per-cell arrays for the step kernel.
__global__ void prepare_kernel(const float *rho, const float *jr, const float *muc, const float *nuc, float dt,
                               long long n, float *buo, float *buo_j, float *mnc) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x) {
        buo[k] = rho[k] != 0.f ? __fdiv_rn(dt, rho[k]) : 0.f;
        if (buo_j) buo_j[k] = jr[k] != 0.f ? __fdiv_rn(dt, jr[k]) : 0.f;
        if (mnc) mnc[k] = __fadd_rn(muc[k], nuc[k]);
    }
}

// ------------------------------------------------------ adjoint interaction

struct DerivCoef {
    float cx1, cx2, cz1, cz2;
};

__device__ __forceinline__ float dxp(const float *u, long long g, int pitch, bool ok, const DerivCoef &c) {
    return ok ? c.cx1 * (u[g + pitch] - u[g]) - c.cx2 * (u[g + 2 * pitch] - u[g - pitch]) : 0.f;
}
__device__ __forceinline__ float dzp(const float *u, long long g, bool ok, const DerivCoef &c) {
    return ok ? c.cz1 * (u[g + 1] - u[g]) - c.cz2 * (u[g + 2] - u[g - 1]) : 0.f;
}

// interaction_muy, solver.py:159-163 with the D+ gradients of solver.py:319-320:
// k_mu += (Dx+ u' Dx+ u + Dz+ u' Dz+ u) * ndt, summed over the batch's shots.
__global__ void interaction_sh_kernel(const float *__restrict__ ua, const float *__restrict__ uf, double *k_mu, int nx,
                                      int nz, int pitch, int nshots, DerivCoef c, double ndt) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= nz) return;
    const bool okx = i >= 1 && i < nx - 2, okz = j >= 1 && j < nz - 2;
    const long long o = (long long)i * pitch + j, field = (long long)nx * pitch;
    double acc = k_mu[o];
    for (int s = 0; s < nshots; s++) {
        const long long g = s * field + o;
        const float ax = dxp(ua, g, pitch, okx, c), az = dzp(ua, g, okz, c);
        const float fx = dxp(uf, g, pitch, okx, c), fz = dzp(uf, g, okz, c);
        acc += ((double)ax * fx + (double)az * fz) * ndt;
    }
    k_mu[o] = acc;
}

// P-SV interaction (no counterpart in the reference, whose P-SV adjoint
// branch solver.py:324-329 cannot run): strains of the adjoint and forward
// displacement from D+ as in div_vxz (solver.py:119-126), correlated every
// sae steps with ndt = sae*dt:
//   k_lam += (exx'+ezz')(exx+ezz),  k_mu += 2(exx' exx + ezz' ezz) + exz' exz,
//   k_rho += vx' vx + vz' vz   (exz = Dz+ ux + Dx+ uz).
__global__ void interaction_psv_kernel(const float *__restrict__ uxa, const float *__restrict__ uza,
                                       const float *__restrict__ uxf, const float *__restrict__ uzf,
                                       const float *__restrict__ vxa, const float *__restrict__ vza,
                                       const float *__restrict__ vxf, const float *__restrict__ vzf, double *k_lam,
                                       double *k_mu, double *k_rho, int nx, int nz, int pitch, int nshots, DerivCoef c,
                                       double ndt) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= nz) return;
    const bool okx = i >= 1 && i < nx - 2, okz = j >= 1 && j < nz - 2;
    const long long o = (long long)i * pitch + j, field = (long long)nx * pitch;
    double al = k_lam ? k_lam[o] : 0.0, am = k_mu ? k_mu[o] : 0.0, ar = k_rho ? k_rho[o] : 0.0;
    const bool rho = k_rho && vxf && vzf;
    for (int s = 0; s < nshots; s++) {
        const long long g = s * field + o;
        const float axx = dxp(uxa, g, pitch, okx, c), axz = dzp(uxa, g, okz, c);
        const float azx = dxp(uza, g, pitch, okx, c), azz = dzp(uza, g, okz, c);
        const float fxx = dxp(uxf, g, pitch, okx, c), fxz = dzp(uxf, g, okz, c);
        const float fzx = dxp(uzf, g, pitch, okx, c), fzz = dzp(uzf, g, okz, c);
        const double ea = (double)(axx + azz), eb = (double)(fxx + fzz);
        const double sa = (double)(axz + azx), sb = (double)(fxz + fzx);
        al += ea * eb * ndt;
        am += (2.0 * ((double)axx * fxx + (double)azz * fzz) + sa * sb) * ndt;
        if (rho) ar += ((double)vxa[g] * vxf[g] + (double)vza[g] * vzf[g]) * ndt;
    }
    if (k_lam) k_lam[o] = al;
    if (k_mu) k_mu[o] = am;
    if (k_rho) k_rho[o] = ar;
}

int launch_interaction(const fwi_batch *b, int isae, cudaStream_t st) {
    DerivCoef c;
    c.cx1 = (float)(9.0 / (8.0 * (double)b->dx));
    c.cx2 = (float)(1.0 / (24.0 * (double)b->dx));
    c.cz1 = (float)(9.0 / (8.0 * (double)b->dz));
    c.cz2 = (float)(1.0 / (24.0 * (double)b->dz));
    const double ndt = (double)b->sae * b->dt;
    const long long field = (long long)b->nshots * b->nx * b->pitch;
    dim3 grid((b->nz + 127) / 128, b->nx);
    if (b->mode == FWI_SH) {
        if (!b->k_mu) return 0;
        interaction_sh_kernel<<<grid, 128, 0, st>>>(b->disp[0], b->snap_u[1] + isae * field, b->k_mu, b->nx, b->nz,
                                                     b->pitch, b->nshots, c, ndt);
    } else {
        const float *vxf = b->snap_v[0] ? b->snap_v[0] + isae * field : nullptr;
        const float *vzf = b->snap_v[2] ? b->snap_v[2] + isae * field : nullptr;
        interaction_psv_kernel<<<grid, 128, 0, st>>>(b->disp[0], b->disp[1], b->snap_u[0] + isae * field,
                                                      b->snap_u[2] + isae * field, b->vel[b->cur][0],
                                                      b->vel[b->cur][1], vxf, vzf, b->k_lam, b->k_mu, b->k_rho,
                                                      b->nx, b->nz, b->pitch, b->nshots, c, ndt);
    }
    return check_launch("interaction");
}

// ------------------------------------------------------ misfit / adjoint src

constexpr int kMisfitBlock = 256;

// diff, waveform.py:5-25.  One thread per (shot, receiver, sample).  The
// Hann-taper weight is computed in double and rounded to float before use,
// as the float32 arithmetic of the reference does.
// GRAD = true writes, instead of the time-reversed adjoint source, the
// derivative of chi = sum taper^2 (syn - data)^2 with respect to each trace
// sample in forward time order: 2 taper^2 (syn - data) = -adstf reversed
// (the input of the exact adjoint, fwi_run_transposed).
template <bool GRAD>
__global__ void misfit_kernel(const float *data, const float *syn, float *adstf, double *partial, int nrec, int nt,
                              double dt) {
    __shared__ double red[kMisfitBlock / 32];
    const int it = blockIdx.x * kMisfitBlock + threadIdx.x;
    const long long row = (long long)blockIdx.z * nrec + blockIdx.y;
    double sq = 0.0;
    if (it < nt) {
        const double t_end = (nt - 1) * dt, tw = t_end / 10, t_min = tw, t_max = t_end - tw, t = it * dt;
        double taper = 1.0;
        if (t <= t_min) taper = 0.5 + 0.5 * cos(M_PI * (t_min - t) / tw);
        else if (t >= t_max) taper = 0.5 + 0.5 * cos(M_PI * (t_max - t) / tw);
        const float tp = (float)taper;
        const long long kt = row * nt + it;
        const float r = __fmul_rn(__fsub_rn(data[kt], syn[kt]), tp);
        const float a = __fmul_rn(__fmul_rn(r, tp), 2.f);
        if (GRAD) adstf[kt] = -a;
        else adstf[row * nt + nt - it - 1] = a;
        sq = (double)r * (double)r;
    }
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xffffffffu, sq, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < kMisfitBlock / 32; w++) s += red[w];
        partial[row * gridDim.x + blockIdx.x] = s;
    }
}

// np.linalg.norm of the residual (waveform.py:34), per shot, fixed order.
__global__ void misfit_finish_kernel(const double *partial, double *misfit, long long per_shot) {
    __shared__ double red[256];
    const double *p = partial + blockIdx.x * per_shot;
    double s = 0.0;
    for (long long q = threadIdx.x; q < per_shot; q += 256) s += p[q];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = 128; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) misfit[blockIdx.x] = sqrt(red[0]);
}

long long misfit_partials(int nrec, int nt) { return (long long)nrec * ((nt + kMisfitBlock - 1) / kMisfitBlock); }

int launch_misfit(const float *data, const float *syn, float *adstf, double *misfit, double *partial, int nshots,
                  int nrec, int nt, double dt, cudaStream_t st, bool grad) {
    dim3 grid((nt + kMisfitBlock - 1) / kMisfitBlock, nrec, nshots);
    if (grad) misfit_kernel<true><<<grid, kMisfitBlock, 0, st>>>(data, syn, adstf, partial, nrec, nt, dt);
    else misfit_kernel<false><<<grid, kMisfitBlock, 0, st>>>(data, syn, adstf, partial, nrec, nt, dt);
    int rc = check_launch("misfit");
    if (rc) return rc;
    misfit_finish_kernel<<<nshots, 256, 0, st>>>(partial, misfit, misfit_partials(nrec, nt));
    return check_launch("misfit_finish");
}

// Suffix sums along time of every trace: out[t] = sum_{s >= t} g[s], one CTA
// per trace walking 256-sample chunks from the end; an FP64 scan inside each
// chunk (warp shuffles, then the warp totals) plus the running carry, so the
// result does not depend on the launch and out may alias g.
__global__ void suffix_sum_kernel(const float *g, float *out, int nt) {
    __shared__ double wsum[8];
    const long long base = (long long)blockIdx.x * nt;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double carry = 0.0;
    for (int end = nt; end > 0; end -= 256) {
        const int t = end - 1 - tid;  // thread i holds the i-th sample counted from the end of the chunk
        double v = t >= 0 ? (double)g[base + t] : 0.0;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double u = __shfl_up_sync(0xffffffffu, v, d);
            if (lane >= d) v += u;
        }
        if (lane == 31) wsum[warp] = v;
        __syncthreads();
        double before = carry, total = carry;
        for (int w = 0; w < 8; w++) {
            if (w < warp) before += wsum[w];
            total += wsum[w];
        }
        if (t >= 0) out[base + t] = (float)(before + v);
        carry = total;
        __syncthreads();
    }
}

// acc[i] += sum over shots s of f[s*field + i]^2 (FP64), shots in order.
__global__ void energy_kernel(const float *f, int nshots, long long field, double *acc) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < field; i += (long long)gridDim.x * blockDim.x) {
        double s = acc[i];
        for (int k = 0; k < nshots; k++) {
            const double v = f[k * field + i];
            s += v * v;
        }
        acc[i] = s;
    }
}

int launch_energy(const float *f, int nshots, long long field, double *acc, cudaStream_t st) {
    long long b = (field + 255) / 256;
    energy_kernel<<<(unsigned)(b > 4736 ? 4736 : b < 1 ? 1 : b), 256, 0, st>>>(f, nshots, field, acc);
    return check_launch("energy");
}

int launch_suffix_sum(const float *g, float *out, long long ntraces, int nt, cudaStream_t st) {
    suffix_sum_kernel<<<(unsigned)ntraces, 256, 0, st>>>(g, out, nt);
    return check_launch("suffix_sum");
}

// ---------------------------------------------------------------- smoothing
// init_gausian / apply_gauxxian_x / apply_gauxxian_z, fd2d.py:76-108.
// gaussian(d) = exp(-d^2 / (2 sigma^2)) / (sqrt(2 pi) sigma), fd2d.py:71-73.

__device__ __forceinline__ double gauss_w(int d, double sigma) {
    return (1.0 / (sqrt(2.0 * M_PI) * sigma)) * exp(-(double)d * d / (2.0 * sigma * sigma));
}

// Pass 1 (x): tmp[i][j] = sum_n w(i-n) in[n][j]
__global__ void smooth_x_kernel(const double *in, int in_pitch, double *tmp, int nx, int nz, int R, double sigma) {
    extern __shared__ double w[];
    for (int d = threadIdx.x; d <= R; d += blockDim.x) w[d] = gauss_w(d, sigma);
    __syncthreads();
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= nz) return;
    const int n0 = max(0, i - R), n1 = min(nx - 1, i + R);
    double s = 0.0;
    for (int n = n0; n <= n1; n++) s += w[abs(i - n)] * in[(long long)n * in_pitch + j];
    tmp[(long long)i * nz + j] = s;
}

// Pass 2 (z) and normalisation by the in-grid Gaussian mass gsum = Sx(i) Sz(j).
__global__ void smooth_z_kernel(const double *tmp, float *out, int out_pitch, int nx, int nz, int R, double sigma) {
    extern __shared__ double w[];
    for (int d = threadIdx.x; d <= R; d += blockDim.x) w[d] = gauss_w(d, sigma);
    __syncthreads();
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= nz) return;
    const int n0 = max(0, j - R), n1 = min(nz - 1, j + R);
    double s = 0.0, sz = 0.0, sx = 0.0;
    const double *row = tmp + (long long)i * nz;
    for (int n = n0; n <= n1; n++) {
        s += w[abs(j - n)] * row[n];
        sz += w[abs(j - n)];
    }
    for (int n = max(0, i - R); n <= min(nx - 1, i + R); n++) sx += w[abs(i - n)];
    out[(long long)i * out_pitch + j] = (float)(s / (sx * sz));
}

int launch_smooth(const double *in, int in_pitch, float *out, int out_pitch, double *tmp, int nx, int nz, int sigma,
                  cudaStream_t st) {
    const int R = min((int)ceil(6.0 * sigma), max(nx, nz));
    const size_t sm = sizeof(double) * (R + 1);
    if (sm > 48 * 1024) return set_error(FWI_ERANGE, "fwi_smooth: truncation radius %d exceeds 6143 taps", R);
    dim3 grid((nz + 127) / 128, nx);
    smooth_x_kernel<<<grid, 128, sm, st>>>(in, in_pitch, tmp, nx, nz, R, (double)sigma);
    int rc = check_launch("smooth_x");
    if (rc) return rc;
    smooth_z_kernel<<<grid, 128, sm, st>>>(tmp, out, out_pitch, nx, nz, R, (double)sigma);
    return check_launch("smooth_z");
}

// ---------------------------------------------------------------- launchers

static dim3 elem_grid(long long n) {
    long long b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    if (b < 1) b = 1;
    return dim3((unsigned)b);
}

int launch_vps2lm(float *lam, float *mu, const float *rho, long long n, cudaStream_t st) {
    vps2lm_kernel<<<elem_grid(n), 256, 0, st>>>(lam, mu, rho, n);
    return check_launch("vps2lm");
}
int launch_lm2vps(float *vp, float *vs, const float *rho, long long n, cudaStream_t st) {
    lm2vps_kernel<<<elem_grid(n), 256, 0, st>>>(vp, vs, rho, n);
    return check_launch("lm2vps");
}
int launch_bound(float *bound, int nx, int nz, int pitch, int width, double alpha, int l, int r, int b, int t,
                 cudaStream_t st) {
    dim3 grid((pitch + 127) / 128, nx);
    bound_kernel<<<grid, 128, 0, st>>>(bound, nx, nz, pitch, width, alpha, l, r, b, t);
    return check_launch("set_bound");
}
int launch_ricker(const double *par, int nsrc, int nt, double dt, float *sx, float *sy, float *sz, cudaStream_t st) {
    dim3 grid((nt + 127) / 128, nsrc);
    ricker_kernel<<<grid, 128, 0, st>>>(par, nsrc, nt, dt, sx, sy, sz);
    return check_launch("ricker");
}
int launch_prepare(const float *rho, const float *jr, const float *muc, const float *nuc, double dt, long long n,
                   float *buo, float *buo_j, float *mnc, cudaStream_t st) {
    prepare_kernel<<<elem_grid(n), 256, 0, st>>>(rho, jr, muc, nuc, (float)dt, n, buo, buo_j, mnc);
    return check_launch("prepare_model");
}

}  // namespace fwi
