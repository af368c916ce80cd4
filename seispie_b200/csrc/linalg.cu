// Vector kernels of the optimizer (L-BFGS / CG / line search): FP64 dot
// products of float32 model-sized vectors, FP64-scalar axpby and the max-norm.
// They replace the numpy calls of seispie/optimize/lbfgs.py:23-59,
// cg.py:20-49 and line_search/bracket.py:23-45 (np.dot, q -= al*y,
// np.amax(abs(.))).  Reductions are two-pass with a fixed block count, so
// results do not depend on scheduling.
#include "common.cuh"

namespace fwi {

constexpr int kRedBlocks = 1184;  // 148 SMs x 8
constexpr int kRedThreads = 256;

__device__ __forceinline__ double block_sum(double v, double *red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kRedThreads / 32; w++) s += red[w];
    return s;
}

__global__ void dot_kernel(const float *x, const float *y, long long n, double *partial) {
    __shared__ double red[kRedThreads / 32];
    double acc = 0.0;
    for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kRedThreads)
        acc += (double)x[i] * (double)y[i];
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void sum_finish_kernel(const double *partial, int np, double *out) {
    __shared__ double red[kRedThreads / 32];
    double acc = 0.0;
    for (int i = threadIdx.x; i < np; i += kRedThreads) acc += partial[i];
    const double s = block_sum(acc, red);
    if (threadIdx.x == 0) *out = s;
}

__global__ void absmax_kernel(const float *x, long long n, float *partial) {
    __shared__ float red[kRedThreads / 32];
    float m = 0.f;
    for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kRedThreads)
        m = fmaxf(m, fabsf(x[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float r = 0.f;
        for (int w = 0; w < kRedThreads / 32; w++) r = fmaxf(r, red[w]);
        partial[blockIdx.x] = r;
    }
}

__global__ void max_finish_kernel(const float *partial, int np, float *out) {
    __shared__ float red[kRedThreads];
    float m = 0.f;
    for (int i = threadIdx.x; i < np; i += kRedThreads) m = fmaxf(m, partial[i]);
    red[threadIdx.x] = m;
    __syncthreads();
    for (int o = kRedThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] = fmaxf(red[threadIdx.x], red[threadIdx.x + o]);
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// out = a*x + b*y, evaluated in double and rounded to float (numpy's
// float64-scalar times float32-array arithmetic).  y may be NULL (b ignored).
__global__ void axpby_kernel(float *out, double a, const float *x, double b, const float *y, long long n) {
    for (long long i = blockIdx.x * (long long)kRedThreads + threadIdx.x; i < n; i += (long long)gridDim.x * kRedThreads) {
        double v = __dmul_rn(a, (double)x[i]);  // unfused, as numpy's separate float64 operations
        if (y) v = __dadd_rn(v, __dmul_rn(b, (double)y[i]));
        out[i] = (float)v;
    }
}

static int blocks_for(long long n) {
    long long b = (n + kRedThreads - 1) / kRedThreads;
    return (int)(b < 1 ? 1 : b > kRedBlocks ? kRedBlocks : b);
}

}  // namespace fwi

using namespace fwi;

extern "C" {

long long fwi_reduce_partials(void) { return kRedBlocks; }

int fwi_dot(const float *x, const float *y, long long n, double *out, double *partial, void *stream) {
    if (!x || !y || !out || !partial || n < 0) return set_error(FWI_EINVAL, "fwi_dot: NULL pointer or negative size");
    const int nb = blocks_for(n);
    dot_kernel<<<nb, kRedThreads, 0, (cudaStream_t)stream>>>(x, y, n, partial);
    int rc = check_launch("dot");
    if (rc) return rc;
    sum_finish_kernel<<<1, kRedThreads, 0, (cudaStream_t)stream>>>(partial, nb, out);
    return check_launch("dot_finish");
}

int fwi_absmax(const float *x, long long n, float *out, float *partial, void *stream) {
    if (!x || !out || !partial || n < 0) return set_error(FWI_EINVAL, "fwi_absmax: NULL pointer or negative size");
    const int nb = blocks_for(n);
    absmax_kernel<<<nb, kRedThreads, 0, (cudaStream_t)stream>>>(x, n, partial);
    int rc = check_launch("absmax");
    if (rc) return rc;
    max_finish_kernel<<<1, kRedThreads, 0, (cudaStream_t)stream>>>(partial, nb, out);
    return check_launch("absmax_finish");
}

int fwi_axpby(float *out, double a, const float *x, double b, const float *y, long long n, void *stream) {
    if (!out || !x || n < 0) return set_error(FWI_EINVAL, "fwi_axpby: NULL pointer or negative size");
    if (n == 0) return 0;
    axpby_kernel<<<blocks_for(n), kRedThreads, 0, (cudaStream_t)stream>>>(out, a, x, b, y, n);
    return check_launch("axpby");
}

}  // extern "C"
