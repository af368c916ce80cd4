// Shared device helpers for libseispie_b200 (sm_100a).
#pragma once
#include <cuda.h>  // CUtensorMap (the driver entry point is fetched at run time)
#include <cuda_runtime.h>
#include <stdint.h>

#include "seispie_b200.h"

namespace fwi {

constexpr int kThreads = 256;  // threads per CTA of the step kernels

// Division by a run-time invariant divisor d >= 1 for 0 <= n < 2^31:
// round-up multiply-high method of Granlund & Montgomery, "Division by
// Invariant Integers using Multiplication" (PLDI 1994), Fig. 4.1.
struct FastDiv {
    uint32_t mul;
    uint32_t sh1, sh2;
    int d;
};

inline FastDiv make_fastdiv(int d) {
    FastDiv f;
    f.d = d;
    uint32_t l = 0;
    while ((1ull << l) < (unsigned long long)d) l++;
    unsigned long long m = ((1ull << 32) * ((1ull << l) - (unsigned long long)d)) / (unsigned long long)d + 1ull;
    f.mul = (uint32_t)m;
    f.sh1 = l > 0 ? 1 : 0;
    f.sh2 = l > 0 ? l - 1 : 0;
    return f;
}

__device__ __forceinline__ int fdiv(int n, const FastDiv &f) {
    uint32_t un = (uint32_t)n;
    uint32_t t = __umulhi(f.mul, un);
    return (int)((t + ((un - t) >> f.sh1)) >> f.sh2);
}

// 16-byte asynchronous global->shared copy; src_bytes == 0 zero-fills.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gmem_src, int src_bytes) {
    uint32_t s = (uint32_t)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem_src), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// mbarrier and TMA helpers shared by the step and U-Net kernels.
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
// Poll limit of the bounded waits (each translation unit has its own copy,
// set through set_wait_limit_here; fwi_set_wait_limit sets them all).
constexpr int kDefaultWaitPolls = 1 << 22;
static __device__ int g_wait_polls = kDefaultWaitPolls;

// Bounded wait: gives up after g_wait_polls polls (each poll may suspend the
// warp for a while), so a lost transaction ends the kernel instead of hanging
// it.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
    const int polls = g_wait_polls;
    for (int i = 0; i < polls; i++)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// Host: set this translation unit's poll limit (synchronous).
static inline cudaError_t set_wait_limit_here(int polls) {
    return cudaMemcpyToSymbol(g_wait_polls, &polls, sizeof(int));
}

// Programmatic dependent launch between consecutive steps of one time loop.
// A step kernel launched with the ProgrammaticStreamSerialization attribute
// may be scheduled while the previous step's kernel in the same stream is
// still running: grid_dep_trigger (at the top of every step kernel) lets the
// next launch be scheduled once every CTA of this grid has started, and
// grid_dep_wait blocks the calling thread until the previous grid has
// completed with all its memory operations visible.  Every access to the
// wavefields, the stores or the gradient comes after grid_dep_wait; only the
// barrier set-up and loads of the model (which no step writes) may precede
// it.  Without the attribute both are no-ops.
__device__ __forceinline__ void grid_dep_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// Host: the attribute (on for the launches after the first of a time loop
// whose batch sets fwi_batch.step_overlap).
inline void set_pdl_attr(cudaLaunchAttribute &at, bool on) {
    at.id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at.val.programmaticStreamSerializationAllowed = on ? 1 : 0;
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

// Untiled bulk copy global -> shared of `bytes` bytes (both addresses 16-byte
// aligned, bytes a multiple of 16), completion counted on `bar`; it lands
// in this CTA's shared memory only, so the source may be any global memory.
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// cuTensorMapEncodeTiled, fetched from the driver at run time.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_fn() {
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

// Error reporting shared by the C entry points (defined in capi.cu).
int set_error(int code, const char *fmt, ...);
int check_launch(const char *what);

// Device-side status words of the kernels with bounded waits, read (and
// optionally cleared) by fwi_device_status; each source file owns its own.
int step_device_status(int clear, int *status);
int march_device_status(int clear, int *status);
int unet_device_status(int clear, int *status);
// Poll limits of the bounded waits of step.cu, march.cu and unet.cu.
cudaError_t step_set_wait_limit(int polls);
cudaError_t march_set_wait_limit(int polls);
cudaError_t unet_set_wait_limit(int polls);

}  // namespace fwi
