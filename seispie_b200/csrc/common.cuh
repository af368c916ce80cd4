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

// Error reporting shared by the C entry points (defined in capi.cu).
int set_error(int code, const char *fmt, ...);
int check_launch(const char *what);

}  // namespace fwi
