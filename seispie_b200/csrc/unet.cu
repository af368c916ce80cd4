// Kernels of the learned preconditioner: a small U-Net in BF16 (weights and
// activations) with FP32 accumulation, for training and inference.  No
// counterpart in the reference, which has no learned component.
//
// Layout.  Activations are NHWC bf16 ([image][row][column][channel]) with a
// channel count that is a multiple of 16, so one pixel's channels are whole
// 16-byte vectors.  3x3 convolution weights are [tap][out channel][in
// channel] bf16 (tap = 3*(dy+1) + (dx+1), input channel innermost), biases
// and all gradients FP32.
//
// Convolutions are implicit GEMMs on the tensor cores (warp-level
// mma.sync m16n8k16, bf16 x bf16 -> f32): M = pixels, N = output channels,
// K = 9 taps x input channels.  A CTA owns 128 pixels (16 per warp) and up to
// 64 output channels; it stages one (tap, 16-channel) slice of the shifted
// input and of the weights per step with cp.async, double-buffered, and feeds
// the fragments with ldmatrix.  The data gradient is the same kernel run on
// the flipped, transposed weights; the weight gradient reduces over pixels
// in fixed blocks whose partial sums are added in block order, so training is
// deterministic.
#include <cuda_bf16.h>

#include "common.cuh"

namespace fwi {
namespace unet {

using bf16 = __nv_bfloat16;

constexpr int kCT = 256;  // threads of a convolution CTA
constexpr int kBM = 128;  // pixels per convolution CTA (16 per warp)
constexpr int kAS = 24;   // shared row stride (bf16) of a 16-channel row: 48 bytes, conflict-free ldmatrix
constexpr int kWgPix = 2048;  // pixels per weight-gradient block
constexpr int kRedPix = 4096;  // pixels per bias / head reduction block

struct Shape {
    int n, h, w;  // images, rows, columns
};

__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(su32(p)));
}
__device__ __forceinline__ void ldsm_x2(uint32_t (&r)[2], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.shared.b16 {%0,%1}, [%2];\n" : "=r"(r[0]), "=r"(r[1]) : "r"(su32(p)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(su32(p)));
}
__device__ __forceinline__ void ldsm_x2_t(uint32_t (&r)[2], const void *p) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x2.trans.shared.b16 {%0,%1}, [%2];\n"
                 : "=r"(r[0]), "=r"(r[1])
                 : "r"(su32(p)));
}
// d += a (16x16, row-major) * b (16x8, column-major), bf16 inputs, f32 accumulators
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2]) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Address of the 8 channels [ch, ch+8) of pixel (n, y, x) of concat(in0, in1)
// (channel counts c0, c1), or NULL outside the image.
__device__ __forceinline__ const bf16 *chan8(const bf16 *in0, int c0, const bf16 *in1, int c1, const Shape &s, int n,
                                             int y, int x, int ch) {
    if (y < 0 || y >= s.h || x < 0 || x >= s.w) return nullptr;
    const long long pix = ((long long)n * s.h + y) * s.w + x;
    return ch < c0 ? in0 + pix * c0 + ch : in1 + pix * c1 + (ch - c0);
}

// out = act(conv3x3(concat(in0, in1)) + bias) over BN output channels
// [blockIdx.y*BN, +BN); output channel co goes to out0 (co < d0) or to out1
// (co - d0).  bias may be NULL.
template <int BN>
__global__ void __launch_bounds__(kCT) conv3x3_kernel(const bf16 *in0, int c0, const bf16 *in1, int c1, const bf16 *wt,
                                                      const float *bias, int cout, bf16 *out0, int d0, bf16 *out1,
                                                      int d1, Shape s, int relu) {
    __shared__ __align__(128) bf16 sA[2][kBM * kAS];
    __shared__ __align__(128) bf16 sB[2][BN * kAS];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long hw = (long long)s.h * s.w, npix = s.n * hw;
    const long long p0 = (long long)blockIdx.x * kBM;
    const int co0 = blockIdx.y * BN;
    const int ct = c0 + c1, nck = ct / 16, nk = 9 * nck;
    // the pixel and 8-channel half this thread stages
    const int apx = tid >> 1, ahalf = tid & 1;
    const long long ap = p0 + apx;
    const bool aok = ap < npix;
    int an = 0, ay = 0, ax = 0;
    if (aok) {
        an = (int)(ap / hw);
        const int rem = (int)(ap - an * hw);
        ay = rem / s.w;
        ax = rem - ay * s.w;
    }
    auto stage = [&](int kc, int buf) {
        const int tap = kc / nck, cc = (kc - tap * nck) * 16;
        const int dy = tap / 3 - 1, dx = tap % 3 - 1;
        const bf16 *src = aok ? chan8(in0, c0, in1, c1, s, an, ay + dy, ax + dx, cc + ahalf * 8) : nullptr;
        cp_async16(&sA[buf][apx * kAS + ahalf * 8], src ? src : in0, src ? 16 : 0);
        if (tid < BN * 2) {
            const int r = tid >> 1, half = tid & 1;
            cp_async16(&sB[buf][r * kAS + half * 8], wt + ((long long)tap * cout + co0 + r) * ct + cc + half * 8, 16);
        }
        cp_async_commit();
    };
    float acc[BN / 8][4];
#pragma unroll
    for (int nb = 0; nb < BN / 8; nb++) acc[nb][0] = acc[nb][1] = acc[nb][2] = acc[nb][3] = 0.f;
    stage(0, 0);
    for (int kc = 0; kc < nk; kc++) {
        const int buf = kc & 1;
        if (kc + 1 < nk) {
            stage(kc + 1, buf ^ 1);
            cp_wait1();
        } else {
            cp_async_wait_all();
        }
        __syncthreads();
        uint32_t a[4];
        ldsm_x4(a, &sA[buf][(warp * 16 + (lane & 15)) * kAS + (lane >> 4) * 8]);
#pragma unroll
        for (int nb = 0; nb < BN / 8; nb++) {
            uint32_t b[2];
            ldsm_x2(b, &sB[buf][(nb * 8 + (lane & 7)) * kAS + ((lane >> 3) & 1) * 8]);
            mma16816(acc[nb], a, b);
        }
        __syncthreads();
    }
    const int r0 = lane >> 2, cq = (lane & 3) * 2;
#pragma unroll
    for (int half = 0; half < 2; half++) {
        const long long p = p0 + warp * 16 + r0 + half * 8;
        if (p >= npix) continue;
#pragma unroll
        for (int nb = 0; nb < BN / 8; nb++) {
            const int co = co0 + nb * 8 + cq;
            float v0 = acc[nb][half * 2], v1 = acc[nb][half * 2 + 1];
            if (bias) {
                v0 += bias[co];
                v1 += bias[co + 1];
            }
            if (relu) {
                v0 = fmaxf(v0, 0.f);
                v1 = fmaxf(v1, 0.f);
            }
            const __nv_bfloat162 v = __floats2bfloat162_rn(v0, v1);
            if (co < d0) *reinterpret_cast<__nv_bfloat162 *>(out0 + p * d0 + co) = v;
            else *reinterpret_cast<__nv_bfloat162 *>(out1 + p * d1 + (co - d0)) = v;
        }
    }
}

// ---------------------------------------------------------------------------
// The same convolution on the 5th-generation tensor cores (tcgen05.mma, FP32
// accumulator in tensor memory).  The halo box may reach past the image on
// every side (images narrower than a strip, or fewer than 3 rows high): the
// tensor map fills what lies outside with zeros.
//
// A CTA owns R strips of kStrip = 128 consecutive pixels (the same columns
// of R consecutive image rows) and BN output channels.  Per 16-channel chunk
// of the (concatenated) input, TMA brings the (R + 2) x 130 halo (rows
// y0-1..y0+R, columns x0-1..x0+128; zero outside the image from the tensor
// map) into shared memory once, as two planes of 8 channels ([row][column][8]
// bf16, 16 bytes per pixel), with the chunk's weights of all 9 taps
// ([tap][BN][8] per plane).  Row r's 9 taps are 9 MMAs (M = 128 pixels,
// N = BN, K = 16) into its own accumulator columns, whose A operand is that
// one halo tile seen from a shifted start: pixel i of tap (dy, dx) sits at
// plane + ((r + dy + 1)*130 + i + dx + 1)*16, which is the K-major,
// no-swizzle canonical layout (8-row core matrices of 16-byte rows, 128
// bytes apart = SBO; the second 8-channel plane LBO bytes further).  No
// per-tap restaging, and neighbouring rows share their halo rows and the
// weights.  (The copies arrive in 16-byte pieces, one per pixel and plane,
// because channels are innermost in memory; the TMA unit's rate for such
// pieces, not the tensor cores, bounds the kernel, hence R > 1.)
//
// Roles: warp 1 lane 0 issues the TMA copies into a ring of stages, warp 0
// lane 0 issues the MMAs and hands each stage back to the producer with
// tcgen05.commit on an mbarrier; then all four warps read the accumulator
// (tensor-memory lane = pixel, column = row * BN + output channel) and write
// bias + ReLU + bf16.  Every wait is bounded; a wait that gives up sets
// g_unet_status, lets the copies in flight land and still frees the tensor
// memory.
constexpr int kStrip = 128;                                // pixels per strip (MMA M)
constexpr int kHaloW = kStrip + 2;                         // staged columns
constexpr int kTcHead = 256;                               // mbarriers, tensor-memory address, flags

template <int BN>
struct TcConv {
    static constexpr int R = BN >= 128 ? 2 : 4;           // image rows per CTA
    static constexpr int kPlaneA = (R + 2) * kHaloW * 16;  // bytes of one 8-channel halo plane
    static constexpr int kPlaneAPad = (kPlaneA + 127) / 128 * 128;  // planes start 128-byte aligned
    static constexpr int kPlaneB = 9 * BN * 16;            // one 8-channel plane of the 9 taps' weights
    static constexpr int kStage = 2 * kPlaneAPad + 2 * kPlaneB;
    static constexpr int kStages = BN >= 64 ? 2 : 3;
    static constexpr int kTmemCols = R * BN <= 32 ? 32 : R * BN <= 64 ? 64 : R * BN <= 128 ? 128 : 256;
    static constexpr uint32_t kTx = 2 * kPlaneA + 2 * kPlaneB;  // bytes the copies of one stage deliver
    static constexpr int kSmemMax = kTcHead + 128 + kStages * kStage;
    static_assert(kTx < (1u << 20), "mbarrier transaction count limit");
    static_assert(BN % 16 == 0 && BN >= 16 && BN <= 256, "MMA N for M = 128");
    static_assert(R * BN <= kTmemCols && R + 2 <= 256, "accumulator columns, box rows");
};

struct TcMaps {
    CUtensorMap in0, in1, wt;
};

__device__ int g_unet_status = 0;

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
// Shared-memory matrix descriptor of tcgen05.mma, K-major without swizzle:
// start address, leading byte offset (distance of the two 8-element K
// halves), stride byte offset (distance of 8-row core matrices), version 1.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: D f32, A and B bf16, both K-major, M = 128.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(
            tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc));
}
__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tmem_ld16(uint32_t (&r)[16], uint32_t taddr) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

template <int BN>
__global__ void __launch_bounds__(128) conv3x3_tc_kernel(const __grid_constant__ TcMaps maps, int c0, int nck,
                                                         const float *bias, bf16 *out0, int d0, bf16 *out1, int d1,
                                                         Shape s, int strips, int groups, int relu) {
    using C = TcConv<BN>;
    extern __shared__ uint8_t tc_smem[];
    uint8_t *base = tc_smem + ((128u - (smem_u32(tc_smem) & 127u)) & 127u);
    uint64_t *full = reinterpret_cast<uint64_t *>(base);  // [kStages]: copies landed
    uint64_t *empty = full + C::kStages;                  // [kStages]: MMAs done reading
    uint64_t *done = empty + C::kStages;                  // every MMA done
    volatile int *info = reinterpret_cast<volatile int *>(done + 1);  // tmem address, error, issued, consumed
    uint8_t *stage0 = base + kTcHead;
    const int nst = nck < C::kStages ? nck : C::kStages;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    constexpr int R = C::R;
    const int t_ = blockIdx.x / strips;  // image * groups + row group
    const int x0 = (blockIdx.x - t_ * strips) * kStrip;
    const int img = t_ / groups, y0 = (t_ - img * groups) * R;
    const int co0 = blockIdx.y * BN;
    if (tid == 0) {
        for (int i = 0; i < nst; i++) {
            mbar_init(&full[i], 1);
            mbar_init(&empty[i], 1);
        }
        mbar_init(done, 1);
        info[1] = 0;
        info[2] = 0;
        info[3] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32((const void *)&info[0])),
                     "r"(C::kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = (uint32_t)info[0];

    if (warp == 1 && lane == 0) {  // producer
        int c = 0;
        for (; c < nck; c++) {
            const int st = c % nst;
            if (c >= nst && !mbar_wait(&empty[st], ((c / nst) - 1) & 1)) {
                info[1] = 1;
                break;
            }
            uint8_t *sp = stage0 + st * C::kStage;
            mbar_expect_tx(&full[st], C::kTx);
            const int ch = c * 16;
            const CUtensorMap *m = ch < c0 ? &maps.in0 : &maps.in1;
            const int cc = ch < c0 ? ch : ch - c0;
#pragma unroll
            for (int j = 0; j < 2; j++) {
                tma_load_4d(sp + j * C::kPlaneAPad, m, cc + 8 * j, x0 - 1, y0 - 1, img, &full[st]);
                tma_load_3d(sp + 2 * C::kPlaneAPad + j * C::kPlaneB, &maps.wt, ch + 8 * j, co0, 0, &full[st]);
            }
        }
        info[2] = c;
    }
    if (warp == 0 && lane == 0) {  // MMA issuer
        constexpr uint32_t idesc = umma_idesc_bf16(BN);
        int c = 0;
        for (; c < nck; c++) {
            const int st = c % nst;
            if (!mbar_wait(&full[st], (c / nst) & 1)) {
                info[1] = 1;
                break;
            }
            tc_fence_after();
            const uint32_t a0 = smem_u32(stage0 + st * C::kStage), b0 = a0 + 2 * C::kPlaneAPad;
#pragma unroll
            for (int r = 0; r < R; r++)
#pragma unroll
                for (int t = 0; t < 9; t++) {
                    const uint64_t ad = umma_desc(a0 + ((r + t / 3) * kHaloW + t % 3) * 16, C::kPlaneAPad, 128);
                    const uint64_t bd = umma_desc(b0 + t * BN * 16, C::kPlaneB, 128);
                    umma_bf16(tmem + r * BN, ad, bd, idesc, (c | t) != 0);
                }
            umma_commit(&empty[st]);
        }
        info[3] = c;
        umma_commit(done);  // arrives once every MMA issued above has completed
    }
    __syncwarp();
    if (!mbar_wait(done, 0)) info[1] = 1;
    __syncthreads();
    if (info[1]) {
        if (tid == 32)  // copies issued but never consumed: one bounded chance to land
            for (int c = info[3]; c < info[2]; c++) mbar_wait(&full[c % nst], (c / nst) & 1);
        if (tid == 0) atomicExch(&g_unet_status, 1);
    } else {
        tc_fence_after();
        const int x = x0 + warp * 32 + lane;
#pragma unroll 1
        for (int q = 0; q < R * (BN / 16); q++) {
            const int rr = q / (BN / 16), g = q - rr * (BN / 16);
            uint32_t r[16];
            tmem_ld16(r, tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(rr * BN + g * 16));
            if (x >= s.w || y0 + rr >= s.h) continue;  // after the warp-wide load
            const long long p = ((long long)img * s.h + y0 + rr) * s.w + x;
            const int co = co0 + g * 16;
            uint32_t packed[8];
#pragma unroll
            for (int i = 0; i < 8; i++) {
                float v0 = __uint_as_float(r[2 * i]), v1 = __uint_as_float(r[2 * i + 1]);
                if (bias) {
                    v0 += bias[co + 2 * i];
                    v1 += bias[co + 2 * i + 1];
                }
                if (relu) {
                    v0 = fmaxf(v0, 0.f);
                    v1 = fmaxf(v1, 0.f);
                }
                const __nv_bfloat162 b2 = __floats2bfloat162_rn(v0, v1);
                packed[i] = *reinterpret_cast<const uint32_t *>(&b2);
            }
            bf16 *dst = co < d0 ? out0 + p * d0 + co : out1 + p * d1 + (co - d0);
            uint4 *d4 = reinterpret_cast<uint4 *>(dst);
            d4[0] = make_uint4(packed[0], packed[1], packed[2], packed[3]);
            d4[1] = make_uint4(packed[4], packed[5], packed[6], packed[7]);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(C::kTmemCols)
                     : "memory");
    }
}

// Weights of the data gradient: wd[8-tap][ci][co] = w[tap][co][ci].
__global__ void flip_weights_kernel(const bf16 *w, bf16 *wd, int cout, int cin) {
    const long long n = 9ll * cout * cin;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int tap = (int)(i / ((long long)cout * cin));
        const int rem = (int)(i - (long long)tap * cout * cin);
        const int co = rem / cin, ci = rem - co * cin;
        wd[((long long)(8 - tap) * cin + ci) * cout + co] = w[i];
    }
}

// g *= (y > 0): the ReLU derivative, y being the layer's output.
__global__ void relu_bwd_kernel(bf16 *g, const bf16 *y, long long n) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        if (!(__bfloat162float(y[i]) > 0.f)) g[i] = __float2bfloat16(0.f);
}

// Weight-gradient partials: part[blk][tap][co][ci] = sum over the pixels of
// block blk of g[p][co] * x[p + off(tap)][ci], x = concat(in0, in1).  CTA
// tile: BMC output x BNC input channels of one tap (grid.z), pixels in steps
// of 32 as the K dimension of the tensor-core products.
template <int BMC, int BNC>
__global__ void __launch_bounds__(128) wgrad_kernel(const bf16 *g, int cout, const bf16 *in0, int c0, const bf16 *in1,
                                                    int c1, float *part, Shape s) {
    __shared__ __align__(128) bf16 sG[32 * (BMC + 8)];
    __shared__ __align__(128) bf16 sX[32 * (BNC + 8)];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int ct = c0 + c1, tiles_n = ct / BNC;
    const int co0 = (blockIdx.y / tiles_n) * BMC, ci0 = (blockIdx.y % tiles_n) * BNC;
    const int tap = blockIdx.z, dy = tap / 3 - 1, dx = tap % 3 - 1;
    const long long hw = (long long)s.h * s.w, npix = s.n * hw;
    const long long pb0 = (long long)blockIdx.x * kWgPix;
    const long long pb1 = pb0 + kWgPix < npix ? pb0 + kWgPix : npix;
    constexpr int WN = BNC / 16, NWARP = (BMC / 16) * WN;
    const int wm = warp / WN, wn = warp - wm * WN;
    float acc[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
    for (long long pc = pb0; pc < pb1; pc += 32) {
        for (int q = tid; q < 32 * (BMC / 8); q += 128) {
            const int px = q / (BMC / 8), ch = (q - px * (BMC / 8)) * 8;
            const long long p = pc + px;
            const bool ok = p < pb1;
            cp_async16(&sG[px * (BMC + 8) + ch], ok ? g + p * cout + co0 + ch : g, ok ? 16 : 0);
        }
        for (int q = tid; q < 32 * (BNC / 8); q += 128) {
            const int px = q / (BNC / 8), ch = (q - px * (BNC / 8)) * 8;
            const long long p = pc + px;
            const bf16 *src = nullptr;
            if (p < pb1) {
                const int n = (int)(p / hw);
                const int rem = (int)(p - n * hw);
                const int y = rem / s.w, x = rem - y * s.w;
                src = chan8(in0, c0, in1, c1, s, n, y + dy, x + dx, ci0 + ch);
            }
            cp_async16(&sX[px * (BNC + 8) + ch], src ? src : in0, src ? 16 : 0);
        }
        cp_async_commit();
        cp_async_wait_all();
        __syncthreads();
        if (warp < NWARP) {
#pragma unroll
            for (int kk = 0; kk < 32; kk += 16) {
                uint32_t a[4];
                {
                    const int j = lane >> 3;
                    ldsm_x4_t(a, &sG[(kk + (j >> 1) * 8 + (lane & 7)) * (BMC + 8) + wm * 16 + (j & 1) * 8]);
                }
#pragma unroll
                for (int nb = 0; nb < 2; nb++) {
                    uint32_t b[2];
                    const int j = (lane >> 3) & 1;
                    ldsm_x2_t(b, &sX[(kk + j * 8 + (lane & 7)) * (BNC + 8) + wn * 16 + nb * 8]);
                    mma16816(acc[nb], a, b);
                }
            }
        }
        __syncthreads();
    }
    if (warp >= NWARP) return;
    const int r0 = lane >> 2, cq = (lane & 3) * 2;
    float *base = part + ((long long)blockIdx.x * 9 + tap) * cout * ct;
#pragma unroll
    for (int half = 0; half < 2; half++) {
        const int co = co0 + wm * 16 + r0 + half * 8;
#pragma unroll
        for (int nb = 0; nb < 2; nb++) {
            const int ci = ci0 + wn * 16 + nb * 8 + cq;
            base[(long long)co * ct + ci] = acc[nb][half * 2];
            base[(long long)co * ct + ci + 1] = acc[nb][half * 2 + 1];
        }
    }
}

// out[i] = sum over blocks b (in order) of part[b][i].
__global__ void block_sum_kernel(const float *part, int nblk, long long n, float *out) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int b = 0; b < nblk; b++) s += part[b * n + i];
        out[i] = s;
    }
}

// Per-block channel sums of g ([pixels][c] bf16): part[blk][co].
__global__ void chan_sum_kernel(const bf16 *g, int c, long long npix, float *part) {
    const long long p0 = (long long)blockIdx.x * kRedPix;
    const long long p1 = p0 + kRedPix < npix ? p0 + kRedPix : npix;
    for (int co = threadIdx.x; co < c; co += blockDim.x) {
        float s = 0.f;
        for (long long p = p0; p < p1; p++) s += __bfloat162float(g[p * c + co]);
        part[(long long)blockIdx.x * c + co] = s;
    }
}

// 2x2 average pooling of [n][h][w][c] into [n][h/2][w/2][c], and its adjoint.
__global__ void pool2_kernel(const bf16 *in, bf16 *out, int c, Shape s) {
    const int ho = s.h / 2, wo = s.w / 2;
    const long long n = (long long)s.n * ho * wo * c;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ch = (int)(i % c);
        const long long pix = i / c;
        const int x = (int)(pix % wo), y = (int)((pix / wo) % ho), im = (int)(pix / ((long long)wo * ho));
        const long long b = (((long long)im * s.h + 2 * y) * s.w + 2 * x) * c + ch;
        const float v = __bfloat162float(in[b]) + __bfloat162float(in[b + c]) +
                        __bfloat162float(in[b + (long long)s.w * c]) + __bfloat162float(in[b + (long long)s.w * c + c]);
        out[i] = __float2bfloat16(0.25f * v);
    }
}
__global__ void pool2_bwd_kernel(const bf16 *gout, bf16 *gin, int c, Shape s, int accumulate) {
    const long long n = (long long)s.n * s.h * s.w * c;
    const int wo = s.w / 2, ho = s.h / 2;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ch = (int)(i % c);
        const long long pix = i / c;
        const int x = (int)(pix % s.w), y = (int)((pix / s.w) % s.h), im = (int)(pix / ((long long)s.w * s.h));
        const float v = 0.25f * __bfloat162float(gout[(((long long)im * ho + y / 2) * wo + x / 2) * c + ch]);
        gin[i] = __float2bfloat16(accumulate ? __bfloat162float(gin[i]) + v : v);
    }
}
// Nearest-neighbour 2x upsampling of [n][h][w][c] into [n][2h][2w][c], and its adjoint.
__global__ void up2_kernel(const bf16 *in, bf16 *out, int c, Shape s) {
    const int ho = 2 * s.h, wo = 2 * s.w;
    const long long n = (long long)s.n * ho * wo * c;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ch = (int)(i % c);
        const long long pix = i / c;
        const int x = (int)(pix % wo), y = (int)((pix / wo) % ho), im = (int)(pix / ((long long)wo * ho));
        out[i] = in[(((long long)im * s.h + y / 2) * s.w + x / 2) * c + ch];
    }
}
__global__ void up2_bwd_kernel(const bf16 *gout, bf16 *gin, int c, Shape s) {
    const long long n = (long long)s.n * s.h * s.w * c;
    const int wo = 2 * s.w;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int ch = (int)(i % c);
        const long long pix = i / c;
        const int x = (int)(pix % s.w), y = (int)((pix / s.w) % s.h), im = (int)(pix / ((long long)s.w * s.h));
        const long long b = (((long long)im * 2 * s.h + 2 * y) * wo + 2 * x) * c + ch;
        const float v = __bfloat162float(gout[b]) + __bfloat162float(gout[b + c]) +
                        __bfloat162float(gout[b + (long long)wo * c]) + __bfloat162float(gout[b + (long long)wo * c + c]);
        gin[i] = __float2bfloat16(v);
    }
}

// 1x1 output head: out[p] = sum_c w[c] x[p][c] + b (FP32 out), and its
// adjoint: gx[p][c] = w[c] gout[p]; part[blk][c] = sum_p x[p][c] gout[p]
// (c < C), part[blk][C] = sum_p gout[p].
template <int C>
__global__ void head_kernel(const bf16 *x, const float *w, const float *b, float *out, long long npix) {
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < npix; p += (long long)gridDim.x * blockDim.x) {
        float s = b[0];
#pragma unroll
        for (int c = 0; c < C; c++) s += w[c] * __bfloat162float(x[p * C + c]);
        out[p] = s;
    }
}
template <int C>
__global__ void head_bwd_kernel(const bf16 *x, const float *w, const float *gout, bf16 *gx, float *part, long long npix) {
    __shared__ float red[C + 1][8];
    const long long p0 = (long long)blockIdx.x * kRedPix;
    const long long p1 = p0 + kRedPix < npix ? p0 + kRedPix : npix;
    float acc[C + 1];
#pragma unroll
    for (int c = 0; c <= C; c++) acc[c] = 0.f;
    for (long long p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
        const float go = gout[p];
#pragma unroll
        for (int c = 0; c < C; c++) {
            gx[p * C + c] = __float2bfloat16(w[c] * go);
            acc[c] += __bfloat162float(x[p * C + c]) * go;
        }
        acc[C] += go;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int c = 0; c <= C; c++) {
        float v = acc[c];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[c][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x <= C) {
        float s = 0.f;
        for (int k = 0; k < 8; k++) s += red[threadIdx.x][k];
        part[(long long)blockIdx.x * (C + 1) + threadIdx.x] = s;
    }
}

// Network input: planes [n][3][h][w] FP32 -> [n][h][w][16] bf16 (channels 3..15 zero).
__global__ void pack_kernel(const float *planes, bf16 *x, Shape s) {
    const long long hw = (long long)s.h * s.w, n = s.n * hw;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < n; p += (long long)gridDim.x * blockDim.x) {
        const long long im = p / hw, r = p - im * hw;
#pragma unroll
        for (int c = 0; c < 16; c++)
            x[p * 16 + c] = __float2bfloat16(c < 3 ? planes[(im * 3 + c) * hw + r] : 0.f);
    }
}

// Adam on FP32 master weights; writes the bf16 copy the kernels use.
__global__ void adam_kernel(float *w, float *m, float *v, const float *g, bf16 *wb, long long n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float wi = w[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        w[i] = wi;
        if (wb) wb[i] = __float2bfloat16(wi);
    }
}

// Mean squared error: gout = 2 (out - tgt) / n, part[blk] = sum (out - tgt)^2 (FP64).
__global__ void mse_kernel(const float *out, const float *tgt, float *gout, long long n, double *part) {
    __shared__ double red[8];
    double acc = 0.0;
    const float inv = 2.f / (float)n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float r = out[i] - tgt[i];
        gout[i] = inv * r;
        acc += (double)r * r;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int k = 0; k < 8; k++) s += red[k];
        part[blockIdx.x] = s;
    }
}
__global__ void mse_finish_kernel(const double *part, int nblk, long long n, double *loss) {
    double s = 0.0;
    for (int b = 0; b < nblk; b++) s += part[b];
    *loss = s / (double)n;
}

constexpr int kElemBlocks = 1184, kElemThreads = 256, kMseBlocks = 296;

static unsigned elem_blocks(long long n) {
    long long b = (n + kElemThreads - 1) / kElemThreads;
    return (unsigned)(b < 1 ? 1 : b > kElemBlocks ? kElemBlocks : b);
}
static bool a16(const void *p) { return ((uintptr_t)p & 15u) == 0; }

}  // namespace unet
}  // namespace fwi

using namespace fwi;
using namespace fwi::unet;

// Convolution kernel selection: 0 = tcgen05 where the image is at least
// kTcMinWidth pixels wide (mma.sync otherwise), 1 = mma.sync only.  Narrower
// images would leave most of the 128 MMA rows of a strip empty.
constexpr int kTcMinWidth = 64;
static int g_conv_path = 0;

// bf16 tiled tensor map, zero fill outside; dims innermost first, strides in
// bytes of dims 1..rank-1.
static int encode_bf16(CUtensorMap *m, const void *base, int rank, const cuuint64_t *dims, const cuuint64_t *strides,
                       const cuuint32_t *box) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) return set_error(FWI_ECUDA, "cuTensorMapEncodeTiled unavailable from the driver");
    const cuuint32_t es[4] = {1, 1, 1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, (cuuint32_t)rank, const_cast<void *>(base), dims, strides, box,
                    es, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return set_error(FWI_ECUDA, "cuTensorMapEncodeTiled (bf16) failed (%d)", (int)r);
    return 0;
}

// Halo map of an NHWC activation: dims (c, w, h, n), box 8 x kHaloW x rows x 1.
static int encode_act(CUtensorMap *m, const bf16 *x, int c, const Shape &s, int rows) {
    const cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)s.w, (cuuint64_t)s.h, (cuuint64_t)s.n};
    const cuuint64_t strides[3] = {(cuuint64_t)c * 2, (cuuint64_t)c * 2 * s.w, (cuuint64_t)c * 2 * s.w * s.h};
    const cuuint32_t box[4] = {8, (cuuint32_t)kHaloW, (cuuint32_t)rows, 1};
    return encode_bf16(m, x, 4, dims, strides, box);
}

template <int BN>
static int launch_tc(const TcMaps &maps, int c0, int nck, const float *bias, bf16 *o0, int d0, bf16 *o1, int d1,
                     const Shape &s, int relu, int cout, cudaStream_t st) {
    using C = TcConv<BN>;
    static bool attr = false;
    if (!attr) {
        if (cudaFuncSetAttribute(conv3x3_tc_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, C::kSmemMax) !=
            cudaSuccess)
            return set_error(FWI_ECUDA, "unet_conv3x3: shared-memory attribute refused");
        attr = true;
    }
    const int strips = (s.w + kStrip - 1) / kStrip, groups = (s.h + C::R - 1) / C::R;
    const long long blocks = (long long)s.n * groups * strips;
    if (blocks >= 0x7fffffffll) return set_error(FWI_ERANGE, "fwi_unet_conv3x3: too many pixel strips");
    const int nst = nck < C::kStages ? nck : C::kStages;
    const size_t smem = kTcHead + 128 + (size_t)nst * C::kStage;
    conv3x3_tc_kernel<BN><<<dim3((unsigned)blocks, cout / BN), 128, smem, st>>>(maps, c0, nck, bias, o0, d0, o1, d1, s,
                                                                               strips, groups, relu);
    return check_launch("unet_conv3x3 (tcgen05)");
}

static int conv3x3_tc(const bf16 *i0, int c0, const bf16 *i1, int c1, const bf16 *wt, const float *bias, int cout,
                      bf16 *o0, int d0, bf16 *o1, int d1, const Shape &s, int relu, cudaStream_t st) {
    const int ct = c0 + c1;
    const int bn = cout % 128 == 0 ? 128 : cout % 64 == 0 ? 64 : cout % 32 == 0 ? 32 : 16;
    const int rows = (bn >= 128 ? TcConv<128>::R : TcConv<16>::R) + 2;
    static_assert(TcConv<16>::R == TcConv<32>::R && TcConv<32>::R == TcConv<64>::R, "rows per CTA");
    TcMaps maps;
    int rc = encode_act(&maps.in0, i0, c0, s, rows);
    if (!rc) rc = c1 ? encode_act(&maps.in1, i1, c1, s, rows) : encode_act(&maps.in1, i0, c0, s, rows);
    const cuuint64_t wdims[3] = {(cuuint64_t)ct, (cuuint64_t)cout, 9};
    const cuuint64_t wstr[2] = {(cuuint64_t)ct * 2, (cuuint64_t)ct * 2 * cout};
    const cuuint32_t wbox[3] = {8, (cuuint32_t)bn, 9};
    if (!rc) rc = encode_bf16(&maps.wt, wt, 3, wdims, wstr, wbox);
    if (rc) return rc;
    const int nck = ct / 16;
    if (bn == 128) return launch_tc<128>(maps, c0, nck, bias, o0, d0, o1, d1, s, relu, cout, st);
    if (bn == 64) return launch_tc<64>(maps, c0, nck, bias, o0, d0, o1, d1, s, relu, cout, st);
    if (bn == 32) return launch_tc<32>(maps, c0, nck, bias, o0, d0, o1, d1, s, relu, cout, st);
    return launch_tc<16>(maps, c0, nck, bias, o0, d0, o1, d1, s, relu, cout, st);
}

int fwi::unet_device_status(int clear, int *status) {
    int v = 0;
    if (cudaMemcpyFromSymbol(&v, g_unet_status, sizeof(int)) != cudaSuccess)
        return set_error(FWI_ECUDA, "fwi_device_status: reading the U-Net kernels' status failed");
    if (clear && v) {
        const int z = 0;
        if (cudaMemcpyToSymbol(g_unet_status, &z, sizeof(int)) != cudaSuccess)
            return set_error(FWI_ECUDA, "fwi_device_status: clearing the U-Net kernels' status failed");
    }
    *status = v;
    return 0;
}

#define UREQ(cond, ...)                                        \
    do {                                                       \
        if (!(cond)) return set_error(FWI_EINVAL, __VA_ARGS__); \
    } while (0)

extern "C" {

int fwi_unet_conv3x3(const void *in0, int c0, const void *in1, int c1, const void *w, const float *bias, int cout,
                     void *out0, int d0, void *out1, int d1, int n, int h, int wd, int relu, void *stream) {
    UREQ(in0 && w && out0, "fwi_unet_conv3x3: NULL pointer");
    UREQ(c0 > 0 && c0 % 16 == 0 && c1 >= 0 && c1 % 16 == 0 && (c1 == 0 || in1),
         "fwi_unet_conv3x3: input channels must be positive multiples of 16");
    UREQ(cout > 0 && cout % 16 == 0 && d0 > 0 && d0 % 16 == 0 && d1 >= 0 && d0 + d1 == cout && (d1 == 0 || out1),
         "fwi_unet_conv3x3: output channels must be multiples of 16 with d0 + d1 = cout");
    UREQ(n > 0 && h > 0 && wd > 0, "fwi_unet_conv3x3: empty image");
    UREQ(a16(in0) && a16(in1) && a16(w) && a16(out0) && a16(out1), "fwi_unet_conv3x3: pointers must be 16-byte aligned");
    const long long npix = (long long)n * h * wd;
    UREQ(npix / kBM < 0x7fffffffll, "fwi_unet_conv3x3: too many pixels");
    const Shape s{n, h, wd};
    cudaStream_t st = (cudaStream_t)stream;
    const bf16 *i0 = (const bf16 *)in0, *i1 = (const bf16 *)in1, *wt = (const bf16 *)w;
    bf16 *o0 = (bf16 *)out0, *o1 = (bf16 *)out1;
    if (g_conv_path == 0 && wd >= kTcMinWidth)
        return conv3x3_tc(i0, c0, i1, c1, wt, bias, cout, o0, d0, o1, d1, s, relu, st);
    const int bn = cout % 64 == 0 ? 64 : cout % 32 == 0 ? 32 : 16;
    dim3 grid((unsigned)((npix + kBM - 1) / kBM), cout / bn);
    if (bn == 64) conv3x3_kernel<64><<<grid, kCT, 0, st>>>(i0, c0, i1, c1, wt, bias, cout, o0, d0, o1, d1, s, relu);
    else if (bn == 32) conv3x3_kernel<32><<<grid, kCT, 0, st>>>(i0, c0, i1, c1, wt, bias, cout, o0, d0, o1, d1, s, relu);
    else conv3x3_kernel<16><<<grid, kCT, 0, st>>>(i0, c0, i1, c1, wt, bias, cout, o0, d0, o1, d1, s, relu);
    return check_launch("unet_conv3x3");
}

int fwi_unet_conv_path(int path) {
    const int old = g_conv_path;
    if (path == 0 || path == 1) g_conv_path = path;
    return old;
}

int fwi_unet_flip_weights(const void *w, void *wd, int cout, int cin, void *stream) {
    UREQ(w && wd && cout > 0 && cin > 0, "fwi_unet_flip_weights: bad arguments");
    flip_weights_kernel<<<elem_blocks(9ll * cout * cin), kElemThreads, 0, (cudaStream_t)stream>>>(
        (const bf16 *)w, (bf16 *)wd, cout, cin);
    return check_launch("unet_flip_weights");
}

int fwi_unet_relu_bwd(void *g, const void *y, long long count, void *stream) {
    UREQ(g && y && count >= 0, "fwi_unet_relu_bwd: bad arguments");
    if (!count) return 0;
    relu_bwd_kernel<<<elem_blocks(count), kElemThreads, 0, (cudaStream_t)stream>>>((bf16 *)g, (const bf16 *)y, count);
    return check_launch("unet_relu_bwd");
}

long long fwi_unet_wgrad_partials(int cout, int cin, int n, int h, int w) {
    const long long npix = (long long)n * h * w;
    const long long blocks = (npix + kWgPix - 1) / kWgPix;
    const long long rblocks = (npix + kRedPix - 1) / kRedPix;
    const long long a = blocks * 9 * cout * cin, b = rblocks * cout;
    return a > b ? a : b;
}

int fwi_unet_conv3x3_wgrad(const void *g, int cout, const void *in0, int c0, const void *in1, int c1, int n, int h,
                           int wd, float *part, float *dw, float *db, void *stream) {
    UREQ(g && in0 && part && dw, "fwi_unet_conv3x3_wgrad: NULL pointer");
    UREQ(c0 > 0 && c0 % 16 == 0 && c1 >= 0 && c1 % 16 == 0 && (c1 == 0 || in1) && cout > 0 && cout % 16 == 0,
         "fwi_unet_conv3x3_wgrad: channel counts must be multiples of 16");
    UREQ(n > 0 && h > 0 && wd > 0, "fwi_unet_conv3x3_wgrad: empty image");
    UREQ(a16(g) && a16(in0) && a16(in1), "fwi_unet_conv3x3_wgrad: pointers must be 16-byte aligned");
    cudaStream_t st = (cudaStream_t)stream;
    const Shape s{n, h, wd};
    const long long npix = (long long)n * h * wd;
    const int ct = c0 + c1;
    const int nblk = (int)((npix + kWgPix - 1) / kWgPix);
    const bf16 *gg = (const bf16 *)g, *i0 = (const bf16 *)in0, *i1 = (const bf16 *)in1;
    const int bmc = cout % 32 == 0 ? 32 : 16, bnc = ct % 32 == 0 ? 32 : 16;
    dim3 grid(nblk, (cout / bmc) * (ct / bnc), 9);
    if (bmc == 32 && bnc == 32) wgrad_kernel<32, 32><<<grid, 128, 0, st>>>(gg, cout, i0, c0, i1, c1, part, s);
    else if (bmc == 32) wgrad_kernel<32, 16><<<grid, 128, 0, st>>>(gg, cout, i0, c0, i1, c1, part, s);
    else if (bnc == 32) wgrad_kernel<16, 32><<<grid, 128, 0, st>>>(gg, cout, i0, c0, i1, c1, part, s);
    else wgrad_kernel<16, 16><<<grid, 128, 0, st>>>(gg, cout, i0, c0, i1, c1, part, s);
    int rc = check_launch("unet_wgrad");
    if (rc) return rc;
    const long long nw = 9ll * cout * ct;
    block_sum_kernel<<<elem_blocks(nw), kElemThreads, 0, st>>>(part, nblk, nw, dw);
    rc = check_launch("unet_wgrad_sum");
    if (rc || !db) return rc;
    const int rblk = (int)((npix + kRedPix - 1) / kRedPix);
    chan_sum_kernel<<<rblk, 128, 0, st>>>(gg, cout, npix, part);
    rc = check_launch("unet_bias_grad");
    if (rc) return rc;
    block_sum_kernel<<<1, 128, 0, st>>>(part, rblk, cout, db);
    return check_launch("unet_bias_grad_sum");
}

int fwi_unet_pool2(const void *in, void *out, int c, int n, int h, int w, void *stream) {
    UREQ(in && out && c > 0 && n > 0 && h > 0 && w > 0 && h % 2 == 0 && w % 2 == 0, "fwi_unet_pool2: bad arguments");
    pool2_kernel<<<elem_blocks((long long)n * h * w * c / 4), kElemThreads, 0, (cudaStream_t)stream>>>(
        (const bf16 *)in, (bf16 *)out, c, Shape{n, h, w});
    return check_launch("unet_pool2");
}

int fwi_unet_pool2_bwd(const void *gout, void *gin, int c, int n, int h, int w, int accumulate, void *stream) {
    UREQ(gout && gin && c > 0 && n > 0 && h > 0 && w > 0 && h % 2 == 0 && w % 2 == 0,
         "fwi_unet_pool2_bwd: bad arguments");
    pool2_bwd_kernel<<<elem_blocks((long long)n * h * w * c), kElemThreads, 0, (cudaStream_t)stream>>>(
        (const bf16 *)gout, (bf16 *)gin, c, Shape{n, h, w}, accumulate);
    return check_launch("unet_pool2_bwd");
}

int fwi_unet_up2(const void *in, void *out, int c, int n, int h, int w, void *stream) {
    UREQ(in && out && c > 0 && n > 0 && h > 0 && w > 0, "fwi_unet_up2: bad arguments");
    up2_kernel<<<elem_blocks(4ll * n * h * w * c), kElemThreads, 0, (cudaStream_t)stream>>>(
        (const bf16 *)in, (bf16 *)out, c, Shape{n, h, w});
    return check_launch("unet_up2");
}

int fwi_unet_up2_bwd(const void *gout, void *gin, int c, int n, int h, int w, void *stream) {
    UREQ(gout && gin && c > 0 && n > 0 && h > 0 && w > 0, "fwi_unet_up2_bwd: bad arguments");
    up2_bwd_kernel<<<elem_blocks((long long)n * h * w * c), kElemThreads, 0, (cudaStream_t)stream>>>(
        (const bf16 *)gout, (bf16 *)gin, c, Shape{n, h, w});
    return check_launch("unet_up2_bwd");
}

int fwi_unet_head(const void *x, const float *w, const float *b, float *out, int n, int h, int wd, void *stream) {
    UREQ(x && w && b && out && n > 0 && h > 0 && wd > 0, "fwi_unet_head: bad arguments");
    const long long npix = (long long)n * h * wd;
    head_kernel<16><<<elem_blocks(npix), kElemThreads, 0, (cudaStream_t)stream>>>((const bf16 *)x, w, b, out, npix);
    return check_launch("unet_head");
}

int fwi_unet_head_bwd(const void *x, const float *w, const float *gout, void *gx, float *part, float *gwb, int n, int h,
                      int wd, void *stream) {
    UREQ(x && w && gout && gx && part && gwb && n > 0 && h > 0 && wd > 0, "fwi_unet_head_bwd: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    const long long npix = (long long)n * h * wd;
    const int rblk = (int)((npix + kRedPix - 1) / kRedPix);
    head_bwd_kernel<16><<<rblk, 256, 0, st>>>((const bf16 *)x, w, gout, (bf16 *)gx, part, npix);
    int rc = check_launch("unet_head_bwd");
    if (rc) return rc;
    block_sum_kernel<<<1, 32, 0, st>>>(part, rblk, 17, gwb);
    return check_launch("unet_head_bwd_sum");
}

int fwi_unet_pack(const float *planes, void *x, int n, int h, int w, void *stream) {
    UREQ(planes && x && n > 0 && h > 0 && w > 0, "fwi_unet_pack: bad arguments");
    pack_kernel<<<elem_blocks((long long)n * h * w), kElemThreads, 0, (cudaStream_t)stream>>>(planes, (bf16 *)x,
                                                                                               Shape{n, h, w});
    return check_launch("unet_pack");
}

int fwi_unet_adam(float *w, float *m, float *v, const float *g, void *wb, long long count, double lr, double beta1,
                  double beta2, double eps, int step, void *stream) {
    UREQ(w && m && v && g && count >= 0 && step >= 1, "fwi_unet_adam: bad arguments");
    if (!count) return 0;
    const float c1 = (float)(1.0 - pow(beta1, step)), c2 = (float)(1.0 - pow(beta2, step));
    adam_kernel<<<elem_blocks(count), kElemThreads, 0, (cudaStream_t)stream>>>(
        w, m, v, g, (bf16 *)wb, count, (float)lr, (float)beta1, (float)beta2, (float)eps, c1, c2);
    return check_launch("unet_adam");
}

long long fwi_unet_mse_partials(void) { return kMseBlocks; }

int fwi_unet_mse(const float *out, const float *tgt, float *gout, double *loss, double *part, long long count,
                 void *stream) {
    UREQ(out && tgt && gout && loss && part && count > 0, "fwi_unet_mse: bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    mse_kernel<<<kMseBlocks, 256, 0, st>>>(out, tgt, gout, count, part);
    int rc = check_launch("unet_mse");
    if (rc) return rc;
    mse_finish_kernel<<<1, 1, 0, st>>>(part, kMseBlocks, count, loss);
    return check_launch("unet_mse_finish");
}

}  // extern "C"

cudaError_t fwi::unet_set_wait_limit(int polls) { return fwi::set_wait_limit_here(polls); }
