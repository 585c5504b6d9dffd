// MLP surrogate of the MRA log-likelihood: n_in -> 128 -> 128 -> 1 with SiLU,
// BF16 weights in the forward and backward passes, FP32 accumulation, FP32
// master parameters updated by Adam (include/mra_surrogate.h).
//
// One kernel does the forward pass, the backward pass and the per-CTA
// gradient sums over a grid-strided set of 16-sample tiles; a second kernel
// adds the per-CTA sums in a fixed order (deterministic) and applies Adam.
// Predictions without input gradients (the screening of candidate parameter
// vectors) run k_mlp_forward_tc instead, whose 128 x 128 layer is a
// tcgen05.mma product in tensor memory.
// Thread h of a CTA owns hidden unit h: row h of W2 sits in its registers for
// the forward product, and the backward product through W2 reads the BF16
// copy of W2 in shared memory column-wise (consecutive threads, consecutive
// addresses).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/mra_surrogate.h"
#include "mra_kernels.cuh"

namespace {

constexpr int H = 128;     // hidden width
constexpr int S = 16;      // samples per tile
constexpr int MAXD = 64;   // largest input width
constexpr long MAXN = 65536;

enum Mode { TRAIN = 0, PREDICT = 1, PREDICT_GRAD = 2 };

struct Layout {
    long W1, b1, W2, b2, w3, b3, P;
    explicit Layout(int D) {
        W1 = 0;
        b1 = W1 + (long)H * D;
        W2 = b1 + H;
        b2 = W2 + (long)H * H;
        w3 = b2 + H;
        b3 = w3 + H;
        P = b3 + 1;
    }
};

struct MlpArgs {
    int D;
    long N;
    long W1, b1, W2, b2, w3, b3, P;
    const float* master;
    const __nv_bfloat16* W1b;   // [H][D]
    const __nv_bfloat16* W2b;   // [H][H]
    const __nv_bfloat16* w3b;   // [H]
    const float* X;             // [N][D]
    const float* T;             // [N]      (TRAIN)
    float* partial;             // [grid][P+1] per-CTA gradient sums, last = loss sum (TRAIN)
    float* Y;                   // [N]      (PREDICT*)
    float* G;                   // [N][D]   (PREDICT_GRAD)
};

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + expf(-z)); }

size_t smem_bytes(int mode, int D) {
    size_t b = (size_t)H * H * sizeof(__nv_bfloat16)   // W2 (row-major)
               + (size_t)D * H * sizeof(__nv_bfloat16) // W1 transposed [d][h]
               + (size_t)S * MAXD * sizeof(float)      // x tile
               + 2 * (size_t)S * H * sizeof(float)     // a1, g_z2 tiles
               + (size_t)S * 4 * sizeof(float);        // y partial sums per warp
    if (mode == TRAIN) b += (size_t)H * H * sizeof(float) + (size_t)D * H * sizeof(float);
    return b;
}

template <int MODE>
__global__ void __launch_bounds__(H) k_mlp_pass(MlpArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int D = a.D;
    const int h = threadIdx.x, warp = h >> 5, lane = h & 31;
    __nv_bfloat16* W2s = reinterpret_cast<__nv_bfloat16*>(smem);
    __nv_bfloat16* W1t = W2s + H * H;
    float* xs = reinterpret_cast<float*>(W1t + D * H);
    float* a1s = xs + S * MAXD;
    float* gzs = a1s + S * H;
    float* red = gzs + S * H;
    float* dW2 = red + S * 4;   // TRAIN only: [o][i], thread i owns column i
    float* dW1 = dW2 + H * H;   // TRAIN only: [d][h]

    // row h of W2 in registers (bf16 pairs)
    __nv_bfloat162 w2r[H / 2];
    const __nv_bfloat162* w2row = reinterpret_cast<const __nv_bfloat162*>(a.W2b + (long)h * H);
#pragma unroll
    for (int q = 0; q < H / 2; ++q) w2r[q] = w2row[q];
    for (int e = h; e < H * H; e += H) W2s[e] = a.W2b[e];
    for (int e = h; e < H * D; e += H) {
        int hh = e / D, d = e % D;
        W1t[d * H + hh] = a.W1b[e];
    }
    const float b1h = a.master[a.b1 + h], b2h = a.master[a.b2 + h], b3 = a.master[a.b3];
    const float w3h = __bfloat162float(a.w3b[h]);
    float db1 = 0.f, db2 = 0.f, dw3 = 0.f, db3 = 0.f, lsum = 0.f;
    if (MODE == TRAIN) {
        for (int o = 0; o < H; ++o) dW2[o * H + h] = 0.f;
        for (int d = 0; d < D; ++d) dW1[d * H + h] = 0.f;
    }
    __syncthreads();

    const long ntiles = (a.N + S - 1) / S;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long s0 = tile * S;
        const int ns = (int)min((long)S, a.N - s0);
        for (int e = h; e < S * D; e += H) {
            int s = e / D, d = e % D;
            xs[s * MAXD + d] = s < ns ? a.X[(s0 + s) * D + d] : 0.f;
        }
        __syncthreads();
        // layer 1
        float z1[S], z2[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            float acc = b1h;
            for (int d = 0; d < D; ++d) acc = fmaf(__bfloat162float(W1t[d * H + h]), xs[s * MAXD + d], acc);
            z1[s] = acc;
            a1s[s * H + h] = acc * sigm(acc);
        }
        __syncthreads();
        // layer 2 and the output
#pragma unroll
        for (int s = 0; s < S; ++s) {
            float acc = b2h;
            const float2* ar = reinterpret_cast<const float2*>(a1s + s * H);
#pragma unroll
            for (int q = 0; q < H / 2; ++q) {
                float2 w = __bfloat1622float2(w2r[q]);
                float2 x = ar[q];
                acc = fmaf(w.x, x.x, acc);
                acc = fmaf(w.y, x.y, acc);
            }
            z2[s] = acc;
            float p = w3h * (acc * sigm(acc));
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) p += __shfl_xor_sync(0xffffffffu, p, o);
            if (lane == 0) red[s * 4 + warp] = p;
        }
        __syncthreads();
        float gy[S];
#pragma unroll
        for (int s = 0; s < S; ++s) {
            float y = b3 + ((red[s * 4 + 0] + red[s * 4 + 1]) + (red[s * 4 + 2] + red[s * 4 + 3]));
            if (MODE == TRAIN) {
                float e = s < ns ? y - a.T[s0 + s] : 0.f;
                gy[s] = 2.f * e / (float)a.N;
                if (h == 0) lsum += e * e;
            } else {
                gy[s] = s < ns ? 1.f : 0.f;
                if (h == 0 && s < ns) a.Y[s0 + s] = y;
            }
        }
        if constexpr (MODE == PREDICT) {
            __syncthreads();
        } else {
            // backward through the output layer
#pragma unroll
            for (int s = 0; s < S; ++s) {
                float sg = sigm(z2[s]);
                float a2 = z2[s] * sg;
                float g = gy[s] * w3h * (sg * (1.f + z2[s] * (1.f - sg)));
                gzs[s * H + h] = g;
                if (MODE == TRAIN) {
                    dw3 = fmaf(gy[s], a2, dw3);
                    db2 += g;
                    if (h == 0) db3 += gy[s];
                }
            }
            __syncthreads();
            float a1h[S];
#pragma unroll
            for (int s = 0; s < S; ++s) a1h[s] = a1s[s * H + h];
            if (MODE == TRAIN) {
                for (int o = 0; o < H; ++o) {
                    float acc = 0.f;
#pragma unroll
                    for (int s = 0; s < S; ++s) acc = fmaf(gzs[s * H + o], a1h[s], acc);
                    dW2[o * H + h] += acc;
                }
            }
            // through W2 and the first activation
            float gz1[S];
#pragma unroll
            for (int s = 0; s < S; ++s) gz1[s] = 0.f;
            for (int o = 0; o < H; ++o) {
                float w = __bfloat162float(W2s[o * H + h]);
#pragma unroll
                for (int s = 0; s < S; ++s) gz1[s] = fmaf(w, gzs[s * H + o], gz1[s]);
            }
#pragma unroll
            for (int s = 0; s < S; ++s) {
                float sg = sigm(z1[s]);
                gz1[s] *= sg * (1.f + z1[s] * (1.f - sg));
            }
            if (MODE == TRAIN) {
#pragma unroll
                for (int s = 0; s < S; ++s) db1 += gz1[s];
                for (int d = 0; d < D; ++d) {
                    float acc = 0.f;
#pragma unroll
                    for (int s = 0; s < S; ++s) acc = fmaf(gz1[s], xs[s * MAXD + d], acc);
                    dW1[d * H + h] += acc;
                }
            } else {
                // d y / d x: sum over hidden units of W1[h][d] g_z1[h]
                __syncthreads();
#pragma unroll
                for (int s = 0; s < S; ++s) gzs[s * H + h] = gz1[s];
                __syncthreads();
                for (int e = h; e < S * D; e += H) {
                    int s = e / D, d = e % D;
                    float acc = 0.f;
                    for (int k = 0; k < H; ++k) acc = fmaf(__bfloat162float(W1t[d * H + k]), gzs[s * H + k], acc);
                    if (s < ns) a.G[(s0 + s) * D + d] = acc;
                }
            }
            __syncthreads();
        }
    }
    if (MODE != TRAIN) return;
    float* out = a.partial + (long)blockIdx.x * (a.P + 1);
    for (int d = 0; d < D; ++d) out[a.W1 + (long)h * D + d] = dW1[d * H + h];
    out[a.b1 + h] = db1;
    for (int o = 0; o < H; ++o) out[a.W2 + (long)o * H + h] = dW2[o * H + h];
    out[a.b2 + h] = db2;
    out[a.w3 + h] = dw3;
    if (h == 0) {
        out[a.b3] = db3;
        out[a.P] = lsum;
    }
}

// Sums the per-CTA partials in CTA order; grad_out != nullptr: store the
// gradient (and loss); else one Adam step on the master weights and their BF16
// copies.  bc1/bc2: 1 - beta^t bias corrections.
__global__ void k_mlp_reduce_adam(long P, int nblk, const float* __restrict__ partial, float* grad_out,
                                  float* loss_out, float* master, float* m, float* v, __nv_bfloat16* W1b,
                                  __nv_bfloat16* W2b, __nv_bfloat16* w3b, long oW2, long ob2, long ow3, long ob3,
                                  long ob1, float lr, float bc1, float bc2) {
    long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p > P) return;
    float g = 0.f;
    for (int c = 0; c < nblk; ++c) g += partial[(long)c * (P + 1) + p];
    if (p == P) {
        if (loss_out) *loss_out = g;
        return;
    }
    if (grad_out) {
        grad_out[p] = g;
        return;
    }
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float mm = b1 * m[p] + (1.f - b1) * g;
    float vv = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    float w = master[p] - lr * (mm / bc1) / (sqrtf(vv / bc2) + eps);
    master[p] = w;
    if (p < ob1) W1b[p] = __float2bfloat16_rn(w);
    else if (p >= oW2 && p < ob2) W2b[p - oW2] = __float2bfloat16_rn(w);
    else if (p >= ow3 && p < ob3) w3b[p - ow3] = __float2bfloat16_rn(w);
}

__global__ void k_mlp_sync_bf16(long P, const float* master, __nv_bfloat16* W1b, __nv_bfloat16* W2b,
                                __nv_bfloat16* w3b, long oW2, long ob2, long ow3, long ob3, long ob1) {
    long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= P) return;
    float w = master[p];
    if (p < ob1) W1b[p] = __float2bfloat16_rn(w);
    else if (p >= oW2 && p < ob2) W2b[p - oW2] = __float2bfloat16_rn(w);
    else if (p >= ow3 && p < ob3) w3b[p - ow3] = __float2bfloat16_rn(w);
}

// ---------------------------------------------------------------------------
// Forward pass on the 5th-generation tensor cores (prediction without input
// gradients).  One CTA of 128 threads takes tiles of 128 samples, thread t =
// sample t of the tile = TMEM lane t:
//   layer 1 (n_in x 128, small) on the FP32 cores, exactly as k_mlp_pass;
//   layer 2 (128 x 128 x 128) as tcgen05.mma kind::tf32 with the product in
//     tensor memory: a1 is split into a TF32 high part and the FP32 remainder
//     (a1 = hi + lo, hi exact in TF32), W2 is BF16 and hence exact in TF32, so
//     hi W2^T + lo W2^T is FP32-accurate (the remainder's own truncation to TF32
//     costs at most 2^-21 |a1|);
//   the output layer on the FP32 cores from the product read back by tcgen05.ld.
// Operands sit in shared memory in the canonical K-major layout without
// swizzle: 8-row x 16-byte core matrices, the two core matrices of one MMA's K
// slice 128 bytes apart (leading byte offset), consecutive 8-row groups 4096
// bytes apart (stride byte offset).  One thread issues the MMAs and commits
// them to an mbarrier; the others wait on it with a bounded spin.
constexpr int TC_M = 128;                    // samples per tile = MMA M = TMEM lanes
constexpr unsigned TC_LBO = 128, TC_SBO = 4096;
constexpr long kTcSpin = 1L << 24;           // bounded waits (about a second)

struct TcSmem {
    float Ahi[TC_M * H];                     // 64 KB each, canonical K-major layout
    float Alo[TC_M * H];
    float W2f[H * H];                        // rows = output units
    __nv_bfloat16 W1t[MAXD * H];             // layer 1 weights [d][h]
    float b1[H], b2[H], w3[H];
    unsigned long long bar;                  // MMA completion
    unsigned tmem_base;
    int abort;
};

// element (row, k) of a 128-row, 128-deep K-major tile of 4-byte elements
__device__ __forceinline__ int tc_idx(int row, int k) {
    return (row >> 3) * (int)(TC_SBO / 4) + (k >> 2) * (int)(TC_LBO / 4) + (row & 7) * 4 + (k & 3);
}
__device__ __forceinline__ unsigned tc_smem(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
// shared-memory matrix descriptor: start, leading / stride byte offsets (>> 4),
// descriptor version 1 (bits 46-47), no swizzle
__device__ __forceinline__ unsigned long long tc_desc(unsigned addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFF) | ((unsigned long long)((TC_LBO >> 4) & 0x3FFF) << 16) |
           ((unsigned long long)((TC_SBO >> 4) & 0x3FFF) << 32) | (1ull << 46);
}
// instruction descriptor: D F32 (bits 4-5 = 1), A and B TF32 (bits 7-9, 10-12 = 2),
// both K-major, N = 128 (bits 17-22 = N >> 3), M = 128 (bits 24-28 = M >> 4)
constexpr unsigned kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(H >> 3) << 17) | ((unsigned)(TC_M >> 4) << 24);

// D[tmem] (+)= A B^T for one K slice of 8, A and B given by their descriptors
__device__ __forceinline__ void tc_mma(unsigned tmem, unsigned long long adesc, unsigned long long bdesc, bool acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
        "l"(adesc), "l"(bdesc), "r"(kTcIdesc), "r"((unsigned)acc)
        : "memory");
}
__device__ __forceinline__ bool tc_try_wait(unsigned long long* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(tc_smem(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// 32 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld32(unsigned taddr, float (&v)[32]) {
    unsigned r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int q = 0; q < 32; ++q) v[q] = __uint_as_float(r[q]);
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// y = MLP(x) for a.N samples (a.Y); *err = 1 if a bounded wait gave up.
__global__ void __launch_bounds__(TC_M, 1) k_mlp_forward_tc(MlpArgs a, int* err) {
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    TcSmem& sm = *reinterpret_cast<TcSmem*>(tc_raw);
    const int tid = threadIdx.x, warp = tid >> 5, D = a.D;
    for (int e = tid; e < H * H; e += TC_M) sm.W2f[tc_idx(e / H, e % H)] = __bfloat162float(a.W2b[e]);
    for (int e = tid; e < H * D; e += TC_M) sm.W1t[(e % D) * H + e / D] = a.W1b[e];
    for (int h = tid; h < H; h += TC_M) {
        sm.b1[h] = a.master[a.b1 + h];
        sm.b2[h] = a.master[a.b2 + h];
        sm.w3[h] = __bfloat162float(a.w3b[h]);
    }
    if (tid == 0) {
        sm.abort = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(tc_smem(&sm.bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) {
        // 128 TMEM columns: the 128 x 128 FP32 product of one tile
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(tc_smem(&sm.tmem_base)),
                     "r"(H)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = sm.tmem_base;
    const unsigned lane_addr = tmem + ((unsigned)(warp * 32) << 16);
    const float b3 = a.master[a.b3];
    const long ntiles = (a.N + TC_M - 1) / TC_M;
    unsigned parity = 0;
    for (long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long s = tile * TC_M + tid;
        const bool valid = s < a.N;
        // layer 1 on the FP32 cores, in k_mlp_pass's order: z1 = b1 + sum_d W1[h][d] x[d]
        float z[H];
#pragma unroll
        for (int h = 0; h < H; ++h) z[h] = sm.b1[h];
        for (int d = 0; d < D; ++d) {
            const float xd = valid ? a.X[s * D + d] : 0.f;
#pragma unroll
            for (int h = 0; h < H; ++h) z[h] = fmaf(__bfloat162float(sm.W1t[d * H + h]), xd, z[h]);
        }
#pragma unroll
        for (int h = 0; h < H; ++h) {
            const float a1 = z[h] * sigm(z[h]);
            const float hi = __uint_as_float(__float_as_uint(a1) & 0xffffe000u);  // exact in TF32
            sm.Ahi[tc_idx(tid, h)] = hi;
            sm.Alo[tc_idx(tid, h)] = a1 - hi;
        }
        // the tile's operands, written by every thread, become visible to the tensor core
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        tc_fence_before();
        __syncthreads();
        if (tid == 0) {
            tc_fence_after();
            const unsigned ahi = tc_smem(sm.Ahi), alo = tc_smem(sm.Alo), bw = tc_smem(sm.W2f);
            for (int k = 0; k < H / 8; ++k) {
                const unsigned off = (unsigned)k * 2u * TC_LBO;  // K slice k: core matrices 2k, 2k+1
                tc_mma(tmem, tc_desc(ahi + off), tc_desc(bw + off), k > 0);
                tc_mma(tmem, tc_desc(alo + off), tc_desc(bw + off), true);
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             tc_smem(&sm.bar))
                         : "memory");
        }
        bool done = false;
        for (long it = 0; it < kTcSpin && !done; ++it) done = tc_try_wait(&sm.bar, parity);
        parity ^= 1u;
        if (__syncthreads_or(done ? 0 : 1)) {
            if (tid == 0) atomicExch(err, 1);
            break;
        }
        tc_fence_after();
        float y = b3;
#pragma unroll
        for (int c = 0; c < H / 32; ++c) {
            float v[32];
            tc_ld32(lane_addr + (unsigned)(32 * c), v);
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int q = 0; q < 32; ++q) {
                const float z2 = v[q] + sm.b2[32 * c + q];
                y = fmaf(sm.w3[32 * c + q], z2 * sigm(z2), y);
            }
        }
        if (valid) a.Y[s] = y;
        // every thread's reads of the product precede the next tile's MMAs into it
        tc_fence_before();
        __syncthreads();
    }
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(H) : "memory");
    }
}

mra_status mfail(mra_status s, const std::string& msg) {
    mra::set_last_error(msg.c_str());
    return s;
}

#define MCU(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return mfail(e_ == cudaErrorMemoryAllocation ? MRA_ERR_OOM : MRA_ERR_CUDA,            \
                         std::string(#call ": ") + cudaGetErrorString(e_));                       \
    } while (0)

}  // namespace

struct mra_mlp {
    int D = 0;
    Layout lay{1};
    int sms = 0;
    int t = 0;  // Adam steps taken
    long N = 0, Nq_cap = 0;
    cudaStream_t stream = nullptr;
    float *master = nullptr, *m = nullptr, *v = nullptr;
    __nv_bfloat16 *W1b = nullptr, *W2b = nullptr, *w3b = nullptr;
    float *X = nullptr, *T = nullptr, *partial = nullptr, *grad = nullptr, *loss = nullptr;
    float *Xq = nullptr, *Yq = nullptr, *Gq = nullptr;
    int grid_train = 1;
    int* tc_err = nullptr;  // bounded-wait status of the tensor-core forward pass
};

namespace {

MlpArgs args_of(const mra_mlp* n, long N, const float* X) {
    MlpArgs a{};
    a.D = n->D;
    a.N = N;
    a.W1 = n->lay.W1; a.b1 = n->lay.b1; a.W2 = n->lay.W2; a.b2 = n->lay.b2;
    a.w3 = n->lay.w3; a.b3 = n->lay.b3; a.P = n->lay.P;
    a.master = n->master;
    a.W1b = n->W1b; a.W2b = n->W2b; a.w3b = n->w3b;
    a.X = X;
    a.T = n->T;
    a.partial = n->partial;
    return a;
}

mra_status launch_train_pass(mra_mlp* n) {
    if (n->N <= 0) return mfail(MRA_ERR_STATE, "mra_mlp: no training data (mra_mlp_set_data)");
    MlpArgs a = args_of(n, n->N, n->X);
    long ntiles = (n->N + S - 1) / S;
    n->grid_train = (int)std::min<long>(ntiles, n->sms);
    k_mlp_pass<TRAIN><<<n->grid_train, H, smem_bytes(TRAIN, n->D), n->stream>>>(a);
    MCU(cudaGetLastError());
    return MRA_OK;
}

mra_status launch_reduce(mra_mlp* n, float* grad_out, float* loss_out, float lr) {
    const Layout& L = n->lay;
    float bc1 = 1.f, bc2 = 1.f;
    if (!grad_out) {
        n->t += 1;
        bc1 = 1.f - std::pow(0.9f, (float)n->t);
        bc2 = 1.f - std::pow(0.999f, (float)n->t);
    }
    long blocks = (L.P + 1 + 255) / 256;
    k_mlp_reduce_adam<<<(unsigned)blocks, 256, 0, n->stream>>>(L.P, n->grid_train, n->partial, grad_out, loss_out,
                                                                n->master, n->m, n->v, n->W1b, n->W2b, n->w3b, L.W2,
                                                                L.b2, L.w3, L.b3, L.b1, lr, bc1, bc2);
    MCU(cudaGetLastError());
    return MRA_OK;
}

mra_status sync_bf16(mra_mlp* n) {
    const Layout& L = n->lay;
    k_mlp_sync_bf16<<<(unsigned)((L.P + 255) / 256), 256, 0, n->stream>>>(L.P, n->master, n->W1b, n->W2b, n->w3b,
                                                                           L.W2, L.b2, L.w3, L.b3, L.b1);
    MCU(cudaGetLastError());
    return MRA_OK;
}

}  // namespace

extern "C" {

mra_status mra_mlp_create(int32_t n_in, int32_t hidden, uint64_t seed, mra_mlp** out) {
    if (!out) return mfail(MRA_ERR_ARG, "mra_mlp_create: out is NULL");
    *out = nullptr;
    if (n_in < 1 || n_in > MAXD) return mfail(MRA_ERR_ARG, "mra_mlp_create: n_in must be in 1..64");
    if (hidden != H) return mfail(MRA_ERR_ARG, "mra_mlp_create: hidden width must be 128");
    int dev = 0, count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) return mfail(MRA_ERR_NO_DEVICE, "no CUDA device");
    MCU(cudaGetDevice(&dev));
    cudaDeviceProp prop;
    MCU(cudaGetDeviceProperties(&prop, dev));
    if (prop.major != 10) return mfail(MRA_ERR_NO_DEVICE, "mra_mlp: needs an sm_100 device");
    mra_mlp* n = new mra_mlp();
    n->D = n_in;
    n->lay = Layout(n_in);
    n->sms = prop.multiProcessorCount;
    const long P = n->lay.P;
    auto fail_free = [&](mra_status s) {
        mra_mlp_destroy(n);
        return s;
    };
#define MALLOC(ptr, bytes)                                                                          \
    do {                                                                                            \
        cudaError_t e_ = cudaMalloc((void**)&(ptr), (bytes));                                       \
        if (e_ != cudaSuccess) return fail_free(mfail(MRA_ERR_OOM, "mra_mlp: device allocation"));  \
    } while (0)
    if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail_free(mfail(MRA_ERR_CUDA, "mra_mlp: stream"));
    MALLOC(n->master, P * sizeof(float));
    MALLOC(n->m, P * sizeof(float));
    MALLOC(n->v, P * sizeof(float));
    MALLOC(n->W1b, (size_t)H * n_in * sizeof(__nv_bfloat16));
    MALLOC(n->W2b, (size_t)H * H * sizeof(__nv_bfloat16));
    MALLOC(n->w3b, (size_t)H * sizeof(__nv_bfloat16));
    MALLOC(n->partial, (size_t)n->sms * (P + 1) * sizeof(float));
    MALLOC(n->grad, (size_t)(P + 1) * sizeof(float));
    MALLOC(n->loss, sizeof(float));
#undef MALLOC
    for (int mode = 0; mode < 3; ++mode) {
        size_t sb = smem_bytes(mode, n_in);
        cudaError_t e = mode == TRAIN ? cudaFuncSetAttribute(k_mlp_pass<TRAIN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb)
                        : mode == PREDICT ? cudaFuncSetAttribute(k_mlp_pass<PREDICT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb)
                                          : cudaFuncSetAttribute(k_mlp_pass<PREDICT_GRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sb);
        if (e != cudaSuccess) return fail_free(mfail(MRA_ERR_CUDA, std::string("mra_mlp: smem attribute: ") + cudaGetErrorString(e)));
    }
    {
        cudaError_t e = cudaFuncSetAttribute(k_mlp_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)sizeof(TcSmem));
        if (e != cudaSuccess) return fail_free(mfail(MRA_ERR_CUDA, std::string("mra_mlp: smem attribute: ") + cudaGetErrorString(e)));
    }
    // Glorot-uniform weights from a host generator, zero biases
    std::vector<float> p(P, 0.f);
    std::mt19937_64 gen(seed);
    auto fill = [&](long off, long count, int fan_in, int fan_out) {
        float lim = std::sqrt(6.f / (float)(fan_in + fan_out));
        std::uniform_real_distribution<float> u(-lim, lim);
        for (long k = 0; k < count; ++k) p[off + k] = u(gen);
    };
    fill(n->lay.W1, (long)H * n_in, n_in, H);
    fill(n->lay.W2, (long)H * H, H, H);
    fill(n->lay.w3, H, H, 1);
    mra_status s = mra_mlp_set_params(n, p.data());
    if (s != MRA_OK) return fail_free(s);
    *out = n;
    return MRA_OK;
}

mra_status mra_mlp_destroy(mra_mlp* n) {
    if (!n) return MRA_OK;
    float* fbufs[] = {n->master, n->m, n->v, n->X, n->T, n->partial, n->grad, n->loss, n->Xq, n->Yq, n->Gq};
    for (float* b : fbufs)
        if (b) cudaFree(b);
    if (n->W1b) cudaFree(n->W1b);
    if (n->W2b) cudaFree(n->W2b);
    if (n->w3b) cudaFree(n->w3b);
    if (n->tc_err) cudaFree(n->tc_err);
    if (n->stream) cudaStreamDestroy(n->stream);
    delete n;
    return MRA_OK;
}

mra_status mra_mlp_num_params(const mra_mlp* n, int64_t* out) {
    if (!n || !out) return mfail(MRA_ERR_ARG, "mra_mlp_num_params: NULL argument");
    *out = n->lay.P;
    return MRA_OK;
}

mra_status mra_mlp_get_params(mra_mlp* n, float* params) {
    if (!n || !params) return mfail(MRA_ERR_ARG, "mra_mlp_get_params: NULL argument");
    MCU(cudaMemcpyAsync(params, n->master, n->lay.P * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    MCU(cudaStreamSynchronize(n->stream));
    return MRA_OK;
}

mra_status mra_mlp_set_params(mra_mlp* n, const float* params) {
    if (!n || !params) return mfail(MRA_ERR_ARG, "mra_mlp_set_params: NULL argument");
    for (long k = 0; k < n->lay.P; ++k)
        if (!std::isfinite(params[k])) return mfail(MRA_ERR_ARG, "mra_mlp_set_params: non-finite parameter");
    const size_t bytes = n->lay.P * sizeof(float);
    MCU(cudaMemcpyAsync(n->master, params, bytes, cudaMemcpyHostToDevice, n->stream));
    MCU(cudaMemsetAsync(n->m, 0, bytes, n->stream));
    MCU(cudaMemsetAsync(n->v, 0, bytes, n->stream));
    n->t = 0;
    mra_status s = sync_bf16(n);
    if (s != MRA_OK) return s;
    MCU(cudaStreamSynchronize(n->stream));
    return MRA_OK;
}

mra_status mra_mlp_set_data(mra_mlp* n, const float* x, const float* t, int64_t N) {
    if (!n || !x || !t) return mfail(MRA_ERR_ARG, "mra_mlp_set_data: NULL argument");
    if (N < 1 || N > MAXN) return mfail(MRA_ERR_ARG, "mra_mlp_set_data: need 1 <= n <= 65536");
    for (long k = 0; k < N * n->D; ++k)
        if (!std::isfinite(x[k])) return mfail(MRA_ERR_ARG, "mra_mlp_set_data: non-finite input");
    for (long k = 0; k < N; ++k)
        if (!std::isfinite(t[k])) return mfail(MRA_ERR_ARG, "mra_mlp_set_data: non-finite target");
    if (!n->X) {
        MCU(cudaMalloc((void**)&n->X, (size_t)MAXN * n->D * sizeof(float)));
        MCU(cudaMalloc((void**)&n->T, (size_t)MAXN * sizeof(float)));
    }
    MCU(cudaMemcpyAsync(n->X, x, (size_t)N * n->D * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    MCU(cudaMemcpyAsync(n->T, t, (size_t)N * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    n->N = N;
    MCU(cudaStreamSynchronize(n->stream));
    return MRA_OK;
}

mra_status mra_mlp_grad(mra_mlp* n, float* grad, float* loss) {
    if (!n || !grad) return mfail(MRA_ERR_ARG, "mra_mlp_grad: NULL argument");
    mra_status s = launch_train_pass(n);
    if (s != MRA_OK) return s;
    s = launch_reduce(n, n->grad, n->loss, 0.f);
    if (s != MRA_OK) return s;
    MCU(cudaMemcpyAsync(grad, n->grad, n->lay.P * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    float l = 0.f;
    MCU(cudaMemcpyAsync(&l, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    MCU(cudaStreamSynchronize(n->stream));
    if (loss) *loss = l / (float)n->N;
    return MRA_OK;
}

mra_status mra_mlp_train(mra_mlp* n, int32_t steps, float lr, float* loss_out) {
    if (!n) return mfail(MRA_ERR_ARG, "mra_mlp_train: NULL argument");
    if (steps < 0 || !(lr > 0.f) || !std::isfinite(lr)) return mfail(MRA_ERR_ARG, "mra_mlp_train: bad steps or lr");
    for (int k = 0; k < steps; ++k) {
        mra_status s = launch_train_pass(n);
        if (s != MRA_OK) return s;
        s = launch_reduce(n, nullptr, n->loss, lr);
        if (s != MRA_OK) return s;
    }
    float l = 0.f;
    MCU(cudaMemcpyAsync(&l, n->loss, sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    MCU(cudaStreamSynchronize(n->stream));
    if (loss_out) *loss_out = n->N ? l / (float)n->N : 0.f;
    return MRA_OK;
}

mra_status mra_mlp_predict(mra_mlp* n, const float* x, int64_t N, float* y, float* dydx) {
    if (!n || !x || !y) return mfail(MRA_ERR_ARG, "mra_mlp_predict: NULL argument");
    if (N < 1 || N > MAXN) return mfail(MRA_ERR_ARG, "mra_mlp_predict: need 1 <= n <= 65536");
    if (!n->Xq) {
        MCU(cudaMalloc((void**)&n->Xq, (size_t)MAXN * n->D * sizeof(float)));
        MCU(cudaMalloc((void**)&n->Yq, (size_t)MAXN * sizeof(float)));
        MCU(cudaMalloc((void**)&n->Gq, (size_t)MAXN * n->D * sizeof(float)));
    }
    if (!n->tc_err) MCU(cudaMalloc((void**)&n->tc_err, sizeof(int)));
    MCU(cudaMemcpyAsync(n->Xq, x, (size_t)N * n->D * sizeof(float), cudaMemcpyHostToDevice, n->stream));
    MlpArgs a = args_of(n, N, n->Xq);
    a.Y = n->Yq;
    a.G = n->Gq;
    if (dydx) {
        const long ntiles = (N + S - 1) / S;
        const int grid = (int)std::min<long>(ntiles, 4L * n->sms);
        k_mlp_pass<PREDICT_GRAD><<<grid, H, smem_bytes(PREDICT_GRAD, n->D), n->stream>>>(a);
    } else {
        // values only: the 128 x 128 layer on the tensor cores (tcgen05), 128 samples per tile
        MCU(cudaMemsetAsync(n->tc_err, 0, sizeof(int), n->stream));
        const long ntiles = (N + TC_M - 1) / TC_M;
        const int grid = (int)std::min<long>(ntiles, n->sms);
        k_mlp_forward_tc<<<grid, TC_M, sizeof(TcSmem), n->stream>>>(a, n->tc_err);
    }
    MCU(cudaGetLastError());
    MCU(cudaMemcpyAsync(y, n->Yq, (size_t)N * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    if (dydx) MCU(cudaMemcpyAsync(dydx, n->Gq, (size_t)N * n->D * sizeof(float), cudaMemcpyDeviceToHost, n->stream));
    int tc_err = 0;
    if (!dydx) MCU(cudaMemcpyAsync(&tc_err, n->tc_err, sizeof(int), cudaMemcpyDeviceToHost, n->stream));
    MCU(cudaStreamSynchronize(n->stream));
    if (tc_err) return mfail(MRA_ERR_TIMEOUT, "mra_mlp_predict: the tensor-core product did not complete in time");
    return MRA_OK;
}

}  // extern "C"
