// Training and inference kernels of the learned proposal spread, and the
// trainer's C ABI (glac_mlp_*).  No counterpart in the reference.
//
// Objective (expected squared jump): each sample i carries the features f_i of a
// link's staple and J_i(eps_k), the mean squared jump ||U' - U||^2 of the
// sampler's NUpdates-hit update of that link with spread eps_k on a grid.  With
// J_i linear between grid points, the loss is L = -(1/n) sum_i J_i(eps(f_i)).
//
// One warp takes 16 samples per tile: the forward pass as in the Metropolis
// kernel, dL/dz from the slope of J_i, and the backward pass with BF16 operands
// and FP32 accumulation on the tensor cores (mma.m16n8k16).  Weight gradients
// are sums over samples, i.e. products with K = samples; their operands are the
// forward activations and deltas transposed in registers (movmatrix).  Each
// block writes its partial sums; a second pass adds the block partials in a
// fixed order, so the gradient is deterministic for a given n.
#include "../../include/glac_b200.h"
#include "learned.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <exception>
#include <random>
#include <string>
#include <vector>

namespace glac {

constexpr int kGradWarps = 4;
constexpr int kGradSlots = kMlpParams + 1;  // parameters + loss
constexpr int kGradMaxBlocks = 296;         // 2 x 148 SMs

// ---------------------------------------------------------------------------
// FP32 master parameters -> BF16 operand fragments
// ---------------------------------------------------------------------------
__device__ __forceinline__ float w1_entry(const float *P, int k, int n) {
    return k < 8 ? P[kMlpW1 + k * 32 + n] : (k == 8 ? P[kMlpB1 + n] : 0.f);
}

__global__ void k_mlp_pack(const float *__restrict__ P, uint32_t *__restrict__ pack) {
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= kPackWords) return;
    uint32_t out = 0;
    if (w < kPackW2) {  // [nt][lane][r]
        const int r = w & 1, lane = (w >> 1) & 31, nt = w >> 6;
        const int g = lane >> 2, t = lane & 3, k = 2 * t + 8 * r, n = 8 * nt + g;
        out = pack_bf16(w1_entry(P, k, n), w1_entry(P, k + 1, n));
    } else if (w < kPackW3) {  // [ks][nt][lane][r]
        const int x = w - kPackW2, r = x & 1, lane = (x >> 1) & 31, nt = (x >> 6) & 3, ks = x >> 8;
        const int g = lane >> 2, t = lane & 3, k = 16 * ks + 2 * t + 8 * r, n = 8 * nt + g;
        out = pack_bf16(P[kMlpW2 + k * 32 + n], P[kMlpW2 + (k + 1) * 32 + n]);
    } else if (w < kPackW2T) {  // [ks][lane][r]
        const int x = w - kPackW3, r = x & 1, lane = (x >> 1) & 31, ks = x >> 6;
        const int g = lane >> 2, t = lane & 3, k = 16 * ks + 2 * t + 8 * r;
        out = g == 0 ? pack_bf16(P[kMlpW3 + k], P[kMlpW3 + k + 1]) : 0u;
    } else if (w < kPackB2) {  // [ks][nt][lane][r], B[k = j][n = i] = W2[i][j]
        const int x = w - kPackW2T, r = x & 1, lane = (x >> 1) & 31, nt = (x >> 6) & 3, ks = x >> 8;
        const int g = lane >> 2, t = lane & 3, k = 16 * ks + 2 * t + 8 * r, n = 8 * nt + g;
        out = pack_bf16(P[kMlpW2 + n * 32 + k], P[kMlpW2 + n * 32 + k + 1]);
    } else if (w < kPackB3) {
        out = __float_as_uint(P[kMlpB2 + (w - kPackB2)]);
    } else if (w == kPackB3) {
        out = __float_as_uint(P[kMlpB3]);
    }
    pack[w] = out;
}

void launch_mlp_pack(const float *params, uint32_t *pack, cudaStream_t st) {
    k_mlp_pack<<<(kPackWords + 255) / 256, 256, 0, st>>>(params, pack);
}

// ---------------------------------------------------------------------------
// Inference over a feature array (the same warp routine the sampler runs)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_mlp_forward(const uint32_t *__restrict__ pack, const float *__restrict__ feat,
                                                     long long n, float eps_min, float eps_max,
                                                     float *__restrict__ eps_out) {
    __shared__ uint32_t smem[4 * 128];
    const long long i = (long long)blockIdx.x * 128 + threadIdx.x;
    float f[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    if (i < n) {
        const float4 a = __ldg(reinterpret_cast<const float4 *>(feat + i * 8));
        const float4 b = __ldg(reinterpret_cast<const float4 *>(feat + i * 8 + 4));
        f[0] = a.x; f[1] = a.y; f[2] = a.z; f[3] = a.w; f[4] = b.x; f[5] = b.y; f[6] = b.z; f[7] = b.w;
    }
    Proposal P;
    P.net = pack;
    P.eps_min = eps_min;
    P.eps_max = eps_max;
    const float e = mlp_spread_warp(f, P, smem + (threadIdx.x >> 5) * 128);
    if (i < n) eps_out[i] = e;
}

void launch_mlp_forward(const uint32_t *pack, const float *features, long long n, float eps_min, float eps_max,
                        float *eps_out, cudaStream_t st) {
    const long long blocks = (n + 127) / 128;
    k_mlp_forward<<<(unsigned)blocks, 128, 0, st>>>(pack, features, n, eps_min, eps_max, eps_out);
}

// ---------------------------------------------------------------------------
// Batched inference on the 5th-generation tensor cores (tcgen05, TMEM).
// A CTA of 4 warps takes 128 rows per tile.  Each layer is one or two
// tcgen05.mma.kind::f16 (M = 128, K = 16; BF16 A and B from shared memory,
// FP32 accumulator in tensor memory), issued by one thread and completed
// through an mbarrier; each warp then reads its 32 rows back (tcgen05.ld
// 32x32b), applies bias and activation, and writes the next layer's operand.
// Shared-memory operands use the canonical K-major layout without swizzle:
// 8-row x 16-byte core matrices, rows 16 B apart, 8-row groups SBO = 128 B
// apart, 16-byte K chunks LBO = rows x 16 B apart.  Rounding points are those
// of the warp-level path: BF16 inputs, weights, first-layer bias and
// activations, FP32 accumulation, FP32 b2 and b3.
// ---------------------------------------------------------------------------
namespace tcf {
constexpr int kA1 = 0;         // 128 x 16 BF16 (features, 1, zeros): 4096 B
constexpr int kA2 = 4096;      // 128 x 32: 8192 B
constexpr int kA3 = 12288;     // 128 x 32: 8192 B
constexpr int kB1 = 20480;     // W1^T with b1: 32 x 16: 1024 B
constexpr int kB2 = 21504;     // W2^T: 32 x 32: 2048 B
constexpr int kB3 = 23552;     // W3^T padded: 16 x 32: 1024 B
constexpr int kBar = 24576;    // mbarrier
constexpr int kSlot = 24584;   // TMEM base address written by tcgen05.alloc
constexpr int kSmem = 61440;   // requested, so that at most 3 CTAs (3 x 128 TMEM columns) share an SM
constexpr int kCols = 128;     // TMEM columns: D1 0-31, D2 32-63, D3 64-79

// byte offset of BF16 element (row, k) in a K-major, no-swizzle operand of `rows` rows
__device__ __forceinline__ uint32_t kmaj(int row, int k, int rows) {
    return (uint32_t)((row & 7) * 16 + (row >> 3) * 128 + (k >> 3) * rows * 16 + (k & 7) * 2);
}
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, int rows) {
    const uint64_t lbo = (uint64_t)(rows * 16) >> 4, sbo = 128 >> 4;
    return (uint64_t)((saddr >> 4) & 0x3FFF) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}
// kind::f16 instruction descriptor: FP32 D, BF16 A and B, both K-major, M = 128
__host__ __device__ constexpr uint32_t idesc(int n) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}
__device__ __forceinline__ void mma(uint32_t dtmem, uint64_t a, uint64_t b, uint32_t id, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(dtmem), "l"(a), "l"(b), "r"(id), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ void commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// Wait for the mbarrier phase for at most limit_ns nanoseconds of the global
// timer (each try_wait suspends for at most kSuspendNs); false on timeout.
constexpr uint32_t kSuspendNs = 1000;
__device__ __forceinline__ bool wait_phase(uint32_t bar, uint32_t phase, uint64_t limit_ns) {
    const uint64_t t0 = globaltimer_ns();
    for (;;) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred P;\n\tmbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2, %3;\n\t"
                     "selp.b32 %0, 1, 0, P;\n\t}\n"
                     : "=r"(done)
                     : "r"(bar), "r"(phase), "r"(kSuspendNs)
                     : "memory");
        if (done) return true;
        if (globaltimer_ns() - t0 > limit_ns) return false;
    }
}
__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
// 32 lanes x 32 columns: this thread's row, columns col .. col+31
__device__ __forceinline__ void ld32(uint32_t taddr, float v[32]) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 32; k++) v[k] = __uint_as_float(r[k]);
}
}  // namespace tcf

// err (atomicMax): 1 = a completion wait ran out and the tensor-core pipeline
// was drained before the TMEM was freed; 2 = it was still not drained after a
// second wait of the same length (the TMEM is freed all the same, as a CTA must
// before it exits, so the caller must stop using this library's tensor-core
// path).  issue = 0 is a test mode: no MMA and no commit are issued, so the
// first wait runs out with nothing in flight (the timeout path, without a
// fault or a hang).
__global__ void __launch_bounds__(128) k_mlp_forward_tc(const float *__restrict__ P, const float *__restrict__ feat,
                                                        long long n, float eps_min, float eps_max,
                                                        float *__restrict__ eps_out, int *__restrict__ err,
                                                        unsigned long long wait_ns, int issue) {
    using namespace tcf;
    extern __shared__ __align__(1024) unsigned char sm[];
    const int tid = threadIdx.x, warp = tid >> 5;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    uint32_t *slot = reinterpret_cast<uint32_t *>(sm + kSlot);
    __nv_bfloat16 *s16 = reinterpret_cast<__nv_bfloat16 *>(sm);
    auto put = [&](int base, int row, int k, int rows, float v) {
        s16[(base + (int)kmaj(row, k, rows)) >> 1] = __float2bfloat16_rn(v);
    };
    // weights (B operands, [n][k] = W[k][n]) once per CTA
    for (int e = tid; e < 32 * 16; e += 128) {
        const int nn = e >> 4, k = e & 15;
        put(kB1, nn, k, 32, k < 8 ? P[kMlpW1 + k * 32 + nn] : (k == 8 ? P[kMlpB1 + nn] : 0.f));
    }
    for (int e = tid; e < 32 * 32; e += 128) {
        const int nn = e >> 5, k = e & 31;
        put(kB2, nn, k, 32, P[kMlpW2 + k * 32 + nn]);
    }
    for (int e = tid; e < 16 * 32; e += 128) {
        const int nn = e >> 5, k = e & 31;
        put(kB3, nn, k, 16, nn == 0 ? P[kMlpW3 + k] : 0.f);
    }
    const float b3 = P[kMlpB3];
    const uint32_t bar = sbase + kBar;
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sbase + kSlot),
                     "r"(kCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    const uint32_t tmem = *slot;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
    uint32_t phase = 0;
    bool ok = true, drained = true;
    const long long tiles = (n + 127) / 128;
    // this thread's feature row of a tile (zeros past the end)
    auto fetch = [&](long long tile, float4 &a, float4 &b) {
        const long long r = tile * 128 + tid;
        if (tile < tiles && r < n) {
            a = __ldg(reinterpret_cast<const float4 *>(feat + r * 8));
            b = __ldg(reinterpret_cast<const float4 *>(feat + r * 8 + 4));
        } else {
            a = make_float4(0.f, 0.f, 0.f, 0.f);
            b = a;
        }
    };
    float4 fa, fb;
    fetch(blockIdx.x, fa, fb);
    for (long long tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
        const long long row = tile * 128 + tid;
        const float f[8] = {fa.x, fa.y, fa.z, fa.w, fb.x, fb.y, fb.z, fb.w};
        fetch(tile + gridDim.x, fa, fb);  // the next tile's row loads while this tile's layers run
        {
            uint4 c0, c1;
            c0.x = pack_bf16(f[0], f[1]); c0.y = pack_bf16(f[2], f[3]);
            c0.z = pack_bf16(f[4], f[5]); c0.w = pack_bf16(f[6], f[7]);
            c1.x = pack_bf16(1.f, 0.f); c1.y = 0u; c1.z = 0u; c1.w = 0u;
            *reinterpret_cast<uint4 *>(sm + kA1 + kmaj(tid, 0, 128)) = c0;
            *reinterpret_cast<uint4 *>(sm + kA1 + kmaj(tid, 8, 128)) = c1;
        }
        float h[32];
        // three layers: (A, K steps, B, B rows, D column, N)
        for (int layer = 0; layer < 3 && ok; layer++) {
            fence_async_smem();
            fence_before();
            __syncthreads();
            fence_after();
            const int A = layer == 0 ? kA1 : (layer == 1 ? kA2 : kA3);
            const int B = layer == 0 ? kB1 : (layer == 1 ? kB2 : kB3);
            const int brows = layer == 2 ? 16 : 32, N = layer == 2 ? 16 : 32, ksteps = layer == 0 ? 1 : 2;
            const uint32_t dcol = 32u * (uint32_t)layer;
            if (tid == 0 && issue) {
                for (int ks = 0; ks < ksteps; ks++)
                    mma(tmem + dcol, sdesc(sbase + A + ks * 2 * 128 * 16, 128),
                        sdesc(sbase + B + ks * 2 * brows * 16, brows), idesc(N), ks > 0 ? 1u : 0u);
                commit(bar);
            }
            // every thread takes the same branch, so no barrier below is skipped by some threads only
            ok = __syncthreads_and(wait_phase(bar, phase, wait_ns)) != 0;
            // on a timeout an issued MMA may still be in flight: one more bounded
            // wait before the loop ends and the TMEM is freed below
            if (!ok && issue) drained = __syncthreads_and(wait_phase(bar, phase, wait_ns)) != 0;
            phase ^= 1u;
            fence_after();
            if (!ok) break;
            ld32(lane_base + dcol, h);
            if (layer < 2) {
                const int Anext = layer == 0 ? kA2 : kA3;
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    float v[8];
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        const float x = layer == 1 ? h[8 * c + k] + P[kMlpB2 + 8 * c + k] : h[8 * c + k];
                        v[k] = leaky(x);
                    }
                    uint4 w;
                    w.x = pack_bf16(v[0], v[1]); w.y = pack_bf16(v[2], v[3]);
                    w.z = pack_bf16(v[4], v[5]); w.w = pack_bf16(v[6], v[7]);
                    *reinterpret_cast<uint4 *>(sm + Anext + kmaj(tid, 8 * c, 128)) = w;
                }
            } else if (row < n) {
                eps_out[row] = spread_of(h[0] + b3, eps_min, eps_max);
            }
        }
    }
    if (!ok && err && tid == 0) atomicMax(err, drained ? 1 : 2);
    fence_before();
    __syncthreads();
    fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols) : "memory");
}

void launch_mlp_forward_tc(const float *params, const float *features, long long n, float eps_min, float eps_max,
                           float *eps_out, int *err, unsigned long long wait_ns, int issue, cudaStream_t st) {
    // per device (cheap): the attribute is not shared between devices
    cudaFuncSetAttribute(k_mlp_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, tcf::kSmem);
    const long long tiles = (n + 127) / 128;
    const int grid = (int)(tiles < 3 * 148 ? tiles : 3 * 148);
    k_mlp_forward_tc<<<grid, 128, tcf::kSmem, st>>>(params, features, n, eps_min, eps_max, eps_out, err, wait_ns,
                                                    issue);
}

// ---------------------------------------------------------------------------
// Loss and gradient
// ---------------------------------------------------------------------------
// J_i(eps) linear between grid points; returns J and its slope.
__device__ __forceinline__ float esj_interp(const float *__restrict__ J, const float *__restrict__ grid, int n_eps,
                                            float eps, float &slope) {
    int k = 0;
    while (k < n_eps - 2 && grid[k + 1] <= eps) k++;
    const float e0 = grid[k], e1 = grid[k + 1];
    const float j0 = __ldg(J + k), j1 = __ldg(J + k + 1);
    slope = (j1 - j0) / (e1 - e0);
    return j0 + slope * (eps - e0);
}

// BF16 value of (C-layout) element c of an 8x8 block word pair: c = 0, 1 -> row g; the
// caller picks the word for rows g / g+8.
__device__ __forceinline__ float bf_el(uint32_t w, int c) { return c == 0 ? bf16_lo(w) : bf16_hi(w); }

__global__ void __launch_bounds__(128) k_mlp_grad(const float *__restrict__ P, const uint32_t *__restrict__ pack,
                                                  const float *__restrict__ feat, const float *__restrict__ esj,
                                                  long long n, int n_eps, const float *__restrict__ eps_grid,
                                                  float eps_min, float eps_max, float *__restrict__ partial) {
    __shared__ float red[kGradWarps][kGradSlots];
    __shared__ float grid_s[64];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    for (int k = threadIdx.x; k < n_eps; k += blockDim.x) grid_s[k] = eps_grid[k];
    __syncthreads();
    const long long ntiles = (n + 15) / 16;
    const long long nw = (long long)gridDim.x * kGradWarps;
    const float inv_n = 1.f / (float)n, span = eps_max - eps_min;
    const uint32_t one = t == 0 ? pack_bf16(1.f, 0.f) : 0u;
    const float *b2 = reinterpret_cast<const float *>(pack + kPackB2);
    const float b3 = reinterpret_cast<const float *>(pack + kPackB3)[0];
    float w3[4][2];
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
        w3[nt][0] = round_bf16(P[kMlpW3 + 8 * nt + 2 * t]);
        w3[nt][1] = round_bf16(P[kMlpW3 + 8 * nt + 2 * t + 1]);
    }
    float gW1[4][4], gW2[2][4][4], gb1[4][2], gb2[4][2], gW3[4][2], gb3 = 0.f, loss = 0.f;
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
#pragma unroll
        for (int c = 0; c < 4; c++) gW1[nt][c] = gW2[0][nt][c] = gW2[1][nt][c] = 0.f;
#pragma unroll
        for (int c = 0; c < 2; c++) gb1[nt][c] = gb2[nt][c] = gW3[nt][c] = 0.f;
    }

    for (long long tile = (long long)blockIdx.x * kGradWarps + warp; tile < ntiles; tile += nw) {
        const long long r0 = tile * 16 + g, r1 = r0 + 8;
        const bool v0 = r0 < n, v1 = r1 < n;
        const float2 x0 = v0 ? __ldg(reinterpret_cast<const float2 *>(feat + r0 * 8 + 2 * t)) : make_float2(0.f, 0.f);
        const float2 x1 = v1 ? __ldg(reinterpret_cast<const float2 *>(feat + r1 * 8 + 2 * t)) : make_float2(0.f, 0.f);
        const uint32_t a0 = pack_bf16(x0.x, x0.y), a1 = pack_bf16(x1.x, x1.y);

        // forward; h1/h2 hold the BF16 activations in the A-operand order, which
        // is also the C layout: [nt >> 1][2 (nt & 1) + half], half 0 = row g, 1 = row g+8
        uint32_t h1[2][4], h2[2][4];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            const uint2 b = ld_frag(pack + kPackW1 + (nt * 32 + lane) * 2);
            mma_bf16(c, a0, a1, one, one, b.x, b.y);
            h1[nt >> 1][2 * (nt & 1)] = pack_bf16(leaky(c[0]), leaky(c[1]));
            h1[nt >> 1][2 * (nt & 1) + 1] = pack_bf16(leaky(c[2]), leaky(c[3]));
        }
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            float c[4] = {b2[8 * nt + 2 * t], b2[8 * nt + 2 * t + 1], b2[8 * nt + 2 * t], b2[8 * nt + 2 * t + 1]};
#pragma unroll
            for (int ks = 0; ks < 2; ks++) {
                const uint2 b = ld_frag(pack + kPackW2 + ((ks * 4 + nt) * 32 + lane) * 2);
                mma_bf16(c, h1[ks][0], h1[ks][1], h1[ks][2], h1[ks][3], b.x, b.y);
            }
            h2[nt >> 1][2 * (nt & 1)] = pack_bf16(leaky(c[0]), leaky(c[1]));
            h2[nt >> 1][2 * (nt & 1) + 1] = pack_bf16(leaky(c[2]), leaky(c[3]));
        }
        float c3[4] = {b3, b3, b3, b3};
#pragma unroll
        for (int ks = 0; ks < 2; ks++) {
            const uint2 b = ld_frag(pack + kPackW3 + (ks * 32 + lane) * 2);
            mma_bf16(c3, h2[ks][0], h2[ks][1], h2[ks][2], h2[ks][3], b.x, b.y);
        }
        const float zq[2] = {__shfl_sync(0xffffffffu, c3[0], lane & ~3), __shfl_sync(0xffffffffu, c3[2], lane & ~3)};

        // dL/dz of rows g and g+8 (every lane of the quad computes both)
        float d3[2];
#pragma unroll
        for (int q = 0; q < 2; q++) {
            const bool v = q ? v1 : v0;
            const long long row = q ? r1 : r0;
            const float sg = 1.f / (1.f + expf(-zq[q]));
            const float eps = eps_min + span * sg;
            float slope = 0.f, Jv = 0.f;
            if (v) Jv = esj_interp(esj + row * n_eps, grid_s, n_eps, eps, slope);
            d3[q] = v ? -inv_n * slope * span * sg * (1.f - sg) : 0.f;
            if (v && t == 0) loss -= inv_n * Jv;
        }

        // layer 3 and delta2
        uint32_t d2[2][4];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            const uint32_t hg = h2[nt >> 1][2 * (nt & 1)], hg8 = h2[nt >> 1][2 * (nt & 1) + 1];
            float e[4];
#pragma unroll
            for (int c = 0; c < 2; c++) {
                const float a = bf_el(hg, c), b = bf_el(hg8, c);
                gW3[nt][c] += d3[0] * a + d3[1] * b;
                e[c] = d3[0] * w3[nt][c] * leaky_slope(a);
                e[2 + c] = d3[1] * w3[nt][c] * leaky_slope(b);
                gb2[nt][c] += e[c] + e[2 + c];
            }
            d2[nt >> 1][2 * (nt & 1)] = pack_bf16(e[0], e[1]);
            d2[nt >> 1][2 * (nt & 1) + 1] = pack_bf16(e[2], e[3]);
        }
        if (t == 0) gb3 += d3[0] + d3[1];

        // dW2 += H1^T delta2  (M = i, N = j, K = the 16 rows)
        uint32_t d2T[4][2];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            d2T[nt][0] = transpose8x8(d2[nt >> 1][2 * (nt & 1)]);
            d2T[nt][1] = transpose8x8(d2[nt >> 1][2 * (nt & 1) + 1]);
        }
#pragma unroll
        for (int mi = 0; mi < 2; mi++) {
            const uint32_t A0 = transpose8x8(h1[mi][0]), A1 = transpose8x8(h1[mi][2]);
            const uint32_t A2 = transpose8x8(h1[mi][1]), A3 = transpose8x8(h1[mi][3]);
#pragma unroll
            for (int nt = 0; nt < 4; nt++) mma_bf16(gW2[mi][nt], A0, A1, A2, A3, d2T[nt][0], d2T[nt][1]);
        }

        // delta1 = (delta2 W2^T) * act'(pre1)
        uint32_t d1[4][2];
#pragma unroll
        for (int nt = 0; nt < 4; nt++) {
            float c[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int ks = 0; ks < 2; ks++) {
                const uint2 b = ld_frag(pack + kPackW2T + ((ks * 4 + nt) * 32 + lane) * 2);
                mma_bf16(c, d2[ks][0], d2[ks][1], d2[ks][2], d2[ks][3], b.x, b.y);
            }
            const uint32_t hg = h1[nt >> 1][2 * (nt & 1)], hg8 = h1[nt >> 1][2 * (nt & 1) + 1];
            const float e0 = c[0] * leaky_slope(bf16_lo(hg)), e1 = c[1] * leaky_slope(bf16_hi(hg));
            const float e2 = c[2] * leaky_slope(bf16_lo(hg8)), e3 = c[3] * leaky_slope(bf16_hi(hg8));
            gb1[nt][0] += e0 + e2;
            gb1[nt][1] += e1 + e3;
            d1[nt][0] = pack_bf16(e0, e1);
            d1[nt][1] = pack_bf16(e2, e3);
        }

        // dW1 += X^T delta1  (M = feature, rows 0-7 kept; N = i; K = the 16 rows)
        const uint32_t X0 = transpose8x8(a0), X1 = transpose8x8(a1);
#pragma unroll
        for (int nt = 0; nt < 4; nt++)
            mma_bf16(gW1[nt], X0, 0u, X1, 0u, transpose8x8(d1[nt][0]), transpose8x8(d1[nt][1]));
    }

    // warp sums of the per-row accumulators (over g: lanes of equal t)
#pragma unroll
    for (int nt = 0; nt < 4; nt++)
#pragma unroll
        for (int c = 0; c < 2; c++)
#pragma unroll
            for (int o = 4; o < 32; o <<= 1) {
                gb1[nt][c] += __shfl_xor_sync(0xffffffffu, gb1[nt][c], o);
                gb2[nt][c] += __shfl_xor_sync(0xffffffffu, gb2[nt][c], o);
                gW3[nt][c] += __shfl_xor_sync(0xffffffffu, gW3[nt][c], o);
            }
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        gb3 += __shfl_xor_sync(0xffffffffu, gb3, o);
        loss += __shfl_xor_sync(0xffffffffu, loss, o);
    }
    float *R = red[warp];
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
        const int i = 8 * nt + 2 * t;
        R[kMlpW1 + g * 32 + i] = gW1[nt][0];
        R[kMlpW1 + g * 32 + i + 1] = gW1[nt][1];
#pragma unroll
        for (int mi = 0; mi < 2; mi++) {
            const int a = 16 * mi + g;
            R[kMlpW2 + a * 32 + i] = gW2[mi][nt][0];
            R[kMlpW2 + a * 32 + i + 1] = gW2[mi][nt][1];
            R[kMlpW2 + (a + 8) * 32 + i] = gW2[mi][nt][2];
            R[kMlpW2 + (a + 8) * 32 + i + 1] = gW2[mi][nt][3];
        }
        if (g == 0) {
            R[kMlpB1 + i] = gb1[nt][0];
            R[kMlpB1 + i + 1] = gb1[nt][1];
            R[kMlpB2 + i] = gb2[nt][0];
            R[kMlpB2 + i + 1] = gb2[nt][1];
            R[kMlpW3 + i] = gW3[nt][0];
            R[kMlpW3 + i + 1] = gW3[nt][1];
        }
    }
    if (lane == 0) {
        R[kMlpB3] = gb3;
        R[kMlpParams] = loss;
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kGradSlots; k += blockDim.x)
        partial[(long long)blockIdx.x * kGradSlots + k] = ((red[0][k] + red[1][k]) + red[2][k]) + red[3][k];
}

__global__ void k_mlp_reduce(const float *__restrict__ partial, int nblocks, float *__restrict__ grad,
                             float *__restrict__ loss) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kGradSlots) return;
    float s = 0.f;
    for (int b = 0; b < nblocks; b++) s += partial[(long long)b * kGradSlots + k];
    if (k < kMlpParams) grad[k] = s;
    else loss[0] = s;
}

static int grad_blocks(long long n) {
    const long long tiles = (n + 15) / 16;
    long long b = (tiles + kGradWarps - 1) / kGradWarps;
    if (b > kGradMaxBlocks) b = kGradMaxBlocks;
    return b < 1 ? 1 : (int)b;
}

size_t mlp_grad_scratch(long long n) { return (size_t)grad_blocks(n) * kGradSlots; }

void launch_mlp_grad(const float *params, const uint32_t *pack, const float *features, const float *esj, long long n,
                     int n_eps, const float *eps_grid_dev, float eps_min, float eps_max, float *partial, float *grad,
                     float *loss, cudaStream_t st) {
    const int nb = grad_blocks(n);
    k_mlp_grad<<<nb, 128, 0, st>>>(params, pack, features, esj, n, n_eps, eps_grid_dev, eps_min, eps_max, partial);
    k_mlp_reduce<<<(kGradSlots + 255) / 256, 256, 0, st>>>(partial, nb, grad, loss);
}

// Adam (Kingma & Ba, arXiv:1412.6980, Algorithm 1), beta1 0.9, beta2 0.999, eps 1e-8.
__global__ void k_adam(float *__restrict__ p, float *__restrict__ m, float *__restrict__ v,
                       const float *__restrict__ grad, float lr, float c1, float c2) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= kMlpParams) return;
    const float gk = grad[k];
    const float mk = 0.9f * m[k] + 0.1f * gk;
    const float vk = 0.999f * v[k] + 0.001f * gk * gk;
    m[k] = mk;
    v[k] = vk;
    p[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + 1e-8f);
}

void launch_adam(float *params, float *m, float *v, const float *grad, int step, float lr, cudaStream_t st) {
    const float c1 = 1.f - powf(0.9f, (float)step), c2 = 1.f - powf(0.999f, (float)step);
    k_adam<<<(kMlpParams + 255) / 256, 256, 0, st>>>(params, m, v, grad, lr, c1, c2);
}

}  // namespace glac

// ---------------------------------------------------------------------------
// C ABI of the trainer
// ---------------------------------------------------------------------------
using namespace glac;

struct glac_mlp {
    int device = 0;
    cudaStream_t stream = nullptr;
    float *params = nullptr, *m = nullptr, *v = nullptr, *grad = nullptr, *loss = nullptr, *grid = nullptr;
    float *partial = nullptr;
    size_t partial_cap = 0;
    uint32_t *pack = nullptr;
    int *err_dev = nullptr;  // wait-timeout flag of the tcgen05 kernel
    int forward_mode = 0;    // 0: the sampler's warp-level routine, 1: tcgen05 tiles
    unsigned long long tc_wait_ns = 1000000000ull;  // completion-wait limit of the tcgen05 kernel (1 s)
    int tc_issue = 1;        // 0: test mode, the tcgen05 kernel issues no MMA (its waits run out)
    bool tc_broken = false;  // a tcgen05 pass timed out without draining: tensor-core path refused
    int step = 0;
    std::string err;
};

namespace {

struct MlpError : std::exception {
    std::string msg;
    explicit MlpError(std::string s) : msg(std::move(s)) {}
    const char *what() const noexcept override { return msg.c_str(); }
};
void mck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw MlpError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename F> glac_status mlp_guarded(glac_mlp *M, F &&f) {
    if (!M) return GLAC_ERR_ARG;
    try {
        mck(cudaSetDevice(M->device), "cudaSetDevice");
        return f();
    } catch (const MlpError &e) {
        M->err = e.msg;
        return GLAC_ERR_CUDA;
    } catch (const std::exception &e) {
        M->err = e.what();
        return GLAC_ERR_CUDA;
    }
}

glac_status check_grid(glac_mlp *M, int n_eps, const double *grid) {
    if (n_eps < 2 || n_eps > 64 || !grid) {
        M->err = "eps grid needs 2..64 points";
        return GLAC_ERR_ARG;
    }
    for (int k = 0; k + 1 < n_eps; k++)
        if (!(grid[k] > 0.0 && grid[k + 1] > grid[k] && grid[k + 1] <= 1.0)) {
            M->err = "eps grid must increase inside (0, 1]";
            return GLAC_ERR_ARG;
        }
    return GLAC_OK;
}

void upload_grid(glac_mlp *M, int n_eps, const double *grid) {
    float g32[64];
    for (int k = 0; k < n_eps; k++) g32[k] = (float)grid[k];
    mck(cudaMemcpyAsync(M->grid, g32, n_eps * sizeof(float), cudaMemcpyHostToDevice, M->stream), "grid upload");
}

void ensure_partial(glac_mlp *M, long long n) {
    const size_t need = mlp_grad_scratch(n);
    if (need > M->partial_cap) {
        if (M->partial) mck(cudaFree(M->partial), "cudaFree");
        M->partial = nullptr;
        mck(cudaMalloc(&M->partial, need * sizeof(float)), "partial alloc");
        M->partial_cap = need;
    }
}

}  // namespace

extern "C" {

glac_status glac_mlp_create(int device, glac_mlp **out) {
    if (!out) return GLAC_ERR_ARG;
    *out = nullptr;
    glac_mlp *M = new glac_mlp;
    M->device = device;
    glac_status s = mlp_guarded(M, [&] {
        mck(cudaStreamCreateWithFlags(&M->stream, cudaStreamNonBlocking), "stream");
        mck(cudaMalloc(&M->params, kMlpParams * sizeof(float)), "alloc");
        mck(cudaMalloc(&M->m, kMlpParams * sizeof(float)), "alloc");
        mck(cudaMalloc(&M->v, kMlpParams * sizeof(float)), "alloc");
        mck(cudaMalloc(&M->grad, kMlpParams * sizeof(float)), "alloc");
        mck(cudaMalloc(&M->loss, sizeof(float)), "alloc");
        mck(cudaMalloc(&M->grid, 64 * sizeof(float)), "alloc");
        mck(cudaMalloc(&M->pack, kPackWords * sizeof(uint32_t)), "alloc");
        mck(cudaMemsetAsync(M->params, 0, kMlpParams * sizeof(float), M->stream), "memset");
        mck(cudaMemsetAsync(M->m, 0, kMlpParams * sizeof(float), M->stream), "memset");
        mck(cudaMemsetAsync(M->v, 0, kMlpParams * sizeof(float), M->stream), "memset");
        launch_mlp_pack(M->params, M->pack, M->stream);
        mck(cudaGetLastError(), "pack");
        mck(cudaStreamSynchronize(M->stream), "sync");
        return GLAC_OK;
    });
    if (s != GLAC_OK) {
        glac_mlp_destroy(M);
        return s;
    }
    *out = M;
    return GLAC_OK;
}

void glac_mlp_destroy(glac_mlp *M) {
    if (!M) return;
    cudaSetDevice(M->device);
    if (M->stream) cudaStreamSynchronize(M->stream);
    for (void *p : {(void *)M->params, (void *)M->m, (void *)M->v, (void *)M->grad, (void *)M->loss, (void *)M->grid,
                    (void *)M->partial, (void *)M->pack, (void *)M->err_dev})
        if (p) cudaFree(p);
    if (M->stream) cudaStreamDestroy(M->stream);
    delete M;
}

const char *glac_mlp_last_error(const glac_mlp *M) { return M ? M->err.c_str() : "null trainer"; }

glac_status glac_mlp_set_params(glac_mlp *M, const float *host) {
    if (!host) return GLAC_ERR_ARG;
    return mlp_guarded(M, [&] {
        for (int k = 0; k < kMlpParams; k++)
            if (!std::isfinite(host[k])) {
                M->err = "non-finite parameter";
                return GLAC_ERR_NONFINITE;
            }
        mck(cudaMemcpyAsync(M->params, host, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, M->stream), "upload");
        mck(cudaMemsetAsync(M->m, 0, kMlpParams * sizeof(float), M->stream), "memset");
        mck(cudaMemsetAsync(M->v, 0, kMlpParams * sizeof(float), M->stream), "memset");
        M->step = 0;
        launch_mlp_pack(M->params, M->pack, M->stream);
        mck(cudaGetLastError(), "pack");
        mck(cudaStreamSynchronize(M->stream), "sync");
        return GLAC_OK;
    });
}

glac_status glac_mlp_get_params(glac_mlp *M, float *host) {
    if (!host) return GLAC_ERR_ARG;
    return mlp_guarded(M, [&] {
        mck(cudaMemcpyAsync(host, M->params, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, M->stream), "download");
        mck(cudaStreamSynchronize(M->stream), "sync");
        return GLAC_OK;
    });
}

glac_status glac_mlp_init(glac_mlp *M, uint64_t seed, double eps_min, double eps_max, double eps0) {
    if (!M) return GLAC_ERR_ARG;
    if (!(eps_min < eps0 && eps0 < eps_max)) {
        M->err = "need eps_min < eps0 < eps_max";
        return GLAC_ERR_ARG;
    }
    // He-normal hidden weights, zero hidden biases, a small output layer whose
    // bias puts the initial spread at eps0.
    std::mt19937_64 rng(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    std::vector<float> P(kMlpParams, 0.f);
    for (int k = 0; k < 256; k++) P[kMlpW1 + k] = (float)(nd(rng) * std::sqrt(2.0 / 8.0));
    for (int k = 0; k < 1024; k++) P[kMlpW2 + k] = (float)(nd(rng) * std::sqrt(2.0 / 32.0));
    for (int k = 0; k < 32; k++) P[kMlpW3 + k] = (float)(nd(rng) * 0.01);
    const double s = (eps0 - eps_min) / (eps_max - eps_min);
    P[kMlpB3] = (float)std::log(s / (1.0 - s));
    return glac_mlp_set_params(M, P.data());
}

glac_status glac_mlp_forward(glac_mlp *M, const float *dev_features, long long n, double eps_min, double eps_max,
                             float *dev_eps) {
    if (!dev_features || !dev_eps || n <= 0 || !(eps_min < eps_max)) return GLAC_ERR_ARG;
    return mlp_guarded(M, [&] {
        if (M->forward_mode == 0) {
            launch_mlp_forward(M->pack, dev_features, n, (float)eps_min, (float)eps_max, dev_eps, M->stream);
            mck(cudaGetLastError(), "forward");
            mck(cudaStreamSynchronize(M->stream), "sync");
            return GLAC_OK;
        }
        if (M->tc_broken) {
            M->err = "an earlier tensor-core pass did not drain after its wait limit; mode 1 is disabled";
            return GLAC_ERR_STATE;
        }
        if (!M->err_dev) mck(cudaMalloc(&M->err_dev, sizeof(int)), "alloc");
        mck(cudaMemsetAsync(M->err_dev, 0, sizeof(int), M->stream), "memset");
        launch_mlp_forward_tc(M->params, dev_features, n, (float)eps_min, (float)eps_max, dev_eps, M->err_dev,
                              M->tc_wait_ns, M->tc_issue, M->stream);
        mck(cudaGetLastError(), "forward (tcgen05)");
        int flag = 0;
        mck(cudaMemcpyAsync(&flag, M->err_dev, sizeof(int), cudaMemcpyDeviceToHost, M->stream), "D2H");
        mck(cudaStreamSynchronize(M->stream), "sync");
        if (flag == 2) {
            M->tc_broken = true;
            M->err = "tensor-core pass did not complete within its wait limit, nor drain after a second wait";
            return GLAC_ERR_TIMEOUT;
        }
        if (flag) {
            M->err = "tensor-core pass did not complete within its wait limit";
            return GLAC_ERR_TIMEOUT;
        }
        return GLAC_OK;
    });
}

glac_status glac_mlp_set_forward_mode(glac_mlp *M, int mode) {
    if (!M || (mode != 0 && mode != 1)) return GLAC_ERR_ARG;
    M->forward_mode = mode;
    return GLAC_OK;
}

glac_status glac_mlp_test_tc_wait(glac_mlp *M, unsigned long long wait_ns, int issue_mma) {
    if (!M || wait_ns == 0 || wait_ns > 10000000000ull || (issue_mma != 0 && issue_mma != 1)) return GLAC_ERR_ARG;
    M->tc_wait_ns = wait_ns;
    M->tc_issue = issue_mma;
    return GLAC_OK;
}

glac_status glac_mlp_loss_grad(glac_mlp *M, const float *dev_features, const float *dev_esj, long long n, int n_eps,
                               const double *eps_grid, double *loss, float *host_grad) {
    if (!dev_features || !dev_esj || n <= 0) return GLAC_ERR_ARG;
    return mlp_guarded(M, [&] {
        glac_status s = check_grid(M, n_eps, eps_grid);
        if (s != GLAC_OK) return s;
        upload_grid(M, n_eps, eps_grid);
        ensure_partial(M, n);
        launch_mlp_grad(M->params, M->pack, dev_features, dev_esj, n, n_eps, M->grid, (float)eps_grid[0],
                        (float)eps_grid[n_eps - 1], M->partial, M->grad, M->loss, M->stream);
        mck(cudaGetLastError(), "grad");
        float l = 0.f;
        mck(cudaMemcpyAsync(&l, M->loss, sizeof(float), cudaMemcpyDeviceToHost, M->stream), "loss");
        if (host_grad)
            mck(cudaMemcpyAsync(host_grad, M->grad, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, M->stream),
                "grad download");
        mck(cudaStreamSynchronize(M->stream), "sync");
        if (loss) *loss = l;
        return GLAC_OK;
    });
}

glac_status glac_mlp_train(glac_mlp *M, const float *dev_features, const float *dev_esj, long long n, int n_eps,
                           const double *eps_grid, int steps, long long batch, double lr, double *host_losses) {
    if (!dev_features || !dev_esj || n <= 0 || steps < 0 || batch <= 0 || !(lr > 0.0)) return GLAC_ERR_ARG;
    return mlp_guarded(M, [&] {
        glac_status s = check_grid(M, n_eps, eps_grid);
        if (s != GLAC_OK) return s;
        if (batch > n) batch = n;
        upload_grid(M, n_eps, eps_grid);
        ensure_partial(M, batch);
        std::vector<float> losses(steps > 0 ? steps : 1);
        float *loss_dev = nullptr;
        mck(cudaMalloc(&loss_dev, losses.size() * sizeof(float)), "loss alloc");
        try {
            const long long nb = n / batch;  // whole batches, cycled in order
            for (int it = 0; it < steps; it++) {
                const long long off = (it % nb) * batch;
                launch_mlp_grad(M->params, M->pack, dev_features + off * 8, dev_esj + off * n_eps, batch, n_eps,
                                M->grid, (float)eps_grid[0], (float)eps_grid[n_eps - 1], M->partial, M->grad,
                                loss_dev + it, M->stream);
                launch_adam(M->params, M->m, M->v, M->grad, ++M->step, (float)lr, M->stream);
                launch_mlp_pack(M->params, M->pack, M->stream);
            }
            mck(cudaGetLastError(), "train");
            if (steps > 0)
                mck(cudaMemcpyAsync(losses.data(), loss_dev, steps * sizeof(float), cudaMemcpyDeviceToHost, M->stream),
                    "losses");
            mck(cudaStreamSynchronize(M->stream), "sync");
        } catch (...) {
            cudaFree(loss_dev);
            throw;
        }
        cudaFree(loss_dev);
        if (host_losses)
            for (int it = 0; it < steps; it++) host_losses[it] = losses[it];
        return GLAC_OK;
    });
}

}  // extern "C"
