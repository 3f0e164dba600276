// Learned Metropolis proposal spread (no counterpart in the reference).
//
// A small MLP maps eight gauge-invariant features of a link's staple A to the
// spread eps of the reference's proposal X = R S T (su3matrixgenerator.h:170-243).
// A is unchanged by the link's own update, so q(U -> U') = q(U' -> U) with the
// same eps(A): the proposal stays symmetric and the accept step of
// GLAC/system.cpp:333-361 keeps the chain exact.
//
// Features of A (W = A A^+, s^2 = Tr W / 3, k = beta s / 3; all invariant under
// A -> Omega(n+mu) A Omega(n)^+ because det Omega = 1):
//   f0 = ln k            f1 = Tr W^2 / (3 s^4) - 1     f2 = Tr W^3 / (3 s^6) - 1
//   f3 = Re det A / s^3  f4 = Im det A / s^3           f5 = |det A| / s^3
//   f6 = 1 / k           f7 = beta / 6 - 1
// Network 8 -> 32 -> 32 -> 1, leaky ReLU (slope 1/16), eps = eps_min +
// (eps_max - eps_min) sigmoid(z).  BF16 operands, FP32 accumulation, on the
// tensor cores through warp-level mma.m16n8k16: one warp evaluates its 32 links
// (two 16-row tiles) from registers, so inference fuses into the Metropolis
// kernel without a round trip through memory.  The first layer's bias rides in
// the padded K dimension (constant feature 1 at column 8).
#pragma once

#include <cuda_bf16.h>

#include "su3.cuh"

namespace glac {

// FP32 master parameters, flat.
constexpr int kMlpW1 = 0;     // [8][32]  W1[f][i]
constexpr int kMlpB1 = 256;   // [32]
constexpr int kMlpW2 = 288;   // [32][32] W2[i][j]
constexpr int kMlpB2 = 1312;  // [32]
constexpr int kMlpW3 = 1344;  // [32]
constexpr int kMlpB3 = 1376;  // [1]
constexpr int kMlpParams = 1377;

// Packed B-operand fragments (32-bit words, two BF16 each), in the register
// order of mma.m16n8k16 for lane l (g = l / 4, t = l % 4):
//   word r of [.., l]: (B[2t + 8r][g], B[2t + 8r + 1][g]) of the 16 x 8 tile.
constexpr int kPackW1 = 0;      // [nt 4][lane 32][2]        B = [W1; b1; 0] (16 x 32)
constexpr int kPackW2 = 256;    // [ks 2][nt 4][lane 32][2]  B = W2 (32 x 32)
constexpr int kPackW3 = 768;    // [ks 2][lane 32][2]        B = [W3, 0...] (32 x 8)
constexpr int kPackW2T = 896;   // [ks 2][nt 4][lane 32][2]  B = W2^T (backward)
constexpr int kPackB2 = 1408;   // 32 floats
constexpr int kPackB3 = 1440;   // 1 float
constexpr int kPackWords = 1472;
constexpr float kLeak = 0.0625f;

struct Proposal {
    const uint32_t *net = nullptr;  // packed fragments; null = the fixed spread
    float eps_min = 0.f, eps_max = 0.f;
    // SU(2) factors of X = R S T: x0 = sign(u0) sqrt(1 - eps^2) as in the reference
    // (true), or x0 = +sqrt(1 - eps^2), every factor near the identity (false)
    bool flips = true;
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}
__device__ __forceinline__ float bf16_lo(uint32_t w) { return __uint_as_float(w << 16); }
__device__ __forceinline__ float bf16_hi(uint32_t w) { return __uint_as_float(w & 0xFFFF0000u); }
__device__ __forceinline__ float round_bf16(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float leaky(float x) { return x > 0.f ? x : kLeak * x; }
__device__ __forceinline__ float leaky_slope(float x) { return x > 0.f ? 1.f : kLeak; }

// D = A B + C, A 16x16 row-major BF16, B 16x8 column-major BF16, C/D FP32.
__device__ __forceinline__ void mma_bf16(float c[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                         uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Transpose of an 8x8 BF16 matrix held one row-pair per lane (lane l: row l/4,
// columns 2(l%4), 2(l%4)+1) into the same layout.
__device__ __forceinline__ uint32_t transpose8x8(uint32_t a) {
    uint32_t d;
    asm volatile("movmatrix.sync.aligned.m8n8.trans.b16 %0, %1;\n" : "=r"(d) : "r"(a));
    return d;
}

__device__ __forceinline__ uint2 ld_frag(const uint32_t *__restrict__ p) {
    return __ldg(reinterpret_cast<const uint2 *>(p));
}

// The eight features of a staple (in T, returned as float).  W = A A^+ from
// its upper triangle; Tr W^3 from Newton's identities with det W = |det A|^2:
// p3 = e1 p2 - e2 p1 + 3 e3, e1 = p1, e2 = (p1^2 - p2) / 2.
template <typename T> __device__ __forceinline__ void staple_features(const M3<T> &A, float beta, float f[8]) {
    T d[3];
#pragma unroll
    for (int i = 0; i < 3; i++)
        d[i] = A(i, 0).re * A(i, 0).re + A(i, 0).im * A(i, 0).im + A(i, 1).re * A(i, 1).re +
               A(i, 1).im * A(i, 1).im + A(i, 2).re * A(i, 2).re + A(i, 2).im * A(i, 2).im;
    T off = T(0);  // sum over i < j of |W_ij|^2
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = i + 1; j < 3; j++) {
            Cx<T> w = cx(T(0), T(0));
            w = cmac_bc(w, A(i, 0), A(j, 0));
            w = cmac_bc(w, A(i, 1), A(j, 1));
            w = cmac_bc(w, A(i, 2), A(j, 2));
            off += w.re * w.re + w.im * w.im;
        }
    const T t1 = d[0] + d[1] + d[2];
    const T t2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + T(2) * off;
    // det A by the first row
    const Cx<T> m0 = A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1);
    const Cx<T> m1 = A(1, 0) * A(2, 2) - A(1, 2) * A(2, 0);
    const Cx<T> m2 = A(1, 0) * A(2, 1) - A(1, 1) * A(2, 0);
    const Cx<T> det = A(0, 0) * m0 - A(0, 1) * m1 + A(0, 2) * m2;
    const T det2 = det.re * det.re + det.im * det.im;
    const T t3 = t1 * t2 - T(0.5) * (t1 * t1 - t2) * t1 + T(3) * det2;
    T s2 = t1 / T(3);
    s2 = s2 > T(1e-30) ? s2 : T(1e-30);
    const T s = sqrt(s2), s3 = s2 * s;
    const T k = T(beta) * s / T(3);
    f[0] = (float)log(k);
    f[1] = (float)(t2 / (T(3) * s2 * s2) - T(1));
    f[2] = (float)(t3 / (T(3) * s2 * s2 * s2) - T(1));
    f[3] = (float)(det.re / s3);
    f[4] = (float)(det.im / s3);
    f[5] = (float)(sqrt(det2) / s3);
    f[6] = (float)(T(1) / k);
    f[7] = beta / 6.f - 1.f;
}

// Forward pass of one 16-row tile whose layer-1 A operand is (a0, a1) (rows g
// and g+8, feature columns 2t, 2t+1; the bias column is added here).  Returns z
// for row g in z[0] and row g+8 in z[1] (valid in the lanes with t = 0).
__device__ __forceinline__ void mlp_tile_forward(uint32_t a0, uint32_t a1, const uint32_t *__restrict__ net,
                                                 float &z_g, float &z_g8) {
    const int lane = threadIdx.x & 31, t = lane & 3;
    const uint32_t one = t == 0 ? pack_bf16(1.f, 0.f) : 0u;
    uint32_t h1[2][4];
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
        float c[4] = {0.f, 0.f, 0.f, 0.f};
        const uint2 b = ld_frag(net + kPackW1 + (nt * 32 + lane) * 2);
        mma_bf16(c, a0, a1, one, one, b.x, b.y);
        h1[nt >> 1][2 * (nt & 1)] = pack_bf16(leaky(c[0]), leaky(c[1]));
        h1[nt >> 1][2 * (nt & 1) + 1] = pack_bf16(leaky(c[2]), leaky(c[3]));
    }
    const float *b2 = reinterpret_cast<const float *>(net + kPackB2);
    uint32_t h2[2][4];
#pragma unroll
    for (int nt = 0; nt < 4; nt++) {
        const float2 bb = __ldg(reinterpret_cast<const float2 *>(b2 + 8 * nt + 2 * t));
        float c[4] = {bb.x, bb.y, bb.x, bb.y};
#pragma unroll
        for (int ks = 0; ks < 2; ks++) {
            const uint2 b = ld_frag(net + kPackW2 + ((ks * 4 + nt) * 32 + lane) * 2);
            mma_bf16(c, h1[ks][0], h1[ks][1], h1[ks][2], h1[ks][3], b.x, b.y);
        }
        h2[nt >> 1][2 * (nt & 1)] = pack_bf16(leaky(c[0]), leaky(c[1]));
        h2[nt >> 1][2 * (nt & 1) + 1] = pack_bf16(leaky(c[2]), leaky(c[3]));
    }
    const float b3 = __ldg(reinterpret_cast<const float *>(net + kPackB3));
    float c[4] = {b3, b3, b3, b3};
#pragma unroll
    for (int ks = 0; ks < 2; ks++) {
        const uint2 b = ld_frag(net + kPackW3 + (ks * 32 + lane) * 2);
        mma_bf16(c, h2[ks][0], h2[ks][1], h2[ks][2], h2[ks][3], b.x, b.y);
    }
    z_g = c[0];
    z_g8 = c[2];
}

__device__ __forceinline__ float spread_of(float z, float eps_min, float eps_max) {
    return eps_min + (eps_max - eps_min) / (1.f + expf(-z));
}

// Proposal spread of this lane's link from its features.  All 32 lanes of the
// warp call it (lanes without a link pass zeros); smem holds 128 words per warp.
__device__ __forceinline__ float mlp_spread_warp(const float f[8], const Proposal &P, uint32_t *smem) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    uint4 w;
    w.x = pack_bf16(f[0], f[1]);
    w.y = pack_bf16(f[2], f[3]);
    w.z = pack_bf16(f[4], f[5]);
    w.w = pack_bf16(f[6], f[7]);
    __syncwarp();
    reinterpret_cast<uint4 *>(smem)[lane] = w;
    __syncwarp();
    float z[2][2];
#pragma unroll
    for (int m = 0; m < 2; m++) {
        const uint32_t a0 = smem[(16 * m + g) * 4 + t], a1 = smem[(16 * m + g + 8) * 4 + t];
        mlp_tile_forward(a0, a1, P.net, z[m][0], z[m][1]);
    }
    // row r of tile m sits in lane 4 (r % 8), slot r / 8
    const int r = lane & 15, src = 4 * (r & 7);
    const float v00 = __shfl_sync(0xffffffffu, z[0][0], src), v01 = __shfl_sync(0xffffffffu, z[0][1], src);
    const float v10 = __shfl_sync(0xffffffffu, z[1][0], src), v11 = __shfl_sync(0xffffffffu, z[1][1], src);
    const float zz = lane < 16 ? (r < 8 ? v00 : v01) : (r < 8 ? v10 : v11);
    return spread_of(zz, P.eps_min, P.eps_max);
}

// Host-side launchers (learned.cu).
void launch_mlp_pack(const float *params, uint32_t *pack, cudaStream_t st);
void launch_mlp_forward(const uint32_t *pack, const float *features, long long n, float eps_min, float eps_max,
                        float *eps_out, cudaStream_t st);
// The same inference on tcgen05 tensor cores from the FP32 parameters (128-row tiles); *err set on a wait timeout.
void launch_mlp_forward_tc(const float *params, const float *features, long long n, float eps_min, float eps_max,
                           float *eps_out, int *err, cudaStream_t st);
// Gradient of L = -(1/n) sum_i J_i(eps_i) (J_i piecewise linear on eps_grid)
// into grad[kMlpParams] and loss[0]; partial: scratch of mlp_grad_scratch(n) floats.
size_t mlp_grad_scratch(long long n);
void launch_mlp_grad(const float *params, const uint32_t *pack, const float *features, const float *esj, long long n,
                     int n_eps, const float *eps_grid_dev, float eps_min, float eps_max, float *partial, float *grad,
                     float *loss, cudaStream_t st);
void launch_adam(float *params, float *m, float *v, const float *grad, int step, float lr, cudaStream_t st);

}  // namespace glac
