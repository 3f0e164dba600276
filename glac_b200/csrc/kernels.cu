// Hot-path kernels for sm_100a: fused flow stage, checkerboard Metropolis,
// fused clover observables with deterministic FP64 reductions, plus field
// initialisation, reunitarisation and layout conversion.
#include "kernels.cuh"
#include "learned.cuh"

#include <algorithm>
#include <stdexcept>

namespace glac {

// ---------------------------------------------------------------------------
// Flow stage (GLAC/flow/flow.cpp:43-73 with getActionDerivative,
// GLAC/actions/wilsongaugeaction.cpp:55-86), one fused pass per RK3 stage:
//   Z = P_ah(U_mu(n) A_mu(n)),  M = alpha Z + beta Zprev,  U' = exp(M) U.
//   stage 0: M = (eps/4) Z0, stores Z0
//   stage 1: M = (8/9 eps) Z1 - (17/36 eps) Z0, stores M
//   stage 2: M = (3/4 eps) Z2 - M_prev
// Reads field `in`, writes `out` (all four Z_mu come from the same field).
// 1-D grid, the 8 (mu, parity) planes interleaved fastest: the blocks that run
// together cover one region of the lattice for all planes, so the neighbour
// links they share are read from HBM once and then hit in L2.
// ---------------------------------------------------------------------------
// Site-block shapes (blocks of 128 threads):
//   shape 0: a block = 128 consecutive sites of one plane, blocks of the 8
//            planes interleaved;
//   shape 1: a block = the same 16 sites in all 8 planes (half-warp per plane),
//            so the neighbour links shared by the 8 link directions of a site
//            are re-read from L1.
//   shape 3: FP32, a thread per site doing its four links in turn, the upper
//            staple product of each plane shared between its two links
//            (flow_stage_site_body below);
//   shape 2: as shape 0, with the 128-site chunks taken in 4 x 4 tiles of
//            (z, t) (tiled_chunk), so that a link's neighbours in t are
//            mostly read while it is still in L2.  An FP64 variant: its
//            144-byte links outgrow L2 in the shape-0 order, and the tiles made
//            the stage 3-6 % faster at 32^3 x 64 and 48^3 x 96 on B200; FP32,
//            whose DRAM traffic is already the algorithmic bytes, ran 4-15 %
//            slower with it.
// Chunk j of the tiled order: j = k + K (zi + 4 (ti + 4 (zT + (Nz/4) tT))) covers
// the k-th of the K chunks of the (z, t) = (4 zT + zi, 4 tT + ti) pair.  The
// identity where a (z, t) pair is not a whole number of chunks or Nz, Nt are
// not multiples of 4.  A bijection of [0, K Nz Nt) either way.
__device__ __forceinline__ int tiled_chunk(const Geom &g, int j) {
    const int hs = g.Nxh * g.N[1];  // sites of one (z, t) pair in a parity plane
    const int K = hs >> 7;
    if (K == 0 || (K << 7) != hs || (g.N[2] & 3) || (g.N[3] & 3)) return j;
    const int k = j % K;
    int r = j / K;
    const int zi = r & 3, ti = (r >> 2) & 3;
    r >>= 4;
    const int nzT = g.N[2] >> 2;
    const int z = (r % nzT) * 4 + zi, t = (r / nzT) * 4 + ti;
    return k + K * (z + g.N[2] * t);
}

template <typename T, int KIND, int STAGE, int SHAPE>
__device__ __forceinline__ void flow_stage_body(const Geom &g, const LinkField<T> &in, const LinkField<T> &out,
                                                const ForceField<T> &zf, T alpha, T beta, int bx) {
    const int plane = SHAPE == 1 ? int(threadIdx.x >> 4) : (bx & 7);
    const int s = SHAPE == 1   ? int(bx * 16 + (threadIdx.x & 15))
                  : SHAPE == 2 ? int(tiled_chunk(g, bx >> 3) * 128 + threadIdx.x)
                               : int((bx >> 3) * 128 + threadIdx.x);
    if (s >= g.Vh) return;
    const int mu = plane >> 1, p = plane & 1;
    const Site n = site_from_ps(g, p, s);
    M3<T> A = staple<T, false, true>(in, g, n, p, mu);
    const M3<T> U = in.load(mu, p, s);
    const AH8<T> Z = project_ah(mul(U, A));
    AH8<T> M;
    if (STAGE == 0) {
        M = ah_scale(alpha, Z);
        zf.store(mu, p, s, Z);
    } else {
        const AH8<T> W = zf.load(mu, p, s);
        M = ah_axpby(alpha, Z, beta, W);
        if (STAGE == 1) zf.store(mu, p, s, M);
    }
    if (KIND == EXP_MORNINGSTAR) {
        // U' = U + (exp(M) - 1) U: the small product first, one rounding at |U|
        out.store(mu, p, s, mul_plus_right(expm_morningstar<T, true>(M), U));
    } else {
        out.store(mu, p, s, mul(expm<T>(KIND, M), U));
    }
}

// Shape 3 (FP32): one thread per site, its four links in turn.  The upper
// staple product of a plane, T_munu = U_nu(n+mu) U_mu(n+nu)^+ (mu < nu), serves
// both links of the plane at the site: link mu adds T U_nu(n)^+ and keeps T in
// the thread's shared-memory slot, link nu later adds T^+ U_mu(n)^+ (the same
// three links) without loading U_nu(n+mu) and U_mu(n+nu) again.  46 SU(3)
// products per site instead of 52 and 64 link loads instead of 76.  Four slots
// per thread suffice in the order mu = 0..3 (T_01 -> 0, T_02 -> 1, T_03 -> 2,
// then T_12 -> 0 and T_13 -> 3 once T_01 is used, T_23 -> 1 once T_02 is).
// Each thread touches only its own slots, laid out slot-major with the thread
// index fastest (no bank conflicts, no barrier).
__host__ __device__ constexpr int tslot(int a, int b) {
    return a == 0 ? b - 1 : (a == 1 ? (b == 2 ? 0 : 3) : 1);
}
constexpr int kSiteBlock = 128;

// MEAS (stage 0 only): also the measurement's clover parts of the planes each
// link direction takes, as flow_stage0_meas_body does (defined further down).
__device__ __forceinline__ bool meas_takes(int mu, int nu);
__host__ __device__ constexpr int plane_of(int a, int b);
template <typename T> __device__ __forceinline__ AH8<T> proj_ah8(const M3<T> &C);
template <typename T> __device__ __forceinline__ AH8<T> ah_neg_if(const AH8<T> &F, bool neg);

template <typename T, int KIND, int STAGE, bool MEAS = false>
__device__ __forceinline__ void flow_stage_site_body(const Geom &g, const LinkField<T> &in, const LinkField<T> &out,
                                                     const ForceField<T> &zf, T alpha, T beta, int bx, T *slots,
                                                     const CloverParts<T> *cp = nullptr) {
    const int p = bx & 1;
    const int s = (bx >> 1) * kSiteBlock + threadIdx.x;
    if (s >= g.Vh) return;
    const int q = p ^ 1;
    const Site n = site_from_ps(g, p, s);
    T *my = slots + threadIdx.x;  // element e of slot k at my[(18 k + e) * kSiteBlock]
#pragma unroll 1
    for (int mu = 0; mu < 4; mu++) {
        M3<T> A;
        set_zero(A);
        T plaq = T(0);
        const int f_mu = step_offset(g, n, mu, +1);
        const int s_mu = (n.lex + f_mu) >> 1;
#pragma unroll 1
        for (int nu = 0; nu < 4; nu++) {
            if (nu == mu) continue;
            const int b_nu = step_offset(g, n, nu, -1);
            if (MEAS && meas_takes(mu, nu)) {
                // the plane this link takes for the measurement: S_up and S_low
                // separately, W = S_up - S_low, the parts P(U W) at n and P(W U) at n + mu
                M3<T> W;
                if (nu > mu) {
                    const int s_nup = (n.lex + step_offset(g, n, nu, +1)) >> 1;
                    const M3<T> t = flow_nd(in.load(nu, q, s_mu), in.load(mu, q, s_nup));
                    T *slot = my + 18 * kSiteBlock * tslot(mu, nu);
#pragma unroll
                    for (int e = 0; e < 9; e++) {
                        slot[(2 * e) * kSiteBlock] = t.e[e].re;
                        slot[(2 * e + 1) * kSiteBlock] = t.e[e].im;
                    }
                    W = flow_nd(t, in.load(nu, p, s));
                } else {
                    const T *slot = my + 18 * kSiteBlock * tslot(nu, mu);
                    M3<T> t;
#pragma unroll
                    for (int e = 0; e < 9; e++) {
                        t.e[e].re = slot[(2 * e) * kSiteBlock];
                        t.e[e].im = slot[(2 * e + 1) * kSiteBlock];
                    }
                    W = flow_dd(t, in.load(nu, p, s));
                }
                add_to(A, W);
                plaq += retr_mul(in.load(mu, p, s), W);  // ReTr(U S_up)
                asm volatile("" ::: "memory");
                {
                    const int s_num = (n.lex + b_nu) >> 1, s_diag = (n.lex + f_mu + b_nu) >> 1;
                    M3<T> t = flow_dd(in.load(nu, p, s_diag), in.load(mu, q, s_num));
                    const M3<T> S = flow_nn(t, in.load(nu, q, s_num));
                    add_to(A, S);
                    sub_from(W, S);
                }
                const bool neg = nu < mu;
                const int pl = neg ? plane_of(nu, mu) : plane_of(mu, nu);
                asm volatile("" ::: "memory");
                cp->ah.store(2 * pl, p, s, ah_neg_if(proj_ah8(mul(in.load(mu, p, s), W)), neg));
                asm volatile("" ::: "memory");
                cp->ah.store(2 * pl + 1, q, s_mu, ah_neg_if(proj_ah8(mul(W, in.load(mu, p, s))), neg));
                continue;
            }
            if (nu > mu) {
                const int s_nup = (n.lex + step_offset(g, n, nu, +1)) >> 1;
                const M3<T> t = flow_nd(in.load(nu, q, s_mu), in.load(mu, q, s_nup));
                T *slot = my + 18 * kSiteBlock * tslot(mu, nu);
#pragma unroll
                for (int e = 0; e < 9; e++) {
                    slot[(2 * e) * kSiteBlock] = t.e[e].re;
                    slot[(2 * e + 1) * kSiteBlock] = t.e[e].im;
                }
                acc_mul_nd(A, t, in.load(nu, p, s));
            } else {
                const T *slot = my + 18 * kSiteBlock * tslot(nu, mu);
                M3<T> t;
#pragma unroll
                for (int e = 0; e < 9; e++) {
                    t.e[e].re = slot[(2 * e) * kSiteBlock];
                    t.e[e].im = slot[(2 * e + 1) * kSiteBlock];
                }
                acc_mul_dd(A, t, in.load(nu, p, s));  // T_numu^+ U_nu(n)^+ = U_nu(n+mu) U_mu(n+nu)^+ U_nu(n)^+
            }
            {
                const int s_num = (n.lex + b_nu) >> 1, s_diag = (n.lex + f_mu + b_nu) >> 1;
                M3<T> t = flow_dd(in.load(nu, p, s_diag), in.load(mu, q, s_num));
                acc_mul(A, t, in.load(nu, q, s_num));
            }
        }
        if (MEAS) cp->plaq[(mu * 2 + p) * g.Vh + s] = plaq;
        const M3<T> U = in.load(mu, p, s);
        const AH8<T> Z = project_ah(mul(U, A));
        AH8<T> M;
        if (STAGE == 0) {
            M = ah_scale(alpha, Z);
            zf.store(mu, p, s, Z);
        } else {
            const AH8<T> W = zf.load(mu, p, s);
            M = ah_axpby(alpha, Z, beta, W);
            if (STAGE == 1) zf.store(mu, p, s, M);
        }
        if (KIND == EXP_MORNINGSTAR) out.store(mu, p, s, mul_plus_right(expm_morningstar<T, true>(M), U));
        else out.store(mu, p, s, mul(expm<T>(KIND, M), U));
    }
}

template <typename T, int KIND, int STAGE>
__global__ void __launch_bounds__(kSiteBlock) k_flow_stage_site(Geom g, LinkField<T> in, LinkField<T> out,
                                                                ForceField<T> zf, T alpha, T beta) {
    __shared__ T slots[4 * 18 * kSiteBlock];
    flow_stage_site_body<T, KIND, STAGE>(g, in, out, zf, alpha, beta, blockIdx.x, slots);
}

// One __global__ per register cap (none: the compiler's own choice under
// 128-thread launch bounds) and site-block shape; the autotuner picks among
// them per lattice.
#define GLAC_FLOW_KERNEL(NAME, ATTR)                                                                      \
    template <typename T, int KIND, int STAGE, int SHAPE>                                                \
    __global__ void ATTR NAME(Geom g, LinkField<T> in, LinkField<T> out, ForceField<T> zf, T alpha,      \
                              T beta) {                                                                  \
        flow_stage_body<T, KIND, STAGE, SHAPE>(g, in, out, zf, alpha, beta, blockIdx.x);                 \
    }
GLAC_FLOW_KERNEL(k_flow_stage, __launch_bounds__(128))
GLAC_FLOW_KERNEL(k_flow_stage_r128, __maxnreg__(128))
GLAC_FLOW_KERNEL(k_flow_stage_r80, __maxnreg__(80))
GLAC_FLOW_KERNEL(k_flow_stage_r96, __maxnreg__(96))

// Launch-bound variants (minimum resident blocks of 128 threads per SM, i.e.
// the register cap) that the autotuner chooses among; variant 0 is the default.
// Register caps per variant ([fp64, fp32]; 0 = no cap, -1 = unused slot); the
// flow family also varies the site-block shape.
const int kFlowRegs[2][kMaxVariants] = {{0, 128, 0, 128}, {0, 80, 0, 96}};
const int kFlowShape[2][kMaxVariants] = {{0, 0, 1, 2}, {0, 0, 3, 0}};
const int kMetroRegs[2][kMaxVariants] = {{0, 128, -1, -1}, {0, 96, 80, 128}};
const int kObsRegs[2][kMaxVariants] = {{0, 128, -1, -1}, {0, 128, 168, -1}};

int num_variants(Family f, bool fp32) {
    const int(*t)[kMaxVariants] = f == FAM_FLOW ? kFlowRegs : f == FAM_METRO ? kMetroRegs : kObsRegs;
    int n = 0;
    while (n < kMaxVariants && t[fp32 ? 1 : 0][n] >= 0) n++;
    return n;
}
int variant_regs(Family f, bool fp32, int v) {
    const int(*t)[kMaxVariants] = f == FAM_FLOW ? kFlowRegs : f == FAM_METRO ? kMetroRegs : kObsRegs;
    return (v >= 0 && v < kMaxVariants) ? t[fp32 ? 1 : 0][v] : 0;
}

int variant_shape(Family f, bool fp32, int v) {
    return (f == FAM_FLOW && v >= 0 && v < kMaxVariants) ? kFlowShape[fp32 ? 1 : 0][v] : 0;
}

template <typename T, int KIND, int STAGE, int SHAPE>
static void flow_dispatch_caps(int regs, cudaStream_t st, const Geom &g, const LinkField<T> &in,
                               const LinkField<T> &out, const ForceField<T> &zf, T a, T b) {
    const dim3 grid(8 * ((g.Vh + 127) / 128));
    switch (regs) {
    case 128: k_flow_stage_r128<T, KIND, STAGE, SHAPE><<<grid, 128, 0, st>>>(g, in, out, zf, a, b); break;
    case 96:
        if constexpr (sizeof(T) == 4) {
            k_flow_stage_r96<T, KIND, STAGE, SHAPE><<<grid, 128, 0, st>>>(g, in, out, zf, a, b);
            break;
        }
        [[fallthrough]];
    case 80:
        if constexpr (sizeof(T) == 4) {
            k_flow_stage_r80<T, KIND, STAGE, SHAPE><<<grid, 128, 0, st>>>(g, in, out, zf, a, b);
            break;
        }
        [[fallthrough]];  // no 80-register FP64 variant
    default: k_flow_stage<T, KIND, STAGE, SHAPE><<<grid, 128, 0, st>>>(g, in, out, zf, a, b); break;
    }
}

template <typename T, int KIND, int STAGE>
static void flow_dispatch(int regs, int shape, cudaStream_t st, const Geom &g, const LinkField<T> &in,
                          const LinkField<T> &out, const ForceField<T> &zf, T a, T b) {
    if constexpr (sizeof(T) == 4) {
        if (shape == 3) {
            const dim3 grid(2 * ((g.Vh + kSiteBlock - 1) / kSiteBlock));
            k_flow_stage_site<T, KIND, STAGE><<<grid, kSiteBlock, 0, st>>>(g, in, out, zf, a, b);
            return;
        }
    }
    if (shape == 1) {
        const dim3 grid((g.Vh + 15) / 16);
        k_flow_stage<T, KIND, STAGE, 1><<<grid, 128, 0, st>>>(g, in, out, zf, a, b);
        return;
    }
    if (shape == 2) flow_dispatch_caps<T, KIND, STAGE, 2>(regs, st, g, in, out, zf, a, b);
    else flow_dispatch_caps<T, KIND, STAGE, 0>(regs, st, g, in, out, zf, a, b);
}

template <typename T>
void launch_flow_stage(const Geom &g, const LinkField<T> &in, const LinkField<T> &out, const ForceField<T> &zf,
                       int stage, int kind, double alpha, double beta, int variant, cudaStream_t st) {
    const dim3 grid(8 * ((g.Vh + 127) / 128));
    const T a = (T)alpha, b = (T)beta;
    const bool fp32 = sizeof(T) == 4;
    if (kind == EXP_MORNINGSTAR) {
        const int regs = variant_regs(FAM_FLOW, fp32, variant), shape = variant_shape(FAM_FLOW, fp32, variant);
        if (stage == 0) flow_dispatch<T, 0, 0>(regs, shape, st, g, in, out, zf, a, b);
        else if (stage == 1) flow_dispatch<T, 0, 1>(regs, shape, st, g, in, out, zf, a, b);
        else flow_dispatch<T, 0, 2>(regs, shape, st, g, in, out, zf, a, b);
        return;
    }
#define GLAC_FLOW_CASE(K, S) \
    if (kind == K && stage == S) { k_flow_stage<T, K, S, 0><<<grid, 128, 0, st>>>(g, in, out, zf, a, b); return; }
    GLAC_FLOW_CASE(1, 0) GLAC_FLOW_CASE(1, 1) GLAC_FLOW_CASE(1, 2)
    GLAC_FLOW_CASE(2, 0) GLAC_FLOW_CASE(2, 1) GLAC_FLOW_CASE(2, 2)
    GLAC_FLOW_CASE(3, 0) GLAC_FLOW_CASE(3, 1) GLAC_FLOW_CASE(3, 2)
#undef GLAC_FLOW_CASE
    throw std::invalid_argument("bad flow stage or exp kind");
}
template void launch_flow_stage<double>(const Geom &, const LinkField<double> &, const LinkField<double> &,
                                        const ForceField<double> &, int, int, double, double, int, cudaStream_t);
template void launch_flow_stage<float>(const Geom &, const LinkField<float> &, const LinkField<float> &,
                                       const ForceField<float> &, int, int, double, double, int, cudaStream_t);

// ---------------------------------------------------------------------------
// Flow stage 0 fused with the measurement of its input field.
//
// The clover of the (mu, nu) plane at n is the sum of its four counterclockwise
// leaves, and the staple pieces that stage 0 computes for the link U_mu(n) are
// three of each leaf's four links:
//   S_up  = U_nu(n+mu) U_mu(n+nu)^+ U_nu(n)^+,  S_low = U_nu(n+mu-nu)^+ U_mu(n-nu)^+ U_nu(n-nu),
//   leaf1(n) = U S_up,  leaf4(n) = (U S_low)^+,  leaf2(n+mu) = S_up U,  leaf3(n+mu) = (S_low U)^+
// with U = U_mu(n).  With P(X) = (X - X^+) - 1/3 Tr(X - X^+) (linear, P(X^+) = -P(X)),
// the projected clover F_munu(n) = P(leaf1 + leaf2 + leaf3 + leaf4)(n) is
//   F_munu(n) = P(U W)(n) + P(W U)(n - mu),   W = S_up - S_low,
// two products per plane once the staple is known, against ten in the
// stand-alone observables kernel (GLAC/observables/mastersamplertopcxyz.cpp:
// 253-340 builds each leaf from four links).  Each of the six planes is taken
// by one link direction (mu = 0: nu = 1, 2; mu = 1: nu = 2, 3; mu = 2: nu = 3;
// mu = 3: nu = 0, stored as -F_30 = F_03); the thread writes P(U W) into the
// plane's "local" slot at n and P(W U) into its "forward" slot at n + mu, and
// ReTr(U S_up) (the plaquette of the plane at n) into its direction's
// plaquette slot.  k_obs_combine then adds the two slots of each plane per
// site and reduces plaquette, Q(t) and E exactly as the observables kernel.
// ---------------------------------------------------------------------------
// (C - C^+) made traceless, in the 8-real form: diagonal 2 i Im C_ii minus a
// third of its trace, off-diagonal C_ij - conj(C_ji).  Linear in C.
template <typename T> __device__ __forceinline__ AH8<T> proj_ah8(const M3<T> &C) {
    AH8<T> F;
    const T two = T(2);
    const T tr = (C(0, 0).im + C(1, 1).im + C(2, 2).im) * T(2.0 / 3.0);
    F.a = two * C(0, 0).im - tr;
    F.d = two * C(1, 1).im - tr;
    F.b = cx(C(0, 1).re - C(1, 0).re, C(0, 1).im + C(1, 0).im);
    F.c = cx(C(0, 2).re - C(2, 0).re, C(0, 2).im + C(2, 0).im);
    F.e = cx(C(1, 2).re - C(2, 1).re, C(1, 2).im + C(2, 1).im);
    return F;
}
template <typename T> __device__ __forceinline__ AH8<T> ah_add(const AH8<T> &X, const AH8<T> &Y) {
    AH8<T> Z;
    Z.a = X.a + Y.a;
    Z.d = X.d + Y.d;
    Z.b = X.b + Y.b;
    Z.c = X.c + Y.c;
    Z.e = X.e + Y.e;
    return Z;
}

// plane index of (a, b), a < b: 01 0, 02 1, 03 2, 12 3, 13 4, 23 5
__host__ __device__ constexpr int plane_of(int a, int b) { return a == 0 ? b - 1 : (a == 1 ? b + 1 : 5); }
// the planes link direction mu takes (nu, or -1)
__device__ __forceinline__ bool meas_takes(int mu, int nu) {
    return (mu == 0 && (nu == 1 || nu == 2)) || (mu == 1 && (nu == 2 || nu == 3)) || (mu == 2 && nu == 3) ||
           (mu == 3 && nu == 0);
}

template <typename T> __device__ __forceinline__ AH8<T> ah_neg_if(const AH8<T> &F, bool neg) {
    return neg ? ah_scale(T(-1), F) : F;
}

template <typename T, int KIND>
__device__ __forceinline__ void flow_stage0_meas_body(const Geom &g, const LinkField<T> &in, const LinkField<T> &out,
                                                      const ForceField<T> &zf, const CloverParts<T> &cp, T alpha,
                                                      int bx) {
    const int plane = bx & 7;
    const int s = (bx >> 3) * 128 + threadIdx.x;
    if (s >= g.Vh) return;
    const int mu = plane >> 1, p = plane & 1, q = p ^ 1;
    const Site n = site_from_ps(g, p, s);
    const int f_mu = sizeof(T) == 4 ? step_offset(g, n, mu, +1) : step_offset_indexed(g, n, mu, +1);
    const int s_mu = (n.lex + f_mu) >> 1;
    M3<T> A;
    set_zero(A);
    T plaq = T(0);
#pragma unroll 1
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        int s_nup, s_num, s_diag;
        if constexpr (sizeof(T) == 4) {
            const int b_nu = step_offset(g, n, nu, -1);
            s_nup = (n.lex + step_offset(g, n, nu, +1)) >> 1;
            s_num = (n.lex + b_nu) >> 1;
            s_diag = (n.lex + f_mu + b_nu) >> 1;
        } else {
            s_nup = lex_step(g, n, nu, +1) >> 1;
            s_num = lex_step(g, n, nu, -1) >> 1;
            s_diag = lex_step2(g, n, mu, +1, nu, -1) >> 1;
        }
        if (!meas_takes(mu, nu)) {
            {
                M3<T> t = flow_nd(in.load(nu, q, s_mu), in.load(mu, q, s_nup));
                acc_mul_nd(A, t, in.load(nu, p, s));
            }
            {
                M3<T> t = flow_dd(in.load(nu, p, s_diag), in.load(mu, q, s_num));
                acc_mul(A, t, in.load(nu, q, s_num));
            }
            continue;
        }
        // this thread's plane: the staple pieces separately, then W = S_up - S_low
        M3<T> W;
        {
            M3<T> t = flow_nd(in.load(nu, q, s_mu), in.load(mu, q, s_nup));
            W = flow_nd(t, in.load(nu, p, s));
        }
        add_to(A, W);
        plaq += retr_mul(in.load(mu, p, s), W);  // ReTr(U S_up), the plaquette of the plane at n
        asm volatile("" ::: "memory");
        {
            M3<T> t = flow_dd(in.load(nu, p, s_diag), in.load(mu, q, s_num));
            M3<T> S = flow_nn(t, in.load(nu, q, s_num));
            add_to(A, S);
            sub_from(W, S);
        }
        const bool neg = nu < mu;  // F_numu = -F_munu
        const int pl = neg ? plane_of(nu, mu) : plane_of(mu, nu);
        asm volatile("" ::: "memory");
        cp.ah.store(2 * pl, p, s, ah_neg_if(proj_ah8(mul(in.load(mu, p, s), W)), neg));
        asm volatile("" ::: "memory");
        cp.ah.store(2 * pl + 1, q, s_mu, ah_neg_if(proj_ah8(mul(W, in.load(mu, p, s))), neg));
    }
    cp.plaq[(mu * 2 + p) * g.Vh + s] = plaq;
    const M3<T> U = in.load(mu, p, s);
    const AH8<T> Z = project_ah(mul(U, A));
    zf.store(mu, p, s, Z);
    const AH8<T> M = ah_scale(alpha, Z);
    if (KIND == EXP_MORNINGSTAR) out.store(mu, p, s, mul_plus_right(expm_morningstar<T, true>(M), U));
    else out.store(mu, p, s, mul(expm<T>(KIND, M), U));
}

#define GLAC_FLOW_MEAS_KERNEL(NAME, ATTR)                                                                  \
    template <typename T, int KIND>                                                                      \
    __global__ void ATTR NAME(Geom g, LinkField<T> in, LinkField<T> out, ForceField<T> zf,               \
                              CloverParts<T> cp, T alpha) {                                              \
        flow_stage0_meas_body<T, KIND>(g, in, out, zf, cp, alpha, blockIdx.x);                           \
    }
GLAC_FLOW_MEAS_KERNEL(k_flow_stage0_meas, __launch_bounds__(128))
GLAC_FLOW_MEAS_KERNEL(k_flow_stage0_meas_r128, __maxnreg__(128))
GLAC_FLOW_MEAS_KERNEL(k_flow_stage0_meas_r96, __maxnreg__(96))
#undef GLAC_FLOW_MEAS_KERNEL

// The site-per-thread form (shape 3 of the flow stage) with the measurement.
template <typename T, int KIND>
__global__ void __launch_bounds__(kSiteBlock) k_flow_stage0_meas_site(Geom g, LinkField<T> in, LinkField<T> out,
                                                                      ForceField<T> zf, CloverParts<T> cp, T alpha) {
    __shared__ T slots[4 * 18 * kSiteBlock];
    flow_stage_site_body<T, KIND, 0, true>(g, in, out, zf, alpha, T(0), blockIdx.x, slots, &cp);
}

template <typename T>
void launch_flow_stage0_meas(const Geom &g, const LinkField<T> &in, const LinkField<T> &out, const ForceField<T> &zf,
                             const CloverParts<T> &cp, int kind, double alpha, int regs, cudaStream_t st) {
    const dim3 grid(8 * ((g.Vh + 127) / 128));
    const T a = (T)alpha;
    if constexpr (sizeof(T) == 4) {
        if (regs == 3) {  // the site-per-thread form
            const dim3 gs(2 * ((g.Vh + kSiteBlock - 1) / kSiteBlock));
            switch (kind) {
            case 0: k_flow_stage0_meas_site<T, 0><<<gs, kSiteBlock, 0, st>>>(g, in, out, zf, cp, a); return;
            case 1: k_flow_stage0_meas_site<T, 1><<<gs, kSiteBlock, 0, st>>>(g, in, out, zf, cp, a); return;
            case 2: k_flow_stage0_meas_site<T, 2><<<gs, kSiteBlock, 0, st>>>(g, in, out, zf, cp, a); return;
            case 3: k_flow_stage0_meas_site<T, 3><<<gs, kSiteBlock, 0, st>>>(g, in, out, zf, cp, a); return;
            default: throw std::invalid_argument("bad exp kind");
            }
        }
    }
#define GLAC_MEAS_CASE(K)                                                                                 \
    if (kind == K) {                                                                                      \
        if (regs == 128) k_flow_stage0_meas_r128<T, K><<<grid, 128, 0, st>>>(g, in, out, zf, cp, a);        \
        else if (regs == 96) k_flow_stage0_meas_r96<T, K><<<grid, 128, 0, st>>>(g, in, out, zf, cp, a);     \
        else k_flow_stage0_meas<T, K><<<grid, 128, 0, st>>>(g, in, out, zf, cp, a);                       \
        return;                                                                                           \
    }
    GLAC_MEAS_CASE(0) GLAC_MEAS_CASE(1) GLAC_MEAS_CASE(2) GLAC_MEAS_CASE(3)
#undef GLAC_MEAS_CASE
    throw std::invalid_argument("bad exp kind");
}
template void launch_flow_stage0_meas<double>(const Geom &, const LinkField<double> &, const LinkField<double> &,
                                              const ForceField<double> &, const CloverParts<double> &, int, double,
                                              int, cudaStream_t);
template void launch_flow_stage0_meas<float>(const Geom &, const LinkField<float> &, const LinkField<float> &,
                                             const ForceField<float> &, const CloverParts<float> &, int, double, int,
                                             cudaStream_t);

// ---------------------------------------------------------------------------
// Checkerboard Metropolis sub-sweep over the links (mu, parity p).
// Staple A once per link, then nhits proposals U' = X U with X = R S T or its
// inverse (GLAC/math/matrices/su3matrixgenerator.h:170-321), accepted iff
// exp(-dS) > r with dS = -(beta/3) ReTr[(U' - U) A] (GLAC/system.cpp:333-361,
// GLAC/actions/wilsongaugeaction.cpp:24-27).  The links of one (mu, parity)
// class do not enter each other's staples, so they update concurrently.
// Each hit needs only ReTr(X W) with W = U A kept up to date, since
// ReTr[(XU - U) A] = ReTr(X W) - ReTr(W); the products X U and X W are formed
// only for accepted proposals.
// Random numbers: Philox4x32-10, key = seed, counter = {2 hit + call,
// mu V + lex, sweep, stream}: words 0-5 carry twelve 16-bit uniforms (low half
// first) for R, S, T; words 6-7 the 53-bit accept uniform; bit 0 of word 7
// picks X or X^+.
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ T su_scalar(double v);
template <> __device__ __forceinline__ double su_scalar<double>(double v) { return v; }
template <> __device__ __forceinline__ float su_scalar<float>(double v) { return (float)v; }

GLAC_HD double u_sym16(uint32_t h) { return ((double)h + 0.5) * (1.0 / 65536.0) - 0.5; }

// The same uniform for the FP32 path without a conversion instruction: 2^23 + h
// read from its bit pattern, minus 2^23, gives h exactly; (h + 1/2) 2^-16 - 1/2
// = (2h + 1 - 2^16) 2^-17 has at most 17 significant bits, so the FMA is exact
// and the value equals u_sym16's bit for bit.
__device__ __forceinline__ float u_sym16f(uint32_t h) {
    const float hf = __uint_as_float(0x4B000000u | h) - 8388608.f;
    return __fmaf_rn(hf, 1.f / 65536.f, 0.5f / 65536.f - 0.5f);
}
template <typename T> __device__ __forceinline__ T proposal_uniform(uint32_t h);
template <> __device__ __forceinline__ double proposal_uniform<double>(uint32_t h) { return u_sym16(h); }
template <> __device__ __forceinline__ float proposal_uniform<float>(uint32_t h) { return u_sym16f(h); }

// Accept uniform in [0, 1): 53 bits for FP64; for FP32 the 23 high bits of word 6
// as the mantissa of a float in [1, 2), minus 1 (no conversion instruction).
template <typename T> __device__ __forceinline__ T accept_uniform(uint32_t w6, uint32_t w7);
template <> __device__ __forceinline__ double accept_uniform<double>(uint32_t w6, uint32_t w7) { return u_53(w6, w7); }
template <> __device__ __forceinline__ float accept_uniform<float>(uint32_t w6, uint32_t) {
    return __uint_as_float(0x3F800000u | (w6 >> 9)) - 1.f;
}

template <typename T>
__device__ __forceinline__ void su2_near_unity(T u0, T u1, T u2, T u3, T eps, T sq1me, bool flips, T out[4]) {
    // x0 = sign(u0) sqrt(1 - eps^2), x = eps u / |u|, normalised
    // (GLAC/math/matrices/su3matrixgenerator.h:202-243); without flips x0 > 0
    T x0 = (flips && u0 < T(0)) ? -sq1me : sq1me;
    T rn = sqrt(u1 * u1 + u2 * u2 + u3 * u3) / eps;
    T x1 = u1 / rn, x2 = u2 / rn, x3 = u3 / rn;
    T nrm = sqrt(x0 * x0 + x1 * x1 + x2 * x2 + x3 * x3);
    out[0] = x0 / nrm; out[1] = x1 / nrm; out[2] = x2 / nrm; out[3] = x3 / nrm;
}
// FP32: the same construction with reciprocal square roots in place of the
// square roots and divisions (which load the special-function pipe).
template <>
__device__ __forceinline__ void su2_near_unity<float>(float u0, float u1, float u2, float u3, float eps, float sq1me,
                                                      bool flips, float out[4]) {
    const float x0 = (flips && u0 < 0.f) ? -sq1me : sq1me;
    const float sc = eps * rsqrtf(u1 * u1 + u2 * u2 + u3 * u3);
    const float x1 = u1 * sc, x2 = u2 * sc, x3 = u3 * sc;
    const float inv = rsqrtf(x0 * x0 + x1 * x1 + x2 * x2 + x3 * x3);
    out[0] = x0 * inv; out[1] = x1 * inv; out[2] = x2 * inv; out[3] = x3 * inv;
}

// X = R S T with the SU(2) elements [[x0 + i x3, x2 + i x1], [-x2 + i x1, x0 - i x3]]
// embedded in the (12), (13), (23) blocks; zero blocks skipped.  inverse -> X^+.
template <typename T>
__device__ __forceinline__ M3<T> rst_matrix(const T r[4], const T s[4], const T t[4], bool inverse) {
    const Cx<T> r00 = cx(r[0], r[3]), r01 = cx(r[2], r[1]), r10 = cx(-r[2], r[1]), r11 = cx(r[0], -r[3]);
    const Cx<T> s00 = cx(s[0], s[3]), s01 = cx(s[2], s[1]), s10 = cx(-s[2], s[1]), s11 = cx(s[0], -s[3]);
    const Cx<T> t00 = cx(t[0], t[3]), t01 = cx(t[2], t[1]), t10 = cx(-t[2], t[1]), t11 = cx(t[0], -t[3]);
    // R S = [[r00 s00, r01, r00 s01], [r10 s00, r11, r10 s01], [s10, 0, s11]]
    const Cx<T> a0 = r00 * s00, a2 = r00 * s01, b0 = r10 * s00, b2 = r10 * s01;
    M3<T> X;
    X(0, 0) = a0;
    X(1, 0) = b0;
    X(2, 0) = s10;
    X(0, 1) = cmac(r01 * t00, a2, t10);
    X(1, 1) = cmac(r11 * t00, b2, t10);
    X(2, 1) = s11 * t10;
    X(0, 2) = cmac(r01 * t01, a2, t11);
    X(1, 2) = cmac(r11 * t01, b2, t11);
    X(2, 2) = s11 * t11;
    return inverse ? dagger(X) : X;
}

template <typename T>
__device__ __forceinline__ void draw_proposal(uint32_t k0, uint32_t k1, uint32_t link_id, uint32_t sweep,
                                              uint32_t stream_id, int hit, T eps, T sq1me, bool flips, M3<T> &X,
                                              T &r) {
    uint32_t w[8];
#pragma unroll
    for (int call = 0; call < 2; call++) {
        U4 c = {(uint32_t)(2 * hit + call), link_id, sweep, stream_id};
        U4 o = philox4x32_10(c, k0, k1);
        w[4 * call] = o.x; w[4 * call + 1] = o.y; w[4 * call + 2] = o.z; w[4 * call + 3] = o.w;
    }
    T su[3][4];
#pragma unroll
    for (int b = 0; b < 3; b++) {
        T u[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int k = 4 * b + c;
            const uint32_t word = w[k >> 1];
            u[c] = proposal_uniform<T>((k & 1) ? (word >> 16) : (word & 0xFFFFu));
        }
        su2_near_unity<T>(u[0], u[1], u[2], u[3], eps, sq1me, flips, su[b]);
    }
    X = rst_matrix<T>(su[0], su[1], su[2], (w[7] & 1u) == 0u);
    r = accept_uniform<T>(w[6], w[7]);
}

// exp(-dS) in the working precision (compared with accept_uniform<T>)
template <typename T> __device__ __forceinline__ T accept_weight(T dS);
template <> __device__ __forceinline__ double accept_weight<double>(double dS) { return exp(-dS); }
template <> __device__ __forceinline__ float accept_weight<float>(float dS) { return expf(-dS); }

template <typename T>
__device__ __forceinline__ T delta_s(const M3<T> &U, const M3<T> &Up, const M3<T> &A, T mfac) {
    M3<T> D = Up;
    sub_from(D, U);
    return retr_mul(D, A) * mfac;
}

__device__ __forceinline__ void block_add_u64(unsigned long long v, unsigned long long *dst) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    __shared__ unsigned long long warp_sum[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) warp_sum[wid] = v;
    __syncthreads();
    if (wid == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        v = lane < nw ? warp_sum[lane] : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0 && v) atomicAdd(dst, v);
    }
}

// NUpdates hits on one link with staple A (GLAC/system.cpp:321-331): W = U A is
// kept so a hit costs Re Tr(X W); returns the accepted count.
template <typename T>
__device__ __forceinline__ unsigned long long metropolis_hits(const LinkField<T> &L, int mu, int p, int s,
                                                              const M3<T> &A, T mfac, T eps, T sq1me, bool flips,
                                                              int nhits, uint32_t k0, uint32_t k1, uint32_t link_id,
                                                              uint32_t sweep, uint32_t stream_id) {
    M3<T> U = L.load_rw(mu, p, s);
    M3<T> W = mul(U, A);
    unsigned long long na = 0;
#pragma unroll 1
    for (int h = 0; h < nhits; h++) {
        M3<T> X;
        T r;
        draw_proposal<T>(k0, k1, link_id, sweep, stream_id, h, eps, sq1me, flips, X, r);
        const T dS = (retr_mul(X, W) - retr(W)) * mfac;
        if (accept_weight<T>(dS) > r) {
            U = mul(X, U);
            W = mul(X, W);
            na++;
        }
    }
    L.store(mu, p, s, U);
    return na;
}

// One (mu, parity) sub-sweep.  LEARNED: the spread of each link's proposals is
// the network's output for its staple's features (every lane of the warp takes
// part in the tensor-core inference; lanes past the plane pass zeros).
template <typename T, bool LEARNED>
__device__ __forceinline__ void metropolis_body(const Geom &g, const LinkField<T> &L, int mu, int p, T mfac, T eps,
                                                T sq1me, int nhits, uint32_t k0, uint32_t k1, uint32_t sweep,
                                                uint32_t stream_id, unsigned long long *acc, const Proposal &P,
                                                float beta, int bx) {
    const int s = bx * blockDim.x + threadIdx.x;
    const bool valid = s < g.Vh;
    unsigned long long na = 0;
    if (LEARNED) {
        __shared__ uint32_t feat[4 * 128];
        float f[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        M3<T> A;
        Site n;
        if (valid) {
            n = site_from_ps(g, p, s);
            A = staple<T, true>(L, g, n, p, mu);
            staple_features(A, beta, f);
        }
        const float e = mlp_spread_warp(f, P, feat + (threadIdx.x >> 5) * 128);
        if (valid) {
            const T et = (T)e;
            na = metropolis_hits<T>(L, mu, p, s, A, mfac, et, sqrt(T(1) - et * et), P.flips, nhits, k0, k1,
                                    (uint32_t)mu * (uint32_t)g.V + (uint32_t)n.lex, sweep, stream_id);
        }
    } else if (valid) {
        const Site n = site_from_ps(g, p, s);
        const M3<T> A = staple<T, true>(L, g, n, p, mu);
        na = metropolis_hits<T>(L, mu, p, s, A, mfac, eps, sq1me, P.flips, nhits, k0, k1,
                                (uint32_t)mu * (uint32_t)g.V + (uint32_t)n.lex, sweep, stream_id);
    }
    block_add_u64(na, acc);
}

#define GLAC_METRO_KERNEL(NAME, ATTR)                                                                        \
    template <typename T, bool LEARNED>                                                                    \
    __global__ void ATTR NAME(Geom g, LinkField<T> L, int mu, int p, T mfac, T eps, T sq1me, int nhits,      \
                              uint32_t k0, uint32_t k1, uint32_t sweep, uint32_t stream_id,                 \
                              unsigned long long *acc, Proposal P, float beta) {                            \
        metropolis_body<T, LEARNED>(g, L, mu, p, mfac, eps, sq1me, nhits, k0, k1, sweep, stream_id, acc, P,  \
                                    beta, blockIdx.x);                                                     \
    }
GLAC_METRO_KERNEL(k_metropolis, __launch_bounds__(128))
GLAC_METRO_KERNEL(k_metropolis_r128, __maxnreg__(128))
GLAC_METRO_KERNEL(k_metropolis_r96, __maxnreg__(96))
GLAC_METRO_KERNEL(k_metropolis_r80, __maxnreg__(80))
#undef GLAC_METRO_KERNEL

template <typename T, bool LEARNED>
static void metro_dispatch(int regs, dim3 grid, cudaStream_t st, const Geom &g, const LinkField<T> &L, int mu,
                           int p, T mfac, T e, T sq, int nhits, uint32_t k0, uint32_t k1, uint32_t sweep,
                           uint32_t stream_id, unsigned long long *acc, const Proposal &P, float beta) {
    switch (regs) {
    case 128: k_metropolis_r128<T, LEARNED><<<grid, 128, 0, st>>>(g, L, mu, p, mfac, e, sq, nhits, k0, k1, sweep, stream_id, acc, P, beta); break;
    case 96: k_metropolis_r96<T, LEARNED><<<grid, 128, 0, st>>>(g, L, mu, p, mfac, e, sq, nhits, k0, k1, sweep, stream_id, acc, P, beta); break;
    case 80: k_metropolis_r80<T, LEARNED><<<grid, 128, 0, st>>>(g, L, mu, p, mfac, e, sq, nhits, k0, k1, sweep, stream_id, acc, P, beta); break;
    default: k_metropolis<T, LEARNED><<<grid, 128, 0, st>>>(g, L, mu, p, mfac, e, sq, nhits, k0, k1, sweep, stream_id, acc, P, beta); break;
    }
}

template <typename T>
void launch_metropolis(const Geom &g, const LinkField<T> &L, int mu, int p, double beta, double eps, int nhits,
                       uint64_t seed, uint32_t sweep, uint32_t stream_id, unsigned long long *acc, int variant,
                       const Proposal &P, cudaStream_t st) {
    const dim3 grid((g.Vh + 127) / 128);  // 128 threads: the learned path's shared memory holds 4 warps
    const T mfac = (T)(-beta / 3.0), e = (T)eps, sq = (T)sqrt(1.0 - eps * eps);
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const int regs = variant_regs(FAM_METRO, sizeof(T) == 4, variant);
    if (P.net)
        metro_dispatch<T, true>(regs, grid, st, g, L, mu, p, mfac, e, sq, nhits, k0, k1, sweep, stream_id, acc, P,
                                (float)beta);
    else
        metro_dispatch<T, false>(regs, grid, st, g, L, mu, p, mfac, e, sq, nhits, k0, k1, sweep, stream_id, acc, P,
                                 (float)beta);
}
template void launch_metropolis<double>(const Geom &, const LinkField<double> &, int, int, double, double, int,
                                        uint64_t, uint32_t, uint32_t, unsigned long long *, int, const Proposal &,
                                        cudaStream_t);
template void launch_metropolis<float>(const Geom &, const LinkField<float> &, int, int, double, double, int,
                                       uint64_t, uint32_t, uint32_t, unsigned long long *, int, const Proposal &,
                                       cudaStream_t);

// ---------------------------------------------------------------------------
// Expected-squared-jump data for the learned spread (no reference counterpart).
// Links s = offset + i stride (i < ns) of each (mu, parity) plane, rows in plane
// order.  Per row: the staple's features, then for every eps_k on the grid the
// mean over `trials` of ||U' - U||^2 = 6 - 2 Re Tr(X_acc) after the sampler's
// nhits-hit update of that link (proposals from a Philox stream of their own:
// stream | 2^31, sweep = snapshot, hit index h + 16 (trial + trials k)).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) k_esj(Geom g, LinkField<T> L, float beta, T mfac, int nhits, int n_eps,
                                             const float *__restrict__ eps_grid, int trials, int stride, int offset,
                                             int ns, uint32_t k0, uint32_t k1, uint32_t snapshot, uint32_t stream_id,
                                             bool flips, float *__restrict__ feat, float *__restrict__ esj,
                                             uint32_t *__restrict__ ids) {
    const long long row = (long long)blockIdx.x * 128 + threadIdx.x;
    if (row >= 8ll * ns) return;
    const int plane = (int)(row / ns), i = (int)(row % ns);
    const int mu = plane >> 1, p = plane & 1, s = offset + i * stride;
    const Site n = site_from_ps(g, p, s);
    const M3<T> A = staple(L, g, n, p, mu);
    float f[8];
    staple_features(A, beta, f);
    float4 *fo = reinterpret_cast<float4 *>(feat + row * 8);
    fo[0] = make_float4(f[0], f[1], f[2], f[3]);
    fo[1] = make_float4(f[4], f[5], f[6], f[7]);
    const uint32_t link_id = (uint32_t)mu * (uint32_t)g.V + (uint32_t)n.lex;
    if (ids) ids[row] = link_id;
    if (n_eps == 0) return;
    const M3<T> W0 = mul(L.load(mu, p, s), A);
    for (int k = 0; k < n_eps; k++) {
        const T eps = (T)eps_grid[k], sq = sqrt(T(1) - eps * eps);
        T J = T(0);
        for (int tr = 0; tr < trials; tr++) {
            M3<T> Xt, Wc = W0;
            set_identity(Xt);
#pragma unroll 1
            for (int h = 0; h < nhits; h++) {
                M3<T> X;
                T r;
                draw_proposal<T>(k0, k1, link_id, snapshot, stream_id, h + 16 * (tr + trials * k), eps, sq, flips, X,
                                 r);
                const T dS = (retr_mul(X, Wc) - retr(Wc)) * mfac;
                if (accept_weight<T>(dS) > r) {
                    Xt = mul(X, Xt);
                    Wc = mul(X, Wc);
                }
            }
            J += T(6) - T(2) * retr(Xt);
        }
        esj[row * n_eps + k] = (float)(J / T(trials));
    }
}

template <typename T>
void launch_esj(const Geom &g, const LinkField<T> &L, double beta, int nhits, int n_eps, const float *eps_grid_dev,
                int trials, int stride, int offset, int ns, uint64_t seed, uint32_t snapshot, uint32_t stream_id,
                bool flips, float *feat, float *esj, uint32_t *ids, cudaStream_t st) {
    const long long rows = 8ll * ns;
    k_esj<T><<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(g, L, (float)beta, (T)(-beta / 3.0), nhits, n_eps,
                                                            eps_grid_dev, trials, stride, offset, ns, (uint32_t)seed,
                                                            (uint32_t)(seed >> 32), snapshot,
                                                            stream_id | 0x80000000u, flips, feat, esj, ids);
}
template void launch_esj<double>(const Geom &, const LinkField<double> &, double, int, int, const float *, int, int,
                                 int, int, uint64_t, uint32_t, uint32_t, bool, float *, float *, uint32_t *,
                                 cudaStream_t);
template void launch_esj<float>(const Geom &, const LinkField<float> &, double, int, int, const float *, int, int,
                                int, int, uint64_t, uint32_t, uint32_t, bool, float *, float *, uint32_t *,
                                cudaStream_t);

// ---------------------------------------------------------------------------
// Observables (GLAC/observables/mastersamplertopcxyz.cpp:236-384): per site,
// for nu = 1..3 and its cyclic complement (rho, sigma), the clovers
//   C = leaf1 - leaf2 + leaf3 - leaf4 projected to (C - C^+) - 1/3 i ImTr,
// plaq += ReTr leaf1, q(t) -= ReTr(C_0nu C_rhosigma), E += ReTr(C C) for both.
// Every block lies in one (t, parity) half-slice, so the block sums are
// per-time-slice partials; FP64 throughout the reduction, fixed order.
// ---------------------------------------------------------------------------
ObsPlan make_obs_plan(const Geom &g) {
    const int half_slice = g.N[0] * g.N[1] * g.N[2] / 2;
    int best = -1, best_score = 1 << 30;
    for (int B = 1; B <= 256 && B <= half_slice; B++) {
        if (half_slice % B) continue;
        int score = (B % 32 == 0 ? 0 : 100000) + std::abs(B - 128);
        if (score < best_score) { best_score = score; best = B; }
    }
    ObsPlan pl;
    pl.Bv = best;
    pl.B = (best + 31) / 32 * 32;
    pl.nb = half_slice / best;
    pl.nblocks = g.N[3] * 2 * pl.nb;
    return pl;
}

// Clover of the (mu, nu) plane at n, projected: F = (C - C^+) - 1/3 i ImTr(C - C^+),
// returned in the 8-real form; *plaq = ReTr(leaf1).  Links are re-read from
// L1/L2 rather than held, to keep register pressure low.  C = leaf1 - leaf2 +
// leaf3 - leaf4 as in the reference (mastersampler.cpp:175-207); FP32 sums the
// leaves in a different order (pairs sharing their first link).  The FP64 form
// runs as a non-inlined call (clover_ah_call): with its own register allocation
// the calling kernels fit a 128-register cap with a small spill, where the
// inlined FP64 form spills kilobytes; the autotuner picks among the caps.
template <typename T>
__device__ __forceinline__ AH8<T> clover_ah_body(const LinkField<T> &L, const Geom &g, const Site &n, int p,
                                                 int mu, int nu, T &plaq) {
    const int q = p ^ 1;
    const int s_n = n.lex >> 1;
    const int s_mup = lex_step(g, n, mu, +1) >> 1;           // n+mu      (q)
    const int s_nup = lex_step(g, n, nu, +1) >> 1;           // n+nu      (q)
    const int s_num = lex_step(g, n, nu, -1) >> 1;           // n-nu      (q)
    const int s_mum = lex_step(g, n, mu, -1) >> 1;           // n-mu      (q)
    const int s_pm = lex_step2(g, n, mu, +1, nu, -1) >> 1;   // n+mu-nu   (p)
    const int s_mm = lex_step2(g, n, mu, -1, nu, -1) >> 1;   // n-mu-nu   (p)
    const int s_mp = lex_step2(g, n, mu, -1, nu, +1) >> 1;   // n-mu+nu   (p)
    AH8<T> F;
    if constexpr (sizeof(T) == 4) {
        // FP32: the four leaves share their first link in pairs, so the clover
        // is formed as C = U_mu(n) (S1 - S2) + U_mu(n-mu)^+ (T3 - T4), 10
        // products instead of 12.  Each three-link piece is a left-to-right
        // chain (one product and one link live at a time); the second half is
        // projected to 8 reals before the first is built, so at most one 3x3 sum
        // is held beside the chain.  (7 % faster than the four-leaf form below
        // in FP32 on B200; slower in FP64, which keeps the four-leaf form.)
        {   // leaf3 - leaf4 = U_mu(n-mu)^+ [U_nu(n-mu-nu)^+ U_mu(n-mu-nu) U_nu(n-nu) - U_nu(n-mu) U_mu(n-mu+nu) U_nu(n)^+]
            M3<T> E = mul(mul_dn(L.load(nu, p, s_mm), L.load(mu, p, s_mm)), L.load(nu, q, s_num));
            asm volatile("" ::: "memory");
            sub_mul_nd(E, mul(L.load(nu, q, s_mum), L.load(mu, p, s_mp)), L.load(nu, p, s_n));
            F = proj_ah8(mul_dn(L.load(mu, q, s_mum), E));
        }
        asm volatile("" ::: "memory");
        {   // leaf1 - leaf2 = U_mu(n) [U_nu(n+mu) U_mu(n+nu)^+ U_nu(n)^+ - U_nu(n+mu-nu)^+ U_mu(n-nu)^+ U_nu(n-nu)]
            M3<T> D = mul_nd(mul_nd(L.load(nu, q, s_mup), L.load(mu, q, s_nup)), L.load(nu, p, s_n));
            plaq = retr_mul(L.load(mu, p, s_n), D);  // ReTr(leaf1)
            asm volatile("" ::: "memory");
            sub_mul(D, mul_dd(L.load(nu, p, s_pm), L.load(mu, q, s_num)), L.load(nu, q, s_num));
            asm volatile("" ::: "memory");  // U_mu(n) is read again (L1) rather than held
            F = ah_add(F, proj_ah8(mul(L.load(mu, p, s_n), D)));
        }
    } else {
        // FP64: each leaf is a left-to-right chain that brings in one link per
        // product, so one product and one link are live at a time; compiler
        // fences between the leaves keep their loads from being hoisted together.
        M3<T> C;
        {   // leaf1 = U_mu(n) U_nu(n+mu) U_mu(n+nu)^+ U_nu(n)^+
            M3<T> t = mul(L.load(mu, p, s_n), L.load(nu, q, s_mup));
            t = mul_nd(t, L.load(mu, q, s_nup));
            C = mul_nd(t, L.load(nu, p, s_n));
            plaq = retr(C);
        }
        asm volatile("" ::: "memory");
        {   // leaf2 = U_mu(n) U_nu(n+mu-nu)^+ U_mu(n-nu)^+ U_nu(n-nu)
            M3<T> t = mul_nd(L.load(mu, p, s_n), L.load(nu, p, s_pm));
            t = mul_nd(t, L.load(mu, q, s_num));
            sub_from(C, mul(t, L.load(nu, q, s_num)));
        }
        asm volatile("" ::: "memory");
        {   // leaf3 = U_mu(n-mu)^+ U_nu(n-mu-nu)^+ U_mu(n-mu-nu) U_nu(n-nu)
            M3<T> t = mul_dd(L.load(mu, q, s_mum), L.load(nu, p, s_mm));
            t = mul(t, L.load(mu, p, s_mm));
            add_to(C, mul(t, L.load(nu, q, s_num)));
        }
        asm volatile("" ::: "memory");
        {   // leaf4 = U_mu(n-mu)^+ U_nu(n-mu) U_mu(n-mu+nu) U_nu(n)^+
            M3<T> t = mul_dn(L.load(mu, q, s_mum), L.load(nu, q, s_mum));
            t = mul(t, L.load(mu, p, s_mp));
            sub_from(C, mul_nd(t, L.load(nu, p, s_n)));
        }
        F = proj_ah8(C);
    }
    return F;
}

template <typename T>
__device__ __noinline__ AH8<T> clover_ah_call(const LinkField<T> &L, const Geom &g, const Site &n, int p, int mu,
                                              int nu, T &plaq) {
    return clover_ah_body<T>(L, g, n, p, mu, nu, plaq);
}
// FP32: inlined (the leaf-pair form fits the 128-register variant with a 4 B
// spill); FP64: a call with its own register allocation.
template <typename T>
__device__ __forceinline__ AH8<T> clover_ah(const LinkField<T> &L, const Geom &g, const Site &n, int p, int mu,
                                            int nu, T &plaq) {
    if constexpr (sizeof(T) == 4) return clover_ah_body<T>(L, g, n, p, mu, nu, plaq);
    else return clover_ah_call<T>(L, g, n, p, mu, nu, plaq);
}

// Re Tr(F G) for traceless anti-Hermitian F, G in the 8-real form:
//   -[a a' + d d' + (a+d)(a'+d')] - 2 Re(b b'* + c c'* + e e'*)
template <typename T>
__device__ __forceinline__ T retr_ah(const AH8<T> &F, const AH8<T> &G) {
    T diag = fmaR(F.a, G.a, F.d * G.d);
    diag = fmaR(F.a + F.d, G.a + G.d, diag);
    T off = fmaR(F.b.re, G.b.re, F.b.im * G.b.im);
    off = fmaR(F.c.re, G.c.re, off);
    off = fmaR(F.c.im, G.c.im, off);
    off = fmaR(F.e.re, G.e.re, off);
    off = fmaR(F.e.im, G.e.im, off);
    return -(diag + off + off);
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Block sums of the three per-thread values in a fixed order (warp shuffles,
// then the warps in order) into partial[3 b .. 3 b + 2] = (plaq, energy, q).
__device__ __forceinline__ void obs_block_reduce(double plaq, double en, double qt, double *partial, int b) {
    __shared__ double sh[3][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    plaq = warp_sum_d(plaq);
    en = warp_sum_d(en);
    qt = warp_sum_d(qt);
    if (lane == 0) { sh[0][wid] = plaq; sh[1][wid] = en; sh[2][wid] = qt; }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double a = 0.0, e = 0.0, q = 0.0;
        for (int w = 0; w < nw; w++) { a += sh[0][w]; e += sh[1][w]; q += sh[2][w]; }
        partial[3 * b] = a;
        partial[3 * b + 1] = e;
        partial[3 * b + 2] = q;
    }
}

// With dq/de set, also the per-site densities in lexicographic order:
// dq[n] = -(1/(16^2 pi^2)) sum ReTr(C_0nu C_rhosigma), de[n] = sum ReTr(C C) (unnormalised),
// the fields LatticeActionChargeDensity writes (latticeactionchargedensity.cpp:169-306).
template <typename T>
__device__ __forceinline__ void observables_body(const Geom &g, const LinkField<T> &L, int nb, int Bv,
                                                 double *partial, int b, double *dq = nullptr,
                                                 double *de = nullptr) {
    const int t = b / (2 * nb);
    const int p = (b / nb) & 1;
    const int j = b % nb;
    const int half_slice = g.Vh / g.N[3];
    const bool valid = (int)threadIdx.x < Bv;
    const int s = t * half_slice + j * Bv + (valid ? (int)threadIdx.x : 0);
    double plaq = 0.0, en = 0.0, qt = 0.0;
    const Site n = site_from_ps(g, p, s);
    if (valid) {
#pragma unroll 1
        for (int nu = 1; nu < 4; nu++) {
            const int rho = nu % 3 + 1, sigma = rho % 3 + 1;
            T pl1, pl2;
            const AH8<T> F1 = clover_ah(L, g, n, p, 0, nu, pl1);
            asm volatile("" ::: "memory");  // one clover at a time: bounds the live registers
            const AH8<T> F2 = clover_ah(L, g, n, p, rho, sigma, pl2);
            plaq += (double)pl1 + (double)pl2;
            qt -= (double)retr_ah(F1, F2);
            en += (double)retr_ah(F1, F1) + (double)retr_ah(F2, F2);
        }
        if (dq) {
            dq[n.lex] = qt * (1.0 / (16 * 16 * M_PI * M_PI));
            de[n.lex] = en;
        }
    }
    obs_block_reduce(plaq, en, qt, partial, b);
}

#define GLAC_OBS_KERNEL(NAME, ATTR)                                                                      \
    template <typename T>                                                                              \
    __global__ void ATTR NAME(Geom g, LinkField<T> L, int nb, int Bv, double *partial) {               \
        observables_body<T>(g, L, nb, Bv, partial, blockIdx.x);                                        \
    }
GLAC_OBS_KERNEL(k_observables, __launch_bounds__(256))
GLAC_OBS_KERNEL(k_observables_r168, __maxnreg__(168))
GLAC_OBS_KERNEL(k_observables_r128, __maxnreg__(128))
GLAC_OBS_KERNEL(k_observables_r96, __maxnreg__(96))
#undef GLAC_OBS_KERNEL

// out = [plaq, topc, energy, topct[Nt]] with the reference's normalisations
// (mastersamplertopcxyz.cpp:13-16, :363-383).
// Per-slice sums by warps (slice t on warp t mod W; lane l adds the partials
// l, l+32, ..., then a fixed xor-shuffle tree), the slices then in order by one
// thread: the same operations in the same order every call.
__device__ __forceinline__ void obs_finalize_body(int Nt, int nb, int V, const double *partial, double *out) {
    __shared__ double sp[1024], se[1024], sq[1024];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int t = warp; t < Nt; t += nwarps) {
        double a = 0.0, e = 0.0, q = 0.0;
        const double *pt = partial + 3 * (size_t)t * 2 * nb;
        for (int k = lane; k < 2 * nb; k += 32) {
            a += pt[3 * k];
            e += pt[3 * k + 1];
            q += pt[3 * k + 2];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            e += __shfl_xor_sync(0xffffffffu, e, o);
            q += __shfl_xor_sync(0xffffffffu, q, o);
        }
        if (lane == 0) { sp[t] = a; se[t] = e; sq[t] = q; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double qfac = 1.0 / (16 * 16 * M_PI * M_PI);
        double a = 0.0, e = 0.0, q = 0.0;
        for (int t = 0; t < Nt; t++) { a += sp[t]; e += se[t]; q += sq[t]; }
        out[0] = a / (18.0 * (double)V);
        out[1] = q * qfac;
        out[2] = e / (double)V;
        for (int t = 0; t < Nt; t++) out[3 + t] = sq[t] * qfac;
    }
}
__global__ void k_obs_finalize(int Nt, int nb, int V, const double *partial, double *out) {
    obs_finalize_body(Nt, nb, V, partial, out);
}

template <typename T>
void launch_observables(const Geom &g, const LinkField<T> &L, const ObsPlan &plan, double *partial, double *out,
                        int variant, cudaStream_t st) {
    if (g.N[3] > 1024) throw std::invalid_argument("Nt > 1024 not supported by the observable reduction");
    switch (variant_regs(FAM_OBS, sizeof(T) == 4, variant)) {
    case 168:
        if constexpr (sizeof(T) == 4) {
            k_observables_r168<T><<<plan.nblocks, plan.B, 0, st>>>(g, L, plan.nb, plan.Bv, partial);
            break;
        }
        [[fallthrough]];
    case 128: k_observables_r128<T><<<plan.nblocks, plan.B, 0, st>>>(g, L, plan.nb, plan.Bv, partial); break;
    case 96: k_observables_r96<T><<<plan.nblocks, plan.B, 0, st>>>(g, L, plan.nb, plan.Bv, partial); break;
    default: k_observables<T><<<plan.nblocks, plan.B, 0, st>>>(g, L, plan.nb, plan.Bv, partial); break;
    }
    k_obs_finalize<<<1, 1024, 0, st>>>(g.N[3], plan.nb, g.V, partial, out);
}
// The measurement from the parts that flow stage 0 wrote (flow_stage0_meas_body):
// per site F of each plane = its local + forward slot, the plaquette = the four
// direction sums; Q(t), E and the plaquette reduced as in observables_body (same
// blocks, same fixed order), then k_obs_finalize.
template <typename T>
__device__ __forceinline__ void combine_site(const Geom &g, const CloverParts<T> &cp, int p, int s, double &plaq,
                                             double &en, double &qt) {
    AH8<T> F[6];
#pragma unroll
    for (int pl = 0; pl < 6; pl++) F[pl] = ah_add(cp.ah.load(2 * pl, p, s), cp.ah.load(2 * pl + 1, p, s));
#pragma unroll
    for (int mu = 0; mu < 4; mu++) plaq += (double)cp.plaq[(mu * 2 + p) * g.Vh + s];
    // q = -[ReTr(F_01 F_23) + ReTr(F_02 F_31) + ReTr(F_03 F_12)], F_31 = -F_13
    qt = -((double)retr_ah(F[0], F[5]) - (double)retr_ah(F[1], F[4]) + (double)retr_ah(F[2], F[3]));
#pragma unroll
    for (int pl = 0; pl < 6; pl++) en += (double)retr_ah(F[pl], F[pl]);
}

template <typename T>
__global__ void __launch_bounds__(256) k_obs_combine(Geom g, CloverParts<T> cp, int nb, int Bv, double *partial) {
    const int b = blockIdx.x;
    const int t = b / (2 * nb);
    const int p = (b / nb) & 1;
    const int j = b % nb;
    const int half_slice = g.Vh / g.N[3];
    const bool valid = (int)threadIdx.x < Bv;
    const int s = t * half_slice + j * Bv + (valid ? (int)threadIdx.x : 0);
    double plaq = 0.0, en = 0.0, qt = 0.0;
    if (valid) combine_site(g, cp, p, s, plaq, en, qt);
    obs_block_reduce(plaq, en, qt, partial, b);
}

// Flow stage 1 that also does the measurement's per-site combination and
// block reduction: the blocks of the mu = 0 planes (shape 0: 128 consecutive
// sites of one parity) combine the clover parts of their own 128 sites after
// their links' stage-1 update.  For lattices whose half time slice is a
// multiple of 128 sites, so that each such block lies in one (t, parity) half
// slice and its partial sums sit where the observable plan's 128-site blocks
// put them (obs_combine_in_stage1).  Launch bounds: six blocks of 128 per SM
// in FP32 (80 registers, 12 B spill; 3 % faster than five blocks at 96 on
// B200), three in FP64.
template <typename T, int KIND>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 6 : 3) k_flow_stage1_combine(Geom g, LinkField<T> in, LinkField<T> out,
                                                             ForceField<T> zf, T alpha, T beta, CloverParts<T> cp,
                                                             double *partial) {
    flow_stage_body<T, KIND, 1, 0>(g, in, out, zf, alpha, beta, blockIdx.x);
    const int plane = blockIdx.x & 7;
    if (plane >= 2) return;  // a whole block returns together
    const int p = plane & 1;
    const int s0 = (blockIdx.x >> 3) * 128, s = s0 + threadIdx.x;
    const int half_slice = g.Vh / g.N[3];
    const int nb = half_slice >> 7;
    const int t = s0 / half_slice, j = (s0 - t * half_slice) >> 7;
    double plaq = 0.0, en = 0.0, qt = 0.0;
    combine_site(g, cp, p, s, plaq, en, qt);
    obs_block_reduce(plaq, en, qt, partial, (t * 2 + p) * nb + j);
}

// The same with the site-per-thread stage (FP32 shape 3): every block covers
// 128 consecutive sites of one parity, does their four links' stage-1 update,
// then combines and reduces the measurement parts of those sites.
template <typename T, int KIND>
__global__ void __launch_bounds__(kSiteBlock) k_flow_stage1_combine_site(Geom g, LinkField<T> in, LinkField<T> out,
                                                                         ForceField<T> zf, T alpha, T beta,
                                                                         CloverParts<T> cp, double *partial) {
    __shared__ T slots[4 * 18 * kSiteBlock];
    flow_stage_site_body<T, KIND, 1>(g, in, out, zf, alpha, beta, blockIdx.x, slots);
    const int p = blockIdx.x & 1;
    const int s0 = (blockIdx.x >> 1) * kSiteBlock, s = s0 + threadIdx.x;
    const int half_slice = g.Vh / g.N[3];
    const int nb = half_slice >> 7;
    const int t = s0 / half_slice, j = (s0 - t * half_slice) >> 7;
    double plaq = 0.0, en = 0.0, qt = 0.0;
    combine_site(g, cp, p, s, plaq, en, qt);
    obs_block_reduce(plaq, en, qt, partial, (t * 2 + p) * nb + j);
}

bool obs_combine_in_stage1(const Geom &g, const ObsPlan &plan) {
    const int half_slice = g.Vh / g.N[3];
    return half_slice % 128 == 0 && plan.Bv == 128 && plan.nb == half_slice / 128;
}

template <typename T>
void launch_flow_stage1_combine(const Geom &g, const LinkField<T> &in, const LinkField<T> &out,
                                const ForceField<T> &zf, int kind, double alpha, double beta,
                                const CloverParts<T> &cp, const ObsPlan &plan, double *partial, double *obs_out,
                                bool site, cudaStream_t st) {
    if (g.N[3] > 1024) throw std::invalid_argument("Nt > 1024 not supported by the observable reduction");
    if (!obs_combine_in_stage1(g, plan)) throw std::invalid_argument("lattice does not allow the stage-1 combine");
    const dim3 grid(8 * (g.Vh / 128));
    const T a = (T)alpha, b = (T)beta;
    if constexpr (sizeof(T) == 4) {
        if (site) {
            const dim3 gs(2 * (g.Vh / kSiteBlock));
            switch (kind) {
            case 0: k_flow_stage1_combine_site<T, 0><<<gs, kSiteBlock, 0, st>>>(g, in, out, zf, a, b, cp, partial); break;
            case 1: k_flow_stage1_combine_site<T, 1><<<gs, kSiteBlock, 0, st>>>(g, in, out, zf, a, b, cp, partial); break;
            case 2: k_flow_stage1_combine_site<T, 2><<<gs, kSiteBlock, 0, st>>>(g, in, out, zf, a, b, cp, partial); break;
            case 3: k_flow_stage1_combine_site<T, 3><<<gs, kSiteBlock, 0, st>>>(g, in, out, zf, a, b, cp, partial); break;
            default: throw std::invalid_argument("bad exp kind");
            }
            k_obs_finalize<<<1, 1024, 0, st>>>(g.N[3], plan.nb, g.V, partial, obs_out);
            return;
        }
    }
    switch (kind) {
    case 0: k_flow_stage1_combine<T, 0><<<grid, 128, 0, st>>>(g, in, out, zf, a, b, cp, partial); break;
    case 1: k_flow_stage1_combine<T, 1><<<grid, 128, 0, st>>>(g, in, out, zf, a, b, cp, partial); break;
    case 2: k_flow_stage1_combine<T, 2><<<grid, 128, 0, st>>>(g, in, out, zf, a, b, cp, partial); break;
    case 3: k_flow_stage1_combine<T, 3><<<grid, 128, 0, st>>>(g, in, out, zf, a, b, cp, partial); break;
    default: throw std::invalid_argument("bad exp kind");
    }
    k_obs_finalize<<<1, 1024, 0, st>>>(g.N[3], plan.nb, g.V, partial, obs_out);
}
template void launch_flow_stage1_combine<double>(const Geom &, const LinkField<double> &, const LinkField<double> &,
                                                 const ForceField<double> &, int, double, double,
                                                 const CloverParts<double> &, const ObsPlan &, double *, double *,
                                                 bool, cudaStream_t);
template void launch_flow_stage1_combine<float>(const Geom &, const LinkField<float> &, const LinkField<float> &,
                                                const ForceField<float> &, int, double, double,
                                                const CloverParts<float> &, const ObsPlan &, double *, double *,
                                                bool, cudaStream_t);

template <typename T>
void launch_obs_combine(const Geom &g, const CloverParts<T> &cp, const ObsPlan &plan, double *partial, double *out,
                        cudaStream_t st) {
    if (g.N[3] > 1024) throw std::invalid_argument("Nt > 1024 not supported by the observable reduction");
    k_obs_combine<T><<<plan.nblocks, plan.B, 0, st>>>(g, cp, plan.nb, plan.Bv, partial);
    k_obs_finalize<<<1, 1024, 0, st>>>(g.N[3], plan.nb, g.V, partial, out);
}
template void launch_obs_combine<double>(const Geom &, const CloverParts<double> &, const ObsPlan &, double *,
                                         double *, cudaStream_t);
template void launch_obs_combine<float>(const Geom &, const CloverParts<float> &, const ObsPlan &, double *, double *,
                                        cudaStream_t);

template <typename T>
__global__ void __launch_bounds__(256) k_observables_density(Geom g, LinkField<T> L, int nb, int Bv, double *partial,
                                                             double *dq, double *de) {
    observables_body<T>(g, L, nb, Bv, partial, blockIdx.x, dq, de);
}
template <typename T>
void launch_observables_density(const Geom &g, const LinkField<T> &L, const ObsPlan &plan, double *partial,
                                double *out, double *dq, double *de, cudaStream_t st) {
    if (g.N[3] > 1024) throw std::invalid_argument("Nt > 1024 not supported by the observable reduction");
    k_observables_density<T><<<plan.nblocks, plan.B, 0, st>>>(g, L, plan.nb, plan.Bv, partial, dq, de);
    k_obs_finalize<<<1, 1024, 0, st>>>(g.N[3], plan.nb, g.V, partial, out);
}
template void launch_observables_density<double>(const Geom &, const LinkField<double> &, const ObsPlan &, double *,
                                                 double *, double *, double *, cudaStream_t);
template void launch_observables_density<float>(const Geom &, const LinkField<float> &, const ObsPlan &, double *,
                                                double *, double *, double *, cudaStream_t);
template void launch_observables<double>(const Geom &, const LinkField<double> &, const ObsPlan &, double *,
                                         double *, int, cudaStream_t);
template void launch_observables<float>(const Geom &, const LinkField<float> &, const ObsPlan &, double *,
                                        double *, int, cudaStream_t);

// ---------------------------------------------------------------------------
// SuperSampler (GLAC/observables/supersampler.cpp:298-496): the observables
// above plus the Weinberg operator.  With the six projected clovers G of a
// site, for nu = 1..3 and (rho, sigma) the cyclic complement of nu:
//   w(t) -= ReTr[(sum_{lambda != nu} G_{0 lambda} G_{nu lambda}) G_{rho sigma}],
// factor 2 * 8 * 8 / (3 * 16^3) (:13).  G_{b a} = G_{a b}^+ for the
// orientations the reference does not store (:421-433).  Partials: 4 per block.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_observables_weinberg(Geom g, LinkField<T> L, int nb, int Bv,
                                                              double *partial) {
    const int b = blockIdx.x;
    const int t = b / (2 * nb);
    const int p = (b / nb) & 1;
    const int j = b % nb;
    const int half_slice = g.Vh / g.N[3];
    const bool valid = (int)threadIdx.x < Bv;
    const int s = t * half_slice + j * Bv + (valid ? (int)threadIdx.x : 0);
    double plaq = 0.0, en = 0.0, qt = 0.0, wt = 0.0;
    if (valid) {
        const Site n = site_from_ps(g, p, s);
        AH8<T> G0[4], Gc[4];  // G0[nu] = G_{0 nu}; Gc[nu] = G_{rho sigma} of nu's complement
#pragma unroll 1
        for (int nu = 1; nu < 4; nu++) {
            const int rho = nu % 3 + 1, sigma = rho % 3 + 1;
            T pl1, pl2;
            G0[nu] = clover_ah(L, g, n, p, 0, nu, pl1);
            Gc[nu] = clover_ah(L, g, n, p, rho, sigma, pl2);
            plaq += (double)pl1 + (double)pl2;
            qt -= (double)retr_ah(G0[nu], Gc[nu]);
            en += (double)retr_ah(G0[nu], G0[nu]) + (double)retr_ah(Gc[nu], Gc[nu]);
        }
        // G_{a b} for spatial a != b from the stored G_{23} = Gc[1], G_{31} = Gc[2], G_{12} = Gc[3]
        auto spatial = [&](int a, int c) -> M3<T> {
            // (a, c) in {(1,2),(2,3),(3,1)} is stored as Gc[the third index]; the reverse is its dagger
            const int k = 6 - a - c;
            const bool stored = (c == a % 3 + 1);
            const M3<T> m = ah_to_m3(Gc[k]);
            return stored ? m : dagger(m);
        };
#pragma unroll 1
        for (int nu = 1; nu < 4; nu++) {
            M3<T> acc;
            set_zero(acc);
#pragma unroll 1
            for (int lam = 1; lam < 4; lam++) {
                if (lam == nu) continue;
                acc_mul(acc, ah_to_m3(G0[lam]), spatial(nu, lam));
            }
            wt -= (double)retr_mul(acc, ah_to_m3(Gc[nu]));
        }
    }
    __shared__ double sh[4][32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    plaq = warp_sum_d(plaq);
    en = warp_sum_d(en);
    qt = warp_sum_d(qt);
    wt = warp_sum_d(wt);
    if (lane == 0) { sh[0][wid] = plaq; sh[1][wid] = en; sh[2][wid] = qt; sh[3][wid] = wt; }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int nw = (blockDim.x + 31) >> 5;
        double a = 0.0, e = 0.0, q = 0.0, w = 0.0;
        for (int k = 0; k < nw; k++) { a += sh[0][k]; e += sh[1][k]; q += sh[2][k]; w += sh[3][k]; }
        partial[4 * b] = a;
        partial[4 * b + 1] = e;
        partial[4 * b + 2] = q;
        partial[4 * b + 3] = w;
    }
}

// out = [plaq, topc, energy, weinberg, topct[Nt], weinbergt[Nt]]
__global__ void k_weinberg_finalize(int Nt, int nb, int V, const double *partial, double *out) {
    __shared__ double sp[1024], se[1024], sq[1024], sw[1024];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int t = warp; t < Nt; t += nwarps) {
        double a = 0.0, e = 0.0, q = 0.0, w = 0.0;
        const double *pt = partial + 4 * (size_t)t * 2 * nb;
        for (int k = lane; k < 2 * nb; k += 32) {
            a += pt[4 * k];
            e += pt[4 * k + 1];
            q += pt[4 * k + 2];
            w += pt[4 * k + 3];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_xor_sync(0xffffffffu, a, o);
            e += __shfl_xor_sync(0xffffffffu, e, o);
            q += __shfl_xor_sync(0xffffffffu, q, o);
            w += __shfl_xor_sync(0xffffffffu, w, o);
        }
        if (lane == 0) { sp[t] = a; se[t] = e; sq[t] = q; sw[t] = w; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double qfac = 1.0 / (16 * 16 * M_PI * M_PI), wfac = 2 * 8.0 * 8.0 / (3 * 16 * 16 * 16);
        double a = 0.0, e = 0.0, q = 0.0, w = 0.0;
        for (int t = 0; t < Nt; t++) { a += sp[t]; e += se[t]; q += sq[t]; w += sw[t]; }
        out[0] = a / (18.0 * (double)V);
        out[1] = q * qfac;
        out[2] = e / (double)V;
        out[3] = w * wfac;
        for (int t = 0; t < Nt; t++) {
            out[4 + t] = sq[t] * qfac;
            out[4 + Nt + t] = sw[t] * wfac;
        }
    }
}

template <typename T>
void launch_weinberg(const Geom &g, const LinkField<T> &L, const ObsPlan &plan, double *partial4, double *out,
                     cudaStream_t st) {
    if (g.N[3] > 1024) throw std::invalid_argument("Nt > 1024 not supported by the observable reduction");
    k_observables_weinberg<T><<<plan.nblocks, plan.B, 0, st>>>(g, L, plan.nb, plan.Bv, partial4);
    k_weinberg_finalize<<<1, 1024, 0, st>>>(g.N[3], plan.nb, g.V, partial4, out);
}
template void launch_weinberg<double>(const Geom &, const LinkField<double> &, const ObsPlan &, double *, double *,
                                      cudaStream_t);
template void launch_weinberg<float>(const Geom &, const LinkField<float> &, const ObsPlan &, double *, double *,
                                     cudaStream_t);

// ---------------------------------------------------------------------------
// Start fields, reunitarisation, layout conversion
// ---------------------------------------------------------------------------
template <typename T> __device__ __forceinline__ M3<T> to_t(const M3<double> &a) {
    M3<T> r;
#pragma unroll
    for (int k = 0; k < 9; k++) { r.e[k].re = (T)a.e[k].re; r.e[k].im = (T)a.e[k].im; }
    return r;
}
template <typename T> __device__ __forceinline__ M3<double> to_d(const M3<T> &a) {
    M3<double> r;
#pragma unroll
    for (int k = 0; k < 9; k++) { r.e[k].re = (double)a.e[k].re; r.e[k].im = (double)a.e[k].im; }
    return r;
}

// grid: x over Vh, y = mu*2 + parity
template <typename T>
__device__ __forceinline__ void haar_link(const Geom &g, const LinkField<T> &L, int mu, int p, int s, uint32_t k0,
                                          uint32_t k1, uint32_t stream_id) {
    const Site n = site_from_ps(g, p, s);
    const uint32_t link_id = (uint32_t)mu * (uint32_t)g.V + (uint32_t)n.lex;
    uint32_t w[20];
#pragma unroll
    for (int call = 0; call < 5; call++) {
        U4 c = {(uint32_t)call, link_id, 0xA11Au, stream_id};
        U4 o = philox4x32_10(c, k0, k1);
        w[4 * call] = o.x; w[4 * call + 1] = o.y; w[4 * call + 2] = o.z; w[4 * call + 3] = o.w;
    }
    M3<double> Z;
#pragma unroll
    for (int e = 0; e < 9; e++) {  // Box-Muller
        double u1 = ((double)w[2 * e] + 1.0) * 2.3283064365386963e-10;
        double u2 = (double)w[2 * e + 1] * 2.3283064365386963e-10;
        double rad = sqrt(-2.0 * log(u1));
        double sn, cs;
        sincospi(2.0 * u2, &sn, &cs);
        Z.e[e] = cx(rad * cs, rad * sn);
    }
    // Gram-Schmidt on columns (QR with positive real R diagonal -> Haar on U(3))
#pragma unroll
    for (int j = 0; j < 3; j++) {
#pragma unroll
        for (int pc = 0; pc < j; pc++) {
            Cx<double> d = cx(0.0, 0.0);
#pragma unroll
            for (int i = 0; i < 3; i++) d = cmac_cj(d, Z(i, pc), Z(i, j));
#pragma unroll
            for (int i = 0; i < 3; i++) Z(i, j) = Z(i, j) - d * Z(i, pc);
        }
        double nrm = 0.0;
#pragma unroll
        for (int i = 0; i < 3; i++) nrm += Z(i, j).re * Z(i, j).re + Z(i, j).im * Z(i, j).im;
        nrm = rsqrt(nrm);
#pragma unroll
        for (int i = 0; i < 3; i++) Z(i, j) = cx(Z(i, j).re * nrm, Z(i, j).im * nrm);
    }
    Cx<double> det = cx(0.0, 0.0);
#pragma unroll
    for (int pc = 0; pc < 3; pc++) {
        const int a = (pc + 1) % 3, b = (pc + 2) % 3;
        det = det + Z(0, pc) * (Z(1, a) * Z(2, b) - Z(1, b) * Z(2, a));
    }
    double sn, cs;
    sincos(-atan2(det.im, det.re) / 3.0, &sn, &cs);
    const Cx<double> f = cx(cs, sn);
#pragma unroll
    for (int e = 0; e < 9; e++) Z.e[e] = Z.e[e] * f;
    L.store(mu, p, s, to_t<T>(Z));
}
template <typename T>
__global__ void k_haar(Geom g, LinkField<T> L, uint32_t k0, uint32_t k1, uint32_t stream_id) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    haar_link(g, L, blockIdx.y >> 1, blockIdx.y & 1, s, k0, k1, stream_id);
}

// Random links near unity: each link is one RST proposal matrix (the
// reference's RST hot start, GLAC/system.cpp:205-210 with generateRST,
// su3matrixgenerator.h:170-196), drawn from the Philox stream with sweep
// counter 0xFFFFFFFF.
template <typename T>
__global__ void k_rst_start(Geom g, LinkField<T> L, double eps, uint32_t k0, uint32_t k1, uint32_t stream_id) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
    const Site n = site_from_ps(g, p, s);
    M3<double> X;
    double r;
    draw_proposal<double>(k0, k1, (uint32_t)mu * (uint32_t)g.V + (uint32_t)n.lex, 0xFFFFFFFFu, stream_id, 0, eps,
                          sqrt(1.0 - eps * eps), true, X, r);
    L.store(mu, p, s, to_t<T>(X));
}
template <typename T>
void launch_rst_start(const Geom &g, const LinkField<T> &L, double eps, uint64_t seed, uint32_t stream_id,
                      cudaStream_t st) {
    k_rst_start<T><<<dim3((g.Vh + 127) / 128, 8), 128, 0, st>>>(g, L, eps, (uint32_t)seed, (uint32_t)(seed >> 32),
                                                                stream_id);
}
template void launch_rst_start<double>(const Geom &, const LinkField<double> &, double, uint64_t, uint32_t,
                                       cudaStream_t);
template void launch_rst_start<float>(const Geom &, const LinkField<float> &, double, uint64_t, uint32_t,
                                      cudaStream_t);

template <typename T>
__global__ void k_cold(Geom g, LinkField<T> L) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    M3<T> I;
    set_identity(I);
    L.store(blockIdx.y >> 1, blockIdx.y & 1, s, I);
}

// Row Gram-Schmidt in FP64, third row = conj(row0 x row1).
__device__ __forceinline__ M3<double> reunit(M3<double> U) {
    double na = 0.0;
#pragma unroll
    for (int j = 0; j < 3; j++) na += U(0, j).re * U(0, j).re + U(0, j).im * U(0, j).im;
    na = rsqrt(na);
#pragma unroll
    for (int j = 0; j < 3; j++) U(0, j) = cx(U(0, j).re * na, U(0, j).im * na);
    Cx<double> d = cx(0.0, 0.0);
#pragma unroll
    for (int j = 0; j < 3; j++) d = cmac_cj(d, U(0, j), U(1, j));
#pragma unroll
    for (int j = 0; j < 3; j++) U(1, j) = U(1, j) - d * U(0, j);
    double nb = 0.0;
#pragma unroll
    for (int j = 0; j < 3; j++) nb += U(1, j).re * U(1, j).re + U(1, j).im * U(1, j).im;
    nb = rsqrt(nb);
#pragma unroll
    for (int j = 0; j < 3; j++) U(1, j) = cx(U(1, j).re * nb, U(1, j).im * nb);
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const int a = (j + 1) % 3, b = (j + 2) % 3;
        U(2, j) = conj(U(0, a) * U(1, b) - U(0, b) * U(1, a));
    }
    return U;
}

template <typename T>
__global__ void k_reunitarize(Geom g, LinkField<T> L) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
    L.store(mu, p, s, to_t<T>(reunit(to_d(L.load_rw(mu, p, s)))));
}

// AoS host layout [mu][lex][18] (FP64) <-> SoA. grid: x over V, y = mu.
template <typename T>
__global__ void k_aos_to_soa(Geom g, const double *aos, LinkField<T> L) {
    const int lex = blockIdx.x * blockDim.x + threadIdx.x;
    if (lex >= g.V) return;
    const int mu = blockIdx.y;
    const double2 *src = reinterpret_cast<const double2 *>(aos + ((size_t)mu * g.V + lex) * 18);
    M3<double> U;
#pragma unroll
    for (int k = 0; k < 9; k++) { double2 v = src[k]; U.e[k] = cx(v.x, v.y); }
    const int p = parity_of_lex(g, lex);
    L.store(mu, p, lex >> 1, to_t<T>(U));
}
template <typename T>
__global__ void k_soa_to_aos(Geom g, LinkField<T> L, double *aos) {
    const int lex = blockIdx.x * blockDim.x + threadIdx.x;
    if (lex >= g.V) return;
    const int mu = blockIdx.y;
    const int p = parity_of_lex(g, lex);
    const M3<double> U = to_d(L.load_rw(mu, p, lex >> 1));
    double2 *dst = reinterpret_cast<double2 *>(aos + ((size_t)mu * g.V + lex) * 18);
#pragma unroll
    for (int k = 0; k < 9; k++) dst[k] = make_double2(U.e[k].re, U.e[k].im);
}
template <typename T>
__global__ void k_copy_field(Geom g, LinkField<T> src, LinkField<T> dst) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
    dst.store(mu, p, s, src.load_rw(mu, p, s));
}

template <typename T>
void launch_haar(const Geom &g, const LinkField<T> &L, uint64_t seed, uint32_t stream_id, cudaStream_t st) {
    k_haar<T><<<dim3((g.Vh + 127) / 128, 8), 128, 0, st>>>(g, L, (uint32_t)seed, (uint32_t)(seed >> 32), stream_id);
}
template <typename T>
void launch_cold(const Geom &g, const LinkField<T> &L, cudaStream_t st) {
    k_cold<T><<<dim3((g.Vh + 255) / 256, 8), 256, 0, st>>>(g, L);
}
template <typename T>
void launch_reunitarize(const Geom &g, const LinkField<T> &L, cudaStream_t st) {
    k_reunitarize<T><<<dim3((g.Vh + 127) / 128, 8), 128, 0, st>>>(g, L);
}
template <typename T>
void launch_aos_to_soa(const Geom &g, const double *aos, const LinkField<T> &L, cudaStream_t st) {
    k_aos_to_soa<T><<<dim3((g.V + 127) / 128, 4), 128, 0, st>>>(g, aos, L);
}
template <typename T>
void launch_soa_to_aos(const Geom &g, const LinkField<T> &L, double *aos, cudaStream_t st) {
    k_soa_to_aos<T><<<dim3((g.V + 127) / 128, 4), 128, 0, st>>>(g, L, aos);
}
template <typename T>
void launch_copy_field(const Geom &g, const LinkField<T> &src, const LinkField<T> &dst, cudaStream_t st) {
    k_copy_field<T><<<dim3((g.Vh + 255) / 256, 8), 256, 0, st>>>(g, src, dst);
}

// ---------------------------------------------------------------------------
// Test exports
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_staples_aos(Geom g, LinkField<T> L, double *out, int force) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
    const Site n = site_from_ps(g, p, s);
    M3<T> A = staple(L, g, n, p, mu);
    if (force) A = ah_to_m3(project_ah(mul(L.load(mu, p, s), A)));
    const M3<double> Ad = to_d(A);
    double2 *dst = reinterpret_cast<double2 *>(out + ((size_t)mu * g.V + n.lex) * 18);
#pragma unroll
    for (int k = 0; k < 9; k++) dst[k] = make_double2(Ad.e[k].re, Ad.e[k].im);
}
template <typename T>
void launch_staples_aos(const Geom &g, const LinkField<T> &L, double *out, cudaStream_t st) {
    k_staples_aos<T><<<dim3((g.Vh + 127) / 128, 8), 128, 0, st>>>(g, L, out, 0);
}
template <typename T>
void launch_force_aos(const Geom &g, const LinkField<T> &L, double *out, cudaStream_t st) {
    k_staples_aos<T><<<dim3((g.Vh + 127) / 128, 8), 128, 0, st>>>(g, L, out, 1);
}

template <typename T>
__device__ __forceinline__ M3<T> load_aos(const double *p) {
    M3<T> U;
#pragma unroll
    for (int k = 0; k < 9; k++) U.e[k] = cx((T)p[2 * k], (T)p[2 * k + 1]);
    return U;
}
template <typename T>
__device__ __forceinline__ void store_aos(double *p, const M3<T> &U) {
#pragma unroll
    for (int k = 0; k < 9; k++) { p[2 * k] = (double)U.e[k].re; p[2 * k + 1] = (double)U.e[k].im; }
}

// exp of n anti-Hermitian traceless matrices given as full 18-double matrices;
// the 8 independent reals are taken as the flow kernels store them.
template <typename T>
__global__ void k_exp_batch(int kind, const double *in, double *out, long n) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const M3<T> M = load_aos<T>(in + 18 * i);
    AH8<T> Z;
    Z.a = M(0, 0).im; Z.d = M(1, 1).im;
    Z.b = M(0, 1); Z.c = M(0, 2); Z.e = M(1, 2);
    store_aos(out + 18 * i, expm<T>(kind, Z));
}
template <typename T>
void launch_exp_batch(int kind, const double *in, double *out, long n, cudaStream_t st) {
    k_exp_batch<T><<<(unsigned)((n + 127) / 128), 128, 0, st>>>(kind, in, out, n);
}

template <typename T>
__global__ void k_accept_fed(T mfac, long nlinks, int nhits, double *U, const double *A, const double *X,
                             const double *r, unsigned char *accept) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nlinks) return;
    M3<T> u = load_aos<T>(U + 18 * k);
    const M3<T> a = load_aos<T>(A + 18 * k);
    for (int h = 0; h < nhits; h++) {
        const M3<T> Up = mul(load_aos<T>(X + 18 * (k * nhits + h)), u);
        const bool acc = accept_weight<T>(delta_s(u, Up, a, mfac)) > r[k * nhits + h];
        accept[k * nhits + h] = acc ? 1 : 0;
        if (acc) u = Up;
    }
    store_aos(U + 18 * k, u);
}
template <typename T>
void launch_accept_fed(double beta, long nlinks, int nhits, double *U, const double *A, const double *X,
                       const double *r, unsigned char *accept, cudaStream_t st) {
    k_accept_fed<T><<<(unsigned)((nlinks + 127) / 128), 128, 0, st>>>((T)(-beta / 3.0), nlinks, nhits, U, A, X, r,
                                                                       accept);
}

template <typename T>
__global__ void k_delta_s(T mfac, long n, const double *U, const double *Up, const double *A, double *out) {
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    out[k] = (double)delta_s(load_aos<T>(U + 18 * k), load_aos<T>(Up + 18 * k), load_aos<T>(A + 18 * k), mfac);
}
template <typename T>
void launch_delta_s(double beta, long n, const double *U, const double *Up, const double *A, double *out,
                    cudaStream_t st) {
    k_delta_s<T><<<(unsigned)((n + 127) / 128), 128, 0, st>>>((T)(-beta / 3.0), n, U, Up, A, out);
}

// max over links of |U U^+ - 1| (entrywise), FP64 result in out[0] via atomicMax on the bit pattern.
template <typename T>
__global__ void k_unitarity(Geom g, LinkField<T> L, unsigned long long *out) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
    const M3<double> U = to_d(L.load_rw(mu, p, s));
    const M3<double> P = mul_nd(U, U);
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double re = P(i, j).re - (i == j ? 1.0 : 0.0);
            m = fmax(m, fmax(fabs(re), fabs(P(i, j).im)));
        }
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
}
template <typename T>
void launch_max_unitarity_dev(const Geom &g, const LinkField<T> &L, double *out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, sizeof(double), st);
    k_unitarity<T><<<dim3((g.Vh + 127) / 128, 8), 128, 0, st>>>(g, L, reinterpret_cast<unsigned long long *>(out));
}

#define GLAC_INST(T)                                                                                             \
    template void launch_haar<T>(const Geom &, const LinkField<T> &, uint64_t, uint32_t, cudaStream_t);          \
    template void launch_cold<T>(const Geom &, const LinkField<T> &, cudaStream_t);                              \
    template void launch_reunitarize<T>(const Geom &, const LinkField<T> &, cudaStream_t);                       \
    template void launch_aos_to_soa<T>(const Geom &, const double *, const LinkField<T> &, cudaStream_t);        \
    template void launch_soa_to_aos<T>(const Geom &, const LinkField<T> &, double *, cudaStream_t);              \
    template void launch_copy_field<T>(const Geom &, const LinkField<T> &, const LinkField<T> &, cudaStream_t);  \
    template void launch_staples_aos<T>(const Geom &, const LinkField<T> &, double *, cudaStream_t);             \
    template void launch_force_aos<T>(const Geom &, const LinkField<T> &, double *, cudaStream_t);               \
    template void launch_exp_batch<T>(int, const double *, double *, long, cudaStream_t);                        \
    template void launch_accept_fed<T>(double, long, int, double *, const double *, const double *,              \
                                       const double *, unsigned char *, cudaStream_t);                           \
    template void launch_max_unitarity_dev<T>(const Geom &, const LinkField<T> &, double *, cudaStream_t);      \
    template void launch_delta_s<T>(double, long, const double *, const double *, const double *, double *,     \
                                    cudaStream_t);
GLAC_INST(double)
GLAC_INST(float)
#undef GLAC_INST

// ---------------------------------------------------------------------------
// Batched ensemble (see LatSlot in kernels.cuh)
// ---------------------------------------------------------------------------
// Lattice of block b: the last i with start[i] <= b.
__device__ __forceinline__ int slot_of(const int *__restrict__ start, int M, int b) {
    int lo = 0, hi = M;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(start + mid) <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}

ObsPlan make_obs_plan_capped(const Geom &g, int max_threads) {
    const int half_slice = g.N[0] * g.N[1] * g.N[2] / 2;
    int best = -1, best_score = 1 << 30;
    for (int B = 1; B <= max_threads && B <= half_slice; B++) {
        if (half_slice % B) continue;
        const int score = (B % 32 == 0 ? 0 : 100000) + std::abs(B - max_threads);
        if (score < best_score) { best_score = score; best = B; }
    }
    ObsPlan pl;
    pl.Bv = best;
    pl.B = (best + 31) / 32 * 32;
    pl.nb = half_slice / best;
    pl.nblocks = g.N[3] * 2 * pl.nb;
    return pl;
}

int ens_blocks(const Geom &g, const ObsPlan &plan, int phase) {
    switch (phase) {
    case ENS_METRO: return (g.Vh + 127) / 128;
    case ENS_FLOW0: return 8 * ((g.Vh + 127) / 128);
    case ENS_FLOW1: return (g.Vh + 15) / 16;
    default: return plan.nblocks;
    }
}

// grid (sum of ENS_METRO blocks, 8 planes)
template <typename T>
__global__ void __launch_bounds__(128) kb_haar(const LatSlot<T> *__restrict__ slots, const int *__restrict__ start,
                                               int M, uint32_t k0, uint32_t k1) {
    const int i = slot_of(start, M, blockIdx.x);
    const LatSlot<T> &S = slots[i];
    const int s = (blockIdx.x - __ldg(start + i)) * 128 + threadIdx.x;
    if (s >= S.g.Vh) return;
    haar_link(S.g, S.f[0], blockIdx.y >> 1, blockIdx.y & 1, s, k0, k1, S.stream);
}
template <typename T>
void launch_ens_haar(const LatSlot<T> *slots, const int *start, int nblocks, int M, uint64_t seed, cudaStream_t st) {
    kb_haar<T><<<dim3(nblocks, 8), 128, 0, st>>>(slots, start, M, (uint32_t)seed, (uint32_t)(seed >> 32));
}

#define GLAC_ENS_METRO_KERNEL(NAME, ATTR)                                                                    \
    template <typename T>                                                                                  \
    __global__ void ATTR NAME(const LatSlot<T> *__restrict__ slots, const int *__restrict__ start, int M,    \
                              int fsel, int mu, int p, T eps, T sq1me, int nhits, uint32_t k0, uint32_t k1,  \
                              const uint32_t *__restrict__ sweep_base, uint32_t sweep_off, bool flips) {     \
        const int i = slot_of(start, M, blockIdx.x);                                                       \
        const LatSlot<T> &S = slots[i];                                                                    \
        Proposal P;                                                                                        \
        P.flips = flips;                                                                                   \
        metropolis_body<T, false>(S.g, S.f[fsel], mu, p, (T)(-S.beta / 3.f), eps, sq1me, nhits, k0, k1,     \
                                  __ldg(sweep_base) + sweep_off, S.stream, S.acc, P, S.beta,               \
                                  blockIdx.x - __ldg(start + i));                                          \
    }
GLAC_ENS_METRO_KERNEL(kb_metropolis, __launch_bounds__(128))
GLAC_ENS_METRO_KERNEL(kb_metropolis_r128, __maxnreg__(128))
GLAC_ENS_METRO_KERNEL(kb_metropolis_r96, __maxnreg__(96))
GLAC_ENS_METRO_KERNEL(kb_metropolis_r80, __maxnreg__(80))
#undef GLAC_ENS_METRO_KERNEL

template <typename T>
void launch_ens_metropolis(const LatSlot<T> *slots, const int *start, int nblocks, int M, int fsel, int mu, int p,
                           double eps, int nhits, uint64_t seed, const uint32_t *sweep_base, uint32_t sweep_off,
                           bool flips, int variant, cudaStream_t st) {
    const T e = (T)eps, sq = (T)sqrt(1.0 - eps * eps);
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    switch (variant_regs(FAM_METRO, sizeof(T) == 4, variant)) {
    case 128: kb_metropolis_r128<T><<<nblocks, 128, 0, st>>>(slots, start, M, fsel, mu, p, e, sq, nhits, k0, k1, sweep_base, sweep_off, flips); break;
    case 96: kb_metropolis_r96<T><<<nblocks, 128, 0, st>>>(slots, start, M, fsel, mu, p, e, sq, nhits, k0, k1, sweep_base, sweep_off, flips); break;
    case 80: kb_metropolis_r80<T><<<nblocks, 128, 0, st>>>(slots, start, M, fsel, mu, p, e, sq, nhits, k0, k1, sweep_base, sweep_off, flips); break;
    default: kb_metropolis<T><<<nblocks, 128, 0, st>>>(slots, start, M, fsel, mu, p, e, sq, nhits, k0, k1, sweep_base, sweep_off, flips); break;
    }
}

#define GLAC_ENS_FLOW_KERNEL(NAME, ATTR)                                                                     \
    template <typename T, int STAGE, int SHAPE>                                                            \
    __global__ void ATTR NAME(const LatSlot<T> *__restrict__ slots, const int *__restrict__ start, int M,    \
                              int src, int dst, T alpha, T beta) {                                         \
        const int i = slot_of(start, M, blockIdx.x);                                                       \
        const LatSlot<T> &S = slots[i];                                                                    \
        flow_stage_body<T, EXP_MORNINGSTAR, STAGE, SHAPE>(S.g, S.f[src], S.f[dst], S.z, alpha, beta,         \
                                                          blockIdx.x - __ldg(start + i));                  \
    }
GLAC_ENS_FLOW_KERNEL(kb_flow_stage, __launch_bounds__(128))
GLAC_ENS_FLOW_KERNEL(kb_flow_stage_r80, __maxnreg__(80))
GLAC_ENS_FLOW_KERNEL(kb_flow_stage_r96, __maxnreg__(96))
GLAC_ENS_FLOW_KERNEL(kb_flow_stage_r128, __maxnreg__(128))
#undef GLAC_ENS_FLOW_KERNEL

template <typename T, int STAGE, int SHAPE>
static void ens_flow_dispatch_caps(int regs, int nblocks, cudaStream_t st, const LatSlot<T> *slots,
                                   const int *start, int M, int src, int dst, T a, T b) {
    switch (regs) {
    case 128: kb_flow_stage_r128<T, STAGE, SHAPE><<<nblocks, 128, 0, st>>>(slots, start, M, src, dst, a, b); break;
    case 96:
        if constexpr (sizeof(T) == 4) {
            kb_flow_stage_r96<T, STAGE, SHAPE><<<nblocks, 128, 0, st>>>(slots, start, M, src, dst, a, b);
            break;
        }
        [[fallthrough]];
    case 80:
        if constexpr (sizeof(T) == 4) {
            kb_flow_stage_r80<T, STAGE, SHAPE><<<nblocks, 128, 0, st>>>(slots, start, M, src, dst, a, b);
            break;
        }
        [[fallthrough]];
    default: kb_flow_stage<T, STAGE, SHAPE><<<nblocks, 128, 0, st>>>(slots, start, M, src, dst, a, b); break;
    }
}

template <typename T, int STAGE>
static void ens_flow_dispatch(int regs, int shape, int nblocks, cudaStream_t st, const LatSlot<T> *slots,
                              const int *start, int M, int src, int dst, T a, T b) {
    if (shape == 1) {
        kb_flow_stage<T, STAGE, 1><<<nblocks, 128, 0, st>>>(slots, start, M, src, dst, a, b);
        return;
    }
    // shape 2 has shape 0's block table (ens_blocks, ENS_FLOW0); only the chunk order differs
    if (shape == 2) ens_flow_dispatch_caps<T, STAGE, 2>(regs, nblocks, st, slots, start, M, src, dst, a, b);
    else ens_flow_dispatch_caps<T, STAGE, 0>(regs, nblocks, st, slots, start, M, src, dst, a, b);
}

// nblocks: the table of the variant's shape (ENS_FLOW0 or ENS_FLOW1)
template <typename T>
void launch_ens_flow_stage(const LatSlot<T> *slots, const int *start, int nblocks, int M, int src, int dst, int stage,
                           double alpha, double beta, int variant, cudaStream_t st) {
    const bool fp32 = sizeof(T) == 4;
    const int regs = variant_regs(FAM_FLOW, fp32, variant), shape = variant_shape(FAM_FLOW, fp32, variant);
    const T a = (T)alpha, b = (T)beta;
    if (stage == 0) ens_flow_dispatch<T, 0>(regs, shape, nblocks, st, slots, start, M, src, dst, a, b);
    else if (stage == 1) ens_flow_dispatch<T, 1>(regs, shape, nblocks, st, slots, start, M, src, dst, a, b);
    else ens_flow_dispatch<T, 2>(regs, shape, nblocks, st, slots, start, M, src, dst, a, b);
}

#define GLAC_ENS_OBS_KERNEL(NAME, ATTR)                                                                      \
    template <typename T>                                                                                  \
    __global__ void ATTR NAME(const LatSlot<T> *__restrict__ slots, const int *__restrict__ start, int M,    \
                              int fsel) {                                                                  \
        const int i = slot_of(start, M, blockIdx.x);                                                       \
        const LatSlot<T> &S = slots[i];                                                                    \
        observables_body<T>(S.g, S.f[fsel], S.nb, S.Bv, S.partial, blockIdx.x - __ldg(start + i));          \
    }
GLAC_ENS_OBS_KERNEL(kb_observables, __launch_bounds__(128))
GLAC_ENS_OBS_KERNEL(kb_observables_r128, __maxnreg__(128))
GLAC_ENS_OBS_KERNEL(kb_observables_r168, __maxnreg__(168))
#undef GLAC_ENS_OBS_KERNEL
template <typename T>
__global__ void kb_obs_finalize(const LatSlot<T> *__restrict__ slots, int meas) {
    const LatSlot<T> &S = slots[blockIdx.x];
    obs_finalize_body(S.g.N[3], S.nb, S.g.V, S.partial, S.obs + (size_t)meas * (3 + S.g.N[3]));
}
template <typename T>
void launch_ens_observables(const LatSlot<T> *slots, const int *start, int nblocks, int M, int fsel, int meas,
                            int variant, cudaStream_t st) {
    switch (variant_regs(FAM_OBS, sizeof(T) == 4, variant)) {
    case 128: kb_observables_r128<T><<<nblocks, 128, 0, st>>>(slots, start, M, fsel); break;
    case 168:
        if constexpr (sizeof(T) == 4) {
            kb_observables_r168<T><<<nblocks, 128, 0, st>>>(slots, start, M, fsel);
            break;
        }
        [[fallthrough]];  // no 168-register FP64 variant
    default: kb_observables<T><<<nblocks, 128, 0, st>>>(slots, start, M, fsel); break;
    }
    kb_obs_finalize<T><<<M, 1024, 0, st>>>(slots, meas);
}

#define GLAC_ENS_MEAS_KERNEL(NAME, ATTR)                                                                     \
    template <typename T>                                                                                  \
    __global__ void ATTR NAME(const LatSlot<T> *__restrict__ slots, const int *__restrict__ start, int M,    \
                              int src, int dst, T alpha) {                                                 \
        const int i = slot_of(start, M, blockIdx.x);                                                       \
        const LatSlot<T> &S = slots[i];                                                                    \
        flow_stage0_meas_body<T, EXP_MORNINGSTAR>(S.g, S.f[src], S.f[dst], S.z, S.cp, alpha,                \
                                                  blockIdx.x - __ldg(start + i));                          \
    }
GLAC_ENS_MEAS_KERNEL(kb_flow_stage0_meas, __launch_bounds__(128))
GLAC_ENS_MEAS_KERNEL(kb_flow_stage0_meas_r128, __maxnreg__(128))
#undef GLAC_ENS_MEAS_KERNEL

template <typename T>
void launch_ens_flow_stage0_meas(const LatSlot<T> *slots, const int *start, int nblocks, int M, int src, int dst,
                                 double alpha, int regs, cudaStream_t st) {
    if (regs == 128) kb_flow_stage0_meas_r128<T><<<nblocks, 128, 0, st>>>(slots, start, M, src, dst, (T)alpha);
    else kb_flow_stage0_meas<T><<<nblocks, 128, 0, st>>>(slots, start, M, src, dst, (T)alpha);
}

template <typename T>
__global__ void __launch_bounds__(128) kb_obs_combine(const LatSlot<T> *__restrict__ slots,
                                                      const int *__restrict__ start, int M) {
    const int i = slot_of(start, M, blockIdx.x);
    const LatSlot<T> &S = slots[i];
    const int b = blockIdx.x - __ldg(start + i);
    const int nb = S.nb, Bv = S.Bv;
    const int t = b / (2 * nb), p = (b / nb) & 1, j = b % nb;
    const int half_slice = S.g.Vh / S.g.N[3];
    const bool valid = (int)threadIdx.x < Bv;
    const int s = t * half_slice + j * Bv + (valid ? (int)threadIdx.x : 0);
    double plaq = 0.0, en = 0.0, qt = 0.0;
    if (valid) combine_site(S.g, S.cp, p, s, plaq, en, qt);
    obs_block_reduce(plaq, en, qt, S.partial, b);
}
template <typename T>
void launch_ens_obs_combine(const LatSlot<T> *slots, const int *start, int nblocks, int M, int meas,
                            cudaStream_t st) {
    kb_obs_combine<T><<<nblocks, 128, 0, st>>>(slots, start, M);
    kb_obs_finalize<T><<<M, 1024, 0, st>>>(slots, meas);
}

// ---------------------------------------------------------------------------
// The whole ensemble schedule in one persistent launch (FP32): every block of
// a cooperative grid (all co-resident) walks the virtual blocks of each phase
// in turn -- the 8 Metropolis sub-sweeps of every sweep, the chain -> flow copy,
// and per flow step stage 0 with the measurement's parts, their combination,
// the per-lattice reduction, stages 1 and 2 -- with a grid-wide barrier between
// phases.  The barrier waits at most wait_ns of the GPU's global timer; when a
// wait runs out the barrier records the error, every block leaves at its next
// barrier, and the host reports a timeout (the field is then undefined).
// test_skip_block0: block 0 leaves at the first barrier without arriving, so
// the others' waits run out (the failure path, without a fault or a hang).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t gtimer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// false: a wait ran out here or elsewhere (the caller leaves)
__device__ bool grid_barrier(GridBarrier *b, uint64_t wait_ns) {
    __shared__ int ok_sh;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned int *vgen = &b->gen;
        volatile int *verr = &b->err;
        const unsigned int gen = *vgen;
        __threadfence();
        if (atomicAdd(&b->count, 1u) + 1u == gridDim.x) {
            atomicExch(&b->count, 0u);
            __threadfence();
            atomicAdd(&b->gen, 1u);
        } else {
            // bounded by the global timer, and by a count of tries as a second
            // bound (a try reads L2 and sleeps, well over 16 ns, so wait_ns / 16
            // tries outlast wait_ns)
            const uint64_t t0 = gtimer_ns();
            for (uint64_t it = 0; *vgen == gen; it++) {
                if (*verr) { ok = 0; break; }
                if (gtimer_ns() - t0 > wait_ns || it > (wait_ns >> 4)) {
                    atomicExch(&b->err, 1);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        if (*verr) ok = 0;
        ok_sh = ok;
    }
    __syncthreads();
    return ok_sh != 0;
}

template <typename T>
__global__ void __launch_bounds__(128, 4) kb_persistent(const LatSlot<T> *__restrict__ slots, EnsSchedule sc,
                                                        GridBarrier *bar) {
    const int M = sc.M;
    const uint32_t sweep0 = *sc.sweep_base;  // advanced at the end, after the last barrier
    Proposal P;
    P.flips = sc.flips;
    bool ok = true;
    if (sc.test_skip_block0 && blockIdx.x == 0) return;
    // Metropolis: 8 (mu, parity) sub-sweeps per sweep on the chain fields
    for (int i = 0; i < sc.n_sweeps && ok; i++)
        for (int k = 0; k < 8 && ok; k++) {
            for (int vb = blockIdx.x; vb < sc.nb_metro; vb += gridDim.x) {
                const int l = slot_of(sc.start_metro, M, vb);
                const LatSlot<T> &S = slots[l];
                metropolis_body<T, false>(S.g, S.f[0], k >> 1, k & 1, (T)(-S.beta / 3.f), (T)sc.eps, (T)sc.sq1me,
                                          sc.nhits, sc.k0, sc.k1, sweep0 + (uint32_t)i, S.stream, S.acc, P, S.beta,
                                          vb - __ldg(sc.start_metro + l));
            }
            ok = grid_barrier(bar, sc.wait_ns);
        }
    if (sc.n_steps < 0) {
        if (ok && blockIdx.x == 0 && threadIdx.x == 0) *sc.sweep_base = sweep0 + (uint32_t)sc.n_sweeps;
        return;
    }
    // the flow fields from the chains (one allocation per role, equal offsets)
    if (ok) {
        const uint4 *src = reinterpret_cast<const uint4 *>(sc.chain);
        uint4 *dst = reinterpret_cast<uint4 *>(sc.flow);
        for (size_t w = (size_t)blockIdx.x * blockDim.x + threadIdx.x; w < sc.field_words;
             w += (size_t)gridDim.x * blockDim.x)
            dst[w] = src[w];
        ok = grid_barrier(bar, sc.wait_ns);
    }
    int cur = 1;
    for (int step = 0; step < sc.n_steps && ok; step++) {
        // stage 0 with the parts of the measurement of the field before the step
        for (int vb = blockIdx.x; vb < sc.nb_flow0 && ok; vb += gridDim.x) {
            const int l = slot_of(sc.start_flow0, M, vb);
            const LatSlot<T> &S = slots[l];
            flow_stage0_meas_body<T, EXP_MORNINGSTAR>(S.g, S.f[cur], S.f[3 - cur], S.z, S.cp, (T)sc.alpha[0],
                                                      vb - __ldg(sc.start_flow0 + l));
        }
        if (ok) ok = grid_barrier(bar, sc.wait_ns);
        for (int vb = blockIdx.x; vb < sc.nb_obs && ok; vb += gridDim.x) {
            const int l = slot_of(sc.start_obs, M, vb);
            const LatSlot<T> &S = slots[l];
            const int b = vb - __ldg(sc.start_obs + l);
            const int t = b / (2 * S.nb), p = (b / S.nb) & 1, j = b % S.nb;
            const int half_slice = S.g.Vh / S.g.N[3];
            const bool valid = (int)threadIdx.x < S.Bv;
            const int s = t * half_slice + j * S.Bv + (valid ? (int)threadIdx.x : 0);
            double plaq = 0.0, en = 0.0, qt = 0.0;
            if (valid) combine_site(S.g, S.cp, p, s, plaq, en, qt);
            obs_block_reduce(plaq, en, qt, S.partial, b);
        }
        if (ok) ok = grid_barrier(bar, sc.wait_ns);
        for (int l = blockIdx.x; l < M && ok; l += gridDim.x) {
            const LatSlot<T> &S = slots[l];
            obs_finalize_body(S.g.N[3], S.nb, S.g.V, S.partial, S.obs + (size_t)step * (3 + S.g.N[3]));
        }
        // (the finalize reads the partials the combine wrote; the next phases do not touch them)
        for (int st = 1; st < 3 && ok; st++) {
            const int src = st == 1 ? 3 - cur : cur, dstf = st == 1 ? cur : 3 - cur;
            for (int vb = blockIdx.x; vb < sc.nb_flow0; vb += gridDim.x) {
                const int l = slot_of(sc.start_flow0, M, vb);
                const LatSlot<T> &S = slots[l];
                if (st == 1)
                    flow_stage_body<T, EXP_MORNINGSTAR, 1, 0>(S.g, S.f[src], S.f[dstf], S.z, (T)sc.alpha[1],
                                                              (T)sc.beta[1], vb - __ldg(sc.start_flow0 + l));
                else
                    flow_stage_body<T, EXP_MORNINGSTAR, 2, 0>(S.g, S.f[src], S.f[dstf], S.z, (T)sc.alpha[2],
                                                              (T)sc.beta[2], vb - __ldg(sc.start_flow0 + l));
            }
            ok = grid_barrier(bar, sc.wait_ns);
        }
        cur = 3 - cur;  // three stages: the field ends in the other buffer
    }
    // the last measurement as a pass of its own
    if (ok) {
        for (int vb = blockIdx.x; vb < sc.nb_obs; vb += gridDim.x) {
            const int l = slot_of(sc.start_obs, M, vb);
            const LatSlot<T> &S = slots[l];
            observables_body<T>(S.g, S.f[cur], S.nb, S.Bv, S.partial, vb - __ldg(sc.start_obs + l));
        }
        ok = grid_barrier(bar, sc.wait_ns);
    }
    if (ok) {
        for (int l = blockIdx.x; l < M; l += gridDim.x) {
            const LatSlot<T> &S = slots[l];
            obs_finalize_body(S.g.N[3], S.nb, S.g.V, S.partial, S.obs + (size_t)sc.n_steps * (3 + S.g.N[3]));
        }
        ok = grid_barrier(bar, sc.wait_ns);
    }
    if (ok && blockIdx.x == 0 && threadIdx.x == 0) *sc.sweep_base = sweep0 + (uint32_t)sc.n_sweeps;
}

int persistent_blocks_per_sm() {
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kb_persistent<float>, 128, 0) != cudaSuccess) return 0;
    return nb;
}

cudaError_t launch_ens_persistent(const LatSlot<float> *slots, const EnsSchedule &sc, GridBarrier *bar, int grid,
                                  cudaStream_t st) {
    void *args[] = {(void *)&slots, (void *)&sc, (void *)&bar};
    return cudaLaunchCooperativeKernel((const void *)kb_persistent<float>, dim3(grid), dim3(128), args, 0, st);
}

__global__ void k_advance(uint32_t *counter, uint32_t by) { counter[0] += by; }
void launch_advance(uint32_t *counter, uint32_t by, cudaStream_t st) { k_advance<<<1, 1, 0, st>>>(counter, by); }

#define GLAC_ENS_INST(T)                                                                                      \
    template void launch_ens_haar<T>(const LatSlot<T> *, const int *, int, int, uint64_t, cudaStream_t);      \
    template void launch_ens_metropolis<T>(const LatSlot<T> *, const int *, int, int, int, int, int, double,  \
                                           int, uint64_t, const uint32_t *, uint32_t, bool, int, cudaStream_t); \
    template void launch_ens_flow_stage<T>(const LatSlot<T> *, const int *, int, int, int, int, int, double,  \
                                           double, int, cudaStream_t);                                        \
    template void launch_ens_observables<T>(const LatSlot<T> *, const int *, int, int, int, int, int,         \
                                            cudaStream_t);                                                    \
    template void launch_ens_flow_stage0_meas<T>(const LatSlot<T> *, const int *, int, int, int, int, double, \
                                                 int, cudaStream_t);                                          \
    template void launch_ens_obs_combine<T>(const LatSlot<T> *, const int *, int, int, int, cudaStream_t);
GLAC_ENS_INST(double)
GLAC_ENS_INST(float)
#undef GLAC_ENS_INST

}  // namespace glac
