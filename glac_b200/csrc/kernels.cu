// Hot-path kernels for sm_100a: fused flow stage, checkerboard Metropolis,
// fused clover observables with deterministic FP64 reductions, plus field
// initialisation, reunitarisation and layout conversion.
#include "kernels.cuh"

#include <algorithm>
#include <cstdlib>
#include <stdexcept>

namespace glac {

// Minimum resident blocks per SM requested from ptxas (caps registers per thread).
template <typename R> struct MinBlocks { static const int flow = 2, metro = 2, obs = 1; };
template <> struct MinBlocks<double> { static const int flow = 3, metro = 3, obs = 1; };

// lanes of a real: the physical sites a thread carries
__device__ __forceinline__ double lane0(double v) { return v; }
__device__ __forceinline__ double lane1(double) { return 0.0; }
__device__ __forceinline__ double lane0(f32x2 v) { return (double)v.v.x; }
__device__ __forceinline__ double lane1(f32x2 v) { return (double)v.v.y; }
__device__ __forceinline__ double lanesum(double v) { return v; }
__device__ __forceinline__ double lanesum(f32x2 v) { return (double)v.v.x + (double)v.v.y; }

template <typename R> GLAC_HD R real_of(double v);
template <> GLAC_HD double real_of<double>(double v) { return v; }
template <> GLAC_HD f32x2 real_of<f32x2>(double v) { return f32x2((float)v); }

// ---------------------------------------------------------------------------
// Exponentials over R (Morningstar-Peardon by default; see expm.cuh)
// ---------------------------------------------------------------------------
__device__ __forceinline__ M3<f32x2> join_lanes(const M3<float> &a, const M3<float> &b) {
    M3<f32x2> r;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        r.e[k].re = f32x2(a.e[k].re, b.e[k].re);
        r.e[k].im = f32x2(a.e[k].im, b.e[k].im);
    }
    return r;
}
__device__ __forceinline__ AH8<float> lane_of(const AH8<f32x2> &Z, int lane) {
    AH8<float> r;
    r.a = lane ? Z.a.v.y : Z.a.v.x;
    r.d = lane ? Z.d.v.y : Z.d.v.x;
    r.b = cx(lane ? Z.b.re.v.y : Z.b.re.v.x, lane ? Z.b.im.v.y : Z.b.im.v.x);
    r.c = cx(lane ? Z.c.re.v.y : Z.c.re.v.x, lane ? Z.c.im.v.y : Z.c.im.v.x);
    r.e = cx(lane ? Z.e.re.v.y : Z.e.re.v.x, lane ? Z.e.im.v.y : Z.e.im.v.x);
    return r;
}

template <typename R, int KIND> struct Expm;
template <int KIND> struct Expm<double, KIND> {
    static __device__ __forceinline__ M3<double> run(const AH8<double> &Z) { return expm<double>(KIND, Z); }
};
template <int KIND> struct Expm<f32x2, KIND> {
    static __device__ __forceinline__ M3<f32x2> run(const AH8<f32x2> &Z) {
        if (KIND == EXP_MORNINGSTAR) return expm_morningstar_pair(Z);
        // alternates: per lane in scalar FP32
        return join_lanes(expm<float>(KIND, lane_of(Z, 0)), expm<float>(KIND, lane_of(Z, 1)));
    }
};

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
template <typename R, int KIND, int STAGE>
__global__ void __launch_bounds__(128, MinBlocks<R>::flow)
    k_flow_stage(Geom g, LinkField<R> in, LinkField<R> out, ForceField<R> zf, R alpha, R beta) {
    const int plane = blockIdx.x & 7;
    const int s = (blockIdx.x >> 3) * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    const int mu = plane >> 1, p = plane & 1;
    const Site n = site_from_ps(g, p, s);
    const M3<R> A = staple(in, g, n, p, mu);
    const M3<R> U = in.load(mu, p, s);
    const AH8<R> Z = project_ah(mul(U, A));
    AH8<R> M;
    if (STAGE == 0) {
        M = ah_scale(alpha, Z);
        zf.store(mu, p, s, Z);
    } else {
        const AH8<R> W = zf.load(mu, p, s);
        M = ah_axpby(alpha, Z, beta, W);
        if (STAGE == 1) zf.store(mu, p, s, M);
    }
    out.store(mu, p, s, mul(Expm<R, KIND>::run(M), U));
}

template <typename R>
void launch_flow_stage(const Geom &g, const LinkField<R> &in, const LinkField<R> &out, const ForceField<R> &zf,
                       int stage, int kind, double alpha, double beta, cudaStream_t st) {
    const dim3 grid(8 * ((g.Vh + 127) / 128));
    const R a = real_of<R>(alpha), b = real_of<R>(beta);
#define GLAC_FLOW_CASE(K, S) \
    if (kind == K && stage == S) { k_flow_stage<R, K, S><<<grid, 128, 0, st>>>(g, in, out, zf, a, b); return; }
    GLAC_FLOW_CASE(0, 0) GLAC_FLOW_CASE(0, 1) GLAC_FLOW_CASE(0, 2)
    GLAC_FLOW_CASE(1, 0) GLAC_FLOW_CASE(1, 1) GLAC_FLOW_CASE(1, 2)
    GLAC_FLOW_CASE(2, 0) GLAC_FLOW_CASE(2, 1) GLAC_FLOW_CASE(2, 2)
    GLAC_FLOW_CASE(3, 0) GLAC_FLOW_CASE(3, 1) GLAC_FLOW_CASE(3, 2)
#undef GLAC_FLOW_CASE
    throw std::invalid_argument("bad flow stage or exp kind");
}

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
// mu V + lex, sweep, stream} (V, lex of the physical lattice): words 0-5 carry
// twelve 16-bit uniforms (low half first) for R, S, T; words 6-7 the 53-bit
// accept uniform; bit 0 of word 7 picks X or X^+.
// ---------------------------------------------------------------------------
GLAC_HD double u_sym16(uint32_t h) { return ((double)h + 0.5) * (1.0 / 65536.0) - 0.5; }

template <typename T>
__device__ __forceinline__ void su2_near_unity(T u0, T u1, T u2, T u3, T eps, T sq1me, T out[4]) {
    // x0 = sign(u0) sqrt(1 - eps^2), x = eps u / |u|, normalised
    // (GLAC/math/matrices/su3matrixgenerator.h:202-243)
    T x0 = u0 < T(0) ? -sq1me : sq1me;
    T rn = sqrt(u1 * u1 + u2 * u2 + u3 * u3) / eps;
    T x1 = u1 / rn, x2 = u2 / rn, x3 = u3 / rn;
    T nrm = sqrt(x0 * x0 + x1 * x1 + x2 * x2 + x3 * x3);
    out[0] = x0 / nrm; out[1] = x1 / nrm; out[2] = x2 / nrm; out[3] = x3 / nrm;
}

// X = R S T with the SU(2) elements [[x0 + i x3, x2 + i x1], [-x2 + i x1, x0 - i x3]]
// embedded in the (12), (13), (23) blocks; zero blocks skipped.
template <typename R>
__device__ __forceinline__ M3<R> rst_matrix(const R r[4], const R s[4], const R t[4]) {
    const Cx<R> r00 = cx(r[0], r[3]), r01 = cx(r[2], r[1]), r10 = cx(-r[2], r[1]), r11 = cx(r[0], -r[3]);
    const Cx<R> s00 = cx(s[0], s[3]), s01 = cx(s[2], s[1]), s10 = cx(-s[2], s[1]), s11 = cx(s[0], -s[3]);
    const Cx<R> t00 = cx(t[0], t[3]), t01 = cx(t[2], t[1]), t10 = cx(-t[2], t[1]), t11 = cx(t[0], -t[3]);
    // R S = [[r00 s00, r01, r00 s01], [r10 s00, r11, r10 s01], [s10, 0, s11]]
    const Cx<R> a0 = r00 * s00, a2 = r00 * s01, b0 = r10 * s00, b2 = r10 * s01;
    M3<R> X;
    X(0, 0) = a0;
    X(1, 0) = b0;
    X(2, 0) = s10;
    X(0, 1) = cmac(r01 * t00, a2, t10);
    X(1, 1) = cmac(r11 * t00, b2, t10);
    X(2, 1) = s11 * t10;
    X(0, 2) = cmac(r01 * t01, a2, t11);
    X(1, 2) = cmac(r11 * t01, b2, t11);
    X(2, 2) = s11 * t11;
    return X;
}

// The SU(2) parameters (3 x 4 reals), inverse flag and accept uniform of one hit.
template <typename T>
__device__ __forceinline__ void draw_hit(uint32_t k0, uint32_t k1, uint32_t link_id, uint32_t sweep,
                                         uint32_t stream_id, int hit, T eps, T sq1me, T su[3][4], bool &inverse,
                                         double &r) {
    uint32_t w[8];
#pragma unroll
    for (int call = 0; call < 2; call++) {
        U4 c = {(uint32_t)(2 * hit + call), link_id, sweep, stream_id};
        U4 o = philox4x32_10(c, k0, k1);
        w[4 * call] = o.x; w[4 * call + 1] = o.y; w[4 * call + 2] = o.z; w[4 * call + 3] = o.w;
    }
#pragma unroll
    for (int b = 0; b < 3; b++) {
        T u[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int k = 4 * b + c;
            const uint32_t word = w[k >> 1];
            u[c] = (T)u_sym16((k & 1) ? (word >> 16) : (word & 0xFFFFu));
        }
        su2_near_unity<T>(u[0], u[1], u[2], u[3], eps, sq1me, su[b]);
    }
    inverse = (w[7] & 1u) == 0u;
    r = u_53(w[6], w[7]);
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

// FP64: one link per thread
__global__ void __launch_bounds__(128, MinBlocks<double>::metro)
    k_metropolis_f64(Geom g, LinkField<double> L, int mu, int p, double mfac, double eps, double sq1me, int nhits,
                     uint32_t k0, uint32_t k1, uint32_t sweep, uint32_t stream_id, unsigned long long *acc) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long na = 0;
    if (s < g.Vh) {
        const Site n = site_from_ps(g, p, s);
        const M3<double> A = staple(L, g, n, p, mu);
        M3<double> U = L.load_rw(mu, p, s);
        M3<double> W = mul(U, A);
        const uint32_t link_id = (uint32_t)mu * (uint32_t)g.V + (uint32_t)n.lex;
#pragma unroll 1
        for (int h = 0; h < nhits; h++) {
            double su[3][4], r;
            bool inv;
            draw_hit<double>(k0, k1, link_id, sweep, stream_id, h, eps, sq1me, su, inv, r);
            M3<double> X = rst_matrix<double>(su[0], su[1], su[2]);
            if (inv) X = dagger(X);
            const double dS = (retr_mul(X, W) - retr(W)) * mfac;
            if (exp(-dS) > r) {
                U = mul(X, U);
                W = mul(X, W);
                na++;
            }
        }
        L.store(mu, p, s, U);
    }
    block_add_u64(na, acc);
}

// FP32: two links per thread (lane x at t, lane y at t + Nt/2), accepted per lane
__device__ __forceinline__ void blend(M3<f32x2> &dst, const M3<f32x2> &src, bool x, bool y) {
#pragma unroll
    for (int k = 0; k < 9; k++) {
        if (x) { dst.e[k].re.v.x = src.e[k].re.v.x; dst.e[k].im.v.x = src.e[k].im.v.x; }
        if (y) { dst.e[k].re.v.y = src.e[k].re.v.y; dst.e[k].im.v.y = src.e[k].im.v.y; }
    }
}

__global__ void __launch_bounds__(128, MinBlocks<f32x2>::metro)
    k_metropolis_f32(Geom g, LinkField<f32x2> L, int mu, int p, float mfac, float eps, float sq1me, int nhits,
                     uint32_t k0, uint32_t k1, uint32_t sweep, uint32_t stream_id, unsigned long long *acc) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    unsigned long long na = 0;
    if (s < g.Vh) {
        const Site n = site_from_ps(g, p, s);
        const M3<f32x2> A = staple(L, g, n, p, mu);
        M3<f32x2> U = L.load_rw(mu, p, s);
        M3<f32x2> W = mul(U, A);
        const uint32_t Vphys = (uint32_t)g.V * 2u;
        const uint32_t id0 = (uint32_t)mu * Vphys + (uint32_t)n.lex;
        const uint32_t id1 = id0 + (uint32_t)g.V;
#pragma unroll 1
        for (int h = 0; h < nhits; h++) {
            float sa[3][4], sb[3][4];
            bool inva, invb;
            double ra, rb;
            draw_hit<float>(k0, k1, id0, sweep, stream_id, h, eps, sq1me, sa, inva, ra);
            draw_hit<float>(k0, k1, id1, sweep, stream_id, h, eps, sq1me, sb, invb, rb);
            f32x2 r4[3][4];
#pragma unroll
            for (int b = 0; b < 3; b++)
#pragma unroll
                for (int c = 0; c < 4; c++) r4[b][c] = f32x2(sa[b][c], sb[b][c]);
            M3<f32x2> X = rst_matrix<f32x2>(r4[0], r4[1], r4[2]);
            if (inva || invb) blend(X, dagger(X), inva, invb);
            const f32x2 dS = (retr_mul(X, W) - retr(W)) * f32x2(mfac);
            const bool ax = (double)expf(-dS.v.x) > ra;
            const bool ay = (double)expf(-dS.v.y) > rb;
            if (ax || ay) {
                blend(U, mul(X, U), ax, ay);
                blend(W, mul(X, W), ax, ay);
                na += (ax ? 1 : 0) + (ay ? 1 : 0);
            }
        }
        L.store(mu, p, s, U);
    }
    block_add_u64(na, acc);
}

template <>
void launch_metropolis<double>(const Geom &g, const LinkField<double> &L, int mu, int p, double beta, double eps,
                               int nhits, uint64_t seed, uint32_t sweep, uint32_t stream_id,
                               unsigned long long *acc, cudaStream_t st) {
    k_metropolis_f64<<<(g.Vh + 127) / 128, 128, 0, st>>>(g, L, mu, p, -beta / 3.0, eps, sqrt(1.0 - eps * eps),
                                                         nhits, (uint32_t)seed, (uint32_t)(seed >> 32), sweep,
                                                         stream_id, acc);
}
template <>
void launch_metropolis<f32x2>(const Geom &g, const LinkField<f32x2> &L, int mu, int p, double beta, double eps,
                              int nhits, uint64_t seed, uint32_t sweep, uint32_t stream_id,
                              unsigned long long *acc, cudaStream_t st) {
    k_metropolis_f32<<<(g.Vh + 127) / 128, 128, 0, st>>>(g, L, mu, p, (float)(-beta / 3.0), (float)eps,
                                                         (float)sqrt(1.0 - eps * eps), nhits, (uint32_t)seed,
                                                         (uint32_t)(seed >> 32), sweep, stream_id, acc);
}

// ---------------------------------------------------------------------------
// Observables (GLAC/observables/mastersamplertopcxyz.cpp:236-384): per site,
// for nu = 1..3 and its cyclic complement (rho, sigma), the clovers
//   C = leaf1 - leaf2 + leaf3 - leaf4 projected to (C - C^+) - 1/3 i ImTr,
// plaq += ReTr leaf1, q(t) -= ReTr(C_0nu C_rhosigma), E += ReTr(C C) for both.
// Every block lies in one (t, parity) half-slice of the stored lattice, so its
// sums are per-time-slice partials (two slices for two lanes); FP64 throughout
// the reduction, fixed order.
// ---------------------------------------------------------------------------
ObsPlan make_obs_plan(const Geom &g) {
    // a block covers Bv <= 32 sites of one (t, parity) half-slice, one warp per plane
    const int half_slice = g.N[0] * g.N[1] * g.N[2] / 2;
    int best = 1;
    for (int B = 1; B <= 32 && B <= half_slice; B++)
        if (half_slice % B == 0) best = B;
    ObsPlan pl;
    pl.Bv = best;
    pl.B = 32;
    pl.nb = half_slice / best;
    pl.nblocks = g.N[3] * 2 * pl.nb;
    return pl;
}

// Clover of the (mu, nu) plane at n, projected: F = (C - C^+) - 1/3 i ImTr(C - C^+),
// in the 8-real form; plaq = ReTr(leaf1).
template <typename R>
__device__ __forceinline__ AH8<R> clover_ah(const LinkField<R> &L, const Geom &g, const Site &n, int p, int mu,
                                            int nu, R &plaq) {
    const int q = p ^ 1;
    const Nb n_0 = nb_self(n);
    const Nb n_mup = nb_step(g, n, mu, +1);           // n+mu      (q)
    const Nb n_nup = nb_step(g, n, nu, +1);           // n+nu      (q)
    const Nb n_num = nb_step(g, n, nu, -1);           // n-nu      (q)
    const Nb n_mum = nb_step(g, n, mu, -1);           // n-mu      (q)
    const Nb n_pm = nb_step2(g, n, mu, +1, nu, -1);   // n+mu-nu   (p)
    const Nb n_mm = nb_step2(g, n, mu, -1, nu, -1);   // n-mu-nu   (p)
    const Nb n_mp = nb_step2(g, n, mu, -1, nu, +1);   // n-mu+nu   (p)
    M3<R> C;
    // compiler fences between the leaves keep their loads from all being
    // hoisted to the top, which would multiply the live registers
    {   // leaf1 = U_mu(n) U_nu(n+mu) U_mu(n+nu)^+ U_nu(n)^+
        const M3<R> P = mul(L.load(mu, p, n_0), L.load(nu, q, n_mup));
        const M3<R> W = mul(L.load(nu, p, n_0), L.load(mu, q, n_nup));
        C = mul_nd(P, W);
        plaq = retr(C);
    }
    asm volatile("" ::: "memory");
    {   // leaf2 = U_mu(n) U_nu(n+mu-nu)^+ U_mu(n-nu)^+ U_nu(n-nu)
        const M3<R> Y = mul(L.load(mu, q, n_num), L.load(nu, p, n_pm));
        const M3<R> t = mul_nd(L.load(mu, p, n_0), Y);
        sub_from(C, mul(t, L.load(nu, q, n_num)));
    }
    asm volatile("" ::: "memory");
    {   // leaf3 = U_mu(n-mu)^+ U_nu(n-mu-nu)^+ U_mu(n-mu-nu) U_nu(n-nu)
        M3<R> t = mul_dd(L.load(mu, q, n_mum), L.load(nu, p, n_mm));
        t = mul(t, L.load(mu, p, n_mm));
        add_to(C, mul(t, L.load(nu, q, n_num)));
    }
    asm volatile("" ::: "memory");
    {   // leaf4 = U_mu(n-mu)^+ U_nu(n-mu) U_mu(n-mu+nu) U_nu(n)^+
        M3<R> t = mul_dn(L.load(mu, q, n_mum), L.load(nu, q, n_mum));
        t = mul(t, L.load(mu, p, n_mp));
        sub_from(C, mul_nd(t, L.load(nu, p, n_0)));
    }
    // (C - C^+): diagonal 2 i Im C_ii, off-diagonal C_ij - conj(C_ji); then traceless
    AH8<R> F;
    const R two = real_of<R>(2.0);
    const R tr = (C(0, 0).im + C(1, 1).im + C(2, 2).im) * real_of<R>(2.0 / 3.0);
    F.a = two * C(0, 0).im - tr;
    F.d = two * C(1, 1).im - tr;
    F.b = cx(C(0, 1).re - C(1, 0).re, C(0, 1).im + C(1, 0).im);
    F.c = cx(C(0, 2).re - C(2, 0).re, C(0, 2).im + C(2, 0).im);
    F.e = cx(C(1, 2).re - C(2, 1).re, C(1, 2).im + C(2, 1).im);
    return F;
}

// Re Tr(F G) for traceless anti-Hermitian F, G in the 8-real form:
//   -[a a' + d d' + (a+d)(a'+d')] - 2 Re(b b'* + c c'* + e e'*)
template <typename R>
__device__ __forceinline__ R retr_ah(const AH8<R> &F, const AH8<R> &G) {
    R diag = fmaR(F.a, G.a, F.d * G.d);
    diag = fmaR(F.a + F.d, G.a + G.d, diag);
    R off = fmaR(F.b.re, G.b.re, F.b.im * G.b.im);
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

// threadIdx.x: site in the block (Bv valid of 32), threadIdx.y: plane 0..5 =
// (0,1) (0,2) (0,3) (2,3) (3,1) (1,2): planes y and y+3 pair up in q.
template <typename R>
__global__ void __launch_bounds__(192, MinBlocks<R>::obs)
    k_observables(Geom g, LinkField<R> L, int nb, int Bv, double *partial) {
    const int b = blockIdx.x;
    const int t = b / (2 * nb);
    const int p = (b / nb) & 1;
    const int j = b % nb;
    const int half_slice = g.Vh / g.N[3];
    const int tx = threadIdx.x, plane = threadIdx.y;
    const bool valid = tx < Bv;
    const int s = t * half_slice + j * Bv + (valid ? tx : 0);
    int mu, nu;
    if (plane < 3) { mu = 0; nu = plane + 1; }
    else { mu = (plane - 3 + 1) % 3 + 1; nu = mu % 3 + 1; }
    __shared__ AH8<R> shF[6][32];
    double plaq = 0.0, en = 0.0, q0 = 0.0, q1 = 0.0;
    AH8<R> F;
    if (valid) {
        const Site n = site_from_ps(g, p, s);
        R pl;
        F = clover_ah(L, g, n, p, mu, nu, pl);
        shF[plane][tx] = F;
        plaq = lanesum(pl);
        en = lanesum(retr_ah(F, F));
    }
    __syncthreads();
    if (valid && plane < 3) {
        const R q = retr_ah(F, shF[plane + 3][tx]);
        q0 = -lane0(q);
        q1 = -lane1(q);
    }
    // deterministic block reduction: warps (= planes) then planes in order
    __shared__ double sh[kObsPartial][6];
    plaq = warp_sum_d(plaq);
    en = warp_sum_d(en);
    q0 = warp_sum_d(q0);
    q1 = warp_sum_d(q1);
    if (tx == 0) { sh[0][plane] = plaq; sh[1][plane] = en; sh[2][plane] = q0; sh[3][plane] = q1; }
    __syncthreads();
    if (plane == 0 && tx < kObsPartial) {
        double a = 0.0;
        for (int w = 0; w < 6; w++) a += sh[tx][w];
        partial[kObsPartial * b + tx] = a;
    }
}

// out = [plaq, topc, energy, topct[Nt]] with the reference's normalisations
// (mastersamplertopcxyz.cpp:13-16, :363-383).  Physical slice t is lane t / NtS
// of stored slice t % NtS.
__global__ void k_obs_finalize(int NtS, int lanes, int nb, double Vphys, const double *partial, double *out) {
    __shared__ double sp[1024], se[1024], sq[1024];
    const int Nt = NtS * lanes;
    for (int t = threadIdx.x; t < Nt; t += blockDim.x) {
        const int ts = t % NtS, lane = t / NtS;
        double a = 0.0, e = 0.0, q = 0.0;
        for (int k = 0; k < 2 * nb; k++) {
            const double *pp = partial + kObsPartial * ((size_t)ts * 2 * nb + k);
            if (lane == 0) { a += pp[0]; e += pp[1]; }
            q += pp[2 + lane];
        }
        sp[t] = a; se[t] = e; sq[t] = q;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double qfac = 1.0 / (16 * 16 * M_PI * M_PI);
        double a = 0.0, e = 0.0, q = 0.0;
        for (int t = 0; t < NtS; t++) { a += sp[t]; e += se[t]; }
        for (int t = 0; t < Nt; t++) q += sq[t];
        out[0] = a / (18.0 * Vphys);
        out[1] = q * qfac;
        out[2] = e / Vphys;
        for (int t = 0; t < Nt; t++) out[3 + t] = sq[t] * qfac;
    }
}

template <typename R>
void launch_observables(const Geom &g, const LinkField<R> &L, const ObsPlan &plan, double *partial, double *out,
                        cudaStream_t st) {
    if (g.N[3] * g.lanes > 1024) throw std::invalid_argument("Nt > 1024 not supported by the observable reduction");
    k_observables<R><<<plan.nblocks, dim3(32, 6), 0, st>>>(g, L, plan.nb, plan.Bv, partial);
    k_obs_finalize<<<1, 256, 0, st>>>(g.N[3], g.lanes, plan.nb, (double)g.V * g.lanes, partial, out);
}

// ---------------------------------------------------------------------------
// Start fields, reunitarisation, layout conversion: per physical link.
// grid: x over the stored plane sites and lanes, y = plane (mu*2 + parity).
// ---------------------------------------------------------------------------
struct LinkRef {
    int mu, p, s, lane, lex_phys;
};
// thread -> one physical link; false if out of range
__device__ __forceinline__ bool link_of_thread(const Geom &g, LinkRef &r) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= g.Vh * g.lanes) return false;
    r.lane = i >= g.Vh ? 1 : 0;
    r.s = i - r.lane * g.Vh;
    r.mu = blockIdx.y >> 1;
    r.p = blockIdx.y & 1;
    const Site n = site_from_ps(g, r.p, r.s);
    r.lex_phys = n.lex + r.lane * g.V;
    return true;
}

template <typename R>
__global__ void k_haar(Geom g, LinkField<R> L, uint32_t k0, uint32_t k1, uint32_t stream_id) {
    LinkRef r;
    if (!link_of_thread(g, r)) return;
    const uint32_t link_id = (uint32_t)r.mu * (uint32_t)(g.V * g.lanes) + (uint32_t)r.lex_phys;
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
        const double u1 = ((double)w[2 * e] + 1.0) * 2.3283064365386963e-10;
        const double u2 = (double)w[2 * e + 1] * 2.3283064365386963e-10;
        const double rad = sqrt(-2.0 * log(u1));
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
    L.store_lane(r.mu, r.p, r.s, r.lane, Z);
}

template <typename R>
__global__ void k_cold(Geom g, LinkField<R> L) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    M3<R> I;
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

template <typename R>
__global__ void k_reunitarize(Geom g, LinkField<R> L) {
    LinkRef r;
    if (!link_of_thread(g, r)) return;
    L.store_lane(r.mu, r.p, r.s, r.lane, reunit(L.load_lane(r.mu, r.p, r.s, r.lane)));
}

// AoS host layout [mu][lex_phys][18] (FP64) <-> device layout
template <typename R>
__global__ void k_aos_to_soa(Geom g, const double *aos, LinkField<R> L) {
    LinkRef r;
    if (!link_of_thread(g, r)) return;
    const double2 *src = reinterpret_cast<const double2 *>(aos + ((size_t)r.mu * g.V * g.lanes + r.lex_phys) * 18);
    M3<double> U;
#pragma unroll
    for (int k = 0; k < 9; k++) { const double2 v = src[k]; U.e[k] = cx(v.x, v.y); }
    L.store_lane(r.mu, r.p, r.s, r.lane, U);
}
template <typename R>
__global__ void k_soa_to_aos(Geom g, LinkField<R> L, double *aos) {
    LinkRef r;
    if (!link_of_thread(g, r)) return;
    const M3<double> U = L.load_lane(r.mu, r.p, r.s, r.lane);
    double2 *dst = reinterpret_cast<double2 *>(aos + ((size_t)r.mu * g.V * g.lanes + r.lex_phys) * 18);
#pragma unroll
    for (int k = 0; k < 9; k++) dst[k] = make_double2(U.e[k].re, U.e[k].im);
}
template <typename R>
__global__ void k_copy_field(Geom g, LinkField<R> src, LinkField<R> dst) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
    dst.store(mu, p, s, src.load_rw(mu, p, s));
}

// max over links of |U U^+ - 1| (entrywise), FP64 result via atomicMax on the bit pattern.
template <typename R>
__global__ void k_unitarity(Geom g, LinkField<R> L, unsigned long long *out) {
    LinkRef r;
    if (!link_of_thread(g, r)) return;
    const M3<double> U = L.load_lane(r.mu, r.p, r.s, r.lane);
    const M3<double> P = mul_nd(U, U);
    double m = 0.0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const double re = P(i, j).re - (i == j ? 1.0 : 0.0);
            m = fmax(m, fmax(fabs(re), fabs(P(i, j).im)));
        }
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

static dim3 link_grid(const Geom &g, int block) { return dim3((g.Vh * g.lanes + block - 1) / block, 8); }

template <typename R>
void launch_haar(const Geom &g, const LinkField<R> &L, uint64_t seed, uint32_t stream_id, cudaStream_t st) {
    k_haar<R><<<link_grid(g, 128), 128, 0, st>>>(g, L, (uint32_t)seed, (uint32_t)(seed >> 32), stream_id);
}
template <typename R>
void launch_cold(const Geom &g, const LinkField<R> &L, cudaStream_t st) {
    k_cold<R><<<dim3((g.Vh + 255) / 256, 8), 256, 0, st>>>(g, L);
}
template <typename R>
void launch_reunitarize(const Geom &g, const LinkField<R> &L, cudaStream_t st) {
    k_reunitarize<R><<<link_grid(g, 128), 128, 0, st>>>(g, L);
}
template <typename R>
void launch_aos_to_soa(const Geom &g, const double *aos, const LinkField<R> &L, cudaStream_t st) {
    k_aos_to_soa<R><<<link_grid(g, 128), 128, 0, st>>>(g, aos, L);
}
template <typename R>
void launch_soa_to_aos(const Geom &g, const LinkField<R> &L, double *aos, cudaStream_t st) {
    k_soa_to_aos<R><<<link_grid(g, 128), 128, 0, st>>>(g, L, aos);
}
template <typename R>
void launch_copy_field(const Geom &g, const LinkField<R> &src, const LinkField<R> &dst, cudaStream_t st) {
    k_copy_field<R><<<dim3((g.Vh + 255) / 256, 8), 256, 0, st>>>(g, src, dst);
}
template <typename R>
void launch_max_unitarity_dev(const Geom &g, const LinkField<R> &L, double *out, cudaStream_t st) {
    cudaMemsetAsync(out, 0, sizeof(double), st);
    k_unitarity<R><<<link_grid(g, 128), 128, 0, st>>>(g, L, reinterpret_cast<unsigned long long *>(out));
}

// ---------------------------------------------------------------------------
// Test exports
// ---------------------------------------------------------------------------
__device__ __forceinline__ void store_aos_lane(double *out, size_t off, const M3<double> &A) {
    double2 *dst = reinterpret_cast<double2 *>(out + off * 18);
#pragma unroll
    for (int k = 0; k < 9; k++) dst[k] = make_double2(A.e[k].re, A.e[k].im);
}
__device__ __forceinline__ M3<double> widen(const M3<double> &A, int) { return A; }
__device__ __forceinline__ M3<double> widen(const M3<f32x2> &A, int lane) {
    M3<double> r;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        r.e[k].re = lane ? (double)A.e[k].re.v.y : (double)A.e[k].re.v.x;
        r.e[k].im = lane ? (double)A.e[k].im.v.y : (double)A.e[k].im.v.x;
    }
    return r;
}

// staples (force = 0) or flow forces as full matrices (force = 1)
template <typename R>
__global__ void k_staples_aos(Geom g, LinkField<R> L, double *out, int force) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= g.Vh) return;
    const int mu = blockIdx.y >> 1, p = blockIdx.y & 1;
    const Site n = site_from_ps(g, p, s);
    M3<R> A = staple(L, g, n, p, mu);
    if (force) A = ah_to_m3(project_ah(mul(L.load(mu, p, s), A)));
    const size_t Vphys = (size_t)g.V * g.lanes;
    for (int lane = 0; lane < g.lanes; lane++)
        store_aos_lane(out, (size_t)mu * Vphys + n.lex + (size_t)lane * g.V, widen(A, lane));
}
template <typename R>
void launch_staples_aos(const Geom &g, const LinkField<R> &L, double *out, int force, cudaStream_t st) {
    k_staples_aos<R><<<dim3((g.Vh + 127) / 128, 8), 128, 0, st>>>(g, L, out, force);
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

template <typename T> __device__ __forceinline__ double accept_weight(T dS);
template <> __device__ __forceinline__ double accept_weight<double>(double dS) { return exp(-dS); }
template <> __device__ __forceinline__ double accept_weight<float>(float dS) { return (double)expf(-dS); }

template <typename T>
__device__ __forceinline__ T delta_s(const M3<T> &U, const M3<T> &Up, const M3<T> &A, T mfac) {
    M3<T> D = Up;
    sub_from(D, U);
    return retr_mul(D, A) * mfac;
}

// the reference's accept step with given proposals (GLAC/system.cpp:340-352)
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

// ---------------------------------------------------------------------------
// Explicit instantiations
// ---------------------------------------------------------------------------
#define GLAC_INST_FIELD(R)                                                                                      \
    template void launch_flow_stage<R>(const Geom &, const LinkField<R> &, const LinkField<R> &,                \
                                       const ForceField<R> &, int, int, double, double, cudaStream_t);          \
    template void launch_observables<R>(const Geom &, const LinkField<R> &, const ObsPlan &, double *, double *, \
                                        cudaStream_t);                                                          \
    template void launch_haar<R>(const Geom &, const LinkField<R> &, uint64_t, uint32_t, cudaStream_t);         \
    template void launch_cold<R>(const Geom &, const LinkField<R> &, cudaStream_t);                             \
    template void launch_reunitarize<R>(const Geom &, const LinkField<R> &, cudaStream_t);                      \
    template void launch_aos_to_soa<R>(const Geom &, const double *, const LinkField<R> &, cudaStream_t);       \
    template void launch_soa_to_aos<R>(const Geom &, const LinkField<R> &, double *, cudaStream_t);             \
    template void launch_copy_field<R>(const Geom &, const LinkField<R> &, const LinkField<R> &, cudaStream_t); \
    template void launch_staples_aos<R>(const Geom &, const LinkField<R> &, double *, int, cudaStream_t);       \
    template void launch_max_unitarity_dev<R>(const Geom &, const LinkField<R> &, double *, cudaStream_t);
GLAC_INST_FIELD(double)
GLAC_INST_FIELD(f32x2)
#undef GLAC_INST_FIELD

#define GLAC_INST_MAT(T)                                                                                 \
    template void launch_exp_batch<T>(int, const double *, double *, long, cudaStream_t);                \
    template void launch_accept_fed<T>(double, long, int, double *, const double *, const double *,      \
                                       const double *, unsigned char *, cudaStream_t);                   \
    template void launch_delta_s<T>(double, long, const double *, const double *, const double *, double *, \
                                    cudaStream_t);
GLAC_INST_MAT(double)
GLAC_INST_MAT(float)
#undef GLAC_INST_MAT

}  // namespace glac
