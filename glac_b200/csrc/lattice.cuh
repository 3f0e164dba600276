// Lattice geometry, the HBM layout of gauge fields, and the Philox streams.
//
// Layout.  Sites are split by parity (even/odd planes of Vh = V/2 sites, site
// index s = lex >> 1 with lex = x + Nx(y + Ny(z + Nz t)), the reference's order,
// GLAC/parallelization/index.h:32-35; Nx must be even), per link direction mu:
// plane = mu*2 + parity.  Inside a plane the sites form tiles of 32; a tile
// holds each 16-byte chunk of its 32 links contiguously, so a warp reading 32
// consecutive sites of one chunk issues fully coalesced 128-bit loads, and the
// chunks of a link sit at fixed 512-byte offsets from one base address.
//
//   FP64 (real type double): the full lattice; 9 double2 chunks per link,
//     chunk k = complex element k (row-major).
//   FP32 (real type f32x2): the lattice is cut into two halves along t; the
//     stored lattice has Nt/2 time slices and every stored site carries two
//     lattice sites in the two FP32 lanes: lane x = (x,y,z,t), lane y =
//     (x,y,z,t + Nt/2) (same parity when Nt/2 is even).  9 float4 chunks per
//     site pair, chunk k = (re_k lane x, re_k lane y, im_k lane x, im_k lane y),
//     i.e. exactly one packed f32x2 complex number, so all FP32 arithmetic is
//     fma.rn.f32x2 with no repacking.  Stepping across the cut in t swaps the
//     lanes of the loaded pair.
//
// Traceless anti-Hermitian flow forces use 8 reals per link (a, d, b, c, e) in
// the same tiling: FP64 4 double2 chunks, FP32 4 float4 chunks.
#pragma once

#include <stdint.h>
#include "su3.cuh"

namespace glac {

// Division by a runtime constant via a multiply-high (Granlund & Montgomery,
// PLDI'94): q = (umulhi(m, n) + n) >> l for n < 2^31.
struct FastDiv {
    uint32_t d, m, l;
    FastDiv() {}
    explicit FastDiv(uint32_t d_) : d(d_) {
        l = 0;
        while ((1ull << l) < d) l++;
        m = (uint32_t)((((1ull << l) - d) << 32) / d + 1);
    }
};
GLAC_HD uint32_t fdiv(uint32_t n, const FastDiv &f) {
#ifdef __CUDA_ARCH__
    return (__umulhi(f.m, n) + n) >> f.l;
#else
    return (uint32_t)((((uint64_t)f.m * n >> 32) + n) >> f.l);
#endif
}

// Geometry of the stored lattice: for lanes == 2 (FP32) its t extent is half
// the physical one and the physical lattice is twice its volume.
struct Geom {
    int N[4];
    int Nxh;
    int Vh;
    int V;
    int stride[4];  // lexicographic strides 1, Nx, Nx Ny, Nx Ny Nz
    int lanes;      // 1 (FP64) or 2 (FP32, lane y = t + N[3])
    FastDiv div_xh, div_y, div_z;
};

// dims are the physical extents; lanes = 2 halves Nt.
inline Geom make_geom(const int dims[4], int lanes = 1) {
    int N[4] = {dims[0], dims[1], dims[2], dims[3] / lanes};
    Geom g;
    g.lanes = lanes;
    for (int d = 0; d < 4; d++) g.N[d] = N[d];
    g.Nxh = N[0] / 2;
    g.V = N[0] * N[1] * N[2] * N[3];
    g.Vh = g.V / 2;
    g.stride[0] = 1;
    g.stride[1] = N[0];
    g.stride[2] = N[0] * N[1];
    g.stride[3] = N[0] * N[1] * N[2];
    g.div_xh = FastDiv((uint32_t)g.Nxh);
    g.div_y = FastDiv((uint32_t)N[1]);
    g.div_z = FastDiv((uint32_t)N[2]);
    return g;
}

// Site with coordinates c[] and its lexicographic index.
struct Site {
    int c[4];
    int lex;
};

// (parity, index in parity plane) -> coordinates
GLAC_HD Site site_from_ps(const Geom &g, int p, int s) {
    Site st;
    uint32_t q = fdiv((uint32_t)s, g.div_xh);
    int xh = s - (int)q * g.Nxh;
    uint32_t q2 = fdiv(q, g.div_y);
    st.c[1] = (int)(q - q2 * g.N[1]);
    uint32_t q3 = fdiv(q2, g.div_z);
    st.c[2] = (int)(q2 - q3 * g.N[2]);
    st.c[3] = (int)q3;
    st.c[0] = 2 * xh + ((st.c[1] + st.c[2] + st.c[3] + p) & 1);
    st.lex = st.c[0] + g.N[0] * (st.c[1] + g.N[1] * (st.c[2] + g.N[2] * st.c[3]));
    return st;
}

// A neighbour: its index in the parity plane and whether the step crossed the
// t cut of a two-lane lattice (then the lanes of what is loaded are swapped).
struct Nb {
    int s;
    int swap;
};

// n + a e_d (a = +1 or -1), periodic
GLAC_HD Nb nb_step(const Geom &g, const Site &n, int d, int a) {
    const int cd = n.c[d];
    int off;
    bool wrap;
    if (a > 0) { wrap = cd == g.N[d] - 1; off = wrap ? -(g.N[d] - 1) * g.stride[d] : g.stride[d]; }
    else { wrap = cd == 0; off = wrap ? (g.N[d] - 1) * g.stride[d] : -g.stride[d]; }
    Nb r;
    r.s = (n.lex + off) >> 1;
    r.swap = (g.lanes == 2 && d == 3 && wrap) ? 1 : 0;
    return r;
}
// n + a e_d + b e_e (d != e)
GLAC_HD Nb nb_step2(const Geom &g, const Site &n, int d, int a, int e, int b) {
    const int cd = n.c[d], ce = n.c[e];
    int off;
    bool wd, we;
    if (a > 0) { wd = cd == g.N[d] - 1; off = wd ? -(g.N[d] - 1) * g.stride[d] : g.stride[d]; }
    else { wd = cd == 0; off = wd ? (g.N[d] - 1) * g.stride[d] : -g.stride[d]; }
    if (b > 0) { we = ce == g.N[e] - 1; off += we ? -(g.N[e] - 1) * g.stride[e] : g.stride[e]; }
    else { we = ce == 0; off += we ? (g.N[e] - 1) * g.stride[e] : -g.stride[e]; }
    Nb r;
    r.s = (n.lex + off) >> 1;
    r.swap = (g.lanes == 2 && ((d == 3 && wd) || (e == 3 && we))) ? 1 : 0;
    return r;
}
GLAC_HD Nb nb_self(const Site &n) {
    Nb r;
    r.s = n.lex >> 1;
    r.swap = 0;
    return r;
}

GLAC_HD int parity_of_lex(const Geom &g, int lex) {
    // parity = (x+y+z+t) & 1; only needed on the host side, slow path
    int x = lex % g.N[0];
    int r = lex / g.N[0];
    int y = r % g.N[1];
    r /= g.N[1];
    int z = r % g.N[2];
    int t = r / g.N[2];
    return (x + y + z + t) & 1;
}

// ---------------------------------------------------------------------------
// Field accessors
// ---------------------------------------------------------------------------
GLAC_HD int round32(int v) { return (v + 31) & ~31; }

GLAC_HD f32x2 lane_swap(f32x2 a) { return f32x2(a.v.y, a.v.x); }
GLAC_HD M3<f32x2> lane_swap(const M3<f32x2> &A) {
    M3<f32x2> B;
#pragma unroll
    for (int k = 0; k < 9; k++) { B.e[k].re = lane_swap(A.e[k].re); B.e[k].im = lane_swap(A.e[k].im); }
    return B;
}

template <typename R> struct LinkField;

template <> struct LinkField<double> {
    double2 *p;
    int Vh, Vh32;
    GLAC_HD size_t base(int mu, int par, int s) const {
        return (size_t)(mu * 2 + par) * 9 * (size_t)Vh32 + (size_t)(s >> 5) * 288 + (size_t)(s & 31);
    }
    __device__ __forceinline__ M3<double> load(int mu, int par, Nb nb) const { return load(mu, par, nb.s); }
    __device__ __forceinline__ M3<double> load(int mu, int par, int s) const {
        const double2 *b = p + base(mu, par, s);
        M3<double> U;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            double2 v = __ldg(b + 32 * k);
            U.e[k].re = v.x; U.e[k].im = v.y;
        }
        return U;
    }
    __device__ __forceinline__ M3<double> load_rw(int mu, int par, int s) const {
        const double2 *b = p + base(mu, par, s);
        M3<double> U;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            double2 v = b[32 * k];
            U.e[k].re = v.x; U.e[k].im = v.y;
        }
        return U;
    }
    __device__ __forceinline__ void store(int mu, int par, int s, const M3<double> &U) const {
        double2 *b = p + base(mu, par, s);
#pragma unroll
        for (int k = 0; k < 9; k++) b[32 * k] = make_double2(U.e[k].re, U.e[k].im);
    }
    // one lattice site (lane ignored for FP64)
    __device__ __forceinline__ M3<double> load_lane(int mu, int par, int s, int) const { return load_rw(mu, par, s); }
    __device__ __forceinline__ void store_lane(int mu, int par, int s, int, const M3<double> &U) const {
        store(mu, par, s, U);
    }
};

// FP32: site pairs in packed lanes (lane x: t < Nt/2, lane y: t + Nt/2)
template <> struct LinkField<f32x2> {
    float4 *p;
    int Vh, Vh32;
    GLAC_HD size_t base(int mu, int par, int s) const {
        return (size_t)(mu * 2 + par) * 9 * (size_t)Vh32 + (size_t)(s >> 5) * 288 + (size_t)(s & 31);
    }
    __device__ __forceinline__ M3<f32x2> load(int mu, int par, int s) const {
        const float4 *b = p + base(mu, par, s);
        M3<f32x2> U;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const float4 v = __ldg(b + 32 * k);
            U.e[k].re = f32x2(v.x, v.y);
            U.e[k].im = f32x2(v.z, v.w);
        }
        return U;
    }
    __device__ __forceinline__ M3<f32x2> load(int mu, int par, Nb nb) const {
        const M3<f32x2> U = load(mu, par, nb.s);
        return nb.swap ? lane_swap(U) : U;
    }
    __device__ __forceinline__ M3<f32x2> load_rw(int mu, int par, int s) const {
        const float4 *b = p + base(mu, par, s);
        M3<f32x2> U;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const float4 v = b[32 * k];
            U.e[k].re = f32x2(v.x, v.y);
            U.e[k].im = f32x2(v.z, v.w);
        }
        return U;
    }
    __device__ __forceinline__ void store(int mu, int par, int s, const M3<f32x2> &U) const {
        float4 *b = p + base(mu, par, s);
#pragma unroll
        for (int k = 0; k < 9; k++)
            b[32 * k] = make_float4(U.e[k].re.v.x, U.e[k].re.v.y, U.e[k].im.v.x, U.e[k].im.v.y);
    }
    // one lattice site: lane 0 or 1 of the pair, widened to FP64
    __device__ __forceinline__ M3<double> load_lane(int mu, int par, int s, int lane) const {
        const float *b = reinterpret_cast<const float *>(p + base(mu, par, s));
        M3<double> U;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            U.e[k].re = (double)b[128 * k + lane];
            U.e[k].im = (double)b[128 * k + 2 + lane];
        }
        return U;
    }
    __device__ __forceinline__ void store_lane(int mu, int par, int s, int lane, const M3<double> &U) const {
        float *b = reinterpret_cast<float *>(p + base(mu, par, s));
#pragma unroll
        for (int k = 0; k < 9; k++) {
            b[128 * k + lane] = (float)U.e[k].re;
            b[128 * k + 2 + lane] = (float)U.e[k].im;
        }
    }
};

template <typename R> struct ForceField;

template <> struct ForceField<double> {
    double2 *p;
    int Vh, Vh32;
    GLAC_HD size_t base(int mu, int par, int s) const {
        return (size_t)(mu * 2 + par) * 4 * (size_t)Vh32 + (size_t)(s >> 5) * 128 + (size_t)(s & 31);
    }
    __device__ __forceinline__ AH8<double> load(int mu, int par, int s) const {
        const double2 *b = p + base(mu, par, s);
        AH8<double> Z;
        const double2 v0 = b[0], v1 = b[32], v2 = b[64], v3 = b[96];
        Z.a = v0.x; Z.d = v0.y;
        Z.b = cx(v1.x, v1.y); Z.c = cx(v2.x, v2.y); Z.e = cx(v3.x, v3.y);
        return Z;
    }
    __device__ __forceinline__ void store(int mu, int par, int s, const AH8<double> &Z) const {
        double2 *b = p + base(mu, par, s);
        b[0] = make_double2(Z.a, Z.d);
        b[32] = make_double2(Z.b.re, Z.b.im);
        b[64] = make_double2(Z.c.re, Z.c.im);
        b[96] = make_double2(Z.e.re, Z.e.im);
    }
};

template <> struct ForceField<f32x2> {
    float4 *p;
    int Vh, Vh32;
    GLAC_HD size_t base(int mu, int par, int s) const {
        return (size_t)(mu * 2 + par) * 4 * (size_t)Vh32 + (size_t)(s >> 5) * 128 + (size_t)(s & 31);
    }
    __device__ __forceinline__ AH8<f32x2> load(int mu, int par, int s) const {
        const float4 *b = p + base(mu, par, s);
        AH8<f32x2> Z;
        const float4 v0 = b[0], v1 = b[32], v2 = b[64], v3 = b[96];
        Z.a = f32x2(v0.x, v0.y); Z.d = f32x2(v0.z, v0.w);
        Z.b = cx(f32x2(v1.x, v1.y), f32x2(v1.z, v1.w));
        Z.c = cx(f32x2(v2.x, v2.y), f32x2(v2.z, v2.w));
        Z.e = cx(f32x2(v3.x, v3.y), f32x2(v3.z, v3.w));
        return Z;
    }
    __device__ __forceinline__ void store(int mu, int par, int s, const AH8<f32x2> &Z) const {
        float4 *b = p + base(mu, par, s);
        b[0] = make_float4(Z.a.v.x, Z.a.v.y, Z.d.v.x, Z.d.v.y);
        b[32] = make_float4(Z.b.re.v.x, Z.b.re.v.y, Z.b.im.v.x, Z.b.im.v.y);
        b[64] = make_float4(Z.c.re.v.x, Z.c.re.v.y, Z.c.im.v.x, Z.c.im.v.y);
        b[96] = make_float4(Z.e.re.v.x, Z.e.re.v.y, Z.e.im.v.x, Z.e.im.v.y);
    }
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11)
// ---------------------------------------------------------------------------
struct U4 { uint32_t x, y, z, w; };

GLAC_HD U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; r++) {
#ifdef __CUDA_ARCH__
        uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
#else
        uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0, hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
#endif
        U4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// uniform in (-1/2, 1/2), never 0
GLAC_HD double u_sym(uint32_t w) { return ((double)w + 0.5) * 2.3283064365386963e-10 - 0.5; }
GLAC_HD float u_symf(uint32_t w) { return ((float)(w >> 8) + 0.5f) * 5.9604644775390625e-8f - 0.5f; }
// uniform in [0,1) with 53 bits
GLAC_HD double u_53(uint32_t hi, uint32_t lo) {
    return (double)(((uint64_t)hi << 21) | (lo >> 11)) * 1.1102230246251565e-16;
}

}  // namespace glac
