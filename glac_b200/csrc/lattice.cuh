// Lattice geometry, the HBM layout of gauge fields, and the Philox streams.
//
// Layout (even/odd split, arrays of 32-site tiles): a field of 4 link
// directions over V = Nx Ny Nz Nt sites is stored per (mu, parity) plane of
// Vh = V/2 sites.  Inside a plane the sites form tiles of 32 (Vh32 = Vh rounded
// up to 32); a tile holds each 16-byte chunk of its 32 links contiguously, so a
// warp reading 32 consecutive sites of one chunk issues fully coalesced 128-bit
// loads, and the chunks of one link sit at fixed 512-byte offsets from one base
// address (no per-chunk address registers):
//   FP64: 9 double2 chunks (chunk k = complex element k, row-major)
//         addr = plane*9*Vh32 + (s>>5)*9*32 + k*32 + (s&31)
//   FP32: 4 float4 chunks (complex elements 2k, 2k+1) in tiles, plus element 8
//         as a plain float2 array:  addr4 = plane*4*Vh32 + (s>>5)*4*32 + k*32 + (s&31),
//         addr2 = plane*Vh + s
//   plane = mu*2 + parity.
// The site index inside a parity plane is s = lex >> 1 with
// lex = x + Nx(y + Ny(z + Nz t)), the reference's site order
// (GLAC/parallelization/index.h:32-35); Nx must be even.
// Traceless anti-Hermitian flow forces use 8 reals per link (a, d, b, c, e) in
// the same tiling: FP64 4 double2 chunks, FP32 2 float4 chunks.
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

struct Geom {
    int N[4];
    int Nxh;
    int Vh;
    int V;
    int stride[4];  // lexicographic strides 1, Nx, Nx Ny, Nx Ny Nz
    FastDiv div_xh, div_y, div_z;
};

inline Geom make_geom(const int N[4]) {
    Geom g;
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

// periodic offset of one step a = +1 or -1 along d, by indexing the arrays
GLAC_HD int step_offset_indexed(const Geom &g, const Site &n, int d, int a) {
    const int cd = n.c[d];
    if (a > 0) return (cd == g.N[d] - 1) ? -(g.N[d] - 1) * g.stride[d] : g.stride[d];
    return (cd == 0) ? (g.N[d] - 1) * g.stride[d] : -g.stride[d];
}
// lexicographic index of n + a e_d (a = +1 or -1), periodic
GLAC_HD int lex_step(const Geom &g, const Site &n, int d, int a) { return n.lex + step_offset_indexed(g, n, d, a); }
// lexicographic index of n + a e_d + b e_e (d != e)
GLAC_HD int lex_step2(const Geom &g, const Site &n, int d, int a, int e, int b) {
    return n.lex + step_offset_indexed(g, n, d, a) + step_offset_indexed(g, n, e, b);
}

// v[d] for a direction d that may be a run-time value, as a chain of selects:
// the arrays stay in registers, where indexing them with a run-time d places
// the Site and the Geom in local memory.  Folds to v[d] for a constant d.  The
// FP32 staple (flow stage, Metropolis) runs faster with it; the FP64 staple and
// the clover run faster with the indexed form above (timed on B200 at 32^3 x 64).
GLAC_HD int pick4(const int v[4], int d) { return d == 0 ? v[0] : d == 1 ? v[1] : d == 2 ? v[2] : v[3]; }

// periodic offset of one step a = +1 or -1 along d, selected without indexing
GLAC_HD int step_offset(const Geom &g, const Site &n, int d, int a) {
    const int cd = pick4(n.c, d), Nd = pick4(g.N, d), sd = pick4(g.stride, d);
    if (a > 0) return (cd == Nd - 1) ? -(Nd - 1) * sd : sd;
    return (cd == 0) ? (Nd - 1) * sd : -sd;
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

// Element offsets inside a field are 32-bit (fewer address instructions per
// neighbour load); glac_create and glac_ensemble_create reject lattices whose
// fields would need more (field_offsets_fit).
inline bool field_offsets_fit(long long V, bool fp64) {
    const long long vh32 = ((V / 2) + 31) / 32 * 32;
    return (fp64 ? 72 : 32) * vh32 < (1ll << 32);
}

// Field loads are plain global loads (L1-cached), not the non-coherent
// read-only path (__ldg): the persistent ensemble kernel reads, after a grid
// barrier, links that other blocks wrote earlier in the same launch, which the
// non-coherent path does not guarantee to see.  (Timed on B200 at 32^3 x 64:
// flow steps and Metropolis sweeps within 2 % of the __ldg build, either way.)
template <typename T> struct LinkField;

template <> struct LinkField<double> {
    double2 *p;
    int Vh, Vh32;
    GLAC_HD uint32_t base(int mu, int par, int s) const {
        return (uint32_t)(mu * 2 + par) * (9u * (uint32_t)Vh32) + (uint32_t)(s >> 5) * 288u + (uint32_t)(s & 31);
    }
    __device__ __forceinline__ M3<double> load(int mu, int par, int s) const {
        const double2 *b = p + base(mu, par, s);
        M3<double> U;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            double2 v = b[32 * k];
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
};

template <> struct LinkField<float> {
    float4 *p4;
    float2 *p2;
    int Vh, Vh32;
    GLAC_HD uint32_t base4(int mu, int par, int s) const {
        return (uint32_t)(mu * 2 + par) * (4u * (uint32_t)Vh32) + (uint32_t)(s >> 5) * 128u + (uint32_t)(s & 31);
    }
    GLAC_HD uint32_t at2(int mu, int par, int s) const { return (uint32_t)(mu * 2 + par) * (uint32_t)Vh + (uint32_t)s; }
    __device__ __forceinline__ M3<float> load(int mu, int par, int s) const {
        const float4 *b = p4 + base4(mu, par, s);
        M3<float> U;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float4 v = b[32 * k];
            U.e[2 * k].re = v.x; U.e[2 * k].im = v.y; U.e[2 * k + 1].re = v.z; U.e[2 * k + 1].im = v.w;
        }
        float2 w = p2[at2(mu, par, s)];
        U.e[8].re = w.x; U.e[8].im = w.y;
        return U;
    }
    __device__ __forceinline__ M3<float> load_rw(int mu, int par, int s) const {
        const float4 *b = p4 + base4(mu, par, s);
        M3<float> U;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            float4 v = b[32 * k];
            U.e[2 * k].re = v.x; U.e[2 * k].im = v.y; U.e[2 * k + 1].re = v.z; U.e[2 * k + 1].im = v.w;
        }
        float2 w = p2[at2(mu, par, s)];
        U.e[8].re = w.x; U.e[8].im = w.y;
        return U;
    }
    __device__ __forceinline__ void store(int mu, int par, int s, const M3<float> &U) const {
        float4 *b = p4 + base4(mu, par, s);
#pragma unroll
        for (int k = 0; k < 4; k++)
            b[32 * k] = make_float4(U.e[2 * k].re, U.e[2 * k].im, U.e[2 * k + 1].re, U.e[2 * k + 1].im);
        p2[at2(mu, par, s)] = make_float2(U.e[8].re, U.e[8].im);
    }
};

template <typename T> struct ForceField;

template <> struct ForceField<double> {
    double2 *p;
    int Vh, Vh32;
    GLAC_HD uint32_t base(int mu, int par, int s) const {
        return (uint32_t)(mu * 2 + par) * (4u * (uint32_t)Vh32) + (uint32_t)(s >> 5) * 128u + (uint32_t)(s & 31);
    }
    __device__ __forceinline__ AH8<double> load(int mu, int par, int s) const {
        const double2 *b = p + base(mu, par, s);
        AH8<double> Z;
        double2 v0 = b[0], v1 = b[32], v2 = b[64], v3 = b[96];
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

template <> struct ForceField<float> {
    float4 *p;
    int Vh, Vh32;
    GLAC_HD uint32_t base(int mu, int par, int s) const {
        return (uint32_t)(mu * 2 + par) * (2u * (uint32_t)Vh32) + (uint32_t)(s >> 5) * 64u + (uint32_t)(s & 31);
    }
    __device__ __forceinline__ AH8<float> load(int mu, int par, int s) const {
        const float4 *b = p + base(mu, par, s);
        AH8<float> Z;
        float4 v0 = b[0], v1 = b[32];
        Z.a = v0.x; Z.d = v0.y; Z.b = cx(v0.z, v0.w);
        Z.c = cx(v1.x, v1.y); Z.e = cx(v1.z, v1.w);
        return Z;
    }
    __device__ __forceinline__ void store(int mu, int par, int s, const AH8<float> &Z) const {
        float4 *b = p + base(mu, par, s);
        b[0] = make_float4(Z.a, Z.d, Z.b.re, Z.b.im);
        b[32] = make_float4(Z.c.re, Z.c.im, Z.e.re, Z.e.im);
    }
};

// Clover parts of the measurement fused into flow stage 0: twelve slots of
// traceless anti-Hermitian 8-real matrices per site (slot 2 pl: plane pl's part
// from the site's own link, 2 pl + 1: the part from the link at n - mu), laid
// out as a ForceField whose "direction" index runs over the 12 slots, and the
// four plaquette sums per site, plaq[(mu * 2 + parity) * Vh + s].
template <typename T> struct CloverParts {
    ForceField<T> ah;
    T *plaq;
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
