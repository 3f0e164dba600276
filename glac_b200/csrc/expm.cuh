// SU(3) exponentials of traceless anti-Hermitian matrices.
//
// Default: Morningstar-Peardon Cayley-Hamilton form (hep-lat/0311018), the
// reference's "morningstar" (GLAC/math/exponentiation/su3exp.cpp:16-79).
// With Q = -i Z (Hermitian, traceless), exp(Z) = exp(iQ) = f0 + f1 Q + f2 Q^2,
// c0 = det Q = Tr(Q^3)/3, c1 = Tr(Q^2)/2.  The coefficients f_j(c0, c1) are
// evaluated two ways:
//  * c1 < 0.1 (spectral radius < 0.37, every flow step at eps <= 0.05): the
//    power series of exp(iQ) reduced by Cayley-Hamilton, Q^3 = c1 Q + c0 1,
//    in the working precision (16 terms FP64, 9 terms FP32).  It has no
//    cancellation at small |Q| and no conditioning problem at degenerate
//    eigenvalues, where the closed form's acos and h_j lose digits.
//  * otherwise: the closed form of su3exp.cpp:28-76, always in FP64 (also on
//    the FP32 path, whose matrix algebra stays FP32).
// Alternates selectable by the run-config's expFunc: "luscher"
// (expluscher.cpp:13-68), "taylor2" (taylor2exp.cpp:8-16), "taylor4"
// (taylor4exp.cpp:8-20).
#pragma once

#include "su3.cuh"

namespace glac {

enum ExpKind { EXP_MORNINGSTAR = 0, EXP_LUSCHER = 1, EXP_TAYLOR2 = 2, EXP_TAYLOR4 = 3 };

struct ExpCoef {
    double f0r, f0i, f1r, f1i, f2r, f2i;
};

// Coefficients from c0 = det Q and c1 = Tr(Q^2)/2 (su3exp.cpp:28-69).
// Z = 0 (c1 = 0) yields the identity here; the reference divides 0 by 0 there.
GLAC_HD ExpCoef ms_coefficients(double c0, double c1) {
    ExpCoef f;
    if (!(c1 > 0.0)) {
        f.f0r = 1.0; f.f0i = 0.0; f.f1r = 0.0; f.f1i = 1.0; f.f2r = -0.5; f.f2i = 0.0;
        return f;
    }
    double c0max = 0.6666666666666666 * c1 * sqrt(c1 * 0.3333333333333333);
    double ratio = c0max > 0.0 ? fabs(c0) / c0max : 1.0;
    ratio = ratio > 1.0 ? 1.0 : ratio;
    double theta = acos(ratio);
    double st3, ct3;
    sincos(0.3333333333333333 * theta, &st3, &ct3);
    double u = sqrt(0.3333333333333333 * c1) * ct3;
    double w = sqrt(c1) * st3;
    double uu = u * u, ww = w * w;
    double su, cu, sw, cw, s2u, c2u;
    sincos(u, &su, &cu);
    sincos(w, &sw, &cw);
    sincos(2.0 * u, &s2u, &c2u);
    double xi0 = fabs(w) > 0.05 ? sw / w : 1.0 - ww * (1.0 - 0.05 * ww * (1.0 - ww / 42.0)) / 6.0;
    double h0r = 8 * uu * cu * cw + 2 * u * xi0 * (3 * uu + ww) * su + (uu - ww) * c2u;
    double h0i = -8 * uu * su * cw + 2 * u * xi0 * (3 * uu + ww) * cu + (uu - ww) * s2u;
    double h1r = -2 * u * cu * cw + 2 * u * c2u + xi0 * (3 * uu - ww) * su;
    double h1i = 2 * u * su * cw + 2 * u * s2u + xi0 * (3 * uu - ww) * cu;
    double h2r = -3 * u * xi0 * su - cu * cw + c2u;
    double h2i = -3 * u * xi0 * cu + su * cw + s2u;
    double den = 9 * uu - ww;
    f.f0r = h0r / den; f.f0i = h0i / den;
    f.f1r = h1r / den; f.f1i = h1i / den;
    f.f2r = h2r / den; f.f2i = h2i / den;
    if (c0 < 0) {  // c0 -> -c0 symmetry (su3exp.cpp:71-76)
        f.f0i = -f.f0i;
        f.f1r = -f.f1r;
        f.f2i = -f.f2i;
    }
    return f;
}

// Hermitian Q = -i Z in compact form: real diagonal q0, q1, q2 and x = Q01,
// y = Q02, z = Q12.
template <typename R> struct HQ {
    R q0, q1, q2;
    Cx<R> x, y, z;
};
template <typename R> GLAC_HD HQ<R> herm_from_ah(const AH8<R> &Z) {
    HQ<R> Q;
    Q.q0 = Z.a;
    Q.q1 = Z.d;
    Q.q2 = -(Z.a + Z.d);
    Q.x = cx(Z.b.im, -Z.b.re);  // -i b
    Q.y = cx(Z.c.im, -Z.c.re);
    Q.z = cx(Z.e.im, -Z.e.re);
    return Q;
}

// Q^2 of a compact Hermitian matrix: diag and the upper triangle.
template <typename R> struct HQ2 {
    R d0, d1, d2;
    Cx<R> x, y, z;
};
template <typename R> GLAC_HD HQ2<R> herm_square(const HQ<R> &Q) {
    HQ2<R> S;
    R nx = fmaR(Q.x.re, Q.x.re, Q.x.im * Q.x.im);
    R ny = fmaR(Q.y.re, Q.y.re, Q.y.im * Q.y.im);
    R nz = fmaR(Q.z.re, Q.z.re, Q.z.im * Q.z.im);
    S.d0 = fmaR(Q.q0, Q.q0, nx + ny);
    S.d1 = fmaR(Q.q1, Q.q1, nx + nz);
    S.d2 = fmaR(Q.q2, Q.q2, ny + nz);
    Cx<R> t;
    // (0,1) = x (q0 + q1) + y conj(z)
    t.re = Q.x.re * (Q.q0 + Q.q1); t.im = Q.x.im * (Q.q0 + Q.q1);
    S.x = cmac_bc(t, Q.y, Q.z);
    // (0,2) = y (q0 + q2) + x z
    t.re = Q.y.re * (Q.q0 + Q.q2); t.im = Q.y.im * (Q.q0 + Q.q2);
    S.y = cmac(t, Q.x, Q.z);
    // (1,2) = z (q1 + q2) + conj(x) y
    t.re = Q.z.re * (Q.q1 + Q.q2); t.im = Q.z.im * (Q.q1 + Q.q2);
    S.z = cmac_cj(t, Q.x, Q.y);
    return S;
}

// c0 = Tr(Q Q^2)/3 = det Q and c1 = Tr(Q^2)/2 in the working precision.
template <typename R> GLAC_HD void invariants(const HQ<R> &Q, const HQ2<R> &S, R &c0, R &c1) {
    c1 = R(0.5f) * (S.d0 + S.d1 + S.d2);
    R t = Q.q0 * S.d0;
    t = fmaR(Q.q1, S.d1, t);
    t = fmaR(Q.q2, S.d2, t);
    R o = Q.x.re * S.x.re;
    o = fmaR(Q.x.im, S.x.im, o);
    o = fmaR(Q.y.re, S.y.re, o);
    o = fmaR(Q.y.im, S.y.im, o);
    o = fmaR(Q.z.re, S.z.re, o);
    o = fmaR(Q.z.im, S.z.im, o);
    c0 = (t + o + o) * R(0.33333333333333333);
}
template <typename R> struct SeriesTerms { static const int n = 9; };
template <> struct SeriesTerms<double> { static const int n = 16; };
#define GLAC_SERIES_C1_MAX 0.1

// exp(iQ) = sum_n i^n Q^n / n!,  Q^n = a_n 1 + b_n Q + g_n Q^2 with
// a_{n+1} = c0 g_n, b_{n+1} = a_n + c1 g_n, g_{n+1} = b_n  (a, b, g carry 1/n!).
// With M1 set, f0 omits the n = 0 term: the coefficients of exp(iQ) - 1.
template <typename R, bool M1 = false> GLAC_HD void ms_series(R c0, R c1, Cx<R> &f0, Cx<R> &f1, Cx<R> &f2) {
    R a = R(1.f), b = rzero<R>(), gg = rzero<R>();
    R z = rzero<R>();
    f0 = cx(z, z); f1 = cx(z, z); f2 = cx(z, z);
#pragma unroll
    for (int n = 0; n < SeriesTerms<R>::n; n++) {
        switch (n & 3) {
        case 0: if (!M1 || n > 0) f0.re = f0.re + a; f1.re = f1.re + b; f2.re = f2.re + gg; break;
        case 1: f0.im = f0.im + a; f1.im = f1.im + b; f2.im = f2.im + gg; break;
        case 2: f0.re = f0.re - a; f1.re = f1.re - b; f2.re = f2.re - gg; break;
        default: f0.im = f0.im - a; f1.im = f1.im - b; f2.im = f2.im - gg; break;
        }
        const R inv = R(1.0f / (float)(n + 1));
        const R a1 = c0 * gg * inv;
        const R b1 = fmaR(c1, gg, a) * inv;
        gg = b * inv;
        a = a1;
        b = b1;
    }
}
template <> GLAC_HD void ms_series<double, false>(double c0, double c1, Cx<double> &f0, Cx<double> &f1,
                                                   Cx<double> &f2) {
    double a = 1.0, b = 0.0, gg = 0.0;
    f0 = cx(0.0, 0.0); f1 = cx(0.0, 0.0); f2 = cx(0.0, 0.0);
#pragma unroll
    for (int n = 0; n < SeriesTerms<double>::n; n++) {
        switch (n & 3) {
        case 0: f0.re += a; f1.re += b; f2.re += gg; break;
        case 1: f0.im += a; f1.im += b; f2.im += gg; break;
        case 2: f0.re -= a; f1.re -= b; f2.re -= gg; break;
        default: f0.im -= a; f1.im -= b; f2.im -= gg; break;
        }
        const double inv = 1.0 / (double)(n + 1);
        const double a1 = c0 * gg * inv;
        const double b1 = fma(c1, gg, a) * inv;
        gg = b * inv;
        a = a1;
        b = b1;
    }
}

template <typename R> GLAC_HD R from_d(double v);
template <> GLAC_HD double from_d<double>(double v) { return v; }
template <> GLAC_HD float from_d<float>(double v) { return (float)v; }

// f0 + f1 Q + f2 Q^2 as a full matrix.
template <typename R>
GLAC_HD M3<R> ms_combine(const HQ<R> &Q, const HQ2<R> &S, Cx<R> f0, Cx<R> f1, Cx<R> f2) {
    M3<R> E;
    // diagonal: f0 + f1 q_i + f2 s_i  (q_i, s_i real)
    E(0, 0) = cx(fmaR(f1.re, Q.q0, fmaR(f2.re, S.d0, f0.re)), fmaR(f1.im, Q.q0, fmaR(f2.im, S.d0, f0.im)));
    E(1, 1) = cx(fmaR(f1.re, Q.q1, fmaR(f2.re, S.d1, f0.re)), fmaR(f1.im, Q.q1, fmaR(f2.im, S.d1, f0.im)));
    E(2, 2) = cx(fmaR(f1.re, Q.q2, fmaR(f2.re, S.d2, f0.re)), fmaR(f1.im, Q.q2, fmaR(f2.im, S.d2, f0.im)));
    // off-diagonal (i<j): f1 Q_ij + f2 S_ij ; (j,i): f1 conj(Q_ij) + f2 conj(S_ij)
    E(0, 1) = cmac(f1 * Q.x, f2, S.x);
    E(1, 0) = cmac(f1 * conj(Q.x), f2, conj(S.x));
    E(0, 2) = cmac(f1 * Q.y, f2, S.y);
    E(2, 0) = cmac(f1 * conj(Q.y), f2, conj(S.y));
    E(1, 2) = cmac(f1 * Q.z, f2, S.z);
    E(2, 1) = cmac(f1 * conj(Q.z), f2, conj(S.z));
    return E;
}

// exp(Z), or with M1 set exp(Z) - 1: the flow's link update U' = U + (exp(Z) - 1) U
// rounds once at the magnitude of U instead of carrying exp(Z)'s rounding at
// ulp(1), which in FP32 is most of a small flow increment's precision.
template <typename R, bool M1 = false> GLAC_HD M3<R> expm_morningstar(const AH8<R> &Z) {
    const HQ<R> Q = herm_from_ah(Z);
    const HQ2<R> S = herm_square(Q);
    R c0, c1;
    invariants(Q, S, c0, c1);
    Cx<R> f0, f1, f2;
    if (c1 < R(GLAC_SERIES_C1_MAX)) {
        ms_series<R, M1>(c0, c1, f0, f1, f2);
    } else {
        const ExpCoef f = ms_coefficients((double)c0, (double)c1);
        f0 = cx(from_d<R>(M1 ? f.f0r - 1.0 : f.f0r), from_d<R>(f.f0i));
        f1 = cx(from_d<R>(f.f1r), from_d<R>(f.f1i));
        f2 = cx(from_d<R>(f.f2r), from_d<R>(f.f2i));
    }
    return ms_combine(Q, S, f0, f1, f2);
}

// ---------------------------------------------------------------------------
// Alternates on full complex matrices (R = double or float)
// ---------------------------------------------------------------------------
template <typename R> GLAC_HD Cx<R> cdivR(Cx<R> a, Cx<R> b) {
    R d = b.re * b.re + b.im * b.im;
    return cx((a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d);
}
template <typename R> GLAC_HD Cx<R> cscale(Cx<R> a, R s) { return cx(a.re * s, a.im * s); }
template <typename R> GLAC_HD Cx<R> cadd_r(Cx<R> a, R s) { return cx(a.re + s, a.im); }

// Luscher's product of SU(2)-block Cayley factors (hep-lat/0409106, App. A).
template <typename R> GLAC_HD M3<R> expm_luscher(const M3<R> &Q) {
    const R third = R(1) / R(3);
    Cx<R> x1 = cscale(Q(0, 0) - Q(1, 1), third), x2 = cscale(Q(0, 0) - Q(2, 2), third),
          x3 = cscale(Q(1, 1) - Q(2, 2), third);
    Cx<R> p12 = Q(0, 1) * Q(1, 0), p13 = Q(0, 2) * Q(2, 0), p23 = Q(1, 2) * Q(2, 1);
    Cx<R> x1s = x1 * x1, x2s = x2 * x2, x3s = x3 * x3;
    const R s16 = R(0.0625), s4 = R(0.25), h = R(0.5);
    Cx<R> d1 = cadd_r(cscale(p12 + x1s, s16), R(-1));
    Cx<R> d2 = cadd_r(cscale(p13 + x2s, s16), R(-1));
    Cx<R> d3 = cadd_r(cscale(p23 + x3s, s4), R(-1));
    M3<R> U1, U2, U3;
    set_zero(U1); set_zero(U2); set_zero(U3);
    Cx<R> one = cx(R(1), R(0));
    Cx<R> t, sq;
    t = cadd_r(cscale(p12, s16) + cscale(x1s, s16) + cscale(x1, h), R(1));
    U1(0, 0) = cdivR(cscale(t, R(-1)), d1);
    U1(0, 1) = cdivR(cscale(Q(0, 1), -h), d1);
    U1(1, 0) = cdivR(cscale(Q(1, 0), -h), d1);
    sq = cadd_r(cscale(x1, s4), R(-1)); sq = sq * sq;
    U1(1, 1) = cdivR(cscale(cscale(p12, s16) + sq, R(-1)), d1);
    U1(2, 2) = one;
    t = cadd_r(cscale(p13, s16) + cscale(x2s, s16) + cscale(x2, h), R(1));
    U2(0, 0) = cdivR(cscale(t, R(-1)), d2);
    U2(0, 2) = cdivR(cscale(Q(0, 2), -h), d2);
    U2(1, 1) = one;
    U2(2, 0) = cdivR(cscale(Q(2, 0), -h), d2);
    sq = cadd_r(cscale(x2, s4), R(-1)); sq = sq * sq;
    U2(2, 2) = cdivR(cscale(cscale(p13, s16) + sq, R(-1)), d2);
    U3(0, 0) = one;
    t = cadd_r(cscale(p23, s4) + cscale(x3s, s4) + x3, R(1));
    U3(1, 1) = cdivR(cscale(t, R(-1)), d3);
    U3(1, 2) = cdivR(cscale(Q(1, 2), R(-1)), d3);
    U3(2, 1) = cdivR(cscale(Q(2, 1), R(-1)), d3);
    sq = cadd_r(cscale(x3, h), R(-1)); sq = sq * sq;
    U3(2, 2) = cdivR(cscale(cscale(p23, s4) + sq, R(-1)), d3);
    M3<R> E = mul(U1, U2);
    E = mul(E, U3);
    E = mul(E, U2);
    return mul(E, U1);
}

// Truncated Taylor series I + Q + ... + Q^deg/deg!
template <typename R> GLAC_HD M3<R> expm_taylor(const M3<R> &Q, int deg) {
    M3<R> S, P;
    set_identity(S);
    set_identity(P);
    R fact = R(1);
    for (int k = 1; k <= deg; k++) {
        P = mul(P, Q);
        fact *= R(k);
        R inv = R(1) / fact;
#pragma unroll
        for (int e = 0; e < 9; e++) S.e[e] = S.e[e] + cscale(P.e[e], inv);
    }
    return S;
}

template <typename R> GLAC_HD M3<R> expm(int kind, const AH8<R> &Z) {
    if (kind == EXP_MORNINGSTAR) return expm_morningstar<R>(Z);
    M3<R> M = ah_to_m3(Z);
    if (kind == EXP_LUSCHER) return expm_luscher(M);
    return expm_taylor(M, kind == EXP_TAYLOR2 ? 2 : 4);
}

}  // namespace glac
