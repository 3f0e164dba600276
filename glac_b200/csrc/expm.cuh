// SU(3) exponentials of traceless anti-Hermitian matrices.
//
// Default: Morningstar-Peardon Cayley-Hamilton form (hep-lat/0311018), the
// reference's "morningstar" (GLAC/math/exponentiation/su3exp.cpp:16-79).
// With Q = -i Z (Hermitian, traceless), exp(Z) = exp(iQ) = f0 + f1 Q + f2 Q^2,
// c0 = det Q = Tr(Q^3)/3, c1 = Tr(Q^2)/2.  The scalar coefficients f_j are
// always evaluated in FP64 -- also on the FP32 path, where the matrix algebra
// stays in FP32; this keeps the near-degenerate region (theta -> 0, where acos
// is ill-conditioned, and small |Q|, where the h_j cancel) accurate.
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

// c1 = Tr(Q^2)/2 and c0 = Tr(Q Q^2)/3 evaluated in FP64.
GLAC_HD void ms_invariants(double q0, double q1, double q2, double xr, double xi, double yr, double yi, double zr,
                           double zi, double s0, double s1, double s2, double sxr, double sxi, double syr,
                           double syi, double szr, double szi, double &c0, double &c1) {
    c1 = 0.5 * (s0 + s1 + s2);
    // Tr(Q S) = sum_i q_i s_i + 2 Re(x conj(Sx) + y conj(Sy) + z conj(Sz))
    double t = q0 * s0 + q1 * s1 + q2 * s2;
    t += 2.0 * (xr * sxr + xi * sxi + yr * syr + yi * syi + zr * szr + zi * szi);
    c0 = t * 0.3333333333333333;
}

template <typename R> GLAC_HD ExpCoef coef_of(const HQ<R> &Q, const HQ2<R> &S);
template <> GLAC_HD ExpCoef coef_of<double>(const HQ<double> &Q, const HQ2<double> &S) {
    double c0, c1;
    ms_invariants(Q.q0, Q.q1, Q.q2, Q.x.re, Q.x.im, Q.y.re, Q.y.im, Q.z.re, Q.z.im, S.d0, S.d1, S.d2, S.x.re,
                  S.x.im, S.y.re, S.y.im, S.z.re, S.z.im, c0, c1);
    return ms_coefficients(c0, c1);
}
template <> GLAC_HD ExpCoef coef_of<float>(const HQ<float> &Q, const HQ2<float> &S) {
    double c0, c1;
    ms_invariants(Q.q0, Q.q1, Q.q2, Q.x.re, Q.x.im, Q.y.re, Q.y.im, Q.z.re, Q.z.im, S.d0, S.d1, S.d2, S.x.re,
                  S.x.im, S.y.re, S.y.im, S.z.re, S.z.im, c0, c1);
    return ms_coefficients(c0, c1);
}

template <typename R> GLAC_HD R from_d(double v);
template <> GLAC_HD double from_d<double>(double v) { return v; }
template <> GLAC_HD float from_d<float>(double v) { return (float)v; }

// exp(Z) as a full matrix (f0 + f1 Q + f2 Q^2).
template <typename R> GLAC_HD M3<R> ms_expm_from(const HQ<R> &Q, const HQ2<R> &S, const ExpCoef &f) {
    Cx<R> f0 = cx(from_d<R>(f.f0r), from_d<R>(f.f0i));
    Cx<R> f1 = cx(from_d<R>(f.f1r), from_d<R>(f.f1i));
    Cx<R> f2 = cx(from_d<R>(f.f2r), from_d<R>(f.f2i));
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

template <typename R> GLAC_HD M3<R> expm_morningstar(const AH8<R> &Z) {
    HQ<R> Q = herm_from_ah(Z);
    HQ2<R> S = herm_square(Q);
    ExpCoef f = coef_of(Q, S);
    return ms_expm_from(Q, S, f);
}

// Packed pair: coefficients per lane in FP64, matrix algebra in packed FP32.
GLAC_HD M3<f32x2> expm_morningstar_pair(const AH8<f32x2> &Z) {
    HQ<f32x2> Q = herm_from_ah(Z);
    HQ2<f32x2> S = herm_square(Q);
    double c0x, c1x, c0y, c1y;
    ms_invariants(Q.q0.v.x, Q.q1.v.x, Q.q2.v.x, Q.x.re.v.x, Q.x.im.v.x, Q.y.re.v.x, Q.y.im.v.x, Q.z.re.v.x,
                  Q.z.im.v.x, S.d0.v.x, S.d1.v.x, S.d2.v.x, S.x.re.v.x, S.x.im.v.x, S.y.re.v.x, S.y.im.v.x,
                  S.z.re.v.x, S.z.im.v.x, c0x, c1x);
    ms_invariants(Q.q0.v.y, Q.q1.v.y, Q.q2.v.y, Q.x.re.v.y, Q.x.im.v.y, Q.y.re.v.y, Q.y.im.v.y, Q.z.re.v.y,
                  Q.z.im.v.y, S.d0.v.y, S.d1.v.y, S.d2.v.y, S.x.re.v.y, S.x.im.v.y, S.y.re.v.y, S.y.im.v.y,
                  S.z.re.v.y, S.z.im.v.y, c0y, c1y);
    ExpCoef a = ms_coefficients(c0x, c1x), b = ms_coefficients(c0y, c1y);
    Cx<f32x2> f0 = cx(f32x2((float)a.f0r, (float)b.f0r), f32x2((float)a.f0i, (float)b.f0i));
    Cx<f32x2> f1 = cx(f32x2((float)a.f1r, (float)b.f1r), f32x2((float)a.f1i, (float)b.f1i));
    Cx<f32x2> f2 = cx(f32x2((float)a.f2r, (float)b.f2r), f32x2((float)a.f2i, (float)b.f2i));
    M3<f32x2> E;
    E(0, 0) = cx(fmaR(f1.re, Q.q0, fmaR(f2.re, S.d0, f0.re)), fmaR(f1.im, Q.q0, fmaR(f2.im, S.d0, f0.im)));
    E(1, 1) = cx(fmaR(f1.re, Q.q1, fmaR(f2.re, S.d1, f0.re)), fmaR(f1.im, Q.q1, fmaR(f2.im, S.d1, f0.im)));
    E(2, 2) = cx(fmaR(f1.re, Q.q2, fmaR(f2.re, S.d2, f0.re)), fmaR(f1.im, Q.q2, fmaR(f2.im, S.d2, f0.im)));
    E(0, 1) = cmac(f1 * Q.x, f2, S.x);
    E(1, 0) = cmac(f1 * conj(Q.x), f2, conj(S.x));
    E(0, 2) = cmac(f1 * Q.y, f2, S.y);
    E(2, 0) = cmac(f1 * conj(Q.y), f2, conj(S.y));
    E(1, 2) = cmac(f1 * Q.z, f2, S.z);
    E(2, 1) = cmac(f1 * conj(Q.z), f2, conj(S.z));
    return E;
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
    if (kind == EXP_MORNINGSTAR) return expm_morningstar(Z);
    M3<R> M = ah_to_m3(Z);
    if (kind == EXP_LUSCHER) return expm_luscher(M);
    return expm_taylor(M, kind == EXP_TAYLOR2 ? 2 : 4);
}

}  // namespace glac
