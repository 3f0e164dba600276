// SU(3) algebra for the device kernels (also compiles for the host).
//
// A matrix is 9 complex numbers, row-major, matching the reference element
// order (i,j) -> re [6i+2j], im [6i+2j+1] (GLAC/math/matrices/su3.h:18-22).
// The real type R is a template parameter: double (FP64 path) or float (FP32
// path).
#pragma once

#include <cuda_runtime.h>
#include <math.h>

#define GLAC_HD __host__ __device__ __forceinline__

namespace glac {

GLAC_HD double fmaR(double a, double b, double c) { return fma(a, b, c); }
GLAC_HD float fmaR(float a, float b, float c) { return fmaf(a, b, c); }

template <typename R> GLAC_HD R rzero() { return R(0); }

// ---------------------------------------------------------------------------
// Complex numbers and 3x3 complex matrices
// ---------------------------------------------------------------------------
template <typename R>
struct Cx {
    R re, im;
};

template <typename R> GLAC_HD Cx<R> cx(R a, R b) { Cx<R> z; z.re = a; z.im = b; return z; }
template <typename R> GLAC_HD Cx<R> operator+(Cx<R> a, Cx<R> b) { return cx(a.re + b.re, a.im + b.im); }
template <typename R> GLAC_HD Cx<R> operator-(Cx<R> a, Cx<R> b) { return cx(a.re - b.re, a.im - b.im); }
template <typename R> GLAC_HD Cx<R> operator-(Cx<R> a) { return cx(-a.re, -a.im); }
template <typename R> GLAC_HD Cx<R> conj(Cx<R> a) { return cx(a.re, -a.im); }
template <typename R> GLAC_HD Cx<R> operator*(Cx<R> a, Cx<R> b) {
    return cx(fmaR(a.re, b.re, -(a.im * b.im)), fmaR(a.re, b.im, a.im * b.re));
}
// acc + a*b
template <typename R> GLAC_HD Cx<R> cmac(Cx<R> acc, Cx<R> a, Cx<R> b) {
    acc.re = fmaR(a.re, b.re, acc.re);
    acc.re = fmaR(-a.im, b.im, acc.re);
    acc.im = fmaR(a.re, b.im, acc.im);
    acc.im = fmaR(a.im, b.re, acc.im);
    return acc;
}
// acc + conj(a)*b
template <typename R> GLAC_HD Cx<R> cmac_cj(Cx<R> acc, Cx<R> a, Cx<R> b) {
    acc.re = fmaR(a.re, b.re, acc.re);
    acc.re = fmaR(a.im, b.im, acc.re);
    acc.im = fmaR(a.re, b.im, acc.im);
    acc.im = fmaR(-a.im, b.re, acc.im);
    return acc;
}
// acc + a*conj(b)
template <typename R> GLAC_HD Cx<R> cmac_bc(Cx<R> acc, Cx<R> a, Cx<R> b) {
    acc.re = fmaR(a.re, b.re, acc.re);
    acc.re = fmaR(a.im, b.im, acc.re);
    acc.im = fmaR(-a.re, b.im, acc.im);
    acc.im = fmaR(a.im, b.re, acc.im);
    return acc;
}
// acc + conj(a)*conj(b)
template <typename R> GLAC_HD Cx<R> cmac_cc(Cx<R> acc, Cx<R> a, Cx<R> b) {
    acc.re = fmaR(a.re, b.re, acc.re);
    acc.re = fmaR(-a.im, b.im, acc.re);
    acc.im = fmaR(-a.re, b.im, acc.im);
    acc.im = fmaR(-a.im, b.re, acc.im);
    return acc;
}

template <typename R>
struct M3 {
    Cx<R> e[9];  // row-major
    GLAC_HD Cx<R> &operator()(int i, int j) { return e[3 * i + j]; }
    GLAC_HD const Cx<R> &operator()(int i, int j) const { return e[3 * i + j]; }
};

template <typename R> GLAC_HD void set_zero(M3<R> &a) {
#pragma unroll
    for (int k = 0; k < 9; k++) { a.e[k].re = rzero<R>(); a.e[k].im = rzero<R>(); }
}
template <typename R> GLAC_HD void set_identity(M3<R> &a) {
    set_zero(a);
    a.e[0].re = R(1.f); a.e[4].re = R(1.f); a.e[8].re = R(1.f);
}
// C = A B
template <typename R> GLAC_HD M3<R> mul(const M3<R> &A, const M3<R> &B) {
    M3<R> C;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s = A(i, 0) * B(0, j);
            s = cmac(s, A(i, 1), B(1, j));
            s = cmac(s, A(i, 2), B(2, j));
            C(i, j) = s;
        }
    return C;
}
// C = A B^+
template <typename R> GLAC_HD M3<R> mul_nd(const M3<R> &A, const M3<R> &B) {
    M3<R> C;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s; s.re = rzero<R>(); s.im = rzero<R>();
            s = cmac_bc(s, A(i, 0), B(j, 0));
            s = cmac_bc(s, A(i, 1), B(j, 1));
            s = cmac_bc(s, A(i, 2), B(j, 2));
            C(i, j) = s;
        }
    return C;
}
// C = A^+ B
template <typename R> GLAC_HD M3<R> mul_dn(const M3<R> &A, const M3<R> &B) {
    M3<R> C;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s; s.re = rzero<R>(); s.im = rzero<R>();
            s = cmac_cj(s, A(0, i), B(0, j));
            s = cmac_cj(s, A(1, i), B(1, j));
            s = cmac_cj(s, A(2, i), B(2, j));
            C(i, j) = s;
        }
    return C;
}
// C = A^+ B^+
template <typename R> GLAC_HD M3<R> mul_dd(const M3<R> &A, const M3<R> &B) {
    M3<R> C;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s; s.re = rzero<R>(); s.im = rzero<R>();
            s = cmac_cc(s, A(0, i), B(j, 0));
            s = cmac_cc(s, A(1, i), B(j, 1));
            s = cmac_cc(s, A(2, i), B(j, 2));
            C(i, j) = s;
        }
    return C;
}
// Products of two SU(3) matrices: the first two rows by the product, the third
// as conj(row 0 x row 1), which every SU(3) matrix satisfies (the rows are
// orthonormal and det = 1); 96 multiply-adds instead of 108.  For factors that
// are SU(3) to rounding, the third row differs from the full product's by the
// factors' distance from SU(3).
// conj(a b - c d)
template <typename R> GLAC_HD Cx<R> conj_cross(Cx<R> a, Cx<R> b, Cx<R> c, Cx<R> d) {
    Cx<R> r;
    r.re = a.re * b.re;
    r.re = fmaR(-a.im, b.im, r.re);
    r.re = fmaR(-c.re, d.re, r.re);
    r.re = fmaR(c.im, d.im, r.re);
    r.im = (-a.re) * b.im;
    r.im = fmaR(-a.im, b.re, r.im);
    r.im = fmaR(c.re, d.im, r.im);
    r.im = fmaR(c.im, d.re, r.im);
    return r;
}
template <typename R> GLAC_HD void su3_third_row(M3<R> &C) {
    C(2, 0) = conj_cross(C(0, 1), C(1, 2), C(0, 2), C(1, 1));
    C(2, 1) = conj_cross(C(0, 2), C(1, 0), C(0, 0), C(1, 2));
    C(2, 2) = conj_cross(C(0, 0), C(1, 1), C(0, 1), C(1, 0));
}
// C = A B^+, A and B in SU(3)
template <typename R> GLAC_HD M3<R> mul_nd_su3(const M3<R> &A, const M3<R> &B) {
    M3<R> C;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s; s.re = rzero<R>(); s.im = rzero<R>();
            s = cmac_bc(s, A(i, 0), B(j, 0));
            s = cmac_bc(s, A(i, 1), B(j, 1));
            s = cmac_bc(s, A(i, 2), B(j, 2));
            C(i, j) = s;
        }
    su3_third_row(C);
    return C;
}
// C = A^+ B^+, A and B in SU(3)
template <typename R> GLAC_HD M3<R> mul_dd_su3(const M3<R> &A, const M3<R> &B) {
    M3<R> C;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s; s.re = rzero<R>(); s.im = rzero<R>();
            s = cmac_cc(s, A(0, i), B(j, 0));
            s = cmac_cc(s, A(1, i), B(j, 1));
            s = cmac_cc(s, A(2, i), B(j, 2));
            C(i, j) = s;
        }
    su3_third_row(C);
    return C;
}
// C = A B, A and B in SU(3)
template <typename R> GLAC_HD M3<R> mul_su3(const M3<R> &A, const M3<R> &B) {
    M3<R> C;
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s = A(i, 0) * B(0, j);
            s = cmac(s, A(i, 1), B(1, j));
            s = cmac(s, A(i, 2), B(2, j));
            C(i, j) = s;
        }
    su3_third_row(C);
    return C;
}

// Acc += A B^+  (fused accumulate, no temporary)
template <typename R> GLAC_HD void acc_mul_nd(M3<R> &Acc, const M3<R> &A, const M3<R> &B) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s = Acc(i, j);
            s = cmac_bc(s, A(i, 0), B(j, 0));
            s = cmac_bc(s, A(i, 1), B(j, 1));
            s = cmac_bc(s, A(i, 2), B(j, 2));
            Acc(i, j) = s;
        }
}
// Acc += A^+ B^+  (fused accumulate, no temporary)
template <typename R> GLAC_HD void acc_mul_dd(M3<R> &Acc, const M3<R> &A, const M3<R> &B) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s = Acc(i, j);
            s = cmac_cc(s, A(0, i), B(j, 0));
            s = cmac_cc(s, A(1, i), B(j, 1));
            s = cmac_cc(s, A(2, i), B(j, 2));
            Acc(i, j) = s;
        }
}
// Acc += A B
// D U + U with each element's small sum D(i,:) U(:,j) formed first and U(i,j)
// added last (one rounding at the magnitude of U); column by column, so a
// column of U is dead once its three outputs are done.
template <typename R> GLAC_HD M3<R> mul_plus_right(const M3<R> &D, const M3<R> &U) {
    M3<R> V;
#pragma unroll
    for (int j = 0; j < 3; j++)
#pragma unroll
        for (int i = 0; i < 3; i++) {
            Cx<R> t = D(i, 0) * U(0, j);
            t = cmac(t, D(i, 1), U(1, j));
            t = cmac(t, D(i, 2), U(2, j));
            V(i, j) = t + U(i, j);
        }
    return V;
}

template <typename R> GLAC_HD void acc_mul(M3<R> &Acc, const M3<R> &A, const M3<R> &B) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s = Acc(i, j);
            s = cmac(s, A(i, 0), B(0, j));
            s = cmac(s, A(i, 1), B(1, j));
            s = cmac(s, A(i, 2), B(2, j));
            Acc(i, j) = s;
        }
}
// Acc -= A B
template <typename R> GLAC_HD void sub_mul(M3<R> &Acc, const M3<R> &A, const M3<R> &B) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s = Acc(i, j);
            s = cmac(s, -A(i, 0), B(0, j));
            s = cmac(s, -A(i, 1), B(1, j));
            s = cmac(s, -A(i, 2), B(2, j));
            Acc(i, j) = s;
        }
}
// Acc -= A B^+
template <typename R> GLAC_HD void sub_mul_nd(M3<R> &Acc, const M3<R> &A, const M3<R> &B) {
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            Cx<R> s = Acc(i, j);
            s = cmac_bc(s, -A(i, 0), B(j, 0));
            s = cmac_bc(s, -A(i, 1), B(j, 1));
            s = cmac_bc(s, -A(i, 2), B(j, 2));
            Acc(i, j) = s;
        }
}
template <typename R> GLAC_HD M3<R> dagger(const M3<R> &A) {
    M3<R> B;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) B(i, j) = conj(A(j, i));
    return B;
}
template <typename R> GLAC_HD void add_to(M3<R> &A, const M3<R> &B) {
#pragma unroll
    for (int k = 0; k < 9; k++) A.e[k] = A.e[k] + B.e[k];
}
template <typename R> GLAC_HD void sub_from(M3<R> &A, const M3<R> &B) {
#pragma unroll
    for (int k = 0; k < 9; k++) A.e[k] = A.e[k] - B.e[k];
}
// Re Tr(A B)
template <typename R> GLAC_HD R retr_mul(const M3<R> &A, const M3<R> &B) {
    R s = rzero<R>();
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int k = 0; k < 3; k++) {
            s = fmaR(A(i, k).re, B(k, i).re, s);
            s = fmaR(-A(i, k).im, B(k, i).im, s);
        }
    return s;
}
template <typename R> GLAC_HD R retr(const M3<R> &A) { return A.e[0].re + A.e[4].re + A.e[8].re; }

// ---------------------------------------------------------------------------
// Traceless anti-Hermitian matrices in 8 reals:
//   Z = [[ i a,    b,      c    ],
//        [ -b*,    i d,    e    ],
//        [ -c*,    -e*,  -i(a+d)]]
// ---------------------------------------------------------------------------
template <typename R>
struct AH8 {
    R a, d;
    Cx<R> b, c, e;
};

// Z = 1/2 [(X^+ - X) - 1/3 i ImTr(X^+ - X)] (GLAC/actions/wilsongaugeaction.cpp:78-85)
template <typename R> GLAC_HD AH8<R> project_ah(const M3<R> &X) {
    AH8<R> Z;
    // (X^+ - X)_ii = -2 i Im X_ii ; trace part removed afterwards
    R d0 = -(X(0, 0).im + X(0, 0).im), d1 = -(X(1, 1).im + X(1, 1).im), d2 = -(X(2, 2).im + X(2, 2).im);
    R tr = (d0 + d1 + d2) * R(1.f / 3.f);
    Z.a = (d0 - tr) * R(0.5f);
    Z.d = (d1 - tr) * R(0.5f);
    // (X^+ - X)_ij = conj(X_ji) - X_ij
    Z.b = cx((X(1, 0).re - X(0, 1).re) * R(0.5f), (-X(1, 0).im - X(0, 1).im) * R(0.5f));
    Z.c = cx((X(2, 0).re - X(0, 2).re) * R(0.5f), (-X(2, 0).im - X(0, 2).im) * R(0.5f));
    Z.e = cx((X(2, 1).re - X(1, 2).re) * R(0.5f), (-X(2, 1).im - X(1, 2).im) * R(0.5f));
    return Z;
}
template <> GLAC_HD AH8<double> project_ah<double>(const M3<double> &X) {
    AH8<double> Z;
    double d0 = -(X(0, 0).im + X(0, 0).im), d1 = -(X(1, 1).im + X(1, 1).im), d2 = -(X(2, 2).im + X(2, 2).im);
    double tr = (d0 + d1 + d2) / 3.0;
    Z.a = (d0 - tr) * 0.5;
    Z.d = (d1 - tr) * 0.5;
    Z.b = cx((X(1, 0).re - X(0, 1).re) * 0.5, (-X(1, 0).im - X(0, 1).im) * 0.5);
    Z.c = cx((X(2, 0).re - X(0, 2).re) * 0.5, (-X(2, 0).im - X(0, 2).im) * 0.5);
    Z.e = cx((X(2, 1).re - X(1, 2).re) * 0.5, (-X(2, 1).im - X(1, 2).im) * 0.5);
    return Z;
}

template <typename R> GLAC_HD M3<R> ah_to_m3(const AH8<R> &Z) {
    M3<R> M;
    R z = rzero<R>();
    M(0, 0) = cx(z, Z.a);
    M(1, 1) = cx(z, Z.d);
    M(2, 2) = cx(z, -(Z.a + Z.d));
    M(0, 1) = Z.b; M(0, 2) = Z.c; M(1, 2) = Z.e;
    M(1, 0) = cx(-Z.b.re, Z.b.im);
    M(2, 0) = cx(-Z.c.re, Z.c.im);
    M(2, 1) = cx(-Z.e.re, Z.e.im);
    return M;
}
// alpha*Z + beta*W
template <typename R> GLAC_HD AH8<R> ah_axpby(R alpha, const AH8<R> &Z, R beta, const AH8<R> &W) {
    AH8<R> r;
    r.a = fmaR(alpha, Z.a, beta * W.a);
    r.d = fmaR(alpha, Z.d, beta * W.d);
    r.b = cx(fmaR(alpha, Z.b.re, beta * W.b.re), fmaR(alpha, Z.b.im, beta * W.b.im));
    r.c = cx(fmaR(alpha, Z.c.re, beta * W.c.re), fmaR(alpha, Z.c.im, beta * W.c.im));
    r.e = cx(fmaR(alpha, Z.e.re, beta * W.e.re), fmaR(alpha, Z.e.im, beta * W.e.im));
    return r;
}
template <typename R> GLAC_HD AH8<R> ah_scale(R alpha, const AH8<R> &Z) {
    AH8<R> r;
    r.a = alpha * Z.a; r.d = alpha * Z.d;
    r.b = cx(alpha * Z.b.re, alpha * Z.b.im);
    r.c = cx(alpha * Z.c.re, alpha * Z.c.im);
    r.e = cx(alpha * Z.e.re, alpha * Z.e.im);
    return r;
}

}  // namespace glac
