/*
 * CPU restatement of GLAC's pure-gauge SU(3) hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker for tests/, smoke() and bench.py's
 * CPU leg).  Every function cites the reference file:line it restates; the
 * project-only parts (Philox, checkerboard sweep, Haar start, reunitarisation)
 * say so.  Written as plain loops for clarity, not speed.
 */
#include "glac_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ------------------------------------------------------------------ */
/* 3x3 complex helpers; m[6i+2j] = Re m_ij, m[6i+2j+1] = Im m_ij       */
/* ------------------------------------------------------------------ */
typedef struct { double re, im; } cplx;

static cplx cmul(cplx a, cplx b) { cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re}; return r; }
static cplx cdiv(cplx a, cplx b) {
    double d = b.re * b.re + b.im * b.im;
    cplx r = {(a.re * b.re + a.im * b.im) / d, (a.im * b.re - a.re * b.im) / d};
    return r;
}
static cplx el(const double *m, int i, int j) { cplx r = {m[6 * i + 2 * j], m[6 * i + 2 * j + 1]}; return r; }
static void setel(double *m, int i, int j, cplx v) { m[6 * i + 2 * j] = v.re; m[6 * i + 2 * j + 1] = v.im; }

/* C = A B (GLAC/math/matrices/su3.h:184-215). */
static void mm(const double *A, const double *B, double *C) {
    double T[18];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            cplx s = {0.0, 0.0};
            for (int k = 0; k < 3; k++) {
                cplx p = cmul(el(A, i, k), el(B, k, j));
                s.re += p.re;
                s.im += p.im;
            }
            setel(T, i, j, s);
        }
    memcpy(C, T, sizeof(T));
}
/* B = A^dagger (GLAC/math/matrices/su3.h:307-329). */
static void dag(const double *A, double *B) {
    double T[18];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            cplx v = el(A, j, i);
            v.im = -v.im;
            setel(T, i, j, v);
        }
    memcpy(B, T, sizeof(T));
}
static void madd(double *A, const double *B) { for (int i = 0; i < 18; i++) A[i] += B[i]; }
static void msub(double *A, const double *B) { for (int i = 0; i < 18; i++) A[i] -= B[i]; }
static void mscale(double *A, double s) { for (int i = 0; i < 18; i++) A[i] *= s; }
static void mident(double *A) { memset(A, 0, 18 * sizeof(double)); A[0] = A[8] = A[16] = 1.0; }
/* Re Tr(A B) (GLAC/math/functions.h:45-53). */
static double retr_mul(const double *A, const double *B) {
    double s = 0.0;
    for (int i = 0; i < 3; i++)
        for (int k = 0; k < 3; k++) s += cmul(el(A, i, k), el(B, k, i)).re;
    return s;
}
static double retr(const double *A) { return A[0] + A[8] + A[16]; }
static double imtr(const double *A) { return A[1] + A[9] + A[17]; }

/* (C - C^dagger) made traceless on the imaginary diagonal; the reference's
 * projection (GLAC/observables/mastersamplertopcxyz.cpp:330-340). */
static void antiherm_traceless(double *C) {
    double D[18];
    dag(C, D);
    msub(C, D);
    double d = imtr(C) / 3.0;
    C[1] -= d;
    C[9] -= d;
    C[17] -= d;
}

void oracle_su3_mul(const double *A, const double *B, double *C) { mm(A, B, C); }
void oracle_su3_dagger(const double *A, double *B) { dag(A, B); }
double oracle_retr_mul(const double *A, const double *B) { return retr_mul(A, B); }

/* ------------------------------------------------------------------ */
/* Lattice indexing: x + Nx(y + Ny(z + Nz t)) (GLAC/parallelization/index.h:32-35) */
/* ------------------------------------------------------------------ */
static long site_of(const int N[4], const int c[4]) {
    return c[0] + (long)N[0] * (c[1] + (long)N[1] * (c[2] + (long)N[2] * c[3]));
}
static void coords_of(const int N[4], long s, int c[4]) {
    for (int d = 0; d < 4; d++) { c[d] = (int)(s % N[d]); s /= N[d]; }
}
/* Site n + a*e_da + b*e_db, periodic (replaces the MPI neighbour getters,
 * GLAC/parallelization/communicator.cpp:83-266). */
static long nbr(const int N[4], const int c[4], int da, int a, int db, int b) {
    int e[4] = {c[0], c[1], c[2], c[3]};
    if (da >= 0) e[da] = (e[da] + a + N[da]) % N[da];
    if (db >= 0) e[db] = (e[db] + b + N[db]) % N[db];
    return site_of(N, e);
}
#define LINK(links, V, mu, s) ((links) + ((long)(mu) * (V) + (s)) * 18)

/* Staple for U_mu(n) (GLAC/actions/wilsongaugeaction.cpp:29-53):
 *   sum_{nu != mu} U_nu(n+mu) U_mu(n+nu)^+ U_nu(n)^+  +  U_nu(n+mu-nu)^+ U_mu(n-nu)^+ U_nu(n-nu). */
static void staple_at(const int N[4], long V, const double *links, const int c[4], int mu, double *A) {
    memset(A, 0, 18 * sizeof(double));
    long n = site_of(N, c);
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        double T1[18], T2[18], D[18];
        /* upper */
        dag(LINK(links, V, mu, nbr(N, c, nu, 1, -1, 0)), D);
        mm(LINK(links, V, nu, nbr(N, c, mu, 1, -1, 0)), D, T1);
        dag(LINK(links, V, nu, n), D);
        mm(T1, D, T1);
        /* lower */
        dag(LINK(links, V, nu, nbr(N, c, mu, 1, nu, -1)), T2);
        dag(LINK(links, V, mu, nbr(N, c, nu, -1, -1, 0)), D);
        mm(T2, D, T2);
        mm(T2, LINK(links, V, nu, nbr(N, c, nu, -1, -1, 0)), T2);
        madd(A, T1);
        madd(A, T2);
    }
}

void oracle_staples(const int N[4], const double *links, double *out) {
    long V = (long)N[0] * N[1] * N[2] * N[3];
    for (long s = 0; s < V; s++) {
        int c[4];
        coords_of(N, s, c);
        for (int mu = 0; mu < 4; mu++) staple_at(N, V, links, c, mu, LINK(out, V, mu, s));
    }
}

/* GLAC/actions/wilsongaugeaction.cpp:24-27 with factor -beta/3 (:9). */
double oracle_delta_s(const double *U, const double *Uprime, const double *A, double beta) {
    double D[18];
    memcpy(D, Uprime, sizeof(D));
    msub(D, U);
    return retr_mul(D, A) * (-beta / 3.0);
}

/* Z = 1/2 [(X^+ - X) - 1/3 i ImTr(X^+ - X)], X = U_mu A_mu
 * (GLAC/actions/wilsongaugeaction.cpp:55-86). */
static void force_from(const double *U, const double *A, double *Z) {
    double X[18], D[18];
    mm(U, A, X);
    dag(X, D);
    msub(D, X);
    double d = imtr(D) / 3.0;
    D[1] -= d;
    D[9] -= d;
    D[17] -= d;
    mscale(D, 0.5);
    memcpy(Z, D, sizeof(D));
}

void oracle_force(const int N[4], const double *links, double *out) {
    long V = (long)N[0] * N[1] * N[2] * N[3];
    for (long s = 0; s < V; s++) {
        int c[4];
        coords_of(N, s, c);
        for (int mu = 0; mu < 4; mu++) {
            double A[18];
            staple_at(N, V, links, c, mu, A);
            force_from(LINK(links, V, mu, s), A, LINK(out, V, mu, s));
        }
    }
}

/* ------------------------------------------------------------------ */
/* Exponentials                                                        */
/* ------------------------------------------------------------------ */

/* Morningstar-Peardon (hep-lat/0311018), as GLAC/math/exponentiation/su3exp.cpp:16-79:
 * Q = -i Z is Hermitian traceless; exp(Z) = exp(iQ) = f0 + f1 Q + f2 Q^2. */
static void exp_morningstar(const double *Zin, double *out) {
    double Q[18], Q2[18], Q3[18];
    for (int k = 0; k < 9; k++) { /* multiply by -i (su3.h:354-365) */
        Q[2 * k] = Zin[2 * k + 1];
        Q[2 * k + 1] = -Zin[2 * k];
    }
    mm(Q, Q, Q2);
    mm(Q, Q2, Q3);
    double c0 = (Q3[0] + Q3[8] + Q3[16]) / 3.0;
    double c1 = 0.5 * (Q2[0] + Q2[8] + Q2[16]);
    double c0max = 2.0 / 3.0 * c1 * sqrt(c1 / 3.0);
    double theta = acos(fabs(c0) / c0max);
    double u = sqrt(c1 / 3.0) * cos(theta / 3.0);
    double w = sqrt(c1) * sin(theta / 3.0);
    double uu = u * u, ww = w * w;
    double cu = cos(u), su = sin(u), cw = cos(w), c2u = cos(2 * u), s2u = sin(2 * u);
    double xi0 = fabs(w) > 0.05 ? sin(w) / w : 1.0 - ww * (1.0 - 0.05 * ww * (1.0 - ww / 42.0)) / 6.0;
    cplx h0 = {8 * uu * cu * cw + 2 * u * xi0 * (3 * uu + ww) * su + (uu - ww) * c2u,
               -8 * uu * su * cw + 2 * u * xi0 * (3 * uu + ww) * cu + (uu - ww) * s2u};
    cplx h1 = {-2 * u * cu * cw + 2 * u * c2u + xi0 * (3 * uu - ww) * su,
               2 * u * su * cw + 2 * u * s2u + xi0 * (3 * uu - ww) * cu};
    cplx h2 = {-3 * u * xi0 * su - cu * cw + c2u, -3 * u * xi0 * cu + su * cw + s2u};
    double den = 9 * uu - ww;
    cplx f0 = {h0.re / den, h0.im / den}, f1 = {h1.re / den, h1.im / den}, f2 = {h2.re / den, h2.im / den};
    if (c0 < 0) { /* symmetry c0 -> -c0 */
        f0.im = -f0.im;
        f1.re = -f1.re;
        f2.im = -f2.im;
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            cplx v = cmul(f1, el(Q, i, j));
            cplx v2 = cmul(f2, el(Q2, i, j));
            v.re += v2.re;
            v.im += v2.im;
            if (i == j) { v.re += f0.re; v.im += f0.im; }
            setel(out, i, j, v);
        }
}

/* Luscher (hep-lat/0409106 App. A) as GLAC/math/exponentiation/expluscher.cpp:13-68:
 * product U1 U2 U3 U2 U1 of Cayley-form SU(2)-block factors. */
static void exp_luscher(const double *Q, double *out) {
    cplx q00 = el(Q, 0, 0), q11 = el(Q, 1, 1), q22 = el(Q, 2, 2);
    cplx q01 = el(Q, 0, 1), q10 = el(Q, 1, 0), q02 = el(Q, 0, 2), q20 = el(Q, 2, 0), q12 = el(Q, 1, 2), q21 = el(Q, 2, 1);
    cplx x1 = {(q00.re - q11.re) / 3.0, (q00.im - q11.im) / 3.0};
    cplx x2 = {(q00.re - q22.re) / 3.0, (q00.im - q22.im) / 3.0};
    cplx x3 = {(q11.re - q22.re) / 3.0, (q11.im - q22.im) / 3.0};
    cplx p12 = cmul(q01, q10), p13 = cmul(q02, q20), p23 = cmul(q12, q21);
    cplx x1s = cmul(x1, x1), x2s = cmul(x2, x2), x3s = cmul(x3, x3);
    cplx one = {1.0, 0.0};
    cplx d1 = {(p12.re + x1s.re) / 16.0 - 1.0, (p12.im + x1s.im) / 16.0};
    cplx d2 = {(p13.re + x2s.re) / 16.0 - 1.0, (p13.im + x2s.im) / 16.0};
    cplx d3 = {(p23.re + x3s.re) / 4.0 - 1.0, (p23.im + x3s.im) / 4.0};
    double U1[18] = {0}, U2[18] = {0}, U3[18] = {0};
    cplx a, b;
    /* U1 acts on the (1,2) block */
    a.re = -(p12.re / 16.0 + x1s.re / 16.0 + x1.re / 2.0 + 1.0); a.im = -(p12.im / 16.0 + x1s.im / 16.0 + x1.im / 2.0);
    setel(U1, 0, 0, cdiv(a, d1));
    a.re = -q01.re / 2.0; a.im = -q01.im / 2.0; setel(U1, 0, 1, cdiv(a, d1));
    a.re = -q10.re / 2.0; a.im = -q10.im / 2.0; setel(U1, 1, 0, cdiv(a, d1));
    b.re = x1.re / 4.0 - 1.0; b.im = x1.im / 4.0; b = cmul(b, b);
    a.re = -(p12.re / 16.0 + b.re); a.im = -(p12.im / 16.0 + b.im); setel(U1, 1, 1, cdiv(a, d1));
    setel(U1, 2, 2, one);
    /* U2 acts on the (1,3) block */
    a.re = -(p13.re / 16.0 + x2s.re / 16.0 + x2.re / 2.0 + 1.0); a.im = -(p13.im / 16.0 + x2s.im / 16.0 + x2.im / 2.0);
    setel(U2, 0, 0, cdiv(a, d2));
    a.re = -q02.re / 2.0; a.im = -q02.im / 2.0; setel(U2, 0, 2, cdiv(a, d2));
    setel(U2, 1, 1, one);
    a.re = -q20.re / 2.0; a.im = -q20.im / 2.0; setel(U2, 2, 0, cdiv(a, d2));
    b.re = x2.re / 4.0 - 1.0; b.im = x2.im / 4.0; b = cmul(b, b);
    a.re = -(p13.re / 16.0 + b.re); a.im = -(p13.im / 16.0 + b.im); setel(U2, 2, 2, cdiv(a, d2));
    /* U3 acts on the (2,3) block */
    setel(U3, 0, 0, one);
    a.re = -(p23.re / 4.0 + x3s.re / 4.0 + x3.re + 1.0); a.im = -(p23.im / 4.0 + x3s.im / 4.0 + x3.im);
    setel(U3, 1, 1, cdiv(a, d3));
    a.re = -q12.re; a.im = -q12.im; setel(U3, 1, 2, cdiv(a, d3));
    a.re = -q21.re; a.im = -q21.im; setel(U3, 2, 1, cdiv(a, d3));
    b.re = x3.re / 2.0 - 1.0; b.im = x3.im / 2.0; b = cmul(b, b);
    a.re = -(p23.re / 4.0 + b.re); a.im = -(p23.im / 4.0 + b.im); setel(U3, 2, 2, cdiv(a, d3));
    double E[18];
    mm(U1, U2, E);
    mm(E, U3, E);
    mm(E, U2, E);
    mm(E, U1, E);
    memcpy(out, E, sizeof(E));
}

/* Truncated Taylor series sum_{k<=deg} Q^k/k! (taylor2exp.cpp:8-16,
 * taylor4exp.cpp:8-20, taylorexp.cpp:14-30). */
static void exp_taylor(const double *Q, int deg, double *out) {
    double S[18], P[18];
    mident(S);
    mident(P);
    double fact = 1.0;
    for (int k = 1; k <= deg; k++) {
        mm(P, Q, P);
        fact *= k;
        double T[18];
        memcpy(T, P, sizeof(T));
        mscale(T, 1.0 / fact);
        madd(S, T);
    }
    memcpy(out, S, sizeof(S));
}

static void exp_one(int kind, int degree, const double *in, double *out) {
    switch (kind) {
    case 0: exp_morningstar(in, out); break;
    case 1: exp_luscher(in, out); break;
    case 2: exp_taylor(in, 2, out); break;
    case 3: exp_taylor(in, 4, out); break;
    default: exp_taylor(in, degree > 0 ? degree : 16, out); break;
    }
}

void oracle_exp(int kind, int degree, const double *in, long n, double *out) {
    for (long i = 0; i < n; i++) exp_one(kind, degree, in + 18 * i, out + 18 * i);
}

/* ------------------------------------------------------------------ */
/* Gradient flow: Luscher RK3 (GLAC/flow/flow.cpp:43-73)               */
/* ------------------------------------------------------------------ */
void oracle_flow(const int N[4], double *links, double eps, int nsteps, int expkind) {
    long V = (long)N[0] * N[1] * N[2] * N[3];
    size_t bytes = (size_t)4 * V * 18 * sizeof(double);
    double *Z = (double *)malloc(bytes), *Zn = (double *)malloc(bytes);
    for (int step = 0; step < nsteps; step++) {
        /* Z0 from W0 for all mu before any update (flow.cpp:50-52) */
        oracle_force(N, links, Z);
        for (long k = 0; k < 4 * V; k++) { /* W1 = exp(eps/4 Z0) W0 (flow.cpp:54-56) */
            double M[18], E[18];
            memcpy(M, Z + 18 * k, sizeof(M));
            mscale(M, eps * 0.25);
            exp_one(expkind, 16, M, E);
            mm(E, links + 18 * k, links + 18 * k);
        }
        oracle_force(N, links, Zn);
        for (long k = 0; k < 4 * V; k++) { /* Z1' = 8/9 eps Z1 - 17/36 eps Z0; W2 = exp(Z1') W1 (:58-64) */
            double *z = Z + 18 * k, E[18];
            for (int i = 0; i < 18; i++) z[i] = Zn[18 * k + i] * (eps * 0.8888888888888888) - z[i] * (eps * 0.4722222222222222);
            exp_one(expkind, 16, z, E);
            mm(E, links + 18 * k, links + 18 * k);
        }
        oracle_force(N, links, Zn);
        for (long k = 0; k < 4 * V; k++) { /* Z2' = 3/4 eps Z2 - Z1'; W3 = exp(Z2') W2 (:66-72) */
            double *z = Z + 18 * k, E[18];
            for (int i = 0; i < 18; i++) z[i] = Zn[18 * k + i] * (0.75 * eps) - z[i];
            exp_one(expkind, 16, z, E);
            mm(E, links + 18 * k, links + 18 * k);
        }
    }
    free(Z);
    free(Zn);
}

/* ------------------------------------------------------------------ */
/* Observables (GLAC/observables/mastersamplertopcxyz.cpp:236-384)      */
/* ------------------------------------------------------------------ */

/* Clover in the (mu,nu) plane from its four leaves, before projection
 * (mastersamplertopcxyz.cpp:253-285): leaf1 - leaf2 + leaf3 - leaf4; leaf1 is
 * the plaquette returned in *plaq_leaf. */
static void clover(const int N[4], long V, const double *L, const int c[4], int mu, int nu, double *C, double *plaq_leaf) {
    long n = site_of(N, c);
    double T[18], D[18];
    /* leaf1 = U_mu(n) U_nu(n+mu) U_mu(n+nu)^+ U_nu(n)^+ */
    mm(LINK(L, V, mu, n), LINK(L, V, nu, nbr(N, c, mu, 1, -1, 0)), T);
    dag(LINK(L, V, mu, nbr(N, c, nu, 1, -1, 0)), D); mm(T, D, T);
    dag(LINK(L, V, nu, n), D); mm(T, D, T);
    memcpy(C, T, sizeof(T));
    memcpy(plaq_leaf, T, sizeof(T));
    /* leaf2 = U_mu(n) U_nu(n+mu-nu)^+ U_mu(n-nu)^+ U_nu(n-nu) */
    dag(LINK(L, V, nu, nbr(N, c, mu, 1, nu, -1)), D); mm(LINK(L, V, mu, n), D, T);
    dag(LINK(L, V, mu, nbr(N, c, nu, -1, -1, 0)), D); mm(T, D, T);
    mm(T, LINK(L, V, nu, nbr(N, c, nu, -1, -1, 0)), T);
    msub(C, T);
    /* leaf3 = U_mu(n-mu)^+ U_nu(n-mu-nu)^+ U_mu(n-mu-nu) U_nu(n-nu) */
    dag(LINK(L, V, mu, nbr(N, c, mu, -1, -1, 0)), T);
    dag(LINK(L, V, nu, nbr(N, c, mu, -1, nu, -1)), D); mm(T, D, T);
    mm(T, LINK(L, V, mu, nbr(N, c, mu, -1, nu, -1)), T);
    mm(T, LINK(L, V, nu, nbr(N, c, nu, -1, -1, 0)), T);
    madd(C, T);
    /* leaf4 = U_mu(n-mu)^+ U_nu(n-mu) U_mu(n-mu+nu) U_nu(n)^+ */
    dag(LINK(L, V, mu, nbr(N, c, mu, -1, -1, 0)), T);
    mm(T, LINK(L, V, nu, nbr(N, c, mu, -1, -1, 0)), T);
    mm(T, LINK(L, V, mu, nbr(N, c, mu, -1, nu, 1)), T);
    dag(LINK(L, V, nu, n), D); mm(T, D, T);
    msub(C, T);
}

void oracle_observables(const int N[4], const double *links, double *out) {
    long V = (long)N[0] * N[1] * N[2] * N[3];
    double plaq = 0.0, energy = 0.0;
    double *qt = out + 3;
    for (int t = 0; t < N[3]; t++) qt[t] = 0.0;
    for (long s = 0; s < V; s++) {
        int c[4];
        coords_of(N, s, c);
        for (int nu = 1; nu < 4; nu++) {
            int rho = nu % 3 + 1, sigma = rho % 3 + 1; /* cyclic complement (:286-289) */
            double C1[18], C2[18], P[18];
            clover(N, V, links, c, 0, nu, C1, P);
            plaq += retr(P);
            clover(N, V, links, c, rho, sigma, C2, P);
            plaq += retr(P);
            antiherm_traceless(C1);
            antiherm_traceless(C2);
            qt[c[3]] -= retr_mul(C1, C2);
            energy += retr_mul(C1, C1) + retr_mul(C2, C2);
        }
    }
    double qfac = 1.0 / (16 * 16 * M_PI * M_PI); /* mastersamplertopcxyz.cpp:13-16 */
    double topc = 0.0;
    for (int t = 0; t < N[3]; t++) { topc += qt[t]; qt[t] *= qfac; }
    out[0] = plaq / (18.0 * (double)V);
    out[1] = topc * qfac;
    out[2] = energy / (double)V;
}

/* SuperSampler::calculate (GLAC/observables/supersampler.cpp:298-496):
 * out = [plaq, topc, energy, weinberg, topct[Nt], weinbergt[Nt]].  The six
 * projected clovers per site; for nu = 1..3, temp = sum over spatial lambda != nu
 * of G_{0 lambda} G_{nu lambda} (G_{b a} = G_{a b}^+ where only (a, b) is
 * formed, :421-433), w(t) -= ReTr(temp G_{rho sigma}); factor 2*8*8/(3*16^3) (:13). */
void oracle_weinberg(const int N[4], const double *links, double *out) {
    long V = (long)N[0] * N[1] * N[2] * N[3];
    int Nt = N[3];
    double plaq = 0.0, energy = 0.0;
    double *qt = out + 4, *wt = out + 4 + Nt;
    for (int t = 0; t < Nt; t++) qt[t] = wt[t] = 0.0;
    for (long s = 0; s < V; s++) {
        int c[4];
        coords_of(N, s, c);
        double G[4][4][18]; /* G[a][b], all ordered spatial/temporal pairs that are used */
        for (int nu = 1; nu < 4; nu++) {
            int rho = nu % 3 + 1, sigma = rho % 3 + 1;
            double P[18];
            clover(N, V, links, c, 0, nu, G[0][nu], P);
            plaq += retr(P);
            clover(N, V, links, c, rho, sigma, G[rho][sigma], P);
            plaq += retr(P);
            antiherm_traceless(G[0][nu]);
            antiherm_traceless(G[rho][sigma]);
            dag(G[rho][sigma], G[sigma][rho]);
            qt[c[3]] -= retr_mul(G[0][nu], G[rho][sigma]);
            energy += retr_mul(G[0][nu], G[0][nu]) + retr_mul(G[rho][sigma], G[rho][sigma]);
        }
        for (int nu = 1; nu < 4; nu++) {
            int rho = nu % 3 + 1, sigma = rho % 3 + 1;
            double T[18] = {0}, M[18];
            for (int lam = 1; lam < 4; lam++) {
                if (lam == nu) continue;
                mm(G[0][lam], G[nu][lam], M);
                madd(T, M);
            }
            wt[c[3]] -= retr_mul(T, G[rho][sigma]);
        }
    }
    double qfac = 1.0 / (16 * 16 * M_PI * M_PI), wfac = 2 * 8.0 * 8.0 / (3 * 16 * 16 * 16);
    double topc = 0.0, w = 0.0;
    for (int t = 0; t < Nt; t++) {
        topc += qt[t];
        w += wt[t];
        qt[t] *= qfac;
        wt[t] *= wfac;
    }
    out[0] = plaq / (18.0 * (double)V);
    out[1] = topc * qfac;
    out[2] = energy / (double)V;
    out[3] = w * wfac;
}

/* Per-site densities of LatticeActionChargeDensity::calculate
 * (GLAC/observables/latticeactionchargedensity.cpp:169-306): q[s] = topological
 * charge density with the factor 1/(16^2 pi^2) (:288-291), e[s] = sum of
 * ReTr(C C) over the six planes, unnormalised (:297-305). */
void oracle_density(const int N[4], const double *links, double *q, double *e) {
    long V = (long)N[0] * N[1] * N[2] * N[3];
    double qfac = 1.0 / (16 * 16 * M_PI * M_PI);
    for (long s = 0; s < V; s++) {
        int c[4];
        coords_of(N, s, c);
        double qs = 0.0, es = 0.0;
        for (int nu = 1; nu < 4; nu++) {
            int rho = nu % 3 + 1, sigma = rho % 3 + 1;
            double C1[18], C2[18], P[18];
            clover(N, V, links, c, 0, nu, C1, P);
            clover(N, V, links, c, rho, sigma, C2, P);
            antiherm_traceless(C1);
            antiherm_traceless(C2);
            qs -= retr_mul(C1, C2);
            es += retr_mul(C1, C1) + retr_mul(C2, C2);
        }
        q[s] = qs * qfac;
        e[s] = es;
    }
}

/* Plaquette (GLAC/observables/plaquette.cpp:26-40), factor 1/(18V) (:23). */
double oracle_plaquette(const int N[4], const double *links) {
    long V = (long)N[0] * N[1] * N[2] * N[3];
    double sum = 0.0;
    for (long s = 0; s < V; s++) {
        int c[4];
        coords_of(N, s, c);
        for (int mu = 0; mu < 4; mu++)
            for (int nu = mu + 1; nu < 4; nu++) {
                double T[18], D[18];
                mm(LINK(links, V, mu, s), LINK(links, V, nu, nbr(N, c, mu, 1, -1, 0)), T);
                dag(LINK(links, V, mu, nbr(N, c, nu, 1, -1, 0)), D); mm(T, D, T);
                dag(LINK(links, V, nu, s), D); mm(T, D, T);
                sum += retr(T);
            }
    }
    return sum / (18.0 * (double)V);
}

/* ------------------------------------------------------------------ */
/* Metropolis proposals and accept step                                 */
/* ------------------------------------------------------------------ */

/* SU(2) near unity (GLAC/math/matrices/su3matrixgenerator.h:202-243):
 * x0 = sign(u0) sqrt(1-eps^2), x = eps u/|u|, normalised; U = x0 + i x.sigma. */
void oracle_su2_near_unity(const double u[4], double eps, double out8[8]) {
    double x[4];
    x[0] = (u[0] < 0 ? -1.0 : 1.0) * sqrt(1.0 - eps * eps);
    double rn = sqrt(u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) / eps;
    for (int i = 1; i < 4; i++) x[i] = u[i] / rn;
    double nrm = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + x[3] * x[3]);
    for (int i = 0; i < 4; i++) x[i] /= nrm;
    /* [[x0 + i x3, x2 + i x1], [-x2 + i x1, x0 - i x3]] */
    out8[0] = x[0]; out8[1] = x[3];
    out8[2] = x[2]; out8[3] = x[1];
    out8[4] = -x[2]; out8[5] = x[1];
    out8[6] = x[0]; out8[7] = -x[3];
}

/* R, S, T embedded in the (12), (13), (23) blocks; X = R S T, or X^+ when
 * inverse (GLAC/math/matrices/su3matrixgenerator.h:245-321). */
void oracle_rst_multiply(const double *r8, const double *s8, const double *t8, int inverse, double *out) {
    double R[18] = {0}, S[18] = {0}, T[18] = {0}, X[18];
    cplx one = {1.0, 0.0};
#define E2(m, i, j) ((cplx){(m)[4 * (i) + 2 * (j)], (m)[4 * (i) + 2 * (j) + 1]})
    setel(R, 0, 0, E2(r8, 0, 0)); setel(R, 0, 1, E2(r8, 0, 1));
    setel(R, 1, 0, E2(r8, 1, 0)); setel(R, 1, 1, E2(r8, 1, 1)); setel(R, 2, 2, one);
    setel(S, 0, 0, E2(s8, 0, 0)); setel(S, 0, 2, E2(s8, 0, 1));
    setel(S, 2, 0, E2(s8, 1, 0)); setel(S, 2, 2, E2(s8, 1, 1)); setel(S, 1, 1, one);
    setel(T, 1, 1, E2(t8, 0, 0)); setel(T, 1, 2, E2(t8, 0, 1));
    setel(T, 2, 1, E2(t8, 1, 0)); setel(T, 2, 2, E2(t8, 1, 1)); setel(T, 0, 0, one);
#undef E2
    mm(R, S, X);
    mm(X, T, X);
    if (inverse) dag(X, X);
    memcpy(out, X, sizeof(X));
}

void oracle_accept_fed(long nlinks, int nhits, double beta, double *U, const double *A,
                       const double *X, const double *r, unsigned char *accept) {
    for (long k = 0; k < nlinks; k++) {
        double *u = U + 18 * k;
        for (int h = 0; h < nhits; h++) {
            double Up[18];
            mm(X + 18 * (k * nhits + h), u, Up); /* U' = X U (system.cpp:321-331) */
            int acc = exp(-oracle_delta_s(u, Up, A + 18 * k, beta)) > r[k * nhits + h]; /* (:347) */
            accept[k * nhits + h] = (unsigned char)acc;
            if (acc) memcpy(u, Up, sizeof(Up));
        }
    }
}

/* ------------------------------------------------------------------ */
/* Project additions: Philox, checkerboard sweep, Haar start            */
/* ------------------------------------------------------------------ */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3], k0 = key[0], k1 = key[1];
    for (int round = 0; round < 10; round++) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0, p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        uint32_t n1 = (uint32_t)p1;
        uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* uniform in (-1/2, 1/2) from 16 bits, never 0 */
static double u_sym16(uint32_t h) { return ((double)h + 0.5) * (1.0 / 65536.0) - 0.5; }
/* uniform in [0, 1) with 53 bits */
static double u_53(uint32_t hi, uint32_t lo) {
    return (double)(((uint64_t)hi << 21) | (lo >> 11)) * 1.1102230246251565e-16;
}

/* Proposal for (link id, hit) from the Philox stream: two calls give 8 words;
 * words 0-5 hold twelve 16-bit uniforms (low half first) that build R, S, T
 * (su3matrixgenerator.h:170-196), words 6-7 the 53-bit accept uniform, and bit
 * 0 of word 7 chooses X or X^+. */
static void proposal(uint32_t key[2], uint32_t link_id, uint32_t sweep, uint32_t stream, int hit,
                     double eps, int flips, double *X, double *r) {
    uint32_t w[8];
    for (int call = 0; call < 2; call++) {
        uint32_t ctr[4] = {(uint32_t)(2 * hit + call), link_id, sweep, stream};
        oracle_philox4x32_10(ctr, key, w + 4 * call);
    }
    double su2[3][8];
    for (int b = 0; b < 3; b++) {
        double u[4];
        for (int c = 0; c < 4; c++) {
            int k = 4 * b + c;
            uint32_t word = w[k >> 1];
            u[c] = u_sym16((k & 1) ? (word >> 16) : (word & 0xFFFFu));
        }
        if (!flips) u[0] = fabs(u[0]); /* x0 = +sqrt(1 - eps^2): every factor near the identity */
        oracle_su2_near_unity(u, eps, su2[b]);
    }
    int inverse = (w[7] & 1u) == 0u;
    oracle_rst_multiply(su2[0], su2[1], su2[2], inverse, X);
    *r = u_53(w[6], w[7]);
}

uint64_t oracle_metropolis_sweep(const int N[4], double *links, double beta, double eps,
                                 int nhits, uint64_t seed, uint32_t stream, uint32_t sweep, int flips) {
    long V = (long)N[0] * N[1] * N[2] * N[3];
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint64_t accepted = 0;
    for (int k = 0; k < 8; k++) {
        int mu = k >> 1, parity = k & 1;
        for (long s = 0; s < V; s++) {
            int c[4];
            coords_of(N, s, c);
            if (((c[0] + c[1] + c[2] + c[3]) & 1) != parity) continue;
            double A[18];
            staple_at(N, V, links, c, mu, A);
            double *u = LINK(links, V, mu, s);
            for (int h = 0; h < nhits; h++) {
                double X[18], Up[18], r;
                proposal(key, (uint32_t)(mu * V + s), sweep, stream, h, eps, flips, X, &r);
                mm(X, u, Up);
                if (exp(-oracle_delta_s(u, Up, A, beta)) > r) {
                    memcpy(u, Up, sizeof(Up));
                    accepted++;
                }
            }
        }
    }
    return accepted;
}

/* Expected squared jump of one link (project design, the learned-spread
 * training data): for each spread eps_grid[k], the mean over `trials` of
 * ||U' - U||^2 = 6 - 2 ReTr(X_acc) after nhits Metropolis hits with staple A
 * (accept iff exp(-dS) > r, dS = -(beta/3)(ReTr(X W) - ReTr W), W = current
 * link times A), proposals from stream | 2^31 with sweep = snapshot and hit
 * index h + 16 (trial + trials k); flips = 0 draws every SU(2) factor near +1. */
void oracle_esj_link(const double *U, const double *A, double beta, int nhits, int n_eps, const double *eps_grid,
                     int trials, uint64_t seed, uint32_t link_id, uint32_t snapshot, uint32_t stream, int flips,
                     double *J) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    double W0[18];
    mm(U, A, W0);
    for (int k = 0; k < n_eps; k++) {
        double acc = 0.0;
        for (int tr = 0; tr < trials; tr++) {
            double Xt[18], Wc[18], X[18], T[18], r;
            mident(Xt);
            memcpy(Wc, W0, sizeof(Wc));
            for (int h = 0; h < nhits; h++) {
                proposal(key, link_id, snapshot, stream | 0x80000000u, h + 16 * (tr + trials * k), eps_grid[k], flips,
                         X, &r);
                double dS = -(beta / 3.0) * (retr_mul(X, Wc) - retr(Wc));
                if (exp(-dS) > r) {
                    mm(X, Xt, T);
                    memcpy(Xt, T, sizeof(T));
                    mm(X, Wc, T);
                    memcpy(Wc, T, sizeof(T));
                }
            }
            acc += 6.0 - 2.0 * retr(Xt);
        }
        J[k] = acc / trials;
    }
}

void oracle_haar_field(const int N[4], double *links, uint64_t seed, uint32_t stream) {
    long V = (long)N[0] * N[1] * N[2] * N[3];
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (long k = 0; k < 4 * V; k++) {
        uint32_t w[20];
        for (int call = 0; call < 5; call++) {
            uint32_t ctr[4] = {(uint32_t)call, (uint32_t)k, 0xA11Au, stream};
            oracle_philox4x32_10(ctr, key, w + 4 * call);
        }
        /* 9 complex Gaussians by Box-Muller */
        cplx z[3][3];
        for (int e = 0; e < 9; e++) {
            double u1 = ((double)w[2 * e] + 1.0) * 2.3283064365386963e-10;
            double u2 = (double)w[2 * e + 1] * 2.3283064365386963e-10;
            double rad = sqrt(-2.0 * log(u1));
            z[e / 3][e % 3].re = rad * cos(2.0 * M_PI * u2);
            z[e / 3][e % 3].im = rad * sin(2.0 * M_PI * u2);
        }
        /* Gram-Schmidt on columns: Q of the QR factorisation with R_ii > 0 */
        for (int j = 0; j < 3; j++) {
            for (int p = 0; p < j; p++) {
                cplx d = {0, 0}; /* <q_p, z_j> */
                for (int i = 0; i < 3; i++) {
                    d.re += z[i][p].re * z[i][j].re + z[i][p].im * z[i][j].im;
                    d.im += z[i][p].re * z[i][j].im - z[i][p].im * z[i][j].re;
                }
                for (int i = 0; i < 3; i++) {
                    cplx q = cmul(d, z[i][p]);
                    z[i][j].re -= q.re;
                    z[i][j].im -= q.im;
                }
            }
            double nrm = 0.0;
            for (int i = 0; i < 3; i++) nrm += z[i][j].re * z[i][j].re + z[i][j].im * z[i][j].im;
            nrm = 1.0 / sqrt(nrm);
            for (int i = 0; i < 3; i++) { z[i][j].re *= nrm; z[i][j].im *= nrm; }
        }
        double *U = links + 18 * k;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) setel(U, i, j, z[i][j]);
        /* det -> 1: multiply by exp(-i arg(det)/3) */
        cplx d = {0, 0};
        for (int p = 0; p < 3; p++) {
            int q = (p + 1) % 3, s = (p + 2) % 3;
            cplx m = cmul(z[1][q], z[2][s]), m2 = cmul(z[1][s], z[2][q]);
            cplx minor = {m.re - m2.re, m.im - m2.im};
            cplx term = cmul(z[0][p], minor);
            d.re += term.re;
            d.im += term.im;
        }
        double ph = -atan2(d.im, d.re) / 3.0;
        cplx f = {cos(ph), sin(ph)};
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) setel(U, i, j, cmul(el(U, i, j), f));
    }
}

void oracle_reunitarize(double *m, long n) {
    for (long k = 0; k < n; k++) {
        double *U = m + 18 * k;
        cplx a[3], b[3];
        for (int j = 0; j < 3; j++) { a[j] = el(U, 0, j); b[j] = el(U, 1, j); }
        double na = 0.0;
        for (int j = 0; j < 3; j++) na += a[j].re * a[j].re + a[j].im * a[j].im;
        na = 1.0 / sqrt(na);
        for (int j = 0; j < 3; j++) { a[j].re *= na; a[j].im *= na; }
        cplx d = {0, 0}; /* sum conj(a_j) b_j */
        for (int j = 0; j < 3; j++) {
            d.re += a[j].re * b[j].re + a[j].im * b[j].im;
            d.im += a[j].re * b[j].im - a[j].im * b[j].re;
        }
        for (int j = 0; j < 3; j++) {
            cplx q = cmul(d, a[j]);
            b[j].re -= q.re;
            b[j].im -= q.im;
        }
        double nb = 0.0;
        for (int j = 0; j < 3; j++) nb += b[j].re * b[j].re + b[j].im * b[j].im;
        nb = 1.0 / sqrt(nb);
        for (int j = 0; j < 3; j++) { b[j].re *= nb; b[j].im *= nb; }
        for (int j = 0; j < 3; j++) {
            int p = (j + 1) % 3, q = (j + 2) % 3;
            cplx c = {0, 0}, t1 = cmul(a[p], b[q]), t2 = cmul(a[q], b[p]);
            c.re = t1.re - t2.re;
            c.im = -(t1.im - t2.im); /* third row = conj(a x b) */
            setel(U, 0, j, a[j]);
            setel(U, 1, j, b[j]);
            setel(U, 2, j, c);
        }
    }
}
