/*
 * CPU restatement of GLAC's pure-gauge SU(3) hot path, plus the project's own
 * additions (Philox streams, checkerboard Metropolis, Haar start,
 * reunitarisation) that have no reference counterpart.
 *
 * TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py as the checker.  Never on the product path.
 *
 * Parity is pinned two ways: against the known-answer fixtures held in the
 * reference's unit tests (tests/golden/), and against the reference itself,
 * compiled from its own sources into oracle/_ref/libglacref.so.
 *
 * Conventions (same as the reference): an SU(3) matrix is 18 doubles, element
 * (i,j) at [6i+2j] (re) and [6i+2j+1] (im) (GLAC/math/matrices/su3.h:18-22).
 * A gauge field is 4 blocks (mu = 0..3) of V matrices, sites in lexicographic
 * order x + Nx(y + Ny(z + Nz t)) (GLAC/parallelization/index.h:32-35).
 */
#ifndef GLAC_ORACLE_H
#define GLAC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): out = bijection(ctr; key). */
void oracle_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Single-matrix algebra (GLAC/math/matrices/su3.h:184-215, 307-329;
 * GLAC/math/functions.h:45-53), exposed for the known-answer fixtures. */
void oracle_su3_mul(const double *A, const double *B, double *C);
void oracle_su3_dagger(const double *A, double *B);
double oracle_retr_mul(const double *A, const double *B);

/* Staple A_mu(n) of every link (GLAC/actions/wilsongaugeaction.cpp:29-53). */
void oracle_staples(const int N[4], const double *links, double *out);
/* dS = -(beta/3) ReTr[(U' - U) A] (GLAC/actions/wilsongaugeaction.cpp:24-27). */
double oracle_delta_s(const double *U, const double *Uprime, const double *A, double beta);
/* Flow force Z_mu(n) as 18-double matrices (GLAC/actions/wilsongaugeaction.cpp:55-86). */
void oracle_force(const int N[4], const double *links, double *out);

/* SU(3) exponentials, n matrices (GLAC/math/exponentiation/):
 * kind 0 Morningstar-Peardon (su3exp.cpp:16-79), 1 Luscher (expluscher.cpp:13-68),
 * 2 Taylor-2 (taylor2exp.cpp:8-16), 3 Taylor-4 (taylor4exp.cpp:8-20),
 * 4 Taylor-N of the given degree (taylorexp.cpp:14-30). */
void oracle_exp(int kind, int degree, const double *in, long n, double *out);

/* nsteps of Luscher RK3 flow, in place (GLAC/flow/flow.cpp:43-73). */
void oracle_flow(const int N[4], double *links, double eps, int nsteps, int expkind);

/* out = [plaq, topc, energy, topct[0..Nt-1]]
 * (GLAC/observables/mastersamplertopcxyz.cpp:236-384). */
void oracle_observables(const int N[4], const double *links, double *out);
/* SuperSampler observables [plaq, topc, energy, weinberg, topct[Nt], weinbergt[Nt]]
 * (GLAC/observables/supersampler.cpp:298-496). */
void oracle_weinberg(const int N[4], const double *links, double *out);
/* Per-site topological charge density q (with 1/(16^2 pi^2)) and unnormalised
 * energy density e, V doubles each (GLAC/observables/latticeactionchargedensity.cpp:169-306). */
void oracle_density(const int N[4], const double *links, double *q, double *e);
/* Plaquette (GLAC/observables/plaquette.cpp:26-40). */
double oracle_plaquette(const int N[4], const double *links);

/* X = R S T or its inverse from three SU(2) 2x2 complex matrices (8 doubles each)
 * (GLAC/math/matrices/su3matrixgenerator.h:245-321). */
void oracle_rst_multiply(const double *r8, const double *s8, const double *t8, int inverse, double *out);
/* SU(2) element near unity from 4 uniforms in (-1/2, 1/2) and spread eps
 * (GLAC/math/matrices/su3matrixgenerator.h:202-243). */
void oracle_su2_near_unity(const double u[4], double eps, double out8[8]);

/* Fed Metropolis on independent links: for link k, nhits proposals X[k][h]
 * and uniforms r[k][h]; U'=X U, accept iff exp(-dS) > r (GLAC/system.cpp:333-361).
 * U is updated in place; accept[k][h] receives the decisions. */
void oracle_accept_fed(long nlinks, int nhits, double beta, double *U, const double *A,
                       const double *X, const double *r, unsigned char *accept);

/* Checkerboard Metropolis with Philox streams (project design, no reference
 * counterpart): sub-sweep k = 2*mu + parity; for each link of that class the
 * staple is taken once and nhits proposals drawn from the Philox stream
 * (key = seed, counter = {2*hit + call, mu*V + site, sweep, stream}).
 * flips = 0 draws every SU(2) factor near +1 (x0 > 0), 1 as the reference.
 * Returns accepted proposals; links updated in place. */
uint64_t oracle_metropolis_sweep(const int N[4], double *links, double beta, double eps,
                                 int nhits, uint64_t seed, uint32_t stream, uint32_t sweep, int flips);

/* Expected squared jump of one link for each spread on a grid (project design,
 * training data of the learned proposal spread); see glac_oracle.c. */
void oracle_esj_link(const double *U, const double *A, double beta, int nhits, int n_eps, const double *eps_grid,
                     int trials, uint64_t seed, uint32_t link_id, uint32_t snapshot, uint32_t stream, int flips,
                     double *J);

/* Seeded Haar-random SU(3) field (QR of a complex Gaussian matrix with phase fix,
 * then det normalisation), 4V links; counter = {call, mu*V + site, 0xA11A, stream}. */
void oracle_haar_field(const int N[4], double *links, uint64_t seed, uint32_t stream);

/* Gram-Schmidt reunitarisation of n matrices in place. */
void oracle_reunitarize(double *m, long n);

#ifdef __cplusplus
}
#endif
#endif
