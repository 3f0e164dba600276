// Device kernels of the hot path and their host-side launchers.
//
// Kernels are written once over the real type R: double for the FP64 path
// (one lattice site per thread) and f32x2 for the FP32 path (two lattice
// sites per thread, one per FP32 lane, see lattice.cuh).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "lattice.cuh"
#include "expm.cuh"

namespace glac {

// Staple A_mu(n) (GLAC/actions/wilsongaugeaction.cpp:29-53, and the same sum in
// getActionDerivative :55-86):
//   sum_{nu != mu}  U_nu(n+mu) U_mu(n+nu)^+ U_nu(n)^+  +  U_nu(n+mu-nu)^+ U_mu(n-nu)^+ U_nu(n-nu)
// n has parity p; n +- nu and n + mu have parity 1-p, n + mu - nu has parity p.
template <typename R>
__device__ __forceinline__ M3<R> staple(const LinkField<R> &L, const Geom &g, const Site &n, int p, int mu) {
    M3<R> A;
    set_zero(A);
    const int q = p ^ 1;
    const Nb n_mu = nb_step(g, n, mu, +1);
    const Nb n_0 = nb_self(n);
#pragma unroll 1
    for (int nu = 0; nu < 4; nu++) {
        if (nu == mu) continue;
        const Nb n_nup = nb_step(g, n, nu, +1);
        const Nb n_num = nb_step(g, n, nu, -1);
        const Nb n_diag = nb_step2(g, n, mu, +1, nu, -1);
        {
            const M3<R> t = mul_nd(L.load(nu, q, n_mu), L.load(mu, q, n_nup));
            acc_mul_nd(A, t, L.load(nu, p, n_0));
        }
        {
            const M3<R> t = mul_dd(L.load(nu, p, n_diag), L.load(mu, q, n_num));
            acc_mul(A, t, L.load(nu, q, n_num));
        }
    }
    return A;
}

// ---------------------------------------------------------------------------
// Launchers (defined in kernels.cu).  All take the stream to launch on.
// ---------------------------------------------------------------------------
struct ObsPlan {
    int Bv;       // sites per block; divides the parity half of a time slice
    int B;        // threads per block (Bv rounded up to a whole warp)
    int nb;       // blocks per (t, parity)
    int nblocks;  // Nt_stored * 2 * nb
};
ObsPlan make_obs_plan(const Geom &g);
constexpr int kObsPartial = 4;  // plaq, energy, q(lane 0), q(lane 1) per block

template <typename R>
void launch_flow_stage(const Geom &g, const LinkField<R> &in, const LinkField<R> &out, const ForceField<R> &zf,
                       int stage, int kind, double alpha, double beta, cudaStream_t st);
template <typename R>
void launch_metropolis(const Geom &g, const LinkField<R> &L, int mu, int p, double beta, double eps, int nhits,
                       uint64_t seed, uint32_t sweep, uint32_t stream_id, unsigned long long *acc, cudaStream_t st);
template <typename R>
void launch_observables(const Geom &g, const LinkField<R> &L, const ObsPlan &plan, double *partial,
                        double *out, cudaStream_t st);
template <typename R>
void launch_haar(const Geom &g, const LinkField<R> &L, uint64_t seed, uint32_t stream_id, cudaStream_t st);
template <typename R>
void launch_cold(const Geom &g, const LinkField<R> &L, cudaStream_t st);
template <typename R>
void launch_reunitarize(const Geom &g, const LinkField<R> &L, cudaStream_t st);
template <typename R>
void launch_aos_to_soa(const Geom &g, const double *aos, const LinkField<R> &L, cudaStream_t st);
template <typename R>
void launch_soa_to_aos(const Geom &g, const LinkField<R> &L, double *aos, cudaStream_t st);
template <typename R>
void launch_copy_field(const Geom &g, const LinkField<R> &src, const LinkField<R> &dst, cudaStream_t st);

// test exports: outputs in the reference's host layout [mu][lex][18] (FP64)
template <typename R>
void launch_staples_aos(const Geom &g, const LinkField<R> &L, double *out, int force, cudaStream_t st);
template <typename R>
void launch_max_unitarity_dev(const Geom &g, const LinkField<R> &L, double *out, cudaStream_t st);
// single matrices (T = double or float)
template <typename T>
void launch_exp_batch(int kind, const double *in, double *out, long n, cudaStream_t st);
template <typename T>
void launch_accept_fed(double beta, long nlinks, int nhits, double *U, const double *A, const double *X,
                       const double *r, unsigned char *accept, cudaStream_t st);
template <typename T>
void launch_delta_s(double beta, long n, const double *U, const double *Up, const double *A, double *out,
                    cudaStream_t st);

}  // namespace glac
