// Device kernels of the hot path and their host-side launchers.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include "lattice.cuh"
#include "learned.cuh"
#include "expm.cuh"

namespace glac {

// SU(3) x SU(3) products of the FP32 flow kernels: the third row from the
// first two (su3.cuh, 96 instead of 108 multiply-adds); FP64 keeps the full
// product, the form the reference computes.
template <typename T> __device__ __forceinline__ M3<T> flow_nd(const M3<T> &a, const M3<T> &b) {
    if constexpr (sizeof(T) == 4) return mul_nd_su3(a, b);
    else return mul_nd(a, b);
}
template <typename T> __device__ __forceinline__ M3<T> flow_dd(const M3<T> &a, const M3<T> &b) {
    if constexpr (sizeof(T) == 4) return mul_dd_su3(a, b);
    else return mul_dd(a, b);
}
template <typename T> __device__ __forceinline__ M3<T> flow_nn(const M3<T> &a, const M3<T> &b) {
    if constexpr (sizeof(T) == 4) return mul_su3(a, b);
    else return mul(a, b);
}

// Staple A_mu(n) (GLAC/actions/wilsongaugeaction.cpp:29-53, and the same sum in
// getActionDerivative :55-86):
//   sum_{nu != mu}  U_nu(n+mu) U_mu(n+nu)^+ U_nu(n)^+  +  U_nu(n+mu-nu)^+ U_mu(n-nu)^+ U_nu(n-nu)
// n has parity p; n +- nu and n + mu have parity 1-p, n + mu - nu has parity p.
// UNROLL: the nu loop unrolled, which made the Metropolis sub-sweep 1-4 % faster
// and the flow stage 2-6 % slower on B200 (the flow keeps the rolled loop).
// RECON: each staple term's first product by flow_nd / flow_dd (the flow
// stage); the Metropolis kernels keep the full products.
template <typename T, bool UNROLL = false, bool RECON = false>
__device__ __forceinline__ M3<T> staple(const LinkField<T> &L, const Geom &g, const Site &n, int p, int mu) {
    M3<T> A;
    set_zero(A);
    const int q = p ^ 1;
    // Neighbour indices: select chains in FP32 (pick4), indexed arrays in FP64;
    // each form is the faster one for its precision.
    const int f_mu = sizeof(T) == 4 ? step_offset(g, n, mu, +1) : step_offset_indexed(g, n, mu, +1);
    const int s_mu = (n.lex + f_mu) >> 1;
#pragma unroll(UNROLL ? 4 : 1)
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
        {
            M3<T> a = L.load(nu, q, s_mu);
            M3<T> b = L.load(mu, q, s_nup);
            M3<T> t = RECON ? flow_nd(a, b) : mul_nd(a, b);
            M3<T> c = L.load(nu, p, n.lex >> 1);
            acc_mul_nd(A, t, c);
        }
        {
            M3<T> a = L.load(nu, p, s_diag);
            M3<T> b = L.load(mu, q, s_num);
            M3<T> t = RECON ? flow_dd(a, b) : mul_dd(a, b);
            M3<T> c = L.load(nu, q, s_num);
            acc_mul(A, t, c);
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
    int nblocks;  // Nt * 2 * nb
};
ObsPlan make_obs_plan(const Geom &g);

// Kernel families with launch variants chosen by the autotuner (glac_autotune).
enum Family { FAM_FLOW = 0, FAM_METRO = 1, FAM_OBS = 2 };
constexpr int kMaxVariants = 4;
int num_variants(Family f, bool fp32);
int variant_regs(Family f, bool fp32, int v);   // register cap of a variant (0 = none)
int variant_shape(Family f, bool fp32, int v);  // flow site-block shape of a variant (0 = one plane per block)

template <typename T>
void launch_flow_stage(const Geom &g, const LinkField<T> &in, const LinkField<T> &out, const ForceField<T> &zf,
                       int stage, int kind, double alpha, double beta, int variant, cudaStream_t st);
// Flow stage 0 that also writes the clover parts of its input field's
// measurement (regs: 0 = the compiler's allocation, 128 = capped), and the
// measurement from those parts ([plaq, topc, energy, topct[Nt]] into out).
template <typename T>
void launch_flow_stage0_meas(const Geom &g, const LinkField<T> &in, const LinkField<T> &out, const ForceField<T> &zf,
                             const CloverParts<T> &cp, int kind, double alpha, int regs, cudaStream_t st);
template <typename T>
void launch_obs_combine(const Geom &g, const CloverParts<T> &cp, const ObsPlan &plan, double *partial, double *out,
                        cudaStream_t st);
// Flow stage 1 with the measurement's combination and reduction folded in
// (where obs_combine_in_stage1 holds), then the final reduction into obs_out.
bool obs_combine_in_stage1(const Geom &g, const ObsPlan &plan);
template <typename T>
void launch_flow_stage1_combine(const Geom &g, const LinkField<T> &in, const LinkField<T> &out,
                                const ForceField<T> &zf, int kind, double alpha, double beta,
                                const CloverParts<T> &cp, const ObsPlan &plan, double *partial, double *obs_out,
                                bool site, cudaStream_t st);
// whether the 12 clover-part slots of a lattice fit 32-bit element offsets
inline bool clover_offsets_fit(long long V, bool fp64) {
    const long long vh32 = ((V / 2) + 31) / 32 * 32;
    return (fp64 ? 96 : 48) * vh32 < (1ll << 32);
}
// P.net set: the learned spread (learned.cuh) replaces eps per link.
template <typename T>
void launch_metropolis(const Geom &g, const LinkField<T> &L, int mu, int p, double beta, double eps, int nhits,
                       uint64_t seed, uint32_t sweep, uint32_t stream_id, unsigned long long *acc, int variant,
                       const Proposal &P, cudaStream_t st);
// Expected-squared-jump rows of 8 * ns sampled links (features [row][8], esj [row][n_eps], ids [row] or null).
template <typename T>
void launch_esj(const Geom &g, const LinkField<T> &L, double beta, int nhits, int n_eps, const float *eps_grid_dev,
                int trials, int stride, int offset, int ns, uint64_t seed, uint32_t snapshot, uint32_t stream_id,
                bool flips, float *feat, float *esj, uint32_t *ids, cudaStream_t st);
// SuperSampler observables: [plaq, topc, energy, weinberg, topct[Nt], weinbergt[Nt]]; partial4: 4 per block.
template <typename T>
void launch_weinberg(const Geom &g, const LinkField<T> &L, const ObsPlan &plan, double *partial4, double *out,
                     cudaStream_t st);
// Observables plus per-site topological-charge and energy densities (V doubles each, lexicographic).
template <typename T>
void launch_observables_density(const Geom &g, const LinkField<T> &L, const ObsPlan &plan, double *partial,
                                double *out, double *dq, double *de, cudaStream_t st);
template <typename T>
void launch_observables(const Geom &g, const LinkField<T> &L, const ObsPlan &plan, double *partial,
                        double *out, int variant, cudaStream_t st);
template <typename T>
void launch_haar(const Geom &g, const LinkField<T> &L, uint64_t seed, uint32_t stream_id, cudaStream_t st);
template <typename T>
void launch_cold(const Geom &g, const LinkField<T> &L, cudaStream_t st);
template <typename T>
void launch_rst_start(const Geom &g, const LinkField<T> &L, double eps, uint64_t seed, uint32_t stream_id,
                      cudaStream_t st);
template <typename T>
void launch_reunitarize(const Geom &g, const LinkField<T> &L, cudaStream_t st);
template <typename T>
void launch_aos_to_soa(const Geom &g, const double *aos, const LinkField<T> &L, cudaStream_t st);
template <typename T>
void launch_soa_to_aos(const Geom &g, const LinkField<T> &L, double *aos, cudaStream_t st);
template <typename T>
void launch_copy_field(const Geom &g, const LinkField<T> &src, const LinkField<T> &dst, cudaStream_t st);

// test exports: outputs in the reference's host layout [mu][lex][18] (FP64)
template <typename T>
void launch_staples_aos(const Geom &g, const LinkField<T> &L, double *out, cudaStream_t st);
template <typename T>
void launch_force_aos(const Geom &g, const LinkField<T> &L, double *out, cudaStream_t st);
template <typename T>
void launch_exp_batch(int kind, const double *in, double *out, long n, cudaStream_t st);
template <typename T>
void launch_accept_fed(double beta, long nlinks, int nhits, double *U, const double *A, const double *X,
                       const double *r, unsigned char *accept, cudaStream_t st);
template <typename T>
void launch_delta_s(double beta, long n, const double *U, const double *Up, const double *A, double *out,
                    cudaStream_t st);
template <typename T>
void launch_max_unitarity_dev(const Geom &g, const LinkField<T> &L, double *out, cudaStream_t st);

// ---------------------------------------------------------------------------
// Batched ensemble: many independent lattices per launch.  Each phase kernel
// walks a prefix table of block counts (start[i] = first block of lattice i,
// start[M] = total) and runs the single-lattice body on lattice i's slot.
// ---------------------------------------------------------------------------
template <typename T> struct LatSlot {
    Geom g;
    LinkField<T> f[3];        // 0: Markov chain, 1 and 2: flow ping-pong
    ForceField<T> z;
    int nb, Bv;               // observable plan (blocks of <= 128 threads)
    double *partial;          // 3 doubles per observable block
    double *obs;              // this lattice's measurement rows (3 + Nt each)
    CloverParts<T> cp;        // clover parts of the measurement inside flow stage 0 (cp.ah.p null: none)
    unsigned long long *acc;  // accepted proposals
    float beta;
    uint32_t stream;          // Philox stream
};
enum EnsPhase { ENS_METRO = 0, ENS_FLOW0 = 1, ENS_FLOW1 = 2, ENS_OBS = 3, ENS_NPHASE = 4 };
// blocks of one lattice per phase (FLOW0/FLOW1: flow site-block shape 0/1)
int ens_blocks(const Geom &g, const ObsPlan &plan, int phase);
ObsPlan make_obs_plan_capped(const Geom &g, int max_threads);

template <typename T>
void launch_ens_haar(const LatSlot<T> *slots, const int *start, int nblocks, int M, uint64_t seed, cudaStream_t st);
template <typename T>
void launch_ens_metropolis(const LatSlot<T> *slots, const int *start, int nblocks, int M, int fsel, int mu, int p,
                           double eps, int nhits, uint64_t seed, const uint32_t *sweep_base, uint32_t sweep_off,
                           bool flips, int variant, cudaStream_t st);
template <typename T>
void launch_ens_flow_stage(const LatSlot<T> *slots, const int *start, int nblocks, int M, int src, int dst, int stage,
                           double alpha, double beta, int variant, cudaStream_t st);
template <typename T>
void launch_ens_observables(const LatSlot<T> *slots, const int *start, int nblocks, int M, int fsel,
                            int meas, int variant, cudaStream_t st);
// Flow stage 0 of every lattice with its measurement's clover parts (block
// table of the shape-0 flow phase), and the measurement from those parts into
// measurement row `meas` (block table of the observable phase).
template <typename T>
void launch_ens_flow_stage0_meas(const LatSlot<T> *slots, const int *start, int nblocks, int M, int src, int dst,
                                 double alpha, int regs, cudaStream_t st);
template <typename T>
void launch_ens_obs_combine(const LatSlot<T> *slots, const int *start, int nblocks, int M, int meas,
                            cudaStream_t st);
void launch_advance(uint32_t *counter, uint32_t by, cudaStream_t st);

// The whole schedule in one persistent cooperative launch (FP32; measurement
// inside stage 0).  A barrier's state, zeroed before the launch.
struct GridBarrier {
    unsigned int count, gen;
    int err;
};
struct EnsSchedule {
    int M, n_sweeps, n_steps;  // n_steps < 0: sweeps only
    const int *start_metro, *start_flow0, *start_obs;
    int nb_metro, nb_flow0, nb_obs;
    double eps, sq1me, alpha[3], beta[3];
    int nhits;
    uint32_t k0, k1;
    uint32_t *sweep_base;
    bool flips;
    const void *chain;  // field role 0 and 1 base pointers, field_words 16-byte words
    void *flow;
    size_t field_words;
    unsigned long long wait_ns;
    int test_skip_block0;
};
int persistent_blocks_per_sm();
cudaError_t launch_ens_persistent(const LatSlot<float> *slots, const EnsSchedule &sc, GridBarrier *bar, int grid,
                                  cudaStream_t st);

}  // namespace glac
