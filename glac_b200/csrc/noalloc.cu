// Allocation-free variant of the observable measurement.
//
// Some callers cannot call cudaMalloc: code running under a host framework that
// owns all device memory through its own pool or arena and forbids allocations
// from libraries, code that must not allocate during a latency-critical phase
// (a driver allocation can synchronise the device and stall other streams), and
// embedded or safety-reviewed deployments where every device allocation is fixed
// at load time.  glac_measure_noalloc serves them: the caller passes the gauge
// field and the output vector in device memory it already owns, and the only
// working memory is the fixed file-scope array below, which every GPU that loads
// this library holds until the process exits.
//
// The field is read in the reference's host layout (4 blocks of V matrices,
// 18 FP64 each, site order x + Nx(y + Ny(z + Nz t))) directly from device
// memory, so no converted copy is needed either.  The arithmetic is the same as
// the context path's observables (clover per plane, FP64 reductions in a fixed
// order), so results agree with glac_measure to rounding.
#include "../../include/glac_b200.h"
#include "su3.cuh"

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

namespace {

constexpr int kBlock = 128;
constexpr int kMaxSlots = 4096;  // (block, time slice) partial sums
constexpr int kSlotDoubles = 3;  // plaq, energy, q

// Scratch for the per-block partial sums: 4096 slots x 3 doubles = 96 KiB per GPU.
static __device__ __align__(256) double g_noalloc_scratch[kMaxSlots * kSlotDoubles];

thread_local std::string g_err;
std::mutex g_mu;
void *g_scratch_ptr[64] = {nullptr};  // per device ordinal, from cudaGetSymbolAddress

using glac::Cx;
using glac::M3;

struct AosField {
    const double *p;
    int N[4];
    long long V;
    __device__ __forceinline__ M3<double> load(int mu, long long lex) const {
        const double2 *src = reinterpret_cast<const double2 *>(p + ((size_t)mu * V + (size_t)lex) * 18);
        M3<double> U;
#pragma unroll
        for (int k = 0; k < 9; k++) {
            const double2 v = __ldg(src + k);
            U.e[k].re = v.x;
            U.e[k].im = v.y;
        }
        return U;
    }
    // lexicographic index of c + a e_d + b e_e (periodic)
    __device__ __forceinline__ long long at(const int c[4], int d, int a, int e, int b) const {
        int x[4] = {c[0], c[1], c[2], c[3]};
        if (d >= 0) x[d] = (x[d] + a + N[d]) % N[d];
        if (e >= 0) x[e] = (x[e] + b + N[e]) % N[e];
        return x[0] + (long long)N[0] * (x[1] + (long long)N[1] * (x[2] + (long long)N[2] * x[3]));
    }
};

// Projected clover of the (mu, nu) plane (GLAC/observables/mastersamplertopcxyz.cpp:253-340):
// F = (C - C^+) - 1/3 i ImTr(C - C^+) with C = leaf1 - leaf2 + leaf3 - leaf4.
__device__ M3<double> clover(const AosField &L, const int c[4], int mu, int nu, double &plaq) {
    using namespace glac;
    const long long n0 = L.at(c, -1, 0, -1, 0);
    M3<double> C = mul_nd(mul(L.load(mu, n0), L.load(nu, L.at(c, mu, 1, -1, 0))),
                          mul(L.load(nu, n0), L.load(mu, L.at(c, nu, 1, -1, 0))));
    plaq = retr(C);
    const long long n_num = L.at(c, nu, -1, -1, 0), n_mum = L.at(c, mu, -1, -1, 0);
    const long long n_mm = L.at(c, mu, -1, nu, -1);
    sub_from(C, mul(mul_nd(L.load(mu, n0), mul(L.load(mu, n_num), L.load(nu, L.at(c, mu, 1, nu, -1)))),
                    L.load(nu, n_num)));
    add_to(C, mul(mul(mul_dd(L.load(mu, n_mum), L.load(nu, n_mm)), L.load(mu, n_mm)), L.load(nu, n_num)));
    sub_from(C, mul_nd(mul(mul_dn(L.load(mu, n_mum), L.load(nu, n_mum)), L.load(mu, L.at(c, mu, -1, nu, 1))),
                       L.load(nu, n0)));
    const M3<double> D = dagger(C);
    sub_from(C, D);
    const double tr = (C(0, 0).im + C(1, 1).im + C(2, 2).im) / 3.0;
    C(0, 0).im -= tr;
    C(1, 1).im -= tr;
    C(2, 2).im -= tr;
    return C;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// grid (K, Nt): block (k, t) strides over the sites of time slice t.
__global__ void __launch_bounds__(kBlock) k_measure_noalloc(AosField L, double *scratch) {
    const int K = gridDim.x, k = blockIdx.x, t = blockIdx.y;
    const long long Vs = (long long)L.N[0] * L.N[1] * L.N[2];
    double plaq = 0.0, en = 0.0, q = 0.0;
    for (long long i = (long long)k * kBlock + threadIdx.x; i < Vs; i += (long long)K * kBlock) {
        int c[4];
        long long r = i;
        c[0] = (int)(r % L.N[0]); r /= L.N[0];
        c[1] = (int)(r % L.N[1]); r /= L.N[1];
        c[2] = (int)r;
        c[3] = t;
        for (int nu = 1; nu < 4; nu++) {
            const int rho = nu % 3 + 1, sigma = rho % 3 + 1;
            double p1, p2;
            const M3<double> C1 = clover(L, c, 0, nu, p1);
            const M3<double> C2 = clover(L, c, rho, sigma, p2);
            plaq += p1 + p2;
            q -= glac::retr_mul(C1, C2);
            en += glac::retr_mul(C1, C1) + glac::retr_mul(C2, C2);
        }
    }
    __shared__ double sh[3][kBlock / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    plaq = warp_sum(plaq);
    en = warp_sum(en);
    q = warp_sum(q);
    if (lane == 0) { sh[0][wid] = plaq; sh[1][wid] = en; sh[2][wid] = q; }
    __syncthreads();
    if (threadIdx.x < 3) {
        double a = 0.0;
        for (int w = 0; w < kBlock / 32; w++) a += sh[threadIdx.x][w];
        scratch[((size_t)t * K + k) * kSlotDoubles + threadIdx.x] = a;
    }
}

// out = [plaq, topc, energy, topct[Nt]] (mastersamplertopcxyz.cpp:13-16, :363-383)
__global__ void k_finalize_noalloc(int Nt, int K, double V, const double *scratch, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double qfac = 1.0 / (16 * 16 * M_PI * M_PI);
    double a = 0.0, e = 0.0, qtot = 0.0;
    for (int t = 0; t < Nt; t++) {
        double qt = 0.0;
        for (int k = 0; k < K; k++) {
            const double *s = scratch + ((size_t)t * K + k) * kSlotDoubles;
            a += s[0];
            e += s[1];
            qt += s[2];
        }
        qtot += qt;
        out[3 + t] = qt * qfac;
    }
    out[0] = a / (18.0 * V);
    out[1] = qtot * qfac;
    out[2] = e / V;
}

}  // namespace

extern "C" const char *glac_noalloc_error(void) { return g_err.c_str(); }

extern "C" glac_status glac_measure_noalloc(const int dims[4], const double *dev_links, double *dev_obs,
                                            void *stream) {
    if (!dims || !dev_links || !dev_obs) {
        g_err = "null argument";
        return GLAC_ERR_ARG;
    }
    // the kernel reads each link as nine 16-byte double2 words and writes
    // doubles: a misaligned buffer is an argument error, not a device fault
    if (reinterpret_cast<uintptr_t>(dev_links) % 16 != 0) {
        g_err = "dev_links must be 16-byte aligned";
        return GLAC_ERR_ARG;
    }
    if (reinterpret_cast<uintptr_t>(dev_obs) % 8 != 0) {
        g_err = "dev_obs must be 8-byte aligned";
        return GLAC_ERR_ARG;
    }
    // V = Nx Ny Nz Nt <= 2^31, checked before each product so it cannot wrap
    const long long kMaxV = 1ll << 31;
    long long V = 1;
    for (int d = 0; d < 4; d++) {
        if (dims[d] < 2) {
            g_err = "every lattice extent must be at least 2";
            return GLAC_ERR_ARG;
        }
        if ((long long)dims[d] > kMaxV / V) {
            g_err = "lattice too large (V > 2^31)";
            return GLAC_ERR_ARG;
        }
        V *= dims[d];
    }
    const int Nt = dims[3];
    if (Nt > kMaxSlots) {
        g_err = "Nt = " + std::to_string(Nt) + " exceeds the scratch capacity of " + std::to_string(kMaxSlots) +
                " time slices";
        return GLAC_ERR_ARG;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        g_err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return GLAC_ERR_CUDA;
    }
    if (dev < 0 || dev >= 64) {
        g_err = "device ordinal " + std::to_string(dev) + " beyond the 64 devices this entry point tracks";
        return GLAC_ERR_CUDA;
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) {
        g_err = std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e);
        return GLAC_ERR_CUDA;
    }
    void *scratch = nullptr;
    {
        // The array's device address belongs to the module loaded in the current
        // context; after cudaDeviceReset (a new primary context) it can move.
        // Outside stream capture it is resolved afresh on every call; during a
        // capture the address of this device's last uncaptured call is used.
        std::lock_guard<std::mutex> lock(g_mu);
        if (cap == cudaStreamCaptureStatusNone) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
                return GLAC_ERR_CUDA;
            }
            g_scratch_ptr[dev] = p;
        } else if (!g_scratch_ptr[dev]) {
            g_err = "the first call on a device must come before any stream capture";
            return GLAC_ERR_STATE;
        }
        scratch = g_scratch_ptr[dev];
    }
    // blocks per time slice: fill the scratch slots without exceeding them
    const long long Vs = V / Nt;
    int K = kMaxSlots / Nt;
    const long long need = (Vs + kBlock - 1) / kBlock;
    if (K > need) K = (int)need;
    if (K > 64) K = 64;
    if (K < 1) K = 1;
    AosField L;
    L.p = dev_links;
    for (int d = 0; d < 4; d++) L.N[d] = dims[d];
    L.V = V;
    k_measure_noalloc<<<dim3(K, Nt), kBlock, 0, st>>>(L, reinterpret_cast<double *>(scratch));
    k_finalize_noalloc<<<1, 32, 0, st>>>(Nt, K, (double)V, reinterpret_cast<const double *>(scratch), dev_obs);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        g_err = std::string("launch: ") + cudaGetErrorString(e);
        return GLAC_ERR_CUDA;
    }
    return GLAC_OK;
}
