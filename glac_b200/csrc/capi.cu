// C ABI (include/glac_b200.h): contexts, device buffers, stream, and the
// sequencing of the hot-path kernels.
#include "../../include/glac_b200.h"
#include "kernels.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

using namespace glac;

struct glac_ctx {
    glac_desc d;
    Geom g;
    ObsPlan plan;
    cudaStream_t stream = nullptr;
    void *field[2] = {nullptr, nullptr};
    int cur = 0;
    void *force = nullptr;
    double *partial = nullptr;
    double *partial4 = nullptr;  // SuperSampler partials, 4 per block (allocated on first use)
    double *obs_dev = nullptr;
    size_t obs_cap = 0;  // doubles in obs_dev
    unsigned long long *acc_dev = nullptr;
    double *staging = nullptr;
    double *scalar_dev = nullptr;
    uint32_t sweep = 0;
    uint64_t launches = 0;
    int tune[3] = {0, 0, 0};  // chosen launch variant per kernel family (flow, metropolis, observables)
    float *net_params = nullptr;  // learned proposal spread: FP32 parameters and their packed fragments
    uint32_t *net_pack = nullptr;
    float *esj_grid = nullptr;    // 64 floats
    Proposal prop;                // prop.net null: the fixed spread su3_eps
    void *clover = nullptr;       // clover parts of the measurement fused into flow stage 0 (first use)
    int fused_measure = 1;        // measure inside flow stage 0 where the lattice allows it (2: 128-register cap)
    bool fused_combine = true;    // that measurement's reduction inside stage 1 where the lattice allows it
    bool has_field = false;
    std::string err;
};

namespace {

thread_local std::string g_global_err;

struct CudaError : std::exception {
    std::string msg;
    explicit CudaError(std::string m) : msg(std::move(m)) {}
    const char *what() const noexcept override { return msg.c_str(); }
};

void ck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}
void ck_launch(const char *what) { ck(cudaGetLastError(), what); }

// 8 planes of Vh32 tiled sites (see lattice.cuh); FP32 adds the plain float2 plane array.
size_t field_bytes(const glac_desc &d, const Geom &g) {
    const size_t vh32 = (size_t)round32(g.Vh);
    if (d.precision == GLAC_FP64) return 8 * vh32 * 9 * sizeof(double2);
    return 8 * vh32 * 4 * sizeof(float4) + 8 * (size_t)g.Vh * sizeof(float2);
}
size_t force_bytes(const glac_desc &d, const Geom &g) {
    const size_t vh32 = (size_t)round32(g.Vh);
    return d.precision == GLAC_FP64 ? 8 * vh32 * 4 * sizeof(double2) : 8 * vh32 * 2 * sizeof(float4);
}

LinkField<double> f64(glac_ctx *c, int i) {
    LinkField<double> L;
    L.p = reinterpret_cast<double2 *>(c->field[i]);
    L.Vh = c->g.Vh;
    L.Vh32 = round32(c->g.Vh);
    return L;
}
LinkField<float> f32(glac_ctx *c, int i) {
    LinkField<float> L;
    L.Vh = c->g.Vh;
    L.Vh32 = round32(c->g.Vh);
    L.p4 = reinterpret_cast<float4 *>(c->field[i]);
    L.p2 = reinterpret_cast<float2 *>(L.p4 + (size_t)8 * 4 * L.Vh32);
    return L;
}
ForceField<double> z64(glac_ctx *c) {
    ForceField<double> Z;
    Z.p = reinterpret_cast<double2 *>(c->force);
    Z.Vh = c->g.Vh;
    Z.Vh32 = round32(c->g.Vh);
    return Z;
}
ForceField<float> z32(glac_ctx *c) {
    ForceField<float> Z;
    Z.p = reinterpret_cast<float4 *>(c->force);
    Z.Vh = c->g.Vh;
    Z.Vh32 = round32(c->g.Vh);
    return Z;
}

// Runs f with the context's device current; maps exceptions to a status.
template <typename F>
glac_status guarded(glac_ctx *c, F &&f) {
    if (!c) return GLAC_ERR_ARG;
    try {
        ck(cudaSetDevice(c->d.device), "cudaSetDevice");
        return f();
    } catch (const CudaError &e) {
        c->err = e.msg;
        return GLAC_ERR_CUDA;
    } catch (const std::exception &e) {
        c->err = e.what();
        return GLAC_ERR_ARG;
    }
}

void ensure_staging(glac_ctx *c) {
    if (!c->staging) ck(cudaMalloc(&c->staging, (size_t)c->g.V * 4 * 18 * sizeof(double)), "cudaMalloc staging");
}
void ensure_obs(glac_ctx *c, size_t n) {
    if (c->obs_cap >= n) return;
    if (c->obs_dev) cudaFree(c->obs_dev);
    c->obs_dev = nullptr;
    ck(cudaMalloc(&c->obs_dev, n * sizeof(double)), "cudaMalloc observables");
    c->obs_cap = n;
}

void measure_into(glac_ctx *c, double *dev_out) {
    if (c->d.precision == GLAC_FP64)
        launch_observables(c->g, f64(c, c->cur), c->plan, c->partial, dev_out, c->tune[FAM_OBS], c->stream);
    else
        launch_observables(c->g, f32(c, c->cur), c->plan, c->partial, dev_out, c->tune[FAM_OBS], c->stream);
    ck_launch("observables");
    c->launches += 2;
}

// Clover parts: 12 slots of 8-real matrices per site (ForceField layout with a
// slot index for the direction) followed by the 4 plaquette sums per site.
size_t clover_ah_bytes(const glac_desc &d, const Geom &g) { return 3 * force_bytes(d, g); }
size_t clover_bytes(const glac_desc &d, const Geom &g) {
    return clover_ah_bytes(d, g) + 8 * (size_t)g.Vh * (d.precision == GLAC_FP64 ? sizeof(double) : sizeof(float));
}
template <typename T> CloverParts<T> clover_view(glac_ctx *c) {
    CloverParts<T> cp;
    cp.ah.p = reinterpret_cast<decltype(cp.ah.p)>(c->clover);
    cp.ah.Vh = c->g.Vh;
    cp.ah.Vh32 = round32(c->g.Vh);
    cp.plaq = reinterpret_cast<T *>(reinterpret_cast<char *>(c->clover) + clover_ah_bytes(c->d, c->g));
    return cp;
}
// The fused measurement needs the clover parts' offsets to fit 32 bits.
bool fused_measure_usable(glac_ctx *c) {
    return c->fused_measure != 0 && clover_offsets_fit(c->g.V, c->d.precision == GLAC_FP64);
}
void ensure_clover(glac_ctx *c) {
    if (!c->clover) ck(cudaMalloc(&c->clover, clover_bytes(c->d, c->g)), "cudaMalloc clover parts");
}

void reunit(glac_ctx *c) {
    if (c->d.precision == GLAC_FP64) launch_reunitarize(c->g, f64(c, c->cur), c->stream);
    else launch_reunitarize(c->g, f32(c, c->cur), c->stream);
    ck_launch("reunitarize");
    c->launches += 1;
}

// One Luscher RK3 step: three fused stages, cur -> other -> cur -> other.
// ev (optional) receives 4 events around the three stage launches, 5 with
// meas_out (the fourth after the measurement's reduction).  meas_out
// (optional, device): the observables of the field before the step, measured
// inside stage 0 (clover parts) and reduced right after it.
void flow_step(glac_ctx *c, cudaEvent_t *ev = nullptr, double *meas_out = nullptr) {
    const double eps = c->d.flow_eps;
    const double alpha[3] = {eps * 0.25, eps * 0.8888888888888888, 0.75 * eps};
    const double beta[3] = {0.0, -(eps * 0.4722222222222222), -1.0};
    if (ev) ck(cudaEventRecord(ev[0], c->stream), "event");
    int e = 1;
    // the measurement's per-site combination and reduction: folded into stage 1
    // where the lattice's half time slices are whole 128-site blocks
    const bool in_stage1 = meas_out && c->fused_combine && obs_combine_in_stage1(c->g, c->plan);
    for (int stage = 0; stage < 3; stage++) {
        const int src = c->cur, dst = c->cur ^ 1;
        if (stage == 1 && in_stage1) {
            // the site-per-thread stage where the flow family's chosen variant has that shape
            const bool site = variant_shape(FAM_FLOW, c->d.precision == GLAC_FP32, c->tune[FAM_FLOW]) == 3;
            if (c->d.precision == GLAC_FP64)
                launch_flow_stage1_combine(c->g, f64(c, src), f64(c, dst), z64(c), c->d.exp_func, alpha[1], beta[1],
                                           clover_view<double>(c), c->plan, c->partial, meas_out, false, c->stream);
            else
                launch_flow_stage1_combine(c->g, f32(c, src), f32(c, dst), z32(c), c->d.exp_func, alpha[1], beta[1],
                                           clover_view<float>(c), c->plan, c->partial, meas_out, site, c->stream);
            ck_launch("flow stage 1 with the measurement's reduction");
            c->launches += 2;
        } else if (stage == 0 && meas_out) {
            ensure_clover(c);
            // 1: link per thread, compiler's registers; 2: the same capped at 128;
            // 3 (FP32): site per thread, upper staple products shared; 4 (FP32):
            // link per thread capped at 96 (five blocks per SM, small spill)
            const int fm = c->fused_measure;
            const int regs = fm == 2 ? 128 : fm == 3 ? 3 : fm == 4 ? 96 : 0;
            if (c->d.precision == GLAC_FP64) {
                const CloverParts<double> cp = clover_view<double>(c);
                launch_flow_stage0_meas(c->g, f64(c, src), f64(c, dst), z64(c), cp, c->d.exp_func, alpha[0], regs,
                                        c->stream);
                ck_launch("flow stage 0 with measurement");
                if (ev) ck(cudaEventRecord(ev[e++], c->stream), "event");
                if (!in_stage1) launch_obs_combine(c->g, cp, c->plan, c->partial, meas_out, c->stream);
            } else {
                const CloverParts<float> cp = clover_view<float>(c);
                launch_flow_stage0_meas(c->g, f32(c, src), f32(c, dst), z32(c), cp, c->d.exp_func, alpha[0], regs,
                                        c->stream);
                ck_launch("flow stage 0 with measurement");
                if (ev) ck(cudaEventRecord(ev[e++], c->stream), "event");
                if (!in_stage1) launch_obs_combine(c->g, cp, c->plan, c->partial, meas_out, c->stream);
            }
            ck_launch("measurement from clover parts");
            c->launches += in_stage1 ? 1 : 3;
        } else {
            if (c->d.precision == GLAC_FP64)
                launch_flow_stage(c->g, f64(c, src), f64(c, dst), z64(c), stage, c->d.exp_func, alpha[stage],
                                  beta[stage], c->tune[FAM_FLOW], c->stream);
            else
                launch_flow_stage(c->g, f32(c, src), f32(c, dst), z32(c), stage, c->d.exp_func, alpha[stage],
                                  beta[stage], c->tune[FAM_FLOW], c->stream);
            ck_launch("flow stage");
            c->launches += 1;
        }
        c->cur = dst;
        if (ev) ck(cudaEventRecord(ev[e++], c->stream), "event");
    }
}

glac_status need_field(glac_ctx *c) {
    if (!c->has_field) {
        c->err = "no gauge field set (call glac_cold_start, glac_hot_start or glac_set_links first)";
        return GLAC_ERR_STATE;
    }
    return GLAC_OK;
}

}  // namespace

extern "C" {

const char *glac_last_error(const glac_ctx *ctx) { return ctx ? ctx->err.c_str() : g_global_err.c_str(); }
const char *glac_global_error(void) { return g_global_err.c_str(); }
void *glac_stream(glac_ctx *ctx) { return ctx ? (void *)ctx->stream : nullptr; }
uint64_t glac_launch_count(const glac_ctx *ctx) { return ctx ? ctx->launches : 0; }

glac_status glac_create(const glac_desc *desc, glac_ctx **out) {
    if (!desc || !out) { g_global_err = "null argument"; return GLAC_ERR_ARG; }
    *out = nullptr;
    const glac_desc &d = *desc;
    long long V = 1;
    for (int k = 0; k < 4; k++) {
        if (d.dims[k] < 4 || (d.dims[k] & 1)) {
            g_global_err = "every lattice extent must be even and at least 4";
            return GLAC_ERR_ARG;
        }
        if (d.dims[k] > (1ll << 29) / V) {  // checked before the product, so V cannot wrap
            g_global_err = "lattice too large (V > 2^29)";
            return GLAC_ERR_ARG;
        }
        V *= d.dims[k];
    }
    if (!field_offsets_fit(V, d.precision == GLAC_FP64)) {
        g_global_err = "lattice too large for 32-bit field offsets (FP64: V < 1.19e8, FP32: V < 2.68e8 sites)";
        return GLAC_ERR_ARG;
    }
    if (d.precision != GLAC_FP64 && d.precision != GLAC_FP32) { g_global_err = "bad precision"; return GLAC_ERR_ARG; }
    if (d.exp_func < 0 || d.exp_func > 3) { g_global_err = "bad exp_func"; return GLAC_ERR_ARG; }
    if (d.n_updates < 0) { g_global_err = "n_updates must be >= 0"; return GLAC_ERR_ARG; }
    if (!(d.su3_eps > 0.0 && d.su3_eps < 1.0)) { g_global_err = "su3_eps must lie in (0, 1)"; return GLAC_ERR_ARG; }
    if (d.dims[3] > 1024) { g_global_err = "Nt > 1024 is not supported"; return GLAC_ERR_ARG; }
    glac_ctx *c = new glac_ctx();
    c->d = d;
    c->g = make_geom(d.dims);
    c->plan = make_obs_plan(c->g);
    // the faster fused-measurement kernel per precision on B200 at 32^3 x 64:
    // FP32 with the 128-register cap (2.50 vs 2.61 ms per measured flow step),
    // FP64 uncapped (6.33 vs 6.77 ms)
    c->fused_measure = d.precision == GLAC_FP32 ? 2 : 1;
    try {
        ck(cudaSetDevice(d.device), "cudaSetDevice");
        ck(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
        for (int i = 0; i < 2; i++) ck(cudaMalloc(&c->field[i], field_bytes(d, c->g)), "cudaMalloc field");
        ck(cudaMalloc(&c->force, force_bytes(d, c->g)), "cudaMalloc force");
        ck(cudaMalloc(&c->partial, (size_t)3 * c->plan.nblocks * sizeof(double)), "cudaMalloc partials");
        ck(cudaMalloc(&c->acc_dev, sizeof(unsigned long long)), "cudaMalloc counter");
        ck(cudaMalloc(&c->scalar_dev, sizeof(double)), "cudaMalloc scalar");
        ensure_obs(c, 3 + (size_t)d.dims[3]);
    } catch (const CudaError &e) {
        g_global_err = e.msg;
        glac_destroy(c);
        return GLAC_ERR_CUDA;
    }
    *out = c;
    return GLAC_OK;
}

void glac_destroy(glac_ctx *c) {
    if (!c) return;
    cudaSetDevice(c->d.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int i = 0; i < 2; i++) if (c->field[i]) cudaFree(c->field[i]);
    if (c->force) cudaFree(c->force);
    if (c->partial) cudaFree(c->partial);
    if (c->partial4) cudaFree(c->partial4);
    if (c->obs_dev) cudaFree(c->obs_dev);
    if (c->acc_dev) cudaFree(c->acc_dev);
    if (c->staging) cudaFree(c->staging);
    if (c->scalar_dev) cudaFree(c->scalar_dev);
    if (c->net_params) cudaFree(c->net_params);
    if (c->net_pack) cudaFree(c->net_pack);
    if (c->esj_grid) cudaFree(c->esj_grid);
    if (c->clover) cudaFree(c->clover);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

glac_status glac_sync(glac_ctx *c) {
    return guarded(c, [&] {
        ck(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
        return GLAC_OK;
    });
}

glac_status glac_set_option(glac_ctx *c, const char *key, long value) {
    if (!c || !key) return GLAC_ERR_ARG;
    if (std::string(key) == "fused_measure") {
        if (value < 0 || value > 4 || (value >= 3 && c->d.precision != GLAC_FP32)) {
            c->err = "fused_measure takes 0 (off), 1 (on), 2 (on, 128-register kernel) or, in FP32, 3 (on, a "
                     "thread per site) or 4 (on, 96-register kernel)";
            return GLAC_ERR_ARG;
        }
        c->fused_measure = (int)value;
        return GLAC_OK;
    }
    if (std::string(key) == "fused_combine") {
        if (value != 0 && value != 1) {
            c->err = "fused_combine takes 0 or 1";
            return GLAC_ERR_ARG;
        }
        c->fused_combine = value != 0;
        return GLAC_OK;
    }
    if (std::string(key) == "su2_sign_flips") {
        if (value != 0 && value != 1) {
            c->err = "su2_sign_flips takes 0 or 1";
            return GLAC_ERR_ARG;
        }
        c->prop.flips = value != 0;
        return GLAC_OK;
    }
    c->err = std::string("unknown option ") + key;
    return GLAC_ERR_ARG;
}

glac_status glac_cold_start(glac_ctx *c) {
    return guarded(c, [&] {
        if (c->d.precision == GLAC_FP64) launch_cold(c->g, f64(c, c->cur), c->stream);
        else launch_cold(c->g, f32(c, c->cur), c->stream);
        ck_launch("cold start");
        c->launches++;
        c->has_field = true;
        return GLAC_OK;
    });
}

glac_status glac_hot_start(glac_ctx *c, uint64_t seed) {
    return guarded(c, [&] {
        if (c->d.precision == GLAC_FP64) launch_haar(c->g, f64(c, c->cur), seed, c->d.stream_id, c->stream);
        else launch_haar(c->g, f32(c, c->cur), seed, c->d.stream_id, c->stream);
        ck_launch("hot start");
        c->launches++;
        c->has_field = true;
        return GLAC_OK;
    });
}

glac_status glac_rst_start(glac_ctx *c, uint64_t seed) {
    return guarded(c, [&] {
        if (c->d.precision == GLAC_FP64) launch_rst_start(c->g, f64(c, c->cur), c->d.su3_eps, seed, c->d.stream_id, c->stream);
        else launch_rst_start(c->g, f32(c, c->cur), c->d.su3_eps, seed, c->d.stream_id, c->stream);
        ck_launch("rst start");
        c->launches++;
        c->has_field = true;
        return GLAC_OK;
    });
}

glac_status glac_set_links_device(glac_ctx *c, const double *dev) {
    return guarded(c, [&] {
        if (!dev) { c->err = "null field"; return GLAC_ERR_ARG; }
        if (c->d.precision == GLAC_FP64) launch_aos_to_soa(c->g, dev, f64(c, c->cur), c->stream);
        else launch_aos_to_soa(c->g, dev, f32(c, c->cur), c->stream);
        ck_launch("aos->soa");
        c->launches++;
        c->has_field = true;
        return GLAC_OK;
    });
}

glac_status glac_get_links_device(glac_ctx *c, double *dev) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        if (c->d.precision == GLAC_FP64) launch_soa_to_aos(c->g, f64(c, c->cur), dev, c->stream);
        else launch_soa_to_aos(c->g, f32(c, c->cur), dev, c->stream);
        ck_launch("soa->aos");
        c->launches++;
        return GLAC_OK;
    });
}

glac_status glac_set_links(glac_ctx *c, const double *host) {
    return guarded(c, [&] {
        if (!host) { c->err = "null field"; return GLAC_ERR_ARG; }
        ensure_staging(c);
        ck(cudaMemcpyAsync(c->staging, host, (size_t)c->g.V * 72 * sizeof(double), cudaMemcpyHostToDevice,
                           c->stream),
           "H2D links");
        glac_status s = glac_set_links_device(c, c->staging);
        if (s != GLAC_OK) return s;
        ck(cudaStreamSynchronize(c->stream), "sync");
        return GLAC_OK;
    });
}

glac_status glac_get_links(glac_ctx *c, double *host) {
    return guarded(c, [&] {
        if (!host) { c->err = "null field"; return GLAC_ERR_ARG; }
        ensure_staging(c);
        glac_status s = glac_get_links_device(c, c->staging);
        if (s != GLAC_OK) return s;
        ck(cudaMemcpyAsync(host, c->staging, (size_t)c->g.V * 72 * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream),
           "D2H links");
        ck(cudaStreamSynchronize(c->stream), "sync");
        return GLAC_OK;
    });
}

glac_status glac_copy_field(glac_ctx *dst, glac_ctx *src) {
    if (!dst || !src) return GLAC_ERR_ARG;
    return guarded(dst, [&] {
        if (!src->has_field) { dst->err = "source has no field"; return GLAC_ERR_STATE; }
        if (src->d.precision != dst->d.precision || memcmp(src->d.dims, dst->d.dims, sizeof(src->d.dims))) {
            dst->err = "contexts differ in precision or dimensions";
            return GLAC_ERR_ARG;
        }
        ck(cudaStreamSynchronize(src->stream), "sync source");
        ck(cudaMemcpyAsync(dst->field[dst->cur], src->field[src->cur], field_bytes(dst->d, dst->g),
                           cudaMemcpyDeviceToDevice, dst->stream),
           "copy field");
        dst->has_field = true;
        return GLAC_OK;
    });
}

glac_status glac_reunitarize(glac_ctx *c) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        reunit(c);
        return GLAC_OK;
    });
}

glac_status glac_unitarity_violation(glac_ctx *c, double *out) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        if (c->d.precision == GLAC_FP64) launch_max_unitarity_dev(c->g, f64(c, c->cur), c->scalar_dev, c->stream);
        else launch_max_unitarity_dev(c->g, f32(c, c->cur), c->scalar_dev, c->stream);
        ck_launch("unitarity");
        c->launches++;
        ck(cudaMemcpyAsync(out, c->scalar_dev, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "sync");
        return GLAC_OK;
    });
}

glac_status glac_metropolis(glac_ctx *c, int n_sweeps, double *acceptance) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        if (n_sweeps < 0) { c->err = "n_sweeps < 0"; return GLAC_ERR_ARG; }
        ck(cudaMemsetAsync(c->acc_dev, 0, sizeof(unsigned long long), c->stream), "memset");
        for (int i = 0; i < n_sweeps; i++) {
            for (int k = 0; k < 8; k++) {
                const int mu = k >> 1, p = k & 1;
                if (c->d.precision == GLAC_FP64)
                    launch_metropolis(c->g, f64(c, c->cur), mu, p, c->d.beta, c->d.su3_eps, c->d.n_updates,
                                      c->d.seed, c->sweep, c->d.stream_id, c->acc_dev, c->tune[FAM_METRO],
                                      c->prop, c->stream);
                else
                    launch_metropolis(c->g, f32(c, c->cur), mu, p, c->d.beta, c->d.su3_eps, c->d.n_updates,
                                      c->d.seed, c->sweep, c->d.stream_id, c->acc_dev, c->tune[FAM_METRO],
                                      c->prop, c->stream);
                ck_launch("metropolis");
                c->launches++;
            }
            c->sweep++;
            if (c->d.reunit_interval > 0 && c->d.precision == GLAC_FP32 && c->sweep % c->d.reunit_interval == 0)
                reunit(c);
        }
        if (acceptance) {
            unsigned long long acc = 0;
            ck(cudaMemcpyAsync(&acc, c->acc_dev, sizeof(acc), cudaMemcpyDeviceToHost, c->stream), "D2H");
            ck(cudaStreamSynchronize(c->stream), "sync");
            const double per = 4.0 * (double)c->d.n_updates * (double)c->g.V * (double)(n_sweeps > 0 ? n_sweeps : 1);
            *acceptance = per > 0 ? (double)acc / per : 0.0;
        }
        return GLAC_OK;
    });
}

glac_status glac_measure(glac_ctx *c, double *obs) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        const size_t n = 3 + (size_t)c->g.N[3];
        ensure_obs(c, n);
        measure_into(c, c->obs_dev);
        if (obs) {
            ck(cudaMemcpyAsync(obs, c->obs_dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H obs");
            ck(cudaStreamSynchronize(c->stream), "sync");
        }
        return GLAC_OK;
    });
}

glac_status glac_measure_density(glac_ctx *c, double *obs, double *q_density, double *e_density) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        if (!q_density || !e_density) {
            c->err = "null density output";
            return GLAC_ERR_ARG;
        }
        const size_t n = 3 + (size_t)c->g.N[3], V = (size_t)c->g.V;
        ensure_obs(c, n);
        ensure_staging(c);  // V * 72 doubles: room for both densities
        double *dq = c->staging, *de = c->staging + V;
        if (c->d.precision == GLAC_FP64)
            launch_observables_density(c->g, f64(c, c->cur), c->plan, c->partial, c->obs_dev, dq, de, c->stream);
        else
            launch_observables_density(c->g, f32(c, c->cur), c->plan, c->partial, c->obs_dev, dq, de, c->stream);
        ck_launch("observables density");
        c->launches += 2;
        if (obs) ck(cudaMemcpyAsync(obs, c->obs_dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaMemcpyAsync(q_density, dq, V * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H q");
        ck(cudaMemcpyAsync(e_density, de, V * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H e");
        ck(cudaStreamSynchronize(c->stream), "sync");
        return GLAC_OK;
    });
}

glac_status glac_measure_weinberg(glac_ctx *c, double *obs) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        if (!obs) {
            c->err = "null output";
            return GLAC_ERR_ARG;
        }
        const size_t n = 4 + 2 * (size_t)c->g.N[3];
        ensure_obs(c, n);
        if (!c->partial4) ck(cudaMalloc(&c->partial4, 4 * (size_t)c->plan.nblocks * sizeof(double)), "partials");
        if (c->d.precision == GLAC_FP64) launch_weinberg(c->g, f64(c, c->cur), c->plan, c->partial4, c->obs_dev, c->stream);
        else launch_weinberg(c->g, f32(c, c->cur), c->plan, c->partial4, c->obs_dev, c->stream);
        ck_launch("weinberg");
        c->launches += 2;
        ck(cudaMemcpyAsync(obs, c->obs_dev, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "D2H");
        ck(cudaStreamSynchronize(c->stream), "sync");
        return GLAC_OK;
    });
}

glac_status glac_get_sweep(glac_ctx *c, uint32_t *sweep) {
    if (!c || !sweep) return GLAC_ERR_ARG;
    *sweep = c->sweep;
    return GLAC_OK;
}

glac_status glac_set_sweep(glac_ctx *c, uint32_t sweep) {
    if (!c) return GLAC_ERR_ARG;
    c->sweep = sweep;
    return GLAC_OK;
}

glac_status glac_flow(glac_ctx *c, int n_steps, double *obs) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        if (n_steps < 0) { c->err = "n_steps < 0"; return GLAC_ERR_ARG; }
        const size_t per = 3 + (size_t)c->g.N[3];
        // Measurement after step i: inside stage 0 of step i + 1 where the lattice
        // allows (the field it flows is the one to measure), else a pass of its
        // own; the last one always a pass of its own.
        const bool fused = obs && fused_measure_usable(c);
        if (obs) {
            ensure_obs(c, per * (size_t)(n_steps + 1));
            if (!fused || n_steps == 0) measure_into(c, c->obs_dev);
        }
        for (int i = 0; i < n_steps; i++) {
            flow_step(c, nullptr, fused ? c->obs_dev + per * (size_t)i : nullptr);
            if (c->d.reunit_interval > 0 && c->d.precision == GLAC_FP32 && (i + 1) % c->d.reunit_interval == 0)
                reunit(c);
            if (obs && (!fused || i == n_steps - 1)) measure_into(c, c->obs_dev + per * (size_t)(i + 1));
        }
        if (obs) {
            ck(cudaMemcpyAsync(obs, c->obs_dev, per * (size_t)(n_steps + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                               c->stream),
               "D2H obs");
            ck(cudaStreamSynchronize(c->stream), "sync");
        }
        return GLAC_OK;
    });
}

glac_status glac_flow_stage_times(glac_ctx *c, int n_steps, double *seconds3) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        if (n_steps <= 0 || !seconds3) { c->err = "n_steps must be > 0"; return GLAC_ERR_ARG; }
        cudaEvent_t ev[4];
        for (int i = 0; i < 4; i++) ck(cudaEventCreate(&ev[i]), "event create");
        double acc[3] = {0, 0, 0};
        for (int k = 0; k < n_steps; k++) {
            flow_step(c, ev);
            ck(cudaEventSynchronize(ev[3]), "event sync");
            for (int i = 0; i < 3; i++) {
                float ms = 0.f;
                ck(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]), "elapsed");
                acc[i] += ms * 1e-3;
            }
        }
        for (int i = 0; i < 4; i++) cudaEventDestroy(ev[i]);
        for (int i = 0; i < 3; i++) seconds3[i] = acc[i] / n_steps;
        return GLAC_OK;
    });
}

glac_status glac_flow_stage_times_measured(glac_ctx *c, int n_steps, double *seconds4) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        if (n_steps <= 0 || !seconds4) { c->err = "n_steps must be > 0"; return GLAC_ERR_ARG; }
        if (!fused_measure_usable(c)) {
            c->err = "the measurement is not fused into flow stage 0 for this context (fused_measure = 0, or the "
                     "lattice is too large for the clover parts' 32-bit offsets)";
            return GLAC_ERR_STATE;
        }
        const size_t per = 3 + (size_t)c->g.N[3];
        ensure_obs(c, per);
        cudaEvent_t ev[5];
        for (int i = 0; i < 5; i++) ck(cudaEventCreate(&ev[i]), "event create");
        double acc[4] = {0, 0, 0, 0};
        for (int k = 0; k < n_steps; k++) {
            flow_step(c, ev, c->obs_dev);
            ck(cudaEventSynchronize(ev[4]), "event sync");
            for (int i = 0; i < 4; i++) {
                float ms = 0.f;
                ck(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]), "elapsed");
                acc[i] += ms * 1e-3;
            }
        }
        for (int i = 0; i < 5; i++) cudaEventDestroy(ev[i]);
        for (int i = 0; i < 4; i++) seconds4[i] = acc[i] / n_steps;
        return GLAC_OK;
    });
}

// Launch-variant autotuner: times every variant of the flow-stage, Metropolis
// and observable kernels on this context's lattice and keeps the fastest.
// The field, the sweep counter and the Philox stream are restored afterwards.
// report (optional, 3 x kMaxVariants doubles) receives the mean seconds per
// call of each variant (0 where a family has fewer variants).
glac_status glac_autotune(glac_ctx *c, int reps, double *report) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        if (reps <= 0) reps = 3;
        const bool fp32 = c->d.precision == GLAC_FP32;
        void *backup = nullptr;
        ck(cudaMalloc(&backup, field_bytes(c->d, c->g)), "cudaMalloc autotune backup");
        ck(cudaMemcpyAsync(backup, c->field[c->cur], field_bytes(c->d, c->g), cudaMemcpyDeviceToDevice, c->stream),
           "backup");
        const uint32_t sweep0 = c->sweep;
        const int cur0 = c->cur;
        cudaEvent_t e0, e1;
        ck(cudaEventCreate(&e0), "event");
        ck(cudaEventCreate(&e1), "event");
        auto restore = [&]() {
            c->cur = cur0;
            c->sweep = sweep0;
            ck(cudaMemcpyAsync(c->field[c->cur], backup, field_bytes(c->d, c->g), cudaMemcpyDeviceToDevice,
                               c->stream),
               "restore");
        };
        double table[3][kMaxVariants] = {{0}};
        for (int fam = 0; fam < 3; fam++) {
            const int nv = num_variants((Family)fam, fp32);
            int best = 0;
            double best_t = 1e300;
            for (int v = 0; v < nv; v++) {
                c->tune[fam] = v;
                for (int pass = 0; pass < 2; pass++) {  // pass 0 warms up
                    ck(cudaEventRecord(e0, c->stream), "event");
                    for (int r = 0; r < reps; r++) {
                        // flows measure after every step where the measurement runs
                        // inside the stages, so the flow family is timed on such steps
                        if (fam == FAM_FLOW) {
                            if (fused_measure_usable(c)) flow_step(c, nullptr, c->obs_dev);
                            else flow_step(c);
                        } else if (fam == FAM_METRO) {
                            for (int k = 0; k < 8; k++) {
                                if (fp32)
                                    launch_metropolis(c->g, f32(c, c->cur), k >> 1, k & 1, c->d.beta, c->d.su3_eps,
                                                      c->d.n_updates, c->d.seed, c->sweep, c->d.stream_id, c->acc_dev,
                                                      v, c->prop, c->stream);
                                else
                                    launch_metropolis(c->g, f64(c, c->cur), k >> 1, k & 1, c->d.beta, c->d.su3_eps,
                                                      c->d.n_updates, c->d.seed, c->sweep, c->d.stream_id, c->acc_dev,
                                                      v, c->prop, c->stream);
                                ck_launch("metropolis");
                            }
                        } else measure_into(c, c->obs_dev);
                    }
                    ck(cudaEventRecord(e1, c->stream), "event");
                    ck(cudaEventSynchronize(e1), "event sync");
                    restore();
                }
                float ms = 0.f;
                ck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
                const double t = ms * 1e-3 / reps;
                table[fam][v] = t;
                if (t < best_t) { best_t = t; best = v; }
            }
            c->tune[fam] = best;
        }
        ck(cudaStreamSynchronize(c->stream), "sync");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaFree(backup);
        if (report)
            for (int f = 0; f < 3; f++)
                for (int v = 0; v < kMaxVariants; v++) report[3 * 0 + f * kMaxVariants + v] = table[f][v];
        return GLAC_OK;
    });
}

glac_status glac_get_tuning(glac_ctx *c, int *variants3) {
    if (!c || !variants3) return GLAC_ERR_ARG;
    for (int f = 0; f < 3; f++) variants3[f] = c->tune[f];
    return GLAC_OK;
}

glac_status glac_set_tuning(glac_ctx *c, const int *variants3) {
    if (!c || !variants3) return GLAC_ERR_ARG;
    const bool fp32 = c->d.precision == GLAC_FP32;
    for (int f = 0; f < 3; f++)
        if (variants3[f] < 0 || variants3[f] >= num_variants((Family)f, fp32)) {
            c->err = "tuning variant out of range";
            return GLAC_ERR_ARG;
        }
    for (int f = 0; f < 3; f++) c->tune[f] = variants3[f];
    return GLAC_OK;
}

glac_status glac_flow_configuration(glac_ctx *c, const double *host_links, int n_steps, double *obs) {
    glac_status s = glac_set_links(c, host_links);
    if (s != GLAC_OK) return s;
    return glac_flow(c, n_steps, obs);
}

glac_status glac_staples(glac_ctx *c, double *host_out) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        ensure_staging(c);
        if (c->d.precision == GLAC_FP64) launch_staples_aos(c->g, f64(c, c->cur), c->staging, c->stream);
        else launch_staples_aos(c->g, f32(c, c->cur), c->staging, c->stream);
        ck_launch("staples");
        c->launches++;
        ck(cudaMemcpyAsync(host_out, c->staging, (size_t)c->g.V * 72 * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream),
           "D2H");
        ck(cudaStreamSynchronize(c->stream), "sync");
        return GLAC_OK;
    });
}

glac_status glac_force(glac_ctx *c, double *host_out) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        ensure_staging(c);
        if (c->d.precision == GLAC_FP64) launch_force_aos(c->g, f64(c, c->cur), c->staging, c->stream);
        else launch_force_aos(c->g, f32(c, c->cur), c->staging, c->stream);
        ck_launch("force");
        c->launches++;
        ck(cudaMemcpyAsync(host_out, c->staging, (size_t)c->g.V * 72 * sizeof(double), cudaMemcpyDeviceToHost,
                           c->stream),
           "D2H");
        ck(cudaStreamSynchronize(c->stream), "sync");
        return GLAC_OK;
    });
}

}  // extern "C"

// Standalone batch entry points (no context): device buffers live for the call.
namespace {
template <typename F>
glac_status standalone(F &&f) {
    try {
        return f();
    } catch (const CudaError &e) {
        g_global_err = e.msg;
        return GLAC_ERR_CUDA;
    } catch (const std::exception &e) {
        g_global_err = e.what();
        return GLAC_ERR_ARG;
    }
}
struct DevBuf {
    void *p = nullptr;
    explicit DevBuf(size_t n) { ck(cudaMalloc(&p, n ? n : 1), "cudaMalloc"); }
    ~DevBuf() { if (p) cudaFree(p); }
};
}  // namespace

extern "C" {

glac_status glac_exp_batch(int precision, int exp_func, const double *host_in, long n, double *host_out) {
    return standalone([&] {
        if (n < 0 || (precision != GLAC_FP64 && precision != GLAC_FP32) || exp_func < 0 || exp_func > 3) {
            g_global_err = "bad argument";
            return GLAC_ERR_ARG;
        }
        if (n == 0) return GLAC_OK;
        const size_t bytes = (size_t)n * 18 * sizeof(double);
        DevBuf in(bytes), out(bytes);
        ck(cudaMemcpy(in.p, host_in, bytes, cudaMemcpyHostToDevice), "H2D");
        if (precision == GLAC_FP64) launch_exp_batch<double>(exp_func, (const double *)in.p, (double *)out.p, n, 0);
        else launch_exp_batch<float>(exp_func, (const double *)in.p, (double *)out.p, n, 0);
        ck_launch("exp batch");
        ck(cudaMemcpy(host_out, out.p, bytes, cudaMemcpyDeviceToHost), "D2H");
        return GLAC_OK;
    });
}

glac_status glac_delta_s_batch(int precision, double beta, long n, const double *host_U, const double *host_Uprime,
                               const double *host_A, double *host_out) {
    return standalone([&] {
        if (n < 0 || (precision != GLAC_FP64 && precision != GLAC_FP32)) {
            g_global_err = "bad argument";
            return GLAC_ERR_ARG;
        }
        if (n == 0) return GLAC_OK;
        const size_t mb = (size_t)n * 18 * sizeof(double);
        DevBuf U(mb), Up(mb), A(mb), out((size_t)n * sizeof(double));
        ck(cudaMemcpy(U.p, host_U, mb, cudaMemcpyHostToDevice), "H2D");
        ck(cudaMemcpy(Up.p, host_Uprime, mb, cudaMemcpyHostToDevice), "H2D");
        ck(cudaMemcpy(A.p, host_A, mb, cudaMemcpyHostToDevice), "H2D");
        if (precision == GLAC_FP64)
            launch_delta_s<double>(beta, n, (const double *)U.p, (const double *)Up.p, (const double *)A.p,
                                   (double *)out.p, 0);
        else
            launch_delta_s<float>(beta, n, (const double *)U.p, (const double *)Up.p, (const double *)A.p,
                                  (double *)out.p, 0);
        ck_launch("delta S");
        ck(cudaMemcpy(host_out, out.p, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost), "D2H");
        return GLAC_OK;
    });
}

glac_status glac_accept_fed(int precision, double beta, long n_links, int n_hits, double *host_U,
                            const double *host_A, const double *host_X, const double *host_r,
                            unsigned char *host_accept) {
    return standalone([&] {
        if (n_links < 0 || n_hits < 0 || (precision != GLAC_FP64 && precision != GLAC_FP32)) {
            g_global_err = "bad argument";
            return GLAC_ERR_ARG;
        }
        if (n_links == 0) return GLAC_OK;
        const size_t mb = (size_t)n_links * 18 * sizeof(double);
        const size_t xb = mb * (size_t)n_hits, rb = (size_t)n_links * n_hits * sizeof(double);
        const size_t ab = (size_t)n_links * n_hits;
        DevBuf U(mb), A(mb), X(xb), r(rb), acc(ab);
        ck(cudaMemcpy(U.p, host_U, mb, cudaMemcpyHostToDevice), "H2D");
        ck(cudaMemcpy(A.p, host_A, mb, cudaMemcpyHostToDevice), "H2D");
        if (xb) ck(cudaMemcpy(X.p, host_X, xb, cudaMemcpyHostToDevice), "H2D");
        if (rb) ck(cudaMemcpy(r.p, host_r, rb, cudaMemcpyHostToDevice), "H2D");
        if (precision == GLAC_FP64)
            launch_accept_fed<double>(beta, n_links, n_hits, (double *)U.p, (const double *)A.p, (const double *)X.p,
                                      (const double *)r.p, (unsigned char *)acc.p, 0);
        else
            launch_accept_fed<float>(beta, n_links, n_hits, (double *)U.p, (const double *)A.p, (const double *)X.p,
                                     (const double *)r.p, (unsigned char *)acc.p, 0);
        ck_launch("accept fed");
        ck(cudaMemcpy(host_U, U.p, mb, cudaMemcpyDeviceToHost), "D2H");
        if (ab) ck(cudaMemcpy(host_accept, acc.p, ab, cudaMemcpyDeviceToHost), "D2H");
        return GLAC_OK;
    });
}


glac_status glac_set_proposal_net(glac_ctx *c, const float *params, double eps_min, double eps_max) {
    return guarded(c, [&] {
        if (!params) {
            c->prop.net = nullptr;
            return GLAC_OK;
        }
        if (!(eps_min > 0.0 && eps_min < eps_max && eps_max <= 1.0)) {
            c->err = "proposal spread range must satisfy 0 < eps_min < eps_max <= 1";
            return GLAC_ERR_ARG;
        }
        for (int k = 0; k < kMlpParams; k++)
            if (!std::isfinite(params[k])) {
                c->err = "non-finite network parameter";
                return GLAC_ERR_NONFINITE;
            }
        if (!c->net_params) ck(cudaMalloc(&c->net_params, kMlpParams * sizeof(float)), "alloc net");
        if (!c->net_pack) ck(cudaMalloc(&c->net_pack, kPackWords * sizeof(uint32_t)), "alloc net");
        ck(cudaMemcpyAsync(c->net_params, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice, c->stream),
           "upload net");
        launch_mlp_pack(c->net_params, c->net_pack, c->stream);
        ck_launch("pack net");
        c->launches++;
        ck(cudaStreamSynchronize(c->stream), "sync");
        c->prop.net = c->net_pack;
        c->prop.eps_min = (float)eps_min;
        c->prop.eps_max = (float)eps_max;
        return GLAC_OK;
    });
}

glac_status glac_esj_data(glac_ctx *c, int n_eps, const double *eps_grid, int trials, int stride, uint32_t snapshot,
                          float *dev_features, float *dev_esj, uint32_t *dev_link_ids, long long capacity,
                          long long *n_rows) {
    return guarded(c, [&] {
        glac_status s = need_field(c);
        if (s != GLAC_OK) return s;
        if (n_eps < 0 || n_eps > 64 || (n_eps > 0 && (!eps_grid || !dev_esj || trials < 1)) || !dev_features ||
            stride < 1 || stride > c->g.Vh) {
            c->err = "esj: need 0 <= n_eps <= 64 (grid, output and trials >= 1 when > 0), features, 1 <= stride <= V/2";
            return GLAC_ERR_ARG;
        }
        if (c->d.n_updates > 16) {
            c->err = "esj: at most 16 hits per link";
            return GLAC_ERR_ARG;
        }
        for (int k = 0; k < n_eps; k++)
            if (!(eps_grid[k] > 0.0 && eps_grid[k] <= 1.0)) {
                c->err = "esj: spreads must lie in (0, 1]";
                return GLAC_ERR_ARG;
            }
        const int ns = c->g.Vh / stride;
        const int offset = (int)((snapshot * 7919u) % (uint32_t)stride);
        const long long rows = 8ll * ns;
        if (n_rows) *n_rows = rows;
        if (rows > capacity) {
            c->err = "esj: capacity below 8 * (V/2 / stride) rows";
            return GLAC_ERR_ARG;
        }
        if (n_eps > 0) {
            if (!c->esj_grid) ck(cudaMalloc(&c->esj_grid, 64 * sizeof(float)), "alloc grid");
            float g32[64];
            for (int k = 0; k < n_eps; k++) g32[k] = (float)eps_grid[k];
            ck(cudaMemcpyAsync(c->esj_grid, g32, n_eps * sizeof(float), cudaMemcpyHostToDevice, c->stream), "grid");
        }
        if (c->d.precision == GLAC_FP64)
            launch_esj(c->g, f64(c, c->cur), c->d.beta, c->d.n_updates, n_eps, c->esj_grid, trials, stride, offset, ns,
                       c->d.seed, snapshot, c->d.stream_id, c->prop.flips, dev_features, dev_esj, dev_link_ids,
                       c->stream);
        else
            launch_esj(c->g, f32(c, c->cur), c->d.beta, c->d.n_updates, n_eps, c->esj_grid, trials, stride, offset, ns,
                       c->d.seed, snapshot, c->d.stream_id, c->prop.flips, dev_features, dev_esj, dev_link_ids,
                       c->stream);
        ck_launch("esj");
        c->launches++;
        ck(cudaStreamSynchronize(c->stream), "sync");
        return GLAC_OK;
    });
}

}  // extern "C"
