// Batched ensemble of independent lattices (glac_ensemble_* in include/glac_b200.h).
// No counterpart in the reference, which runs one lattice per job.
//
// All lattices of an ensemble share one device allocation per field role (the
// Markov chain and two flow buffers, identical offsets) plus one force buffer.
// Each phase of the schedule -- a (mu, parity) Metropolis sub-sweep, an RK3
// flow stage, an observable pass -- is one launch over every lattice: blocks
// find their lattice in a prefix table of per-lattice block counts and run the
// single-lattice kernel body on it, so small lattices fill the GPU together.
// glac_ensemble_run records the whole schedule (sweeps, the copy into the flow
// buffers, flow steps with a measurement after each) as one CUDA graph, captured
// on the first call for a (sweeps, steps) pair and replayed after; the sweep
// counter of the Philox streams lives in device memory, so replays draw fresh
// numbers.
#include "../../include/glac_b200.h"
#include "kernels.cuh"

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <exception>
#include <string>
#include <vector>

using namespace glac;

struct glac_ensemble {
    glac_desc d;  // common settings; dims unused
    int M = 0;
    std::vector<Geom> geo;
    std::vector<ObsPlan> plan;
    std::vector<double> beta;
    std::vector<size_t> off_field, off_force, off_partial;  // bytes, bytes, doubles
    size_t field_total = 0, force_total = 0, partial_total = 0;
    void *field[3] = {nullptr, nullptr, nullptr};
    void *force = nullptr;
    double *partial = nullptr;
    void *slots = nullptr;
    int *start[ENS_NPHASE] = {nullptr, nullptr, nullptr, nullptr};
    int nblk[ENS_NPHASE] = {0, 0, 0, 0};
    unsigned long long *acc = nullptr;
    uint32_t *sweep_dev = nullptr;
    uint32_t sweep = 0;
    double *obs = nullptr;
    size_t obs_cap = 0;
    int obs_steps = -1;  // the layout the slots' obs pointers describe
    double *staging = nullptr;
    size_t staging_cap = 0;
    void *clover = nullptr;                // clover parts of the measurement inside flow stage 0
    std::vector<size_t> off_clover;        // bytes
    bool fused_measure = true;             // measure inside flow stage 0 (all lattices fit the parts' offsets)
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    int graph_sweeps = -1, graph_steps = -1;
    bool flips = true;
    bool has_field = false;
    int tune[3] = {0, 0, 0};
    GridBarrier *barrier = nullptr;             // the persistent launch's grid barrier (first use)
    unsigned long long persistent_wait_ns = 5000000000ull;  // its wait limit (5 s)
    int persistent_test_stall = 0;              // test mode: one block never arrives
    uint64_t launches = 0;
    std::string err;
};

namespace {

thread_local std::string g_ens_err;

struct EnsError : std::exception {
    std::string msg;
    explicit EnsError(std::string m) : msg(std::move(m)) {}
    const char *what() const noexcept override { return msg.c_str(); }
};
void eck(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw EnsError(std::string(what) + ": " + cudaGetErrorString(e));
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

size_t lattice_field_bytes(int prec, const Geom &g) {
    const size_t vh32 = (size_t)round32(g.Vh);
    if (prec == GLAC_FP64) return 8 * vh32 * 9 * sizeof(double2);
    return 8 * vh32 * 4 * sizeof(float4) + 8 * (size_t)g.Vh * sizeof(float2);
}
size_t lattice_force_bytes(int prec, const Geom &g) {
    const size_t vh32 = (size_t)round32(g.Vh);
    return prec == GLAC_FP64 ? 8 * vh32 * 4 * sizeof(double2) : 8 * vh32 * 2 * sizeof(float4);
}

template <typename T> LinkField<T> field_of(glac_ensemble *E, int role, int i);
template <> LinkField<double> field_of<double>(glac_ensemble *E, int role, int i) {
    LinkField<double> L;
    L.p = reinterpret_cast<double2 *>(static_cast<char *>(E->field[role]) + E->off_field[i]);
    L.Vh = E->geo[i].Vh;
    L.Vh32 = round32(L.Vh);
    return L;
}
template <> LinkField<float> field_of<float>(glac_ensemble *E, int role, int i) {
    LinkField<float> L;
    L.Vh = E->geo[i].Vh;
    L.Vh32 = round32(L.Vh);
    L.p4 = reinterpret_cast<float4 *>(static_cast<char *>(E->field[role]) + E->off_field[i]);
    L.p2 = reinterpret_cast<float2 *>(L.p4 + (size_t)8 * 4 * L.Vh32);
    return L;
}
template <typename T> ForceField<T> force_of(glac_ensemble *E, int i);
template <> ForceField<double> force_of<double>(glac_ensemble *E, int i) {
    ForceField<double> Z;
    Z.p = reinterpret_cast<double2 *>(static_cast<char *>(E->force) + E->off_force[i]);
    Z.Vh = E->geo[i].Vh;
    Z.Vh32 = round32(Z.Vh);
    return Z;
}
template <> ForceField<float> force_of<float>(glac_ensemble *E, int i) {
    ForceField<float> Z;
    Z.p = reinterpret_cast<float4 *>(static_cast<char *>(E->force) + E->off_force[i]);
    Z.Vh = E->geo[i].Vh;
    Z.Vh32 = round32(Z.Vh);
    return Z;
}

// Row offset (doubles) of lattice i's measurements when each lattice holds `rows` rows.
size_t obs_offset(const glac_ensemble *E, int i, int rows) {
    size_t o = 0;
    for (int j = 0; j < i; j++) o += (size_t)rows * (3 + E->geo[j].N[3]);
    return o;
}

// clover parts of lattice i: 12 slots in the force layout, then 4 plaquette sums per site
size_t lattice_clover_bytes(int prec, const Geom &g) {
    return 3 * lattice_force_bytes(prec, g) + 8 * (size_t)g.Vh * (prec == GLAC_FP64 ? sizeof(double) : sizeof(float));
}
template <typename T> CloverParts<T> clover_of(glac_ensemble *E, int i) {
    CloverParts<T> cp;
    char *base = E->clover ? static_cast<char *>(E->clover) + E->off_clover[i] : nullptr;
    cp.ah.p = reinterpret_cast<decltype(cp.ah.p)>(base);
    cp.ah.Vh = E->geo[i].Vh;
    cp.ah.Vh32 = round32(E->geo[i].Vh);
    cp.plaq = base ? reinterpret_cast<T *>(base + 3 * lattice_force_bytes(E->d.precision, E->geo[i])) : nullptr;
    return cp;
}

template <typename T> void upload_slots(glac_ensemble *E, int rows) {
    std::vector<LatSlot<T>> S(E->M);
    for (int i = 0; i < E->M; i++) {
        S[i].g = E->geo[i];
        for (int r = 0; r < 3; r++) S[i].f[r] = field_of<T>(E, r, i);
        S[i].z = force_of<T>(E, i);
        S[i].cp = clover_of<T>(E, i);
        S[i].nb = E->plan[i].nb;
        S[i].Bv = E->plan[i].Bv;
        S[i].partial = E->partial + E->off_partial[i];
        S[i].obs = E->obs ? E->obs + obs_offset(E, i, rows) : nullptr;
        S[i].acc = E->acc + i;
        S[i].beta = (float)E->beta[i];
        S[i].stream = E->d.stream_id + (uint32_t)i;
    }
    eck(cudaMemcpyAsync(E->slots, S.data(), S.size() * sizeof(LatSlot<T>), cudaMemcpyHostToDevice, E->stream),
        "upload slots");
    eck(cudaStreamSynchronize(E->stream), "sync");
    E->obs_steps = rows - 1;
}

void ensure_obs(glac_ensemble *E, int n_steps) {
    const size_t need = obs_offset(E, E->M, n_steps + 1);
    if (need > E->obs_cap) {
        if (E->graph) {  // a captured graph refers to the old buffer
            cudaGraphExecDestroy(E->graph);
            E->graph = nullptr;
        }
        if (E->obs) eck(cudaFree(E->obs), "cudaFree");
        E->obs = nullptr;
        eck(cudaMalloc(&E->obs, need * sizeof(double)), "obs alloc");
        E->obs_cap = need;
        E->obs_steps = -1;
    }
    if (E->obs_steps != n_steps) {
        if (E->d.precision == GLAC_FP64) upload_slots<double>(E, n_steps + 1);
        else upload_slots<float>(E, n_steps + 1);
    }
}

template <typename T> const LatSlot<T> *slots_of(glac_ensemble *E) {
    return static_cast<const LatSlot<T> *>(E->slots);
}

template <typename T> void sweeps_t(glac_ensemble *E, int fsel, int n) {
    for (int i = 0; i < n; i++)
        for (int k = 0; k < 8; k++) {
            launch_ens_metropolis<T>(slots_of<T>(E), E->start[ENS_METRO], E->nblk[ENS_METRO], E->M, fsel, k >> 1,
                                     k & 1, E->d.su3_eps, E->d.n_updates, E->d.seed, E->sweep_dev, (uint32_t)i,
                                     E->flips, E->tune[FAM_METRO], E->stream);
            E->launches++;
        }
}

template <typename T> void observe_t(glac_ensemble *E, int fsel, int meas) {
    launch_ens_observables<T>(slots_of<T>(E), E->start[ENS_OBS], E->nblk[ENS_OBS], E->M, fsel, meas,
                              E->tune[FAM_OBS], E->stream);
    E->launches += 2;
}

// Flow buffers 1/2 from the chain; measurement 0, then n steps with a measurement after each.
template <typename T> void flow_t(glac_ensemble *E, int n, bool measure) {
    eck(cudaMemcpyAsync(E->field[1], E->field[0], E->field_total, cudaMemcpyDeviceToDevice, E->stream),
        "copy to flow field");
    const double eps = E->d.flow_eps;
    const double alpha[3] = {eps * 0.25, eps * 0.8888888888888888, 0.75 * eps};
    const double bet[3] = {0.0, -(eps * 0.4722222222222222), -1.0};
    const bool fp32 = sizeof(T) == 4;
    const int phase = variant_shape(FAM_FLOW, fp32, E->tune[FAM_FLOW]) == 1 ? ENS_FLOW1 : ENS_FLOW0;
    int cur = 1;
    // the measurement after step k inside stage 0 of step k + 1 (the field that
    // stage flows is the one to measure), the last one in a pass of its own
    const bool fused = measure && E->fused_measure && E->clover;
    if (measure && (!fused || n == 0)) observe_t<T>(E, cur, 0);
    for (int step = 0; step < n; step++) {
        for (int stage = 0; stage < 3; stage++) {
            if (stage == 0 && fused) {
                // FP32: the 128-register kernel, FP64: the compiler's own allocation
                launch_ens_flow_stage0_meas<T>(slots_of<T>(E), E->start[ENS_FLOW0], E->nblk[ENS_FLOW0], E->M, cur,
                                               3 - cur, alpha[0], sizeof(T) == 4 ? 128 : 0, E->stream);
                launch_ens_obs_combine<T>(slots_of<T>(E), E->start[ENS_OBS], E->nblk[ENS_OBS], E->M, step,
                                          E->stream);
                E->launches += 3;
            } else {
                launch_ens_flow_stage<T>(slots_of<T>(E), E->start[phase], E->nblk[phase], E->M, cur, 3 - cur, stage,
                                         alpha[stage], bet[stage], E->tune[FAM_FLOW], E->stream);
                E->launches++;
            }
            cur = 3 - cur;
        }
        if (measure && (!fused || step == n - 1)) observe_t<T>(E, cur, step + 1);
    }
}

void schedule(glac_ensemble *E, int n_sweeps, int n_steps) {
    if (E->d.precision == GLAC_FP64) {
        sweeps_t<double>(E, 0, n_sweeps);
        launch_advance(E->sweep_dev, (uint32_t)n_sweeps, E->stream);
        if (n_steps >= 0) flow_t<double>(E, n_steps, true);
    } else {
        sweeps_t<float>(E, 0, n_sweeps);
        launch_advance(E->sweep_dev, (uint32_t)n_sweeps, E->stream);
        if (n_steps >= 0) flow_t<float>(E, n_steps, true);
    }
    E->launches++;
}

void read_acceptance(glac_ensemble *E, int n_sweeps, double *acceptance) {
    std::vector<unsigned long long> a(E->M);
    eck(cudaMemcpyAsync(a.data(), E->acc, E->M * sizeof(unsigned long long), cudaMemcpyDeviceToHost, E->stream),
        "D2H acc");
    eck(cudaStreamSynchronize(E->stream), "sync");
    for (int i = 0; i < E->M; i++) {
        const double per = 4.0 * E->d.n_updates * (double)E->geo[i].V * (double)(n_sweeps > 0 ? n_sweeps : 1);
        acceptance[i] = (double)a[i] / per;
    }
}

void read_obs(glac_ensemble *E, int n_steps, double *obs) {
    eck(cudaMemcpyAsync(obs, E->obs, obs_offset(E, E->M, n_steps + 1) * sizeof(double), cudaMemcpyDeviceToHost,
                        E->stream),
        "D2H obs");
    eck(cudaStreamSynchronize(E->stream), "sync");
}

template <typename F> glac_status eguarded(glac_ensemble *E, F &&f) {
    if (!E) return GLAC_ERR_ARG;
    try {
        eck(cudaSetDevice(E->d.device), "cudaSetDevice");
        return f();
    } catch (const EnsError &e) {
        E->err = e.msg;
        return GLAC_ERR_CUDA;
    } catch (const std::exception &e) {
        E->err = e.what();
        return GLAC_ERR_CUDA;
    }
}

glac_status need_field(glac_ensemble *E) {
    if (!E->has_field) {
        E->err = "no gauge fields set (call glac_ensemble_hot_start or glac_ensemble_set_links first)";
        return GLAC_ERR_STATE;
    }
    return GLAC_OK;
}

void drop_graph(glac_ensemble *E) {
    if (E->graph) cudaGraphExecDestroy(E->graph);
    E->graph = nullptr;
    E->graph_sweeps = E->graph_steps = -1;
}

}  // namespace

extern "C" {

const char *glac_ensemble_global_error(void) { return g_ens_err.c_str(); }

glac_status glac_ensemble_create(int n, const int *dims, const double *betas, const glac_desc *common,
                                 glac_ensemble **out) {
    if (!out) return GLAC_ERR_ARG;
    *out = nullptr;
    if (n < 1 || !dims || !betas || !common) {
        g_ens_err = "need n >= 1 lattices, their dims and betas, and the common settings";
        return GLAC_ERR_ARG;
    }
    if (common->precision != GLAC_FP64 && common->precision != GLAC_FP32) {
        g_ens_err = "precision must be GLAC_FP64 or GLAC_FP32";
        return GLAC_ERR_ARG;
    }
    if (common->exp_func != GLAC_EXP_MORNINGSTAR) {
        g_ens_err = "the ensemble flow uses the Morningstar exponential";
        return GLAC_ERR_ARG;
    }
    if (common->n_updates < 1 || !(common->su3_eps > 0 && common->su3_eps < 1) || !(common->flow_eps > 0)) {
        g_ens_err = "need n_updates >= 1, 0 < su3_eps < 1, flow_eps > 0";
        return GLAC_ERR_ARG;
    }
    for (int i = 0; i < n; i++) {
        long long V = 1;
        for (int k = 0; k < 4; k++) {
            const int N = dims[4 * i + k];
            if (N < 4 || (N & 1)) {
                g_ens_err = "lattice " + std::to_string(i) + ": every extent must be even and >= 4";
                return GLAC_ERR_ARG;
            }
            V *= N;
        }
        if (V > (1ll << 29) || dims[4 * i + 3] > 1024) {
            g_ens_err = "lattice " + std::to_string(i) + ": V <= 2^29 and Nt <= 1024";
            return GLAC_ERR_ARG;
        }
        if (!field_offsets_fit(V, common->precision == GLAC_FP64)) {
            g_ens_err = "lattice " + std::to_string(i) + ": too large for 32-bit field offsets";
            return GLAC_ERR_ARG;
        }
    }
    glac_ensemble *E = new glac_ensemble;
    E->d = *common;
    E->M = n;
    glac_status s = eguarded(E, [&] {
        size_t fo = 0, zo = 0, po = 0, co = 0;
        std::vector<int> st[ENS_NPHASE];
        for (int k = 0; k < ENS_NPHASE; k++) st[k].push_back(0);
        for (int i = 0; i < n; i++) {
            const Geom g = make_geom(dims + 4 * i);
            const ObsPlan pl = make_obs_plan_capped(g, 128);
            E->geo.push_back(g);
            E->plan.push_back(pl);
            E->beta.push_back(betas[i]);
            E->off_field.push_back(fo);
            E->off_force.push_back(zo);
            E->off_partial.push_back(po);
            E->off_clover.push_back(co);
            co += align256(lattice_clover_bytes(E->d.precision, g));
            if (!clover_offsets_fit(g.V, E->d.precision == GLAC_FP64)) E->fused_measure = false;
            fo += align256(lattice_field_bytes(E->d.precision, g));
            zo += align256(lattice_force_bytes(E->d.precision, g));
            po += 3 * (size_t)pl.nblocks;
            for (int k = 0; k < ENS_NPHASE; k++) st[k].push_back(st[k].back() + ens_blocks(g, pl, k));
        }
        E->field_total = fo;
        E->force_total = zo;
        E->partial_total = po;
        eck(cudaStreamCreateWithFlags(&E->stream, cudaStreamNonBlocking), "stream");
        for (int r = 0; r < 3; r++) eck(cudaMalloc(&E->field[r], fo), "field alloc");
        eck(cudaMalloc(&E->force, zo), "force alloc");
        eck(cudaMalloc(&E->partial, po * sizeof(double)), "partial alloc");
        if (E->fused_measure) eck(cudaMalloc(&E->clover, co), "clover parts alloc");
        const size_t slot_bytes = E->d.precision == GLAC_FP64 ? sizeof(LatSlot<double>) : sizeof(LatSlot<float>);
        eck(cudaMalloc(&E->slots, n * slot_bytes), "slots alloc");
        eck(cudaMalloc(&E->acc, n * sizeof(unsigned long long)), "acc alloc");
        eck(cudaMalloc(&E->sweep_dev, sizeof(uint32_t)), "counter alloc");
        eck(cudaMemsetAsync(E->sweep_dev, 0, sizeof(uint32_t), E->stream), "memset");
        for (int k = 0; k < ENS_NPHASE; k++) {
            E->nblk[k] = st[k].back();
            eck(cudaMalloc(&E->start[k], st[k].size() * sizeof(int)), "table alloc");
            eck(cudaMemcpyAsync(E->start[k], st[k].data(), st[k].size() * sizeof(int), cudaMemcpyHostToDevice,
                                E->stream),
                "table upload");
        }
        ensure_obs(E, 0);
        return GLAC_OK;
    });
    if (s != GLAC_OK) {
        g_ens_err = E->err;
        glac_ensemble_destroy(E);
        return s;
    }
    *out = E;
    return GLAC_OK;
}

void glac_ensemble_destroy(glac_ensemble *E) {
    if (!E) return;
    cudaSetDevice(E->d.device);
    if (E->stream) cudaStreamSynchronize(E->stream);
    drop_graph(E);
    for (void *p : {E->field[0], E->field[1], E->field[2], E->force, (void *)E->partial, E->slots, (void *)E->acc,
                    (void *)E->sweep_dev, (void *)E->obs, (void *)E->staging, E->clover, (void *)E->barrier})
        if (p) cudaFree(p);
    for (int k = 0; k < ENS_NPHASE; k++)
        if (E->start[k]) cudaFree(E->start[k]);
    if (E->stream) cudaStreamDestroy(E->stream);
    delete E;
}

const char *glac_ensemble_last_error(const glac_ensemble *E) { return E ? E->err.c_str() : g_ens_err.c_str(); }

uint64_t glac_ensemble_launch_count(const glac_ensemble *E) { return E ? E->launches : 0; }

glac_status glac_ensemble_set_option(glac_ensemble *E, const char *key, long value) {
    if (!E || !key) return GLAC_ERR_ARG;
    if (std::string(key) == "su2_sign_flips" && (value == 0 || value == 1)) {
        E->flips = value != 0;
        drop_graph(E);
        return GLAC_OK;
    }
    if (std::string(key) == "persistent_wait_ms" && value > 0 && value <= 60000) {
        E->persistent_wait_ns = (unsigned long long)value * 1000000ull;
        return GLAC_OK;
    }
    if (std::string(key) == "persistent_test_stall" && (value == 0 || value == 1)) {
        E->persistent_test_stall = (int)value;
        return GLAC_OK;
    }
    if (std::string(key) == "fused_measure" && (value == 0 || value == 1)) {
        if (value == 1 && !E->clover) {
            E->err = "fused_measure: a lattice of this ensemble is too large for the clover parts' 32-bit offsets";
            return GLAC_ERR_ARG;
        }
        E->fused_measure = value != 0;
        drop_graph(E);
        return GLAC_OK;
    }
    E->err = std::string("unknown option or value: ") + key;
    return GLAC_ERR_ARG;
}

glac_status glac_ensemble_hot_start(glac_ensemble *E, uint64_t seed) {
    return eguarded(E, [&] {
        if (E->d.precision == GLAC_FP64)
            launch_ens_haar<double>(slots_of<double>(E), E->start[ENS_METRO], E->nblk[ENS_METRO], E->M, seed, E->stream);
        else
            launch_ens_haar<float>(slots_of<float>(E), E->start[ENS_METRO], E->nblk[ENS_METRO], E->M, seed, E->stream);
        eck(cudaGetLastError(), "hot start");
        E->launches++;
        eck(cudaStreamSynchronize(E->stream), "sync");
        E->has_field = true;
        return GLAC_OK;
    });
}

static glac_status ens_links(glac_ensemble *E, int i, double *host, bool set) {
    return eguarded(E, [&] {
        if (i < 0 || i >= E->M || !host) {
            E->err = "lattice index out of range or null field";
            return GLAC_ERR_ARG;
        }
        const size_t bytes = (size_t)E->geo[i].V * 72 * sizeof(double);
        if (bytes > E->staging_cap) {
            if (E->staging) eck(cudaFree(E->staging), "cudaFree");
            E->staging = nullptr;
            eck(cudaMalloc(&E->staging, bytes), "staging alloc");
            E->staging_cap = bytes;
        }
        if (set) {
            eck(cudaMemcpyAsync(E->staging, host, bytes, cudaMemcpyHostToDevice, E->stream), "H2D");
            if (E->d.precision == GLAC_FP64) launch_aos_to_soa(E->geo[i], E->staging, field_of<double>(E, 0, i), E->stream);
            else launch_aos_to_soa(E->geo[i], E->staging, field_of<float>(E, 0, i), E->stream);
            eck(cudaGetLastError(), "layout");
            E->launches++;
            E->has_field = true;
        } else {
            glac_status s = need_field(E);
            if (s != GLAC_OK) return s;
            if (E->d.precision == GLAC_FP64) launch_soa_to_aos(E->geo[i], field_of<double>(E, 0, i), E->staging, E->stream);
            else launch_soa_to_aos(E->geo[i], field_of<float>(E, 0, i), E->staging, E->stream);
            eck(cudaGetLastError(), "layout");
            E->launches++;
            eck(cudaMemcpyAsync(host, E->staging, bytes, cudaMemcpyDeviceToHost, E->stream), "D2H");
        }
        eck(cudaStreamSynchronize(E->stream), "sync");
        return GLAC_OK;
    });
}

glac_status glac_ensemble_set_links(glac_ensemble *E, int i, const double *host) {
    return ens_links(E, i, const_cast<double *>(host), true);
}
glac_status glac_ensemble_get_links(glac_ensemble *E, int i, double *host) { return ens_links(E, i, host, false); }

glac_status glac_ensemble_metropolis(glac_ensemble *E, int n_sweeps, double *acceptance) {
    return eguarded(E, [&] {
        glac_status s = need_field(E);
        if (s != GLAC_OK) return s;
        if (n_sweeps < 0) { E->err = "n_sweeps < 0"; return GLAC_ERR_ARG; }
        eck(cudaMemsetAsync(E->acc, 0, E->M * sizeof(unsigned long long), E->stream), "memset");
        schedule(E, n_sweeps, -1);
        eck(cudaGetLastError(), "metropolis");
        E->sweep += (uint32_t)n_sweeps;
        if (acceptance) read_acceptance(E, n_sweeps, acceptance);
        else eck(cudaStreamSynchronize(E->stream), "sync");
        return GLAC_OK;
    });
}

long long glac_ensemble_obs_count(const glac_ensemble *E, int n_steps) {
    if (!E || n_steps < 0) return -1;
    return (long long)obs_offset(E, E->M, n_steps + 1);
}

glac_status glac_ensemble_flow(glac_ensemble *E, int n_steps, double *obs) {
    return eguarded(E, [&] {
        glac_status s = need_field(E);
        if (s != GLAC_OK) return s;
        if (n_steps < 0) { E->err = "n_steps < 0"; return GLAC_ERR_ARG; }
        ensure_obs(E, n_steps);
        if (E->d.precision == GLAC_FP64) flow_t<double>(E, n_steps, true);
        else flow_t<float>(E, n_steps, true);
        eck(cudaGetLastError(), "flow");
        if (obs) read_obs(E, n_steps, obs);
        else eck(cudaStreamSynchronize(E->stream), "sync");
        return GLAC_OK;
    });
}

glac_status glac_ensemble_run(glac_ensemble *E, int n_sweeps, int n_steps, double *acceptance, double *obs,
                              double *gpu_seconds) {
    return eguarded(E, [&] {
        glac_status s = need_field(E);
        if (s != GLAC_OK) return s;
        if (n_sweeps < 0 || n_steps < 0) { E->err = "negative count"; return GLAC_ERR_ARG; }
        ensure_obs(E, n_steps);
        if (!E->graph || E->graph_sweeps != n_sweeps || E->graph_steps != n_steps) {
            drop_graph(E);
            cudaGraph_t g = nullptr;
            eck(cudaStreamBeginCapture(E->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            const uint64_t before = E->launches;
            try {
                eck(cudaMemsetAsync(E->acc, 0, E->M * sizeof(unsigned long long), E->stream), "memset");
                schedule(E, n_sweeps, n_steps);
            } catch (...) {
                cudaStreamEndCapture(E->stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            E->launches = before;  // counted when the graph runs
            eck(cudaStreamEndCapture(E->stream, &g), "end capture");
            cudaError_t ie = cudaGraphInstantiate(&E->graph, g, 0);
            cudaGraphDestroy(g);
            eck(ie, "instantiate");
            E->graph_sweeps = n_sweeps;
            E->graph_steps = n_steps;
        }
        cudaEvent_t e0, e1;
        eck(cudaEventCreate(&e0), "event");
        eck(cudaEventCreate(&e1), "event");
        eck(cudaEventRecord(e0, E->stream), "event");
        eck(cudaGraphLaunch(E->graph, E->stream), "graph launch");
        eck(cudaEventRecord(e1, E->stream), "event");
        eck(cudaEventSynchronize(e1), "sync");
        float ms = 0.f;
        eck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        E->launches += 8ull * n_sweeps + 1 + (n_steps >= 0 ? 2 + 5ull * n_steps : 0);
        E->sweep += (uint32_t)n_sweeps;
        if (gpu_seconds) *gpu_seconds = ms * 1e-3;
        if (acceptance) read_acceptance(E, n_sweeps, acceptance);
        if (obs) read_obs(E, n_steps, obs);
        return GLAC_OK;
    });
}

glac_status glac_ensemble_run_persistent(glac_ensemble *E, int n_sweeps, int n_steps, double *acceptance,
                                         double *obs, double *gpu_seconds) {
    return eguarded(E, [&] {
        glac_status s = need_field(E);
        if (s != GLAC_OK) return s;
        if (n_sweeps < 0 || n_steps < 0) { E->err = "negative count"; return GLAC_ERR_ARG; }
        if (E->d.precision != GLAC_FP32 || !E->clover || !E->fused_measure) {
            E->err = "the persistent launch runs FP32 ensembles with the measurement inside flow stage 0";
            return GLAC_ERR_STATE;
        }
        int coop = 0, sms = 0;
        eck(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, E->d.device), "attribute");
        eck(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, E->d.device), "attribute");
        const int per_sm = persistent_blocks_per_sm();
        if (!coop || per_sm <= 0) {
            E->err = "cooperative launch not available for the persistent kernel on this device";
            return GLAC_ERR_CUDA;
        }
        ensure_obs(E, n_steps);
        if (!E->barrier) eck(cudaMalloc(&E->barrier, sizeof(GridBarrier)), "barrier alloc");
        eck(cudaMemsetAsync(E->barrier, 0, sizeof(GridBarrier), E->stream), "memset");
        eck(cudaMemsetAsync(E->acc, 0, E->M * sizeof(unsigned long long), E->stream), "memset");
        const double eps = E->d.flow_eps;
        EnsSchedule sc;
        std::memset(&sc, 0, sizeof(sc));
        sc.M = E->M;
        sc.n_sweeps = n_sweeps;
        sc.n_steps = n_steps;
        sc.start_metro = E->start[ENS_METRO];
        sc.start_flow0 = E->start[ENS_FLOW0];
        sc.start_obs = E->start[ENS_OBS];
        sc.nb_metro = E->nblk[ENS_METRO];
        sc.nb_flow0 = E->nblk[ENS_FLOW0];
        sc.nb_obs = E->nblk[ENS_OBS];
        sc.eps = E->d.su3_eps;
        sc.sq1me = std::sqrt(1.0 - E->d.su3_eps * E->d.su3_eps);
        const double alpha[3] = {eps * 0.25, eps * 0.8888888888888888, 0.75 * eps};
        const double beta[3] = {0.0, -(eps * 0.4722222222222222), -1.0};
        for (int k = 0; k < 3; k++) { sc.alpha[k] = alpha[k]; sc.beta[k] = beta[k]; }
        sc.nhits = E->d.n_updates;
        sc.k0 = (uint32_t)E->d.seed;
        sc.k1 = (uint32_t)(E->d.seed >> 32);
        sc.sweep_base = E->sweep_dev;
        sc.flips = E->flips;
        sc.chain = E->field[0];
        sc.flow = E->field[1];
        sc.field_words = E->field_total / 16;
        sc.wait_ns = E->persistent_wait_ns;
        sc.test_skip_block0 = E->persistent_test_stall;
        cudaEvent_t e0, e1;
        eck(cudaEventCreate(&e0), "event");
        eck(cudaEventCreate(&e1), "event");
        eck(cudaEventRecord(e0, E->stream), "event");
        eck(launch_ens_persistent(static_cast<const LatSlot<float> *>(E->slots), sc, E->barrier, per_sm * sms,
                                  E->stream),
            "persistent launch");
        eck(cudaEventRecord(e1, E->stream), "event");
        eck(cudaEventSynchronize(e1), "sync");
        float ms = 0.f;
        eck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        E->launches += 1;
        GridBarrier b;
        eck(cudaMemcpy(&b, E->barrier, sizeof(b), cudaMemcpyDeviceToHost), "D2H barrier");
        if (b.err) {
            E->err = "a grid barrier of the persistent launch waited past its limit; the fields are undefined";
            return GLAC_ERR_TIMEOUT;
        }
        E->sweep += (uint32_t)n_sweeps;
        if (gpu_seconds) *gpu_seconds = ms * 1e-3;
        if (acceptance) read_acceptance(E, n_sweeps, acceptance);
        if (obs) read_obs(E, n_steps, obs);
        return GLAC_OK;
    });
}

glac_status glac_ensemble_get_tuning(const glac_ensemble *E, int *v) {
    if (!E || !v) return GLAC_ERR_ARG;
    for (int k = 0; k < 3; k++) v[k] = E->tune[k];
    return GLAC_OK;
}

glac_status glac_ensemble_set_tuning(glac_ensemble *E, const int *v) {
    if (!E || !v) return GLAC_ERR_ARG;
    const bool fp32 = E->d.precision == GLAC_FP32;
    for (int f = 0; f < 3; f++)
        if (v[f] < 0 || v[f] >= num_variants((Family)f, fp32)) {
            E->err = "launch variant out of range";
            return GLAC_ERR_ARG;
        }
    for (int k = 0; k < 3; k++) E->tune[k] = v[k];
    drop_graph(E);
    return GLAC_OK;
}

// Times every launch variant of the flow, Metropolis and observable families on
// the whole ensemble (in the flow buffers: the chain, its sweep counter and the
// acceptance counters are left as they were) and keeps the fastest.
// report[4 f + v] = seconds per flow step / per sweep / per measurement (0 for
// absent variants).
glac_status glac_ensemble_autotune(glac_ensemble *E, int reps, double *report) {
    return eguarded(E, [&] {
        glac_status s = need_field(E);
        if (s != GLAC_OK) return s;
        if (reps < 1) reps = 1;
        const bool fp32 = E->d.precision == GLAC_FP32;
        std::vector<unsigned long long> acc_save(E->M);
        eck(cudaMemcpyAsync(acc_save.data(), E->acc, E->M * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                            E->stream),
            "save acc");
        double rep[12] = {0};
        cudaEvent_t e0, e1;
        eck(cudaEventCreate(&e0), "event");
        eck(cudaEventCreate(&e1), "event");
        // the observable family measures the flow buffer into row 0 of each lattice's
        // rows (allocated since creation)
        for (int fam = 0; fam < 3; fam++) {
            const int nv = num_variants((Family)fam, fp32);
            int best = E->tune[fam];
            double best_t = 1e30;
            for (int v = 0; v < nv; v++) {
                E->tune[fam] = v;
                for (int pass = 0; pass < 2; pass++) {  // pass 0 warms up
                    eck(cudaMemcpyAsync(E->field[1], E->field[0], E->field_total, cudaMemcpyDeviceToDevice, E->stream),
                        "copy");
                    eck(cudaEventRecord(e0, E->stream), "event");
                    for (int r = 0; r < reps; r++) {
                        if (fam == FAM_METRO) {
                            if (fp32) sweeps_t<float>(E, 1, 1);
                            else sweeps_t<double>(E, 1, 1);
                        } else if (fam == FAM_OBS) {
                            if (fp32) observe_t<float>(E, 1, 0);
                            else observe_t<double>(E, 1, 0);
                        } else {
                            if (fp32) flow_t<float>(E, 1, false);
                            else flow_t<double>(E, 1, false);
                        }
                    }
                    eck(cudaEventRecord(e1, E->stream), "event");
                    eck(cudaEventSynchronize(e1), "sync");
                }
                float ms = 0.f;
                eck(cudaEventElapsedTime(&ms, e0, e1), "elapsed");
                const double t = ms * 1e-3 / reps;
                rep[4 * fam + v] = t;
                if (t < best_t) { best_t = t; best = v; }
            }
            E->tune[fam] = best;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        eck(cudaMemcpyAsync(E->acc, acc_save.data(), E->M * sizeof(unsigned long long), cudaMemcpyHostToDevice,
                            E->stream),
            "restore acc");
        eck(cudaStreamSynchronize(E->stream), "sync");
        drop_graph(E);
        if (report)
            for (int k = 0; k < 12; k++) report[k] = rep[k];
        return GLAC_OK;
    });
}

}  // extern "C"
