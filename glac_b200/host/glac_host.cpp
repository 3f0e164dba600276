// Host driver of the drop-in: run-configuration, System, output files.
#include "glac_host.h"

#include <sys/stat.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>

#include "json_lite.h"

namespace glac_host {

namespace {

const Json &req(const Json &j, const char *key) {
    if (!j.has(key)) throw std::runtime_error(std::string("configuration key '") + key + "' is missing");
    return j[key];
}

std::string default_format(double v) {
    std::ostringstream o;
    o << v;
    return o.str();
}

}  // namespace

// GLAC/config/configloader.cpp:55-181: the same keys; the test and
// performance-test keys are accepted and ignored.
Parameters Parameters::load(const std::string &path) {
    std::ifstream f(path);
    if (!f.good()) throw std::runtime_error("File " + path + " does not exist");
    std::stringstream ss;
    ss << f.rdbuf();
    const Json j = Json::parse(ss.str());
    Parameters p;
    p.NSpatial = (unsigned)req(j, "NSpatial").number();
    p.NTemporal = (unsigned)req(j, "NTemporal").number();
    p.beta = req(j, "beta").number();
    p.NCf = (unsigned)req(j, "NCf").number();
    p.NCor = (unsigned)req(j, "NCor").number();
    p.NTherm = (unsigned)req(j, "NTherm").number();
    p.NFlows = (unsigned)req(j, "NFlows").number();
    p.NUpdates = (unsigned)req(j, "NUpdates").number();
    p.action = req(j, "action").string();
    p.outputFolder = req(j, "outputFolder").string();
    p.inputFolder = req(j, "inputFolder").string();
    p.storeConfigurations = req(j, "storeConfigurations").boolean();
    p.storeThermalizationObservables = req(j, "storeThermalizationObservables").boolean();
    p.verbose = req(j, "verbose").boolean();
    p.pwd = req(j, "pwd").string();
    p.batchName = req(j, "batchName").string();
    p.hotStart = req(j, "hotStart").boolean();
    p.RSTHotStart = req(j, "RSTHotStart").boolean();
    if (j.has("subDims"))
        for (size_t i = 0; i < j["subDims"].size(); i++) p.subDims.push_back((unsigned)j["subDims"][i].number());
    p.expFunc = req(j, "expFunc").string();
    p.observables = req(j, "observables").strings();
    p.flowObservables = req(j, "flowObservables").strings();
    p.loadFieldConfigurations = j.has("load_field_configs") && j["load_field_configs"].boolean();
    if (p.loadFieldConfigurations) {
        p.fieldConfigs = j["field_configs"].strings();
        p.chromaConfig = j.has("chroma_config") && j["chroma_config"].boolean();
    }
    if (j.has("load_config_and_run")) p.loadConfigAndRun = j["load_config_and_run"].string();
    if (!p.loadConfigAndRun.empty()) {
        p.fieldConfigs = {p.loadConfigAndRun};
        p.chromaConfig = j.has("chroma_config") && j["chroma_config"].boolean();
    }
    if (j.has("config_start_number") && !j["config_start_number"].is_null())
        p.configStartNumber = (int)j["config_start_number"].number();
    if (j.has("unitTesting")) p.unitTesting = j["unitTesting"].boolean();
    if (j.has("performanceTesting")) p.performanceTesting = j["performanceTesting"].boolean();
    if (j.has("debug")) p.debug = j["debug"].boolean();
    p.SU3Eps = req(j, "SU3Eps").number();
    p.flowEpsilon = req(j, "flowEpsilon").number();
    // seed 0 means time-seeded (configloader.cpp:163-177)
    const double ms = req(j, "metropolisSeed").number(), rs = req(j, "randomMatrixSeed").number();
    p.metropolisSeed = ms != 0 ? ms : (double)std::time(nullptr) + 1.0;
    p.randomMatrixSeed = rs != 0 ? rs : (double)std::time(nullptr);
    if (j.has("samplingFrequency")) p.samplingFrequency = (int)j["samplingFrequency"].number();
    if (j.has("precision")) p.precision = j["precision"].string();
    if (j.has("device")) p.device = (int)j["device"].number();
    if (j.has("reunitInterval")) p.reunitInterval = (int)j["reunitInterval"].number();
    if (j.has("autotune")) p.autotune = j["autotune"].boolean();
    if (p.precision != "fp64" && p.precision != "fp32")
        throw std::runtime_error("precision must be \"fp64\" or \"fp32\", not \"" + p.precision + "\"");
    if (p.action != "wilson" && p.action != "wilsonExplicitDer")
        throw std::runtime_error("ERROR: Action type " + p.action + "not recognized.");
    return p;
}

std::string Parameters::to_json() const {
    std::ostringstream o;
    auto list = [&](const std::vector<std::string> &v) {
        std::string s = "[";
        for (size_t i = 0; i < v.size(); i++) s += (i ? ", \"" : "\"") + v[i] + "\"";
        return s + "]";
    };
    o << std::setprecision(17) << "{\"NSpatial\": " << NSpatial << ", \"NTemporal\": " << NTemporal
      << ", \"beta\": " << beta << ", \"NCf\": " << NCf << ", \"NCor\": " << NCor << ", \"NTherm\": " << NTherm
      << ", \"NFlows\": " << NFlows << ", \"NUpdates\": " << NUpdates << ", \"action\": \"" << action
      << "\", \"hotStart\": " << (hotStart ? "true" : "false") << ", \"RSTHotStart\": "
      << (RSTHotStart ? "true" : "false") << ", \"expFunc\": \"" << expFunc << "\", \"observables\": "
      << list(observables) << ", \"flowObservables\": " << list(flowObservables)
      << ", \"load_field_configs\": " << (loadFieldConfigurations ? "true" : "false") << ", \"field_configs\": "
      << list(fieldConfigs) << ", \"load_config_and_run\": \"" << loadConfigAndRun
      << "\", \"config_start_number\": " << configStartNumber << ", \"SU3Eps\": " << SU3Eps
      << ", \"flowEpsilon\": " << flowEpsilon << ", \"metropolisSeed\": " << metropolisSeed
      << ", \"randomMatrixSeed\": " << randomMatrixSeed << ", \"precision\": \"" << precision
      << "\", \"device\": " << device << ", \"reunitInterval\": " << reunitInterval
      << ", \"autotune\": " << (autotune ? "true" : "false") << ", \"outputFolder\": \"" << outputFolder
      << "\", \"inputFolder\": \"" << inputFolder << "\", \"pwd\": \"" << pwd << "\", \"batchName\": \""
      << batchName << "\"}";
    return o.str();
}

// GLAC/observables/tools/observablestorer.cpp:77-98
void ObservableStorer::run_statistics() {
    const double n = (double)values.size();
    double s = 0, s2 = 0;
    for (double v : values) { s += v; s2 += v * v; }
    mean = s / n;
    variance = (s2 / n - mean * mean) / n;
    stdev = std::sqrt(variance);
}

// GLAC/system.cpp:62-125
Sampler select_sampler(const std::vector<std::string> &names) {
    bool plaq = false, topc = false, energy = false, topct = false, density = false, weinberg = false;
    for (const std::string &n : names) {
        if (n == "plaq") plaq = true;
        else if (n == "topc") topc = true;
        else if (n == "energy") energy = true;
        else if (n == "topct") topct = true;
        else if (n == "energyTopcFieldDensity") density = true;
        else if (n == "weinberg") weinberg = true;
        else throw std::runtime_error("observable \"" + n + "\" is not provided by this implementation");
    }
    if (weinberg) return Sampler::Super;
    if ((topc || energy) && !topct) return Sampler::Master;
    if (plaq && !topc && !energy && !topct) return Sampler::Plaquette;
    if (density && !plaq && !topc && !energy && !topct) return Sampler::ChargeDensity;
    return Sampler::MasterTopcXYZ;
}
std::vector<std::string> sampler_names(Sampler s, bool flow) {
    if (s == Sampler::Plaquette) return {"plaq"};
    if (s == Sampler::ChargeDensity) return {"plaq", "topc", "energy"};
    if (s == Sampler::Super)  // GLAC/observables/supersampler.cpp:134-174
        return flow ? std::vector<std::string>{"plaq", "topc", "weinberg", "energy", "topct", "weinbergt"}
                    : std::vector<std::string>{"plaq", "topc", "energy", "weinberg"};
    if (s == Sampler::Master || !flow) return {"plaq", "topc", "energy"};
    return {"plaq", "topc", "energy", "topct"};
}

size_t row_width(Sampler s, unsigned Nt) { return s == Sampler::Super ? 4 + 2 * (size_t)Nt : 3 + (size_t)Nt; }
size_t row_offset(Sampler s, const std::string &name, unsigned Nt) {
    if (name == "plaq") return 0;
    if (name == "topc") return 1;
    if (name == "energy") return 2;
    if (name == "weinberg") return 3;
    if (name == "topct") return s == Sampler::Super ? 4 : 3;
    if (name == "weinbergt") return 4 + (size_t)Nt;
    throw std::runtime_error("no observable " + name);
}

void makeDirs(const std::string &path) {
    std::string cur;
    for (size_t i = 0; i < path.size(); i++) {
        cur += path[i];
        if (path[i] == '/' || i + 1 == path.size()) mkdir(cur.c_str(), 0755);
    }
}

static std::string cfg_number(const Parameters &P, unsigned n) {
    char buf[16];
    std::snprintf(buf, sizeof(buf), "%05d", (int)n + P.configStartNumber);
    return buf;
}

// GLAC/io/fieldio.cpp:72-79
std::string fieldFileName(const Parameters &P, unsigned configNumber) {
    return P.batchName + "_b" + std::to_string(P.beta) + "_N" + std::to_string(P.NSpatial) + "_NT" +
           std::to_string(P.NTemporal) + "_np1_config" + cfg_number(P, configNumber) + ".bin";
}

void writeScalarField(const Parameters &P, const std::string &observable, const std::vector<double> &field,
                      unsigned configNumber) {
    const std::string dir = P.pwd + P.outputFolder + P.batchName + "/scalar_fields/" + observable + "/";
    makeDirs(dir);
    const std::string fname = dir + fieldFileName(P, configNumber);
    std::FILE *f = std::fopen(fname.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + fname);
    const size_t n = std::fwrite(field.data(), sizeof(double), field.size(), f);
    std::fclose(f);
    if (n != field.size()) throw std::runtime_error("short write " + fname);
    std::printf("\n    %s written.", fname.c_str());
}

// GLAC/io/observablesio.cpp:29-78
void writeObservablesToFile(const Parameters &P, double acceptance, const ObservableStorer &o) {
    const std::string dir = P.pwd + P.outputFolder + P.batchName + "/observables/";
    makeDirs(dir);
    const std::string fname = dir + o.name + "_" + P.batchName + ".dat";
    std::ofstream f(fname);
    f << "beta " << default_format(P.beta) << "\n";
    f << "acceptanceCounter " << default_format(acceptance) << "\n";
    f << "NCor " << P.NCor << "\n";
    f << "NCf " << P.NCf << "\n";
    f << "NTherm " << P.NTherm << "\n";
    f << std::fixed << std::setprecision(15);
    f << "Average" << o.name << " " << o.mean << "\n";
    f << "Variance" << o.name << " " << o.variance << "\n";
    f << "std" << o.name << " " << o.stdev << "\n";
    for (double v : o.values) f << v << "\n";
    std::printf("\n%s written.", fname.c_str());
}

static std::ofstream flow_file(const Parameters &P, const std::string &name, unsigned configNumber) {
    const std::string dir = P.pwd + P.outputFolder + P.batchName + "/flow_observables/" + name + "/";
    makeDirs(dir);
    std::ofstream f(dir + P.batchName + "_" + name + "_flow_config" + cfg_number(P, configNumber) + ".dat");
    f << "beta " << default_format(P.beta) << "\n";
    f << "NFlows " << P.NFlows << "\n";
    f << "FlowEpsilon " << default_format(P.flowEpsilon) << "\n";
    f << std::fixed << std::setprecision(15);
    return f;
}

// GLAC/io/observablesio.cpp:80-139
void writeFlowObservableToFile(const Parameters &P, const std::string &name, const std::vector<double> &values,
                               unsigned configNumber) {
    std::ofstream f = flow_file(P, name, configNumber);
    for (unsigned i = 0; i < P.NFlows + 1; i++) f << i * P.flowEpsilon << " " << values[i] << "\n";
}

// GLAC/io/observablesio.cpp:141-193
void writeMatrixToFile(const Parameters &P, const std::string &name, const std::vector<double> &values,
                       unsigned configNumber, unsigned N) {
    std::ofstream f = flow_file(P, name, configNumber);
    for (unsigned i = 0; i < P.NFlows + 1; i++) {
        f << i * P.flowEpsilon;
        for (unsigned k = 0; k < N; k++) f << " " << values[(size_t)i * N + k];
        f << "\n";
    }
}

// ---------------------------------------------------------------------------
// System
// ---------------------------------------------------------------------------
System::System(const Parameters &p) : P(p) {
    cfgSampler = select_sampler(P.observables);
    flowSampler = select_sampler(P.flowObservables);
    V = P.NSpatial * P.NSpatial * P.NSpatial * P.NTemporal;
    if (cfgSampler == Sampler::ChargeDensity || flowSampler == Sampler::ChargeDensity) {
        // one configuration, none stored, to keep the number of field files down (GLAC/system.cpp:105-113)
        P.NCf = 1;
        P.storeConfigurations = false;
    }
}

void System::measureInto(glac_ctx *c, Sampler s, unsigned index, bool write, std::vector<double> &obs) {
    obs.resize(row_width(s, P.NTemporal));
    if (s == Sampler::Super) {
        if (glac_measure_weinberg(c, obs.data()) != GLAC_OK)
            throw std::runtime_error(std::string("measure: ") + glac_last_error(c));
        return;
    }
    if (s != Sampler::ChargeDensity || !write) {
        if (glac_measure(c, obs.data()) != GLAC_OK) throw std::runtime_error(std::string("measure: ") + glac_last_error(c));
        return;
    }
    std::vector<double> q(V), e(V);
    if (glac_measure_density(c, obs.data(), q.data(), e.data()) != GLAC_OK)
        throw std::runtime_error(std::string("measure density: ") + glac_last_error(c));
    writeScalarField(P, "topc", q, index);
    writeScalarField(P, "energy", e, index);
}

System::~System() {
    if (flowCtx) glac_destroy(flowCtx);
    if (ctx) glac_destroy(ctx);
}

void System::ck(glac_status s, const char *what) {
    if (s != GLAC_OK) {
        const char *m = ctx ? glac_last_error(ctx) : glac_global_error();
        throw std::runtime_error(std::string(what) + ": " + (m ? m : "?"));
    }
}

std::string System::outDir() const { return P.pwd + P.outputFolder + P.batchName + "/"; }

void System::latticeSetup() {
    if (!P.subDims.empty())
        std::printf("\nsubDims ignored: the whole lattice lives on one GPU");
    glac_desc d{};
    d.dims[0] = d.dims[1] = d.dims[2] = (int)P.NSpatial;
    d.dims[3] = (int)P.NTemporal;
    d.beta = P.beta;
    d.precision = P.precision == "fp32" ? GLAC_FP32 : GLAC_FP64;
    d.n_updates = (int)P.NUpdates;
    d.su3_eps = P.SU3Eps;
    d.flow_eps = P.flowEpsilon;
    d.exp_func = P.expFunc == "luscher" ? GLAC_EXP_LUSCHER : P.expFunc == "taylor2" ? GLAC_EXP_TAYLOR2
                 : P.expFunc == "taylor4" ? GLAC_EXP_TAYLOR4 : GLAC_EXP_MORNINGSTAR;
    d.seed = (uint64_t)P.metropolisSeed;
    d.stream_id = 0;
    d.reunit_interval = P.reunitInterval;
    d.device = P.device;
    ck(glac_create(&d, &ctx), "glac_create");
    if (!P.loadFieldConfigurations && P.loadConfigAndRun.empty()) {
        if (P.hotStart) {
            if (P.RSTHotStart) ck(glac_rst_start(ctx, (uint64_t)P.randomMatrixSeed), "RST hot start");
            else ck(glac_hot_start(ctx, (uint64_t)P.randomMatrixSeed), "hot start");
        } else {
            ck(glac_cold_start(ctx), "cold start");
        }
        if (P.autotune) ck(glac_autotune(ctx, 3, nullptr), "autotune");
        std::printf("\nLattice setup complete\n");
    }
    std::printf("\nLattice %u^3 x %u, beta %g, %s, NUpdates %u, SU3Eps %g, flowEpsilon %g, expFunc %s",
                P.NSpatial, P.NTemporal, P.beta, P.precision.c_str(), P.NUpdates, P.SU3Eps, P.flowEpsilon,
                P.expFunc.c_str());
}

void System::checkLattice(const std::string &where) {
    if (!P.debug) return;
    double dev = 0;
    ck(glac_unitarity_violation(ctx, &dev), "unitarity check");
    if (!std::isfinite(dev) || dev > 1e-3) throw std::runtime_error("Configuration is corrupt " + where);
}

void System::storeConfigObservables(unsigned index, const std::vector<double> &obs) {
    const std::vector<std::string> names = sampler_names(cfgSampler, false);
    if (cfgObs.empty())
        for (const std::string &n : names) cfgObs.push_back(ObservableStorer{n, {}});
    for (size_t k = 0; k < names.size(); k++) {
        if (cfgObs[k].values.size() <= index) cfgObs[k].values.resize(index + 1, 0.0);
        cfgObs[k].values[index] = obs[row_offset(cfgSampler, names[k], P.NTemporal)];
    }
}

// GLAC/system.cpp:262-319
void System::thermalize() {
    std::printf("\nInitiating thermalization.");
    std::vector<double> obs(row_width(cfgSampler, P.NTemporal));
    if (P.storeThermalizationObservables) {
        NThermSteps = 1 + P.NTherm;
        measureInto(ctx, cfgSampler, 0, true, obs);
        storeConfigObservables(0, obs);
    }
    double accept = 0.0;
    for (unsigned i = 1; i < P.NTherm + 1; i++) {
        const auto t0 = std::chrono::steady_clock::now();
        double a = 0;
        ck(glac_metropolis(ctx, 1, &a), "metropolis");
        updateSeconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        accept += a;
        if (i % 20 == 0)
            std::printf("\n%6.2f %% done. Avg. update time: %10.6f sec", 100.0 * i / P.NTherm, updateSeconds / i);
        if (P.storeThermalizationObservables) {
            measureInto(ctx, cfgSampler, i, true, obs);
            storeConfigObservables(i, obs);
        }
    }
    if (P.NTherm) std::printf("\nTermalization complete. Acceptance rate: %f", accept / P.NTherm);
    thermalized = true;
}

// GLAC/system.cpp:363-469
void System::runMetropolis() {
    if (!thermalized) thermalize();
    std::printf("\ni    %-20s Avg.Update-time  Accept/reject", "observables");
    acceptanceScore = 0.0;
    double seconds = 0.0;
    std::vector<double> obs(row_width(cfgSampler, P.NTemporal));
    for (unsigned iConfig = 0; iConfig < P.NCf; iConfig++) {
        const auto t0 = std::chrono::steady_clock::now();
        double a = 0;
        ck(glac_metropolis(ctx, (int)P.NCor, &a), "metropolis");
        seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        acceptanceScore += a * P.NCor;
        checkLattice("in system right before copying to flow lattice");
        if (P.NFlows != 0) {
            flowConfiguration(iConfig);  // flows a copy; the chain field stays in ctx
            // the flow sampler's t = 0 values, by name, into the config sampler's row
            obs.assign(row_width(cfgSampler, P.NTemporal), 0.0);
            const std::vector<std::string> fnames = sampler_names(flowSampler, true);
            for (const std::string &n : sampler_names(cfgSampler, false))
                if (std::find(fnames.begin(), fnames.end(), n) != fnames.end() || n == "plaq" || n == "topc" ||
                    n == "energy")
                    obs[row_offset(cfgSampler, n, P.NTemporal)] = lastFlowT0[row_offset(flowSampler, n, P.NTemporal)];
        } else {
            measureInto(ctx, cfgSampler, iConfig + NThermSteps, true, obs);
        }
        storeConfigObservables(iConfig + NThermSteps, obs);
        std::printf("\n%-4u %-20.8f %-12.8f", iConfig, obs[0], seconds / ((iConfig + 1) * (double)P.NCor));
        if (iConfig % 10 == 0) std::printf("     %-10.8f", acceptanceScore / ((iConfig + 1) * (double)P.NCor));
        if (P.storeConfigurations) writeFieldToFile(iConfig);
    }
    std::printf("\nSystem completed.\nAcceptancerate: %.16f \nAverage update time: %.6f sec.\n", acceptanceRate(),
                (P.NCf * P.NCor) != 0 ? seconds / (P.NCf * P.NCor) : 0.0);
    for (ObservableStorer &o : cfgObs) {
        o.run_statistics();
        writeObservablesToFile(P, acceptanceRate(), o);
    }
}

double System::acceptanceRate() const {
    return (P.NCf * P.NCor) != 0 ? acceptanceScore / (double)(P.NCf * P.NCor) : 0.0;
}

// GLAC/system.cpp:471-517: flow a copy of the chain field, measuring at t = 0
// and after every step, then write the flow observables of this config.
void System::flowConfiguration(unsigned iConfig) {
    if (!flowCtx) {
        glac_desc d{};
        d.dims[0] = d.dims[1] = d.dims[2] = (int)P.NSpatial;
        d.dims[3] = (int)P.NTemporal;
        d.beta = P.beta;
        d.precision = P.precision == "fp32" ? GLAC_FP32 : GLAC_FP64;
        d.n_updates = (int)P.NUpdates;
        d.su3_eps = P.SU3Eps;
        d.flow_eps = P.flowEpsilon;
        d.exp_func = P.expFunc == "luscher" ? GLAC_EXP_LUSCHER : P.expFunc == "taylor2" ? GLAC_EXP_TAYLOR2
                     : P.expFunc == "taylor4" ? GLAC_EXP_TAYLOR4 : GLAC_EXP_MORNINGSTAR;
        d.seed = (uint64_t)P.metropolisSeed;
        d.reunit_interval = P.reunitInterval;
        d.device = P.device;
        ck(glac_create(&d, &flowCtx), "glac_create (flow lattice)");
    }
    ck(glac_copy_field(flowCtx, ctx), "copy to flow lattice");
    const size_t per = row_width(flowSampler, P.NTemporal);
    std::vector<double> obs((size_t)(P.NFlows + 1) * per);
    if (flowSampler == Sampler::ChargeDensity || flowSampler == Sampler::Super) {
        // step by step: the per-site fields every samplingFrequency flow steps
        // (LatticeActionChargeDensity::calculate, :277-294; file number = flow step)
        std::vector<double> o;
        const unsigned sf = P.samplingFrequency > 0 ? (unsigned)P.samplingFrequency : 1u;
        for (unsigned i = 0; i <= P.NFlows; i++) {
            if (i > 0 && glac_flow(flowCtx, 1, nullptr) != GLAC_OK)
                throw std::runtime_error(std::string("flow: ") + glac_last_error(flowCtx));
            measureInto(flowCtx, flowSampler, i, i % sf == 0, o);
            std::copy(o.begin(), o.end(), obs.begin() + (size_t)i * per);
        }
    } else {
        glac_status st = glac_flow(flowCtx, (int)P.NFlows, obs.data());
        if (st != GLAC_OK) throw std::runtime_error(std::string("flow: ") + glac_last_error(flowCtx));
    }
    lastFlowT0.assign(obs.begin(), obs.begin() + per);
    if (P.verbose)
        for (unsigned i = 0; i < P.NFlows + 1; i++)
            std::printf("\n%-4u %-3.3f  %-20.15f %-20.15f %-20.15f", i, i * P.flowEpsilon, obs[(size_t)i * per],
                        obs[(size_t)i * per + 1], obs[(size_t)i * per + 2]);
    for (const std::string &name : sampler_names(flowSampler, true)) {
        const size_t k = row_offset(flowSampler, name, P.NTemporal);
        if (name == "topct" || name == "weinbergt") {
            std::vector<double> m((size_t)(P.NFlows + 1) * P.NTemporal);
            for (unsigned i = 0; i < P.NFlows + 1; i++)
                for (unsigned t = 0; t < P.NTemporal; t++) m[(size_t)i * P.NTemporal + t] = obs[(size_t)i * per + k + t];
            writeMatrixToFile(P, name, m, iConfig, P.NTemporal);
        } else {
            std::vector<double> v(P.NFlows + 1);
            for (unsigned i = 0; i < P.NFlows + 1; i++) v[i] = obs[(size_t)i * per + k];
            writeFlowObservableToFile(P, name, v, iConfig);
        }
    }
}

// GLAC/system.cpp:541-568 (reads into the flow lattice when flowing,
// GLAC/io/fieldio.cpp:195-315)
void System::load(const std::string &name) {
    const std::string path = P.pwd + P.inputFolder + name;
    std::vector<double> host((size_t)V * 72);
    const int dims[4] = {(int)P.NSpatial, (int)P.NSpatial, (int)P.NSpatial, (int)P.NTemporal};
    glac_status st = glac_read_field(path.c_str(), dims, P.chromaConfig ? 1 : 0, host.data());
    if (st != GLAC_OK) throw std::runtime_error(glac_io_error());
    ck(glac_set_links(ctx, host.data()), "set links");
    std::printf("\nConfiguration %s loaded", path.c_str());
    // random-stream checkpoint written beside stored configurations: continue the chain's stream
    std::ifstream rng(path + ".rng");
    std::string key;
    double seed = 0;
    unsigned sweep = 0;
    if (rng >> key >> seed >> key >> sweep) {
        if (seed == P.metropolisSeed) {
            ck(glac_set_sweep(ctx, sweep), "set sweep");
            std::printf("; random stream continues at sweep %u", sweep);
        } else {
            std::printf("; its random-stream checkpoint is for metropolisSeed %g, not %g: stream restarts", seed,
                        P.metropolisSeed);
        }
    }
}

// GLAC/system.cpp:519-539
void System::loadConfigurationAndRunMetropolis() {
    thermalized = true;
    if (P.fieldConfigs.size() != 1)
        throw std::runtime_error("Should only be one configuration loaded(there are currently " +
                                 std::to_string(P.fieldConfigs.size()) + "configurations.");
    load(P.fieldConfigs[0]);
    runMetropolis();
}

// GLAC/system.cpp:570-602
void System::flowConfigurations() {
    if (P.fieldConfigs.empty())
        throw std::runtime_error("Missing configurations to flow. Check input folder: " + P.inputFolder);
    for (size_t i = 0; i < P.fieldConfigs.size(); i++) {
        load(P.fieldConfigs[i]);
        flowConfiguration((unsigned)i);
    }
    std::printf("\nFlowing of %zu configurations done.", P.fieldConfigs.size());
}

// GLAC/io/fieldio.cpp:61-135
void System::writeFieldToFile(unsigned iConfig) {
    const std::string dir = outDir() + "field_configurations/";
    makeDirs(dir);
    std::vector<double> host((size_t)V * 72);
    ck(glac_get_links(ctx, host.data()), "get links");
    const int dims[4] = {(int)P.NSpatial, (int)P.NSpatial, (int)P.NSpatial, (int)P.NTemporal};
    const std::string fname = fieldFileName(P, iConfig);
    if (glac_write_field((dir + fname).c_str(), dims, host.data()) != GLAC_OK) throw std::runtime_error(glac_io_error());
    // random-stream checkpoint (no counterpart in the reference): seed and Philox sweep counter
    uint32_t sweep = 0;
    ck(glac_get_sweep(ctx, &sweep), "get sweep");
    std::ofstream rng(dir + fname + ".rng");
    rng << "metropolisSeed " << std::setprecision(17) << P.metropolisSeed << "\nsweep " << sweep << "\n";
    std::printf("    %s written.", fname.c_str());
}

// GLAC/system.cpp:239-260
void System::run() {
    if (!P.loadFieldConfigurations && P.loadConfigAndRun.empty()) runMetropolis();
    else if (!P.loadConfigAndRun.empty()) loadConfigurationAndRunMetropolis();
    else flowConfigurations();
}

}  // namespace glac_host
