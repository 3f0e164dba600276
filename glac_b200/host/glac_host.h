// Host side of the drop-in: GLAC's run-configuration, its System driver and its
// output files, over the C ABI of include/glac_b200.h.
//
// Mirrors the reference's call surface for the hot path:
//   ConfigLoader::load(json)  -> Parameters        (GLAC/config/configloader.cpp:55-181)
//   System::latticeSetup()/run()                   (GLAC/system.cpp:193-260)
//   thermalize / update / runMetropolis            (GLAC/system.cpp:262-469)
//   flowConfiguration / flowConfigurations         (GLAC/system.cpp:471-602)
//   IO::writeObservablesToFile / writeFlowObservableToFile / writeMatrixToFile
//                                                  (GLAC/io/observablesio.cpp:29-193)
//   IO::FieldIO::writeFieldToFile / load*          (GLAC/io/fieldio.cpp:61-315)
// The physics runs on the GPU through glac_metropolis / glac_flow / glac_measure.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/glac_b200.h"

namespace glac_host {

// Every key GLAC's job driver writes (createJobs.py _create_json), plus the
// optional keys of this implementation ("precision", "device",
// "reunitInterval", "autotune"), which default to the reference's behaviour.
struct Parameters {
    unsigned NSpatial = 8, NTemporal = 16;
    std::vector<unsigned> subDims;
    double beta = 6.0;
    unsigned NCf = 0, NCor = 0, NTherm = 0, NFlows = 0, NUpdates = 10;
    std::string action = "wilson";
    std::string outputFolder = "/output/", inputFolder = "/input/";
    bool storeConfigurations = false, storeThermalizationObservables = false, verbose = false;
    std::string pwd = ".", batchName = "run";
    bool hotStart = false, RSTHotStart = false;
    std::string expFunc = "morningstar";
    std::vector<std::string> observables = {"plaq"}, flowObservables = {"plaq", "topc", "energy"};
    bool loadFieldConfigurations = false, chromaConfig = false;
    std::vector<std::string> fieldConfigs;
    std::string loadConfigAndRun;
    int configStartNumber = 0;
    bool unitTesting = false, performanceTesting = false, debug = false;
    double SU3Eps = 0.24, flowEpsilon = 0.01;
    double metropolisSeed = 0, randomMatrixSeed = 0;
    int samplingFrequency = 25;
    // optional keys of this implementation
    std::string precision = "fp64";
    int device = 0;
    int reunitInterval = 0;
    bool autotune = false;

    static Parameters load(const std::string &json_path);  // GLAC/config/configloader.cpp:55-181
    std::string to_json() const;
};

// Per-observable storage, mean and variance (GLAC/observables/tools/observablestorer.cpp:14-160).
struct ObservableStorer {
    std::string name;
    std::vector<double> values;
    double mean = 0, variance = 0, stdev = 0;
    void run_statistics();
};

// Which observables a list selects (GLAC/system.cpp:62-125): plaquette only, the
// three-observable MasterSampler, MasterSamplerTopcXYZ (adds topct), or
// LatticeActionChargeDensity (energyTopcFieldDensity alone: per-site q and E
// fields written to scalar_fields/).
// "weinberg" anywhere in the list selects SuperSampler (adds weinberg, weinbergt).
enum class Sampler { Plaquette, Master, MasterTopcXYZ, ChargeDensity, Super };
Sampler select_sampler(const std::vector<std::string> &names);
std::vector<std::string> sampler_names(Sampler s, bool flow);
// Layout of a measurement row: scalars [plaq, topc, energy(, weinberg)], then
// topct[Nt] (and weinbergt[Nt] for SuperSampler).
size_t row_width(Sampler s, unsigned Nt);
size_t row_offset(Sampler s, const std::string &name, unsigned Nt);

class System {
public:
    explicit System(const Parameters &p);
    ~System();
    void latticeSetup();  // GLAC/system.cpp:193-231
    void run();           // GLAC/system.cpp:239-260
    double acceptanceRate() const;

private:
    void thermalize();
    void runMetropolis();
    void loadConfigurationAndRunMetropolis();
    void flowConfigurations();
    void flowConfiguration(unsigned iConfig);
    void load(const std::string &name);
    void writeFieldToFile(unsigned iConfig);
    void storeConfigObservables(unsigned index, const std::vector<double> &obs);
    void checkLattice(const std::string &where);
    // glac_measure, or for the charge-density sampler also the per-site fields,
    // written when `write` (LatticeActionChargeDensity::calculate, :277-305)
    void measureInto(glac_ctx *c, Sampler s, unsigned index, bool write, std::vector<double> &obs);
    void ck(glac_status s, const char *what);
    std::string outDir() const;

    Parameters P;
    glac_ctx *ctx = nullptr;      // the Markov-chain lattice (System::m_lattice)
    glac_ctx *flowCtx = nullptr;  // the flow lattice (System::m_flowLattice)
    std::vector<double> lastFlowT0;
    unsigned V = 0;
    Sampler cfgSampler, flowSampler;
    std::vector<ObservableStorer> cfgObs;
    double acceptanceScore = 0.0;
    double updateSeconds = 0.0;
    unsigned NThermSteps = 0;
    bool thermalized = false;
};

// Output files in the reference's formats.
void writeObservablesToFile(const Parameters &P, double acceptance, const ObservableStorer &o);
void writeFlowObservableToFile(const Parameters &P, const std::string &name, const std::vector<double> &values,
                               unsigned configNumber);
void writeMatrixToFile(const Parameters &P, const std::string &name, const std::vector<double> &values,
                       unsigned configNumber, unsigned N);
std::string fieldFileName(const Parameters &P, unsigned configNumber);
// scalar_fields/<observable>/<field file name>: V doubles, x fastest (GLAC/io/fieldio.cpp:137-193)
void writeScalarField(const Parameters &P, const std::string &observable, const std::vector<double> &field,
                      unsigned configNumber);
void makeDirs(const std::string &path);

}  // namespace glac_host
