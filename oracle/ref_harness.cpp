/*
 * C entry points around the reference GLAC objects, compiled from the
 * reference's own sources (see oracle/Makefile) with the single-rank MPI
 * stand-in in oracle/mpishim.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the bridge that lets the parity
 * tests and the CPU-baseline leg of bench.py call the reference's code
 * (WilsonGaugeAction, Flow, SU3Exp/ExpLuscher/Taylor*, MasterSamplerTopcXYZ,
 * Plaquette, SU3MatrixGenerator, System::update, IO::FieldIO) on host arrays.
 * It never runs on the product path.
 *
 * Host array layout used by every entry point: 4 blocks (mu = 0..3) of V
 * matrices, each 18 doubles (re, im row-major), sites in the reference's
 * Index::getIndex order (x fastest) -- exactly the memory of Lattice<SU3>[4]
 * (GLAC/math/lattice.h:23-180, GLAC/parallelization/index.h:32-35).
 */
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>
#include <random>
#include <chrono>
#include <iostream>
#include <fstream>
#include <sstream>
#include <map>
#include <algorithm>
#include <functional>
#include <memory>

// Private members (the staple held by WilsonGaugeAction, System::update, the
// RST multiplication) are read directly by this test bridge.
#define private public
#define protected public
#include "system.h"
#include "config/parameters.h"
#include "parallelization/parallel.h"
#include "parallelization/communicator.h"
#include "actions/actions.h"
#include "observables/observables.h"
#include "flow/flow.h"
#include "math/exponentiation/su3exp.h"
#include "math/exponentiation/expluscher.h"
#include "math/exponentiation/taylor2exp.h"
#include "math/exponentiation/taylor4exp.h"
#include "math/exponentiation/taylorexp.h"
#include "math/matrices/su3matrixgenerator.h"
#include "io/fieldio.h"
#undef private
#undef protected

namespace {

bool g_comm_ready = false;
int g_N[4] = {0, 0, 0, 0};
unsigned long g_V = 0;

std::vector<unsigned int> dims() {
    return {unsigned(g_N[0]), unsigned(g_N[1]), unsigned(g_N[2]), unsigned(g_N[3])};
}

void to_lattice(const double *links, Lattice<SU3> *L) {
    for (int mu = 0; mu < 4; mu++) {
        L[mu].allocate(dims());
        for (unsigned long s = 0; s < g_V; s++)
            std::memcpy(L[mu].m_sites[s].mat, links + (mu * g_V + s) * 18, 18 * sizeof(double));
    }
}

void from_lattice(Lattice<SU3> *L, double *links) {
    for (int mu = 0; mu < 4; mu++)
        for (unsigned long s = 0; s < g_V; s++)
            std::memcpy(links + (mu * g_V + s) * 18, L[mu].m_sites[s].mat, 18 * sizeof(double));
}

/* System::subLatticeSetup allocates the flow lattice only when NFlows > 0, while
 * ~System deletes it unconditionally: give it a valid null in that case. */
void setup_system(System &sys) {
    sys.m_flowLattice = nullptr;
    sys.subLatticeSetup();
}

void load_su3(SU3 &A, const double *p) { std::memcpy(A.mat, p, 18 * sizeof(double)); }
void store_su3(const SU3 &A, double *p) { std::memcpy(p, A.mat, 18 * sizeof(double)); }

}  // namespace

extern "C" {

/* Sets the reference's static Parameters for an Ns^3 x Nt lattice on one rank
 * (GLAC/config/configloader.cpp:55-181 does the same from JSON). */
int ref_configure(int Ns, int Nt, double beta, double su3eps, double flowEps, const char *expFunc,
                  double metropolisSeed, double randomMatrixSeed, int NUpdates, int NFlows) {
    if (!g_comm_ready) {
        static char a0[] = "glacref", a1[] = "none.json";
        static char *argv_[] = {a0, a1, nullptr};
        int argc = 2;
        char **argv = argv_;
        Parallel::Communicator::init(&argc, &argv);
        g_comm_ready = true;
    }
    Parameters::setLatticeSize(1);
    Parameters::setNSpatial(Ns);
    Parameters::setNTemporal(Nt);
    Parallel::Index::setNTot(Ns, Nt);
    Parameters::setSubLatticePreset(false);
    Parameters::setBeta(beta);
    Parameters::setSU3Eps(su3eps);
    Parameters::setFlowEpsilon(flowEps);
    Parameters::setExpFuncName(std::string(expFunc));
    Parameters::setMetropolisSeed(metropolisSeed);
    Parameters::setRandomMatrixSeed(randomMatrixSeed);
    Parameters::setNUpdates(NUpdates);
    Parameters::setNFlows(NFlows);
    Parameters::setNCf(1);
    Parameters::setNCor(1);
    Parameters::setNTherm(0);
    Parameters::setActionType("wilson");
    Parameters::setStoreThermalizationObservables(false);
    Parameters::setStoreConfigurations(false);
    Parameters::setVerbose(false);
    Parameters::setDebug(false);
    Parameters::setUnitTesting(false);
    Parameters::setLoadFieldConfigurations(false);
    Parameters::setLoadConfigAndRun(false);
    Parameters::setConfigStartNumber(0);
    Parameters::setObservableList({"plaq"});
    Parameters::setFlowObservablesList({"plaq", "topc", "energy", "topct"});
    Parameters::setFilePath("");
    Parameters::setInputFolder("");
    Parameters::setOutputFolder("");
    Parameters::setBatchName("ref");
    Parallel::Communicator::initializeSubLattice();
    IO::FieldIO::init();
    g_N[0] = g_N[1] = g_N[2] = Ns;
    g_N[3] = Nt;
    g_V = (unsigned long)Ns * Ns * Ns * Nt;
    return 0;
}

/* WilsonGaugeAction::computeStaple (GLAC/actions/wilsongaugeaction.cpp:29-53) for every link. */
void ref_staples(const double *links, double *out) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    WilsonGaugeAction S;
    for (int t = 0; t < g_N[3]; t++)
        for (int z = 0; z < g_N[2]; z++)
            for (int y = 0; y < g_N[1]; y++)
                for (int x = 0; x < g_N[0]; x++)
                    for (int mu = 0; mu < 4; mu++) {
                        S.computeStaple(L.get(), x, y, z, t, mu);
                        unsigned long s = Parallel::Index::getIndex(x, y, z, t);
                        store_su3(S.m_staple, out + (mu * g_V + s) * 18);
                    }
}

/* WilsonGaugeAction::getDeltaAction (GLAC/actions/wilsongaugeaction.cpp:24-27). */
double ref_delta_s(const double *U, const double *Uprime, const double *staple) {
    WilsonGaugeAction S;
    SU3 a, b;
    load_su3(a, U);
    load_su3(b, Uprime);
    load_su3(S.m_staple, staple);
    return S.getDeltaAction(a, b);
}

/* WilsonGaugeAction::getActionDerivative (GLAC/actions/wilsongaugeaction.cpp:55-86), all mu. */
void ref_action_derivative(const double *links, double *out) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    WilsonGaugeAction S;
    for (int mu = 0; mu < 4; mu++) {
        Lattice<SU3> Z = S.getActionDerivative(L.get(), mu);
        for (unsigned long s = 0; s < g_V; s++) store_su3(Z.m_sites[s], out + (mu * g_V + s) * 18);
    }
}

/* Exponentials (GLAC/math/exponentiation/): kind 0 Morningstar (su3exp.cpp:16-79),
 * 1 Luscher (expluscher.cpp:13-68), 2 Taylor-2, 3 Taylor-4, 4 Taylor-N (degree). */
void ref_exp(int kind, int degree, const double *in, long n, double *out) {
    SU3Exp ms;
    ExpLuscher lu;
    Taylor2Exp t2;
    Taylor4Exp t4;
    TaylorExp tn(degree > 0 ? degree : 16);
    for (long i = 0; i < n; i++) {
        SU3 Q, R;
        load_su3(Q, in + 18 * i);
        switch (kind) {
        case 0: R = ms.exp(Q); break;
        case 1: R = lu.exp(Q); break;
        case 2: R = t2.exp(Q); break;
        case 3: R = t4.exp(Q); break;
        default: R = tn.exp(Q); break;
        }
        store_su3(R, out + 18 * i);
    }
}

/* Flow::flowField (GLAC/flow/flow.cpp:43-73), nsteps times, in place. */
void ref_flow(double *links, int nsteps) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    WilsonGaugeAction S;
    Flow F(&S);
    for (int i = 0; i < nsteps; i++) F.flowField(L.get());
    from_lattice(L.get(), links);
}

/* MasterSamplerTopcXYZ::calculate (GLAC/observables/mastersamplertopcxyz.cpp:236-384):
 * out = [plaq, topc, energy, topct[0..Nt-1]]. */
void ref_observables(const double *links, double *out) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    MasterSamplerTopcXYZ M(true);
    M.reset();
    M.calculate(L.get(), 0);
    std::vector<double> v = M.getObservablesVector(0);
    for (size_t i = 0; i < v.size(); i++) out[i] = v[i];
}

/* MasterSampler::calculate (GLAC/observables/mastersampler.cpp:161-287): out = [plaq, topc, energy]. */
void ref_observables_nt(const double *links, double *out) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    MasterSampler M(true);
    M.reset();
    M.calculate(L.get(), 0);
    std::vector<double> v = M.getObservablesVector(0);
    for (size_t i = 0; i < 3; i++) out[i] = v[i];
}

/* SuperSampler::calculate (GLAC/observables/supersampler.cpp:298-496) at
 * measurement 0: out = [plaq, topc, energy, weinberg, topct[Nt], weinbergt[Nt]]. */
void ref_supersampler(const double *links, double *out) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    SuperSampler S(true);
    S.reset();
    S.calculate(L.get(), 0);
    const int Nt = g_N[3];
    out[0] = (*S.m_plaqObservable)[0];
    out[1] = (*S.m_topcObservable)[0];
    out[2] = (*S.m_energyObservable)[0];
    out[3] = (*S.m_wObservable)[0];
    for (int t = 0; t < Nt; t++) {
        out[4 + t] = (*S.m_topctObservable)[t];
        out[4 + Nt + t] = (*S.m_wtObservable)[t];
    }
}

/* LatticeActionChargeDensity::calculate (GLAC/observables/latticeactionchargedensity.cpp:169-306)
 * as a flow sampler at a measurement index the sampling frequency skips, so
 * nothing is written; the per-site fields are read from the sampler. */
void ref_density(const double *links, double *q, double *e, double *obs3) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    const int sf = Parameters::getSamplingFrequency();
    Parameters::setSamplingFrequency(1 << 30);
    {
        LatticeActionChargeDensity S(true);
        S.calculate(L.get(), 1);
        for (unsigned long s = 0; s < g_V; s++) {
            q[s] = S.m_topCharge.m_sites[s];
            e[s] = S.m_energy.m_sites[s];
        }
        std::vector<double> v = S.getObservablesVector(1);
        for (int i = 0; i < 3; i++) obs3[i] = v[i];
    }
    Parameters::setSamplingFrequency(sf);
}

/* Plaquette::calculate (GLAC/observables/plaquette.cpp:26-40). */
double ref_plaquette(const double *links) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    Plaquette P(true);
    P.calculate(L.get(), 0);
    return (*P.m_observable)[0];
}

/* SU3MatrixGenerator (GLAC/math/matrices/su3matrixgenerator.h:98-196), seeded from
 * Parameters::getRandomMatrixSeed and SU3Eps: kind 0 generateRST, 1 generateRandom. */
void ref_generate(int kind, long n, double *out) {
    SU3MatrixGenerator G;
    for (long i = 0; i < n; i++) {
        SU3 X = kind == 0 ? G.generateRST() : G.generateRandom();
        store_su3(X, out + 18 * i);
    }
}

/* SU3MatrixGenerator::RSTMatrixMultiplication / ...Inverse (su3matrixgenerator.h:245-321). */
void ref_rst_multiply(const double *r8, const double *s8, const double *t8, int inverse, double *out) {
    SU3MatrixGenerator G;
    SU2 r, s, t;
    std::memcpy(r.mat, r8, 8 * sizeof(double));
    std::memcpy(s.mat, s8, 8 * sizeof(double));
    std::memcpy(t.mat, t8, 8 * sizeof(double));
    SU3 X = inverse ? G.RSTMatrixMultiplicationInverse(r, s, t) : G.RSTMatrixMultiplication(r, s, t);
    store_su3(X, out);
}

/* Runs System::update (GLAC/system.cpp:333-361) nsweeps times on the given field,
 * in place; returns the mean acceptance per sweep (system.cpp:359). */
double ref_metropolis(double *links, int nsweeps) {
    System sys;
    setup_system(sys);
    for (int mu = 0; mu < 4; mu++)
        for (unsigned long s = 0; s < g_V; s++)
            std::memcpy(sys.m_lattice[mu].m_sites[s].mat, links + (mu * g_V + s) * 18, 18 * sizeof(double));
    for (int i = 0; i < nsweeps; i++) sys.update();
    for (int mu = 0; mu < 4; mu++)
        for (unsigned long s = 0; s < g_V; s++)
            std::memcpy(links + (mu * g_V + s) * 18, sys.m_lattice[mu].m_sites[s].mat, 18 * sizeof(double));
    return sys.m_acceptanceScore / double(nsweeps > 0 ? nsweeps : 1);
}

/* A Markov chain of nsweeps System::update sweeps from one System (so its
 * generators run on, as in System::runMetropolis, GLAC/system.cpp:363-469),
 * with the plaquette (GLAC/observables/plaquette.cpp:26-40) after every sweep
 * in plaq[nsweeps].  Returns the mean acceptance per sweep. */
double ref_metropolis_chain(double *links, int nsweeps, double *plaq) {
    System sys;
    setup_system(sys);
    for (int mu = 0; mu < 4; mu++)
        for (unsigned long s = 0; s < g_V; s++)
            std::memcpy(sys.m_lattice[mu].m_sites[s].mat, links + (mu * g_V + s) * 18, 18 * sizeof(double));
    Plaquette P(true);
    for (int i = 0; i < nsweeps; i++) {
        sys.update();
        P.calculate(sys.m_lattice, 0);
        plaq[i] = (*P.m_observable)[0];
    }
    for (int mu = 0; mu < 4; mu++)
        for (unsigned long s = 0; s < g_V; s++)
            std::memcpy(links + (mu * g_V + s) * 18, sys.m_lattice[mu].m_sites[s].mat, 18 * sizeof(double));
    return sys.m_acceptanceScore / double(nsweeps > 0 ? nsweeps : 1);
}

/* One Metropolis sweep in System::update's order (x, y, z, t outer to inner, then
 * mu; GLAC/system.cpp:338-357) with the draws recorded: for each visited link in
 * visiting order, the link before its hits, its staple, the NUpdates proposals X
 * (generateRST, su3matrixgenerator.h:170-196), the accept uniforms r
 * (system.cpp:347) and the decisions.  Uses System's own generators, seeded as
 * System::System does (system.cpp:36-41).  links is updated in place; order
 * receives (mu, site) of each visited link. */
long ref_metropolis_trace(double *links, double *U_before, double *staples, double *X,
                          double *r, unsigned char *accept, int *order) {
    System sys;
    setup_system(sys);
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    WilsonGaugeAction S;
    const unsigned int nup = Parameters::getNUpdates();
    long k = 0;
    for (int x = 0; x < g_N[0]; x++)
        for (int y = 0; y < g_N[1]; y++)
            for (int z = 0; z < g_N[2]; z++)
                for (int t = 0; t < g_N[3]; t++)
                    for (int mu = 0; mu < 4; mu++) {
                        unsigned long s = Parallel::Index::getIndex(x, y, z, t);
                        S.computeStaple(L.get(), x, y, z, t, mu);
                        store_su3(L[mu].m_sites[s], U_before + 18 * k);
                        store_su3(S.m_staple, staples + 18 * k);
                        order[2 * k] = mu;
                        order[2 * k + 1] = int(s);
                        for (unsigned int n = 0; n < nup; n++) {
                            SU3 Xn = sys.m_SU3Generator->generateRST();
                            SU3 Up = Xn * L[mu].m_sites[s];
                            double rn = sys.m_uniform_distribution(sys.m_generator);
                            bool acc = std::exp(-S.getDeltaAction(L[mu].m_sites[s], Up)) > rn;
                            store_su3(Xn, X + 18 * (k * nup + n));
                            r[k * nup + n] = rn;
                            accept[k * nup + n] = acc ? 1 : 0;
                            if (acc) L[mu].m_sites[s] = Up;
                        }
                        k++;
                    }
    from_lattice(L.get(), links);
    return k;
}

/* IO::FieldIO::loadFieldConfiguration / loadChromaFieldConfiguration
 * (GLAC/io/fieldio.cpp:195-315) from a full path. */
void ref_load_field(const char *path, int chroma, double *links) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    for (int mu = 0; mu < 4; mu++) L[mu].allocate(dims());
    Parameters::setFilePath("");
    Parameters::setInputFolder("");
    if (chroma) IO::FieldIO::loadChromaFieldConfiguration(std::string(path), L.get());
    else IO::FieldIO::loadFieldConfiguration(std::string(path), L.get());
    from_lattice(L.get(), links);
}

/* IO::FieldIO::writeFieldToFile (GLAC/io/fieldio.cpp:61-135) into
 * <dir>/<batch>/field_configurations/; returns 0 on success. */
int ref_write_field(const double *links, const char *dir, const char *batch, int configNumber) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    Parameters::setFilePath(std::string(dir));
    Parameters::setOutputFolder("");
    Parameters::setBatchName(std::string(batch));
    Parameters::setUnitTesting(true);
    IO::FieldIO::writeFieldToFile(L.get(), configNumber);
    Parameters::setUnitTesting(false);
    return 0;
}

/* PerformanceTests::testFlow-style timing (GLAC/tests/performancetests.cpp:433-509):
 * seconds for nsteps of Flow::flowField on the given field (in place). */
double ref_time_flow(double *links, int nsteps) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    WilsonGaugeAction S;
    Flow F(&S);
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < nsteps; i++) F.flowField(L.get());
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    from_lattice(L.get(), links);
    return dt;
}

/* Seconds for nsteps of (Flow::flowField + MasterSamplerTopcXYZ::calculate), the
 * per-step work of System::flowConfiguration (GLAC/system.cpp:490-510). */
double ref_time_flow_measure(double *links, int nsteps) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    WilsonGaugeAction S;
    Flow F(&S);
    MasterSamplerTopcXYZ M(true);
    M.reset();
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < nsteps; i++) {
        F.flowField(L.get());
        M.calculate(L.get(), (unsigned)((i + 1) % (Parameters::getNFlows() + 1)));
    }
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    from_lattice(L.get(), links);
    return dt;
}

/* Seconds for nsweeps of System::update (the reference's own per-sweep timer
 * brackets the same call, GLAC/system.cpp:395-401). */
double ref_time_metropolis(double *links, int nsweeps, double *acceptance) {
    System sys;
    setup_system(sys);
    for (int mu = 0; mu < 4; mu++)
        for (unsigned long s = 0; s < g_V; s++)
            std::memcpy(sys.m_lattice[mu].m_sites[s].mat, links + (mu * g_V + s) * 18, 18 * sizeof(double));
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < nsweeps; i++) sys.update();
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int mu = 0; mu < 4; mu++)
        for (unsigned long s = 0; s < g_V; s++)
            std::memcpy(links + (mu * g_V + s) * 18, sys.m_lattice[mu].m_sites[s].mat, 18 * sizeof(double));
    if (acceptance) *acceptance = sys.m_acceptanceScore / double(nsweeps > 0 ? nsweeps : 1);
    return dt;
}

/* Seconds for nmeas MasterSamplerTopcXYZ::calculate calls on the given field. */
double ref_time_observables(const double *links, int nmeas) {
    std::unique_ptr<Lattice<SU3>[]> L(new Lattice<SU3>[4]);
    to_lattice(links, L.get());
    MasterSamplerTopcXYZ M(true);
    auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < nmeas; i++) { M.reset(); M.calculate(L.get(), 0); }
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // extern "C"
