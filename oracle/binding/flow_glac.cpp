// GLAC's Flow operator bound to the glac_b200 C ABI: the binding a maintainer
// keeping the reference's own System, correlators and IO would add.  This file
// takes the place of GLAC/flow/flow.cpp (GLAC/flow/flow.h:42 declares the
// class) in a build of the reference sources; everything else -- configuration
// loading, the run modes of System (system.cpp:471-602), the
// MasterSamplerTopcXYZ measurement, the output files -- stays the reference's.
//
// Flow::flowField (flow.cpp:43-73, one Luscher RK3 step of all four link
// directions) becomes: the Lattice<SU3>[4] memory (4 blocks of V SU3 = 18
// doubles, exactly the C ABI's host layout) copied into a glac_b200 context,
// one RK3 step on the GPU (glac_flow), the field copied back.  The context is
// made on the first call from the reference's static Parameters (lattice size,
// flowEpsilon, expFunc) and lives until exit.  On a status other than
// GLAC_OK the message is printed and the run ends through MPIExit, as the
// reference ends on its own errors (communicator.cpp:526-537).
//
// TEST INFRASTRUCTURE: built by oracle/Makefile (target ref-bin-bound) into
// oracle/_ref/bin/GLAC_bound and run by tests/test_reference_binding.py.
#include "flow/flow.h"

#include <cstring>
#include <string>
#include <vector>

#include "config/parameters.h"
#include "glac_b200.h"
#include "parallelization/communicator.h"

namespace {

glac_ctx *g_ctx = nullptr;
std::vector<double> g_host;

void check(glac_status s, const char *what) {
    if (s == GLAC_OK) return;
    std::string msg = std::string("glac_b200 ") + what + ": " + (g_ctx ? glac_last_error(g_ctx) : glac_global_error());
    Parallel::Communicator::MPIExit(msg);
}

int exp_kind(const std::string &name) {
    if (name == "luscher") return GLAC_EXP_LUSCHER;
    if (name == "taylor2") return GLAC_EXP_TAYLOR2;
    if (name == "taylor4") return GLAC_EXP_TAYLOR4;
    return GLAC_EXP_MORNINGSTAR;  // the reference's default and its fallback (flow.cpp:75-93)
}

void ensure_context() {
    if (g_ctx) return;
    glac_desc d;
    std::memset(&d, 0, sizeof(d));
    const std::vector<unsigned int> N = Parameters::getN();  // this rank's (= the whole) lattice
    for (int k = 0; k < 4; k++) d.dims[k] = (int)N[k];
    d.beta = Parameters::getBeta();
    d.precision = GLAC_FP64;
    d.n_updates = (int)Parameters::getNUpdates();
    d.su3_eps = Parameters::getSU3Eps();
    d.flow_eps = Parameters::getFlowEpsilon();
    d.exp_func = exp_kind(Parameters::getExpFuncName());
    d.seed = (uint64_t)Parameters::getMetropolisSeed();
    check(glac_create(&d, &g_ctx), "glac_create");
}

}  // namespace

Flow::Flow(Action *S) {
    m_N = Parameters::getN();
    m_epsilon = Parameters::getFlowEpsilon();
    m_subLatticeSize = Parameters::getSubLatticeSize();
    m_tempLattice = nullptr;  // the device context holds the stage temporaries
    m_S = S;
}

Flow::~Flow() {}

void Flow::setSU3ExpFunc() {}

void Flow::flowField(Lattice<SU3> *lattice) {
    ensure_context();
    const size_t V = lattice[0].m_sites.size();
    g_host.resize(4 * V * 18);
    for (int mu = 0; mu < 4; mu++) std::memcpy(&g_host[mu * V * 18], lattice[mu].m_sites.data(), V * sizeof(SU3));
    check(glac_set_links(g_ctx, g_host.data()), "glac_set_links");
    check(glac_flow(g_ctx, 1, nullptr), "glac_flow");
    check(glac_get_links(g_ctx, g_host.data()), "glac_get_links");
    for (int mu = 0; mu < 4; mu++) std::memcpy(lattice[mu].m_sites.data(), &g_host[mu * V * 18], V * sizeof(SU3));
}
