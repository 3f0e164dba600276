// GLAC-compatible program entry: `GLAC config.json` (GLAC/main.cpp:50-84).
// Runs on one GPU; tolerates being started under `mpirun -np 1` as
// createJobs.py does.  `GLAC --print-config config.json` prints the parsed
// run-configuration as JSON and exits (no GPU needed).
#include <chrono>
#include <cstdio>
#include <cstring>
#include <exception>

#include "glac_host.h"

int main(int argc, char **argv) {
    if (argc == 3 && std::strcmp(argv[1], "--print-config") == 0) {
        try {
            std::printf("%s\n", glac_host::Parameters::load(argv[2]).to_json().c_str());
            return 0;
        } catch (const std::exception &e) {
            std::printf("\n%s\n", e.what());
            return 1;
        }
    }
    if (argc != 2) {
        std::printf("\nError: please provide a json file to parse.\n");
        return 1;
    }
    const auto t0 = std::chrono::steady_clock::now();
    try {
        glac_host::Parameters p = glac_host::Parameters::load(argv[1]);
        if (p.unitTesting || p.performanceTesting)
            std::printf("\nunitTesting / performanceTesting are the reference's in-binary suites; "
                        "this implementation's tests live in tests/ (pytest).");
        glac_host::System pureGauge(p);
        pureGauge.latticeSetup();
        pureGauge.run();
    } catch (const std::exception &e) {
        std::printf("\n%s\n", e.what());
        return 1;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("\nProgram complete. Time used: %f hours (%f seconds)\n", secs / 3600.0, secs);
    return 0;
}
