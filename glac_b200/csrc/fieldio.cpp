// GLAC .bin gauge-field files (GLAC/io/fieldio.cpp): per site (x fastest, then
// y, z, t) the 4 links mu = 0..3, each 18 doubles (re, im row-major), native
// byte order (writeFieldToFile :61-135, loadFieldConfiguration :195-257); the
// Chroma variant holds the same layout with each double byte-reversed
// (loadChromaFieldConfiguration :259-315, reverseDouble :317-330).
#include "../../include/glac_b200.h"

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {
thread_local std::string g_io_err;

long long volume(const int dims[4]) {
    long long V = 1;
    for (int k = 0; k < 4; k++) V *= dims[k];
    return V;
}
void swap_bytes(double &v) {
    unsigned char b[8];
    std::memcpy(b, &v, 8);
    for (int i = 0; i < 4; i++) { unsigned char t = b[i]; b[i] = b[7 - i]; b[7 - i] = t; }
    std::memcpy(&v, b, 8);
}
}  // namespace

extern "C" const char *glac_io_error(void) { return g_io_err.c_str(); }

extern "C" glac_status glac_read_field(const char *path, const int dims[4], int chroma, double *host_links) {
    if (!path || !dims || !host_links) { g_io_err = "null argument"; return GLAC_ERR_ARG; }
    for (int k = 0; k < 4; k++)
        if (dims[k] <= 0) { g_io_err = "bad dims"; return GLAC_ERR_ARG; }
    const long long V = volume(dims);
    FILE *f = std::fopen(path, "rb");
    if (!f) { g_io_err = std::string("File ") + path + " does not exist"; return GLAC_ERR_IO; }
    std::fseek(f, 0, SEEK_END);
    const long long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    const long long want = V * 4 * 18 * (long long)sizeof(double);
    if (size != want) {
        std::fclose(f);
        g_io_err = std::string("File ") + path + " has " + std::to_string(size) + " bytes, expected " +
                   std::to_string(want);
        return GLAC_ERR_IO;
    }
    std::vector<double> row((size_t)dims[0] * 4 * 18);
    const long long rows = V / dims[0];
    for (long long r = 0; r < rows; r++) {
        if (std::fread(row.data(), sizeof(double), row.size(), f) != row.size()) {
            std::fclose(f);
            g_io_err = "short read";
            return GLAC_ERR_IO;
        }
        for (int x = 0; x < dims[0]; x++) {
            const long long site = r * dims[0] + x;
            for (int mu = 0; mu < 4; mu++) {
                double *dst = host_links + ((size_t)mu * V + site) * 18;
                const double *src = row.data() + ((size_t)x * 4 + mu) * 18;
                for (int i = 0; i < 18; i++) {
                    double v = src[i];
                    if (chroma) swap_bytes(v);
                    dst[i] = v;
                }
            }
        }
    }
    std::fclose(f);
    return GLAC_OK;
}

extern "C" glac_status glac_write_field(const char *path, const int dims[4], const double *host_links) {
    if (!path || !dims || !host_links) { g_io_err = "null argument"; return GLAC_ERR_ARG; }
    const long long V = volume(dims);
    FILE *f = std::fopen(path, "wb");
    if (!f) { g_io_err = std::string("cannot open ") + path; return GLAC_ERR_IO; }
    std::vector<double> row((size_t)dims[0] * 4 * 18);
    const long long rows = V / dims[0];
    for (long long r = 0; r < rows; r++) {
        for (int x = 0; x < dims[0]; x++) {
            const long long site = r * dims[0] + x;
            for (int mu = 0; mu < 4; mu++)
                std::memcpy(row.data() + ((size_t)x * 4 + mu) * 18, host_links + ((size_t)mu * V + site) * 18,
                            18 * sizeof(double));
        }
        if (std::fwrite(row.data(), sizeof(double), row.size(), f) != row.size()) {
            std::fclose(f);
            g_io_err = "short write";
            return GLAC_ERR_IO;
        }
    }
    std::fclose(f);
    return GLAC_OK;
}
