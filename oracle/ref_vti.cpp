// ref_vti.cpp -- test-only C wrapper around the reference's own header-only
// readVTI (include/vti/VTIReader.hpp:35-160), compiled against the reference
// tree where it lies (oracle/build_oracle.py); the checker for fm_vti_read.
#include <cstdint>
#include <cstring>
#include <stdexcept>
#include <string>

#include "vti/VTIReader.hpp"

static thread_local std::string g_err;

extern "C" {

// 0 on success; -1 with the exception text in ref_vti_error() otherwise.
// mask may be NULL (dimensions only); cap is its capacity in cells.
int ref_vti_read(const char* path, double threshold, int* nx, int* ny, int* nz, uint8_t* mask, long long cap)
{
    try {
        VTIResult r = readVTI(path, threshold);
        *nx = r.Nx;
        *ny = r.Ny;
        *nz = r.Nz;
        if (mask) {
            if ((long long)r.mask.size() > cap) throw std::runtime_error("mask capacity too small");
            std::memcpy(mask, r.mask.data(), r.mask.size());
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

const char* ref_vti_error() { return g_err.c_str(); }
}
