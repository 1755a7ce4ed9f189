// ref_params_driver.cpp -- TEST INFRASTRUCTURE.
// Exposes the reference's own icy::SimParams::Reset / ParseFile
// (simulation/parameters_sim.cpp, compiled unmodified) through a C call so the
// tests can pin this library's JSON reader and derived constants against it.
#include <cstring>
#include <string>
#include <stdexcept>

#include "parameters_sim.h"
#include "ref_driver_common.h"

extern "C" {

void ref_params_reset(icy_sim_params *out) {
    icy::SimParams p{};  // zero the fields Reset() leaves unset
    p.Reset();
    std::memcpy(out, &p, sizeof(p));
}

// Parse a JSON file the way the reference does.  Returns 0 on success,
// 1 if the reference threw (message copied to err).
int ref_params_parse_file(icy_sim_params *inout, const char *path, char *raw, size_t cap,
                          char *err, size_t errcap) {
    icy::SimParams p;
    std::memcpy(&p, inout, sizeof(p));
    try {
        std::string r = p.ParseFile(path);
        std::strncpy(raw, r.c_str(), cap - 1);
        raw[cap - 1] = 0;
    } catch (const std::exception &e) {
        std::memcpy(inout, &p, sizeof(p));
        std::strncpy(err, e.what(), errcap - 1);
        err[errcap - 1] = 0;
        return 1;
    }
    std::memcpy(inout, &p, sizeof(p));
    return 0;
}

void ref_params_compute_helpers(icy_sim_params *inout) {
    icy::SimParams p;
    std::memcpy(&p, inout, sizeof(p));
    p.ComputeHelperVariables();
    std::memcpy(inout, &p, sizeof(p));
}

}  // extern "C"
