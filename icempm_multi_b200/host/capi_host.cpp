// capi_host.cpp -- C entry points of libicempm_host.so (include/icempm_host.h).
#include <cstring>
#include <exception>
#include <string>

#include "../../include/icempm_host.h"
#include "h5lite.hpp"
#include "icy_host.hpp"

namespace {
thread_local std::string g_host_error;

int failed(int code, const std::exception &e)
{
    g_host_error = e.what();
    return code;
}
}  // namespace

extern "C" {

const char *icy_host_last_error(void) { return g_host_error.c_str(); }

int icy_h5_count(const char *path, unsigned *n_points)
{
    if (!path || !n_points) return ICY_ERR_INVALID_ARGUMENT;
    try {
        icy::h5::File f(path);
        const auto d = f.dims("llGrainIDs");
        if (d.size() != 1) { g_host_error = "llGrainIDs is not one-dimensional"; return ICY_ERR_FILE; }
        *n_points = (unsigned)d[0];
        return ICY_OK;
    } catch (const std::exception &e) {
        return failed(ICY_ERR_FILE, e);
    }
}

int icy_h5_load(icy_sim_params *p, const char *path, double *hssoa, unsigned capacity, unsigned *n_points)
{
    if (!p || !path || !hssoa || !n_points) return ICY_ERR_INVALID_ARGUMENT;
    try {
        icy::h5::File f(path);
        const auto d = f.dims("llGrainIDs");
        if (d.size() != 1) { g_host_error = "llGrainIDs is not one-dimensional"; return ICY_ERR_FILE; }
        const unsigned n = (unsigned)d[0];
        if (n > capacity) { g_host_error = "point cloud larger than the HSSOA capacity"; return ICY_ERR_CAPACITY; }
        const auto x = f.read_double("x"), y = f.read_double("y");
        const auto g = f.read_uint64("llGrainIDs");
        if (x.size() != n || y.size() != n) { g_host_error = "x, y and llGrainIDs differ in length"; return ICY_ERR_FILE; }
        for (int l = 0; l < ICY_N_PTS_ARRAYS; l++) std::memset(hssoa + (size_t)l * capacity, 0, sizeof(double) * n);
        std::memcpy(hssoa, g.data(), sizeof(uint64_t) * n);
        std::memcpy(hssoa + (size_t)ICY_POSX * capacity, x.data(), sizeof(double) * n);
        std::memcpy(hssoa + (size_t)(ICY_POSX + 1) * capacity, y.data(), sizeof(double) * n);
        const float volume = (float)f.attribute_double("llGrainIDs", "volume");
        unsigned kept = n;
        const int rc = icy_scene_place(p, hssoa, capacity, &kept, (double)volume);
        if (rc != ICY_OK) { g_host_error = "icy_scene_place failed"; return rc; }
        *n_points = kept;
        return ICY_OK;
    } catch (const std::exception &e) {
        return failed(ICY_ERR_FILE, e);
    }
}

int icy_format_double(double v, char *buf, size_t cap)
{
    if (!buf || cap == 0) return ICY_ERR_INVALID_ARGUMENT;
    const std::string s = icy::format_double(v);
    if (s.size() + 1 > cap) return ICY_ERR_CAPACITY;
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return ICY_OK;
}

}  // extern "C"
