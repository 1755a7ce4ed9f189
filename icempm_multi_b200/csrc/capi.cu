// capi.cu -- the C-ABI of include/icempm.h: one simulation instance
// (one partition, one GPU) and its per-phase and multi-step entry points.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/icempm.h"
#include "instance.cuh"

namespace {
thread_local std::string g_last_error;
}

void icy_set_error(const char *where, cudaError_t e)
{
    char buf[512];
    std::snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
    g_last_error = buf;
}
void icy_set_error_msg(const std::string &m) { g_last_error = m; }

#define CK(call)                                                  \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) { icy_set_error(#call, e_); return ICY_ERR_CUDA; } \
    } while (0)

using namespace icy_dev;

StepParams icy_step_params(const icy_sim_params &p)
{
    StepParams s;
    s.h = p.cellsize; s.hinv = p.cellsize_inv; s.dt = p.InitialTimeStep;
    s.dt_vol_Dpinv = p.dt_vol_Dpinv; s.dt_gravity = p.dt_Gravity;
    s.vmax = p.vmax; s.vmax_sq = p.vmax_squared; s.ind_rsq = p.IndRSq; s.ind_v = p.IndVelocity;
    s.mass_ice = p.ParticleMass; s.mass_water = p.WaterParticleMass;
    s.mu = p.mu; s.kappa = p.kappa; s.tan_phi = p.DP_tan_phi; s.dp_p = p.DP_threshold_p;
    s.pmax = p.IceCompressiveStrength; s.pmin_t = p.IceTensileStrength; s.qmax_s = p.IceShearStrength;
    s.t2 = p.IceTensileStrength2; s.beta = p.NACC_beta; s.grain_var = p.GrainVariability;
    s.gridx = p.GridXTotal; s.gridy = p.GridY; s.halo = p.GridHaloSize; s.nsub = p.n_indenter_subdivisions;
    return s;
}

static int set_device(icy_mpm *h)
{
    CK(cudaSetDevice(h->device));
    return ICY_OK;
}

extern "C" {

const char *icy_version(void) { return "icempm_b200 sm_100a"; }

int icy_host_alloc(size_t bytes, void **ptr)
{
    if (!ptr || bytes == 0) return ICY_ERR_INVALID_ARGUMENT;
    *ptr = nullptr;
    cudaError_t e = cudaMallocHost(ptr, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        icy_set_error("cudaMallocHost", e);
        *ptr = nullptr;
        return ICY_ERR_OUT_OF_MEMORY;
    }
    std::memset(*ptr, 0, bytes);
    return ICY_OK;
}

int icy_host_free(void *ptr)
{
    if (ptr) CK(cudaFreeHost(ptr));
    return ICY_OK;
}
const char *icy_last_error(void) { return g_last_error.c_str(); }

int icy_mpm_create(const icy_sim_params *p, int device, unsigned capacity, int precision, icy_mpm **out)
{
    return icy_mpm_create_on(p, device, capacity, precision, nullptr, out);
}
}  // extern "C"

int icy_mpm_create_on(const icy_sim_params *p, int device, unsigned capacity, int precision, cudaStream_t stream,
                      icy_mpm **out)
{
    if (!p || !out || capacity == 0) return ICY_ERR_INVALID_ARGUMENT;
    if (precision != ICY_PRECISION_FP64 && precision != ICY_PRECISION_FP32_SPLIT) return ICY_ERR_INVALID_ARGUMENT;
    if (p->GridXTotal < 4 || p->GridY < 4 || p->GridHaloSize < 0 || p->n_indenter_subdivisions < 1)
        return ICY_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    icy_mpm *h = new icy_mpm();
    h->device = device;
    h->prm = *p;
    h->precision = precision;
    int rc = icy_instance_allocate(h, capacity, stream);
    if (rc != ICY_OK) {
        icy_instance_free(h, rc == ICY_ERR_OUT_OF_MEMORY);
        delete h;
        return rc;
    }
    *out = h;
    return ICY_OK;
}

extern "C" {

int icy_mpm_destroy(icy_mpm *h)
{
    if (!h) return ICY_OK;
    cudaSetDevice(h->device);
    icy_instance_free(h);
    delete h;
    return ICY_OK;
}

int icy_mpm_set_stream(icy_mpm *h, void *stream)
{
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    h->stream = stream ? (cudaStream_t)stream : h->own_stream;
    return ICY_OK;
}

void *icy_mpm_get_stream(icy_mpm *h) { return h ? (void *)h->stream : nullptr; }

int icy_mpm_update_constants(icy_mpm *h, const icy_sim_params *p)
{
    if (!h || !p) return ICY_ERR_INVALID_ARGUMENT;
    if (p->GridXTotal != h->prm.GridXTotal || p->GridY != h->prm.GridY || p->GridHaloSize != h->prm.GridHaloSize ||
        p->n_indenter_subdivisions != h->prm.n_indenter_subdivisions)
        return ICY_ERR_INVALID_ARGUMENT;  // grid shape is fixed at creation
    if (set_device(h)) return ICY_ERR_CUDA;
    h->prm = *p;
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream));
    return icy_instance_constants(h);
}

int icy_mpm_transfer_points_to_device(icy_mpm *h, const double *hssoa, unsigned capacity, unsigned size)
{
    if (!h || !hssoa || size > capacity) return ICY_ERR_INVALID_ARGUMENT;
    if (size > h->capacity) return ICY_ERR_NO_SPACE;
    if (set_device(h)) return ICY_ERR_CUDA;
    return icy_instance_upload(h, hssoa, capacity, size);
}

int icy_mpm_transfer_from_device(icy_mpm *h, double *hssoa, unsigned capacity, unsigned *size,
                                 double *bins)
{
    if (!h || !hssoa) return ICY_ERR_INVALID_ARGUMENT;
    if (h->n > capacity) return ICY_ERR_CAPACITY;
    if (set_device(h)) return ICY_ERR_CUDA;
    int rc = icy_instance_download(h, hssoa, capacity);
    if (rc) return rc;
    if (bins)
        CK(cudaMemcpyAsync(bins, h->d_acc, sizeof(double) * 2 * h->prm.n_indenter_subdivisions,
                           cudaMemcpyDeviceToHost, h->stream));
    int code = 0;
    CK(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    code = *h->h_status;
    if (size) *size = h->n;
    if (code) return code;
    // active point count (simulation/gpu_implementation5.cpp:399-433)
    long active = 0;
    for (unsigned i = 0; i < h->n; i++) {
        long long u;
        std::memcpy(&u, hssoa + i, 8);
        if (!(u & ICY_STATUS_DISABLED)) active++;
    }
    if (active != h->prm.nPtsTotal) {
        icy_set_error_msg("transfer_from_device(): active point count mismatch");
        return ICY_ERR_POINT_COUNT;
    }
    return ICY_OK;
}

int icy_mpm_reset_indenter_force_accumulator(icy_mpm *h)
{
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    if (set_device(h)) return ICY_ERR_CUDA;
    CK(cudaMemsetAsync(h->d_acc, 0, sizeof(double) * 2 * h->prm.n_indenter_subdivisions, h->stream));
    return ICY_OK;
}

int icy_mpm_indenter_force(icy_mpm *h, double *force_xy, double *bins)
{
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    if (set_device(h)) return ICY_ERR_CUDA;
    const int nb = 2 * h->prm.n_indenter_subdivisions;
    std::vector<double> b(nb);
    CK(cudaMemcpyAsync(b.data(), h->d_acc, sizeof(double) * nb, cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (bins) std::memcpy(bins, b.data(), sizeof(double) * nb);
    if (force_xy) {
        // GPU_Implementation5::transfer_from_device sums the bins (gpu_implementation5.cpp:392-396)
        double fx = 0, fy = 0;
        for (int j = 0; j < nb / 2; j++) { fx += b[2 * j]; fy += b[2 * j + 1]; }
        force_xy[0] = fx;
        force_xy[1] = fy;
    }
    return ICY_OK;
}

int icy_mpm_reset_grid(icy_mpm *h)
{
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    if (set_device(h)) return ICY_ERR_CUDA;
    return icy_phase_reset_grid(h);
}

int icy_mpm_p2g(icy_mpm *h)
{
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    if (set_device(h)) return ICY_ERR_CUDA;
    return icy_phase_p2g(h);
}

int icy_mpm_receive_halos(icy_mpm *h) { return h ? ICY_OK : ICY_ERR_INVALID_ARGUMENT; }
int icy_mpm_receive_points(icy_mpm *h) { return h ? ICY_OK : ICY_ERR_INVALID_ARGUMENT; }

int icy_mpm_update_nodes(icy_mpm *h, double ind_x, double ind_y, double simulation_time)
{
    (void)simulation_time;  // unused by the reference kernel outside commented-out code
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    if (set_device(h)) return ICY_ERR_CUDA;
    return icy_phase_update(h, ind_x, ind_y);
}

int icy_mpm_g2p(icy_mpm *h, int recordPQ, int enablePointTransfer)
{
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    if (enablePointTransfer) return ICY_ERR_NOT_SUPPORTED;  // one domain: nothing to transfer
    if (set_device(h)) return ICY_ERR_CUDA;
    return icy_phase_g2p(h, recordPQ != 0);
}

int icy_mpm_step(icy_mpm *h, int step0, int nsteps, double *sim_time)
{
    if (!h || !sim_time || nsteps < 0) return ICY_ERR_INVALID_ARGUMENT;
    if (h->prm.UpdateEveryNthStep <= 0) return ICY_ERR_INVALID_ARGUMENT;
    if (set_device(h)) return ICY_ERR_CUDA;
    return icy_instance_steps(h, step0, nsteps, sim_time);
}

int icy_mpm_synchronize(icy_mpm *h)
{
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    if (set_device(h)) return ICY_ERR_CUDA;
    CK(cudaStreamSynchronize(h->stream));
    return ICY_OK;
}

int icy_mpm_status(icy_mpm *h)
{
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    if (set_device(h)) return ICY_ERR_CUDA;
    CK(cudaMemcpyAsync(h->h_status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return *h->h_status;
}

int64_t icy_mpm_kernel_launches(icy_mpm *h) { return h ? h->launches : 0; }

int icy_mpm_counters(icy_mpm *h, int64_t *moved_points, int64_t *fused_launches, int64_t *fallback_launches)
{
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    unsigned long long c[3] = {0, 0, 0};
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(c, h->d_moved, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    if (moved_points) *moved_points = (int64_t)c[0];
    if (fused_launches) *fused_launches = (int64_t)c[1];
    if (fallback_launches) *fallback_launches = (int64_t)c[2];
    return ICY_OK;
}

int icy_mpm_set_option(icy_mpm *h, const char *name, double value)
{
    if (!h || !name) return ICY_ERR_INVALID_ARGUMENT;
    const std::string k(name);
    if (k == "resort_every") {
        if (value < 0) return ICY_ERR_INVALID_ARGUMENT;
        h->resort_every = (int)value;
    } else if (k == "profile_every") {
        if (value < 1 || value > (1 << 20)) return ICY_ERR_INVALID_ARGUMENT;
        h->prof_every = (int)value;
    } else if (k == "pipe") {
        h->pipe = value != 0;
    } else if (k == "pipe_fault_test") {
        h->pipe_fault_test = value != 0;
    } else if (k == "tiled") {
        h->tiled = value != 0;
        h->primed = false;
    } else if (k == "fuse_update") {
        h->fuse_update = value != 0;
    } else if (k == "tile_shape") {
        return icy_instance_set_shape(h, (int)value);
    } else {
        return ICY_ERR_INVALID_ARGUMENT;
    }
    return ICY_OK;
}

}  // extern "C"

// ---------------------------------------------------------------- profiling
const char *const icy_kernel_names[K_N_KERNELS] = {
    "k_p2g_simple", "k_update_simple", "k_g2p_simple", "memset_grid",
    "bin_sort", "k_tile_g2p2g", "k_tile_p2g", "k_tile_g2p", "k_update_nodes", "k_unpermute",
};

static cudaEvent_t pool_get(icy_mpm *h)
{
    if (h->event_pool.empty()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        return e;
    }
    cudaEvent_t e = h->event_pool.back();
    h->event_pool.pop_back();
    return e;
}

void icy_prof_begin(icy_mpm *h, int kernel)
{
    h->prof_cur = false;
    if (!h->profiling) return;
    if (h->prof_seen.size() != K_N_KERNELS) h->prof_seen.assign(K_N_KERNELS, 0);
    // every re-binning is timed (it is rare, and its share of a step is amortised
    // from its own time); other kernels every prof_every-th launch
    if (h->prof_seen[kernel]++ % h->prof_every != 0 && kernel != K_BIN) return;   // not a sampled launch
    icy_mpm::ProfRec r{kernel, pool_get(h), pool_get(h)};
    if (!r.a || !r.b) return;
    cudaEventRecord(r.a, h->stream);
    h->prof_recs.push_back(r);
    h->prof_cur = true;
}

void icy_prof_end(icy_mpm *h)
{
    if (!h->profiling || !h->prof_cur || h->prof_recs.empty()) return;
    cudaEventRecord(h->prof_recs.back().b, h->stream);
    h->prof_cur = false;
}

int icy_prof_resolve(icy_mpm *h)
{
    if (h->prof_recs.empty()) return ICY_OK;
    CK(cudaStreamSynchronize(h->stream));
    if (h->prof_ms.size() != K_N_KERNELS) { h->prof_ms.assign(K_N_KERNELS, 0.0); h->prof_n.assign(K_N_KERNELS, 0); }
    for (auto &r : h->prof_recs) {
        float ms = 0;
        if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
            h->prof_ms[r.kernel] += ms;
            h->prof_n[r.kernel] += 1;
        }
        h->event_pool.push_back(r.a);
        h->event_pool.push_back(r.b);
    }
    h->prof_recs.clear();
    return ICY_OK;
}

void icy_prof_free(icy_mpm *h)
{
    for (auto &r : h->prof_recs) { h->event_pool.push_back(r.a); h->event_pool.push_back(r.b); }
    h->prof_recs.clear();
    for (auto e : h->event_pool) cudaEventDestroy(e);
    h->event_pool.clear();
}

extern "C" {

int icy_mpm_profile(icy_mpm *h, int enable)
{
    if (!h) return ICY_ERR_INVALID_ARGUMENT;
    if (set_device(h)) return ICY_ERR_CUDA;
    if (enable) {
        int rc = icy_prof_resolve(h);
        if (rc) return rc;
        h->prof_ms.assign(K_N_KERNELS, 0.0);
        h->prof_n.assign(K_N_KERNELS, 0);
        h->prof_seen.assign(K_N_KERNELS, 0);
    }
    h->profiling = enable != 0;
    return ICY_OK;
}

int icy_mpm_profile_read(icy_mpm *h, int max, char *names, double *ms_total, int64_t *launches, int *count)
{
    if (!h || max < 0) return ICY_ERR_INVALID_ARGUMENT;
    if (set_device(h)) return ICY_ERR_CUDA;
    int rc = icy_prof_resolve(h);
    if (rc) return rc;
    int c = 0;
    for (int k = 0; k < (int)h->prof_n.size(); k++) {
        if (h->prof_n[k] == 0) continue;
        if (c < max) {
            if (names) { std::strncpy(names + 48 * c, icy_kernel_names[k], 47); names[48 * c + 47] = 0; }
            if (ms_total) ms_total[c] = h->prof_ms[k];
            if (launches) launches[c] = h->prof_n[k];
        }
        c++;
    }
    if (count) *count = c;
    return ICY_OK;
}

}  // extern "C"
