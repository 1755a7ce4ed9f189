// noalloc.cu -- icy_step_noalloc: the step loop on point data the caller keeps
// in device memory, for callers that cannot allocate device memory.
//
// Who needs it: applications whose device memory is owned by someone else --
// a host framework with its own pooling allocator that forbids cudaMalloc /
// cudaFree from plug-ins (both can synchronise the device and fragment the
// pool), code on a latency-critical path that must not allocate after start-up,
// or a process that has handed nearly all device memory to another component.
// Such a caller passes its particle buffer in; this entry point allocates
// nothing: the grid and the status word it needs live in one file-scope
// __device__ array of fixed size, which every GPU that loads the library holds
// until the process exits.
//
// The array is shared by all calls and keeps the last call's contents; each
// call clears the parts that must start at zero.  Calls that overlap on the
// GPU (on different streams, or from different host threads) race on it.
#include <cuda_runtime.h>

#include <climits>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/icempm.h"
#include "mpm_math.cuh"

using icy_dev::StepParams;

StepParams icy_step_params(const icy_sim_params &p);
void icy_set_error(const char *where, cudaError_t e);
void icy_set_error_msg(const std::string &m);
cudaError_t icy_launch_p2g_simple(cudaStream_t s, const StepParams &P, const double *pts, long pitch, int n,
                                  double *grid, long n_nodes, int *status);
cudaError_t icy_launch_update_simple(cudaStream_t s, const StepParams &P, double *grid, long n_nodes, double ind_x,
                                     double ind_y, double *acc);
cudaError_t icy_launch_g2p_simple(cudaStream_t s, const StepParams &P, double *pts, long pitch, int n, double *grid,
                                  long n_nodes, int recordPQ, int *status);

namespace {

constexpr size_t kScratchBytes = ICY_NOALLOC_SCRATCH_BYTES;
static_assert(kScratchBytes % 256 == 0, "scratch size");

// The scratch: [grid: 5 x n_nodes doubles][status: 256 B][indenter bins when
// the caller passes none].  In host code this name is a host-side stand-in,
// not a device address; the address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
struct Resolved { void *ctx; void *addr; };
Resolved g_scratch[kMaxDevices] = {};

// The driver's cuCtxGetCurrent, through the runtime's entry-point query (the
// library does not link the driver library itself).
typedef int (*CtxGetCurrentFn)(void **);
CtxGetCurrentFn ctx_get_current()
{
    static CtxGetCurrentFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    return fn;
}

// Device address of the scratch array on the current device, resolved with
// that device current at the first call, and again whenever the device's
// context has changed since (after cudaDeviceReset the module, and with it
// the array, is loaded anew and may sit at another address).
int scratch_address(int device, unsigned char **out)
{
    if (device < 0 || device >= kMaxDevices) return ICY_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(g_mutex);
    void *ctx = nullptr;
    if (CtxGetCurrentFn f = ctx_get_current()) f(&ctx);
    Resolved &r = g_scratch[device];
    if (!r.addr || r.ctx != ctx) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            icy_set_error("cudaGetSymbolAddress(g_noalloc_scratch)", e);
            return ICY_ERR_CUDA;
        }
        if (!ctx && ctx_get_current()) ctx_get_current()(&ctx);   // the call above made the context current
        r.addr = p;
        r.ctx = ctx;
    }
    *out = static_cast<unsigned char *>(r.addr);
    return ICY_OK;
}

#define CKN(call)                                                                 \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) { icy_set_error(#call, e_); return ICY_ERR_CUDA; } \
    } while (0)

}  // namespace

extern "C" int icy_step_noalloc(const icy_sim_params *p, double *d_hssoa, unsigned pitch, unsigned n, int step0,
                                int nsteps, double *sim_time, double *d_indenter_bins, void *stream)
{
    if (!p || !sim_time || nsteps < 0 || (n > 0 && !d_hssoa) || pitch < n || n > (unsigned)INT_MAX)
        return ICY_ERR_INVALID_ARGUMENT;
    if (p->UpdateEveryNthStep <= 0 || p->GridXTotal < 4 || p->GridY < 4 || p->GridHaloSize < 0 ||
        p->n_indenter_subdivisions < 1)
        return ICY_ERR_INVALID_ARGUMENT;
    const long n_nodes = (long)p->GridY * (p->GridXTotal + 2 * p->GridHaloSize);
    const size_t grid_bytes = sizeof(double) * 5 * (size_t)n_nodes;
    const size_t status_off = (grid_bytes + 255) / 256 * 256;
    const size_t bins_off = status_off + 256;
    const size_t need = bins_off + (d_indenter_bins ? 0 : sizeof(double) * 2 * p->n_indenter_subdivisions);
    if (need > kScratchBytes) {
        char msg[256];
        std::snprintf(msg, sizeof(msg),
                      "icy_step_noalloc: grid of %ld nodes needs %zu bytes of scratch, limit %zu bytes", n_nodes, need,
                      kScratchBytes);
        icy_set_error_msg(msg);
        return ICY_ERR_CAPACITY;
    }
    int device = 0;
    CKN(cudaGetDevice(&device));
    unsigned char *base = nullptr;
    if (int rc = scratch_address(device, &base)) return rc;
    double *grid = reinterpret_cast<double *>(base);
    int *status = reinterpret_cast<int *>(base + status_off);
    double *bins = d_indenter_bins ? d_indenter_bins : reinterpret_cast<double *>(base + bins_off);
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // what must start at zero: the status word, the velocity arrays (read by
    // G2P only where this call's P2G put mass, but cleared so nothing from an
    // earlier call can leak in) and our own bin copy; the accumulators are
    // cleared before every sub-step
    CKN(cudaMemsetAsync(status, 0, sizeof(int), s));
    CKN(cudaMemsetAsync(grid + 3 * n_nodes, 0, sizeof(double) * 2 * n_nodes, s));
    if (!d_indenter_bins) CKN(cudaMemsetAsync(bins, 0, sizeof(double) * 2 * p->n_indenter_subdivisions, s));

    const StepParams P = icy_step_params(*p);
    double t = *sim_time;
    double t_done = t;   // time of the last sub-step whose G2P was queued
    cudaError_t e = cudaSuccess;
    const char *where = nullptr;
    for (int k = 0; k < nsteps; k++) {
        // icy::Model::Step sub-step (simulation/model.cpp:40-49)
        t += p->InitialTimeStep;
        const double ind_x = p->indenter_x_initial + t * p->IndVelocity;
        const int rec = ((step0 + k) % p->UpdateEveryNthStep) == 0;
        if ((e = cudaMemsetAsync(grid, 0, sizeof(double) * 3 * n_nodes, s)) != cudaSuccess) where = "cudaMemsetAsync(grid)";
        else if ((e = icy_launch_p2g_simple(s, P, d_hssoa, (long)pitch, (int)n, grid, n_nodes, status)) != cudaSuccess)
            where = "icy_launch_p2g_simple";
        else if ((e = icy_launch_update_simple(s, P, grid, n_nodes, ind_x, p->indenter_y, bins)) != cudaSuccess)
            where = "icy_launch_update_simple";
        else if ((e = icy_launch_g2p_simple(s, P, d_hssoa, (long)pitch, (int)n, grid, n_nodes, rec, status)) !=
                 cudaSuccess)
            where = "icy_launch_g2p_simple";
        if (where) break;
        t_done = t;
    }
    if (where) {
        // the sub-steps queued before the failure still run: wait for them, so
        // that d_hssoa is no longer changing, and report how far it advanced
        icy_set_error(where, e);
        cudaStreamSynchronize(s);
        *sim_time = t_done;
        return ICY_ERR_CUDA;
    }
    int code = 0;
    CKN(cudaMemcpyAsync(&code, status, sizeof(int), cudaMemcpyDeviceToHost, s));
    CKN(cudaStreamSynchronize(s));
    *sim_time = t;
    return code;
}
