// instance.cuh -- device state of one simulation instance (one domain, one GPU).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/icempm.h"
#include "mpm_math.cuh"

struct icy_mpm {
    int device = 0;
    int precision = ICY_PRECISION_FP64;
    icy_sim_params prm{};
    cudaStream_t stream = nullptr, own_stream = nullptr;

    // particles: 16 lines of `pitch` doubles (HSSOA line order)
    unsigned capacity = 0, n = 0;
    long pitch = 0;
    double *d_pts = nullptr;

    // grid: nodes gx in [-halo, GridX+halo), gy in [0, GridY), column gx+halo,
    // five arrays of n_nodes doubles: m, px, py (accumulated), vx, vy (updated)
    long n_nodes = 0;
    double *d_grid = nullptr;

    // binning by tile (tiled path): second particle buffer for the permutation,
    // upload index of every slot, sort scratch, tile ranges, node-tile marks
    double *d_pts_alt = nullptr;
    int *d_oidx = nullptr, *d_oidx_alt = nullptr, *d_keys = nullptr, *d_ranks = nullptr;
    int *d_counts = nullptr, *d_start = nullptr, *d_active = nullptr, *d_nactive = nullptr;
    int *d_block_sums = nullptr;

    // FP32 split-precision state (precision == ICY_PRECISION_FP32_SPLIT):
    // 17 words per point in 32-point blocks (kernels_split.cuh), an FP32 grid,
    // FP64 staging for the HSSOA conversion
    unsigned *d_st = nullptr, *d_st_alt = nullptr;
    double *d_stage = nullptr;
    long stage_n = 0;
    float *d_gridf = nullptr;       // m, px, py, then two velocity buffers (vx, vy each)
    int vpar = 0;                   // which velocity buffer G2P reads (the update writes the other)
    int *d_nexp = nullptr, *d_ncnt = nullptr;   // fused grid update: per node tile expected / finished
    int *d_unsafe = nullptr;        // [2] margin flags of the last launches, by parity
    int fuse_seq = 0;               // fused-capable launches since the last binning
    bool fuse_update = false;       // grid update fused into the tile kernel where safe (option "fuse_update")
    int shape = 0;                  // FP32 tile shape (option "tile_shape", kernels_split.cuh SHAPE_*)
    void *d_grainf = nullptr;
    int tile_grid_f32 = 0;
    icy_dev::GrainConst *d_grain = nullptr;   // failure-surface constants per grain slot
    int scan_blocks = 0;
    unsigned *d_flags = nullptr;
    int2 *d_tlist = nullptr;        // node tiles written since the last grid update (once each)
    unsigned *d_tlist_n = nullptr;  // [0] entries, [1] CTAs of the update done
    unsigned long long *d_moved = nullptr;
    int ntx = 0, nty = 0, ntiles = 0;
    int tile_grid = 0, update_grid = 0, pipe_grid = 0, update_grid_f32 = 0;
    bool binned = false;        // points sorted by tile since the last upload
    bool permuted = false;      // device order differs from upload order
    bool primed = false;        // accumulators hold P2G of the current state
    int steps_since_bin = 0;
    int resort_every = 64;      // re-bin interval in steps (0 = never)
    bool tiled = true;          // tiled kernels (false: one-thread-per-item kernels)
    bool pipe = false;          // fused step fed by the bulk-copy producer warp
    bool pipe_fault_test = false;   // pipe kernel leaves its first stage unfilled (timeout test)

    double *d_acc = nullptr;      // indenter force bins, 2*n_indenter_subdivisions
    int *d_status = nullptr;      // device error code (reference codes 70..73, 5)
    int *h_status = nullptr;      // pinned host mirror

    int64_t launches = 0;

    // per-kernel event profiling (icy_mpm_profile)
    struct ProfRec { int kernel; cudaEvent_t a, b; };
    bool profiling = false;
    int prof_every = 1;                // time every prof_every-th launch of each kernel
    bool prof_cur = false;             // the open launch is timed
    std::vector<int64_t> prof_seen;    // launches of each kernel since profiling started
    std::vector<ProfRec> prof_recs;
    std::vector<cudaEvent_t> event_pool;
    std::vector<double> prof_ms;
    std::vector<int64_t> prof_n;
};

// kernel ids for profiling
enum IcyKernel {
    K_P2G_SIMPLE = 0, K_UPDATE_SIMPLE, K_G2P_SIMPLE, K_MEMSET_GRID,
    K_BIN, K_TILE_G2P2G, K_TILE_P2G, K_TILE_G2P, K_UPDATE_TILES, K_UNPERMUTE,
    K_N_KERNELS
};
extern const char *const icy_kernel_names[K_N_KERNELS];
void icy_prof_begin(icy_mpm *h, int kernel);
void icy_prof_end(icy_mpm *h);
int icy_prof_resolve(icy_mpm *h);
void icy_prof_free(icy_mpm *h);

icy_dev::StepParams icy_step_params(const icy_sim_params &p);
void icy_set_error(const char *where, cudaError_t e);
void icy_set_error_msg(const std::string &m);

// Allocates and clears an instance's device memory.  With work_stream, the
// allocations and clearing are queued there and the call returns without
// waiting for them (work_stream becomes the instance's stream); otherwise on
// the instance's own stream, waited for.
int icy_instance_allocate(icy_mpm *h, unsigned capacity, cudaStream_t work_stream = nullptr);
// icy_mpm_create with the allocation work queued on `stream` (not waited for;
// nullptr: the instance's own stream, waited for)
int icy_mpm_create_on(const icy_sim_params *p, int device, unsigned capacity, int precision, cudaStream_t stream,
                      icy_mpm **out);
// trim: give unused pool memory back; wait = false: the memory is freed in
// the order of h->stream only (the caller knows that nothing on another stream
// still uses it)
void icy_instance_free(icy_mpm *h, bool trim = false, bool wait = true);
// Grows the device's instance memory pool to hold at least `bytes` (kept).
int icy_instance_pool_reserve(int device, size_t bytes);
int icy_instance_upload(icy_mpm *h, const double *hssoa, unsigned cap, unsigned size);
int icy_instance_download(icy_mpm *h, double *hssoa, unsigned cap);
int icy_phase_reset_grid(icy_mpm *h);
int icy_phase_p2g(icy_mpm *h);
int icy_phase_update(icy_mpm *h, double ind_x, double ind_y);
int icy_phase_g2p(icy_mpm *h, bool recordPQ);
int icy_instance_steps(icy_mpm *h, int step0, int nsteps, double *sim_time);
int icy_instance_bin(icy_mpm *h);
int icy_instance_constants(icy_mpm *h);
int icy_instance_set_shape(icy_mpm *h, int shape);
