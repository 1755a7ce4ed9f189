// instance.cu -- allocation, host<->device transfer, binning and the step loop
// of one simulation instance.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <vector>

#include "instance.cuh"
#include "kernels_split.cuh"

using namespace icy_dev;

#define CK(call)                                                                  \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) { icy_set_error(#call, e_); return ICY_ERR_CUDA; } \
    } while (0)
#define CK_LAUNCH(where)                                                          \
    do {                                                                          \
        cudaError_t e_ = cudaGetLastError();                                      \
        if (e_ != cudaSuccess) { icy_set_error(where, e_); return ICY_ERR_CUDA; } \
        h->launches++;                                                            \
    } while (0)

static GridView grid_view(icy_mpm *h)
{
    GridView g;
    g.m = h->d_grid;
    g.px = h->d_grid + h->n_nodes;
    g.py = h->d_grid + 2 * h->n_nodes;
    g.vx = h->d_grid + 3 * h->n_nodes;
    g.vy = h->d_grid + 4 * h->n_nodes;
    g.ny = h->prm.GridY;
    g.halo = h->prm.GridHaloSize;
    return g;
}

static TileGeom tile_geom(icy_mpm *h) { return TileGeom{h->ntx, h->nty, h->ntiles}; }

// Device memory of instances comes from one stream-ordered pool per device
// that keeps freed blocks for reuse (release threshold: never), so that
// creating and destroying instances -- as the serving loop does all the
// time -- neither synchronises the device nor goes back to the driver.
static cudaMemPool_t instance_pool(int device)
{
    static std::mutex m;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> g(m);
    auto it = pools.find(device);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) return nullptr;
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    pools[device] = pool;
    return pool;
}

int icy_instance_pool_reserve(int device, size_t bytes)
{
    CK(cudaSetDevice(device));
    cudaMemPool_t pool = instance_pool(device);
    if (!pool) return ICY_ERR_OUT_OF_MEMORY;
    size_t have = 0;
    CK(cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &have));
    if (have >= bytes) return ICY_OK;
    cudaStream_t s;
    CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    void *p = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(&p, bytes - have, pool, s);
    if (e == cudaSuccess) e = cudaFreeAsync(p, s);   // kept by the pool (release threshold: never)
    const cudaError_t e2 = cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    if (e != cudaSuccess || e2 != cudaSuccess) {
        icy_set_error("icy_mpm_reserve", e != cudaSuccess ? e : e2);
        return e == cudaErrorMemoryAllocation ? ICY_ERR_OUT_OF_MEMORY : ICY_ERR_CUDA;
    }
    return ICY_OK;
}

template <typename T>
static cudaError_t dalloc(icy_mpm *h, T **p, size_t count)
{
    cudaMemPool_t pool = instance_pool(h->device);
    if (!pool) return cudaErrorMemoryAllocation;
    return cudaMallocFromPoolAsync((void **)p, sizeof(T) * std::max<size_t>(count, 1), pool, h->stream);
}

// One pinned int per instance for reading the device status back, from a
// process-wide page-locked block (pinning four bytes costs as much as pinning
// megabytes, and instances come and go).
static std::mutex g_slot_mutex;
static std::vector<int *> g_free_slots;

static int *status_slot_get()
{
    std::lock_guard<std::mutex> g(g_slot_mutex);
    if (g_free_slots.empty()) {
        int *block = nullptr;
        if (cudaMallocHost(&block, sizeof(int) * 1024) != cudaSuccess) return nullptr;
        for (int k = 1023; k >= 0; k--) g_free_slots.push_back(block + k);
    }
    int *s = g_free_slots.back();
    g_free_slots.pop_back();
    return s;
}

static void status_slot_put(int *s)
{
    if (!s) return;
    std::lock_guard<std::mutex> g(g_slot_mutex);
    g_free_slots.push_back(s);
}

// tile dimensions of the instance: FP32 instances take their shape, FP64 32 x 8
static void tile_dims(const icy_mpm *h, int &tx, int &ty)
{
    tx = TX;
    ty = TY;
    if (h->precision == ICY_PRECISION_FP32_SPLIT)
        with_shape(h->shape, [&](auto sh) {
            tx = decltype(sh)::TX;
            ty = decltype(sh)::TY;
        });
}

// The arrays whose size depends on the tile shape (cell ranges, sort counts,
// tile lists and marks) and the launch sizes of the tile kernels.
static int alloc_tiles(icy_mpm *h)
{
    int tx, ty;
    tile_dims(h, tx, ty);
    const int nx = h->prm.GridXTotal + 2 * h->prm.GridHaloSize;
    h->ntx = (nx + tx - 1) / tx;
    h->nty = (h->prm.GridY + ty - 1) / ty;
    h->ntiles = h->ntx * h->nty;
    const long nkeys = (long)h->ntiles * tx * ty + 1;   // cells + the disabled / out-of-grid bucket
    h->scan_blocks = (int)((nkeys + SCAN_BLOCK - 1) / SCAN_BLOCK);
    CK(dalloc(h, &h->d_counts, nkeys));
    CK(dalloc(h, &h->d_start, nkeys + 1));
    CK(dalloc(h, &h->d_block_sums, h->scan_blocks));
    CK(dalloc(h, &h->d_active, h->ntiles));
    CK(dalloc(h, &h->d_flags, h->ntiles));
    CK(dalloc(h, &h->d_tlist, h->ntiles));
    CK(dalloc(h, &h->d_nexp, h->ntiles));
    CK(dalloc(h, &h->d_ncnt, h->ntiles));
    CK(cudaMemsetAsync(h->d_flags, 0, sizeof(unsigned) * h->ntiles, h->stream));
    CK(cudaMemsetAsync(h->d_nexp, 0, sizeof(int) * h->ntiles, h->stream));
    CK(cudaMemsetAsync(h->d_ncnt, 0, sizeof(int) * h->ntiles, h->stream));
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    h->update_grid = (int)std::max(1L, std::min((long)(h->ntiles + 1) / 2, (long)sms * 8));
    if (h->precision == ICY_PRECISION_FP32_SPLIT) {
        cudaError_t e = cudaSuccess;
        with_shape(h->shape, [&](auto sh) {
            using S = decltype(sh);
            int per_sm = 0;
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_tile_f32<true, true, false, false, false, S>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MOMF_BYTES);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_tile_f32<false, true, false, false, false, S>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MOMF_BYTES);
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile_f32<true, true, false, false, false, S>,
                                                                  TILE_THREADS_F32, MOMF_BYTES);
            h->tile_grid_f32 = std::max(1, sms * std::max(per_sm, 1));
            per_sm = 0;
            if (e == cudaSuccess)
                e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_update_tiles_f32<S>, S::TT, 0);
            h->update_grid_f32 = (int)std::max(1L, std::min((long)h->ntiles, (long)sms * std::max(per_sm, 1)));
        });
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_tile_f32<true, true, false, false, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MOMF_BYTES);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(k_tile_f32<false, true, false, false, true>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MOMF_BYTES);
        CK(e);
    }
    return ICY_OK;
}

static void free_tiles(icy_mpm *h)
{
    void *ptrs[] = {h->d_counts, h->d_start, h->d_block_sums, h->d_active, h->d_flags, h->d_tlist, h->d_nexp,
                    h->d_ncnt};
    for (void *p : ptrs)
        if (p) cudaFreeAsync(p, h->stream);
    h->d_counts = h->d_start = h->d_block_sums = h->d_active = nullptr;
    h->d_flags = nullptr;
    h->d_tlist = nullptr;
    h->d_nexp = h->d_ncnt = nullptr;
}

// FP32 tile shape of an instance (option "tile_shape"): the shape-dependent
// arrays are made anew and the points binned again at the next step.
int icy_instance_set_shape(icy_mpm *h, int shape)
{
    if (shape < 0 || shape >= N_SHAPES) return ICY_ERR_INVALID_ARGUMENT;
    if (h->precision != ICY_PRECISION_FP32_SPLIT || shape == h->shape) {
        if (h->precision != ICY_PRECISION_FP32_SPLIT && shape != SHAPE_32X8) return ICY_ERR_NOT_SUPPORTED;
        return ICY_OK;
    }
    CK(cudaSetDevice(h->device));
    free_tiles(h);
    h->shape = shape;
    if (int rc = alloc_tiles(h)) return rc;
    CK(cudaMemsetAsync(h->d_tlist_n, 0, sizeof(unsigned) * 2, h->stream));
    CK(cudaMemsetAsync(h->d_nactive, 0, sizeof(int), h->stream));
    h->binned = false;
    h->primed = false;
    return ICY_OK;
}

int icy_instance_allocate(icy_mpm *h, unsigned capacity, cudaStream_t work_stream)
{
    const bool split = h->precision == ICY_PRECISION_FP32_SPLIT;
    CK(cudaSetDevice(h->device));
    if (work_stream) {
        h->stream = work_stream;   // no stream of its own (creating one cost 2 ms)
    } else {
        CK(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
        h->stream = h->own_stream;
    }
    h->capacity = capacity;
    h->pitch = ((long)capacity + 31) / 32 * 32;
    const int nx = h->prm.GridXTotal + 2 * h->prm.GridHaloSize;
    h->n_nodes = (long)h->prm.GridY * nx;
    if (nx > 32767 || h->prm.GridY > 32767) return ICY_ERR_INVALID_ARGUMENT;   // packed 16-bit base/cell indices
    cudaError_t e;
    if (split) {
        // FP32 state (two buffers for the binning permutation), FP32 grid,
        // FP64 staging for the HSSOA conversion at upload/download
        h->stage_n = std::min<long>(h->pitch, 1L << 20);
        if ((e = dalloc(h, &h->d_st, S_NLINES * h->pitch)) != cudaSuccess ||
            (e = dalloc(h, &h->d_st_alt, S_NLINES * h->pitch)) != cudaSuccess ||
            (e = dalloc(h, &h->d_stage, 16 * h->stage_n)) != cudaSuccess) {
            icy_set_error("cudaMalloc(particles)", e);
            return ICY_ERR_OUT_OF_MEMORY;
        }
        if ((e = dalloc(h, &h->d_gridf, 7 * h->n_nodes)) != cudaSuccess) {   // either layout of GridViewF
            icy_set_error("cudaMalloc(grid)", e);
            return ICY_ERR_OUT_OF_MEMORY;
        }
        CK(dalloc(h, reinterpret_cast<GrainConstF **>(&h->d_grainf), GRAIN_TAB_F32));
        CK(cudaMemsetAsync(h->d_st, 0, sizeof(unsigned) * S_NLINES * h->pitch, h->stream));
        CK(cudaMemsetAsync(h->d_gridf, 0, sizeof(float) * 7 * h->n_nodes, h->stream));
    } else {
        if ((e = dalloc(h, &h->d_pts, 16 * h->pitch)) != cudaSuccess ||
            (e = dalloc(h, &h->d_pts_alt, 16 * h->pitch)) != cudaSuccess) {
            icy_set_error("cudaMalloc(particles)", e);
            return ICY_ERR_OUT_OF_MEMORY;
        }
        if ((e = dalloc(h, &h->d_grid, 5 * h->n_nodes)) != cudaSuccess) {
            icy_set_error("cudaMalloc(grid)", e);
            return ICY_ERR_OUT_OF_MEMORY;
        }
        CK(cudaMemsetAsync(h->d_pts, 0, sizeof(double) * 16 * h->pitch, h->stream));
        CK(cudaMemsetAsync(h->d_grid, 0, sizeof(double) * 5 * h->n_nodes, h->stream));
    }
    CK(dalloc(h, &h->d_oidx, h->pitch));
    CK(dalloc(h, &h->d_oidx_alt, h->pitch));
    CK(dalloc(h, &h->d_keys, h->pitch));
    CK(dalloc(h, &h->d_ranks, h->pitch));
    if (int rc = alloc_tiles(h)) return rc;
    CK(dalloc(h, &h->d_nactive, 1));
    CK(dalloc(h, &h->d_tlist_n, 2));
    CK(dalloc(h, &h->d_unsafe, 2));
    CK(dalloc(h, &h->d_moved, 3));
    CK(dalloc(h, &h->d_acc, 2 * h->prm.n_indenter_subdivisions));
    CK(dalloc(h, &h->d_status, 1));
    CK(dalloc(h, &h->d_grain, GRAIN_TAB));
    h->h_status = status_slot_get();
    if (!h->h_status) return ICY_ERR_OUT_OF_MEMORY;
    CK(cudaMemsetAsync(h->d_tlist_n, 0, sizeof(unsigned) * 2, h->stream));
    CK(cudaMemsetAsync(h->d_unsafe, 0xff, sizeof(int) * 2, h->stream));
    CK(cudaMemsetAsync(h->d_nactive, 0, sizeof(int), h->stream));
    CK(cudaMemsetAsync(h->d_moved, 0, sizeof(unsigned long long) * 3, h->stream));
    CK(cudaMemsetAsync(h->d_acc, 0, sizeof(double) * 2 * h->prm.n_indenter_subdivisions, h->stream));
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream));
    // persistent grid sizes
    int sms = 0, per_sm = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    CK(cudaFuncSetAttribute(k_tile<true, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TILE_DYN_SMEM));
    CK(cudaFuncSetAttribute(k_tile<false, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TILE_DYN_SMEM));
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile<true, true, false>, TILE_THREADS, TILE_DYN_SMEM));
    h->tile_grid = std::max(1, sms * std::max(per_sm, 1));
    CK(cudaFuncSetAttribute(k_tile_pipe, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PIPE_SMEM));
    h->pipe_grid = sms;
    if (int rc = icy_instance_constants(h)) return rc;
    // a caller's stream is not waited for: waiting here, behind the kernels
    // already queued on a busy device, cost a served batch 12 ms per admission
    if (!work_stream) CK(cudaStreamSynchronize(h->stream));
    return ICY_OK;
}

void icy_instance_free(icy_mpm *h, bool trim, bool wait)
{
    icy_prof_free(h);
    if (wait && h->own_stream) cudaStreamSynchronize(h->own_stream);
    if (wait && h->stream && h->stream != h->own_stream) cudaStreamSynchronize(h->stream);
    void *ptrs[] = {h->d_pts, h->d_pts_alt, h->d_grid, h->d_oidx, h->d_oidx_alt, h->d_keys, h->d_ranks,
                    h->d_counts, h->d_start, h->d_active, h->d_nactive, h->d_flags, h->d_moved, h->d_acc,
                    h->d_status, h->d_block_sums, h->d_grain, h->d_st, h->d_st_alt, h->d_stage, h->d_gridf,
                    h->d_grainf, h->d_tlist, h->d_tlist_n, h->d_nexp, h->d_ncnt, h->d_unsafe};
    cudaStream_t fs = h->stream ? h->stream : h->own_stream;
    for (void *p : ptrs)
        if (p) cudaFreeAsync(p, fs);   // back to the pool, after the stream's work
    if (trim && fs) {
        // a refused allocation: the blocks this instance did get (up to the
        // whole device) go back to the driver now, not to the pool's cache
        cudaStreamSynchronize(fs);
        if (cudaMemPool_t pool = instance_pool(h->device)) cudaMemPoolTrimTo(pool, 0);
    }
    h->d_st = h->d_st_alt = nullptr;
    h->d_stage = nullptr;
    h->d_gridf = nullptr;
    h->d_grainf = nullptr;
    status_slot_put(h->h_status);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    h->d_pts = h->d_pts_alt = h->d_grid = h->d_acc = nullptr;
    h->d_oidx = h->d_oidx_alt = h->d_keys = h->d_ranks = h->d_counts = h->d_start = nullptr;
    h->d_active = h->d_nactive = h->d_status = h->h_status = h->d_block_sums = nullptr;
    h->d_flags = nullptr;
    h->d_tlist = nullptr;
    h->d_tlist_n = nullptr;
    h->d_nexp = h->d_ncnt = h->d_unsafe = nullptr;
    h->d_moved = nullptr;
    h->d_grain = nullptr;
    h->own_stream = h->stream = nullptr;
}

static bool is_split(const icy_mpm *h) { return h->precision == ICY_PRECISION_FP32_SPLIT; }

int icy_instance_upload(icy_mpm *h, const double *hssoa, unsigned cap, unsigned size)
{
    if (is_split(h)) {
        // FP64 HSSOA -> FP32 state, in chunks through the staging buffer
        for (long a = 0; a < (long)size; a += h->stage_n) {
            const long cnt = std::min<long>(h->stage_n, (long)size - a);
            CK(cudaMemcpy2DAsync(h->d_stage, sizeof(double) * h->stage_n, hssoa + a, sizeof(double) * cap,
                                 sizeof(double) * cnt, 16, cudaMemcpyHostToDevice, h->stream));
            k_split_from_hssoa<<<(unsigned)((cnt + 255) / 256), 256, 0, h->stream>>>(
                h->d_stage, h->stage_n, (int)cnt, h->d_st, h->pitch, (int)a, h->prm.cellsize_inv);
            CK_LAUNCH("k_split_from_hssoa");
        }
    } else if (size) {
        // one 2-D copy: 16 lines of `size` doubles, host line stride = cap
        CK(cudaMemcpy2DAsync(h->d_pts, sizeof(double) * h->pitch, hssoa, sizeof(double) * cap,
                             sizeof(double) * size, 16, cudaMemcpyHostToDevice, h->stream));
    }
    h->n = size;
    h->binned = false;
    h->permuted = false;
    h->primed = false;
    if (size) {
        k_iota<<<(size + 255) / 256, 256, 0, h->stream>>>(h->d_oidx, (int)size);
        CK_LAUNCH("k_iota");
    }
    return ICY_OK;
}

int icy_instance_download(icy_mpm *h, double *hssoa, unsigned cap)
{
    if (!h->n) return ICY_OK;
    if (is_split(h)) {
        // FP32 state -> FP64 HSSOA in upload order, in chunks through the staging buffer
        const int *inv = nullptr;
        if (h->permuted) {
            k_inverse_perm<<<(h->n + 255) / 256, 256, 0, h->stream>>>(h->d_oidx, (int)h->n, h->d_keys);
            CK_LAUNCH("k_inverse_perm");
            inv = h->d_keys;
        }
        for (long a = 0; a < (long)h->n; a += h->stage_n) {
            const long cnt = std::min<long>(h->stage_n, (long)h->n - a);
            k_split_to_hssoa<<<(unsigned)((cnt + 255) / 256), 256, 0, h->stream>>>(
                h->d_st, h->pitch, inv, (int)a, (int)cnt, h->d_stage, h->stage_n, h->prm.cellsize);
            CK_LAUNCH("k_split_to_hssoa");
            CK(cudaMemcpy2DAsync(hssoa + a, sizeof(double) * cap, h->d_stage, sizeof(double) * h->stage_n,
                                 sizeof(double) * cnt, 16, cudaMemcpyDeviceToHost, h->stream));
        }
        return ICY_OK;
    }
    const double *src = h->d_pts;
    if (h->permuted) {
        icy_prof_begin(h, K_UNPERMUTE);
        k_unpermute<<<(h->n + 255) / 256, 256, 0, h->stream>>>(h->d_pts, h->d_pts_alt, h->pitch, (int)h->n,
                                                               h->d_oidx);
        icy_prof_end(h);
        CK_LAUNCH("k_unpermute");
        src = h->d_pts_alt;
    }
    CK(cudaMemcpy2DAsync(hssoa, sizeof(double) * cap, src, sizeof(double) * h->pitch, sizeof(double) * h->n, 16,
                         cudaMemcpyDeviceToHost, h->stream));
    return ICY_OK;
}

// Counting sort of the points by tile (stable per warp, not globally):
// count -> scan (+ list of non-empty tiles) -> scatter into the second buffer.
int icy_instance_bin(icy_mpm *h)
{
    if (!h->n) { h->binned = true; return ICY_OK; }
    StepParams P = icy_step_params(h->prm);
    const int nb = (h->n + 255) / 256;
    int stx, sty;
    tile_dims(h, stx, sty);
    const int nkeys = h->ntiles * stx * sty + 1;
    icy_prof_begin(h, K_BIN);
    CK(cudaMemsetAsync(h->d_counts, 0, sizeof(int) * nkeys, h->stream));
    if (is_split(h))
        with_shape(h->shape, [&](auto sh) {
            k_bin_count_f32<decltype(sh)><<<nb, 256, 0, h->stream>>>(P, tile_geom(h), h->d_st, (int)h->n, h->d_keys,
                                                                      h->d_ranks, h->d_counts, h->d_status);
        });
    else
        k_bin_count<<<nb, 256, 0, h->stream>>>(P, tile_geom(h), h->d_pts, h->pitch, (int)h->n, h->d_keys,
                                               h->d_ranks, h->d_counts, h->d_status);
    CK_LAUNCH("k_bin_count");
    k_scan_reduce<<<h->scan_blocks, SCAN_NT, 0, h->stream>>>(h->d_counts, nkeys, h->d_block_sums);
    CK_LAUNCH("k_scan_reduce");
    k_scan_blocks<<<1, 1024, 0, h->stream>>>(h->d_block_sums, h->scan_blocks);
    CK_LAUNCH("k_scan_blocks");
    k_scan_apply<<<h->scan_blocks, SCAN_NT, 0, h->stream>>>(h->d_counts, nkeys, h->d_block_sums, h->d_start);
    CK_LAUNCH("k_scan_apply");
    if (is_split(h))
        with_shape(h->shape, [&](auto sh) {
            k_tiles_active<decltype(sh)::TT><<<1, 1024, 0, h->stream>>>(h->d_start, h->ntiles, h->d_active,
                                                                         h->d_nactive);
        });
    else
        k_tiles_active<<<1, 1024, 0, h->stream>>>(h->d_start, h->ntiles, h->d_active, h->d_nactive);
    CK_LAUNCH("k_tiles_active");
    if (is_split(h)) {
        // fused grid update: contributors per node tile for this binning, counts and
        // margin flags from zero
        with_shape(h->shape, [&](auto sh) {
            k_node_tile_expect<decltype(sh)><<<(h->ntiles + 255) / 256, 256, 0, h->stream>>>(tile_geom(h), h->d_start,
                                                                                           h->d_nexp);
        });
        CK_LAUNCH("k_node_tile_expect");
        CK(cudaMemsetAsync(h->d_ncnt, 0, sizeof(int) * h->ntiles, h->stream));
        CK(cudaMemsetAsync(h->d_unsafe, 0xff, sizeof(int) * 2, h->stream));
        h->fuse_seq = 0;
    }
    if (is_split(h)) {
        k_bin_scatter_f32<<<nb, 256, 0, h->stream>>>(h->d_st, h->d_st_alt, h->pitch, (int)h->n, h->d_keys,
                                                     h->d_ranks, h->d_start, h->d_oidx, h->d_oidx_alt);
        std::swap(h->d_st, h->d_st_alt);
    } else {
        k_bin_scatter<<<nb, 256, 0, h->stream>>>(h->d_pts, h->d_pts_alt, h->pitch, (int)h->n, h->d_keys,
                                                 h->d_ranks, h->d_start, h->d_oidx, h->d_oidx_alt);
        std::swap(h->d_pts, h->d_pts_alt);
    }
    CK_LAUNCH("k_bin_scatter");
    icy_prof_end(h);
    std::swap(h->d_oidx, h->d_oidx_alt);
    h->binned = true;
    h->permuted = true;
    h->steps_since_bin = 0;
    return ICY_OK;
}

static TileArgs tile_args(icy_mpm *h, bool record)
{
    TileArgs A;
    A.P = icy_step_params(h->prm);
    A.G = tile_geom(h);
    A.g = grid_view(h);
    A.pts = h->d_pts;
    A.pitch = h->pitch;
    A.cell_start = h->d_start;
    A.active = h->d_active;
    A.n_active = h->d_nactive;
    A.flags = h->d_flags;
    A.tlist = h->d_tlist;
    A.tlist_n = h->d_tlist_n;
    A.status = h->d_status;
    A.moved = h->d_moved;
    A.grain_tab = h->d_grain;
    A.record_pq = record ? 1 : 0;
    A.fault_test = h->pipe_fault_test ? 1 : 0;
    return A;
}

static GridViewF grid_view_f32(icy_mpm *h)
{
    GridViewF g;
    g.m = h->d_gridf;
    g.px = h->d_gridf + h->n_nodes;
    g.py = h->d_gridf + 2 * h->n_nodes;
    // two velocity buffers: G2P reads buffer vpar, the grid update writes the other
    float *v0 = h->d_gridf + 3 * h->n_nodes, *v1 = h->d_gridf + 5 * h->n_nodes;
    g.vx = h->vpar ? v1 : v0;
    g.vy = g.vx + h->n_nodes;
    g.nvx = h->vpar ? v0 : v1;
    g.mp = reinterpret_cast<float4 *>(h->d_gridf);               // 16-byte aligned (pool blocks: 256 B)
    g.v = reinterpret_cast<float2 *>(h->d_gridf + 4 * h->n_nodes);
    g.ny = h->prm.GridY;
    g.halo = h->prm.GridHaloSize;
    return g;
}

static SplitArgs split_args(icy_mpm *h, bool record)
{
    SplitArgs A;
    A.P = icy_step_params(h->prm);
    A.Q = split_consts(A.P);
    A.G = tile_geom(h);
    A.g = grid_view_f32(h);
    A.st = h->d_st;
    A.pitch = h->pitch;
    A.cell_start = h->d_start;
    A.active = h->d_active;
    A.n_active = h->d_nactive;
    A.flags = h->d_flags;
    A.tlist = h->d_tlist;
    A.tlist_n = h->d_tlist_n;
    A.inst = 0;
    A.status = h->d_status;
    A.moved = h->d_moved;
    A.claim = nullptr;   // batches only
    A.grain_tab = static_cast<const GrainConstF *>(h->d_grainf);
    A.record_pq = record ? 1 : 0;
    A.acc = h->d_acc;
    A.n_nodes = h->n_nodes;
    A.nexp = h->d_nexp;
    A.ncnt = h->d_ncnt;
    A.unsafe = h->d_unsafe;
    A.seq = 0;
    A.safe_m = 0.f;
    A.ind_x = A.ind_y = 0.0;
    return A;
}

// CTAs of the list-driven update queued after a fused tile launch: it has no
// work unless the tile kernel fell back to marking tiles, which a re-binning
// soon ends, so a small grid keeps its empty launch cheap.
static int fallback_ctas(icy_mpm *h)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
    return std::max(1, std::min(h->update_grid_f32, sms));
}

// Largest move of a point in one step, in cells: the grid update clamps node
// speeds to vmax = 0.5 h / dt, and the indenter can add twice its own speed;
// a margin for rounding on top.
static double step_move_cells(const icy_sim_params &p)
{
    return 0.5 + 2.0 * std::fabs(p.IndVelocity) * p.InitialTimeStep * p.cellsize_inv + 1e-3;
}

// which: 0 = G2P + P2G, 1 = P2G only, 2 = G2P only (writes vel and Bp).
// A G2P + P2G launch also updates the grid for the next step (indenter at
// (ind_x, ind_y)) where it is safe to (see k_tile_f32), the list-driven
// update queued after it doing the rest.
static int launch_tile_split(icy_mpm *h, int which, bool record, double ind_x = 0.0, double ind_y = 0.0)
{
    SplitArgs A = split_args(h, record);
    if (which != 2 && h->fuse_update && h->shape == SHAPE_32X8) {
        // every launch with a P2G tests whether a point can leave the staged margin
        // in the step after it (the P2G-only launch that starts a call too, so that
        // the test covers every step a fused launch follows); only G2P + P2G
        // launches fuse the update
        const double delta = step_move_cells(h->prm);
        if (delta < 1.0) {   // beyond one cell a point that has not moved could leave the margin
            A.seq = ++h->fuse_seq;
            A.safe_m = (float)(1.5 - delta);
            A.ind_x = ind_x;
            A.ind_y = ind_y;
        }
    }
    const bool fuse = A.seq > 0;   // only with the 32 x 8 shape (see above)
    const int kinds[3] = {K_TILE_G2P2G, K_TILE_P2G, K_TILE_G2P};
    icy_prof_begin(h, kinds[which < 0 || which > 2 ? 2 : which]);
    with_shape(h->shape, [&](auto sh) {
        using S = decltype(sh);
        const int grid = h->tile_grid_f32;
        switch (which) {
        case 0:
            if (fuse)
                k_tile_f32<true, true, false, false, true><<<grid, TILE_THREADS_F32, MOMF_BYTES, h->stream>>>(A);
            else
                k_tile_f32<true, true, false, false, false, S><<<grid, TILE_THREADS_F32, MOMF_BYTES, h->stream>>>(A);
            break;
        case 1:
            if (fuse)
                k_tile_f32<false, true, false, false, true><<<grid, TILE_THREADS_F32, MOMF_BYTES, h->stream>>>(A);
            else
                k_tile_f32<false, true, false, false, false, S><<<grid, TILE_THREADS_F32, MOMF_BYTES, h->stream>>>(A);
            break;
        default:
            k_tile_f32<true, false, true, false, false, S><<<grid, TILE_THREADS_F32, 0, h->stream>>>(A);
            break;
        }
    });
    icy_prof_end(h);
    CK_LAUNCH("k_tile_f32");
    return ICY_OK;
}

// which: 0 = G2P+P2G, 1 = P2G only, 2 = G2P only (writes vel and Bp)
static int launch_tile(icy_mpm *h, int which, bool record, double ind_x = 0.0, double ind_y = 0.0)
{
    if (!h->n) return ICY_OK;
    if (!h->binned) {
        int rc = icy_instance_bin(h);
        if (rc) return rc;
    }
    if (is_split(h)) return launch_tile_split(h, which, record, ind_x, ind_y);
    TileArgs A = tile_args(h, record);
    switch (which) {
    case 0:
        icy_prof_begin(h, K_TILE_G2P2G);
        if (h->pipe) k_tile_pipe<<<h->pipe_grid, PIPE_THREADS, PIPE_SMEM, h->stream>>>(A);
        else k_tile<true, true, false><<<h->tile_grid, TILE_THREADS, TILE_DYN_SMEM, h->stream>>>(A);
        break;
    case 1:
        icy_prof_begin(h, K_TILE_P2G);
        k_tile<false, true, false><<<h->tile_grid, TILE_THREADS, TILE_DYN_SMEM, h->stream>>>(A);
        break;
    default:
        icy_prof_begin(h, K_TILE_G2P);
        k_tile<true, false, true><<<h->tile_grid, TILE_THREADS, 0, h->stream>>>(A);
        break;
    }
    icy_prof_end(h);
    CK_LAUNCH("k_tile");
    return ICY_OK;
}

// The list-driven grid update.  FP32: it writes the velocity buffer G2P does
// not read, and the buffers swap after it (also after a fused launch, whose
// update it completes); `ctas` = 0: the usual grid.
static int launch_update_tiles(icy_mpm *h, double ind_x, double ind_y, int ctas = 0)
{
    StepParams P = icy_step_params(h->prm);
    icy_prof_begin(h, K_UPDATE_TILES);
    if (is_split(h)) {
        with_shape(h->shape, [&](auto sh) {
            using S = decltype(sh);
            k_update_tiles_f32<S><<<ctas > 0 ? ctas : h->update_grid_f32, S::TT, 0, h->stream>>>(
                split_args(h, false), h->d_tlist, h->d_tlist_n, ind_x, ind_y);
        });
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemsetAsync(h->d_tlist_n, 0, sizeof(unsigned) * 2, h->stream);
        if (e != cudaSuccess) { icy_set_error("k_update_tiles_f32", e); return ICY_ERR_CUDA; }
        h->vpar ^= 1;
    } else
        k_update_list<<<h->update_grid, 256, sizeof(double) * 2 * P.nsub, h->stream>>>(
            P, tile_geom(h), grid_view(h), h->d_flags, h->d_tlist, h->d_tlist_n, ind_x, ind_y, h->d_acc);
    icy_prof_end(h);
    CK_LAUNCH("k_update_nodes");
    return ICY_OK;
}

// per-instance tables that depend on the parameters
int icy_instance_constants(icy_mpm *h)
{
    k_grain_table<<<(GRAIN_TAB + 255) / 256, 256, 0, h->stream>>>(icy_step_params(h->prm), h->d_grain);
    CK_LAUNCH("k_grain_table");
    if (is_split(h)) {
        k_grain_table_f32<<<(GRAIN_TAB_F32 + 255) / 256, 256, 0, h->stream>>>(h->d_grain,
                                                                        static_cast<GrainConstF *>(h->d_grainf));
        CK_LAUNCH("k_grain_table_f32");
    }
    return ICY_OK;
}

int icy_phase_reset_grid(icy_mpm *h)
{
    icy_prof_begin(h, K_MEMSET_GRID);
    if (is_split(h)) CK(cudaMemsetAsync(h->d_gridf, 0, sizeof(float) * 3 * h->n_nodes, h->stream));
    else CK(cudaMemsetAsync(h->d_grid, 0, sizeof(double) * 3 * h->n_nodes, h->stream));
    icy_prof_end(h);
    if (h->tiled || is_split(h)) {
        CK(cudaMemsetAsync(h->d_flags, 0, sizeof(unsigned) * h->ntiles, h->stream));
        CK(cudaMemsetAsync(h->d_tlist_n, 0, sizeof(unsigned) * 2, h->stream));
    }
    h->primed = false;
    return ICY_OK;
}

int icy_phase_p2g(icy_mpm *h)
{
    if (!h->n) return ICY_OK;
    if (h->tiled || is_split(h)) return launch_tile(h, 1, false);
    StepParams P = icy_step_params(h->prm);
    const int tpb = 256;
    icy_prof_begin(h, K_P2G_SIMPLE);
    k_p2g_simple<<<(h->n + tpb - 1) / tpb, tpb, 0, h->stream>>>(P, h->d_pts, h->pitch, (int)h->n, grid_view(h),
                                                                h->d_status);
    icy_prof_end(h);
    CK_LAUNCH("k_p2g_simple");
    return ICY_OK;
}

int icy_phase_update(icy_mpm *h, double ind_x, double ind_y)
{
    if (h->tiled || is_split(h)) return launch_update_tiles(h, ind_x, ind_y);
    StepParams P = icy_step_params(h->prm);
    const int tpb = 256;
    const long nb = (h->n_nodes + tpb - 1) / tpb;
    icy_prof_begin(h, K_UPDATE_SIMPLE);
    k_update_simple<<<(unsigned)nb, tpb, sizeof(double) * 2 * P.nsub, h->stream>>>(P, grid_view(h), h->n_nodes,
                                                                                 ind_x, ind_y, h->d_acc);
    icy_prof_end(h);
    CK_LAUNCH("k_update_simple");
    return ICY_OK;
}

int icy_phase_g2p(icy_mpm *h, bool recordPQ)
{
    if (!h->n) return ICY_OK;
    h->primed = false;
    if (h->tiled || is_split(h)) return launch_tile(h, 2, recordPQ);
    StepParams P = icy_step_params(h->prm);
    const int tpb = 128;
    icy_prof_begin(h, K_G2P_SIMPLE);
    k_g2p_simple<<<(h->n + tpb - 1) / tpb, tpb, 0, h->stream>>>(P, h->d_pts, h->pitch, (int)h->n, grid_view(h),
                                                                recordPQ ? 1 : 0, h->d_status);
    icy_prof_end(h);
    CK_LAUNCH("k_g2p_simple");
    return ICY_OK;
}

int icy_instance_steps(icy_mpm *h, int step0, int nsteps, double *sim_time)
{
    double t = *sim_time;
    const icy_sim_params &p = h->prm;
    int rc;
    if (!h->tiled && !is_split(h)) {
        for (int k = 0; k < nsteps; k++) {
            // icy::Model::Step sub-step (simulation/model.cpp:40-49)
            t += p.InitialTimeStep;
            const double ind_x = p.indenter_x_initial + t * p.IndVelocity;
            if ((rc = icy_phase_reset_grid(h))) return rc;
            if ((rc = icy_phase_p2g(h))) return rc;
            if ((rc = icy_phase_update(h, ind_x, p.indenter_y))) return rc;
            const bool rec = ((step0 + k) % p.UpdateEveryNthStep) == 0;
            if ((rc = icy_phase_g2p(h, rec))) return rc;
        }
        *sim_time = t;
        return ICY_OK;
    }
    if (nsteps == 0) return ICY_OK;
    if (is_split(h)) {
        // FP32: P2G(first) and its update, then [G2P(k) + P2G(k+1) + update(k+1)]
        // per step (the update fused into the tile kernel where safe, the list
        // update after it completing it otherwise), last G2P alone.  Each update
        // takes the indenter position of its own sub-step, t += dt;
        // indenter_x = x0 + t V (simulation/model.cpp:40-41).
        if (!h->primed) {
            const double t1 = t + p.InitialTimeStep;
            if ((rc = launch_tile(h, 1, false))) return rc;
            if ((rc = launch_update_tiles(h, p.indenter_x_initial + t1 * p.IndVelocity, p.indenter_y))) return rc;
            h->primed = true;
        }
        for (int k = 0; k < nsteps; k++) {
            t += p.InitialTimeStep;
            const bool rec = ((step0 + k) % p.UpdateEveryNthStep) == 0;
            if (k == nsteps - 1) {
                if ((rc = launch_tile(h, 2, rec))) return rc;
                h->primed = false;
            } else {
                const double tn = t + p.InitialTimeStep;
                const double ind_x = p.indenter_x_initial + tn * p.IndVelocity;
                if ((rc = launch_tile(h, 0, rec, ind_x, p.indenter_y))) return rc;
                // the fused update's fallback: empty unless the tile kernel marked tiles
                if ((rc = launch_update_tiles(h, ind_x, p.indenter_y, h->fuse_update ? fallback_ctas(h) : 0)))
                    return rc;
                if (h->resort_every > 0 && ++h->steps_since_bin >= h->resort_every)
                    if ((rc = icy_instance_bin(h))) return rc;
            }
        }
        *sim_time = t;
        return ICY_OK;
    }
    // tiled path: P2G(first), then [update(k); G2P(k)+P2G(k+1)] ..., last G2P alone
    if (!h->primed) {
        if ((rc = launch_tile(h, 1, false))) return rc;
        h->primed = true;
    }
    for (int k = 0; k < nsteps; k++) {
        t += p.InitialTimeStep;
        const double ind_x = p.indenter_x_initial + t * p.IndVelocity;
        if ((rc = launch_update_tiles(h, ind_x, p.indenter_y))) return rc;
        const bool rec = ((step0 + k) % p.UpdateEveryNthStep) == 0;
        if (k == nsteps - 1) {
            if ((rc = launch_tile(h, 2, rec))) return rc;
            h->primed = false;
        } else {
            if ((rc = launch_tile(h, 0, rec))) return rc;
            if (h->resort_every > 0 && ++h->steps_since_bin >= h->resort_every)
                if ((rc = icy_instance_bin(h))) return rc;
        }
    }
    *sim_time = t;
    return ICY_OK;
}

// ---------------------------------------------------------------- launch helpers
// The one-thread-per-item kernels on caller-supplied buffers, for entry points
// defined in other translation units (icy_step_noalloc in noalloc.cu).  grid
// holds five arrays of n_nodes doubles: m, px, py, vx, vy.
static GridView raw_grid_view(double *grid, long n_nodes, int ny, int halo)
{
    GridView g;
    g.m = grid;
    g.px = grid + n_nodes;
    g.py = grid + 2 * n_nodes;
    g.vx = grid + 3 * n_nodes;
    g.vy = grid + 4 * n_nodes;
    g.ny = ny;
    g.halo = halo;
    return g;
}

cudaError_t icy_launch_p2g_simple(cudaStream_t s, const StepParams &P, const double *pts, long pitch, int n,
                                  double *grid, long n_nodes, int *status)
{
    if (n > 0)
        k_p2g_simple<<<(n + 255) / 256, 256, 0, s>>>(P, pts, pitch, n, raw_grid_view(grid, n_nodes, P.gridy, P.halo),
                                                     status);
    return cudaGetLastError();
}

cudaError_t icy_launch_update_simple(cudaStream_t s, const StepParams &P, double *grid, long n_nodes, double ind_x,
                                     double ind_y, double *acc)
{
    const long nb = (n_nodes + 255) / 256;
    k_update_simple<<<(unsigned)nb, 256, sizeof(double) * 2 * P.nsub, s>>>(
        P, raw_grid_view(grid, n_nodes, P.gridy, P.halo), n_nodes, ind_x, ind_y, acc);
    return cudaGetLastError();
}

cudaError_t icy_launch_g2p_simple(cudaStream_t s, const StepParams &P, double *pts, long pitch, int n, double *grid,
                                  long n_nodes, int recordPQ, int *status)
{
    if (n > 0)
        k_g2p_simple<<<(n + 127) / 128, 128, 0, s>>>(P, pts, pitch, n, raw_grid_view(grid, n_nodes, P.gridy, P.halo),
                                                     recordPQ, status);
    return cudaGetLastError();
}
