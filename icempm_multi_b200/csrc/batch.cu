// batch.cu -- many independent simulation instances advanced together.
//
// Every member is an FP32 split-precision instance with its own parameters,
// grid and points.  One step of the whole batch is four launches, whatever the
// number of members: advance the members' clocks, update all marked grid
// nodes, clear the marks, and the tile kernel over the (instance, tile) work
// list of all members.  A sequence of steps is captured once per length as a
// CUDA graph and replayed.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cstring>
#include <map>
#include <vector>

#include "../../include/icempm.h"
#include "instance.cuh"
#include "kernels_split.cuh"

using namespace icy_dev;

namespace icy_dev {   // batch_cargs.cu
int batch_const_slots();
bool batch_const_acquire(int device, const void *batch);
void batch_const_release(int device, const void *batch);
cudaError_t batch_const_upload(const SplitArgs *args, const SplitArgs *d_args, int n, SplitMember *staging,
                               cudaStream_t s);
cudaError_t batch_const_setup();
cudaError_t batch_upd_const_upload(const SplitArgs *args, int n, UpdMember *staging, cudaStream_t s);
void batch_upd_const_launch(int shape, int grid, cudaStream_t s, const BatchClock *clk, const int2 *tlist,
                            unsigned *tlist_n);
void batch_const_launch_tile(int kind, int shape, int grid, cudaStream_t s, const SplitArgs &none, const SplitArgs *args,
                             const BatchItem *work, const int *nwork, const int *rec);
}

#define CKB(call)                                                                 \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) { icy_set_error(#call, e_); return ICY_ERR_CUDA; } \
    } while (0)

// A retired member: its download is in flight on the side stream.
struct Retiring {
    icy_mpm *h = nullptr;
    cudaEvent_t done = nullptr;
    const double *hssoa = nullptr;   // destination of the download (NULL: none)
    double *bins = nullptr;          // caller's force bins, filled at collection (NULL: none)
    double *h_bins = nullptr;        // page-locked staging of the bins (a pageable target would block)
    int nbins = 0, bins_cap = 0;
};

struct icy_batch {
    int device = 0;
    cudaStream_t stream = nullptr;   // rounds, re-binning, work-list rebuilds
    cudaStream_t side = nullptr;     // admissions (upload, binning) and retirements (download)
    cudaEvent_t ev_join = nullptr, ev_round = nullptr;
    int nslots = 0;
    std::vector<icy_mpm *> members;
    std::vector<Retiring> retiring;
    BatchClock *h_clk = nullptr;     // page-locked: the clocks of retired members
    SplitArgs *d_args = nullptr;
    BatchClock *d_clk = nullptr;
    int *d_rec = nullptr;
    int2 *d_tlist = nullptr;         // node tiles written since the last update, all members
    unsigned *d_tlist_n = nullptr;   // [0] entries, [1] CTAs of the update done
    BatchItem *d_work = nullptr;
    long work_cap = 0;
    int *d_woff = nullptr, *d_nwork = nullptr;
    int *d_claim = nullptr;          // work-item counters of the tile kernel
    bool dirty = true;
    int steps_since_bin = 0, resort_every = 256;
    static constexpr int NEV = 8;
    cudaEvent_t ev_steps[NEV] = {};   // ring: recorded after each icy_batch_step
    int64_t steps_queued = 0;
    std::map<int, cudaGraphExec_t> graphs;
    std::map<int, int> graph_launches;   // kernels per replay
    int tile_grid = 0, update_grid = 0;
    int shape = SHAPE_32X8;         // members' tile shape (option "tile_shape", set while the batch is empty)
    bool cargs = false;              // owns the device's constant-bank argument table (batch_cargs.cu)
    int64_t launches = 0;
    // page-locked staging of the argument tables a rebuild uploads, a ring of
    // NARGS (a copy from pageable memory would wait for the queued rounds)
    static constexpr int NARGS = 3;
    SplitArgs *h_args[NARGS] = {};
    SplitMember *h_mem[NARGS] = {};
    UpdMember *h_upd[NARGS] = {};
    cudaEvent_t ev_args[NARGS] = {};
    bool args_used[NARGS] = {};
    int args_next = 0;
    // the members' re-binning tables (batched binning), staged the same way
    BinMember *d_bin = nullptr;
    BinMember *h_bin[NARGS] = {};
    cudaEvent_t ev_bin[NARGS] = {};
    bool bin_used[NARGS] = {};
    int bin_next = 0;
};

// A member's device memory back to the pool in the order of the batch's second
// stream, where its last work (upload or download) ran: no host wait.
static void member_destroy(icy_batch *b, icy_mpm *h)
{
    h->stream = b->side;
    icy_instance_free(h, false, false);
    delete h;
}

static SplitArgs member_args(icy_batch *b, icy_mpm *h, int slot)
{
    SplitArgs A{};
    A.P = icy_step_params(h->prm);
    A.Q = split_consts(A.P);
    A.G = TileGeom{h->ntx, h->nty, h->ntiles};
    GridViewF g;
    g.m = h->d_gridf;
    g.px = h->d_gridf + h->n_nodes;
    g.py = h->d_gridf + 2 * h->n_nodes;
    g.vx = h->d_gridf + 3 * h->n_nodes;
    g.vy = h->d_gridf + 4 * h->n_nodes;
    g.mp = reinterpret_cast<float4 *>(h->d_gridf);               // 16-byte aligned (pool blocks: 256 B)
    g.v = reinterpret_cast<float2 *>(h->d_gridf + 4 * h->n_nodes);
    g.ny = h->prm.GridY;
    g.halo = h->prm.GridHaloSize;
    A.g = g;
    A.st = h->d_st;
    A.pitch = h->pitch;
    A.cell_start = h->d_start;
    A.active = h->d_active;
    A.n_active = h->d_nactive;
    A.flags = h->d_flags;
    A.tlist = b->d_tlist;
    A.tlist_n = b->d_tlist_n;
    A.inst = slot;
    A.status = h->d_status;
    A.moved = h->d_moved;
    A.grain_tab = static_cast<const GrainConstF *>(h->d_grainf);
    A.record_pq = 0;
    A.acc = h->d_acc;
    A.n_nodes = h->n_nodes;
    return A;
}

static void drop_graphs(icy_batch *b)
{
    for (auto &kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
    b->graph_launches.clear();
}

// Upload the members' kernel arguments and work list (and grow the work and
// node-tile lists to the members' total tile count).
static int rebuild(icy_batch *b)
{
    // the staging buffer of the rebuild NARGS ago: its copies are long done
    const int k = b->args_next;
    b->args_next = (k + 1) % icy_batch::NARGS;
    if (b->args_used[k]) CKB(cudaEventSynchronize(b->ev_args[k]));
    SplitArgs *args = b->h_args[k];
    long tiles = 0;
    for (int s = 0; s < b->nslots; s++)
        tiles += b->members[s] ? b->members[s]->ntiles : 0;
    if (tiles > b->work_cap) {
        cudaFree(b->d_work);
        b->d_work = nullptr;
        drop_graphs(b);   // the graphs hold the old work-list address
        cudaFree(b->d_tlist);
        b->d_tlist = nullptr;
        const long cap = std::max(tiles, 2 * b->work_cap);
        cudaError_t e = cudaMalloc(&b->d_work, sizeof(BatchItem) * std::max(cap, 1L));
        if (e == cudaSuccess) e = cudaMalloc(&b->d_tlist, sizeof(int2) * std::max(cap, 1L));
        if (e != cudaSuccess) { icy_set_error("cudaMalloc(batch work list)", e); return ICY_ERR_OUT_OF_MEMORY; }
        b->work_cap = cap;
    }
    for (int s = 0; s < b->nslots; s++) args[s] = b->members[s] ? member_args(b, b->members[s], s) : SplitArgs{};
    CKB(cudaMemcpyAsync(b->d_args, args, sizeof(SplitArgs) * b->nslots, cudaMemcpyHostToDevice, b->stream));
    if (b->cargs) {
        CKB(batch_const_upload(args, b->d_args, b->nslots, b->h_mem[k], b->stream));
        CKB(batch_upd_const_upload(args, b->nslots, b->h_upd[k], b->stream));
    }
    CKB(cudaEventRecord(b->ev_args[k], b->stream));
    b->args_used[k] = true;
    k_batch_work_offsets<<<1, 1024, 0, b->stream>>>(b->d_args, b->d_clk, b->nslots, b->d_woff, b->d_nwork);
    k_batch_work_fill<<<dim3(8, b->nslots), 256, 0, b->stream>>>(b->d_args, b->d_clk, b->d_woff, b->d_work);
    CKB(cudaGetLastError());
    b->launches += 2;
    b->dirty = false;
    return ICY_OK;
}

// Every member with points binned again (icy_instance_bin's work), all
// members in seven launches on the batch stream.
static int rebin_members(icy_batch *b)
{
    const int k = b->bin_next;
    b->bin_next = (k + 1) % icy_batch::NARGS;
    if (b->bin_used[k]) CKB(cudaEventSynchronize(b->ev_bin[k]));
    BinMember *tab = b->h_bin[k];
    int nm = 0;
    long blocks = 0, sblocks = 0;
    for (icy_mpm *h : b->members) {
        if (!h || !h->n) continue;
        BinMember &m = tab[nm++];
        m.st = h->d_st;
        m.st_alt = h->d_st_alt;
        m.pitch = h->pitch;
        m.n = (int)h->n;
        m.blk0 = (int)blocks;
        m.sblk0 = (int)sblocks;
        m.halo = h->prm.GridHaloSize;
        m.gridx = h->prm.GridXTotal;
        m.gridy = h->prm.GridY;
        m.G = TileGeom{h->ntx, h->nty, h->ntiles};
        m.keys = h->d_keys;
        m.ranks = h->d_ranks;
        m.counts = h->d_counts;
        m.start = h->d_start;
        m.block_sums = h->d_block_sums;
        m.active = h->d_active;
        m.nactive = h->d_nactive;
        m.nexp = h->d_nexp;
        m.ncnt = h->d_ncnt;
        m.unsafe = h->d_unsafe;
        m.status = h->d_status;
        m.oidx = h->d_oidx;
        m.oidx_alt = h->d_oidx_alt;
        blocks += (h->n + 255) / 256;
        sblocks += h->scan_blocks;
    }
    if (blocks > INT_MAX || sblocks > INT_MAX) return ICY_ERR_INVALID_ARGUMENT;
    if (nm > 0) {
        CKB(cudaMemcpyAsync(b->d_bin, tab, sizeof(BinMember) * nm, cudaMemcpyHostToDevice, b->stream));
        CKB(cudaEventRecord(b->ev_bin[k], b->stream));
        b->bin_used[k] = true;
        with_shape(b->shape, [&](auto sh) {
            using S = decltype(sh);
            k_bin_clear_batch<S><<<dim3(64, nm), 256, 0, b->stream>>>(b->d_bin);
            k_bin_count_batch<S><<<(int)blocks, 256, 0, b->stream>>>(b->d_bin, nm);
            k_bin_scan_reduce_batch<S><<<(int)sblocks, SCAN_NT, 0, b->stream>>>(b->d_bin, nm);
            k_bin_scan_blocks_batch<S><<<nm, 1024, 0, b->stream>>>(b->d_bin);
            k_bin_scan_apply_batch<S><<<(int)sblocks, SCAN_NT, 0, b->stream>>>(b->d_bin, nm);
            k_bin_tiles_batch<S><<<nm, 1024, 0, b->stream>>>(b->d_bin);
            k_bin_scatter_batch<<<(int)blocks, 256, 0, b->stream>>>(b->d_bin, nm);
        });
        CKB(cudaGetLastError());
        b->launches += 7;
        for (icy_mpm *h : b->members) {
            if (!h || !h->n) continue;
            std::swap(h->d_st, h->d_st_alt);
            std::swap(h->d_oidx, h->d_oidx_alt);
            h->binned = h->permuted = true;
            h->steps_since_bin = 0;
            h->fuse_seq = 0;
        }
    }
    b->steps_since_bin = 0;
    b->dirty = true;
    return ICY_OK;
}

// The batched tile kernel (kind 0: first P2G, 1: fused, 2: last G2P): the
// constant-bank variant when this batch owns the device's table.
template <bool DO_G2P, bool DO_P2G, bool WRITE_VB>
static void launch_tile_batch(icy_batch *b, const SplitArgs &none, size_t smem, int kind)
{
    if (b->cargs)
        batch_const_launch_tile(kind, b->shape, b->tile_grid, b->stream, none, b->d_args, b->d_work, b->d_nwork,
                                b->d_rec);
    else
        with_shape(b->shape, [&](auto sh) {
            k_tile_f32<DO_G2P, DO_P2G, WRITE_VB, true, false, decltype(sh)>
                <<<b->tile_grid, TILE_THREADS_F32, smem, b->stream>>>(none, b->d_args, b->d_work, b->d_nwork, b->d_rec);
        });
}

// Capture [P2G] + nsteps x [advance, update, G2P(+P2G)] as a graph.
static int capture(icy_batch *b, int nsteps, cudaGraphExec_t *out, int *nlaunch)
{
    SplitArgs none{};
    none.claim = b->d_claim;
    cudaGraph_t g = nullptr;
    int n = 0;
    CKB(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    launch_tile_batch<false, true, false>(b, none, MOMF_BYTES, 0);
    n++;
    for (int k = 0; k < nsteps; k++) {
        k_batch_advance<<<(b->nslots + 127) / 128, 128, 0, b->stream>>>(b->d_clk, b->d_rec, b->nslots);
        if (b->cargs)
            batch_upd_const_launch(b->shape, b->update_grid, b->stream, b->d_clk, b->d_tlist, b->d_tlist_n);
        else
            with_shape(b->shape, [&](auto sh) {
                k_update_list_f32<decltype(sh), GlobalMembers><<<b->update_grid, 256, 0, b->stream>>>(
                    GlobalMembers{b->d_args}, b->d_clk, b->d_tlist, b->d_tlist_n);
            });
        if (k + 1 < nsteps)
            launch_tile_batch<true, true, false>(b, none, MOMF_BYTES, 1);
        else
            launch_tile_batch<true, false, true>(b, none, 0, 2);
        n += 3;
    }
    cudaError_t e = cudaStreamEndCapture(b->stream, &g);
    if (e != cudaSuccess) { icy_set_error("cudaStreamEndCapture", e); return ICY_ERR_CUDA; }
    e = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { icy_set_error("cudaGraphInstantiate", e); return ICY_ERR_CUDA; }
    *nlaunch = n;
    return ICY_OK;
}

extern "C" int64_t icy_mpm_device_bytes(const icy_sim_params *p, unsigned capacity, int precision);

static int64_t icy_instance_device_bytes(icy_mpm *h)
{
    return icy_mpm_device_bytes(&h->prm, h->capacity, h->precision);
}

extern "C" {

int icy_mpm_reserve(int device, int64_t bytes)
{
    if (bytes < 0) return ICY_ERR_INVALID_ARGUMENT;
    return icy_instance_pool_reserve(device, (size_t)bytes);
}

// Device memory an instance of this size takes (as allocated by
// icy_instance_allocate), for admission by memory budget.
int64_t icy_mpm_device_bytes(const icy_sim_params *p, unsigned capacity, int precision)
{
    if (!p) return 0;
    const long pitch = ((long)capacity + 31) / 32 * 32;
    const long nx = p->GridXTotal + 2L * p->GridHaloSize;
    const long n_nodes = (long)p->GridY * nx;
    const long ntiles = ((nx + TX - 1) / TX) * ((p->GridY + TY - 1) / TY);
    const long nkeys = ntiles * TT + 1;
    int64_t b = 0;
    if (precision == ICY_PRECISION_FP32_SPLIT)
        b += 2 * (int64_t)S_NLINES * 4 * pitch + 16 * 8 * (int64_t)std::min(pitch, 1L << 20) + 7 * 4 * (int64_t)n_nodes +
             4 * 2 * (int64_t)ntiles + 16;
    else
        b += 2 * 16 * 8 * (int64_t)pitch + 5 * 8 * (int64_t)n_nodes;
    b += 4 * 4 * (int64_t)pitch + 4 * (2 * nkeys + 1) + 4 * 2 * ntiles + 2 * 8 * p->n_indenter_subdivisions + 65536;
    return b;
}

int icy_batch_create(int device, int max_instances, icy_batch **out)
{
    if (!out || max_instances < 1 || max_instances > 65535) return ICY_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    icy_batch *b = new icy_batch();
    b->device = device;
    b->nslots = max_instances;
    b->members.assign(max_instances, nullptr);
    auto fail = [&](cudaError_t e, const char *w) {
        icy_set_error(w, e);
        icy_batch_destroy(b);
        return ICY_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaSetDevice(device)) != cudaSuccess) return fail(e, "cudaSetDevice");
    b->retiring.assign(max_instances, Retiring{});
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(e, "stream");
    if ((e = cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming)) != cudaSuccess ||
        (e = cudaEventCreateWithFlags(&b->ev_round, cudaEventDisableTiming)) != cudaSuccess)
        return fail(e, "event");
    for (cudaEvent_t &ev : b->ev_steps)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    if ((e = cudaMallocHost(&b->h_clk, sizeof(BatchClock) * max_instances)) != cudaSuccess)
        return fail(e, "cudaMallocHost(batch clocks)");
    for (int k = 0; k < icy_batch::NARGS; k++) {
        if ((e = cudaMallocHost(&b->h_args[k], sizeof(SplitArgs) * max_instances)) != cudaSuccess)
            return fail(e, "cudaMallocHost(batch arguments)");
        if (max_instances <= batch_const_slots() &&
            ((e = cudaMallocHost(&b->h_mem[k], sizeof(SplitMember) * max_instances)) != cudaSuccess ||
             (e = cudaMallocHost(&b->h_upd[k], sizeof(UpdMember) * max_instances)) != cudaSuccess))
            return fail(e, "cudaMallocHost(batch arguments)");
        if ((e = cudaEventCreateWithFlags(&b->ev_args[k], cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&b->ev_bin[k], cudaEventDisableTiming)) != cudaSuccess)
            return fail(e, "event");
        if ((e = cudaMallocHost(&b->h_bin[k], sizeof(BinMember) * max_instances)) != cudaSuccess)
            return fail(e, "cudaMallocHost(batch binning)");
    }
    if ((e = cudaMalloc(&b->d_bin, sizeof(BinMember) * max_instances)) != cudaSuccess)
        return fail(e, "cudaMalloc(batch binning)");
    if ((e = cudaMalloc(&b->d_args, sizeof(SplitArgs) * max_instances)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_clk, sizeof(BatchClock) * max_instances)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_rec, sizeof(int) * max_instances)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_tlist_n, sizeof(unsigned) * 2)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_woff, sizeof(int) * max_instances)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_nwork, sizeof(int))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_claim, sizeof(int) * 2)) != cudaSuccess)
        return fail(e, "cudaMalloc(batch)");
    cudaMemsetAsync(b->d_clk, 0, sizeof(BatchClock) * max_instances, b->stream);
    cudaMemsetAsync(b->d_rec, 0, sizeof(int) * max_instances, b->stream);
    cudaMemsetAsync(b->d_nwork, 0, sizeof(int), b->stream);
    cudaMemsetAsync(b->d_claim, 0, sizeof(int) * 2, b->stream);
    cudaMemsetAsync(b->d_tlist_n, 0, sizeof(unsigned) * 2, b->stream);
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    for (int sh = 0; sh < N_SHAPES; sh++)
        with_shape(sh, [&](auto s) {
            using S = decltype(s);
            cudaFuncSetAttribute(k_tile_f32<true, true, false, true, false, S>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MOMF_BYTES);
            cudaFuncSetAttribute(k_tile_f32<false, true, false, true, false, S>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MOMF_BYTES);
        });
    if ((e = batch_const_setup()) != cudaSuccess) return fail(e, "cudaFuncSetAttribute");
    b->cargs = max_instances <= batch_const_slots() && batch_const_acquire(device, b);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tile_f32<true, true, false, true>, TILE_THREADS_F32,
                                                  MOMF_BYTES);
    b->tile_grid = std::max(1, sms * std::max(per_sm, 1));
    b->update_grid = std::max(1, sms * 8);
    if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return fail(e, "batch init");
    *out = b;
    return ICY_OK;
}

int icy_batch_destroy(icy_batch *b)
{
    if (!b) return ICY_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->side) cudaStreamSynchronize(b->side);
    drop_graphs(b);
    for (icy_mpm *h : b->members)
        if (h) member_destroy(b, h);
    for (Retiring &r : b->retiring) {
        if (r.h) member_destroy(b, r.h);
        if (r.done) cudaEventDestroy(r.done);
        if (r.h_bins) cudaFreeHost(r.h_bins);
    }
    cudaFree(b->d_args);
    cudaFree(b->d_clk);
    cudaFree(b->d_rec);
    cudaFree(b->d_tlist);
    cudaFree(b->d_tlist_n);
    cudaFree(b->d_work);
    cudaFree(b->d_woff);
    cudaFree(b->d_nwork);
    cudaFree(b->d_claim);
    if (b->cargs) batch_const_release(b->device, b);
    if (b->h_clk) cudaFreeHost(b->h_clk);
    for (int k = 0; k < icy_batch::NARGS; k++) {
        if (b->h_args[k]) cudaFreeHost(b->h_args[k]);
        if (b->h_mem[k]) cudaFreeHost(b->h_mem[k]);
        if (b->h_upd[k]) cudaFreeHost(b->h_upd[k]);
        if (b->ev_args[k]) cudaEventDestroy(b->ev_args[k]);
        if (b->h_bin[k]) cudaFreeHost(b->h_bin[k]);
        if (b->ev_bin[k]) cudaEventDestroy(b->ev_bin[k]);
    }
    cudaFree(b->d_bin);
    for (cudaEvent_t ev : b->ev_steps)
        if (ev) cudaEventDestroy(ev);
    if (b->ev_join) cudaEventDestroy(b->ev_join);
    if (b->ev_round) cudaEventDestroy(b->ev_round);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return ICY_OK;
}

// Admission on the side stream (upload, HSSOA conversion, binning), joined
// into the batch stream by an event: the rounds already queued run on
// meanwhile, the next one waits for it.
static int add_member(icy_batch *b, const icy_sim_params *p, const double *hssoa, unsigned capacity, unsigned size,
                      int *slot)
{
    if (!b || !p || !hssoa || !slot || size > capacity || p->UpdateEveryNthStep <= 0) return ICY_ERR_INVALID_ARGUMENT;
    int s = -1;
    for (int k = 0; k < b->nslots; k++)
        if (!b->members[k] && !b->retiring[k].h) { s = k; break; }
    if (s < 0) return ICY_ERR_NO_SPACE;
    CKB(cudaSetDevice(b->device));
    // the member's memory is allocated and cleared on the batch's second stream,
    // behind nothing but earlier admissions and retirements, without waiting
    icy_mpm *h = nullptr;
    int rc = icy_mpm_create_on(p, b->device, std::max(size, 1u), ICY_PRECISION_FP32_SPLIT, b->side, &h);
    if (rc) return rc;
    if (b->shape != SHAPE_32X8 && (rc = icy_instance_set_shape(h, b->shape))) {
        icy_mpm_destroy(h);
        return rc;
    }
    h->stream = b->side;
    if ((rc = icy_mpm_update_constants(h, p)) || (rc = icy_mpm_transfer_points_to_device(h, hssoa, capacity, size)) ||
        (rc = icy_mpm_reset_indenter_force_accumulator(h)) || (rc = icy_instance_bin(h))) {
        member_destroy(b, h);
        return rc;
    }
    BatchClock c{};
    c.t = 0.0;
    c.dt = p->InitialTimeStep;
    c.x0 = p->indenter_x_initial;
    c.y0 = p->indenter_y;
    c.v = p->IndVelocity;
    c.ind_x = p->indenter_x_initial;
    c.step = 0;
    c.every = p->UpdateEveryNthStep;
    c.live = 1;
    CKB(cudaEventRecord(b->ev_join, b->side));
    CKB(cudaStreamWaitEvent(b->stream, b->ev_join, 0));
    // the clock on the batch stream, after the queued rounds (whose clock
    // kernels advance every live slot); from pageable memory, so staged
    // before the call returns
    CKB(cudaMemcpyAsync(b->d_clk + s, &c, sizeof(c), cudaMemcpyHostToDevice, b->stream));
    h->stream = b->stream;   // the member's later work (re-binning, downloads) in the batch's order
    b->members[s] = h;
    b->dirty = true;
    *slot = s;
    return ICY_OK;
}

int icy_batch_add(icy_batch *b, const icy_sim_params *p, const double *hssoa, unsigned capacity, unsigned size,
                  int *slot)
{
    int rc = add_member(b, p, hssoa, capacity, size, slot);
    if (rc) return rc;
    CKB(cudaStreamSynchronize(b->side));
    return ICY_OK;
}

int icy_batch_add_async(icy_batch *b, const icy_sim_params *p, const double *hssoa, unsigned capacity,
                        unsigned size, int *slot)
{
    return add_member(b, p, hssoa, capacity, size, slot);
}

static __global__ void k_batch_leave(BatchClock *clk, int slot, int live) { clk[slot].live = live; }

int icy_batch_retire(icy_batch *b, int slot, double *hssoa, unsigned capacity, double *bins)
{
    if (!b || slot < 0 || slot >= b->nslots || !b->members[slot]) return ICY_ERR_INVALID_ARGUMENT;
    icy_mpm *h = b->members[slot];
    if (hssoa && h->n > capacity) return ICY_ERR_CAPACITY;
    CKB(cudaSetDevice(b->device));
    Retiring &r = b->retiring[slot];
    // host-side preparation that can fail comes before the member leaves the
    // device work list, so that a failure here leaves it a member on both sides
    if (!r.done) CKB(cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming));
    const int nbins = 2 * h->prm.n_indenter_subdivisions;
    if (bins && r.bins_cap < nbins) {
        if (r.h_bins) CKB(cudaFreeHost(r.h_bins));
        r.h_bins = nullptr;
        r.bins_cap = 0;
        CKB(cudaMallocHost(&r.h_bins, sizeof(double) * nbins));
        r.bins_cap = nbins;
    }
    // leaves the batch after the work already queued; its clock stays for the readback
    k_batch_leave<<<1, 1, 0, b->stream>>>(b->d_clk, slot, 0);
    CKB(cudaGetLastError());
    b->launches++;
    // a failure from here on puts the member back into the batch on the device
    // (no round can have been queued in between) and leaves it a member
    auto undo = [&](int rc) {
        h->stream = b->stream;
        k_batch_leave<<<1, 1, 0, b->stream>>>(b->d_clk, slot, 1);
        if (cudaGetLastError() == cudaSuccess) b->launches++;
        return rc;
    };
    cudaError_t e;
    if ((e = cudaEventRecord(b->ev_round, b->stream)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(b->side, b->ev_round, 0)) != cudaSuccess) {
        icy_set_error("icy_batch_retire(event)", e);
        return undo(ICY_ERR_CUDA);
    }
    h->stream = b->side;
    if (hssoa)
        if (int rc = icy_instance_download(h, hssoa, capacity)) return undo(rc);
    r.bins = bins;
    r.nbins = nbins;
    if ((bins && (e = cudaMemcpyAsync(r.h_bins, h->d_acc, sizeof(double) * nbins, cudaMemcpyDeviceToHost,
                                      b->side)) != cudaSuccess) ||
        (e = cudaMemcpyAsync(h->h_status, h->d_status, sizeof(int), cudaMemcpyDeviceToHost, b->side)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(b->h_clk + slot, b->d_clk + slot, sizeof(BatchClock), cudaMemcpyDeviceToHost,
                             b->side)) != cudaSuccess ||
        (e = cudaEventRecord(r.done, b->side)) != cudaSuccess) {
        icy_set_error("icy_batch_retire(readback)", e);
        r.bins = nullptr;
        return undo(ICY_ERR_CUDA);
    }
    r.h = h;
    r.hssoa = hssoa;
    b->members[slot] = nullptr;
    b->dirty = true;
    return ICY_OK;
}

int icy_batch_collect(icy_batch *b, int slot, int wait, int *done, unsigned *size, double *sim_time, int64_t *step)
{
    if (!b || slot < 0 || slot >= b->nslots || !b->retiring[slot].h || !done) return ICY_ERR_INVALID_ARGUMENT;
    CKB(cudaSetDevice(b->device));
    Retiring &r = b->retiring[slot];
    if (wait) {
        CKB(cudaEventSynchronize(r.done));
    } else {
        const cudaError_t q = cudaEventQuery(r.done);
        if (q == cudaErrorNotReady) {
            *done = 0;
            return ICY_OK;
        }
        CKB(q);
    }
    *done = 1;
    icy_mpm *h = r.h;
    const int code = *h->h_status;
    if (r.bins) std::memcpy(r.bins, r.h_bins, sizeof(double) * r.nbins);
    if (size) *size = h->n;
    if (sim_time) *sim_time = b->h_clk[slot].t;
    if (step) *step = b->h_clk[slot].step;
    // active point count of the downloaded state (simulation/gpu_implementation5.cpp:399-433)
    long active = 0;
    if (r.hssoa)
        for (unsigned i = 0; i < h->n; i++) {
            long long u;
            std::memcpy(&u, r.hssoa + i, 8);
            if (!(u & ICY_STATUS_DISABLED)) active++;
        }
    const bool count_ok = !r.hssoa || active == h->prm.nPtsTotal;
    member_destroy(b, h);
    r.h = nullptr;
    r.hssoa = nullptr;
    r.bins = nullptr;
    if (code) return code;
    if (!count_ok) {
        icy_set_error_msg("icy_batch_collect(): active point count mismatch");
        return ICY_ERR_POINT_COUNT;
    }
    return ICY_OK;
}

int icy_batch_remove(icy_batch *b, int slot)
{
    if (!b || slot < 0 || slot >= b->nslots || !b->members[slot]) return ICY_ERR_INVALID_ARGUMENT;
    CKB(cudaSetDevice(b->device));
    CKB(cudaStreamSynchronize(b->stream));
    CKB(cudaStreamSynchronize(b->side));
    BatchClock c{};
    CKB(cudaMemcpy(b->d_clk + slot, &c, sizeof(c), cudaMemcpyHostToDevice));
    member_destroy(b, b->members[slot]);
    b->members[slot] = nullptr;
    b->dirty = true;
    return ICY_OK;
}

int icy_batch_step(icy_batch *b, int nsteps)
{
    if (!b || nsteps < 0) return ICY_ERR_INVALID_ARGUMENT;
    if (nsteps == 0) return ICY_OK;
    CKB(cudaSetDevice(b->device));
    if (b->dirty)
        if (int rc = rebuild(b)) return rc;
    auto it = b->graphs.find(nsteps);
    if (it == b->graphs.end()) {
        cudaGraphExec_t ge;
        int nl = 0;
        if (int rc = capture(b, nsteps, &ge, &nl)) return rc;
        it = b->graphs.emplace(nsteps, ge).first;
        b->graph_launches[nsteps] = nl;
    }
    CKB(cudaGraphLaunch(it->second, b->stream));
    b->launches += b->graph_launches[nsteps];
    b->steps_since_bin += nsteps;
    if (b->resort_every > 0 && b->steps_since_bin >= b->resort_every)
        if (int rc = rebin_members(b)) return rc;
    CKB(cudaEventRecord(b->ev_steps[b->steps_queued % icy_batch::NEV], b->stream));
    b->steps_queued++;
    return ICY_OK;
}

int icy_batch_wait_steps(icy_batch *b, int in_flight)
{
    if (!b || in_flight < 0) return ICY_ERR_INVALID_ARGUMENT;
    CKB(cudaSetDevice(b->device));
    if (in_flight == 0) {
        CKB(cudaStreamSynchronize(b->stream));
        return ICY_OK;
    }
    // the newest call that must have finished (the ring holds the last NEV calls:
    // a larger in_flight waits as for NEV - 1)
    const int64_t k = b->steps_queued - 1 - std::min(in_flight, icy_batch::NEV - 1);
    if (k >= 0) CKB(cudaEventSynchronize(b->ev_steps[k % icy_batch::NEV]));
    return ICY_OK;
}

int icy_batch_set_clock(icy_batch *b, int slot, double sim_time, int64_t step)
{
    if (!b || slot < 0 || slot >= b->nslots || !b->members[slot] || step < 0) return ICY_ERR_INVALID_ARGUMENT;
    CKB(cudaSetDevice(b->device));
    BatchClock c;
    CKB(cudaMemcpyAsync(&c, b->d_clk + slot, sizeof(c), cudaMemcpyDeviceToHost, b->stream));
    CKB(cudaStreamSynchronize(b->stream));
    c.t = sim_time;
    c.step = step;
    c.ind_x = c.x0 + c.t * c.v;   // recomputed on the device before every step
    CKB(cudaMemcpyAsync(b->d_clk + slot, &c, sizeof(c), cudaMemcpyHostToDevice, b->stream));
    CKB(cudaStreamSynchronize(b->stream));
    return ICY_OK;
}

int icy_batch_download(icy_batch *b, int slot, double *hssoa, unsigned capacity, unsigned *size, double *bins,
                       double *sim_time, int64_t *step)
{
    if (!b || slot < 0 || slot >= b->nslots || !b->members[slot]) return ICY_ERR_INVALID_ARGUMENT;
    CKB(cudaSetDevice(b->device));
    BatchClock c;
    CKB(cudaMemcpyAsync(&c, b->d_clk + slot, sizeof(c), cudaMemcpyDeviceToHost, b->stream));
    int rc = icy_mpm_transfer_from_device(b->members[slot], hssoa, capacity, size, bins);
    if (sim_time) *sim_time = c.t;
    if (step) *step = c.step;
    return rc;
}

int icy_batch_synchronize(icy_batch *b)
{
    if (!b) return ICY_ERR_INVALID_ARGUMENT;
    CKB(cudaSetDevice(b->device));
    CKB(cudaStreamSynchronize(b->stream));
    CKB(cudaStreamSynchronize(b->side));
    return ICY_OK;
}

int icy_batch_set_option(icy_batch *b, const char *name, double value)
{
    if (!b || !name) return ICY_ERR_INVALID_ARGUMENT;
    if (std::strcmp(name, "resort_every") == 0 && value >= 0) {
        b->resort_every = (int)value;
        return ICY_OK;
    }
    if (std::strcmp(name, "tile_ctas") == 0 && value >= 1 && value <= (1 << 20)) {   // persistent CTAs, tile kernel
        b->tile_grid = (int)value;
        drop_graphs(b);
        return ICY_OK;
    }
    if (std::strcmp(name, "update_ctas") == 0 && value >= 1 && value <= (1 << 20)) {   // CTAs of the grid update
        b->update_grid = (int)value;
        drop_graphs(b);
        return ICY_OK;
    }
    if (std::strcmp(name, "tile_shape") == 0 && value >= 0 && value < N_SHAPES) {   // members' tile shape
        for (int k = 0; k < b->nslots; k++)
            if (b->members[k] || b->retiring[k].h) return ICY_ERR_NOT_SUPPORTED;   // only while empty
        b->shape = (int)value;
        drop_graphs(b);
        return ICY_OK;
    }
    return ICY_ERR_INVALID_ARGUMENT;
}

int icy_batch_info(icy_batch *b, int *live, int64_t *points, int64_t *kernel_launches, void **stream)
{
    if (!b) return ICY_ERR_INVALID_ARGUMENT;
    int nl = 0;
    int64_t np = 0;
    for (icy_mpm *h : b->members)
        if (h) { nl++; np += h->n; }
    if (live) *live = nl;
    if (points) *points = np;
    if (kernel_launches) *kernel_launches = b->launches;
    if (stream) *stream = b->stream;
    return ICY_OK;
}

int64_t icy_batch_device_bytes(icy_batch *b, int slot)
{
    if (!b || slot < 0 || slot >= b->nslots || !b->members[slot]) return 0;
    return icy_instance_device_bytes(b->members[slot]);
}

}  // extern "C"
