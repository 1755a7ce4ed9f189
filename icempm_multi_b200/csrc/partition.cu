// partition.cu -- one instance split into slabs of grid columns (partitions),
// on one GPU or one GPU each: the reference's multi-partition layout
// (simulation/gpu_implementation5.cpp:31-204,284-326, kernels
// simulation/kernels.cuh:416-513) for instances larger than one device.
//
// Partition i owns grid columns [x0_i, x0_i + width_i) and the points whose
// stencil base lies there; its grid holds its columns plus `halo` columns on
// each side, so the 2*halo columns around a boundary exist in both
// neighbours.  Per sub-step, on each partition's own stream:
//   reset grid; P2G (one thread per point, FP64 reductions);
//   halo exchange: the 2*halo boundary columns of mass and momentum are
//     copied into the neighbour's own receive buffer (cudaMemcpyPeerAsync:
//     NVLink between GPUs, a device copy on one GPU) and added there, so both
//     sides hold the full sums (the receive buffers alternate by step parity:
//     a partition may run one step ahead of its neighbour's add);
//   grid update; G2P;
//   every UpdateEveryNthStep / PointTransferFrequency steps, points whose
//     base has moved more than 3 columns past the slab leave it
//     (simulation/kernels.cuh:416-461): they are packed into the partition's
//     outgoing buffer and disabled; each neighbour then appends them to its
//     own point array, reading the outgoing buffer and its count directly
//     from the sender's memory (peer loads) -- no host round trip.
// Each node's indenter force is counted by the partition owning its column
// (the reference adds the overlap columns' forces in both partitions).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/icempm.h"
#include "kernels_simple.cuh"

using namespace icy_dev;

StepParams icy_step_params(const icy_sim_params &p);
void icy_set_error(const char *where, cudaError_t e);
void icy_set_error_msg(const std::string &m);

namespace {

constexpr int FLY = 3;                 // columns past the slab before a point moves (kernels.cuh:418)
constexpr int XFER_WORDS = 17;         // a migrating point: 16 HSSOA values + its upload index

struct Slab {
    int device = 0;
    cudaStream_t s = nullptr;
    int x0 = 0, width = 0;             // grid columns [x0, x0 + width)
    long n_nodes = 0;                  // GridY * (width + 2 halo)
    double *grid = nullptr;            // m, px, py, vx, vy: 5 * n_nodes
    double *pts = nullptr;             // 16 HSSOA lines of `pitch` doubles
    long pitch = 0;
    unsigned cap = 0;
    int *oidx = nullptr;               // upload index of each slot (-1: moved away)
    int *count = nullptr;              // [0] slots in use, [1] points appended this exchange
    int *xfer_n = nullptr;             // [0] to the left, [1] to the right
    double *out[2] = {nullptr, nullptr};       // outgoing points, left / right
    double *halo_in[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};   // [side][step parity]
    double *acc = nullptr;             // indenter force bins
    int *status = nullptr;
    cudaEvent_t ev_halo = nullptr, ev_moved = nullptr;
};

#define CKP(call)                                                                 \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) { icy_set_error(#call, e_); return ICY_ERR_CUDA; } \
    } while (0)

// boundary columns shared with the neighbour: [m, px, py] x 2 halo columns
__global__ void k_part_halo_add(double *grid, long n_nodes, long first, long count, const double *in)
{
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= count) return;
#pragma unroll
    for (int a = 0; a < 3; a++) grid[a * n_nodes + first + k] += in[a * count + k];
}

__global__ void k_part_p2g(StepParams P, const double *__restrict__ pts, long pitch, const int *count, GridView g,
                           int *status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count[0]) p2g_one(P, pts, pitch, i, g, status);
}

__global__ void k_part_g2p(StepParams P, double *__restrict__ pts, long pitch, const int *count, GridView g,
                           int recordPQ, int *status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count[0]) g2p_one(P, pts, pitch, i, g, recordPQ, status);
}

// After G2P on an exchange step: a point whose base lies more than FLY
// columns past the slab is packed into the outgoing buffer of its side and
// disabled here (kernels.cuh:416-461); a full buffer keeps it for the next
// exchange, as the reference does.
__global__ void k_part_pack(double hinv, double *__restrict__ pts, long pitch, int *oidx, const int *count, int x0,
                            int width, double *out_left, double *out_right, int *xfer_n, int xcap)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count[0]) return;
    const long long util = __double_as_longlong(pts[i]);
    if (util & kDisabled) return;
    const int bx = (int)(pts[i + pitch * 4] * hinv - 0.5);
    int side = -1;
    if (bx - x0 < -FLY) side = 0;
    else if (bx - (x0 + width - 3) > FLY) side = 1;
    if (side < 0) return;
    const int k = atomicAdd(xfer_n + side, 1);
    if (k >= xcap) return;
    double *o = (side ? out_right : out_left) + (long)k * XFER_WORDS;
#pragma unroll
    for (int l = 0; l < 16; l++) o[l] = pts[i + pitch * l];
    o[16] = (double)oidx[i];
    pts[i] = __longlong_as_double((long long)kDisabled);
    oidx[i] = -1;
}

// Appends the points the neighbours packed (their outgoing buffers and counts,
// read from the neighbours' memory) after this partition's slots.
__global__ void k_part_append(double *__restrict__ pts, long pitch, int *oidx, int *count, unsigned cap,
                              const double *from_left, const int *n_left, const double *from_right,
                              const int *n_right, int xcap, int *status)
{
    const int nl = from_left ? min(*n_left, xcap) : 0, nr = from_right ? min(*n_right, xcap) : 0;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= nl + nr) return;
    const long slot = (long)count[0] + j;
    if (slot >= (long)cap) {   // no space for incoming points (kernels.cuh:506)
        *status = 5;
        return;
    }
    const double *src = j < nl ? from_left + (long)j * XFER_WORDS : from_right + (long)(j - nl) * XFER_WORDS;
#pragma unroll
    for (int l = 0; l < 16; l++) pts[slot + pitch * l] = src[l];
    oidx[slot] = (int)src[16];
    if (j == 0) count[1] = nl + nr;
}

__global__ void k_part_count(int *count, unsigned cap)
{
    count[0] = (int)min((unsigned)(count[0] + count[1]), cap);
    count[1] = 0;
}

}  // namespace

struct icy_part {
    icy_sim_params prm{};
    StepParams P{};
    int n = 0, halo = 0, xcap = 0;
    std::vector<Slab> s;
    unsigned size = 0;                 // points uploaded
    int64_t steps_done = 0;
};

static GridView slab_view(const icy_part *h, const Slab &q)
{
    GridView g;
    g.m = q.grid;
    g.px = q.grid + q.n_nodes;
    g.py = q.grid + 2 * q.n_nodes;
    g.vx = q.grid + 3 * q.n_nodes;
    g.vy = q.grid + 4 * q.n_nodes;
    g.ny = h->prm.GridY;
    g.halo = h->halo - q.x0;
    g.xlo = q.x0 - h->halo;
    g.xhi = q.x0 + q.width + h->halo - 3;
    const int last = &q == &h->s.back();
    g.flo = &q == &h->s.front() ? -(1 << 30) : q.x0;
    g.fhi = last ? (1 << 30) : q.x0 + q.width;
    return g;
}

static void free_slab(Slab &q)
{
    if (q.s) {
        cudaSetDevice(q.device);
        cudaStreamSynchronize(q.s);
    }
    void *ptrs[] = {q.grid, q.pts, q.oidx, q.count, q.xfer_n, q.out[0], q.out[1], q.halo_in[0][0], q.halo_in[0][1],
                    q.halo_in[1][0], q.halo_in[1][1], q.acc, q.status};
    for (void *p : ptrs)
        if (p) cudaFree(p);
    if (q.ev_halo) cudaEventDestroy(q.ev_halo);
    if (q.ev_moved) cudaEventDestroy(q.ev_moved);
    if (q.s) cudaStreamDestroy(q.s);
    q = Slab{};
}

extern "C" {

int icy_part_plan(const icy_sim_params *p, const double *hssoa, unsigned capacity, unsigned size, int n_partitions,
                  int *x0, int *width, unsigned *first, unsigned *count)
{
    // GPU_Implementation5::split_hssoa_into_partitions (gpu_implementation5.cpp:284-326):
    // points sorted by cell, equal shares, each boundary at the x cell of the
    // first point of the next share
    if (!p || !hssoa || n_partitions < 1 || !x0 || !width || !first || !count || size > capacity)
        return ICY_ERR_INVALID_ARGUMENT;
    unsigned done = 0;
    int off = 0;
    for (int i = 0; i < n_partitions; i++) {
        const unsigned share = (size - done) / (unsigned)(n_partitions - i);
        x0[i] = off;
        first[i] = done;
        count[i] = share;
        if (i < n_partitions - 1) {
            const double x = hssoa[(size_t)capacity * ICY_POSX + done + share];
            const int cell = (int)(x * p->cellsize_inv + 0.5);   // ProxyPoint::getXIndex (proxypoint2d.cpp)
            width[i] = cell - off;
            off = cell;
        } else {
            width[i] = p->GridXTotal - off;
        }
        // a slab narrower than both boundary regions would let the points of the
        // slabs two away reach columns that no exchange covers
        if (width[i] < 2 * p->GridHaloSize) {
            icy_set_error_msg("icy_part_plan: a slab of " + std::to_string(width[i]) + " columns, fewer than 2 x " +
                              "GridHaloSize: use fewer partitions");
            return ICY_ERR_INVALID_ARGUMENT;
        }
        done += share;
    }
    return ICY_OK;
}

int icy_part_create(const icy_sim_params *p, int n_partitions, const int *devices, unsigned capacity_per_partition,
                    icy_part **out)
{
    if (!p || !out || n_partitions < 1 || n_partitions > 64 || capacity_per_partition == 0 ||
        p->UpdateEveryNthStep < 1 || p->PointTransferFrequency < 1 || p->GridHaloSize < 4)
        return ICY_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    icy_part *h = new icy_part();
    h->prm = *p;
    h->P = icy_step_params(*p);
    h->n = n_partitions;
    h->halo = p->GridHaloSize;
    h->s.resize(n_partitions);
    h->xcap = std::max(64, (int)(capacity_per_partition * std::max(p->PointsTransferBufferFraction, 0.01)));
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) {
        delete h;
        icy_set_error_msg("icy_part_create: no CUDA device");
        return ICY_ERR_CUDA;
    }
    for (int i = 0; i < n_partitions; i++) {
        Slab &q = h->s[i];
        q.device = devices ? devices[i] : 0;
        if (q.device < 0 || q.device >= ndev) {
            for (Slab &r : h->s) free_slab(r);
            delete h;
            return ICY_ERR_INVALID_ARGUMENT;
        }
        q.cap = capacity_per_partition;
        q.pitch = ((long)capacity_per_partition + 31) / 32 * 32;
    }
    // peer access between neighbours on different devices (NVLink loads and copies)
    for (int i = 0; i + 1 < n_partitions; i++) {
        const int a = h->s[i].device, b = h->s[i + 1].device;
        if (a == b) continue;
        for (int k = 0; k < 2; k++) {
            const int from = k ? b : a, to = k ? a : b;
            int ok = 0;
            cudaDeviceCanAccessPeer(&ok, from, to);
            if (!ok) {
                for (Slab &r : h->s) free_slab(r);
                delete h;
                icy_set_error_msg("icy_part_create: no peer access between neighbouring partitions' devices");
                return ICY_ERR_NOT_SUPPORTED;
            }
            cudaSetDevice(from);
            const cudaError_t e = cudaDeviceEnablePeerAccess(to, 0);
            if (e != cudaSuccess && e != cudaErrorPeerAccessAlreadyEnabled) {
                for (Slab &r : h->s) free_slab(r);
                delete h;
                icy_set_error("cudaDeviceEnablePeerAccess", e);
                return ICY_ERR_CUDA;
            }
            cudaGetLastError();
        }
    }
    *out = h;
    return ICY_OK;
}

static int slab_allocate(icy_part *h, Slab &q)
{
    const icy_sim_params &p = h->prm;
    CKP(cudaSetDevice(q.device));
    if (!q.s) CKP(cudaStreamCreateWithFlags(&q.s, cudaStreamNonBlocking));
    q.n_nodes = (long)p.GridY * (q.width + 2 * h->halo);
    const long hcount = 3L * 2 * h->halo * p.GridY;
    auto al = [&](void **ptr, size_t bytes) { return cudaMalloc(ptr, std::max<size_t>(bytes, 16)); };
    cudaError_t e;
    if ((e = al((void **)&q.grid, sizeof(double) * 5 * q.n_nodes)) != cudaSuccess ||
        (e = al((void **)&q.pts, sizeof(double) * 16 * q.pitch)) != cudaSuccess ||
        (e = al((void **)&q.oidx, sizeof(int) * q.pitch)) != cudaSuccess ||
        (e = al((void **)&q.count, sizeof(int) * 2)) != cudaSuccess ||
        (e = al((void **)&q.xfer_n, sizeof(int) * 2)) != cudaSuccess ||
        (e = al((void **)&q.out[0], sizeof(double) * XFER_WORDS * h->xcap)) != cudaSuccess ||
        (e = al((void **)&q.out[1], sizeof(double) * XFER_WORDS * h->xcap)) != cudaSuccess ||
        (e = al((void **)&q.acc, sizeof(double) * 2 * p.n_indenter_subdivisions)) != cudaSuccess ||
        (e = al((void **)&q.status, sizeof(int))) != cudaSuccess) {
        icy_set_error("cudaMalloc(partition)", e);
        return ICY_ERR_OUT_OF_MEMORY;
    }
    for (int side = 0; side < 2; side++)
        for (int par = 0; par < 2; par++)
            if ((e = al((void **)&q.halo_in[side][par], sizeof(double) * hcount)) != cudaSuccess) {
                icy_set_error("cudaMalloc(partition halo)", e);
                return ICY_ERR_OUT_OF_MEMORY;
            }
    CKP(cudaEventCreateWithFlags(&q.ev_halo, cudaEventDisableTiming));
    CKP(cudaEventCreateWithFlags(&q.ev_moved, cudaEventDisableTiming));
    CKP(cudaMemsetAsync(q.grid, 0, sizeof(double) * 5 * q.n_nodes, q.s));
    CKP(cudaMemsetAsync(q.pts, 0, sizeof(double) * 16 * q.pitch, q.s));
    CKP(cudaMemsetAsync(q.count, 0, sizeof(int) * 2, q.s));
    CKP(cudaMemsetAsync(q.xfer_n, 0, sizeof(int) * 2, q.s));
    CKP(cudaMemsetAsync(q.acc, 0, sizeof(double) * 2 * p.n_indenter_subdivisions, q.s));
    CKP(cudaMemsetAsync(q.status, 0, sizeof(int), q.s));
    return ICY_OK;
}

int icy_part_upload(icy_part *h, const double *hssoa, unsigned capacity, unsigned size)
{
    if (!h || (!hssoa && size)) return ICY_ERR_INVALID_ARGUMENT;
    std::vector<int> x0(h->n), width(h->n);
    std::vector<unsigned> first(h->n), count(h->n);
    if (int rc = icy_part_plan(&h->prm, hssoa, capacity, size, h->n, x0.data(), width.data(), first.data(),
                               count.data()))
        return rc;
    for (int i = 0; i < h->n; i++) {
        Slab &q = h->s[i];
        if (count[i] > q.cap) return ICY_ERR_CAPACITY;
        if (q.grid && q.width != width[i]) {   // a new split: the grid size changes
            const int dev = q.device;
            const unsigned cap = q.cap;
            const long pitch = q.pitch;
            free_slab(q);
            q.device = dev;
            q.cap = cap;
            q.pitch = pitch;
        }
        q.x0 = x0[i];
        q.width = width[i];
        if (!q.grid)
            if (int rc = slab_allocate(h, q)) return rc;
        CKP(cudaSetDevice(q.device));
        if (count[i])
            CKP(cudaMemcpy2DAsync(q.pts, sizeof(double) * q.pitch, hssoa + first[i], sizeof(double) * capacity,
                                  sizeof(double) * count[i], 16, cudaMemcpyHostToDevice, q.s));
        std::vector<int> idx(std::max(count[i], 1u));
        for (unsigned k = 0; k < count[i]; k++) idx[k] = (int)(first[i] + k);
        CKP(cudaMemcpyAsync(q.oidx, idx.data(), sizeof(int) * count[i], cudaMemcpyHostToDevice, q.s));
        const int c[2] = {(int)count[i], 0};
        CKP(cudaMemcpyAsync(q.count, c, sizeof(c), cudaMemcpyHostToDevice, q.s));
        CKP(cudaStreamSynchronize(q.s));   // the host vectors above go out of scope
    }
    h->size = size;
    return ICY_OK;
}

int icy_part_step(icy_part *h, int step0, int nsteps, double *sim_time)
{
    if (!h || !sim_time || nsteps < 0 || h->s.empty() || !h->s[0].grid) return ICY_ERR_INVALID_ARGUMENT;
    const icy_sim_params &p = h->prm;
    const StepParams &P = h->P;
    const int tpb = 256;
    const long hcols = 2L * h->halo * p.GridY;   // nodes of the shared boundary columns
    const int every = std::max(1, p.UpdateEveryNthStep / p.PointTransferFrequency);
    double t = *sim_time;
    for (int k = 0; k < nsteps; k++) {
        // icy::Model::Step sub-step (simulation/model.cpp:40-52)
        t += p.InitialTimeStep;
        const double ind_x = p.indenter_x_initial + t * p.IndVelocity;
        const int step = step0 + k;
        const int par = step & 1;
        const bool rec = step % p.UpdateEveryNthStep == 0;
        const bool xfer = h->n > 1 && step % every == 0;
        // reset grid, P2G, boundary columns to the neighbours
        for (int i = 0; i < h->n; i++) {
            Slab &q = h->s[i];
            CKP(cudaSetDevice(q.device));
            const GridView g = slab_view(h, q);
            CKP(cudaMemsetAsync(q.grid, 0, sizeof(double) * 3 * q.n_nodes, q.s));
            k_part_p2g<<<(q.cap + tpb - 1) / tpb, tpb, 0, q.s>>>(P, q.pts, q.pitch, q.count, g, q.status);
            CKP(cudaGetLastError());
            for (int side = 0; side < 2; side++) {
                const int j = side ? i + 1 : i - 1;
                if (j < 0 || j >= h->n) continue;
                Slab &r = h->s[j];
                // my left boundary columns (local 0 .. 2 halo) go to the left neighbour's
                // right receive buffer, my right ones (local width .. width + 2 halo) to
                // the right neighbour's left buffer
                const long first = side ? (long)q.width * p.GridY : 0;
                for (int a = 0; a < 3; a++)
                    CKP(cudaMemcpyPeerAsync(r.halo_in[1 - side][par] + a * hcols, r.device,
                                            q.grid + a * q.n_nodes + first, q.device, sizeof(double) * hcols, q.s));
            }
            CKP(cudaEventRecord(q.ev_halo, q.s));
        }
        // add the neighbours' boundary columns, update, G2P, pack the leaving points
        for (int i = 0; i < h->n; i++) {
            Slab &q = h->s[i];
            CKP(cudaSetDevice(q.device));
            const GridView g = slab_view(h, q);
            for (int side = 0; side < 2; side++) {
                const int j = side ? i + 1 : i - 1;
                if (j < 0 || j >= h->n) continue;
                CKP(cudaStreamWaitEvent(q.s, h->s[j].ev_halo, 0));
                const long first = side ? (long)q.width * p.GridY : 0;
                k_part_halo_add<<<(unsigned)((hcols + tpb - 1) / tpb), tpb, 0, q.s>>>(q.grid, q.n_nodes, first, hcols,
                                                                                    q.halo_in[side][par]);
                CKP(cudaGetLastError());
            }
            const long nb = (q.n_nodes + tpb - 1) / tpb;
            k_update_simple<<<(unsigned)nb, tpb, sizeof(double) * 2 * P.nsub, q.s>>>(P, g, q.n_nodes, ind_x,
                                                                                   p.indenter_y, q.acc);
            CKP(cudaGetLastError());
            k_part_g2p<<<(q.cap + 127) / 128, 128, 0, q.s>>>(P, q.pts, q.pitch, q.count, g, rec ? 1 : 0, q.status);
            CKP(cudaGetLastError());
            if (xfer) {
                CKP(cudaMemsetAsync(q.xfer_n, 0, sizeof(int) * 2, q.s));
                k_part_pack<<<(q.cap + tpb - 1) / tpb, tpb, 0, q.s>>>(P.hinv, q.pts, q.pitch, q.oidx, q.count, q.x0,
                                                                    q.width, q.out[0], q.out[1], q.xfer_n, h->xcap);
                CKP(cudaGetLastError());
            }
            CKP(cudaEventRecord(q.ev_moved, q.s));
        }
        if (!xfer) continue;
        // each partition appends what its neighbours packed for it
        for (int i = 0; i < h->n; i++) {
            Slab &q = h->s[i];
            CKP(cudaSetDevice(q.device));
            const Slab *L = i > 0 ? &h->s[i - 1] : nullptr, *R = i + 1 < h->n ? &h->s[i + 1] : nullptr;
            if (L) CKP(cudaStreamWaitEvent(q.s, L->ev_moved, 0));
            if (R) CKP(cudaStreamWaitEvent(q.s, R->ev_moved, 0));
            k_part_append<<<(2 * h->xcap + tpb - 1) / tpb, tpb, 0, q.s>>>(
                q.pts, q.pitch, q.oidx, q.count, q.cap, L ? L->out[1] : nullptr, L ? L->xfer_n + 1 : nullptr,
                R ? R->out[0] : nullptr, R ? R->xfer_n : nullptr, h->xcap, q.status);
            CKP(cudaGetLastError());
            k_part_count<<<1, 1, 0, q.s>>>(q.count, q.cap);
            CKP(cudaGetLastError());
            CKP(cudaEventRecord(q.ev_moved, q.s));
        }
        // the outgoing buffers may be refilled only after both neighbours appended
        for (int i = 0; i < h->n; i++) {
            Slab &q = h->s[i];
            CKP(cudaSetDevice(q.device));
            if (i > 0) CKP(cudaStreamWaitEvent(q.s, h->s[i - 1].ev_moved, 0));
            if (i + 1 < h->n) CKP(cudaStreamWaitEvent(q.s, h->s[i + 1].ev_moved, 0));
        }
    }
    h->steps_done += nsteps;
    *sim_time = t;
    return ICY_OK;
}

int icy_part_download(icy_part *h, double *hssoa, unsigned capacity, unsigned *size, double *bins)
{
    if (!h || !hssoa || capacity < h->size) return ICY_ERR_INVALID_ARGUMENT;
    const int nb = 2 * h->prm.n_indenter_subdivisions;
    if (bins) std::fill(bins, bins + nb, 0.0);
    int code = 0;
    unsigned seen = 0;
    std::vector<double> buf, b(nb);
    std::vector<int> oidx;
    for (int i = 0; i < h->n; i++) {
        Slab &q = h->s[i];
        CKP(cudaSetDevice(q.device));
        int c[2] = {0, 0}, st = 0;
        CKP(cudaMemcpyAsync(c, q.count, sizeof(c), cudaMemcpyDeviceToHost, q.s));
        CKP(cudaMemcpyAsync(&st, q.status, sizeof(int), cudaMemcpyDeviceToHost, q.s));
        CKP(cudaMemcpyAsync(b.data(), q.acc, sizeof(double) * nb, cudaMemcpyDeviceToHost, q.s));
        CKP(cudaStreamSynchronize(q.s));
        if (st && !code) code = st;
        if (bins)
            for (int k = 0; k < nb; k++) bins[k] += b[k];
        const unsigned n = (unsigned)c[0];
        buf.resize((size_t)16 * std::max(n, 1u));
        oidx.resize(std::max(n, 1u));
        if (n) {
            CKP(cudaMemcpy2DAsync(buf.data(), sizeof(double) * n, q.pts, sizeof(double) * q.pitch, sizeof(double) * n,
                                  16, cudaMemcpyDeviceToHost, q.s));
            CKP(cudaMemcpyAsync(oidx.data(), q.oidx, sizeof(int) * n, cudaMemcpyDeviceToHost, q.s));
            CKP(cudaStreamSynchronize(q.s));
        }
        for (unsigned k = 0; k < n; k++) {
            const int o = oidx[k];
            if (o < 0) continue;   // moved to a neighbour
            if ((unsigned)o >= h->size) {
                icy_set_error_msg("icy_part_download: corrupt upload index");
                return ICY_ERR_POINT_COUNT;
            }
            for (int l = 0; l < 16; l++) hssoa[(size_t)capacity * l + o] = buf[(size_t)n * l + k];
            seen++;
        }
    }
    if (size) *size = h->size;
    if (code) return code;
    if (seen != h->size) {
        icy_set_error_msg("icy_part_download: points lost between partitions");
        return ICY_ERR_POINT_COUNT;
    }
    return ICY_OK;
}

int icy_part_info(icy_part *h, int part, int *x0, int *width, unsigned *count, int *device)
{
    if (!h || part < 0 || part >= h->n) return ICY_ERR_INVALID_ARGUMENT;
    const Slab &q = h->s[part];
    if (x0) *x0 = q.x0;
    if (width) *width = q.width;
    if (device) *device = q.device;
    if (count) {
        int c[2] = {0, 0};
        if (q.count) {
            CKP(cudaSetDevice(q.device));
            CKP(cudaMemcpyAsync(c, q.count, sizeof(c), cudaMemcpyDeviceToHost, q.s));
            CKP(cudaStreamSynchronize(q.s));
        }
        *count = (unsigned)c[0];
    }
    return ICY_OK;
}

int icy_part_destroy(icy_part *h)
{
    if (!h) return ICY_OK;
    for (Slab &q : h->s) free_slab(q);
    delete h;
    return ICY_OK;
}

}  // extern "C"
