// kernels_tiled.cuh -- binned, tile-staged FP64 step kernels (the fast path).
//
// Points are kept sorted by the cell of their stencil base node, cells grouped
// in tiles of TX x TY bases.  One CTA owns one tile at a time:
//   * the node velocities of the tile's region (its bases, a drift margin of
//     RM cells and the +2 stencil reach) are staged in shared memory;
//   * phase 1, one thread per point (coalesced): G2P + return mapping of step
//     n, the new state is written back, and the point's P2G moments for step
//     n+1 (mass, momentum, affine/stress matrix, base, offset) go to shared
//     memory -- the point state is read once and written once per step;
//   * phase 2, one thread per cell: the 27 node contributions of the cell's
//     points are summed in registers -- no atomics;
//   * phase 3, one thread per node: each node adds the partials of the (up to)
//     9 cells whose stencil covers it, in a fixed order, and the tile's
//     non-empty nodes are flushed to the global grid with one FP64 reduction
//     per value, marking the node tiles written.
// The grid update then visits only marked node tiles (simulation/kernels.cuh:164-301)
// and zeroes the accumulators for the next step.  A point whose base is no
// longer its sorted cell (it moved since the last binning) is still handled
// exactly: by shared-memory atomics inside the staged region, through global
// memory beyond it; such points are counted so the host can re-bin.
#pragma once
#include "kernels_simple.cuh"

namespace icy_dev {

constexpr int TX = 16, TY = 8, TT = TX * TY;   // stencil bases (cells) per tile
constexpr int RM = 1;                          // drift margin (cells) of the staged region
constexpr int RX = TX + 2 + 2 * RM, RY = TY + 2 + 2 * RM, RN = RX * RY;
constexpr int TILE_THREADS = 256;
constexpr int CAP = 640;                       // points staged per chunk
constexpr int NMOM = 9;                        // P2G moments per point
constexpr int BASE_NONE = 0x7fffffff;
constexpr size_t TILE_DYN_SMEM = sizeof(double) * NMOM * CAP + sizeof(int) * CAP;
static_assert(27 * TT <= NMOM * CAP, "cell partials alias the moment buffer");

// Tiles cover bases bx in [-halo, -halo + ntx*TX), by in [0, nty*TY);
// tile id = ty*ntx + tx; cell key = tile*TT + lx*TY + ly; node tiles use the
// same partition of the nodes.
struct TileGeom {
    int ntx, nty, ntiles;
    __device__ __forceinline__ int cell_key(int bx, int by, int halo) const
    {
        const int gx = bx + halo;
        return ((by / TY) * ntx + gx / TX) * TT + (gx % TX) * TY + (by % TY);
    }
};

struct TileArgs {
    StepParams P;
    TileGeom G;
    GridView g;
    double *pts;
    long pitch;
    const int *cell_start;   // ntiles*TT + 2 entries; [ntiles*TT] = start of the disabled bucket
    const int *active;       // tiles with points, ascending
    const int *n_active;
    unsigned *flags;         // node tiles written by P2G since the last update
    int *status;
    unsigned long long *moved;  // points whose base is not their sorted cell (re-binning hint)
    const GrainConst *grain_tab;  // failure-surface constants per grain slot
    int record_pq;
};

__global__ void k_grain_table(StepParams P, GrainConst *tab)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < GRAIN_TAB) tab[s] = grain_constants(P, s / GRAIN_N11 - 29, s % GRAIN_N11 - 10);
}

__device__ __forceinline__ bool node_in_grid(const StepParams &P, int gx, int gy)
{
    return gx >= -P.halo && gx < P.gridx + P.halo && gy >= 0 && gy < P.gridy;
}

__device__ __forceinline__ int pack_base(int bx, int by) { return ((bx + 32768) << 16) | by; }
__device__ __forceinline__ void unpack_base(int k, int &bx, int &by)
{
    bx = (int)((unsigned)k >> 16) - 32768;
    by = k & 0xffff;
}

// ---------------------------------------------------------------- scans
// Exclusive block scan of one int per thread (NT threads); returns the prefix.
template <int NT>
__device__ __forceinline__ int block_exclusive_scan(int v, int *s_warp, int &total)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < NT / 32 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < NT / 32) s_warp[lane] = s;
    }
    __syncthreads();
    const int prefix = (w > 0 ? s_warp[w - 1] : 0) + x - v;
    total = s_warp[NT / 32 - 1];
    __syncthreads();
    return prefix;
}

constexpr int SCAN_NT = 256, SCAN_PER = 16, SCAN_BLOCK = SCAN_NT * SCAN_PER;

__global__ void __launch_bounds__(SCAN_NT) k_scan_reduce(const int *in, int n, int *block_sum)
{
    __shared__ int s_warp[SCAN_NT / 32];
    const long base = (long)blockIdx.x * SCAN_BLOCK;
    int s = 0;
    for (int k = 0; k < SCAN_PER; k++) {
        const long i = base + (long)k * SCAN_NT + threadIdx.x;
        if (i < n) s += in[i];
    }
    int total;
    block_exclusive_scan<SCAN_NT>(s, s_warp, total);
    if (threadIdx.x == 0) block_sum[blockIdx.x] = total;
}

// one CTA: exclusive scan of the nb block sums, in place
__global__ void __launch_bounds__(1024) k_scan_blocks(int *block_sum, int nb)
{
    __shared__ int s_warp[32];
    const int per = (nb + 1023) / 1024;
    const int b = min((int)threadIdx.x * per, nb), e = min(b + per, nb);
    int s = 0;
    for (int k = b; k < e; k++) s += block_sum[k];
    int total;
    int run = block_exclusive_scan<1024>(s, s_warp, total);
    for (int k = b; k < e; k++) {
        const int c = block_sum[k];
        block_sum[k] = run;
        run += c;
    }
}

// start[i] = exclusive prefix of in[] (n items); start[n] = total
__global__ void __launch_bounds__(SCAN_NT) k_scan_apply(const int *in, int n, const int *block_off, int *start)
{
    __shared__ int s_warp[SCAN_NT / 32];
    const long base = (long)blockIdx.x * SCAN_BLOCK + (long)threadIdx.x * SCAN_PER;
    int v[SCAN_PER], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER; k++) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int run = block_exclusive_scan<SCAN_NT>(s, s_warp, total) + block_off[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_PER; k++) {
        if (base + k < n) start[base + k] = run;
        run += v[k];
    }
    if (base + SCAN_PER >= n && base < n) start[n] = run;   // the thread holding the last item
}

// one CTA: ordered list of tiles that hold points
__global__ void __launch_bounds__(1024) k_tiles_active(const int *cell_start, int ntiles, int *active, int *n_active)
{
    __shared__ int s_warp[32];
    const int per = (ntiles + 1023) / 1024;
    const int b = min((int)threadIdx.x * per, ntiles), e = min(b + per, ntiles);
    int s = 0;
    for (int t = b; t < e; t++) s += cell_start[(long)(t + 1) * TT] > cell_start[(long)t * TT];
    int total;
    int run = block_exclusive_scan<1024>(s, s_warp, total);
    for (int t = b; t < e; t++)
        if (cell_start[(long)(t + 1) * TT] > cell_start[(long)t * TT]) active[run++] = t;
    if (threadIdx.x == 0) *n_active = total;
}

// ---------------------------------------------------------------- binning
__global__ void k_bin_count(StepParams P, TileGeom G, const double *__restrict__ pts, long pitch, int n,
                            int *keys, int *ranks, int *counts, int *status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < n;
    int key = G.ntiles * TT;   // disabled / out-of-grid bucket
    if (in) {
        long long u = __double_as_longlong(pts[i]);
        if (!(u & kDisabled)) {
            const double x = pts[i + pitch * 4], y = pts[i + pitch * 5];
            const int bx = (int)(x * P.hinv - 0.5), by = (int)(y * P.hinv - 0.5);
            const int e = base_error(P, bx, by);
            if (e) *status = e;
            else key = G.cell_key(bx, by, P.halo);
        }
    }
    const unsigned act = __ballot_sync(0xffffffffu, in);
    if (!in) return;
    // warp-aggregated rank: points are mostly sorted, so lanes share keys
    const unsigned peers = __match_any_sync(act, key);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&counts[key], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    keys[i] = key;
    ranks[i] = base + __popc(peers & ((1u << lane) - 1u));
}

__global__ void k_bin_scatter(const double *__restrict__ src, double *__restrict__ dst, long pitch, int n,
                              const int *__restrict__ keys, const int *__restrict__ ranks,
                              const int *__restrict__ start, const int *__restrict__ oidx_src,
                              int *__restrict__ oidx_dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int d = start[keys[i]] + ranks[i];
#pragma unroll
    for (int l = 0; l < 16; l++) dst[d + pitch * l] = src[i + pitch * l];
    oidx_dst[d] = oidx_src[i];
}

__global__ void k_iota(int *a, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

// HSSOA back in upload order: dst[l][oidx[i]] = src[l][i]
__global__ void k_unpermute(const double *__restrict__ src, double *__restrict__ dst, long pitch, int n,
                            const int *__restrict__ oidx)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int o = oidx[i];
#pragma unroll
    for (int l = 0; l < 16; l++) dst[o + pitch * l] = src[i + pitch * l];
}

// ---------------------------------------------------------------- P2G helpers
// The 27 contributions of one point, in the reference's expression order
// (simulation/kernels.cuh:105-121), handed to `sink(a, b, dm, dpx, dpy)`.
template <typename Sink>
__device__ __forceinline__ void point_contributions(double h, double fx, double fy, double mass, double mvx,
                                                    double mvy, double s00, double s01, double s10, double s11,
                                                    Sink &&sink)
{
    double wx[3], wy[3];
    bspline_weights(fx, wx);
    bspline_weights(fy, wy);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double d0 = ((double)a - fx) * h;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const double W = wx[a] * wy[b];
            const double d1 = ((double)b - fy) * h;
            sink(a, b, W * mass, W * (mvx + (s00 * d0 + s01 * d1)), W * (mvy + (s10 * d0 + s11 * d1)));
        }
    }
}

// P2G of one point straight into the global grid (its base left the staged region).
__device__ __noinline__ void p2g_global(GridView g, unsigned *flags, int ntx, int halo, double h, int bx, int by,
                                        double fx, double fy, double mass, double mvx, double mvy, double s00,
                                        double s01, double s10, double s11)
{
    point_contributions(h, fx, fy, mass, mvx, mvy, s00, s01, s10, s11,
                        [&](int a, int b, double dm, double dpx, double dpy) {
                            const long k = g.idx(bx + a, by + b);
                            atomicAdd(g.m + k, dm);
                            atomicAdd(g.px + k, dpx);
                            atomicAdd(g.py + k, dpy);
                        });
    const int t0x = (bx + halo) / TX, t1x = (bx + 2 + halo) / TX;
    const int t0y = by / TY, t1y = (by + 2) / TY;
    flags[t0y * ntx + t0x] = 1u;
    flags[t0y * ntx + t1x] = 1u;
    flags[t1y * ntx + t0x] = 1u;
    flags[t1y * ntx + t1x] = 1u;
}

// ---------------------------------------------------------------- phase 1
// G2P + return mapping of point i (if DO_G2P) and its P2G moments (if DO_P2G)
// into slot j of the shared moment buffer.
template <bool DO_G2P, bool DO_P2G, bool WRITE_VB>
__device__ __forceinline__ void tile_point(const TileArgs &A, long i, int j, int RX0, int RY0,
                                           const double (*s_v)[RN], double *s_mom, int *s_base)
{
    const StepParams &P = A.P;
    double *__restrict__ pts = A.pts;
    const long pitch = A.pitch;
    long long util = __double_as_longlong(pts[i]);
    if (util & kDisabled) {
        if (DO_P2G) s_base[j] = BASE_NONE;
        return;
    }
    const bool liquid = (util & kLiquid) != 0;
    double x = pts[i + pitch * 4], y = pts[i + pitch * 5];
    M2<double> F{pts[i + pitch * 8], pts[i + pitch * 9], pts[i + pitch * 10], pts[i + pitch * 11]};
    double Jp = pts[i + pitch * 3];
    double vx, vy;
    M2<double> B;
    if (DO_G2P) {
        const int bx = (int)(x * P.hinv - 0.5), by = (int)(y * P.hinv - 0.5);
        const double fx = x * P.hinv - (double)bx, fy = y * P.hinv - (double)by;
        const int e = base_error(P, bx, by);
        if (e) {
            *A.status = e;
            if (DO_P2G) s_base[j] = BASE_NONE;
            return;
        }
        double wx[3], wy[3];
        bspline_weights(fx, wx);
        bspline_weights(fy, wy);
        vx = 0; vy = 0;
        B = {0, 0, 0, 0};
        const int lx = bx - RX0, ly = by - RY0;
        const bool staged = lx >= 0 && lx + 2 < RX && ly >= 0 && ly + 2 < RY;
        const double s4 = 4. * P.hinv;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const double d0 = (double)a - fx;
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const double d1 = (double)b - fy;
                const double w = wx[a] * wy[b];
                double nvx, nvy;
                if (staged) {
                    const int k = (lx + a) * RY + (ly + b);
                    nvx = s_v[0][k];
                    nvy = s_v[1][k];
                } else {
                    const long k = A.g.idx(bx + a, by + b);
                    nvx = A.g.vx[k];
                    nvy = A.g.vy[k];
                }
                vx = vx + w * nvx;
                vy = vy + w * nvy;
                const double s = s4 * w;
                const double snx = s * nvx, sny = s * nvy;
                B.a00 = B.a00 + snx * d0; B.a01 = B.a01 + snx * d1;
                B.a10 = B.a10 + sny * d0; B.a11 = B.a11 + sny * d1;
            }
        }
        x = x + vx * P.dt;
        y = y + vy * P.dt;
        const M2<double> Am{1.0 + P.dt * B.a00, P.dt * B.a01, P.dt * B.a10, 1.0 + P.dt * B.a11};
        const M2<double> Fn{Am.a00 * F.a00 + Am.a01 * F.a10, Am.a00 * F.a01 + Am.a01 * F.a11,
                            Am.a10 * F.a00 + Am.a11 * F.a10, Am.a10 * F.a01 + Am.a11 * F.a11};
        F = Fn;
        double ptr = 0, qtr = 0;
        if (liquid) {
            Jp = Jp * (Am.a00 * Am.a11 - Am.a10 * Am.a01);
        } else {
            double Je;
            compute_pq(F, P.mu, P.kappa, Je, ptr, qtr);
            if (!(util & kCrushed)) {
                const GrainConst *gc = A.grain_tab + grain_slot((short)util);
                const GrainConst c{__ldg(&gc->pmin2), __ldg(&gc->k), __ldg(&gc->msq)};
                if (failure_surface_crushed_tab(P, c, ptr, qtr)) util |= kCrushed;
            }
            if (util & kCrushed) return_map(P, F, Jp, ptr, qtr, Je);
        }
        pts[i] = __longlong_as_double(util);
        pts[i + pitch * 3] = Jp;
        pts[i + pitch * 4] = x;
        pts[i + pitch * 5] = y;
        pts[i + pitch * 8] = F.a00; pts[i + pitch * 9] = F.a01;
        pts[i + pitch * 10] = F.a10; pts[i + pitch * 11] = F.a11;
        if (WRITE_VB) {
            pts[i + pitch * 6] = vx; pts[i + pitch * 7] = vy;
            pts[i + pitch * 12] = B.a00; pts[i + pitch * 13] = B.a01;
            pts[i + pitch * 14] = B.a10; pts[i + pitch * 15] = B.a11;
        }
        if (A.record_pq) { pts[i + pitch * 1] = ptr; pts[i + pitch * 2] = qtr; }
    } else {
        vx = pts[i + pitch * 6];
        vy = pts[i + pitch * 7];
        B = {pts[i + pitch * 12], pts[i + pitch * 13], pts[i + pitch * 14], pts[i + pitch * 15]};
    }
    if (DO_P2G) {
        // P2G moments of the (updated) point (simulation/kernels.cuh:57-92)
        const double mass = liquid ? P.mass_water : P.mass_ice;
        const M2<double> tau = liquid ? water_stress(Jp, P.kappa) : kirchhoff(F, P.mu, P.kappa);
        const int bx = (int)(x * P.hinv - 0.5), by = (int)(y * P.hinv - 0.5);
        const int e = base_error(P, bx, by);
        if (e) {
            *A.status = e;
            s_base[j] = BASE_NONE;
            return;
        }
        s_base[j] = pack_base(bx, by);
        s_mom[0 * CAP + j] = x * P.hinv - (double)bx;
        s_mom[1 * CAP + j] = y * P.hinv - (double)by;
        s_mom[2 * CAP + j] = mass;
        s_mom[3 * CAP + j] = vx * mass;
        s_mom[4 * CAP + j] = vy * mass;
        s_mom[5 * CAP + j] = mass * B.a00 - P.dt_vol_Dpinv * tau.a00;
        s_mom[6 * CAP + j] = mass * B.a01 - P.dt_vol_Dpinv * tau.a01;
        s_mom[7 * CAP + j] = mass * B.a10 - P.dt_vol_Dpinv * tau.a10;
        s_mom[8 * CAP + j] = mass * B.a11 - P.dt_vol_Dpinv * tau.a11;
    }
}

// One persistent CTA loop over the non-empty tiles.
//   <true, true, false>  G2P(n) + P2G(n+1)          (steady state of a run)
//   <false, true, false> P2G only                   (first step, per-phase p2g)
//   <true, false, true>  G2P only, writes vel & Bp  (last step, per-phase g2p)
template <bool DO_G2P, bool DO_P2G, bool WRITE_VB>
__global__ void __launch_bounds__(TILE_THREADS, 2) k_tile(TileArgs A)
{
    __shared__ double s_v[2][RN];      // staged node velocities (G2P)
    __shared__ double s_odd[3][RN];    // contributions of points off their sorted cell
    __shared__ int s_cs[TT + 1];       // cell ranges of the tile
    __shared__ unsigned s_touch;
    extern __shared__ double s_dyn[];  // moments [NMOM][CAP] | cell partials [27][TT]; then bases [CAP]
    double *s_mom = s_dyn;
    int *s_base = reinterpret_cast<int *>(s_dyn + NMOM * CAP);
    const StepParams &P = A.P;
    const int na = *A.n_active;
    const int tid = threadIdx.x;
    unsigned moved = 0;
    for (int ti = blockIdx.x; ti < na; ti += gridDim.x) {
        const int t = A.active[ti];
        const int tx = t % A.G.ntx, ty = t / A.G.ntx;
        const int X0 = tx * TX - P.halo, Y0 = ty * TY;
        const int RX0 = X0 - RM, RY0 = Y0 - RM;
        for (int c = tid; c <= TT; c += blockDim.x) s_cs[c] = A.cell_start[(long)t * TT + c];
        if (tid == 0) s_touch = 0;
        for (int k = tid; k < RN; k += blockDim.x) {
            if (DO_G2P) {
                const int gx = RX0 + k / RY, gy = RY0 + k % RY;
                double vx = 0, vy = 0;
                if (node_in_grid(P, gx, gy)) {
                    const long q = A.g.idx(gx, gy);
                    vx = A.g.vx[q];
                    vy = A.g.vy[q];
                }
                s_v[0][k] = vx;
                s_v[1][k] = vy;
            }
            if (DO_P2G) { s_odd[0][k] = 0; s_odd[1][k] = 0; s_odd[2][k] = 0; }
        }
        __syncthreads();
        const int ps = s_cs[0], pe = s_cs[TT];
        if (!DO_P2G) {
            for (int i = ps + tid; i < pe; i += blockDim.x)
                tile_point<DO_G2P, DO_P2G, WRITE_VB>(A, i, 0, RX0, RY0, s_v, s_mom, s_base);
            __syncthreads();
            continue;
        }
        for (int cs = ps; cs < pe; cs += CAP) {
            const int ce = min(cs + CAP, pe);
            // phase 1: one thread per point
            for (int j = tid; j < ce - cs; j += blockDim.x)
                tile_point<DO_G2P, DO_P2G, WRITE_VB>(A, cs + j, j, RX0, RY0, s_v, s_mom, s_base);
            __syncthreads();
            // phase 2: one thread per cell, partials in registers
            double acc[27];
#pragma unroll
            for (int q = 0; q < 27; q++) acc[q] = 0;
            if (tid < TT) {
                const int bxc = X0 + tid / TY, byc = Y0 + tid % TY;
                const int r0 = max(s_cs[tid], cs) - cs, r1 = min(s_cs[tid + 1], ce) - cs;
                for (int j = r0; j < r1; j++) {
                    const int pb = s_base[j];
                    if (pb == BASE_NONE) continue;
                    int bx, by;
                    unpack_base(pb, bx, by);
                    const double fx = s_mom[j], fy = s_mom[CAP + j], mass = s_mom[2 * CAP + j];
                    const double mvx = s_mom[3 * CAP + j], mvy = s_mom[4 * CAP + j];
                    const double s00 = s_mom[5 * CAP + j], s01 = s_mom[6 * CAP + j];
                    const double s10 = s_mom[7 * CAP + j], s11 = s_mom[8 * CAP + j];
                    if (bx == bxc && by == byc) {
                        point_contributions(P.h, fx, fy, mass, mvx, mvy, s00, s01, s10, s11,
                                            [&](int a, int b, double dm, double dpx, double dpy) {
                                                const int q = (a * 3 + b) * 3;
                                                acc[q] += dm;
                                                acc[q + 1] += dpx;
                                                acc[q + 2] += dpy;
                                            });
                    } else {
                        moved++;
                        const int lx = bx - RX0, ly = by - RY0;
                        if (lx >= 0 && lx + 2 < RX && ly >= 0 && ly + 2 < RY) {
                            point_contributions(P.h, fx, fy, mass, mvx, mvy, s00, s01, s10, s11,
                                                [&](int a, int b, double dm, double dpx, double dpy) {
                                                    const int k = (lx + a) * RY + (ly + b);
                                                    atomicAdd(&s_odd[0][k], dm);
                                                    atomicAdd(&s_odd[1][k], dpx);
                                                    atomicAdd(&s_odd[2][k], dpy);
                                                });
                        } else {
                            p2g_global(A.g, A.flags, A.G.ntx, P.halo, P.h, bx, by, fx, fy, mass, mvx, mvy, s00,
                                       s01, s10, s11);
                        }
                    }
                }
            }
            __syncthreads();   // all moments read: the buffer becomes the cell partials
            if (tid < TT) {
#pragma unroll
                for (int q = 0; q < 27; q++) s_mom[q * TT + tid] = acc[q];
            }
            __syncthreads();
            // phase 3: one thread per region node, 9 partials in a fixed order, flush
            unsigned touch = 0;
            for (int k = tid; k < RN; k += blockDim.x) {
                const int i = k / RY, jj = k % RY;        // region coordinates
                const int nx = i - RM, ny = jj - RM;       // node relative to the tile's first base
                double m = 0, px = 0, py = 0;
#pragma unroll
                for (int a = 0; a < 3; a++) {
                    const int cx = nx - a;
                    if (cx < 0 || cx >= TX) continue;
#pragma unroll
                    for (int b = 0; b < 3; b++) {
                        const int cy = ny - b;
                        if (cy < 0 || cy >= TY) continue;
                        const int c = cx * TY + cy, q = (a * 3 + b) * 3;
                        m += s_mom[q * TT + c];
                        px += s_mom[(q + 1) * TT + c];
                        py += s_mom[(q + 2) * TT + c];
                    }
                }
                m += s_odd[0][k]; px += s_odd[1][k]; py += s_odd[2][k];
                s_odd[0][k] = 0; s_odd[1][k] = 0; s_odd[2][k] = 0;
                if (m != 0.0 || px != 0.0 || py != 0.0) {
                    const int gx = RX0 + i, gy = RY0 + jj;   // inside the grid: only valid bases scatter
                    const long q = A.g.idx(gx, gy);
                    atomicAdd(A.g.m + q, m);
                    atomicAdd(A.g.px + q, px);
                    atomicAdd(A.g.py + q, py);
                    const int dx = (gx + P.halo) / TX - tx + 1, dy = gy / TY - ty + 1;
                    touch |= 1u << (dy * 3 + dx);
                }
            }
            touch = __reduce_or_sync(0xffffffffu, touch);
            if ((tid & 31) == 0 && touch) atomicOr(&s_touch, touch);
            __syncthreads();
        }
        if (tid < 9 && ((s_touch >> tid) & 1u)) {
            const int ntx = tx + tid % 3 - 1, nty = ty + tid / 3 - 1;
            A.flags[nty * A.G.ntx + ntx] = 1u;
        }
        __syncthreads();
    }
    if (DO_P2G) {
        moved = __reduce_add_sync(0xffffffffu, moved);
        if ((tid & 31) == 0 && moved) atomicAdd(A.moved, (unsigned long long)moved);
    }
}

// Grid update of the nodes of marked tiles (simulation/kernels.cuh:164-301),
// one thread per node; zeroes the accumulators for the next step.  The marks
// are cleared by the caller afterwards.
__global__ void __launch_bounds__(256) k_update_nodes(StepParams P, TileGeom G, GridView g,
                                                      const unsigned *__restrict__ flags, long n_nodes,
                                                      double ind_x, double ind_y, double *acc)
{
    extern __shared__ double s_acc[];   // 2*nsub
    for (int k = threadIdx.x; k < 2 * P.nsub; k += blockDim.x) s_acc[k] = 0;
    __syncthreads();
    bool any = false;
    const int nn = (int)n_nodes;   // < 2^31 nodes per instance
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < nn; q += gridDim.x * blockDim.x) {
        const int col = q / g.ny;
        const int gx = col - g.halo, gy = q - col * g.ny;
        if (!flags[(gy / TY) * G.ntx + (gx + g.halo) / TX]) continue;
        double vx = 0, vy = 0, fx, fy;
        int bin;
        if (node_update(P, gx, gy, g.m[q], g.px[q], g.py[q], ind_x, ind_y, vx, vy, bin, fx, fy) && bin >= 0) {
            atomicAdd(&s_acc[2 * bin], fx);
            atomicAdd(&s_acc[2 * bin + 1], fy);
            any = true;
        }
        g.vx[q] = vx;
        g.vy[q] = vy;
        g.m[q] = 0.0;
        g.px[q] = 0.0;
        g.py[q] = 0.0;
    }
    if (!__syncthreads_or(any)) return;
    for (int k = threadIdx.x; k < 2 * P.nsub; k += blockDim.x)
        if (s_acc[k] != 0.0) atomicAdd(acc + k, s_acc[k]);
}

}  // namespace icy_dev
