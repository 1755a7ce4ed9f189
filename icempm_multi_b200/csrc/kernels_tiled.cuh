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
#include "tma_pipe.cuh"

namespace icy_dev {

constexpr int TX = 32, TY = 8, TT = TX * TY;   // stencil bases (cells) per tile
constexpr int RM = 1;                          // drift margin (cells) of the staged region
constexpr int RX = TX + 2 + 2 * RM, RY = TY + 2 + 2 * RM, RN = RX * RY;
constexpr int TILE_THREADS = 256;
constexpr int CAP = 1056;                      // points staged per chunk (a tile holds 1,024 at 4 per cell)
constexpr int BASE_NONE = 0x7fffffff;
constexpr int ICY_TIMEOUT_CODE = 108;          // ICY_ERR_TIMEOUT

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
    // the same for tiles of STX x STY cells
    template <int STX, int STY>
    __device__ __forceinline__ int cell_key_s(int bx, int by, int halo) const
    {
        const int gx = bx + halo;
        return ((by / STY) * ntx + gx / STX) * (STX * STY) + (gx % STX) * STY + (by % STY);
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
    int2 *tlist;             // those tiles, each once: (instance, tile)
    unsigned *tlist_n;       // [0] entries in tlist, [1] CTAs done (reset by the update)
    int *status;
    unsigned long long *moved;  // points whose base is not their sorted cell (re-binning hint)
    const GrainConst *grain_tab;  // failure-surface constants per grain slot
    int record_pq;
    int fault_test;          // pipe kernel: leave the first stage unfilled (timeout test)
};

// Marks node tile (tx, ty) as written by P2G since the last grid update and
// appends (inst, ty << 16 | tx) to the list the update visits, once per tile.
__device__ __forceinline__ void mark_tile(unsigned *flags, int2 *tlist, unsigned *tlist_n, int inst, int tx, int ty,
                                          int ntx)
{
    const int t = ty * ntx + tx;
    if (*(volatile unsigned *)(flags + t) == 0u && atomicExch(flags + t, 1u) == 0u)
        tlist[atomicAdd(tlist_n, 1u)] = make_int2(inst, (ty << 16) | tx);
}

// Called by thread 0 of every CTA of a list-driven grid update after its last
// read of the list: the last CTA to finish empties the list for the next step.
__device__ __forceinline__ void tile_list_done(unsigned *tlist_n)
{
    __threadfence();
    if (atomicAdd(tlist_n + 1, 1u) == gridDim.x - 1) {
        tlist_n[0] = 0u;
        tlist_n[1] = 0u;
        __threadfence();
    }
}

static __global__ void k_grain_table(StepParams P, GrainConst *tab)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < GRAIN_TAB) tab[s] = grain_constants(P, s / GRAIN_N11 - 29, s % GRAIN_N11 - 10);
}

template <class PT>
__device__ __forceinline__ bool node_in_grid(const PT &P, int gx, int gy)
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

static __global__ void __launch_bounds__(SCAN_NT) k_scan_reduce(const int *in, int n, int *block_sum)
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
static __global__ void __launch_bounds__(1024) k_scan_blocks(int *block_sum, int nb)
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
static __global__ void __launch_bounds__(SCAN_NT) k_scan_apply(const int *in, int n, const int *block_off, int *start)
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
template <int CELLS = TT>
static __global__ void __launch_bounds__(1024) k_tiles_active(const int *cell_start, int ntiles, int *active, int *n_active)
{
    constexpr int TT = CELLS;   // cells per tile
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
static __global__ void k_bin_count(StepParams P, TileGeom G, const double *__restrict__ pts, long pitch, int n,
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

static __global__ void k_bin_scatter(const double *__restrict__ src, double *__restrict__ dst, long pitch, int n,
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

static __global__ void k_iota(int *a, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) a[i] = i;
}

// HSSOA back in upload order: dst[l][oidx[i]] = src[l][i]
static __global__ void k_unpermute(const double *__restrict__ src, double *__restrict__ dst, long pitch, int n,
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
    // node (a, b) gets W m and W (m v + S d), d = ((a - fx) h, (b - fy) h),
    // W = wx[a] wy[b]; S d is affine in (a, b): c0 + a S(:,0) h + b S(:,1) h
    double wx[3], wy[3];
    bspline_weights(fx, wx);
    bspline_weights(fy, wy);
    const double s00h = s00 * h, s01h = s01 * h, s10h = s10 * h, s11h = s11 * h;
    const double c0x = mvx - (s00h * fx + s01h * fy), c0y = mvy - (s10h * fx + s11h * fy);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double ax = c0x + (double)a * s00h, ay = c0y + (double)a * s10h;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const double W = wx[a] * wy[b];
            sink(a, b, W, W * mass, ax + (double)b * s01h, ay + (double)b * s11h);
        }
    }
}

// P2G of one point straight into the global grid (its base left the staged region).
static __device__ __noinline__ void p2g_global(GridView g, unsigned *flags, int2 *tlist, unsigned *tlist_n, int ntx,
                                               int halo, double h, int bx, int by, double fx, double fy, double mass,
                                               double mvx, double mvy, double s00, double s01, double s10, double s11)
{
    point_contributions(h, fx, fy, mass, mvx, mvy, s00, s01, s10, s11,
                        [&](int a, int b, double W, double dm, double tx, double ty) {
                            const long k = g.idx(bx + a, by + b);
                            atomicAdd(g.m + k, dm);
                            atomicAdd(g.px + k, W * tx);
                            atomicAdd(g.py + k, W * ty);
                        });
    const int t0x = (bx + halo) / TX, t1x = (bx + 2 + halo) / TX;
    const int t0y = by / TY, t1y = (by + 2) / TY;
    mark_tile(flags, tlist, tlist_n, 0, t0x, t0y, ntx);
    if (t1x != t0x) mark_tile(flags, tlist, tlist_n, 0, t1x, t0y, ntx);
    if (t1y != t0y) {
        mark_tile(flags, tlist, tlist_n, 0, t0x, t1y, ntx);
        if (t1x != t0x) mark_tile(flags, tlist, tlist_n, 0, t1x, t1y, ntx);
    }
}

// ---------------------------------------------------------------- per point
// State of one point during G2P (HSSOA fields) plus its p, q on record steps.
struct PointState {
    long long util;
    double x, y, Jp, vx, vy, ptr, qtr;
    M2<double> F, B;
};

// The return mapping (simulation/kernels.cuh:540-545, 623-674) out of line:
// only crushed points take it, and its registers stay out of the tile
// kernel's main path.
struct ReturnMapped { M2<double> F; double Jp; };
static __device__ __noinline__ ReturnMapped return_map_out(const StepParams &P, M2<double> F, double Jp, double ptr,
                                                           double qtr, double Je)
{
    return_map(P, F, Jp, ptr, qtr, Je);
    return ReturnMapped{F, Jp};
}

// G2P + return mapping of one point (simulation/kernels.cuh:305-407).
// vsrc(bx, by, nv) supplies the 3 x 3 node velocities.  Returns false (and
// records the reference's error code) if the stencil leaves the grid.
template <typename VSrc>
__device__ __forceinline__ bool g2p_update(const StepParams &P, const GrainConst *grain_tab, PointState &s,
                                           int *status, VSrc &&vsrc)
{
    const int bx = (int)(s.x * P.hinv - 0.5), by = (int)(s.y * P.hinv - 0.5);
    const double fx = s.x * P.hinv - (double)bx, fy = s.y * P.hinv - (double)by;
    const int e = base_error(P, bx, by);
    if (e) { *status = e; return false; }
    double wx[3], wy[3];
    bspline_weights(fx, wx);
    bspline_weights(fy, wy);
    // v = sum W v_i, Bp = 4/h sum W v_i (i - f)^T (kernels.cuh:357-372), as
    // per-column sums over b with wy, then over a with wx
    double2 nv[9];
    vsrc(bx, by, nv);
    double cvx[3], cvy[3], cbx[3], cby[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double2 n0 = nv[a * 3], n1 = nv[a * 3 + 1], n2 = nv[a * 3 + 2];
        cvx[a] = wy[0] * n0.x + wy[1] * n1.x + wy[2] * n2.x;
        cvy[a] = wy[0] * n0.y + wy[1] * n1.y + wy[2] * n2.y;
        cbx[a] = wy[1] * n1.x + 2.0 * (wy[2] * n2.x);
        cby[a] = wy[1] * n1.y + 2.0 * (wy[2] * n2.y);
    }
    const double vx = wx[0] * cvx[0] + wx[1] * cvx[1] + wx[2] * cvx[2];
    const double vy = wx[0] * cvy[0] + wx[1] * cvy[1] + wx[2] * cvy[2];
    const double sax = wx[1] * cvx[1] + 2.0 * (wx[2] * cvx[2]), say = wx[1] * cvy[1] + 2.0 * (wx[2] * cvy[2]);
    const double sbx = wx[0] * cbx[0] + wx[1] * cbx[1] + wx[2] * cbx[2];
    const double sby = wx[0] * cby[0] + wx[1] * cby[1] + wx[2] * cby[2];
    const double s4 = 4. * P.hinv;
    const M2<double> B{s4 * (sax - fx * vx), s4 * (sbx - fy * vx), s4 * (say - fx * vy), s4 * (sby - fy * vy)};
    s.x = s.x + vx * P.dt;
    s.y = s.y + vy * P.dt;
    const M2<double> Am{1.0 + P.dt * B.a00, P.dt * B.a01, P.dt * B.a10, 1.0 + P.dt * B.a11};
    const M2<double> F = s.F;
    s.F = {Am.a00 * F.a00 + Am.a01 * F.a10, Am.a00 * F.a01 + Am.a01 * F.a11,
           Am.a10 * F.a00 + Am.a11 * F.a10, Am.a10 * F.a01 + Am.a11 * F.a11};
    s.ptr = 0;
    s.qtr = 0;
    if (s.util & kLiquid) {
        s.Jp = s.Jp * (Am.a00 * Am.a11 - Am.a10 * Am.a01);
    } else {
        double Je;
        compute_pq(s.F, P.mu, P.kappa, Je, s.ptr, s.qtr);   // kernels.cuh:547-557
        if (!(s.util & kCrushed)) {
            const GrainConst *gc = grain_tab + grain_slot((short)s.util);
            const GrainConst c{__ldg(&gc->pmin2), __ldg(&gc->k), __ldg(&gc->msq)};
            if (failure_surface_crushed_tab(P, c, s.ptr, s.qtr)) s.util |= kCrushed;
        }
        if (s.util & kCrushed) {
            const ReturnMapped r = return_map_out(P, s.F, s.Jp, s.ptr, s.qtr, Je);
            s.F = r.F;
            s.Jp = r.Jp;
        }
    }
    s.vx = vx;
    s.vy = vy;
    s.B = B;
    return true;
}

__device__ __forceinline__ void store_point(double *__restrict__ pts, long pitch, long i, const PointState &s,
                                            bool write_vb, bool record_pq)
{
    pts[i] = __longlong_as_double(s.util);
    pts[i + pitch * 3] = s.Jp;
    pts[i + pitch * 4] = s.x;
    pts[i + pitch * 5] = s.y;
    pts[i + pitch * 8] = s.F.a00; pts[i + pitch * 9] = s.F.a01;
    pts[i + pitch * 10] = s.F.a10; pts[i + pitch * 11] = s.F.a11;
    if (write_vb) {
        pts[i + pitch * 6] = s.vx; pts[i + pitch * 7] = s.vy;
        pts[i + pitch * 12] = s.B.a00; pts[i + pitch * 13] = s.B.a01;
        pts[i + pitch * 14] = s.B.a10; pts[i + pitch * 15] = s.B.a11;
    }
    if (record_pq) { pts[i + pitch * 1] = s.ptr; pts[i + pitch * 2] = s.qtr; }
}

// Shared buffer of P2G moments: five vectors of two doubles per staged point,
//   (fx, fy), (m, m vx), (m vy, S00), (S01, S10), (S11, base)
// with one padding column after every 4 points (cell threads read points about
// 4 apart).  After the cell phase the same buffer holds the cell partials
// (27 x TT doubles).
// Moments of a point, four double2 vectors and a 64-bit word per slot, one
// padding slot after every 4 points (the cell phase reads points about 4
// apart per lane): (fx, fy), (m vx, m vy), (S00, S01), (S10, S11) with
// S = m Bp - dt vol Dp_inv tau, and the packed stencil base (low 32 bits)
// with the liquid flag (bit 32) that selects the point's mass.
constexpr int MOM_N = CAP + CAP / 4;
constexpr size_t MOM_BYTES = (sizeof(double2) * 4 + sizeof(unsigned long long)) * MOM_N;
constexpr unsigned long long MOM_LIQUID = 1ull << 32;
static_assert(27 * TT * sizeof(double) <= MOM_BYTES, "cell partials alias the moment buffer");
__device__ __forceinline__ int mom_col(int j) { return j + (j >> 2); }
constexpr size_t TILE_DYN_SMEM = MOM_BYTES;

// P2G moments of a point (simulation/kernels.cuh:57-92) into column j.
__device__ __forceinline__ void p2g_moments(const StepParams &P, const PointState &s, double *mom, int j,
                                            int *status)
{
    double2 *m = reinterpret_cast<double2 *>(mom);
    unsigned long long *mb = reinterpret_cast<unsigned long long *>(m + 4 * MOM_N);
    const int c = mom_col(j);
    const bool liquid = (s.util & kLiquid) != 0;
    const double mass = liquid ? P.mass_water : P.mass_ice;
    const int bx = (int)(s.x * P.hinv - 0.5), by = (int)(s.y * P.hinv - 0.5);
    const int e = base_error(P, bx, by);
    if (e) {
        *status = e;
        mb[c] = (unsigned)BASE_NONE;
        return;
    }
    const M2<double> tau = liquid ? water_stress(s.Jp, P.kappa) : kirchhoff(s.F, P.mu, P.kappa);
    m[c] = make_double2(s.x * P.hinv - (double)bx, s.y * P.hinv - (double)by);
    m[MOM_N + c] = make_double2(s.vx * mass, s.vy * mass);
    m[2 * MOM_N + c] = make_double2(mass * s.B.a00 - P.dt_vol_Dpinv * tau.a00, mass * s.B.a01 - P.dt_vol_Dpinv * tau.a01);
    m[3 * MOM_N + c] = make_double2(mass * s.B.a10 - P.dt_vol_Dpinv * tau.a10, mass * s.B.a11 - P.dt_vol_Dpinv * tau.a11);
    mb[c] = (unsigned long long)(unsigned)pack_base(bx, by) | (liquid ? MOM_LIQUID : 0ull);
}

__device__ __forceinline__ void mom_none(double *mom, int j)
{
    reinterpret_cast<unsigned long long *>(reinterpret_cast<double2 *>(mom) + 4 * MOM_N)[mom_col(j)] = (unsigned)BASE_NONE;
}

// Phases 2 and 3 for one chunk of points [cs, ce) of tile (tx, ty): cell
// threads (tid < TT) sum their points' contributions in registers, then every
// region node adds its 9 cell partials in a fixed order plus the off-cell
// contributions and flushes to the global grid.  `sync` is a barrier over
// the NT participating threads.  `nxt`: the next tile's prologue, overlapped
// with the node phase (nxt.load() before the node loop issues its global
// loads, nxt.store() after it puts them into shared memory).
struct NoNextTile {
    __device__ __forceinline__ void load() const {}
    __device__ __forceinline__ void store() const {}
};
template <class L, class St>
struct NextTileOps {
    L l;
    St st;
    __device__ __forceinline__ void load() const { l(); }
    __device__ __forceinline__ void store() const { st(); }
};
// `s_oddf` (or nullptr: always the full region): set when a point of the
// chunk added to the drift buffer s_odd; without one the node phase walks only
// the (TX + 2) x (TY + 2) nodes that cell sums reach and leaves s_odd alone.
template <int NT, typename Sync, class Next = NoNextTile>
__device__ __forceinline__ void p2g_cells_and_flush(const TileArgs &A, int tid, int tx, int ty, int cs, int ce,
                                                    const int *s_cs, double *mom, double (*s_odd)[RN],
                                                    int *s_oddf, unsigned &touch, unsigned &moved, Sync &&sync,
                                                    Next &&nxt = NoNextTile{})
{
    const StepParams &P = A.P;
    const int X0 = tx * TX - P.halo, Y0 = ty * TY;
    const int RX0 = X0 - RM, RY0 = Y0 - RM;
    static_assert(NT >= TT, "one thread per cell");
    double acc[27];
#pragma unroll
    for (int q = 0; q < 27; q++) acc[q] = 0;
    if (tid < TT) {
        const int bxc = X0 + tid / TY, byc = Y0 + tid % TY;
        const int r0 = max(s_cs[tid], cs) - cs, r1 = min(s_cs[tid + 1], ce) - cs;
        for (int j = r0; j < r1; j++) {
            const double2 *mv = reinterpret_cast<const double2 *>(mom);
            const int c = mom_col(j);
            const unsigned long long bw = reinterpret_cast<const unsigned long long *>(mv + 4 * MOM_N)[c];
            const int pb = (int)(unsigned)bw;
            if (pb == BASE_NONE) continue;
            int bx, by;
            unpack_base(pb, bx, by);
            const double2 q0 = mv[c], q1 = mv[MOM_N + c], q2 = mv[2 * MOM_N + c], q3 = mv[3 * MOM_N + c];
            const double mass = (bw & MOM_LIQUID) ? P.mass_water : P.mass_ice;
            const double fx = q0.x, fy = q0.y, mvx = q1.x, mvy = q1.y;
            const double s00 = q2.x, s01 = q2.y, s10 = q3.x, s11 = q3.y;
            if (bx == bxc && by == byc) {
                point_contributions(P.h, fx, fy, mass, mvx, mvy, s00, s01, s10, s11,
                                    [&](int a, int b, double W, double dm, double tx, double ty) {
                                        const int q = (a * 3 + b) * 3;
                                        acc[q] += dm;
                                        acc[q + 1] += W * tx;
                                        acc[q + 2] += W * ty;
                                    });
            } else {
                moved++;
                const int lx = bx - RX0, ly = by - RY0;
                if (lx >= 0 && lx + 2 < RX && ly >= 0 && ly + 2 < RY) {
                    if (s_oddf) *s_oddf = 1;
                    point_contributions(P.h, fx, fy, mass, mvx, mvy, s00, s01, s10, s11,
                                        [&](int a, int b, double W, double dm, double tx, double ty) {
                                            const int k = (lx + a) * RY + (ly + b);
                                            atomicAdd(&s_odd[0][k], dm);
                                            atomicAdd(&s_odd[1][k], W * tx);
                                            atomicAdd(&s_odd[2][k], W * ty);
                                        });
                } else {
                    p2g_global(A.g, A.flags, A.tlist, A.tlist_n, A.G.ntx, P.halo, P.h, bx, by, fx, fy, mass, mvx, mvy, s00, s01, s10,
                               s11);
                }
            }
        }
    }
    sync();   // all moments read: the buffer becomes the cell partials
    // partials per (node offset, cell): (m, px) as a vector, then py
    double2 *pmx = reinterpret_cast<double2 *>(mom);
    double *ppy = mom + 2 * 9 * TT;
    if (tid < TT) {
#pragma unroll
        for (int q = 0; q < 9; q++) {
            pmx[q * TT + tid] = make_double2(acc[3 * q], acc[3 * q + 1]);
            ppy[q * TT + tid] = acc[3 * q + 2];
        }
    }
    sync();
    nxt.load();
    const bool odd = !s_oddf || *s_oddf != 0;
    constexpr int CY = TY + 2;
    const int kn = odd ? RN : (TX + 2) * CY;
    for (int k = tid; k < kn; k += NT) {
        int i, jj;                                 // region coordinates
        if (odd) {
            i = k / RY;
            jj = k % RY;
        } else {
            i = RM + k / CY;
            jj = RM + k % CY;
        }
        const int kk = i * RY + jj;
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
                const int c = cx * TY + cy, q = a * 3 + b;
                const double2 v = pmx[q * TT + c];
                m += v.x;
                px += v.y;
                py += ppy[q * TT + c];
            }
        }
        if (odd) {
            m += s_odd[0][kk]; px += s_odd[1][kk]; py += s_odd[2][kk];
            s_odd[0][kk] = 0; s_odd[1][kk] = 0; s_odd[2][kk] = 0;
        }
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
    nxt.store();
    sync();   // partials consumed before the buffer is refilled
    if (s_oddf && tid == 0) *s_oddf = 0;   // the next chunk's cell phase sets it after a barrier
}

__device__ __forceinline__ void mark_node_tiles(const TileArgs &A, int tx, int ty, unsigned touch, int lane9)
{
    if (lane9 < 9 && ((touch >> lane9) & 1u)) {
        const int ntx = tx + lane9 % 3 - 1, nty = ty + lane9 / 3 - 1;
        mark_tile(A.flags, A.tlist, A.tlist_n, 0, ntx, nty, A.G.ntx);
    }
}

// L2 prefetch of [p, p + bytes) rounded inward to 16-byte boundaries (never
// past either end): cp.async.bulk.prefetch.L2 from this GPU's global memory.
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes)
{
    const uintptr_t a = ((uintptr_t)p + 15) & ~uintptr_t(15), e = ((uintptr_t)p + bytes) & ~uintptr_t(15);
    if (e > a) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"((uint32_t)(e - a)) : "memory");
}

// Prefetches into L2 one column of the node region a tile stages (RY nodes of
// column RX0 + col from row RY0, clipped to the grid) of one node array:
// the first and the last node's lines (a column spans at most two lines).
template <typename T>
__device__ __forceinline__ void prefetch_region_column(const T *arr, int gridx, int gridy, int halo, int ny, int RX0,
                                                       int RY0, int col, int RY = icy_dev::RY)
{
    const int gx = RX0 + col;
    if (gx < -halo || gx >= gridx + halo) return;
    const int y0 = max(RY0, 0), y1 = min(RY0 + RY, gridy);
    if (y1 <= y0) return;
    const T *c = arr + (long)(gx + halo) * ny;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(c + y0));
    asm volatile("prefetch.global.L2 [%0];" ::"l"(c + y1 - 1));
}

// Starts moving the next tile's point lines that G2P reads (which < 8: utility,
// Jp, x, y, Fe00..Fe11) or its cell ranges (which == 8) into L2 while this CTA
// is in its cell phase.
constexpr int TILE_PREFETCHES = 9;
__device__ __forceinline__ void prefetch_next_tile(const TileArgs &A, int next, int na, int which)
{
    if (next >= na) return;
    const int *cs = A.cell_start + (long)A.active[next] * TT;
    if (which == 8) {
        prefetch_l2(cs, (TT + 1) * sizeof(int));
        return;
    }
    const int line = which < 1 ? 0 : which < 4 ? which + 2 : which + 4;   // 0, 3, 4, 5, 8, 9, 10, 11
    const int ps = cs[0], pe = cs[TT];
    if (pe > ps) prefetch_l2(A.pts + A.pitch * line + ps, (size_t)(pe - ps) * sizeof(double));
}

// ---------------------------------------------------------------- plain tile kernel
// One persistent CTA loop over the non-empty tiles, points read straight from
// global memory.  Used for the first step of a run (<false, true, false>: P2G
// only) and the last (<true, false, true>: G2P only, writes vel and Bp), and
// by the per-phase calls.
template <bool DO_G2P, bool DO_P2G, bool WRITE_VB>
static __global__ void __launch_bounds__(TILE_THREADS, 2) k_tile(const __grid_constant__ TileArgs A)
{
    __shared__ double2 s_v[RN];        // staged node velocities (G2P)
    __shared__ double s_odd[3][RN];    // contributions of points off their sorted cell
    __shared__ int s_cs[TT + 1];       // cell ranges of the tile
    __shared__ unsigned s_touch;
    __shared__ int s_oddf;             // a point of the chunk used s_odd
    extern __shared__ double2 s_mom2[];   // moments | 27 x TT cell partials
    double *const s_mom = reinterpret_cast<double *>(s_mom2);
    const StepParams &P = A.P;
    const int na = *A.n_active;
    const int tid = threadIdx.x;
    unsigned moved = 0;
    for (int k = tid; k < RN; k += blockDim.x) { s_odd[0][k] = 0; s_odd[1][k] = 0; s_odd[2][k] = 0; }
    if (tid == 0) s_oddf = 0;
    // the tile's prologue (cell ranges, staged node velocities) was done during
    // the previous tile's node phase
    bool staged = false;
    for (int ti = blockIdx.x; ti < na; ti += gridDim.x) {
        const int t = A.active[ti];
        const int tx = t % A.G.ntx, ty = t / A.G.ntx;
        const int RX0 = tx * TX - P.halo - RM, RY0 = ty * TY - RM;
        if (!staged) {
            for (int c = tid; c <= TT; c += blockDim.x) s_cs[c] = A.cell_start[(long)t * TT + c];
            if (DO_G2P) {
                for (int k = tid; k < RN; k += blockDim.x) {
                    const int gx = RX0 + k / RY, gy = RY0 + k % RY;
                    double vx = 0, vy = 0;
                    if (node_in_grid(P, gx, gy)) {
                        const long q = A.g.idx(gx, gy);
                        vx = A.g.vx[q];
                        vy = A.g.vy[q];
                    }
                    s_v[k] = make_double2(vx, vy);
                }
            }
        }
        if (tid == 0) s_touch = 0;
        __syncthreads();
        const int ps = s_cs[0], pe = s_cs[TT];
        // the 3 x 3 node velocities of a stencil: from the staged region (one check
        // per point), else from the grid
        auto vsrc = [&](int bx, int by, double2 *nv) {
            const int lx = bx - RX0, ly = by - RY0;
            if (lx >= 0 && lx + 2 < RX && ly >= 0 && ly + 2 < RY) {
                const double2 *r = s_v + lx * RY + ly;
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) nv[a * 3 + b] = r[a * RY + b];
            } else {
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) {
                        const long k = A.g.idx(bx + a, by + b);
                        nv[a * 3 + b] = make_double2(A.g.vx[k], A.g.vy[k]);
                    }
            }
        };
        unsigned touch = 0;
        bool next_staged = false;
        for (int cs = ps; cs < pe; cs += CAP) {
            const int ce = min(cs + CAP, pe);
            for (int j = tid; j < ce - cs; j += blockDim.x) {
                const long i = cs + j;
                PointState s;
                // all eight lines requested before the first is tested (one memory latency)
                const long pitch = A.pitch;
                s.util = __double_as_longlong(A.pts[i]);
                s.x = A.pts[i + pitch * 4];
                s.y = A.pts[i + pitch * 5];
                s.Jp = A.pts[i + pitch * 3];
                s.F = {A.pts[i + pitch * 8], A.pts[i + pitch * 9], A.pts[i + pitch * 10], A.pts[i + pitch * 11]};
                if (s.util & kDisabled) {
                    if (DO_P2G) mom_none(s_mom, j);
                    continue;
                }
                if (DO_G2P) {
                    if (!g2p_update(P, A.grain_tab, s, A.status, vsrc)) {
                        if (DO_P2G) mom_none(s_mom, j);
                        continue;
                    }
                    store_point(A.pts, pitch, i, s, WRITE_VB, A.record_pq != 0);
                } else {
                    s.vx = A.pts[i + pitch * 6];
                    s.vy = A.pts[i + pitch * 7];
                    s.B = {A.pts[i + pitch * 12], A.pts[i + pitch * 13], A.pts[i + pitch * 14],
                           A.pts[i + pitch * 15]};
                }
                if (DO_P2G) p2g_moments(P, s, s_mom, j, A.status);
            }
            __syncthreads();
            // the last threads start the next tile's loads during the cell phase
            if (DO_P2G && cs == ps && tid >= TILE_THREADS - TILE_PREFETCHES)
                prefetch_next_tile(A, ti + gridDim.x, na, tid - (TILE_THREADS - TILE_PREFETCHES));
            const int nti = ti + gridDim.x;
            if (DO_P2G && ce == pe && nti < na) {
                // the last chunk: the next tile's prologue during this node phase
                constexpr int NC = (TT + 1 + TILE_THREADS - 1) / TILE_THREADS, NV = (RN + TILE_THREADS - 1) / TILE_THREADS;
                int ncs[NC];
                double2 nvel[NV];
                auto ld = [&] {
                    const int tn = A.active[nti];
#pragma unroll
                    for (int u = 0; u < NC; u++) {
                        const int c = tid + u * TILE_THREADS;
                        ncs[u] = c <= TT ? A.cell_start[(long)tn * TT + c] : 0;
                    }
                    if (DO_G2P) {
                        const int rx0 = (tn % A.G.ntx) * TX - P.halo - RM, ry0 = (tn / A.G.ntx) * TY - RM;
#pragma unroll
                        for (int u = 0; u < NV; u++) {
                            const int k = tid + u * TILE_THREADS;
                            const int gx = rx0 + k / RY, gy = ry0 + k % RY;
                            double vx = 0, vy = 0;
                            if (k < RN && node_in_grid(P, gx, gy)) {
                                const long q = A.g.idx(gx, gy);
                                vx = A.g.vx[q];
                                vy = A.g.vy[q];
                            }
                            nvel[u] = make_double2(vx, vy);
                        }
                    }
                };
                auto st = [&] {
#pragma unroll
                    for (int u = 0; u < NC; u++) {
                        const int c = tid + u * TILE_THREADS;
                        if (c <= TT) s_cs[c] = ncs[u];
                    }
                    if (DO_G2P) {
#pragma unroll
                        for (int u = 0; u < NV; u++) {
                            const int k = tid + u * TILE_THREADS;
                            if (k < RN) s_v[k] = nvel[u];
                        }
                    }
                };
                p2g_cells_and_flush<TILE_THREADS>(A, tid, tx, ty, cs, ce, s_cs, s_mom, s_odd, &s_oddf, touch, moved,
                                                  [] { __syncthreads(); }, NextTileOps<decltype(ld), decltype(st)>{ld, st});
                next_staged = true;
            } else if (DO_P2G) {
                p2g_cells_and_flush<TILE_THREADS>(A, tid, tx, ty, cs, ce, s_cs, s_mom, s_odd, &s_oddf, touch, moved,
                                                  [] { __syncthreads(); });
            }
        }
        if (DO_P2G) {
            touch = __reduce_or_sync(0xffffffffu, touch);
            if ((tid & 31) == 0 && touch) atomicOr(&s_touch, touch);
            __syncthreads();
            mark_node_tiles(A, tx, ty, s_touch, tid);
        }
        __syncthreads();
        staged = next_staged;
    }
    if (DO_P2G) {
        moved = __reduce_add_sync(0xffffffffu, moved);
        if ((tid & 31) == 0 && moved) atomicAdd(A.moved, (unsigned long long)moved);
    }
}

// ---------------------------------------------------------------- pipelined fused kernel
// G2P(n) + P2G(n+1) with the point stream fed by bulk copies: warp PIPE_CONS/32
// (the producer) walks the same chunk sequence as the consumers and, for each
// chunk, loads the tile's node velocities and cell ranges with plain loads and
// the chunk's 8 state lines with cp.async.bulk into one of NSTAGE ring slots;
// the 8 consumer warps compute from shared memory and write the new state to
// global memory.  One CTA per SM.
constexpr int PIPE_CONS = 256, PIPE_THREADS = PIPE_CONS + 32, NSTAGE = 2;
constexpr int NLINE = 8;                          // utility, Jp, x, y, Fe00..Fe11
constexpr int PIPE_CAP = 704;                     // points per staged chunk of the pipelined kernel
constexpr int LINE_CAP = PIPE_CAP + 2;            // slack for 16-byte alignment of the copy
static_assert((LINE_CAP * sizeof(double)) % 16 == 0, "16-byte aligned staged lines");
static __device__ __constant__ const int kPipeLines[NLINE] = {0, 3, 4, 5, 8, 9, 10, 11};
constexpr uint64_t PIPE_WAIT_NS = 1000000000ull;  // a wait gives up after 1 s ...
constexpr long PIPE_WAIT_POLLS = 1L << 26;         // ... or this many polls

struct PipeSmem {
    double line[NSTAGE][NLINE][LINE_CAP];        // staged point lines
    double2 v[NSTAGE][RN];                       // staged node velocities
    int cs[NSTAGE][TT + 1];                      // staged cell ranges
    int meta[NSTAGE][4];                         // tile, cs, ce, first aligned index
    alignas(16) double mom[MOM_BYTES / sizeof(double)];   // moments | cell partials
    double odd[3][RN];
    unsigned long long full[NSTAGE], empty[NSTAGE];
    unsigned touch;
    int abort;
};
constexpr size_t PIPE_SMEM = sizeof(PipeSmem) + 128;

static __global__ void __launch_bounds__(PIPE_THREADS, 1) k_tile_pipe(const __grid_constant__ TileArgs A)
{
    extern __shared__ unsigned char s_raw[];
    PipeSmem &S = *reinterpret_cast<PipeSmem *>((reinterpret_cast<uintptr_t>(s_raw) + 127) & ~uintptr_t(127));
    const StepParams &P = A.P;
    const int tid = threadIdx.x;
    const int na = *A.n_active;
    if (tid == 0) {
        for (int s = 0; s < NSTAGE; s++) {
            mbar_init(reinterpret_cast<uint64_t *>(&S.full[s]), 1);
            mbar_init(reinterpret_cast<uint64_t *>(&S.empty[s]), 1);
        }
        mbar_init_fence();
        S.touch = 0;
        S.abort = 0;
    }
    for (int k = tid; k < RN; k += PIPE_THREADS) { S.odd[0][k] = 0; S.odd[1][k] = 0; S.odd[2][k] = 0; }
    __syncthreads();

    if (tid >= PIPE_CONS) {
        // ------------------------------------------------ producer warp
        const int lane = tid - PIPE_CONS;
        int c = 0;
        bool ok = true;
        for (int ti = blockIdx.x; ti < na && ok; ti += gridDim.x) {
            const int t = A.active[ti];
            const int ps = A.cell_start[(long)t * TT], pe = A.cell_start[(long)(t + 1) * TT];
            const int tx = t % A.G.ntx, ty = t / A.G.ntx;
            const int RX0 = tx * TX - P.halo - RM, RY0 = ty * TY - RM;
            for (int cs = ps; cs < pe; cs += PIPE_CAP, c++) {
                const int st = c % NSTAGE, use = c / NSTAGE;
                if (use > 0 && !mbar_wait(reinterpret_cast<uint64_t *>(&S.empty[st]), (use - 1) & 1,
                                          PIPE_WAIT_NS, PIPE_WAIT_POLLS)) {
                    *A.status = ICY_TIMEOUT_CODE;
                    ok = false;
                    break;
                }
                fence_proxy_async_smem();
                const int ce = min(cs + PIPE_CAP, pe);
                const int a0 = cs & ~1, a1 = (ce + 1) & ~1;
                for (int k = lane; k < RN; k += 32) {
                    const int gx = RX0 + k / RY, gy = RY0 + k % RY;
                    double vx = 0, vy = 0;
                    if (node_in_grid(P, gx, gy)) {
                        const long q = A.g.idx(gx, gy);
                        vx = A.g.vx[q];
                        vy = A.g.vy[q];
                    }
                    S.v[st][k] = make_double2(vx, vy);
                }
                for (int k = lane; k <= TT; k += 32) S.cs[st][k] = A.cell_start[(long)t * TT + k];
                if (lane == 0) {
                    S.meta[st][0] = t;
                    S.meta[st][1] = cs;
                    S.meta[st][2] = ce;
                    S.meta[st][3] = a0;
                }
                __syncwarp();
                // fault_test: the first stage is never filled, so every wait on it
                // runs out (the timeout path, exercised by a test)
                if (lane == 0 && !(A.fault_test && c == 0)) {
                    const uint32_t bytes = (uint32_t)((a1 - a0) * sizeof(double));
                    uint64_t *bar = reinterpret_cast<uint64_t *>(&S.full[st]);
                    mbar_arrive_expect_tx(bar, bytes * NLINE);
                    for (int l = 0; l < NLINE; l++)
                        bulk_g2s(&S.line[st][l][0], A.pts + A.pitch * kPipeLines[l] + a0, bytes, bar);
                }
                __syncwarp();
            }
        }
        // before leaving, wait (bounded) for this warp's last copies: consumers
        // that gave up no longer wait for them, and none may be in flight when
        // the CTA ends (chunks [0, c) were issued; each stage's last phase is final)
        if (lane == 0)
            for (int k = max(0, c - NSTAGE); k < c; k++)
                mbar_wait(reinterpret_cast<uint64_t *>(&S.full[k % NSTAGE]), (k / NSTAGE) & 1, PIPE_WAIT_NS, PIPE_WAIT_POLLS);
        return;
    }

    // ---------------------------------------------------- consumer warps
    unsigned moved = 0;
    int c = 0;
    unsigned touch = 0;
    auto csync = [] { consumer_sync<PIPE_CONS>(); };
    bool ok = true;
    for (int ti = blockIdx.x; ti < na && ok; ti += gridDim.x) {
        const int t = A.active[ti];
        const int ps = A.cell_start[(long)t * TT], pe = A.cell_start[(long)(t + 1) * TT];
        const int tx = t % A.G.ntx, ty = t / A.G.ntx;
        const int RX0 = tx * TX - P.halo - RM, RY0 = ty * TY - RM;
        touch = 0;
        for (int cs = ps; cs < pe; cs += PIPE_CAP, c++) {
            const int st = c % NSTAGE, use = c / NSTAGE;
            // the decision to give up is made CTA-uniform through S.abort
            if (!mbar_wait(reinterpret_cast<uint64_t *>(&S.full[st]), use & 1, PIPE_WAIT_NS, PIPE_WAIT_POLLS)) {
                *A.status = ICY_TIMEOUT_CODE;
                S.abort = 1;
            }
            csync();
            if (S.abort) { ok = false; break; }
            const int ce = S.meta[st][2], off = cs - S.meta[st][3];
            const double2 *sv = S.v[st];
            // the 3 x 3 node velocities of a stencil: from the staged region (one check
            // per point), else from the grid
            auto vsrc = [&](int bx, int by, double2 *nv) {
                const int lx = bx - RX0, ly = by - RY0;
                if (lx >= 0 && lx + 2 < RX && ly >= 0 && ly + 2 < RY) {
                    const double2 *r = sv + lx * RY + ly;
    #pragma unroll
                    for (int a = 0; a < 3; a++)
    #pragma unroll
                        for (int b = 0; b < 3; b++) nv[a * 3 + b] = r[a * RY + b];
                } else {
    #pragma unroll
                    for (int a = 0; a < 3; a++)
    #pragma unroll
                        for (int b = 0; b < 3; b++) {
                            const long k = A.g.idx(bx + a, by + b);
                            nv[a * 3 + b] = make_double2(A.g.vx[k], A.g.vy[k]);
                        }
                }
            };
            // phase 1: one thread per point, state from the staged lines
            for (int j = tid; j < ce - cs; j += PIPE_CONS) {
                const int q = off + j;
                PointState s;
                s.util = __double_as_longlong(S.line[st][0][q]);
                if (s.util & kDisabled) { mom_none(S.mom, j); continue; }
                s.Jp = S.line[st][1][q];
                s.x = S.line[st][2][q];
                s.y = S.line[st][3][q];
                s.F = {S.line[st][4][q], S.line[st][5][q], S.line[st][6][q], S.line[st][7][q]};
                if (!g2p_update(P, A.grain_tab, s, A.status, vsrc)) { mom_none(S.mom, j); continue; }
                store_point(A.pts, A.pitch, cs + j, s, false, A.record_pq != 0);
                p2g_moments(P, s, S.mom, j, A.status);
            }
            csync();
            p2g_cells_and_flush<PIPE_CONS>(A, tid, tx, ty, cs, ce, S.cs[st], S.mom, S.odd, nullptr, touch, moved,
                                           csync);
            // the stage (lines, velocities, cell ranges) is no longer read: release it
            if (tid == 0) mbar_arrive(reinterpret_cast<uint64_t *>(&S.empty[st]));
        }
        if (!ok) break;
        touch = __reduce_or_sync(0xffffffffu, touch);
        if ((tid & 31) == 0 && touch) atomicOr(&S.touch, touch);
        csync();
        const unsigned tt = S.touch;
        csync();
        if (tid == 0) S.touch = 0;
        mark_node_tiles(A, tx, ty, tt, tid);
    }
    moved = __reduce_add_sync(0xffffffffu, moved);
    if ((tid & 31) == 0 && moved) atomicAdd(A.moved, (unsigned long long)moved);
}

constexpr int UPD_TILES64 = 2;

// Grid update of the nodes of the listed tiles (simulation/kernels.cuh:164-301):
// each group of TT threads takes one TX x TY node tile (one thread per node, the
// TY nodes of a tile column contiguous in memory), computes the velocities, zeroes the
// accumulators for the next step and clears the tile's mark; the last CTA
// empties the list.
static __global__ void __launch_bounds__(256, 4) k_update_list(StepParams P, TileGeom G, GridView g, unsigned *flags,
                                                            const int2 *__restrict__ tlist, unsigned *tlist_n,
                                                            double ind_x, double ind_y, double *acc)
{
    extern __shared__ double s_acc[];   // 2*nsub
    for (int k = threadIdx.x; k < 2 * P.nsub; k += blockDim.x) s_acc[k] = 0;
    __syncthreads();
    bool any = false;
    const unsigned n = *(volatile unsigned *)tlist_n;
    constexpr int TPC = 256 / TT;   // node tiles per CTA pass
    static_assert(256 % TT == 0, "whole node tiles per 256-thread CTA");
    const int l = threadIdx.x % TT;
    const unsigned stride = gridDim.x * TPC;
    // UPD_TILES64 tiles per pass, their loads issued together
    for (unsigned e0 = blockIdx.x * TPC + threadIdx.x / TT; e0 < n; e0 += stride * UPD_TILES64) {
        long q[UPD_TILES64];
        int gx[UPD_TILES64], gy[UPD_TILES64];
        double m[UPD_TILES64], px[UPD_TILES64], py[UPD_TILES64];
#pragma unroll
        for (int u = 0; u < UPD_TILES64; u++) {
            const unsigned e = e0 + u * stride;
            q[u] = -1;
            if (e >= n) continue;
            const int e2 = tlist[e].y;
            const int tx = e2 & 0xffff, ty = e2 >> 16;
            if (l == 0) flags[ty * G.ntx + tx] = 0u;
            gx[u] = tx * TX + l / TY - P.halo;
            gy[u] = ty * TY + (l & (TY - 1));
            if (gx[u] >= P.gridx + P.halo || gy[u] >= P.gridy) continue;   // past the grid edge
            q[u] = g.idx(gx[u], gy[u]);
            m[u] = g.m[q[u]];
            px[u] = g.px[q[u]];
            py[u] = g.py[q[u]];
        }
#pragma unroll
        for (int u = 0; u < UPD_TILES64; u++) {
            if (q[u] < 0) continue;
            double vx = 0, vy = 0, fx, fy;
            int bin;
            if (node_update(P, gx[u], gy[u], m[u], px[u], py[u], ind_x, ind_y, vx, vy, bin, fx, fy) && bin >= 0) {
                atomicAdd(&s_acc[2 * bin], fx);
                atomicAdd(&s_acc[2 * bin + 1], fy);
                any = true;
            }
            g.vx[q[u]] = vx;
            g.vy[q[u]] = vy;
            g.m[q[u]] = 0.0;
            g.px[q[u]] = 0.0;
            g.py[q[u]] = 0.0;
        }
    }
    if (__syncthreads_or(any))
        for (int k = threadIdx.x; k < 2 * P.nsub; k += blockDim.x)
            if (s_acc[k] != 0.0) atomicAdd(acc + k, s_acc[k]);
    if (threadIdx.x == 0) tile_list_done(tlist_n);
}

}  // namespace icy_dev
