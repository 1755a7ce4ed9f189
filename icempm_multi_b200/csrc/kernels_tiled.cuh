// kernels_tiled.cuh -- binned, tile-staged FP64 step kernels (the fast path).
//
// Points are kept sorted by the tile of their stencil base node (TX x TY
// bases per tile).  One CTA owns one tile at a time:
//   * the node velocities of the tile's region (the bases of the tile plus a
//     margin of RM cells, and the +2 stencil reach) are staged in shared
//     memory for the G2P gather;
//   * G2P + return mapping of step n and P2G of step n+1 run back to back on
//     each point while its state is in registers, so the point state is read
//     once and written once per step;
//   * P2G contributions are summed into a shared-memory copy of the region
//     and flushed to the global grid once per tile (global FP64 reductions
//     only for the region's non-empty nodes);
//   * the flush marks the node tiles it wrote; the grid update then visits
//     only marked tiles, computes velocities (simulation/kernels.cuh:164-301)
//     and zeroes the accumulators for the next step.
// A point that drifted out of its tile's region since the last binning is
// still handled exactly, through global memory, and counted so the host can
// re-bin.
#pragma once
#include "kernels_simple.cuh"

namespace icy_dev {

constexpr int TX = 16, TY = 8, TT = TX * TY;   // stencil bases per tile
constexpr int RM = 1;                          // drift margin (cells) of the staged region
constexpr int RX = TX + 2 + 2 * RM, RY = TY + 2 + 2 * RM, RN = RX * RY;
constexpr int TILE_THREADS = 256;

// Tiles cover bases bx in [-halo, -halo + ntx*TX), by in [0, nty*TY);
// tile id = ty*ntx + tx; node tiles use the same partition of the nodes.
struct TileGeom {
    int ntx, nty, ntiles;
    __device__ __forceinline__ int tile_of(int bx, int by, int halo) const
    {
        return (by / TY) * ntx + (bx + halo) / TX;
    }
};

struct TileArgs {
    StepParams P;
    TileGeom G;
    GridView g;
    double *pts;
    long pitch;
    const int *tile_start;   // ntiles + 2 entries: first point of each tile; [ntiles] = disabled bucket
    const int *active;       // tiles with points, ascending
    const int *n_active;
    unsigned *flags;         // node tiles written by P2G since the last update
    int *status;
    unsigned long long *moved;  // points whose base left their tile (re-binning hint)
    int record_pq;
};

__device__ __forceinline__ bool node_in_grid(const StepParams &P, int gx, int gy)
{
    return gx >= -P.halo && gx < P.gridx + P.halo && gy >= 0 && gy < P.gridy;
}

// ---------------------------------------------------------------- binning
__global__ void k_bin_count(StepParams P, TileGeom G, const double *__restrict__ pts, long pitch, int n,
                            int *keys, int *ranks, int *counts, int *status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < n;
    int key = G.ntiles;
    if (in) {
        long long u = __double_as_longlong(pts[i]);
        if (!(u & kDisabled)) {
            const double x = pts[i + pitch * 4], y = pts[i + pitch * 5];
            const int bx = (int)(x * P.hinv - 0.5), by = (int)(y * P.hinv - 0.5);
            const int e = base_error(P, bx, by);
            if (e) *status = e;
            else key = G.tile_of(bx, by, P.halo);
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

// Exclusive scan of counts[0..ntiles] (one CTA) and the list of non-empty tiles.
__global__ void __launch_bounds__(1024) k_bin_scan(const int *counts, int ntiles, int *start, int *active,
                                                   int *n_active)
{
    __shared__ int s_sum[1024], s_act[1024];
    const int tid = threadIdx.x, total = ntiles + 1;
    const int per = (total + 1023) / 1024;
    const int b = min(tid * per, total), e = min(b + per, total);
    int sum = 0, act = 0;
    for (int k = b; k < e; k++) {
        const int c = counts[k];
        sum += c;
        act += (k < ntiles && c > 0);
    }
    s_sum[tid] = sum;
    s_act[tid] = act;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const int vs = tid >= off ? s_sum[tid - off] : 0, va = tid >= off ? s_act[tid - off] : 0;
        __syncthreads();
        s_sum[tid] += vs;
        s_act[tid] += va;
        __syncthreads();
    }
    int run = s_sum[tid] - sum, arun = s_act[tid] - act;
    for (int k = b; k < e; k++) {
        const int c = counts[k];
        start[k] = run;
        run += c;
        if (k < ntiles && c > 0) active[arun++] = k;
    }
    if (tid == 1023) {
        start[total] = s_sum[1023];
        *n_active = s_act[1023];
    }
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

// ---------------------------------------------------------------- per point
// Global-memory P2G of one point whose stencil is outside the staged region.
__device__ __noinline__ void p2g_global(GridView g, unsigned *flags, int ntx, int halo, double h, int bx, int by,
                                        double wx0, double wx1, double wx2, double wy0, double wy1, double wy2,
                                        double fx, double fy, double mass, double mvx, double mvy, double s00,
                                        double s01, double s10, double s11)
{
    const double wx[3] = {wx0, wx1, wx2}, wy[3] = {wy0, wy1, wy2};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double d0 = ((double)a - fx) * h;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const double W = wx[a] * wy[b];
            const double d1 = ((double)b - fy) * h;
            const long k = g.idx(bx + a, by + b);
            atomicAdd(g.m + k, W * mass);
            atomicAdd(g.px + k, W * (mvx + (s00 * d0 + s01 * d1)));
            atomicAdd(g.py + k, W * (mvy + (s10 * d0 + s11 * d1)));
        }
    }
    // node tiles touched: those of (bx, by) and (bx+2, by+2)
    const int t0x = (bx + halo) / TX, t1x = (bx + 2 + halo) / TX;
    const int t0y = by / TY, t1y = (by + 2) / TY;
    flags[t0y * ntx + t0x] = 1u;
    flags[t0y * ntx + t1x] = 1u;
    flags[t1y * ntx + t0x] = 1u;
    flags[t1y * ntx + t1x] = 1u;
}

template <bool DO_G2P, bool DO_P2G, bool WRITE_VB>
__device__ __forceinline__ void tile_point(const TileArgs &A, long i, int X0, int Y0, const double (*s_v)[RN],
                                           double (*s_a)[RN], unsigned &moved)
{
    const StepParams &P = A.P;
    double *__restrict__ pts = A.pts;
    const long pitch = A.pitch;
    long long util = __double_as_longlong(pts[i]);
    if (util & kDisabled) return;
    const bool liquid = (util & kLiquid) != 0;
    const int RX0 = X0 - RM, RY0 = Y0 - RM;
    double x = pts[i + pitch * 4], y = pts[i + pitch * 5];
    M2<double> F{pts[i + pitch * 8], pts[i + pitch * 9], pts[i + pitch * 10], pts[i + pitch * 11]};
    double Jp = pts[i + pitch * 3];
    double vx, vy;
    M2<double> B;
    if (DO_G2P) {
        const int bx = (int)(x * P.hinv - 0.5), by = (int)(y * P.hinv - 0.5);
        const double fx = x * P.hinv - (double)bx, fy = y * P.hinv - (double)by;
        const int e = base_error(P, bx, by);
        if (e) { *A.status = e; return; }
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
            if (!(util & kCrushed) && failure_surface_crushed(P, (short)util, ptr, qtr)) util |= kCrushed;
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
        // P2G of the (updated) point (simulation/kernels.cuh:57-121)
        const double mass = liquid ? P.mass_water : P.mass_ice;
        const M2<double> tau = liquid ? water_stress(Jp, P.kappa) : kirchhoff(F, P.mu, P.kappa);
        const M2<double> S{mass * B.a00 - P.dt_vol_Dpinv * tau.a00, mass * B.a01 - P.dt_vol_Dpinv * tau.a01,
                           mass * B.a10 - P.dt_vol_Dpinv * tau.a10, mass * B.a11 - P.dt_vol_Dpinv * tau.a11};
        const int bx = (int)(x * P.hinv - 0.5), by = (int)(y * P.hinv - 0.5);
        const double fx = x * P.hinv - (double)bx, fy = y * P.hinv - (double)by;
        const int e = base_error(P, bx, by);
        if (e) { *A.status = e; return; }
        double wx[3], wy[3];
        bspline_weights(fx, wx);
        bspline_weights(fy, wy);
        const double mvx = vx * mass, mvy = vy * mass;
        const int lx = bx - RX0, ly = by - RY0;
        if (bx < X0 || bx >= X0 + TX || by < Y0 || by >= Y0 + TY) moved++;
        if (lx >= 0 && lx + 2 < RX && ly >= 0 && ly + 2 < RY) {
#pragma unroll
            for (int a = 0; a < 3; a++) {
                const double d0 = ((double)a - fx) * P.h;
#pragma unroll
                for (int b = 0; b < 3; b++) {
                    const double W = wx[a] * wy[b];
                    const double d1 = ((double)b - fy) * P.h;
                    const int k = (lx + a) * RY + (ly + b);
                    atomicAdd(&s_a[0][k], W * mass);
                    atomicAdd(&s_a[1][k], W * (mvx + (S.a00 * d0 + S.a01 * d1)));
                    atomicAdd(&s_a[2][k], W * (mvy + (S.a10 * d0 + S.a11 * d1)));
                }
            }
        } else {
            p2g_global(A.g, A.flags, A.G.ntx, P.halo, P.h, bx, by, wx[0], wx[1], wx[2], wy[0], wy[1], wy[2], fx, fy,
                       mass, mvx, mvy, S.a00, S.a01, S.a10, S.a11);
        }
    }
}

// One persistent CTA loop over the non-empty tiles.
//   <true, true, false>  G2P(n) + P2G(n+1)         (steady state of a run)
//   <false, true, false> P2G only                  (first step, per-phase p2g)
//   <true, false, true>  G2P only, writes vel & Bp (last step, per-phase g2p)
template <bool DO_G2P, bool DO_P2G, bool WRITE_VB>
__global__ void __launch_bounds__(TILE_THREADS, 2) k_tile(TileArgs A)
{
    __shared__ double s_v[2][RN];
    __shared__ double s_a[3][RN];
    __shared__ unsigned s_touch;
    const StepParams &P = A.P;
    const int na = *A.n_active;
    unsigned moved = 0;
    for (int ti = blockIdx.x; ti < na; ti += gridDim.x) {
        const int t = A.active[ti];
        const int tx = t % A.G.ntx, ty = t / A.G.ntx;
        const int X0 = tx * TX - P.halo, Y0 = ty * TY;
        const int RX0 = X0 - RM, RY0 = Y0 - RM;
        const int ps = A.tile_start[t], pe = A.tile_start[t + 1];
        if (threadIdx.x == 0) s_touch = 0;
        for (int k = threadIdx.x; k < RN; k += blockDim.x) {
            const int gx = RX0 + k / RY, gy = RY0 + k % RY;
            if (DO_G2P) {
                double vx = 0, vy = 0;
                if (node_in_grid(P, gx, gy)) {
                    const long q = A.g.idx(gx, gy);
                    vx = A.g.vx[q];
                    vy = A.g.vy[q];
                }
                s_v[0][k] = vx;
                s_v[1][k] = vy;
            }
            if (DO_P2G) { s_a[0][k] = 0; s_a[1][k] = 0; s_a[2][k] = 0; }
        }
        __syncthreads();
        for (int i = ps + threadIdx.x; i < pe; i += blockDim.x)
            tile_point<DO_G2P, DO_P2G, WRITE_VB>(A, i, X0, Y0, s_v, s_a, moved);
        __syncthreads();
        if (DO_P2G) {
            unsigned touch = 0;
            for (int k = threadIdx.x; k < RN; k += blockDim.x) {
                const double m = s_a[0][k], px = s_a[1][k], py = s_a[2][k];
                if (m != 0.0 || px != 0.0 || py != 0.0) {
                    const int gx = RX0 + k / RY, gy = RY0 + k % RY;   // in the grid: only valid bases scatter
                    const long q = A.g.idx(gx, gy);
                    atomicAdd(A.g.m + q, m);
                    atomicAdd(A.g.px + q, px);
                    atomicAdd(A.g.py + q, py);
                    const int dx = (gx + P.halo) / TX - tx + 1, dy = gy / TY - ty + 1;
                    touch |= 1u << (dy * 3 + dx);
                }
            }
            touch = __reduce_or_sync(0xffffffffu, touch);
            if ((threadIdx.x & 31) == 0 && touch) atomicOr(&s_touch, touch);
            __syncthreads();
            if (threadIdx.x < 9 && ((s_touch >> threadIdx.x) & 1u)) {
                const int ntx = tx + (int)(threadIdx.x % 3) - 1, nty = ty + (int)(threadIdx.x / 3) - 1;
                A.flags[nty * A.G.ntx + ntx] = 1u;
            }
        }
        __syncthreads();
    }
    if (DO_P2G) {
        moved = __reduce_add_sync(0xffffffffu, moved);
        if ((threadIdx.x & 31) == 0 && moved) atomicAdd(A.moved, (unsigned long long)moved);
    }
}

// Grid update of the marked node tiles (simulation/kernels.cuh:164-301); zeroes
// the accumulators and clears the marks for the next step.
__global__ void __launch_bounds__(TT) k_update_tiles(StepParams P, TileGeom G, GridView g, unsigned *flags,
                                                    double ind_x, double ind_y, double *acc)
{
    extern __shared__ double s_acc[];   // 2*nsub
    for (int k = threadIdx.x; k < 2 * P.nsub; k += blockDim.x) s_acc[k] = 0;
    __syncthreads();
    bool any = false;
    for (int t = blockIdx.x; t < G.ntiles; t += gridDim.x) {
        if (flags[t] == 0u) continue;   // uniform over the CTA
        const int tx = t % G.ntx, ty = t / G.ntx;
        const int gx = tx * TX - P.halo + (int)threadIdx.x / TY, gy = ty * TY + (int)threadIdx.x % TY;
        if (gx < P.gridx + P.halo && gy < P.gridy) {
            const long q = g.idx(gx, gy);
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
        __syncthreads();
        if (threadIdx.x == 0) flags[t] = 0u;
    }
    if (!__syncthreads_or(any)) return;
    for (int k = threadIdx.x; k < 2 * P.nsub; k += blockDim.x)
        if (s_acc[k] != 0.0) atomicAdd(acc + k, s_acc[k]);
}

}  // namespace icy_dev
