// kernels_simple.cuh -- one-thread-per-item FP64 kernels for the per-phase API.
//
// These serve icy_mpm_p2g / icy_mpm_update_nodes / icy_mpm_g2p, the calls a
// GPU_Implementation5-style caller makes one phase at a time
// (simulation/gpu_implementation5.h:44-51).  They work on the particle SoA in
// its current order with global FP64 reductions (red.global.add.f64), and
// never touch memory outside the grid: a particle whose stencil leaves the
// grid records the reference's error code and is skipped.
#pragma once
#include "mpm_math.cuh"

namespace icy_dev {

struct GridView {
    double *m, *px, *py;   // accumulators
    double *vx, *vy;       // node velocities
    int ny;                // node stride along x (= GridY)
    int halo;              // x offset: node gx is stored at column gx + halo (for a slab of the
                           // grid starting at column x0: halo - x0)
    // stencil bases gx in [xlo, xhi] lie in this grid's columns (the whole grid:
    // -halo .. GridX + halo - 3, as base_error's x test); nodes gx in [flo, fhi)
    // count their indenter force (a slab: its own columns, not the neighbours')
    int xlo = -(1 << 30), xhi = 1 << 30, flo = -(1 << 30), fhi = 1 << 30;
    __device__ __forceinline__ long idx(int gx, int gy) const { return (long)(gx + halo) * ny + gy; }
};

__device__ __forceinline__ long long ld_util(const double *pts, long i)
{
    return __double_as_longlong(pts[i]);
}

// P2G of point i (kernels.cuh:46-122)
__device__ __forceinline__ void p2g_one(const StepParams &P, const double *__restrict__ pts, long pitch, int i,
                                        const GridView &g, int *status)
{
    long long util = ld_util(pts, i);
    if (util & kDisabled) return;
    const bool liquid = (util & kLiquid) != 0;
    const double mass = liquid ? P.mass_water : P.mass_ice;
    const double x = pts[i + pitch * 4], y = pts[i + pitch * 5];
    const double vx = pts[i + pitch * 6], vy = pts[i + pitch * 7];
    M2<double> F{pts[i + pitch * 8], pts[i + pitch * 9], pts[i + pitch * 10], pts[i + pitch * 11]};
    M2<double> B{pts[i + pitch * 12], pts[i + pitch * 13], pts[i + pitch * 14], pts[i + pitch * 15]};
    M2<double> tau = liquid ? water_stress(pts[i + pitch * 3], P.kappa) : kirchhoff(F, P.mu, P.kappa);
    M2<double> S{mass * B.a00 - P.dt_vol_Dpinv * tau.a00, mass * B.a01 - P.dt_vol_Dpinv * tau.a01,
                 mass * B.a10 - P.dt_vol_Dpinv * tau.a10, mass * B.a11 - P.dt_vol_Dpinv * tau.a11};
    const int bx = (int)(x * P.hinv - 0.5), by = (int)(y * P.hinv - 0.5);
    const double fx = x * P.hinv - (double)bx, fy = y * P.hinv - (double)by;
    int e = base_error(P, bx, by);
    if (!e && (bx < g.xlo || bx > g.xhi)) e = bx < g.xlo ? 70 : 72;   // beyond the slab's columns
    if (e) { *status = e; return; }
    double wx[3], wy[3];
    bspline_weights(fx, wx);
    bspline_weights(fy, wy);
    const double mvx = vx * mass, mvy = vy * mass;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double d0 = ((double)a - fx) * P.h;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const double W = wx[a] * wy[b];
            const double d1 = ((double)b - fy) * P.h;
            const long k = g.idx(bx + a, by + b);
            atomicAdd(g.m + k, W * mass);
            atomicAdd(g.px + k, W * (mvx + (S.a00 * d0 + S.a01 * d1)));
            atomicAdd(g.py + k, W * (mvy + (S.a10 * d0 + S.a11 * d1)));
        }
    }
}

// P2G, one thread per particle
static __global__ void k_p2g_simple(StepParams P, const double *__restrict__ pts, long pitch, int n, GridView g,
                                    int *status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p2g_one(P, pts, pitch, i, g, status);
}

// indenter force bins are accumulated per block in shared memory first
// and added to the global accumulator once per block
static __global__ void k_update_simple(StepParams P, GridView g, long n_nodes, double ind_x, double ind_y,
                                double *acc)
{
    extern __shared__ double s_acc[];   // 2*nsub
    for (int k = threadIdx.x; k < 2 * P.nsub; k += blockDim.x) s_acc[k] = 0;
    __syncthreads();
    bool any = false;
    long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < n_nodes) {
        int gix = (int)(idx / g.ny) - g.halo, giy = (int)(idx % g.ny);
        double vx, vy, fx, fy;
        int bin;
        if (node_update(P, gix, giy, g.m[idx], g.px[idx], g.py[idx], ind_x, ind_y, vx, vy, bin, fx, fy)) {
            g.vx[idx] = vx;
            g.vy[idx] = vy;
            if (bin >= 0 && gix >= g.flo && gix < g.fhi) {
                atomicAdd(&s_acc[2 * bin], fx);
                atomicAdd(&s_acc[2 * bin + 1], fy);
                any = true;
            }
        } else {
            g.vx[idx] = 0.0;
            g.vy[idx] = 0.0;
        }
    }
    if (!__syncthreads_or(any)) return;
    for (int k = threadIdx.x; k < 2 * P.nsub; k += blockDim.x)
        if (s_acc[k] != 0.0) atomicAdd(acc + k, s_acc[k]);
}

// G2P + plasticity of point i (kernels.cuh:305-414)
__device__ __forceinline__ void g2p_one(const StepParams &P, double *__restrict__ pts, long pitch, int i,
                                        const GridView &g, int recordPQ, int *status)
{
    long long util = ld_util(pts, i);
    if (util & kDisabled) return;
    const bool liquid = (util & kLiquid) != 0;
    double x = pts[i + pitch * 4], y = pts[i + pitch * 5];
    M2<double> F{pts[i + pitch * 8], pts[i + pitch * 9], pts[i + pitch * 10], pts[i + pitch * 11]};
    double Jp = pts[i + pitch * 3];
    const int grain = (short)util;
    const int bx = (int)(x * P.hinv - 0.5), by = (int)(y * P.hinv - 0.5);
    const double fx = x * P.hinv - (double)bx, fy = y * P.hinv - (double)by;
    int e = base_error(P, bx, by);
    if (!e && (bx < g.xlo || bx > g.xhi)) e = bx < g.xlo ? 70 : 72;   // beyond the slab's columns
    if (e) { *status = e; return; }
    double wx[3], wy[3];
    bspline_weights(fx, wx);
    bspline_weights(fy, wy);
    double vx = 0, vy = 0;
    M2<double> B{0, 0, 0, 0};
    const double s4 = 4. * P.hinv;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const double d0 = (double)a - fx;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const double d1 = (double)b - fy;
            const double w = wx[a] * wy[b];
            const long k = g.idx(bx + a, by + b);
            const double nvx = g.vx[k], nvy = g.vy[k];
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
    M2<double> A{1.0 + P.dt * B.a00, P.dt * B.a01, P.dt * B.a10, 1.0 + P.dt * B.a11};
    M2<double> Fn{A.a00 * F.a00 + A.a01 * F.a10, A.a00 * F.a01 + A.a01 * F.a11,
                  A.a10 * F.a00 + A.a11 * F.a10, A.a10 * F.a01 + A.a11 * F.a11};
    double ptr = 0, qtr = 0;
    if (liquid) {
        Jp = Jp * (A.a00 * A.a11 - A.a10 * A.a01);
    } else {
        double Je;
        compute_pq(Fn, P.mu, P.kappa, Je, ptr, qtr);
        if (!(util & kCrushed) && failure_surface_crushed(P, grain, ptr, qtr)) util |= kCrushed;
        if (util & kCrushed) return_map(P, Fn, Jp, ptr, qtr, Je);
    }
    pts[i] = __longlong_as_double(util);
    pts[i + pitch * 3] = Jp;
    pts[i + pitch * 4] = x;
    pts[i + pitch * 5] = y;
    pts[i + pitch * 6] = vx;
    pts[i + pitch * 7] = vy;
    pts[i + pitch * 8] = Fn.a00; pts[i + pitch * 9] = Fn.a01; pts[i + pitch * 10] = Fn.a10; pts[i + pitch * 11] = Fn.a11;
    pts[i + pitch * 12] = B.a00; pts[i + pitch * 13] = B.a01; pts[i + pitch * 14] = B.a10; pts[i + pitch * 15] = B.a11;
    if (recordPQ) { pts[i + pitch * 1] = ptr; pts[i + pitch * 2] = qtr; }
}

// G2P + plasticity, one thread per particle
static __global__ void k_g2p_simple(StepParams P, double *__restrict__ pts, long pitch, int n, GridView g, int recordPQ,
                                    int *status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) g2p_one(P, pts, pitch, i, g, recordPQ, status);
}

}  // namespace icy_dev
