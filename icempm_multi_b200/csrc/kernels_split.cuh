// kernels_split.cuh -- FP32 "split precision" variant of the tiled step.
//
// Device state per point (17 lines of 4 bytes, `pitch` entries each):
//   utility (low 32 bits of the reference's 64-bit word), packed integer cell
//   (cx + 32768) << 16 | cy, FP32 offset inside the cell (ox, oy in [0,1)),
//   FP32 De = Fe - I, Jp, then vx, vy, Bp (4), P, Q.
// Positions as integer cell + FP32 offset keep ~1e-8 cells of resolution on
// any grid; holding Fe - I instead of Fe keeps full FP32 precision of the
// small elastic strain, and det(Fe) - 1 and dev(Fe Fe^T) are formed from De
// without cancellation.  Grid mass and momentum are FP32.  FP64 is kept for
// the return mapping of crushed points (the projected Fe is formed in FP64
// and stored back as Fe - I, so nearly equal singular values lose nothing)
// and for the indenter force bins.  The tiling, sorting and the three phases
// are those of the FP64 kernels in kernels_tiled.cuh.
#pragma once
#include "kernels_tiled.cuh"

namespace icy_dev {

enum SplitLine {
    S_UTIL = 0, S_CELL, S_OX, S_OY, S_D00, S_D01, S_D10, S_D11, S_JP,
    S_VX, S_VY, S_B00, S_B01, S_B10, S_B11, S_P, S_Q, S_NLINES
};

struct GrainConstF { float pmin2, k, msq; };

// FP32 copies of the per-step constants
struct SplitConsts {
    float h, hinv, dt, dt_hinv, s4, dtvd, dtg, vmax, vmax_sq, mass_ice, mass_water, mu, kappa, beta, pmax;
};

__host__ __device__ inline SplitConsts split_consts(const StepParams &P)
{
    SplitConsts c;
    c.h = (float)P.h; c.hinv = (float)P.hinv; c.dt = (float)P.dt; c.dt_hinv = (float)(P.dt * P.hinv);
    c.s4 = (float)(4. * P.hinv); c.dtvd = (float)P.dt_vol_Dpinv; c.dtg = (float)P.dt_gravity;
    c.vmax = (float)P.vmax; c.vmax_sq = (float)P.vmax_sq;
    c.mass_ice = (float)P.mass_ice; c.mass_water = (float)P.mass_water;
    c.mu = (float)P.mu; c.kappa = (float)P.kappa; c.beta = (float)P.beta; c.pmax = (float)P.pmax;
    return c;
}

static __global__ void k_grain_table_f32(const GrainConst *tab, GrainConstF *out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < GRAIN_TAB) out[s] = GrainConstF{(float)tab[s].pmin2, (float)tab[s].k, (float)tab[s].msq};
}

__device__ __forceinline__ unsigned pack_cell(int cx, int cy) { return ((unsigned)(cx + 32768) << 16) | (unsigned)cy; }
__device__ __forceinline__ void unpack_cell(unsigned k, int &cx, int &cy)
{
    cx = (int)(k >> 16) - 32768;
    cy = (int)(k & 0xffffu);
}

// Stencil base with the reference's truncation, (int)(x/h - 0.5) (kernels.cuh:90),
// from cell c and offset o (x/h = c + o), and the offset f = x/h - base.
__device__ __forceinline__ void split_base(int c, float o, int &base, float &f)
{
    const bool nonneg = c >= 1 || (c == 0 && o >= 0.5f);   // c + o - 0.5 >= 0
    base = nonneg ? (o >= 0.5f ? c : c - 1) : (o > 0.5f ? c + 1 : c);
    f = (float)(c - base) + o;
}

__device__ __forceinline__ void split_renorm(int &c, float &o)
{
    if (o >= 1.0f) { c += 1; o -= 1.0f; }
    else if (o < 0.0f) { c -= 1; o += 1.0f; }
    if (o >= 1.0f) o = 0.99999994f;   // o = 1 - ulp after rounding
}

// dev(Fe Fe^T) and J = det Fe from De = Fe - I, without cancellation:
// Fe Fe^T - I = De + De^T + De De^T, J - 1 = tr De + det De.
__device__ __forceinline__ void split_dev(const M2<float> &D, float &jm1, float &d00, float &d01)
{
    jm1 = (D.a00 + D.a11) + (D.a00 * D.a11 - D.a10 * D.a01);
    const float b00 = 2.f * D.a00 + D.a00 * D.a00 + D.a01 * D.a01;
    const float b11 = 2.f * D.a11 + D.a10 * D.a10 + D.a11 * D.a11;
    d00 = 0.5f * (b00 - b11);
    d01 = D.a01 + D.a10 + D.a00 * D.a10 + D.a01 * D.a11;
}

struct PointF {
    unsigned util;
    int cx, cy;
    float ox, oy, Jp, vx, vy, ptr, qtr;
    M2<float> D, B;
};

// The return mapping of a crushed point in FP64 (kernels.cuh:540-545, 623-674)
// from its FP32 state, out of line: few points take it, and keeping its FP64
// registers out of the tile kernel's main path leaves room for more warps.
struct SplitRm { float d00, d01, d10, d11, jp; };
static __device__ __noinline__ SplitRm return_map_split(const StepParams &P, float d00, float d01, float d10,
                                                        float d11, float jp)
{
    M2<double> F{1.0 + (double)d00, (double)d01, (double)d10, 1.0 + (double)d11};
    double Jp = jp;
    double Je64 = det2(F), p64 = (-(P.kappa / 2.)) * (Je64 * Je64 - 1.);
    M2<double> dv = dev_ffT(F);
    double q64 = ((kCoeff1 * P.mu) * (1. / Je64)) *
                 sqrt(((dv.a00 * dv.a00 + dv.a10 * dv.a10) + dv.a01 * dv.a01) + dv.a11 * dv.a11);
    return_map(P, F, Jp, p64, q64, Je64);
    return SplitRm{(float)(F.a00 - 1.0), (float)F.a01, (float)F.a10, (float)(F.a11 - 1.0), (float)Jp};
}

template <typename VSrc>
__device__ __forceinline__ bool g2p_update_f32(const StepParams &P, const SplitConsts &Q, const GrainConstF *tab,
                                               PointF &s, int *status, VSrc &&vsrc)
{
    int bx, by;
    float fx, fy;
    split_base(s.cx, s.ox, bx, fx);
    split_base(s.cy, s.oy, by, fy);
    const int e = base_error(P, bx, by);
    if (e) { *status = e; return false; }
    float wx[3], wy[3];
    bspline_weights(fx, wx);
    bspline_weights(fy, wy);
    // v = sum W v_i and Bp = 4/h sum W v_i (i - f)^T (kernels.cuh:357-372),
    // separably: sums over b with wy per column a, then over a with wx;
    // sum W v_i (i - f) = sum W v_i i - f v
    float2 nv[9];
    vsrc(bx, by, nv);
    float cvx[3], cvy[3], cbx[3], cby[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float2 n0 = nv[a * 3], n1 = nv[a * 3 + 1], n2 = nv[a * 3 + 2];
        cvx[a] = wy[0] * n0.x + wy[1] * n1.x + wy[2] * n2.x;
        cvy[a] = wy[0] * n0.y + wy[1] * n1.y + wy[2] * n2.y;
        cbx[a] = wy[1] * n1.x + 2.f * (wy[2] * n2.x);
        cby[a] = wy[1] * n1.y + 2.f * (wy[2] * n2.y);
    }
    const float vx = wx[0] * cvx[0] + wx[1] * cvx[1] + wx[2] * cvx[2];
    const float vy = wx[0] * cvy[0] + wx[1] * cvy[1] + wx[2] * cvy[2];
    const float sax = wx[1] * cvx[1] + 2.f * (wx[2] * cvx[2]), say = wx[1] * cvy[1] + 2.f * (wx[2] * cvy[2]);
    const float sbx = wx[0] * cbx[0] + wx[1] * cbx[1] + wx[2] * cbx[2];
    const float sby = wx[0] * cby[0] + wx[1] * cby[1] + wx[2] * cby[2];
    const M2<float> B{Q.s4 * (sax - fx * vx), Q.s4 * (sbx - fy * vx), Q.s4 * (say - fx * vy), Q.s4 * (sby - fy * vy)};
    // advection in cell units, x += v dt (kernels.cuh:375)
    s.ox += vx * Q.dt_hinv;
    s.oy += vy * Q.dt_hinv;
    split_renorm(s.cx, s.ox);
    split_renorm(s.cy, s.oy);
    // Fe <- (I + dt Bp) Fe  as  De <- De + T + T De,  T = dt Bp (kernels.cuh:376)
    const M2<float> T{Q.dt * B.a00, Q.dt * B.a01, Q.dt * B.a10, Q.dt * B.a11};
    const M2<float> D = s.D;
    s.D = {D.a00 + T.a00 + (T.a00 * D.a00 + T.a01 * D.a10), D.a01 + T.a01 + (T.a00 * D.a01 + T.a01 * D.a11),
           D.a10 + T.a10 + (T.a10 * D.a00 + T.a11 * D.a10), D.a11 + T.a11 + (T.a10 * D.a01 + T.a11 * D.a11)};
    s.ptr = 0.f;
    s.qtr = 0.f;
    if (s.util & (unsigned)kLiquid) {
        s.Jp *= (1.f + T.a00) * (1.f + T.a11) - T.a10 * T.a01;   // kernels.cuh:380
    } else {
        // ComputePQ (kernels.cuh:547-557) from De
        float jm1, d00, d01;
        split_dev(s.D, jm1, d00, d01);
        const float Je = 1.f + jm1;
        s.ptr = -(Q.kappa * 0.5f) * (jm1 * (Je + 1.f));
        s.qtr = __fdividef(2.f * Q.mu, Je) * sqrtf(d00 * d00 + d01 * d01);   // sqrt(2) mu/J |dev|, |dev| = sqrt(2(d00^2+d01^2))
        if (!(s.util & (unsigned)kCrushed)) {
            const GrainConstF *gc = tab + grain_slot((short)s.util);
            const float pmin2 = __ldg(&gc->pmin2), k = __ldg(&gc->k), msq = __ldg(&gc->msq);
            bool crushed;
            if (s.ptr < 0.f) crushed = s.ptr < pmin2 || s.qtr > k * (s.ptr - pmin2);
            else crushed = (1.f + 2.f * Q.beta) * s.qtr * s.qtr + msq * (s.ptr + Q.beta * Q.pmax) * (s.ptr - Q.pmax) > 0.f;
            if (crushed) s.util |= (unsigned)kCrushed;
        }
        if (s.util & (unsigned)kCrushed) {
            const SplitRm r = return_map_split(P, s.D.a00, s.D.a01, s.D.a10, s.D.a11, s.Jp);
            s.D = {r.d00, r.d01, r.d10, r.d11};
            s.Jp = r.jp;
        }
    }
    s.vx = vx;
    s.vy = vy;
    s.B = B;
    return true;
}

__device__ __forceinline__ void store_point_f32(unsigned *__restrict__ st, long pitch, long i, const PointF &s,
                                                bool write_vb, bool record_pq)
{
    float *f = reinterpret_cast<float *>(st);
    st[i] = s.util;
    st[i + pitch * S_CELL] = pack_cell(s.cx, s.cy);
    f[i + pitch * S_OX] = s.ox;
    f[i + pitch * S_OY] = s.oy;
    f[i + pitch * S_D00] = s.D.a00; f[i + pitch * S_D01] = s.D.a01;
    f[i + pitch * S_D10] = s.D.a10; f[i + pitch * S_D11] = s.D.a11;
    f[i + pitch * S_JP] = s.Jp;
    if (write_vb) {
        f[i + pitch * S_VX] = s.vx; f[i + pitch * S_VY] = s.vy;
        f[i + pitch * S_B00] = s.B.a00; f[i + pitch * S_B01] = s.B.a01;
        f[i + pitch * S_B10] = s.B.a10; f[i + pitch * S_B11] = s.B.a11;
    }
    if (record_pq) { f[i + pitch * S_P] = s.ptr; f[i + pitch * S_Q] = s.qtr; }
}

__device__ __forceinline__ void load_point_f32(const unsigned *__restrict__ st, long pitch, long i, PointF &s)
{
    const float *f = reinterpret_cast<const float *>(st);
    unpack_cell(st[i + pitch * S_CELL], s.cx, s.cy);
    s.ox = f[i + pitch * S_OX];
    s.oy = f[i + pitch * S_OY];
    s.D = {f[i + pitch * S_D00], f[i + pitch * S_D01], f[i + pitch * S_D10], f[i + pitch * S_D11]};
    s.Jp = f[i + pitch * S_JP];
}

// ---------------------------------------------------------------- P2G (FP32)
// Moments of a point as three vectors in shared memory, one padding column
// after every 4 points (the cell phase reads points about 4 apart per lane):
//   m0 = (fx, fy, mass, m vx),  m1 = (m vy, S00, S01, S10),  m2 = (S11, base)
// with S = m Bp - dt vol Dp_inv tau (simulation/kernels.cuh:57-92).
constexpr int CAPF = 1280;                // points per chunk of the FP32 tile kernel
constexpr int MOMF_N = CAPF + CAPF / 4;
constexpr size_t MOMF_BYTES = (2 * sizeof(float4) + sizeof(float2)) * MOMF_N;
static_assert(9 * TT * sizeof(float4) <= MOMF_BYTES, "cell partials alias the moment buffer");
__device__ __forceinline__ int momf_col(int j) { return j + (j >> 2); }
struct MomF {
    float4 *m0, *m1;
    float2 *m2;
    __device__ __forceinline__ explicit MomF(float *base)
        : m0(reinterpret_cast<float4 *>(base)), m1(reinterpret_cast<float4 *>(base) + MOMF_N),
          m2(reinterpret_cast<float2 *>(reinterpret_cast<float4 *>(base) + 2 * MOMF_N)) {}
    __device__ __forceinline__ void none(int j) const { m2[momf_col(j)] = make_float2(0.f, __int_as_float(BASE_NONE)); }
};

__device__ __forceinline__ void p2g_moments_f32(const StepParams &P, const SplitConsts &Q, const PointF &s,
                                                float *mom, int j, int *status)
{
    const MomF M(mom);
    const bool liquid = (s.util & (unsigned)kLiquid) != 0;
    const float mass = liquid ? Q.mass_water : Q.mass_ice;
    int bx, by;
    float fx, fy;
    split_base(s.cx, s.ox, bx, fx);
    split_base(s.cy, s.oy, by, fy);
    const int e = base_error(P, bx, by);
    if (e) {
        *status = e;
        M.none(j);
        return;
    }
    M2<float> tau;
    if (liquid) {
        const float sw = (float)(P.kappa * (1. - pow((double)s.Jp, -5.0)));   // Water (kernels.cuh:37-44)
        tau = {sw, 0.f, 0.f, sw};
    } else {
        // KirchhoffStress_Wolper (kernels.cuh:24-34) from De
        float jm1, d00, d01;
        split_dev(s.D, jm1, d00, d01);
        const float Je = 1.f + jm1;
        const float s1 = __fdividef(Q.mu, Je), s2 = (Q.kappa * 0.5f) * (jm1 * (Je + 1.f));
        tau = {s1 * d00 + s2, s1 * d01, s1 * d01, -s1 * d00 + s2};
    }
    const int c = momf_col(j);
    M.m0[c] = make_float4(fx, fy, mass, s.vx * mass);
    M.m1[c] = make_float4(s.vy * mass, mass * s.B.a00 - Q.dtvd * tau.a00, mass * s.B.a01 - Q.dtvd * tau.a01,
                          mass * s.B.a10 - Q.dtvd * tau.a10);
    M.m2[c] = make_float2(mass * s.B.a11 - Q.dtvd * tau.a11, __int_as_float(pack_base(bx, by)));
}

// FP32 grid of n nodes in one allocation of 6 n floats, in one of two layouts.
// Alone: five arrays m, px, py, vx, vy (scalar atomics; the bases are
// constant-bank operands).  In a batch (AOS): per node (m, px, py, -) as a
// float4 taken by one vector atomic, then a float2 velocity array: two bases
// to look up per member and fewer live addresses (the batched kernel spills
// less and runs 10 % faster; alone the scalar layout is 2.5 % faster).
struct GridViewF {
    float *m, *px, *py, *vx, *vy;   // alone
    float4 *mp;                     // in a batch (same memory)
    float2 *v;
    int ny, halo;
    // node (m, px, py) += (dm, dpx, dpy)
    template <bool AOS>
    __device__ __forceinline__ void add(long k, float dm, float dpx, float dpy) const
    {
        if constexpr (AOS) {
            atomicAdd(mp + k, make_float4(dm, dpx, dpy, 0.f));
        } else {
            atomicAdd(m + k, dm);
            atomicAdd(px + k, dpx);
            atomicAdd(py + k, dpy);
        }
    }
    template <bool AOS>
    __device__ __forceinline__ float2 vel(long k) const
    {
        if constexpr (AOS) return v[k];
        else return make_float2(vx[k], vy[k]);
    }
    __device__ __forceinline__ long idx(int gx, int gy) const { return (long)(gx + halo) * ny + gy; }
};

struct SplitArgs {
    StepParams P;
    SplitConsts Q;
    TileGeom G;
    GridViewF g;
    unsigned *st;
    long pitch;
    const int *cell_start, *active, *n_active;
    unsigned *flags;
    int2 *tlist;        // node tiles written since the last update, each once: (inst, tile)
    unsigned *tlist_n;  // [0] entries, [1] CTAs of the update done
    int inst;           // this instance's slot in a batch (0 alone)
    int *status;
    unsigned long long *moved;
    int *claim;         // batch: [0] next work item to hand out, [1] CTAs finished (zero between launches)
    const GrainConstF *grain_tab;
    int record_pq;
    double *acc;        // indenter force bins
    long n_nodes;       // nodes of the grid
};

#ifdef ICY_BATCH_CONST_ARGS
// Only in batch_cargs.cu: the member arguments of a batch of at most
// BATCH_CONST_SLOTS slots, copied to the constant bank, where the batched
// tile kernel reads them as the single-instance kernel reads its own (no
// global loads and fewer spills in the point loop).  In its own translation
// unit so that the kernels reading the global table compile as before.
constexpr int BATCH_CONST_SLOTS = 128;
static __constant__ SplitArgs c_batch_args[BATCH_CONST_SLOTS];
#endif

// P2G contributions of one point to its 3 x 3 nodes (simulation/kernels.cuh:
// 100-120): node (a, b) gets W m and W (m v + S d) with W = wx[a] wy[b] and
// d = ((a - fx) h, (b - fy) h).  S d is affine in (a, b), so it is evaluated
// as c0 + a S(:,0) h + b S(:,1) h: per node one product for W and one
// multiply-add per component.
template <typename Sink>
__device__ __forceinline__ void point_contributions_f32(float h, float fx, float fy, float mass, float mvx,
                                                        float mvy, float s00, float s01, float s10, float s11,
                                                        Sink &&sink)
{
    float wx[3], wy[3];
    bspline_weights(fx, wx);
    bspline_weights(fy, wy);
    const float s00h = s00 * h, s01h = s01 * h, s10h = s10 * h, s11h = s11 * h;
    const float c0x = mvx - (s00h * fx + s01h * fy), c0y = mvy - (s10h * fx + s11h * fy);
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float ax = c0x + (float)a * s00h, ay = c0y + (float)a * s10h;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const float W = wx[a] * wy[b];
            sink(a, b, W, W * mass, ax + (float)b * s01h, ay + (float)b * s11h);
        }
    }
}

template <bool AOS>
static __device__ __noinline__ void p2g_global_f32(GridViewF g, unsigned *flags, int2 *tlist, unsigned *tlist_n,
                                                   int inst, int ntx, int halo, float h, int bx, int by, float fx,
                                                   float fy, float mass, float mvx, float mvy, float s00, float s01,
                                                   float s10, float s11)
{
    point_contributions_f32(h, fx, fy, mass, mvx, mvy, s00, s01, s10, s11,
                            [&](int a, int b, float W, float dm, float tx, float ty) {
                                g.add<AOS>(g.idx(bx + a, by + b), dm, W * tx, W * ty);
                            });
    const int t0x = (bx + halo) / TX, t1x = (bx + 2 + halo) / TX;
    const int t0y = by / TY, t1y = (by + 2) / TY;
    mark_tile(flags, tlist, tlist_n, inst, t0x, t0y, ntx);
    if (t1x != t0x) mark_tile(flags, tlist, tlist_n, inst, t1x, t0y, ntx);
    if (t1y != t0y) {
        mark_tile(flags, tlist, tlist_n, inst, t0x, t1y, ntx);
        if (t1x != t0x) mark_tile(flags, tlist, tlist_n, inst, t1x, t1y, ntx);
    }
}

// phases 2 and 3 (see p2g_cells_and_flush in kernels_tiled.cuh), in FP32
template <int NT, bool AOS, typename Sync>
__device__ __forceinline__ void p2g_cells_and_flush_f32(const SplitArgs &A, int tid, int tx, int ty, int cs, int ce,
                                                        const int *s_cs, float *mom, float (*s_odd)[RN],
                                                        unsigned &touch, unsigned &moved, Sync &&sync)
{
    const StepParams &P = A.P;
    const int X0 = tx * TX - P.halo, Y0 = ty * TY;
    const int RX0 = X0 - RM, RY0 = Y0 - RM;
    float acc[27];
#pragma unroll
    for (int q = 0; q < 27; q++) acc[q] = 0.f;
    if (tid < TT) {
        const int bxc = X0 + tid / TY, byc = Y0 + tid % TY;
        const int r0 = max(s_cs[tid], cs) - cs, r1 = min(s_cs[tid + 1], ce) - cs;
        const MomF M(mom);
        for (int j = r0; j < r1; j++) {
            const int c = momf_col(j);
            const float2 q2 = M.m2[c];
            const int pb = __float_as_int(q2.y);
            if (pb == BASE_NONE) continue;
            int bx, by;
            unpack_base(pb, bx, by);
            const float4 q0 = M.m0[c], q1 = M.m1[c];
            const float fx = q0.x, fy = q0.y, mass = q0.z, mvx = q0.w, mvy = q1.x;
            const float s00 = q1.y, s01 = q1.z, s10 = q1.w, s11 = q2.x;
            if (bx == bxc && by == byc) {
                point_contributions_f32(A.Q.h, fx, fy, mass, mvx, mvy, s00, s01, s10, s11,
                                        [&](int a, int b, float W, float dm, float tx, float ty) {
                                            const int q = (a * 3 + b) * 3;
                                            acc[q] += dm;
                                            acc[q + 1] += W * tx;
                                            acc[q + 2] += W * ty;
                                        });
            } else {
                moved++;
                const int lx = bx - RX0, ly = by - RY0;
                if (lx >= 0 && lx + 2 < RX && ly >= 0 && ly + 2 < RY) {
                    point_contributions_f32(A.Q.h, fx, fy, mass, mvx, mvy, s00, s01, s10, s11,
                                            [&](int a, int b, float W, float dm, float tx, float ty) {
                                                const int k = (lx + a) * RY + (ly + b);
                                                atomicAdd(&s_odd[0][k], dm);
                                                atomicAdd(&s_odd[1][k], W * tx);
                                                atomicAdd(&s_odd[2][k], W * ty);
                                            });
                } else {
                    p2g_global_f32<AOS>(A.g, A.flags, A.tlist, A.tlist_n, A.inst, A.G.ntx, P.halo, A.Q.h, bx, by, fx, fy, mass, mvx, mvy, s00, s01,
                                   s10, s11);
                }
            }
        }
    }
    sync();
    float4 *part = reinterpret_cast<float4 *>(mom);   // [9 node offsets][TT cells], aliasing the moments
    if (tid < TT) {
#pragma unroll
        for (int q = 0; q < 9; q++) part[q * TT + tid] = make_float4(acc[3 * q], acc[3 * q + 1], acc[3 * q + 2], 0.f);
    }
    sync();
    for (int k = tid; k < RN; k += NT) {
        const int i = k / RY, jj = k % RY;
        const int nx = i - RM, ny = jj - RM;
        float m = 0.f, px = 0.f, py = 0.f;
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const int cx = nx - a;
            if (cx < 0 || cx >= TX) continue;
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const int cy = ny - b;
                if (cy < 0 || cy >= TY) continue;
                const float4 v = part[(a * 3 + b) * TT + cx * TY + cy];
                m += v.x;
                px += v.y;
                py += v.z;
            }
        }
        m += s_odd[0][k]; px += s_odd[1][k]; py += s_odd[2][k];
        s_odd[0][k] = 0.f; s_odd[1][k] = 0.f; s_odd[2][k] = 0.f;
        if (m != 0.f || px != 0.f || py != 0.f) {
            const int gx = RX0 + i, gy = RY0 + jj;
            A.g.add<AOS>(A.g.idx(gx, gy), m, px, py);
            const int dx = (gx + P.halo) / TX - tx + 1, dy = gy / TY - ty + 1;
            touch |= 1u << (dy * 3 + dx);
        }
    }
    sync();
}

// Threads and resident CTAs per SM of the FP32 tile kernel.
constexpr int TILE_THREADS_F32 = 256, TILE_CTAS_F32 = 3;

// Work items of a batch: (instance, tile) pairs over all instances.
struct BatchItem { int inst, tile; };

// Starts moving the next work item's point lines (line `which` < S_JP + 1) or
// cell ranges (which == S_JP + 1) into L2 while this CTA is in its cell phase.
template <bool BATCH>
__device__ __forceinline__ void prefetch_next_item(const SplitArgs &A1, const SplitArgs *Aarr, const BatchItem *work,
                                                   int next, int na, int which)
{
    if (next >= na) return;
    const BatchItem w = BATCH ? work[next] : BatchItem{0, A1.active[next]};
    const SplitArgs &A = BATCH ? Aarr[w.inst] : A1;
    const int *cs = A.cell_start + (long)w.tile * TT;
    if (which == S_JP + 1) {
        prefetch_l2(cs, (TT + 1) * sizeof(int));
        return;
    }
    const int ps = cs[0], pe = cs[TT];
    if (pe > ps) prefetch_l2(A.st + A.pitch * which + ps, (size_t)(pe - ps) * sizeof(unsigned));
}

// Tile kernel over the FP32 state: <G2P, P2G, write vel/Bp> as k_tile.
// With BATCH, the CTAs walk the (instance, tile) list of many independent
// instances, each with its own parameters, grid and points (Aarr[inst]), and
// the record-PQ flag of each instance comes from rec[inst].
template <bool DO_G2P, bool DO_P2G, bool WRITE_VB, bool BATCH = false>
static __global__ void __launch_bounds__(TILE_THREADS_F32, TILE_CTAS_F32)
    k_tile_f32(const __grid_constant__ SplitArgs A1, const SplitArgs *__restrict__ Aarr = nullptr, const BatchItem *__restrict__ work = nullptr,
               const int *__restrict__ nwork = nullptr, const int *__restrict__ rec = nullptr)
{
    __shared__ float2 s_v[RN];
    __shared__ float s_odd[3][RN];
    __shared__ int s_cs[TT + 1];
    __shared__ unsigned s_touch;
    __shared__ int s_claim;
    extern __shared__ float4 s_momf4[];
    float *const s_momf = reinterpret_cast<float *>(s_momf4);
    const int na = BATCH ? *nwork : *A1.n_active;
    const int tid = threadIdx.x;
    // Alone, CTA c takes the tiles c, c + gridDim.x, ... (equal tiles, and no
    // claim to wait for: 5 % faster).  In a batch, where the items differ in
    // size, they are handed out one at a time (A1.claim[0]), each CTA claiming
    // its next item when it starts one, so that the CTAs finish together (4 %).
    if (BATCH && tid == 0) s_claim = atomicAdd(A1.claim, 1);
    for (int k = tid; k < RN; k += blockDim.x) { s_odd[0][k] = 0.f; s_odd[1][k] = 0.f; s_odd[2][k] = 0.f; }
    __syncthreads();
    int ti = BATCH ? s_claim : (int)blockIdx.x;
    __syncthreads();   // everybody has read s_claim; later reads of it come before the item's last barrier
    while (ti < na) {
        const BatchItem w = BATCH ? work[ti] : BatchItem{0, A1.active[ti]};
        if (BATCH && tid == 0) s_claim = atomicAdd(A1.claim, 1);
#ifdef ICY_BATCH_CONST_ARGS
        const SplitArgs &A = BATCH ? c_batch_args[w.inst] : A1;
#else
        const SplitArgs &A = BATCH ? Aarr[w.inst] : A1;
#endif
        const StepParams &P = A.P;
        const bool record = BATCH ? rec[w.inst] != 0 : A.record_pq != 0;
        const float *fst = reinterpret_cast<const float *>(A.st);
        unsigned moved = 0;
        const int t = w.tile;
        const int tx = t % A.G.ntx, ty = t / A.G.ntx;
        const int RX0 = tx * TX - P.halo - RM, RY0 = ty * TY - RM;
        for (int c = tid; c <= TT; c += blockDim.x) s_cs[c] = A.cell_start[(long)t * TT + c];
        if (tid == 0) s_touch = 0;
        if (DO_G2P) {
            for (int k = tid; k < RN; k += blockDim.x) {
                const int gx = RX0 + k / RY, gy = RY0 + k % RY;
                s_v[k] = node_in_grid(P, gx, gy) ? A.g.vel<BATCH>(A.g.idx(gx, gy)) : make_float2(0.f, 0.f);
            }
        }
        __syncthreads();
        const int next = BATCH ? s_claim : ti + (int)gridDim.x;
        const int ps = s_cs[0], pe = s_cs[TT];
        // the 3 x 3 node velocities of a stencil: from the staged region (one check
        // per point), else from the grid
        auto vsrc = [&](int bx, int by, float2 *nv) {
            const int lx = bx - RX0, ly = by - RY0;
            if (lx >= 0 && lx + 2 < RX && ly >= 0 && ly + 2 < RY) {
                const float2 *r = s_v + lx * RY + ly;
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) nv[a * 3 + b] = r[a * RY + b];
            } else {
#pragma unroll
                for (int a = 0; a < 3; a++)
#pragma unroll
                    for (int b = 0; b < 3; b++) nv[a * 3 + b] = A.g.vel<BATCH>(A.g.idx(bx + a, by + b));
            }
        };
        unsigned touch = 0;
        for (int cs = ps; cs < pe; cs += CAPF) {
            const int ce = min(cs + CAPF, pe);
            for (int j = tid; j < ce - cs; j += blockDim.x) {
                const long i = cs + j;
                PointF s;
                s.util = A.st[i];
                if (s.util & (unsigned)kDisabled) {
                    if (DO_P2G) MomF(s_momf).none(j);
                    continue;
                }
                load_point_f32(A.st, A.pitch, i, s);
                if (DO_G2P) {
                    if (!g2p_update_f32(P, A.Q, A.grain_tab, s, A.status, vsrc)) {
                        if (DO_P2G) MomF(s_momf).none(j);
                        continue;
                    }
                    store_point_f32(A.st, A.pitch, i, s, WRITE_VB, record);
                } else {
                    s.vx = fst[i + A.pitch * S_VX];
                    s.vy = fst[i + A.pitch * S_VY];
                    s.B = {fst[i + A.pitch * S_B00], fst[i + A.pitch * S_B01], fst[i + A.pitch * S_B10],
                           fst[i + A.pitch * S_B11]};
                }
                if (DO_P2G) p2g_moments_f32(P, A.Q, s, s_momf, j, A.status);
            }
            __syncthreads();
            // threads without a cell in the cell phase (else the last ones) start the
            // next item's loads
            constexpr int PF0 = TT < TILE_THREADS_F32 ? TT : TILE_THREADS_F32 - (S_JP + 2);
            if (DO_P2G && cs == ps && tid >= PF0 && tid < PF0 + S_JP + 2)
                prefetch_next_item<BATCH>(A1, Aarr, work, next, na, tid - PF0);
            // and the first threads its staged node velocities (columns of vx and vy,
            // or of the float2 velocities of a batch member)
            if (DO_G2P && DO_P2G && cs == ps && tid < (BATCH ? 1 : 2) * RX && next < na) {
                const BatchItem wn = BATCH ? work[next] : BatchItem{0, A1.active[next]};
                const SplitArgs &An = BATCH ? Aarr[wn.inst] : A1;
                const int nx0 = (wn.tile % An.G.ntx) * TX - An.P.halo - RM, ny0 = (wn.tile / An.G.ntx) * TY - RM;
                if (BATCH)
                    prefetch_region_column(An.g.v, An.P.gridx, An.P.gridy, An.P.halo, An.g.ny, nx0, ny0, tid);
                else
                    prefetch_region_column(tid < RX ? An.g.vx : An.g.vy, An.P.gridx, An.P.gridy, An.P.halo, An.g.ny,
                                           nx0, ny0, tid % RX);
            }
            if (DO_P2G)
                p2g_cells_and_flush_f32<TILE_THREADS_F32, BATCH>(A, tid, tx, ty, cs, ce, s_cs, s_momf, s_odd, touch, moved,
                                                      [] { __syncthreads(); });
        }
        if (DO_P2G) {
            touch = __reduce_or_sync(0xffffffffu, touch);
            if ((tid & 31) == 0 && touch) atomicOr(&s_touch, touch);
            __syncthreads();
            if (tid < 9 && ((s_touch >> tid) & 1u)) {
                const int ntx = tx + tid % 3 - 1, nty = ty + tid / 3 - 1;
                mark_tile(A.flags, A.tlist, A.tlist_n, A.inst, ntx, nty, A.G.ntx);
            }
            moved = __reduce_add_sync(0xffffffffu, moved);
            if ((tid & 31) == 0 && moved) atomicAdd(A.moved, (unsigned long long)moved);
        }
        __syncthreads();
        ti = next;
    }
    // the last CTA to finish resets the counters for the next launch: every
    // CTA's last claim came before its count
    if (BATCH && tid == 0) {
        __threadfence();
        if (atomicAdd(A1.claim + 1, 1) == (int)gridDim.x - 1) {
            A1.claim[0] = 0;
            A1.claim[1] = 0;
            __threadfence();
        }
    }
}

// Grid update of one node in FP32 (simulation/kernels.cuh:175-300) from its
// mass and momentum, the indenter geometry and the force in FP64: the new
// velocity, and the force bin of a contact node (-1 if none).
__device__ __forceinline__ int node_velocity_f32(const StepParams &P, const SplitConsts &Q, int gx, int gy, float mass,
                                                 float px, float py, double ind_x, double ind_y, float &vx, float &vy,
                                                 double &fxd, double &fyd)
{
    vx = 0.f;
    vy = 0.f;
    int bin = -1;
    if (mass != 0.f) {
        const float rm = __fdividef(1.f, mass);   // fast reciprocal (FP32 path)
        vx = px * rm;
        vy = py * rm;
        vy -= Q.dtg;
        const float v2 = vx * vx + vy * vy;
        if (v2 > Q.vmax_sq) {
            const float r = sqrtf(v2);
            vx = vx / r * Q.vmax;
            vy = vy / r * Q.vmax;
        }
        double nx = (double)gx * P.h - ind_x, ny = (double)gy * P.h - ind_y;
        if (nx * nx + ny * ny < P.ind_rsq) {
            const double r = sqrt(nx * nx + ny * ny);
            if (r > 0) { nx /= r; ny /= r; }
            const float fnx = (float)nx, fny = (float)ny;
            const float vrx = vx - (float)P.ind_v, vry = vy;
            const float vn = vrx * fnx + vry * fny;
            if (vn < 0.f) {
                const float vtx = vrx - fnx * vn, vty = vry - fny * vn;
                const float pvx = vx, pvy = vy;
                vx = (float)P.ind_v + vtx;
                vy = vty;
                fxd = (double)(pvx - vx) * mass / P.dt;
                fyd = (double)(pvy - vy) * mass / P.dt;
                float angle = atan2f(fnx, fny);
                angle = (float)((double)angle + kPi);
                angle = (float)((double)angle * (P.nsub / (2 * kPi)));
                bin = min(max((int)angle, 0), P.nsub - 1);
            }
        }
        if (gy <= 2) { vx = 0.f; vy = 0.f; }
        if (gy >= P.gridy - 3 && vy > 0.f) vy = 0.f;
        if (gx <= 2 && vx < 0.f) vx = 0.f;
        else if (gx >= P.gridx - 3 && vx > 0.f) vx = 0.f;
    }
    return bin;
}

struct BatchClock;
constexpr int UPD_TILES = 4;

// Grid update of the listed node tiles (see k_update_list in kernels_tiled.cuh),
// defined after BatchClock below.
template <bool BATCH>
static __global__ void __launch_bounds__(256, 4) k_update_list_f32(const __grid_constant__ SplitArgs A1,
                                                                const SplitArgs *__restrict__ Aarr,
                                                                const BatchClock *__restrict__ clk,
                                                                const int2 *__restrict__ tlist, unsigned *tlist_n,
                                                                double ind_x, double ind_y);

// ---------------------------------------------------------------- binning / conversion
static __global__ void k_bin_count_f32(StepParams P, TileGeom G, const unsigned *__restrict__ st, long pitch, int n,
                                int *keys, int *ranks, int *counts, int *status)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool in = i < n;
    int key = G.ntiles * TT;
    if (in) {
        const unsigned u = st[i];
        if (!(u & (unsigned)kDisabled)) {
            int cx, cy, bx, by;
            float fx, fy;
            unpack_cell(st[i + pitch * S_CELL], cx, cy);
            const float *f = reinterpret_cast<const float *>(st);
            split_base(cx, f[i + pitch * S_OX], bx, fx);
            split_base(cy, f[i + pitch * S_OY], by, fy);
            const int e = base_error(P, bx, by);
            if (e) *status = e;
            else key = G.cell_key(bx, by, P.halo);
        }
    }
    const unsigned act = __ballot_sync(0xffffffffu, in);
    if (!in) return;
    const unsigned peers = __match_any_sync(act, key);
    const int lane = threadIdx.x & 31, leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(&counts[key], __popc(peers));
    base = __shfl_sync(peers, base, leader);
    keys[i] = key;
    ranks[i] = base + __popc(peers & ((1u << lane) - 1u));
}

static __global__ void k_bin_scatter_f32(const unsigned *__restrict__ src, unsigned *__restrict__ dst, long pitch, int n,
                                  const int *__restrict__ keys, const int *__restrict__ ranks,
                                  const int *__restrict__ start, const int *__restrict__ oidx_src,
                                  int *__restrict__ oidx_dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int d = start[keys[i]] + ranks[i];
#pragma unroll
    for (int l = 0; l < S_NLINES; l++) dst[d + pitch * l] = src[i + pitch * l];
    oidx_dst[d] = oidx_src[i];
}

// FP64 HSSOA chunk (16 lines, stride cpitch) -> FP32 state slots [first, first+count)
static __global__ void k_split_from_hssoa(const double *__restrict__ chunk, long cpitch, int count, unsigned *st,
                                   long pitch, int first, double hinv)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const long i = first + j;
    float *f = reinterpret_cast<float *>(st);
    auto L = [&](int l) { return chunk[j + cpitch * l]; };
    st[i] = (unsigned)(unsigned long long)__double_as_longlong(L(0));
    int c[2];
    float o[2];
    for (int k = 0; k < 2; k++) {
        const double xs = L(4 + k) * hinv;
        const double fl = floor(xs);
        c[k] = (int)fl;
        o[k] = (float)(xs - fl);
        if (o[k] >= 1.0f) { c[k] += 1; o[k] = 0.0f; }
    }
    st[i + pitch * S_CELL] = pack_cell(c[0], c[1]);
    f[i + pitch * S_OX] = o[0];
    f[i + pitch * S_OY] = o[1];
    f[i + pitch * S_D00] = (float)(L(8) - 1.0);
    f[i + pitch * S_D01] = (float)L(9);
    f[i + pitch * S_D10] = (float)L(10);
    f[i + pitch * S_D11] = (float)(L(11) - 1.0);
    f[i + pitch * S_JP] = (float)L(3);
    f[i + pitch * S_VX] = (float)L(6);
    f[i + pitch * S_VY] = (float)L(7);
    for (int k = 0; k < 4; k++) f[i + pitch * (S_B00 + k)] = (float)L(12 + k);
    f[i + pitch * S_P] = (float)L(1);
    f[i + pitch * S_Q] = (float)L(2);
}

// FP32 state -> FP64 HSSOA chunk of upload positions [first, first+count);
// inv[o] is the slot holding the point uploaded at position o.
static __global__ void k_split_to_hssoa(const unsigned *__restrict__ st, long pitch, const int *__restrict__ inv, int first,
                                 int count, double *__restrict__ chunk, long cpitch, double h)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const long i = inv ? inv[first + j] : first + j;
    const float *f = reinterpret_cast<const float *>(st);
    auto W = [&](int l, double v) { chunk[j + cpitch * l] = v; };
    W(0, __longlong_as_double((long long)st[i]));
    int cx, cy;
    unpack_cell(st[i + pitch * S_CELL], cx, cy);
    W(4, ((double)cx + (double)f[i + pitch * S_OX]) * h);
    W(5, ((double)cy + (double)f[i + pitch * S_OY]) * h);
    W(8, 1.0 + (double)f[i + pitch * S_D00]);
    W(9, (double)f[i + pitch * S_D01]);
    W(10, (double)f[i + pitch * S_D10]);
    W(11, 1.0 + (double)f[i + pitch * S_D11]);
    W(3, (double)f[i + pitch * S_JP]);
    W(6, (double)f[i + pitch * S_VX]);
    W(7, (double)f[i + pitch * S_VY]);
    for (int k = 0; k < 4; k++) W(12 + k, (double)f[i + pitch * (S_B00 + k)]);
    W(1, (double)f[i + pitch * S_P]);
    W(2, (double)f[i + pitch * S_Q]);
}

static __global__ void k_inverse_perm(const int *__restrict__ oidx, int n, int *__restrict__ inv)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) inv[oidx[i]] = i;
}

}  // namespace icy_dev

namespace icy_dev {

// ---------------------------------------------------------------- batches
// Time stepping of one batch member on the device, so that a sequence of
// sub-steps can be replayed as a CUDA graph: the reference's
// `t += dt; indenter_x = indenter_x_initial + t * IndVelocity`
// (simulation/model.cpp:40-41), evaluated with explicit round-to-nearest
// operations (no FMA contraction), as the host does it.
struct BatchClock {
    double t, dt, x0, y0, v, ind_x;
    long long step;   // index of the next sub-step
    int every;        // UpdateEveryNthStep
    int live;         // 0 = free slot
};

static __global__ void k_batch_advance(BatchClock *clk, int *rec, int nslots)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nslots || !clk[i].live) return;
    BatchClock c = clk[i];
    c.t = __dadd_rn(c.t, c.dt);
    c.ind_x = __dadd_rn(c.x0, __dmul_rn(c.t, c.v));
    rec[i] = (c.step % c.every) == 0;
    c.step += 1;
    clk[i] = c;
}

// Grid update of the listed node tiles: each group of TT threads takes one
// TX x TY node tile (one thread per node), clears its mark, and the last CTA empties
// the list.  Alone (BATCH = false) the forces are summed per CTA in shared
// memory; in a batch every entry names its member, whose indenter position
// comes from the member's clock and whose force bins take the force directly.
template <bool BATCH>
static __global__ void __launch_bounds__(256, 4) k_update_list_f32(const __grid_constant__ SplitArgs A1,
                                                                const SplitArgs *__restrict__ Aarr,
                                                                const BatchClock *__restrict__ clk,
                                                                const int2 *__restrict__ tlist, unsigned *tlist_n,
                                                                double ind_x, double ind_y)
{
    extern __shared__ double s_acc[];   // 2*nsub (alone only)
    if (!BATCH) {
        for (int k = threadIdx.x; k < 2 * A1.P.nsub; k += blockDim.x) s_acc[k] = 0;
        __syncthreads();
    }
    bool any = false;
    const unsigned n = *(volatile unsigned *)tlist_n;
    constexpr int TPC = 256 / TT;   // node tiles per CTA pass
    static_assert(256 % TT == 0, "whole node tiles per 256-thread CTA");
    const int l = threadIdx.x % TT;
    const unsigned stride = gridDim.x * TPC;
    // UPD_TILES tiles per pass, their loads issued together
    for (unsigned e0 = blockIdx.x * TPC + threadIdx.x / TT; e0 < n; e0 += stride * UPD_TILES) {
        long q[UPD_TILES];
        int inst[UPD_TILES], gx[UPD_TILES], gy[UPD_TILES];
        float m[UPD_TILES], px[UPD_TILES], py[UPD_TILES];
#pragma unroll
        for (int u = 0; u < UPD_TILES; u++) {
            const unsigned e = e0 + u * stride;
            q[u] = -1;
            if (e >= n) continue;
            const int2 it = tlist[e];
            inst[u] = it.x;
            const SplitArgs &A = BATCH ? Aarr[it.x] : A1;
            const int tx = it.y & 0xffff, ty = it.y >> 16;
            if (l == 0) A.flags[ty * A.G.ntx + tx] = 0u;
            gx[u] = tx * TX + l / TY - A.P.halo;
            gy[u] = ty * TY + (l & (TY - 1));
            if (gx[u] >= A.P.gridx + A.P.halo || gy[u] >= A.P.gridy) continue;   // past the grid edge
            q[u] = A.g.idx(gx[u], gy[u]);
            if constexpr (BATCH) {
                const float4 a = A.g.mp[q[u]];
                m[u] = a.x;
                px[u] = a.y;
                py[u] = a.z;
            } else {
                m[u] = A.g.m[q[u]];
                px[u] = A.g.px[q[u]];
                py[u] = A.g.py[q[u]];
            }
        }
#pragma unroll
        for (int u = 0; u < UPD_TILES; u++) {
            if (q[u] < 0) continue;
            const SplitArgs &A = BATCH ? Aarr[inst[u]] : A1;
            float vx, vy;
            double fx = 0, fy = 0;
            const int bin = node_velocity_f32(A.P, A.Q, gx[u], gy[u], m[u], px[u], py[u],
                                              BATCH ? clk[inst[u]].ind_x : ind_x, BATCH ? clk[inst[u]].y0 : ind_y,
                                              vx, vy, fx, fy);
            if constexpr (BATCH) {
                A.g.v[q[u]] = make_float2(vx, vy);
                A.g.mp[q[u]] = make_float4(0.f, 0.f, 0.f, 0.f);
            } else {
                A.g.vx[q[u]] = vx;
                A.g.vy[q[u]] = vy;
                A.g.m[q[u]] = 0.f;
                A.g.px[q[u]] = 0.f;
                A.g.py[q[u]] = 0.f;
            }
            if (bin >= 0) {
                if (BATCH) {
                    atomicAdd(A.acc + 2 * bin, fx);
                    atomicAdd(A.acc + 2 * bin + 1, fy);
                } else {
                    atomicAdd(&s_acc[2 * bin], fx);
                    atomicAdd(&s_acc[2 * bin + 1], fy);
                    any = true;
                }
            }
        }
    }
    if (!BATCH && __syncthreads_or(any))
        for (int k = threadIdx.x; k < 2 * A1.P.nsub; k += blockDim.x)
            if (s_acc[k] != 0.0) atomicAdd(A1.acc + k, s_acc[k]);
    if (BATCH) __syncthreads();
    if (threadIdx.x == 0) tile_list_done(tlist_n);
}

// (instance, tile) work list: offsets by an exclusive scan over the members'
// non-empty-tile counts (one CTA), then a fill
static __global__ void __launch_bounds__(1024) k_batch_work_offsets(const SplitArgs *__restrict__ Aarr,
                                                                    const BatchClock *__restrict__ clk, int nslots,
                                                                    int *off, int *nwork)
{
    __shared__ int s_warp[32];
    const int per = (nslots + 1023) / 1024;
    const int b = min((int)threadIdx.x * per, nslots), e = min(b + per, nslots);
    int s = 0;
    for (int i = b; i < e; i++) s += clk[i].live ? *Aarr[i].n_active : 0;
    int total;
    int run = block_exclusive_scan<1024>(s, s_warp, total);
    for (int i = b; i < e; i++) {
        off[i] = run;
        run += clk[i].live ? *Aarr[i].n_active : 0;
    }
    if (threadIdx.x == 0) *nwork = total;
}

static __global__ void k_batch_work_fill(const SplitArgs *__restrict__ Aarr, const BatchClock *__restrict__ clk,
                                         const int *__restrict__ off, BatchItem *work)
{
    const int s = blockIdx.y;
    if (!clk[s].live) return;
    const int n = *Aarr[s].n_active;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        work[off[s] + k] = BatchItem{s, Aarr[s].active[k]};
}

}  // namespace icy_dev
