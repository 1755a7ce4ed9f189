// kernels_split.cuh -- FP32 "split precision" variant of the tiled step.
//
// Device state, in blocks of 32 points (point i: block i / 32, lane i % 32),
// `pitch` points of capacity (a multiple of 32), 17 words per point:
//   hot part, read and written at every step, 288 words per block:
//     words [0, 128)    one 16-byte vector per point: (base word, gx, gy, utility),
//                       the utility word's bits 19-29 holding the point's
//                       failure-surface table entry, marked by bit 30, where
//                       the input left bits 19-31 clear
//     words [128, 256)  one 16-byte vector per point: De = Fe - I by columns (d00, d10, d01, d11)
//     words [256, 288)  Jp_inv per point
//   cold part (from word 9 * pitch on), written on the last step of a call
//   and on record steps only, 256 words per block:
//     words [0, 128)    (vx, vy, P, Q) per point
//     words [128, 256)  Bp by columns (b00, b10, b01, b11) per point
// so that a thread reads and writes a point's step state with two 128-bit
// and one 32-bit access, a warp's accesses are contiguous, and a tile's
// points (consecutive after binning) are one contiguous range of the hot part.
//
// Position: the reference's stencil base b = (int)(x/h - 0.5) (truncation,
// simulation/kernels.cuh:90), packed with 16 bits per axis in the base word,
// and g = x/h - b - 1 in FP32: g lies in [-0.5, 0.5) wherever x/h >= 0.5
// (elsewhere the truncation puts it in (-1.5, -0.5]).  The quadratic
// B-spline weights are 0.5 (0.5 - g)^2, 0.75 - g^2, 0.5 (0.5 + g)^2, the node
// offsets (i - fx) are (i - 1 - g), nothing is re-based between G2P and P2G,
// and moving a point to the next base (g -= 1 or g += 1 from [0.5, 1) or
// [-1, -0.5)) is exact.  g keeps ~3e-8 cells of resolution on any grid.
// Holding Fe - I instead of Fe keeps full FP32 precision of the small elastic
// strain, and det(Fe) - 1 and dev(Fe Fe^T) are formed from De without
// cancellation.  Grid mass and momentum are FP32.  FP64 is kept for the
// return mapping of crushed points (the projected Fe is formed in FP64 and
// stored back as Fe - I, so nearly equal singular values lose nothing) and
// for the indenter force bins.  The tiling, sorting and the three phases are
// those of the FP64 kernels in kernels_tiled.cuh.
#pragma once
#include "kernels_tiled.cuh"

namespace icy_dev {

// Tile shapes of the FP32 path: TX x TY cells (stencil bases) per tile and
// the tile's staged node region (its bases, a drift margin of RM cells and
// the +2 stencil reach).  32 x 8 is the default; the autotuner times the
// others per workload (icempm_multi_b200/autotune.py).  Functions templated
// on a shape declare its constants locally (ICY_TILE_SHAPE), shadowing the
// 32 x 8 constants of kernels_tiled.cuh.
template <int TX_, int TY_>
struct TileShape {
    static constexpr int TX = TX_, TY = TY_, TT = TX_ * TY_;
    static constexpr int RX = TX_ + 2 + 2 * RM, RY = TY_ + 2 + 2 * RM, RN = RX * RY;
};
using Shape32x8 = TileShape<32, 8>;
using Shape16x16 = TileShape<16, 16>;
using Shape16x8 = TileShape<16, 8>;
enum { SHAPE_32X8 = 0, SHAPE_16X16 = 1, SHAPE_16X8 = 2, N_SHAPES = 3 };
#define ICY_TILE_SHAPE(S)                                                                                  \
    [[maybe_unused]] constexpr int TX = S::TX, TY = S::TY, TT = S::TT, RX = S::RX, RY = S::RY, RN = S::RN

// Runs f(S{}) with S the tile shape numbered `shape` (host code).
template <class F>
inline void with_shape(int shape, F &&f)
{
    switch (shape) {
    case SHAPE_16X16: f(Shape16x16{}); break;
    case SHAPE_16X8: f(Shape16x8{}); break;
    default: f(Shape32x8{}); break;
    }
}

constexpr int SB = 32;                   // points per block of the state
constexpr int HOT_WORDS = 9 * SB;        // words of a block's hot part
constexpr int COLD_WORDS = 8 * SB;       // words of a block's cold part
constexpr int S_NLINES = 17;             // words per point, hot + cold
constexpr int S_HOT = 9;                 // the cold part starts at word S_HOT * pitch
// Device error code of a fused launch in which a point left the staged
// margin (ICY_ERR_DRIFT): the margin test of the launch before excludes it.
constexpr int ICY_DRIFT_CODE = 110;

struct GrainConstF { float pmin2, k, msq, pad; };

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

// Failure-surface constants in FP32: [0, GRAIN_TAB) by grain slot as the FP64
// table, then [GRAIN_TAB, GRAIN_TAB + 330) by grain id modulo 330.  The
// reference varies the constants with (grain + 3) % 30 and (grain + 4) % 11
// of the grain id as a short (simulation/kernels.cuh:341,560-576): for a
// non-negative id that is periodic in 330, so one remainder finds the entry;
// a negative id (C remainders are negative) takes the slot table.
constexpr int GRAIN_PERIOD = 330, GRAIN_TAB_F32 = GRAIN_TAB + GRAIN_PERIOD;
static __global__ void k_grain_table_f32(const GrainConst *tab, GrainConstF *out)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= GRAIN_TAB_F32) return;
    const GrainConst c = tab[s < GRAIN_TAB ? s : grain_slot(s - GRAIN_TAB)];
    out[s] = GrainConstF{(float)c.pmin2, (float)c.k, (float)c.msq, 0.f};
}
__device__ __forceinline__ int grain_entry_f32(unsigned util)
{
    const short g = (short)util;
    return g >= 0 ? GRAIN_TAB + (int)((unsigned)g % GRAIN_PERIOD) : grain_slot(g);
}
// Bits 19-29 of a point's utility word in the FP32 state hold its table entry
// (cached at upload, with bit 30 set) where the input word leaves bits 19-31
// clear; the download clears them again.
constexpr unsigned GE_SHIFT = 19, GE_MASK = 0x7ffu, GE_CACHED = 1u << 30;
static_assert(GRAIN_TAB_F32 <= (int)GE_MASK + 1, "table entries fit the cached field");
__device__ __forceinline__ int grain_entry_cached(unsigned util)
{
    return (util & GE_CACHED) ? (int)((util >> GE_SHIFT) & GE_MASK) : grain_entry_f32(util);
}

// base word: 16 bits per axis, each offset by 32768
__host__ __device__ __forceinline__ unsigned split_pack(int bx, int by)
{
    return ((unsigned)(bx + 32768) << 16) | ((unsigned)(by + 32768) & 0xffffu);
}
__host__ __device__ __forceinline__ void split_unpack(unsigned w, int &bx, int &by)
{
    bx = (int)(w >> 16) - 32768;
    by = (int)(w & 0xffffu) - 32768;
}

// Moves (b, g) to the base of the new position after g changed by at most a
// cell or so: the reference's truncating base (int)(b + g + 0.5)
// (simulation/kernels.cuh:90) and g = x/h - b - 1.  Returns false on the
// common path (g still in [-0.5, 0.5): the base is unchanged).
__device__ __forceinline__ bool split_rebase(int &b, float &g)
{
    if (g >= -0.5f && g < 0.5f) return false;
    // floor semantics first (bounded: a step moves a point by at most half a cell)
    for (int k = 0; k < 4 && g >= 0.5f; k++) { b += 1; g -= 1.0f; }
    for (int k = 0; k < 4 && g < -0.5f; k++) { b -= 1; g += 1.0f; }
    // truncation toward zero where x/h - 0.5 = b + (g + 0.5) is negative and not whole
    if (b < 0 && g > -0.5f) { b += 1; g -= 1.0f; }
    return true;
}

// Paired FP32 arithmetic of sm_100 (the FFMA2 / FADD2 / FMUL2 instructions):
// two independent operations in one instruction, each component rounded as
// the scalar __fmaf_rn / __fadd_rn / __fmul_rn.  A pair holds the two
// components of a vector (a velocity, a momentum, a column of De, Bp or the
// affine moment), or one value twice (p_dup: a weight scaling both).
__device__ __forceinline__ float2 p_fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 p_add(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 p_mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 p_dup(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 p_neg(float2 a) { return make_float2(-a.x, -a.y); }

// quadratic B-spline weights of the stencil columns 0, 1, 2 (simulation/kernels.cuh:100-103)
// with fx = 1 + g, for the two offsets of g at once: 0.5 (0.5 - g)^2,
// 0.75 - g^2, 0.5 (0.5 + g)^2 (g = (t, t) gives each weight twice)
__device__ __forceinline__ void weights_g2(float2 g, float2 w[3])
{
    const float2 h = p_dup(0.5f);
    const float2 a0 = p_add(h, p_neg(g)), a2 = p_add(h, g);
    w[0] = p_mul(p_mul(h, a0), a0);
    w[1] = p_fma(p_neg(g), g, p_dup(0.75f));
    w[2] = p_mul(p_mul(h, a2), a2);
}

// dev(Fe Fe^T) and J = det Fe from De = Fe - I, given by its columns
// d0 = (d00, d10), d1 = (d01, d11), without cancellation:
// Fe Fe^T - I = De + De^T + De De^T, J - 1 = tr De + det De.
__device__ __forceinline__ void split_dev(float2 d0, float2 d1, float &jm1, float &d00, float &d01)
{
    const float a00 = d0.x, a10 = d0.y, a01 = d1.x, a11 = d1.y;
    jm1 = (a00 + a11) + (a00 * a11 - a10 * a01);
    const float b00 = 2.f * a00 + a00 * a00 + a01 * a01;
    const float b11 = 2.f * a11 + a10 * a10 + a11 * a11;
    d00 = 0.5f * (b00 - b11);
    d01 = a01 + a10 + a00 * a10 + a01 * a11;
}

struct PointF {
    unsigned util, bw;   // utility (low 32 bits), base word
    int bx, by;
    float gx, gy, Jp, ptr, qtr;
    float2 v;            // (vx, vy)
    float2 d0, d1, b0, b1;   // columns of De = Fe - I and of Bp: (a00, a10), (a01, a11)
    // J and dev(Fe Fe^T) of the current D from ComputePQ, reused by P2G's stress
    // (dev_ok: D unchanged since, i.e. no return mapping)
    float je, dv0, dv1;
    bool dev_ok;
};

// addresses of point i's vectors in the blocked state
__device__ __forceinline__ unsigned *hot_vec(unsigned *st, long i) { return st + (i >> 5) * HOT_WORDS + (i & 31) * 4; }
__device__ __forceinline__ const unsigned *hot_vec(const unsigned *st, long i)
{
    return st + (i >> 5) * HOT_WORDS + (i & 31) * 4;
}
__device__ __forceinline__ long hot_jp(long i) { return (i >> 5) * HOT_WORDS + 256 + (i & 31); }
__device__ __forceinline__ long cold_vec(long pitch, long i) { return S_HOT * pitch + (i >> 5) * COLD_WORDS + (i & 31) * 4; }

// The parameters a batch member's tile kernel reads from the constant bank:
// the grid extent as ints, and the FP64 block (in global memory) for the
// rare paths -- the crushed-point return mapping and liquid points.
struct MemberP {
    int halo, gridx, gridy;
    unsigned blo, bhi;           // the valid stencil bases (-halo, 0) .. (gridx + halo - 3, gridy - 3), packed
    const StepParams *p64;
};
__device__ __forceinline__ const StepParams &rare_params(const StepParams &P) { return P; }
__device__ __forceinline__ const StepParams &rare_params(const MemberP &P) { return *P.p64; }

// The reference's error code of a stencil base outside the grid (0 inside).
// A batch member tests both axes at once on the packed base word bw, against
// two packed bounds (the three separate bounds of base_error cost the batched
// kernel registers and spills: 3 % of a batched step).
__device__ __forceinline__ int split_base_error(const StepParams &P, unsigned, int bx, int by)
{
    return base_error(P, bx, by);
}
__device__ __forceinline__ int split_base_error(const MemberP &P, unsigned bw, int, int)
{
    const unsigned lo = __vcmpgeu2(bw, P.blo), hi = __vcmpgeu2(P.bhi, bw);   // per 16-bit half: 0xffff if in
    if ((lo & hi) == 0xffffffffu) return 0;
    int e = 0;                       // codes in base_error's order: the last that applies
    if (!(lo >> 16)) e = 70;
    if (!(lo & 0xffffu)) e = 71;
    if (!(hi >> 16)) e = 72;
    if (!(hi & 0xffffu)) e = 73;
    return e;
}

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

template <class PT, typename VSrc>
__device__ __forceinline__ bool g2p_update_f32(const PT &P, const SplitConsts &Q, const GrainConstF *tab,
                                               PointF &s, int *status, VSrc &&vsrc)
{
    const int e = split_base_error(P, s.bw, s.bx, s.by);
    if (e) { *status = e; return false; }
    // the weights of each axis, each held twice: it scales both velocity components
    float2 wx[3], wy[3];
    weights_g2(p_dup(s.gx), wx);
    weights_g2(p_dup(s.gy), wy);
    // v = sum W v_i and Bp = 4/h sum W v_i (i - f)^T (kernels.cuh:357-372),
    // separably: sums over b with wy per column a, then over a with wx;
    // sum W v_i (i - f) = sum W v_i (i - 1) - g v; (vx, vy) paired throughout
    float2 nv[9];
    vsrc(s.bx, s.by, nv);
    float2 cv[3], cb[3];
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float2 n0 = nv[a * 3], n1 = nv[a * 3 + 1], n2 = nv[a * 3 + 2];
        cv[a] = p_fma(wy[2], n2, p_fma(wy[1], n1, p_mul(wy[0], n0)));
        cb[a] = p_fma(wy[2], n2, p_neg(p_mul(wy[0], n0)));
    }
    const float2 v = p_fma(wx[2], cv[2], p_fma(wx[1], cv[1], p_mul(wx[0], cv[0])));
    const float2 sa = p_fma(wx[2], cv[2], p_neg(p_mul(wx[0], cv[0])));
    const float2 sb = p_fma(wx[2], cb[2], p_fma(wx[1], cb[1], p_mul(wx[0], cb[0])));
    // the columns of Bp: (B00, B10) = 4/h (sa - gx v), (B01, B11) = 4/h (sb - gy v)
    const float2 s4 = p_dup(Q.s4);
    const float2 b0 = p_mul(s4, p_fma(p_dup(-s.gx), v, sa));
    const float2 b1 = p_mul(s4, p_fma(p_dup(-s.gy), v, sb));
    // advection in cell units, x += v dt (kernels.cuh:375)
    s.gx += v.x * Q.dt_hinv;
    s.gy += v.y * Q.dt_hinv;
    const bool mx = split_rebase(s.bx, s.gx);
    const bool my = split_rebase(s.by, s.gy);
    if (mx || my) s.bw = split_pack(s.bx, s.by);
    // Fe <- (I + dt Bp) Fe  as  De <- De + T + T De,  T = dt Bp (kernels.cuh:376),
    // by columns: column j of T De is T(:,0) De(0,j) + T(:,1) De(1,j)
    const float2 dtp = p_dup(Q.dt);
    const float2 t0 = p_mul(dtp, b0), t1 = p_mul(dtp, b1);
    const float2 d0 = s.d0, d1 = s.d1;
    s.d0 = p_add(p_add(d0, t0), p_fma(t1, p_dup(d0.y), p_mul(t0, p_dup(d0.x))));
    s.d1 = p_add(p_add(d1, t1), p_fma(t1, p_dup(d1.y), p_mul(t0, p_dup(d1.x))));
    s.ptr = 0.f;
    s.qtr = 0.f;
    s.dev_ok = false;
    if (s.util & (unsigned)kLiquid) {
        s.Jp *= (1.f + t0.x) * (1.f + t1.y) - t0.y * t1.x;   // kernels.cuh:380
    } else {
        // ComputePQ (kernels.cuh:547-557) from De
        float jm1, d00, d01;
        split_dev(s.d0, s.d1, jm1, d00, d01);
        const float Je = 1.f + jm1;
        s.ptr = -(Q.kappa * 0.5f) * (jm1 * (Je + 1.f));
        s.je = Je;
        s.dv0 = d00;
        s.dv1 = d01;
        s.dev_ok = true;
        // sqrt(2) mu/J |dev|, |dev| = sqrt(2(d00^2+d01^2)); the square root to FP32
        // accuracy by the hardware approximation (relative error 2^-23)
        float sq;
        asm("sqrt.approx.f32 %0, %1;" : "=f"(sq) : "f"(d00 * d00 + d01 * d01));
        s.qtr = __fdividef(2.f * Q.mu, Je) * sq;   // sqrt(2) mu/J |dev|, |dev| = sqrt(2(d00^2+d01^2))
        if (!(s.util & (unsigned)kCrushed)) {
            const float4 gc = __ldg(reinterpret_cast<const float4 *>(tab) + grain_entry_cached(s.util));
            const float pmin2 = gc.x, k = gc.y, msq = gc.z;
            bool crushed;
            if (s.ptr < 0.f) crushed = s.ptr < pmin2 || s.qtr > k * (s.ptr - pmin2);
            else crushed = (1.f + 2.f * Q.beta) * s.qtr * s.qtr + msq * (s.ptr + Q.beta * Q.pmax) * (s.ptr - Q.pmax) > 0.f;
            if (crushed) s.util |= (unsigned)kCrushed;
        }
        if (s.util & (unsigned)kCrushed) {
            const SplitRm r = return_map_split(rare_params(P), s.d0.x, s.d1.x, s.d0.y, s.d1.y, s.Jp);
            s.d0 = make_float2(r.d00, r.d10);
            s.d1 = make_float2(r.d01, r.d11);
            s.Jp = r.jp;
            s.dev_ok = false;
        }
    }
    s.v = v;
    s.b0 = b0;
    s.b1 = b1;
    return true;
}

__device__ __forceinline__ void store_point_f32(unsigned *__restrict__ st, long pitch, long i, const PointF &s,
                                                bool write_vb, bool record_pq)
{
    unsigned *v = hot_vec(st, i);
    *reinterpret_cast<uint4 *>(v) = make_uint4(s.bw, __float_as_uint(s.gx), __float_as_uint(s.gy), s.util);
    *reinterpret_cast<float4 *>(v + 128) = make_float4(s.d0.x, s.d0.y, s.d1.x, s.d1.y);
    reinterpret_cast<float *>(st)[hot_jp(i)] = s.Jp;
    if (write_vb || record_pq) {
        float *c = reinterpret_cast<float *>(st) + cold_vec(pitch, i);
        if (write_vb) {
            *reinterpret_cast<float2 *>(c) = s.v;
            *reinterpret_cast<float4 *>(c + 128) = make_float4(s.b0.x, s.b0.y, s.b1.x, s.b1.y);
        }
        if (record_pq) *reinterpret_cast<float2 *>(c + 2) = make_float2(s.ptr, s.qtr);
    }
}

// Loads point i's step state; returns false for a disabled point.
__device__ __forceinline__ bool load_point_f32(const unsigned *__restrict__ st, long i, PointF &s)
{
    const unsigned *v = hot_vec(st, i);
    const uint4 a = *reinterpret_cast<const uint4 *>(v);
    const float4 d = *reinterpret_cast<const float4 *>(v + 128);
    s.Jp = reinterpret_cast<const float *>(st)[hot_jp(i)];
    s.bw = a.x;
    s.gx = __uint_as_float(a.y);
    s.gy = __uint_as_float(a.z);
    s.util = a.w;
    s.d0 = make_float2(d.x, d.y);
    s.d1 = make_float2(d.z, d.w);
    s.dev_ok = false;
    split_unpack(s.bw, s.bx, s.by);
    return !(s.util & (unsigned)kDisabled);
}

// ---------------------------------------------------------------- P2G (FP32)
// Moments of a point as three vectors in shared memory, one padding column
// after every 4 points (the cell phase reads points about 4 apart per lane):
//   m0 = (gx, gy, cx, cy),  m1 = (S00, S10, S01, S11) h,  m2 = (mass, base word)
// with S = m Bp - dt vol Dp_inv tau (simulation/kernels.cuh:57-92) and
// c = m v - S h g, the node-independent part of the affine momentum
// m v + S d (d = ((a - 1 - gx) h, (b - 1 - gy) h)), formed here in paired
// arithmetic so that the cell phase starts from it.
constexpr int CAPF = 1280;                // points per chunk of the FP32 tile kernel
constexpr int MOMF_N = CAPF + CAPF / 4;
constexpr size_t MOMF_BYTES = (2 * sizeof(float4) + sizeof(float2)) * MOMF_N;
__device__ __forceinline__ int momf_col(int j) { return j + (j >> 2); }
struct MomF {
    float4 *m0, *m1;
    float2 *m2;
    __device__ __forceinline__ explicit MomF(float *base)
        : m0(reinterpret_cast<float4 *>(base)), m1(reinterpret_cast<float4 *>(base) + MOMF_N),
          m2(reinterpret_cast<float2 *>(reinterpret_cast<float4 *>(base) + 2 * MOMF_N)) {}
    __device__ __forceinline__ void none(int j) const { m2[momf_col(j)] = make_float2(0.f, __int_as_float(BASE_NONE)); }
};

// REUSE: take J and the deviator from ComputePQ when D is unchanged (the
// batched kernel: 1.8 % faster; alone, where keeping them live costs
// spills, 2.6 % slower, so the single-instance kernel forms them again)
template <bool REUSE, class PT>
__device__ __forceinline__ void p2g_moments_f32(const PT &P, const SplitConsts &Q, const PointF &s,
                                                float *mom, int j, int *status)
{
    const MomF M(mom);
    const bool liquid = (s.util & (unsigned)kLiquid) != 0;
    const float mass = liquid ? Q.mass_water : Q.mass_ice;
    const int e = split_base_error(P, s.bw, s.bx, s.by);
    if (e) {
        *status = e;
        M.none(j);
        return;
    }
    float2 tau0, tau1;   // columns of tau
    if (liquid) {
        const float sw = (float)(rare_params(P).kappa * (1. - pow((double)s.Jp, -5.0)));   // Water (kernels.cuh:37-44)
        tau0 = make_float2(sw, 0.f);
        tau1 = make_float2(0.f, sw);
    } else {
        // KirchhoffStress_Wolper (kernels.cuh:24-34) from De: mu/J dev(Fe Fe^T) +
        // kappa/2 (J^2 - 1) I, the second term -p of ComputePQ; J and the
        // deviator as ComputePQ formed them when D is unchanged since
        float Je, d00, d01, s2;
        if (REUSE && s.dev_ok) {
            Je = s.je;
            d00 = s.dv0;
            d01 = s.dv1;
            s2 = -s.ptr;
        } else {
            float jm1;
            split_dev(s.d0, s.d1, jm1, d00, d01);
            Je = 1.f + jm1;
            s2 = (Q.kappa * 0.5f) * (jm1 * (Je + 1.f));
        }
        const float s1 = __fdividef(Q.mu, Je);
        tau0 = make_float2(s1 * d00 + s2, s1 * d01);
        tau1 = make_float2(s1 * d01, -s1 * d00 + s2);
    }
    const int c = momf_col(j);
    const float2 mh = p_dup(mass * Q.h), ndth = p_dup(-Q.dtvd * Q.h);
    const float2 S0 = p_fma(mh, s.b0, p_mul(ndth, tau0)), S1 = p_fma(mh, s.b1, p_mul(ndth, tau1));   // S h
    const float2 cc = p_add(p_mul(p_dup(mass), s.v), p_neg(p_fma(S1, p_dup(s.gy), p_mul(S0, p_dup(s.gx)))));
    M.m0[c] = make_float4(s.gx, s.gy, cc.x, cc.y);
    M.m1[c] = make_float4(S0.x, S0.y, S1.x, S1.y);
    M.m2[c] = make_float2(mass, __uint_as_float(s.bw));
}

// (m, px, py) += (dm, dpx, dpy) on a float4 node with one vector reduction
// (red: no value comes back, unlike atomicAdd on a float4, which returns the
// old value and costs registers and latency); each component is added
// atomically on its own, as with atomicAdd.
__device__ __forceinline__ void red_add_f4(float4 *p, float dm, float dpx, float dpy)
{
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p), "f"(dm), "f"(dpx), "f"(dpy), "f"(0.f));
}

// FP32 grid of n nodes in one allocation of 6 n floats, in one of two layouts.
// Alone: five arrays m, px, py, vx, vy (scalar atomics; the bases are
// constant-bank operands).  In a batch (AOS): per node (m, px, py, -) as a
// float4 taken by one vector atomic, then a float2 velocity array: two bases
// to look up per member and fewer live addresses (the batched kernel spills
// less and runs 10 % faster; alone the scalar layout is 2.5 % faster).
struct GridViewF {
    float *m, *px, *py, *vx, *vy;   // alone: accumulators, velocities G2P reads
    float *nvx;                     // alone: velocities the grid update writes, the next step's vx
                                    // (its vy follows n_nodes floats later)
    float4 *mp;                     // in a batch (same memory)
    float2 *v;
    int ny, halo;
    // node (m, px, py) += (dm, dpx, dpy)
    template <bool AOS>
    __device__ __forceinline__ void add(long k, float dm, float dpx, float dpy) const
    {
        if constexpr (AOS) {
            red_add_f4(mp + k, dm, dpx, dpy);
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
    unsigned *st;       // blocked state: hot part, then the cold part from word S_HOT * pitch
    long pitch;
    const int *cell_start, *active, *n_active;
    unsigned *flags;
    int2 *tlist;        // node tiles written since the last update, each once: (inst, tile)
    unsigned *tlist_n;  // [0] entries, [1] CTAs of the update done
    int inst;           // this instance's slot in a batch (0 alone)
    int seq;            // fused grid update: this launch's number since the last binning (>= 1); 0 = none
    int *status;
    unsigned long long *moved;   // [0] points off their sorted cell (counted per P2G), [1] fused launches,
                                 // [2] launches that fell back to the update kernel (single instance)
    int *claim;         // batch: [0] next work item to hand out, [1] CTAs finished (zero between launches)
    const GrainConstF *grain_tab;   // GRAIN_TAB_F32 entries
    int record_pq;
    float safe_m;       // fused grid update: a point at offset u (cells) from its sorted cell stays
                        // in the staged margin during one step if -safe_m <= u < safe_m
    double *acc;        // indenter force bins
    long n_nodes;       // nodes of the grid
    // grid update fused into the tile kernel (single instance): each node tile
    // is updated by the CTA that brings its count of finished neighbouring
    // cell tiles to the expected number; see k_tile_f32
    const int *nexp;    // per node tile: active cell tiles in its 3 x 3 neighbourhood
    int *ncnt;          // per node tile: neighbouring cell tiles finished in this launch
    int *unsafe;        // [2]: by launch parity, the last launch that found a point able to leave
                        // the staged margin during the next step
    double ind_x, ind_y;   // indenter position of the fused update
};

// A batch member's FP32 grid as the batched tile kernel sees it: (m, px, py, -)
// float4 accumulators and float2 velocities (GridViewF's batch layout).
struct GridViewB {
    float4 *mp;
    float2 *v;
    int ny, halo;
    template <bool AOS>
    __device__ __forceinline__ void add(long k, float dm, float dpx, float dpy) const
    {
        static_assert(AOS, "batch layout");
        red_add_f4(mp + k, dm, dpx, dpy);
    }
    template <bool AOS>
    __device__ __forceinline__ float2 vel(long k) const
    {
        static_assert(AOS, "batch layout");
        return v[k];
    }
    __device__ __forceinline__ long idx(int gx, int gy) const { return (long)(gx + halo) * ny + gy; }
};

// The member arguments the batched tile kernel reads per work item, 208 of
// SplitArgs' bytes: the FP64 parameters stay in the global table (p64), read
// only by the rare paths.  300 members fit the 64 KB constant bank.
struct SplitMember {
    MemberP P;
    SplitConsts Q;
    TileGeom G;
    GridViewB g;
    unsigned *st;
    long pitch;
    const int *cell_start;
    const GrainConstF *grain_tab;
    int *status;
    unsigned *flags;
    int2 *tlist;
    unsigned *tlist_n;
    unsigned long long *moved;
    int inst;
};
constexpr int BATCH_CONST_SLOTS = 300;
static_assert(sizeof(SplitMember) * BATCH_CONST_SLOTS <= 64000, "the members' arguments fit the constant bank");

// member i of a batch whose argument table is `d_args` on the device
inline SplitMember split_member(const SplitArgs &a, const SplitArgs *d_args_i)
{
    SplitMember m{};
    m.P = MemberP{a.P.halo, a.P.gridx, a.P.gridy, split_pack(-a.P.halo, 0),
                  split_pack(a.P.gridx + a.P.halo - 3, a.P.gridy - 3), &d_args_i->P};
    m.Q = a.Q;
    m.G = a.G;
    m.g = GridViewB{a.g.mp, a.g.v, a.g.ny, a.g.halo};
    m.st = a.st;
    m.pitch = a.pitch;
    m.cell_start = a.cell_start;
    m.grain_tab = a.grain_tab;
    m.status = a.status;
    m.flags = a.flags;
    m.tlist = a.tlist;
    m.tlist_n = a.tlist_n;
    m.moved = a.moved;
    m.inst = a.inst;
    return m;
}

// Where the batched tile kernel finds its members' arguments: the global
// table, or (batch_cargs.cu, batches of at most BATCH_CONST_SLOTS slots) a
// compact copy in the constant bank, read as the single-instance kernel
// reads its own (no global loads and fewer spills in the point loop).
struct GlobalMembers {
    const SplitArgs *a;
    __device__ __forceinline__ const SplitArgs &operator[](int i) const { return a[i]; }
};
#ifdef ICY_BATCH_CONST_ARGS
static __constant__ SplitMember c_batch_mem[BATCH_CONST_SLOTS];
struct ConstMembers {
    __device__ __forceinline__ const SplitMember &operator[](int i) const { return c_batch_mem[i]; }
};
using BatchMembers = ConstMembers;
#else
using BatchMembers = GlobalMembers;
#endif

// The arguments of member `inst` (a batch), or the launch's own (alone).
template <bool BATCH, class TAB>
__device__ __forceinline__ decltype(auto) member_at(const SplitArgs &A1, const TAB &tab, int inst)
{
    if constexpr (BATCH) return tab[inst];
    else return (A1);
}

// P2G contributions of one point to its 3 x 3 nodes (simulation/kernels.cuh:
// 100-120): node (a, b) gets W m and W (m v + S d) with W = wx[a] wy[b] and
// d = ((a - fx) h, (b - fy) h) = ((a - 1 - gx) h, (b - 1 - gy) h).  m v + S d is
// affine in (a, b), so it is evaluated as c + (a - 1) S(:,0) h + (b - 1) S(:,1) h
// from c = m v - S h g and the columns S0h, S1h of S h (the point's moments):
// per node one product for W and one addition per component.  In scalar
// arithmetic: the paired form of this loop (W twice, (tx, ty) and the
// momentum sums as pairs) needs aligned register pairs for the 9 momentum
// sums of the cell phase, and at 80 registers the tile kernel then spills
// four times as much.
__device__ __forceinline__ void weights_g(float g, float w[3])
{
    const float a0 = 0.5f - g, a2 = 0.5f + g;
    w[0] = (0.5f * a0) * a0;
    w[1] = 0.75f - g * g;
    w[2] = (0.5f * a2) * a2;
}
template <typename Sink>
__device__ __forceinline__ void point_contributions_f32(float gx, float gy, float mass, float2 c, float2 S0h,
                                                        float2 S1h, Sink &&sink)
{
    float wx[3], wy[3];
    weights_g(gx, wx);
    weights_g(gy, wy);
    const float s00h = S0h.x, s01h = S1h.x, s10h = S0h.y, s11h = S1h.y;
    const float cx = c.x, cy = c.y;
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float ax = a == 0 ? cx - s00h : a == 1 ? cx : cx + s00h;
        const float ay = a == 0 ? cy - s10h : a == 1 ? cy : cy + s10h;
#pragma unroll
        for (int b = 0; b < 3; b++) {
            const float W = wx[a] * wy[b];
            const float tx = b == 0 ? ax - s01h : b == 1 ? ax : ax + s01h;
            const float ty = b == 0 ? ay - s11h : b == 1 ? ay : ay + s11h;
            sink(a, b, W, W * mass, tx, ty);
        }
    }
}

template <bool AOS, class S, class GV>
static __device__ __noinline__ void p2g_global_f32(GV g, unsigned *flags, int2 *tlist, unsigned *tlist_n,
                                                   int inst, int ntx, int halo, int bx, int by, float gx,
                                                   float gy, float mass, float2 c, float2 S0h, float2 S1h)
{
    ICY_TILE_SHAPE(S);
    point_contributions_f32(gx, gy, mass, c, S0h, S1h, [&](int a, int b, float W, float dm, float tx, float ty) {
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

// Cells of a tile in the order the cell phase takes them: by point count,
// largest first, so that the 32 cells of a warp hold about the same number of
// points (the warp's loop runs as long as its fullest cell; in input order a
// warp's fullest cell holds about twice the mean).  rank[c] = (count bucket
// << 16) | rank of cell c within its bucket, from shared atomics on hist; the
// first warp then turns the buckets into perm (position -> cell).  Any order
// gives the same sums: each cell's partials have a fixed place.
constexpr int CNT_BUCKETS = 16;
// every thread of the tile (tid < TT): its cell's count
template <int NC>
__device__ __forceinline__ void cell_order_count(int (&hist)[CNT_BUCKETS], int (&rank)[NC], int tid, int cnt)
{
    const int b = CNT_BUCKETS - 1 - min(cnt, CNT_BUCKETS - 1);   // largest first
    rank[tid] = (b << 16) | atomicAdd(hist + b, 1);
}
// the first warp, after a barrier that follows every count
template <int NC>
__device__ __forceinline__ void cell_order_build(int (&hist)[CNT_BUCKETS], const int (&rank)[NC], int (&perm)[NC],
                                                 int lane)
{
    const int h = lane < CNT_BUCKETS ? hist[lane] : 0;
    int x = h;
#pragma unroll
    for (int o = 1; o < CNT_BUCKETS; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    const int off = x - h;   // exclusive prefix of the bucket
    __syncwarp();
    if (lane < CNT_BUCKETS) hist[lane] = 0;   // ready for the next tile
#pragma unroll
    for (int c = lane; c < NC; c += 32) {
        const int r = rank[c];
        perm[__shfl_sync(0xffffffffu, off, r >> 16) + (r & 0xffff)] = c;
    }
}

// phases 2 and 3 (see p2g_cells_and_flush in kernels_tiled.cuh), in FP32
// `nxt`: the next work item's prologue, overlapped with this tile's node
// phase (nxt.load() issues its global loads before the node loop, nxt.store()
// puts the values into shared memory after it).  `s_oddf`: set when a point
// of the chunk added to the drift buffer s_odd (a point off its binned cell:
// 0.01-0.07 % of the points per step on the 9.6 M-point indentation case, in
// about one tile in eight); without one the node phase walks only the
// (TX + 2) x (TY + 2) nodes that cell sums reach and leaves s_odd alone.
template <int NT, bool AOS, bool FUSE, class S, class AT, typename Sync, class Next>
__device__ __forceinline__ void p2g_cells_and_flush_f32(const AT &A, int tid, int tx, int ty, int cs, int ce,
                                                        const int *s_cs, const int *s_perm, float *mom,
                                                        float (*s_odd)[S::RN], int *s_oddf, unsigned &touch,
                                                        unsigned &moved, bool fused, Sync &&sync, Next &&nxt)
{
    ICY_TILE_SHAPE(S);
    const auto &P = A.P;
    const int X0 = tx * TX - P.halo, Y0 = ty * TY;
    const int RX0 = X0 - RM, RY0 = Y0 - RM;
    float accm[9];     // per node of the stencil: mass and momentum
    float2 accp[9];
#pragma unroll
    for (int q = 0; q < 9; q++) {
        accm[q] = 0.f;
        accp[q] = make_float2(0.f, 0.f);
    }
    if (tid < TT) {
        const int cell = s_perm[tid];
        const unsigned pbc = split_pack(X0 + cell / TY, Y0 + cell % TY);
        const int r0 = max(s_cs[cell], cs) - cs, r1 = min(s_cs[cell + 1], ce) - cs;
        const MomF M(mom);
        for (int j = r0; j < r1; j++) {
            const int c = momf_col(j);
            const float2 q2 = M.m2[c];
            const unsigned pb = __float_as_uint(q2.y);
            if (pb == (unsigned)BASE_NONE) continue;
            const float4 q0 = M.m0[c], q1 = M.m1[c];
            const float gx = q0.x, gy = q0.y, mass = q2.x;
            const float2 c0 = make_float2(q0.z, q0.w), S0h = make_float2(q1.x, q1.y), S1h = make_float2(q1.z, q1.w);
            if (pb == pbc) {
                point_contributions_f32(gx, gy, mass, c0, S0h, S1h,
                                        [&](int a, int b, float W, float dm, float tx, float ty) {
                                            const int q = a * 3 + b;
                                            accm[q] += dm;
                                            accp[q].x += W * tx;
                                            accp[q].y += W * ty;
                                        });
            } else {
                moved++;
                int bx, by;
                split_unpack(pb, bx, by);
                if constexpr (FUSE) {
                    // can this point leave the staged margin during the next step?  (its
                    // offset from its sorted cell, in cells, against the largest move of a
                    // step; near the low edges, where the base truncates, always)
                    if (A.seq > 0) {
                        int sx, sy;
                        split_unpack(pbc, sx, sy);
                        const float ux = (float)(bx - sx) + gx, uy = (float)(by - sy) + gy;
                        if (!(ux >= -A.safe_m && ux < A.safe_m && uy >= -A.safe_m && uy < A.safe_m) || bx <= 0 ||
                            by <= 0)
                            A.unsafe[A.seq & 1] = A.seq;
                    }
                }
                const int lx = bx - RX0, ly = by - RY0;
                if (lx >= 0 && lx + 2 < RX && ly >= 0 && ly + 2 < RY) {
                    *s_oddf = 1;
                    point_contributions_f32(gx, gy, mass, c0, S0h, S1h,
                                            [&](int a, int b, float W, float dm, float tx, float ty) {
                                                const int k = (lx + a) * RY + (ly + b);
                                                atomicAdd(&s_odd[0][k], dm);
                                                atomicAdd(&s_odd[1][k], W * tx);
                                                atomicAdd(&s_odd[2][k], W * ty);
                                            });
                } else {
                    if (FUSE && fused) *A.status = ICY_DRIFT_CODE;   // excluded by the margin test of the last launch
                    p2g_global_f32<AOS, S>(A.g, A.flags, A.tlist, A.tlist_n, A.inst, A.G.ntx, P.halo, bx, by, gx,
                                           gy, mass, c0, S0h, S1h);
                }
            }
        }
    }
    sync();
    // [9 node offsets][TT cells] of (px, py, m, -), aliasing the moments
    float4 *part = reinterpret_cast<float4 *>(mom);
    if (tid < TT) {
        const int cell = s_perm[tid];
#pragma unroll
        for (int q = 0; q < 9; q++) part[q * TT + cell] = make_float4(accp[q].x, accp[q].y, accm[q], 0.f);
    }
    sync();
    nxt.load();
    const bool odd = *s_oddf != 0;
    // without drifted points in the staged region, only the core nodes (the
    // tile's bases + 2) have sums, and the drift buffer is all zero
    constexpr int CX = TX + 2, CY = TY + 2;
    const int kn = odd ? RN : CX * CY;
    for (int k = tid; k < kn; k += NT) {
        int i, jj;
        if (odd) {
            i = k / RY;
            jj = k % RY;
        } else {
            i = RM + k / CY;
            jj = RM + k % CY;
        }
        const int kk = i * RY + jj;
        const int nx = i - RM, ny = jj - RM;
        float m = 0.f;
        float2 pp = make_float2(0.f, 0.f);
#pragma unroll
        for (int a = 0; a < 3; a++) {
            const int cx = nx - a;
            if (cx < 0 || cx >= TX) continue;
#pragma unroll
            for (int b = 0; b < 3; b++) {
                const int cy = ny - b;
                if (cy < 0 || cy >= TY) continue;
                const float4 v = part[(a * 3 + b) * TT + cx * TY + cy];
                pp = p_add(pp, make_float2(v.x, v.y));
                m += v.z;
            }
        }
        float px = pp.x, py = pp.y;
        if (odd) {
            m += s_odd[0][kk]; px += s_odd[1][kk]; py += s_odd[2][kk];
            s_odd[0][kk] = 0.f; s_odd[1][kk] = 0.f; s_odd[2][kk] = 0.f;
        }
        if (m != 0.f || px != 0.f || py != 0.f) {
            const int gx = RX0 + i, gy = RY0 + jj;
            A.g.add<AOS>(A.g.idx(gx, gy), m, px, py);
            if (!FUSE || !fused) {
                const int dx = (gx + P.halo) / TX - tx + 1, dy = gy / TY - ty + 1;
                touch |= 1u << (dy * 3 + dx);
            }
        }
    }
    nxt.store();
    sync();
    if (tid == 0) *s_oddf = 0;   // the next chunk's cell phase sets it after a barrier
}

// Grid update of one node in FP32 (simulation/kernels.cuh:175-300) from its
// mass and momentum, the indenter geometry and the force in FP64: the new
// velocity, and the force bin of a contact node (-1 if none).
// (P: h, dt, ind_rsq, ind_v, nsub, gridx, gridy as in StepParams; Q: h, dtg,
// vmax, vmax_sq as in SplitConsts)
template <class PT, class QT>
__device__ __forceinline__ int node_velocity_f32(const PT &P, const QT &Q, int gx, int gy, float mass,
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
        // indenter contact (kernels.cuh:264-287) decided in FP64, as the reference
        // does; an FP32 test with a 1 mm margin (FP32 errors here are ~1e-5 m)
        // first lets the nodes far from the indenter skip the FP64 arithmetic
        const float ex = (float)gx * Q.h - (float)ind_x, ey = (float)gy * Q.h - (float)ind_y;
        const float rr = sqrtf((float)P.ind_rsq) + 1e-3f;
        double nx = 0.0, ny = 0.0;
        if (ex * ex + ey * ey < rr * rr && ((nx = (double)gx * P.h - ind_x), (ny = (double)gy * P.h - ind_y),
                                            nx * nx + ny * ny < P.ind_rsq)) {
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

// Grid update of node tile (ntx_, nty_) by one CTA of TT threads, one node
// each (the fused update of k_tile_f32): reads the finished sums (through L2:
// other CTAs added them), writes the next velocities, clears the sums and
// adds the indenter force of contact nodes to the bins.
template <class S>
__device__ __forceinline__ void update_node_tile_f32(const SplitArgs &A, int ntx_, int nty_, int l, double ind_x,
                                                     double ind_y)
{
    ICY_TILE_SHAPE(S);
    const StepParams &P = A.P;
    if (l >= TT) return;
    const int gx = ntx_ * TX + l / TY - P.halo, gy = nty_ * TY + l % TY;
    if (gx >= P.gridx + P.halo || gy >= P.gridy) return;   // past the grid edge
    const long k = A.g.idx(gx, gy);
    const float m = __ldcg(A.g.m + k), px = __ldcg(A.g.px + k), py = __ldcg(A.g.py + k);
    float vx, vy;
    double fx = 0, fy = 0;
    const int bin = node_velocity_f32(P, A.Q, gx, gy, m, px, py, ind_x, ind_y, vx, vy, fx, fy);
    A.g.nvx[k] = vx;
    A.g.nvx[k + A.n_nodes] = vy;
    if (m != 0.f || px != 0.f || py != 0.f) {
        A.g.m[k] = 0.f;
        A.g.px[k] = 0.f;
        A.g.py[k] = 0.f;
    }
    if (bin >= 0) {
        atomicAdd(A.acc + 2 * bin, fx);
        atomicAdd(A.acc + 2 * bin + 1, fy);
    }
}

// Threads and resident CTAs per SM of the FP32 tile kernel.
constexpr int TILE_THREADS_F32 = 256, TILE_CTAS_F32 = 3;

// The next work item's prologue run inside a tile's node phase (see
// p2g_cells_and_flush_f32), or nothing.
struct NoNext {
    __device__ __forceinline__ void load() const {}
    __device__ __forceinline__ void store() const {}
};
template <class L, class St>
struct NextOps {
    L l;
    St st;
    __device__ __forceinline__ void load() const { l(); }
    __device__ __forceinline__ void store() const { st(); }
};

// Work items of a batch: (instance, tile) pairs over all instances.
struct BatchItem { int inst, tile; };

// Starts moving the next work item's hot state (pieces which < 8 of its
// contiguous block range) or cell ranges (which == 8) into L2 while this CTA
// is in its cell phase.
constexpr int PF_PIECES = 8;
template <bool BATCH, class S, class TAB>
__device__ __forceinline__ void prefetch_next_item(const SplitArgs &A1, const TAB &tab, const BatchItem *work,
                                                   int next, int na, int which)
{
    ICY_TILE_SHAPE(S);
    if (next >= na) return;
    const BatchItem w = BATCH ? work[next] : BatchItem{0, A1.active[next]};
    const auto &A = member_at<BATCH>(A1, tab, w.inst);
    const int *cs = A.cell_start + (long)w.tile * TT;
    if (which == PF_PIECES) {
        prefetch_l2(cs, (TT + 1) * sizeof(int));
        return;
    }
    const int ps = cs[0], pe = cs[TT];
    if (pe <= ps) return;
    const int b0 = ps >> 5, nb = ((pe - 1) >> 5) + 1 - b0;
    const int k0 = b0 + nb * which / PF_PIECES, k1 = b0 + nb * (which + 1) / PF_PIECES;
    if (k1 > k0) prefetch_l2(A.st + (long)k0 * HOT_WORDS, (size_t)(k1 - k0) * HOT_WORDS * sizeof(unsigned));
}

// Tile kernel over the FP32 state: <G2P, P2G, write vel/Bp> as k_tile.
// With BATCH, the CTAs walk the (instance, tile) list of many independent
// instances, each with its own parameters, grid and points (Aarr[inst]), and
// the record-PQ flag of each instance comes from rec[inst].  FUSE (single
// instance, option "fuse_update"): P2G tests the drift margin for the next
// step, and a G2P + P2G launch updates the grid itself where that is safe.
template <bool DO_G2P, bool DO_P2G, bool WRITE_VB, bool BATCH = false, bool FUSE = false, class S = Shape32x8>
static __global__ void __launch_bounds__(TILE_THREADS_F32, TILE_CTAS_F32)
    k_tile_f32(const __grid_constant__ SplitArgs A1, const SplitArgs *__restrict__ Aarr = nullptr, const BatchItem *__restrict__ work = nullptr,
               const int *__restrict__ nwork = nullptr, const int *__restrict__ rec = nullptr)
{
    ICY_TILE_SHAPE(S);
    static_assert(TT <= TILE_THREADS_F32, "at most one cell per thread in the cell phase");
    static_assert(9 * TT * sizeof(float4) <= MOMF_BYTES, "cell partials alias the moment buffer");
    __shared__ float2 s_v[RN];
    __shared__ float s_odd[3][RN];
    __shared__ int s_cs[TT + 1];
    __shared__ int s_hist[CNT_BUCKETS], s_rank[TT], s_perm[TT];
    __shared__ unsigned s_touch;
    __shared__ int s_oddf;
    __shared__ int s_claim;
    extern __shared__ float4 s_momf4[];
    float *const s_momf = reinterpret_cast<float *>(s_momf4);
    const int na = BATCH ? *nwork : *A1.n_active;
    const int tid = threadIdx.x;
    // This launch updates the grid itself (see the end of the tile loop) unless
    // the launch before found a point that could leave its tile's staged margin
    // in this step: its contributions could then reach node tiles beyond the 3 x 3
    // neighbourhood after they were updated, so the tiles are marked for the
    // list-driven update that follows instead.  The flag of launch s is
    // unsafe[s & 1]: this launch reads the other one, which nobody writes now.
    static_assert(!(FUSE && BATCH), "the fused grid update is single-instance only");
    const bool fused = FUSE && DO_G2P && DO_P2G && A1.seq > 0 && A1.unsafe[(A1.seq - 1) & 1] != A1.seq - 1;
    if (FUSE && DO_G2P && DO_P2G && A1.seq > 0 && blockIdx.x == 0 && tid == 0)
        atomicAdd(A1.moved + (fused ? 1 : 2), 1ull);
    // Alone, CTA c takes the tiles c, c + gridDim.x, ... (equal tiles, and no
    // claim to wait for: 5 % faster).  In a batch, where the items differ in
    // size, they are handed out one at a time (A1.claim[0]), each CTA claiming
    // its next item when it starts one, so that the CTAs finish together (4 %).
    if (BATCH && tid == 0) s_claim = atomicAdd(A1.claim, 1);
    for (int k = tid; k < RN; k += blockDim.x) { s_odd[0][k] = 0.f; s_odd[1][k] = 0.f; s_odd[2][k] = 0.f; }
    if (tid < CNT_BUCKETS) s_hist[tid] = 0;
    if (tid == 0) s_oddf = 0;
    __syncthreads();
    int ti = BATCH ? s_claim : (int)blockIdx.x;
    __syncthreads();   // everybody has read s_claim; later reads of it come before the item's last barrier
    // the current item's prologue (cell ranges and order counts, staged node
    // velocities) was done during the previous item's node phase
    bool staged = false;
    while (ti < na) {
        const BatchItem w = BATCH ? work[ti] : BatchItem{0, A1.active[ti]};
        if (BATCH && tid == 0) s_claim = atomicAdd(A1.claim, 1);
#ifdef ICY_BATCH_CONST_ARGS
        const BatchMembers tab{};
#else
        const BatchMembers tab{Aarr};
#endif
        const auto &A = member_at<BATCH>(A1, tab, w.inst);
        const auto &P = A.P;
        const bool record = BATCH ? rec[w.inst] != 0 : A1.record_pq != 0;
        unsigned moved = 0;
        const int t = w.tile;
        const int tx = t % A.G.ntx, ty = t / A.G.ntx;
        const int RX0 = tx * TX - P.halo - RM, RY0 = ty * TY - RM;
        if (!staged) {
            // cell ranges; each thread counts its own cell's points for the cell order
            const int *cst = A.cell_start + (long)t * TT;
            if (tid < TT) {
                const int c0 = cst[tid], c1 = cst[tid + 1];
                s_cs[tid] = c0;
                if (tid == TT - 1) s_cs[TT] = c1;
                if (DO_P2G) cell_order_count(s_hist, s_rank, tid, c1 - c0);
            }
            if (DO_G2P) {
                for (int k = tid; k < RN; k += blockDim.x) {
                    const int gx = RX0 + k / RY, gy = RY0 + k % RY;
                    s_v[k] = node_in_grid(P, gx, gy) ? A.g.vel<BATCH>(A.g.idx(gx, gy)) : make_float2(0.f, 0.f);
                }
            }
        }
        if (tid == 0) s_touch = 0;
        __syncthreads();
        const int next = BATCH ? s_claim : ti + (int)gridDim.x;
        const int ps = s_cs[0], pe = s_cs[TT];
        unsigned touch = 0;
        bool next_staged = false;
        for (int cs = ps; cs < pe; cs += CAPF) {
            const int ce = min(cs + CAPF, pe);
            for (int j = tid; j < ce - cs; j += blockDim.x) {
                const long i = cs + j;
                // a batch member's arguments read from the constant bank again in
                // every iteration (the index is opaque to the compiler) instead of
                // held in registers across the loop: fewer spills (batched step
                // -2.5 %); alone they are constant-bank operands either way
                int inst_o = w.inst;
                if (BATCH) asm volatile("" : "+r"(inst_o));
                const auto &A = member_at<BATCH>(A1, tab, inst_o);
                const auto &P = A.P;
                // the 3 x 3 node velocities of a stencil: from the staged region (one
                // check per point), else from the grid
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
                            for (int b = 0; b < 3; b++)
                                nv[a * 3 + b] = A.g.template vel<BATCH>(A.g.idx(bx + a, by + b));
                    }
                };
                PointF s;
                if (!load_point_f32(A.st, i, s)) {
                    if (DO_P2G) MomF(s_momf).none(j);
                    continue;
                }
                if (DO_G2P) {
                    if (!g2p_update_f32(P, A.Q, A.grain_tab, s, A.status, vsrc)) {
                        if (DO_P2G) MomF(s_momf).none(j);
                        continue;
                    }
                    store_point_f32(A.st, A.pitch, i, s, WRITE_VB, record);
                } else {
                    const float *c = reinterpret_cast<const float *>(A.st) + cold_vec(A.pitch, i);
                    const float4 v = *reinterpret_cast<const float4 *>(c);
                    const float4 b = *reinterpret_cast<const float4 *>(c + 128);
                    s.v = make_float2(v.x, v.y);
                    s.b0 = make_float2(b.x, b.y);
                    s.b1 = make_float2(b.z, b.w);
                }
                if (DO_P2G) p2g_moments_f32<BATCH>(P, A.Q, s, s_momf, j, A.status);
            }
            __syncthreads();
            // the last threads start the next item's loads: its hot state in pieces
            // and its cell ranges
            constexpr int PF0 = TILE_THREADS_F32 - (PF_PIECES + 1);
            if (DO_P2G && cs == ps && tid >= PF0)
                prefetch_next_item<BATCH, S>(A1, tab, work, next, na, tid - PF0);
            // and the first threads its staged node velocities (columns of vx and vy,
            // or of the float2 velocities of a batch member)
            static_assert(2 * RX <= PF0, "velocity-column and state prefetches on different threads");
            if (DO_G2P && DO_P2G && cs == ps && tid < (BATCH ? 1 : 2) * RX && next < na) {
                const BatchItem wn = BATCH ? work[next] : BatchItem{0, A1.active[next]};
                const auto &An = member_at<BATCH>(A1, tab, wn.inst);
                const int nx0 = (wn.tile % An.G.ntx) * TX - An.P.halo - RM, ny0 = (wn.tile / An.G.ntx) * TY - RM;
                if constexpr (BATCH)
                    prefetch_region_column(An.g.v, An.P.gridx, An.P.gridy, An.P.halo, An.g.ny, nx0, ny0, tid, RY);
                else
                    prefetch_region_column(tid < RX ? An.g.vx : An.g.vy, An.P.gridx, An.P.gridy, An.P.halo, An.g.ny,
                                           nx0, ny0, tid % RX, RY);
            }
            if (DO_P2G) {
                if (cs == ps) {
                    // the cell order, by the first warp while the point loop's registers are free
                    if (tid < 32) cell_order_build(s_hist, s_rank, s_perm, tid);
                    __syncthreads();
                }
                auto sync = [] { __syncthreads(); };
                if (ce == pe && next < na) {
                    // the last chunk: the next item's prologue during this node phase
                    // (its global loads into registers before the node loop, into
                    // shared memory after it; the staging pass cost 7 % when alone)
                    constexpr int NV = (RN + TILE_THREADS_F32 - 1) / TILE_THREADS_F32;
                    int nc0 = 0, nc1 = 0;
                    float2 nvel[NV];
                    auto ld = [&] {
                        const BatchItem wn = BATCH ? work[next] : BatchItem{0, A1.active[next]};
                        const auto &An = member_at<BATCH>(A1, tab, wn.inst);
                        const int tn = wn.tile;
                        if (tid < TT) {
                            const int *cst = An.cell_start + (long)tn * TT;
                            nc0 = cst[tid];
                            nc1 = cst[tid + 1];
                        }
                        if (DO_G2P) {
                            const int rx0 = (tn % An.G.ntx) * TX - An.P.halo - RM, ry0 = (tn / An.G.ntx) * TY - RM;
#pragma unroll
                            for (int u = 0; u < NV; u++) {
                                const int k = tid + u * TILE_THREADS_F32;
                                const int gx = rx0 + k / RY, gy = ry0 + k % RY;
                                nvel[u] = k < RN && node_in_grid(An.P, gx, gy)
                                              ? An.g.template vel<BATCH>(An.g.idx(gx, gy))
                                              : make_float2(0.f, 0.f);
                            }
                        }
                    };
                    auto st = [&] {
                        if (tid < TT) {
                            s_cs[tid] = nc0;
                            if (tid == TT - 1) s_cs[TT] = nc1;
                            cell_order_count(s_hist, s_rank, tid, nc1 - nc0);
                        }
                        if (DO_G2P) {
#pragma unroll
                            for (int u = 0; u < NV; u++) {
                                const int k = tid + u * TILE_THREADS_F32;
                                if (k < RN) s_v[k] = nvel[u];
                            }
                        }
                    };
                    p2g_cells_and_flush_f32<TILE_THREADS_F32, BATCH, FUSE, S>(
                        A, tid, tx, ty, cs, ce, s_cs, s_perm, s_momf, s_odd, &s_oddf, touch, moved, fused, sync,
                        NextOps<decltype(ld), decltype(st)>{ld, st});
                    next_staged = true;
                } else {
                    p2g_cells_and_flush_f32<TILE_THREADS_F32, BATCH, FUSE, S>(
                        A, tid, tx, ty, cs, ce, s_cs, s_perm, s_momf, s_odd, &s_oddf, touch, moved, fused, sync, NoNext{});
                }
            }
        }
        bool tail_done = false;
        if constexpr (FUSE) {
            if (DO_P2G && fused) {
                tail_done = true;
                // Fused grid update: this tile's sums are in; count it finished for each
                // of the 9 node tiles around it.  The CTA that brings a node tile's count
                // to the number of active cell tiles around it (nexp, from the binning)
                // updates that node tile: all its contributions have landed, since in a
                // fused launch every contribution to a node tile comes from the cell tiles
                // around it.  Release: the CTA's reductions, barrier, then a fence and the
                // count by the counting threads (the barrier orders the other threads'
                // reductions before the fence, which is cumulative); acquire: count,
                // fence, barrier, reads through L2 -- the pattern of a grid-wide barrier.
                __syncthreads();
                if (tid < 9) {
                    const int nx = tx + tid % 3 - 1, ny = ty + tid / 3 - 1;
                    bool ready = false;
                    if (nx >= 0 && nx < A.G.ntx && ny >= 0 && ny < A.G.nty) {
                        const int X = ny * A.G.ntx + nx;
                        __threadfence();
                        ready = atomicAdd(A.ncnt + X, 1) == A.nexp[X] - 1;
                        if (ready) {
                            A.ncnt[X] = 0;   // the last one: ready for the next launch
                            __threadfence();
                        }
                    }
                    const unsigned r = __ballot_sync(0x1ffu, ready);
                    if (tid == 0) s_touch = r;
                }
                __syncthreads();
                unsigned r = s_touch;
                if (r) {
                    do {
                        const int q = __ffs(r) - 1;
                        r &= r - 1;
                        update_node_tile_f32<S>(A, tx + q % 3 - 1, ty + q / 3 - 1, tid, A.ind_x, A.ind_y);
                    } while (r);
                }
                moved = __reduce_add_sync(0xffffffffu, moved);
                if ((tid & 31) == 0 && moved) atomicAdd(A.moved, (unsigned long long)moved);
            }
        }
        if (DO_P2G && !tail_done) {
            // each warp marks the node tiles it wrote (no barrier: the node phase's
            // last barrier already ended every use of the shared buffers)
            touch = __reduce_or_sync(0xffffffffu, touch);
            const int lane = tid & 31;
            if (lane < 9 && ((touch >> lane) & 1u)) {
                const int ntx = tx + lane % 3 - 1, nty = ty + lane / 3 - 1;
                mark_tile(A.flags, A.tlist, A.tlist_n, A.inst, ntx, nty, A.G.ntx);
            }
            moved = __reduce_add_sync(0xffffffffu, moved);
            if ((tid & 31) == 0 && moved) atomicAdd(A.moved, (unsigned long long)moved);
        }
        if (FUSE || !DO_P2G) __syncthreads();   // the fused path reads s_touch; G2P only: s_v, s_cs reused
        staged = next_staged;
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

struct BatchClock;
constexpr int UPD_TILES = 4;


// ---------------------------------------------------------------- binning / conversion
// Binning key and rank of point i of the blocked state st (n points): its
// tile cell (or the disabled / out-of-grid bucket), its place among the
// points of that cell (warp-aggregated atomics on counts).  P: any block of
// the ints halo, gridx, gridy.
template <class S, class PT>
__device__ __forceinline__ void bin_count_point(const PT &P, const TileGeom &G, const unsigned *__restrict__ st, int n,
                                                int i, int *keys, int *ranks, int *counts, int *status)
{
    ICY_TILE_SHAPE(S);
    const bool in = i < n;
    int key = G.ntiles * TT;
    if (in) {
        const uint4 a = *reinterpret_cast<const uint4 *>(hot_vec(st, i));
        if (!(a.w & (unsigned)kDisabled)) {
            int bx, by;
            split_unpack(a.x, bx, by);
            const int e = base_error(P, bx, by);
            if (e) *status = e;
            else key = G.cell_key_s<TX, TY>(bx, by, P.halo);
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

template <class S>
static __global__ void k_bin_count_f32(StepParams P, TileGeom G, const unsigned *__restrict__ st, int n, int *keys,
                                       int *ranks, int *counts, int *status)
{
    bin_count_point<S>(P, G, st, n, blockIdx.x * blockDim.x + threadIdx.x, keys, ranks, counts, status);
}

// point i of src to its binned place start[keys[i]] + ranks[i] in dst, with its
// upload index
__device__ __forceinline__ void bin_scatter_point(const unsigned *__restrict__ src, unsigned *__restrict__ dst,
                                                  long pitch, int i, const int *__restrict__ keys,
                                                  const int *__restrict__ ranks, const int *__restrict__ start,
                                                  const int *__restrict__ oidx_src, int *__restrict__ oidx_dst)
{
    const long d = start[keys[i]] + ranks[i];
    *reinterpret_cast<uint4 *>(hot_vec(dst, d)) = *reinterpret_cast<const uint4 *>(hot_vec(src, i));
    *reinterpret_cast<uint4 *>(hot_vec(dst, d) + 128) = *reinterpret_cast<const uint4 *>(hot_vec(src, i) + 128);
    dst[hot_jp(d)] = src[hot_jp(i)];
    *reinterpret_cast<uint4 *>(dst + cold_vec(pitch, d)) = *reinterpret_cast<const uint4 *>(src + cold_vec(pitch, i));
    *reinterpret_cast<uint4 *>(dst + cold_vec(pitch, d) + 128) =
        *reinterpret_cast<const uint4 *>(src + cold_vec(pitch, i) + 128);
    oidx_dst[d] = oidx_src[i];
}

static __global__ void k_bin_scatter_f32(const unsigned *__restrict__ src, unsigned *__restrict__ dst, long pitch, int n,
                                         const int *__restrict__ keys, const int *__restrict__ ranks,
                                         const int *__restrict__ start, const int *__restrict__ oidx_src,
                                         int *__restrict__ oidx_dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) bin_scatter_point(src, dst, pitch, i, keys, ranks, start, oidx_src, oidx_dst);
}

// FP64 HSSOA chunk (16 lines, stride cpitch) -> FP32 state slots [first, first+count)
static __global__ void k_split_from_hssoa(const double *__restrict__ chunk, long cpitch, int count, unsigned *st,
                                          long pitch, int first, double hinv)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const long i = first + j;
    auto L = [&](int l) { return chunk[j + cpitch * l]; };
    int b[2];
    float g[2];
    for (int k = 0; k < 2; k++) {
        const double xs = L(4 + k) * hinv;                // pos * cellsize_inv (kernels.cuh:90)
        b[k] = (int)(xs - 0.5);
        g[k] = (float)(xs - (double)b[k] - 1.0);
    }
    PointF s;
    s.bw = split_pack(b[0], b[1]);
    s.gx = g[0];
    s.gy = g[1];
    s.util = (unsigned)(unsigned long long)__double_as_longlong(L(0));
    if ((s.util >> GE_SHIFT) == 0u) s.util |= GE_CACHED | ((unsigned)grain_entry_f32(s.util) << GE_SHIFT);
    s.d0 = make_float2((float)(L(8) - 1.0), (float)L(10));   // columns of Fe - I
    s.d1 = make_float2((float)L(9), (float)(L(11) - 1.0));
    s.Jp = (float)L(3);
    s.v = make_float2((float)L(6), (float)L(7));
    s.b0 = make_float2((float)L(12), (float)L(14));            // columns of Bp
    s.b1 = make_float2((float)L(13), (float)L(15));
    s.ptr = (float)L(1);
    s.qtr = (float)L(2);
    store_point_f32(st, pitch, i, s, true, true);
}

// FP32 state -> FP64 HSSOA chunk of upload positions [first, first+count);
// inv[o] is the slot holding the point uploaded at position o.
static __global__ void k_split_to_hssoa(const unsigned *__restrict__ st, long pitch, const int *__restrict__ inv,
                                        int first, int count, double *__restrict__ chunk, long cpitch, double h)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    const long i = inv ? inv[first + j] : first + j;
    auto W = [&](int l, double v) { chunk[j + cpitch * l] = v; };
    PointF s;
    load_point_f32(st, i, s);
    const float *c = reinterpret_cast<const float *>(st) + cold_vec(pitch, i);
    const float4 v = *reinterpret_cast<const float4 *>(c);
    const float4 bp = *reinterpret_cast<const float4 *>(c + 128);
    const unsigned u = (s.util & GE_CACHED) ? s.util & ~(GE_CACHED | (GE_MASK << GE_SHIFT)) : s.util;
    W(0, __longlong_as_double((long long)u));
    W(4, ((double)s.bx + 1.0 + (double)s.gx) * h);
    W(5, ((double)s.by + 1.0 + (double)s.gy) * h);
    W(8, 1.0 + (double)s.d0.x);
    W(9, (double)s.d1.x);
    W(10, (double)s.d0.y);
    W(11, 1.0 + (double)s.d1.y);
    W(3, (double)s.Jp);
    W(6, (double)v.x);
    W(7, (double)v.y);
    W(12, (double)bp.x);   // Bp by columns: (b00, b10, b01, b11)
    W(13, (double)bp.z);
    W(14, (double)bp.y);
    W(15, (double)bp.w);
    W(1, (double)v.z);
    W(2, (double)v.w);
}

static __global__ void k_inverse_perm(const int *__restrict__ oidx, int n, int *__restrict__ inv)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) inv[oidx[i]] = i;
}

// Per node tile: the number of cell tiles with points in its 3 x 3
// neighbourhood (the contributors the fused grid update waits for).
template <class S>
static __global__ void k_node_tile_expect(TileGeom G, const int *__restrict__ cell_start, int *__restrict__ nexp)
{
    ICY_TILE_SHAPE(S);
    const int X = blockIdx.x * blockDim.x + threadIdx.x;
    if (X >= G.ntiles) return;
    const int x = X % G.ntx, y = X / G.ntx;
    int e = 0;
    for (int dy = -1; dy <= 1; dy++)
        for (int dx = -1; dx <= 1; dx++) {
            const int tx = x + dx, ty = y + dy;
            if (tx < 0 || tx >= G.ntx || ty < 0 || ty >= G.nty) continue;
            const long t = (long)ty * G.ntx + tx;
            e += cell_start[(t + 1) * TT] > cell_start[t * TT];
        }
    nexp[X] = e;
}

// ---------------------------------------------------------------- batched re-binning
// The binning of every member of a batch in seven launches (clear, count, the
// three phases of the scan, active tiles, scatter) instead of about ten per
// member: with a hundred members the per-member launches cost the serving
// loop 30 ms of host time per re-binning.  Member m's points are blocks
// [blk0, blk0 + ceil(n / 256)) of the count and scatter grids, its keys scan
// blocks [sblk0, sblk0 + ceil(nkeys / SCAN_BLOCK)) of the scan grids.
struct BinMember {
    const unsigned *st;
    unsigned *st_alt;
    long pitch;
    int n, blk0, sblk0;
    int halo, gridx, gridy;   // for base_error
    TileGeom G;
    int *keys, *ranks, *counts, *start, *block_sums, *active, *nactive, *nexp, *ncnt, *unsafe, *status;
    const int *oidx;
    int *oidx_alt;
};

// the member whose block range holds block b (members in ascending blk0, sblk0)
template <bool SCAN>
__device__ __forceinline__ int bin_member_of(const BinMember *mem, int nmem, int b)
{
    int lo = 0, hi = nmem;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if ((SCAN ? mem[mid].sblk0 : mem[mid].blk0) <= b) lo = mid;
        else hi = mid;
    }
    return lo;
}

// counts of every member to zero (grid: 64 CTAs per member)
template <class S>
static __global__ void k_bin_clear_batch(const BinMember *__restrict__ mem)
{
    ICY_TILE_SHAPE(S);
    const BinMember &M = mem[blockIdx.y];
    const long nkeys = (long)M.G.ntiles * TT + 1;
    for (long k = (long)blockIdx.x * blockDim.x + threadIdx.x; k < nkeys; k += (long)gridDim.x * blockDim.x)
        M.counts[k] = 0;
}

template <class S>
static __global__ void k_bin_count_batch(const BinMember *__restrict__ mem, int nmem)
{
    const BinMember &M = mem[bin_member_of<false>(mem, nmem, blockIdx.x)];
    bin_count_point<S>(M, M.G, M.st, M.n, (blockIdx.x - M.blk0) * blockDim.x + threadIdx.x, M.keys, M.ranks,
                       M.counts, M.status);
}

// the scan of each member's counts (k_scan_reduce / k_scan_blocks /
// k_scan_apply over every member): start[i] = exclusive prefix, start[nkeys] = total
template <class S>
static __global__ void __launch_bounds__(SCAN_NT) k_bin_scan_reduce_batch(const BinMember *__restrict__ mem, int nmem)
{
    ICY_TILE_SHAPE(S);
    __shared__ int s_warp[SCAN_NT / 32];
    const BinMember &M = mem[bin_member_of<true>(mem, nmem, blockIdx.x)];
    const long nkeys = (long)M.G.ntiles * TT + 1;
    const int blk = blockIdx.x - M.sblk0;
    const long base = (long)blk * SCAN_BLOCK;
    int s = 0;
    for (int k = 0; k < SCAN_PER; k++) {
        const long i = base + (long)k * SCAN_NT + threadIdx.x;
        if (i < nkeys) s += M.counts[i];
    }
    int total;
    block_exclusive_scan<SCAN_NT>(s, s_warp, total);
    if (threadIdx.x == 0) M.block_sums[blk] = total;
}

template <class S>
static __global__ void __launch_bounds__(1024) k_bin_scan_blocks_batch(const BinMember *__restrict__ mem)
{
    ICY_TILE_SHAPE(S);
    __shared__ int s_warp[32];
    const BinMember &M = mem[blockIdx.x];
    const int nb = (int)(((long)M.G.ntiles * TT + 1 + SCAN_BLOCK - 1) / SCAN_BLOCK);
    const int per = (nb + 1023) / 1024;
    const int b = min((int)threadIdx.x * per, nb), e = min(b + per, nb);
    int s = 0;
    for (int k = b; k < e; k++) s += M.block_sums[k];
    int total;
    int run = block_exclusive_scan<1024>(s, s_warp, total);
    for (int k = b; k < e; k++) {
        const int c = M.block_sums[k];
        M.block_sums[k] = run;
        run += c;
    }
}

template <class S>
static __global__ void __launch_bounds__(SCAN_NT) k_bin_scan_apply_batch(const BinMember *__restrict__ mem, int nmem)
{
    ICY_TILE_SHAPE(S);
    __shared__ int s_warp[SCAN_NT / 32];
    const BinMember &M = mem[bin_member_of<true>(mem, nmem, blockIdx.x)];
    const long n = (long)M.G.ntiles * TT + 1;
    const int blk = blockIdx.x - M.sblk0;
    const long base = (long)blk * SCAN_BLOCK + (long)threadIdx.x * SCAN_PER;
    int v[SCAN_PER], s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_PER; k++) {
        v[k] = (base + k < n) ? M.counts[base + k] : 0;
        s += v[k];
    }
    int total;
    int run = block_exclusive_scan<SCAN_NT>(s, s_warp, total) + M.block_sums[blk];
#pragma unroll
    for (int k = 0; k < SCAN_PER; k++) {
        if (base + k < n) M.start[base + k] = run;
        run += v[k];
    }
    if (base + SCAN_PER >= n && base < n) M.start[n] = run;   // the thread holding the last item
}

// one CTA of 1024 threads per member: the list of tiles with points, the
// contributors per node tile, and the fused update's counters reset
template <class S>
static __global__ void __launch_bounds__(1024) k_bin_tiles_batch(const BinMember *__restrict__ mem)
{
    ICY_TILE_SHAPE(S);
    __shared__ int s_warp[32];
    const BinMember &M = mem[blockIdx.x];
    const int nt = M.G.ntiles;
    const int per = (nt + 1023) / 1024;
    const int t0 = min((int)threadIdx.x * per, nt), t1 = min(t0 + per, nt);
    int s = 0;
    for (int t = t0; t < t1; t++) s += M.start[(long)(t + 1) * TT] > M.start[(long)t * TT];
    int total;
    int run = block_exclusive_scan<1024>(s, s_warp, total);
    for (int t = t0; t < t1; t++)
        if (M.start[(long)(t + 1) * TT] > M.start[(long)t * TT]) M.active[run++] = t;
    if (threadIdx.x == 0) {
        *M.nactive = total;
        M.unsafe[0] = M.unsafe[1] = -1;
    }
    for (int X = threadIdx.x; X < nt; X += blockDim.x) {
        const int x = X % M.G.ntx, y = X / M.G.ntx;
        int e = 0;
        for (int dy = -1; dy <= 1; dy++)
            for (int dx = -1; dx <= 1; dx++) {
                const int tx = x + dx, ty = y + dy;
                if (tx < 0 || tx >= M.G.ntx || ty < 0 || ty >= M.G.nty) continue;
                const long t = (long)ty * M.G.ntx + tx;
                e += M.start[(t + 1) * TT] > M.start[t * TT];
            }
        M.nexp[X] = e;
        M.ncnt[X] = 0;
    }
}

static __global__ void k_bin_scatter_batch(const BinMember *__restrict__ mem, int nmem)
{
    const BinMember &M = mem[bin_member_of<false>(mem, nmem, blockIdx.x)];
    const int i = (blockIdx.x - M.blk0) * blockDim.x + threadIdx.x;
    if (i < M.n) bin_scatter_point(M.st, M.st_alt, M.pitch, i, M.keys, M.ranks, M.start, M.oidx, M.oidx_alt);
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

// Grid update of the node tiles P2G listed (single instance): TT threads per
// CTA, one node of each of UPD_FLAT list entries per thread and pass, their
// loads issued together so that many tiles' loads are in flight; contact
// forces go to the bins directly (a few hundred nodes touch the indenter);
// the velocities go to the buffer the next G2P reads.  The host clears the
// list after the kernel.
constexpr int UPD_FLAT = 2;
template <class S>
static __global__ void __launch_bounds__(S::TT) k_update_tiles_f32(const __grid_constant__ SplitArgs A,
                                                                  const int2 *__restrict__ tlist,
                                                                  const unsigned *__restrict__ tlist_n, double ind_x,
                                                                  double ind_y)
{
    ICY_TILE_SHAPE(S);
    const StepParams &P = A.P;
    const unsigned n = *tlist_n;
    const int l = threadIdx.x;
    for (unsigned e0 = blockIdx.x; e0 < n; e0 += gridDim.x * UPD_FLAT) {
        long q[UPD_FLAT];
        int gx[UPD_FLAT], gy[UPD_FLAT];
        float m[UPD_FLAT], px[UPD_FLAT], py[UPD_FLAT];
#pragma unroll
        for (int u = 0; u < UPD_FLAT; u++) {
            const unsigned e = e0 + u * gridDim.x;
            q[u] = -1;
            if (e >= n) continue;
            const int2 it = tlist[e];
            const int tx = it.y & 0xffff, ty = it.y >> 16;
            if (l == 0) A.flags[ty * A.G.ntx + tx] = 0u;
            gx[u] = tx * TX + l / TY - P.halo;
            gy[u] = ty * TY + l % TY;
            if (gx[u] >= P.gridx + P.halo || gy[u] >= P.gridy) continue;   // past the grid edge
            q[u] = A.g.idx(gx[u], gy[u]);
            m[u] = A.g.m[q[u]];
            px[u] = A.g.px[q[u]];
            py[u] = A.g.py[q[u]];
        }
#pragma unroll
        for (int u = 0; u < UPD_FLAT; u++) {
            if (q[u] < 0) continue;
            float vx, vy;
            double fx = 0, fy = 0;
            const int bin = node_velocity_f32(P, A.Q, gx[u], gy[u], m[u], px[u], py[u], ind_x, ind_y, vx, vy, fx, fy);
            A.g.nvx[q[u]] = vx;
            A.g.nvx[q[u] + A.n_nodes] = vy;
            if (m[u] != 0.f || px[u] != 0.f || py[u] != 0.f) {
                A.g.m[q[u]] = 0.f;
                A.g.px[q[u]] = 0.f;
                A.g.py[q[u]] = 0.f;
            }
            if (bin >= 0) {
                atomicAdd(A.acc + 2 * bin, fx);
                atomicAdd(A.acc + 2 * bin + 1, fy);
            }
        }
    }
}

// The arguments a batch member's grid update reads: 104 of SplitArgs' bytes,
// so that 300 members' fit the constant bank beside nothing else
// (batch_uargs.cu); field names as in SplitArgs.
struct UpdMember {
    struct {
        double h, dt, ind_rsq, ind_v;
        int nsub, gridx, gridy, halo;
    } P;
    struct {
        float h, dtg, vmax, vmax_sq;
    } Q;
    TileGeom G;
    GridViewB g;
    unsigned *flags;
    double *acc;
};
static_assert(sizeof(UpdMember) * 300 <= 64000, "300 members' update arguments fit the constant bank");

inline UpdMember upd_member(const SplitArgs &a)
{
    UpdMember m{};
    m.P.h = a.P.h;
    m.P.dt = a.P.dt;
    m.P.ind_rsq = a.P.ind_rsq;
    m.P.ind_v = a.P.ind_v;
    m.P.nsub = a.P.nsub;
    m.P.gridx = a.P.gridx;
    m.P.gridy = a.P.gridy;
    m.P.halo = a.P.halo;
    m.Q.h = a.Q.h;
    m.Q.dtg = a.Q.dtg;
    m.Q.vmax = a.Q.vmax;
    m.Q.vmax_sq = a.Q.vmax_sq;
    m.G = a.G;
    m.g = GridViewB{a.g.mp, a.g.v, a.g.ny, a.g.halo};
    m.flags = a.flags;
    m.acc = a.acc;
    return m;
}

#ifdef ICY_BATCH_UPD_CONST_ARGS
static __constant__ UpdMember c_upd_mem[BATCH_CONST_SLOTS];
struct ConstUpdMembers {
    __device__ __forceinline__ const UpdMember &operator[](int i) const { return c_upd_mem[i]; }
};
#endif

// Grid update of a batch's listed node tiles (all members): UPD_TILES node
// tiles per pass, their loads issued together; each member's velocities are
// updated in place (the next launch reads them) and its accumulators
// cleared; contact forces go to the member's bins.  TAB: where the members'
// arguments are (the global table, or the constant-bank copy of batch_uargs.cu).
template <class S, class TAB>
static __global__ void __launch_bounds__(256, 4) k_update_list_f32(TAB tab, const BatchClock *__restrict__ clk,
                                                                const int2 *__restrict__ tlist, unsigned *tlist_n)
{
    ICY_TILE_SHAPE(S);
    const unsigned n = *(volatile unsigned *)tlist_n;
    constexpr int TPC = 256 / TT;   // node tiles per CTA pass
    static_assert(256 % TT == 0, "whole node tiles per 256-thread CTA");
    const int l = threadIdx.x % TT;
    const unsigned stride = gridDim.x * TPC;
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
            const auto &A = tab[it.x];
            const int tx = it.y & 0xffff, ty = it.y >> 16;
            if (l == 0) A.flags[ty * A.G.ntx + tx] = 0u;
            gx[u] = tx * TX + l / TY - A.P.halo;
            gy[u] = ty * TY + (l & (TY - 1));
            if (gx[u] >= A.P.gridx + A.P.halo || gy[u] >= A.P.gridy) continue;   // past the grid edge
            q[u] = A.g.idx(gx[u], gy[u]);
            const float4 a = A.g.mp[q[u]];
            m[u] = a.x;
            px[u] = a.y;
            py[u] = a.z;
        }
#pragma unroll
        for (int u = 0; u < UPD_TILES; u++) {
            if (q[u] < 0) continue;
            const auto &A = tab[inst[u]];
            float vx, vy;
            double fx = 0, fy = 0;
            const int bin = node_velocity_f32(A.P, A.Q, gx[u], gy[u], m[u], px[u], py[u], clk[inst[u]].ind_x,
                                              clk[inst[u]].y0, vx, vy, fx, fy);
            A.g.v[q[u]] = make_float2(vx, vy);
            A.g.mp[q[u]] = make_float4(0.f, 0.f, 0.f, 0.f);
            if (bin >= 0) {
                atomicAdd(A.acc + 2 * bin, fx);
                atomicAdd(A.acc + 2 * bin + 1, fy);
            }
        }
    }
    __syncthreads();
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
