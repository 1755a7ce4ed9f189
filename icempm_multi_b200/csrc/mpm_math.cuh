// mpm_math.cuh -- per-particle and per-node MLS-MPM math for the device.
//
// Each function states the reference expression it evaluates
// (simulation/kernels.cuh, helper_math.cuh, givens.cuh).  The order of every
// sum and product follows the reference's Eigen expressions (linear
// reductions, (s*A)*B for a scalar in front of a product, normalize() of a
// zero vector is a no-op), so that FP64 results differ from the CPU oracle
// only by FMA contraction and atomic summation order.  Matrices are four
// named scalars m00, m01, m10, m11 (row, column).
#pragma once
#include <cstdint>

namespace icy_dev {

constexpr double kPi = 3.14159265358979323846;
constexpr double kCoeff1 = 1.4142135623730950;     // sqrt((6-d)/2), d = 2
constexpr double kCoeff1Inv = 0.7071067811865475;
constexpr long long kCrushed = 0x10000, kDisabled = 0x20000, kLiquid = 0x40000;

template <typename T> struct M2 { T a00, a01, a10, a11; };

// Parameters one kernel needs, filled from icy_sim_params on the host.
struct StepParams {
    double h, hinv, dt, dt_vol_Dpinv, dt_gravity, vmax, vmax_sq, ind_rsq, ind_v;
    double mass_ice, mass_water, mu, kappa, tan_phi, dp_p, pmax, pmin_t, qmax_s, t2, beta, grain_var;
    int gridx, gridy, halo, nsub;
};

template <typename T> __device__ __forceinline__ T sqrt_t(T x);
template <> __device__ __forceinline__ double sqrt_t<double>(double x) { return sqrt(x); }
template <> __device__ __forceinline__ float sqrt_t<float>(float x) { return sqrtf(x); }

// quadratic B-spline weights of one axis (kernels.cuh:99-103)
template <typename T>
__device__ __forceinline__ void bspline_weights(T f, T w[3])
{
    T a0 = T(1.5) - f, a1 = f - T(1.0), a2 = f - T(0.5);
    w[0] = (T(0.5) * a0) * a0;
    w[1] = T(0.75) - a1 * a1;
    w[2] = (T(0.5) * a2) * a2;
}

// dev(F F^T) (kernels.cuh:31, 591-594)
template <typename T>
__device__ __forceinline__ M2<T> dev_ffT(const M2<T> &F)
{
    T b00 = F.a00 * F.a00 + F.a01 * F.a01;
    T b01 = F.a00 * F.a10 + F.a01 * F.a11;
    T b11 = F.a10 * F.a10 + F.a11 * F.a11;
    T hh = (b00 + b11) / T(2);
    return {b00 - hh, b01, b01, b11 - hh};
}

template <typename T>
__device__ __forceinline__ T det2(const M2<T> &F) { return F.a00 * F.a11 - F.a10 * F.a01; }

// KirchhoffStress_Wolper (kernels.cuh:24-34): mu/J dev(FF^T) + kappa/2 (J^2-1) I
template <typename T>
__device__ __forceinline__ M2<T> kirchhoff(const M2<T> &F, T mu, T kappa)
{
    T Je = det2(F);
    M2<T> d = dev_ffT(F);
    T s1 = mu * (T(1) / Je);
    T s2 = (kappa * T(0.5)) * (Je * Je - T(1));
    return {s1 * d.a00 + s2, s1 * d.a01, s1 * d.a10, s1 * d.a11 + s2};
}

// Water (kernels.cuh:37-44): kappa (1 - J^-5) I
__device__ __forceinline__ M2<double> water_stress(double J, double kappa)
{
    double s = kappa * (1. - pow(J, -5.0));
    return {s, 0., 0., s};
}

// ComputePQ (kernels.cuh:547-557)
template <typename T>
__device__ __forceinline__ void compute_pq(const M2<T> &F, T mu, T kappa, T &Je, T &p, T &q)
{
    Je = det2(F);
    p = (-(kappa / T(2))) * (Je * Je - T(1));
    M2<T> d = dev_ffT(F);
    // Frobenius norm, column-major summation order
    T sq = ((d.a00 * d.a00 + d.a10 * d.a10) + d.a01 * d.a01) + d.a11 * d.a11;
    q = ((T(kCoeff1) * mu) * (T(1) / Je)) * sqrt_t(sq);
}

// Grain-dependent constants of the failure surface.  GetParametersForGrain
// (kernels.cuh:560-576) varies them with (grain+3) % 30 and (grain+4) % 11
// only, so they take 59 x 21 distinct values (C++ remainders of a signed
// 16-bit grain id lie in [-29, 29] and [-10, 10]); a per-instance table of
// the exact same expressions replaces 3 divisions and a square root per point.
constexpr int GRAIN_N30 = 59, GRAIN_N11 = 21, GRAIN_TAB = GRAIN_N30 * GRAIN_N11;
struct GrainConst { double pmin2, k, msq; };

__device__ __forceinline__ GrainConst grain_constants(const StepParams &P, int r30, int r11)
{
    double var2 = 1.0 + P.grain_var * 0.033 * (double)(-15 + r30);
    double var3 = 1.0 + P.grain_var * 0.1 * (double)(-10 + r11);
    double pmax = P.pmax, pmin = -P.pmin_t;
    double qmax = P.qmax_s * var3;
    double pmin2 = -P.t2 * var2;
    double beta = P.beta;
    GrainConst c;
    c.msq = (4 * qmax * qmax * (1 + 2 * beta)) / ((pmax - pmin) * (pmax - pmin));
    double q0 = 2 * sqrt(-pmax * pmin) * qmax / (pmax - pmin);
    c.k = -q0 / pmin2;
    c.pmin2 = pmin2;
    return c;
}

__device__ __forceinline__ int grain_slot(int grain)
{
    return ((grain + 3) % 30 + 29) * GRAIN_N11 + ((grain + 4) % 11 + 10);
}

// CheckIfPointIsInsideFailureSurface with the grain constants looked up (kernels.cuh:598-619)
__device__ __forceinline__ bool failure_surface_crushed_tab(const StepParams &P, const GrainConst &c, double p,
                                                            double q)
{
    if (p < 0) {
        if (p < c.pmin2) return true;
        double q_limit = c.k * (p - c.pmin2);
        return q > q_limit;
    }
    double y = (1. + 2. * P.beta) * q * q + c.msq * (p + P.beta * P.pmax) * (p - P.pmax);
    return y > 0;
}

// GetParametersForGrain + CheckIfPointIsInsideFailureSurface (kernels.cuh:560-619)
__device__ __forceinline__ bool failure_surface_crushed(const StepParams &P, int grain, double p, double q)
{
    double var2 = 1.0 + P.grain_var * 0.033 * (double)(-15 + (grain + 3) % 30);
    double var3 = 1.0 + P.grain_var * 0.1 * (double)(-10 + (grain + 4) % 11);
    double pmax = P.pmax, pmin = -P.pmin_t;
    double qmax = P.qmax_s * var3;
    double pmin2 = -P.t2 * var2;
    double beta = P.beta;
    double mSq = (4 * qmax * qmax * (1 + 2 * beta)) / ((pmax - pmin) * (pmax - pmin));
    if (p < 0) {
        if (p < pmin2) return true;
        double q0 = 2 * sqrt(-pmax * pmin) * qmax / (pmax - pmin);
        double k = -q0 / pmin2;
        double q_limit = k * (p - pmin2);
        return q > q_limit;
    }
    double y = (1. + 2. * beta) * q * q + mSq * (p + beta * pmax) * (p - pmax);
    return y > 0;
}

// 2x2 SVD as the reference builds it: polar decomposition by one Givens
// rotation, then one Jacobi rotation of the symmetric factor, singular values
// sorted descending (helper_math.cuh:27-46, 81-140; givens.cuh:99-166;
// kernels.cuh:521-538).  Returns the rotations (uc, us) and (vc, vs) such that
// U = [[uc, us], [-us, uc]] and V = [[vc, vs], [-vs, vc]] in the reference's
// row-wise fill convention.
__device__ __forceinline__ void svd2x2(const M2<double> &F, double &uc, double &us, double &s0,
                                       double &s1, double &vc, double &vs)
{
    // column-major a = {F00, F10, F01, F11}
    double a0 = F.a00, a1 = F.a10, a2 = F.a01, a3 = F.a11;
    double x0 = a0 + a3, x1 = a1 - a2;
    double den = sqrt(x0 * x0 + x1 * x1);
    uc = 1; us = 0;
    if (den != 0) { uc = x0 / den; us = -x1 / den; }
    // S = G a, column by column
    double S0 = uc * a0 - us * a1;   // S(0,0)
    double S2 = uc * a2 - us * a3;   // S(0,1)
    double S3 = us * a2 + uc * a3;   // S(1,1)
    double x = S0, y = S2, z = S3, y2 = y * y;
    double cosine, sine;
    if (y2 == 0) {
        cosine = 1; sine = 0; s0 = x; s1 = z;
    } else {
        double tau = 0.5 * (x - z);
        double w = sqrt(tau * tau + y2);
        double t = (tau > 0) ? y / (tau + w) : y / (tau - w);
        cosine = 1.0 / sqrt(t * t + 1.0);
        sine = -t * cosine;
        double c2 = cosine * cosine, csy = 2 * cosine * sine * y, sn2 = sine * sine;
        s0 = c2 * x - csy + sn2 * z;
        s1 = sn2 * x + csy + c2 * z;
    }
    if (s0 < s1) { double tmp = s0; s0 = s1; s1 = tmp; vc = -sine; vs = cosine; }
    else { vc = cosine; vs = sine; }
    double nc = uc * vc - us * vs, ns = us * vc + uc * vs;
    uc = nc; us = ns;
}

// Fe = U diag(s) V^T evaluated as (U*D)*V^T (kernels.cuh:642,671)
__device__ __forceinline__ M2<double> usv(double uc, double us, double s0, double s1, double vc, double vs)
{
    // U = [[uc, us], [-us, uc]], V = [[vc, vs], [-vs, vc]]
    double ud00 = uc * s0, ud01 = us * s1, ud10 = -us * s0, ud11 = uc * s1;
    return {ud00 * vc + ud01 * vs, ud00 * (-vs) + ud01 * vc,
            ud10 * vc + ud11 * vs, ud10 * (-vs) + ud11 * vc};
}

// ComputeSVD + Wolper_Drucker_Prager for a crushed point (kernels.cuh:540-545, 623-674)
__device__ __forceinline__ void return_map(const StepParams &P, M2<double> &F, double &Jp, double ptr,
                                           double qtr, double Je)
{
    double uc, us, s0, s1, vc, vs;
    svd2x2(F, uc, us, s0, s1, vc, vs);
    double sq0 = s0 * s0, sq1 = s1 * s1;
    double hs = (sq0 + sq1) / 2;
    double f = P.mu / Je;
    double vsh0 = f * (sq0 - hs), vsh1 = f * (sq1 - hs);
    if (ptr < -P.dp_p || Jp < 1) {
        double p_new = -P.dp_p;
        double Je_new = sqrt(-2. * p_new / P.kappa + 1.);
        double sj = sqrt(Je_new);
        F = usv(uc, us, sj, sj, vc, vs);
        Jp = Jp * (Je_new / Je);
    } else {
        double q_n_1;
        if (ptr > P.pmax) {
            q_n_1 = 0;
        } else {
            double q_from_dp = (ptr + P.dp_p) * P.tan_phi;
            double pmin = -P.pmin_t;
            double q_from_fs = 2 * sqrt((P.pmax - ptr) * (ptr - pmin)) * P.qmax_s / (P.pmax - pmin);
            q_n_1 = fmin(q_from_fs, q_from_dp);
        }
        if (qtr >= q_n_1) {
            double snorm = q_n_1 * kCoeff1Inv;
            double z = vsh0 * vsh0 + vsh1 * vsh1;
            double n0 = vsh0, n1 = vsh1;
            if (z > 0) { double r = sqrt(z); n0 = vsh0 / r; n1 = vsh1 / r; }
            double k = snorm * (Je / P.mu);
            double tr = (sq0 + sq1) / 2.;
            F = usv(uc, us, sqrt(k * n0 + tr), sqrt(k * n1 + tr), vc, vs);
        }
    }
}

// Grid-node velocity update (kernels.cuh:175-300).  gix, giy: node indices
// in the whole grid.  Returns false for an empty node (left untouched).
// On indenter contact, *bin and (fx, fy) receive the reaction force sample.
__device__ __forceinline__ bool node_update(const StepParams &P, int gix, int giy, double mass, double px,
                                            double py, double ind_x, double ind_y, double &vx, double &vy,
                                            int &bin, double &fx, double &fy)
{
    bin = -1;
    if (mass == 0) return false;
    double gnx = (double)gix * P.h, gny = (double)giy * P.h;
    vx = px / mass;
    vy = py / mass;
    vy = vy - P.dt_gravity;
    if (vx * vx + vy * vy > P.vmax_sq) {
        double r = sqrt(vx * vx + vy * vy);
        vx = (vx / r) * P.vmax;
        vy = (vy / r) * P.vmax;
    }
    double nx = gnx - ind_x, ny = gny - ind_y;
    if (nx * nx + ny * ny < P.ind_rsq) {
        double vrx = vx - P.ind_v, vry = vy;
        double z = nx * nx + ny * ny;
        if (z > 0) { double r = sqrt(z); nx = nx / r; ny = ny / r; }
        double vn = vrx * nx + vry * ny;
        if (vn < 0) {
            double vtx = vrx - nx * vn, vty = vry - ny * vn;
            double pvx = vx, pvy = vy;
            vx = P.ind_v + vtx;
            vy = vty;
            fx = (pvx - vx) * mass / P.dt;
            fy = (pvy - vy) * mass / P.dt;
            float angle = atan2f((float)nx, (float)ny);
            angle = (float)((double)angle + kPi);
            angle = (float)((double)angle * (P.nsub / (2 * kPi)));
            int index = (int)angle;
            bin = min(max(index, 0), P.nsub - 1);
        }
    }
    if (giy <= 2) { vx = 0; vy = 0; }
    if (giy >= P.gridy - 3 && vy > 0) vy = 0;
    if (gix <= 2 && vx < 0) vx = 0;
    else if (gix >= P.gridx - 3 && vx > 0) vx = 0;
    return true;
}

// reference error codes for a stencil base outside the grid (kernels.cuh:94-97)
// (P: any parameter block with the int fields halo, gridx, gridy)
template <class PT>
__device__ __forceinline__ int base_error(const PT &P, int bx, int by)
{
    int e = 0;
    if (bx < -P.halo) e = 70;
    if (by < 0) e = 71;
    if (bx > P.gridx + P.halo - 3) e = 72;
    if (by > P.gridy - 3) e = 73;
    return e;
}

}  // namespace icy_dev
