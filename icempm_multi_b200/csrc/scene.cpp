// scene.cpp -- seeded synthetic ice block in the reference HSSOA layout.
//
// Stands in for the HDF5 point clouds of the reference (no HDF5 library is
// available): the points are generated here, then placed exactly as
// SnapshotManager::LoadRawPoints places a loaded cloud
// (simulation/snapshotmanager.cpp:62-109).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/icempm.h"

namespace {

uint64_t mix64(uint64_t z)
{
    // splitmix64 finaliser: a counter-based hash, so point k of cell c
    // gets the same jitter whatever order the cells are generated in
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

double unit(uint64_t seed, uint64_t a, uint64_t b, uint64_t c)
{
    uint64_t h = mix64(seed ^ mix64(a ^ mix64(b ^ mix64(c))));
    return (double)(h >> 11) * (1.0 / 9007199254740992.0);  // [0,1)
}

double as_double(long long v) { double d; std::memcpy(&d, &v, 8); return d; }

void block_cells(const icy_sim_params *p, double bw, double bh, long *ncx, long *ncy)
{
    const double h = p->GridXDimension / p->GridXTotal;
    *ncx = std::max(1L, std::lround(bw / h));
    *ncy = std::max(1L, std::lround(bh / h));
}

}  // namespace

extern "C" {

/* LoadRawPoints' placement of a point cloud already in the HSSOA
   (simulation/snapshotmanager.cpp:62-109); see include/icempm.h. */
int icy_scene_place(icy_sim_params *p, double *hssoa, unsigned capacity, unsigned *n_points, double volume)
{
    if (!p || !hssoa || !n_points || *n_points == 0 || *n_points > capacity || !(volume > 0))
        return ICY_ERR_INVALID_ARGUMENT;
    icy_params_compute_helpers(p);
    const double h = p->cellsize;
    const size_t N0 = *n_points;
    size_t N = N0;
    p->nPtsTotal = (int)N;
    p->Volume = volume;
    double *X = hssoa + (size_t)ICY_POSX * capacity, *Y = hssoa + (size_t)(ICY_POSX + 1) * capacity;
    double xmin = *std::min_element(X, X + N), xmax = *std::max_element(X, X + N);
    double ymin = *std::min_element(Y, Y + N), ymax = *std::max_element(Y, Y + N);
    p->xmin = xmin; p->xmax = xmax; p->ymin = ymin; p->ymax = ymax;
    const double box_x = p->GridXTotal * h;
    const double length = xmax - xmin;
    const double x_offset = (box_x - length) / 2;
    const double y_offset = 2 * h;
    for (size_t i = 0; i < N; i++) { X[i] += x_offset; Y[i] += y_offset; }

    // RemoveDisabledAndSort (host_side_soa.cpp:50-61): drop points with the disabled bit
    // (keeping the order of the rest), then sort by the cell index of ProxyPoint::getCellIndex (proxypoint2d.cpp:114-119),
    // stable so the order is the same on every platform
    std::vector<uint32_t> perm;
    perm.reserve(N);
    for (size_t i = 0; i < N; i++) {
        long long u;
        std::memcpy(&u, hssoa + i, 8);
        if (!(u & ICY_STATUS_DISABLED)) perm.push_back((uint32_t)i);
    }
    std::vector<long> key(N);
    const double hinv = p->cellsize_inv;
    for (size_t i = 0; i < N; i++)
        key[i] = (long)(int)(X[i] * hinv + 0.5) * p->GridY + (int)(Y[i] * hinv + 0.5);
    std::stable_sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) { return key[a] < key[b]; });
    std::vector<double> tmp(perm.size());
    for (int l : {0, (int)ICY_POSX, (int)ICY_POSX + 1}) {
        double *L = hssoa + (size_t)l * capacity;
        for (size_t i = 0; i < perm.size(); i++) tmp[i] = L[perm[i]];
        std::memcpy(L, tmp.data(), sizeof(double) * perm.size());
    }
    N = perm.size();
    // the other lines start at zero (HostSideSOA::Allocate clears the buffer,
    // host_side_soa.cpp:64-79), then InitializeBlock (host_side_soa.cpp:94-105)
    for (int l = 1; l < ICY_N_PTS_ARRAYS; l++)
        if (l != ICY_POSX && l != ICY_POSX + 1) std::memset(hssoa + (size_t)l * capacity, 0, sizeof(double) * N0);
    for (size_t i = 0; i < N; i++) {
        hssoa[(size_t)ICY_IDX_JP_INV * capacity + i] = 1.0;
        hssoa[(size_t)ICY_FE00 * capacity + i] = 1.0;
        hssoa[(size_t)(ICY_FE00 + 3) * capacity + i] = 1.0;
    }
    // indenter start (snapshotmanager.cpp:84-105)
    const double block_left = x_offset;
    const double block_top = p->ymax + y_offset;
    const double r = p->IndDiameter / 2;
    const double ht = r - p->IndDepth;
    const double x_ind_offset = std::sqrt(r * r - ht * ht);
    p->indenter_x = std::floor((block_left - x_ind_offset) / h) * h;
    if (p->SetupType == 0) p->indenter_y = block_top + ht;
    else if (p->SetupType == 1) p->indenter_y = std::ceil(block_top / h) * h;
    else p->indenter_x = p->indenter_y = -1;
    p->indenter_x_initial = p->indenter_x;
    p->indenter_y_initial = p->indenter_y;
    // particle volume and mass (snapshotmanager.cpp:108-109)
    p->ParticleVolume = p->Volume / N0;
    icy_params_compute_helpers(p);
    *n_points = (unsigned)N;
    return ICY_OK;
}

unsigned icy_scene_block_count(const icy_sim_params *p, double block_w, double block_h, int ppc)
{
    long ncx, ncy;
    block_cells(p, block_w, block_h, &ncx, &ncy);
    return (unsigned)(ncx * ncy * std::max(ppc, 1));
}

int icy_scene_block(icy_sim_params *p, double block_w, double block_h, int ppc, uint64_t seed,
                    int n_grains, double *hssoa, unsigned capacity, unsigned *n_points)
{
    if (!p || !hssoa || ppc < 1 || block_w <= 0 || block_h <= 0) return ICY_ERR_INVALID_ARGUMENT;
    icy_params_compute_helpers(p);  // cellsize from GridXDimension / GridX
    const double h = p->cellsize;
    long ncx, ncy;
    block_cells(p, block_w, block_h, &ncx, &ncy);
    const size_t N = (size_t)ncx * ncy * ppc;
    if (N > capacity) return ICY_ERR_CAPACITY;
    for (int l = 0; l < ICY_N_PTS_ARRAYS; l++) std::memset(hssoa + (size_t)l * capacity, 0, sizeof(double) * N);

    // grain sites on a jittered coarse lattice (approximate Voronoi grains)
    const double area = (double)ncx * ncy * h * h;
    long gnx = 1, gny = 1;
    double gsp = 1;
    if (n_grains > 0) {
        gsp = std::sqrt(area / n_grains);
        gnx = std::max(1L, (long)std::ceil(ncx * h / gsp));
        gny = std::max(1L, (long)std::ceil(ncy * h / gsp));
    }
    std::vector<double> sx(gnx * gny), sy(gnx * gny);
    for (long i = 0; i < gnx; i++)
        for (long j = 0; j < gny; j++) {
            sx[i * gny + j] = (i + unit(seed, 0x51, i, j)) * gsp;
            sy[i * gny + j] = (j + unit(seed, 0x52, i, j)) * gsp;
        }

    // stratified jitter: ppc = m*m points on an m x m sub-lattice of the cell
    int m = (int)std::lround(std::sqrt((double)ppc));
    bool strat = (m * m == ppc);
    double *X = hssoa + (size_t)ICY_POSX * capacity, *Y = hssoa + (size_t)(ICY_POSX + 1) * capacity;
    size_t q = 0;
    for (long cx = 0; cx < ncx; cx++)
        for (long cy = 0; cy < ncy; cy++) {
            uint64_t cell = (uint64_t)cx * (uint64_t)ncy + cy;
            for (int k = 0; k < ppc; k++, q++) {
                double u = unit(seed, cell, k, 1), v = unit(seed, cell, k, 2);
                if (strat) { u = ((k % m) + u) / m; v = ((k / m) + v) / m; }
                double x = (cx + u) * h, y = (cy + v) * h;
                X[q] = x;
                Y[q] = y;
                long long grain = 0;
                if (n_grains > 0) {
                    long gi = std::min(gnx - 1, (long)(x / gsp)), gj = std::min(gny - 1, (long)(y / gsp));
                    double best = 1e300;
                    for (long a = std::max(0L, gi - 2); a <= std::min(gnx - 1, gi + 2); a++)
                        for (long b = std::max(0L, gj - 2); b <= std::min(gny - 1, gj + 2); b++) {
                            double dx = sx[a * gny + b] - x, dy = sy[a * gny + b] - y, d2 = dx * dx + dy * dy;
                            if (d2 < best) { best = d2; grain = (a * gny + b) % 65536; }
                        }
                }
                hssoa[q] = as_double(grain);
            }
        }

    unsigned n = (unsigned)N;
    int rc = icy_scene_place(p, hssoa, capacity, &n, area);
    if (rc != ICY_OK) return rc;
    if (n_points) *n_points = n;
    return ICY_OK;
}

}  // extern "C"
