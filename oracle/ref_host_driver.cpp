// ref_host_driver.cpp -- TEST INFRASTRUCTURE / CPU baseline.
// Runs the reference's own P2G / update / G2P kernels (simulation/kernels.cuh,
// included unmodified from the reference tree) on the host: each CUDA thread
// becomes one loop iteration of an OpenMP parallel-for, atomics become OpenMP
// atomics (see oracle/refshim/hostcuda/cuda_runtime.h).  The step loop
// mirrors icy::Model::Step for one partition without point transfer
// (simulation/model.cpp:38-54) and GPU_Partition's launch wrappers
// (simulation/gpu_partition.cu:221-293).
#include <cstring>
#include <vector>
#include <omp.h>

#include "gpu_partition.h"
#include "helper_math.cuh"
#include "kernels.cuh"
#include "ref_driver_common.h"

thread_local icempm_uint3 blockIdx, threadIdx, blockDim;

template <typename F>
static void launch(int nthreads_total, F &&body) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nthreads_total; i++) {
        blockIdx = {(unsigned)i, 0, 0};
        blockDim = {1, 1, 1};
        threadIdx = {0, 0, 0};
        body();
    }
}

extern "C" {

// nsteps sub-steps on the HSSOA in place (line stride = cap, n points).
// bins: 2*n_indenter_subdivisions doubles, accumulated.  nthreads <= 0: all.
// Returns the reference's device error byte after the run.
int ref_host_run(const icy_sim_params *prm, double *soa, unsigned cap, unsigned n,
                 int step0, int nsteps, double *sim_time, double *bins, int nthreads)
{
    if (nthreads > 0) omp_set_num_threads(nthreads);
    std::memcpy(&gprms, prm, sizeof(icy::SimParams));
    gpu_error_indicator = 0;
    const size_t pitch_grid = ref_grid_pitch(prm);
    std::vector<double> grid(3 * pitch_grid);
    std::vector<double> acc(2 * prm->n_indenter_subdivisions, 0.0);
    double t = *sim_time;
    const int nNodes = ref_update_nodes(prm);
    for (int k = 0; k < nsteps; k++) {
        t += prm->InitialTimeStep;
        double ind_x = prm->indenter_x_initial + t * prm->IndVelocity;
        std::memset(grid.data(), 0, grid.size() * sizeof(double));
        launch((int)n, [&] {
            partition_kernel_p2g(prm->GridXTotal, 0, (int)pitch_grid, (int)n, (int)cap, soa, grid.data());
        });
        Eigen::Vector2d c(ind_x, prm->indenter_y);
        launch(nNodes, [&] {
            partition_kernel_update_nodes(c, nNodes, 0, (int)pitch_grid, grid.data(), acc.data(), t);
        });
        bool rec = ((step0 + k) % prm->UpdateEveryNthStep) == 0;
        launch((int)n, [&] {
            partition_kernel_g2p(rec, false, prm->GridXTotal, 0, (int)pitch_grid, (int)n, (int)cap,
                                 soa, grid.data(), nullptr, 0, nullptr, nullptr);
        });
    }
    *sim_time = t;
    if (bins)
        for (size_t i = 0; i < acc.size(); i++) bins[i] += acc[i];
    return gpu_error_indicator;
}

int ref_host_max_threads(void) { return omp_get_max_threads(); }

// The reference's device math on one matrix, for unit pins of the oracle.
void ref_host_svd(const double F[4], double U[4], double S[2], double V[4]) {
    Eigen::Matrix2d A, mU, mV;
    Eigen::Vector2d mS;
    A << F[0], F[1], F[2], F[3];
    svd2x2(A, mU, mS, mV);
    for (int r = 0; r < 2; r++)
        for (int c = 0; c < 2; c++) { U[r * 2 + c] = mU(r, c); V[r * 2 + c] = mV(r, c); }
    S[0] = mS[0]; S[1] = mS[1];
}

void ref_host_kirchhoff(const icy_sim_params *prm, const double F[4], double tau[4]) {
    std::memcpy(&gprms, prm, sizeof(icy::SimParams));
    Eigen::Matrix2d A;
    A << F[0], F[1], F[2], F[3];
    Eigen::Matrix2d T = KirchhoffStress_Wolper(A);
    for (int r = 0; r < 2; r++)
        for (int c = 0; c < 2; c++) tau[r * 2 + c] = T(r, c);
}

// ComputePQ + failure check + return mapping of one point, as G2P runs them
// (simulation/kernels.cuh:383-390).  util in/out.
void ref_host_plasticity(const icy_sim_params *prm, double F[4], double *Jp, long long *util,
                         double *ptr, double *qtr) {
    std::memcpy(&gprms, prm, sizeof(icy::SimParams));
    icy::Point p;
    p.Fe << F[0], F[1], F[2], F[3];
    p.Jp_inv = *Jp;
    p.utility_data = *util;
    p.grain = (short)p.utility_data;
    ComputePQ(p, gprms.kappa, gprms.mu);
    if (!(p.utility_data & status_crushed)) CheckIfPointIsInsideFailureSurface(p);
    if (p.utility_data & status_crushed) {
        ComputeSVD(p, gprms.kappa, gprms.mu);
        Wolper_Drucker_Prager(p);
    }
    for (int r = 0; r < 2; r++)
        for (int c = 0; c < 2; c++) F[r * 2 + c] = p.Fe(r, c);
    *Jp = p.Jp_inv;
    *util = p.utility_data;
    *ptr = p.p_tr;
    *qtr = p.q_tr;
}

}  // extern "C"
