// ref_cuda_driver.cu -- TEST INFRASTRUCTURE / reference-on-the-same-GPU arm.
// Runs the reference's own CUDA kernels (simulation/kernels.cuh, compiled
// unmodified from the reference tree for sm_100a) as ONE partition with the
// launch shapes and order of GPU_Partition (simulation/gpu_partition.cu:221-293)
// and icy::Model::Step without point transfer (simulation/model.cpp:38-54).
//
// The reference kernels do not stop at an out-of-grid particle
// (simulation/kernels.cuh:94-97 only record a code), so callers must only
// pass inputs that the CPU oracle has shown to stay inside the grid.
#include <cstring>
#include <cuda_runtime.h>

#include "gpu_partition.h"
#include "helper_math.cuh"
#include "kernels.cuh"
#include "ref_driver_common.h"

extern "C" {

// nsteps sub-steps on the HSSOA in place (host memory, line stride = cap).
// bins accumulates the indenter force; *ms receives the device time of the
// step loop (CUDA events).  Returns the device error byte, or -1 on a CUDA error.
int ref_cuda_run(const icy_sim_params *prm, double *soa, unsigned cap, unsigned n,
                 int step0, int nsteps, double *sim_time, double *bins, float *ms)
{
    const size_t pitch_grid = ref_grid_pitch(prm);
    const int nNodes = ref_update_nodes(prm);
    const size_t acc_bytes = sizeof(double) * 2 * prm->n_indenter_subdivisions;
    double *d_pts = nullptr, *d_grid = nullptr, *d_acc = nullptr;
    cudaStream_t s;
    cudaEvent_t e0, e1;
    int rc = -1;
    uint8_t code = 0;
    if (cudaStreamCreate(&s) != cudaSuccess) return -1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    if (cudaMalloc(&d_pts, sizeof(double) * cap * 16) != cudaSuccess) goto done;
    if (cudaMalloc(&d_grid, sizeof(double) * pitch_grid * 3) != cudaSuccess) goto done;
    if (cudaMalloc(&d_acc, acc_bytes) != cudaSuccess) goto done;
    cudaMemsetAsync(d_acc, 0, acc_bytes, s);
    cudaMemcpyAsync(d_pts, soa, sizeof(double) * cap * 16, cudaMemcpyHostToDevice, s);
    if (cudaMemcpyToSymbol(gprms, prm, sizeof(icy::SimParams)) != cudaSuccess) goto done;
    if (cudaMemcpyToSymbol(gpu_error_indicator, &code, 1) != cudaSuccess) goto done;
    {
        double t = *sim_time;
        cudaEventRecord(e0, s);
        for (int k = 0; k < nsteps; k++) {
            t += prm->InitialTimeStep;
            double ind_x = prm->indenter_x_initial + t * prm->IndVelocity;
            cudaMemsetAsync(d_grid, 0, sizeof(double) * pitch_grid * 3, s);
            int tpb = prm->tpb_P2G;
            partition_kernel_p2g<<<(n + tpb - 1) / tpb, tpb, 0, s>>>(prm->GridXTotal, 0, (int)pitch_grid,
                                                                     (int)n, (int)cap, d_pts, d_grid);
            tpb = prm->tpb_Upd;
            Eigen::Vector2d c(ind_x, prm->indenter_y);
            partition_kernel_update_nodes<<<(nNodes + tpb - 1) / tpb, tpb, 0, s>>>(c, nNodes, 0, (int)pitch_grid,
                                                                                 d_grid, d_acc, t);
            bool rec = ((step0 + k) % prm->UpdateEveryNthStep) == 0;
            tpb = prm->tpb_G2P;
            partition_kernel_g2p<<<(n + tpb - 1) / tpb, tpb, 0, s>>>(rec, false, prm->GridXTotal, 0,
                                                                     (int)pitch_grid, (int)n, (int)cap, d_pts,
                                                                     d_grid, nullptr, 0, nullptr, nullptr);
        }
        cudaEventRecord(e1, s);
        *sim_time = t;
    }
    cudaMemcpyAsync(soa, d_pts, sizeof(double) * cap * 16, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) goto done;
    if (ms) cudaEventElapsedTime(ms, e0, e1);
    if (bins) {
        double *h = new double[2 * prm->n_indenter_subdivisions];
        cudaMemcpy(h, d_acc, acc_bytes, cudaMemcpyDeviceToHost);
        for (int i = 0; i < 2 * prm->n_indenter_subdivisions; i++) bins[i] += h[i];
        delete[] h;
    }
    if (cudaMemcpyFromSymbol(&code, gpu_error_indicator, 1) != cudaSuccess) goto done;
    rc = code;
done:
    cudaFree(d_pts);
    cudaFree(d_grid);
    cudaFree(d_acc);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    return rc;
}

}  // extern "C"
