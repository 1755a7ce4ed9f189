// instance.cu -- allocation, host<->device transfer and the step loop of one
// simulation instance.
#include <cuda_runtime.h>

#include "instance.cuh"
#include "kernels_simple.cuh"

using namespace icy_dev;

#define CK(call)                                                                  \
    do {                                                                          \
        cudaError_t e_ = (call);                                                  \
        if (e_ != cudaSuccess) { icy_set_error(#call, e_); return ICY_ERR_CUDA; } \
    } while (0)
#define CK_LAUNCH(where)                                                          \
    do {                                                                          \
        cudaError_t e_ = cudaGetLastError();                                      \
        if (e_ != cudaSuccess) { icy_set_error(where, e_); return ICY_ERR_CUDA; } \
        h->launches++;                                                            \
    } while (0)

static GridView grid_view(icy_mpm *h)
{
    GridView g;
    g.m = h->d_grid;
    g.px = h->d_grid + h->n_nodes;
    g.py = h->d_grid + 2 * h->n_nodes;
    g.vx = h->d_grid + 3 * h->n_nodes;
    g.vy = h->d_grid + 4 * h->n_nodes;
    g.ny = h->prm.GridY;
    g.halo = h->prm.GridHaloSize;
    return g;
}

int icy_instance_allocate(icy_mpm *h, unsigned capacity)
{
    if (h->precision != ICY_PRECISION_FP64) return ICY_ERR_NOT_SUPPORTED;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;
    h->capacity = capacity;
    h->pitch = ((long)capacity + 31) / 32 * 32;
    h->n_nodes = (long)h->prm.GridY * (h->prm.GridXTotal + 2 * h->prm.GridHaloSize);
    cudaError_t e;
    if ((e = cudaMalloc(&h->d_pts, sizeof(double) * 16 * h->pitch)) != cudaSuccess) {
        icy_set_error("cudaMalloc(particles)", e);
        return ICY_ERR_OUT_OF_MEMORY;
    }
    if ((e = cudaMalloc(&h->d_grid, sizeof(double) * 5 * h->n_nodes)) != cudaSuccess) {
        icy_set_error("cudaMalloc(grid)", e);
        return ICY_ERR_OUT_OF_MEMORY;
    }
    CK(cudaMalloc(&h->d_acc, sizeof(double) * 2 * h->prm.n_indenter_subdivisions));
    CK(cudaMalloc(&h->d_status, sizeof(int)));
    CK(cudaMallocHost(&h->h_status, sizeof(int)));
    CK(cudaMemsetAsync(h->d_pts, 0, sizeof(double) * 16 * h->pitch, h->stream));
    CK(cudaMemsetAsync(h->d_grid, 0, sizeof(double) * 5 * h->n_nodes, h->stream));
    CK(cudaMemsetAsync(h->d_acc, 0, sizeof(double) * 2 * h->prm.n_indenter_subdivisions, h->stream));
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(int), h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return ICY_OK;
}

void icy_instance_free(icy_mpm *h)
{
    icy_prof_free(h);
    if (h->own_stream) cudaStreamSynchronize(h->own_stream);
    if (h->stream && h->stream != h->own_stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->d_pts);
    cudaFree(h->d_grid);
    cudaFree(h->d_acc);
    cudaFree(h->d_status);
    cudaFreeHost(h->h_status);
    if (h->own_stream) cudaStreamDestroy(h->own_stream);
    h->d_pts = h->d_grid = h->d_acc = nullptr;
    h->d_status = h->h_status = nullptr;
    h->own_stream = h->stream = nullptr;
}

int icy_instance_upload(icy_mpm *h, const double *hssoa, unsigned cap, unsigned size)
{
    // one 2-D copy: 16 lines of `size` doubles, host line stride = cap
    if (size)
        CK(cudaMemcpy2DAsync(h->d_pts, sizeof(double) * h->pitch, hssoa, sizeof(double) * cap,
                             sizeof(double) * size, 16, cudaMemcpyHostToDevice, h->stream));
    h->n = size;
    return ICY_OK;
}

int icy_instance_download(icy_mpm *h, double *hssoa, unsigned cap)
{
    if (h->n)
        CK(cudaMemcpy2DAsync(hssoa, sizeof(double) * cap, h->d_pts, sizeof(double) * h->pitch,
                             sizeof(double) * h->n, 16, cudaMemcpyDeviceToHost, h->stream));
    return ICY_OK;
}

int icy_phase_reset_grid(icy_mpm *h)
{
    icy_prof_begin(h, K_MEMSET_GRID);
    CK(cudaMemsetAsync(h->d_grid, 0, sizeof(double) * 3 * h->n_nodes, h->stream));
    icy_prof_end(h);
    return ICY_OK;
}

int icy_phase_p2g(icy_mpm *h)
{
    if (!h->n) return ICY_OK;
    StepParams P = icy_step_params(h->prm);
    const int tpb = 256;
    icy_prof_begin(h, K_P2G_SIMPLE);
    k_p2g_simple<<<(h->n + tpb - 1) / tpb, tpb, 0, h->stream>>>(P, h->d_pts, h->pitch, (int)h->n, grid_view(h),
                                                                h->d_status);
    icy_prof_end(h);
    CK_LAUNCH("k_p2g_simple");
    return ICY_OK;
}

int icy_phase_update(icy_mpm *h, double ind_x, double ind_y)
{
    StepParams P = icy_step_params(h->prm);
    const int tpb = 256;
    const long nb = (h->n_nodes + tpb - 1) / tpb;
    icy_prof_begin(h, K_UPDATE_SIMPLE);
    k_update_simple<<<(unsigned)nb, tpb, sizeof(double) * 2 * P.nsub, h->stream>>>(P, grid_view(h), h->n_nodes,
                                                                                 ind_x, ind_y, h->d_acc);
    icy_prof_end(h);
    CK_LAUNCH("k_update_simple");
    return ICY_OK;
}

int icy_phase_g2p(icy_mpm *h, bool recordPQ)
{
    if (!h->n) return ICY_OK;
    StepParams P = icy_step_params(h->prm);
    const int tpb = 128;
    icy_prof_begin(h, K_G2P_SIMPLE);
    k_g2p_simple<<<(h->n + tpb - 1) / tpb, tpb, 0, h->stream>>>(P, h->d_pts, h->pitch, (int)h->n, grid_view(h),
                                                                recordPQ ? 1 : 0, h->d_status);
    icy_prof_end(h);
    CK_LAUNCH("k_g2p_simple");
    return ICY_OK;
}

int icy_instance_steps(icy_mpm *h, int step0, int nsteps, double *sim_time)
{
    double t = *sim_time;
    const icy_sim_params &p = h->prm;
    for (int k = 0; k < nsteps; k++) {
        // icy::Model::Step sub-step (simulation/model.cpp:40-49)
        t += p.InitialTimeStep;
        const double ind_x = p.indenter_x_initial + t * p.IndVelocity;
        int rc;
        if ((rc = icy_phase_reset_grid(h))) return rc;
        if ((rc = icy_phase_p2g(h))) return rc;
        if ((rc = icy_phase_update(h, ind_x, p.indenter_y))) return rc;
        const bool rec = ((step0 + k) % p.UpdateEveryNthStep) == 0;
        if ((rc = icy_phase_g2p(h, rec))) return rc;
    }
    *sim_time = t;
    return ICY_OK;
}
