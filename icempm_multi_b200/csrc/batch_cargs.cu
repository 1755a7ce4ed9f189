// batch_cargs.cu -- the batched tile kernel for batches of at most
// BATCH_CONST_SLOTS (300) slots, reading its members' arguments from a
// compact constant-bank copy of the batch's argument table (SplitMember,
// ICY_BATCH_CONST_ARGS in kernels_split.cuh).  The kernels of batch.cu read
// the global table, for larger batches.
#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <vector>

#include "../../include/icempm.h"
#define ICY_BATCH_CONST_ARGS
#include "kernels_split.cuh"

using namespace icy_dev;

namespace icy_dev {

int batch_const_slots() { return BATCH_CONST_SLOTS; }

// The table is one per device for the whole process: one batch at a time
// owns it (the first small batch created on the device); the others read
// their global tables.
static std::mutex g_owner_mutex;
static std::map<int, const void *> g_owner;

bool batch_const_acquire(int device, const void *batch)
{
    std::lock_guard<std::mutex> g(g_owner_mutex);
    auto it = g_owner.find(device);
    if (it != g_owner.end() && it->second) return it->second == batch;
    g_owner[device] = batch;
    return true;
}

void batch_const_release(int device, const void *batch)
{
    std::lock_guard<std::mutex> g(g_owner_mutex);
    auto it = g_owner.find(device);
    if (it != g_owner.end() && it->second == batch) it->second = nullptr;
}

// args[0 .. n) (whose device copy is d_args) into the constant bank of this
// module as compact member arguments, through `staging` (page-locked, n
// entries, not reused before the copy is done), on stream s
// (n <= BATCH_CONST_SLOTS)
cudaError_t batch_const_upload(const SplitArgs *args, const SplitArgs *d_args, int n, SplitMember *staging,
                               cudaStream_t s)
{
    if (n > BATCH_CONST_SLOTS || !staging) return cudaErrorInvalidValue;
    for (int i = 0; i < n; i++) staging[i] = split_member(args[i], d_args + i);
    return cudaMemcpyToSymbolAsync(c_batch_mem, staging, sizeof(SplitMember) * n, 0, cudaMemcpyHostToDevice, s);
}

cudaError_t batch_const_setup()
{
    cudaError_t e = cudaSuccess;
    for (int sh = 0; sh < N_SHAPES; sh++)
        with_shape(sh, [&](auto s) {
            using S = decltype(s);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_tile_f32<true, true, false, true, false, S>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MOMF_BYTES);
            if (e == cudaSuccess)
                e = cudaFuncSetAttribute(k_tile_f32<false, true, false, true, false, S>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MOMF_BYTES);
        });
    return e;
}

// kind 0: first P2G, 1: fused G2P + P2G, 2: last G2P (as in batch.cu), tile shape `shape`
void batch_const_launch_tile(int kind, int shape, int grid, cudaStream_t s, const SplitArgs &none,
                             const SplitArgs *args, const BatchItem *work, const int *nwork, const int *rec)
{
    with_shape(shape, [&](auto sh) {
        using S = decltype(sh);
        if (kind == 0)
            k_tile_f32<false, true, false, true, false, S><<<grid, TILE_THREADS_F32, MOMF_BYTES, s>>>(none, args, work,
                                                                                                      nwork, rec);
        else if (kind == 1)
            k_tile_f32<true, true, false, true, false, S><<<grid, TILE_THREADS_F32, MOMF_BYTES, s>>>(none, args, work,
                                                                                                     nwork, rec);
        else
            k_tile_f32<true, false, true, true, false, S><<<grid, TILE_THREADS_F32, 0, s>>>(none, args, work, nwork,
                                                                                            rec);
    });
}

}  // namespace icy_dev
