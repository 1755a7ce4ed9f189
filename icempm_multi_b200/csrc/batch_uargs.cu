// batch_uargs.cu -- the batched grid update for batches of at most
// BATCH_CONST_SLOTS (300) slots, reading its members' arguments from a
// compact constant-bank copy of the batch's argument table (UpdMember,
// ICY_BATCH_UPD_CONST_ARGS in kernels_split.cuh): in a translation unit of its
// own, whose constant bank holds nothing else.  The batch that owns the tile
// kernel's constant-bank table (batch_cargs.cu) owns this one too.
#include <cuda_runtime.h>

#include "../../include/icempm.h"
#define ICY_BATCH_UPD_CONST_ARGS
#include "kernels_split.cuh"

using namespace icy_dev;

namespace icy_dev {

// args[0 .. n) into the constant bank of this module as compact update
// arguments, through `staging` (page-locked, n entries, not reused before
// the copy is done), on stream s (n <= BATCH_CONST_SLOTS)
cudaError_t batch_upd_const_upload(const SplitArgs *args, int n, UpdMember *staging, cudaStream_t s)
{
    if (n > BATCH_CONST_SLOTS || !staging) return cudaErrorInvalidValue;
    for (int i = 0; i < n; i++) staging[i] = upd_member(args[i]);
    return cudaMemcpyToSymbolAsync(c_upd_mem, staging, sizeof(UpdMember) * n, 0, cudaMemcpyHostToDevice, s);
}

void batch_upd_const_launch(int shape, int grid, cudaStream_t s, const BatchClock *clk, const int2 *tlist,
                            unsigned *tlist_n)
{
    with_shape(shape, [&](auto sh) {
        k_update_list_f32<decltype(sh), ConstUpdMembers><<<grid, 256, 0, s>>>(ConstUpdMembers{}, clk, tlist, tlist_n);
    });
}

}  // namespace icy_dev
