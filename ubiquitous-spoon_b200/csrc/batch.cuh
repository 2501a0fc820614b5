// Batched launches: one kernel launch covers the same stage of many
// independent instances of different sizes.
//
// Every kernel body takes its block index as an argument.  The single-instance
// kernel passes blockIdx; the batched kernel receives a device array of
// per-instance records (the instance's geometry and arguments, its own grid
// and the first flat block it owns), finds its record by a binary search over
// the records' first blocks, and runs the same body with the local block
// index.  Records are built on the host by the batch (instance.cu) and live in
// device memory for as long as the launches (or the CUDA graph holding them)
// may run.
#pragma once

#include "engine.cuh"

namespace cf {

template <class Args>
struct BatchRec {
    Geo G;
    Args A;
    unsigned gx, gy, gz;   // this instance's grid
    unsigned begin;        // its first flat block in the batched launch
};

// Flat block of this launch -> its record and the block index within it.
template <class Rec>
__device__ __forceinline__ const Rec& batch_locate(const Rec* __restrict__ r, int n, uint3& bid)
{
    const unsigned b = blockIdx.x;
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (r[mid].begin <= b) lo = mid;
        else hi = mid - 1;
    }
    const Rec& R = r[lo];
    unsigned l = b - R.begin;
    bid.x = l % R.gx;
    l /= R.gx;
    bid.y = l % R.gy;
    bid.z = l / R.gy;
    return R;
}

// One batched launch: `recs` points at n device records whose grids add up
// to `blocks` flat blocks; `smem` is the dynamic shared memory of the
// largest instance; `block` the block shape of the kernels with a tuned
// shape (every record's grid was formed with it).
struct BatchLaunch {
    const void* recs;
    int n;
    unsigned blocks;
    size_t smem;
    dim3 block;
};

}  // namespace cf
