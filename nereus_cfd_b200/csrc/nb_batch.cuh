// Device tables of a batch of solves (nb_batch.cu): many requests advanced by the same launches. A batched launch has
// grid z = the batch's capacity; block z runs the request at list[z] of the current work list while z < *count, with
// that request's own level data, vectors and reductions, on the x, y tiles of the grid a single solve of it would
// launch. Requests that converged leave the list, so their tiles cost an empty block each.
#pragma once
#include "nb_device.cuh"

namespace nb
{

// one level of one request
struct BatchLevel
{
    LevelView v;
    const uint8_t *du;   // the level's diagonal units (colour-split layout)
    const uint8_t *pext; // its red cells' prolongation bytes toward the next coarser level
    float *r, *e, *res;  // its FP32 vectors
};

// one request
struct BatchReq
{
    Reducer red;  // its own partial sums, counter and scalar slots (red.out)
    int *it;      // its CG iteration number
    int singular; // all-Neumann: the CG scalars remove z's mean
    long long vecLen;
    float *x, *p0, *p1, *q; // level 0's CG vectors (z is level 0's e, r its r)
    const double *b;        // the right-hand side (grid layout)
    double *xin, *xout;     // this refinement pass's FP64 iterates (grid layout)
    double scale, sfac;
    const void *tail; // its coarse end's TailArgs<float> (device memory)
};

// the requests a launch runs
struct BatchList
{
    const int *list;
    const int *count;
};

// The request of this block, or -1 when the block's slot is past the list (it then returns at once).
__device__ __forceinline__ int BatchReqOf(const BatchList &a)
{
    const int z = (int)blockIdx.z;
    return z < *a.count ? a.list[z] : -1;
}

} // namespace nb
