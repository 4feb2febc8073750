// Host-side declarations of the B200 pressure-projection kernels' launchers.
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/nereus_b200.h"
#include "nb_batch.cuh"
#include "nb_device.cuh"

namespace nb
{

// Kernel launches made by this library in this process (nereus_b200_kernel_launches).
extern std::atomic<long long> g_launches;
#define NB_COUNT_LAUNCH() ::nb::g_launches.fetch_add(1, std::memory_order_relaxed)
#define NB_COUNT_LAUNCHES(n) ::nb::g_launches.fetch_add((n), std::memory_order_relaxed)

// ---- nb_exact.cu: reference-exact kernels ----
void LaunchLabelCells(int dim, int Nx, int Ny, int Nz, const double *cx, const double *cy, const double *cz,
                      const nb_scene &s, uint8_t *types, cudaStream_t st);
int NumberUnknowns(const LevelView &v, int32_t *idp, int *lineCounts, int *lineOffsets, void *scanTmp,
                   size_t scanTmpBytes, int *hostTotal, cudaStream_t st);
size_t ScanTempBytes(int n);
int ExportMatrix(const LevelView &v, const int32_t *idp, int n, double scale, int *rowLen, int *rowPtr,
                 int32_t *col, double *val, int *flag, void *scanTmp, size_t scanTmpBytes, int *hostNnz,
                 int *hostSingular, cudaStream_t st);
void LaunchRhs(const LevelView &v, const double *u, const double *vv, const double *w, const double *p, double rhoDt,
               double scale, double dh, double *b, cudaStream_t st);
void LaunchMaxDiv(const LevelView &v, const double *u, const double *vv, const double *w, double dh,
                  const Reducer &R, int slot, cudaStream_t st);
template <typename T>
void LaunchResidual64(const LevelView &v, const double *b, const double *x, T *rOut, double scale, double sfac,
                      const Reducer &R, int slot, cudaStream_t st);
template <typename T>
// swap (may be null): when *swap is odd the kernel reads xout and writes xin (a device-side refinement loop)
void LaunchRefine64(const LevelView &v, const double *b, const double *xin, const T *e, double *xout, T *rOut,
                    double scale, double sfac, const Reducer &R, int slot, cudaStream_t st,
                    const int *swap = nullptr);
enum : int { CELL_DELTA = 0, CELL_RING_DELTA, CELL_NEG, CELL_TAKE, CELL_SUM, CELL_RESTORE };
void LaunchCellwise(const LevelView &v, int op, double *a, const double *b, double *out, cudaStream_t st);
void LaunchSumUnknowns(const LevelView &v, const double *x, const Reducer &R, int slot, cudaStream_t st);
void LaunchSubMeanScatter(const LevelView &v, double *x, const double *sums, int n, int sub, double *p,
                          cudaStream_t st);
void LaunchRing(const LevelView &v, double *p, cudaStream_t st);
void LaunchProject(const LevelView &g, double *u, double *v, double *w, const double *p, double dtOverRho,
                   cudaStream_t st);
void LaunchGather(const LevelView &v, const int32_t *idp, const double *grid, double *compact, cudaStream_t st);
void LaunchScatterVolume(const LevelView &v, const int32_t *idp, const double *compact, double *grid, int volume,
                         cudaStream_t st);

// ---- nb_tail.cu: the coarse end of the V-cycle in one thread block, in shared memory ----
constexpr int kMaxTailLevels = 8;
constexpr size_t kTailMaxSmem = 200 * 1024;
template <typename T> size_t TailSmemBytes(const LevelView *levels, int nlev);
template <typename T> bool PrepareTail(size_t bytes);
// the per-colour lists of the tail levels' unknowns (once per layout): TailListEntries entries, 2 * nlev counts
long long TailListEntries(const LevelView *levels, int nlev);
void LaunchTailLists(const LevelView *levels, int nlev, unsigned *lists, int *counts, cudaStream_t st);
template <typename T>
void LaunchTail(const LevelView *levels, int nlev, const T *rIn, T *eOut, int pre, int post, int coarseSweeps,
                const unsigned *lists, const int *counts, cudaStream_t st);

// the batched coarse end (nb_batch.cu): one request's TailArgs<float> for the batch's table (sizes first with
// out = null), and the launch (grid z = the capacity; smem: the largest request's dynamic shared memory)
void TailArgsFor(const LevelView *levels, int nlev, const float *rIn, float *eOut, int pre, int post,
                 int coarseSweeps, const unsigned *lists, const int *counts, void *out, size_t *bytes, size_t *smem);
void LaunchBatchTail(const BatchReq *rq, BatchList a, int cap, size_t smem, cudaStream_t st);

// ---- nb_pairs.cu: FP32 kernels for 3D levels of a uniform grid with Nz even (cell pairs, unmasked stencil) ----
bool PairLevelShape(const LevelView &v);
void LaunchBuildDu(const LevelView &v, uint8_t *du, cudaStream_t st);
void LaunchPairFirst(const LevelView &v, const uint8_t *du, const float *r, float *e, cudaStream_t st);
void LaunchPairHalf(const LevelView &v, const uint8_t *du, const float *r, float *e, int colour, cudaStream_t st);
// stretched levels: the coefficients from the level's tables, the diagonal from its code (first: red from zero)
void LaunchPairHalfSt(const LevelView &v, const float *r, float *e, int colour, bool first, cudaStream_t st);
void LaunchPairHalfStDot(const LevelView &v, const float *r, float *e, int colour, const Reducer &R, const int *it,
                         int baseEven, int baseOdd, cudaStream_t st);
void LaunchPairResidualSt(const LevelView &v, const float *r, const float *e, float *res, cudaStream_t st);
// the same sweep, also summing (r.z, z, r) into the scalar block of the iteration's parity (k_dot's output)
void LaunchPairHalfDot(const LevelView &v, const uint8_t *du, const float *r, float *e, int colour, const Reducer &R,
                       const int *it, int baseEven, int baseOdd, cudaStream_t st);
void LaunchPairResidual(const LevelView &v, const uint8_t *du, const float *r, const float *e, float *res,
                        cudaStream_t st);
void LaunchPairPApply(const LevelView &v, const uint8_t *du, const float *z, float *p0, float *p1, float *q,
                      const Reducer &R, const double *S, const int *it, int baseEven, int baseOdd, int slotN,
                      int singular, int slotPQ, cudaStream_t st);
void LaunchBuildPext(const LevelView &fine, const LevelView &coarse, uint8_t *pext, cudaStream_t st);
void LaunchPairProlong(const LevelView &fine, const LevelView &coarse, const uint8_t *pext, const float *eCoarse,
                       float *eFine, cudaStream_t st);
void LaunchPairRestrict(const LevelView &fine, const LevelView &coarse, const uint8_t *pext, const float *resFine,
                        float *rCoarse, cudaStream_t st);
// the FP64 refinement step x_out = x_in + e, r = sfac (b - A x_out) on a uniform 3D level 0 (k_residual64's)
void LaunchPairRefine64(const LevelView &v, const uint8_t *du, const double *b, const double *xin, const float *e,
                        double *xout, float *r, double scale, double sfac, const Reducer &R, int slot,
                        cudaStream_t st, const int *swap = nullptr);
void LaunchLinDot(long long cells, const float *r, const float *z, const Reducer &R, const int *it, int baseEven,
                  int baseOdd, cudaStream_t st);
// the same on a colour-split level 0 (v), skipping the tiles its activity marks empty (all tiles without one)
void LaunchSplitLinXR(const LevelView &v, long long vecLen, float *x, float *r, const float *p0, const float *p1,
                      const float *q, const Reducer &R, const double *S, int *it, int baseEven, int baseOdd, int slotN,
                      int singular, int slotPQ, int slotRR, cudaStream_t st);
void LaunchBatchLinXR(const BatchLevel *lv, int ls, const BatchReq *rq, BatchList a, int cap, int baseEven,
                      int baseOdd, int slotN, int slotPQ, int slotRR, cudaStream_t st);
void LaunchLinXR(long long cells, float *x, float *r, const float *p0, const float *p1, const float *q,
                 const Reducer &R, const double *S, int *it, int baseEven, int baseOdd, int slotN, int singular,
                 int slotPQ, int slotRR, cudaStream_t st);

// ---- nb_split.cu: FP32 kernels for 3D levels with Nz even in the colour-split layout (LevelView::sRS) ----
// uniform levels only; du: the level's diagonal units in that layout; pext: the red cells' bytes
// reads the kernels' occupancy (their grids follow it); call before capturing launches into a graph
void PrepareSplitKernels();
// the first red-black sweep from a zero iterate
void LaunchSplitFirst(const LevelView &v, const uint8_t *du, const float *r, float *e, cudaStream_t st);
void LaunchSplitHalf(const LevelView &v, const uint8_t *du, const float *r, float *e, int colour, cudaStream_t st);
// the post-smoothing's last sweep on level 0: the black half (last = false) sums its (r.z, z, r) into
// out[partSlot..], the red half (last = true) adds its own into the scalar block of the iteration's parity
void LaunchSplitHalfDot(const LevelView &v, const uint8_t *du, const float *r, float *e, int colour, bool last,
                        const Reducer &R, const int *it, int baseEven, int baseOdd, int partSlot, cudaStream_t st);
// the red residual after a sweep that ended black (into the first half of res)
void LaunchSplitResidual(const LevelView &v, const uint8_t *du, const float *r, const float *e, float *res,
                         cudaStream_t st);
void LaunchSplitProlong(const LevelView &fine, const LevelView &coarse, const uint8_t *pext, const float *eCoarse,
                        float *eFine, cudaStream_t st);
// mode: 0 by the coarse level's size, 1 one thread per coarse cell, 2 one thread per 4 coarse cells (same result)
void LaunchSplitRestrict(const LevelView &fine, const LevelView &coarse, const uint8_t *pext, const float *resFine,
                         float *rCoarse, int mode, cudaStream_t st);
void LaunchSplitPApply(const LevelView &v, const uint8_t *du, const float *z, float *p0, float *p1, float *q,
                       const Reducer &R, const double *S, const int *it, int baseEven, int baseOdd, int slotN,
                       int singular, int slotPQ, cudaStream_t st);
void LaunchSplitScaleSum(const LevelView &v, const double *b, float *r, double sfac, const Reducer &R, int slot,
                         cudaStream_t st);
// the tiles of a plane of a colour-split level (1024 elements each, the cells one quad-kernel block owns), and the
// activity bytes of every (plane, tile): nonzero where a tile holds an unknown of either colour (LevelView::act)
int SplitActivityTiles(const LevelView &v);
void LaunchSplitActivity(const LevelView &v, const uint8_t *du, uint8_t *act, int tiles, cudaStream_t st);
// the batched forms (nb_batch.cu): kind NB_BK_*; S the march length of the non-reducing kernels; coarse: the next
// coarser level (restriction, prolongation); mode: the restriction's kernel (1 per coarse cell, else per 4)
enum : int { NB_BK_FIRST = 0, NB_BK_HALF, NB_BK_RESIDUAL, NB_BK_RESTRICT, NB_BK_PROLONG, NB_BK_COUNT };
int SplitDefaultS(const LevelView &v, int kind);
void LaunchBatchSplit(int kind, const LevelView &v, const LevelView *coarse, int S, int mode, const BatchLevel *lv,
                      int ls, int l, const BatchReq *rq, BatchList a, int cap, int colour, cudaStream_t st);
void LaunchBatchSplitHalfDot(const LevelView &v, const BatchLevel *lv, int ls, const BatchReq *rq, BatchList a,
                             int cap, int colour, bool last, int baseEven, int baseOdd, int partSlot, cudaStream_t st);
void LaunchBatchSplitPApply(const LevelView &v, const BatchLevel *lv, int ls, const BatchReq *rq, BatchList a,
                            int cap, int baseEven, int baseOdd, int slotN, int slotPQ, cudaStream_t st);
void LaunchBatchSplitScaleSum(const BatchLevel *lv, int ls, const BatchReq *rq, BatchList a, int cap, int slot,
                              cudaStream_t st);
void LaunchBatchSplitRefine64(const LevelView &v, const BatchLevel *lv, int ls, const BatchReq *rq, BatchList a,
                              int cap, const int *parity, int slot, cudaStream_t st);
void LaunchSplitRefine64(const LevelView &v, const uint8_t *du, const double *b, const double *xin, const float *e,
                         double *xout, float *r, double scale, double sfac, const Reducer &R, int slot,
                         cudaStream_t st, const int *swap = nullptr);

// ---- nb_kernels.cu: multigrid and PCG kernels, T = float (inner solve) or double (plain FP64) ----
void LaunchBuildCodes(const LevelView &v, uint8_t *code, cudaStream_t st);
// out[slot] = unknowns, out[slot + 1] = unknowns whose row reaches a Dirichlet value (0: the system is singular)
void LaunchCountUnknowns(const LevelView &v, const Reducer &R, int slot, cudaStream_t st);
void LaunchCoarsenTypes(const LevelView &fine, const LevelView &coarse, uint8_t *coarseTypes, cudaStream_t st);

template <typename T> void LaunchSmoothFirst(const LevelView &v, const T *r, T *e, cudaStream_t st);
template <typename T> void LaunchSmooth(const LevelView &v, const T *r, T *e, int colour, cudaStream_t st);
template <typename T> void LaunchLevelResidual(const LevelView &v, const T *r, const T *e, T *res, cudaStream_t st);
template <typename T>
void LaunchRestrict(const LevelView &fine, const LevelView &coarse, const T *resFine, T *rCoarse, cudaStream_t st);
template <typename T>
void LaunchProlong(const LevelView &fine, const LevelView &coarse, const T *eCoarse, T *eFine, cudaStream_t st);
template <typename T> void LaunchCoarseSolve(const LevelView &v, const T *r, T *e, int sweeps, cudaStream_t st);

// PCG on the unit-form operator M = -A/scale of level 0. A singular (all-Neumann) system removes the mean of the
// preconditioned residual z over the unknowns; its effect on r.z is carried in the scalars, so z itself is not
// rewritten: with S[b..b+2] = (sum r.z, sum z, sum r), rz_eff = S[b] - (S[b+1]/n) S[b+2], n = S[slotN] (the count of
// unknowns, kept on the device).
//   dot:   out[base..base+2] = (sum r.z, sum z, sum r)
//   pupd:  beta = first ? 0 : rz_eff(new)/rz_eff(old); pOut = (z - mean) + beta pIn; q = M pOut;
//          out[slotPQ] = sum pOut.q
//   xr:    alpha = rz_eff/S[pq]; x += alpha p; r -= alpha q; out[slotRR] = sum r.r
// The iteration number lives on the device (*it, advanced by the x,r update's last block), so one captured graph
// serves every iteration: even iterations read p0 and write p1 and use the scalar block baseEven, odd ones the
// other way round; iteration 0 takes beta = 0.
template <typename T>
void LaunchDot(const LevelView &v, const T *r, const T *z, const Reducer &R, const int *it, int baseEven, int baseOdd,
               cudaStream_t st);
template <typename T>
void LaunchUpdatePApply(const LevelView &v, const T *z, T *p0, T *p1, T *q, const Reducer &R, const double *S,
                        const int *it, int baseEven, int baseOdd, int slotN, int singular, int slotPQ, int exact,
                        cudaStream_t st);
template <typename T>
void LaunchUpdateXR(const LevelView &v, T *x, T *r, const T *p0, const T *p1, const T *q, const Reducer &R,
                    const double *S, int *it, int baseEven, int baseOdd, int slotN, int singular, int slotPQ, int slotRR,
                    cudaStream_t st);
// r = sfac * b over all `cells` and out[slot..slot+1] = (sum b^2, sum b): the residual of a zero iterate
template <typename T>
void LaunchScaleSum(long long cells, const double *b, T *r, double sfac, const Reducer &R, int slot, cudaStream_t st);
// y = s * x over the level's unknowns (x and y may alias)
template <typename Tin, typename Tout>
void LaunchScaleCopy(const LevelView &v, const Tin *x, Tout *y, double s, cudaStream_t st);

} // namespace nb
