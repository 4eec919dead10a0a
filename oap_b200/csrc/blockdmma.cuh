// FP64 block operator pass W = A X on the FP64 tensor cores (DMMA,
// mma.sync m16n8k4 f64), stream-K scheduled.
//
// The work of one pass is tiles x kchunks iterations (128 operator rows x 16
// columns each).  A persistent grid of G CTAs (148 x resident CTAs per SM)
// splits that range into G equal contiguous pieces, so every SM gets the same
// number of FP64 MMAs whatever n is.  A CTA that crosses a tile boundary
// writes one partial per tile it touched; k_dmma_reduce sums the partials of
// each tile in CTA order (deterministic).
#pragma once

#include <cuda_runtime.h>

namespace oapb {

struct DmmaPlan {
  int n;
  long tiles, kchunks, total;   // iterations = tiles x kchunks
  int grid;                     // CTAs
  int slots;                    // partial slots per CTA (tiles one CTA can touch)
};

// Plan for an n x n operator; returns false when the DMMA pass does not
// apply (n odd: rows of A are not 16-byte aligned).
bool dmma_plan(int n, DmmaPlan* p);

// Doubles of partial workspace for b <= 32 vectors at either occupancy.
size_t dmma_workspace(const DmmaPlan& p);

// W (planes wr / wi, vector q at offset q n) = A X; X planes likewise.
// Are / Aim / X 16-byte aligned.  ws: dmma_workspace() doubles.  The grid
// is re-planned per launch for the occupancy of the n-tile count.
int launch_block_matvec_dmma(const double* Are, const double* Aim, int n, const double* xr, const double* xi,
                             int b, double* wr, double* wi, const DmmaPlan& p, double* ws, cudaStream_t s);

}  // namespace oapb
