// One pass of a transform run along a strided register (any register but the
// last): the geometry of its columns, its diagonal runs and its four-step
// twiddle.  Shared by the CUDA-core column kernel (kernels_col.cu) and the
// tensor-core one (kernels_tc.cu).
#pragma once

#include "cvdv_internal.cuh"

namespace cvdv {

constexpr int kColThreads = 256;
constexpr int kMaxColOps = 24;
constexpr int kMaxColDiags = 10;

enum ColOpKind : int { kColDft = 0, kColDiag = 1 };

// Pass shapes: the first half of a transform (diagonal runs on the loads, DFT,
// four-step twiddle), a shared middle pass (DFT, runs, DFT, twiddle), the second
// half (DFT, runs on the stores), or a whole run on a short register (the op list).
enum ColKind : int { kColFirst = 0, kColMiddle = 1, kColLast = 2, kColWhole = 3 };

struct ColOp {
  int kind;
  int dir;   // DFT: +1 forward, -1 inverse
  int diag;  // diagonal run: index into ColPass::diag
};

struct ColPass {
  uint64_t nCols;
  int logS;           // inner size S = 2^logS
  int logA;           // log2 of the middle index range of a column's base
  uint64_t midIn, outerIn, axisIn;     // strides (amplitudes) of the input
  uint64_t midOut, outerOut, axisOut;  // strides of the output
  int logN;           // four-step twiddle: multiply point m of column (mid) by w_N^{mid m}
  int logTwN;
  const double2* tw;  // w_{2^logTwN}^e table of the context
  int nOps, nDiag;
  ColOp ops[kMaxColOps];
  // diagonal runs, evaluated at input addresses before the first DFT, output ones
  // after: diag[d] per point, and the run's bilinear terms c x_reg x_other (control
  // bit off the register) lin[d][0..nLin[d]) as a linear phase along the column
  FactorList diag[kMaxColDiags];
  int nLin[kMaxColDiags];
  XXFactor lin[kMaxColDiags][kMaxXX];  // side 1: the other register
  int logQ;            // register length 2^logQ
  double regC, regDx;  // centre and spacing of the register's grid
};

}  // namespace cvdv
