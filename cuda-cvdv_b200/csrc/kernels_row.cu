// Row programs: a run of basis changes and diagonal gates on the contiguous
// (last) register, executed in ONE read + write of the state.
//
// A conditional displacement is FtQ2P . CPhaseX . FtP2Q (src/cuda/gates.cu:163-204);
// the reference spends 9 elementwise passes and two cuFFT transforms on it.
// Here the whole sequence -- pre-twiddle, forward DFT, post-twiddle / scale /
// phase kick / next pre-twiddle, inverse DFT, post-twiddle / scale and any
// following diagonal gates -- runs on a row held on chip.
//
// Tiling.  A CTA of 256 threads holds a tile of 4096 (complex128) or 8192
// (complex64) amplitudes, 16 or 32 per thread, in one shared-memory buffer;
// each Stockham stage gathers its operands into registers, synchronises and
// scatters the results back in place.  Two CTAs fit an SM.  A register of
// N <= tile points is processed as tile/N whole rows per CTA.  A longer row
// runs on "big" CTAs of 512 threads (twice the tile, one CTA per SM) and, past
// that, is split across a thread-block cluster of C = N / tile CTAs (C = 2 or
// 4): CTA c holds the contiguous chunk [c M, (c+1) M), M = N / C, and the DFT
// of the row is one radix-C butterfly across the cluster (operands read from
// the other CTAs' shared memory, DSMEM) plus an M-point DFT inside each CTA:
//   forward  X[k1 + C k2] = sum_m w_M^{m k2} [ w_N^{m k1} sum_j1 w_C^{j1 k1} x[j1 M + m] ]
//            -> CTA k1 holds X[k1 + C k2] at local position k2 ("transposed");
//   inverse  x[j1 M + m]  = sum_k1 w_C^{-j1 k1} w_N^{-m k1} sum_k2 w_M^{-m k2} X[k1 + C k2]
//            -> consumes the transposed layout and returns the natural one,
// so FFT . diag . IFFT never reshuffles data between CTAs.  A program that
// starts with an inverse transform loads straight into the transposed layout,
// and one that ends in it stores from it (CTA k1 writes every C-th element;
// L2 merges the sectors before they reach HBM).  Diagonal tables applied while
// the layout is transposed are built permuted to match.
//
// The M-point DFT runs as Stockham stages of radix 16 (plus one radix-2/4/8
// stage when log2 M is not a multiple of 4).  Twiddles come from two small
// shared-memory tables (w^e = hi[e >> 6] lo[e & 63]) and, inside a butterfly,
// from powers of its base twiddle.  A diagonal run is applied as
//   (per-row scalar) x (combined table of the row register)[ctrl segment][k]
// where the per-row scalar collects every factor that does not depend on the
// row register (qubit phases, other modes) and is computed once per row.

#include <cooperative_groups.h>

#include "cvdv_internal.cuh"
#include "row_fft.cuh"

namespace cg = cooperative_groups;

namespace cvdv {

constexpr int kRowMinLogN = 8;  // shorter registers use the pass kernels

template <typename C> struct RowCfg;
template <> struct RowCfg<double2> {
  static constexpr int LOGE = 4;  // 16 amplitudes per thread
  static constexpr int E = 16;
};
template <> struct RowCfg<float2> {
  static constexpr int LOGE = 5;  // 32 amplitudes per thread
  static constexpr int E = 32;
};

struct RowOp {
  int kind;
  int dir;   // fft: +1 forward, -1 inverse
  int diag;  // diag: index into RowProgram::diag
};

struct RowDiag {
  const double2* tab;  // [2^nCtrl][N] combined factor of the row register, or null
  int permuted;        // tab stored as [seg][rank][m] for k = rank + C m (transposed layout)
  int nCtrl;
  int ctrlShift[2];    // flat-index bits selecting the table segment (row bits)
  int hasRowF, hasElemF;
  FactorList rowF;     // factors constant along a row
  FactorList elemF;    // per-element factors (bilinear terms with the row register)
  // Bilinear terms c x_row x_other (other register and control bit off the row)
  // taken out of elemF for k_rowr: along one row they are the linear phase
  // a (m - regC) regDx with a = sum c x_other (+-1 by the control bit), so a
  // thread needs two sincos per run instead of one per amplitude.  The other
  // register is side 1 of each XXFactor.
  int nLin;
  double regC, regDx;
  XXFactor lin[kMaxXX];
  // k_rowq: a run whose register terms are linear phases (no table): transform
  // twiddles, the sum of their signs s giving exp(i pi s (N-1)(2n-N+1)/(2N)) at
  // point n, and terms c x_n (x_n = (n - regC) regDx), each negated when its
  // control bit (a row bit, or none: -1) is set
  int ftSign;
  int nPl;
  double plC[2];
  int plCtrl[2];
};

struct RowProgram {
  int logN;     // register length
  int logM;     // row elements held by one CTA
  int logRows;  // rows per CTA (cluster size 1 only)
  int nOps;
  int nDiag;
  int logTwN;
  int loadT;    // cluster rows: start transposed (1: from the natural layout, 2: from the blocked one)
  int storeBlocked;  // cluster rows ending transposed: write the blocked layout
  int logS;          // k_rowr on a strided register: log2 of the amplitudes below it (0: rows)
  const double2* tw;
  double* rowSums;        // non-null: per-warp partial sums of |psi|^2 of every row's result
  unsigned int* waitErr;  // set when a bounded wait on the cluster peers gives up
  RowOp ops[kMaxRowOps];
  RowDiag diag[kMaxRowDiags];
};

// ---------------------------------------------------------------- twiddles in smem
// w_L^e = hi[e >> 6] * lo[e & 63] for e < L (L = M for the CTA-local DFT, N for
// the cross-cluster butterfly); forward convention exp(-2 pi i e / L).
struct TwTables {
  double2* loM;
  double2* hiM;
  double2* loN;
  double2* hiN;
};

// One Stockham stage of radix RHO, in place on the single tile buffer: every
// thread gathers its butterflies' operands into registers, the CTA syncs, and
// the results are scattered to their autosorted positions.
template <typename C, int DIR, int RHO, int LOGT>
__device__ __forceinline__ void row_stage(C* sm, int RS, int logM, int logNs, const TwTables& T) {
  constexpr int LOGRHO = RHO == 16 ? 4 : (RHO == 8 ? 3 : (RHO == 4 ? 2 : 1));
  constexpr int NT = 1 << LOGT;
  constexpr int K = RowCfg<C>::E / RHO;  // butterflies per thread
  const int logNbf = logM - LOGRHO;
  const int ns = 1 << logNs;
  const int sc = logM - (logNs + LOGRHO);  // w_{ns RHO}^x = w_M^{x << sc}
  C v[K][RHO];
#pragma unroll
  for (int k = 0; k < K; ++k) {
    int bf = threadIdx.x + k * NT;
    int row = bf >> logNbf;
    int jb = bf & ((1 << logNbf) - 1);
    const C* col = sm + row * RS;
#pragma unroll
    for (int u = 0; u < RHO; ++u) v[k][u] = col[rpad<C>(jb + (u << logNbf))];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) {
    int bf = threadIdx.x + k * NT;
    int row = bf >> logNbf;
    int jb = bf & ((1 << logNbf) - 1);
    int jm = jb & (ns - 1);
    if (jm) {
      // powers w^u of the butterfly's base twiddle as a tree of depth log2(RHO):
      // w^(u + 2^j) = w^u * w^(2^j), so no product waits on more than four others
      C w[RHO];
      w[1] = tw2<C, DIR>(T.loM, T.hiM, jm << sc);
#pragma unroll
      for (int p = 1; p < RHO / 2; p <<= 1) {
        w[2 * p] = cmul(w[p], w[p]);
#pragma unroll
        for (int u = 1; u < p; ++u) w[p + u] = cmul(w[p], w[u]);
      }
#pragma unroll
      for (int u = RHO / 2 + 1; u < RHO; ++u) w[u] = cmul(w[RHO / 2], w[u - RHO / 2]);
#pragma unroll
      for (int u = 1; u < RHO; ++u) v[k][u] = cmul(v[k][u], w[u]);
    }
    bfly<C, DIR, RHO>(v[k]);
    C* out = sm + row * RS;
    int base = ((jb >> logNs) << (logNs + LOGRHO)) + jm;
#pragma unroll
    for (int u = 0; u < RHO; ++u) out[rpad<C>(base + u * ns)] = v[k][u];
  }
  __syncthreads();
}

// M-point DFT of every row segment of the tile
template <typename C, int DIR, int LOGT>
__device__ void local_fft(C* sm, int RS, int logM, const TwTables& T) {
  int logNs = 0, rem = logM;
  while (rem >= 4) {
    row_stage<C, DIR, 16, LOGT>(sm, RS, logM, logNs, T);
    logNs += 4;
    rem -= 4;
  }
  if (rem == 3) row_stage<C, DIR, 8, LOGT>(sm, RS, logM, logNs, T);
  else if (rem == 2) row_stage<C, DIR, 4, LOGT>(sm, RS, logM, logNs, T);
  else if (rem == 1) row_stage<C, DIR, 2, LOGT>(sm, RS, logM, logNs, T);
}

// ---------------------------------------------------------------- cross-CTA steps
// Each cross-CTA step reads the cluster peers' tiles (DSMEM) and overwrites its
// own tile in place, in two halves: all CTAs read half 0, sync, write half 0,
// read half 1 (disjoint positions), sync, write half 1.  Holding only half of a
// thread's outputs keeps the step within 128 registers.
template <typename C, int LOGC, int LOGT, typename F>
__device__ __forceinline__ void cluster_exchange(C* sm, F f) {
  constexpr int NT = 1 << LOGT;
  constexpr int H = RowCfg<C>::E / 2;
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();  // every tile of the cluster is complete
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    C y[H];
#pragma unroll
    for (int k = 0; k < H; ++k) y[k] = f(threadIdx.x + (h * H + k) * NT);
    cl.sync();  // every CTA has read these positions
#pragma unroll
    for (int k = 0; k < H; ++k) sm[rpad<C>(threadIdx.x + (h * H + k) * NT)] = y[k];
  }
  __syncthreads();
}

// forward DIF radix-C butterfly: this CTA produces output k1 = rank at every m
template <typename C, int LOGC, int LOGT>
__device__ void cross_forward(C* sm, const TwTables& T) {
  constexpr int NC = 1 << LOGC;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const C* peer[NC];
#pragma unroll
  for (int j = 0; j < NC; ++j) peer[j] = cl.map_shared_rank(sm, j);
  cluster_exchange<C, LOGC, LOGT>(sm, [=](int m) -> C {
    int p = rpad<C>(m);
    C x[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) x[j] = peer[j][p];
    C acc;  // sum_j1 w_C^{j1 rank} x_j1
    if constexpr (NC == 2) {
      acc = rank ? csub(x[0], x[1]) : cadd(x[0], x[1]);
    } else {
      C s02 = cadd(x[0], x[2]), d02 = csub(x[0], x[2]);
      C s13 = cadd(x[1], x[3]), d13 = rot_mi<C, 1>(csub(x[1], x[3]));
      acc = rank == 0 ? cadd(s02, s13) : rank == 1 ? cadd(d02, d13) : rank == 2 ? csub(s02, s13) : csub(d02, d13);
    }
    int e = m * rank;  // w_N^{m rank}
    return e ? cmul(acc, tw2<C, 1>(T.loN, T.hiN, e)) : acc;
  });
}

// inverse DIT radix-C butterfly: this CTA (rank = j1) produces x[j1 M + m]
template <typename C, int LOGC, int LOGT>
__device__ void cross_inverse(C* sm, const TwTables& T) {
  constexpr int NC = 1 << LOGC;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const C* peer[NC];
#pragma unroll
  for (int j = 0; j < NC; ++j) peer[j] = cl.map_shared_rank(sm, j);
  cluster_exchange<C, LOGC, LOGT>(sm, [=](int m) -> C {
    int p = rpad<C>(m);
    C z[NC];
    z[0] = peer[0][p];
    C w1 = m ? tw2<C, -1>(T.loN, T.hiN, m) : fromd<C>(make_double2(1.0, 0.0));
    C w = w1;  // z_k1 * w_N^{-m k1}
#pragma unroll
    for (int k1 = 1; k1 < NC; ++k1) {
      z[k1] = cmul(peer[k1][p], w);
      if (k1 + 1 < NC) w = cmul(w, w1);
    }
    C acc;  // sum_k1 w_C^{-rank k1} z_k1
    if constexpr (NC == 2) {
      acc = rank ? csub(z[0], z[1]) : cadd(z[0], z[1]);
    } else {
      C s02 = cadd(z[0], z[2]), d02 = csub(z[0], z[2]);
      C s13 = cadd(z[1], z[3]), d13 = rot_mi<C, -1>(csub(z[1], z[3]));
      acc = rank == 0 ? cadd(s02, s13) : rank == 1 ? cadd(d02, d13) : rank == 2 ? csub(s02, s13) : csub(d02, d13);
    }
    return acc;
  });
}

// layout change: natural (CTA j1 holds k = j1 M + m) <-> transposed (CTA k1 holds k = k1 + C m)
template <typename C, int LOGC, int LOGT>
__device__ void redistribute(C* sm, int logM, bool toNatural) {
  // Unlike the butterflies, output position m reads a different position of a
  // sibling, so every read must finish before any CTA writes: one full round.
  constexpr int NC = 1 << LOGC;
  constexpr int NT = 1 << LOGT;
  constexpr int E = RowCfg<C>::E;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  cl.sync();
  C y[E];
#pragma unroll
  for (int k = 0; k < E; ++k) {
    int m = threadIdx.x + k * NT;
    int kk, srcRank, srcPos;
    if (toNatural) {
      kk = (rank << logM) + m;
      srcRank = kk & (NC - 1);
      srcPos = kk >> LOGC;
    } else {
      kk = rank + (m << LOGC);
      srcRank = kk >> logM;
      srcPos = kk & ((1 << logM) - 1);
    }
    y[k] = cl.map_shared_rank(sm, srcRank)[rpad<C>(srcPos)];
  }
  cl.sync();
#pragma unroll
  for (int k = 0; k < E; ++k) sm[rpad<C>(threadIdx.x + k * NT)] = y[k];
  __syncthreads();
}

// ---------------------------------------------------------------- the kernel
// Single-CTA rows run two CTAs per SM (one loads while the other computes);
// cluster rows hold the cross-step operands in registers and get the full file.
template <typename C, int LOGC, int LOGT>
__global__ void __launch_bounds__(1 << LOGT, (LOGC > 0 || LOGT > 8) ? 1 : 2)
    k_row(const C* __restrict__ in, C* __restrict__ out, const __grid_constant__ RowProgram P) {
  constexpr int NT = 1 << LOGT;
  constexpr int E = RowCfg<C>::E;
  constexpr int TILE = NT * E;
  extern __shared__ __align__(16) unsigned char smraw[];
  const int logM = P.logM;
  const int M = 1 << logM;
  const int RS = rpad<C>(M);
  const int rows = 1 << P.logRows;
  C* sm = reinterpret_cast<C*>(smraw);
  double2* twbase = reinterpret_cast<double2*>(sm + RS * rows);
  TwTables T;
  T.loM = twbase;
  T.hiM = T.loM + 64;
  T.loN = T.hiM + 128;
  T.hiN = T.loN + 64;
  double2* rowScalar = T.hiN + 512;  // [rows][nDiag]
  int* rowSeg = reinterpret_cast<int*>(rowScalar + rows * P.nDiag);

  int rank = 0;
  uint64_t base;  // flat index of element 0 of this CTA's first row
  if (LOGC == 0) {
    base = (uint64_t)blockIdx.x * TILE;
  } else {
    rank = (int)cg::this_cluster().block_rank();
    base = ((uint64_t)blockIdx.x >> LOGC) << P.logN;
  }
  const uint64_t chunk = base + ((uint64_t)rank << logM);  // first element held here

  const bool tailDiag = P.nOps > 1 && P.ops[P.nOps - 1].kind == kRowDiag;
  const int opEnd = tailDiag ? P.nOps - 1 : P.nOps;

  // ---- twiddle tables and per-row diagonal scalars
  {
    const int scM = P.logTwN - logM, scN = P.logTwN - P.logN;
    for (int i = threadIdx.x; i < 64 + 128 + 64 + 512; i += NT) {
      double2 w = make_double2(1.0, 0.0);
      if (i < 64) { if (i < M) w = __ldg(P.tw + ((size_t)i << scM)); }
      else if (i < 192) { int h = i - 64; if ((h << 6) < M) w = __ldg(P.tw + ((size_t)(h << 6) << scM)); }
      else if (i < 256) { int l = i - 192; if (LOGC && l < (1 << P.logN)) w = __ldg(P.tw + ((size_t)l << scN)); }
      else { int h = i - 256; if (LOGC && (h << 6) < (1 << P.logN)) w = __ldg(P.tw + ((size_t)(h << 6) << scN)); }
      twbase[i] = w;
    }
    for (int i = threadIdx.x; i < rows * P.nDiag; i += NT) {
      int r = i / P.nDiag, d = i - r * P.nDiag;
      const RowDiag& D = P.diag[d];
      uint64_t rb = base + ((uint64_t)r << P.logN);
      rowScalar[i] = D.hasRowF ? eval_factor(D.rowF, rb) : make_double2(1.0, 0.0);
      int seg = 0;
      for (int c = 0; c < D.nCtrl; ++c) seg |= (int)((rb >> D.ctrlShift[c]) & 1ull) << c;
      rowSeg[i] = seg << P.logN;
    }
  }
  __syncthreads();

  // A program whose first transform is inverse loads the row straight into the
  // transposed layout (stride-C reads; siblings share the sectors through L2).
  bool transposed = LOGC > 0 && P.loadT;
  auto gaddrT = [&](int e) -> uint64_t { return base + (uint64_t)rank + ((uint64_t)e << LOGC); };
  // table entry of diag d for tile element (row, m): the table of an op that
  // runs in the transposed layout is stored permuted, so every read is contiguous
  auto tab_at = [&](int d, int row, int m) -> double2 {
    const RowDiag& D = P.diag[d];
    if (!D.tab) return make_double2(1.0, 0.0);
    int k = LOGC == 0 ? m : (rank << logM) + m;
    return __ldg(D.tab + rowSeg[row * P.nDiag + d] + k);
  };
  auto factor_with = [&](int d, int row, int m, double2 t) -> C {
    const RowDiag& D = P.diag[d];
    double2 f = dmul(rowScalar[row * P.nDiag + d], t);
    if (D.hasElemF) {
      int k = LOGC == 0 ? m : (transposed ? rank + (m << LOGC) : (rank << logM) + m);
      f = dmul(f, eval_factor(D.elemF, base + ((uint64_t)row << P.logN) + (uint64_t)k));
    }
    return fromd<C>(f);
  };

  // ---- load the tile: all E requests in flight per thread
  {
    C v[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
      int e = threadIdx.x + k * NT;
      v[k] = in[transposed ? gaddrT(e) : chunk + e];
    }
#pragma unroll
    for (int k = 0; k < E; ++k) {
      int e = threadIdx.x + k * NT;
      sm[(e >> logM) * RS + rpad<C>(e & (M - 1))] = v[k];
    }
  }
  __syncthreads();

  for (int o = 0; o < opEnd; ++o) {
    const RowOp op = P.ops[o];
    if (op.kind == kRowDiag) {
#pragma unroll 1
      for (int k0 = 0; k0 < E; k0 += 8) {
        double2 t[8];  // 8 table reads in flight before any is used
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          int e = threadIdx.x + (k0 + k) * NT;
          t[k] = tab_at(op.diag, e >> logM, e & (M - 1));
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          int e = threadIdx.x + (k0 + k) * NT;
          int row = e >> logM, m = e & (M - 1);
          C* p = sm + row * RS + rpad<C>(m);
          *p = cmul(*p, factor_with(op.diag, row, m, t[k]));
        }
      }
      __syncthreads();
    } else if (op.dir > 0) {
      if constexpr (LOGC > 0) {
        if (transposed) redistribute<C, LOGC, LOGT>(sm, logM, true);
        cross_forward<C, LOGC, LOGT>(sm, T);
        transposed = true;
      }
      local_fft<C, 1, LOGT>(sm, RS, logM, T);
    } else {
      if constexpr (LOGC > 0) {
        if (!transposed) {
          redistribute<C, LOGC, LOGT>(sm, logM, false);
          transposed = true;
        }
      }
      local_fft<C, -1, LOGT>(sm, RS, logM, T);
      if constexpr (LOGC > 0) {
        cross_inverse<C, LOGC, LOGT>(sm, T);
        transposed = false;
      }
    }
  }
  // ---- store (trailing diagonal run applied on the way out).  A row that ends
  // transposed is written in place with stride C: the sectors this CTA leaves
  // half-written are completed by its cluster siblings in L2.
  const bool storeT = LOGC > 0 && transposed;
  if (tailDiag) {
    const int dd = P.ops[P.nOps - 1].diag;
#pragma unroll 1
    for (int k0 = 0; k0 < E; k0 += 8) {
      double2 t[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        int e = threadIdx.x + (k0 + k) * NT;
        t[k] = tab_at(dd, e >> logM, e & (M - 1));
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        int e = threadIdx.x + (k0 + k) * NT;
        int row = e >> logM, m = e & (M - 1);
        out[storeT ? gaddrT(e) : chunk + e] = cmul(sm[row * RS + rpad<C>(m)], factor_with(dd, row, m, t[k]));
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < E; ++k) {
      int e = threadIdx.x + k * NT;
      out[storeT ? gaddrT(e) : chunk + e] = sm[(e >> logM) * RS + rpad<C>(e & (M - 1))];
    }
  }
  if constexpr (LOGC > 0) cg::this_cluster().sync();  // no CTA leaves while peers may read it
}

// ---------------------------------------------------------------- register-resident rows
// Rows that fit one CTA (up to 2^13 complex128 / 2^14 complex64 points) run in
// k_rowr: each thread keeps E = 16 (or 32) amplitudes of one row in registers
// for the whole program -- elements t + TPR v (v < E) of its row, TPR = M / E
// threads per row.  A Stockham stage of radix R gives thread t the butterflies
// j = t + b TPR (b < E/R); their inputs j + u M/R are exactly the thread's E
// elements (register b + (E/R) u), and the last stage's outputs land on the same
// positions.  So the global load, the store and every diagonal run between
// transforms work on registers in place; only the stages inside a transform
// exchange data, through one padded shared-memory row.  Row length, radices and
// strides are template constants, so every shared-memory address is a
// per-thread base plus an immediate offset.

// exp(i pi s (N-1)(2n-N+1)/(2N)) with the angle reduced exactly in integers, and
// its ratio between n + d and n, exp(i pi s (N-1) d / N)
__device__ __forceinline__ double2 ft_tw_at(long long n, long long N, int s) {
  long long m = ((N - 1) * (2 * n - N + 1) * s) % (4 * N);
  if (m < 0) m += 4 * N;
  double sn, c;
  sincospi((double)m / (double)(2 * N), &sn, &c);
  return make_double2(c, sn);
}
__device__ __forceinline__ double2 ft_tw_ratio(long long d, long long N, int s) {
  long long m = ((N - 1) * d * s) % (2 * N);
  if (m < 0) m += 2 * N;
  double sn, c;
  sincospi((double)m / (double)N, &sn, &c);
  return make_double2(c, sn);
}

template <typename C, int LOGM, int LOGE>
__device__ __forceinline__ void rr_diag(C (&v)[1 << LOGE], const RowDiag& D, uint64_t rowBase, int t) {
  constexpr int E = 1 << LOGE, TPR = 1 << (LOGM - LOGE);
  const double2 rs = D.hasRowF ? eval_factor(D.rowF, rowBase) : make_double2(1.0, 0.0);
  // running factor of element t + k TPR: rs times the linear phase, advanced by st per k
  double2 f = rs, st = make_double2(1.0, 0.0);
  const bool lin = D.nLin || D.nPl || D.ftSign;
  if (lin) {
    // bilinear terms with other registers and c x terms (controls off the row) are
    // one linear phase a (m - regC) regDx along the row; the transform twiddle is
    // exact at the first point and as a ratio per step
    double a = 0.0;
    for (int l = 0; l < D.nLin; ++l) {
      const XXFactor& X = D.lin[l];
      const int j = (int)((rowBase >> X.shift1) & (uint64_t)X.mask1);
      double c = X.coeff * (((double)j - X.c1) * X.dx1);
      if (X.ctrlShift >= 0 && ((rowBase >> X.ctrlShift) & 1ull)) c = -c;
      a += c;
    }
    for (int k = 0; k < D.nPl; ++k)
      a += (D.plCtrl[k] >= 0 && ((rowBase >> D.plCtrl[k]) & 1ull)) ? -D.plC[k] : D.plC[k];
    a *= D.regDx;
    double s0, c0;
    sincos(a * ((double)t - D.regC), &s0, &c0);
    sincos(a * (double)TPR, &st.y, &st.x);
    f = dmul(rs, make_double2(c0, s0));
    if (D.ftSign) {
      f = dmul(f, ft_tw_at(t, 1ll << LOGM, D.ftSign));
      st = dmul(st, ft_tw_ratio(TPR, 1ll << LOGM, D.ftSign));
    }
  }
  if (D.tab) {
    int seg = 0;
    for (int c = 0; c < D.nCtrl; ++c) seg |= (int)((rowBase >> D.ctrlShift[c]) & 1ull) << c;
    const double2* tp = D.tab + ((size_t)seg << LOGM) + t;
#pragma unroll
    for (int k0 = 0; k0 < E; k0 += 8) {
      double2 w[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) w[k] = __ldg(tp + (k0 + k) * TPR);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (D.hasRowF || lin) w[k] = dmul(w[k], f);
        if (lin) f = dmul(f, st);
        v[k0 + k] = cmul(v[k0 + k], fromd<C>(w[k]));
      }
    }
  } else if (lin) {
#pragma unroll
    for (int k = 0; k < E; ++k) {
      v[k] = cmul(v[k], fromd<C>(f));
      f = dmul(f, st);
    }
  } else if (D.hasRowF) {
    const C c = fromd<C>(rs);
#pragma unroll
    for (int k = 0; k < E; ++k) v[k] = cmul(v[k], c);
  }
}

// 256-thread CTAs run two per SM; 512- and 1024-thread CTAs one
// Ask L2 to fetch [p, p + bytes) ahead of use: bulk prefetches of 16 KB, one per
// lane of the first warp (bytes a multiple of 16 KB, at most 32 x 16 KB).
__device__ __forceinline__ void l2_prefetch_tile(const void* p, uint32_t bytes) {
  const uint32_t chunk = 16384;
  const uint32_t i = threadIdx.x;
  if (i < bytes / chunk) {
    const char* a = static_cast<const char*>(p) + (size_t)i * chunk;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(chunk) : "memory");
  }
}

// Tiles of one CTA per SM (more than 256 threads) run persistent: each CTA walks
// tiles blockIdx.x, + gridDim.x, ... and asks L2 for its next tile before working
// on the current one, so the next load finds its data on chip while this tile's
// butterflies run.  Smaller tiles run two CTAs per SM, which already overlap one
// CTA's loads with the other's work; they get one tile per CTA.
//
// With COL the "rows" are the columns of a strided register (P.logS amplitudes
// below it): column c is inner index c mod S and outer index c / S, and element m
// sits m S amplitudes after its first.  The CTA's 2^LOGR columns (at least two
// within 512 threads) are adjacent inner indices interleaved lane by lane, so a
// warp's load covers runs of 2^LOGR amplitudes; the rest of each sector is read
// from L2 by the CTAs of the neighbouring columns.
// The sum of |psi|^2 (FP64) over the E amplitudes of each of a group of W lanes
// (W = 32, or the lanes of one row when a warp holds several), written by the
// group's first lane.
template <typename C, int E, int W>
__device__ __forceinline__ void row_sum_part(const C (&v)[E], double* out) {
  double a = 0.0;
#pragma unroll
  for (int k = 0; k < E; ++k) a += (double)v[k].x * (double)v[k].x + (double)v[k].y * (double)v[k].y;
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if ((threadIdx.x & (W - 1)) == 0) *out = a;
}

template <typename C, int LOGM, int LOGR, int LOGE, bool COL>
__global__ void __launch_bounds__(1 << (LOGM - LOGE + LOGR), (LOGM - LOGE + LOGR) > 8 ? 1 : 2)
    k_rowr(const C* __restrict__ in, C* __restrict__ out, uint64_t nTiles, const __grid_constant__ RowProgram P) {
  constexpr int E = 1 << LOGE, M = 1 << LOGM, TPR = M >> LOGE, NT = TPR << LOGR, RS = M + (M >> 4);
  constexpr uint32_t TILE_BYTES = (uint32_t)sizeof(C) << (LOGM + LOGR);
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  double2* lo = reinterpret_cast<double2*>(sm + (RS << LOGR));  // w_M^e, e < 64
  double2* hi = lo + 64;                                         // w_M^(64 h), h < M / 64
  const int tid = threadIdx.x;
  // column form: the CTA's 2^LOGR adjacent columns interleave lane by lane, so a
  // warp's load covers 32 / 2^LOGR points of every column in runs of 2^LOGR
  const int row = COL ? (tid & ((1 << LOGR) - 1)) : tid >> (LOGM - LOGE);
  const int t = COL ? (tid >> LOGR) : tid & (TPR - 1);
  C* smrow = sm + row * RS;
  const int logS = COL ? P.logS : 0;

  const int scM = P.logTwN - LOGM;
  for (int i = tid; i < 64 + (M >> 6); i += NT) {
    const int e = i < 64 ? i : (i - 64) << 6;
    lo[i] = __ldg(P.tw + ((size_t)e << scM));  // lo and hi are one array
  }
  __syncthreads();
  // No barrier between tiles: after a transform's last exchange (which ends in a
  // barrier) a thread touches shared memory again only in the next tile's first
  // exchange, and every thread has left the old tile's exchanges by then.
  for (uint64_t tile = blockIdx.x; tile < nTiles; tile += gridDim.x) {
    uint64_t rowBase;
    if constexpr (COL) {
      const uint64_t c = (tile << LOGR) + (uint64_t)row;
      rowBase = (c & ((1ull << logS) - 1)) + ((c >> logS) << (LOGM + logS));
    } else {
      if (NT > 256 && tile + gridDim.x < nTiles)
        l2_prefetch_tile(in + ((tile + gridDim.x) << (LOGM + LOGR)), TILE_BYTES);
      rowBase = (tile << (LOGM + LOGR)) + ((uint64_t)row << LOGM);
    }
    C v[E];
#pragma unroll
    for (int k = 0; k < E; ++k) v[k] = in[rowBase + ((uint64_t)(t + k * TPR) << logS)];
    for (int o = 0; o < P.nOps; ++o) {
      const RowOp& op = P.ops[o];
      if (op.kind == kRowDiag) rr_diag<C, LOGM, LOGE>(v, P.diag[op.diag], rowBase, t);
      else if (op.dir > 0) rr_stages<C, 1, LOGM, 0, LOGE>(v, smrow, t, lo, hi);
      else rr_stages<C, -1, LOGM, 0, LOGE>(v, smrow, t, lo, hi);
    }
    if constexpr (!COL) {
      // the row's |psi|^2 in TPR / 32 partials (one when a warp holds several rows)
      constexpr int W = TPR < 32 ? TPR : 32, PARTS = TPR < 32 ? 1 : TPR / 32;
      if (P.rowSums) row_sum_part<C, E, W>(v, P.rowSums + (rowBase >> LOGM) * PARTS + t / 32);
    }
#pragma unroll
    for (int k = 0; k < E; ++k) out[rowBase + ((uint64_t)(t + k * TPR) << logS)] = v[k];
  }
}

// largest row k_rowr takes (one CTA: 2^13 complex128 / 2^14 complex64 points)
static int rowr_max_log(int precision) { return precision == kC128 ? 13 : 14; }

// complex64 rows of 2^13 and 2^14 points keep 32 amplitudes per thread (256 / 512
// threads); everything else 16
template <typename C, int LOGM>
struct RrShape {
  static constexpr int LOGE = (sizeof(C) == sizeof(float2) && LOGM >= 13) ? 5 : 4;
  static constexpr int LOGR = LOGM - LOGE < 8 ? 8 - (LOGM - LOGE) : 0;
};

template <typename C, int LOGM, bool COL>
static cudaError_t launch_rowr_t(Context* ctx, const RowProgram& P) {
  constexpr int LOGE = RrShape<C, LOGM>::LOGE, LOGR0 = RrShape<C, LOGM>::LOGR;
  // column form: at least two columns a CTA while it stays within 512 threads
  constexpr int LOGR = (COL && LOGR0 == 0 && (LOGM - LOGE) < 9) ? 1 : LOGR0;
  constexpr int NT = 1 << (LOGM - LOGE + LOGR);
  constexpr int M = 1 << LOGM;
  const size_t smem = (size_t)(M + (M >> 4)) * (1 << LOGR) * sizeof(C) + (64 + (M >> 6)) * sizeof(double2);
  auto kern = k_rowr<C, LOGM, LOGR, LOGE, COL>;
  static int resident = 0;  // CTAs per SM of this instantiation, asked once
  cudaError_t e = cudaSuccess;
  if (!resident) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, kern, NT, smem);
    if (e != cudaSuccess || resident < 1) return e != cudaSuccess ? e : cudaErrorInvalidConfiguration;
  }
  const uint64_t nTiles = ctx->size() >> (LOGM + LOGR);
  uint64_t grid = NT > 256 ? (uint64_t)ctx->numSMs * resident : nTiles;
  if (grid > nTiles) grid = nTiles;
  kern<<<(unsigned)grid, NT, smem, ctx->stream>>>((const C*)ctx->state(), (C*)ctx->other(), nTiles, P);
  return cudaGetLastError();
}

template <typename C, bool COL>
static cudaError_t launch_rowr(Context* ctx, const RowProgram& P, int q) {
  switch (q) {
    case 8: return launch_rowr_t<C, 8, COL>(ctx, P);
    case 9: return launch_rowr_t<C, 9, COL>(ctx, P);
    case 10: return launch_rowr_t<C, 10, COL>(ctx, P);
    case 11: return launch_rowr_t<C, 11, COL>(ctx, P);
    case 12: return launch_rowr_t<C, 12, COL>(ctx, P);
    case 13: return launch_rowr_t<C, 13, COL>(ctx, P);
    default:
      if constexpr (sizeof(C) == sizeof(float2)) return launch_rowr_t<C, 14, COL>(ctx, P);
      return cudaErrorInvalidValue;
  }
}

// A program on a register that is not the last one runs on k_rowr in column
// form for registers of 2^9 .. 2^14 (complex64) or 2^13 (complex128) points, at
// least as many columns as one CTA takes.  The column loads are strided, but one
// pass replaces the two per transform of the column kernel (with the linear-phase
// runs taken without tables this also wins in complex128: 5.1 against 5.7 ms of
// column work per [13, 13] layer); registers of up to 2^8 points run whole on the
// column kernel anyway.
bool col_program_ok(Context* ctx, int reg) {
  const int q = ctx->q[reg];
  if (!ctx->colProg || ctx->flw[reg] == 0 || q <= 8 ||
      q > rowr_max_log(ctx->precision))
    return false;
  if (ctx->colFft && col_fft_ok(ctx, reg) && tc_col_ok(ctx, reg)) return false;  // chained tensor-core passes
  const int logE = (ctx->precision == kC64 && q >= 13) ? 5 : 4;
  const int logR = q - logE < 8 ? 8 - (q - logE) : (q - logE < 9 ? 1 : 0);
  return ctx->totalQbt - q >= logR;
}

// ---------------------------------------------------------------- cluster register-resident rows
// A row of N = C M points is split over a cluster of C CTAs of M / 16 threads
// (2^14-point complex128 rows: C = 8, 2048 points and 128 threads per CTA, 38 KB
// of shared memory, so CTAs of four clusters share an SM and the rows' loads,
// exchanges and butterflies overlap).  Every thread keeps 16 amplitudes in
// registers.  With I = 16 / C, Q = M / C and m_i = r Q + t + TPR i for thread t
// of CTA r (i < I), two layouts occur:
//   S ("strips"):     v[I j1 + i] = x[j1 M + m_i]   (CTA r holds part r of each
//                     C-th of the row: coalesced loads and stores)
//   T ("transposed"): v[w] = X[r + C k2] at k2 = t + TPR w   (w < 16)
// Forward, S -> T: radix-C butterflies over j1 in registers give
//   y_k1[m_i] = w_N^{m_i k1} sum_j1 w_C^{j1 k1} x[j1 M + m_i];
//   thread t hands y_k1[m_i] (k1 != r) to thread t of CTA k1, after which every
//   thread holds y_r[t + TPR k] for all 16 k, and an M-point DFT of y_r gives
//   X[r + C k2] in the natural Stockham order.
// Inverse, T -> S: an M-point inverse DFT gives z_r[m] at m = t + TPR w; thread t
//   hands z_r[m] for CTA q's part (w = I q + i) to thread t of CTA q, then
//   x[j1 M + m_i] = sum_k1 w_C^{-j1 k1} w_N^{-m_i k1} z_k1[m_i]   (radix C again).
// So each transform moves 16 - I of a thread's 16 amplitudes once, and only
// between threads of the same index: the sender writes them straight into the
// receiving CTA's shared memory (slot (I src + i) TPR + t); the I it keeps never
// leave its registers.  Diagonal runs in T read tables stored permuted for C CTAs
// (position r M + k2 holds index r + C k2).
// XX: the run may hold bilinear terms (D.nLin); programs without them use the
// instantiation that has no code for them.
template <typename C, int LOGM, int LOGC, bool XX>
__device__ __forceinline__ void rq_diag(C (&v)[16], const RowDiag& D, uint64_t rowBase, int t, int r,
                                        bool layoutT) {
  constexpr int M = 1 << LOGM, TPR = M / 16, IPS = 16 >> LOGC, Q = M >> LOGC, NC = 1 << LOGC;
  constexpr long long N = (long long)M << LOGC;
  const double2 rs = D.hasRowF ? eval_factor(D.rowF, rowBase) : make_double2(1.0, 0.0);
  const bool lin = D.ftSign || D.nPl || (XX && D.nLin);
  if (lin) {
    // linear phases as running products from values at a thread's first point (a
    // thread's points are arithmetic progressions in n): T holds
    // n = r + C (t + TPR w), S holds n = j1 M + r Q + t + TPR i at v[I j1 + i].
    // The transform twiddle's values are exact (integer-reduced angles); c x terms
    // and bilinear terms with other registers add to one coefficient of x.
    double c = 0.0;
    for (int k = 0; k < D.nPl; ++k)
      c += (D.plCtrl[k] >= 0 && ((rowBase >> D.plCtrl[k]) & 1ull)) ? -D.plC[k] : D.plC[k];
    if constexpr (XX)
      for (int l = 0; l < D.nLin; ++l) {
        const XXFactor& X = D.lin[l];
        const int j = (int)((rowBase >> X.shift1) & (uint64_t)X.mask1);
        double cc = X.coeff * (((double)j - X.c1) * X.dx1);
        if (X.ctrlShift >= 0 && ((rowBase >> X.ctrlShift) & 1ull)) cc = -cc;
        c += cc;
      }
    c *= D.regDx;
    auto at = [&](long long n) {
      double2 f = D.ftSign ? ft_tw_at(n, N, D.ftSign) : make_double2(1.0, 0.0);
      if (c != 0.0) {
        double sn, cs;
        sincos(c * ((double)n - D.regC), &sn, &cs);
        f = dmul(f, make_double2(cs, sn));
      }
      return f;
    };
    auto ratio = [&](long long d) {
      double2 f = D.ftSign ? ft_tw_ratio(d, N, D.ftSign) : make_double2(1.0, 0.0);
      if (c != 0.0) {
        double sn, cs;
        sincos(c * (double)d, &sn, &cs);
        f = dmul(f, make_double2(cs, sn));
      }
      return f;
    };
    if (layoutT) {
      double2 f = dmul(at(r + NC * t), rs);
      const double2 st = ratio((long long)NC * TPR);
#pragma unroll
      for (int w = 0; w < 16; ++w) {
        v[w] = cmul(v[w], fromd<C>(f));
        f = dmul(f, st);
      }
    } else {
      double2 f = dmul(at(r * Q + t), rs);
      const double2 si = ratio(TPR), sj = ratio(M);
#pragma unroll
      for (int j1 = 0; j1 < NC; ++j1) {
        double2 g = f;
#pragma unroll
        for (int i = 0; i < IPS; ++i) {
          v[IPS * j1 + i] = cmul(v[IPS * j1 + i], fromd<C>(g));
          g = dmul(g, si);
        }
        f = dmul(f, sj);
      }
    }
    if constexpr (!XX) return;  // (without bilinear terms a run is linear or tabled)
  }
  if (D.tab) {
    int seg = 0;
    for (int c = 0; c < D.nCtrl; ++c) seg |= (int)((rowBase >> D.ctrlShift[c]) & 1ull) << c;
    const double2* tp = D.tab + ((size_t)seg << (LOGM + LOGC));
    // T: permuted table at r M + k2; S: natural index j1 M + r Q + t + TPR i
    const double2* base = layoutT ? tp + r * M + t : tp + r * Q + t;
#pragma unroll
    for (int k0 = 0; k0 < 16; k0 += 8) {
      double2 w[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int kk = k0 + k;
        w[k] = __ldg(base + (layoutT ? TPR * kk : (kk / IPS) * M + TPR * (kk % IPS)));
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        if (D.hasRowF && !(XX && lin)) w[k] = dmul(w[k], rs);  // (a linear pass carried rs)
        v[k0 + k] = cmul(v[k0 + k], fromd<C>(w[k]));
      }
    }
  } else if (D.hasRowF && !(XX && lin)) {
    const C c = fromd<C>(rs);
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = cmul(v[k], c);
  }
}

// ---- cluster primitives (distributed shared memory pushed by st.async)
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ uint32_t cluster_map(uint32_t a, int rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(rank));
  return r;
}
__device__ __forceinline__ void cluster_arrive_release() {
  asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory");
}
__device__ __forceinline__ void cluster_wait_acquire() {
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void mbar_init(uint32_t bar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void st_async(uint32_t addr, double2 v, uint32_t bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f64 [%0], {%1, %2}, [%3];" ::"r"(addr),
               "d"(v.x), "d"(v.y), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void st_async(uint32_t addr, float2 v, uint32_t bar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];" ::"r"(addr),
               "f"(v.x), "f"(v.y), "r"(bar)
               : "memory");
}

// Bounded wait for the phase `parity` of a local mbarrier.  A wait that gives up
// (a peer that never delivers: a fault elsewhere) records it in *err and returns,
// so the kernel still reaches its cluster barriers and ends.
__device__ __forceinline__ void mbar_wait_bounded(uint32_t bar, uint32_t parity, unsigned int* err) {
  for (uint32_t it = 0; it < (1u << 22); ++it)
    if (mbar_try_wait(bar, parity)) return;
  if (err) atomicOr(err, 1u);
}

// Thread t hands its amplitudes v[I q + i] (q != r, i < I = 16 / C) to thread t of
// CTA q, slot (I r + i) TPR + t of that CTA's buffer, and takes v[I q + i] from
// slot (I q + i) TPR + t of its own, which thread t of CTA q wrote.  The writes
// are st.async into the peer's shared memory, each completing 16 (complex128) or
// 8 bytes on the peer's mbarrier, which expects (16 - I) TPR amplitudes per
// exchange; so a CTA waits only for its own data, with no cluster-wide barrier or
// fence.  The caller has arrived on the cluster barrier once its buffer was free
// (at start, or after its last local use); the wait here orders the remote writes
// after every peer's arrival.
template <typename C, int TPR, int LOGC>
__device__ __forceinline__ void rq_exchange(C (&v)[16], C* buf, uint32_t bar, uint32_t& parity, int t, int r,
                                            const uint32_t* peerBuf, const uint32_t* peerBar, unsigned int* err) {
  constexpr int NC = 1 << LOGC, IPS = 16 >> LOGC;
  if (t == 0) mbar_expect_tx(bar, (uint32_t)((16 - IPS) * TPR * sizeof(C)));
  cluster_wait_acquire();
#pragma unroll
  for (int q = 0; q < NC; ++q) {
    if (q == r) continue;
    const uint32_t dst = peerBuf[q], dbar = peerBar[q];  // the peer's buffer and mbarrier
#pragma unroll
    for (int i = 0; i < IPS; ++i)
      st_async(dst + (uint32_t)(((IPS * r + i) * TPR + t) * sizeof(C)), v[IPS * q + i], dbar);
  }
  mbar_wait_bounded(bar, parity, err);
  parity ^= 1u;
#pragma unroll
  for (int k = 0; k < 16; ++k)
    if (k / IPS != r) v[k] = buf[k * TPR + t];
  __syncthreads();  // every thread has read its slots before the buffer is reused
}

// radix-C butterfly across the cluster at point i of every strip: forward
// y_k1 = w_N^{m k1} sum_j1 w_C^{j1 k1} x_j1, inverse x_j1 = sum_k1 w_C^{-j1 k1} w_N^{-m k1} z_k1
template <typename C, int DIR, int LOGC>
__device__ __forceinline__ void rq_cross(C (&v)[16], int i, const double2* loN, const double2* hiN, int m) {
  constexpr int NC = 1 << LOGC, IPS = 16 >> LOGC;
  C a[NC], w[NC];
  w[0] = mk((decltype(v[0].x))1, (decltype(v[0].x))0);
  w[1] = tw2<C, DIR>(loN, hiN, m);
#pragma unroll
  for (int k = 2; k < NC; ++k) w[k] = cmul(w[k >> 1], w[k - (k >> 1)]);
#pragma unroll
  for (int j = 0; j < NC; ++j) a[j] = DIR > 0 ? v[IPS * j + i] : cmul(v[IPS * j + i], w[j]);
  if constexpr (NC == 4) bf4<C, DIR>(a[0], a[1], a[2], a[3]);
  else if constexpr (NC == 8) bf8<C, DIR>(a);
  else bf16<C, DIR>(a);
#pragma unroll
  for (int j = 0; j < NC; ++j) v[IPS * j + i] = DIR > 0 ? cmul(a[j], w[j]) : a[j];
}

template <typename C, int LOGN, int LOGC, bool XX>
__global__ void __launch_bounds__(1 << (LOGN - LOGC - 4), 1 << (LOGC - 1))
    k_rowq(const C* __restrict__ in, C* __restrict__ out, uint64_t nRows, const __grid_constant__ RowProgram P) {
  constexpr int LOGM = LOGN - LOGC, M = 1 << LOGM, TPR = M / 16, NC = 1 << LOGC, IPS = 16 >> LOGC, Q = M >> LOGC;
  constexpr int RS = M + (M >> 4);
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  double2* loM = reinterpret_cast<double2*>(sm + RS);  // w_M^e, e < 64
  double2* hiM = loM + 64;                              // w_M^(64 h), h < M / 64
  double2* loN = hiM + (M >> 6);                        // w_N^e, e < 64
  double2* hiN = loN + 64;                              // w_N^(64 h), h < M / 64
  __shared__ __align__(8) uint64_t xbar;  // completes when the peers' (16 - I) TPR amplitudes have landed
  cg::cluster_group cl = cg::this_cluster();
  const int r = (int)cl.block_rank();
  const int t = threadIdx.x;
  const uint32_t bar = smem_addr(&xbar);
  uint32_t parity = 0;
  // the peers' buffer and mbarrier addresses in the cluster window, mapped once
  __shared__ uint32_t peerBuf[NC], peerBar[NC];
  if (t == 0) mbar_init(bar, 1);
  if (t < NC) {
    peerBuf[t] = cluster_map(smem_addr(sm), t);
    peerBar[t] = cluster_map(bar, t);
  }
  {
    const int scM = P.logTwN - LOGM, scN = P.logTwN - LOGN;
    constexpr int NTAB = 2 * (64 + (M >> 6));
    for (int i = t; i < NTAB; i += TPR) {
      const int half = i >= NTAB / 2, j = half ? i - NTAB / 2 : i;
      const int e = j < 64 ? j : (j - 64) << 6;
      loM[i] = __ldg(P.tw + ((size_t)e << (half ? scN : scM)));  // loM..hiN are one array
    }
  }
  __syncthreads();  // mbarrier and twiddle tables
  // A CTA arrives on the cluster barrier when its buffer is free (and, the first
  // time, its mbarrier set up); each exchange waits for every CTA's arrival before
  // writing into the peers.  A program that starts with a forward transform
  // arrives at the start of each row, so the wait comes after the loads and
  // butterflies; one that starts with an inverse transform uses its buffer for
  // the local stages first and arrives after them.
  bool fwdFirst = false;
  for (int o = 0; o < P.nOps; ++o)
    if (P.ops[o].kind != kRowDiag) {
      fwdFirst = P.ops[o].dir > 0;
      break;
    }
  // persistent clusters: cluster c takes rows c, c + nClusters, ...
  const uint64_t nClusters = gridDim.x >> LOGC;
  for (uint64_t row = blockIdx.x >> LOGC; row < nRows; row += nClusters) {
    const uint64_t rowBase = row << LOGN;
    bool arrived = fwdFirst;
    if (arrived) cluster_arrive_release();
    C v[16];
    bool layoutT = P.loadT != 0;
    if (P.loadT == 2) {  // blocked: X[r + C k2] contiguous at r M + k2
#pragma unroll
      for (int w = 0; w < 16; ++w) v[w] = in[rowBase + (uint64_t)r * M + t + TPR * w];
    } else if (P.loadT == 1) {  // transposed from the natural layout (every C-th element)
#pragma unroll
      for (int w = 0; w < 16; ++w) v[w] = in[rowBase + r + NC * (uint64_t)(t + TPR * w)];
    } else {
#pragma unroll
      for (int k = 0; k < 16; ++k) v[k] = in[rowBase + (uint64_t)(k / IPS) * M + r * Q + t + TPR * (k % IPS)];
    }

    for (int o = 0; o < P.nOps; ++o) {
      const RowOp& op = P.ops[o];
      if (op.kind == kRowDiag) {
        rq_diag<C, LOGM, LOGC, XX>(v, P.diag[op.diag], rowBase, t, r, layoutT);
      } else if (op.dir > 0) {  // S -> T
#pragma unroll
        for (int i = 0; i < IPS; ++i) rq_cross<C, 1, LOGC>(v, i, loN, hiN, r * Q + t + TPR * i);
        if (!arrived) cluster_arrive_release();  // this CTA is done with its buffer
        rq_exchange<C, TPR, LOGC>(v, sm, bar, parity, t, r, peerBuf, peerBar, P.waitErr);
        arrived = false;
        rr_stages<C, 1, LOGM, 0, 4>(v, sm, t, loM, hiM);
        layoutT = true;
      } else {  // T -> S
        // the buffer is free once the stages' last exchange is read: arrive there,
        // so the last stage's butterflies overlap the peers' progress
        if (!arrived) {
          struct Arrive {
            __device__ __forceinline__ void operator()() const { cluster_arrive_release(); }
          };
          rr_stages<C, -1, LOGM, 0, 4, Arrive>(v, sm, t, loM, hiM, Arrive());
        } else {
          rr_stages<C, -1, LOGM, 0, 4>(v, sm, t, loM, hiM);
        }
        rq_exchange<C, TPR, LOGC>(v, sm, bar, parity, t, r, peerBuf, peerBar, P.waitErr);
        arrived = false;
#pragma unroll
        for (int i = 0; i < IPS; ++i) rq_cross<C, -1, LOGC>(v, i, loN, hiN, r * Q + t + TPR * i);
        layoutT = false;
      }
    }

    if (arrived) cluster_wait_acquire();  // pair an arrival no exchange waited for
    // the row's |psi|^2 in C * TPR / 32 partials (one per warp of the cluster)
    if (P.rowSums) row_sum_part<C, 16, 32>(v, P.rowSums + row * (NC * TPR / 32) + r * (TPR / 32) + t / 32);
    if (!layoutT) {
#pragma unroll
      for (int k = 0; k < 16; ++k) out[rowBase + (uint64_t)(k / IPS) * M + r * Q + t + TPR * (k % IPS)] = v[k];
    } else if (P.storeBlocked) {
#pragma unroll
      for (int w = 0; w < 16; ++w) out[rowBase + (uint64_t)r * M + t + TPR * w] = v[w];
    } else {
#pragma unroll
      for (int w = 0; w < 16; ++w) out[rowBase + r + NC * (uint64_t)(t + TPR * w)] = v[w];
    }
    // The next row's first arrival says this CTA's buffer is free again: the last
    // reads of it (the last exchange or stage) ended in a CTA barrier.
  }
}
template <typename C, int LOGN, int LOGC, bool XX>
static cudaError_t launch_rowq_t(Context* ctx, const RowProgram& P) {
  constexpr int M = 1 << (LOGN - LOGC), NC = 1 << LOGC;
  const size_t smem = (size_t)(M + (M >> 4)) * sizeof(C) + 2 * (64 + (M >> 6)) * sizeof(double2);
  auto kern = k_rowq<C, LOGN, LOGC, XX>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e == cudaSuccess && NC > 8) e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  const uint64_t nRows = ctx->size() >> LOGN;
  cudaLaunchConfig_t cfg{};
  cfg.blockDim = dim3(M / 16);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = NC;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // as many clusters as are resident at once (asked once per device), each
  // walking its share of the rows
  static int clusters[64] = {};
  const int dev = ctx->device >= 0 && ctx->device < 64 ? ctx->device : 0;
  if (!clusters[dev]) {
    cfg.gridDim = dim3((unsigned)(NC * 1024));
    int n = 0;
    e = cudaOccupancyMaxActiveClusters(&n, kern, &cfg);
    if (e != cudaSuccess) return e;
    clusters[dev] = n > 0 ? n : 1;
  }
  const uint64_t nc = nRows < (uint64_t)clusters[dev] ? nRows : (uint64_t)clusters[dev];
  cfg.gridDim = dim3((unsigned)(NC * nc));
  return cudaLaunchKernelEx(&cfg, kern, (const C*)ctx->state(), (C*)ctx->other(), nRows, P);
}

// ---------------------------------------------------------------- host side
int row_log_tile(int precision) { return precision == kC128 ? 12 : 13; }

bool row_eligible(Context* ctx, int reg) {
  if (ctx->flw[reg] != 0) return false;
  int lt = row_log_tile(ctx->precision);
  int q = ctx->q[reg];
  if (q > lt + 3 || q < kRowMinLogN) return false;  // big tile x cluster of 4 at most
  if (ctx->totalQbt < lt) return false;            // tile larger than the state
  return true;
}

// Split a diagonal run for a row program on `reg`.  Returns false when it does
// not fit (more than two control bits on the row register, too many terms, or a
// remainder that does not fit one factor list).
static bool split_row_diag(Context* ctx, int reg, const std::vector<Term>& terms,
                           std::vector<Term>* regTerms, std::vector<int>* ctrlBits,
                           std::vector<Term>* rowTerms, std::vector<Term>* elemTerms) {
  int lo = ctx->flw[reg], hi = lo + ctx->q[reg];
  auto inReg = [&](int bit) { return bit >= lo && bit < hi; };
  for (const Term& t : terms) {
    if (t.kind == kTermXX) {
      // bilinear terms touching the row register (or controlled from it) vary along the row
      if (t.r == reg || t.s == reg || (t.ctrlBit >= 0 && inReg(t.ctrlBit))) elemTerms->push_back(t);
      else rowTerms->push_back(t);
      continue;
    }
    if (t.kind != kTermScalar && t.r == reg) {
      if (t.kind == kTermPoly && t.ctrlBit >= 0 && !inReg(t.ctrlBit)) {
        bool found = false;
        for (int c : *ctrlBits) found |= c == t.ctrlBit;
        if (!found) ctrlBits->push_back(t.ctrlBit);
      }
      regTerms->push_back(t);
      continue;
    }
    if (t.kind == kTermPoly && t.ctrlBit >= 0 && inReg(t.ctrlBit)) {
      elemTerms->push_back(t);  // another register's phase controlled by a row qubit
      continue;
    }
    rowTerms->push_back(t);
  }
  if (ctrlBits->size() > 2 || regTerms->size() > (size_t)kMaxTermsPerTable) return false;
  // rowTerms and elemTerms must each fit one factor list
  auto fits = [&](const std::vector<Term>& ts) {
    std::vector<std::pair<int, int>> groups;
    std::vector<int> counts;
    int nxx = 0;
    for (const Term& t : ts) {
      if (t.kind == kTermScalar) continue;
      if (t.kind == kTermXX) {
        ++nxx;
        continue;
      }
      int c = -1;
      if (t.kind == kTermPoly && t.ctrlBit >= 0) {
        int l2 = ctx->flw[t.r], h2 = l2 + ctx->q[t.r];
        if (!(t.ctrlBit >= l2 && t.ctrlBit < h2)) c = t.ctrlBit;
      }
      std::pair<int, int> key{t.r, c};
      size_t g = 0;
      while (g < groups.size() && groups[g] != key) ++g;
      if (g == groups.size()) {
        groups.push_back(key);
        counts.push_back(0);
      }
      ++counts[g];
    }
    int tables = 0;
    for (int n : counts) tables += (n + kMaxTermsPerTable - 1) / kMaxTermsPerTable;
    return tables <= kMaxTab && nxx <= kMaxXX;
  };
  return fits(*rowTerms) && fits(*elemTerms);
}

// A bilinear term c x_reg x_other whose control bit (if any) lies off register
// reg: along a row of reg it is a linear phase (RowDiag::lin).
static bool linear_xx(Context* ctx, int reg, const Term& t) {
  const int lo = ctx->flw[reg], hi = lo + ctx->q[reg];
  return t.kind == kTermXX && ((t.r == reg) != (t.s == reg)) && (t.ctrlBit < 0 || t.ctrlBit < lo || t.ctrlBit >= hi);
}

static bool all_linear(Context* ctx, int reg, const std::vector<Term>& elemTerms) {
  for (const Term& t : elemTerms)
    if (!linear_xx(ctx, reg, t)) return false;
  return true;
}

// Programs on a strided register run on k_rowr only, which takes no per-element
// factor other than linear phases.
bool row_diag_fits(Context* ctx, int reg, const std::vector<Term>& terms) {
  std::vector<Term> a, b, c;
  std::vector<int> bits;
  if (!split_row_diag(ctx, reg, terms, &a, &bits, &b, &c)) return false;
  return ctx->flw[reg] == 0 || all_linear(ctx, reg, c);
}

template <typename C, int LOGC, int LOGT>
static cudaError_t launch_row_t(Context* ctx, const RowProgram& P, uint64_t nCta, size_t smem) {
  auto kern = k_row<C, LOGC, LOGT>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)nCta);
  cfg.blockDim = dim3(1u << LOGT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = ctx->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 1u << LOGC;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kern, (const C*)ctx->state(), (C*)ctx->other(), P);
}

// 2^14-point complex128 rows run on the eight-CTA kernel (k_rowq).  Complex64 rows
// of that length fit one CTA, k_rowr, which measured faster for them than k_rowq
// (1.43 against 1.61 ms per 2^28-amplitude launch); so did the one-CTA k_rowr for
// 2^13-point complex128 rows against a four-CTA k_rowq (3.30 against 3.41 ms of
// row programs per layer of the two-mode [13, 13] network).
static bool rowc_shape(Context* ctx, int reg, const std::vector<HostRowOp>& ops) {
  if (ctx->precision != kC128 || ctx->q[reg] != 14 || !row_eligible(ctx, reg)) return false;
  int lastDir = 0;
  for (const HostRowOp& h : ops)
    if (h.kind == kRowFft) {
      if (h.dir == lastDir) return false;
      lastDir = h.dir;
    }
  return true;
}

// log2 of the cluster that runs 2^14-point complex128 row programs (k_rowq: eight
// 128-thread CTAs); the blocked layout between paired programs follows it.
int rowc_log_cluster() { return 3; }

bool rowc_takes(Context* ctx, int reg, const std::vector<HostRowOp>& ops) {
  if (!rowc_shape(ctx, reg, ops)) return false;
  for (const HostRowOp& h : ops) {
    if (h.kind != kRowDiag) continue;
    std::vector<Term> regTerms, rowTerms, elemTerms;
    std::vector<int> bits;
    if (!split_row_diag(ctx, reg, h.terms, &regTerms, &bits, &rowTerms, &elemTerms) ||
        !all_linear(ctx, reg, elemTerms) || elemTerms.size() > (size_t)kMaxXX)
      return false;
  }
  return true;
}

bool launch_row_program(Context* ctx, int reg, const std::vector<HostRowOp>& ops, bool blockedIn,
                        bool blockedOut, bool rowSums) {
  RowProgram P{};
  // Registers up to the normal tile run two 256-thread CTAs per SM; longer ones
  // use the big tile (512 threads, twice the amplitudes, one CTA per SM) and, past
  // that, a cluster of 2 or 4 big tiles.
  int q = ctx->q[reg];
  const bool col = ctx->flw[reg] != 0;  // a strided register: k_rowr in column form, or the column kernel
  if (col && !col_program_ok(ctx, reg)) return launch_col_chain(ctx, reg, ops);
  int logT = q <= row_log_tile(ctx->precision) ? 8 : 9;
  int lt = row_log_tile(ctx->precision) + (logT - 8);
  int logC = q > lt ? q - lt : 0;
  const bool useC = !col && rowc_takes(ctx, reg, ops);  // the cluster register-resident kernels
  if (useC) logC = rowc_log_cluster();
  if (col) logC = 0;
  // k_rowr runs the program when every per-element factor is a linear phase
  bool toRowr = logC == 0 && q <= rowr_max_log(ctx->precision);
  for (const HostRowOp& h : ops) {
    if (!toRowr || h.kind != kRowDiag) continue;
    std::vector<Term> regTerms, rowTerms, elemTerms;
    std::vector<int> bits;
    toRowr = split_row_diag(ctx, reg, h.terms, &regTerms, &bits, &rowTerms, &elemTerms) &&
             all_linear(ctx, reg, elemTerms);
  }
  if (col && !toRowr) {
    set_error(ctx, kErrUnsupported, "column program on register %d needs per-element factors", reg);
    return false;
  }
  P.logS = col ? ctx->flw[reg] : 0;
  P.logN = q;
  P.logM = q - logC;
  P.logRows = q < lt ? lt - q : 0;
  P.logTwN = 0;
  while ((1 << P.logTwN) < ctx->twN) ++P.logTwN;
  P.tw = ctx->twiddle;
  P.waitErr = ctx->waitErr;
  // Layout at every op, as the kernel will see it: a program whose first
  // transform is inverse starts transposed; a forward transform leaves the
  // cluster transposed, an inverse natural; the tail runs in the final layout.
  P.loadT = 0;
  if (logC > 0) {
    for (const HostRowOp& h : ops)
      if (h.kind == kRowFft) {
        P.loadT = h.dir < 0 ? 1 : 0;
        break;
      }
  }
  bool transposedSim = P.loadT != 0;
  for (const HostRowOp& h : ops) {
    bool opTransposed = logC > 0 && transposedSim;
    if (h.kind == kRowFft) transposedSim = logC > 0 && h.dir > 0;
    if (P.nOps >= kMaxRowOps) {
      set_error(ctx, kErrUnsupported, "row program too long");
      return false;
    }
    RowOp& o = P.ops[P.nOps++];
    o.kind = h.kind;
    o.dir = h.dir;
    o.diag = -1;
    if (h.kind != kRowDiag) continue;
    if (P.nDiag >= kMaxRowDiags) {
      set_error(ctx, kErrUnsupported, "row program has too many diagonal runs");
      return false;
    }
    std::vector<Term> regTerms, rowTerms, elemTerms;
    std::vector<int> bits;
    if (!split_row_diag(ctx, reg, h.terms, &regTerms, &bits, &rowTerms, &elemTerms)) {
      set_error(ctx, kErrUnsupported, "row program diagonal run does not fit");
      return false;
    }
    RowDiag& D = P.diag[P.nDiag];
    D.nCtrl = (int)bits.size();
    for (int c = 0; c < D.nCtrl; ++c) D.ctrlShift[c] = bits[c];
    D.tab = nullptr;
    D.permuted = opTransposed ? 1 : 0;
    D.ftSign = 0;
    D.nPl = 0;
    // On the cluster kernel a run whose register terms are linear phases (transform
    // twiddles, c x terms controlled by row bits) needs no table.
    {
      const int lo = ctx->flw[reg], hi = lo + q;
      bool linOnly = (useC || toRowr) && !regTerms.empty();
      int nPl = 0;
      for (const Term& t : regTerms) {
        if (t.kind == kTermFtTw && t.ctrlBit < 0) continue;
        const bool rowCtrl = t.ctrlBit < 0 || t.ctrlBit < lo || t.ctrlBit >= hi;
        if (t.kind == kTermPoly && t.power == 1 && rowCtrl && nPl < 2) {
          ++nPl;
          continue;
        }
        linOnly = false;
      }
      if (linOnly) {
        for (const Term& t : regTerms) {
          if (t.kind == kTermFtTw) {
            D.ftSign += t.sign;
            continue;
          }
          D.plC[D.nPl] = t.coeff;
          D.plCtrl[D.nPl++] = t.ctrlBit;
        }
        D.regC = (double)((1 << q) - 1) * 0.5;
        D.regDx = ctx->dx[reg];
        regTerms.clear();
        bits.clear();
        D.nCtrl = 0;
      }
    }
    if (!regTerms.empty()) {
      double2* tab = (double2*)arena_alloc(ctx, ((size_t)1 << (q + D.nCtrl)) * sizeof(double2));
      if (!tab) return false;
      if (!launch_build_table_ext(ctx, reg, D.nCtrl, bits.data(), regTerms.data(),
                                  (int)regTerms.size(), tab, D.permuted ? logC : 0))
        return false;
      D.tab = tab;
    }
    D.nLin = 0;
    if (toRowr || useC) {
      const int lo = ctx->flw[reg];
      std::vector<Term> rest;
      for (const Term& t : elemTerms) {
        if (!linear_xx(ctx, reg, t) || D.nLin >= kMaxXX) {
          rest.push_back(t);
          continue;
        }
        const int o = t.r == reg ? t.s : t.r;
        XXFactor& X = D.lin[D.nLin++];
        X.shift1 = ctx->flw[o];
        X.mask1 = (1 << ctx->q[o]) - 1;
        X.c1 = (double)((1 << ctx->q[o]) - 1) * 0.5;
        X.dx1 = ctx->dx[o];
        X.shift2 = lo;
        X.mask2 = (1 << q) - 1;
        X.c2 = (double)((1 << q) - 1) * 0.5;
        X.dx2 = ctx->dx[reg];
        X.coeff = t.coeff;
        X.ctrlShift = t.ctrlBit;
      }
      elemTerms.swap(rest);
      D.regC = (double)((1 << q) - 1) * 0.5;
      D.regDx = ctx->dx[reg];
    }
    std::vector<Term> left;
    if (!build_factor_list(ctx, rowTerms, &D.rowF, &left) || !left.empty()) return false;
    if (!build_factor_list(ctx, elemTerms, &D.elemF, &left) || !left.empty()) return false;
    D.hasRowF = !factor_empty(D.rowF);
    D.hasElemF = !factor_empty(D.elemF);
    o.diag = P.nDiag++;
  }
  bool elemF = false;
  for (int d = 0; d < P.nDiag; ++d) elemF |= P.diag[d].hasElemF != 0;
  if ((blockedIn || blockedOut) && !useC) {
    set_error(ctx, kErrUnsupported, "blocked layout requested for a program the cluster kernel does not run");
    return false;
  }
  // the cluster kernel needs transforms that alternate in direction (each forward
  // leaves the transposed layout an inverse consumes)
  bool alternating = true;
  int lastDir = 0;
  for (int o = 0; o < P.nOps; ++o)
    if (P.ops[o].kind == kRowFft) {
      alternating &= P.ops[o].dir != lastDir;
      lastDir = P.ops[o].dir;
    }
  if (useC && !elemF && alternating) {
    if (blockedIn) P.loadT = 2;
    P.storeBlocked = blockedOut ? 1 : 0;
    if (rowSums) {
      P.rowSums = ctx->rowSums;
      ctx->rowSumParts = 32;  // 8 CTAs x 4 warps
    }
    cudaError_t er;
    {
      LaunchScope _ls(ctx, kKFft);
      bool xx = false;
      for (int d = 0; d < P.nDiag; ++d) xx |= P.diag[d].nLin > 0;
      er = xx ? launch_rowq_t<double2, 14, 3, true>(ctx, P) : launch_rowq_t<double2, 14, 3, false>(ctx, P);
    }
    if (!cuda_ok(ctx, er, "row program launch")) return false;
    ctx->cur ^= 1;
    return true;
  }
  if (toRowr) {
    if (elemF) {
      set_error(ctx, kErrUnsupported, "row program: per-element factors left for k_rowr");
      return false;
    }
    if (rowSums && !col) {
      const int logE = (ctx->precision == kC64 && q >= 13) ? 5 : 4, tpr = 1 << (q - logE);
      P.rowSums = ctx->rowSums;
      ctx->rowSumParts = tpr < 32 ? 1 : tpr / 32;
    }
    cudaError_t er;
    {
      LaunchScope _ls(ctx, col ? kKCol : kKFft);
      if (col)
        er = ctx->precision == kC128 ? launch_rowr<double2, true>(ctx, P, q) : launch_rowr<float2, true>(ctx, P, q);
      else
        er = ctx->precision == kC128 ? launch_rowr<double2, false>(ctx, P, q) : launch_rowr<float2, false>(ctx, P, q);
    }
    if (!cuda_ok(ctx, er, "row program launch")) return false;
    ctx->cur ^= 1;
    return true;
  }
  uint64_t tile = 1ull << lt;
  uint64_t nCta = ctx->size() / tile;
  size_t rs = (size_t)((1 << P.logM) + ((1 << P.logM) >> 4));
  size_t rows = 1ull << P.logRows;
  size_t smem = rs * rows * ctx->elemBytes + (64 + 128 + 64 + 512) * sizeof(double2) +
                rows * P.nDiag * (sizeof(double2) + sizeof(int)) + 16;
  cudaError_t e;
  {
    LaunchScope _ls(ctx, kKFft);
    if (ctx->precision == kC128) {
      if (logT == 8) e = launch_row_t<double2, 0, 8>(ctx, P, nCta, smem);
      else if (logC == 0) e = launch_row_t<double2, 0, 9>(ctx, P, nCta, smem);
      else if (logC == 1) e = launch_row_t<double2, 1, 9>(ctx, P, nCta, smem);
      else e = launch_row_t<double2, 2, 9>(ctx, P, nCta, smem);
    } else {
      if (logT == 8) e = launch_row_t<float2, 0, 8>(ctx, P, nCta, smem);
      else if (logC == 0) e = launch_row_t<float2, 0, 9>(ctx, P, nCta, smem);
      else if (logC == 1) e = launch_row_t<float2, 1, 9>(ctx, P, nCta, smem);
      else e = launch_row_t<float2, 2, 9>(ctx, P, nCta, smem);
    }
  }
  if (!cuda_ok(ctx, e, "row program launch")) return false;
  ctx->cur ^= 1;
  return true;
}

}  // namespace cvdv
