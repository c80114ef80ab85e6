// Transforms along a strided register (any register but the last): register-
// resident column DFTs in coalesced passes, with runs of transforms chained.
//
// The state is an [O][N][S] array around register r (N = 2^q points, S = 2^f
// amplitudes below it).  A "column" is one transform line: fixed outer and inner
// indices, stride S along the register.  A CTA of 256 threads takes W adjacent
// columns (adjacent inner indices, so every load and store instruction covers W
// consecutive amplitudes) and keeps each column's L points in registers, 8 per
// thread; the Stockham stages of the row kernels (row_fft.cuh) exchange through
// one padded shared-memory line per column.  A pass runs a small program on its
// columns: DFTs, diagonal runs (factor lists of the flat index) and the four-step
// twiddle.
//
// Registers of up to 2^8 points hold the whole column: a run of transforms and
// diagonal gates is one pass.  Longer ones use the four-step split N = N1 N2,
// j = j1 + N1 j2, k = k2 + N2 k1:
//   pass 1: u[j1, k2] = w_N^{j1 k2} sum_j2 w_N2^{j2 k2} x[j1 + N1 j2]   (stored at j1 + N1 k2)
//   pass 2: X[k2 + N2 k1] = sum_j1 w_N1^{j1 k1} u[j1, k2]            (stored in natural order)
// For fixed k2, pass 2 of one transform writes the positions k2 + N2 k1, and
// pass 1 of a next transform split the other way round (N1' = N2, N2' = N1) reads,
// for fixed j1' = k2, exactly the positions j1' + N1' j2'.  So consecutive
// transforms alternate their split and share a pass: pass 2 of transform t, the
// diagonal run between, and pass 1 of transform t + 1 run on one column load --
// T transforms take T + 1 passes instead of 2T.

#include "col_pass.cuh"
#include "cvdv_internal.cuh"
#include "row_fft.cuh"

namespace cvdv {

// CE: log2 of the points a thread holds (16 or 8); the shared line of a column is
// padded once per radix (16 or 8 points) and has an odd length, so the W columns
// of a warp fall on distinct banks
template <int LOGL, int CE>
struct ColShape {
  static constexpr int E = 1 << CE, L = 1 << LOGL, TPC = L >> CE, W = kColThreads / TPC;
  static constexpr int RS = (L + (L >> (CE >= 4 ? 4 : 3))) | 1;
  static constexpr int HI = L >= 64 ? (L >> 6) : 1;
};

// points per thread of the column kernel (log2): 8, so that three complex128 CTAs
// (four complex64 ones) fit an SM instead of two -- 0.71 against 0.80 ms per
// complex128 pass of a 2^26-amplitude state, 0.54 against 0.65 in complex64
template <typename C> struct ColCE { static constexpr int v = 3; };


// The linear phase of diagonal run d on the points t + TPC k (k < E) of a column
// whose point m sits at b + m ax: a (j - regC) regDx at register index j = j0 + u m,
// a = sum c x_other (sign by the control bit); two sincos, then a running product.
template <typename C, int LOGL, int CE>
__device__ __forceinline__ void col_lin(C (&v)[1 << CE], const ColPass& P, int d, uint64_t b, uint64_t ax,
                                        int t) {
  constexpr int TPC = ColShape<LOGL, CE>::TPC;
  double a = 0.0;
  for (int l = 0; l < P.nLin[d]; ++l) {
    const XXFactor& X = P.lin[d][l];
    const int j = (int)((b >> X.shift1) & (uint64_t)X.mask1);
    double cc = X.coeff * (((double)j - X.c1) * X.dx1);
    if (X.ctrlShift >= 0 && ((b >> X.ctrlShift) & 1ull)) cc = -cc;
    a += cc;
  }
  a *= P.regDx;
  const double j0 = (double)((b >> P.logS) & ((1ull << P.logQ) - 1));
  const double u = (double)(ax >> P.logS);
  double2 f, st;
  sincos(a * (j0 + u * (double)t - P.regC), &f.y, &f.x);
  sincos(a * u * (double)TPC, &st.y, &st.x);
#pragma unroll
  for (int k = 0; k < (1 << CE); ++k) {
    v[k] = cmul(v[k], fromd<C>(f));
    f = dmul(f, st);
  }
}

template <typename C, int LOGL, int CE>
__device__ __forceinline__ void col_lins(C (&v)[1 << CE], const ColPass& P, uint64_t b, uint64_t ax, int t) {
  for (int d = 0; d < P.nDiag; ++d)
    if (P.nLin[d]) col_lin<C, LOGL, CE>(v, P, d, b, ax, t);
}

template <typename C, int LOGL, int CE>
__device__ __forceinline__ void col_diags(C (&v)[1 << CE], const ColPass& P, uint64_t b, uint64_t ax, int t) {
  constexpr int TPC = ColShape<LOGL, CE>::TPC;
  for (int d = 0; d < P.nDiag; ++d) {
#pragma unroll
    for (int k = 0; k < (1 << CE); ++k)
      v[k] = cmul(v[k], fromd<C>(eval_factor(P.diag[d], b + (uint64_t)(t + TPC * k) * ax)));
    if (P.nLin[d]) col_lin<C, LOGL, CE>(v, P, d, b, ax, t);
  }
}

template <typename C, int LOGL, int KIND, int D1, int D2, int CE = ColCE<C>::v>
__global__ void __launch_bounds__(kColThreads, CE >= 4 ? 2 : (sizeof(C) == sizeof(float2) ? 4 : 3))
    k_colr(const C* __restrict__ in, C* __restrict__ out, const __grid_constant__ ColPass P) {
  using S = ColShape<LOGL, CE>;
  constexpr int TPC = S::TPC, W = S::W, E = S::E;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  double2* loL = reinterpret_cast<double2*>(sm + (size_t)W * S::RS);  // w_L^e, e < 64
  double2* hiL = loL + 64;                                            // w_L^(64 h)
  double2* loN = hiL + S::HI;                                         // w_N^e, e < 64
  double2* hiN = loN + 64;                                            // w_N^(64 h), h < N / 64
  const int tid = threadIdx.x, w = tid % W, t = tid / W;
  {
    const int nHiN = P.logN >= 6 ? 1 << (P.logN - 6) : 1;
    const int total = 64 + S::HI + 64 + nHiN;
    for (int i = tid; i < total; i += kColThreads) {
      int e, logM;
      double2* dst;
      if (i < 64 + S::HI) {
        e = i < 64 ? i : (i - 64) << 6;
        logM = LOGL;
        dst = loL + i;
      } else {
        const int j = i - 64 - S::HI;
        e = j < 64 ? j : (j - 64) << 6;
        logM = P.logN > 0 ? P.logN : LOGL;
        dst = loN + j;
      }
      *dst = (e < (1 << logM)) ? __ldg(P.tw + ((size_t)e << (P.logTwN - logM))) : make_double2(1.0, 0.0);
    }
  }
  __syncthreads();
  const uint64_t c = (uint64_t)blockIdx.x * W + w;
  const uint64_t i = c & ((1ull << P.logS) - 1);
  const uint64_t mid = (c >> P.logS) & ((1ull << P.logA) - 1);
  const uint64_t o = c >> (P.logS + P.logA);
  const uint64_t bIn = i + mid * P.midIn + o * P.outerIn;
  const uint64_t bOut = i + mid * P.midOut + o * P.outerOut;
  C* smcol = sm + (size_t)w * S::RS;
  C v[E];
  // the first half's diagonal runs ride on the loads, the last half's on the stores
#pragma unroll
  for (int k = 0; k < E; ++k) {
    const uint64_t a = bIn + (uint64_t)(t + TPC * k) * P.axisIn;
    v[k] = in[a];
    if constexpr (KIND == kColFirst)
      for (int d = 0; d < P.nDiag; ++d) v[k] = cmul(v[k], fromd<C>(eval_factor(P.diag[d], a)));
  }
  if constexpr (KIND == kColFirst) col_lins<C, LOGL, CE>(v, P, bIn, P.axisIn, t);
  if constexpr (KIND == kColWhole) {
    // input and output addresses coincide (one pass over the whole register)
    for (int p = 0; p < P.nOps; ++p) {
      const ColOp& op = P.ops[p];
      if (op.kind == kColDft) {
        if (op.dir > 0) rr_stages<C, 1, LOGL, 0, CE>(v, smcol, t, loL, hiL);
        else rr_stages<C, -1, LOGL, 0, CE>(v, smcol, t, loL, hiL);
      } else {
        const FactorList& F = P.diag[op.diag];
#pragma unroll
        for (int k = 0; k < E; ++k)
          v[k] = cmul(v[k], fromd<C>(eval_factor(F, bOut + (uint64_t)(t + TPC * k) * P.axisOut)));
        if (P.nLin[op.diag]) col_lin<C, LOGL, CE>(v, P, op.diag, bOut, P.axisOut, t);
      }
    }
  } else {
    rr_stages<C, D1, LOGL, 0, CE>(v, smcol, t, loL, hiL);
    if constexpr (KIND == kColMiddle) {
      col_diags<C, LOGL, CE>(v, P, bOut, P.axisOut, t);
      rr_stages<C, D2, LOGL, 0, CE>(v, smcol, t, loL, hiL);
    }
  }
  if constexpr (KIND == kColLast) col_lins<C, LOGL, CE>(v, P, bOut, P.axisOut, t);
  constexpr int DT = KIND == kColMiddle ? D2 : D1;  // direction of the four-step twiddle
  const int nMask = (1 << P.logN) - 1;
#pragma unroll
  for (int k = 0; k < E; ++k) {
    const int m = t + TPC * k;
    const uint64_t a = bOut + (uint64_t)m * P.axisOut;
    C x = v[k];
    if constexpr (KIND == kColFirst || KIND == kColMiddle) {
      const int e = (int)((mid * (uint64_t)m) & (uint64_t)nMask);
      if (e) x = cmul(x, tw2<C, DT>(loN, hiN, e));
    }
    if constexpr (KIND == kColLast)
      for (int d = 0; d < P.nDiag; ++d) x = cmul(x, fromd<C>(eval_factor(P.diag[d], a)));
    out[a] = x;
  }
}

template <typename C, int LOGL, int KIND, int D1, int D2>
static cudaError_t col_launch_t(Context* ctx, const ColPass& P) {
  using S = ColShape<LOGL, ColCE<C>::v>;
  const int nHiN = P.logN >= 6 ? 1 << (P.logN - 6) : 1;
  const size_t smem = (size_t)S::W * S::RS * sizeof(C) + (64 + S::HI + 64 + nHiN) * sizeof(double2);
  const unsigned grid = (unsigned)(P.nCols / S::W);
  auto kern = k_colr<C, LOGL, KIND, D1, D2>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  kern<<<grid, kColThreads, smem, ctx->stream>>>((const C*)ctx->state(), (C*)ctx->other(), P);
  return cudaGetLastError();
}

template <typename C, int LOGL>
static cudaError_t col_launch(Context* ctx, const ColPass& P, int kind, int d1, int d2) {
  switch (kind) {
    case kColFirst:
      return d1 > 0 ? col_launch_t<C, LOGL, kColFirst, 1, 0>(ctx, P) : col_launch_t<C, LOGL, kColFirst, -1, 0>(ctx, P);
    case kColLast:
      return d1 > 0 ? col_launch_t<C, LOGL, kColLast, 1, 0>(ctx, P) : col_launch_t<C, LOGL, kColLast, -1, 0>(ctx, P);
    case kColMiddle:
      if (d1 > 0) return d2 > 0 ? col_launch_t<C, LOGL, kColMiddle, 1, 1>(ctx, P) : col_launch_t<C, LOGL, kColMiddle, 1, -1>(ctx, P);
      return d2 > 0 ? col_launch_t<C, LOGL, kColMiddle, -1, 1>(ctx, P) : col_launch_t<C, LOGL, kColMiddle, -1, -1>(ctx, P);
    default:
      return col_launch_t<C, LOGL, kColWhole, 1, 0>(ctx, P);
  }
}

template <typename C>
static cudaError_t col_dispatch(Context* ctx, int logL, const ColPass& P, int kind, int d1, int d2) {
  switch (logL) {
    case 4: return col_launch<C, 4>(ctx, P, kind, d1, d2);
    case 5: return col_launch<C, 5>(ctx, P, kind, d1, d2);
    case 6: return col_launch<C, 6>(ctx, P, kind, d1, d2);
    case 7: return col_launch<C, 7>(ctx, P, kind, d1, d2);
    default: return col_launch<C, 8>(ctx, P, kind, d1, d2);
  }
}

cudaError_t launch_col_tc(Context* ctx, const ColPass& P, int logL, int kind, int d1, int d2);  // kernels_tc.cu

// Whether the column kernel takes transforms of register `reg`: 2^4..2^16 points
// and at least 8 amplitudes below it (runs of 8 contiguous columns for the loads
// and stores).  A pass of 2^l points has 2^(n-l) columns and 2^(11-l) columns per
// CTA (8 points a thread), so n >= 12 fills every CTA.
bool col_fft_ok(Context* ctx, int reg) {
  const int q = ctx->q[reg], logS = ctx->flw[reg];
  return q >= 4 && q <= 16 && logS >= 3 && ctx->totalQbt >= 12;
}

// A diagonal run of a column pass: the per-point factor list and the bilinear terms
// applied as a linear phase.
struct ColRun {
  FactorList F;
  int nLin = 0;
  XXFactor lin[kMaxXX];
};

// The bilinear terms c x_reg x_other with the control bit off register reg (at most
// kMaxXX) become linear phases; the rest goes to one factor list (false: it does not fit).
static bool split_col_run(Context* ctx, int reg, const std::vector<Term>& terms, ColRun* R) {
  const int lo = ctx->flw[reg], hi = lo + ctx->q[reg];
  std::vector<Term> rest;
  R->nLin = 0;
  for (const Term& t : terms) {
    const bool ctrlIn = t.ctrlBit >= lo && t.ctrlBit < hi;
    if (t.kind != kTermXX || (t.r == reg) == (t.s == reg) || ctrlIn || R->nLin >= kMaxXX) {
      rest.push_back(t);
      continue;
    }
    const int o = t.r == reg ? t.s : t.r;
    XXFactor& X = R->lin[R->nLin++];
    X = XXFactor{};
    X.shift1 = ctx->flw[o];
    X.mask1 = (1 << ctx->q[o]) - 1;
    X.c1 = (double)((1 << ctx->q[o]) - 1) * 0.5;
    X.dx1 = ctx->dx[o];
    X.coeff = t.coeff;
    X.ctrlShift = t.ctrlBit;
  }
  std::vector<Term> left;
  return build_factor_list(ctx, rest, &R->F, &left) && left.empty();
}

// A run of T >= 1 transforms (directions dirs) with the diagonal runs around
// them: slots[0] before the first, slots[t] between transform t-1 and t,
// slots[T] after the last (each slot a list of diagonal runs).
static bool run_col_chain(Context* ctx, int reg, const std::vector<int>& dirs,
                          const std::vector<std::vector<ColRun>>& slots) {
  const int q = ctx->q[reg], logS = ctx->flw[reg], n = ctx->totalQbt;
  const int T = (int)dirs.size();
  const uint64_t S = 1ull << logS, N = 1ull << q;
  int logTwN = 0;
  while ((1 << logTwN) < ctx->twN) ++logTwN;
  auto base = [&](ColPass& P) {
    P = ColPass{};
    P.logS = logS;
    P.logTwN = logTwN;
    P.tw = ctx->twiddle;
    P.outerIn = P.outerOut = N * S;
    P.logQ = q;
    P.regC = (double)(N - 1) * 0.5;
    P.regDx = ctx->dx[reg];
  };
  auto add_op = [&](ColPass& P, int kind, int dir, const ColRun* F) -> bool {
    if (P.nOps >= kMaxColOps || (kind == kColDiag && P.nDiag >= kMaxColDiags)) return false;
    ColOp& op = P.ops[P.nOps++];
    op.kind = kind;
    op.dir = dir;
    op.diag = -1;
    if (kind == kColDiag) {
      P.diag[P.nDiag] = F->F;
      P.nLin[P.nDiag] = F->nLin;
      for (int l = 0; l < F->nLin; ++l) P.lin[P.nDiag][l] = F->lin[l];
      op.diag = P.nDiag++;
    }
    return true;
  };
  auto add_slot = [&](ColPass& P, int s) -> bool {
    for (const ColRun& F : slots[s])
      if ((!factor_empty(F.F) || F.nLin) && !add_op(P, kColDiag, 0, &F)) return false;
    return true;
  };
  // complex64 passes of 64 or 128 points run as DFT-matrix products on the tensor cores
  const bool tc = tc_col_ok(ctx, reg);
  auto go = [&](const ColPass& P, int logL, int kind, int d1, int d2) -> bool {
    cudaError_t e;
    if (tc && kind != kColWhole && (logL == 6 || logL == 7) && P.logA >= 7 - logL) {
      LaunchScope _ls(ctx, kKColTc);
      e = launch_col_tc(ctx, P, logL, kind, d1, d2);
    } else {
      LaunchScope _ls(ctx, kKCol);
      e = ctx->precision == kC128 ? col_dispatch<double2>(ctx, logL, P, kind, d1, d2)
                                  : col_dispatch<float2>(ctx, logL, P, kind, d1, d2);
    }
    if (!cuda_ok(ctx, e, "column transform launch")) return false;
    ctx->cur ^= 1;
    return true;
  };
  auto too_long = [&]() {
    set_error(ctx, kErrUnsupported, "column transform run too long");
    return false;
  };
  ColPass P;
  if (q <= 8) {  // the whole run in one pass
    base(P);
    P.nCols = 1ull << (n - q);
    P.axisIn = P.axisOut = S;
    for (int t = 0; t <= T; ++t) {
      if (!add_slot(P, t)) return too_long();
      if (t < T && !add_op(P, kColDft, dirs[t], nullptr)) return too_long();
    }
    return go(P, q, kColWhole, 0, 0);
  }
  const int a = (q + 1) / 2, b = q - a;
  auto n1 = [&](int t) { return (t & 1) ? b : a; };  // log N1 of transform t
  auto n2 = [&](int t) { return (t & 1) ? a : b; };
  // pass 0: transform 0's N2-point DFTs along j2 (stride N1 S), columns (i, j1, o)
  base(P);
  P.nCols = 1ull << (n - n2(0));
  P.logA = n1(0);
  P.midIn = P.midOut = S;
  P.axisIn = P.axisOut = (1ull << n1(0)) * S;
  P.logN = q;
  if (!add_slot(P, 0)) return too_long();
  if (!go(P, n2(0), kColFirst, dirs[0], 0)) return false;
  // pass t: transform t-1's N1-point DFTs along j1 (stride S), columns (i, k2, o),
  // then (t < T) the run between and transform t's first half on the same points
  for (int t = 1; t <= T; ++t) {
    base(P);
    P.nCols = 1ull << (n - n1(t - 1));
    P.logA = n2(t - 1);
    P.midIn = (1ull << n1(t - 1)) * S;
    P.axisIn = S;
    P.midOut = S;
    P.axisOut = (1ull << n2(t - 1)) * S;
    P.logN = t < T ? q : 0;
    if (!add_slot(P, t)) return too_long();
    if (!go(P, n1(t - 1), t < T ? kColMiddle : kColLast, dirs[t - 1], t < T ? dirs[t] : 0)) return false;
  }
  return true;
}

bool launch_col_fft(Context* ctx, int reg, int dir, const FactorList& pre, const FactorList& post) {
  ColRun a, b;
  a.F = pre;
  b.F = post;
  return run_col_chain(ctx, reg, {dir}, {{a}, {b}});
}

// A row-program style run (transforms of `reg` and diagonal runs, in order) on a
// strided register: one pass for registers of up to 2^8 points, T + 1 chained
// passes for longer ones.
bool launch_col_chain(Context* ctx, int reg, const std::vector<HostRowOp>& ops) {
  std::vector<int> dirs;
  std::vector<std::vector<ColRun>> slots(1);
  for (const HostRowOp& h : ops) {
    if (h.kind == kRowFft) {
      dirs.push_back(h.dir);
      slots.emplace_back();
      continue;
    }
    ColRun R;
    if (!split_col_run(ctx, reg, h.terms, &R)) {
      set_error(ctx, kErrUnsupported, "column transform run: diagonal run does not fit");
      return false;
    }
    slots.back().push_back(R);
  }
  if (dirs.empty()) {
    set_error(ctx, kErrUnsupported, "column transform run without a transform");
    return false;
  }
  return run_col_chain(ctx, reg, dirs, slots);
}

}  // namespace cvdv
