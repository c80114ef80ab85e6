// Transforms along a strided register (any register but the last): register-
// resident column DFTs, one or two HBM passes.
//
// The state is an [O][N][S] array around register r (N = 2^q points, S = 2^f
// amplitudes below it).  A "column" is one transform line: fixed outer and inner
// indices, stride S along the register.  A CTA of 256 threads takes W adjacent
// columns (adjacent inner indices, so every load and store instruction covers W
// consecutive amplitudes) and keeps each column's L points in registers, 16 per
// thread; the Stockham stages of the row kernels (row_fft.cuh) exchange through
// one padded shared-memory line per column.
//
// Registers of up to 2^8 points take one pass.  Longer ones use the four-step
// split N = N1 N2, j = j1 + N1 j2, k = k2 + N2 k1:
//   pass 1: u[j1, k2] = w_N^{j1 k2} sum_j2 w_N2^{j2 k2} x[j1 + N1 j2]   (stored at j1 + N1 k2)
//   pass 2: X[k2 + N2 k1] = sum_j1 w_N1^{j1 k1} u[j1, k2]            (stored in natural order)
// The diagonal run before the transform is applied on pass 1's loads and the
// one after it on the last pass's stores, as factors of the flat index.

#include "cvdv_internal.cuh"
#include "row_fft.cuh"

namespace cvdv {

constexpr int kColThreads = 256;

struct ColPass {
  uint64_t nCols;
  int logS;           // inner size S = 2^logS
  int logA;           // log2 of the middle index range of a column's base
  uint64_t midIn, outerIn, axisIn;     // strides (amplitudes) of the input
  uint64_t midOut, outerOut, axisOut;  // strides of the output
  int logN;           // > 0: multiply output point m of column (mid) by w_N^{mid m}
  int logTwN;
  const double2* tw;  // w_{2^logTwN}^e table of the context
  int hasPre, hasPost;
  FactorList pre, post;
};

template <int LOGL>
struct ColShape {
  static constexpr int L = 1 << LOGL, TPC = L >> 4, W = kColThreads / TPC;
  static constexpr int RS = (L + (L >> 4)) | 1;  // odd: the W columns of a warp fall on distinct banks
  static constexpr int HI = L >= 64 ? (L >> 6) : 1;
};

template <typename C, int LOGL, int DIR>
__global__ void __launch_bounds__(kColThreads, 2)
    k_colr(const C* __restrict__ in, C* __restrict__ out, const __grid_constant__ ColPass P) {
  using S = ColShape<LOGL>;
  constexpr int L = S::L, TPC = S::TPC, W = S::W;
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
  C v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const uint64_t a = bIn + (uint64_t)(t + TPC * k) * P.axisIn;
    v[k] = in[a];
    if (P.hasPre) v[k] = cmul(v[k], fromd<C>(eval_factor(P.pre, a)));
  }
  rr_stages<C, DIR, LOGL, 0, 4>(v, sm + (size_t)w * S::RS, t, loL, hiL);
  const int nMask = (1 << P.logN) - 1;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int m = t + TPC * k;
    const uint64_t a = bOut + (uint64_t)m * P.axisOut;
    C x = v[k];
    if (P.logN > 0) {
      const int e = (int)((mid * (uint64_t)m) & (uint64_t)nMask);
      if (e) x = cmul(x, tw2<C, DIR>(loN, hiN, e));
    }
    if (P.hasPost) x = cmul(x, fromd<C>(eval_factor(P.post, a)));
    out[a] = x;
  }
}

template <typename C, int LOGL>
static cudaError_t col_launch(Context* ctx, const void* in, void* out, const ColPass& P, int dir) {
  using S = ColShape<LOGL>;
  const int nHiN = P.logN >= 6 ? 1 << (P.logN - 6) : 1;
  const size_t smem = (size_t)S::W * S::RS * sizeof(C) + (64 + S::HI + 64 + nHiN) * sizeof(double2);
  const unsigned grid = (unsigned)(P.nCols / S::W);
  cudaError_t e;
  if (dir > 0) {
    e = cudaFuncSetAttribute(k_colr<C, LOGL, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_colr<C, LOGL, 1><<<grid, kColThreads, smem, ctx->stream>>>((const C*)in, (C*)out, P);
  } else {
    e = cudaFuncSetAttribute(k_colr<C, LOGL, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) k_colr<C, LOGL, -1><<<grid, kColThreads, smem, ctx->stream>>>((const C*)in, (C*)out, P);
  }
  return e != cudaSuccess ? e : cudaGetLastError();
}

template <typename C>
static cudaError_t col_dispatch(Context* ctx, int logL, const void* in, void* out, const ColPass& P, int dir) {
  switch (logL) {
    case 4: return col_launch<C, 4>(ctx, in, out, P, dir);
    case 5: return col_launch<C, 5>(ctx, in, out, P, dir);
    case 6: return col_launch<C, 6>(ctx, in, out, P, dir);
    case 7: return col_launch<C, 7>(ctx, in, out, P, dir);
    default: return col_launch<C, 8>(ctx, in, out, P, dir);
  }
}

// Whether launch_col_fft takes a transform of register `reg`: 2^4..2^16 points and
// at least 8 amplitudes below it (runs of 8 contiguous columns for the loads and
// stores).  A pass of 2^l points has 2^(n-l) columns and 2^(12-l) columns per
// CTA, so n >= 12 fills every CTA.
bool col_fft_ok(Context* ctx, int reg) {
  const int q = ctx->q[reg], logS = ctx->flw[reg];
  return q >= 4 && q <= 16 && logS >= 3 && ctx->totalQbt >= 12;
}

bool launch_col_fft(Context* ctx, int reg, int dir, const FactorList& pre, const FactorList& post) {
  const int q = ctx->q[reg], logS = ctx->flw[reg], n = ctx->totalQbt;
  const uint64_t S = 1ull << logS, N = 1ull << q;
  int logTwN = 0;
  while ((1 << logTwN) < ctx->twN) ++logTwN;
  ColPass P{};
  P.logS = logS;
  P.logTwN = logTwN;
  P.tw = ctx->twiddle;
  const bool two = q > 8;
  const int a = two ? (q + 1) / 2 : q, b = q - a;  // N1 = 2^a, N2 = 2^b
  cudaError_t e;
  const void* src = ctx->state();
  void* dst = ctx->other();
  {
    LaunchScope _ls(ctx, kKCol);
    if (!two) {
      P.nCols = 1ull << (n - q);
      P.logA = 0;
      P.midIn = P.midOut = 0;
      P.outerIn = P.outerOut = N * S;
      P.axisIn = P.axisOut = S;
      P.logN = 0;
      P.hasPre = !factor_empty(pre);
      P.hasPost = !factor_empty(post);
      P.pre = pre;
      P.post = post;
      e = ctx->precision == kC128 ? col_dispatch<double2>(ctx, q, src, dst, P, dir)
                                  : col_dispatch<float2>(ctx, q, src, dst, P, dir);
    } else {
      // pass 1: N2-point DFTs along j2 (stride N1 S), columns (i, j1, o); twiddle w_N^{j1 k2}
      P.nCols = 1ull << (n - b);
      P.logA = a;
      P.midIn = P.midOut = S;
      P.outerIn = P.outerOut = N * S;
      P.axisIn = P.axisOut = (1ull << a) * S;
      P.logN = q;
      P.hasPre = !factor_empty(pre);
      P.pre = pre;
      P.hasPost = 0;
      e = ctx->precision == kC128 ? col_dispatch<double2>(ctx, b, src, dst, P, dir)
                                  : col_dispatch<float2>(ctx, b, src, dst, P, dir);
    }
  }
  if (!cuda_ok(ctx, e, "column transform launch")) return false;
  ctx->cur ^= 1;
  if (!two) return true;
  {
    // pass 2: N1-point DFTs along j1 (stride S), columns (i, k2, o); output k2 + N2 k1
    LaunchScope _ls(ctx, kKCol);
    ColPass Q{};
    Q.logS = logS;
    Q.logTwN = logTwN;
    Q.tw = ctx->twiddle;
    Q.nCols = 1ull << (n - a);
    Q.logA = b;
    Q.midIn = (1ull << a) * S;
    Q.midOut = S;
    Q.outerIn = Q.outerOut = N * S;
    Q.axisIn = S;
    Q.axisOut = (1ull << b) * S;
    Q.logN = 0;
    Q.hasPre = 0;
    Q.hasPost = !factor_empty(post);
    Q.post = post;
    e = ctx->precision == kC128 ? col_dispatch<double2>(ctx, a, ctx->state(), ctx->other(), Q, dir)
                                : col_dispatch<float2>(ctx, a, ctx->state(), ctx->other(), Q, dir);
  }
  if (!cuda_ok(ctx, e, "column transform launch")) return false;
  ctx->cur ^= 1;
  return true;
}

}  // namespace cvdv
