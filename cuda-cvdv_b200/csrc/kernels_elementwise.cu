// Elementwise kernels: diagonal factor tables, fused diagonal runs, 2x2 qubit
// pairs, register permutations and the separable-product initialiser.
//
// Every kernel here is one coalesced read + write of the state (HBM-bound);
// the per-element work is a handful of FP64 multiplies against factor tables
// that stay resident in L1/L2.

#include "cvdv_internal.cuh"

namespace cvdv {

// ----------------------------------------------------------------- tables
struct TTerm {
  int kind;        // kTermPoly / kTermFtTw / kTermBit
  int power;
  int sign;
  int bit;         // kTermBit: bit inside the register
  int ctrlMode;    // 0 none, 1 external control (table half), 2 control bit inside the register
  int ctrlLocal;   // ctrlMode 2: bit inside the register
  double coeff;
  double2 g0, g1;
};

struct TableJob {
  int N;
  int ctrl;        // number of external control bits: the table has 2^ctrl segments
  int permLogC;    // > 0: entries stored permuted (see launch_build_table_ext)
  int permLogM;
  double dx;
  int nTerms;
  TTerm t[kMaxTermsPerTable];
};

// Table entry (b, j) = prod over terms.  Polynomial terms are summed into one
// FP64 phase first (the same x_j expression as gridX in the reference,
// src/cuda/kernels/utils.cuh:5-7, and the same coeff*x*x*... evaluation order
// as kernelPhaseX/X2/X3, src/cuda/kernels/gates.cuh:5-16,184-209); the FT
// twiddle is generated exactly from the integer (N-1)(2j-N+1) mod 4N so its
// argument carries no rounding however large N is.
__global__ void k_build_table(TableJob job, double2* out) {
  int total = job.N << job.ctrl;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    int j = e % job.N;
    int b = e / job.N;
    if (job.permLogC) j = ((j & ((1 << job.permLogM) - 1)) << job.permLogC) + (j >> job.permLogM);
    double x = ((double)j - (double)(job.N - 1) * 0.5) * job.dx;
    double ph = 0.0;
    bool anyPoly = false;
    double2 f = make_double2(1.0, 0.0);
    for (int t = 0; t < job.nTerms; ++t) {
      const TTerm& T = job.t[t];
      if (T.kind == kTermPoly) {
        double v;
        if (T.power == 1) v = T.coeff * x;
        else if (T.power == 2) v = T.coeff * x * x;
        else v = T.coeff * x * x * x;
        bool neg = (T.ctrlMode == 1 && ((b >> T.ctrlLocal) & 1)) ||
                   (T.ctrlMode == 2 && ((j >> T.ctrlLocal) & 1));
        ph += neg ? -v : v;
        anyPoly = true;
      } else if (T.kind == kTermFtTw) {
        long long N = job.N;
        long long m = (N - 1) * (2LL * j - N + 1);
        long long M4 = 4 * N;
        m %= M4;
        if (m < 0) m += M4;
        double s, c;
        sincospi((double)(T.sign) * (double)m / (double)(2 * N), &s, &c);
        f = dmul(f, make_double2(c, s));
      } else if (T.kind == kTermBit) {
        f = dmul(f, ((j >> T.bit) & 1) ? T.g1 : T.g0);
      }
    }
    if (anyPoly) {
      double s, c;
      sincos(ph, &s, &c);
      f = dmul(make_double2(c, s), f);
    }
    out[e] = f;
  }
}

// Table over register r with nExt external control bits (extBits, flat-index
// positions outside r): entry [seg][j], seg bit c = value of extBits[c].
bool launch_build_table_ext(Context* ctx, int r, int nExt, const int* extBits, const Term* terms,
                            int nTerms, double2* out, int permLogC) {
  TableJob job{};
  job.N = 1 << ctx->q[r];
  job.ctrl = nExt;
  job.permLogC = permLogC;
  job.permLogM = ctx->q[r] - permLogC;
  job.dx = ctx->dx[r];
  job.nTerms = nTerms;
  int lo = ctx->flw[r], hi = ctx->flw[r] + ctx->q[r];
  for (int t = 0; t < nTerms; ++t) {
    const Term& T = terms[t];
    TTerm& D = job.t[t];
    D.kind = T.kind;
    D.power = T.power;
    D.sign = T.sign;
    D.bit = T.bit;
    D.coeff = T.coeff;
    D.g0 = T.g0;
    D.g1 = T.g1;
    D.ctrlMode = 0;
    D.ctrlLocal = 0;
    if (T.kind == kTermPoly && T.ctrlBit >= 0) {
      if (T.ctrlBit >= lo && T.ctrlBit < hi) {
        D.ctrlMode = 2;
        D.ctrlLocal = T.ctrlBit - lo;
      } else {
        D.ctrlMode = 1;
        for (int c = 0; c < nExt; ++c)
          if (extBits[c] == T.ctrlBit) D.ctrlLocal = c;
      }
    }
  }
  int total = job.N << nExt;
  int threads = 256;
  int blocks = (total + threads - 1) / threads;
  if (blocks > 1184) blocks = 1184;
  {
    LaunchScope _ls(ctx, kKTable);
    k_build_table<<<blocks, threads, 0, ctx->stream>>>(job, out);
  }
  return cuda_ok(ctx, cudaGetLastError(), "build_table launch");
}

bool launch_build_table(Context* ctx, int r, bool ctrl, const Term* terms, int nTerms,
                        double2* out) {
  int bit = -1;
  if (ctrl) {
    int lo = ctx->flw[r], hi = lo + ctx->q[r];
    for (int t = 0; t < nTerms; ++t)
      if (terms[t].kind == kTermPoly && terms[t].ctrlBit >= 0 &&
          !(terms[t].ctrlBit >= lo && terms[t].ctrlBit < hi))
        bit = terms[t].ctrlBit;
  }
  return launch_build_table_ext(ctx, r, ctrl ? 1 : 0, &bit, terms, nTerms, out,
                                r == ctx->permReg ? ctx->permLogC : 0);
}

// ----------------------------------------------------------------- diag run
// A thread takes V = 4 amplitudes i0 + 256 k with i0 a multiple of 1024 plus the
// thread index: its indices differ only in bits 8-9, which hold k.  A register
// field that misses those bits has the same index for all four, so its table
// entry is loaded once; a field that contains both (and reaches bit 8 or lower)
// advances by 2^(8 - shift) per k, so a bilinear term c x_r x_s whose sides are
// each fixed or advancing (and whose control, if any, is not bit 8 or 9) is
// linear in k: its value at k = 0 and the ratio between steps, two sincos,
// replace the four per-amplitude ones.  Other factors are evaluated per amplitude.
template <typename C>
__global__ void __launch_bounds__(256) k_diag(C* __restrict__ st, uint64_t n, FactorList F) {
  constexpr int V = 4;  // 256 threads x V amplitudes span bits 0..9
  // -1: the field holds one of bits 8, 9 only; 0: neither; else the step per k
  auto field = [](int shift, int mask) -> int {
    const int q = __popc(mask);
    if (shift >= 10 || shift + q <= 8) return 0;
    return (shift <= 8 && shift + q >= 10) ? (1 << (8 - shift)) : -1;
  };
  auto ctrl_fixed = [](int c) { return c < 8 || c > 9; };  // (-1: no control)
  const uint64_t stride = (uint64_t)gridDim.x * 256 * V;
  for (uint64_t base = (uint64_t)blockIdx.x * 256 * V + threadIdx.x; base < n; base += stride) {
    C v[V];
#pragma unroll
    for (int k = 0; k < V; ++k) {
      const uint64_t i = base + (uint64_t)k * 256;
      if (i < n) v[k] = st[i];
    }
    double2 g[V];
#pragma unroll
    for (int k = 0; k < V; ++k) g[k] = F.hasScalar ? F.scalar : make_double2(1.0, 0.0);
#pragma unroll
    for (int t = 0; t < kMaxTab; ++t) {
      if (t >= F.nTab) break;
      const TabFactor& T = F.tab[t];
      if (field(T.shift, T.mask) == 0 && ctrl_fixed(T.ctrlShift)) {
        int j = (int)((base >> T.shift) & (uint64_t)T.mask);
        if (T.ctrlShift >= 0) j += (int)((base >> T.ctrlShift) & 1ull) * T.half;
        const double2 a = __ldg(T.ptr + j);
#pragma unroll
        for (int k = 0; k < V; ++k) g[k] = dmul(g[k], a);
      } else {
        double2 a[V];
#pragma unroll
        for (int k = 0; k < V; ++k) {
          const uint64_t i = base + (uint64_t)k * 256;
          int j = (int)((i >> T.shift) & (uint64_t)T.mask);
          if (T.ctrlShift >= 0) j += (int)((i >> T.ctrlShift) & 1ull) * T.half;
          a[k] = __ldg(T.ptr + j);
        }
#pragma unroll
        for (int k = 0; k < V; ++k) g[k] = dmul(g[k], a[k]);
      }
    }
#pragma unroll 1
    for (int x = 0; x < F.nXX; ++x) {
      const XXFactor& X = F.xx[x];
      const int s1 = field(X.shift1, X.mask1), s2 = field(X.shift2, X.mask2);
      if (s1 >= 0 && s2 >= 0 && ctrl_fixed(X.ctrlShift)) {
        const double x1 = ((double)((base >> X.shift1) & (uint64_t)X.mask1) - X.c1) * X.dx1;
        const double x2 = ((double)((base >> X.shift2) & (uint64_t)X.mask2) - X.c2) * X.dx2;
        double c = X.coeff;
        if (X.ctrlShift >= 0 && ((base >> X.ctrlShift) & 1ull)) c = -c;
        // (the two registers differ, so at most one side advances)
        const double d = s1 ? c * ((double)s1 * X.dx1) * x2 : s2 ? c * x1 * ((double)s2 * X.dx2) : 0.0;
        double sn, cs;
        sincos(c * x1 * x2, &sn, &cs);
        double2 e = make_double2(cs, sn), stp;
        sincos(d, &stp.y, &stp.x);
#pragma unroll
        for (int k = 0; k < V; ++k) {
          g[k] = dmul(g[k], e);
          e = dmul(e, stp);
        }
      } else {
#pragma unroll
        for (int k = 0; k < V; ++k) {
          const uint64_t i = base + (uint64_t)k * 256;
          const double x1 = ((double)((i >> X.shift1) & (uint64_t)X.mask1) - X.c1) * X.dx1;
          const double x2 = ((double)((i >> X.shift2) & (uint64_t)X.mask2) - X.c2) * X.dx2;
          double ph = X.coeff * x1 * x2;
          if (X.ctrlShift >= 0 && ((i >> X.ctrlShift) & 1ull)) ph = -ph;
          double sn, cs;
          sincos(ph, &sn, &cs);
          g[k] = dmul(g[k], make_double2(cs, sn));
        }
      }
    }
#pragma unroll
    for (int k = 0; k < V; ++k) {
      const uint64_t i = base + (uint64_t)k * 256;
      if (i < n) st[i] = cmul(v[k], fromd<C>(g[k]));
    }
  }
}

static int grid_for(uint64_t work, int threads, int perThread) {
  uint64_t b = (work + (uint64_t)threads * perThread - 1) / ((uint64_t)threads * perThread);
  uint64_t cap = 148ull * 16;
  if (b > cap) b = cap;
  if (b < 1) b = 1;
  return (int)b;
}

bool launch_diag(Context* ctx, const FactorList& F) {
  uint64_t n = ctx->size();
  int blocks = grid_for(n, 256, 4);
  if (ctx->precision == kC128)
    {
      LaunchScope _ls(ctx, kKDiag);
      k_diag<double2><<<blocks, 256, 0, ctx->stream>>>((double2*)ctx->state(), n, F);
    }
  else
    {
      LaunchScope _ls(ctx, kKDiag);
      k_diag<float2><<<blocks, 256, 0, ctx->stream>>>((float2*)ctx->state(), n, F);
    }
  return cuda_ok(ctx, cudaGetLastError(), "diag launch");
}

// ----------------------------------------------------------------- pair (2x2)
// Pair indexing as qubitPairIndices (src/cuda/kernels/utils.cuh:79-84).
// Each thread takes kPairV pairs per iteration, all loads issued first.  The
// factor-free instance (the common case: neighbouring diagonal runs usually
// ride on a row program) is a separate, lean specialisation.
constexpr int kPairV = 4;

// MAXT: 0 = no factors; 2 = at most two tables and no bilinear terms (the
// usual neighbouring run: a qubit phase and one mode table); kMaxTab = general.
template <typename C, int MAXT>
__global__ void __launch_bounds__(256) k_pair(C* __restrict__ st, uint64_t npairs, int bit,
                                             double2 m00, double2 m01, double2 m10, double2 m11,
                                             const __grid_constant__ FactorList pre,
                                             const __grid_constant__ FactorList post) {
  constexpr int V = MAXT == 0 ? kPairV : (MAXT == 2 ? 2 : 1);
  constexpr bool XX = MAXT == kMaxTab;
  const uint64_t lowMask = (1ull << bit) - 1;
  const C a00 = fromd<C>(m00), a01 = fromd<C>(m01), a10 = fromd<C>(m10), a11 = fromd<C>(m11);
  const bool hasPre = MAXT > 0 && !factor_empty(pre), hasPost = MAXT > 0 && !factor_empty(post);
  const uint64_t step = (uint64_t)gridDim.x * blockDim.x * V;
  for (uint64_t p0 = (uint64_t)blockIdx.x * blockDim.x * V + threadIdx.x; p0 < npairs;
       p0 += step) {
    C a[V], b[V];
    uint64_t i0[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      uint64_t p = p0 + (uint64_t)v * blockDim.x;
      i0[v] = ((p & ~lowMask) << 1) | (p & lowMask);
      if (p < npairs) {
        a[v] = st[i0[v]];
        b[v] = st[i0[v] | (1ull << bit)];
      }
    }
#pragma unroll
    for (int v = 0; v < V; ++v) {
      uint64_t p = p0 + (uint64_t)v * blockDim.x;
      if (p >= npairs) continue;
      uint64_t i1 = i0[v] | (1ull << bit);
      C x = a[v], y = b[v];
      if constexpr (MAXT > 0) {
        if (hasPre) {
          x = cmul(x, fromd<C>(eval_factor_t<(MAXT > 0 ? MAXT : 1), XX>(pre, i0[v])));
          y = cmul(y, fromd<C>(eval_factor_t<(MAXT > 0 ? MAXT : 1), XX>(pre, i1)));
        }
      }
      C nx = cadd(cmul(a00, x), cmul(a01, y));
      C ny = cadd(cmul(a10, x), cmul(a11, y));
      if constexpr (MAXT > 0) {
        if (hasPost) {
          nx = cmul(nx, fromd<C>(eval_factor_t<(MAXT > 0 ? MAXT : 1), XX>(post, i0[v])));
          ny = cmul(ny, fromd<C>(eval_factor_t<(MAXT > 0 ? MAXT : 1), XX>(post, i1)));
        }
      }
      st[i0[v]] = nx;
      st[i1] = ny;
    }
  }
}

template <typename C>
static void pair_launch(Context* ctx, uint64_t np, int bit, const double2 m[4],
                        const FactorList& pre, const FactorList& post) {
  LaunchScope _ls(ctx, kKPair);
  bool none = factor_empty(pre) && factor_empty(post);
  bool small = pre.nTab <= 2 && post.nTab <= 2 && pre.nXX == 0 && post.nXX == 0;
  C* st = (C*)ctx->state();
  if (none)
    k_pair<C, 0><<<grid_for(np, 256, kPairV), 256, 0, ctx->stream>>>(st, np, bit, m[0], m[1], m[2],
                                                                      m[3], pre, post);
  else if (small)
    k_pair<C, 2><<<grid_for(np, 256, 2), 256, 0, ctx->stream>>>(st, np, bit, m[0], m[1], m[2],
                                                                m[3], pre, post);
  else
    k_pair<C, kMaxTab><<<grid_for(np, 256, 1), 256, 0, ctx->stream>>>(st, np, bit, m[0], m[1],
                                                                      m[2], m[3], pre, post);
}

bool launch_pair(Context* ctx, int bit, const double2 m[4], const FactorList& pre,
                 const FactorList& post) {
  uint64_t np = ctx->size() / 2;
  if (ctx->precision == kC128) pair_launch<double2>(ctx, np, bit, m, pre, post);
  else pair_launch<float2>(ctx, np, bit, m, pre, post);
  return cuda_ok(ctx, cudaGetLastError(), "pair launch");
}

// ----------------------------------------------------------------- permutations
// Out-of-place gather out[i] = in[src(i)].  src is an involution:
//  parity       j_r -> N-1-j_r  (kernelParity, gates.cuh:113-131)
//  cond parity  the pair {j, N-1-j} is exchanged iff the control bit of the
//               element with the smaller local index is 1
//               (kernelConditionalParity, gates.cuh:134-158)
//  swap         (j_r1, j_r2) -> (j_r2, j_r1)   (kernelSwapRegisters, gates.cuh:161-182)
struct PermDesc {
  int kind;
  int shift1, q1, shift2;
  int ctrlBit;
};

__device__ __forceinline__ uint64_t perm_src(const PermDesc& P, uint64_t i) {
  uint64_t m1 = ((1ull << P.q1) - 1) << P.shift1;
  if (P.kind == kPermParity) return i ^ m1;
  if (P.kind == kPermCondParity) {
    uint64_t loc = (i & m1) >> P.shift1;
    uint64_t N = 1ull << P.q1;
    uint64_t small = loc < (N - 1 - loc) ? loc : (N - 1 - loc);
    uint64_t is = (i & ~m1) | (small << P.shift1);
    return ((is >> P.ctrlBit) & 1ull) ? (i ^ m1) : i;
  }
  uint64_t m2 = ((1ull << P.q1) - 1) << P.shift2;
  uint64_t a = (i & m1) >> P.shift1;
  uint64_t b = (i & m2) >> P.shift2;
  return (i & ~(m1 | m2)) | (b << P.shift1) | (a << P.shift2);
}

// Each thread issues its V gathers before evaluating any factor, so V loads are in
// flight per thread.
template <typename C>
__global__ void __launch_bounds__(256) k_perm(const C* __restrict__ in, C* __restrict__ out,
                                             uint64_t n, PermDesc P, FactorList pre,
                                             FactorList post) {
  constexpr int V = 4;
  const bool hasPre = !factor_empty(pre), hasPost = !factor_empty(post);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x * V;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x * V + threadIdx.x; base < n; base += stride) {
    C v[V];
    uint64_t s[V];
#pragma unroll
    for (int k = 0; k < V; ++k) {
      const uint64_t i = base + (uint64_t)k * blockDim.x;
      s[k] = i < n ? perm_src(P, i) : 0;
      if (i < n) v[k] = in[s[k]];
    }
#pragma unroll
    for (int k = 0; k < V; ++k) {
      const uint64_t i = base + (uint64_t)k * blockDim.x;
      if (i >= n) continue;
      if (hasPre) v[k] = cmul(v[k], fromd<C>(eval_factor(pre, s[k])));
      if (hasPost) v[k] = cmul(v[k], fromd<C>(eval_factor(post, i)));
      out[i] = v[k];
    }
  }
}

bool launch_perm(Context* ctx, const Stage& st, const FactorList& pre, const FactorList& post) {
  PermDesc P{};
  P.kind = st.perm;
  P.shift1 = ctx->flw[st.reg];
  P.q1 = ctx->q[st.reg];
  P.shift2 = st.reg2 >= 0 ? ctx->flw[st.reg2] : 0;
  P.ctrlBit = st.bit;
  uint64_t n = ctx->size();
  int blocks = grid_for(n, 256, 4);
  if (ctx->precision == kC128)
    {
      LaunchScope _ls(ctx, kKPerm);
      k_perm<double2><<<blocks, 256, 0, ctx->stream>>>((const double2*)ctx->state(),
                                                       (double2*)ctx->other(), n, P, pre, post);
    }
  else
    {
      LaunchScope _ls(ctx, kKPerm);
      k_perm<float2><<<blocks, 256, 0, ctx->stream>>>((const float2*)ctx->state(),
                                                      (float2*)ctx->other(), n, P, pre, post);
    }
  if (!cuda_ok(ctx, cudaGetLastError(), "perm launch")) return false;
  ctx->cur ^= 1;
  return true;
}

// ----------------------------------------------------------------- separable init
// psi[i] = prod_r phi_r[j_r(i)], last register fastest (cvdvInitFromSeparable,
// src/cuda/context.cu:75-115; no normalisation).  Two steps: the product over
// all registers but the last into a small "outer" table, then one complex
// multiply per amplitude.
struct InitDesc {
  int numReg;
  int qLast;
  const double2* arr;   // concatenated register arrays
  int off[kMaxRegs];
  int shift[kMaxRegs];  // flw of each register minus qLast (index into outer)
  int mask[kMaxRegs];
};

__global__ void k_init_outer(InitDesc D, double2* outer, uint64_t nOuter) {
  for (uint64_t h = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; h < nOuter;
       h += (uint64_t)gridDim.x * blockDim.x) {
    double2 p = make_double2(1.0, 0.0);
    for (int r = D.numReg - 2; r >= 0; --r) {
      int j = (int)((h >> D.shift[r]) & (uint64_t)D.mask[r]);
      p = dmul(p, D.arr[D.off[r] + j]);
    }
    outer[h] = p;
  }
}

template <typename C>
__global__ void __launch_bounds__(256) k_init_product(C* __restrict__ st, uint64_t n, int qLast,
                                                     const double2* __restrict__ last,
                                                     const double2* __restrict__ outer) {
  const uint64_t lm = (1ull << qLast) - 1;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    double2 v = dmul(__ldg(last + (i & lm)), __ldg(outer + (i >> qLast)));
    st[i] = fromd<C>(v);
  }
}

static InitDesc init_desc(Context* ctx, const double2* const* regArrays) {
  int R = ctx->numReg;
  int qLast = ctx->q[R - 1];
  InitDesc D{};
  D.numReg = R;
  D.qLast = qLast;
  D.arr = regArrays[0];
  for (int r = 0; r < R; ++r) {
    D.off[r] = (int)(regArrays[r] - regArrays[0]);
    D.shift[r] = ctx->flw[r] - qLast;
    D.mask[r] = (1 << ctx->q[r]) - 1;
  }
  return D;
}

bool launch_outer(Context* ctx, const double2* const* regArrays, double2* outer) {
  int R = ctx->numReg;
  uint64_t nOuter = 1ull << (ctx->totalQbt - ctx->q[R - 1]);
  if (R >= 2) {
    InitDesc D = init_desc(ctx, regArrays);
    {
      LaunchScope _ls(ctx, kKInit);
      k_init_outer<<<grid_for(nOuter, 256, 1), 256, 0, ctx->stream>>>(D, outer, nOuter);
    }
    return cuda_ok(ctx, cudaGetLastError(), "outer launch");
  }
  static const double2 one = {1.0, 0.0};
  return cuda_ok(ctx, cudaMemcpyAsync(outer, &one, sizeof(one), cudaMemcpyHostToDevice, ctx->stream),
                 "outer copy");
}

bool launch_init_product(Context* ctx, const double2* const* regArrays) {
  // regArrays: device pointers to our own copies (arena), one per register
  int R = ctx->numReg;
  int qLast = ctx->q[R - 1];
  uint64_t nOuter = 1ull << (ctx->totalQbt - qLast);
  double2* outer = (double2*)arena_alloc(ctx, nOuter * sizeof(double2));
  if (!outer) return false;
  if (!launch_outer(ctx, regArrays, outer)) return false;
  uint64_t n = ctx->size();
  int blocks = grid_for(n, 256, 4);
  if (ctx->precision == kC128)
    {
      LaunchScope _ls(ctx, kKInit);
      k_init_product<double2><<<blocks, 256, 0, ctx->stream>>>((double2*)ctx->state(), n, qLast,
                                                               regArrays[R - 1], outer);
    }
  else
    {
      LaunchScope _ls(ctx, kKInit);
      k_init_product<float2><<<blocks, 256, 0, ctx->stream>>>((float2*)ctx->state(), n, qLast,
                                                              regArrays[R - 1], outer);
    }
  return cuda_ok(ctx, cudaGetLastError(), "init launch");
}

}  // namespace cvdv
