// Qubit-gate sequences: a run of 2x2 gates on up to four qubit bits, with the
// diagonal runs between them, in ONE read + write of the state.
//
// The state-transfer circuit, once its basis changes cancel, is a chain
//   H(q0) . CPhaseX(ctrl q0) . Rz(q0) . H(q1) . CPhaseX(ctrl q1) . Rz(q1) ...
// which the pair kernel runs as one HBM pass per qubit.  Here each thread owns a
// "site": the 2^NB amplitudes whose flat indices differ only in the NB selected
// bits.  It loads them once, applies every gate of the sequence in registers and
// stores them once.  Sites are numbered so that consecutive threads differ in
// the lowest unselected index bits, keeping loads and stores coalesced.
//
// Diagonal runs are table factors (the same tables the other kernels use).
// Inside a site a table index is idx0 + sum of per-bit offsets of the selected
// bits set in k.  The planner admits only tables that depend on at most one
// selected bit, so a run costs two table loads per table per site; tables that
// depend on the same bit are multiplied together first and the site is scaled
// once per dependent bit (once in total in the common case).

#include <algorithm>

#include "cvdv_internal.cuh"

namespace cvdv {

struct SeqTab {
  const double2* ptr;
  int shift, mask, ctrlShift, half;
  int gbit;  // selected-bit number (0..NB-1) the index depends on, or -1
  int d1;    // index offset when that bit is set
};

struct SeqDiag {
  double2 scalar;
  int nTab;
  SeqTab tab[kSeqMaxTabs];
};

enum SeqOpKind : int { kSeqPair = 0, kSeqPairReal = 1, kSeqDiag = 2 };

struct SeqOp {
  int kind;
  int bit;   // pair: selected-bit number
  int diag;  // diag: index into SeqProgram::diag
  double2 m[4];
};

struct SeqProgram {
  int bits[kSeqMaxBits];  // global bit positions, ascending
  int nOps;
  SeqOp ops[kSeqMaxOps];
  SeqDiag diag[kSeqMaxDiags];
};

template <typename C> struct SeqReal;
template <> struct SeqReal<double2> { using t = double; };
template <> struct SeqReal<float2> { using t = float; };

template <typename C, int NB, int B>
__device__ __forceinline__ void seq_pair(C* v, const double2* m) {
  const C a00 = fromd<C>(m[0]), a01 = fromd<C>(m[1]), a10 = fromd<C>(m[2]), a11 = fromd<C>(m[3]);
#pragma unroll
  for (int k = 0; k < (1 << NB); ++k) {
    if (k & (1 << B)) continue;
    const C x = v[k], y = v[k | (1 << B)];
    v[k] = cadd(cmul(a00, x), cmul(a01, y));
    v[k | (1 << B)] = cadd(cmul(a10, x), cmul(a11, y));
  }
}

// real 2x2 matrix (H, Ry): four real-by-complex products per butterfly
template <typename C, int NB, int B>
__device__ __forceinline__ void seq_pair_real(C* v, const double2* m) {
  using R = typename SeqReal<C>::t;
  const R a00 = (R)m[0].x, a01 = (R)m[1].x, a10 = (R)m[2].x, a11 = (R)m[3].x;
#pragma unroll
  for (int k = 0; k < (1 << NB); ++k) {
    if (k & (1 << B)) continue;
    const C x = v[k], y = v[k | (1 << B)];
    v[k] = mk(a00 * x.x + a01 * y.x, a00 * x.y + a01 * y.y);
    v[k | (1 << B)] = mk(a10 * x.x + a11 * y.x, a10 * x.y + a11 * y.y);
  }
}

template <typename C, int NB, int B>
__device__ __forceinline__ void seq_scale(C* v, double2 f0, double2 f1) {
  const C c0 = fromd<C>(f0), c1 = fromd<C>(f1);
#pragma unroll
  for (int k = 0; k < (1 << NB); ++k) v[k] = cmul(v[k], (k & (1 << B)) ? c1 : c0);
}

template <typename C, int NB>
__device__ __forceinline__ void seq_diag(C* v, const SeqDiag& D, uint64_t base) {
  double2 a = D.scalar;  // factor common to the whole site
  double2 p0[NB], p1[NB];
#pragma unroll
  for (int b = 0; b < NB; ++b) p0[b] = p1[b] = make_double2(1.0, 0.0);
  unsigned used = 0;
  for (int t = 0; t < D.nTab; ++t) {
    const SeqTab& T = D.tab[t];
    int idx = (int)((base >> T.shift) & (uint64_t)T.mask);
    if (T.ctrlShift >= 0) idx += (int)((base >> T.ctrlShift) & 1ull) * T.half;
    const double2 w0 = __ldg(T.ptr + idx);
    if (T.gbit < 0) {
      a = dmul(a, w0);
      continue;
    }
    const double2 w1 = __ldg(T.ptr + idx + T.d1);
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const bool hit = T.gbit == b;
      p0[b] = dmul(p0[b], hit ? w0 : make_double2(1.0, 0.0));
      p1[b] = dmul(p1[b], hit ? w1 : make_double2(1.0, 0.0));
    }
    used |= 1u << T.gbit;
  }
  if (!used) {
    const C c = fromd<C>(a);
#pragma unroll
    for (int k = 0; k < (1 << NB); ++k) v[k] = cmul(v[k], c);
    return;
  }
  bool folded = false;
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    if (!(used & (1u << b))) continue;
    double2 f0 = p0[b], f1 = p1[b];
    if (!folded) {
      f0 = dmul(f0, a);
      f1 = dmul(f1, a);
      folded = true;
    }
    if (b == 0) seq_scale<C, NB, 0>(v, f0, f1);
    if constexpr (NB > 1) if (b == 1) seq_scale<C, NB, 1>(v, f0, f1);
    if constexpr (NB > 2) if (b == 2) seq_scale<C, NB, 2>(v, f0, f1);
    if constexpr (NB > 3) if (b == 3) seq_scale<C, NB, 3>(v, f0, f1);
  }
}

template <typename C, int NB>
__global__ void __launch_bounds__(256, 2) k_seq(C* __restrict__ st, uint64_t nSites,
                                            const __grid_constant__ SeqProgram P) {
  constexpr int K = 1 << NB;
  for (uint64_t s = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nSites;
       s += (uint64_t)gridDim.x * blockDim.x) {
    // site base: s with a zero inserted at every selected bit (ascending order)
    uint64_t base = s;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const uint64_t low = (1ull << P.bits[b]) - 1;
      base = ((base & ~low) << 1) | (base & low);
    }
    C v[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      uint64_t o = base;
#pragma unroll
      for (int b = 0; b < NB; ++b)
        if (k & (1 << b)) o |= 1ull << P.bits[b];
      v[k] = st[o];
    }
    for (int o = 0; o < P.nOps; ++o) {
      const SeqOp& op = P.ops[o];
      if (op.kind == kSeqDiag) {
        seq_diag<C, NB>(v, P.diag[op.diag], base);
      } else if (op.kind == kSeqPairReal) {
        if (op.bit == 0) seq_pair_real<C, NB, 0>(v, op.m);
        if constexpr (NB > 1) if (op.bit == 1) seq_pair_real<C, NB, 1>(v, op.m);
        if constexpr (NB > 2) if (op.bit == 2) seq_pair_real<C, NB, 2>(v, op.m);
        if constexpr (NB > 3) if (op.bit == 3) seq_pair_real<C, NB, 3>(v, op.m);
      } else {
        if (op.bit == 0) seq_pair<C, NB, 0>(v, op.m);
        if constexpr (NB > 1) if (op.bit == 1) seq_pair<C, NB, 1>(v, op.m);
        if constexpr (NB > 2) if (op.bit == 2) seq_pair<C, NB, 2>(v, op.m);
        if constexpr (NB > 3) if (op.bit == 3) seq_pair<C, NB, 3>(v, op.m);
      }
    }
#pragma unroll
    for (int k = 0; k < K; ++k) {
      uint64_t o = base;
#pragma unroll
      for (int b = 0; b < NB; ++b)
        if (k & (1 << b)) o |= 1ull << P.bits[b];
      st[o] = v[k];
    }
  }
}

// ---------------------------------------------------------------- host side

// Number of selected bits a table of register r (with external control bit
// ctrl, or -1) depends on.
static int seq_deps(Context* ctx, const std::vector<int>& bits, int r, int ctrl) {
  const int lo = ctx->flw[r], hi = lo + ctx->q[r];
  int n = 0;
  for (int b : bits) n += ((b >= lo && b < hi) || b == ctrl) ? 1 : 0;
  return n;
}

bool seq_diag_ok(Context* ctx, const std::vector<int>& bits, const std::vector<Term>& terms) {
  // mirror build_factor_list's grouping: one table per (register, external control)
  std::vector<std::pair<int, int>> groups;
  std::vector<int> count;
  for (const Term& t : terms) {
    if (t.kind == kTermScalar) continue;
    if (t.kind == kTermXX) return false;
    int ctrl = -1;
    if (t.kind == kTermPoly && t.ctrlBit >= 0) {
      const int lo = ctx->flw[t.r], hi = lo + ctx->q[t.r];
      if (!(t.ctrlBit >= lo && t.ctrlBit < hi)) ctrl = t.ctrlBit;
    }
    if (seq_deps(ctx, bits, t.r, ctrl) > 1) return false;
    // an uncontrolled group may be folded into a controlled one of the same register
    if (ctrl < 0)
      for (const Term& u : terms)
        if (u.kind == kTermPoly && u.r == t.r && u.ctrlBit >= 0 && seq_deps(ctx, bits, t.r, u.ctrlBit) > 1)
          return false;
    std::pair<int, int> key{t.r, ctrl};
    size_t g = 0;
    while (g < groups.size() && groups[g] != key) ++g;
    if (g == groups.size()) {
      groups.push_back(key);
      count.push_back(0);
    }
    ++count[g];
  }
  int tables = 0;
  for (int c : count) tables += (c + kMaxTermsPerTable - 1) / kMaxTermsPerTable;
  return tables <= kSeqMaxTabs;
}

template <typename C>
static void seq_dispatch(Context* ctx, int nb, unsigned blocks, uint64_t nSites, const SeqProgram& P) {
  C* st = (C*)ctx->state();
  switch (nb) {
    case 1: k_seq<C, 1><<<blocks, 256, 0, ctx->stream>>>(st, nSites, P); break;
    case 2: k_seq<C, 2><<<blocks, 256, 0, ctx->stream>>>(st, nSites, P); break;
    case 3: k_seq<C, 3><<<blocks, 256, 0, ctx->stream>>>(st, nSites, P); break;
    default: k_seq<C, 4><<<blocks, 256, 0, ctx->stream>>>(st, nSites, P); break;
  }
}

bool launch_seq(Context* ctx, const std::vector<HostSeqOp>& ops) {
  std::vector<int> bits;
  for (const HostSeqOp& op : ops)
    if (op.kind == 0 && std::find(bits.begin(), bits.end(), op.bit) == bits.end()) bits.push_back(op.bit);
  std::sort(bits.begin(), bits.end());
  const int nb = (int)bits.size();
  if (nb < 1 || nb > kSeqMaxBits || (int)ops.size() > kSeqMaxOps) {
    set_error(ctx, kErrUnsupported, "qubit-gate sequence outside the kernel limits");
    return false;
  }
  SeqProgram P{};
  for (int b = 0; b < nb; ++b) P.bits[b] = bits[b];
  int nd = 0;
  for (const HostSeqOp& h : ops) {
    SeqOp& o = P.ops[P.nOps++];
    if (h.kind == 0) {
      o.bit = (int)(std::find(bits.begin(), bits.end(), h.bit) - bits.begin());
      bool real = true;
      for (int k = 0; k < 4; ++k) {
        o.m[k] = h.m[k];
        real = real && h.m[k].y == 0.0;
      }
      o.kind = real ? kSeqPairReal : kSeqPair;
      continue;
    }
    if (nd >= kSeqMaxDiags) {
      set_error(ctx, kErrUnsupported, "qubit-gate sequence has too many diagonal runs");
      return false;
    }
    FactorList F;
    std::vector<Term> left;
    if (!build_factor_list(ctx, h.terms, &F, &left)) return false;
    if (!left.empty() || F.nXX || F.nTab > kSeqMaxTabs) {
      set_error(ctx, kErrUnsupported, "diagonal run does not fit a qubit-gate sequence");
      return false;
    }
    SeqDiag& D = P.diag[nd];
    D.scalar = F.hasScalar ? F.scalar : make_double2(1.0, 0.0);
    D.nTab = F.nTab;
    for (int t = 0; t < F.nTab; ++t) {
      const TabFactor& T = F.tab[t];
      SeqTab& S = D.tab[t];
      S.ptr = T.ptr;
      S.shift = T.shift;
      S.mask = T.mask;
      S.ctrlShift = T.ctrlShift;
      S.half = T.half;
      S.gbit = -1;
      S.d1 = 0;
      for (int b = 0; b < nb; ++b) {
        const uint64_t i = 1ull << bits[b];
        int d = (int)((i >> T.shift) & (uint64_t)T.mask);
        if (T.ctrlShift >= 0) d += (int)((i >> T.ctrlShift) & 1ull) * T.half;
        if (!d) continue;
        if (S.gbit >= 0) {
          set_error(ctx, kErrUnsupported, "table depends on two bits of a qubit-gate sequence");
          return false;
        }
        S.gbit = b;
        S.d1 = d;
      }
    }
    o.kind = kSeqDiag;
    o.diag = nd++;
  }
  const uint64_t nSites = ctx->size() >> nb;
  uint64_t blocks = (nSites + 255) / 256;
  if (blocks > 148ull * 8) blocks = 148ull * 8;
  {
    LaunchScope _ls(ctx, kKSeq);
    if (ctx->precision == kC128) seq_dispatch<double2>(ctx, nb, (unsigned)blocks, nSites, P);
    else seq_dispatch<float2>(ctx, nb, (unsigned)blocks, nSites, P);
  }
  return cuda_ok(ctx, cudaGetLastError(), "qubit-gate sequence launch");
}

}  // namespace cvdv
