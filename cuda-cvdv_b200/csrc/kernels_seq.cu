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
  int dep;   // index depends on the run's selected bit
  int d1;    // index offset when that bit is set
  int conj;  // the entry at +d1 is the conjugate of the one at +0 (a controlled phase)
};

struct SeqDiag {
  double2 scalar;   // the run's constant factor where its dependent bit is 0
  double2 scalar1;  // ... and where it is 1 (single-qubit phases folded in)
  int nTab;
  int g;  // selected-bit number (0..NB-1) the run depends on, or -1
  SeqTab tab[kSeqMaxTabs];
};

// kSeqPairH: c [[1, 1], [1, -1]] (Hadamard) -- sums and differences, with the
// real factor c carried along and folded into the next diagonal run
enum SeqOpKind : int { kSeqPair = 0, kSeqPairReal = 1, kSeqPairH = 2, kSeqDiag = 3 };

struct SeqOp {
  int kind;
  int bit;   // pair: selected-bit number
  int diag;  // diag: index into SeqProgram::diag
  double2 m[4];
};

struct SeqProgram {
  int bits[kSeqMaxBits];  // global bit positions, ascending
  // the state is the product last[i mod 2^prodQ] * outer[i >> prodQ], formed here
  const double2* prodLast;
  const double2* prodOuter;
  int prodQ;
  int nOps;
  SeqOp ops[kSeqMaxOps];
  SeqDiag diag[kSeqMaxDiags];
};

template <typename C> struct SeqReal;
template <> struct SeqReal<double2> { using t = double; };
template <> struct SeqReal<float2> { using t = float; };

// the 2x2 matrix arrives as four values (not a pointer into the kernel's
// parameters, which would make the compiler copy them to the stack)
struct Mat2 {
  double2 m0, m1, m2, m3;
};

template <typename C, int NB, int B>
__device__ __forceinline__ void seq_pair(C* v, const Mat2 m) {
  const C a00 = fromd<C>(m.m0), a01 = fromd<C>(m.m1), a10 = fromd<C>(m.m2), a11 = fromd<C>(m.m3);
#pragma unroll
  for (int k = 0; k < (1 << NB); ++k) {
    if (k & (1 << B)) continue;
    const C x = v[k], y = v[k | (1 << B)];
    v[k] = cadd(cmul(a00, x), cmul(a01, y));
    v[k | (1 << B)] = cadd(cmul(a10, x), cmul(a11, y));
  }
}

// real 2x2 matrix (Ry): four real-by-complex products per butterfly
template <typename C, int NB, int B>
__device__ __forceinline__ void seq_pair_real(C* v, const Mat2 m) {
  using R = typename SeqReal<C>::t;
  const R a00 = (R)m.m0.x, a01 = (R)m.m1.x, a10 = (R)m.m2.x, a11 = (R)m.m3.x;
#pragma unroll
  for (int k = 0; k < (1 << NB); ++k) {
    if (k & (1 << B)) continue;
    const C x = v[k], y = v[k | (1 << B)];
    v[k] = mk(a00 * x.x + a01 * y.x, a00 * x.y + a01 * y.y);
    v[k | (1 << B)] = mk(a10 * x.x + a11 * y.x, a10 * x.y + a11 * y.y);
  }
}

template <typename C, int NB, int B>
__device__ __forceinline__ void seq_pair_h(C* v) {
#pragma unroll
  for (int k = 0; k < (1 << NB); ++k) {
    if (k & (1 << B)) continue;
    const C x = v[k], y = v[k | (1 << B)];
    v[k] = cadd(x, y);
    v[k | (1 << B)] = csub(x, y);
  }
}

template <typename C, int NB, int B>
__device__ __forceinline__ void seq_scale(C* v, double2 f0, double2 f1) {
  const C c0 = fromd<C>(f0), c1 = fromd<C>(f1);
#pragma unroll
  for (int k = 0; k < (1 << NB); ++k) v[k] = cmul(v[k], (k & (1 << B)) ? c1 : c0);
}

#define SEQ_BIT_SWITCH(b, CALL)                          \
  switch (b) {                                           \
    case 0: { constexpr int B_ = 0; CALL; } break;       \
    case 1: if constexpr (NBL > 1) { constexpr int B_ = 1; CALL; } break; \
    case 2: if constexpr (NBL > 2) { constexpr int B_ = 2; CALL; } break; \
    case 3: if constexpr (NBL > 3) { constexpr int B_ = 3; CALL; } break; \
    default: if constexpr (NBL > 4) { constexpr int B_ = 4; CALL; } break; \
  }

template <typename C> __device__ __forceinline__ C shfl_xor_c(C v, int m);
template <> __device__ __forceinline__ double2 shfl_xor_c<double2>(double2 v, int m) {
  return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
template <> __device__ __forceinline__ float2 shfl_xor_c<float2>(float2 v, int m) {
  return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

// 2x2 gate on a bit split across lanes: the partner amplitude (same local index)
// lives in lane ^ lm; `hi` is this lane's value of the bit
template <typename C, int KL>
__device__ __forceinline__ void seq_pair_lanes(C* v, int kind, const Mat2 m, int lm, int hi) {
  using R = typename SeqReal<C>::t;
  // four amplitudes at a time: the warp barrier between groups keeps the compiler
  // from hoisting all KL shuffles ahead (which would double the live registers)
  if (kind == kSeqPairH) {
#pragma unroll
    for (int k0 = 0; k0 < KL; k0 += 4) {
#pragma unroll
      for (int k = k0; k < k0 + 4; ++k) {
        const C o = shfl_xor_c(v[k], lm);
        v[k] = hi ? csub(o, v[k]) : cadd(v[k], o);
      }
      __syncwarp();
    }
  } else if (kind == kSeqPairReal) {
    const R c0 = (R)(hi ? m.m2.x : m.m0.x), c1 = (R)(hi ? m.m3.x : m.m1.x);
#pragma unroll
    for (int k0 = 0; k0 < KL; k0 += 4) {
#pragma unroll
      for (int k = k0; k < k0 + 4; ++k) {
        const C o = shfl_xor_c(v[k], lm);
        const C x0 = hi ? o : v[k], x1 = hi ? v[k] : o;
        v[k] = mk(c0 * x0.x + c1 * x1.x, c0 * x0.y + c1 * x1.y);
      }
      __syncwarp();
    }
  } else {
    const C c0 = fromd<C>(hi ? m.m2 : m.m0), c1 = fromd<C>(hi ? m.m3 : m.m1);
#pragma unroll
    for (int k0 = 0; k0 < KL; k0 += 4) {
#pragma unroll
      for (int k = k0; k < k0 + 4; ++k) {
        const C o = shfl_xor_c(v[k], lm);
        const C x0 = hi ? o : v[k], x1 = hi ? v[k] : o;
        v[k] = cadd(cmul(c0, x0), cmul(c1, x1));
      }
      __syncwarp();
    }
  }
}

// A site of 2^NB amplitudes is held by 2^SPLIT consecutive lanes: the top SPLIT
// selected bits pick the lane, the other NB - SPLIT the register.  Gates on a
// lane bit exchange partners with warp shuffles.  GEN = false: the sequence's 2x2
// gates are all Hadamard-type, and the general-matrix paths are compiled out
// (fewer live registers, fewer spills of the site).
//
// PROD: the state is not written yet; each amplitude is formed from the product
// tables (the register arrays' outer product and the last register's array), so
// the product costs no pass of its own.
template <typename C, int NB, int SPLIT, typename IDX, bool GEN, bool PROD>
__global__ void __launch_bounds__(256, 2) k_seq(C* __restrict__ st, IDX nSites,
                                               const __grid_constant__ SeqProgram P) {
  constexpr int NBL = NB - SPLIT;  // bits held in registers
  constexpr int KL = 1 << NBL;
  using R = typename SeqReal<C>::t;
  // offsets of a site's register amplitudes from its base (the same for every
  // site), kept in shared memory rather than in 2^NBL registers per thread
  __shared__ IDX soff[KL];
  if (threadIdx.x < KL) {
    IDX o = 0;
    for (int b = 0; b < NBL; ++b)
      if (threadIdx.x & (1u << b)) o += (IDX)1 << P.bits[b];
    soff[threadIdx.x] = o;
  }
  __syncthreads();
  // every lane of a site runs every iteration: total is a multiple of the warp
  // size (the host keeps 2^(n - NB + SPLIT) >= 32 when SPLIT > 0)
  const IDX total = nSites << SPLIT;
  for (IDX g = (IDX)blockIdx.x * blockDim.x + threadIdx.x; g < total; g += (IDX)gridDim.x * blockDim.x) {
    const IDX s = g >> SPLIT;
    const int part = (int)(g & (IDX)((1 << SPLIT) - 1));
    // site base: s with a zero inserted at every selected bit (ascending order)
    IDX base = s;
#pragma unroll
    for (int b = 0; b < NB; ++b) {
      const IDX low = ((IDX)1 << P.bits[b]) - 1;
      base = ((base & ~low) << 1) | (base & low);
    }
    IDX hoff = 0;
#pragma unroll
    for (int i = 0; i < SPLIT; ++i)
      if ((part >> i) & 1) hoff += (IDX)1 << P.bits[NBL + i];
    // the offsets are re-read from shared memory (a broadcast) at every use rather
    // than held in KL registers across the site's gates
    const volatile IDX* vso = soff;
    C v[KL];
    if constexpr (PROD) {
      const IDX lm = ((IDX)1 << P.prodQ) - 1;
#pragma unroll
      for (int k = 0; k < KL; ++k) {
        const IDX a = base + hoff + vso[k];
        v[k] = fromd<C>(dmul(__ldg(P.prodLast + (a & lm)), __ldg(P.prodOuter + (a >> P.prodQ))));
      }
    } else {
#pragma unroll
      for (int k = 0; k < KL; ++k) v[k] = st[base + hoff + vso[k]];
    }
    R sc = (R)1;  // pending real factor of Hadamard-type pairs
    for (int o = 0; o < P.nOps; ++o) {
      const SeqOp& op = P.ops[o];
      if (op.kind != kSeqDiag) {
        if constexpr (!GEN) {  // Hadamard-type pairs only
          sc *= (R)op.m[0].x;
          if (SPLIT > 0 && op.bit >= NBL) {
            const int lb = op.bit - NBL;
            seq_pair_lanes<C, KL>(v, kSeqPairH, Mat2{}, 1 << lb, (part >> lb) & 1);
          } else {
            SEQ_BIT_SWITCH(op.bit, (seq_pair_h<C, NBL, B_>(v)))
          }
        } else {
          const Mat2 mm{op.m[0], op.m[1], op.m[2], op.m[3]};
          if (op.kind == kSeqPairH) sc *= (R)mm.m0.x;
          if (SPLIT > 0 && op.bit >= NBL) {
            const int lb = op.bit - NBL;
            seq_pair_lanes<C, KL>(v, op.kind, mm, 1 << lb, (part >> lb) & 1);
          } else if (op.kind == kSeqPairH) {
            SEQ_BIT_SWITCH(op.bit, (seq_pair_h<C, NBL, B_>(v)))
          } else if (op.kind == kSeqPairReal) {
            SEQ_BIT_SWITCH(op.bit, (seq_pair_real<C, NBL, B_>(v, mm)))
          } else {
            SEQ_BIT_SWITCH(op.bit, (seq_pair<C, NBL, B_>(v, mm)))
          }
        }
      } else {
        const SeqDiag& D = P.diag[op.diag];
        double2 w0 = D.scalar, w1 = D.scalar1;
        for (int t = 0; t < D.nTab; ++t) {
          const SeqTab& T = D.tab[t];
          int idx = (int)((base >> T.shift) & (IDX)T.mask);
          if (T.ctrlShift >= 0) idx += (int)((base >> T.ctrlShift) & (IDX)1) * T.half;
          const double2 a = __ldg(T.ptr + idx);
          const double2 b = T.dep ? (T.conj ? make_double2(a.x, -a.y) : __ldg(T.ptr + idx + T.d1)) : a;
          w0 = dmul(w0, a);
          w1 = dmul(w1, b);
        }
        const double dsc = (double)sc;
        w0 = make_double2(w0.x * dsc, w0.y * dsc);
        w1 = make_double2(w1.x * dsc, w1.y * dsc);
        sc = (R)1;
        if (D.g < 0 || (SPLIT > 0 && D.g >= NBL)) {
          // the factor does not vary over this lane's registers
          const C c = fromd<C>((D.g >= 0 && ((part >> (D.g - NBL)) & 1)) ? w1 : w0);
#pragma unroll
          for (int k = 0; k < KL; ++k) v[k] = cmul(v[k], c);
        } else {
          SEQ_BIT_SWITCH(D.g, (seq_scale<C, NBL, B_>(v, w0, w1)))
        }
      }
    }
    if (sc != (R)1) {
#pragma unroll
      for (int k = 0; k < KL; ++k) v[k] = mk(v[k].x * sc, v[k].y * sc);
    }
#pragma unroll
    for (int k = 0; k < KL; ++k) st[base + hoff + vso[k]] = v[k];
  }
}

// ---------------------------------------------------------------- host side

bool seq_diag_ok(Context* ctx, const std::vector<int>& bits, const std::vector<Term>& terms) {
  // mirror build_factor_list's grouping: one table per (register, external
  // control); every table may depend on one selected bit, the same for all
  std::vector<std::pair<int, int>> groups;
  std::vector<int> count;
  int depBit = -1;
  auto dep_ok = [&](int r, int ctrl) {
    const int lo = ctx->flw[r], hi = lo + ctx->q[r];
    for (int b : bits)
      if ((b >= lo && b < hi) || b == ctrl) {
        if (depBit >= 0 && depBit != b) return false;
        depBit = b;
      }
    return true;
  };
  for (const Term& t : terms) {
    if (t.kind == kTermScalar) continue;
    if (t.kind == kTermXX) return false;
    int ctrl = -1;
    if (t.kind == kTermPoly && t.ctrlBit >= 0) {
      const int lo = ctx->flw[t.r], hi = lo + ctx->q[t.r];
      if (!(t.ctrlBit >= lo && t.ctrlBit < hi)) ctrl = t.ctrlBit;
    }
    if (!dep_ok(t.r, ctrl)) return false;
    // an uncontrolled group may be folded into a controlled one of the same register
    if (ctrl < 0)
      for (const Term& u : terms)
        if (u.kind == kTermPoly && u.r == t.r && u.ctrlBit >= 0 && !dep_ok(t.r, u.ctrlBit)) return false;
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

// Bits per sequence: 16 (complex128) or 32 (complex64) amplitudes per thread;
// complex128 sequences of five bits split each site over 2 lanes when the state
// is large enough that every warp holds whole sites (2^(n - NB + SPLIT) >= 32).
// (Splitting complex64 sites over 2 or 4 lanes for 6-7 bits measured slower per
// pass than the extra pass it saves, so complex64 stops at 5.)
int seq_max_bits(Context* ctx) {
  if (ctx->precision == kC128) return ctx->totalQbt >= 9 ? 5 : 4;
  return 5;
}

template <typename C, int NB, int SPLIT, typename IDX>
static void seq_go(Context* ctx, unsigned blocks, uint64_t nSites, const SeqProgram& P) {
  bool gen = false;
  for (int o = 0; o < P.nOps; ++o) gen |= P.ops[o].kind == kSeqPair || P.ops[o].kind == kSeqPairReal;
  C* st = (C*)ctx->state();
  if (P.prodLast) {
    if (gen) k_seq<C, NB, SPLIT, IDX, true, true><<<blocks, 256, 0, ctx->stream>>>(st, (IDX)nSites, P);
    else k_seq<C, NB, SPLIT, IDX, false, true><<<blocks, 256, 0, ctx->stream>>>(st, (IDX)nSites, P);
  } else {
    if (gen) k_seq<C, NB, SPLIT, IDX, true, false><<<blocks, 256, 0, ctx->stream>>>(st, (IDX)nSites, P);
    else k_seq<C, NB, SPLIT, IDX, false, false><<<blocks, 256, 0, ctx->stream>>>(st, (IDX)nSites, P);
  }
}

template <typename C, typename IDX>
static void seq_dispatch(Context* ctx, int nb, unsigned blocks, uint64_t nSites, const SeqProgram& P) {
  switch (nb) {
    case 1: seq_go<C, 1, 0, IDX>(ctx, blocks, nSites, P); break;
    case 2: seq_go<C, 2, 0, IDX>(ctx, blocks, nSites, P); break;
    case 3: seq_go<C, 3, 0, IDX>(ctx, blocks, nSites, P); break;
    case 4: seq_go<C, 4, 0, IDX>(ctx, blocks, nSites, P); break;
    default:
      if constexpr (sizeof(C) == sizeof(float2)) seq_go<C, 5, 0, IDX>(ctx, blocks, nSites, P);
      else seq_go<C, 5, 1, IDX>(ctx, blocks, nSites, P);
      break;
  }
}

// lanes per site of the kernel seq_dispatch picks
static int seq_split(Context* ctx, int nb) { return (ctx->precision == kC128 && nb >= 5) ? 1 : 0; }

bool launch_seq(Context* ctx, const std::vector<HostSeqOp>& ops) {
  std::vector<int> bits;
  for (const HostSeqOp& op : ops)
    if (op.kind == 0 && std::find(bits.begin(), bits.end(), op.bit) == bits.end()) bits.push_back(op.bit);
  std::sort(bits.begin(), bits.end());
  const int nb = (int)bits.size();
  if (nb < 1 || nb > seq_max_bits(ctx) || (int)ops.size() > kSeqMaxOps) {
    set_error(ctx, kErrUnsupported, "qubit-gate sequence outside the kernel limits");
    return false;
  }
  SeqProgram P{};
  for (int b = 0; b < nb; ++b) P.bits[b] = bits[b];
  if (ctx->seqProdLast) {  // this pass forms the product state
    P.prodLast = ctx->seqProdLast;
    P.prodOuter = ctx->seqProdOuter;
    P.prodQ = ctx->q[ctx->numReg - 1];
    ctx->seqProdLast = ctx->seqProdOuter = nullptr;
  }
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
      const bool had = real && h.m[0].x == h.m[1].x && h.m[0].x == h.m[2].x && h.m[0].x == -h.m[3].x;
      o.kind = had ? kSeqPairH : real ? kSeqPairReal : kSeqPair;
      continue;
    }
    if (nd >= kSeqMaxDiags) {
      set_error(ctx, kErrUnsupported, "qubit-gate sequence has too many diagonal runs");
      return false;
    }
    // a phase on one selected qubit (Rz) is a pair of constants, g0 / g1 by that
    // bit: fold it into the run's scalars instead of a two-entry table
    std::vector<Term> rest;
    double2 s0 = make_double2(1.0, 0.0), s1 = s0;
    int foldBit = -1;
    for (const Term& t : h.terms) {
      const int gb = t.kind == kTermBit ? ctx->flw[t.r] + t.bit : -1;
      if (gb >= 0 && std::find(bits.begin(), bits.end(), gb) != bits.end() && (foldBit < 0 || foldBit == gb)) {
        foldBit = gb;
        s0 = make_double2(s0.x * t.g0.x - s0.y * t.g0.y, s0.x * t.g0.y + s0.y * t.g0.x);
        s1 = make_double2(s1.x * t.g1.x - s1.y * t.g1.y, s1.x * t.g1.y + s1.y * t.g1.x);
        continue;
      }
      rest.push_back(t);
    }
    FactorList F;
    std::vector<Term> left;
    if (!build_factor_list(ctx, rest, &F, &left)) return false;
    if (!left.empty() || F.nXX || F.nTab > kSeqMaxTabs) {
      set_error(ctx, kErrUnsupported, "diagonal run does not fit a qubit-gate sequence");
      return false;
    }
    SeqDiag& D = P.diag[nd];
    D.scalar = F.hasScalar ? F.scalar : make_double2(1.0, 0.0);
    D.scalar1 = make_double2(D.scalar.x * s1.x - D.scalar.y * s1.y, D.scalar.x * s1.y + D.scalar.y * s1.x);
    D.scalar = make_double2(D.scalar.x * s0.x - D.scalar.y * s0.y, D.scalar.x * s0.y + D.scalar.y * s0.x);
    D.nTab = F.nTab;
    D.g = -1;
    for (int t = 0; t < F.nTab; ++t) {
      const TabFactor& T = F.tab[t];
      SeqTab& S = D.tab[t];
      S.ptr = T.ptr;
      S.shift = T.shift;
      S.mask = T.mask;
      S.ctrlShift = T.ctrlShift;
      S.half = T.half;
      S.dep = 0;
      S.d1 = 0;
      S.conj = 0;
      for (int b = 0; b < nb; ++b) {
        const uint64_t i = 1ull << bits[b];
        int d = (int)((i >> T.shift) & (uint64_t)T.mask);
        if (T.ctrlShift >= 0) d += (int)((i >> T.ctrlShift) & 1ull) * T.half;
        if (!d) continue;
        if (S.dep || (D.g >= 0 && D.g != b)) {
          set_error(ctx, kErrUnsupported, "diagonal run depends on two bits of a qubit-gate sequence");
          return false;
        }
        S.dep = 1;
        S.d1 = d;
        S.conj = T.conjHalf && d == T.half;
        D.g = b;
      }
    }
    if (foldBit >= 0) {
      const int gi = (int)(std::find(bits.begin(), bits.end(), foldBit) - bits.begin());
      if (D.g >= 0 && D.g != gi) {
        set_error(ctx, kErrUnsupported, "diagonal run depends on two bits of a qubit-gate sequence");
        return false;
      }
      D.g = gi;
    }
    o.kind = kSeqDiag;
    o.diag = nd++;
  }
  const uint64_t nSites = ctx->size() >> nb;
  uint64_t blocks = ((nSites << seq_split(ctx, nb)) + 255) / 256;
  // the grid-stride loop runs on up to 32 CTAs per SM (two resident at a time): of
  // 2, 4, 8, 32 and 128 per SM, 32 measured fastest on a 2^28-amplitude state
  const uint64_t cap = 32ull * (uint64_t)ctx->numSMs;
  if (blocks > cap) blocks = cap;
  const bool narrow = ctx->totalQbt <= 31;  // every flat index fits 32 bits
  {
    LaunchScope _ls(ctx, kKSeq);
    if (ctx->precision == kC128) {
      if (narrow) seq_dispatch<double2, uint32_t>(ctx, nb, (unsigned)blocks, nSites, P);
      else seq_dispatch<double2, uint64_t>(ctx, nb, (unsigned)blocks, nSites, P);
    } else {
      if (narrow) seq_dispatch<float2, uint32_t>(ctx, nb, (unsigned)blocks, nSites, P);
      else seq_dispatch<float2, uint64_t>(ctx, nb, (unsigned)blocks, nSites, P);
    }
  }
  return cuda_ok(ctx, cudaGetLastError(), "qubit-gate sequence launch");
}

}  // namespace cvdv
