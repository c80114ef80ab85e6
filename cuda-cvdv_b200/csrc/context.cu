// Context lifecycle, error reporting, scratch memory, state I/O and the flush
// planner.
//
// Reference interfaces replaced here: cvdvCreate / cvdvDestroy / cvdvFree /
// cvdvInitFromSeparable / cvdvSetStateFromDevicePtr and the getters
// (src/cuda/context.cu:7-163, declared in src/cuda/api.h:14-23).  Unlike the
// reference, no entry point throws or exits: failures are recorded and can be
// read back with cvdvGetLastError.

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <atomic>
#include <map>
#include <mutex>

#include <algorithm>

#include "cvdv_internal.cuh"

namespace cvdv {

static std::mutex g_errMu;
static int g_lastErr = kOk;
static std::string g_lastMsg;

void set_error(Context* ctx, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) {
    ctx->lastErr = code;
    ctx->lastMsg = buf;
  }
  std::lock_guard<std::mutex> lk(g_errMu);
  g_lastErr = code;
  g_lastMsg = buf;
  if (getenv("CVDV_VERBOSE")) fprintf(stderr, "cvdv error %d: %s\n", code, buf);
}

// ----------------------------------------------------------------- launch accounting
std::atomic<unsigned long long> g_launches{0};
static thread_local int t_scopeDepth = 0;

static cudaEvent_t pool_event(Context* c) {
  if (!c->eventPool.empty()) {
    cudaEvent_t e = c->eventPool.back();
    c->eventPool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

void launch_begin(Context* c, int kind) {
  if (t_scopeDepth++ > 0) return;  // nested scopes count once
  g_launches.fetch_add(1, std::memory_order_relaxed);
  if (c && c->timing) {
    TimingRec r{pool_event(c), pool_event(c), kind};
    cudaEventRecord(r.a, c->stream);
    c->timingRecs.push_back(r);
  }
}

void launch_end(Context* c) {
  if (--t_scopeDepth > 0) return;
  if (c && c->timing && !c->timingRecs.empty()) cudaEventRecord(c->timingRecs.back().b, c->stream);
}

void harvest_timing(Context* c) {
  if (c->timingRecs.empty()) return;
  cudaStreamSynchronize(c->stream);
  for (auto& r : c->timingRecs) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      c->kindMs[r.kind] += ms;
      c->kindCount[r.kind] += 1;
    } else {
      cudaGetLastError();
    }
    c->eventPool.push_back(r.a);
    c->eventPool.push_back(r.b);
  }
  c->timingRecs.clear();
}

int global_error(char* msg, int len) {
  std::lock_guard<std::mutex> lk(g_errMu);
  if (msg && len > 0) {
    strncpy(msg, g_lastMsg.c_str(), (size_t)len - 1);
    msg[len - 1] = 0;
  }
  return g_lastErr;
}

bool cuda_ok(Context* ctx, cudaError_t e, const char* what) {
  if (e == cudaSuccess) return true;
  set_error(ctx, kErrCuda, "%s: %s", what, cudaGetErrorString(e));
  return false;
}

bool stream_sync(Context* ctx, const char* what) {
  if (!cuda_ok(ctx, cudaStreamSynchronize(ctx->stream), what)) return false;
  if (ctx->waitErr && *(volatile unsigned int*)ctx->waitErr) {
    *(volatile unsigned int*)ctx->waitErr = 0;
    set_error(ctx, kErrCuda, "%s: a kernel's wait for its cluster peers timed out; the state is not valid", what);
    return false;
  }
  return true;
}

// ----------------------------------------------------------------- arena
// Small per-flush scratch (factor tables, partial sums).  Allocation never
// invalidates pointers handed out since the last reset: when the arena is full
// a new block is chained; the next reset merges all blocks into one.
void arena_reset(Context* ctx) {
  if (!ctx->arenaExtra.empty()) {
    size_t total = ctx->arenaCap;
    for (auto& b : ctx->arenaExtra) total += b.cap;
    cudaStreamSynchronize(ctx->stream);
    for (auto& b : ctx->arenaExtra) cudaFree(b.p);
    ctx->arenaExtra.clear();
    if (ctx->arena) cudaFree(ctx->arena);
    ctx->arena = nullptr;
    ctx->arenaCap = 0;
    if (cudaMalloc(&ctx->arena, total) == cudaSuccess) ctx->arenaCap = total;
    else cudaGetLastError();
  }
  ctx->arenaTop = 0;
}

void* arena_alloc(Context* ctx, size_t bytes) {
  bytes = (bytes + 255) & ~(size_t)255;
  if (ctx->arena && ctx->arenaTop + bytes <= ctx->arenaCap) {
    void* p = ctx->arena + ctx->arenaTop;
    ctx->arenaTop += bytes;
    return p;
  }
  if (!ctx->arenaExtra.empty()) {
    ArenaBlock& b = ctx->arenaExtra.back();
    if (b.top + bytes <= b.cap) {
      void* p = b.p + b.top;
      b.top += bytes;
      return p;
    }
  }
  size_t cap = bytes < (64ull << 20) ? (64ull << 20) : bytes;
  char* p = nullptr;
  if (cudaMalloc(&p, cap) != cudaSuccess) {
    cudaGetLastError();
    set_error(ctx, kErrAlloc, "arena: cudaMalloc(%zu) failed", cap);
    return nullptr;
  }
  ctx->arenaExtra.push_back({p, cap, bytes});
  return p;
}

void* big_scratch(Context* ctx, size_t bytes) {
  if (bytes <= ctx->bigCap) return ctx->big;
  cudaStreamSynchronize(ctx->stream);
  if (ctx->big) cudaFree(ctx->big);
  ctx->big = nullptr;
  ctx->bigCap = 0;
  if (cudaMalloc(&ctx->big, bytes) != cudaSuccess) {
    cudaGetLastError();
    set_error(ctx, kErrAlloc, "scratch: cudaMalloc(%zu) failed", bytes);
    return nullptr;
  }
  ctx->bigCap = bytes;
  return ctx->big;
}

double* host_scratch(Context* ctx, size_t count) {
  size_t bytes = count * sizeof(double);
  if (bytes <= ctx->hostScratchCap) return ctx->hostScratch;
  if (ctx->hostScratch) cudaFreeHost(ctx->hostScratch);
  ctx->hostScratch = nullptr;
  ctx->hostScratchCap = 0;
  if (cudaMallocHost(&ctx->hostScratch, bytes) != cudaSuccess) {
    set_error(ctx, kErrAlloc, "pinned host scratch (%zu bytes) failed", bytes);
    return nullptr;
  }
  ctx->hostScratchCap = bytes;
  return ctx->hostScratch;
}

bool ensure_state(Context* ctx) {
  if (ctx->numReg == 0) {
    set_error(ctx, kErrNotInitialized, "context has no registers");
    return false;
  }
  uint64_t n = ctx->size();
  if (ctx->allocElems >= n && ctx->buf[0] && ctx->buf[1]) return true;
  for (int k = 0; k < 2; ++k) {
    if (ctx->buf[k]) cudaFree(ctx->buf[k]);
    ctx->buf[k] = nullptr;
  }
  for (int k = 0; k < 2; ++k) {
    if (cudaMalloc(&ctx->buf[k], n * ctx->elemBytes) != cudaSuccess) {
      cudaGetLastError();
      set_error(ctx, kErrAlloc, "state buffer %d: cudaMalloc(%llu bytes) failed", k,
                (unsigned long long)(n * ctx->elemBytes));
      if (ctx->buf[0]) cudaFree(ctx->buf[0]);
      ctx->buf[0] = nullptr;
      return false;
    }
  }
  ctx->allocElems = n;
  ctx->cur = 0;
  return true;
}

// ----------------------------------------------------------------- factor lists
struct TableKey {
  int r;
  int ctrl;  // external control bit or -1
  bool operator<(const TableKey& o) const { return r != o.r ? r < o.r : ctrl < o.ctrl; }
};

static inline double2 hmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Turn a diagonal run into a FactorList.  Terms that do not fit are returned in
// `leftover` (diagonal terms commute, so they can run as a separate pass).
bool build_factor_list(Context* ctx, const std::vector<Term>& terms, FactorList* F,
                       std::vector<Term>* leftover) {
  memset(F, 0, sizeof(*F));
  F->scalar = make_double2(1.0, 0.0);
  std::map<TableKey, std::vector<Term>> groups;
  std::vector<const Term*> xx;
  for (const Term& t : terms) {
    if (t.kind == kTermScalar) {
      F->scalar = hmul(F->scalar, t.g0);
      F->hasScalar = 1;
      continue;
    }
    if (t.kind == kTermXX) {
      xx.push_back(&t);
      continue;
    }
    int ctrl = -1;
    if (t.kind == kTermPoly && t.ctrlBit >= 0) {
      int lo = ctx->flw[t.r], hi = lo + ctx->q[t.r];
      if (!(t.ctrlBit >= lo && t.ctrlBit < hi)) ctrl = t.ctrlBit;
    }
    groups[{t.r, ctrl}].push_back(t);
  }
  // fold each register's uncontrolled terms into one of its controlled tables
  for (auto it = groups.begin(); it != groups.end();) {
    if (it->first.ctrl == -1) {
      auto jt = groups.end();
      for (auto kt = groups.begin(); kt != groups.end(); ++kt)
        if (kt->first.r == it->first.r && kt->first.ctrl >= 0) {
          jt = kt;
          break;
        }
      if (jt != groups.end() &&
          jt->second.size() + it->second.size() <= (size_t)kMaxTermsPerTable) {
        jt->second.insert(jt->second.end(), it->second.begin(), it->second.end());
        it = groups.erase(it);
        continue;
      }
    }
    ++it;
  }
  for (auto& g : groups) {
    const std::vector<Term>& ts = g.second;
    for (size_t start = 0; start < ts.size(); start += kMaxTermsPerTable) {
      size_t cnt = ts.size() - start;
      if (cnt > (size_t)kMaxTermsPerTable) cnt = kMaxTermsPerTable;
      if (F->nTab >= kMaxTab) {
        leftover->insert(leftover->end(), ts.begin() + start, ts.begin() + start + cnt);
        continue;
      }
      int r = g.first.r;
      bool ctrl = g.first.ctrl >= 0;
      int N = 1 << ctx->q[r];
      double2* tab = (double2*)arena_alloc(ctx, (size_t)N * (ctrl ? 2 : 1) * sizeof(double2));
      if (!tab) return false;
      if (!launch_build_table(ctx, r, ctrl, ts.data() + start, (int)cnt, tab)) return false;
      TabFactor& T = F->tab[F->nTab++];
      T.ptr = tab;
      T.shift = ctx->flw[r];
      T.mask = N - 1;
      T.ctrlShift = ctrl ? g.first.ctrl : -1;
      T.half = N;
      // only controlled phases (Z = +-1 flips their sign): the halves are conjugate
      T.conjHalf = ctrl ? 1 : 0;
      for (size_t k = start; k < start + cnt && T.conjHalf; ++k)
        T.conjHalf = ts[k].kind == kTermPoly && ts[k].ctrlBit == g.first.ctrl;
    }
  }
  for (const Term* t : xx) {
    if (F->nXX >= kMaxXX) {
      leftover->push_back(*t);
      continue;
    }
    XXFactor& X = F->xx[F->nXX++];
    X.shift1 = ctx->flw[t->r];
    X.mask1 = (1 << ctx->q[t->r]) - 1;
    X.shift2 = ctx->flw[t->s];
    X.mask2 = (1 << ctx->q[t->s]) - 1;
    X.c1 = (double)((1 << ctx->q[t->r]) - 1) * 0.5;
    X.dx1 = ctx->dx[t->r];
    X.c2 = (double)((1 << ctx->q[t->s]) - 1) * 0.5;
    X.dx2 = ctx->dx[t->s];
    X.coeff = t->coeff;
    X.ctrlShift = t->ctrlBit;
  }
  return true;
}

static bool run_leftover(Context* ctx, std::vector<Term> terms) {
  while (!terms.empty()) {
    FactorList F;
    std::vector<Term> rest;
    if (!build_factor_list(ctx, terms, &F, &rest)) return false;
    if (!factor_empty(F) && !launch_diag(ctx, F)) return false;
    if (rest.size() == terms.size()) {
      set_error(ctx, kErrUnsupported, "diagonal run could not be planned");
      return false;
    }
    terms.swap(rest);
  }
  return true;
}

// ----------------------------------------------------------------- flush
// Whether a diagonal run fits one factor list (no leftover).
static bool diag_fits(Context* ctx, const std::vector<Term>& terms) {
  std::vector<std::pair<int, int>> groups;
  int nxx = 0;
  std::vector<int> perGroup;
  for (const Term& t : terms) {
    if (t.kind == kTermScalar) continue;
    if (t.kind == kTermXX) {
      ++nxx;
      continue;
    }
    int ctrl = -1;
    if (t.kind == kTermPoly && t.ctrlBit >= 0) {
      int lo = ctx->flw[t.r], hi = lo + ctx->q[t.r];
      if (!(t.ctrlBit >= lo && t.ctrlBit < hi)) ctrl = t.ctrlBit;
    }
    std::pair<int, int> key{t.r, ctrl};
    size_t g = 0;
    while (g < groups.size() && groups[g] != key) ++g;
    if (g == groups.size()) {
      groups.push_back(key);
      perGroup.push_back(0);
    }
    ++perGroup[g];
  }
  int tables = 0;
  for (int c : perGroup) tables += (c + kMaxTermsPerTable - 1) / kMaxTermsPerTable;
  return tables <= kMaxTab && nxx <= kMaxXX;
}

// Whether a diagonal run fits a program on register reg: the row kernels' split
// (row programs, and column programs on k_rowr), else one factor list (column
// transform runs).
static bool program_diag_fits(Context* ctx, int reg, const std::vector<Term>& terms) {
  if (ctx->flw[reg] == 0 || col_program_ok(ctx, reg)) return row_diag_fits(ctx, reg, terms);
  return diag_fits(ctx, terms);
}

struct Op {
  const Stage* st = nullptr;        // pass-kernel op (FFT pass / pair / permutation)
  std::vector<Term> pre, post;
  int rowReg = -1;                  // row program on this register when >= 0
  std::vector<HostRowOp> row;
  bool blockedIn = false, blockedOut = false;
};

// Whether an op reads register r other than through factor tables over r (built
// permuted while r is blocked): a 2x2 gate on one of r's bits, a control bit
// inside r for a term on another register, a bilinear term on r.  Those index
// r's bits directly and need its natural order.
static bool reads_reg_bits(Context* ctx, const Op& b, int r) {
  const int lo = ctx->flw[r], hi = lo + ctx->q[r];
  auto inReg = [&](int bit) { return bit >= lo && bit < hi; };
  if (b.st && b.st->kind == kStPair && inReg(b.st->bit)) return true;
  for (const std::vector<Term>* v : {&b.pre, &b.post})
    for (const Term& t : *v) {
      if (t.kind == kTermXX && (t.r == r || t.s == r)) return true;
      if (t.ctrlBit >= 0 && inReg(t.ctrlBit) && t.r != r) return true;
    }
  return false;
}

// Pair a row program that ends with a forward 2^14-point transform (cluster
// kernel) with the next row program on the same register that starts with the
// inverse one, when everything in between only reads that register through
// factor tables (qubit gates on other registers, transforms of other registers,
// diagonal runs without bilinear terms on it or controls inside it).  The pair
// keeps the register in the blocked order in between, which saves the two
// layout swaps.
static void pair_blocked_programs(Context* ctx, std::vector<Op>& ops) {
  for (size_t i = 0; i < ops.size(); ++i) {
    Op& a = ops[i];
    if (a.rowReg < 0 || !rowc_takes(ctx, a.rowReg, a.row)) continue;
    int lastDir = 0, firstDir = 0;
    for (const HostRowOp& h : a.row)
      if (h.kind == kRowFft) lastDir = h.dir;
    if (lastDir <= 0) continue;
    const int r = a.rowReg;
    for (size_t j = i + 1; j < ops.size(); ++j) {
      Op& b = ops[j];
      if (b.rowReg == r) {
        for (const HostRowOp& h : b.row)
          if (h.kind == kRowFft) {
            firstDir = h.dir;
            break;
          }
        if (firstDir < 0 && rowc_takes(ctx, r, b.row)) {
          a.blockedOut = true;
          b.blockedIn = true;
          i = j - 1;  // b may itself end forward and pair with a later program
        }
        break;
      }
      if (b.rowReg >= 0) break;
      if (b.st && b.st->kind == kStPerm) break;
      if (b.st && b.st->kind == kStFft && b.st->reg == r) break;
      if (reads_reg_bits(ctx, b, r)) break;
    }
  }
}

// Number of consecutive pair ops from ops[i] that one qubit-gate sequence can
// take: at most kSeqMaxBits distinct bits, and every diagonal run among them
// (each pair's `pre`, the last op's `post`) still fitting with the final bit set.
static size_t seq_extent(Context* ctx, const std::vector<Op>& ops, size_t i) {
  std::vector<int> bits;
  int nOps = 0, nDiag = 0;
  size_t j = i;
  for (; j < ops.size(); ++j) {
    const Op& op = ops[j];
    if (op.rowReg >= 0 || !op.st || op.st->kind != kStPair) break;
    std::vector<int> nb = bits;
    if (std::find(nb.begin(), nb.end(), op.st->bit) == nb.end()) nb.push_back(op.st->bit);
    const int addDiag = (op.pre.empty() ? 0 : 1) + (op.post.empty() ? 0 : 1);
    if ((int)nb.size() > seq_max_bits(ctx) || nOps + 1 + addDiag > kSeqMaxOps ||
        nDiag + addDiag > kSeqMaxDiags)
      break;
    bool ok = true;
    for (size_t k = i; k <= j && ok; ++k)
      ok = (ops[k].pre.empty() || seq_diag_ok(ctx, nb, ops[k].pre)) &&
           (ops[k].post.empty() || seq_diag_ok(ctx, nb, ops[k].post));
    if (!ok) break;
    bits.swap(nb);
    nOps += 1 + addDiag;
    nDiag += addDiag;
  }
  return j - i;
}

// Whether a diagonal run depends on flat-index bit b.
static bool terms_touch_bit(Context* ctx, const std::vector<Term>& terms, int b) {
  auto inReg = [&](int r) { return r >= 0 && b >= ctx->flw[r] && b < ctx->flw[r] + ctx->q[r]; };
  for (const Term& t : terms) {
    if (t.kind == kTermScalar) continue;
    const bool ctrl = (t.kind == kTermPoly || t.kind == kTermXX) && t.ctrlBit == b;
    if (inReg(t.r) || ctrl || (t.kind == kTermXX && inReg(t.s))) return true;
  }
  return false;
}

// A qubit gate that opens a chain of qubit gates but is separated from it by a
// basis change of another register (H(q0) . FtQ2P(mode) . CPhaseX(ctrl q0) ...)
// commutes with that basis change: move it past the transform and every other
// commuting stage, so it runs in the chain's qubit-gate sequence instead of in
// a pass of its own.  Only stages that commute exactly are crossed.
static void hoist_pairs_past_transforms(Context* ctx, std::vector<Stage>& st) {
  for (size_t i = 0; i < st.size(); ++i) {
    if (st[i].kind != kStPair || (i > 0 && st[i - 1].kind == kStPair)) continue;
    const int b = st[i].bit;
    size_t j = i + 1;
    bool crossedFft = false;
    for (; j < st.size(); ++j) {
      const Stage& t = st[j];
      if (t.kind == kStFft) {
        if (b >= ctx->flw[t.reg] && b < ctx->flw[t.reg] + ctx->q[t.reg]) break;
        crossedFft = true;
      } else if (t.kind == kStDiag) {
        if (terms_touch_bit(ctx, t.terms, b)) break;
      } else {
        break;
      }
    }
    if (!crossedFft || j >= st.size() || (st[j].kind != kStDiag && st[j].kind != kStPair)) continue;
    Stage moved = std::move(st[i]);
    for (size_t k = i; k + 1 < j; ++k) st[k] = std::move(st[k + 1]);
    st[j - 1] = std::move(moved);
  }
}

// Whether a stage acts on register r (reads or changes its amplitudes' indices
// or phases through it).
static bool stage_touches_reg(Context* ctx, const Stage& s, int r) {
  const int lo = ctx->flw[r], hi = lo + ctx->q[r];
  auto inReg = [&](int b) { return b >= lo && b < hi; };
  switch (s.kind) {
    case kStFft: return s.reg == r;
    case kStPair: return inReg(s.bit);
    case kStPerm: return s.reg == r || s.reg2 == r || (s.bit >= 0 && inReg(s.bit));
    default:
      for (const Term& t : s.terms) {
        if (t.kind == kTermScalar) continue;
        if (t.r == r || (t.kind == kTermXX && t.s == r) || (t.ctrlBit >= 0 && inReg(t.ctrlBit))) return true;
      }
      return false;
  }
}

// Whether stage y may run before stage x (they commute exactly).
static bool stage_commutes(Context* ctx, const Stage& y, const Stage& x) {
  if (y.kind == kStDiag && x.kind == kStDiag) return true;
  if (y.kind == kStFft) return !stage_touches_reg(ctx, x, y.reg);
  if (y.kind != kStDiag) return false;
  switch (x.kind) {
    case kStFft: return !stage_touches_reg(ctx, y, x.reg);
    case kStPair: return !terms_touch_bit(ctx, y.terms, x.bit);
    case kStPerm:
      return !stage_touches_reg(ctx, y, x.reg) && (x.reg2 < 0 || !stage_touches_reg(ctx, y, x.reg2)) &&
             (x.bit < 0 || !terms_touch_bit(ctx, y.terms, x.bit));
    default: return false;
  }
}

// Product deferral.  After cvdvInitFromSeparable the state is the product of the
// register arrays.  A stage that acts on register r alone, queued ahead of every
// stage that couples r to another register, commutes with the stages before it
// (they act on other registers or on r alone), so it can run on r's array before
// the product is formed.  Such stages of registers of kFactorMinQ..kFactorMaxQ
// qubits run, in queue order, in a one-register complex128 context on this
// context's stream; qubit registers keep theirs (they join the qubit-gate
// sequences).  Stages that stay are left in order; the product is formed from
// the updated arrays before the flush's first launch (launch_product).
constexpr int kFactorMinQ = 8, kFactorMaxQ = 14;

static Stage factor_stage(Context* ctx, Stage s, int r) {
  const int f = ctx->flw[r];
  switch (s.kind) {
    case kStFft: s.reg = 0; break;
    case kStPair: s.bit -= f; break;
    case kStPerm:
      s.reg = 0;
      if (s.reg2 >= 0) s.reg2 = 0;
      if (s.bit >= 0) s.bit -= f;
      break;
    default:
      for (Term& t : s.terms) {
        if (t.kind == kTermScalar) continue;
        t.r = 0;
        if (t.kind == kTermXX) t.s = 0;
        if (t.ctrlBit >= 0) t.ctrlBit -= f;
      }
  }
  if (s.ftTag) s.ftReg = 0;
  return s;
}

static bool run_factors(Context* ctx, std::vector<Stage>& stages, std::vector<const double2*>& arrs) {
  const int R = ctx->numReg;
  std::vector<std::vector<Stage>> per(R);
  std::vector<char> coupled(R, 0);
  std::vector<Stage> rest;
  rest.reserve(stages.size());
  for (Stage& s : stages) {
    int reg = -1, n = 0;
    for (int r = 0; r < R; ++r)
      if (stage_touches_reg(ctx, s, r)) {
        reg = r;
        ++n;
      }
    if (n == 1 && !coupled[reg] && ctx->q[reg] >= kFactorMinQ && ctx->q[reg] <= kFactorMaxQ) {
      per[reg].push_back(factor_stage(ctx, std::move(s), reg));
      continue;
    }
    if (n > 1)
      for (int r = 0; r < R; ++r)
        if (stage_touches_reg(ctx, s, r)) coupled[r] = 1;
    rest.push_back(std::move(s));
  }
  arrs.assign(R, nullptr);
  size_t off = 0;
  for (int r = 0; r < R; ++r) {
    arrs[r] = ctx->factors + off;
    off += (size_t)1 << ctx->q[r];
  }
  for (int r = 0; r < R; ++r) {
    if (per[r].empty()) continue;
    Context* f = factor_context(ctx, r);
    if (!f) return false;
    const size_t bytes = ((size_t)1 << ctx->q[r]) * sizeof(double2);
    bool ok = ensure_state(f) &&
              cuda_ok(f, cudaMemcpyAsync(f->state(), arrs[r], bytes, cudaMemcpyDeviceToDevice, f->stream),
                      "register array in");
    if (ok) {
      f->initialized = true;
      f->cancelFt = ctx->cancelFt;
      f->fuseSeq = ctx->fuseSeq;
      f->colFft = ctx->colFft;
      f->colProg = ctx->colProg;
      // (transform pairs were cancelled when they were queued on this context, so
      // cvdvCancelledTransforms already counts them)
      f->pending = std::move(per[r]);
      ok = flush(f) && cuda_ok(f, cudaMemcpyAsync((void*)arrs[r], f->state(), bytes,
                                                   cudaMemcpyDeviceToDevice, f->stream),
                               "register array out");
    }
    if (!ok) {
      set_error(ctx, f->lastErr != kOk ? f->lastErr : kErrCuda, "register %d before the product: %s", r,
                f->lastMsg.c_str());
      return false;
    }
  }
  stages.swap(rest);
  return true;
}

// Whether the flush's first op on register r is a cluster row program that starts
// (after diagonal runs) with an inverse transform, with everything before it
// reading r only through factor tables; it is then marked to load r blocked.
static bool starts_blocked(Context* ctx, std::vector<Op>& ops, int r) {
  for (Op& b : ops) {
    if (b.rowReg == r) {
      int firstDir = 0;
      for (const HostRowOp& h : b.row)
        if (h.kind == kRowFft) {
          firstDir = h.dir;
          break;
        }
      if (firstDir >= 0 || b.blockedIn || !rowc_takes(ctx, r, b.row)) return false;
      b.blockedIn = true;
      return true;
    }
    if (b.rowReg >= 0) return false;
    if (b.st && b.st->kind == kStPerm) return false;
    if (b.st && b.st->kind == kStFft && b.st->reg == r) return false;
    if (reads_reg_bits(ctx, b, r)) return false;
  }
  return false;
}

// The product of the register arrays.  With blockedReg >= 0 (the last register)
// that register's array is first put in the blocked order of a cluster of
// C = 2^rowc_log_cluster() CTAs (position h M + k2 holds index h + C k2, M = N / C),
// so the state comes out blocked in it.
static bool blocked_array(Context* ctx, std::vector<const double2*>& arrs, int blockedReg) {
  if (blockedReg < 0) return true;
  const int nC = 1 << rowc_log_cluster();
  const size_t M = ((size_t)1 << ctx->q[blockedReg]) / nC;
  double2* t = (double2*)arena_alloc(ctx, nC * M * sizeof(double2));
  bool ok = t != nullptr;
  for (int h = 0; ok && h < nC; ++h)
    ok = cuda_ok(ctx, cudaMemcpy2DAsync(t + h * M, sizeof(double2), arrs[blockedReg] + h, nC * sizeof(double2),
                                        sizeof(double2), M, cudaMemcpyDeviceToDevice, ctx->stream),
                 "blocked register array");
  if (ok) arrs[blockedReg] = t;
  return ok;
}

// The product formed by the flush's first qubit-gate sequence: only the tables
// (the other registers' outer product, the last register's array) are made here.
static bool product_tables(Context* ctx, std::vector<const double2*>& arrs, int blockedReg) {
  const int R = ctx->numReg;
  double2* outer = (double2*)arena_alloc(ctx, ((size_t)1 << (ctx->totalQbt - ctx->q[R - 1])) * sizeof(double2));
  const bool ok = outer && blocked_array(ctx, arrs, blockedReg) && launch_outer(ctx, arrs.data(), outer);
  ctx->productPending = false;
  if (!ok) {
    ctx->initialized = false;
    return false;
  }
  ctx->seqProdLast = arrs[R - 1];
  ctx->seqProdOuter = outer;
  return true;
}

static bool launch_product(Context* ctx, std::vector<const double2*>& arrs, int blockedReg) {
  bool ok = blocked_array(ctx, arrs, blockedReg);
  ok = ok && launch_init_product(ctx, arrs.data());
  // The register arrays already carry the stages run on them and the rest of the
  // queue is dropped with the flush, so a product that could not be formed leaves
  // no valid state: later calls report the state uninitialised.
  ctx->productPending = false;
  if (!ok) ctx->initialized = false;
  return ok;
}

bool flush(Context* ctx) {
  if (ctx->pending.empty() && !ctx->productPending) return true;
  if (!ctx->initialized) {
    set_error(ctx, kErrNotInitialized, "gates queued before the state was initialised");
    ctx->pending.clear();
    return false;
  }
  arena_reset(ctx);
  std::vector<Stage> stages;
  stages.swap(ctx->pending);
  const bool product = ctx->productPending;
  std::vector<const double2*> arrs;
  if (product) {
    if (!run_factors(ctx, stages, arrs)) {
      // the state is lost with the product: later calls report it uninitialised
      ctx->productPending = false;
      ctx->initialized = false;
      return false;
    }
    if (stages.empty()) return launch_product(ctx, arrs, -1);
  }
  if (ctx->fuseSeq) hoist_pairs_past_transforms(ctx, stages);
  std::vector<Op> ops;
  std::vector<Term> diag;
  // A program on one register takes every later transform of that register and
  // every diagonal run that commutes with all the stages it would jump over
  // (transforms of other registers, qubit gates, runs that do not fit), up to
  // the program limits: gates on different registers are interleaved in the
  // queue (a beam splitter, then a gate on each mode) and would otherwise cut
  // the programs short.
  constexpr size_t kLookahead = 256, kMaxSkipped = 96;
  std::vector<char> taken(stages.size(), 0);
  size_t i = 0;
  while (i < stages.size()) {
    if (taken[i]) {
      ++i;
      continue;
    }
    const Stage& s = stages[i];
    if (s.kind == kStDiag) {
      diag.insert(diag.end(), s.terms.begin(), s.terms.end());
      taken[i] = 1;
      ++i;
      continue;
    }
    const bool chain = s.kind == kStFft && ctx->colFft && col_fft_ok(ctx, s.reg);
    if (s.kind == kStFft && (row_eligible(ctx, s.reg) || col_program_ok(ctx, s.reg) || chain)) {
      Op op;
      op.rowReg = s.reg;
      int nDiag = 0;
      auto addDiag = [&](const std::vector<Term>& t) -> bool {
        if (!op.row.empty() && op.row.back().kind == kRowDiag) {
          std::vector<Term> merged = op.row.back().terms;
          merged.insert(merged.end(), t.begin(), t.end());
          if (!program_diag_fits(ctx, s.reg, merged)) return false;
          op.row.back().terms = std::move(merged);
          return true;
        }
        if (nDiag >= kMaxRowDiags || (int)op.row.size() >= kMaxRowOps ||
            !program_diag_fits(ctx, s.reg, t))
          return false;
        op.row.push_back({kRowDiag, 0, t});
        ++nDiag;
        return true;
      };
      if (!diag.empty() && !addDiag(diag)) {
        // unusual: the leading run is too large for a program; it runs on its own first
        ops.push_back(Op{});
        ops.back().pre = diag;
        op.row.clear();
        nDiag = 0;
      }
      diag.clear();
      std::vector<size_t> skipped;
      for (size_t j = i; j < stages.size() && j < i + kLookahead; ++j) {
        if (taken[j]) continue;
        const Stage& t = stages[j];
        bool free = true;
        for (size_t k : skipped)
          if (!stage_commutes(ctx, t, stages[k])) {
            free = false;
            break;
          }
        bool took = false;
        if (free && t.kind == kStFft && t.reg == s.reg) {
          if ((int)op.row.size() + 2 > kMaxRowOps) break;
          op.row.push_back({kRowFft, t.dir, {}});
          took = true;
        } else if (free && t.kind == kStDiag) {
          took = addDiag(t.terms);
        }
        if (took) {
          taken[j] = 1;
        } else {
          skipped.push_back(j);
          if (skipped.size() > kMaxSkipped) break;
        }
      }
      ops.push_back(std::move(op));
      ++i;
      continue;
    }
    Op op;
    op.st = &s;
    op.pre = diag;
    ops.push_back(std::move(op));
    diag.clear();
    taken[i] = 1;
    ++i;
  }
  if (ops.empty()) return (!product || launch_product(ctx, arrs, -1)) && run_leftover(ctx, diag);
  if (!diag.empty()) {
    if (ops.back().rowReg >= 0) {
      // (only reachable when the program hit its limits) run the tail alone
      ops.push_back(Op{});
      ops.back().pre = diag;
    } else {
      ops.back().post = diag;
    }
  }
  pair_blocked_programs(ctx, ops);
  struct PermReset {  // the blocked layout never outlives the flush, errors included
    Context* c;
    ~PermReset() { c->permReg = -1; }
  } permReset{ctx};
  if (product) {
    // a first program on the last register that reads it blocked gets the product blocked
    const int last = ctx->numReg - 1;
    const int blocked = starts_blocked(ctx, ops, last) ? last : -1;
    // when the flush opens with a qubit-gate sequence, that pass forms the product
    const bool inSeq = ctx->fuseSeq && ctx->numReg >= 2 && ops[0].st && ops[0].st->kind == kStPair &&
                       seq_extent(ctx, ops, 0) >= 2;
    if (!(inSeq ? product_tables(ctx, arrs, blocked) : launch_product(ctx, arrs, blocked))) return false;
    if (blocked >= 0) {
      ctx->permReg = blocked;
      ctx->permLogC = rowc_log_cluster();
    }
  }
  for (size_t oi = 0; oi < ops.size(); ++oi) {
    Op& op = ops[oi];
    if (ctx->fuseSeq && op.st && op.st->kind == kStPair) {
      const size_t ext = seq_extent(ctx, ops, oi);
      if (ext >= 2) {
        std::vector<HostSeqOp> seq;
        for (size_t k = oi; k < oi + ext; ++k) {
          if (!ops[k].pre.empty()) seq.push_back({1, -1, {}, ops[k].pre});
          HostSeqOp p{0, ops[k].st->bit, {}, {}};
          for (int e = 0; e < 4; ++e) p.m[e] = ops[k].st->m[e];
          seq.push_back(std::move(p));
          if (!ops[k].post.empty()) seq.push_back({1, -1, {}, ops[k].post});
        }
        const bool forms = ctx->seqProdLast != nullptr;
        if (!launch_seq(ctx, seq)) {
          ctx->seqProdLast = ctx->seqProdOuter = nullptr;
          if (forms) ctx->initialized = false;  // the product state was never written
          return false;
        }
        oi += ext - 1;
        continue;
      }
    }
    if (op.rowReg >= 0) {
      if (op.blockedIn) ctx->permReg = -1;  // this program reads the blocked layout itself
      // the flush's last op on the last register may also write the row sums a
      // marginal readout asked for
      const bool sums = ctx->rowSums && oi + 1 == ops.size() && op.rowReg == ctx->numReg - 1 && !op.blockedOut;
      if (!launch_row_program(ctx, op.rowReg, op.row, op.blockedIn, op.blockedOut, sums)) return false;
      if (op.blockedOut) {
        ctx->permReg = op.rowReg;
        ctx->permLogC = rowc_log_cluster();
      }
      continue;
    }
    if (!op.st) {  // standalone diagonal run
      if (!run_leftover(ctx, op.pre)) return false;
      continue;
    }
    FactorList pre, post;
    std::vector<Term> lpre, lpost;
    if (!build_factor_list(ctx, op.pre, &pre, &lpre)) return false;
    if (!build_factor_list(ctx, op.post, &post, &lpost)) return false;
    if (!run_leftover(ctx, lpre)) return false;
    const Stage& s = *op.st;
    bool ok = true;
    if (s.kind == kStFft) ok = launch_fft(ctx, s.reg, s.dir, pre, post);
    else if (s.kind == kStPair) ok = launch_pair(ctx, s.bit, s.m, pre, post);
    else if (s.kind == kStPerm) ok = launch_perm(ctx, s, pre, post);
    if (!ok) return false;
    if (!run_leftover(ctx, lpost)) return false;
  }
  return true;
}

}  // namespace cvdv
