// extern "C" entry points: context lifecycle, state I/O and gates.
//
// Each gate is decomposed exactly as the reference's src/cuda/gates.cu does
// (same primitive order, thresholds, rounding functions and global phases) but
// the primitives are queued as stages instead of being launched one by one:
//   FtQ2P(r)  = diag{twiddle} . FFT_r . diag{twiddle, 1/sqrt(N) e^{i pi (N-1)^2/(2N)}}
//   diagonal gates (PhaseX/X2/X3/XX, their controlled forms, Rz, Z) = diag terms
//   Hadamard / Rx / Ry = pair stages;  parity / cparity / swap = permutation stages.

#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/cvdv.h"
#include "cvdv_internal.cuh"

using namespace cvdv;

struct CVDVContext : public cvdv::Context {};

namespace {

constexpr double PI = CVDV_PI;
constexpr double SQRT2 = 1.41421356237309504880;

bool reg_ok(Context* c, int r, const char* what) {
  if (r < 0 || r >= c->numReg) {
    set_error(c, kErrInvalidArg, "%s: invalid register index %d", what, r);
    return false;
  }
  return true;
}

bool qubit_ok(Context* c, int r, int k, const char* what) {
  if (!reg_ok(c, r, what)) return false;
  if (k < 0 || k >= c->q[r]) {
    set_error(c, kErrInvalidArg, "%s: invalid qubit index %d of register %d", what, k, r);
    return false;
  }
  return true;
}

bool gate_ready(Context* c, const char* what) {
  if (c->numReg == 0) {
    set_error(c, kErrNotInitialized, "%s: context has no registers", what);
    return false;
  }
  if (!c->initialized) {
    set_error(c, kErrNotInitialized, "%s: state not initialised", what);
    return false;
  }
  return true;
}

int qubit_bit(Context* c, int r, int k) { return c->flw[r] + c->q[r] - 1 - k; }

Term poly(int r, int power, double coeff, int ctrlBit = -1) {
  Term t{};
  t.kind = kTermPoly;
  t.r = r;
  t.s = -1;
  t.power = power;
  t.coeff = coeff;
  t.ctrlBit = ctrlBit;
  return t;
}

void push_diag(Context* c, std::vector<Term> terms) {
  Stage s;
  s.kind = kStDiag;
  s.terms = std::move(terms);
  c->pending.push_back(std::move(s));
  if (c->pending.size() > 512) flush(c);
}

void push_stage(Context* c, Stage s) {
  c->pending.push_back(std::move(s));
  if (c->pending.size() > 512) flush(c);
}

// exp(i pi m / (2N)) with m = (N-1)^2 mod 4N, i.e. the FT global phase
// pi (N-1)^2 / (2N) reduced exactly (gates.cu:63-66, 119-121).
double2 ft_global(int N, int sign, double scale) {
  long long m = ((long long)(N - 1) * (long long)(N - 1)) % (4LL * N);
  double a = sign * PI * (double)m / (2.0 * (double)N);
  return make_double2(scale * cos(a), scale * sin(a));
}

// Whether a queued stage leaves register r untouched (so it commutes with any
// operator acting on r alone).
bool touches_bit(Context* c, int r, int bit) {
  return bit >= c->flw[r] && bit < c->flw[r] + c->q[r];
}

bool commutes_with_reg(Context* c, const Stage& s, int r) {
  switch (s.kind) {
    case kStDiag:
      for (const Term& t : s.terms) {
        if (t.kind == kTermScalar) continue;
        if (t.r == r || (t.kind == kTermXX && t.s == r)) return false;
        if (t.ctrlBit >= 0 && touches_bit(c, r, t.ctrlBit)) return false;
      }
      return true;
    case kStFft:
      return s.reg != r;
    case kStPair:
      return !touches_bit(c, r, s.bit);
    case kStPerm:
      if (s.reg == r || s.reg2 == r) return false;
      return !(s.perm == kPermCondParity && touches_bit(c, r, s.bit));
  }
  return false;
}

void queue_ft(Context* c, int r, int dir) {
  if (c->cancelFt) {
    // FtQ2P(r) . FtP2Q(r) = FtP2Q(r) . FtQ2P(r) = I exactly (conjugate twiddles and
    // global phases, unitary scale); stages in between that leave r alone commute.
    for (int i = (int)c->pending.size() - 1; i >= 0; --i) {
      const Stage& s = c->pending[i];
      if (s.ftTag && s.ftReg == r) {
        if (s.ftDir == -dir) {
          int tag = s.ftTag;
          std::vector<Stage> kept;
          kept.reserve(c->pending.size());
          for (Stage& t : c->pending)
            if (t.ftTag != tag) kept.push_back(std::move(t));
          c->pending.swap(kept);
          ++c->ftCancelled;
          return;
        }
        break;
      }
      if (!commutes_with_reg(c, s, r)) break;
    }
  }
  int N = 1 << c->q[r];
  int tag = c->nextFtTag++;
  Term tw{};
  tw.kind = kTermFtTw;
  tw.r = r;
  tw.s = -1;
  tw.ctrlBit = -1;
  tw.sign = dir;
  Stage pre;
  pre.kind = kStDiag;
  pre.terms = {tw};
  Stage f;
  f.kind = kStFft;
  f.reg = r;
  f.dir = dir;
  Term sc{};
  sc.kind = kTermScalar;
  sc.ctrlBit = -1;
  sc.g0 = ft_global(N, dir, 1.0 / sqrt((double)N));
  Stage post;
  post.kind = kStDiag;
  post.terms = {tw, sc};
  for (Stage* s : {&pre, &f, &post}) {
    s->ftTag = tag;
    s->ftReg = r;
    s->ftDir = dir;
  }
  // the three stages enter the queue together (a flush never splits them)
  c->pending.push_back(std::move(pre));
  c->pending.push_back(std::move(f));
  c->pending.push_back(std::move(post));
  if (c->pending.size() > 512) flush(c);
}

void queue_pair(Context* c, int bit, double2 m00, double2 m01, double2 m10, double2 m11) {
  Stage s;
  s.kind = kStPair;
  s.bit = bit;
  s.m[0] = m00;
  s.m[1] = m01;
  s.m[2] = m10;
  s.m[3] = m11;
  push_stage(c, std::move(s));
}

void queue_perm(Context* c, int kind, int r, int r2, int ctrlBit) {
  Stage s;
  s.kind = kStPerm;
  s.perm = kind;
  s.reg = r;
  s.reg2 = r2;
  s.bit = ctrlBit;
  push_stage(c, std::move(s));
}

void queue_pauli(Context* c, int r, int k, int axis, double theta) {
  double co = cos(theta / 2.0), si = sin(theta / 2.0);
  int bit = qubit_bit(c, r, k);
  if (axis == 2) {  // Rz is diagonal: (c - is) on |0>, (c + is) on |1>  (gates.cuh:86-90)
    Term t{};
    t.kind = kTermBit;
    t.r = r;
    t.s = -1;
    t.ctrlBit = -1;
    t.bit = c->q[r] - 1 - k;
    t.g0 = make_double2(co, -si);
    t.g1 = make_double2(co, si);
    push_diag(c, {t});
  } else if (axis == 0) {
    queue_pair(c, bit, make_double2(co, 0), make_double2(0, -si), make_double2(0, -si),
               make_double2(co, 0));
  } else {
    queue_pair(c, bit, make_double2(co, 0), make_double2(-si, 0), make_double2(si, 0),
               make_double2(co, 0));
  }
}

// C rint (half to even under the default rounding mode) and C round (half away)
double c_rint(double x) { return rint(x); }
double c_round(double x) { return round(x); }

void rotation_small(Context* c, int r, double th) {
  if (fabs(th) < 1e-15) return;
  double t = tan(th / 2.0), s = sin(th);
  push_diag(c, {poly(r, 2, -0.5 * t)});
  queue_ft(c, r, 1);
  push_diag(c, {poly(r, 2, -0.5 * s)});
  queue_ft(c, r, -1);
  push_diag(c, {poly(r, 2, -0.5 * t)});
}

void crotation_small(Context* c, int t, int cb, double th) {
  if (fabs(th) < 1e-15) return;
  double tt = tan(th / 2.0), s = sin(th);
  push_diag(c, {poly(t, 2, -0.5 * tt, cb)});
  queue_ft(c, t, 1);
  push_diag(c, {poly(t, 2, -0.5 * s, cb)});
  queue_ft(c, t, -1);
  push_diag(c, {poly(t, 2, -0.5 * tt, cb)});
}

Term xx(int r1, int r2, double coeff, int cb = -1) {
  Term t{};
  t.kind = kTermXX;
  t.r = r1;
  t.s = r2;
  t.coeff = coeff;
  t.ctrlBit = cb;
  return t;
}

void bs_small(Context* c, int r1, int r2, double th, int cb) {
  if (fabs(th) < 1e-15) return;
  double cq = -tan(0.25 * th), cp = -sin(0.5 * th);
  push_diag(c, {xx(r1, r2, cq, cb)});
  queue_ft(c, r1, 1);
  queue_ft(c, r2, 1);
  push_diag(c, {xx(r1, r2, cp, cb)});
  queue_ft(c, r1, -1);
  queue_ft(c, r2, -1);
  push_diag(c, {xx(r1, r2, cq, cb)});
}

Context* C(CVDVContext* p) { return static_cast<Context*>(p); }

}  // namespace

// ====================================================================== lifecycle
extern "C" {

CVDVContext* cvdvCreateEx(int numReg, int* numQubits, int precision) {
  CVDVContext* ctx = new (std::nothrow) CVDVContext();
  if (!ctx) return nullptr;
  Context* c = C(ctx);
  if (numReg <= 0 || numQubits == nullptr) return ctx;  // empty context (context.cu:10-12)
  if (numReg > kMaxRegs) {
    set_error(c, kErrInvalidArg, "cvdvCreate: %d registers (max %d)", numReg, kMaxRegs);
    return ctx;
  }
  if (precision != kC128 && precision != kC64) {
    set_error(c, kErrInvalidArg, "cvdvCreate: unknown precision %d", precision);
    return ctx;
  }
  int total = 0, qmax = 1;
  for (int r = 0; r < numReg; ++r) {
    if (numQubits[r] < 1 || numQubits[r] > kMaxTotalQubits) {
      set_error(c, kErrInvalidArg, "cvdvCreate: register %d has %d qubits", r, numQubits[r]);
      return ctx;
    }
    total += numQubits[r];
    if (numQubits[r] > qmax) qmax = numQubits[r];
  }
  if (total > kMaxTotalQubits) {
    set_error(c, kErrInvalidArg, "cvdvCreate: %d total qubits (max %d)", total, kMaxTotalQubits);
    return ctx;
  }
  c->precision = precision;
  c->elemBytes = precision == kC128 ? 16 : 8;
  c->numReg = numReg;
  c->totalQbt = total;
  c->q.assign(numQubits, numQubits + numReg);
  c->flw.assign(numReg, 0);
  c->dx.assign(numReg, 0.0);
  for (int r = 0; r < numReg; ++r) {
    int f = 0;
    for (int s = r + 1; s < numReg; ++s) f += numQubits[s];
    c->flw[r] = f;
    c->dx[r] = sqrt(2.0 * PI / (double)(1 << numQubits[r]));  // context.cu:30-31
  }
  cudaGetDevice(&c->device);
  if (cudaDeviceGetAttribute(&c->numSMs, cudaDevAttrMultiProcessorCount, c->device) != cudaSuccess ||
      c->numSMs < 1) {
    cudaGetLastError();
    c->numSMs = 148;
  }
  if (!cuda_ok(c, cudaStreamCreate(&c->stream), "cvdvCreate stream")) {
    c->numReg = 0;
    return ctx;
  }
  if (!make_twiddle(c, qmax < 3 ? 3 : qmax)) {
    c->numReg = 0;
    return ctx;
  }
  size_t cap = 16ull << 20;
  if (cudaMalloc((void**)&c->arena, cap) == cudaSuccess) c->arenaCap = cap;
  else cudaGetLastError();
  if (!cuda_ok(c, cudaHostAlloc((void**)&c->waitErr, 64, cudaHostAllocMapped), "cvdvCreate wait flag")) {
    c->waitErr = nullptr;
    c->numReg = 0;
    return ctx;
  }
  *c->waitErr = 0;
  // load the device code of cvdvMeasureMultipleNoAlloc on this device now, so
  // that its first call takes no device memory (a failure shows up there)
  no_alloc_prepare(c->device, false);
  return ctx;
}

CVDVContext* cvdvCreate(int numReg, int* numQubits) {
  return cvdvCreateEx(numReg, numQubits, kC128);
}

}  // extern "C"

namespace cvdv {

Context* factor_context(Context* ctx, int r) {
  if ((int)ctx->factorCtx.size() < ctx->numReg) ctx->factorCtx.resize(ctx->numReg, nullptr);
  if (ctx->factorCtx[r]) return ctx->factorCtx[r];
  int q = ctx->q[r];
  CVDVContext* h = cvdvCreateEx(1, &q, kC128);
  if (!h) {
    set_error(ctx, kErrAlloc, "register %d context: out of host memory", r);
    return nullptr;
  }
  Context* f = h;
  if (f->numReg != 1) {
    set_error(ctx, f->lastErr != kOk ? f->lastErr : kErrAlloc, "register %d context: %s", r,
              f->lastMsg.c_str());
    cvdvDestroy(h);
    return nullptr;
  }
  cudaStreamSynchronize(f->stream);  // its twiddle table
  cudaStreamDestroy(f->stream);
  f->stream = ctx->stream;  // stream order keeps its kernels between this context's
  cudaFreeHost(f->waitErr);
  f->waitErr = ctx->waitErr;  // its kernels' failed waits show at this context's syncs
  ctx->factorCtx[r] = f;
  return f;
}

}  // namespace cvdv

extern "C" {

static void release(Context* c) {
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (Context* f : c->factorCtx)
    if (f) {
      f->stream = nullptr;  // this context's stream and wait flag, released with it
      f->waitErr = nullptr;
      cvdvDestroy(static_cast<CVDVContext*>(f));
    }
  c->factorCtx.clear();
  if (c->factors) cudaFree(c->factors);
  c->factors = nullptr;
  c->factorsCap = 0;
  c->productPending = false;
  for (int k = 0; k < 2; ++k) {
    if (c->buf[k]) cudaFree(c->buf[k]);
    c->buf[k] = nullptr;
  }
  if (c->twiddle) cudaFree(c->twiddle);
  c->twiddle = nullptr;
  if (c->arena) cudaFree(c->arena);
  c->arena = nullptr;
  c->arenaCap = c->arenaTop = 0;
  for (auto& b : c->arenaExtra) cudaFree(b.p);
  c->arenaExtra.clear();
  if (c->big) cudaFree(c->big);
  if (c->rowSumBuf) cudaFree(c->rowSumBuf);
  c->big = nullptr;
  c->bigCap = 0;
  if (c->waitErr) cudaFreeHost(c->waitErr);
  c->waitErr = nullptr;
  for (void*& p : c->tcImage) {
    if (p) cudaFree(p);
    p = nullptr;
  }
  if (c->hostScratch) cudaFreeHost(c->hostScratch);
  c->hostScratch = nullptr;
  c->hostScratchCap = 0;
  c->allocElems = 0;
  c->initialized = false;
  c->pending.clear();
}

void cvdvDestroy(CVDVContext* ctx) {
  if (!ctx) return;
  Context* c = C(ctx);
  release(c);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete ctx;
}

void cvdvFree(CVDVContext* ctx) {
  if (!ctx) return;
  Context* c = C(ctx);
  release(c);
  c->numReg = 0;
  c->totalQbt = 0;
  c->q.clear();
  c->flw.clear();
  c->dx.clear();
}

void cvdvInitFromSeparable(CVDVContext* ctx, void** devicePtrs, int numReg) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (c->numReg == 0) {
    set_error(c, kErrNotInitialized,
              "cvdvInitFromSeparable: create the context with registers first");
    return;
  }
  if (numReg != c->numReg || devicePtrs == nullptr) {
    set_error(c, kErrInvalidArg, "cvdvInitFromSeparable: numReg mismatch (context %d, got %d)",
              c->numReg, numReg);
    return;
  }
  for (int r = 0; r < numReg; ++r)
    if (!devicePtrs[r]) {
      set_error(c, kErrInvalidArg, "cvdvInitFromSeparable: register %d pointer is NULL", r);
      return;
    }
  c->pending.clear();  // a new state replaces whatever the queued gates would have produced
  c->productPending = false;
  if (!ensure_state(c)) return;
  size_t totalN = 0;
  for (int r = 0; r < numReg; ++r) totalN += (size_t)1 << c->q[r];
  if (c->deferProduct && numReg >= 2) {
    // keep the arrays; the next flush forms the product (context.cu, form_product)
    if (c->factorsCap < totalN) {
      if (c->factors) cudaFree(c->factors);
      c->factors = nullptr;
      c->factorsCap = 0;
      if (cudaMalloc((void**)&c->factors, totalN * sizeof(double2)) != cudaSuccess) {
        cudaGetLastError();
        set_error(c, kErrAlloc, "cvdvInitFromSeparable: register arrays (%zu bytes)",
                  totalN * sizeof(double2));
        return;
      }
      c->factorsCap = totalN;
    }
    size_t off = 0;
    for (int r = 0; r < numReg; ++r) {
      size_t N = (size_t)1 << c->q[r];
      if (!cuda_ok(c, cudaMemcpyAsync(c->factors + off, devicePtrs[r], N * sizeof(double2),
                                      cudaMemcpyDefault, c->stream),
                   "cvdvInitFromSeparable copy"))
        return;
      off += N;
    }
    c->productPending = true;
    c->initialized = true;
    return;
  }
  arena_reset(c);
  double2* base = (double2*)arena_alloc(c, totalN * sizeof(double2));
  if (!base) return;
  std::vector<const double2*> arrs(numReg);
  size_t off = 0;
  for (int r = 0; r < numReg; ++r) {
    size_t N = (size_t)1 << c->q[r];
    if (!cuda_ok(c, cudaMemcpyAsync(base + off, devicePtrs[r], N * sizeof(double2),
                                    cudaMemcpyDefault, c->stream),
                 "cvdvInitFromSeparable copy"))
      return;
    arrs[r] = base + off;
    off += N;
  }
  if (!launch_init_product(c, arrs.data())) return;
  c->initialized = true;
}

}  // extern "C"

extern "C" {

void cvdvSetStateFromDevicePtr(CVDVContext* ctx, void* d_src) {
  if (!ctx || !d_src) return;
  Context* c = C(ctx);
  c->pending.clear();
  c->productPending = false;
  if (!ensure_state(c)) return;
  uint64_t n = c->size();
  if (c->precision == kC128) {
    if (!cuda_ok(c, cudaMemcpyAsync(c->state(), d_src, n * sizeof(double2), cudaMemcpyDefault,
                                    c->stream),
                 "cvdvSetStateFromDevicePtr"))
      return;
  } else {
    // stage the complex128 source in the second buffer (2 x the c64 size), convert
    void* tmp = big_scratch(c, n * sizeof(double2));
    if (!tmp) return;
    if (!cuda_ok(c, cudaMemcpyAsync(tmp, d_src, n * sizeof(double2), cudaMemcpyDefault,
                                    c->stream),
                 "cvdvSetStateFromDevicePtr"))
      return;
    if (!launch_convert_c128_to_c64(c, (const double2*)tmp, (float2*)c->state(), n)) return;
  }
  cudaStreamSynchronize(c->stream);  // the caller may free the source on return
  c->initialized = true;
}

int cvdvGetNumRegisters(CVDVContext* ctx) { return ctx ? C(ctx)->numReg : 0; }

size_t cvdvGetTotalSize(CVDVContext* ctx) {
  if (!ctx || C(ctx)->numReg == 0) return ctx ? 1 : 0;  // 1 << 0, as the reference
  return (size_t)C(ctx)->size();
}

void cvdvGetRegisterInfo(CVDVContext* ctx, int* qubitCountsOut, double* gridStepsOut) {
  if (!ctx || C(ctx)->numReg == 0) return;
  Context* c = C(ctx);
  if (qubitCountsOut) memcpy(qubitCountsOut, c->q.data(), c->numReg * sizeof(int));
  if (gridStepsOut) memcpy(gridStepsOut, c->dx.data(), c->numReg * sizeof(double));
}

int cvdvGetRegisterDim(CVDVContext* ctx, int regIdx) {
  if (!ctx || regIdx < 0 || regIdx >= C(ctx)->numReg) return -1;
  return 1 << C(ctx)->q[regIdx];
}

double cvdvGetRegisterDx(CVDVContext* ctx, int regIdx) {
  if (!ctx || regIdx < 0 || regIdx >= C(ctx)->numReg) return -1.0;
  return C(ctx)->dx[regIdx];
}

int cvdvGetPrecision(CVDVContext* ctx) { return ctx ? C(ctx)->precision : -1; }

int cvdvGetLastError(CVDVContext* ctx, char* msg, int len);  // context_errors below

void cvdvSynchronize(CVDVContext* ctx) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!flush(c)) return;
  if (c->stream) stream_sync(c, "cvdvSynchronize");
}

void cvdvFlush(CVDVContext* ctx) {
  if (!ctx) return;
  flush(C(ctx));
}

int cvdvPendingStages(CVDVContext* ctx) { return ctx ? (int)C(ctx)->pending.size() : 0; }

void* cvdvGetStateDevicePtr(CVDVContext* ctx) {
  if (!ctx) return nullptr;
  Context* c = C(ctx);
  if (!c->initialized || !flush(c)) return nullptr;
  return c->state();
}

void* cvdvGetStream(CVDVContext* ctx) { return ctx ? (void*)C(ctx)->stream : nullptr; }

unsigned long long cvdvLaunchCount(void) { return cvdv::g_launches.load(); }

void cvdvSetFusion(CVDVContext* ctx, int flags) {
  if (!ctx) return;
  C(ctx)->cancelFt = (flags & 1) != 0;
  C(ctx)->fuseSeq = (flags & 2) != 0;
  C(ctx)->colFft = (flags & 4) != 0;
  C(ctx)->colProg = (flags & 8) != 0;
  C(ctx)->deferProduct = (flags & 16) != 0;
  C(ctx)->tcCol = (flags & 32) != 0;
}

long long cvdvCancelledTransforms(CVDVContext* ctx) { return ctx ? C(ctx)->ftCancelled * 2 : 0; }

void cvdvSetTiming(CVDVContext* ctx, int on) {
  if (!ctx) return;
  Context* c = C(ctx);
  harvest_timing(c);
  c->timing = on != 0;
}

int cvdvGetKernelStats(CVDVContext* ctx, double* msOut, long long* countOut, int n) {
  if (!ctx) return 0;
  Context* c = C(ctx);
  harvest_timing(c);
  int k = n < kKindCount ? n : kKindCount;
  for (int i = 0; i < k; ++i) {
    if (msOut) msOut[i] = c->kindMs[i];
    if (countOut) countOut[i] = c->kindCount[i];
    c->kindMs[i] = 0.0;
    c->kindCount[i] = 0;
  }
  return kKindCount;
}

// ====================================================================== gates
void cvdvFtQ2P(CVDVContext* ctx, int regIdx) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!reg_ok(c, regIdx, "cvdvFtQ2P") || !gate_ready(c, "cvdvFtQ2P")) return;
  queue_ft(c, regIdx, 1);
}

void cvdvFtP2Q(CVDVContext* ctx, int regIdx) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!reg_ok(c, regIdx, "cvdvFtP2Q") || !gate_ready(c, "cvdvFtP2Q")) return;
  queue_ft(c, regIdx, -1);
}

void cvdvDisplacement(CVDVContext* ctx, int regIdx, double betaRe, double betaIm) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!reg_ok(c, regIdx, "cvdvDisplacement") || !gate_ready(c, "cvdvDisplacement")) return;
  if (fabs(betaIm) > 1e-12) push_diag(c, {poly(regIdx, 1, SQRT2 * betaIm)});
  if (fabs(betaRe) > 1e-12) {
    queue_ft(c, regIdx, 1);
    push_diag(c, {poly(regIdx, 1, -SQRT2 * betaRe)});
    queue_ft(c, regIdx, -1);
  }
}

void cvdvConditionalDisplacement(CVDVContext* ctx, int targetReg, int ctrlReg, int ctrlQubit,
                                 double alphaRe, double alphaIm) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvConditionalDisplacement";
  if (!reg_ok(c, targetReg, w) || !qubit_ok(c, ctrlReg, ctrlQubit, w) || !gate_ready(c, w))
    return;
  int cb = qubit_bit(c, ctrlReg, ctrlQubit);
  if (fabs(alphaIm) > 1e-12) push_diag(c, {poly(targetReg, 1, SQRT2 * alphaIm, cb)});
  if (fabs(alphaRe) > 1e-12) {
    queue_ft(c, targetReg, 1);
    push_diag(c, {poly(targetReg, 1, -SQRT2 * alphaRe, cb)});
    queue_ft(c, targetReg, -1);
  }
}

void cvdvPauliRotation(CVDVContext* ctx, int regIdx, int qubitIdx, int axis, double theta) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvPauliRotation";
  if (!qubit_ok(c, regIdx, qubitIdx, w) || !gate_ready(c, w)) return;
  if (axis < 0 || axis > 2) {
    set_error(c, kErrInvalidArg, "%s: axis %d", w, axis);
    return;
  }
  queue_pauli(c, regIdx, qubitIdx, axis, theta);
}

void cvdvHadamard(CVDVContext* ctx, int regIdx, int qubitIdx) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvHadamard";
  if (!qubit_ok(c, regIdx, qubitIdx, w) || !gate_ready(c, w)) return;
  const double h = 1.0 / SQRT2;  // gates.cuh:103
  queue_pair(c, qubit_bit(c, regIdx, qubitIdx), make_double2(h, 0), make_double2(h, 0),
             make_double2(h, 0), make_double2(-h, 0));
}

void cvdvParity(CVDVContext* ctx, int regIdx) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!reg_ok(c, regIdx, "cvdvParity") || !gate_ready(c, "cvdvParity")) return;
  queue_perm(c, kPermParity, regIdx, -1, -1);
}

void cvdvConditionalParity(CVDVContext* ctx, int targetReg, int ctrlReg, int ctrlQubit) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvConditionalParity";
  if (!reg_ok(c, targetReg, w) || !qubit_ok(c, ctrlReg, ctrlQubit, w) || !gate_ready(c, w))
    return;
  queue_perm(c, kPermCondParity, targetReg, -1, qubit_bit(c, ctrlReg, ctrlQubit));
}

void cvdvSwapRegisters(CVDVContext* ctx, int reg1, int reg2) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvSwapRegisters";
  if (!reg_ok(c, reg1, w) || !reg_ok(c, reg2, w) || !gate_ready(c, w)) return;
  if (c->q[reg1] != c->q[reg2]) {
    set_error(c, kErrInvalidArg, "%s: registers need the same number of qubits", w);
    return;
  }
  if (reg1 == reg2) return;
  queue_perm(c, kPermSwap, reg1, reg2, -1);
}

void cvdvPhaseSquare(CVDVContext* ctx, int regIdx, double t) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!reg_ok(c, regIdx, "cvdvPhaseSquare") || !gate_ready(c, "cvdvPhaseSquare")) return;
  push_diag(c, {poly(regIdx, 2, t)});
}

void cvdvPhaseCubic(CVDVContext* ctx, int regIdx, double t) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!reg_ok(c, regIdx, "cvdvPhaseCubic") || !gate_ready(c, "cvdvPhaseCubic")) return;
  push_diag(c, {poly(regIdx, 3, t)});
}

void cvdvRotation(CVDVContext* ctx, int regIdx, double theta) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!reg_ok(c, regIdx, "cvdvRotation") || !gate_ready(c, "cvdvRotation")) return;
  double theta0 = c_rint(theta / (PI / 2.0)) * (PI / 2.0);
  double rem = theta - theta0;
  int qt = (int)c_rint(theta0 / (PI / 2.0));
  qt = ((qt % 4) + 4) % 4;
  if (qt == 1) queue_ft(c, regIdx, 1);
  else if (qt == 2) queue_perm(c, kPermParity, regIdx, -1, -1);
  else if (qt == 3) queue_ft(c, regIdx, -1);
  rotation_small(c, regIdx, rem);
}

void cvdvConditionalRotation(CVDVContext* ctx, int targetReg, int ctrlReg, int ctrlQubit,
                             double theta) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvConditionalRotation";
  if (!reg_ok(c, targetReg, w) || !qubit_ok(c, ctrlReg, ctrlQubit, w) || !gate_ready(c, w))
    return;
  int cb = qubit_bit(c, ctrlReg, ctrlQubit);
  double theta0 = c_rint(theta / (PI / 2.0)) * (PI / 2.0);
  double rem = theta - theta0;
  int qt = (int)c_rint(theta0 / (PI / 2.0));
  qt = ((qt % 4) + 4) % 4;
  if (qt == 1) {
    queue_ft(c, targetReg, 1);
    queue_perm(c, kPermCondParity, targetReg, -1, cb);
    queue_pauli(c, ctrlReg, ctrlQubit, 2, PI / 2);
  } else if (qt == 2) {
    queue_perm(c, kPermParity, targetReg, -1, -1);
    queue_pauli(c, ctrlReg, ctrlQubit, 2, PI);
  } else if (qt == 3) {
    queue_ft(c, targetReg, -1);
    queue_perm(c, kPermCondParity, targetReg, -1, cb);
    queue_pauli(c, ctrlReg, ctrlQubit, 2, -PI / 2);
  }
  crotation_small(c, targetReg, cb, rem);
}

void cvdvSqueeze(CVDVContext* ctx, int regIdx, double r) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!reg_ok(c, regIdx, "cvdvSqueeze") || !gate_ready(c, "cvdvSqueeze")) return;
  double a = exp(0.5 * r), b = exp(-0.5 * r), s = sqrt(fabs(exp(r) - 1.0));
  double sg = (r >= 0) ? 1.0 : -1.0;
  queue_ft(c, regIdx, 1);
  push_diag(c, {poly(regIdx, 2, -0.5 * a * s)});
  queue_ft(c, regIdx, -1);
  push_diag(c, {poly(regIdx, 2, 0.5 * b * s * sg)});
  queue_ft(c, regIdx, 1);
  push_diag(c, {poly(regIdx, 2, 0.5 * b * s)});
  queue_ft(c, regIdx, -1);
  push_diag(c, {poly(regIdx, 2, -0.5 * a * s * sg)});
}

void cvdvConditionalSqueeze(CVDVContext* ctx, int targetReg, int ctrlReg, int ctrlQubit,
                            double r) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvConditionalSqueeze";
  if (!reg_ok(c, targetReg, w) || !qubit_ok(c, ctrlReg, ctrlQubit, w) || !gate_ready(c, w))
    return;
  int cb = qubit_bit(c, ctrlReg, ctrlQubit);
  double ch = cosh(r), sh = sinh(r), s = sqrt(2.0 * fabs(sinh(0.5 * r)));
  push_diag(c, {poly(targetReg, 2, 0.5 * s * ch), poly(targetReg, 2, -0.5 * s * sh, cb)});
  queue_ft(c, targetReg, 1);
  push_diag(c, {poly(targetReg, 2, 0.5 * (ch - 1) / s), poly(targetReg, 2, 0.5 * sh / s, cb)});
  queue_ft(c, targetReg, -1);
  push_diag(c, {poly(targetReg, 2, -0.5 * s)});
  queue_ft(c, targetReg, 1);
  push_diag(c, {poly(targetReg, 2, 0.5 * (ch - 1) / s), poly(targetReg, 2, -0.5 * sh / s, cb)});
  queue_ft(c, targetReg, -1);
}

void cvdvBeamSplitter(CVDVContext* ctx, int reg1, int reg2, double theta) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvBeamSplitter";
  if (!reg_ok(c, reg1, w) || !reg_ok(c, reg2, w) || !gate_ready(c, w)) return;
  if (reg1 == reg2) {
    set_error(c, kErrInvalidArg, "%s: needs two different registers", w);
    return;
  }
  double theta0 = c_round(theta / PI) * PI;
  double rem = theta - theta0;
  int ht = (int)c_round(theta0 / PI);
  ht = ((ht % 4) + 4) % 4;
  bool sameQ = c->q[reg1] == c->q[reg2];
  if (ht == 1) {
    queue_ft(c, reg1, 1);
    queue_ft(c, reg2, 1);
    if (sameQ) queue_perm(c, kPermSwap, reg1, reg2, -1);
  } else if (ht == 2) {
    queue_perm(c, kPermParity, reg1, -1, -1);
    queue_perm(c, kPermParity, reg2, -1, -1);
  } else if (ht == 3) {
    queue_ft(c, reg1, -1);
    queue_ft(c, reg2, -1);
    if (sameQ) queue_perm(c, kPermSwap, reg1, reg2, -1);
  }
  if ((ht == 1 || ht == 3) && !sameQ)
    set_error(c, kErrInvalidArg, "%s: swap needs registers with the same number of qubits", w);
  bs_small(c, reg1, reg2, rem, -1);
}

void cvdvConditionalBeamSplitter(CVDVContext* ctx, int reg1, int reg2, int ctrlReg, int ctrlQubit,
                                 double theta) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvConditionalBeamSplitter";
  if (!reg_ok(c, reg1, w) || !reg_ok(c, reg2, w) || !qubit_ok(c, ctrlReg, ctrlQubit, w) ||
      !gate_ready(c, w))
    return;
  if (reg1 == reg2) {
    set_error(c, kErrInvalidArg, "%s: needs two different registers", w);
    return;
  }
  int cb = qubit_bit(c, ctrlReg, ctrlQubit);
  double theta0 = c_round(theta / PI) * PI;
  double rem = theta - theta0;
  int ht = (int)c_round(theta0 / PI);
  ht = ((ht % 4) + 4) % 4;
  bool sameQ = c->q[reg1] == c->q[reg2];
  if (ht == 1 || ht == 3) {
    int d = ht == 1 ? 1 : -1;
    queue_ft(c, reg1, d);
    queue_ft(c, reg2, d);
    queue_perm(c, kPermCondParity, reg1, -1, cb);
    queue_perm(c, kPermCondParity, reg2, -1, cb);
    if (sameQ) queue_perm(c, kPermSwap, reg1, reg2, -1);
    else set_error(c, kErrInvalidArg, "%s: swap needs registers with the same number of qubits", w);
  } else if (ht == 2) {
    queue_perm(c, kPermParity, reg1, -1, -1);
    queue_perm(c, kPermParity, reg2, -1, -1);
  }
  bs_small(c, reg1, reg2, rem, cb);
}

void cvdvQ1Q2Gate(CVDVContext* ctx, int reg1, int reg2, double coeff) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvQ1Q2Gate";
  if (!reg_ok(c, reg1, w) || !reg_ok(c, reg2, w) || !gate_ready(c, w)) return;
  if (reg1 == reg2) {
    set_error(c, kErrInvalidArg, "%s: cannot couple a register with itself", w);
    return;
  }
  push_diag(c, {xx(reg1, reg2, coeff)});
}

}  // extern "C"
