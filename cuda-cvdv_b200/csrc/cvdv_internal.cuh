// Internal definitions shared by the libcvdv translation units.
//
// State layout in HBM: one contiguous array of 2^n complex amplitudes
// (complex128 = double2, or complex64 = float2 in the mixed-precision form),
// register 0 most significant, the last register fastest.  Register r owns the
// bit field [flw_r, flw_r + q_r) of the flat index; its local index is
// j_r = (i >> flw_r) & (N_r - 1) and its grid point x_j = (j - (N_r-1)/2) dx_r,
// dx_r = sqrt(2 pi / N_r)  (reference: src/cuda/context.cu:26-38,
// src/cuda/kernels/utils.cuh:5-7,34-37).
//
// Execution model: gate calls append stages to a per-context queue; a flush
// (any readout, state I/O, or an explicit cvdvSynchronize) plans the queue
// into kernels.  Runs of diagonal stages become factor lists that ride on the
// neighbouring kernel's load (pre) or store (post), so a diagonal gate never
// costs a pass of its own unless nothing else is queued.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>
#include <vector>

#ifndef CVDV_PI
#define CVDV_PI 3.14159265358979323846
#endif

namespace cvdv {

// ----------------------------------------------------------------- limits
constexpr int kMaxRegs = 64;          // registers per context
constexpr int kMaxTotalQubits = 34;   // n <= 34 (c64: 128 GiB per buffer)
constexpr int kMaxTab = 6;            // table factors per factor list
constexpr int kMaxXX = 2;             // bilinear factors per factor list
constexpr int kMaxTermsPerTable = 24; // terms folded into one table
constexpr int kFftTile = 4096;        // complex elements per FFT tile (c128)

enum Precision : int { kC128 = 0, kC64 = 1 };

// Error codes returned by cvdvGetLastError (0 = none).
enum ErrCode : int {
  kOk = 0,
  kErrInvalidArg = 1,
  kErrNotInitialized = 2,
  kErrCuda = 3,
  kErrAlloc = 4,
  kErrUnsupported = 5,
};

// ----------------------------------------------------------------- complex helpers
template <typename T> struct Cx;
template <> struct Cx<double> { using t = double2; };
template <> struct Cx<float> { using t = float2; };

__host__ __device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }
__host__ __device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }

template <typename C>
__host__ __device__ __forceinline__ C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename C>
__host__ __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C>
__host__ __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C>
__host__ __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }

// complex from a double2 factor, in the compute type of C
template <typename C> __device__ __forceinline__ C fromd(double2 v);
template <> __device__ __forceinline__ double2 fromd<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ float2 fromd<float2>(double2 v) {
  return make_float2((float)v.x, (float)v.y);
}

// ----------------------------------------------------------------- factor lists
// A factor list is the product of a diagonal run evaluated at one flat index:
//   scalar * prod_t tab_t[idx_t(i)] * prod_x exp(i c s(i) x_r x_s)
// Tables are double2, built on the device by build_tables().
struct TabFactor {
  const double2* ptr;
  int shift;      // flw of the register
  int mask;       // N - 1
  int ctrlShift;  // global bit of a control qubit, -1 if none
  int half;       // N (offset of the ctrl=1 half)
  int conjHalf;   // the ctrl=1 half is the complex conjugate of the ctrl=0 half
};

struct XXFactor {
  int shift1, mask1, shift2, mask2;
  double c1, dx1, c2, dx2;  // x = (j - c) * dx
  double coeff;
  int ctrlShift;            // -1 if none
};

struct FactorList {
  int nTab;
  int nXX;
  int hasScalar;
  double2 scalar;
  TabFactor tab[kMaxTab];
  XXFactor xx[kMaxXX];
};

__device__ __forceinline__ double2 dmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Evaluate the factor at flat index i (FP64); an empty list gives 1.  XX = false
// leaves out the bilinear terms (lists the caller knows have none).
template <int MAXT = kMaxTab, bool XX = true>
__device__ __forceinline__ double2 eval_factor_t(const FactorList& F, uint64_t i) {
  double2 f = F.hasScalar ? F.scalar : make_double2(1.0, 0.0);
  // issue every table load before the products so they overlap
  double2 tv[MAXT];
#pragma unroll
  for (int t = 0; t < MAXT; ++t) {
    if (t < F.nTab) {
      const TabFactor& T = F.tab[t];
      int j = (int)((i >> T.shift) & (uint64_t)T.mask);
      if (T.ctrlShift >= 0) j += (int)((i >> T.ctrlShift) & 1ull) * T.half;
      tv[t] = __ldg(T.ptr + j);
    }
  }
#pragma unroll
  for (int t = 0; t < MAXT; ++t)
    if (t < F.nTab) f = dmul(f, tv[t]);
  if constexpr (XX) {
#pragma unroll 1
    for (int t = 0; t < F.nXX; ++t) {
      const XXFactor& X = F.xx[t];
      int j1 = (int)((i >> X.shift1) & (uint64_t)X.mask1);
      int j2 = (int)((i >> X.shift2) & (uint64_t)X.mask2);
      double x1 = ((double)j1 - X.c1) * X.dx1;
      double x2 = ((double)j2 - X.c2) * X.dx2;
      double ph = X.coeff * x1 * x2;
      if (X.ctrlShift >= 0 && ((i >> X.ctrlShift) & 1ull)) ph = -ph;
      double s, c;
      sincos(ph, &s, &c);
      f = dmul(f, make_double2(c, s));
    }
  }
  return f;
}

__device__ __forceinline__ double2 eval_factor(const FactorList& F, uint64_t i) {
  return eval_factor_t<kMaxTab, true>(F, i);
}

__host__ __device__ __forceinline__ bool factor_empty(const FactorList& F) {
  return F.nTab == 0 && F.nXX == 0 && !F.hasScalar;
}

// ----------------------------------------------------------------- stages
enum TermKind : int {
  kTermPoly = 0,   // coeff * x_r^power, optionally * Z(ctrl)
  kTermFtTw = 1,   // exact centred-grid FT twiddle exp(i sign pi (N-1)(2j-N+1)/(2N))
  kTermBit = 2,    // g0 if bit(j) == 0 else g1   (qubit-diagonal gates)
  kTermXX = 3,     // coeff * x_r * x_s, optionally * Z(ctrl)
  kTermScalar = 4, // global complex scalar
};

struct Term {
  int kind;
  int r, s;        // registers
  int ctrlBit;     // global bit index or -1
  int power;       // 1..3 for kTermPoly
  int sign;        // +-1 for kTermFtTw
  int bit;         // bit inside register r for kTermBit
  double coeff;
  double2 g0, g1;  // kTermBit factors / kTermScalar value (g0)
};

enum StageKind : int { kStDiag = 0, kStFft = 1, kStPair = 2, kStPerm = 3 };
enum PermKind : int { kPermParity = 0, kPermCondParity = 1, kPermSwap = 2 };

struct Stage {
  int kind;
  int ftTag = 0;      // > 0: one of the three stages of one FtQ2P / FtP2Q
  int ftReg = -1;     // register of that basis change
  int ftDir = 0;      // its direction (+1 FtQ2P, -1 FtP2Q)
  int reg = -1, reg2 = -1;
  int dir = 1;        // FFT: +1 forward (e^{-2 pi i jk/N}), -1 inverse (unnormalised)
  int bit = -1;       // pair: global bit; perm: control bit
  int perm = 0;       // PermKind
  double2 m[4];       // pair matrix row-major
  std::vector<Term> terms;  // diag
};

// ----------------------------------------------------------------- context
struct ArenaBlock {
  char* p;
  size_t cap;
  size_t top;
};

// Kernel kinds for the optional per-launch timing (cvdvSetTiming).
enum KernelKind : int {
  kKFft = 0,
  kKPair = 1,
  kKDiag = 2,
  kKPerm = 3,
  kKTable = 4,
  kKInit = 5,
  kKReduce = 6,
  kKPhaseSpace = 7,
  kKSeq = 8,
  kKCol = 9,
  kKColTc = 10,  // column passes on the tensor cores
  kKindCount = 11,
};

struct TimingRec {
  cudaEvent_t a, b;
  int kind;
};

struct Context {
  // per-launch timing (off by default): event pairs around every launch
  bool timing = false;
  std::vector<TimingRec> timingRecs;
  std::vector<cudaEvent_t> eventPool;
  double kindMs[kKindCount] = {};
  long long kindCount[kKindCount] = {};

  int numReg = 0;
  int totalQbt = 0;
  int precision = kC128;
  size_t elemBytes = 16;
  std::vector<int> q, flw;
  std::vector<double> dx;

  // state: ping-pong buffers; cur indexes the live one
  void* buf[2] = {nullptr, nullptr};
  int cur = 0;
  size_t allocElems = 0;
  bool initialized = false;

  cudaStream_t stream = nullptr;
  int numSMs = 148;  // of the context's device
  int device = 0;

  // twiddle table W[m] = exp(-2 pi i m / twN) for the largest register
  double2* twiddle = nullptr;
  int twN = 0;

  // device scratch arena (tables, partial sums, readout buffers)
  char* arena = nullptr;
  size_t arenaCap = 0;
  size_t arenaTop = 0;
  std::vector<ArenaBlock> arenaExtra;  // chained when a flush outgrows the arena
  // large scratch (Wigner / Husimi work areas)
  void* big = nullptr;
  size_t bigCap = 0;

  // pinned host staging for small D2H results
  double* hostScratch = nullptr;
  size_t hostScratchCap = 0;

  std::vector<Stage> pending;
  // Basis-change cancellation: FtQ2P(r) after FtP2Q(r) (or the reverse) with only
  // stages that leave register r untouched in between is the identity; both are
  // dropped from the queue.  On by default (cvdvSetFusion).
  bool cancelFt = true;
  bool fuseSeq = true;  // run chains of qubit gates as one qubit-gate sequence pass
  bool colFft = true;   // transforms of strided registers by the register-resident column kernel
  bool colProg = true;  // programs on strided registers by the register-resident row kernel in column form
  bool tcCol = false;   // complex64 column passes of 2^12..2^14-point registers on the tensor cores (opt-in)
  void* tcImage[2] = {nullptr, nullptr};  // their DFT matrices (64-point blocks, 128-point), made on first use
  // Product deferral (on by default, cvdvSetFusion bit 4): cvdvInitFromSeparable
  // keeps the register arrays and the next flush forms the product, after the
  // queued stages that act on one register alone, ahead of every stage that
  // couples it to another register, have run on that register's array.
  bool deferProduct = true;
  bool productPending = false;
  double2* factors = nullptr;       // the register arrays, concatenated (complex128)
  size_t factorsCap = 0;            // in elements
  std::vector<Context*> factorCtx;  // one-register contexts for them, made on first use
  // Inside one flush, between a forward and an inverse 2^14-point transform of
  // the last register run by a cluster row kernel of C = 2^permLogC CTAs, that
  // register may be stored "blocked": position r M + k2 (M = N / C) holds logical
  // index r + C k2 (each CTA's natural output order).  While permReg >= 0, tables
  // over it are built permuted.
  int permReg = -1;
  int permLogC = 0;
  // Inside one flush: the product state not yet written; the first qubit-gate
  // sequence forms each amplitude as last[i mod N_last] * outer[i / N_last] from
  // these tables instead of reading the state (set by flush, taken by launch_seq)
  const double2* seqProdLast = nullptr;
  const double2* seqProdOuter = nullptr;
  // Set by a marginal readout of registers above the last one before it flushes:
  // a row program on the last register that ends the flush also writes each
  // row's sum of |psi|^2 there (rowSumParts partials per row; 0 = not written).
  double* rowSums = nullptr;
  int rowSumParts = 0;
  double* rowSumBuf = nullptr;  // owned buffer for them
  size_t rowSumCap = 0;         // in doubles
  int nextFtTag = 1;
  long long ftCancelled = 0;

  int lastErr = kOk;
  std::string lastMsg;
  // Mapped pinned word a kernel sets when a bounded wait on its cluster peers
  // gives up; read on the host after every synchronisation (stream_sync).
  unsigned int* waitErr = nullptr;

  uint64_t size() const { return 1ull << totalQbt; }
  void* state() const { return buf[cur]; }
  void* other() const { return buf[cur ^ 1]; }
};

// ----------------------------------------------------------------- host helpers (context.cu)
// Every kernel launch of the library is bracketed by a LaunchScope: it counts
// the launch (cvdvLaunchCount) and, when timing is on, records an event pair.
void launch_begin(Context* ctx, int kind);
void launch_end(Context* ctx);
struct LaunchScope {
  Context* c;
  LaunchScope(Context* ctx, int kind) : c(ctx) { launch_begin(ctx, kind); }
  ~LaunchScope() { launch_end(c); }
};
void harvest_timing(Context* ctx);
extern std::atomic<unsigned long long> g_launches;

void set_error(Context* ctx, int code, const char* fmt, ...);
bool cuda_ok(Context* ctx, cudaError_t e, const char* what);
// synchronise the context's stream and report a failed kernel-side wait
bool stream_sync(Context* ctx, const char* what);
void* arena_alloc(Context* ctx, size_t bytes);   // reset per flush / readout
void arena_reset(Context* ctx);
void* big_scratch(Context* ctx, size_t bytes);   // persistent, grown on demand
double* host_scratch(Context* ctx, size_t count);
bool ensure_state(Context* ctx);                  // allocate both buffers
// complex128 context of the one register r of ctx, on ctx's stream (api_gates.cu)
Context* factor_context(Context* ctx, int r);
bool flush(Context* ctx);                         // run pending stages
// scratch address of cvdvMeasureMultipleNoAlloc on device dev (current), with its
// device code loaded; nullptr on failure (recorded as the last error if report)
double* no_alloc_prepare(int dev, bool report);

// factor lists of a diagonal run (context.cu)
bool build_factor_list(Context* ctx, const std::vector<Term>& terms, FactorList* out,
                       std::vector<Term>* leftover);

// kernel launchers (kernels_*.cu); all enqueue on ctx->stream
bool launch_build_table(Context* ctx, int r, bool ctrl, const Term* terms, int nTerms,
                        double2* out);
// permLogC > 0 stores the table permuted for a cluster of 2^permLogC CTAs in the
// transposed layout: position rank * (N >> permLogC) + m holds index rank + (m << permLogC)
bool launch_build_table_ext(Context* ctx, int r, int nExt, const int* extBits, const Term* terms,
                            int nTerms, double2* out, int permLogC = 0);
bool launch_diag(Context* ctx, const FactorList& F);
bool launch_pair(Context* ctx, int bit, const double2 m[4], const FactorList& pre,
                 const FactorList& post);
bool launch_perm(Context* ctx, const Stage& st, const FactorList& pre, const FactorList& post);
bool launch_fft(Context* ctx, int reg, int dir, const FactorList& pre, const FactorList& post);
bool col_fft_ok(Context* ctx, int reg);
bool col_program_ok(Context* ctx, int reg);
bool tc_col_ok(Context* ctx, int reg);  // kernels_tc.cu
bool launch_col_fft(Context* ctx, int reg, int dir, const FactorList& pre, const FactorList& post);
bool launch_fft_generic(Context* ctx, const void* in, void* out, void* tmp, uint64_t O,
                        int q, uint64_t S, int dir, int prec);
bool launch_init_product(Context* ctx, const double2* const* regArrays);

// row programs (kernels_row.cu): FFTs and diagonal runs on the contiguous register
constexpr int kMaxRowOps = 24;
constexpr int kMaxRowDiags = 10;
enum RowOpKind : int { kRowDiag = 0, kRowFft = 1 };
struct HostRowOp {
  int kind;
  int dir;
  std::vector<Term> terms;
};
bool row_eligible(Context* ctx, int reg);
bool row_diag_fits(Context* ctx, int reg, const std::vector<Term>& terms);
// a run of transforms and diagonal runs on a strided register (kernels_col.cu)
bool launch_col_chain(Context* ctx, int reg, const std::vector<HostRowOp>& ops);
// blockedIn: the register is stored blocked and the program starts with an
// inverse transform; blockedOut: leave it blocked after the final forward transform
bool launch_row_program(Context* ctx, int reg, const std::vector<HostRowOp>& ops, bool blockedIn = false,
                        bool blockedOut = false, bool rowSums = false);
// largest number of row-sum partials per row a row program writes (32)
constexpr int kRowSumMaxParts = 32;
// whether launch_row_program runs this program on the cluster kernel (which can
// store and load the blocked layout)
bool rowc_takes(Context* ctx, int reg, const std::vector<HostRowOp>& ops);
int rowc_log_cluster();  // log2 CTAs per 2^14-point complex128 row (the blocked layout's permLogC)
// qubit-gate sequences (kernels_seq.cu): 2x2 gates on up to four bits and the
// diagonal runs between them in one pass
constexpr int kSeqMaxBits = 5;  // see seq_max_bits
constexpr int kSeqMaxOps = 24;
constexpr int kSeqMaxDiags = 10;
constexpr int kSeqMaxTabs = 4;
struct HostSeqOp {
  int kind;  // 0 pair (bit, m), 1 diagonal run (terms)
  int bit;
  double2 m[4];
  std::vector<Term> terms;
};
// whether a diagonal run can ride in a sequence over `bits` (global bit positions)
bool seq_diag_ok(Context* ctx, const std::vector<int>& bits, const std::vector<Term>& terms);
bool launch_seq(Context* ctx, const std::vector<HostSeqOp>& ops);
int seq_max_bits(Context* ctx);
// outer[h] = prod over registers but the last of phi_r[j_r(h)], h < 2^(n - q_last)
bool launch_outer(Context* ctx, const double2* const* regArrays, double2* outer);
// FFT of the live state along `reg` into `out` (state untouched); `tmp` is the
// temporary of a two-pass transform.  pre is applied on the first pass's load.
bool launch_fft_into(Context* ctx, int reg, int dir, const FactorList& pre, void* out, void* tmp);
int global_error(char* msg, int len);
bool make_twiddle(Context* ctx, int logN);
bool launch_convert_c128_to_c64(Context* ctx, const double2* src, float2* dst, uint64_t n);

}  // namespace cvdv
