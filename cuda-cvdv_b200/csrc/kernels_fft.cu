// q<->p basis change: a hand-written strided batched FFT along one register.
//
// A register of N = 2^q points with stride S = 2^flw is transformed by one or
// more out-of-place Stockham passes.  Pass k has radix R_k <= 4096 and works on
// tiles of R_k x B complex values (B adjacent "columns" of the batch); the tile
// is staged in shared memory, the inter-pass twiddle is applied on load, the
// length-R_k DFT runs as radix-8/4/2 Stockham stages between registers and
// shared memory, and the tile is written back in the autosorted position, so
// the last pass leaves the spectrum in natural order.  The centred-grid
// pre/post twiddles of the reference's FtQ2P/FtP2Q (src/cuda/gates.cu:19-122),
// the 1/sqrt(N) scale, the global phase and any neighbouring diagonal gates ride
// in the first pass's load and the last pass's store as factor lists.
//
// Load/store thread mapping: element (t, b) of a tile is visited in the order
// (b mod W) fastest, then t, then b / W, with W = min(B, memory stride of t).
// That order is the memory order, so every warp touches contiguous runs for
// contiguous registers (S = 1), inner registers and outer registers alike.

#include "cvdv_internal.cuh"

namespace cvdv {

constexpr int kFftThreads = 256;
constexpr int kFftPerThread = kFftTile / kFftThreads;  // 16 complex per thread

struct PassDesc {
  int logN, logR, logNs, logS, logB;
  int logWl, logWs;       // log2 of the load / store inner widths
  int first, last;        // apply pre / post factor lists
  int twShift;            // log2(twN) - log2(Ns*R): twiddle index scale for the pass twiddle
  int logTwN;
  const double2* tw;      // W[m] = exp(-2 pi i m / twN)
};

__device__ __forceinline__ int padt(int t) { return t + (t >> 3); }

template <typename C, int DIR>
__device__ __forceinline__ C twiddle(const double2* tw, int m) {
  double2 w = __ldg(tw + m);
  if (DIR < 0) w.y = -w.y;
  return fromd<C>(w);
}

// y_k = sum_u w^{uk} x_u with w = exp(-DIR*2 pi i / rho)
template <typename C, int DIR>
__device__ __forceinline__ void dft2(C& a, C& b) {
  C t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <typename C, int DIR>
__device__ __forceinline__ C mul_mi(C a) {  // multiply by -DIR*i  (= w4 for DIR=+1)
  return DIR > 0 ? mk(a.y, -a.x) : mk(-a.y, a.x);
}

template <typename C, int DIR>
__device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3) {
  C s02 = cadd(a0, a2), d02 = csub(a0, a2);
  C s13 = cadd(a1, a3), d13 = mul_mi<C, DIR>(csub(a1, a3));
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, d13);
  a3 = csub(d02, d13);
}

template <typename C, int DIR>
__device__ __forceinline__ void dft8(C* v) {
  using T = decltype(v[0].x);
  const T h = (T)0.70710678118654752440;
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<C, DIR>(e0, e1, e2, e3);
  dft4<C, DIR>(o0, o1, o2, o3);
  // w8^k, w8 = exp(-DIR i pi/4)
  C t1 = DIR > 0 ? mk(h * (o1.x + o1.y), h * (o1.y - o1.x)) : mk(h * (o1.x - o1.y), h * (o1.y + o1.x));
  C t2 = mul_mi<C, DIR>(o2);
  C t3 = DIR > 0 ? mk(h * (o3.y - o3.x), -h * (o3.x + o3.y)) : mk(-h * (o3.x + o3.y), h * (o3.x - o3.y));
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, t1);
  v[5] = csub(e1, t1);
  v[2] = cadd(e2, t2);
  v[6] = csub(e2, t2);
  v[3] = cadd(e3, t3);
  v[7] = csub(e3, t3);
}

// One Stockham stage inside the tile: radix RHO, previous product ns.
// Butterfly jb of a column reads x[jb + u R/RHO], multiplies by
// w_{ns RHO}^{(jb mod ns) u}, and writes y[(jb/ns) ns RHO + (jb mod ns) + v ns].
template <typename C, int DIR, int RHO>
__device__ __forceinline__ void tile_stage(C* sm, int RP, int logR, int logB, int logNs,
                                           const double2* tw, int logTwN) {
  constexpr int LOGRHO = RHO == 8 ? 3 : (RHO == 4 ? 2 : 1);
  constexpr int KMAX = kFftPerThread / RHO;
  const int logNbf = logR - LOGRHO;
  const int total = 1 << (logNbf + logB);
  const int ns = 1 << logNs;
  const int sc = logTwN - (logNs + LOGRHO);
  C v[KMAX][RHO];
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
    int bf = threadIdx.x + k * kFftThreads;
    if (bf < total) {
      int b = bf >> logNbf;
      int jb = bf & ((1 << logNbf) - 1);
      const C* col = sm + b * RP;
#pragma unroll
      for (int u = 0; u < RHO; ++u) v[k][u] = col[padt(jb + (u << logNbf))];
      int jm = jb & (ns - 1);
      if (jm) {
#pragma unroll
        for (int u = 1; u < RHO; ++u) v[k][u] = cmul(v[k][u], twiddle<C, DIR>(tw, (jm * u) << sc));
      }
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < KMAX; ++k) {
    int bf = threadIdx.x + k * kFftThreads;
    if (bf < total) {
      int b = bf >> logNbf;
      int jb = bf & ((1 << logNbf) - 1);
      if constexpr (RHO == 8) dft8<C, DIR>(v[k]);
      else if constexpr (RHO == 4) dft4<C, DIR>(v[k][0], v[k][1], v[k][2], v[k][3]);
      else dft2<C, DIR>(v[k][0], v[k][1]);
      C* col = sm + b * RP;
      int base = ((jb >> logNs) << (logNs + LOGRHO)) + (jb & (ns - 1));
#pragma unroll
      for (int u = 0; u < RHO; ++u) col[padt(base + u * ns)] = v[k][u];
    }
  }
  __syncthreads();
}

template <typename C, int DIR>
__global__ void __launch_bounds__(kFftThreads) k_fft_pass(const C* __restrict__ in,
                                                         C* __restrict__ out, PassDesc P,
                                                         FactorList pre, FactorList post) {
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  const int R = 1 << P.logR;
  const int RP = (padt(R) | 1);
  const int logNR = P.logN - P.logR;
  const uint64_t c0 = (uint64_t)blockIdx.x << P.logB;
  const uint64_t Smask = (1ull << P.logS) - 1;
  const uint64_t NRmask = (1ull << logNR) - 1;
  const int nsMask = (1 << P.logNs) - 1;
  const bool doPre = P.first && !factor_empty(pre);
  const bool doPost = P.last && !factor_empty(post);
  const int total = R << P.logB;

  // ---- load (memory order: inner b, t, outer b).  All of a thread's loads are
  // issued before any is used, so each thread keeps kFftPerThread requests in
  // flight.
  {
    const int Wl = 1 << P.logWl;
    C v[kFftPerThread];
#pragma unroll
    for (int k = 0; k < kFftPerThread; ++k) {
      int l = threadIdx.x + k * kFftThreads;
      if (l < total) {
        int inner = l & (Wl - 1);
        int t = (l >> P.logWl) & (R - 1);
        int b = ((l >> (P.logWl + P.logR)) << P.logWl) | inner;
        uint64_t c = c0 + b;
        uint64_t tmp = c >> P.logS;
        uint64_t addr = ((((tmp >> logNR) << P.logN) + (tmp & NRmask) + ((uint64_t)t << logNR))
                         << P.logS) + (c & Smask);
        v[k] = in[addr];
      }
    }
#pragma unroll
    for (int k = 0; k < kFftPerThread; ++k) {
      int l = threadIdx.x + k * kFftThreads;
      if (l < total) {
        int inner = l & (Wl - 1);
        int t = (l >> P.logWl) & (R - 1);
        int b = ((l >> (P.logWl + P.logR)) << P.logWl) | inner;
        uint64_t c = c0 + b;
        uint64_t tmp = c >> P.logS;
        uint64_t jj = tmp & NRmask;
        C x = v[k];
        if (doPre) {
          uint64_t addr = ((((tmp >> logNR) << P.logN) + jj + ((uint64_t)t << logNR)) << P.logS) +
                          (c & Smask);
          x = cmul(x, fromd<C>(eval_factor(pre, addr)));
        }
        int jm = (int)(jj & nsMask);
        if (jm && t) x = cmul(x, twiddle<C, DIR>(P.tw, (jm * t) << P.twShift));
        sm[b * RP + padt(t)] = x;
      }
    }
  }
  __syncthreads();

  // ---- length-R DFT of every column, radix 8 first
  {
    int logNs = 0;
    int rem = P.logR;
    while (rem >= 3) {
      tile_stage<C, DIR, 8>(sm, RP, P.logR, P.logB, logNs, P.tw, P.logTwN);
      logNs += 3;
      rem -= 3;
    }
    if (rem == 2) tile_stage<C, DIR, 4>(sm, RP, P.logR, P.logB, logNs, P.tw, P.logTwN);
    else if (rem == 1) tile_stage<C, DIR, 2>(sm, RP, P.logR, P.logB, logNs, P.tw, P.logTwN);
  }

  // ---- store (autosorted position)
  {
    const int Ws = 1 << P.logWs;
#pragma unroll
    for (int kk = 0; kk < kFftPerThread; ++kk) {
      int l = threadIdx.x + kk * kFftThreads;
      if (l < total) {
        int inner = l & (Ws - 1);
        int t = (l >> P.logWs) & (R - 1);
        int b = ((l >> (P.logWs + P.logR)) << P.logWs) | inner;
        uint64_t c = c0 + b;
        uint64_t s = c & Smask;
        uint64_t tmp = c >> P.logS;
        uint64_t jj = tmp & NRmask;
        uint64_t o = tmp >> logNR;
        uint64_t k = ((jj >> P.logNs) << (P.logNs + P.logR)) + (jj & (uint64_t)nsMask) +
                     ((uint64_t)t << P.logNs);
        uint64_t addr = (((o << P.logN) + k) << P.logS) + s;
        C v = sm[b * RP + padt(t)];
        if (doPost) v = cmul(v, fromd<C>(eval_factor(post, addr)));
        out[addr] = v;
      }
    }
  }
}

// ----------------------------------------------------------------- twiddle table
__global__ void k_twiddle(double2* W, int logN) {
  int N = 1 << logN;
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < N; m += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)m / (double)N, &s, &c);
    W[m] = make_double2(c, -s);
  }
}

bool make_twiddle(Context* ctx, int logN) {
  int N = 1 << logN;
  if (!cuda_ok(ctx, cudaMalloc(&ctx->twiddle, (size_t)N * sizeof(double2)), "twiddle alloc"))
    return false;
  ctx->twN = N;
  {
    LaunchScope _ls(ctx, kKTable);
    k_twiddle<<<(N + 255) / 256 < 1184 ? (N + 255) / 256 : 1184, 256, 0, ctx->stream>>>(ctx->twiddle,
                                                                                      logN);
  }
  return cuda_ok(ctx, cudaGetLastError(), "twiddle launch");
}

// ----------------------------------------------------------------- planning
static int ilog2u(uint64_t v) {
  int r = 0;
  while ((1ull << r) < v) ++r;
  return r;
}

// Split q into pass radices (log2), each <= 12.
static std::vector<int> pass_radices(int q, int logS) {
  std::vector<int> r;
  if (q <= 0) return r;
  bool single = q <= 12 && (logS == 0 || q <= 11);
  int p = single ? 1 : (q + 11) / 12;
  if (!single && p < 2) p = 2;
  int base = q / p, extra = q % p;
  for (int k = 0; k < p; ++k) r.push_back(base + (k < extra ? 1 : 0));
  return r;
}

template <typename C>
static bool run_passes(Context* ctx, const void* src, void* const* dsts, uint64_t O, int q,
                       int logS, int dir, const FactorList& pre, const FactorList& post) {
  std::vector<int> rad = pass_radices(q, logS);
  static const FactorList empty{};
  int logNs = 0;
  const void* in = src;
  uint64_t totalLog = (uint64_t)ilog2u(O) + q + logS;
  for (size_t k = 0; k < rad.size(); ++k) {
    PassDesc P{};
    P.logN = q;
    P.logR = rad[k];
    P.logNs = logNs;
    P.logS = logS;
    int logTile = ilog2u(kFftTile);
    int logB = logTile - P.logR;
    int logCols = (int)totalLog - P.logR;
    if (logB > logCols) logB = logCols;
    if (logB < 0) logB = 0;
    P.logB = logB;
    int logLoadStride = (q - P.logR) + logS;
    int logStoreStride = logNs + logS;
    P.logWl = logB < logLoadStride ? logB : logLoadStride;
    P.logWs = logB < logStoreStride ? logB : logStoreStride;
    P.first = k == 0;
    P.last = k + 1 == rad.size();
    P.logTwN = ilog2u((uint64_t)ctx->twN);
    P.twShift = P.logTwN - (logNs + P.logR);
    P.tw = ctx->twiddle;
    void* outp = dsts[k];
    uint64_t blocks = 1ull << (logCols - logB);
    int RP = (P.logR >= 3 ? ((1 << P.logR) + ((1 << P.logR) >> 3)) : (1 << P.logR)) | 1;
    size_t smem = (size_t)RP * (1ull << logB) * sizeof(C);
    const FactorList& fpre = P.first ? pre : empty;
    const FactorList& fpost = P.last ? post : empty;
    if (dir > 0) {
      cudaFuncSetAttribute(k_fft_pass<C, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      {
        LaunchScope _ls(ctx, kKFft);
        k_fft_pass<C, 1><<<(unsigned)blocks, kFftThreads, smem, ctx->stream>>>(
            (const C*)in, (C*)outp, P, fpre, fpost);
      }
    } else {
      cudaFuncSetAttribute(k_fft_pass<C, -1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem);
      {
        LaunchScope _ls(ctx, kKFft);
        k_fft_pass<C, -1><<<(unsigned)blocks, kFftThreads, smem, ctx->stream>>>(
            (const C*)in, (C*)outp, P, fpre, fpost);
      }
    }
    if (!cuda_ok(ctx, cudaGetLastError(), "fft pass launch")) return false;
    in = outp;
    logNs += P.logR;
  }
  return true;
}

// FFT along register `reg` of the live state (ping-pong buffers).
bool launch_fft(Context* ctx, int reg, int dir, const FactorList& pre, const FactorList& post) {
  if (ctx->colFft && col_fft_ok(ctx, reg)) return launch_col_fft(ctx, reg, dir, pre, post);
  int q = ctx->q[reg];
  int logS = ctx->flw[reg];
  uint64_t O = 1ull << (ctx->totalQbt - q - logS);
  std::vector<int> rad = pass_radices(q, logS);
  std::vector<void*> dsts;
  int c = ctx->cur;
  for (size_t k = 0; k < rad.size(); ++k) {
    c ^= 1;
    dsts.push_back(ctx->buf[c]);
  }
  bool ok = ctx->precision == kC128
                ? run_passes<double2>(ctx, ctx->state(), dsts.data(), O, q, logS, dir, pre, post)
                : run_passes<float2>(ctx, ctx->state(), dsts.data(), O, q, logS, dir, pre, post);
  if (ok) ctx->cur = c;
  return ok;
}

bool launch_fft_into(Context* ctx, int reg, int dir, const FactorList& pre, void* out, void* tmp) {
  int q = ctx->q[reg];
  int logS = ctx->flw[reg];
  uint64_t O = 1ull << (ctx->totalQbt - q - logS);
  std::vector<int> rad = pass_radices(q, logS);
  if (rad.size() > 2) return false;
  void* dsts[2];
  if (rad.size() == 1) {
    dsts[0] = out;
  } else {
    dsts[0] = tmp;
    dsts[1] = out;
  }
  static const FactorList empty{};
  return ctx->precision == kC128
             ? run_passes<double2>(ctx, ctx->state(), dsts, O, q, logS, dir, pre, empty)
             : run_passes<float2>(ctx, ctx->state(), dsts, O, q, logS, dir, pre, empty);
}

// FFT along the middle axis of an [O][2^q][S] array in a caller buffer, result in
// `out`; `tmp` must hold the same size when more than one pass is needed.
bool launch_fft_generic(Context* ctx, const void* in, void* out, void* tmp, uint64_t O, int q,
                        uint64_t S, int dir, int prec) {
  int logS = ilog2u(S);
  std::vector<int> rad = pass_radices(q, logS);
  if (rad.size() > 2) return false;
  void* dsts[2];
  if (rad.size() == 1) {
    dsts[0] = out;
  } else {
    dsts[0] = tmp;
    dsts[1] = out;
  }
  static const FactorList empty{};
  return prec == kC128 ? run_passes<double2>(ctx, in, dsts, O, q, logS, dir, empty, empty)
                       : run_passes<float2>(ctx, in, dsts, O, q, logS, dir, empty, empty);
}

}  // namespace cvdv
