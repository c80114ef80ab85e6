// Column transform passes of complex64 states on the tensor cores (tcgen05).
//
// A pass of the four-step split of a transform along a strided register (see
// kernels_col.cu: first half, shared middle pass, second half) is, per column,
// an L-point DFT (L = 64 or 128) with diagonal factors and the four-step twiddle
// around it.  Here the DFTs of a tile of 32 adjacent columns are one DFT-matrix
// product on the tensor cores, Y = F X with F the 128 x 128 matrix (L = 128) or
// two 64 x 64 blocks on its diagonal (L = 64, two lines of a column per tile),
// as split-BF16 three-term products accumulated in FP32 in tensor memory
// (tc_dft.cuh).  The CUDA cores load the tile (coalesced rows of 32 amplitudes),
// apply diagonal runs (FP64 factors; bilinear phases reduced mod 2 pi in FP64,
// sine and cosine in FP32), split it into BF16 pairs, and in the epilogue read the
// accumulators back, combine real and imaginary parts, twiddle and store.
//
// One persistent CTA per SM (the F operand takes 128 KB of shared memory): tiles
// alternate between two operand buffers and two accumulator pairs, so the
// tensor-core products of tile i run while the CUDA cores finish tile i - 1 and
// load tile i + 1.  (A warp-specialised form -- eight producer warps filling a
// four-tile ring of 16-column tiles, one MMA warp, four epilogue warps -- measured
// slower: 1.95 against 1.25 ms per 2^26-amplitude pass, the per-tile factor and
// barrier latency doubling with the tile count.)
//
// This replaces, for complex64 states, the reference's cuFFT Z2Z transform along a
// register (src/cuda/gates.cu:42-50, 98-105).

#include <cuda_bf16.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "col_pass.cuh"
#include "cvdv_internal.cuh"
#include "row_fft.cuh"
#include "tc_dft.cuh"

namespace cvdv {

namespace {
constexpr int kTcW = 32;                       // columns per tile
constexpr int kTcNB = 2 * kTcW;                // B rows: [Xr | Xi]
constexpr int kTcThreads = 256;
constexpr int kTcBBytes = kTcNB * tc::kK * 2;  // one BF16 copy of a tile (16 KB)
constexpr int kTcBufBytes = 2 * kTcBBytes;     // hi + lo (32 KB)
constexpr uint32_t kTcCols = 4 * kTcNB;        // TMEM: D1, D2 of two tile buffers
constexpr int kTcHiN = 256;                    // w_N high table, N <= 2^14
constexpr size_t kTcSmem = 4 * tc::kABytes + 2 * kTcBufBytes + (64 + kTcHiN) * sizeof(double2);
}  // namespace

struct TcPass {
  ColPass P;
  const uint4* aImg;  // F in the A layout: Re hi, Re lo, Im hi, Im lo (4 x 32 KB)
  int logL;           // 6 (two lines per tile, block-diagonal F) or 7
  uint64_t nTiles;
  unsigned int* err;  // set when a wait for the tensor cores gives up
};

__device__ __forceinline__ float2 cmulf2(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// Classes of the table factors of a pass's diagonal runs, by the address bits they
// read (their register and control bit): the strided register (one value per tile
// row), the registers below it (one per tile column), the registers above it (one
// per tile), or a mix (looked up per point).
enum TcTabClass : uint8_t { kTcRow = 0, kTcCol = 1, kTcConst = 2, kTcMixed = 3 };

__device__ __forceinline__ double2 tab_at(const TabFactor& T, uint64_t a) {
  int j = (int)((a >> T.shift) & (uint64_t)T.mask);
  if (T.ctrlShift >= 0) j += (int)((a >> T.ctrlShift) & 1ull) * T.half;
  return __ldg(T.ptr + j);
}

// BF16 pair split of two values: hi = bf16(x), lo = bf16(x - hi)
__device__ __forceinline__ void split2(float x0, float x1, __nv_bfloat162& hi, __nv_bfloat162& lo) {
  hi = __floats2bfloat162_rn(x0, x1);
  const float2 h = __bfloat1622float2(hi);
  lo = __floats2bfloat162_rn(x0 - h.x, x1 - h.y);
}

// e^{i ph} for a phase computed in FP64: reduced mod 2 pi in FP64, then an FP32 sine and cosine
__device__ __forceinline__ float2 cis_reduced(double ph) {
  const double k = rint(ph * 0.15915494309189534561);
  const float red = (float)fma(-k, 6.28318530717958647693, ph);
  float s, c;
  sincosf(red, &s, &c);
  return make_float2(c, s);
}

template <int KIND, int D1, int D2>
__global__ void __launch_bounds__(kTcThreads, 1)
    k_coltc(const float2* __restrict__ in, float2* __restrict__ out, const __grid_constant__ TcPass T) {
  const ColPass& P = T.P;
  extern __shared__ __align__(1024) unsigned char smraw[];
  unsigned char* A = smraw;                           // F: 4 x 32 KB
  unsigned char* Bbuf = smraw + 4 * tc::kABytes;      // two tile buffers of 32 KB (hi, lo)
  double2* loN = reinterpret_cast<double2*>(Bbuf + 2 * kTcBufBytes);  // w_N^e, e < 64
  double2* hiN = loN + 64;                                            // w_N^(64 h)
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmemBase;
  // diagonal runs of the current tile, factored by the address bits they read
  __shared__ uint8_t cls[kMaxColDiags][kMaxTab];
  __shared__ int perPoint, anyLin;
  __shared__ float2 rowF[tc::kK], colF[kTcW], constF;
  __shared__ double rowJ[tc::kK], colA[kTcW];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  for (int i = tid; i < 4 * tc::kABytes / 16; i += kTcThreads) reinterpret_cast<uint4*>(A)[i] = __ldg(T.aImg + i);
  if (KIND != kColLast) {
    const int nHi = P.logN >= 6 ? 1 << (P.logN - 6) : 1;
    for (int i = tid; i < 64 + nHi; i += kTcThreads) {
      const int e = i < 64 ? i : (i - 64) << 6;
      loN[i] = e < (1 << P.logN) ? __ldg(P.tw + ((size_t)e << (P.logTwN - P.logN))) : make_double2(1.0, 0.0);
    }
  }
  if (tid == 0) {
    tc::bar_init(tc::saddr(&mbar[0]), 1);
    tc::bar_init(tc::saddr(&mbar[1]), 1);
    const int rlo = P.logS, rhi = P.logS + P.logQ;
    int pp = 0, lin = 0;
    for (int d = 0; d < P.nDiag; ++d) {
      const FactorList& F = P.diag[d];
      for (int t = 0; t < F.nTab; ++t) {
        const TabFactor& X = F.tab[t];
        const int lo = X.shift, hi = X.shift + (32 - __clz(X.mask)), c = X.ctrlShift;
        uint8_t k;
        if (lo >= rlo && hi <= rhi && (c < 0 || (c >= rlo && c < rhi))) k = kTcRow;
        else if (hi <= rlo && (c < 0 || c < rlo)) k = kTcCol;
        else if (lo >= rhi && (c < 0 || c >= rhi)) k = kTcConst;
        else k = kTcMixed;
        cls[d][t] = k;
        pp |= k == kTcMixed;
      }
      pp |= F.nXX > 0;
      lin |= P.nLin[d] > 0;
    }
    perPoint = pp;
    anyLin = lin;
  }
  if (warp == 0) tc::tmem_alloc(tc::saddr(&tmemBase), kTcCols);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tbase = tmemBase;
  uint32_t phase[2] = {0u, 0u};

  const int logL = T.logL, L = 1 << logL, lpt = tc::kK >> logL;  // points per line, lines per tile
  const uint64_t nIb = (1ull << P.logS) / kTcW, nMid = (1ull << P.logA) / lpt;
  const int nMask = (1 << P.logN) - 1;
  auto geo = [&](uint64_t tile, uint64_t& i0, uint64_t& mid0, uint64_t& o) {
    i0 = (tile % nIb) * kTcW;
    const uint64_t rest = tile / nIb;
    mid0 = (rest % nMid) * lpt;
    o = rest / nMid;
  };

  // The tile's diagonal factor at (row kr, column c) is rowF[kr] colF[c] constF
  // e^{i colA[c] rowJ[kr]} times the per-point tables; rows are placed by the input
  // strides (first half) or the output ones.  Ends with a CTA barrier.
  uint64_t rowKey = ~0ull;  // (mid0, o) of the row factors in rowF / rowJ
  auto factors = [&](uint64_t i0, uint64_t mid0, uint64_t o, uint64_t midS, uint64_t axS) {
    const uint64_t key = mid0 + (o << 32);
    const bool rows = key != rowKey;  // uniform: every thread walks the same tiles
    rowKey = key;
    if (tid < tc::kK) {
      if (rows) {
        const int kr = tid, lx = kr >> logL, m = kr & (L - 1);
        const uint64_t ar = (mid0 + lx) * midS + (uint64_t)m * axS;  // the register's bits only
        double2 f = make_double2(1.0, 0.0);
        for (int d = 0; d < P.nDiag; ++d)
          for (int t = 0; t < P.diag[d].nTab; ++t)
            if (cls[d][t] == kTcRow) f = dmul(f, tab_at(P.diag[d].tab[t], ar));
        rowF[kr] = make_float2((float)f.x, (float)f.y);
        rowJ[kr] = ((double)((ar >> P.logS) & ((1ull << P.logQ) - 1)) - P.regC) * P.regDx;
      }
    } else if (tid < tc::kK + kTcW) {
      const int c = tid - tc::kK;
      const uint64_t ac = i0 + c + o * P.outerIn;
      double2 f = make_double2(1.0, 0.0);
      double a = 0.0;
      for (int d = 0; d < P.nDiag; ++d) {
        for (int t = 0; t < P.diag[d].nTab; ++t)
          if (cls[d][t] == kTcCol) f = dmul(f, tab_at(P.diag[d].tab[t], ac));
        for (int l = 0; l < P.nLin[d]; ++l) {
          const XXFactor& X = P.lin[d][l];
          const int jo = (int)((ac >> X.shift1) & (uint64_t)X.mask1);
          double cc = X.coeff * (((double)jo - X.c1) * X.dx1);
          if (X.ctrlShift >= 0 && ((ac >> X.ctrlShift) & 1ull)) cc = -cc;
          a += cc;
        }
      }
      colF[c] = make_float2((float)f.x, (float)f.y);
      colA[c] = a;
    } else if (tid == tc::kK + kTcW) {
      const uint64_t ak = o * P.outerIn;
      double2 f = make_double2(1.0, 0.0);
      for (int d = 0; d < P.nDiag; ++d) {
        if (P.diag[d].hasScalar) f = dmul(f, P.diag[d].scalar);
        for (int t = 0; t < P.diag[d].nTab; ++t)
          if (cls[d][t] == kTcConst) f = dmul(f, tab_at(P.diag[d].tab[t], ak));
      }
      constF = make_float2((float)f.x, (float)f.y);
    }
    __syncthreads();
  };
  // the remaining factors of point a: tables reading bits of several ranges, and
  // bilinear terms of two other registers (FP64)
  auto point_factor = [&](uint64_t a) -> float2 {
    double2 f = make_double2(1.0, 0.0);
    for (int d = 0; d < P.nDiag; ++d) {
      const FactorList& F = P.diag[d];
      for (int t = 0; t < F.nTab; ++t)
        if (cls[d][t] == kTcMixed) f = dmul(f, tab_at(F.tab[t], a));
      for (int t = 0; t < F.nXX; ++t) {
        const XXFactor& X = F.xx[t];
        const double x1 = ((double)(int)((a >> X.shift1) & (uint64_t)X.mask1) - X.c1) * X.dx1;
        const double x2 = ((double)(int)((a >> X.shift2) & (uint64_t)X.mask2) - X.c2) * X.dx2;
        double ph = X.coeff * x1 * x2;
        if (X.ctrlShift >= 0 && ((a >> X.ctrlShift) & 1ull)) ph = -ph;
        const float2 e = cis_reduced(ph);
        f = dmul(f, make_double2(e.x, e.y));
      }
    }
    return make_float2((float)f.x, (float)f.y);
  };
  auto factor = [&](int kr, int c, uint64_t a) -> float2 {
    float2 f = cmulf2(cmulf2(rowF[kr], colF[c]), constF);
    if (anyLin) f = cmulf2(f, cis_reduced(colA[c] * rowJ[kr]));
    if (perPoint) f = cmulf2(f, point_factor(a));
    return f;
  };

  // D[buf] = F B[buf]: 2 parts (Re F, Im F) x 8 K-steps x 3 split terms
  auto issue = [&](int buf) {
    const uint32_t idesc = tc::instr_desc_bf16(tc::kM, kTcNB, true);
    const uint32_t aB = tc::saddr(A);
    const uint32_t bh = tc::saddr(Bbuf + buf * kTcBufBytes), bl = bh + kTcBBytes;
    constexpr uint32_t LBO = (kTcNB / 8) * 128;
    for (int part = 0; part < 2; ++part) {
      const uint32_t d = tbase + (uint32_t)((2 * buf + part) * kTcNB);
      const uint32_t ah = aB + 2 * part * tc::kABytes, al = ah + tc::kABytes;
#pragma unroll
      for (int s = 0; s < tc::kK / 16; ++s) {
        const uint64_t dAh = tc::smem_desc(ah + s * 256, 128, 2048), dAl = tc::smem_desc(al + s * 256, 128, 2048);
        const uint64_t dBh = tc::smem_desc(bh + s * 2 * LBO, LBO, 128), dBl = tc::smem_desc(bl + s * 2 * LBO, LBO, 128);
        tc::mma_bf16(d, dAh, dBh, idesc, s > 0);
        tc::mma_bf16(d, dAh, dBl, idesc, 1);
        tc::mma_bf16(d, dAl, dBh, idesc, 1);
      }
    }
    tc::mma_commit(tc::saddr(&mbar[buf]));
  };

  // a tile's 128 rows (line lx = kr / L, point m = kr % L) x 32 columns into B[buf];
  // a warp reads two rows of 256 bytes per instruction, all eight rows of a thread
  // in flight at once
  auto load = [&](uint64_t tile, int buf) {
    uint64_t i0, mid0, o;
    geo(tile, i0, mid0, o);
    unsigned char* Bh = Bbuf + buf * kTcBufBytes;
    unsigned char* Bl = Bh + kTcBBytes;
    const int h = lane >> 4, cc = 2 * (lane & 15);
    float4 v[tc::kK / 16];
#pragma unroll
    for (int rr = 0; rr < tc::kK / 16; ++rr) {
      const int kr = 16 * rr + 2 * warp + h;
      const int lx = kr >> logL, m = kr & (L - 1);
      const uint64_t a = i0 + cc + (mid0 + lx) * P.midIn + o * P.outerIn + (uint64_t)m * P.axisIn;
      v[rr] = __ldg(reinterpret_cast<const float4*>(in + a));
    }
    // the tile's factors while its loads are in flight
    if (KIND == kColFirst && P.nDiag) factors(i0, mid0, o, P.midIn, P.axisIn);
#pragma unroll
    for (int rr = 0; rr < tc::kK / 16; ++rr) {
      const int kr = 16 * rr + 2 * warp + h;
      float2 x0 = make_float2(v[rr].x, v[rr].y), x1 = make_float2(v[rr].z, v[rr].w);
      if (KIND == kColFirst && P.nDiag) {
        const int lx = kr >> logL, m = kr & (L - 1);
        const uint64_t a = i0 + cc + (mid0 + lx) * P.midIn + o * P.outerIn + (uint64_t)m * P.axisIn;
        x0 = cmulf2(x0, factor(kr, cc, a));
        x1 = cmulf2(x1, factor(kr, cc + 1, a + 1));
      }
      __nv_bfloat162 hi, lo;
      split2(x0.x, x1.x, hi, lo);
      *reinterpret_cast<__nv_bfloat162*>(Bh + tc::b_off(cc, kr, kTcNB)) = hi;
      *reinterpret_cast<__nv_bfloat162*>(Bl + tc::b_off(cc, kr, kTcNB)) = lo;
      split2(x0.y, x1.y, hi, lo);
      *reinterpret_cast<__nv_bfloat162*>(Bh + tc::b_off(kTcW + cc, kr, kTcNB)) = hi;
      *reinterpret_cast<__nv_bfloat162*>(Bl + tc::b_off(kTcW + cc, kr, kTcNB)) = lo;
    }
  };

  // this thread's 16 results of D[buf]: row kr = 32 (warp % 4) + lane, columns
  // c0 .. c0 + 15 with c0 = 16 (warp / 4); dir -1 conjugates F
  const int kr = 32 * (warp & 3) + lane, c0 = 16 * (warp >> 2);
  const int lxE = kr >> logL, mE = kr & (L - 1);
  auto read = [&](int buf, int dir, float2 (&y)[16]) {
    const uint32_t d1 = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + (uint32_t)(2 * buf * kTcNB);
    const uint32_t d2 = d1 + kTcNB;
    float a[16], b[16], c[16], e[16];
    tc::tmem_ld16(d1 + c0, a);
    tc::tmem_ld16(d1 + kTcW + c0, b);
    tc::tmem_ld16(d2 + c0, c);
    tc::tmem_ld16(d2 + kTcW + c0, e);
    tc::tmem_ld_wait();
#pragma unroll
    for (int i = 0; i < 16; ++i)
      y[i] = dir > 0 ? make_float2(a[i] - e[i], b[i] + c[i]) : make_float2(a[i] + e[i], b[i] - c[i]);
  };
  auto wait = [&](int buf) {
    tc::bar_wait(tc::saddr(&mbar[buf]), phase[buf], T.err);
    phase[buf] ^= 1u;
    tc::fence_after_sync();
  };

  auto epilogue = [&](uint64_t tile, int buf) {
    uint64_t i0, mid0, o;
    geo(tile, i0, mid0, o);
    if (KIND != kColFirst && P.nDiag) factors(i0, mid0, o, P.midOut, P.axisOut);
    const uint64_t aOut = i0 + c0 + (mid0 + lxE) * P.midOut + o * P.outerOut + (uint64_t)mE * P.axisOut;
    float2 y[16];
    wait(buf);
    read(buf, D1, y);
    if constexpr (KIND == kColMiddle) {
      // the run between the two transforms, then the second DFT on the same points
      if (P.nDiag)
#pragma unroll
        for (int i = 0; i < 16; ++i) y[i] = cmulf2(y[i], factor(kr, c0 + i, aOut + i));
      unsigned char* Bh = Bbuf + buf * kTcBufBytes;
      unsigned char* Bl = Bh + kTcBBytes;
#pragma unroll
      for (int g = 0; g < 2; ++g) {
        float xr[8], xi[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          xr[q] = y[8 * g + q].x;
          xi[q] = y[8 * g + q].y;
        }
        uint4 hi, lo;
        tc::split8(xr, hi, lo);
        *reinterpret_cast<uint4*>(Bh + tc::b_off(c0 + 8 * g, kr, kTcNB)) = hi;
        *reinterpret_cast<uint4*>(Bl + tc::b_off(c0 + 8 * g, kr, kTcNB)) = lo;
        tc::split8(xi, hi, lo);
        *reinterpret_cast<uint4*>(Bh + tc::b_off(kTcW + c0 + 8 * g, kr, kTcNB)) = hi;
        *reinterpret_cast<uint4*>(Bl + tc::b_off(kTcW + c0 + 8 * g, kr, kTcNB)) = lo;
      }
      tc::fence_async_smem();
      tc::fence_before_sync();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after_sync();
        issue(buf);
      }
      wait(buf);
      read(buf, D2, y);
    }
    if constexpr (KIND == kColFirst || KIND == kColMiddle) {
      constexpr int DT = KIND == kColMiddle ? D2 : D1;  // direction of the four-step twiddle
      const int e = (int)(((mid0 + lxE) * (uint64_t)mE) & (uint64_t)nMask);
      if (e) {
        const float2 w = tw2<float2, DT>(loN, hiN, e);
#pragma unroll
        for (int i = 0; i < 16; ++i) y[i] = cmulf2(y[i], w);
      }
    }
    if constexpr (KIND == kColLast) {
      if (P.nDiag)
#pragma unroll
        for (int i = 0; i < 16; ++i) y[i] = cmulf2(y[i], factor(kr, c0 + i, aOut + i));
    }
    float4* dst = reinterpret_cast<float4*>(out + aOut);
#pragma unroll
    for (int i = 0; i < 8; ++i) dst[i] = make_float4(y[2 * i].x, y[2 * i].y, y[2 * i + 1].x, y[2 * i + 1].y);
  };

  // tile i's products overlap the epilogue of tile i - 1 and the loads of tile i + 1
  uint64_t prev = ~0ull;
  int pbuf = 0, it = 0;
  for (uint64_t tile = blockIdx.x; tile < T.nTiles; tile += gridDim.x, ++it) {
    const int buf = it & 1;
    load(tile, buf);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      issue(buf);
    }
    if (prev != ~0ull) epilogue(prev, pbuf);
    prev = tile;
    pbuf = buf;
  }
  if (prev != ~0ull) epilogue(prev, pbuf);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, kTcCols);
}

// ---------------------------------------------------------------- host side
// F in the A operand layout, split into BF16 pairs (Re hi, Re lo, Im hi, Im lo),
// 128 x 128: the 128-point DFT matrix, or two 64-point ones on the diagonal.
static uint16_t bf16_bits(float x) {
  const __nv_bfloat16 b = __float2bfloat16_rn(x);
  return *reinterpret_cast<const uint16_t*>(&b);
}

const uint4* tc_dft_image(Context* ctx, int logL) {
  const int slot = logL - 6;
  if (slot < 0 || slot > 1) return nullptr;
  if (ctx->tcImage[slot]) return (const uint4*)ctx->tcImage[slot];
  const int L = 1 << logL;
  std::vector<uint16_t> img(4 * tc::kABytes / 2, 0);
  for (int m = 0; m < tc::kM; ++m)
    for (int k = 0; k < tc::kK; ++k) {
      if ((m >> logL) != (k >> logL)) continue;  // block-diagonal for L = 64
      const int e = ((m & (L - 1)) * (k & (L - 1))) & (L - 1);
      const double ang = -2.0 * CVDV_PI * (double)e / (double)L;
      const float re = (float)cos(ang), im = (float)sin(ang);
      const uint16_t rh = bf16_bits(re), ih = bf16_bits(im);
      const float rhf = __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(&rh));
      const float ihf = __bfloat162float(*reinterpret_cast<const __nv_bfloat16*>(&ih));
      const uint32_t o = tc::a_off(m, k) / 2;
      img[0 * (tc::kABytes / 2) + o] = rh;
      img[1 * (tc::kABytes / 2) + o] = bf16_bits(re - rhf);
      img[2 * (tc::kABytes / 2) + o] = ih;
      img[3 * (tc::kABytes / 2) + o] = bf16_bits(im - ihf);
    }
  void* d = nullptr;
  if (!cuda_ok(ctx, cudaMalloc(&d, 4 * tc::kABytes), "tensor-core DFT matrix")) return nullptr;
  if (!cuda_ok(ctx, cudaMemcpyAsync(d, img.data(), 4 * tc::kABytes, cudaMemcpyHostToDevice, ctx->stream),
               "tensor-core DFT matrix") ||
      !cuda_ok(ctx, cudaStreamSynchronize(ctx->stream), "tensor-core DFT matrix")) {
    cudaFree(d);
    return nullptr;
  }
  ctx->tcImage[slot] = d;
  return (const uint4*)d;
}

// Whether a transform of register reg runs its four-step passes on the tensor
// cores: complex64, 2^12 .. 2^14 points (passes of 64 or 128 points), at least 32
// amplitudes below it (tiles of 32 adjacent columns), and fusion bit 5 set.
bool tc_col_ok(Context* ctx, int reg) {
  const int q = ctx->q[reg], logS = ctx->flw[reg];
  return ctx->tcCol && ctx->precision == kC64 && q >= 12 && q <= 14 && logS >= 5;
}

template <int KIND, int D1, int D2>
static cudaError_t tc_launch_t(Context* ctx, const TcPass& T) {
  auto kern = k_coltc<KIND, D1, D2>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
  if (e != cudaSuccess) return e;
  const uint64_t grid = T.nTiles < (uint64_t)ctx->numSMs ? T.nTiles : (uint64_t)ctx->numSMs;
  kern<<<(unsigned)grid, kTcThreads, kTcSmem, ctx->stream>>>((const float2*)ctx->state(), (float2*)ctx->other(), T);
  return cudaGetLastError();
}

// One pass of a column chain (kernels_col.cu: run_col_chain) on the tensor cores;
// logL is the pass's DFT length, kind / d1 / d2 as for k_colr.
cudaError_t launch_col_tc(Context* ctx, const ColPass& P, int logL, int kind, int d1, int d2) {
  if (logL < 6 || logL > 7 || P.logS < 5 || P.logN > 14 || kind == kColWhole) return cudaErrorInvalidValue;
  const int lpt = 1 << (7 - logL);
  if (P.logA < 7 - logL) return cudaErrorInvalidValue;
  TcPass T;
  T.P = P;
  T.aImg = tc_dft_image(ctx, logL);
  if (!T.aImg) return cudaErrorMemoryAllocation;
  T.logL = logL;
  T.nTiles = P.nCols / (uint64_t)(kTcW * lpt);
  T.err = ctx->waitErr;
  switch (kind) {
    case kColFirst: return d1 > 0 ? tc_launch_t<kColFirst, 1, 0>(ctx, T) : tc_launch_t<kColFirst, -1, 0>(ctx, T);
    case kColLast: return d1 > 0 ? tc_launch_t<kColLast, 1, 0>(ctx, T) : tc_launch_t<kColLast, -1, 0>(ctx, T);
    default:
      if (d1 > 0) return d2 > 0 ? tc_launch_t<kColMiddle, 1, 1>(ctx, T) : tc_launch_t<kColMiddle, 1, -1>(ctx, T);
      return d2 > 0 ? tc_launch_t<kColMiddle, -1, 1>(ctx, T) : tc_launch_t<kColMiddle, -1, -1>(ctx, T);
  }
}

}  // namespace cvdv
