// Readouts: state I/O, norm, fidelities, marginals and <n>.
//
// Reductions are two-level and deterministic where they produce a scalar: a
// fixed grid writes one partial per block, a single block sums the partials in
// a fixed order.  Marginals accumulate per-block shared-memory histograms with
// warp aggregation (one shared atomic per warp when every lane of the warp
// falls in the same bin, which is the case whenever the selected registers are
// not the lowest 5 index bits), then sum the per-block histograms bin by bin.

#include <cmath>
#include <cstring>
#include <mutex>

#include "../../include/cvdv.h"
#include "cvdv_internal.cuh"

using namespace cvdv;
struct CVDVContext : public cvdv::Context {};

namespace cvdv {

constexpr int kRedBlocks = 148 * 4;
constexpr int kRedThreads = 256;

template <typename C> __device__ __forceinline__ double2 tod(C v);
template <> __device__ __forceinline__ double2 tod<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ double2 tod<float2>(float2 v) {
  return make_double2((double)v.x, (double)v.y);
}

__device__ __forceinline__ double2 block_sum2(double2 v) {
  __shared__ double2 ws[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) ws[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < (int)(blockDim.x >> 5) ? ws[lane] : make_double2(0.0, 0.0);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      v.x += __shfl_down_sync(0xffffffffu, v.x, o);
      v.y += __shfl_down_sync(0xffffffffu, v.y, o);
    }
  }
  return v;
}

__global__ void k_final_sum(const double2* __restrict__ part, int n, double2* out) {
  double2 a = make_double2(0.0, 0.0);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    a.x += part[i].x;
    a.y += part[i].y;
  }
  a = block_sum2(a);
  if (threadIdx.x == 0) *out = a;
}

// ---- functors for the generic reduction: return a double2 per index
template <typename C>
struct OpNorm {  // sum |psi|^2    (measure.cu:276-300)
  const C* st;
  __device__ double2 operator()(uint64_t i) const {
    double2 v = tod<C>(st[i]);
    return make_double2(v.x * v.x + v.y * v.y, 0.0);
  }
};

template <typename C>
struct OpX2 {  // sum |psi|^2 x_j^2   (kernelExpectX2, measure.cuh:158-178)
  const C* st;
  int shift, mask;
  double c, dx;
  __device__ double2 operator()(uint64_t i) const {
    double2 v = tod<C>(st[i]);
    double x = ((double)((i >> shift) & (uint64_t)mask) - c) * dx;
    return make_double2((v.x * v.x + v.y * v.y) * x * x, 0.0);
  }
};

template <typename C1, typename C2>
struct OpDot {  // sum conj(a) b   (kernelInnerProductStatevectors, measure.cuh:227-252)
  const C1* a;
  const C2* b;
  __device__ double2 operator()(uint64_t i) const {
    double2 x = tod<C1>(a[i]), y = tod<C2>(b[i]);
    return make_double2(x.x * y.x + x.y * y.y, x.x * y.y - x.y * y.x);
  }
};

template <typename C>
struct OpSep {  // sum conj(psi) * outer[i >> qLast] * last[i & m]   (measure.cuh:182-223)
  const C* st;
  const double2* outer;
  const double2* last;
  int qLast;
  __device__ double2 operator()(uint64_t i) const {
    double2 v = tod<C>(st[i]);
    double2 p = dmul(__ldg(last + (i & ((1ull << qLast) - 1))), __ldg(outer + (i >> qLast)));
    return make_double2(v.x * p.x + v.y * p.y, v.x * p.y - v.y * p.x);
  }
};

template <typename Op>
__global__ void __launch_bounds__(kRedThreads) k_reduce(Op op, uint64_t n, double2* part) {
  double2 a = make_double2(0.0, 0.0);
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  // four terms evaluated before they are added, so four loads are in flight
  for (; i + 3 * stride < n; i += 4 * stride) {
    const double2 v0 = op(i), v1 = op(i + stride), v2 = op(i + 2 * stride), v3 = op(i + 3 * stride);
    a.x += (v0.x + v1.x) + (v2.x + v3.x);
    a.y += (v0.y + v1.y) + (v2.y + v3.y);
  }
  for (; i < n; i += stride) {
    const double2 v = op(i);
    a.x += v.x;
    a.y += v.y;
  }
  a = block_sum2(a);
  if (threadIdx.x == 0) part[blockIdx.x] = a;
}

template <typename Op>
static bool reduce(Context* ctx, Op op, uint64_t n, double2* result) {
  double2* part = (double2*)arena_alloc(ctx, (kRedBlocks + 1) * sizeof(double2));
  if (!part) return false;
  double* hs = host_scratch(ctx, 2);
  if (!hs) return false;
  {
    LaunchScope _ls(ctx, kKReduce);
    k_reduce<Op><<<kRedBlocks, kRedThreads, 0, ctx->stream>>>(op, n, part);
  }
  {
    LaunchScope _ls(ctx, kKReduce);
    k_final_sum<<<1, 1024, 0, ctx->stream>>>(part, kRedBlocks, part + kRedBlocks);
  }
  if (!cuda_ok(ctx, cudaGetLastError(), "reduce launch")) return false;
  if (!cuda_ok(ctx, cudaMemcpyAsync(hs, part + kRedBlocks, sizeof(double2), cudaMemcpyDeviceToHost,
                                    ctx->stream),
               "reduce copy"))
    return false;
  if (!stream_sync(ctx, "reduce sync")) return false;
  *result = make_double2(hs[0], hs[1]);
  return true;
}

// ----------------------------------------------------------------- marginals
struct MargDesc {
  int nSel;
  int shift[16];
  int mask[16];
  long long stride[16];
  long long outSize;
};

__device__ __forceinline__ long long marg_bin(const MargDesc& D, uint64_t i) {
  long long oi = 0;
  for (int s = 0; s < D.nSel; ++s) oi += (long long)((i >> D.shift[s]) & (uint64_t)D.mask[s]) * D.stride[s];
  return oi;
}

// smem histogram per block -> part[block][bin]
template <typename C>
__global__ void __launch_bounds__(256) k_marg_smem(const C* __restrict__ st, uint64_t n,
                                                  MargDesc D, double* __restrict__ part) {
  extern __shared__ double hist[];
  for (int b = threadIdx.x; b < D.outSize; b += blockDim.x) hist[b] = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const uint64_t warpStride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n;
       base += warpStride) {
    uint64_t i = base + lane;
    double p = 0.0;
    long long bin = 0;
    if (i < n) {
      double2 v = tod<C>(st[i]);
      p = v.x * v.x + v.y * v.y;
      bin = marg_bin(D, i);
    }
    long long b0 = __shfl_sync(0xffffffffu, bin, 0);
    bool same = __all_sync(0xffffffffu, (i >= n) || bin == b0);
    if (same) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) p += __shfl_down_sync(0xffffffffu, p, o);
      if (lane == 0) atomicAdd(&hist[b0], p);
    } else if (i < n) {
      atomicAdd(&hist[bin], p);
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < D.outSize; b += blockDim.x)
    part[(size_t)blockIdx.x * D.outSize + b] = hist[b];
}

__global__ void k_marg_final(const double* __restrict__ part, int nb, long long outSize,
                             double* __restrict__ out) {
  for (long long b = (long long)blockIdx.x * blockDim.x + threadIdx.x; b < outSize;
       b += (long long)gridDim.x * blockDim.x) {
    double a = 0.0;
    for (int k = 0; k < nb; ++k) a += part[(size_t)k * outSize + b];
    out[b] = a;
  }
}

// large outputs: global atomics (warp-aggregated when the warp shares a bin)
template <typename C>
__global__ void __launch_bounds__(256) k_marg_global(const C* __restrict__ st, uint64_t n,
                                                    MargDesc D, double* __restrict__ out) {
  const int lane = threadIdx.x & 31;
  const uint64_t warpStride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n;
       base += warpStride) {
    uint64_t i = base + lane;
    double p = 0.0;
    long long bin = 0;
    if (i < n) {
      double2 v = tod<C>(st[i]);
      p = v.x * v.x + v.y * v.y;
      bin = marg_bin(D, i);
    }
    long long b0 = __shfl_sync(0xffffffffu, bin, 0);
    bool same = __all_sync(0xffffffffu, (i >= n) || bin == b0);
    if (same) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) p += __shfl_down_sync(0xffffffffu, p, o);
      if (lane == 0) atomicAdd(&out[b0], p);
    } else if (i < n) {
      atomicAdd(&out[bin], p);
    }
  }
}

// Tiled marginals: several outputs (each the joint marginal of some registers) in
// one pass.  A block reads tiles of 256 x 16 consecutive amplitudes.  An output
// whose registers all lie above the tile's 12 index bits has one bin per tile:
// the block sums the tile once and thread 0 adds it (no atomics at all, which
// is the case for every qubit register of a mode-last layout).  Other outputs
// bin each amplitude with warp-aggregated shared atomics.
constexpr int kMargLogV = 4;
constexpr int kMargLogTile = 8 + kMargLogV;
constexpr int kMargMaxOut = 16;
constexpr int kMargSmemBins = 4096;

struct MargOut {
  int nSel, sel0, off, high;
};
struct MargPlan {
  int nOut, nHigh, totalBins;
  int shift[16], mask[16], stride[16];
  MargOut out[kMargMaxOut];
};

__device__ __forceinline__ int marg_out_bin(const MargPlan& P, const MargOut& O, uint64_t i) {
  int b = 0;
  for (int s = 0; s < O.nSel; ++s)
    b += (int)((i >> P.shift[O.sel0 + s]) & (uint64_t)P.mask[O.sel0 + s]) * P.stride[O.sel0 + s];
  return b;
}

template <typename C>
__global__ void __launch_bounds__(256) k_marg_tiles(const C* __restrict__ st, uint64_t nTiles,
                                                   const __grid_constant__ MargPlan P,
                                                   double* __restrict__ part) {
  constexpr int V = 1 << kMargLogV;
  extern __shared__ double hist[];
  __shared__ double red[8];
  for (int b = threadIdx.x; b < P.totalBins; b += blockDim.x) hist[b] = 0.0;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (uint64_t tile = blockIdx.x; tile < nTiles; tile += gridDim.x) {
    const uint64_t t0 = tile << kMargLogTile;
    double p[V];
#pragma unroll
    for (int v = 0; v < V; ++v) {
      const double2 a = tod<C>(st[t0 + threadIdx.x + (v << 8)]);
      p[v] = a.x * a.x + a.y * a.y;
    }
    if (P.nHigh < P.nOut) {
      for (int o = 0; o < P.nOut; ++o) {
        const MargOut& O = P.out[o];
        if (O.high) continue;
#pragma unroll
        for (int v = 0; v < V; ++v) {
          const int bin = marg_out_bin(P, O, t0 + threadIdx.x + (v << 8));
          const int b0 = __shfl_sync(0xffffffffu, bin, 0);
          if (__all_sync(0xffffffffu, bin == b0)) {
            double q = p[v];
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) q += __shfl_down_sync(0xffffffffu, q, d);
            if (lane == 0) atomicAdd(&hist[O.off + b0], q);
          } else {
            atomicAdd(&hist[O.off + bin], p[v]);
          }
        }
      }
    }
    if (P.nHigh) {
      double q = 0.0;
#pragma unroll
      for (int v = 0; v < V; ++v) q += p[v];
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) q += __shfl_down_sync(0xffffffffu, q, d);
      if (lane == 0) red[warp] = q;
      __syncthreads();
      if (threadIdx.x == 0) {
        double S = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) S += red[w];
        for (int o = 0; o < P.nOut; ++o)
          if (P.out[o].high) hist[P.out[o].off + marg_out_bin(P, P.out[o], t0)] += S;
      }
      __syncthreads();
    }
  }
  __syncthreads();
  for (int b = threadIdx.x; b < P.totalBins; b += blockDim.x)
    part[(size_t)blockIdx.x * P.totalBins + b] = hist[b];
}

// One pass for `outs` (each a list of registers, first fastest); every output
// must have at most kMargSmemBins bins in total and the state at least one tile.
// dOut receives the outputs back to back.
static bool marginals_tiled(Context* ctx, const std::vector<std::vector<int>>& outs, double* dOut) {
  MargPlan P{};
  int sel = 0;
  for (const auto& regs : outs) {
    MargOut& O = P.out[P.nOut++];
    O.nSel = (int)regs.size();
    O.sel0 = sel;
    O.off = P.totalBins;
    O.high = 1;
    int stride = 1;
    for (int r : regs) {
      P.shift[sel] = ctx->flw[r];
      P.mask[sel] = (1 << ctx->q[r]) - 1;
      P.stride[sel] = stride;
      stride <<= ctx->q[r];
      if (ctx->flw[r] < kMargLogTile) O.high = 0;
      ++sel;
    }
    P.nHigh += O.high;
    P.totalBins += stride;
  }
  const uint64_t nTiles = ctx->size() >> kMargLogTile;
  uint64_t blocks = P.totalBins <= 256 ? 148ull * 4 : 148ull * 2;
  if (blocks > nTiles) blocks = nTiles;
  double* part = (double*)arena_alloc(ctx, (size_t)blocks * P.totalBins * sizeof(double));
  if (!part) return false;
  const size_t smem = (size_t)P.totalBins * sizeof(double);
  {
    LaunchScope _ls(ctx, kKReduce);
    if (ctx->precision == kC128)
      k_marg_tiles<double2><<<(unsigned)blocks, 256, smem, ctx->stream>>>((const double2*)ctx->state(), nTiles, P, part);
    else
      k_marg_tiles<float2><<<(unsigned)blocks, 256, smem, ctx->stream>>>((const float2*)ctx->state(), nTiles, P, part);
  }
  {
    LaunchScope _ls(ctx, kKReduce);
    k_marg_final<<<(P.totalBins + 255) / 256, 256, 0, ctx->stream>>>(part, (int)blocks, P.totalBins, dOut);
  }
  return cuda_ok(ctx, cudaGetLastError(), "marginal launch");
}

// Marginals of registers above the last one from the row sums the flush's last
// row program wrote (a row = one value of every register but the last): the rows'
// partials are added in a fixed order, then one CTA per output bin adds the rows
// with that register value in a fixed tree.
__global__ void k_row_total(const double* __restrict__ parts, int P, uint64_t rows, double* __restrict__ tot) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
    double a = 0.0;
    for (int p = 0; p < P; ++p) a += parts[r * P + p];
    tot[r] = a;
  }
}

struct RowMarg {
  int nOut;
  int shift[kMargMaxOut], q[kMargMaxOut], off[kMargMaxOut];  // register field in the row index; output offset
};

__global__ void __launch_bounds__(256) k_row_marg(const double* __restrict__ tot, uint64_t rows,
                                                  const __grid_constant__ RowMarg M, double* __restrict__ out) {
  int o = 0;
  while (o + 1 < M.nOut && (int)blockIdx.x >= M.off[o + 1]) ++o;
  const uint64_t v = (uint64_t)(blockIdx.x - M.off[o]);
  const int sh = M.shift[o], q = M.q[o];
  const uint64_t cnt = rows >> q, low = (1ull << sh) - 1;
  double a = 0.0;
  for (uint64_t i = threadIdx.x; i < cnt; i += blockDim.x)
    a += tot[((i & ~low) << q) | (v << sh) | (i & low)];
  const double2 s = block_sum2(make_double2(a, 0.0));
  if (threadIdx.x == 0) out[blockIdx.x] = s.x;
}

static bool marginals_from_rows(Context* ctx, const std::vector<std::vector<int>>& outs, int parts, double* dOut) {
  const int last = ctx->numReg - 1;
  const uint64_t rows = ctx->size() >> ctx->q[last];
  RowMarg M{};
  int bins = 0;
  for (const auto& regs : outs) {
    const int r = regs[0];
    M.shift[M.nOut] = ctx->flw[r] - ctx->q[last];
    M.q[M.nOut] = ctx->q[r];
    M.off[M.nOut++] = bins;
    bins += 1 << ctx->q[r];
  }
  double* tot = (double*)arena_alloc(ctx, rows * sizeof(double));
  if (!tot) return false;
  {
    LaunchScope _ls(ctx, kKReduce);
    k_row_total<<<(unsigned)((rows + 255) / 256 < 1184 ? (rows + 255) / 256 : 1184), 256, 0, ctx->stream>>>(
        ctx->rowSumBuf, parts, rows, tot);
  }
  {
    LaunchScope _ls(ctx, kKReduce);
    k_row_marg<<<bins, 256, 0, ctx->stream>>>(tot, rows, M, dOut);
  }
  return cuda_ok(ctx, cudaGetLastError(), "row-sum marginal launch");
}

// Ask the next flush for row sums when every register read is a single register
// above the last one; false (nothing asked) otherwise.
static bool request_row_sums(Context* c, const std::vector<std::vector<int>>& outs) {
  if (c->numReg < 2 || outs.empty()) return false;
  for (const auto& regs : outs)
    if (regs.size() != 1 || regs[0] == c->numReg - 1) return false;
  const size_t need = (c->size() >> c->q[c->numReg - 1]) * kRowSumMaxParts;
  if (need > c->rowSumCap) {
    cudaStreamSynchronize(c->stream);
    if (c->rowSumBuf) cudaFree(c->rowSumBuf);
    c->rowSumBuf = nullptr;
    c->rowSumCap = 0;
    if (cudaMalloc(&c->rowSumBuf, need * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      return false;
    }
    c->rowSumCap = need;
  }
  c->rowSums = c->rowSumBuf;
  c->rowSumParts = 0;
  return true;
}

static bool tiled_ok(Context* ctx, long long bins) {
  return bins <= kMargSmemBins && ctx->totalQbt >= kMargLogTile;
}

static bool marginal_device(Context* ctx, const int* regs, int nr, double** dOut, long long* outSize) {
  MargDesc D{};
  D.nSel = nr;
  long long stride = 1;
  for (int s = 0; s < nr; ++s) {
    D.shift[s] = ctx->flw[regs[s]];
    D.mask[s] = (1 << ctx->q[regs[s]]) - 1;
    D.stride[s] = stride;  // column-major: first selected register fastest (measure.cu:89-91)
    stride *= (long long)1 << ctx->q[regs[s]];
  }
  D.outSize = stride;
  *outSize = stride;
  uint64_t n = ctx->size();
  double* out = (double*)arena_alloc(ctx, (size_t)stride * sizeof(double));
  if (!out) return false;
  if (stride <= 4096) {
    int blocks = 148 * 2;
    uint64_t maxBlocks = (n + 255) / 256;
    if ((uint64_t)blocks > maxBlocks) blocks = (int)maxBlocks;
    double* part = (double*)arena_alloc(ctx, (size_t)blocks * stride * sizeof(double));
    if (!part) return false;
    size_t smem = (size_t)stride * sizeof(double);
    if (ctx->precision == kC128)
      {
        LaunchScope _ls(ctx, kKReduce);
        k_marg_smem<double2><<<blocks, 256, smem, ctx->stream>>>((const double2*)ctx->state(), n, D, part);
      }
    else
      {
        LaunchScope _ls(ctx, kKReduce);
        k_marg_smem<float2><<<blocks, 256, smem, ctx->stream>>>((const float2*)ctx->state(), n, D, part);
      }
    int fb = (int)((stride + 255) / 256);
    {
      LaunchScope _ls(ctx, kKReduce);
      k_marg_final<<<fb, 256, 0, ctx->stream>>>(part, blocks, stride, out);
    }
  } else {
    if (!cuda_ok(ctx, cudaMemsetAsync(out, 0, (size_t)stride * sizeof(double), ctx->stream), "memset"))
      return false;
    int blocks = 148 * 8;
    if (ctx->precision == kC128)
      {
        LaunchScope _ls(ctx, kKReduce);
        k_marg_global<double2><<<blocks, 256, 0, ctx->stream>>>((const double2*)ctx->state(), n, D, out);
      }
    else
      {
        LaunchScope _ls(ctx, kKReduce);
        k_marg_global<float2><<<blocks, 256, 0, ctx->stream>>>((const float2*)ctx->state(), n, D, out);
      }
  }
  if (!cuda_ok(ctx, cudaGetLastError(), "marginal launch")) return false;
  *dOut = out;
  return true;
}

// ----------------------------------------------------------------- conversions
__global__ void k_c128_to_c64(const double2* __restrict__ s, float2* __restrict__ d, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    d[i] = make_float2((float)s[i].x, (float)s[i].y);
}

bool launch_convert_c128_to_c64(Context* ctx, const double2* src, float2* dst, uint64_t n) {
  {
    LaunchScope _ls(ctx, kKInit);
    k_c128_to_c64<<<148 * 8, 256, 0, ctx->stream>>>(src, dst, n);
  }
  return cuda_ok(ctx, cudaGetLastError(), "convert launch");
}

template <typename C>
__global__ void k_split(const C* __restrict__ st, uint64_t off, uint64_t cnt, double* __restrict__ re,
                        double* __restrict__ im) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt;
       i += (uint64_t)gridDim.x * blockDim.x) {
    double2 v = tod<C>(st[off + i]);
    re[i] = v.x;
    im[i] = v.y;
  }
}

}  // namespace cvdv

// ====================================================================== C API
static Context* C(CVDVContext* p) { return static_cast<Context*>(p); }

static bool ready(Context* c, const char* what) {
  if (c->numReg == 0 || !c->initialized) {
    set_error(c, kErrNotInitialized, "%s: state not initialised", what);
    return false;
  }
  return flush(c);
}

extern "C" {

int cvdvGetLastError(CVDVContext* ctx, char* msg, int len);

void cvdvGetState(CVDVContext* ctx, double* realOut, double* imagOut) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!ready(c, "cvdvGetState") || !realOut || !imagOut) return;
  uint64_t n = c->size();
  const uint64_t chunk = 1ull << 22;
  uint64_t cnt0 = n < chunk ? n : chunk;
  double* dre = (double*)arena_alloc(c, cnt0 * sizeof(double));
  double* dim = (double*)arena_alloc(c, cnt0 * sizeof(double));
  if (!dre || !dim) return;
  for (uint64_t off = 0; off < n; off += chunk) {
    uint64_t cnt = n - off < chunk ? n - off : chunk;
    int blocks = (int)((cnt + 255) / 256 < 1184 ? (cnt + 255) / 256 : 1184);
    if (c->precision == kC128)
      {
        LaunchScope _ls(ctx, kKReduce);
        k_split<double2><<<blocks, 256, 0, c->stream>>>((const double2*)c->state(), off, cnt, dre, dim);
      }
    else
      {
        LaunchScope _ls(ctx, kKReduce);
        k_split<float2><<<blocks, 256, 0, c->stream>>>((const float2*)c->state(), off, cnt, dre, dim);
      }
    if (!cuda_ok(c, cudaMemcpyAsync(realOut + off, dre, cnt * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream), "getState copy re") ||
        !cuda_ok(c, cudaMemcpyAsync(imagOut + off, dim, cnt * sizeof(double), cudaMemcpyDeviceToHost,
                                    c->stream), "getState copy im"))
      return;
  }
  stream_sync(c, "getState sync");
}

double cvdvGetNorm(CVDVContext* ctx) {
  if (!ctx) return 0.0;
  Context* c = C(ctx);
  if (!ready(c, "cvdvGetNorm")) return 0.0;
  arena_reset(c);
  double2 r;
  bool ok = c->precision == kC128
                ? reduce(c, OpNorm<double2>{(const double2*)c->state()}, c->size(), &r)
                : reduce(c, OpNorm<float2>{(const float2*)c->state()}, c->size(), &r);
  return ok ? r.x : 0.0;
}

static bool measure(Context* c, const int* regIdxs, int numRegs, double* probsOut, const char* w) {
  if (!regIdxs || numRegs <= 0 || !probsOut) {
    set_error(c, kErrInvalidArg, "%s: empty register list", w);
    return false;
  }
  if (numRegs > 16) {
    set_error(c, kErrInvalidArg, "%s: at most 16 registers", w);
    return false;
  }
  for (int s = 0; s < numRegs; ++s)
    if (regIdxs[s] < 0 || regIdxs[s] >= c->numReg) {
      set_error(c, kErrInvalidArg, "%s: invalid register index %d", w, regIdxs[s]);
      return false;
    }
  if (!ready(c, w)) return false;
  arena_reset(c);
  long long bins = 1;
  for (int s = 0; s < numRegs; ++s) bins <<= c->q[regIdxs[s]];
  double* dOut;
  long long outSize = bins;
  if (tiled_ok(c, bins)) {
    dOut = (double*)arena_alloc(c, (size_t)bins * sizeof(double));
    if (!dOut || !marginals_tiled(c, {std::vector<int>(regIdxs, regIdxs + numRegs)}, dOut)) return false;
  } else if (!marginal_device(c, regIdxs, numRegs, &dOut, &outSize)) {
    return false;
  }
  if (!cuda_ok(c, cudaMemcpyAsync(probsOut, dOut, (size_t)outSize * sizeof(double),
                                  cudaMemcpyDeviceToHost, c->stream), "marginal copy"))
    return false;
  return stream_sync(c, "marginal sync");
}

void cvdvMeasureMultiple(CVDVContext* ctx, const int* regIdxs, int numRegs, double* probsOut) {
  if (!ctx) return;
  measure(C(ctx), regIdxs, numRegs, probsOut, "cvdvMeasureMultiple");
}

void cvdvMeasureMultipleCT(CVDVContext* ctx, const int* regIdxs, int numRegs, double* probsOut) {
  if (!ctx) return;
  measure(C(ctx), regIdxs, numRegs, probsOut, "cvdvMeasureMultipleCT");
}

void cvdvMeasureEach(CVDVContext* ctx, const int* regIdxs, int numRegs, double* probsOut) {
  if (!ctx) return;
  Context* c = C(ctx);
  const char* w = "cvdvMeasureEach";
  if (!regIdxs || numRegs <= 0 || numRegs > kMargMaxOut || !probsOut) {
    set_error(c, kErrInvalidArg, "%s: need 1..%d registers and an output", w, kMargMaxOut);
    return;
  }
  for (int k = 0; k < numRegs; ++k)
    if (regIdxs[k] < 0 || regIdxs[k] >= c->numReg) {
      set_error(c, kErrInvalidArg, "%s: invalid register index %d", w, regIdxs[k]);
      return;
    }
  // registers whose marginals fit the shared histogram go in one pass; larger
  // ones are read one at a time
  std::vector<std::vector<int>> outs;
  std::vector<size_t> outPos, bigPos;
  std::vector<int> big;
  size_t off = 0;
  long long tiledBins = 0;
  for (int k = 0; k < numRegs; ++k) {
    const long long b = 1ll << c->q[regIdxs[k]];
    if (tiled_ok(c, tiledBins + b)) {
      outs.push_back({regIdxs[k]});
      outPos.push_back(off);
      tiledBins += b;
    } else {
      big.push_back(regIdxs[k]);
      bigPos.push_back(off);
    }
    off += (size_t)b;
  }
  for (size_t k = 0; k < big.size(); ++k)
    if (!measure(c, &big[k], 1, probsOut + bigPos[k], w)) return;
  if (outs.empty()) return;
  // qubit registers after a row program on the last register: the program writes
  // the row sums on its way out and the marginals come from them, not another pass
  const bool asked = request_row_sums(c, outs);
  const bool ok = ready(c, w);
  c->rowSums = nullptr;
  if (!ok) return;
  const int parts = asked ? c->rowSumParts : 0;
  c->rowSumParts = 0;
  arena_reset(c);
  double* dOut = (double*)arena_alloc(c, (size_t)tiledBins * sizeof(double));
  if (!dOut) return;
  if (!(parts > 0 ? marginals_from_rows(c, outs, parts, dOut) : marginals_tiled(c, outs, dOut))) return;
  size_t src = 0;
  for (size_t k = 0; k < outs.size(); ++k) {
    const size_t b = (size_t)1 << c->q[outs[k][0]];
    if (!cuda_ok(c, cudaMemcpyAsync(probsOut + outPos[k], dOut + src, b * sizeof(double),
                                    cudaMemcpyDeviceToHost, c->stream), "marginal copy"))
      return;
    src += b;
  }
  stream_sync(c, "marginal sync");
}

void cvdvGetFidelity(CVDVContext* ctx, void** devicePtrs, int numReg, double* fidOut) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (fidOut) *fidOut = 0.0;
  if (!fidOut || !devicePtrs) {
    set_error(c, kErrInvalidArg, "cvdvGetFidelity: NULL argument");
    return;
  }
  if (numReg != c->numReg) {
    set_error(c, kErrInvalidArg, "cvdvGetFidelity: numReg mismatch (context %d, got %d)",
              c->numReg, numReg);
    return;
  }
  if (!ready(c, "cvdvGetFidelity")) return;
  arena_reset(c);
  size_t totalN = 0;
  for (int r = 0; r < numReg; ++r) totalN += (size_t)1 << c->q[r];
  double2* base = (double2*)arena_alloc(c, totalN * sizeof(double2));
  if (!base) return;
  std::vector<const double2*> arrs(numReg);
  size_t off = 0;
  for (int r = 0; r < numReg; ++r) {
    size_t N = (size_t)1 << c->q[r];
    if (!cuda_ok(c, cudaMemcpyAsync(base + off, devicePtrs[r], N * sizeof(double2), cudaMemcpyDefault,
                                    c->stream), "cvdvGetFidelity copy"))
      return;
    arrs[r] = base + off;
    off += N;
  }
  // outer product of all registers but the last (same helper as the initialiser)
  int R = c->numReg, qLast = c->q[R - 1];
  uint64_t nOuter = 1ull << (c->totalQbt - qLast);
  double2* outer = (double2*)arena_alloc(c, nOuter * sizeof(double2));
  if (!outer) return;
  if (!launch_outer(c, arrs.data(), outer)) return;
  double2 ip;
  bool ok = c->precision == kC128
                ? reduce(c, OpSep<double2>{(const double2*)c->state(), outer, arrs[R - 1], qLast}, c->size(), &ip)
                : reduce(c, OpSep<float2>{(const float2*)c->state(), outer, arrs[R - 1], qLast}, c->size(), &ip);
  if (ok) *fidOut = ip.x * ip.x + ip.y * ip.y;
}

double cvdvGetPhotonNumber(CVDVContext* ctx, int regIdx) {
  if (!ctx) return -1.0;
  Context* c = C(ctx);
  if (regIdx < 0 || regIdx >= c->numReg) {
    set_error(c, kErrInvalidArg, "cvdvGetPhotonNumber: invalid register index %d", regIdx);
    return -1.0;
  }
  if (!ready(c, "cvdvGetPhotonNumber")) return -1.0;
  arena_reset(c);
  int N = 1 << c->q[regIdx];
  double cc = (double)(N - 1) * 0.5, dx = c->dx[regIdx];
  int sh = c->flw[regIdx];
  double2 q2, p2;
  bool ok = c->precision == kC128
                ? reduce(c, OpX2<double2>{(const double2*)c->state(), sh, N - 1, cc, dx}, c->size(), &q2)
                : reduce(c, OpX2<float2>{(const float2*)c->state(), sh, N - 1, cc, dx}, c->size(), &q2);
  if (!ok) return -1.0;
  // <p^2>: |FtQ2P psi|^2 = |FFT(pre-twiddle * psi)|^2 / N, computed out of place
  Term tw{};
  tw.kind = kTermFtTw;
  tw.r = regIdx;
  tw.s = -1;
  tw.ctrlBit = -1;
  tw.sign = 1;
  Term sc{};
  sc.kind = kTermScalar;
  sc.ctrlBit = -1;
  sc.g0 = make_double2(1.0 / sqrt((double)N), 0.0);
  FactorList pre;
  std::vector<Term> left;
  if (!build_factor_list(c, {tw, sc}, &pre, &left)) return -1.0;
  size_t bytes = (size_t)c->size() * c->elemBytes;
  char* scratch = (char*)big_scratch(c, bytes);
  if (!scratch) return -1.0;
  // the second state buffer is free between flushes: it serves as the pass temporary
  if (!launch_fft_into(c, regIdx, 1, pre, scratch, c->other())) return -1.0;
  ok = c->precision == kC128
           ? reduce(c, OpX2<double2>{(const double2*)scratch, sh, N - 1, cc, dx}, c->size(), &p2)
           : reduce(c, OpX2<float2>{(const float2*)scratch, sh, N - 1, cc, dx}, c->size(), &p2);
  if (!ok) return -1.0;
  return (q2.x + p2.x - 1.0) / 2.0;
}

void cvdvFidelityStatevectors(CVDVContext* ctx1, CVDVContext* ctx2, double* fidOut) {
  if (fidOut) *fidOut = 0.0;
  if (!ctx1 || !ctx2 || !fidOut) return;
  Context* a = C(ctx1);
  Context* b = C(ctx2);
  if (a->totalQbt != b->totalQbt || a->numReg == 0 || b->numReg == 0) {
    set_error(a, kErrInvalidArg, "cvdvFidelityStatevectors: total qubit count mismatch (%d vs %d)",
              a->totalQbt, b->totalQbt);
    return;
  }
  if (!ready(a, "cvdvFidelityStatevectors") || !ready(b, "cvdvFidelityStatevectors")) return;
  if (a != b && !stream_sync(b, "fidelity sync")) return;
  arena_reset(a);
  double2 ip;
  bool ok;
  uint64_t n = a->size();
  if (a->precision == kC128 && b->precision == kC128)
    ok = reduce(a, OpDot<double2, double2>{(const double2*)a->state(), (const double2*)b->state()}, n, &ip);
  else if (a->precision == kC128)
    ok = reduce(a, OpDot<double2, float2>{(const double2*)a->state(), (const float2*)b->state()}, n, &ip);
  else if (b->precision == kC128)
    ok = reduce(a, OpDot<float2, double2>{(const float2*)a->state(), (const double2*)b->state()}, n, &ip);
  else
    ok = reduce(a, OpDot<float2, float2>{(const float2*)a->state(), (const float2*)b->state()}, n, &ip);
  if (ok) *fidOut = ip.x * ip.x + ip.y * ip.y;
}

int cvdvGetLastError(CVDVContext* ctx, char* msg, int len) {
  if (!ctx) return global_error(msg, len);
  Context* c = C(ctx);
  if (msg && len > 0) {
    strncpy(msg, c->lastMsg.c_str(), (size_t)len - 1);
    msg[len - 1] = 0;
  }
  return c->lastErr;
}

void cvdvClearError(CVDVContext* ctx) {
  if (!ctx) return;
  C(ctx)->lastErr = kOk;
  C(ctx)->lastMsg.clear();
}

}  // extern "C"

// ====================================================================== marginal without allocation
// Some callers cannot let a library call cudaMalloc: an application whose
// device memory is owned by another allocator (a framework's caching pool
// that has reserved the GPU, so a plain cudaMalloc fails although the pool has
// room), a service that sizes its device memory once at start-up and must not
// grow it afterwards, or a loop that cannot afford the device-wide
// synchronisation that cudaMalloc and cudaFree may perform.  For them,
// cvdvMeasureMultipleNoAlloc computes the same joint marginal as
// cvdvMeasureMultiple on a state they own, writes it to an output they own,
// and keeps its per-block partial histograms in the fixed array below.
//
// The array is part of this library's device code: every GPU that loads the
// library holds it (kNoAllocBlocks x kNoAllocMaxBins doubles = 4.625 MiB) until
// the process exits.  Every call shares it and it keeps the last call's
// contents; nothing in it has to start at zero, because each block writes its
// whole histogram row before the final kernel reads it.  Calls whose kernels
// overlap on the GPU (different streams, no ordering between them) race on it.
namespace cvdv {

constexpr int kNoAllocBlocks = 148;
constexpr int kNoAllocMaxBins = 4096;  // 2^12: joint marginals of up to 12 qubits
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noAllocScratch[kNoAllocBlocks * kNoAllocMaxBins];

static std::mutex g_noAllocMu;
static double* g_noAllocPtr[kNoAllocMaxDevices];  // device address per device, set up on first use

// Device address of the scratch array on the current device.  The array's name
// in host code is only a handle for the runtime; the address the kernels use is
// looked up once per device, with that device current.
static double* no_alloc_scratch(int dev, bool report) {
  std::lock_guard<std::mutex> lk(g_noAllocMu);
  if (!g_noAllocPtr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noAllocScratch);
    if (e != cudaSuccess) {
      cudaGetLastError();
      if (report)
        set_error(nullptr, kErrCuda, "cvdvMeasureMultipleNoAlloc: scratch lookup on device %d: %s", dev,
                  cudaGetErrorString(e));
      return nullptr;
    }
    g_noAllocPtr[dev] = (double*)p;
  }
  return g_noAllocPtr[dev];
}

// Loads, on device dev (current), the part of this library's device code that
// holds the array and the two kernels the entry point launches, and records the
// array's address.  Under CUDA's lazy module loading (the default since 12.2)
// that code is loaded on its first use, which takes device memory (the array and
// the kernels' code); cvdvCreate / cvdvCreateEx call this for their device so a
// process that made a context makes its first cvdvMeasureMultipleNoAlloc call
// without that load.
static std::atomic<bool> g_noAllocLoaded[kNoAllocMaxDevices];

double* no_alloc_prepare(int dev, bool report) {
  if (dev < 0 || dev >= kNoAllocMaxDevices) return nullptr;
  double* p = no_alloc_scratch(dev, report);
  if (!p || g_noAllocLoaded[dev].load()) return p;
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, k_marg_smem<double2>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_marg_smem<float2>);
  if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k_marg_final);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (report)
      set_error(nullptr, kErrCuda, "cvdvMeasureMultipleNoAlloc: loading its kernels on device %d: %s", dev,
                cudaGetErrorString(e));
    return nullptr;
  }
  g_noAllocLoaded[dev].store(true);
  return p;
}

static bool device_pointer_on(const void* p, int dev) {
  cudaPointerAttributes a{};
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) && a.device == dev;
}

}  // namespace cvdv

extern "C" int cvdvMeasureMultipleNoAlloc(const void* state, int precision, const int* numQubits,
                                          int numReg, const int* regIdxs, int numRegs, double* probsOut,
                                          void* stream) {
  const char* fn = "cvdvMeasureMultipleNoAlloc";
  if (!state || !probsOut || !numQubits || !regIdxs) {
    set_error(nullptr, kErrInvalidArg, "%s: null pointer argument", fn);
    return kErrInvalidArg;
  }
  if (precision != kC128 && precision != kC64) {
    set_error(nullptr, kErrInvalidArg, "%s: precision %d (0 = complex128, 1 = complex64)", fn, precision);
    return kErrInvalidArg;
  }
  if (numReg < 1 || numReg > kMaxRegs) {
    set_error(nullptr, kErrInvalidArg, "%s: numReg %d outside 1..%d", fn, numReg, kMaxRegs);
    return kErrInvalidArg;
  }
  int flw[kMaxRegs];
  int total = 0;
  for (int r = numReg - 1; r >= 0; --r) {
    if (numQubits[r] < 1 || numQubits[r] > kMaxTotalQubits) {
      set_error(nullptr, kErrInvalidArg, "%s: register %d has %d qubits", fn, r, numQubits[r]);
      return kErrInvalidArg;
    }
    flw[r] = total;
    total += numQubits[r];
  }
  if (total > kMaxTotalQubits) {
    set_error(nullptr, kErrInvalidArg, "%s: %d qubits in total exceed %d", fn, total, kMaxTotalQubits);
    return kErrInvalidArg;
  }
  if (numRegs < 1 || numRegs > 16 || numRegs > numReg) {
    set_error(nullptr, kErrInvalidArg, "%s: numRegs %d outside 1..min(16, numReg)", fn, numRegs);
    return kErrInvalidArg;
  }
  MargDesc D{};
  D.nSel = numRegs;
  long long bins = 1;
  for (int s = 0; s < numRegs; ++s) {
    int r = regIdxs[s];
    if (r < 0 || r >= numReg) {
      set_error(nullptr, kErrInvalidArg, "%s: register index %d outside 0..%d", fn, r, numReg - 1);
      return kErrInvalidArg;
    }
    for (int t = 0; t < s; ++t)
      if (regIdxs[t] == r) {
        set_error(nullptr, kErrInvalidArg, "%s: register %d selected twice", fn, r);
        return kErrInvalidArg;
      }
    bins <<= numQubits[r];  // at most 2^12 * 2^34, no overflow
    if (bins > kNoAllocMaxBins) break;
    D.shift[s] = flw[r];
    D.mask[s] = (1 << numQubits[r]) - 1;
    D.stride[s] = bins >> numQubits[r];  // first selected register fastest, as cvdvMeasureMultiple
  }
  if (bins > kNoAllocMaxBins) {
    set_error(nullptr, kErrInvalidArg,
              "%s: the selected registers span more than %d outcomes; this entry point holds at most "
              "%d (12 qubits) -- use cvdvMeasureMultiple for larger marginals",
              fn, kNoAllocMaxBins, kNoAllocMaxBins);
    return kErrInvalidArg;
  }
  D.outSize = bins;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices) {
    cudaGetLastError();
    set_error(nullptr, kErrCuda, "%s: no usable current device", fn);
    return kErrCuda;
  }
  const size_t elem = precision == kC128 ? sizeof(double2) : sizeof(float2);
  if (((uintptr_t)state % elem) || ((uintptr_t)probsOut % sizeof(double)) ||
      !device_pointer_on(state, dev) || !device_pointer_on(probsOut, dev)) {
    set_error(nullptr, kErrInvalidArg,
              "%s: state and probsOut must be aligned device memory of the current device %d", fn, dev);
    return kErrInvalidArg;
  }
  double* scratch = no_alloc_prepare(dev, true);
  if (!scratch) return kErrCuda;
  cudaStream_t s = (cudaStream_t)stream;
  const uint64_t n = 1ull << total;
  uint64_t maxBlocks = (n + 255) / 256;
  int blocks = kNoAllocBlocks < maxBlocks ? kNoAllocBlocks : (int)maxBlocks;
  size_t smem = (size_t)bins * sizeof(double);
  // an error the caller's own earlier CUDA work left pending is theirs: it is
  // neither reported as this call's nor cleared
  const cudaError_t before = cudaPeekAtLastError();
  {
    LaunchScope _ls(nullptr, kKReduce);
    if (precision == kC128)
      k_marg_smem<double2><<<blocks, 256, smem, s>>>((const double2*)state, n, D, scratch);
    else
      k_marg_smem<float2><<<blocks, 256, smem, s>>>((const float2*)state, n, D, scratch);
  }
  {
    LaunchScope _ls(nullptr, kKReduce);
    k_marg_final<<<(int)((bins + 255) / 256), 256, 0, s>>>(scratch, blocks, bins, probsOut);
  }
  e = cudaPeekAtLastError();
  if (e != cudaSuccess && e != before) {
    cudaGetLastError();
    set_error(nullptr, kErrCuda, "%s: launch: %s", fn, cudaGetErrorString(e));
    return kErrCuda;
  }
  return kOk;
}
