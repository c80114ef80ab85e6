// Batched variational circuits: many parameter sets of one circuit of qubit
// rotations Rx(theta) and real conditional displacements cd(beta) on a layout
// [qubit registers..., mode], run side by side, with the adjoint sweep that gives
// the gradient of a fidelity loss.
//
// The states of the batch are one caller-owned array: instance b occupies
// [b 2^n, (b + 1) 2^n), the mode is the last (contiguous) register of q bits,
// and each instance has its own angle theta_b / displacement beta_b per gate.
//
// cd(beta) = FtP2Q . exp(i beta K) . FtQ2P with K = -sqrt2 Z x_k, Z = +1 when the
// control qubit is 0 (src/cuda/gates.cu:163-204).  The two basis changes'
// twiddles meet in the middle: FtQ2P's post-twiddle and FtP2Q's pre-twiddle are
// conjugate and their global phases cancel, so a cd row program is
//   exp(i theta_j) . DFT . [exp(i beta K_k) / N] . IDFT . exp(-i theta_j)
// with theta_j = pi (N-1)(2j-N+1) / (2N), run on one row held in registers.
//
// Adjoint: with psi_l the state after gate l and lambda_l = U_{l+1}^+ ... U_L^+ t,
// d<t|psi>/dp_l = i <lambda_l| G_l |psi_l> for U_l = exp(i p_l G_l).  One kernel
// per gate computes g_l = <lambda_l| G_l |psi_l> and applies U_l^+ to both
// states: G = -X/2 for Rx, and <lambda|K_cd|psi> = <F lambda| K |F psi> (F =
// FtQ2P) for cd, taken between the two transforms.

#include <cooperative_groups.h>

#include <cmath>

#include "../../include/cvdv.h"
#include "cvdv_internal.cuh"
#include "row_fft.cuh"

namespace cg = cooperative_groups;

namespace cvdv {

constexpr int kBatchThreads = 256;

template <typename C> __device__ __forceinline__ double2 tod_b(C v);
template <> __device__ __forceinline__ double2 tod_b<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ double2 tod_b<float2>(float2 v) {
  return make_double2((double)v.x, (double)v.y);
}

// sum over the CTA (valid in thread 0)
__device__ __forceinline__ double2 block_sum2_b(double2 v) {
  __shared__ double2 ws[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_down_sync(0xffffffffu, v.x, o);
    v.y += __shfl_down_sync(0xffffffffu, v.y, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
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

// exp(i theta_j) of the centred-grid transform, exact (integer argument mod 4N)
__device__ __forceinline__ double2 ft_twiddle(int j, int N, int sign) {
  long long m = (long long)(N - 1) * (2LL * j - N + 1);
  const long long M4 = 4LL * N;
  m %= M4;
  if (m < 0) m += M4;
  double s, c;
  sincospi((double)sign * (double)m / (double)(2 * N), &s, &c);
  return make_double2(c, s);
}

// Ratio of ft_twiddle between j + d and j: exp(i sign pi (N-1) d / N), the angle
// reduced exactly in integers.  A thread's points t + k TPR take the twiddle as a
// running product from its exact value at t (16 steps: a few units of 1e-16).
__device__ __forceinline__ double2 ft_twiddle_step(int d, int N, int sign) {
  const long long m = ((long long)(N - 1) * d) % (2LL * N);
  double s, c;
  sincospi((double)sign * (double)m / (double)N, &s, &c);
  return make_double2(c, s);
}

// ---------------------------------------------------------------- Rx
template <typename C>
__global__ void __launch_bounds__(kBatchThreads) k_b_rx(C* __restrict__ st, uint64_t nPairs, int n, int bit,
                                                       const double* __restrict__ th, double sign) {
  for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nPairs;
       p += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b = p >> (n - 1);
    const uint64_t lp = p & ((1ull << (n - 1)) - 1);
    const uint64_t i0 = (b << n) | ((lp >> bit) << (bit + 1)) | (lp & ((1ull << bit) - 1));
    const uint64_t i1 = i0 | (1ull << bit);
    double s, c;
    sincos(0.5 * sign * __ldg(th + b), &s, &c);
    const double2 x = tod_b(st[i0]), y = tod_b(st[i1]);
    // [[c, -i s], [-i s, c]]
    st[i0] = fromd<C>(make_double2(c * x.x + s * y.y, c * x.y - s * y.x));
    st[i1] = fromd<C>(make_double2(s * x.y + c * y.x, -s * x.x + c * y.y));
  }
}

// g = <lambda| (-X/2) |psi> over the pairs of one instance chunk, then
// Rx(-theta) on both states.  One partial per CTA; a CTA stays in one instance.
template <typename C>
__global__ void __launch_bounds__(kBatchThreads) k_b_rx_adj(C* __restrict__ psi, C* __restrict__ lam, int n,
                                                           int bit, const double* __restrict__ th,
                                                           int ctaPerInst, double2* __restrict__ part) {
  const uint64_t pairsPerInst = 1ull << (n - 1);
  const int b = blockIdx.x / ctaPerInst, c = blockIdx.x % ctaPerInst;
  const uint64_t chunk = pairsPerInst / ctaPerInst;
  double s, co;
  sincos(-0.5 * __ldg(th + b), &s, &co);
  double gx = 0.0, gy = 0.0;
  for (uint64_t lp = c * chunk + threadIdx.x; lp < (c + 1) * chunk; lp += blockDim.x) {
    const uint64_t i0 = ((uint64_t)b << n) | ((lp >> bit) << (bit + 1)) | (lp & ((1ull << bit) - 1));
    const uint64_t i1 = i0 | (1ull << bit);
    const double2 p0 = tod_b(psi[i0]), p1 = tod_b(psi[i1]);
    const double2 l0 = tod_b(lam[i0]), l1 = tod_b(lam[i1]);
    // conj(l0) (-p1/2) + conj(l1) (-p0/2)
    gx -= 0.5 * (l0.x * p1.x + l0.y * p1.y + l1.x * p0.x + l1.y * p0.y);
    gy -= 0.5 * (l0.x * p1.y - l0.y * p1.x + l1.x * p0.y - l1.y * p0.x);
    psi[i0] = fromd<C>(make_double2(co * p0.x + s * p1.y, co * p0.y - s * p1.x));
    psi[i1] = fromd<C>(make_double2(s * p0.y + co * p1.x, -s * p0.x + co * p1.y));
    lam[i0] = fromd<C>(make_double2(co * l0.x + s * l1.y, co * l0.y - s * l1.x));
    lam[i1] = fromd<C>(make_double2(s * l0.y + co * l1.x, -s * l0.x + co * l1.y));
  }
  const double2 g = block_sum2_b(make_double2(gx, gy));
  if (threadIdx.x == 0) part[blockIdx.x] = g;
}

// ---------------------------------------------------------------- cd rows
// R rows of N = 2^LOGQ points per CTA (TPR = N/16 threads per row).
template <int LOGQ>
struct BRow {
  static constexpr int N = 1 << LOGQ, TPR = N >> 4;
  static constexpr int LOGR = LOGQ >= 12 ? 0 : 12 - LOGQ;
  static constexpr int NT = TPR << LOGR;
  static constexpr int RS = N + (N >> 4);
};

template <int LOGQ>
__device__ __forceinline__ void b_fill_twiddles(double2* lo, int tid, int nt) {
  constexpr int N = 1 << LOGQ;
  for (int i = tid; i < 64 + (N >> 6); i += nt) {
    const int e = i < 64 ? i : (i - 64) << 6;
    double s, c;
    sincospi(-2.0 * (double)e / (double)N, &s, &c);
    lo[i] = make_double2(c, s);
  }
}

// exp(i sgn beta K_k) / N with K_k = -sqrt2 z x_k
__device__ __forceinline__ double2 b_kick(int k, int N, double coef) {
  const double dx = sqrt(2.0 * M_PI / (double)N);
  const double x = ((double)k - 0.5 * (double)(N - 1)) * dx;
  double s, c;
  sincos(coef * x, &s, &c);
  const double inv = 1.0 / (double)N;
  return make_double2(c * inv, s * inv);
}

// exp(i coef dx d): the ratio of b_kick between k + d and k
__device__ __forceinline__ double2 b_kick_step(int d, int N, double coef) {
  const double dx = sqrt(2.0 * M_PI / (double)N);
  double s, c;
  sincos(coef * dx * (double)d, &s, &c);
  return make_double2(c, s);
}

template <typename C, int LOGQ>
__global__ void __launch_bounds__(BRow<LOGQ>::NT, 2)
    k_b_cd(C* __restrict__ st, uint64_t nRows, int n, int ctrlBit, const double* __restrict__ beta, double sign) {
  using G = BRow<LOGQ>;
  constexpr int N = G::N, TPR = G::TPR;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  double2* lo = reinterpret_cast<double2*>(sm + (G::RS << G::LOGR));
  double2* hi = lo + 64;
  const int tid = threadIdx.x, row = tid / TPR, t = tid % TPR;
  C* smrow = sm + row * G::RS;
  const uint64_t gRow = ((uint64_t)blockIdx.x << G::LOGR) + row;
  const bool valid = gRow < nRows;  // the last CTA may hold fewer rows; its spare rows only sync
  const uint64_t rowBase = (valid ? gRow : 0) << LOGQ;
  const uint64_t b = rowBase >> n;
  const double zs = ((rowBase >> ctrlBit) & 1ull) ? -1.0 : 1.0;
  const double coef = sign * __ldg(beta + b) * (-M_SQRT2) * zs;
  b_fill_twiddles<LOGQ>(lo, tid, G::NT);
  C v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = st[rowBase + t + k * TPR];
  const double2 tw0 = ft_twiddle(t, N, 1), tws = ft_twiddle_step(TPR, N, 1);
  double2 f = tw0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    v[k] = cmul(v[k], fromd<C>(f));
    f = dmul(f, tws);
  }
  __syncthreads();
  rr_stages<C, 1, LOGQ, 0, 4>(v, smrow, t, lo, hi);
  f = b_kick(t, N, coef);
  const double2 ks = b_kick_step(TPR, N, coef);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    v[k] = cmul(v[k], fromd<C>(f));
    f = dmul(f, ks);
  }
  rr_stages<C, -1, LOGQ, 0, 4>(v, smrow, t, lo, hi);
  if (!valid) return;
  f = cconj(tw0);  // ft_twiddle(j, N, -1) = conj(ft_twiddle(j, N, 1))
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    st[rowBase + t + k * TPR] = cmul(v[k], fromd<C>(f));
    f = dmul(f, cconj(tws));
  }
}

// g = <F lambda| K |F psi> for every row (one partial per row), then cd(-beta)
// on both states.
template <typename C, int LOGQ>
__global__ void __launch_bounds__(BRow<LOGQ>::NT, 1)
    k_b_cd_adj(C* __restrict__ psi, C* __restrict__ lam, uint64_t nRows, int n, int ctrlBit,
               const double* __restrict__ beta, double2* __restrict__ part) {
  using G = BRow<LOGQ>;
  constexpr int N = G::N, TPR = G::TPR;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  C* keep = sm + (G::RS << G::LOGR);  // the transformed psi rows, one slot per thread and k
  double2* lo = reinterpret_cast<double2*>(keep + (N << G::LOGR));
  double2* hi = lo + 64;
  const int tid = threadIdx.x, row = tid / TPR, t = tid % TPR;
  C* smrow = sm + row * G::RS;
  C* krow = keep + row * N;
  const uint64_t gRow = ((uint64_t)blockIdx.x << G::LOGR) + row;
  const bool valid = gRow < nRows;  // spare rows of the last CTA only take part in the syncs
  const uint64_t rowBase = (valid ? gRow : 0) << LOGQ;
  const uint64_t b = rowBase >> n;
  const double zs = ((rowBase >> ctrlBit) & 1ull) ? -1.0 : 1.0;
  const double kz = -M_SQRT2 * zs;                // K_k = kz x_k
  const double coef = -__ldg(beta + b) * kz;      // exp(-i beta K)
  const double dx = sqrt(2.0 * M_PI / (double)N);
  b_fill_twiddles<LOGQ>(lo, tid, G::NT);
  const double2 tw0 = ft_twiddle(t, N, 1), tws = ft_twiddle_step(TPR, N, 1);
  C v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = psi[rowBase + t + k * TPR];
  double2 f = tw0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    v[k] = cmul(v[k], fromd<C>(f));
    f = dmul(f, tws);
  }
  __syncthreads();
  rr_stages<C, 1, LOGQ, 0, 4>(v, smrow, t, lo, hi);
#pragma unroll
  for (int k = 0; k < 16; ++k) krow[t + k * TPR] = v[k];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = lam[rowBase + t + k * TPR];
  f = tw0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    v[k] = cmul(v[k], fromd<C>(f));
    f = dmul(f, tws);
  }
  rr_stages<C, 1, LOGQ, 0, 4>(v, smrow, t, lo, hi);
  // <F lambda| K |F psi> = (1/N) sum_k conj(L_k) K_k P_k for the unnormalised transforms
  double gx = 0.0, gy = 0.0;
  f = b_kick(t, N, coef);
  const double2 ks = b_kick_step(TPR, N, coef);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int kk = t + k * TPR;
    const double2 P = tod_b(krow[kk]), L = tod_b(v[k]);
    const double w = kz * ((double)kk - 0.5 * (double)(N - 1)) * dx / (double)N;
    gx += w * (L.x * P.x + L.y * P.y);
    gy += w * (L.x * P.y - L.y * P.x);
    const C fc = fromd<C>(f);
    v[k] = cmul(v[k], fc);
    krow[kk] = cmul(krow[kk], fc);
    f = dmul(f, ks);
  }
  rr_stages<C, -1, LOGQ, 0, 4>(v, smrow, t, lo, hi);
  if (valid) {
    f = cconj(tw0);  // ft_twiddle(j, N, -1) = conj(ft_twiddle(j, N, 1))
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      lam[rowBase + t + k * TPR] = cmul(v[k], fromd<C>(f));
      f = dmul(f, cconj(tws));
    }
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = krow[t + k * TPR];
  rr_stages<C, -1, LOGQ, 0, 4>(v, smrow, t, lo, hi);
  if (valid) {
    f = cconj(tw0);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      psi[rowBase + t + k * TPR] = cmul(v[k], fromd<C>(f));
      f = dmul(f, cconj(tws));
    }
  }
  // per-row sum: lanes of one row (TPR >= 16 consecutive threads), then the row's warps
  __shared__ double2 racc[1 << G::LOGR];
  if (tid < (1 << G::LOGR)) racc[tid] = make_double2(0.0, 0.0);
  __syncthreads();
  constexpr int W = TPR < 32 ? TPR : 32;
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) {
    gx += __shfl_down_sync(0xffffffffu, gx, o, W);
    gy += __shfl_down_sync(0xffffffffu, gy, o, W);
  }
  if ((tid & (W - 1)) == 0) {
    atomicAdd(&racc[row].x, gx);
    atomicAdd(&racc[row].y, gy);
  }
  __syncthreads();
  if (tid < (1 << G::LOGR) && ((uint64_t)blockIdx.x << G::LOGR) + tid < nRows)
    part[((uint64_t)blockIdx.x << G::LOGR) + tid] = racc[tid];
}

// ---------------------------------------------------------------- Rx then cd, fused
// A layer Rx(theta) on qubit bit q followed by cd(beta) controlled by the same bit
// runs as one pass: a cluster of two CTAs holds the two rows (mode arrays) that
// differ only in that bit, CTA rank = the bit's value.  Each loads its row, the
// Rx mixes it with the partner's row read from the partner's shared memory, and
// the cd runs on the row in registers.  Rows of 2^9 .. 2^12 points, one CTA each.
template <int LOGQ>
struct BPair {
  static constexpr int N = 1 << LOGQ, TPR = N >> 4, RS = N + (N >> 4);
};

// the row of cluster rank r for pair index p: the bit at position rb of the row
// index (the qubit bit above the mode) set to r
__device__ __forceinline__ uint64_t pair_row(uint64_t p, int rb, int r) {
  return ((p >> rb) << (rb + 1)) | (p & ((1ull << rb) - 1)) | ((uint64_t)r << rb);
}

template <typename C, int LOGQ>
__global__ void __launch_bounds__(BPair<LOGQ>::TPR, 1)
    k_b_rxcd(C* __restrict__ st, int n, int bit, const double* __restrict__ th, const double* __restrict__ beta) {
  using G = BPair<LOGQ>;
  constexpr int N = G::N, TPR = G::TPR;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  double2* lo = reinterpret_cast<double2*>(sm + G::RS);
  double2* hi = lo + 64;
  cg::cluster_group cl = cg::this_cluster();
  const int r = (int)cl.block_rank(), t = threadIdx.x;
  const uint64_t rowBase = pair_row(blockIdx.x >> 1, bit - LOGQ, r) << LOGQ;
  const uint64_t b = rowBase >> n;
  b_fill_twiddles<LOGQ>(lo, t, TPR);
  C v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = st[rowBase + t + k * TPR];
  // Rx: v <- c v - i s w with w the partner row's amplitude at the same point
  // ([[c, -i s], [-i s, c]] is symmetric in the two rows)
#pragma unroll
  for (int k = 0; k < 16; ++k) sm[t + k * TPR] = v[k];
  cl.sync();
  {
    const C* pw = cl.map_shared_rank(sm, r ^ 1);
    double s, c;
    sincos(0.5 * __ldg(th + b), &s, &c);
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      const double2 x = tod_b(v[k]), y = tod_b(pw[t + k * TPR]);
      v[k] = fromd<C>(make_double2(c * x.x + s * y.y, c * x.y - s * y.x));
    }
  }
  cl.sync();  // the partner has read this CTA's row before the stages reuse the buffer
  // cd controlled by the bit (value r): as k_b_cd
  const double coef = __ldg(beta + b) * (-M_SQRT2) * (r ? -1.0 : 1.0);
  const double2 tw0 = ft_twiddle(t, N, 1), tws = ft_twiddle_step(TPR, N, 1);
  double2 f = tw0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    v[k] = cmul(v[k], fromd<C>(f));
    f = dmul(f, tws);
  }
  rr_stages<C, 1, LOGQ, 0, 4>(v, sm, t, lo, hi);
  f = b_kick(t, N, coef);
  const double2 ks = b_kick_step(TPR, N, coef);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    v[k] = cmul(v[k], fromd<C>(f));
    f = dmul(f, ks);
  }
  rr_stages<C, -1, LOGQ, 0, 4>(v, sm, t, lo, hi);
  f = cconj(tw0);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    st[rowBase + t + k * TPR] = cmul(v[k], fromd<C>(f));
    f = dmul(f, cconj(tws));
  }
}

// Adjoint of the fused layer, walked backwards: the cd's g_cd = <F lambda| K |F psi>
// and cd^+ on both states (as k_b_cd_adj), then the Rx's
// g_rx = <lambda| (-X/2) |psi> and Rx(-theta) on both, the partner rows read from
// the partner's shared memory.  One partial of each per row.
// With a single qubit bit above the mode (one cluster per instance) the cluster
// adds its two rows' partials itself and writes gCd / gRx (partCd, partRx null).
template <typename C, int LOGQ>
__global__ void __launch_bounds__(BPair<LOGQ>::TPR, 1)
    k_b_cdrx_adj(C* __restrict__ psi, C* __restrict__ lam, int n, int bit, const double* __restrict__ th,
                 const double* __restrict__ beta, double2* __restrict__ partCd, double2* __restrict__ partRx,
                 double* __restrict__ gCd, double* __restrict__ gRx) {
  __shared__ double2 sums[2];  // this row's g_cd and g_rx
  using G = BPair<LOGQ>;
  constexpr int N = G::N, TPR = G::TPR;
  extern __shared__ __align__(16) unsigned char smraw[];
  C* sm = reinterpret_cast<C*>(smraw);
  C* keep = sm + G::RS;  // the transformed psi row, then psi after cd^+
  C* park = keep + N;    // lambda after cd^+
  double2* lo = reinterpret_cast<double2*>(park + N);
  double2* hi = lo + 64;
  cg::cluster_group cl = cg::this_cluster();
  const int r = (int)cl.block_rank(), t = threadIdx.x;
  const uint64_t row = pair_row(blockIdx.x >> 1, bit - LOGQ, r);
  const uint64_t rowBase = row << LOGQ;
  const uint64_t b = rowBase >> n;
  const double kz = -M_SQRT2 * (r ? -1.0 : 1.0);  // K_k = kz x_k
  const double coef = -__ldg(beta + b) * kz;       // exp(-i beta K)
  const double dx = sqrt(2.0 * M_PI / (double)N);
  b_fill_twiddles<LOGQ>(lo, t, TPR);
  const double2 tw0 = ft_twiddle(t, N, 1), tws = ft_twiddle_step(TPR, N, 1);
  C v[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = psi[rowBase + t + k * TPR];
  double2 f = tw0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    v[k] = cmul(v[k], fromd<C>(f));
    f = dmul(f, tws);
  }
  __syncthreads();
  rr_stages<C, 1, LOGQ, 0, 4>(v, sm, t, lo, hi);
#pragma unroll
  for (int k = 0; k < 16; ++k) keep[t + k * TPR] = v[k];
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = lam[rowBase + t + k * TPR];
  f = tw0;
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    v[k] = cmul(v[k], fromd<C>(f));
    f = dmul(f, tws);
  }
  rr_stages<C, 1, LOGQ, 0, 4>(v, sm, t, lo, hi);
  double gx = 0.0, gy = 0.0;
  f = b_kick(t, N, coef);
  const double2 ks = b_kick_step(TPR, N, coef);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    const int kk = t + k * TPR;
    const double2 P = tod_b(keep[kk]), L = tod_b(v[k]);
    const double w = kz * ((double)kk - 0.5 * (double)(N - 1)) * dx / (double)N;
    gx += w * (L.x * P.x + L.y * P.y);
    gy += w * (L.x * P.y - L.y * P.x);
    const C fc = fromd<C>(f);
    v[k] = cmul(v[k], fc);
    keep[kk] = cmul(keep[kk], fc);
    f = dmul(f, ks);
  }
  rr_stages<C, -1, LOGQ, 0, 4>(v, sm, t, lo, hi);
  f = cconj(tw0);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    park[t + k * TPR] = cmul(v[k], fromd<C>(f));
    f = dmul(f, cconj(tws));
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) v[k] = keep[t + k * TPR];
  rr_stages<C, -1, LOGQ, 0, 4>(v, sm, t, lo, hi);
  f = cconj(tw0);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    keep[t + k * TPR] = cmul(v[k], fromd<C>(f));
    f = dmul(f, cconj(tws));
  }
  // this row's g_cd
  {
    const double2 g = block_sum2_b(make_double2(gx, gy));
    if (t == 0) {
      sums[0] = g;
      if (partCd) partCd[row] = g;
    }
  }
  cl.sync();  // both rows of the pair are in shared memory (psi in keep, lambda in park)
  // Rx(-theta) and this row's half of g_rx = sum conj(l_r) (-p_{1-r} / 2)
  {
    const C* pk = cl.map_shared_rank(keep, r ^ 1);
    const C* pp = cl.map_shared_rank(park, r ^ 1);
    double s, co;
    sincos(-0.5 * __ldg(th + b), &s, &co);
    gx = gy = 0.0;
#pragma unroll 4
    for (int k = 0; k < 16; ++k) {
      const int kk = t + k * TPR;
      const double2 p0 = tod_b(keep[kk]), p1 = tod_b(pk[kk]);
      const double2 l0 = tod_b(park[kk]), l1 = tod_b(pp[kk]);
      gx -= 0.5 * (l0.x * p1.x + l0.y * p1.y);
      gy -= 0.5 * (l0.x * p1.y - l0.y * p1.x);
      psi[rowBase + kk] = fromd<C>(make_double2(co * p0.x + s * p1.y, co * p0.y - s * p1.x));
      lam[rowBase + kk] = fromd<C>(make_double2(co * l0.x + s * l1.y, co * l0.y - s * l1.x));
    }
    const double2 g = block_sum2_b(make_double2(gx, gy));
    if (t == 0) {
      sums[1] = g;
      if (partRx) partRx[row] = g;
    }
  }
  cl.sync();  // both rows' sums are in shared memory; no CTA leaves while its partner reads it
  if (!partCd && r == 0 && t < 2) {
    const double2* ps = cl.map_shared_rank(sums, 1);
    const double2 a = sums[t], c = ps[t];
    double* out = t == 0 ? gCd : gRx;
    out[2 * b] = a.x + c.x;
    out[2 * b + 1] = a.y + c.y;
  }
  cl.sync();
}

// <t| a_b> per CTA chunk (t shared by every instance when tStride == 0)
template <typename C>
__global__ void __launch_bounds__(kBatchThreads) k_b_dot(const C* __restrict__ a, const C* __restrict__ tg,
                                                        int n, uint64_t tStride, int ctaPerInst,
                                                        double2* __restrict__ part) {
  const uint64_t per = 1ull << n;
  const int b = blockIdx.x / ctaPerInst, c = blockIdx.x % ctaPerInst;
  const uint64_t chunk = per / ctaPerInst;
  double gx = 0.0, gy = 0.0;
  for (uint64_t i = c * chunk + threadIdx.x; i < (c + 1) * chunk; i += blockDim.x) {
    const double2 x = tod_b(tg[b * tStride + i]), y = tod_b(a[((uint64_t)b << n) + i]);
    gx += x.x * y.x + x.y * y.y;
    gy += x.x * y.y - x.y * y.x;
  }
  const double2 g = block_sum2_b(make_double2(gx, gy));
  if (threadIdx.x == 0) part[blockIdx.x] = g;
}

__global__ void k_b_sum(const double2* __restrict__ part, int per, int B, double* __restrict__ out) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    double x = 0.0, y = 0.0;
    for (int c = 0; c < per; ++c) {
      x += part[b * per + c].x;
      y += part[b * per + c].y;
    }
    out[2 * b] = x;
    out[2 * b + 1] = y;
  }
}

// ---------------------------------------------------------------- host side
static bool b_check(const char* fn, const void* p, int precision, int batch, int n) {
  if (!p || batch < 1 || n < 2 || n > kMaxTotalQubits || (precision != kC128 && precision != kC64)) {
    set_error(nullptr, kErrInvalidArg, "%s: invalid state, batch, qubit count or precision", fn);
    return false;
  }
  return true;
}

static bool b_launch_ok(const char* fn) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error(nullptr, kErrCuda, "%s: %s", fn, cudaGetErrorString(e));
    return false;
  }
  return true;
}

static int b_grid(uint64_t work) {
  uint64_t g = (work + kBatchThreads - 1) / kBatchThreads;
  return (int)(g > 148ull * 8 ? 148ull * 8 : (g < 1 ? 1 : g));
}

// CTAs per instance for the reductions: enough to fill the GPU, dividing the work
static int b_cta_per_inst(int batch, uint64_t unitsPerInst) {
  int c = 1;
  while ((uint64_t)c * 2 * kBatchThreads <= unitsPerInst && batch * c < 148 * 4) c *= 2;
  return c;
}

template <typename C, int LOGQ>
static cudaError_t b_cd_t(void* st, void* lam, int batch, int n, int ctrlBit, const double* beta, double sign,
                          double2* part, cudaStream_t s) {
  using G = BRow<LOGQ>;
  const uint64_t nRows = (uint64_t)batch << (n - LOGQ);
  const unsigned grid = (unsigned)((nRows + (1u << G::LOGR) - 1) >> G::LOGR);
  if (!lam) {
    const size_t smem = (size_t)(G::RS << G::LOGR) * sizeof(C) + (64 + (G::N >> 6)) * sizeof(double2);
    auto kern = k_b_cd<C, LOGQ>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, G::NT, smem, s>>>((C*)st, nRows, n, ctrlBit, beta, sign);
  } else {
    const size_t smem = (size_t)((G::RS + G::N) << G::LOGR) * sizeof(C) + (64 + (G::N >> 6)) * sizeof(double2);
    auto kern = k_b_cd_adj<C, LOGQ>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, G::NT, smem, s>>>((C*)st, (C*)lam, nRows, n, ctrlBit, beta, part);
  }
  return cudaGetLastError();
}

template <typename C>
static cudaError_t b_cd(void* st, void* lam, int batch, int n, int q, int ctrlBit, const double* beta,
                        double sign, double2* part, cudaStream_t s) {
  switch (q) {
    case 8: return b_cd_t<C, 8>(st, lam, batch, n, ctrlBit, beta, sign, part, s);
    case 9: return b_cd_t<C, 9>(st, lam, batch, n, ctrlBit, beta, sign, part, s);
    case 10: return b_cd_t<C, 10>(st, lam, batch, n, ctrlBit, beta, sign, part, s);
    case 11: return b_cd_t<C, 11>(st, lam, batch, n, ctrlBit, beta, sign, part, s);
    case 12: return b_cd_t<C, 12>(st, lam, batch, n, ctrlBit, beta, sign, part, s);
    default: return cudaErrorInvalidValue;
  }
}

static bool b_cd_args(const char* fn, int n, int q, int ctrlBit) {
  if (q < 8 || q > 12 || q >= n || ctrlBit < q || ctrlBit >= n) {
    set_error(nullptr, kErrInvalidArg,
              "%s: the mode must be the last register with 8..12 qubits and the control a bit above it", fn);
    return false;
  }
  return true;
}

// partial sums -> out[2 b], out[2 b + 1]; the partials live in stream-ordered memory
static bool b_finish(const char* fn, double2* part, int per, int batch, double* out, cudaStream_t s) {
  {
    LaunchScope _ls(nullptr, kKReduce);
    k_b_sum<<<(batch + 255) / 256, 256, 0, s>>>(part, per, batch, out);
  }
  bool ok = b_launch_ok(fn);
  cudaFreeAsync(part, s);
  return ok;
}

// the fused layer: rows of 2^9 .. 2^12 points, a cluster of two CTAs per row pair
template <typename C, int LOGQ>
static cudaError_t b_rxcd_t(void* st, void* lam, int batch, int n, int bit, const double* th, const double* beta,
                            double2* partCd, double2* partRx, double* gCd, double* gRx, cudaStream_t s) {
  using G = BPair<LOGQ>;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)((uint64_t)batch << (n - LOGQ)));
  cfg.blockDim = dim3(G::TPR);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = 2;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const size_t tw = (64 + (G::N >> 6)) * sizeof(double2);
  if (!lam) {
    cfg.dynamicSmemBytes = (size_t)G::RS * sizeof(C) + tw;
    auto kern = k_b_rxcd<C, LOGQ>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.dynamicSmemBytes);
    if (e != cudaSuccess) return e;
    return cudaLaunchKernelEx(&cfg, kern, (C*)st, n, bit, th, beta);
  }
  cfg.dynamicSmemBytes = (size_t)(G::RS + 2 * G::N) * sizeof(C) + tw;
  auto kern = k_b_cdrx_adj<C, LOGQ>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cfg.dynamicSmemBytes);
  if (e != cudaSuccess) return e;
  return cudaLaunchKernelEx(&cfg, kern, (C*)st, (C*)lam, n, bit, th, beta, partCd, partRx, gCd, gRx);
}

template <typename C>
static cudaError_t b_rxcd(void* st, void* lam, int batch, int n, int q, int bit, const double* th,
                          const double* beta, double2* partCd, double2* partRx, double* gCd, double* gRx,
                          cudaStream_t s) {
  switch (q) {
    case 9: return b_rxcd_t<C, 9>(st, lam, batch, n, bit, th, beta, partCd, partRx, gCd, gRx, s);
    case 10: return b_rxcd_t<C, 10>(st, lam, batch, n, bit, th, beta, partCd, partRx, gCd, gRx, s);
    case 11: return b_rxcd_t<C, 11>(st, lam, batch, n, bit, th, beta, partCd, partRx, gCd, gRx, s);
    case 12: return b_rxcd_t<C, 12>(st, lam, batch, n, bit, th, beta, partCd, partRx, gCd, gRx, s);
    default: return cudaErrorInvalidValue;
  }
}

static bool b_rxcd_args(const char* fn, int n, int q, int bit) {
  if (q < 9 || q > 12 || q >= n || bit < q || bit >= n) {
    set_error(nullptr, kErrInvalidArg,
              "%s: the mode must be the last register with 9..12 qubits and the qubit a bit above it", fn);
    return false;
  }
  return true;
}

}  // namespace cvdv

using namespace cvdv;

extern "C" {

int cvdvBatchRxCondDisp(void* states, int precision, int batch, int n, int modeQubits, int bit,
                        const double* thetas, const double* betas, void* stream) {
  const char* fn = "cvdvBatchRxCondDisp";
  if (!b_check(fn, states, precision, batch, n) || !b_rxcd_args(fn, n, modeQubits, bit)) return kErrInvalidArg;
  if (!thetas || !betas) {
    set_error(nullptr, kErrInvalidArg, "%s: null angles or displacements", fn);
    return kErrInvalidArg;
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  {
    LaunchScope _ls(nullptr, kKFft);
    e = precision == kC128 ? b_rxcd<double2>(states, nullptr, batch, n, modeQubits, bit, thetas, betas, nullptr,
                                             nullptr, nullptr, nullptr, s)
                           : b_rxcd<float2>(states, nullptr, batch, n, modeQubits, bit, thetas, betas, nullptr,
                                            nullptr, nullptr, nullptr, s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(nullptr, kErrCuda, "%s: %s", fn, cudaGetErrorString(e));
    return kErrCuda;
  }
  return kOk;
}

int cvdvBatchRxCondDispAdjoint(void* psi, void* lam, int precision, int batch, int n, int modeQubits, int bit,
                               const double* thetas, const double* betas, double* gRx, double* gCd,
                               void* stream) {
  const char* fn = "cvdvBatchRxCondDispAdjoint";
  if (!b_check(fn, psi, precision, batch, n) || !b_rxcd_args(fn, n, modeQubits, bit)) return kErrInvalidArg;
  if (!lam || !thetas || !betas || !gRx || !gCd) {
    set_error(nullptr, kErrInvalidArg, "%s: null argument", fn);
    return kErrInvalidArg;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int per = 1 << (n - modeQubits);  // rows per instance, one partial of each kind per row
  if (per == 2) {  // one cluster per instance: it writes the sums itself
    cudaError_t e;
    {
      LaunchScope _ls(nullptr, kKFft);
      e = precision == kC128 ? b_rxcd<double2>(psi, lam, batch, n, modeQubits, bit, thetas, betas, nullptr,
                                               nullptr, gCd, gRx, s)
                             : b_rxcd<float2>(psi, lam, batch, n, modeQubits, bit, thetas, betas, nullptr,
                                              nullptr, gCd, gRx, s);
    }
    if (e != cudaSuccess) {
      cudaGetLastError();
      set_error(nullptr, kErrCuda, "%s: %s", fn, cudaGetErrorString(e));
      return kErrCuda;
    }
    return kOk;
  }
  const size_t np = (size_t)batch * per;
  double2* part = nullptr;
  if (cudaMallocAsync((void**)&part, 2 * np * sizeof(double2), s) != cudaSuccess) {
    cudaGetLastError();
    set_error(nullptr, kErrAlloc, "%s: partial sums", fn);
    return kErrAlloc;
  }
  cudaError_t e;
  {
    LaunchScope _ls(nullptr, kKFft);
    e = precision == kC128 ? b_rxcd<double2>(psi, lam, batch, n, modeQubits, bit, thetas, betas, part, part + np,
                                             nullptr, nullptr, s)
                           : b_rxcd<float2>(psi, lam, batch, n, modeQubits, bit, thetas, betas, part, part + np,
                                            nullptr, nullptr, s);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    set_error(nullptr, kErrCuda, "%s: %s", fn, cudaGetErrorString(e));
    cudaFreeAsync(part, s);
    return kErrCuda;
  }
  {
    LaunchScope _ls(nullptr, kKReduce);
    k_b_sum<<<(batch + 255) / 256, 256, 0, s>>>(part, per, batch, gCd);
    k_b_sum<<<(batch + 255) / 256, 256, 0, s>>>(part + np, per, batch, gRx);
  }
  const bool ok = b_launch_ok(fn);
  cudaFreeAsync(part, s);
  return ok ? kOk : kErrCuda;
}


int cvdvBatchRx(void* states, int precision, int batch, int n, int bit, const double* thetas, double sign,
                void* stream) {
  const char* fn = "cvdvBatchRx";
  if (!b_check(fn, states, precision, batch, n)) return kErrInvalidArg;
  if (!thetas || bit < 0 || bit >= n) {
    set_error(nullptr, kErrInvalidArg, "%s: invalid bit or null angles", fn);
    return kErrInvalidArg;
  }
  const uint64_t nPairs = (uint64_t)batch << (n - 1);
  cudaStream_t s = (cudaStream_t)stream;
  {
    LaunchScope _ls(nullptr, kKPair);
    if (precision == kC128)
      k_b_rx<double2><<<b_grid(nPairs), kBatchThreads, 0, s>>>((double2*)states, nPairs, n, bit, thetas, sign);
    else
      k_b_rx<float2><<<b_grid(nPairs), kBatchThreads, 0, s>>>((float2*)states, nPairs, n, bit, thetas, sign);
  }
  return b_launch_ok(fn) ? kOk : kErrCuda;
}

int cvdvBatchCondDisp(void* states, int precision, int batch, int n, int modeQubits, int ctrlBit,
                      const double* betas, double sign, void* stream) {
  const char* fn = "cvdvBatchCondDisp";
  if (!b_check(fn, states, precision, batch, n) || !b_cd_args(fn, n, modeQubits, ctrlBit)) return kErrInvalidArg;
  if (!betas) {
    set_error(nullptr, kErrInvalidArg, "%s: null displacements", fn);
    return kErrInvalidArg;
  }
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  {
    LaunchScope _ls(nullptr, kKFft);
    e = precision == kC128 ? b_cd<double2>(states, nullptr, batch, n, modeQubits, ctrlBit, betas, sign, nullptr, s)
                           : b_cd<float2>(states, nullptr, batch, n, modeQubits, ctrlBit, betas, sign, nullptr, s);
  }
  if (e != cudaSuccess) {
    set_error(nullptr, kErrCuda, "%s: %s", fn, cudaGetErrorString(e));
    return kErrCuda;
  }
  return kOk;
}

int cvdvBatchRxAdjoint(void* psi, void* lam, int precision, int batch, int n, int bit, const double* thetas,
                       double* gOut, void* stream) {
  const char* fn = "cvdvBatchRxAdjoint";
  if (!b_check(fn, psi, precision, batch, n) || !lam || !thetas || !gOut || bit < 0 || bit >= n) {
    set_error(nullptr, kErrInvalidArg, "%s: invalid arguments", fn);
    return kErrInvalidArg;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int per = b_cta_per_inst(batch, 1ull << (n - 1));
  double2* part = nullptr;
  if (cudaMallocAsync((void**)&part, (size_t)batch * per * sizeof(double2), s) != cudaSuccess) {
    cudaGetLastError();
    set_error(nullptr, kErrAlloc, "%s: partial sums", fn);
    return kErrAlloc;
  }
  {
    LaunchScope _ls(nullptr, kKPair);
    if (precision == kC128)
      k_b_rx_adj<double2><<<batch * per, kBatchThreads, 0, s>>>((double2*)psi, (double2*)lam, n, bit, thetas, per, part);
    else
      k_b_rx_adj<float2><<<batch * per, kBatchThreads, 0, s>>>((float2*)psi, (float2*)lam, n, bit, thetas, per, part);
  }
  if (!b_launch_ok(fn)) return kErrCuda;
  return b_finish(fn, part, per, batch, gOut, s) ? kOk : kErrCuda;
}

int cvdvBatchCondDispAdjoint(void* psi, void* lam, int precision, int batch, int n, int modeQubits,
                             int ctrlBit, const double* betas, double* gOut, void* stream) {
  const char* fn = "cvdvBatchCondDispAdjoint";
  if (!b_check(fn, psi, precision, batch, n) || !b_cd_args(fn, n, modeQubits, ctrlBit)) return kErrInvalidArg;
  if (!lam || !betas || !gOut) {
    set_error(nullptr, kErrInvalidArg, "%s: null argument", fn);
    return kErrInvalidArg;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int per = 1 << (n - modeQubits);  // rows per instance, one partial each
  double2* part = nullptr;
  if (cudaMallocAsync((void**)&part, (size_t)batch * per * sizeof(double2), s) != cudaSuccess) {
    cudaGetLastError();
    set_error(nullptr, kErrAlloc, "%s: partial sums", fn);
    return kErrAlloc;
  }
  cudaError_t e;
  {
    LaunchScope _ls(nullptr, kKFft);
    e = precision == kC128 ? b_cd<double2>(psi, lam, batch, n, modeQubits, ctrlBit, betas, -1.0, part, s)
                           : b_cd<float2>(psi, lam, batch, n, modeQubits, ctrlBit, betas, -1.0, part, s);
  }
  if (e != cudaSuccess) {
    set_error(nullptr, kErrCuda, "%s: %s", fn, cudaGetErrorString(e));
    cudaFreeAsync(part, s);
    return kErrCuda;
  }
  return b_finish(fn, part, per, batch, gOut, s) ? kOk : kErrCuda;
}

int cvdvBatchOverlap(const void* states, const void* target, int precision, int batch, int n, int targetPerInstance,
                     double* out, void* stream) {
  const char* fn = "cvdvBatchOverlap";
  if (!b_check(fn, states, precision, batch, n) || !target || !out) {
    set_error(nullptr, kErrInvalidArg, "%s: invalid arguments", fn);
    return kErrInvalidArg;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int per = b_cta_per_inst(batch, 1ull << n);
  double2* part = nullptr;
  if (cudaMallocAsync((void**)&part, (size_t)batch * per * sizeof(double2), s) != cudaSuccess) {
    cudaGetLastError();
    set_error(nullptr, kErrAlloc, "%s: partial sums", fn);
    return kErrAlloc;
  }
  const uint64_t ts = targetPerInstance ? (1ull << n) : 0;
  {
    LaunchScope _ls(nullptr, kKReduce);
    if (precision == kC128)
      k_b_dot<double2><<<batch * per, kBatchThreads, 0, s>>>((const double2*)states, (const double2*)target, n, ts,
                                                             per, part);
    else
      k_b_dot<float2><<<batch * per, kBatchThreads, 0, s>>>((const float2*)states, (const float2*)target, n, ts,
                                                            per, part);
  }
  if (!b_launch_ok(fn)) return kErrCuda;
  return b_finish(fn, part, per, batch, out, s) ? kOk : kErrCuda;
}

}  // extern "C"
