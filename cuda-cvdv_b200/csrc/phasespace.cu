// Phase-space readouts: Wigner and Husimi-Q of one register, other registers
// traced out.
//
// Wigner (reference: cvdvGetWigner, src/cuda/bosonic.cu:103-132 with kernels
// src/cuda/kernels/bosonic.cuh:7-52).  The reference builds
//   G[i,k] = sum_o conj(psi_o[i+kd]) psi_o[i-kd],  kd = k - (N-1)/2,
// with one thread per (i,k) looping over all M other-register slices through
// uncoalesced gathers, O(N^2 M).  Here the same sum is read off the reduced
// density matrix rho[a][b] = sum_o psi_o[a] conj(psi_o[b]), formed as a tiled
// Hermitian GEMM (upper-triangle tiles only, FP64 accumulation, shared-memory
// operand tiles, only the entries with a + b even that the gather reads), then
// G[i,k] = rho[i-kd][i+kd] is gathered, a batched inverse
// FFT runs along k, and a transposing epilogue applies the phase correction,
// the fftshift and dx/pi.
//
// Husimi-Q (reference: husimiFromOverlap, bosonic.cu:10-61 and
// husimiFromWignerFft2, bosonic.cu:63-101) follows the same two routes and the
// same memory rule for choosing between them.

#include <cmath>
#include <cstring>

#include "../../include/cvdv.h"
#include "cvdv_internal.cuh"
#include "row_fft.cuh"

using namespace cvdv;
struct CVDVContext : public cvdv::Context {};

namespace cvdv {

template <typename C> __device__ __forceinline__ double2 tod2(C v);
template <> __device__ __forceinline__ double2 tod2<double2>(double2 v) { return v; }
template <> __device__ __forceinline__ double2 tod2<float2>(float2 v) {
  return make_double2((double)v.x, (double)v.y);
}

// psi_o[a]: slice o of register r (low bits below the register, then high bits),
// local index a -- the ordering of kernelExtractChunkPsi (bosonic.cuh:93-106).
__device__ __forceinline__ uint64_t slice_addr(uint64_t o, uint64_t a, int flw, int q) {
  uint64_t lowMask = (1ull << flw) - 1;
  return ((o & ~lowMask) << q) | (a << flw) | (o & lowMask);
}

// ----------------------------------------------------------------- rho GEMM
constexpr int kRT = 64;   // output tile
constexpr int kRK = 8;    // slices per k-step (two buffers of 2 x 8 x 65 complex: 33 KB)

// The Wigner gather reads rho[a][b] only at a + b even (a = i - kd, b = i + kd), so
// the GEMM forms the two same-parity blocks, a = 2 a' + par and b = 2 b' + par
// (par = blockIdx.z), each an N/2 x N/2 Hermitian product: a quarter of the full
// N x N x M work instead of half.  Tile indices below are in the halved index.
template <typename C>
__global__ void __launch_bounds__(256, 2) k_rho(const C* __restrict__ st, int N, int q, int flw,
                                            uint64_t M, double2* __restrict__ rho, int aFast) {
  int ta = blockIdx.y, tb = blockIdx.x;
  if (ta > tb) return;  // Hermitian: upper tiles only
  // two operand buffers: the next k-step's slices are loaded into registers while
  // the current one is multiplied, then stored to the other buffer (one barrier a step)
  __shared__ double2 sA[2][kRK][kRT + 1];
  __shared__ double2 sB[2][kRK][kRT + 1];
  const int par = blockIdx.z, Nh = N >> 1;
  const int a0 = ta * kRT, b0 = tb * kRT;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  constexpr int PER = kRK * kRT / 256;  // operand elements a thread loads per step
  double2 acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);
  double2 ra[PER], rb[PER];
  auto fetch = [&](uint64_t o0) {
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int e = threadIdx.x + 256 * u;
      const int kk = aFast ? e / kRT : e % kRK, a = aFast ? e % kRT : e / kRK;
      const uint64_t o = o0 + kk;
      double2 va = make_double2(0.0, 0.0), vb = make_double2(0.0, 0.0);
      if (o < M) {
        if (a0 + a < Nh) va = tod2<C>(st[slice_addr(o, 2 * (a0 + a) + par, flw, q)]);
        if (b0 + a < Nh) vb = tod2<C>(st[slice_addr(o, 2 * (b0 + a) + par, flw, q)]);
      }
      ra[u] = va;
      rb[u] = vb;
    }
  };
  auto put = [&](int buf) {
#pragma unroll
    for (int u = 0; u < PER; ++u) {
      const int e = threadIdx.x + 256 * u;
      const int kk = aFast ? e / kRT : e % kRK, a = aFast ? e % kRT : e / kRK;
      sA[buf][kk][a] = ra[u];
      sB[buf][kk][a] = rb[u];
    }
  };
  fetch(0);
  put(0);
  __syncthreads();
  int buf = 0;
  for (uint64_t o0 = 0; o0 < M; o0 += kRK) {
    const bool more = o0 + kRK < M;
    if (more) fetch(o0 + kRK);
#pragma unroll 4
    for (int kk = 0; kk < kRK; ++kk) {
      double2 av[4], bv[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) av[i] = sA[buf][kk][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < 4; ++j) bv[j] = sB[buf][kk][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          // a * conj(b)
          acc[i][j].x += av[i].x * bv[j].x + av[i].y * bv[j].y;
          acc[i][j].y += av[i].y * bv[j].x - av[i].x * bv[j].y;
        }
    }
    if (more) put(buf ^ 1);  // that buffer was last read before the previous barrier
    __syncthreads();
    buf ^= 1;
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      int a = a0 + ty + 16 * i, b = b0 + tx + 16 * j;
      if (a < Nh && b < Nh) rho[(size_t)(2 * a + par) * N + 2 * b + par] = acc[i][j];
    }
}

// G[i][k] = rho[i-kd][i+kd] (conj-symmetric lookup), 0 off the grid
__global__ void k_wigner_gather(const double2* __restrict__ rho, int N, double2* __restrict__ G) {
  uint64_t NN = (uint64_t)N * N;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < NN;
       e += (uint64_t)gridDim.x * blockDim.x) {
    int i = (int)(e / N), k = (int)(e % N);
    int kd = k - (N - 1) / 2;
    int ip = i + kd, im = i - kd;
    double2 v = make_double2(0.0, 0.0);
    if (ip >= 0 && ip < N && im >= 0 && im < N) {
      if (im <= ip) {
        v = rho[(size_t)im * N + ip];
      } else {
        v = rho[(size_t)ip * N + im];
        v.y = -v.y;
      }
    }
    G[e] = v;
  }
}

// W[jc][i] = Re(H[i][(jc+N/2)%N] e^{i phi_jc}) dx/pi, phi_jc = -pi (jc-N/2)(N-1)/N
// (kernelFinalizeWigner, bosonic.cuh:39-52; phase reduced exactly).
// Writes real (complexOut == nullptr) or complex (w, 0) output.
__global__ void k_wigner_finalize(const double2* __restrict__ H, int N, double dx,
                                  double* __restrict__ out, double2* __restrict__ complexOut) {
  __shared__ double tile[32][33];
  int jc0 = blockIdx.x * 32, i0 = blockIdx.y * 32;
  int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
  for (int r = ty; r < 32; r += 8) {
    int i = i0 + r, jc = jc0 + tx;
    if (i < N && jc < N) {
      int kf = (jc + N / 2) % N;
      double2 g = H[(size_t)i * N + kf];
      long long m = -(long long)(jc - N / 2) * (long long)(N - 1);
      long long M2 = 2LL * N;
      m %= M2;
      if (m < 0) m += M2;
      double s, c;
      sincospi((double)m / (double)N, &s, &c);
      tile[r][tx] = (g.x * c - g.y * s) * dx / CVDV_PI;
    }
  }
  __syncthreads();
  for (int r = ty; r < 32; r += 8) {
    int jc = jc0 + r, i = i0 + tx;
    if (i < N && jc < N) {
      double w = tile[tx][r];
      if (complexOut) complexOut[(size_t)jc * N + i] = make_double2(w, 0.0);
      else out[(size_t)jc * N + i] = w;
    }
  }
}

// ----------------------------------------------------------------- Husimi kernels
template <typename C>
__global__ void k_extract_slices(const C* __restrict__ st, int N, int q, int flw, uint64_t s0,
                                 uint64_t cnt, double2* __restrict__ X) {
  uint64_t tot = cnt * (uint64_t)N;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t s = e / N, x = e % N;
    X[e] = tod2<C>(st[slice_addr(s0 + s, x, flw, q)]);
  }
}

// G[k] = pi^{1/4} sqrt(2/dx) exp(-p^2/2), p = 2 pi k_signed / (N dx)  (bosonic.cuh:82-89)
__device__ __forceinline__ double husimi_g(int k, int N, double dx) {
  int ks = (k <= N / 2) ? k : k - N;
  double p = 2.0 * CVDV_PI * ks / ((double)N * dx);
  return pow(CVDV_PI, 0.25) * sqrt(2.0 / dx) * exp(-0.5 * p * p);
}

// A[s][m][k] = Psi_s[(m+k) & (N-1)] G[k]   (kernelFillHusimiABatched, bosonic.cuh:112-125)
__global__ void k_husimi_fill(const double2* __restrict__ Psi, int N, double dx, uint64_t cnt,
                              double2* __restrict__ A) {
  uint64_t NN = (uint64_t)N * N, tot = cnt * NN;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
       e += (uint64_t)gridDim.x * blockDim.x) {
    uint64_t s = e / NN;
    uint64_t rem = e % NN;
    int m = (int)(rem / N), k = (int)(rem % N);
    double2 p = Psi[s * N + ((m + k) & (N - 1))];
    double g = husimi_g(k, N, dx);
    A[e] = make_double2(p.x * g, p.y * g);
  }
}

// acc[m][j] += sum_s |H[s][m][j]|^2   (kernelAccumHusimiPowerChunked, bosonic.cuh:142-150)
__global__ void k_husimi_accum(const double2* __restrict__ H, uint64_t NN, uint64_t cnt,
                               double* __restrict__ acc) {
  for (uint64_t pos = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; pos < NN;
       pos += (uint64_t)gridDim.x * blockDim.x) {
    double a = 0.0;
    for (uint64_t s = 0; s < cnt; ++s) {
      double2 v = H[s * NN + pos];
      a += v.x * v.x + v.y * v.y;
    }
    acc[pos] += a;
  }
}

// Q[jc][q] = acc[(jc+N/2)%N][q] / (pi N^2)   (kernelFinalizeHusimi, bosonic.cuh:128-138)
__global__ void k_husimi_finalize(const double* __restrict__ acc, int N, double* __restrict__ out) {
  uint64_t NN = (uint64_t)N * N;
  double norm = CVDV_PI * (double)N * (double)N;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < NN;
       e += (uint64_t)gridDim.x * blockDim.x) {
    int jc = (int)(e / N), qq = (int)(e % N);
    int m = (jc + N / 2) % N;
    out[e] = acc[(size_t)m * N + qq] / norm;
  }
}

// x exp(-(wq^2 + wp^2)/4) in 2-D frequency space (kernelApplyHusimiGaussian2DFreq,
// bosonic.cuh:158-177)
__global__ void k_husimi_gauss2d(double2* __restrict__ spec, int N, double dx) {
  uint64_t NN = (uint64_t)N * N;
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < NN;
       e += (uint64_t)gridDim.x * blockDim.x) {
    int p = (int)(e / N), qq = (int)(e % N);
    int kq = (qq <= N / 2) ? qq : qq - N;
    int kp = (p <= N / 2) ? p : p - N;
    double Lq = (double)N * dx;
    double dp = CVDV_PI / ((double)N * dx);
    double Lp = (double)N * dp;
    double wq = 2.0 * CVDV_PI * (double)kq / Lq;
    double wp = 2.0 * CVDV_PI * (double)kp / Lp;
    double g = exp(-0.25 * (wq * wq + wp * wp));
    spec[e] = make_double2(spec[e].x * g, spec[e].y * g);
  }
}

// G[k] once per readout
__global__ void k_husimi_g(int N, double dx, double* __restrict__ G) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < N; k += gridDim.x * blockDim.x) G[k] = husimi_g(k, N, dx);
}

// The overlap route in one pass per output row.  Row m of the result is
//   Q[(m + N/2) mod N][q] = 1/(pi N^2) sum_s |H_s[q]|^2,  H_s = IDFT_k( Psi_s[(m + k) mod N] G[k] ),
// so a thread group of N/16 threads forms A_s[k] for its 16 points k = t + (N/16) e
// straight from the transformed slices Psi (S N values, read from L2 for every m),
// runs the inverse N-point DFT in registers (the row kernels' Stockham stages,
// one padded shared-memory row), adds |H_s|^2 to its 16 accumulators, and after
// the last slice writes its part of the output row.  The S N^2 circulant the
// reference materialises (bosonic.cu:10-61, bosonic.cuh:112-150) is never stored,
// and no atomics or separate accumulation and finalisation passes are needed.
template <int LOGN>
__global__ void __launch_bounds__((1 << (LOGN - 4)) > 256 ? (1 << (LOGN - 4)) : 256)
    k_husimi_rows(const double2* __restrict__ Psi, const double* __restrict__ G, uint64_t S,
                  const double2* __restrict__ tw, int logTwN, double* __restrict__ out) {
  constexpr int N = 1 << LOGN, E = 16, TPR = N / E;
  constexpr int ROWS = TPR >= 256 ? 1 : (256 / TPR < N ? 256 / TPR : N);  // output rows per CTA
  constexpr int RS = N + (N >> 4);
  constexpr int NHI = N >= 64 ? N / 64 : 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  double2* sm = reinterpret_cast<double2*>(smraw);
  double2* lo = sm + ROWS * RS;  // w_N^e, e < 64
  double2* hi = lo + 64;         // w_N^(64 h), h < N / 64
  const int tid = threadIdx.x, row = tid / TPR, t = tid % TPR;
  for (int i = tid; i < 64 + NHI; i += TPR * ROWS) {
    const int e = i < 64 ? i : (i - 64) << 6;
    lo[i] = e < N ? __ldg(tw + ((size_t)e << (logTwN - LOGN))) : make_double2(1.0, 0.0);
  }
  __syncthreads();
  const int m = blockIdx.x * ROWS + row;
  double2* smrow = sm + row * RS;
  double g[E], acc[E];
#pragma unroll
  for (int k = 0; k < E; ++k) {
    g[k] = __ldg(G + t + TPR * k);
    acc[k] = 0.0;
  }
  for (uint64_t s = 0; s < S; ++s) {
    const double2* ps = Psi + s * N;
    double2 v[E];
#pragma unroll
    for (int k = 0; k < E; ++k) {
      const double2 p = __ldg(ps + ((m + t + TPR * k) & (N - 1)));
      v[k] = make_double2(p.x * g[k], p.y * g[k]);
    }
    rr_stages<double2, -1, LOGN, 0, 4>(v, smrow, t, lo, hi);  // v[k] = H_s[t + TPR k]
#pragma unroll
    for (int k = 0; k < E; ++k) acc[k] += v[k].x * v[k].x + v[k].y * v[k].y;
  }
  const double norm = 1.0 / (CVDV_PI * (double)N * (double)N);
  double* o = out + (size_t)((m + N / 2) & (N - 1)) * N;
#pragma unroll
  for (int k = 0; k < E; ++k) o[t + TPR * k] = acc[k] * norm;
}

template <int LOGN>
static cudaError_t husimi_rows_t(Context* c, const double2* Psi, const double* G, uint64_t S, double* out) {
  constexpr int N = 1 << LOGN, TPR = N / 16, ROWS = TPR >= 256 ? 1 : (256 / TPR < N ? 256 / TPR : N);
  const size_t smem = (size_t)ROWS * (N + (N >> 4)) * sizeof(double2) + (64 + (N >= 64 ? N / 64 : 1)) * sizeof(double2);
  auto kern = k_husimi_rows<LOGN>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int logTwN = 0;
  while ((1 << logTwN) < c->twN) ++logTwN;
  kern<<<N / ROWS, TPR * ROWS, smem, c->stream>>>(Psi, G, S, c->twiddle, logTwN, out);
  return cudaGetLastError();
}

static cudaError_t husimi_rows(Context* c, int q, const double2* Psi, const double* G, uint64_t S, double* out) {
  switch (q) {
    case 4: return husimi_rows_t<4>(c, Psi, G, S, out);
    case 5: return husimi_rows_t<5>(c, Psi, G, S, out);
    case 6: return husimi_rows_t<6>(c, Psi, G, S, out);
    case 7: return husimi_rows_t<7>(c, Psi, G, S, out);
    case 8: return husimi_rows_t<8>(c, Psi, G, S, out);
    case 9: return husimi_rows_t<9>(c, Psi, G, S, out);
    case 10: return husimi_rows_t<10>(c, Psi, G, S, out);
    case 11: return husimi_rows_t<11>(c, Psi, G, S, out);
    case 12: return husimi_rows_t<12>(c, Psi, G, S, out);
    case 13: return husimi_rows_t<13>(c, Psi, G, S, out);
    default: return cudaErrorInvalidValue;
  }
}

// max(Re / N^2, 0)   (kernelComplexToRealNormalizedClamp, bosonic.cuh:180-186)
__global__ void k_real_clamp(const double2* __restrict__ in, uint64_t NN, double norm,
                             double* __restrict__ out) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < NN;
       e += (uint64_t)gridDim.x * blockDim.x) {
    double v = in[e].x / norm;
    out[e] = v < 0.0 ? 0.0 : v;
  }
}

static int gblocks(uint64_t work) {
  uint64_t b = (work + 255) / 256;
  return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

// Wigner into device memory: real W (out) or complex (w, 0) (complexOut).
// Scratch layout in big: [rho | G/H | tmp] each N^2 complex.
static bool wigner_device(Context* c, int r, double* out, double2* complexOut, double2* work) {
  int q = c->q[r], flw = c->flw[r];
  int N = 1 << q;
  uint64_t M = c->size() >> q;
  size_t NN = (size_t)N * N;
  double2* rho = work;
  double2* G = work + NN;
  double2* T = work + 2 * NN;
  const int nt = ((N >> 1) + kRT - 1) / kRT;  // tiles of the halved index
  dim3 g(nt, nt, 2);
  int aFast = flw == 0 ? 1 : 0;
  if (c->precision == kC128)
    {
      LaunchScope _ls(c, kKPhaseSpace);
      k_rho<double2><<<g, 256, 0, c->stream>>>((const double2*)c->state(), N, q, flw, M, rho, aFast);
    }
  else
    {
      LaunchScope _ls(c, kKPhaseSpace);
      k_rho<float2><<<g, 256, 0, c->stream>>>((const float2*)c->state(), N, q, flw, M, rho, aFast);
    }
  {
    LaunchScope _ls(c, kKPhaseSpace);
    k_wigner_gather<<<gblocks(NN), 256, 0, c->stream>>>(rho, N, G);
  }
  if (!cuda_ok(c, cudaGetLastError(), "wigner launch")) return false;
  // inverse FFT along k (rows contiguous); the result lands in rho's buffer
  if (!launch_fft_generic(c, G, rho, T, (uint64_t)N, q, 1, -1, kC128)) {
    set_error(c, kErrUnsupported, "wigner: register too large for the row FFT");
    return false;
  }
  dim3 fg((N + 31) / 32, (N + 31) / 32);
  {
    LaunchScope _ls(c, kKPhaseSpace);
    k_wigner_finalize<<<fg, dim3(32, 8), 0, c->stream>>>(rho, N, c->dx[r], out, complexOut);
  }
  return cuda_ok(c, cudaGetLastError(), "wigner finalize");
}

}  // namespace cvdv

static Context* C(CVDVContext* p) { return static_cast<Context*>(p); }

static bool prep(Context* c, int regIdx, void* out, const char* w) {
  if (regIdx < 0 || regIdx >= c->numReg || !out) {
    set_error(c, kErrInvalidArg, "%s: invalid register index %d", w, regIdx);
    return false;
  }
  if (c->numReg == 0 || !c->initialized) {
    set_error(c, kErrNotInitialized, "%s: state not initialised", w);
    return false;
  }
  return flush(c);
}

static void husimi_wigner_route(Context* c, int r, double* husimiOut) {
  int q = c->q[r];
  int N = 1 << q;
  size_t NN = (size_t)N * N;
  double2* work = (double2*)big_scratch(c, 4 * NN * sizeof(double2));
  if (!work) return;
  double2* Wc = work + 3 * NN;
  if (!wigner_device(c, r, nullptr, Wc, work)) return;
  double2* A = work;
  double2* B = work + NN;
  // 2-D FFT: along q (contiguous rows), then along p (stride N)
  if (!launch_fft_generic(c, Wc, A, B, (uint64_t)N, q, 1, 1, kC128) ||
      !launch_fft_generic(c, A, Wc, B, 1, q, (uint64_t)N, 1, kC128)) {
    set_error(c, kErrUnsupported, "husimi: register too large");
    return;
  }
  {
    LaunchScope _ls(c, kKPhaseSpace);
    k_husimi_gauss2d<<<gblocks(NN), 256, 0, c->stream>>>(Wc, N, c->dx[r]);
  }
  if (!launch_fft_generic(c, Wc, A, B, (uint64_t)N, q, 1, -1, kC128) ||
      !launch_fft_generic(c, A, Wc, B, 1, q, (uint64_t)N, -1, kC128))
    return;
  double* dOut = (double*)B;
  {
    LaunchScope _ls(c, kKPhaseSpace);
    k_real_clamp<<<gblocks(NN), 256, 0, c->stream>>>(Wc, NN, (double)NN, dOut);
  }
  if (!cuda_ok(c, cudaMemcpyAsync(husimiOut, dOut, NN * sizeof(double), cudaMemcpyDeviceToHost,
                                  c->stream), "husimi copy"))
    return;
  stream_sync(c, "husimi sync");
}

static void husimi_overlap_route(Context* c, int r, double* husimiOut) {
  int q = c->q[r], flw = c->flw[r];
  int N = 1 << q;
  uint64_t S = c->size() >> q;
  size_t NN = (size_t)N * N;
  if (q >= 4 && q <= 13) {
    // slices, their transforms and the transform's scratch (3 S N), G (N), the output (N^2)
    char* work = (char*)big_scratch(c, (3 * S * N) * sizeof(double2) + (N + NN) * sizeof(double));
    if (!work) return;
    double2* X = (double2*)work;
    double2* Psi = X + S * N;
    double2* T = Psi + S * N;
    double* G = (double*)(T + S * N);
    double* dOut = G + N;
    {
      LaunchScope _ls(c, kKPhaseSpace);
      if (c->precision == kC128)
        k_extract_slices<double2><<<gblocks(S * N), 256, 0, c->stream>>>((const double2*)c->state(), N, q, flw, 0, S, X);
      else
        k_extract_slices<float2><<<gblocks(S * N), 256, 0, c->stream>>>((const float2*)c->state(), N, q, flw, 0, S, X);
    }
    if (!launch_fft_generic(c, X, Psi, T, S, q, 1, 1, kC128)) {
      set_error(c, kErrUnsupported, "husimi: register too large");
      return;
    }
    {
      LaunchScope _ls(c, kKPhaseSpace);
      k_husimi_g<<<gblocks(N), 256, 0, c->stream>>>(N, c->dx[r], G);
    }
    cudaError_t e;
    {
      LaunchScope _ls(c, kKPhaseSpace);
      e = husimi_rows(c, q, Psi, G, S, dOut);
    }
    if (!cuda_ok(c, e, "husimi launch")) return;
    if (!cuda_ok(c, cudaMemcpyAsync(husimiOut, dOut, NN * sizeof(double), cudaMemcpyDeviceToHost, c->stream),
                 "husimi copy"))
      return;
    stream_sync(c, "husimi sync");
    return;
  }
  // longer registers: the circulant in chunks of slices, transformed by the pass kernel
  // slices per chunk: the circulant A of a chunk holds cs * N^2 complex values
  uint64_t cs = ((uint64_t)1 << 25) / NN;
  if (cs < 1) cs = 1;
  if (cs > S) cs = S;
  size_t need = (size_t)(2 * S * N + 3 * cs * NN) * sizeof(double2) + NN * sizeof(double);
  char* work = (char*)big_scratch(c, need);
  if (!work) return;
  double2* X = (double2*)work;
  double2* Psi = X + S * N;
  double2* A = Psi + S * N;
  double2* H = A + cs * NN;
  double2* T = H + cs * NN;  // temporary of a two-pass row transform
  double* acc = (double*)(T + cs * NN);
  if (c->precision == kC128)
    {
      LaunchScope _ls(c, kKPhaseSpace);
      k_extract_slices<double2><<<gblocks(S * N), 256, 0, c->stream>>>((const double2*)c->state(), N, q, flw, 0, S, X);
    }
  else
    {
      LaunchScope _ls(c, kKPhaseSpace);
      k_extract_slices<float2><<<gblocks(S * N), 256, 0, c->stream>>>((const float2*)c->state(), N, q, flw, 0, S, X);
    }
  if (!launch_fft_generic(c, X, Psi, A, S, q, 1, 1, kC128)) {
    set_error(c, kErrUnsupported, "husimi: register too large");
    return;
  }
  cudaMemsetAsync(acc, 0, NN * sizeof(double), c->stream);
  for (uint64_t s0 = 0; s0 < S; s0 += cs) {
    uint64_t cnt = S - s0 < cs ? S - s0 : cs;
    {
      LaunchScope _ls(c, kKPhaseSpace);
      k_husimi_fill<<<gblocks(cnt * NN), 256, 0, c->stream>>>(Psi + s0 * N, N, c->dx[r], cnt, A);
    }
    // inverse FFT of every (s, m) row
    if (!launch_fft_generic(c, A, H, T, cnt * N, q, 1, -1, kC128)) return;
    {
      LaunchScope _ls(c, kKPhaseSpace);
      k_husimi_accum<<<gblocks(NN), 256, 0, c->stream>>>(H, NN, cnt, acc);
    }
  }
  double* dOut = (double*)A;
  {
    LaunchScope _ls(c, kKPhaseSpace);
    k_husimi_finalize<<<gblocks(NN), 256, 0, c->stream>>>(acc, N, dOut);
  }
  if (!cuda_ok(c, cudaGetLastError(), "husimi launch")) return;
  if (!cuda_ok(c, cudaMemcpyAsync(husimiOut, dOut, NN * sizeof(double), cudaMemcpyDeviceToHost,
                                  c->stream), "husimi copy"))
    return;
  stream_sync(c, "husimi sync");
}

// The reference chooses the Wigner route when the overlap route's buffers would
// exceed 80% of free device memory (bosonic.cu:14-25); the same rule applies.
static bool overlap_fits(Context* c, int r) {
  size_t N = (size_t)1 << c->q[r];
  size_t S = (size_t)(c->size() >> c->q[r]);
  size_t fixedBytes = N * 16 + 2 * N * N * 8;
  double dyn = (double)S * N * 16 + (double)S * N * N * 16;
  size_t freeB = 0, totalB = 0;
  if (cudaMemGetInfo(&freeB, &totalB) != cudaSuccess) return false;
  return (double)fixedBytes + dyn <= 0.8 * (double)freeB;
}

extern "C" {

void cvdvGetWigner(CVDVContext* ctx, int regIdx, double* wignerOut) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!prep(c, regIdx, wignerOut, "cvdvGetWigner")) return;
  int N = 1 << c->q[regIdx];
  size_t NN = (size_t)N * N;
  double2* work = (double2*)big_scratch(c, 3 * NN * sizeof(double2) + NN * sizeof(double));
  if (!work) return;
  double* dOut = (double*)(work + 3 * NN);
  if (!wigner_device(c, regIdx, dOut, nullptr, work)) return;
  if (!cuda_ok(c, cudaMemcpyAsync(wignerOut, dOut, NN * sizeof(double), cudaMemcpyDeviceToHost,
                                  c->stream), "wigner copy"))
    return;
  stream_sync(c, "wigner sync");
}

void cvdvGetHusimiQ(CVDVContext* ctx, int regIdx, double* husimiOut) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!prep(c, regIdx, husimiOut, "cvdvGetHusimiQ")) return;
  if (overlap_fits(c, regIdx)) husimi_overlap_route(c, regIdx, husimiOut);
  else husimi_wigner_route(c, regIdx, husimiOut);
}

void cvdvGetHusimiQOverlap(CVDVContext* ctx, int regIdx, double* husimiOut) {
  cvdvGetHusimiQ(ctx, regIdx, husimiOut);  // bosonic.cu:140-144 has the same fallback
}

void cvdvGetHusimiQWigner(CVDVContext* ctx, int regIdx, double* husimiOut) {
  if (!ctx) return;
  Context* c = C(ctx);
  if (!prep(c, regIdx, husimiOut, "cvdvGetHusimiQWigner")) return;
  husimi_wigner_route(c, regIdx, husimiOut);
}

}  // extern "C"
