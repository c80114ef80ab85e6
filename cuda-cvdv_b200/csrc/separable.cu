// Register arrays of separable states, generated on the device.
//
// The input format of cvdvInitFromSeparable is one complex128 array per register
// (src/separable.py:13-138 builds them in torch; the legacy library had kernels
// for them, src/cvdv.cu:187-295).  cvdvSeparableFill writes one such array for a
// register of 2^numQubits points x_j = (j - (N-1)/2) dx, dx = sqrt(2 pi / N):
//   kind 0  basis state j0                       (setZero: j0 = 0)
//   kind 1  uniform 1/sqrt(N)                    (setUniform)
//   kind 2  coherent |alpha>:  pi^-1/4 sqrt(dx) exp(-(x - q0)^2 / 2) exp(i (p0 x - p0 q0 / 2)),
//           q0 = sqrt2 Re alpha, p0 = sqrt2 Im alpha               (setCoherent)
//   kind 3  Fock |n> by the normalised Hermite-function recurrence  (setFock)
//           psi_0 = pi^-1/4 sqrt(dx) exp(-x^2/2), psi_k = sqrt(2/k) x psi_{k-1} - sqrt((k-1)/k) psi_{k-2}
//   kind 4  sum_n c_n |n> with the coefficients as given            (setFocks)
//   kind 5  sum_k c_k |alpha_k>, normalised to unit norm            (setCat)
//   kind 6  squeezed coherent D(alpha) S(r)|0> (no reference setter):
//           (e^{2 r} / pi)^{1/4} sqrt(dx) exp(-e^{2 r} (x - q0)^2 / 2) exp(i p0 (x - q0)),
//           the state the library's squeeze and displacement gates make from the
//           vacuum (r > 0 narrows the position distribution; the displacement
//           gate's global phase differs from setCoherent's by exp(-i Re a Im a))
// All arithmetic is FP64; a kind-5 array is normalised by a block-wide sum.
#include <cmath>

#include "../../include/cvdv.h"
#include "cvdv_internal.cuh"

namespace cvdv {

constexpr int kSepMaxParams = 256;

struct SepParams {
  int kind, q, n;  // n: parameter count
  double dx;
  double p[kSepMaxParams];
};

// (e^{2r}/pi)^{1/4} sqrt(dx) exp(-e^{2r} (x - q0)^2 / 2) exp(i (p0 x - ph p0 q0)):
// ph = 1/2 is setCoherent's phase convention, 1 the displacement gate's
__device__ __forceinline__ double2 sep_coherent(double x, double dx, double are, double aim, double e2r,
                                                double ph) {
  const double q0 = 1.41421356237309504880 * are, p0 = 1.41421356237309504880 * aim;
  const double amp = pow(e2r / CVDV_PI, 0.25) * sqrt(dx) * exp(-0.5 * e2r * (x - q0) * (x - q0));
  double s, c;
  sincos(p0 * x - ph * p0 * q0, &s, &c);
  return make_double2(amp * c, amp * s);
}

// one CTA per array: every thread walks points j = tid, tid + blockDim, ...; kind 5
// sums |psi|^2 over the CTA and rescales
__global__ void __launch_bounds__(1024) k_sep_fill(double2* __restrict__ out, const __grid_constant__ SepParams P) {
  const uint64_t N = 1ull << P.q;
  const double c0 = 0.5 * (double)(N - 1);
  __shared__ double part[32];
  double local = 0.0;
  for (uint64_t j = threadIdx.x; j < N; j += blockDim.x) {
    const double x = ((double)j - c0) * P.dx;
    double2 v = make_double2(0.0, 0.0);
    switch (P.kind) {
      case 0:
        v = make_double2(j == (uint64_t)P.p[0] ? 1.0 : 0.0, 0.0);
        break;
      case 1:
        v = make_double2(1.0 / sqrt((double)N), 0.0);
        break;
      case 2:
        v = sep_coherent(x, P.dx, P.p[0], P.p[1], 1.0, 0.5);
        break;
      case 3:
      case 4: {
        // Hermite functions psi_0 .. psi_n at x, summed with the coefficients (kind 4)
        const int nmax = P.kind == 3 ? (int)P.p[0] : P.n / 2 - 1;
        double prev = 0.0, cur = 0.7511255444649425 * sqrt(P.dx) * exp(-0.5 * x * x);  // pi^-1/4
        if (P.kind == 4) v = make_double2(P.p[0] * cur, P.p[1] * cur);
        for (int k = 1; k <= nmax; ++k) {
          const double nxt = sqrt(2.0 / k) * x * cur - sqrt((k - 1.0) / k) * prev;
          prev = cur;
          cur = nxt;
          if (P.kind == 4) {
            v.x += P.p[2 * k] * cur;
            v.y += P.p[2 * k + 1] * cur;
          }
        }
        if (P.kind == 3) v = make_double2(cur, 0.0);
        break;
      }
      case 5:
        for (int k = 0; k + 3 < P.n; k += 4) {
          const double2 a = sep_coherent(x, P.dx, P.p[k], P.p[k + 1], 1.0, 0.5);
          v.x += P.p[k + 2] * a.x - P.p[k + 3] * a.y;
          v.y += P.p[k + 2] * a.y + P.p[k + 3] * a.x;
        }
        local += v.x * v.x + v.y * v.y;
        break;
      default:  // 6: r, Re alpha, Im alpha
        v = sep_coherent(x, P.dx, P.p[1], P.p[2], exp(2.0 * P.p[0]), 1.0);
        break;
    }
    out[j] = v;
  }
  if (P.kind != 5) return;
  for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = local;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (threadIdx.x == 0) part[0] = t;
  }
  __syncthreads();
  const double inv = 1.0 / sqrt(part[0]);
  for (uint64_t j = threadIdx.x; j < N; j += blockDim.x) {
    const double2 v = out[j];  // this thread wrote it above
    out[j] = make_double2(v.x * inv, v.y * inv);
  }
}

}  // namespace cvdv

using namespace cvdv;

extern "C" int cvdvSeparableFill(void* out, int numQubits, int kind, const double* params, int nParams,
                                 void* stream) {
  const char* fn = "cvdvSeparableFill";
  if (!out || (nParams > 0 && !params)) {
    set_error(nullptr, kErrInvalidArg, "%s: null pointer argument", fn);
    return kErrInvalidArg;
  }
  if (numQubits < 1 || numQubits > 24) {
    set_error(nullptr, kErrInvalidArg, "%s: %d qubits (1..24)", fn, numQubits);
    return kErrInvalidArg;
  }
  static const int minParams[7] = {1, 0, 2, 1, 2, 4, 3};
  if (kind < 0 || kind > 6 || nParams < minParams[kind] || nParams > kSepMaxParams ||
      ((kind == 4 && (nParams & 1)) || (kind == 5 && (nParams & 3)))) {
    set_error(nullptr, kErrInvalidArg, "%s: kind %d with %d parameters (at most %d)", fn, kind, nParams,
              kSepMaxParams);
    return kErrInvalidArg;
  }
  if ((kind == 0 && (params[0] < 0 || params[0] >= (double)(1ull << numQubits))) ||
      (kind == 3 && (params[0] < 0 || params[0] > 100000))) {
    set_error(nullptr, kErrInvalidArg, "%s: index or Fock number %g out of range", fn, params[0]);
    return kErrInvalidArg;
  }
  SepParams P{};
  P.kind = kind;
  P.q = numQubits;
  P.n = nParams;
  P.dx = sqrt(2.0 * CVDV_PI / (double)(1ull << numQubits));
  for (int i = 0; i < nParams; ++i) P.p[i] = params[i];
  const cudaError_t before = cudaPeekAtLastError();
  {
    LaunchScope _ls(nullptr, kKInit);
    k_sep_fill<<<1, 1024, 0, (cudaStream_t)stream>>>((double2*)out, P);
  }
  const cudaError_t e = cudaPeekAtLastError();
  if (e != cudaSuccess && e != before) {
    cudaGetLastError();
    set_error(nullptr, kErrCuda, "%s: launch: %s", fn, cudaGetErrorString(e));
    return kErrCuda;
  }
  return kOk;
}
