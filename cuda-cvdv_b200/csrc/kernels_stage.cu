// Batched independent circuits: one persistent launch per gate stage.
//
// Every instance of the batch has its own layout [1-qubit registers..., mode]
// and gate list; at stage s each instance applies its s-th gate.  The host turns
// those gates into tasks (CvdvBatchTask): a row program -- the mode's transforms,
// parity and diagonal phases, on a group of rows -- or a 2x2 gate on a qubit bit
// over a range of pairs.  A grid of persistent 512-thread CTAs walks the stage's
// task list; the task decides the code path, so instances with different gates
// and mode sizes share one launch.
//
// Row programs keep each row in registers (16 amplitudes per thread for modes
// up to 2^12 points, 32 for 2^13 and 2^14) and use the Stockham stages of the
// row kernels; diagonal phases are evaluated per element from a small phase
// polynomial (FP64 argument with exact transform twiddles, reduced mod 2 pi,
// then sin/cos in the state's precision), so nothing has to be tabulated per
// instance.

#include <cmath>

#include "../../include/cvdv.h"
#include "cvdv_internal.cuh"
#include "row_fft.cuh"

namespace cvdv {

constexpr int kStageThreads = 512;

// Amplitudes per thread of a row task, 2^LOGE with LOGE = 3, 4 or 5 (radix-8, 16 or
// 32 Stockham stages; 512 2^LOGE / N rows per CTA), chosen per task (the
// autotuner's knob).  A row must fit the 512 threads (N / 2^LOGE <= 512) and the
// CTA's rows the shared memory (complex128: 2^LOGE <= 16).  The default is 32 for
// complex64 rows of 2^13 and 2^14 points, else 16.
template <typename C> constexpr int stage_max_log() { return sizeof(C) == sizeof(float2) ? 14 : 13; }
template <typename C> constexpr int stage_max_loge() { return sizeof(C) == sizeof(float2) ? 5 : 4; }
template <typename C, int LOGN, int LOGE>
constexpr bool stage_shape_ok() {
  return LOGE >= 3 && LOGE <= stage_max_loge<C>() && LOGN >= LOGE && (LOGN - LOGE) <= 9;
}

// shared memory of the largest row group (512 threads x E amplitudes, padded) + twiddles;
// the radix-8 shape's rows (512 x 8 amplitudes, padded by 1/8) are smaller
template <typename C>
constexpr size_t stage_smem() {
  constexpr int L = stage_max_log<C>();
  constexpr int E = 1 << stage_max_loge<C>();
  return (size_t)(kStageThreads * E + kStageThreads * E / 16) * sizeof(C) + (64 + (1 << (L - 6))) * sizeof(double2);
}

template <typename C> struct StageReal;
template <> struct StageReal<double2> { using t = double; };
template <> struct StageReal<float2> { using t = float; };

template <typename C>
__device__ __forceinline__ C phase_factor(const CvdvBatchPhase& P, int j, int N, double zs) {
  // exact multiple of theta_j = pi (N-1)(2j-N+1) / (2N): integer argument mod 4N
  const int M4 = 4 * N;
  int m = (int)(((long long)(N - 1) * (2 * j - N + 1)) % M4);
  m = (int)(((long long)m * P.tw) % M4);
  if (m < 0) m += M4;
  const double dx = sqrt(2.0 * M_PI / (double)N);
  const double x = ((double)j - 0.5 * (double)(N - 1)) * dx;
  double ph = M_PI * (double)m / (double)(2 * N) + P.g0 + zs * P.h0 +
              x * ((P.a1 + zs * P.b1) + x * ((P.a2 + zs * P.b2) + x * P.a3));
  ph -= 2.0 * M_PI * rint(ph * (0.5 / M_PI));
  using R = typename StageReal<C>::t;
  R s, c;
  if constexpr (sizeof(R) == sizeof(float)) {
    __sincosf((float)ph, &s, &c);  // |ph| <= pi after the FP64 reduction
  } else {
    sincos(ph, &s, &c);
  }
  const R sc = (R)P.scale;
  return mk(sc * c, sc * s);
}

template <typename C, int LOGN, int LOGE>
__device__ __forceinline__ void stage_row_task(C* __restrict__ st, const CvdvBatchTask& T,
                                               const CvdvBatchProgram& Pg, unsigned char* smraw) {
  constexpr int E = 1 << LOGE, N = 1 << LOGN, TPR = N >> LOGE, R = kStageThreads / TPR;
  // the Stockham exchanges pad a row once per radix: every 8 points for radix-8
  // stages (LOGE 3), every 16 or 32 otherwise
  constexpr int RS = N + (N >> (LOGE == 3 ? 3 : 4));
  C* sm = reinterpret_cast<C*>(smraw);
  double2* lo = reinterpret_cast<double2*>(sm + (size_t)RS * R);
  double2* hi = lo + 64;
  const int tid = threadIdx.x, row = tid / TPR, t = tid % TPR;
  const bool valid = row < T.count;  // rows past the task's count only take part in the syncs
  const uint64_t rowIdx = (uint64_t)T.first + (valid ? row : 0);
  C* src = st + T.stateOffset + (rowIdx << LOGN);
  C* smrow = sm + row * RS;
  for (int i = tid; i < 64 + (N >> 6); i += kStageThreads) {
    const int e = i < 64 ? i : (i - 64) << 6;
    double s, c;
    sincospi(-2.0 * (double)e / (double)N, &s, &c);
    lo[i] = make_double2(c, s);
  }
  C v[E];
#pragma unroll
  for (int k = 0; k < E; ++k) v[k] = src[t + k * TPR];
  __syncthreads();
  int d = 0;
  for (int o = 0; o < Pg.nOps; ++o) {
    const int op = Pg.op[o];
    if (op == 0) {
      const CvdvBatchPhase P = Pg.phase[d++];
      const double zs = (P.ctrlBit >= 0 && (((rowIdx << LOGN) >> P.ctrlBit) & 1ull)) ? -1.0 : 1.0;
#pragma unroll
      for (int k = 0; k < E; ++k) v[k] = cmul(v[k], phase_factor<C>(P, t + k * TPR, N, zs));
    } else if (op == 1 || op == 2) {
      // one transform body for both directions (keeps the kernel's code small):
      // the unnormalised inverse DFT is conj(DFT(conj(x)))
      if (op == 2) {
#pragma unroll
        for (int k = 0; k < E; ++k) v[k].y = -v[k].y;
      }
      rr_stages<C, 1, LOGN, 0, LOGE>(v, smrow, t, lo, hi);
      if (op == 2) {
#pragma unroll
        for (int k = 0; k < E; ++k) v[k].y = -v[k].y;
      }
    } else {  // parity: element j <- element N-1-j of the same row
#pragma unroll
      for (int k = 0; k < E; ++k) smrow[rpad<C>(N - 1 - (t + k * TPR))] = v[k];
      __syncthreads();
#pragma unroll
      for (int k = 0; k < E; ++k) v[k] = smrow[rpad<C>(t + k * TPR)];
      __syncthreads();
    }
  }
  if (valid) {
#pragma unroll
    for (int k = 0; k < E; ++k) src[t + k * TPR] = v[k];
  }
  __syncthreads();  // shared memory is reused by the CTA's next task
}

template <typename C, int LOGN>
__device__ __forceinline__ void stage_row_dispatch(C* __restrict__ st, const CvdvBatchTask& T,
                                                   const CvdvBatchProgram& Pg, unsigned char* smraw, int le) {
  // (the host checks every task's shape against stage_shape_ok before launching)
  if (le == 3) {
    if constexpr (stage_shape_ok<C, LOGN, 3>()) stage_row_task<C, LOGN, 3>(st, T, Pg, smraw);
  } else if (le == 4) {
    if constexpr (stage_shape_ok<C, LOGN, 4>()) stage_row_task<C, LOGN, 4>(st, T, Pg, smraw);
  } else {
    if constexpr (stage_shape_ok<C, LOGN, 5>()) stage_row_task<C, LOGN, 5>(st, T, Pg, smraw);
  }
}

template <typename C>
__device__ __forceinline__ void stage_pair_task(C* __restrict__ st, const CvdvBatchTask& T) {
  const C a00 = fromd<C>(make_double2(T.m[0], T.m[1])), a01 = fromd<C>(make_double2(T.m[2], T.m[3]));
  const C a10 = fromd<C>(make_double2(T.m[4], T.m[5])), a11 = fromd<C>(make_double2(T.m[6], T.m[7]));
  C* base = st + T.stateOffset;
  const uint64_t low = (1ull << T.bit) - 1;
  for (int p = threadIdx.x; p < T.count; p += kStageThreads) {
    const uint64_t lp = (uint64_t)T.first + p;
    const uint64_t i0 = ((lp & ~low) << 1) | (lp & low);
    const uint64_t i1 = i0 | (1ull << T.bit);
    const C x = base[i0], y = base[i1];
    base[i0] = cadd(cmul(a00, x), cmul(a01, y));
    base[i1] = cadd(cmul(a10, x), cmul(a11, y));
  }
}

template <typename C>
__global__ void __launch_bounds__(kStageThreads, 1)
    k_batch_stage(C* __restrict__ st, const CvdvBatchTask* __restrict__ tasks, int nTasks,
                  const CvdvBatchProgram* __restrict__ progs) {
  extern __shared__ __align__(16) unsigned char smraw[];
  for (int ti = blockIdx.x; ti < nTasks; ti += gridDim.x) {
    const CvdvBatchTask T = tasks[ti];
    if (T.kind == 1) {
      stage_pair_task<C>(st, T);
      continue;
    }
    const CvdvBatchProgram& Pg = progs[T.program];
    const int le = T.logE ? T.logE : ((sizeof(C) == sizeof(float2) && T.logRow >= 13) ? 5 : 4);
    switch (T.logRow) {
      case 8: stage_row_dispatch<C, 8>(st, T, Pg, smraw, le); break;
      case 9: stage_row_dispatch<C, 9>(st, T, Pg, smraw, le); break;
      case 10: stage_row_dispatch<C, 10>(st, T, Pg, smraw, le); break;
      case 11: stage_row_dispatch<C, 11>(st, T, Pg, smraw, le); break;
      case 12: stage_row_dispatch<C, 12>(st, T, Pg, smraw, le); break;
      case 13: stage_row_dispatch<C, 13>(st, T, Pg, smraw, le); break;
      default:
        if constexpr (stage_max_log<C>() >= 14) stage_row_dispatch<C, 14>(st, T, Pg, smraw, le);
        break;
    }
  }
}

}  // namespace cvdv

using namespace cvdv;

extern "C" {

void cvdvBatchStructSizes(int* sizes) {
  if (!sizes) return;
  sizes[0] = (int)sizeof(CvdvBatchPhase);
  sizes[1] = (int)sizeof(CvdvBatchProgram);
  sizes[2] = (int)sizeof(CvdvBatchTask);
}

int cvdvBatchRunStage(void* states, int precision, const CvdvBatchTask* tasks, int nTasks,
                      const CvdvBatchProgram* programs, int gridCtas, void* stream) {
  const char* fn = "cvdvBatchRunStage";
  if (!states || !tasks || nTasks < 0 || gridCtas < 1 || (precision != kC128 && precision != kC64)) {
    set_error(nullptr, kErrInvalidArg, "%s: invalid arguments", fn);
    return kErrInvalidArg;
  }
  if (nTasks == 0) return kOk;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e = cudaSuccess;
  // the shared-memory opt-in is set once per process (so later calls can be captured)
  static bool attr128 = false, attr64 = false;
  {
    LaunchScope _ls(nullptr, kKFft);
    if (precision == kC128) {
      const size_t smem = stage_smem<double2>();
      if (!attr128) {
        e = cudaFuncSetAttribute(k_batch_stage<double2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr128 = e == cudaSuccess;
      }
      if (e == cudaSuccess) {
        k_batch_stage<double2><<<gridCtas, kStageThreads, smem, s>>>((double2*)states, tasks, nTasks, programs);
        e = cudaGetLastError();
      }
    } else {
      const size_t smem = stage_smem<float2>();
      if (!attr64) {
        e = cudaFuncSetAttribute(k_batch_stage<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr64 = e == cudaSuccess;
      }
      if (e == cudaSuccess) {
        k_batch_stage<float2><<<gridCtas, kStageThreads, smem, s>>>((float2*)states, tasks, nTasks, programs);
        e = cudaGetLastError();
      }
    }
  }
  if (e != cudaSuccess) {
    set_error(nullptr, kErrCuda, "%s: %s", fn, cudaGetErrorString(e));
    return kErrCuda;
  }
  return kOk;
}

}  // extern "C"
