// Device building blocks of the register-resident row transforms, shared by
// the row-program kernels (kernels_row.cu) and the batched circuit kernels
// (kernels_batch.cu): radix-2/4/8/16 butterflies, two-level twiddle tables in
// shared memory, and Stockham stages on E amplitudes per thread.
#pragma once

#include "cvdv_internal.cuh"

namespace cvdv {

// shared-memory position of element e of a row: one padding slot every 16
// (the radix-16 stride), which keeps the strided butterfly accesses conflict-free
template <typename C, int LOGP = 4>
__device__ __forceinline__ int rpad(int e) {
  return e + (e >> LOGP);
}

// ---------------------------------------------------------------- butterflies
template <typename C, int DIR>
__device__ __forceinline__ C rot_mi(C a) {  // * (-DIR i)
  return DIR > 0 ? mk(a.y, -a.x) : mk(-a.y, a.x);
}

template <typename C, int DIR>
__device__ __forceinline__ void bf2(C& a, C& b) {
  C t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <typename C, int DIR>
__device__ __forceinline__ void bf4(C& a0, C& a1, C& a2, C& a3) {
  C s02 = cadd(a0, a2), d02 = csub(a0, a2);
  C s13 = cadd(a1, a3), d13 = rot_mi<C, DIR>(csub(a1, a3));
  a0 = cadd(s02, s13);
  a2 = csub(s02, s13);
  a1 = cadd(d02, d13);
  a3 = csub(d02, d13);
}

// multiply by w8^K, w8 = exp(-DIR i pi / 4)
template <typename C, int DIR, int K>
__device__ __forceinline__ C w8mul(C o) {
  using T = decltype(o.x);
  const T h = (T)0.70710678118654752440;
  if constexpr (K == 0) return o;
  else if constexpr (K == 1)
    return DIR > 0 ? mk(h * (o.x + o.y), h * (o.y - o.x)) : mk(h * (o.x - o.y), h * (o.y + o.x));
  else if constexpr (K == 2) return rot_mi<C, DIR>(o);
  else
    return DIR > 0 ? mk(h * (o.y - o.x), -h * (o.x + o.y)) : mk(-h * (o.x + o.y), h * (o.x - o.y));
}

template <typename C, int DIR>
__device__ __forceinline__ void bf8(C* v) {
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  bf4<C, DIR>(e0, e1, e2, e3);
  bf4<C, DIR>(o0, o1, o2, o3);
  o1 = w8mul<C, DIR, 1>(o1);
  o2 = w8mul<C, DIR, 2>(o2);
  o3 = w8mul<C, DIR, 3>(o3);
  v[0] = cadd(e0, o0);
  v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1);
  v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2);
  v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3);
  v[7] = csub(e3, o3);
}

// radix 16 = 4 x 4: y[k1 + 4 k2] = sum_n2 w4^{n2 k2} [ w16^{n2 k1} sum_n1 w4^{n1 k1} x[4 n1 + n2] ]
template <typename C, int DIR>
__device__ __forceinline__ void bf16(C* v) {
  using T = decltype(v[0].x);
  const T c1 = (T)0.92387953251128675613, s1 = (T)0.38268343236508977173;
  const T sg = DIR > 0 ? (T)-1 : (T)1;  // sign of the imaginary part of w16
  C a[16];
#pragma unroll
  for (int n2 = 0; n2 < 4; ++n2) {
    C x0 = v[n2], x1 = v[4 + n2], x2 = v[8 + n2], x3 = v[12 + n2];
    bf4<C, DIR>(x0, x1, x2, x3);
    a[n2 * 4 + 0] = x0;
    a[n2 * 4 + 1] = x1;
    a[n2 * 4 + 2] = x2;
    a[n2 * 4 + 3] = x3;
  }
  auto mulw = [&](C x, T c, T s) { return mk(x.x * c - x.y * s, x.x * s + x.y * c); };
  a[5] = mulw(a[5], c1, sg * s1);     // w^1
  a[6] = w8mul<C, DIR, 1>(a[6]);      // w^2
  a[7] = mulw(a[7], s1, sg * c1);     // w^3
  a[9] = w8mul<C, DIR, 1>(a[9]);      // w^2
  a[10] = rot_mi<C, DIR>(a[10]);      // w^4
  a[11] = w8mul<C, DIR, 3>(a[11]);    // w^6
  a[13] = mulw(a[13], s1, sg * c1);   // w^3
  a[14] = w8mul<C, DIR, 3>(a[14]);    // w^6
  a[15] = mulw(a[15], -c1, -sg * s1); // w^9 = -w^1
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
    C y0 = a[k1], y1 = a[4 + k1], y2 = a[8 + k1], y3 = a[12 + k1];
    bf4<C, DIR>(y0, y1, y2, y3);
    v[k1 + 0] = y0;
    v[k1 + 4] = y1;
    v[k1 + 8] = y2;
    v[k1 + 12] = y3;
  }
}

// radix 32 = 2 x 16: y[k] = E[k] + w32^k O[k], y[k + 16] = E[k] - w32^k O[k] with E, O
// the 16-point DFTs of the even and odd inputs (complex64 rows, 32 amplitudes a thread)
template <typename C, int DIR>
__device__ __forceinline__ void bf32(C* v) {
  using T = decltype(v[0].x);
  // cos(k pi / 16), k = 0..8
  constexpr double cs[9] = {1.0,
                            0.98078528040323044913,
                            0.92387953251128675613,
                            0.83146961230254523708,
                            0.70710678118654752440,
                            0.55557023301960222474,
                            0.38268343236508977173,
                            0.19509032201612826785,
                            0.0};
  C e[16], o[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    e[i] = v[2 * i];
    o[i] = v[2 * i + 1];
  }
  bf16<C, DIR>(e);
  bf16<C, DIR>(o);
#pragma unroll
  for (int k = 0; k < 16; ++k) {
    // w32^k = cos(k pi / 16) - DIR i sin(k pi / 16)
    const T c = (T)(k <= 8 ? cs[k] : -cs[16 - k]);
    const T sn = (T)(k <= 8 ? cs[8 - k] : cs[k - 8]);
    const T si = DIR > 0 ? -sn : sn;
    const C t = mk(o[k].x * c - o[k].y * si, o[k].x * si + o[k].y * c);
    v[k] = cadd(e[k], t);
    v[k + 16] = csub(e[k], t);
  }
}

template <typename C, int DIR, int RHO>
__device__ __forceinline__ void bfly(C* v) {
  if constexpr (RHO == 32) bf32<C, DIR>(v);
  else if constexpr (RHO == 16) bf16<C, DIR>(v);
  else if constexpr (RHO == 8) bf8<C, DIR>(v);
  else if constexpr (RHO == 4) bf4<C, DIR>(v[0], v[1], v[2], v[3]);
  else bf2<C, DIR>(v[0], v[1]);
}

// w_L^e = hi[e >> 6] * lo[e & 63] for e < L, forward convention exp(-2 pi i e / L);
// the conjugate for DIR < 0
template <typename C, int DIR>
__device__ __forceinline__ C tw2(const double2* lo, const double2* hi, int e) {
  double2 a = hi[e >> 6], b = lo[e & 63];
  double2 w = make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
  if (DIR < 0) w.y = -w.y;
  return fromd<C>(w);
}

template <typename C, int DIR, int LOGM, int LOGRAD, int LOGNS, int LOGE>
__device__ __forceinline__ void rr_butterflies(C (&v)[1 << LOGE], int t, const double2* lo,
                                               const double2* hi) {
  constexpr int E = 1 << LOGE, RAD = 1 << LOGRAD, NB = E / RAD, TPR = 1 << (LOGM - LOGE);
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    C x[RAD];
#pragma unroll
    for (int u = 0; u < RAD; ++u) x[u] = v[b + NB * u];
    if constexpr (LOGNS > 0) {
      const int jm = (t + b * TPR) & ((1 << LOGNS) - 1);
      // w_{ns R}^{jm u} = w_M^{(jm u) << (LOGM - LOGNS - LOGRAD)}; powers as a tree
      // powers w^u as a tree (w^(u + 2^j) = w^u w^(2^j)); for radix 32 the upper
      // half is formed as it is applied, so only 17 powers are live at once
      constexpr int RT = RAD > 16 ? 16 : RAD;
      C w[RT + 1];
      w[1] = tw2<C, DIR>(lo, hi, jm << (LOGM - LOGNS - LOGRAD));
#pragma unroll
      for (int p = 1; p < RT / 2; p <<= 1) {
        w[2 * p] = cmul(w[p], w[p]);
#pragma unroll
        for (int u = 1; u < p; ++u) w[p + u] = cmul(w[p], w[u]);
      }
#pragma unroll
      for (int u = RT / 2 + 1; u < RT; ++u) w[u] = cmul(w[RT / 2], w[u - RT / 2]);
      if constexpr (RAD > 16) w[16] = cmul(w[8], w[8]);
#pragma unroll
      for (int u = 1; u < RT; ++u) x[u] = cmul(x[u], w[u]);
      if constexpr (RAD > 16) {
        x[16] = cmul(x[16], w[16]);
#pragma unroll
        for (int u = 17; u < RAD; ++u) x[u] = cmul(x[u], cmul(w[16], w[u - 16]));
      }
    }
    bfly<C, DIR, RAD>(x);
#pragma unroll
    for (int u = 0; u < RAD; ++u) v[b + NB * u] = x[u];
  }
}

// outputs of a stage to their autosorted positions, then the next stage's inputs
// (padding period 2^LOGP elements: 16 for radix-16 stages, 32 for radix-32 ones,
// so the first stage's writes at stride RAD stay free of bank conflicts)
template <typename C, int LOGM, int LOGRAD, int LOGNS, int LOGE, int LOGP = 4>
__device__ __forceinline__ void rr_exchange(C (&v)[1 << LOGE], C* smrow, int t) {
  constexpr int E = 1 << LOGE, RAD = 1 << LOGRAD, NB = E / RAD, TPR = 1 << (LOGM - LOGE);
#pragma unroll
  for (int b = 0; b < NB; ++b) {
    const int j = t + b * TPR;
    const int y = ((j >> LOGNS) << (LOGNS + LOGRAD)) + (j & ((1 << LOGNS) - 1));
#pragma unroll
    for (int u = 0; u < RAD; ++u) smrow[rpad<C, LOGP>(y + (u << LOGNS))] = v[b + NB * u];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < E; ++k) v[k] = smrow[rpad<C, LOGP>(t + k * TPR)];
  __syncthreads();
}

// The stages of one transform: radix 16 (radix 32 with 32 amplitudes a thread,
// radix 8 with 8), then the remaining radix.  The shared row holds at least
// M + M/16 elements (M + M/8 with 8 amplitudes a thread).
// AFTER: a callable run once the shared row is no longer needed (after the last
// exchange, before the last stage's butterflies)
struct NoHook {
  __device__ __forceinline__ void operator()() const {}
};
template <typename C, int DIR, int LOGM, int S, int LOGE = 4, typename H = NoHook>
__device__ __forceinline__ void rr_stages(C (&v)[1 << LOGE], C* smrow, int t, const double2* lo,
                                          const double2* hi, H after = H()) {
  constexpr int LR = LOGE >= 5 ? 5 : (LOGE == 3 ? 3 : 4);  // log2 of the full stages' radix
  constexpr int NF = LOGM / LR, REM = LOGM % LR;
  if constexpr (S < NF) {
    rr_butterflies<C, DIR, LOGM, LR, LR * S, LOGE>(v, t, lo, hi);
    if constexpr (S + 1 < NF || REM) rr_exchange<C, LOGM, LR, LR * S, LOGE, LR>(v, smrow, t);
    if constexpr ((REM > 0 && S + 1 == NF) || (REM == 0 && S + 2 == NF)) after();
    rr_stages<C, DIR, LOGM, S + 1, LOGE, H>(v, smrow, t, lo, hi, after);
  } else if constexpr (REM > 0) {
    rr_butterflies<C, DIR, LOGM, REM, LR * NF, LOGE>(v, t, lo, hi);
  }
}

}  // namespace cvdv
