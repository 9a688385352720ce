// Device-side definitions shared by the execution translation units of libcfft_b200:
// the plan geometry block, complex helpers, small DFT butterflies, the shared-memory
// Stockham pass and the 8-point Walsh-Hadamard transform.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace cfft {
namespace {

constexpr int kMaxRem = 192;

struct DevGeom {
  int N[3], M[3], H[3], L[3];
  int P, d, n_ch, centered;
  int n_spec, n_orbits, n_rem, n_mask_words;
  int chan_of_parity[8];
  int off_idx[8];          // WHT index (o0 + 2 o1 + 4 o2) of each channel
  int rep_R[8][9];
  int rep_t[8][3];
  int rem_R[kMaxRem][9];
  int rem_s[kMaxRem][3];
  int nf[3];
  int radix[3][8];
  // offsets (in complex elements) into the table buffer
  int tw_off[3];           // e^{-2 pi i j / H_d}, j < H_d
  int ftw_off[3];          // e^{-2 pi i j / M_d}, j < H_d  (fold twiddles)
  int ph_off;              // e^{-2 pi i j / P}, j < P
  int pmask;               // P - 1 when P is a power of two, else -1
  int rep_tp[8][3];        // t_b,d * (P / N_d): phase numerators per unit frequency
  int rep_perm;            // 1 if every R_b^T is a signed permutation
  int rep_ps[8][3];        // (R_b^T h)_d = sign * h[src]: packed as src + 4 * (sign < 0)
  int rep_diag8;           // 1 if d = 8 and the rep ops are the 8 diagonal sign matrices
  int sign_op[8];          // sign pattern s (bit d = axis d negated) -> representative index
};

template <typename T> struct Cx;
template <> struct Cx<float> { using type = float2; };
template <> struct Cx<double> { using type = double2; };

template <typename C> __device__ __forceinline__ C mk(decltype(C::x) a, decltype(C::x) b) { C c; c.x = a; c.y = b; return c; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) { return mk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) { return mk<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }  // a * conj(b)
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk<C>(a.x, -a.y); }
template <typename C> __device__ __forceinline__ C cscale(C a, decltype(C::x) s) { return mk<C>(a.x * s, a.y * s); }
// multiply by -i (forward) or +i (inverse)
template <typename C, bool INV> __device__ __forceinline__ C mul_mi(C a) { return INV ? mk<C>(-a.y, a.x) : mk<C>(a.y, -a.x); }

// FP32 complex arithmetic on sm_100's packed two-lane instructions (FADD2 / FMUL2 /
// FFMA2 through __fadd2_rn, __fmul2_rn, __ffma2_rn): a complex add or subtract is one
// instruction instead of two.  Each lane rounds like the scalar operation it replaces
// (round to nearest), so results are unchanged except where the scalar code would
// have fused a multiply-add differently.  Off with -DCFFT_NO_PACKED_F32.
#ifndef CFFT_NO_PACKED_F32
template <> __device__ __forceinline__ float2 cadd<float2>(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 csub<float2>(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.f, -1.f), a);
}
template <> __device__ __forceinline__ float2 cmul<float2>(float2 a, float2 b) {
  return __ffma2_rn(make_float2(a.x, a.x), b, __fmul2_rn(make_float2(a.y, a.y), make_float2(-b.y, b.x)));
}
template <> __device__ __forceinline__ float2 cmulc<float2>(float2 a, float2 b) {  // a * conj(b)
  return __ffma2_rn(make_float2(a.x, a.x), make_float2(b.x, -b.y), __fmul2_rn(make_float2(a.y, a.y), make_float2(b.y, b.x)));
}
template <> __device__ __forceinline__ float2 cscale<float2>(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
#endif

// ---------------------------------------------------------------- small DFTs
template <typename C, bool INV> __device__ __forceinline__ void dft2(C* v) {
  C a = v[0], b = v[1];
  v[0] = cadd(a, b); v[1] = csub(a, b);
}
template <typename C, bool INV> __device__ __forceinline__ void dft4(C& x0, C& x1, C& x2, C& x3) {
  C t0 = cadd(x0, x2), t1 = csub(x0, x2), t2 = cadd(x1, x3), t3 = mul_mi<C, INV>(csub(x1, x3));
  x0 = cadd(t0, t2); x2 = csub(t0, t2); x1 = cadd(t1, t3); x3 = csub(t1, t3);
}
template <typename C, bool INV> __device__ __forceinline__ void dft3(C* v) {
  using T = decltype(C::x);
  const T s3 = static_cast<T>(0.86602540378443864676);  // sqrt(3)/2
  C t = cadd(v[1], v[2]);
  C u = csub(v[1], v[2]);
  C m = mk<C>(v[0].x - static_cast<T>(0.5) * t.x, v[0].y - static_cast<T>(0.5) * t.y);
  C ju = mul_mi<C, INV>(u);  // -i u (forward)
  v[0] = cadd(v[0], t);
  v[1] = mk<C>(m.x + s3 * ju.x, m.y + s3 * ju.y);
  v[2] = mk<C>(m.x - s3 * ju.x, m.y - s3 * ju.y);
}
template <typename C, bool INV> __device__ __forceinline__ void dft5(C* v) {
  using T = decltype(C::x);
  const T c1 = static_cast<T>(0.30901699437494742410), c2 = static_cast<T>(-0.80901699437494742410);
  const T s1 = static_cast<T>(0.95105651629515357212), s2 = static_cast<T>(0.58778525229247312917);
  C a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]), a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  C x0 = v[0];
  C r1 = mk<C>(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
  C r2 = mk<C>(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
  C i1 = mul_mi<C, INV>(mk<C>(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
  C i2 = mul_mi<C, INV>(mk<C>(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
  v[0] = cadd(x0, cadd(a1, a2));
  v[1] = cadd(r1, i1); v[4] = csub(r1, i1);
  v[2] = cadd(r2, i2); v[3] = csub(r2, i2);
}
template <typename C, bool INV> __device__ __forceinline__ void dft8(C* v) {
  using T = decltype(C::x);
  const T r = static_cast<T>(0.70710678118654752440);
  C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<C, INV>(e0, e1, e2, e3);
  dft4<C, INV>(o0, o1, o2, o3);
  // W8^1 = (1 -/+ i)/sqrt2, W8^2 = -/+ i, W8^3 = (-1 -/+ i)/sqrt2
  C w1 = INV ? mk<C>(r * (o1.x - o1.y), r * (o1.x + o1.y)) : mk<C>(r * (o1.x + o1.y), r * (o1.y - o1.x));
  C w2 = mul_mi<C, INV>(o2);
  C w3 = INV ? mk<C>(-r * (o3.x + o3.y), r * (o3.x - o3.y)) : mk<C>(r * (o3.y - o3.x), -r * (o3.x + o3.y));
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, w1); v[5] = csub(e1, w1);
  v[2] = cadd(e2, w2); v[6] = csub(e2, w2);
  v[3] = cadd(e3, w3); v[7] = csub(e3, w3);
}
template <typename C, bool INV, int R> __device__ __forceinline__ void dftR(C* v) {
  if constexpr (R == 2) dft2<C, INV>(v);
  else if constexpr (R == 3) dft3<C, INV>(v);
  else if constexpr (R == 4) dft4<C, INV>(v[0], v[1], v[2], v[3]);
  else if constexpr (R == 5) dft5<C, INV>(v);
  else dft8<C, INV>(v);
}

// One Stockham autosort pass (radix R, span Ns) over `nlines` lines of length n,
// out of place between two shared-memory buffers.  Element i of line l lives at
// base(l) + i * es with base(l) = (l / G) * gs + (l % G) * ls in both buffers.
// Threads loop over butterflies, so any block size works.
template <typename C, bool INV, int R>
__device__ __forceinline__ void stockham_pass(const C* __restrict__ src, C* __restrict__ dst, int n, int Ns,
                                              int nlines, int G, int gs, int ls, int es, const C* tw, int tid,
                                              int nth) {
  const int nb = n / R;
  const int total = nb * nlines;
  const int step = n / (Ns * R);
  for (int b = tid; b < total; b += nth) {
    int l, j;
    if (es == 1) { l = b / nb; j = b - l * nb; } else { j = b / nlines; l = b - j * nlines; }
    const int base = (l / G) * gs + (l % G) * ls;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src[base + (j + r * nb) * es];
    const int k = j % Ns;
#pragma unroll
    for (int r = 1; r < R; ++r) {
      const C w = tw[r * k * step];
      v[r] = INV ? cmulc(v[r], w) : cmul(v[r], w);
    }
    dftR<C, INV, R>(v);
    const int o = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; ++r) dst[base + (o + r * Ns) * es] = v[r];
  }
  __syncthreads();
}

// Runs all passes; returns the buffer (a or b) that holds the result.
template <typename C, bool INV>
__device__ C* fft_lines(C* a, C* b, int n, int nf, const int* radix, int nlines, int G, int gs, int ls, int es,
                        const C* tw, int tid, int nth) {
  int Ns = 1;
  for (int p = 0; p < nf; ++p) {
    const int R = radix[p];
    switch (R) {
      case 2: stockham_pass<C, INV, 2>(a, b, n, Ns, nlines, G, gs, ls, es, tw, tid, nth); break;
      case 3: stockham_pass<C, INV, 3>(a, b, n, Ns, nlines, G, gs, ls, es, tw, tid, nth); break;
      case 4: stockham_pass<C, INV, 4>(a, b, n, Ns, nlines, G, gs, ls, es, tw, tid, nth); break;
      case 5: stockham_pass<C, INV, 5>(a, b, n, Ns, nlines, G, gs, ls, es, tw, tid, nth); break;
      default: stockham_pass<C, INV, 8>(a, b, n, Ns, nlines, G, gs, ls, es, tw, tid, nth); break;
    }
    C* t = a; a = b; b = t;
    Ns *= R;
  }
  return a;
}

// Walsh-Hadamard transform of 8 complex values (two real transforms in the lanes).
template <typename C> __device__ __forceinline__ void wht8c(C* v) {
#pragma unroll
  for (int s = 1; s < 8; s <<= 1)
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (!(i & s)) { const C a = v[i], b = v[i + s]; v[i] = cadd(a, b); v[i + s] = csub(a, b); }
}

// Walsh-Hadamard transform of 8 values indexed e0 + 2 e1 + 4 e2 (three butterfly stages).
template <typename T> __device__ __forceinline__ void wht8(T* v) {
#pragma unroll
  for (int s = 1; s < 8; s <<= 1)
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (!(i & s)) { T a = v[i], b = v[i + s]; v[i] = a + b; v[i + s] = a - b; }
}

// 16-byte vector loads/stores of real values (4 floats or 2 doubles).
template <typename T> struct Vec16;
template <> struct Vec16<float> { using type = float4; };
template <> struct Vec16<double> { using type = double2; };
template <typename T> __device__ __forceinline__ void vload(T* out, const T* p);
template <> __device__ __forceinline__ void vload<float>(float* out, const float* p) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
}
template <> __device__ __forceinline__ void vload<double>(double* out, const double* p) {
  const double2 v = *reinterpret_cast<const double2*>(p);
  out[0] = v.x; out[1] = v.y;
}
template <typename T> __device__ __forceinline__ void vstore(T* p, const T* in);
template <> __device__ __forceinline__ void vstore<float>(float* p, const float* in) {
  *reinterpret_cast<float4*>(p) = make_float4(in[0], in[1], in[2], in[3]);
}
template <> __device__ __forceinline__ void vstore<double>(double* p, const double* in) {
  *reinterpret_cast<double2*>(p) = make_double2(in[0], in[1]);
}

// Streaming (evict-first) 16-byte loads and stores for data touched once per pass (the
// caller's f0 in the fold and the unfold), so they do not push the channel workspace out
// of L2 between the kernels that produce and consume it.  -DCFFT_NO_CACHE_HINTS turns
// them into plain accesses.
template <typename T> __device__ __forceinline__ void vload_stream(T* out, const T* p) {
#ifdef CFFT_NO_CACHE_HINTS
  vload<T>(out, p);
#else
  if constexpr (sizeof(T) == 4) {
    const float4 v = __ldcs(reinterpret_cast<const float4*>(p));
    out[0] = v.x; out[1] = v.y; out[2] = v.z; out[3] = v.w;
  } else {
    const double2 v = __ldcs(reinterpret_cast<const double2*>(p));
    out[0] = v.x; out[1] = v.y;
  }
#endif
}
template <typename T> __device__ __forceinline__ void vstore_stream(T* p, const T* in) {
#ifdef CFFT_NO_CACHE_HINTS
  vstore<T>(p, in);
#else
  if constexpr (sizeof(T) == 4) __stcs(reinterpret_cast<float4*>(p), make_float4(in[0], in[1], in[2], in[3]));
  else __stcs(reinterpret_cast<double2*>(p), make_double2(in[0], in[1]));
#endif
}

template <int M> __device__ __forceinline__ int mod_m(int v) {
  if constexpr ((M & (M - 1)) == 0) {
    return v & (M - 1);
  } else {
    const int r = v % M;
    return r < 0 ? r + M : r;
  }
}

}  // namespace
}  // namespace cfft
