// Device execution layer of libcfft_b200 (sm_100a).
//
// Forward KRFFT per batch of fields (centred fold path; the plain M2 path is the
// same pipeline with one channel and no fold):
//   k_plane_fwd   f0 (HBM) -> [fold (WHT8) + twiddle] -> x/y FFT in shared memory
//                 -> channel workspace   (one CTA per z-plane pair per field)
//   k_fft_z       z FFT of the channel workspace in place (one CTA per xz-plane)
//   k_recon       spectral-ASU gather: F(h) = sum_b e^{-2 pi i h.t_b/N} G0(R_b^T h mod M)
//                 (indices and phases computed on the fly from the representative ops)
// Backward:
//   k_inv_recon   G0 at orbit representatives from the aliasing identity
//                 G0(q) = (1/d) sum_a F(q + M.alpha_a), expanded to the whole orbit
//                 with G0(R^T q) = e^{2 pi i q.s/M} G0(q)
//   k_fft_z (inverse), k_plane_bwd (inverse x/y FFT + unfold (inverse WHT / 8) -> f0)
// The diffusion kernel K multiplies inside k_recon, and e^{-w dt/2} inside the
// plane kernels, so one SCFT contour step is six launches with no extra passes.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <cstdlib>
#include <mutex>

#include "exec.h"

namespace cfft {

namespace {

thread_local int64_t g_launches = 0;

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

// Walsh-Hadamard transform of 8 values indexed e0 + 2 e1 + 4 e2 (three butterfly stages).
template <typename T> __device__ __forceinline__ void wht8(T* v) {
#pragma unroll
  for (int s = 1; s < 8; s <<= 1)
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (!(i & s)) { T a = v[i], b = v[i + s]; v[i] = a + b; v[i + s] = a - b; }
}

// ---------------------------------------------------------------- plane kernels
// Forward: build the n_ch channel planes of z-index iz (fold or plain load), x/y FFT,
// store to the channel workspace W[b][c][iz][y][x].
template <typename T, bool USE_E>
__global__ void k_plane_fwd(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                            const T* __restrict__ f0, const T* __restrict__ E, typename Cx<T>::type* __restrict__ W) {
  using C = typename Cx<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int H1 = g->H[0], H2 = g->H[1], H3 = g->H[2];
  const int M1 = g->M[0], M2 = g->M[1];
  const int nch = g->n_ch;
  const int plane = H1 * H2;
  C* tmp = buf + nch * plane;
  C* twx = tmp + nch * plane;
  C* twy = twx + H1;
  const int iz = blockIdx.x, b = blockIdx.y;
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int i = tid; i < H1; i += nth) twx[i] = tables[g->tw_off[0] + i];
  for (int i = tid; i < H2; i += nth) twy[i] = tables[g->tw_off[1] + i];
  const size_t mvol = static_cast<size_t>(g->M[0]) * g->M[1] * g->M[2];
  const T* src = f0 + static_cast<size_t>(b) * mvol;
  const T* Eb = USE_E ? E + static_cast<size_t>(b) * mvol : nullptr;
  if (!g->centered) {
    const T* s = src + static_cast<size_t>(iz) * M1 * M2;
    for (int e = tid; e < plane; e += nth) {
      T v = s[e];
      if (USE_E) v *= Eb[static_cast<size_t>(iz) * M1 * M2 + e];
      buf[e] = mk<C>(v, static_cast<T>(0));
    }
  } else {
    const C* ftx = tables + g->ftw_off[0];
    const C* fty = tables + g->ftw_off[1];
    const C ftz = tables[g->ftw_off[2] + iz];
    for (int e = tid; e < plane; e += nth) {
      const int ix = e % H1, iy = e / H1;
      T v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const size_t idx = (static_cast<size_t>(iz + ((k >> 2) & 1) * H3) * M2 + iy + ((k >> 1) & 1) * H2) * M1 +
                           ix + (k & 1) * H1;
        v[k] = src[idx];
        if (USE_E) v[k] *= Eb[idx];
      }
      wht8(v);
      const C tx = ftx[ix], ty = fty[iy];
      for (int c = 0; c < nch; ++c) {
        const int o = g->off_idx[c];
        C w = mk<C>(static_cast<T>(1), static_cast<T>(0));
        if (o & 1) w = tx;
        if (o & 2) w = cmul(w, ty);
        if (o & 4) w = cmul(w, ftz);
        buf[c * plane + e] = mk<C>(v[o] * w.x, v[o] * w.y);
      }
    }
  }
  __syncthreads();
  // x lines: nch*H2 lines of length H1, contiguous
  C* r1 = fft_lines<C, false>(buf, tmp, H1, g->nf[0], g->radix[0], nch * H2, nch * H2, 0, H1, 1, twx, tid, nth);
  // y lines: nch*H1 lines of length H2, stride H1
  C* r2 = fft_lines<C, false>(r1, r1 == buf ? tmp : buf, H2, g->nf[1], g->radix[1], nch * H1, H1, plane, 1, H1,
                              twy, tid, nth);
  const size_t hvol = static_cast<size_t>(plane) * H3;
  for (int c = 0; c < nch; ++c) {
    C* dst = W + (static_cast<size_t>(b) * nch + c) * hvol + static_cast<size_t>(iz) * plane;
    for (int e = tid; e < plane; e += nth) dst[e] = r2[c * plane + e];
  }
}

// Backward: inverse x/y FFT of the n_ch channel planes at z-index iz, then unfold
// (inverse WHT / 8 after the conjugate twiddle, real part) or take the real part.
template <typename T, bool USE_E>
__global__ void k_plane_bwd(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                            const typename Cx<T>::type* __restrict__ W, const T* __restrict__ E, T* __restrict__ f0) {
  using C = typename Cx<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int H1 = g->H[0], H2 = g->H[1], H3 = g->H[2];
  const int M1 = g->M[0], M2 = g->M[1];
  const int nch = g->n_ch;
  const int plane = H1 * H2;
  C* tmp = buf + nch * plane;
  C* twx = tmp + nch * plane;
  C* twy = twx + H1;
  const int iz = blockIdx.x, b = blockIdx.y;
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int i = tid; i < H1; i += nth) twx[i] = tables[g->tw_off[0] + i];
  for (int i = tid; i < H2; i += nth) twy[i] = tables[g->tw_off[1] + i];
  const size_t hvol = static_cast<size_t>(plane) * H3;
  for (int c = 0; c < nch; ++c) {
    const C* s = W + (static_cast<size_t>(b) * nch + c) * hvol + static_cast<size_t>(iz) * plane;
    for (int e = tid; e < plane; e += nth) buf[c * plane + e] = s[e];
  }
  __syncthreads();
  C* r1 = fft_lines<C, true>(buf, tmp, H1, g->nf[0], g->radix[0], nch * H2, nch * H2, 0, H1, 1, twx, tid, nth);
  buf = fft_lines<C, true>(r1, r1 == buf ? tmp : buf, H2, g->nf[1], g->radix[1], nch * H1, H1, plane, 1, H1, twy,
                           tid, nth);
  const size_t mvol = static_cast<size_t>(g->M[0]) * g->M[1] * g->M[2];
  T* dst = f0 + static_cast<size_t>(b) * mvol;
  const T* Eb = USE_E ? E + static_cast<size_t>(b) * mvol : nullptr;
  if (!g->centered) {
    const T scale = static_cast<T>(1.0 / static_cast<double>(mvol));
    for (int e = tid; e < plane; e += nth) {
      const size_t idx = static_cast<size_t>(iz) * M1 * M2 + e;
      T v = buf[e].x * scale;
      if (USE_E) v *= Eb[idx];
      dst[idx] = v;
    }
  } else {
    const T scale = static_cast<T>(1.0 / (8.0 * static_cast<double>(hvol)));
    const C* ftx = tables + g->ftw_off[0];
    const C* fty = tables + g->ftw_off[1];
    const C ftz = tables[g->ftw_off[2] + iz];
    for (int e = tid; e < plane; e += nth) {
      const int ix = e % H1, iy = e / H1;
      T v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) v[k] = static_cast<T>(0);
      const C tx = ftx[ix], ty = fty[iy];
      for (int c = 0; c < nch; ++c) {
        const int o = g->off_idx[c];
        C w = mk<C>(static_cast<T>(1), static_cast<T>(0));
        if (o & 1) w = tx;
        if (o & 2) w = cmul(w, ty);
        if (o & 4) w = cmul(w, ftz);
        const C x = buf[c * plane + e];
        v[o] = x.x * w.x + x.y * w.y;  // Re(x * conj(w))
      }
      wht8(v);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const size_t idx = (static_cast<size_t>(iz + ((k >> 2) & 1) * H3) * M2 + iy + ((k >> 1) & 1) * H2) * M1 +
                           ix + (k & 1) * H1;
        T val = v[k] * scale;
        if (USE_E) val *= Eb[idx];
        dst[idx] = val;
      }
    }
  }
}

// z FFT of the channel workspace: one CTA per (y, channel, field) xz-plane.
template <typename T, bool INV>
__global__ void k_fft_z(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                        typename Cx<T>::type* __restrict__ W) {
  using C = typename Cx<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int H1 = g->H[0], H2 = g->H[1], H3 = g->H[2];
  const int iy = blockIdx.x, c = blockIdx.y, b = blockIdx.z;
  const int tid = threadIdx.x, nth = blockDim.x;
  C* tmp = buf + H1 * H3;
  C* twz = tmp + H1 * H3;
  for (int i = tid; i < H3; i += nth) twz[i] = tables[g->tw_off[2] + i];
  const size_t plane = static_cast<size_t>(H1) * H2;
  C* base = W + (static_cast<size_t>(b) * g->n_ch + c) * plane * H3 + static_cast<size_t>(iy) * H1;
  const int tot = H1 * H3;
  for (int e = tid; e < tot; e += nth) {
    const int x = e % H1, z = e / H1;
    buf[e] = base[static_cast<size_t>(z) * plane + x];
  }
  __syncthreads();
  const C* res = fft_lines<C, INV>(buf, tmp, H3, g->nf[2], g->radix[2], H1, H1, 0, 1, H1, twz, tid, nth);
  for (int e = tid; e < tot; e += nth) {
    const int x = e % H1, z = e / H1;
    base[static_cast<size_t>(z) * plane + x] = res[e];
  }
}

// ---------------------------------------------------------------- spectral gathers
__device__ __forceinline__ int fmod_pos(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }

template <typename T, bool USE_K>
__global__ void k_recon(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                        const uint32_t* __restrict__ spec_h, const T* __restrict__ K,
                        const typename Cx<T>::type* __restrict__ W, typename Cx<T>::type* __restrict__ F) {
  using C = typename Cx<T>::type;
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (s >= g->n_spec) return;
  const uint32_t hp = spec_h[s];
  const int h[3] = {static_cast<int>(hp & 1023u), static_cast<int>((hp >> 10) & 1023u), static_cast<int>((hp >> 20) & 1023u)};
  const int H1 = g->H[0], H2 = g->H[1], H3 = g->H[2];
  const size_t hvol = static_cast<size_t>(H1) * H2 * H3;
  const C* Wb = W + static_cast<size_t>(b) * g->n_ch * hvol;
  const C* ph = tables + g->ph_off;
  const int P = g->P;
  C acc = mk<C>(static_cast<T>(0), static_cast<T>(0));
  for (int r = 0; r < g->d; ++r) {
    int q[3];
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      const int v = g->rep_R[r][0 * 3 + dd] * h[0] + g->rep_R[r][1 * 3 + dd] * h[1] + g->rep_R[r][2 * 3 + dd] * h[2];
      q[dd] = fmod_pos(v, g->M[dd]);
    }
    size_t idx;
    if (g->centered) {
      const int c = g->chan_of_parity[(q[0] & 1) + 2 * (q[1] & 1) + 4 * (q[2] & 1)];
      if (c < 0) continue;
      idx = static_cast<size_t>(c) * hvol + (static_cast<size_t>(q[2] >> 1) * H2 + (q[1] >> 1)) * H1 + (q[0] >> 1);
    } else {
      idx = (static_cast<size_t>(q[2]) * H2 + q[1]) * H1 + q[0];
    }
    int jj = h[0] * g->rep_tp[r][0] + h[1] * g->rep_tp[r][1] + h[2] * g->rep_tp[r][2];
    jj = g->pmask >= 0 ? (jj & g->pmask) : ((jj % P) + P) % P;
    acc = cadd(acc, cmul(Wb[idx], ph[jj]));
  }
  if (USE_K) acc = cscale(acc, K[s]);
  F[static_cast<size_t>(b) * g->n_spec + s] = acc;
}

template <typename T>
__global__ void k_inv_recon(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                            const int32_t* __restrict__ orbit_rep, const int32_t* __restrict__ inv_spec,
                            const int32_t* __restrict__ inv_phase, const uint32_t* __restrict__ img_mask,
                            const typename Cx<T>::type* __restrict__ F, typename Cx<T>::type* __restrict__ W) {
  using C = typename Cx<T>::type;
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (o >= g->n_orbits) return;
  const int d = g->d;
  const C* Fb = F + static_cast<size_t>(b) * g->n_spec;
  const C* ph = tables + g->ph_off;
  C acc = mk<C>(static_cast<T>(0), static_cast<T>(0));
  for (int a = 0; a < d; ++a) {
    const int s = inv_spec[static_cast<size_t>(o) * d + a];
    if (s == 0) continue;
    C f = Fb[(s > 0 ? s : -s) - 1];
    if (s < 0) f = cconj(f);
    acc = cadd(acc, cmulc(f, ph[inv_phase[static_cast<size_t>(o) * d + a]]));  // f * e^{+2 pi i j/P}
  }
  acc = cscale(acc, static_cast<T>(1.0 / static_cast<double>(d)));
  const int m = orbit_rep[o];
  const int M1 = g->M[0], M2 = g->M[1], M3 = g->M[2];
  const int q[3] = {m % M1, (m / M1) % M2, m / (M1 * M2)};
  const int H1 = g->H[0], H2 = g->H[1], H3 = g->H[2];
  const size_t hvol = static_cast<size_t>(H1) * H2 * H3;
  C* Wb = W + static_cast<size_t>(b) * g->n_ch * hvol;
  const int P = g->P;
  const int nw = g->n_mask_words;
  for (int i = 0; i < g->n_rem; ++i) {
    if (!((img_mask[static_cast<size_t>(o) * nw + (i >> 5)] >> (i & 31)) & 1u)) continue;
    int qq[3];
    long long j = 0;
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      const int v = g->rem_R[i][0 * 3 + dd] * q[0] + g->rem_R[i][1 * 3 + dd] * q[1] + g->rem_R[i][2 * 3 + dd] * q[2];
      qq[dd] = fmod_pos(v, g->M[dd]);
      j += static_cast<long long>(q[dd]) * g->rem_s[i][dd] * (P / g->M[dd]);
    }
    const int jj = static_cast<int>(((j % P) + P) % P);
    const C val = cmulc(acc, ph[jj]);  // acc * e^{+2 pi i q.s/M}
    size_t idx;
    if (g->centered) {
      const int c = g->chan_of_parity[(qq[0] & 1) + 2 * (qq[1] & 1) + 4 * (qq[2] & 1)];
      if (c < 0) continue;  // even-translation images stay in alive classes; guard anyway
      idx = static_cast<size_t>(c) * hvol + (static_cast<size_t>(qq[2] >> 1) * H2 + (qq[1] >> 1)) * H1 + (qq[0] >> 1);
    } else {
      idx = (static_cast<size_t>(qq[2]) * H2 + qq[1]) * H1 + qq[0];
    }
    Wb[idx] = val;
  }
  (void)M3;
}

// ---------------------------------------------------------------- compile-time sized path
// For cubic channel grids with H in {4, 6, 8, 12, 16, 24, 32, 48} every line FFT is a
// fully unrolled mixed-radix Stockham in registers (one thread per line), with its
// twiddles in constant memory, so no runtime division or shared-memory pass remains
// inside an FFT.  Shared-memory rows are padded to an odd stride (H + 1 complex) so
// row and column accesses of a warp are bank-conflict free.

constexpr int kTwOff4 = 0, kTwOff6 = 4, kTwOff8 = 10, kTwOff12 = 18, kTwOff16 = 30, kTwOff24 = 46,
              kTwOff32 = 70, kTwOff48 = 102, kTwTotal = 150;
__constant__ float2 c_tw_f[kTwTotal];
__constant__ double2 c_tw_d[kTwTotal];

template <int N> constexpr int tw_offset() {
  return N == 4 ? kTwOff4 : N == 6 ? kTwOff6 : N == 8 ? kTwOff8 : N == 12 ? kTwOff12 : N == 16 ? kTwOff16
       : N == 24 ? kTwOff24 : N == 32 ? kTwOff32 : kTwOff48;
}
constexpr int pick_radix(int rem) { return rem % 8 == 0 ? 8 : rem % 4 == 0 ? 4 : rem % 2 == 0 ? 2 : rem % 3 == 0 ? 3 : 5; }

template <typename C> __device__ __forceinline__ C ctw(int i);
template <> __device__ __forceinline__ float2 ctw<float2>(int i) { return c_tw_f[i]; }
template <> __device__ __forceinline__ double2 ctw<double2>(int i) { return c_tw_d[i]; }

template <typename C, bool INV, int N, int Ns, int Rem>
struct RegFFT {
  static __device__ __forceinline__ void run(C* v) {
    constexpr int R = pick_radix(Rem);
    constexpr int NB = N / R;
    constexpr int STEP = N / (Ns * R);
    C w[N];
#pragma unroll
    for (int j = 0; j < NB; ++j) {
      const int k = j % Ns;
      C x[R];
#pragma unroll
      for (int r = 0; r < R; ++r) x[r] = v[j + r * NB];
      if (k != 0) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const C t = ctw<C>(tw_offset<N>() + r * k * STEP);
          x[r] = INV ? cmulc(x[r], t) : cmul(x[r], t);
        }
      }
      dftR<C, INV, R>(x);
      const int o = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) w[o + r * Ns] = x[r];
    }
#pragma unroll
    for (int i = 0; i < N; ++i) v[i] = w[i];
    RegFFT<C, INV, N, Ns * R, Rem / R>::run(v);
  }
};
template <typename C, bool INV, int N, int Ns>
struct RegFFT<C, INV, N, Ns, 1> {
  static __device__ __forceinline__ void run(C*) {}
};
template <typename C, bool INV, int N> __device__ __forceinline__ void reg_fft(C* v) { RegFFT<C, INV, N, 1, N>::run(v); }

// FFT of `count` lines of length H in padded shared memory, one thread per line.
// Line l starts at line_base(l) and has element stride es.
template <typename C, bool INV, int H>
__device__ __forceinline__ void smem_lines(C* buf, int count, int group, int gstride, int lstride, int es) {
  for (int l = threadIdx.x; l < count; l += blockDim.x) {
    C* p = buf + (l / group) * gstride + (l % group) * lstride;
    C v[H];
#pragma unroll
    for (int i = 0; i < H; ++i) v[i] = p[i * es];
    reg_fft<C, INV, H>(v);
#pragma unroll
    for (int i = 0; i < H; ++i) p[i * es] = v[i];
  }
}

// Two real fields share one complex transform on the fast path: slot s of the
// channel workspace holds g_a + i g_b for fields a = 2s and b = 2s + 1 (b may be
// absent at the end of a batch).  The forward gather separates them with
// G_a(p) = (X(p) + conj X(-p)) / 2 and G_b(p) = (X(p) - conj X(-p)) / 2i, the backward
// builds X = G_a + i G_b and the unfold reads field a from the real part and field b
// from the imaginary part.  This halves the FFT work and the workspace traffic.

// Row / column FFTs of nch padded H x H planes (row stride S = H + 1, plane stride
// H * S), one thread per line, compile-time strides.
template <typename C, bool INV, int H>
__device__ __forceinline__ void smem_rows(C* buf, int nlines) {
  constexpr int S = H + 1;
  for (int l = threadIdx.x; l < nlines; l += blockDim.x) {
    C* p = buf + l * S;
    C v[H];
#pragma unroll
    for (int i = 0; i < H; ++i) v[i] = p[i];
    reg_fft<C, INV, H>(v);
#pragma unroll
    for (int i = 0; i < H; ++i) p[i] = v[i];
  }
}
template <typename C, bool INV, int H>
__device__ __forceinline__ void smem_cols(C* buf, int nlines) {
  constexpr int S = H + 1;
  for (int l = threadIdx.x; l < nlines; l += blockDim.x) {
    C* p = buf + (l / H) * (H * S) + (l % H);
    C v[H];
#pragma unroll
    for (int i = 0; i < H; ++i) v[i] = p[i * S];
    reg_fft<C, INV, H>(v);
#pragma unroll
    for (int i = 0; i < H; ++i) p[i * S] = v[i];
  }
}

// Forward plane kernel, cubic H: fold (or plain load) of two fields + x FFT + y FFT
// -> W[slot][c][z][y][x].
template <typename T, int H, bool USE_E>
__global__ void k_plane_fwd_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                              const T* __restrict__ f0, const T* __restrict__ E, typename Cx<T>::type* __restrict__ W,
                              int nfields) {
  using C = typename Cx<T>::type;
  constexpr int S = H + 1;
  constexpr int PL = H * S;  // padded plane
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int nch = g->n_ch;
  const int iz = blockIdx.x, slot = blockIdx.y;
  const int fa = 2 * slot;
  const bool has_b = fa + 1 < nfields;
  const int tid = threadIdx.x, nth = blockDim.x;
  const size_t mvol = static_cast<size_t>(g->M[0]) * g->M[1] * g->M[2];
  const T* srca = f0 + static_cast<size_t>(fa) * mvol;
  const T* srcb = srca + mvol;
  const T* Ea = USE_E ? E + static_cast<size_t>(fa) * mvol : nullptr;
  const T* Eb = USE_E ? Ea + mvol : nullptr;
  const T zero = static_cast<T>(0);
  if (!g->centered) {
    const size_t zoff = static_cast<size_t>(iz) * H * H;
    for (int e = tid; e < H * H; e += nth) {
      T va = srca[zoff + e];
      T vb = has_b ? srcb[zoff + e] : zero;
      if (USE_E) { va *= Ea[zoff + e]; if (has_b) vb *= Eb[zoff + e]; }
      buf[(e / H) * S + (e % H)] = mk<C>(va, vb);
    }
  } else {
    constexpr int M = 2 * H;
    const C* ftx = tables + g->ftw_off[0];
    const C ftz = tables[g->ftw_off[2] + iz];
    for (int e = tid; e < H * H; e += nth) {
      const int ix = e % H, iy = e / H;
      T va[8], vb[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const size_t idx = (static_cast<size_t>(iz + ((k >> 2) & 1) * H) * M + iy + ((k >> 1) & 1) * H) * M + ix + (k & 1) * H;
        va[k] = srca[idx];
        vb[k] = has_b ? srcb[idx] : zero;
        if (USE_E) { va[k] *= Ea[idx]; if (has_b) vb[k] *= Eb[idx]; }
      }
      wht8(va);
      wht8(vb);
      const C tx = ftx[ix], ty = ftx[iy];  // cubic: the y fold twiddle table equals x's
      for (int c = 0; c < nch; ++c) {
        const int o = g->off_idx[c];
        C w = mk<C>(static_cast<T>(1), zero);
        if (o & 1) w = tx;
        if (o & 2) w = cmul(w, ty);
        if (o & 4) w = cmul(w, ftz);
        buf[c * PL + iy * S + ix] = cmul(mk<C>(va[o], vb[o]), w);
      }
    }
  }
  __syncthreads();
  smem_rows<C, false, H>(buf, nch * H);   // x lines
  __syncthreads();
  smem_cols<C, false, H>(buf, nch * H);   // y lines
  __syncthreads();
  constexpr int HV = H * H * H;
  C* dst0 = W + static_cast<size_t>(slot) * nch * HV + iz * H * H;
  for (int c = 0; c < nch; ++c)
    for (int e = tid; e < H * H; e += nth) dst0[c * HV + e] = buf[c * PL + (e / H) * S + (e % H)];
}

// Backward plane kernel, cubic H: inverse x/y FFT of W[slot][c][iz] + unfold of the two
// fields (real part -> field a, imaginary part -> field b).
template <typename T, int H, bool USE_E>
__global__ void k_plane_bwd_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                              const typename Cx<T>::type* __restrict__ W, const T* __restrict__ E, T* __restrict__ f0,
                              int nfields) {
  using C = typename Cx<T>::type;
  constexpr int S = H + 1;
  constexpr int PL = H * S;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int nch = g->n_ch;
  const int iz = blockIdx.x, slot = blockIdx.y;
  const int fa = 2 * slot;
  const bool has_b = fa + 1 < nfields;
  const int tid = threadIdx.x, nth = blockDim.x;
  const size_t hvol = static_cast<size_t>(H) * H * H;
  constexpr int HV = H * H * H;
  const C* src0 = W + static_cast<size_t>(slot) * nch * HV + iz * H * H;
  for (int c = 0; c < nch; ++c)
    for (int e = tid; e < H * H; e += nth) buf[c * PL + (e / H) * S + (e % H)] = src0[c * HV + e];
  __syncthreads();
  smem_rows<C, true, H>(buf, nch * H);
  __syncthreads();
  smem_cols<C, true, H>(buf, nch * H);
  __syncthreads();
  const size_t mvol = static_cast<size_t>(g->M[0]) * g->M[1] * g->M[2];
  T* dsta = f0 + static_cast<size_t>(fa) * mvol;
  T* dstb = dsta + mvol;
  const T* Ea = USE_E ? E + static_cast<size_t>(fa) * mvol : nullptr;
  const T* Eb = USE_E ? Ea + mvol : nullptr;
  if (!g->centered) {
    const T scale = static_cast<T>(1.0 / static_cast<double>(mvol));
    const size_t zoff = static_cast<size_t>(iz) * H * H;
    for (int e = tid; e < H * H; e += nth) {
      const C x = buf[(e / H) * S + (e % H)];
      T va = x.x * scale, vb = x.y * scale;
      if (USE_E) { va *= Ea[zoff + e]; if (has_b) vb *= Eb[zoff + e]; }
      dsta[zoff + e] = va;
      if (has_b) dstb[zoff + e] = vb;
    }
  } else {
    constexpr int M = 2 * H;
    const T scale = static_cast<T>(1.0 / (8.0 * static_cast<double>(hvol)));
    const C* ftx = tables + g->ftw_off[0];
    const C ftz = tables[g->ftw_off[2] + iz];
    for (int e = tid; e < H * H; e += nth) {
      const int ix = e % H, iy = e / H;
      T va[8], vb[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) { va[k] = static_cast<T>(0); vb[k] = static_cast<T>(0); }
      const C tx = ftx[ix], ty = ftx[iy];
      for (int c = 0; c < nch; ++c) {
        const int o = g->off_idx[c];
        C w = mk<C>(static_cast<T>(1), static_cast<T>(0));
        if (o & 1) w = tx;
        if (o & 2) w = cmul(w, ty);
        if (o & 4) w = cmul(w, ftz);
        const C y = cmulc(buf[c * PL + iy * S + ix], w);  // x * conj(w)
        va[o] = y.x;
        vb[o] = y.y;
      }
      wht8(va);
      wht8(vb);
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const size_t idx = (static_cast<size_t>(iz + ((k >> 2) & 1) * H) * M + iy + ((k >> 1) & 1) * H) * M + ix + (k & 1) * H;
        T a = va[k] * scale, bq = vb[k] * scale;
        if (USE_E) { a *= Ea[idx]; if (has_b) bq *= Eb[idx]; }
        dsta[idx] = a;
        if (has_b) dstb[idx] = bq;
      }
    }
  }
}

constexpr int kZB = 4;  // xz-planes (y values) per CTA in the z kernels

// Forward z FFT, cubic H: W[slot][c][z][y][x] (in) -> WT[slot][c][x][y][z] (z fastest,
// out, same storage: each CTA reads and writes exactly the same addresses).  Thread
// (yy, x) loads its z line straight into registers (coalesced across x); the
// transposed store goes through shared memory.
template <typename T, int H>
__global__ void k_fft_z_fwd_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* W,
                              typename Cx<T>::type* WT) {
  using C = typename Cx<T>::type;
  constexpr int S = H + 1;
  constexpr int HV = H * H * H;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);  // [yy][x][z] padded
  const int y0 = blockIdx.x * kZB, c = blockIdx.y, slot = blockIdx.z;
  const int ny = min(kZB, H - y0);
  const int tid = threadIdx.x;
  const size_t base = (static_cast<size_t>(slot) * g->n_ch + c) * HV;
  const int yy = tid / H, x = tid % H;
  if (yy < ny) {
    const C* src = W + base + (y0 + yy) * H + x;
    C v[H];
#pragma unroll
    for (int z = 0; z < H; ++z) v[z] = src[z * H * H];
    reg_fft<C, false, H>(v);
    C* row = buf + (yy * H + x) * S;
#pragma unroll
    for (int z = 0; z < H; ++z) row[z] = v[z];
  }
  __syncthreads();
  C* dst = WT + base;
  const int run = ny * H;  // contiguous (yy, z) run per x
  for (int e = tid; e < H * run; e += blockDim.x) {
    const int xx = e / run, r = e % run;
    const int y2 = r / H, z = r % H;
    dst[(xx * H + y0) * H + r] = buf[(y2 * H + xx) * S + z];
  }
}

// Backward: expand G0 from orbit representatives (ET table) + inverse z FFT, cubic H:
// G0R[slot][o] -> W[slot][c][z][y][x].
template <typename T, int H>
__global__ void k_expand_ifft_z_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                                  const int2* __restrict__ ET, const typename Cx<T>::type* __restrict__ G0R,
                                  typename Cx<T>::type* __restrict__ W) {
  using C = typename Cx<T>::type;
  constexpr int S = H + 1;
  constexpr int PL = H * S;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int y0 = blockIdx.x * kZB, c = blockIdx.y, slot = blockIdx.z;
  const int ny = min(kZB, H - y0);
  const int tid = threadIdx.x, nth = blockDim.x;
  const size_t hvol = static_cast<size_t>(H) * H * H;
  const int2* et = ET + static_cast<size_t>(c) * hvol;
  const C* rep = G0R + static_cast<size_t>(slot) * g->n_orbits;
  const C* ph = tables + g->ph_off;
  for (int e = tid; e < ny * H * H; e += nth) {
    const int x = e % H, z = (e / H) % H, yy = e / (H * H);
    const int2 t = et[(static_cast<size_t>(z) * H + y0 + yy) * H + x];
    buf[yy * PL + z * S + x] = cmulc(rep[t.x], ph[t.y]);  // G0R * e^{+2 pi i j/P}
  }
  __syncthreads();
  smem_lines<C, true, H>(buf, ny * H, H, PL, 1, S);
  __syncthreads();
  C* dst = W + (static_cast<size_t>(slot) * g->n_ch + c) * hvol;
  for (int e = tid; e < ny * H * H; e += nth) {
    const int x = e % H, z = (e / H) % H, yy = e / (H * H);
    dst[(static_cast<size_t>(z) * H + y0 + yy) * H + x] = buf[yy * PL + z * S + x];
  }
}

template <int M> __device__ __forceinline__ int mod_m(int v) {
  if constexpr ((M & (M - 1)) == 0) {
    return v & (M - 1);
  } else {
    const int r = v % M;
    return r < 0 ? r + M : r;
  }
}

// Spectral-ASU gather from the z-fastest packed workspace, cubic M (= 2H centred,
// = H plain), D representative operations; separates the two fields of the slot on
// the fly.  The geometry is staged in shared memory once per CTA.
template <typename T, int M, int D, bool USE_K, bool PERM>
__global__ void k_recon_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                          const uint32_t* __restrict__ spec_h, const T* __restrict__ K,
                          const typename Cx<T>::type* __restrict__ WT, typename Cx<T>::type* __restrict__ F,
                          int nfields) {
  using C = typename Cx<T>::type;
  __shared__ int sR[D][9];
  __shared__ int sPS[D][3];
  __shared__ int sTP[D][3];
  __shared__ int sCh[8];
  const int tid = threadIdx.x;
  if (tid < D * 9) sR[tid / 9][tid % 9] = g->rep_R[tid / 9][tid % 9];
  if (tid < D * 3) { sPS[tid / 3][tid % 3] = g->rep_ps[tid / 3][tid % 3]; sTP[tid / 3][tid % 3] = g->rep_tp[tid / 3][tid % 3]; }
  if (tid < 8) sCh[tid] = g->chan_of_parity[tid];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + tid;
  const int slot = blockIdx.y;
  if (s >= g->n_spec) return;
  const int fa = 2 * slot;
  const bool has_b = fa + 1 < nfields;
  const uint32_t hp = spec_h[s];
  const int h[3] = {static_cast<int>(hp & 1023u), static_cast<int>((hp >> 10) & 1023u), static_cast<int>((hp >> 20) & 1023u)};
  const bool cen = g->centered;
  constexpr int Hc2 = M / 2;
  const int Hc = cen ? Hc2 : M;
  const int ls = cen ? 1 : 0;  // channel coordinate = q >> ls
  const size_t hvol = static_cast<size_t>(Hc) * Hc * Hc;
  const C* Wb = WT + static_cast<size_t>(slot) * g->n_ch * hvol;
  const C* ph = tables + g->ph_off;
  const int P = g->P, pmask = g->pmask;
  const T half = static_cast<T>(0.5);
  C acca = mk<C>(static_cast<T>(0), static_cast<T>(0));
  C accb = acca;
#pragma unroll
  for (int r = 0; r < D; ++r) {
    int q[3], qn[3];
#pragma unroll
    for (int dd = 0; dd < 3; ++dd) {
      int v;
      if (PERM) {
        const int ps = sPS[r][dd];
        v = h[ps & 3];
        if (ps & 4) v = -v;
      } else {
        v = sR[r][dd] * h[0] + sR[r][3 + dd] * h[1] + sR[r][6 + dd] * h[2];
      }
      q[dd] = mod_m<M>(v);
      qn[dd] = mod_m<M>(M - q[dd]);
    }
    int c = 0;
    if (cen) {
      c = sCh[(q[0] & 1) + 2 * (q[1] & 1) + 4 * (q[2] & 1)];
      if (c < 0) continue;
    }
    const size_t base = static_cast<size_t>(c) * hvol;
    const size_t idx = base + (static_cast<size_t>(q[0] >> ls) * Hc + (q[1] >> ls)) * Hc + (q[2] >> ls);
    const size_t idn = base + (static_cast<size_t>(qn[0] >> ls) * Hc + (qn[1] >> ls)) * Hc + (qn[2] >> ls);
    const C X = Wb[idx], Xn = Wb[idn];
    const C Ga = mk<C>(half * (X.x + Xn.x), half * (X.y - Xn.y));   // (X + conj Xn) / 2
    const C Gb = mk<C>(half * (X.y + Xn.y), half * (Xn.x - X.x));   // (X - conj Xn) / 2i
    int j = h[0] * sTP[r][0] + h[1] * sTP[r][1] + h[2] * sTP[r][2];
    j = pmask >= 0 ? (j & pmask) : ((j % P) + P) % P;
    const C w = ph[j];
    acca = cadd(acca, cmul(Ga, w));
    accb = cadd(accb, cmul(Gb, w));
  }
  if (USE_K) { const T k = K[s]; acca = cscale(acca, k); accb = cscale(accb, k); }
  F[static_cast<size_t>(fa) * g->n_spec + s] = acca;
  if (has_b) F[static_cast<size_t>(fa + 1) * g->n_spec + s] = accb;
}

// Spectral-ASU gather when the 8 representative operations are the diagonal sign
// matrices diag(+-1, +-1, +-1) (any translations): the 8 taps read G0 at the sign
// images s.h of h, which all lie in one parity channel, and the Hermitian partner
// X(-q) of tap s is tap ~s.  Eight workspace loads per point and slot.
template <typename T, int M, bool USE_K>
__global__ void k_recon_diag8(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                              const uint32_t* __restrict__ spec_h, const T* __restrict__ K,
                              const typename Cx<T>::type* __restrict__ WT, typename Cx<T>::type* __restrict__ F,
                              int nfields) {
  using C = typename Cx<T>::type;
  __shared__ int sTP[8][3];  // indexed by sign pattern
  __shared__ int sCh[8];
  const int tid = threadIdx.x;
  if (tid < 24) sTP[tid / 3][tid % 3] = g->rep_tp[g->sign_op[tid / 3]][tid % 3];
  if (tid < 8) sCh[tid] = g->chan_of_parity[tid];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + tid;
  const int slot = blockIdx.y;
  if (s >= g->n_spec) return;
  const int fa = 2 * slot;
  const bool has_b = fa + 1 < nfields;
  const uint32_t hp = spec_h[s];
  const int h0 = static_cast<int>(hp & 1023u), h1 = static_cast<int>((hp >> 10) & 1023u), h2 = static_cast<int>((hp >> 20) & 1023u);
  const bool cen = g->centered;
  const int Hc = cen ? M / 2 : M;
  const int ls = cen ? 1 : 0;
  const int hvol = Hc * Hc * Hc;
  // per-axis (+h, -h) positions mod M, in channel coordinates
  const int p0 = mod_m<M>(h0), p1 = mod_m<M>(h1), p2 = mod_m<M>(h2);
  const int m0 = mod_m<M>(M - p0), m1 = mod_m<M>(M - p1), m2 = mod_m<M>(M - p2);
  int c = 0;
  if (cen) c = sCh[(p0 & 1) + 2 * (p1 & 1) + 4 * (p2 & 1)];
  if (c < 0) {  // extinct parity class: every tap reads zero
    const C z = mk<C>(static_cast<T>(0), static_cast<T>(0));
    F[static_cast<size_t>(fa) * g->n_spec + s] = z;
    if (has_b) F[static_cast<size_t>(fa + 1) * g->n_spec + s] = z;
    return;
  }
  const int X0[2] = {(p0 >> ls) * Hc * Hc, (m0 >> ls) * Hc * Hc};
  const int X1[2] = {(p1 >> ls) * Hc, (m1 >> ls) * Hc};
  const int X2[2] = {p2 >> ls, m2 >> ls};
  const C* Wb = WT + (static_cast<size_t>(slot) * g->n_ch + c) * hvol;
  C X[8];
#pragma unroll
  for (int sg = 0; sg < 8; ++sg) X[sg] = Wb[X0[sg & 1] + X1[(sg >> 1) & 1] + X2[(sg >> 2) & 1]];
  const C* ph = tables + g->ph_off;
  const int P = g->P, pmask = g->pmask;
  const T half = static_cast<T>(0.5);
  C acca = mk<C>(static_cast<T>(0), static_cast<T>(0));
  C accb = acca;
#pragma unroll
  for (int sg = 0; sg < 8; ++sg) {
    const C Xs = X[sg], Xn = X[7 - sg];
    const C Ga = mk<C>(half * (Xs.x + Xn.x), half * (Xs.y - Xn.y));
    const C Gb = mk<C>(half * (Xs.y + Xn.y), half * (Xn.x - Xs.x));
    int j = h0 * sTP[sg][0] + h1 * sTP[sg][1] + h2 * sTP[sg][2];
    j = pmask >= 0 ? (j & pmask) : ((j % P) + P) % P;
    const C w = ph[j];
    acca = cadd(acca, cmul(Ga, w));
    accb = cadd(accb, cmul(Gb, w));
  }
  if (USE_K) { const T k = K[s]; acca = cscale(acca, k); accb = cscale(accb, k); }
  F[static_cast<size_t>(fa) * g->n_spec + s] = acca;
  if (has_b) F[static_cast<size_t>(fa + 1) * g->n_spec + s] = accb;
}

// G0 at orbit representatives of the two fields of a slot, packed as G_a + i G_b.
// Each thread serves SPT consecutive slots, reusing the table entries and keeping
// several independent spectrum gathers in flight.
constexpr int kRepSlots = 4;
template <typename T>
__global__ void k_inv_recon_reps(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                                 const int32_t* __restrict__ inv_spec, const int32_t* __restrict__ inv_phase,
                                 const typename Cx<T>::type* __restrict__ F, typename Cx<T>::type* __restrict__ G0R,
                                 int nfields) {
  using C = typename Cx<T>::type;
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= g->n_orbits) return;
  const int slot0 = blockIdx.y * kRepSlots;
  const int nslots = (nfields + 1) / 2;
  const int d = g->d;
  const int ns = g->n_spec;
  const C* ph = tables + g->ph_off;
  C acc[2 * kRepSlots];
#pragma unroll
  for (int k = 0; k < 2 * kRepSlots; ++k) acc[k] = mk<C>(static_cast<T>(0), static_cast<T>(0));
  for (int a = 0; a < d; ++a) {
    const int s = inv_spec[static_cast<size_t>(o) * d + a];
    if (s == 0) continue;
    const int si = (s > 0 ? s : -s) - 1;
    const C w = ph[inv_phase[static_cast<size_t>(o) * d + a]];
#pragma unroll
    for (int k = 0; k < 2 * kRepSlots; ++k) {
      const int f = 2 * slot0 + k;
      if (f < nfields) {
        C v = F[static_cast<size_t>(f) * ns + si];
        if (s < 0) v = cconj(v);
        acc[k] = cadd(acc[k], cmulc(v, w));
      }
    }
  }
  const T inv_d = static_cast<T>(1.0 / static_cast<double>(d));
#pragma unroll
  for (int k = 0; k < kRepSlots; ++k) {
    const int slot = slot0 + k;
    if (slot < nslots) {
      const C a = acc[2 * k], b = acc[2 * k + 1];
      G0R[static_cast<size_t>(slot) * g->n_orbits + o] = mk<C>(inv_d * (a.x - b.y), inv_d * (a.y + b.x));
    }
  }
}

// G0 at orbit representatives for one field, with the field's whole spectrum staged
// in shared memory (one CTA per field and representative range): every alias gather
// is a shared-memory read.  Aliases are packed as spec+1 (bits 0-19), conjugation
// (bit 20) and phase numerator (bits 21-31); with d = 8 a thread reads its
// representative's 8 entries as two 16-byte loads.  Output layout: G0RP[slot][o][f&1].
template <typename T, int D>
__global__ void k_inv_recon_reps_smem(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                                      const uint32_t* __restrict__ inv_pk, const typename Cx<T>::type* __restrict__ F,
                                      typename Cx<T>::type* __restrict__ G0RP, int reps_per_part) {
  using C = typename Cx<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* sF = reinterpret_cast<C*>(smem_raw);
  const int ns = g->n_spec;
  const int f = blockIdx.y;
  const C* Ff = F + static_cast<size_t>(f) * ns;
  for (int i = threadIdx.x; i < ns; i += blockDim.x) sF[i] = Ff[i];
  __syncthreads();
  const C* ph = tables + g->ph_off;
  const T inv_d = static_cast<T>(1.0 / static_cast<double>(D));
  const int o0 = blockIdx.x * reps_per_part;
  const int o1 = min(g->n_orbits, o0 + reps_per_part);
  C* out = G0RP + static_cast<size_t>(f >> 1) * g->n_orbits * 2 + (f & 1);
  for (int o = o0 + threadIdx.x; o < o1; o += blockDim.x) {
    uint32_t e[D];
    if constexpr (D == 8) {
      const uint4* p4 = reinterpret_cast<const uint4*>(inv_pk + static_cast<size_t>(o) * 8);
      const uint4 u0 = p4[0], u1 = p4[1];
      e[0] = u0.x; e[1] = u0.y; e[2] = u0.z; e[3] = u0.w; e[4] = u1.x; e[5] = u1.y; e[6] = u1.z; e[7] = u1.w;
    } else {
#pragma unroll
      for (int a = 0; a < D; ++a) e[a] = inv_pk[static_cast<size_t>(o) * D + a];
    }
    C acc = mk<C>(static_cast<T>(0), static_cast<T>(0));
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const uint32_t sp = e[a] & 0xFFFFFu;
      if (sp == 0) continue;
      C v = sF[sp - 1];
      if (e[a] & (1u << 20)) v = cconj(v);
      acc = cadd(acc, cmulc(v, ph[e[a] >> 21]));
    }
    out[static_cast<size_t>(o) * 2] = cscale(acc, inv_d);
  }
}

// Backward expansion from per-field representatives (G0RP[slot][o][a|b]) + inverse z
// FFT: thread (yy, x) assembles its z line X = (G_a + i G_b) e^{+2 pi i j/P} in
// registers, transforms it and stores it coalesced across x.  No shared memory.
template <typename T, int H>
__global__ void k_expand2_ifft_z_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                                   const int2* __restrict__ ET, const typename Cx<T>::type* __restrict__ G0RF,
                                   typename Cx<T>::type* __restrict__ W, int nfields) {
  using C = typename Cx<T>::type;
  constexpr int HV = H * H * H;
  const int y0 = blockIdx.x * kZB, c = blockIdx.y, slot = blockIdx.z;
  const int ny = min(kZB, H - y0);
  const int tid = threadIdx.x;
  const int yy = tid / H, x = tid % H;
  if (yy >= ny) return;
  const int y = y0 + yy;
  const int2* et = ET + static_cast<size_t>(c) * HV + y * H + x;
  const bool has_b = 2 * slot + 1 < nfields;
  const C* rp = G0RF + static_cast<size_t>(slot) * g->n_orbits * 2;
  const C* ph = tables + g->ph_off;
  C v[H];
#pragma unroll
  for (int z = 0; z < H; ++z) {
    const int2 t = et[z * H * H];
    const C a = rp[2 * t.x];
    const C b = has_b ? rp[2 * t.x + 1] : mk<C>(static_cast<T>(0), static_cast<T>(0));
    v[z] = cmulc(mk<C>(a.x - b.y, a.y + b.x), ph[t.y]);
  }
  reg_fft<C, true, H>(v);
  C* dst = W + (static_cast<size_t>(slot) * g->n_ch + c) * HV + y * H + x;
#pragma unroll
  for (int z = 0; z < H; ++z) dst[z * H * H] = v[z];
}

// ---------------------------------------------------------------- elementwise
template <typename T>
__global__ void k_interaction(const T* __restrict__ w, T* __restrict__ E, T half_dt, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x)
    E[i] = exp(-w[i] * half_dt);
}

template <typename T>
__global__ void k_full_to_sub(const T* __restrict__ u, T* __restrict__ f0, int N1, int N2, int L1, int L2, int L3,
                              int M1, int M2, size_t mvol, size_t nvol, int B) {
  const size_t tot = mvol * B;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < tot; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t b = i / mvol, r = i % mvol;
    const size_t x = r % M1, y = (r / M1) % M2, z = r / (static_cast<size_t>(M1) * M2);
    f0[i] = u[b * nvol + (z * L3 * N2 + y * L2) * N1 + x * L1];
  }
}

template <typename T>
__global__ void k_sub_to_full(const T* __restrict__ f0, const int32_t* __restrict__ fill_map, T* __restrict__ u,
                              size_t mvol, size_t nvol, int B) {
  const size_t tot = nvol * B;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < tot; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const size_t b = i / nvol, r = i % nvol;
    u[i] = f0[b * mvol + fill_map[r]];
  }
}

// ---------------------------------------------------------------- host helpers
std::string cuda_msg(cudaError_t e, const char* what) {
  return std::string(what) + ": " + cudaGetErrorString(e);
}

#define CFFT_CUDA(call, what)                          \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) {                           \
      *err = cuda_msg(e_, what);                       \
      return Status::kCuda;                            \
    }                                                  \
  } while (0)

bool factor_radices(int n, int* nf, int* radix) {
  *nf = 0;
  const int order[5] = {8, 4, 2, 3, 5};
  for (int r : order)
    while (n > 1 && n % r == 0) {
      if (*nf >= 8) return false;
      radix[(*nf)++] = r;
      n /= r;
    }
  return n == 1;
}

// One thread per four elements, in whole warps, 64 to 512 threads per CTA.
int round_threads(long elems) {
  long t = (elems + 3) / 4;
  t = ((t + 31) / 32) * 32;
  return static_cast<int>(std::max(64L, std::min(512L, t)));
}

// Allow the largest dynamic shared memory a CTA may have (227 KB) once per kernel,
// so plans of different sizes can coexist.
constexpr int kMaxDynSmem = 227 * 1024;
template <typename T>
void set_smem_attrs() {
  cudaFuncSetAttribute(k_plane_fwd<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  cudaFuncSetAttribute(k_plane_fwd<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  cudaFuncSetAttribute(k_plane_bwd<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  cudaFuncSetAttribute(k_plane_bwd<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  cudaFuncSetAttribute(k_fft_z<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  cudaFuncSetAttribute(k_fft_z<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
}

template <typename T>
std::vector<unsigned char> make_table_bytes(const Plan& p, DevGeom* g) {
  using C = typename Cx<T>::type;
  std::vector<C> tab;
  auto push = [&](double re, double im) { C c; c.x = static_cast<T>(re); c.y = static_cast<T>(im); tab.push_back(c); };
  for (int d = 0; d < 3; ++d) {
    g->tw_off[d] = static_cast<int>(tab.size());
    const int n = p.T.H[d];
    for (int j = 0; j < n; ++j) push(std::cos(2.0 * M_PI * j / n), -std::sin(2.0 * M_PI * j / n));
  }
  for (int d = 0; d < 3; ++d) {
    g->ftw_off[d] = static_cast<int>(tab.size());
    const int m = p.T.M[d];
    for (int j = 0; j < p.T.H[d]; ++j) push(std::cos(2.0 * M_PI * j / m), -std::sin(2.0 * M_PI * j / m));
  }
  g->ph_off = static_cast<int>(tab.size());
  for (int j = 0; j < p.T.P; ++j) push(std::cos(2.0 * M_PI * j / p.T.P), -std::sin(2.0 * M_PI * j / p.T.P));
  std::vector<unsigned char> bytes(tab.size() * sizeof(C));
  std::memcpy(bytes.data(), tab.data(), bytes.size());
  return bytes;
}

// Compile-time sized kernels are instantiated for these cubic channel-grid edges.
template <typename T> constexpr bool fast_ok(int H) {
  return H == 4 || H == 6 || H == 8 || H == 12 || H == 16 || H == 24 || H == 32 || (H == 48 && sizeof(T) == 4);
}

#define CFFT_FOR_H(H, ...)                                        \
  switch (H) {                                                     \
    case 4: { constexpr int HH = 4; __VA_ARGS__; } break;                 \
    case 6: { constexpr int HH = 6; __VA_ARGS__; } break;                 \
    case 8: { constexpr int HH = 8; __VA_ARGS__; } break;                 \
    case 12: { constexpr int HH = 12; __VA_ARGS__; } break;               \
    case 16: { constexpr int HH = 16; __VA_ARGS__; } break;               \
    case 24: { constexpr int HH = 24; __VA_ARGS__; } break;               \
    case 32: { constexpr int HH = 32; __VA_ARGS__; } break;               \
    default: { constexpr int HH = 48; __VA_ARGS__; } break;               \
  }

#define CFFT_FOR_M(M, ...)                                        \
  switch (M) {                                                     \
    case 4: { constexpr int MM = 4; __VA_ARGS__; } break;                 \
    case 6: { constexpr int MM = 6; __VA_ARGS__; } break;                 \
    case 8: { constexpr int MM = 8; __VA_ARGS__; } break;                 \
    case 12: { constexpr int MM = 12; __VA_ARGS__; } break;               \
    case 16: { constexpr int MM = 16; __VA_ARGS__; } break;               \
    case 24: { constexpr int MM = 24; __VA_ARGS__; } break;               \
    case 32: { constexpr int MM = 32; __VA_ARGS__; } break;               \
    case 48: { constexpr int MM = 48; __VA_ARGS__; } break;               \
    case 64: { constexpr int MM = 64; __VA_ARGS__; } break;               \
    default: { constexpr int MM = 96; __VA_ARGS__; } break;               \
  }

template <typename T>
void set_fast_attrs() {
  for (int H : {4, 6, 8, 12, 16, 24, 32, 48}) {
    if (!fast_ok<T>(H)) continue;
    CFFT_FOR_H(H, {
      cudaFuncSetAttribute(k_plane_fwd_h<T, HH, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
      cudaFuncSetAttribute(k_plane_fwd_h<T, HH, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
      cudaFuncSetAttribute(k_plane_bwd_h<T, HH, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
      cudaFuncSetAttribute(k_plane_bwd_h<T, HH, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
      cudaFuncSetAttribute(k_fft_z_fwd_h<T, HH>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
      cudaFuncSetAttribute(k_expand_ifft_z_h<T, HH>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
    });
  }
  cudaFuncSetAttribute(k_inv_recon_reps_smem<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  cudaFuncSetAttribute(k_inv_recon_reps_smem<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  cudaFuncSetAttribute(k_inv_recon_reps_smem<T, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
  cudaFuncSetAttribute(k_inv_recon_reps_smem<T, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmem);
}

// Constant-memory twiddles e^{-2 pi i j / N} for the register FFTs (FP64 values rounded).
Status upload_const_twiddles(std::string* err) {
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  CFFT_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  std::lock_guard<std::mutex> lock(mu);
  if (dev >= 0 && dev < 64 && done[dev]) return Status::kOk;
  std::vector<float2> tf(kTwTotal);
  std::vector<double2> td(kTwTotal);
  const int sizes[8] = {4, 6, 8, 12, 16, 24, 32, 48};
  const int offs[8] = {kTwOff4, kTwOff6, kTwOff8, kTwOff12, kTwOff16, kTwOff24, kTwOff32, kTwOff48};
  for (int k = 0; k < 8; ++k)
    for (int j = 0; j < sizes[k]; ++j) {
      const double c = std::cos(2.0 * M_PI * j / sizes[k]), sn = -std::sin(2.0 * M_PI * j / sizes[k]);
      td[offs[k] + j] = make_double2(c, sn);
      tf[offs[k] + j] = make_float2(static_cast<float>(c), static_cast<float>(sn));
    }
  CFFT_CUDA(cudaMemcpyToSymbol(c_tw_f, tf.data(), sizeof(float2) * kTwTotal), "upload twiddles");
  CFFT_CUDA(cudaMemcpyToSymbol(c_tw_d, td.data(), sizeof(double2) * kTwTotal), "upload twiddles");
  set_fast_attrs<float>();
  set_fast_attrs<double>();
  CFFT_CUDA(cudaGetLastError(), "set shared-memory attributes");
  if (dev >= 0 && dev < 64) done[dev] = true;
  return Status::kOk;
}

// Stages of one forward + backward: 0 plane/fold + x/y FFT, 1 z FFT, 2 reconstruct,
// 3 inverse reconstruct (+ orbit expansion), 4 inverse z FFT, 5 inverse x/y FFT + unfold.
// `nb` fields starting at the caller's pointers; the workspace holds one chunk.
template <typename T>
void launch_stage(Plan* p, int stage, const T* f0, typename Cx<T>::type* F, const typename Cx<T>::type* Fin,
                  T* f0_out, const T* E, bool use_K, int nb, cudaStream_t st) {
  using C = typename Cx<T>::type;
  const DevGeom* g = static_cast<const DevGeom*>(p->d_geom);
  const C* tab = static_cast<const C*>(p->d_tables);
  C* W = static_cast<C*>(p->d_work_T);
  const PlanTables& T_ = p->T;
  const int H = p->fast_h;
  const size_t cs = sizeof(C);
  if (H > 0) {
    const int nch = T_.n_ch;
    const int nslots = (nb + 1) / 2;
    const int thr_plane = std::max(128, ((nch * H + 31) / 32) * 32);
    const size_t smem_plane = static_cast<size_t>(nch) * H * (H + 1) * cs;
    const int thr_z = std::max(64, ((kZB * H + 31) / 32) * 32);
    const size_t smem_z = static_cast<size_t>(kZB) * H * (H + 1) * cs;
    const dim3 gz((H + kZB - 1) / kZB, nch, nslots);
    switch (stage) {
      case 0:
        CFFT_FOR_H(H, {
          if (E) k_plane_fwd_h<T, HH, true><<<dim3(H, nslots), thr_plane, smem_plane, st>>>(g, tab, f0, E, W, nb);
          else k_plane_fwd_h<T, HH, false><<<dim3(H, nslots), thr_plane, smem_plane, st>>>(g, tab, f0, nullptr, W, nb);
        });
        break;
      case 1:
        CFFT_FOR_H(H, { k_fft_z_fwd_h<T, HH><<<gz, thr_z, smem_z, st>>>(g, W, W); });
        break;
      case 2: {
        const int ns = static_cast<int>(T_.spec.size());
        const dim3 gr((ns + 255) / 256, nslots);
        const int M = T_.centered ? 2 * H : H;
        const T* K = static_cast<const T*>(p->d_K);
        const uint32_t* sh = static_cast<const uint32_t*>(p->d_spec_h);
        const bool perm = p->rep_perm;
        if (p->rep_diag8) {
          CFFT_FOR_M(M, {
            if (use_K) k_recon_diag8<T, MM, true><<<gr, 256, 0, st>>>(g, tab, sh, K, W, F, nb);
            else k_recon_diag8<T, MM, false><<<gr, 256, 0, st>>>(g, tab, sh, nullptr, W, F, nb);
          });
          break;
        }
#define CFFT_RECON_D(DD)                                                                                  \
  CFFT_FOR_M(M, {                                                                                         \
    if (use_K) {                                                                                          \
      if (perm) k_recon_h<T, MM, DD, true, true><<<gr, 256, 0, st>>>(g, tab, sh, K, W, F, nb);            \
      else k_recon_h<T, MM, DD, true, false><<<gr, 256, 0, st>>>(g, tab, sh, K, W, F, nb);                \
    } else {                                                                                              \
      if (perm) k_recon_h<T, MM, DD, false, true><<<gr, 256, 0, st>>>(g, tab, sh, nullptr, W, F, nb);     \
      else k_recon_h<T, MM, DD, false, false><<<gr, 256, 0, st>>>(g, tab, sh, nullptr, W, F, nb);         \
    }                                                                                                     \
  })
        switch (T_.d) {
          case 1: CFFT_RECON_D(1); break;
          case 2: CFFT_RECON_D(2); break;
          case 4: CFFT_RECON_D(4); break;
          default: CFFT_RECON_D(8); break;
        }
#undef CFFT_RECON_D
        break;
      }
      case 3: {
        const int no = static_cast<int>(T_.orbit_rep.size());
        if (p->reps_smem) {
          const int parts = nb >= 100 ? 1 : std::max(1, std::min((148 + nb - 1) / nb, (no + 1023) / 1024));
          const int per = (no + parts - 1) / parts;
          const size_t smem = T_.spec.size() * cs;
          const uint32_t* pk = static_cast<const uint32_t*>(p->d_inv_pk);
          switch (T_.d) {
            case 1: k_inv_recon_reps_smem<T, 1><<<dim3(parts, nb), 1024, smem, st>>>(g, tab, pk, Fin, static_cast<C*>(p->d_g0r), per); break;
            case 2: k_inv_recon_reps_smem<T, 2><<<dim3(parts, nb), 1024, smem, st>>>(g, tab, pk, Fin, static_cast<C*>(p->d_g0r), per); break;
            case 4: k_inv_recon_reps_smem<T, 4><<<dim3(parts, nb), 1024, smem, st>>>(g, tab, pk, Fin, static_cast<C*>(p->d_g0r), per); break;
            default: k_inv_recon_reps_smem<T, 8><<<dim3(parts, nb), 1024, smem, st>>>(g, tab, pk, Fin, static_cast<C*>(p->d_g0r), per); break;
          }
          break;
        }
        k_inv_recon_reps<T><<<dim3((no + 127) / 128, (nslots + kRepSlots - 1) / kRepSlots), 128, 0, st>>>(
            g, tab, static_cast<const int32_t*>(p->d_inv_spec), static_cast<const int32_t*>(p->d_inv_phase), Fin,
            static_cast<C*>(p->d_g0r), nb);
        break;
      }
      case 4:
        CFFT_FOR_H(H, {
          if (p->reps_smem)
            k_expand2_ifft_z_h<T, HH><<<gz, thr_z, 0, st>>>(g, tab, static_cast<const int2*>(p->d_expand),
                                                            static_cast<const C*>(p->d_g0r), W, nb);
          else
            k_expand_ifft_z_h<T, HH><<<gz, thr_z, smem_z, st>>>(g, tab, static_cast<const int2*>(p->d_expand),
                                                                static_cast<const C*>(p->d_g0r), W);
        });
        break;
      default:
        CFFT_FOR_H(H, {
          if (E) k_plane_bwd_h<T, HH, true><<<dim3(H, nslots), thr_plane, smem_plane, st>>>(g, tab, W, E, f0_out, nb);
          else k_plane_bwd_h<T, HH, false><<<dim3(H, nslots), thr_plane, smem_plane, st>>>(g, tab, W, nullptr, f0_out, nb);
        });
        break;
    }
    ++g_launches;
    return;
  }
  switch (stage) {
    case 0:
      if (E) k_plane_fwd<T, true><<<dim3(T_.H[2], nb), p->threads_xy, p->smem_xy, st>>>(g, tab, f0, E, W);
      else k_plane_fwd<T, false><<<dim3(T_.H[2], nb), p->threads_xy, p->smem_xy, st>>>(g, tab, f0, nullptr, W);
      break;
    case 1:
      if (T_.H[2] <= 1) return;
      k_fft_z<T, false><<<dim3(T_.H[1], T_.n_ch, nb), p->threads_z, p->smem_z, st>>>(g, tab, W);
      break;
    case 2: {
      const int ns = static_cast<int>(T_.spec.size());
      const dim3 gr((ns + 255) / 256, nb);
      if (use_K)
        k_recon<T, true><<<gr, 256, 0, st>>>(g, tab, static_cast<const uint32_t*>(p->d_spec_h), static_cast<const T*>(p->d_K), W, F);
      else
        k_recon<T, false><<<gr, 256, 0, st>>>(g, tab, static_cast<const uint32_t*>(p->d_spec_h), nullptr, W, F);
      break;
    }
    case 3: {
      const int no = static_cast<int>(T_.orbit_rep.size());
      k_inv_recon<T><<<dim3((no + 127) / 128, nb), 128, 0, st>>>(
          g, tab, static_cast<const int32_t*>(p->d_orbit_rep), static_cast<const int32_t*>(p->d_inv_spec),
          static_cast<const int32_t*>(p->d_inv_phase), static_cast<const uint32_t*>(p->d_img_mask), Fin, W);
      break;
    }
    case 4:
      if (T_.H[2] <= 1) return;
      k_fft_z<T, true><<<dim3(T_.H[1], T_.n_ch, nb), p->threads_z, p->smem_z, st>>>(g, tab, W);
      break;
    default:
      if (E) k_plane_bwd<T, true><<<dim3(T_.H[2], nb), p->threads_xy, p->smem_xy, st>>>(g, tab, W, E, f0_out);
      else k_plane_bwd<T, false><<<dim3(T_.H[2], nb), p->threads_xy, p->smem_xy, st>>>(g, tab, W, nullptr, f0_out);
      break;
  }
  ++g_launches;
}

// Forward and/or backward over B fields in workspace-sized chunks.  F holds the
// spectra of all B fields (the forward output, the backward input).
template <typename T>
Status run_chunks(Plan* p, bool fwd, bool bwd, const T* f0, typename Cx<T>::type* F, T* f0_out, const T* E,
                  bool use_K, int B, cudaStream_t st, std::string* err) {
  const size_t mvol = static_cast<size_t>(p->T.M[0]) * p->T.M[1] * p->T.M[2];
  const size_t ns = p->T.spec.size();
  for (int b0 = 0; b0 < B; b0 += p->chunk) {
    const int nb = std::min(p->chunk, B - b0);
    const T* fin = f0 ? f0 + b0 * mvol : nullptr;
    T* fout = f0_out ? f0_out + b0 * mvol : nullptr;
    const T* Ec = E ? E + b0 * mvol : nullptr;
    auto* Fc = F + b0 * ns;
    if (fwd)
      for (int s = 0; s < 3; ++s) launch_stage<T>(p, s, fin, Fc, nullptr, nullptr, Ec, use_K, nb, st);
    if (bwd)
      for (int s = 3; s < 6; ++s) launch_stage<T>(p, s, nullptr, nullptr, Fc, fout, Ec, false, nb, st);
  }
  CFFT_CUDA(cudaGetLastError(), fwd ? "forward launch" : "backward launch");
  return Status::kOk;
}

template <typename T>
Status profile_roundtrip(Plan* p, const T* f0, typename Cx<T>::type* F, T* f0_out, int B, cudaStream_t st,
                         float* ms, int* n, std::string* err) {
  cudaEvent_t ev[7];
  for (int i = 0; i < 7; ++i) CFFT_CUDA(cudaEventCreate(&ev[i]), "event create");
  for (int s = 0; s < 6; ++s) ms[s] = 0.f;
  const size_t mvol = static_cast<size_t>(p->T.M[0]) * p->T.M[1] * p->T.M[2];
  const size_t ns = p->T.spec.size();
  for (int b0 = 0; b0 < B; b0 += p->chunk) {
    const int nb = std::min(p->chunk, B - b0);
    CFFT_CUDA(cudaEventRecord(ev[0], st), "event record");
    for (int s = 0; s < 6; ++s) {
      launch_stage<T>(p, s, f0 + b0 * mvol, F + b0 * ns, F + b0 * ns, f0_out + b0 * mvol, nullptr, false, nb, st);
      CFFT_CUDA(cudaEventRecord(ev[s + 1], st), "event record");
    }
    CFFT_CUDA(cudaGetLastError(), "profile launch");
    CFFT_CUDA(cudaEventSynchronize(ev[6]), "event sync");
    for (int s = 0; s < 6; ++s) {
      float t = 0.f;
      CFFT_CUDA(cudaEventElapsedTime(&t, ev[s], ev[s + 1]), "elapsed");
      ms[s] += t;
    }
  }
  *n = 6;
  for (int i = 0; i < 7; ++i) cudaEventDestroy(ev[i]);
  return Status::kOk;
}

Status check_batch(const Plan* p, int B, std::string* err) {
  if (B < 1 || B > p->max_batch) { *err = "batch must be in [1, max_batch]"; return Status::kInvalid; }
  return Status::kOk;
}

}  // namespace

int64_t launch_count(bool reset) {
  const int64_t v = g_launches;
  if (reset) g_launches = 0;
  return v;
}

Status plan_device_init(Plan* p, std::string* err) {
  const PlanTables& T = p->T;
  DevGeom g;
  std::memset(&g, 0, sizeof(g));
  for (int d = 0; d < 3; ++d) {
    g.N[d] = T.N[d]; g.M[d] = T.M[d]; g.H[d] = T.H[d]; g.L[d] = T.L[d];
    if (!factor_radices(T.H[d], &g.nf[d], g.radix[d])) { *err = "FFT length must factor into 2, 3, 5"; return Status::kUnsupported; }
  }
  g.P = T.P; g.d = T.d; g.n_ch = T.n_ch; g.centered = T.centered ? 1 : 0;
  g.pmask = (T.P & (T.P - 1)) == 0 ? T.P - 1 : -1;
  g.n_spec = static_cast<int>(T.spec.size());
  g.n_orbits = static_cast<int>(T.orbit_rep.size());
  g.n_rem = static_cast<int>(T.rem_ops.size());
  if (g.n_rem > kMaxRem) { *err = "too many even-translation operations"; return Status::kUnsupported; }
  if (T.d > 8) { *err = "fiber length above 8"; return Status::kUnsupported; }
  if (T.P > 8192) { *err = "phase denominator lcm(N) above 8192"; return Status::kUnsupported; }
  p->n_mask_words = (g.n_rem + 31) / 32;
  g.n_mask_words = p->n_mask_words;
  for (int k = 0; k < 8; ++k) g.chan_of_parity[k] = T.chan_of_parity[k];
  for (int c = 0; c < T.n_ch; ++c) g.off_idx[c] = T.offsets[c][0] + 2 * T.offsets[c][1] + 4 * T.offsets[c][2];
  for (int r = 0; r < T.d; ++r) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) g.rep_R[r][i * 3 + j] = T.rep_ops[r].R[i][j];
    for (int i = 0; i < 3; ++i) {
      g.rep_t[r][i] = T.rep_ops[r].t[i];
      g.rep_tp[r][i] = T.rep_ops[r].t[i] * (T.P / T.N[i]);
    }
  }
  for (int r = 0; r < g.n_rem; ++r) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) g.rem_R[r][i * 3 + j] = T.rem_ops[r].R[i][j];
    for (int i = 0; i < 3; ++i) g.rem_s[r][i] = T.rem_ops[r].t[i];
  }
  // Signed-permutation form of R_b^T (column dd of R_b holds a single +-1).
  g.rep_perm = 1;
  for (int r = 0; r < T.d && g.rep_perm; ++r)
    for (int dd = 0; dd < 3; ++dd) {
      int nz = 0, src = 0, neg = 0;
      for (int d2 = 0; d2 < 3; ++d2) {
        const int v = T.rep_ops[r].R[d2][dd];
        if (v == 0) continue;
        ++nz; src = d2; neg = v < 0;
        if (v != 1 && v != -1) nz = 9;
      }
      if (nz != 1) { g.rep_perm = 0; break; }
      g.rep_ps[r][dd] = src + 4 * neg;
    }
  p->rep_perm = g.rep_perm != 0;
  // The 8 representatives are exactly the 8 diagonal sign matrices?
  g.rep_diag8 = T.d == 8 ? 1 : 0;
  for (int k = 0; k < 8; ++k) g.sign_op[k] = -1;
  for (int r = 0; r < T.d && g.rep_diag8; ++r) {
    int sg = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
        const int v = T.rep_ops[r].R[i][j];
        if (i != j && v != 0) g.rep_diag8 = 0;
        if (i == j && v != 1 && v != -1) g.rep_diag8 = 0;
        if (i == j && v == -1) sg |= 1 << i;
      }
    if (g.rep_diag8 && g.sign_op[sg] >= 0) g.rep_diag8 = 0;
    if (g.rep_diag8) g.sign_op[sg] = r;
  }
  p->rep_diag8 = g.rep_diag8 != 0;
  // Fast (compile-time sized) path for cubic channel grids.
  const bool cubic = T.H[0] == T.H[1] && T.H[1] == T.H[2];
  p->fast_h = (cubic && (p->precision == 8 ? fast_ok<double>(T.H[0]) : fast_ok<float>(T.H[0]))) ? T.H[0] : 0;
  if (const char* f = std::getenv("CFFT_DISABLE_FAST")) {
    if (f[0] == '1') p->fast_h = 0;
  }
  // distinct-image masks: op i contributes only if no earlier op maps the representative to the same point
  std::vector<uint32_t> masks(static_cast<size_t>(g.n_orbits) * p->n_mask_words, 0u);
  const size_t hvol = static_cast<size_t>(T.H[0]) * T.H[1] * T.H[2];
  std::vector<int2> expand;
  if (p->fast_h) expand.assign(static_cast<size_t>(T.n_ch) * hvol, make_int2(-1, 0));
  for (int o = 0; o < g.n_orbits; ++o) {
    const int m = T.orbit_rep[o];
    const int q[3] = {m % T.M[0], (m / T.M[0]) % T.M[1], m / (T.M[0] * T.M[1])};
    std::vector<long> seen;
    for (int i = 0; i < g.n_rem; ++i) {
      long li = 0, stride = 1;
      int qq[3];
      for (int dd = 0; dd < 3; ++dd) {
        long v = 0;
        for (int d2 = 0; d2 < 3; ++d2) v += static_cast<long>(T.rem_ops[i].R[d2][dd]) * q[d2];
        qq[dd] = static_cast<int>(floor_mod(v, T.M[dd]));
        li += qq[dd] * stride;
        stride *= T.M[dd];
      }
      if (std::find(seen.begin(), seen.end(), li) != seen.end()) continue;
      seen.push_back(li);
      masks[static_cast<size_t>(o) * p->n_mask_words + (i >> 5)] |= 1u << (i & 31);
      if (p->fast_h) {
        long j = 0;
        for (int dd = 0; dd < 3; ++dd) j += static_cast<long>(q[dd]) * T.rem_ops[i].t[dd] * (T.P / T.M[dd]);
        size_t pos;
        if (T.centered) {
          const int c = T.chan_of_parity[(qq[0] & 1) + 2 * (qq[1] & 1) + 4 * (qq[2] & 1)];
          if (c < 0) { *err = "orbit image outside the alive channels"; return Status::kInvalid; }
          pos = static_cast<size_t>(c) * hvol + (static_cast<size_t>(qq[2] >> 1) * T.H[1] + (qq[1] >> 1)) * T.H[0] + (qq[0] >> 1);
        } else {
          pos = (static_cast<size_t>(qq[2]) * T.H[1] + qq[1]) * T.H[0] + qq[0];
        }
        expand[pos] = make_int2(o, static_cast<int>(floor_mod(j, T.P)));
      }
    }
  }
  for (const int2& e : expand)
    if (e.x < 0) { *err = "orbit expansion does not cover the channel grid"; return Status::kInvalid; }
  std::vector<uint32_t> hp(T.spec.size());
  for (size_t s = 0; s < T.spec.size(); ++s)
    hp[s] = static_cast<uint32_t>(T.spec[s].h[0]) | (static_cast<uint32_t>(T.spec[s].h[1]) << 10) |
            (static_cast<uint32_t>(T.spec[s].h[2]) << 20);
  std::vector<unsigned char> tab = p->precision == 8 ? make_table_bytes<double>(*p, &g) : make_table_bytes<float>(*p, &g);

  const size_t rs = p->precision;          // real size
  const size_t cs = 2 * rs;                // complex size
  const size_t mvol = static_cast<size_t>(T.M[0]) * T.M[1] * T.M[2];
  const size_t B = p->max_batch;
  // Chunk the batch: each chunk's channel workspace is at most `budget` bytes (64 MiB by
  // default; measured: fewer, larger launches beat keeping the workspace L2-resident).
  // On the fast path two fields share one workspace slot, and chunks hold whole pairs.
  size_t budget = static_cast<size_t>(64) << 20;
  if (const char* cb = std::getenv("CFFT_CHUNK_BYTES")) budget = std::strtoull(cb, nullptr, 10);
  const size_t per_field = T.n_ch * hvol * cs / (p->fast_h ? 2 : 1);
  size_t ch = std::max<size_t>(1, std::min<size_t>(B, budget / std::max<size_t>(per_field, 1)));
  if (p->fast_h && ch < B && ch > 1) ch &= ~static_cast<size_t>(1);
  p->chunk = static_cast<int>(ch);
  // launch geometry and shared memory (generic path)
  const long pe = static_cast<long>(T.n_ch) * T.H[0] * T.H[1];
  const long ze = static_cast<long>(T.H[0]) * T.H[2];
  p->threads_xy = round_threads(pe);
  p->threads_z = round_threads(ze);
  p->smem_xy = (2 * pe + T.H[0] + T.H[1]) * cs;
  p->smem_z = (2 * ze + T.H[2]) * cs;
  if (!p->fast_h && (p->smem_xy > 227 * 1024 || p->smem_z > 227 * 1024)) { *err = "shared memory above 227 KB"; return Status::kUnsupported; }

  auto alloc = [&](void** ptr, size_t bytes, const char* what) -> Status {
    cudaError_t e = cudaMalloc(ptr, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) { *err = cuda_msg(e, what); return Status::kAlloc; }
    p->workspace_bytes += bytes;
    return Status::kOk;
  };
  const size_t chunk = static_cast<size_t>(p->chunk);
  Status st;
  if ((st = alloc(&p->d_geom, sizeof(DevGeom), "geometry")) != Status::kOk) return st;
  if ((st = alloc(&p->d_tables, tab.size(), "tables")) != Status::kOk) return st;
  if ((st = alloc(&p->d_spec_h, hp.size() * 4, "spectral points")) != Status::kOk) return st;
  if ((st = alloc(&p->d_K, T.spec.size() * rs, "kernel")) != Status::kOk) return st;
  if ((st = alloc(&p->d_orbit_rep, T.orbit_rep.size() * 4, "orbit reps")) != Status::kOk) return st;
  if ((st = alloc(&p->d_inv_spec, T.inv_spec.size() * 4, "inverse spec")) != Status::kOk) return st;
  if ((st = alloc(&p->d_inv_phase, T.inv_phase.size() * 4, "inverse phase")) != Status::kOk) return st;
  if ((st = alloc(&p->d_img_mask, masks.size() * 4, "image masks")) != Status::kOk) return st;
  if ((st = alloc(&p->d_work_T, chunk * T.n_ch * hvol * cs, "channel workspace")) != Status::kOk) return st;
  if ((st = alloc(&p->d_work_F, B * T.spec.size() * cs, "spectrum workspace")) != Status::kOk) return st;
  if ((st = alloc(&p->d_work_E, B * mvol * rs, "interaction workspace")) != Status::kOk) return st;
  // Per-field representative gather from a shared-memory copy of the spectrum.
  std::vector<uint32_t> inv_pk;
  p->reps_smem = p->fast_h && T.spec.size() * cs <= 200 * 1024 && T.spec.size() < (1u << 20) - 1 && T.P <= 2048;
  if (p->reps_smem) {
    inv_pk.resize(T.inv_spec.size());
    for (size_t k = 0; k < inv_pk.size(); ++k) {
      const int sp = T.inv_spec[k];
      const uint32_t a = static_cast<uint32_t>(sp < 0 ? -sp : sp);
      inv_pk[k] = a | (sp < 0 ? (1u << 20) : 0u) | (static_cast<uint32_t>(T.inv_phase[k]) << 21);
    }
    if ((st = alloc(&p->d_inv_pk, inv_pk.size() * 4, "packed inverse table")) != Status::kOk) return st;
  }
  if (p->fast_h) {
    if ((st = alloc(&p->d_expand, expand.size() * sizeof(int2), "expansion table")) != Status::kOk) return st;
    if ((st = alloc(&p->d_g0r, (chunk + 1) * T.orbit_rep.size() * cs, "representative workspace")) != Status::kOk) return st;
  }
  CFFT_CUDA(cudaMemcpy(p->d_geom, &g, sizeof(g), cudaMemcpyHostToDevice), "upload geometry");
  CFFT_CUDA(cudaMemcpy(p->d_tables, tab.data(), tab.size(), cudaMemcpyHostToDevice), "upload tables");
  CFFT_CUDA(cudaMemcpy(p->d_spec_h, hp.data(), hp.size() * 4, cudaMemcpyHostToDevice), "upload spectral points");
  if (!T.orbit_rep.empty()) {
    CFFT_CUDA(cudaMemcpy(p->d_orbit_rep, T.orbit_rep.data(), T.orbit_rep.size() * 4, cudaMemcpyHostToDevice), "upload reps");
    CFFT_CUDA(cudaMemcpy(p->d_inv_spec, T.inv_spec.data(), T.inv_spec.size() * 4, cudaMemcpyHostToDevice), "upload inv spec");
    CFFT_CUDA(cudaMemcpy(p->d_inv_phase, T.inv_phase.data(), T.inv_phase.size() * 4, cudaMemcpyHostToDevice), "upload inv phase");
    CFFT_CUDA(cudaMemcpy(p->d_img_mask, masks.data(), masks.size() * 4, cudaMemcpyHostToDevice), "upload masks");
  }
  if (p->fast_h)
    CFFT_CUDA(cudaMemcpy(p->d_expand, expand.data(), expand.size() * sizeof(int2), cudaMemcpyHostToDevice), "upload expansion");
  if (p->reps_smem)
    CFFT_CUDA(cudaMemcpy(p->d_inv_pk, inv_pk.data(), inv_pk.size() * 4, cudaMemcpyHostToDevice), "upload packed table");
  // Orbit expansion writes only alive positions; channel positions never written stay zero.
  CFFT_CUDA(cudaMemset(p->d_work_T, 0, chunk * T.n_ch * hvol * cs), "clear workspace");
  if (p->precision == 8) set_smem_attrs<double>();
  else set_smem_attrs<float>();
  CFFT_CUDA(cudaGetLastError(), "set shared-memory attributes");
  if ((st = upload_const_twiddles(err)) != Status::kOk) return st;
  cudaStream_t s;
  CFFT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "create stream");
  p->own_stream = s;
  return plan_upload_kernel(p, err);
}

Status plan_upload_kernel(Plan* p, std::string* err) {
  compute_kernel(p->T, p->lattice, p->ds, &p->T.K);
  if (p->precision == 8) {
    CFFT_CUDA(cudaMemcpy(p->d_K, p->T.K.data(), p->T.K.size() * 8, cudaMemcpyHostToDevice), "upload K");
  } else {
    std::vector<float> k(p->T.K.begin(), p->T.K.end());
    CFFT_CUDA(cudaMemcpy(p->d_K, k.data(), k.size() * 4, cudaMemcpyHostToDevice), "upload K");
  }
  return Status::kOk;
}

void plan_device_free(Plan* p) {
  void** bufs[] = {&p->d_geom, &p->d_tables, &p->d_spec_h, &p->d_K, &p->d_orbit_rep, &p->d_inv_spec,
                   &p->d_inv_phase, &p->d_img_mask, &p->d_fill_map, &p->d_work_T, &p->d_work_F,
                   &p->d_work_E, &p->d_stage_in, &p->d_stage_out, &p->d_expand, &p->d_g0r, &p->d_inv_pk};
  for (void** b : bufs)
    if (*b) { cudaFree(*b); *b = nullptr; }
  if (p->own_stream) { cudaStreamDestroy(static_cast<cudaStream_t>(p->own_stream)); p->own_stream = nullptr; }
}

Status exec_forward(Plan* p, const void* f0, void* F, int B, void* stream, std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  if (!f0 || !F) { *err = "null pointer"; return Status::kInvalid; }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->precision == 8)
    return run_chunks<double>(p, true, false, static_cast<const double*>(f0), static_cast<double2*>(F), nullptr, nullptr, false, B, s, err);
  return run_chunks<float>(p, true, false, static_cast<const float*>(f0), static_cast<float2*>(F), nullptr, nullptr, false, B, s, err);
}

Status exec_profile_roundtrip(Plan* p, const void* f0, void* F, void* f0_out, int B, void* stream, float* ms,
                              int* n, std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  if (!f0 || !F || !f0_out || !ms || !n) { *err = "null pointer"; return Status::kInvalid; }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->precision == 8)
    return profile_roundtrip<double>(p, static_cast<const double*>(f0), static_cast<double2*>(F), static_cast<double*>(f0_out), B, s, ms, n, err);
  return profile_roundtrip<float>(p, static_cast<const float*>(f0), static_cast<float2*>(F), static_cast<float*>(f0_out), B, s, ms, n, err);
}

Status exec_backward(Plan* p, const void* F, void* f0, int B, void* stream, std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  if (!f0 || !F) { *err = "null pointer"; return Status::kInvalid; }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->precision == 8)
    return run_chunks<double>(p, false, true, nullptr, const_cast<double2*>(static_cast<const double2*>(F)), static_cast<double*>(f0), nullptr, false, B, s, err);
  return run_chunks<float>(p, false, true, nullptr, const_cast<float2*>(static_cast<const float2*>(F)), static_cast<float*>(f0), nullptr, false, B, s, err);
}

Status exec_scft_step(Plan* p, void* f0, int B, void* stream, std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  if (!f0) { *err = "null pointer"; return Status::kInvalid; }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->precision == 8)
    return run_chunks<double>(p, true, true, static_cast<const double*>(f0), static_cast<double2*>(p->d_work_F), static_cast<double*>(f0), nullptr, true, B, s, err);
  return run_chunks<float>(p, true, true, static_cast<const float*>(f0), static_cast<float2*>(p->d_work_F), static_cast<float*>(f0), nullptr, true, B, s, err);
}

Status exec_step_diffusion(Plan* p, void* q, const void* w, double dt, int n_steps, int B, void* stream,
                           std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  if (!q || !w || n_steps < 0) { *err = "invalid argument"; return Status::kInvalid; }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t n = static_cast<size_t>(B) * p->T.M[0] * p->T.M[1] * p->T.M[2];
  const int grid = static_cast<int>(std::min<size_t>((n + 255) / 256, 148 * 16));
  if (p->precision == 8) {
    k_interaction<double><<<grid, 256, 0, s>>>(static_cast<const double*>(w), static_cast<double*>(p->d_work_E), dt / 2, n);
    ++g_launches;
    for (int i = 0; i < n_steps; ++i) {
      st = run_chunks<double>(p, true, true, static_cast<const double*>(q), static_cast<double2*>(p->d_work_F),
                              static_cast<double*>(q), static_cast<const double*>(p->d_work_E), true, B, s, err);
      if (st != Status::kOk) return st;
    }
  } else {
    k_interaction<float><<<grid, 256, 0, s>>>(static_cast<const float*>(w), static_cast<float*>(p->d_work_E),
                                              static_cast<float>(dt / 2), n);
    ++g_launches;
    for (int i = 0; i < n_steps; ++i) {
      st = run_chunks<float>(p, true, true, static_cast<const float*>(q), static_cast<float2*>(p->d_work_F),
                             static_cast<float*>(q), static_cast<const float*>(p->d_work_E), true, B, s, err);
      if (st != Status::kOk) return st;
    }
  }
  CFFT_CUDA(cudaGetLastError(), "step_diffusion launch");
  return Status::kOk;
}

// _build_fill_map (src/q_fused_krfft.jl:733-783): for each grid point the first
// operation that lands it on the stride-L subgrid.
static Status ensure_fill_map(Plan* p, std::string* err) {
  if (p->d_fill_map) return Status::kOk;
  const PlanTables& T = p->T;
  const long n1 = T.N[0], n2 = T.N[1], n3 = T.N[2];
  p->fill_map.assign(n1 * n2 * n3, -1);
  for (long z = 0; z < n3; ++z)
    for (long y = 0; y < n2; ++y)
      for (long x = 0; x < n1; ++x) {
        const long X[3] = {x, y, z};
        for (const auto& op : T.ops) {
          long sub = 0, stride = 1;
          bool on = true;
          for (int d = 0; d < 3 && on; ++d) {
            long v = op.t[d];
            for (int j = 0; j < 3; ++j) v += static_cast<long>(op.R[d][j]) * X[j];
            v = floor_mod(v, T.N[d]);
            if (v % T.L[d] != 0) on = false;
            sub += (v / T.L[d]) * stride;
            stride *= T.M[d];
          }
          if (on) { p->fill_map[x + n1 * (y + n2 * z)] = static_cast<int32_t>(sub); break; }
        }
        if (p->fill_map[x + n1 * (y + n2 * z)] < 0) {
          *err = "No symmetry operation maps a grid point to the subgrid";
          return Status::kInvalid;
        }
      }
  CFFT_CUDA(cudaMalloc(&p->d_fill_map, p->fill_map.size() * 4), "alloc fill map");
  CFFT_CUDA(cudaMemcpy(p->d_fill_map, p->fill_map.data(), p->fill_map.size() * 4, cudaMemcpyHostToDevice), "upload fill map");
  return Status::kOk;
}

Status exec_full_to_sub(Plan* p, const void* u, void* f0, int B, void* stream, std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  const PlanTables& T = p->T;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t mvol = static_cast<size_t>(T.M[0]) * T.M[1] * T.M[2];
  const size_t nvol = static_cast<size_t>(T.N[0]) * T.N[1] * T.N[2];
  const int grid = static_cast<int>(std::min<size_t>((mvol * B + 255) / 256, 148 * 16));
  if (p->precision == 8)
    k_full_to_sub<double><<<grid, 256, 0, s>>>(static_cast<const double*>(u), static_cast<double*>(f0), T.N[0], T.N[1],
                                               T.L[0], T.L[1], T.L[2], T.M[0], T.M[1], mvol, nvol, B);
  else
    k_full_to_sub<float><<<grid, 256, 0, s>>>(static_cast<const float*>(u), static_cast<float*>(f0), T.N[0], T.N[1],
                                              T.L[0], T.L[1], T.L[2], T.M[0], T.M[1], mvol, nvol, B);
  ++g_launches;
  CFFT_CUDA(cudaGetLastError(), "fullgrid_to_subgrid launch");
  return Status::kOk;
}

Status exec_sub_to_full(Plan* p, const void* f0, void* u, int B, void* stream, std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  if ((st = ensure_fill_map(p, err)) != Status::kOk) return st;
  const PlanTables& T = p->T;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t mvol = static_cast<size_t>(T.M[0]) * T.M[1] * T.M[2];
  const size_t nvol = static_cast<size_t>(T.N[0]) * T.N[1] * T.N[2];
  const int grid = static_cast<int>(std::min<size_t>((nvol * B + 255) / 256, 148 * 16));
  if (p->precision == 8)
    k_sub_to_full<double><<<grid, 256, 0, s>>>(static_cast<const double*>(f0), static_cast<const int32_t*>(p->d_fill_map),
                                               static_cast<double*>(u), mvol, nvol, B);
  else
    k_sub_to_full<float><<<grid, 256, 0, s>>>(static_cast<const float*>(f0), static_cast<const int32_t*>(p->d_fill_map),
                                              static_cast<float*>(u), mvol, nvol, B);
  ++g_launches;
  CFFT_CUDA(cudaGetLastError(), "subgrid_to_fullgrid launch");
  return Status::kOk;
}

// which: 0 forward, 1 backward, 2 scft step (in place on the host buffer `out`)
Status exec_host(Plan* p, int which, const void* in, void* out, int B, std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  const PlanTables& T = p->T;
  const size_t rs = p->precision, cs = 2 * rs;
  const size_t fbytes = static_cast<size_t>(B) * T.M[0] * T.M[1] * T.M[2] * rs;
  const size_t sbytes = static_cast<size_t>(B) * T.spec.size() * cs;
  const size_t fmax = static_cast<size_t>(p->max_batch) * T.M[0] * T.M[1] * T.M[2] * rs;
  const size_t smax = static_cast<size_t>(p->max_batch) * T.spec.size() * cs;
  if (!p->d_stage_in) {
    CFFT_CUDA(cudaMalloc(&p->d_stage_in, std::max(fmax, smax)), "alloc staging");
    CFFT_CUDA(cudaMalloc(&p->d_stage_out, std::max(fmax, smax)), "alloc staging");
    p->workspace_bytes += 2 * std::max(fmax, smax);
  }
  cudaStream_t s = static_cast<cudaStream_t>(p->own_stream);
  if (which == 0) {
    CFFT_CUDA(cudaMemcpyAsync(p->d_stage_in, in, fbytes, cudaMemcpyHostToDevice, s), "H2D");
    if ((st = exec_forward(p, p->d_stage_in, p->d_stage_out, B, s, err)) != Status::kOk) return st;
    CFFT_CUDA(cudaMemcpyAsync(out, p->d_stage_out, sbytes, cudaMemcpyDeviceToHost, s), "D2H");
  } else if (which == 1) {
    CFFT_CUDA(cudaMemcpyAsync(p->d_stage_in, in, sbytes, cudaMemcpyHostToDevice, s), "H2D");
    if ((st = exec_backward(p, p->d_stage_in, p->d_stage_out, B, s, err)) != Status::kOk) return st;
    CFFT_CUDA(cudaMemcpyAsync(out, p->d_stage_out, fbytes, cudaMemcpyDeviceToHost, s), "D2H");
  } else {
    CFFT_CUDA(cudaMemcpyAsync(p->d_stage_in, out, fbytes, cudaMemcpyHostToDevice, s), "H2D");
    if ((st = exec_scft_step(p, p->d_stage_in, B, s, err)) != Status::kOk) return st;
    CFFT_CUDA(cudaMemcpyAsync(out, p->d_stage_in, fbytes, cudaMemcpyDeviceToHost, s), "D2H");
  }
  CFFT_CUDA(cudaStreamSynchronize(s), "synchronize");
  return Status::kOk;
}

// ---------------------------------------------------------------- allocation-free forward
// cfft_forward_noalloc: the forward transform for callers that may not allocate
// device memory (for example a process whose device memory belongs entirely to
// another allocator, or code that must not call into the driver's allocator while
// it runs).  The channel workspace, the geometry and the twiddle/phase tables live in
// one file-scope static device array instead of cudaMalloc'd plan buffers, so a plan
// built with cfft_plan_create_host (host memory only) is enough.  Every GPU that
// loads this library holds the array (kNoAllocBytes) until the process exits.
namespace {

constexpr size_t kNoAllocBytes = static_cast<size_t>(32) << 20;  // 32 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];
std::mutex g_noalloc_mu;
constexpr int kNoAllocMaxDevices = 64;
unsigned char* g_noalloc_addr[kNoAllocMaxDevices] = {nullptr};

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Device address of the static scratch for the current device, looked up once per
// device (the array's name is only a host-side stand-in in host code).
Status noalloc_scratch_for_current_device(unsigned char** out, std::string* err) {
  int dev = 0;
  CFFT_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices) { *err = "device ordinal above the supported range"; return Status::kUnsupported; }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_addr[dev]) {
    void* ptr = nullptr;
    CFFT_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress(static scratch)");
    set_smem_attrs<float>();
    set_smem_attrs<double>();
    CFFT_CUDA(cudaGetLastError(), "set shared-memory attributes");
    g_noalloc_addr[dev] = static_cast<unsigned char*>(ptr);
  }
  *out = g_noalloc_addr[dev];
  return Status::kOk;
}

template <typename T>
Status noalloc_forward(const Plan* p, const T* f0, typename Cx<T>::type* F, int B, cudaStream_t st,
                       std::string* err) {
  using C = typename Cx<T>::type;
  const PlanTables& Tb = p->T;
  DevGeom g;
  std::memset(&g, 0, sizeof(g));
  for (int d = 0; d < 3; ++d) {
    g.N[d] = Tb.N[d]; g.M[d] = Tb.M[d]; g.H[d] = Tb.H[d]; g.L[d] = Tb.L[d];
    if (!factor_radices(Tb.H[d], &g.nf[d], g.radix[d])) { *err = "FFT length must factor into 2, 3, 5"; return Status::kUnsupported; }
  }
  if (Tb.d > 8) { *err = "fiber length above 8"; return Status::kUnsupported; }
  if (Tb.P > 8192) { *err = "phase denominator lcm(N) above 8192"; return Status::kUnsupported; }
  g.P = Tb.P; g.d = Tb.d; g.n_ch = Tb.n_ch; g.centered = Tb.centered ? 1 : 0;
  g.pmask = (Tb.P & (Tb.P - 1)) == 0 ? Tb.P - 1 : -1;
  g.n_spec = static_cast<int>(Tb.spec.size());
  for (int k = 0; k < 8; ++k) g.chan_of_parity[k] = Tb.chan_of_parity[k];
  for (int c = 0; c < Tb.n_ch; ++c) g.off_idx[c] = Tb.offsets[c][0] + 2 * Tb.offsets[c][1] + 4 * Tb.offsets[c][2];
  for (int r = 0; r < Tb.d; ++r) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) g.rep_R[r][i * 3 + j] = Tb.rep_ops[r].R[i][j];
    for (int i = 0; i < 3; ++i) {
      g.rep_t[r][i] = Tb.rep_ops[r].t[i];
      g.rep_tp[r][i] = Tb.rep_ops[r].t[i] * (Tb.P / Tb.N[i]);
    }
  }
  std::vector<uint32_t> hp(Tb.spec.size());
  for (size_t s = 0; s < Tb.spec.size(); ++s)
    hp[s] = static_cast<uint32_t>(Tb.spec[s].h[0]) | (static_cast<uint32_t>(Tb.spec[s].h[1]) << 10) |
            (static_cast<uint32_t>(Tb.spec[s].h[2]) << 20);
  const std::vector<unsigned char> tab = make_table_bytes<T>(*p, &g);
  const size_t cs = sizeof(C);
  const size_t hvol = static_cast<size_t>(Tb.H[0]) * Tb.H[1] * Tb.H[2];
  const size_t off_tab = align256(sizeof(DevGeom));
  const size_t off_spec = off_tab + align256(tab.size());
  const size_t off_W = off_spec + align256(hp.size() * 4);
  const size_t per_field = align256(static_cast<size_t>(Tb.n_ch) * hvol * cs);
  if (off_W + per_field > kNoAllocBytes) {
    *err = "the allocation-free forward needs " + std::to_string(off_W + per_field) +
           " bytes of scratch for one field; its static scratch holds " + std::to_string(kNoAllocBytes) + " bytes";
    return Status::kUnsupported;
  }
  const int chunk = static_cast<int>((kNoAllocBytes - off_W) / per_field);
  const long pe = static_cast<long>(Tb.n_ch) * Tb.H[0] * Tb.H[1];
  const long ze = static_cast<long>(Tb.H[0]) * Tb.H[2];
  const int thr_xy = round_threads(pe), thr_z = round_threads(ze);
  const size_t smem_xy = (2 * pe + Tb.H[0] + Tb.H[1]) * cs, smem_z = (2 * ze + Tb.H[2]) * cs;
  if (smem_xy > 227 * 1024 || smem_z > 227 * 1024) { *err = "shared memory above 227 KB"; return Status::kUnsupported; }

  unsigned char* base = nullptr;
  Status s = noalloc_scratch_for_current_device(&base, err);
  if (s != Status::kOk) return s;
  // Pageable-source copies return once the host data is staged, so the locals may go.
  CFFT_CUDA(cudaMemcpyAsync(base, &g, sizeof(g), cudaMemcpyHostToDevice, st), "upload geometry");
  CFFT_CUDA(cudaMemcpyAsync(base + off_tab, tab.data(), tab.size(), cudaMemcpyHostToDevice, st), "upload tables");
  CFFT_CUDA(cudaMemcpyAsync(base + off_spec, hp.data(), hp.size() * 4, cudaMemcpyHostToDevice, st), "upload points");
  const DevGeom* dg = reinterpret_cast<const DevGeom*>(base);
  const C* dtab = reinterpret_cast<const C*>(base + off_tab);
  const uint32_t* dspec = reinterpret_cast<const uint32_t*>(base + off_spec);
  C* W = reinterpret_cast<C*>(base + off_W);
  const size_t mvol = static_cast<size_t>(Tb.M[0]) * Tb.M[1] * Tb.M[2];
  const int ns = g.n_spec;
  for (int b0 = 0; b0 < B; b0 += chunk) {
    const int nb = std::min(chunk, B - b0);
    k_plane_fwd<T, false><<<dim3(Tb.H[2], nb), thr_xy, smem_xy, st>>>(dg, dtab, f0 + b0 * mvol, nullptr, W);
    ++g_launches;
    if (Tb.H[2] > 1) {
      k_fft_z<T, false><<<dim3(Tb.H[1], Tb.n_ch, nb), thr_z, smem_z, st>>>(dg, dtab, W);
      ++g_launches;
    }
    k_recon<T, false><<<dim3((ns + 255) / 256, nb), 256, 0, st>>>(dg, dtab, dspec, nullptr, W,
                                                                    F + static_cast<size_t>(b0) * ns);
    ++g_launches;
  }
  CFFT_CUDA(cudaGetLastError(), "allocation-free forward launch");
  return Status::kOk;
}

}  // namespace

Status exec_forward_noalloc(const Plan* p, const void* f0, void* F, int B, void* stream, std::string* err) {
  if (B < 1 || !f0 || !F) { *err = "invalid argument (batch < 1 or null pointer)"; return Status::kInvalid; }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->precision == 8)
    return noalloc_forward<double>(p, static_cast<const double*>(f0), static_cast<double2*>(F), B, s, err);
  return noalloc_forward<float>(p, static_cast<const float*>(f0), static_cast<float2*>(F), B, s, err);
}

}  // namespace cfft
