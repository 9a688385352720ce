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
#include <cstdint>
#include <cstdlib>
#include <mutex>
#include <tuple>

#include "device_common.cuh"
#include "exec.h"
#include "fast_api.h"

namespace cfft {

namespace {

thread_local int64_t g_launches = 0;

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

// ---------------------------------------------------------------- elementwise
template <typename T>
__global__ void k_interaction(const T* __restrict__ w, T* __restrict__ E, T half_dt, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x)
    E[i] = exp(-w[i] * half_dt);
}

// Subgrid spectrum G0 = FFT_M(f0) of each field from the forward workspace of the
// compile-time sized path (slot s holds X = G0_a + i G0_b, z-fastest per channel):
// G0_a(q) = (X(q) + conj X(-q)) / 2, G0_b(q) = (X(q) - conj X(-q)) / 2i.  On the
// centred path q = 2k + off reads channel chan_of_parity(off) at k, and -q at
// k' = off ? H - 1 - k : (H - k) mod H; parity classes without a channel are 0.
// Output [field][q3][q2][q1] complex (x fastest), one thread per subgrid point.
template <typename T>
__global__ void k_unpack_g0(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ WT,
                            typename Cx<T>::type* __restrict__ G0, int nfields) {
  using C = typename Cx<T>::type;
  const long mvol = static_cast<long>(g->M[0]) * g->M[1] * g->M[2];
  const long q = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (q >= mvol) return;
  const int slot = blockIdx.y;
  const int qv[3] = {static_cast<int>(q % g->M[0]), static_cast<int>((q / g->M[0]) % g->M[1]),
                     static_cast<int>(q / (static_cast<long>(g->M[0]) * g->M[1]))};
  const int H0 = g->H[0], H1 = g->H[1], H2 = g->H[2];
  const long hv = static_cast<long>(H0) * H1 * H2;
  int c = 0, k[3], km[3];
  if (g->centered) {
    c = g->chan_of_parity[(qv[0] & 1) + 2 * (qv[1] & 1) + 4 * (qv[2] & 1)];
    const int Hd[3] = {H0, H1, H2};
    for (int d = 0; d < 3; ++d) {
      k[d] = qv[d] >> 1;
      km[d] = (qv[d] & 1) ? Hd[d] - 1 - k[d] : (Hd[d] - k[d]) % Hd[d];
    }
  } else {
    const int Md[3] = {g->M[0], g->M[1], g->M[2]};
    for (int d = 0; d < 3; ++d) {
      k[d] = qv[d];
      km[d] = (Md[d] - qv[d]) % Md[d];
    }
  }
  C ga = mk<C>(static_cast<T>(0), static_cast<T>(0)), gb = ga;
  if (c >= 0) {
    const C* w = WT + (static_cast<long>(slot) * g->n_ch + c) * hv;
    const C x = w[(static_cast<long>(k[0]) * H1 + k[1]) * H2 + k[2]];
    const C xm = w[(static_cast<long>(km[0]) * H1 + km[1]) * H2 + km[2]];
    const T h = static_cast<T>(0.5);
    ga = mk<C>(h * (x.x + xm.x), h * (x.y - xm.y));
    gb = mk<C>(h * (x.y + xm.y), h * (xm.x - x.x));
  }
  G0[(2L * slot) * mvol + q] = ga;
  if (2 * slot + 1 < nfields) G0[(2L * slot + 1) * mvol + q] = gb;
}

// Per-block FFT of the legacy block plan (plan_cfft + mul!/ldiv!, src/cfft_plan.jl,
// src/execution.jl): blocks are concatenated, each column-major (x fastest) with
// dims[b] = (n1, n2, n3).  One pass transforms one axis of every block; a CTA takes one
// work item (block b, first line l0, cnt lines along the axis), stages the lines in
// shared memory, builds the n twiddles e^{-2 pi i m / n} once, and runs the mixed-radix
// Stockham passes (radices 8, 4, 2, 3, 5) of fft_lines; a length with another prime
// factor is transformed as a DFT from the same twiddle table (index j k mod n exact).
// y(k) = sum_j x(j) e^{-+2 pi i j k / n}; the inverse's 1/n is k_block_scale.
template <typename T>
__global__ void k_block_fft_axis(const int32_t* __restrict__ dims, const long long* __restrict__ off,
                                 const int4* __restrict__ items, const typename Cx<T>::type* __restrict__ src,
                                 typename Cx<T>::type* __restrict__ dst, int axis, int inverse) {
  using C = typename Cx<T>::type;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int4 it = items[blockIdx.x];
  const int b = it.x, l0 = it.y, cnt = it.z;
  const int n0 = dims[3 * b], n1 = dims[3 * b + 1];
  const int n = dims[3 * b + axis];
  C* bufa = reinterpret_cast<C*>(smem_raw);
  C* bufb = bufa + static_cast<size_t>(cnt) * n;
  C* tw = bufb + static_cast<size_t>(cnt) * n;
  const int tid = threadIdx.x, nth = blockDim.x;
  // line l of the block along `axis`: base offset and element stride
  auto line_base = [&](int l, long long* stride) -> long long {
    if (axis == 0) { *stride = 1; return off[b] + static_cast<long long>(l) * n0; }
    if (axis == 1) {
      *stride = n0;
      const int c0 = l % n0, c2 = l / n0;
      return off[b] + c0 + static_cast<long long>(c2) * n0 * n1;
    }
    *stride = static_cast<long long>(n0) * n1;
    return off[b] + l;
  };
  for (int m = tid; m < n; m += nth) {
    T sv, cv;
    if constexpr (sizeof(T) == 8) sincospi(-2.0 * m / n, &sv, &cv);
    else sincospif(-2.0f * m / n, &sv, &cv);
    tw[m] = mk<C>(cv, sv);
  }
  for (int e = tid; e < cnt * n; e += nth) {
    const int l = e / n, j = e % n;
    long long st;
    const long long base = line_base(l0 + l, &st);
    bufa[e] = src[base + j * st];
  }
  __syncthreads();
  int radix[24], nf = 0, r = n;
  while (r > 1 && nf < 24) {
    int f = 0;
    if (r % 8 == 0) f = 8; else if (r % 4 == 0) f = 4; else if (r % 2 == 0) f = 2;
    else if (r % 3 == 0) f = 3; else if (r % 5 == 0) f = 5;
    if (!f) break;
    radix[nf++] = f;
    r /= f;
  }
  const C* res;
  if (r == 1) {
    res = inverse ? fft_lines<C, true>(bufa, bufb, n, nf, radix, cnt, cnt, 0, n, 1, tw, tid, nth)
                  : fft_lines<C, false>(bufa, bufb, n, nf, radix, cnt, cnt, 0, n, 1, tw, tid, nth);
  } else {
    for (int e = tid; e < cnt * n; e += nth) {
      const int l = e / n, k = e % n;
      const C* x = bufa + static_cast<size_t>(l) * n;
      C acc = mk<C>(static_cast<T>(0), static_cast<T>(0));
      for (int j = 0; j < n; ++j) {
        const C w = tw[static_cast<int>((static_cast<long long>(j) * k) % n)];
        acc = cadd(acc, inverse ? cmulc(x[j], w) : cmul(x[j], w));
      }
      bufb[e] = acc;
    }
    __syncthreads();
    res = bufb;
  }
  for (int e = tid; e < cnt * n; e += nth) {
    const int l = e / n, j = e % n;
    long long st;
    const long long base = line_base(l0 + l, &st);
    dst[base + j * st] = res[e];
  }
}

// Inverse normalisation of the block plan: each block's elements times 1/(n1 n2 n3).
template <typename T>
__global__ void k_block_scale(const int32_t* __restrict__ dims, const long long* __restrict__ off, int n_blocks,
                              typename Cx<T>::type* __restrict__ x) {
  const long long total = off[n_blocks];
  for (long long e = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; e < total;
       e += static_cast<long long>(gridDim.x) * blockDim.x) {
    int lo = 0, hi = n_blocks - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (off[mid] <= e) lo = mid; else hi = mid - 1;
    }
    const T inv = static_cast<T>(1.0 / (static_cast<double>(dims[3 * lo]) * dims[3 * lo + 1] * dims[3 * lo + 2]));
    x[e] = cscale(x[e], inv);
  }
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

// Units of the fused z FFT + diagonal-sign gather (stage 6): in each channel, every
// channel row y is paired with its mirror y' = (M - p1) >> ls (p1 = 2 y + the channel's
// y parity when centred, p1 = y otherwise); self-mirrored rows are paired with each
// other.  Every spectral point joins the unit holding its row, so all eight taps of the
// point lie in that unit's two rows.  Units are ordered by point count, largest first.
// Leaves the fusion off (plan unchanged) when a point falls in a parity class without
// a channel or CFFT_ZRECON=0.
Status build_zrecon_units(Plan* p, std::string* err) {
  if (const char* e = std::getenv("CFFT_ZRECON")) if (e[0] == '0') return Status::kOk;
  const PlanTables& T = p->T;
  const int H = p->fast_h, nch = T.n_ch;
  const int M = T.M[0];
  const int ls = T.centered ? 1 : 0;
  if (M != (T.centered ? 2 * H : H) || H > 255 || nch > 255) return Status::kOk;
  struct Unit { int c, ya, yb; std::vector<uint32_t> pts; };
  std::vector<Unit> units;
  std::vector<int> unit_of_row(static_cast<size_t>(nch) * H, -1);
  for (int c = 0; c < nch; ++c) {
    int ypar = 0;
    if (T.centered) {
      int o = -1;
      for (int k = 0; k < 8; ++k)
        if (T.chan_of_parity[k] == c) { o = k; break; }
      if (o < 0) return Status::kOk;
      ypar = (o >> 1) & 1;
    }
    std::vector<int> singles;
    for (int y = 0; y < H; ++y) {
      if (unit_of_row[static_cast<size_t>(c) * H + y] >= 0) continue;
      const int p1 = T.centered ? 2 * y + ypar : y;
      const int y2 = (p1 ? M - p1 : 0) >> ls;
      if (y2 == y) { singles.push_back(y); continue; }
      units.push_back({c, y, y2, {}});
      unit_of_row[static_cast<size_t>(c) * H + y] = unit_of_row[static_cast<size_t>(c) * H + y2] =
          static_cast<int>(units.size()) - 1;
    }
    for (size_t i = 0; i < singles.size(); i += 2) {
      const int yb = i + 1 < singles.size() ? singles[i + 1] : -1;
      units.push_back({c, singles[i], yb, {}});
      unit_of_row[static_cast<size_t>(c) * H + singles[i]] = static_cast<int>(units.size()) - 1;
      if (yb >= 0) unit_of_row[static_cast<size_t>(c) * H + yb] = static_cast<int>(units.size()) - 1;
    }
  }
  for (size_t sidx = 0; sidx < T.spec.size(); ++sidx) {
    int pp[3];
    for (int d = 0; d < 3; ++d) pp[d] = static_cast<int>(floor_mod(T.spec[sidx].h[d], M));
    const int c = T.centered ? T.chan_of_parity[(pp[0] & 1) + 2 * (pp[1] & 1) + 4 * (pp[2] & 1)] : 0;
    if (c < 0) return Status::kOk;
    const int u = unit_of_row[static_cast<size_t>(c) * H + (pp[1] >> ls)];
    if (u < 0) { *err = "fused gather: spectral point outside the unit rows"; return Status::kInvalid; }
    units[u].pts.push_back(static_cast<uint32_t>(sidx));
  }
  std::stable_sort(units.begin(), units.end(), [](const Unit& a, const Unit& b) { return a.pts.size() > b.pts.size(); });
  std::vector<uint4> ut;
  std::vector<uint32_t> pts;
  for (const Unit& u : units) {
    if (u.pts.empty()) continue;
    ut.push_back(make_uint4(static_cast<uint32_t>(u.c) | (static_cast<uint32_t>(u.ya) << 8) |
                                (static_cast<uint32_t>(u.yb + 1) << 16),
                            static_cast<uint32_t>(pts.size()), static_cast<uint32_t>(u.pts.size()), 0u));
    pts.insert(pts.end(), u.pts.begin(), u.pts.end());
  }
  if (ut.empty()) return Status::kOk;
  // Plan-owned device tables: counted in the plan's device bytes, allocation failures
  // reported as such (like the other plan buffers).
  for (auto [ptr, bytes, what] : {std::tuple<void**, size_t, const char*>{&p->d_zr_units, ut.size() * sizeof(uint4), "fused gather units"},
                                  std::tuple<void**, size_t, const char*>{&p->d_zr_pts, pts.size() * 4, "fused gather points"}}) {
    const cudaError_t e = cudaMalloc(ptr, bytes);
    if (e != cudaSuccess) { *err = cuda_msg(e, what); return Status::kAlloc; }
    p->workspace_bytes += bytes;
  }
  CFFT_CUDA(cudaMemcpy(p->d_zr_units, ut.data(), ut.size() * sizeof(uint4), cudaMemcpyHostToDevice), "upload units");
  CFFT_CUDA(cudaMemcpy(p->d_zr_pts, pts.data(), pts.size() * 4, cudaMemcpyHostToDevice), "upload unit points");
  p->zr_units = static_cast<int>(ut.size());
  p->zrecon = true;
  return Status::kOk;
}

// Stages of one forward + backward: 0 plane/fold + x/y FFT, 1 z FFT, 2 reconstruct,
// 3 inverse reconstruct (+ orbit expansion), 4 inverse z FFT, 5 inverse x/y FFT + unfold.
// `nb` fields starting at the caller's pointers; the workspace holds one chunk.
template <typename T>
Status launch_stage(Plan* p, int stage, const T* f0, typename Cx<T>::type* F, const typename Cx<T>::type* Fin,
                    T* f0_out, const T* E, bool use_K, int nb, cudaStream_t st, std::string* err, int lane = 0,
                    bool q_step = false) {
  using C = typename Cx<T>::type;
  const DevGeom* g = static_cast<const DevGeom*>(p->d_geom);
  const C* tab = static_cast<const C*>(p->d_tables);
  C* W = reinterpret_cast<C*>(static_cast<char*>(p->d_work_T) + lane * p->w_lane_bytes);
  const PlanTables& T_ = p->T;
  if (p->fast_h > 0) {
    if (p->cluster && (stage == 1 || stage == 4)) return Status::kOk;  // fused into stages 0 and 5
    FastArgs a;
    a.geom = p->d_geom; a.tables = p->d_tables; a.spec_h = p->d_spec_h; a.K = p->d_K;
    a.inv_spec = p->d_inv_spec; a.inv_phase = p->d_inv_phase; a.inv_pk = p->d_inv_pk; a.expand = p->d_expand;
    a.W = W;
    a.G0R = p->d_g0r ? static_cast<char*>(p->d_g0r) + lane * p->g0r_lane_bytes : nullptr;
    a.FT = p->d_ft ? static_cast<char*>(p->d_ft) + lane * p->ft_lane_bytes : nullptr;
    a.f0 = f0; a.F = F; a.Fin = Fin; a.f0_out = f0_out; a.E = E;
    a.stage = stage; a.nb = nb; a.H = p->fast_h; a.n_ch = T_.n_ch; a.centered = T_.centered ? 1 : 0;
    a.cent_type = p->cent_type; a.d = T_.d;
    a.n_spec = static_cast<int>(T_.spec.size()); a.n_orbits = static_cast<int>(T_.orbit_rep.size());
    a.use_K = use_K; a.rep_diag8 = p->rep_diag8; a.rep_perm = p->rep_perm; a.reps_quad = p->reps_quad;
    a.reps_wide = p->reps_wide && !p->cluster;
    a.zr_units = p->d_zr_units; a.zr_pts = p->d_zr_pts; a.zr_n_units = p->zr_units;
    a.cluster = p->cluster;
    a.cluster_ctas = p->cluster_ctas;
    a.status = p->d_status;
    a.timeout_ns = p->timeout_ns;
    a.zr_slots = p->tune.zr_slots;
    a.tma = p->tune.tma;
    if (q_step) {  // stage 4: Q-multiply + inverse z FFT into the Q workspace; stage 5 reads it
      a.q_step = true;
      a.QT = p->d_qt;
      a.GT = p->d_gt;
      a.qsep = p->qsep;
      a.QS = p->d_qsep;
      C* WQ = reinterpret_cast<C*>(static_cast<char*>(p->d_work_Q) + lane * p->w_lane_bytes);
      if (stage == 4) a.W2 = WQ;
      else if (stage == 5) a.W = WQ;
    }
    a.stream = st;
    const bool planes = stage == 0 || stage == 5;
    Status s = sizeof(T) == 4 ? (planes ? fast_planes_f32(a, err) : fast_other_f32(a, err))
                              : (planes ? fast_planes_f64(a, err) : fast_other_f64(a, err));
    g_launches += (stage == 3 && p->reps_quad && !q_step) ? 2 : 1;  // regroup + gather
    return s;
  }
  switch (stage) {
    case 0:
      if (E) k_plane_fwd<T, true><<<dim3(T_.H[2], nb), p->threads_xy, p->smem_xy, st>>>(g, tab, f0, E, W);
      else k_plane_fwd<T, false><<<dim3(T_.H[2], nb), p->threads_xy, p->smem_xy, st>>>(g, tab, f0, nullptr, W);
      break;
    case 1:
      if (T_.H[2] <= 1) return Status::kOk;
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
      if (T_.H[2] <= 1) return Status::kOk;
      k_fft_z<T, true><<<dim3(T_.H[1], T_.n_ch, nb), p->threads_z, p->smem_z, st>>>(g, tab, W);
      break;
    default:
      if (E) k_plane_bwd<T, true><<<dim3(T_.H[2], nb), p->threads_xy, p->smem_xy, st>>>(g, tab, W, E, f0_out);
      else k_plane_bwd<T, false><<<dim3(T_.H[2], nb), p->threads_xy, p->smem_xy, st>>>(g, tab, W, nullptr, f0_out);
      break;
  }
  ++g_launches;
  return Status::kOk;
}

// Forward and/or backward over B fields in workspace-sized chunks.  F holds the
// spectra of all B fields (the forward output, the backward input).
template <typename T>
Status run_chunks(Plan* p, bool fwd, bool bwd, const T* f0, typename Cx<T>::type* F, T* f0_out, const T* E,
                  bool use_K, int B, cudaStream_t st, std::string* err) {
  const size_t mvol = static_cast<size_t>(p->T.M[0]) * p->T.M[1] * p->T.M[2];
  const size_t ns = p->T.spec.size();
  const int nchunks = (B + p->chunk - 1) / p->chunk;
  const int lanes = std::min(p->lanes, nchunks);
  // Two or more chunks run concurrently on the plan's lane streams (fork/join with
  // events on the caller's stream), each lane with its own workspace.
  if (lanes > 1) {
    CFFT_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(p->ev_fork), st), "fork event");
    for (int l = 0; l < lanes; ++l)
      CFFT_CUDA(cudaStreamWaitEvent(static_cast<cudaStream_t>(p->lane_stream[l]), static_cast<cudaEvent_t>(p->ev_fork), 0), "fork wait");
  }
  for (int i = 0; i < nchunks; ++i) {
    const int b0 = i * p->chunk;
    const int nb = std::min(p->chunk, B - b0);
    const int lane = lanes > 1 ? i % lanes : 0;
    cudaStream_t ls = lanes > 1 ? static_cast<cudaStream_t>(p->lane_stream[lane]) : st;
    const T* fin = f0 ? f0 + b0 * mvol : nullptr;
    T* fout = f0_out ? f0_out + b0 * mvol : nullptr;
    const T* Ec = E ? E + b0 * mvol : nullptr;
    auto* Fc = F + b0 * ns;
    if (fwd && bwd && use_K && p->qmode) {
      // Q-matrix diffusion step: forward transform to G0, Q-multiply + inverse z FFT,
      // inverse x/y FFT + unfold (no spectral-ASU round trip).
      for (int s : {0, 1, 4, 5}) {
        Status r = launch_stage<T>(p, s, fin, Fc, Fc, fout, Ec, false, nb, ls, err, lane, true);
        if (r != Status::kOk) return r;
      }
      continue;
    }
    if (fwd)
      for (int s : {0, 1, 2}) {
        if (p->zrecon && s == 1) continue;  // stage 6 = z FFT + gather
        Status r = launch_stage<T>(p, p->zrecon && s == 2 ? 6 : s, fin, Fc, nullptr, nullptr, Ec, use_K, nb, ls, err, lane);
        if (r != Status::kOk) return r;
      }
    if (bwd)
      for (int s = 3; s < 6; ++s) {
        Status r = launch_stage<T>(p, s, nullptr, nullptr, Fc, fout, Ec, false, nb, ls, err, lane);
        if (r != Status::kOk) return r;
      }
  }
  if (lanes > 1) {
    for (int l = 0; l < lanes; ++l) {
      CFFT_CUDA(cudaEventRecord(static_cast<cudaEvent_t>(p->ev_join[l]), static_cast<cudaStream_t>(p->lane_stream[l])), "join event");
      CFFT_CUDA(cudaStreamWaitEvent(st, static_cast<cudaEvent_t>(p->ev_join[l]), 0), "join wait");
    }
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
      // With the fused stage 6 the z FFT and the gather are one launch, timed as stage 1.
      if (!(p->zrecon && s == 2)) {
        Status r = launch_stage<T>(p, p->zrecon && s == 1 ? 6 : s, f0 + b0 * mvol, F + b0 * ns, F + b0 * ns,
                                   f0_out + b0 * mvol, nullptr, false, nb, st, err);
        if (r != Status::kOk) return r;
      }
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
  if (p->h_status && *static_cast<volatile int*>(p->h_status) != 0) {
    *err = "a bounded device wait of an earlier call on this plan gave up (cfft_plan_device_status clears it)";
    return Status::kTimeout;
  }
  return Status::kOk;
}

}  // namespace

void add_launches(int64_t n) { g_launches += n; }

Status exec_contour_step(Plan* p, const void* in, void* out, const void* E, int B, void* stream, std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  if (!in || !out || !E || in == out) { *err = "invalid argument"; return Status::kInvalid; }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (p->precision == 8)
    return run_chunks<double>(p, true, true, static_cast<const double*>(in), static_cast<double2*>(p->d_work_F),
                              static_cast<double*>(out), static_cast<const double*>(E), true, B, s, err);
  return run_chunks<float>(p, true, true, static_cast<const float*>(in), static_cast<float2*>(p->d_work_F),
                           static_cast<float*>(out), static_cast<const float*>(E), true, B, s, err);
}

int64_t launch_count(bool reset) {
  const int64_t v = g_launches;
  if (reset) g_launches = 0;
  return v;
}

// M-grid column-major index of channel point (c, x, y, z) of the channel grid.
static long q_of_channel_point(const PlanTables& T, int c, int x, int y, int z) {
  if (!T.centered) return x + static_cast<long>(T.M[0]) * (y + static_cast<long>(T.M[1]) * z);
  const auto& o = T.offsets[c];
  return (2 * x + o[0]) + static_cast<long>(T.M[0]) * ((2 * y + o[1]) + static_cast<long>(T.M[1]) * (2 * z + o[2]));
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
  // Compile-time centring type of the plane kernels (plain path: 0).
  p->cent_type = !T.centered ? 0 : T.centering == kCentI ? 1 : T.centering == kCentF ? 2 : T.centering == kCentC ? 3 : 4;
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
  p->fast_h = (cubic && fast_size_ok(T.H[0], p->precision)) ? T.H[0] : 0;
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
  if (p->tune.chunk_bytes > 0) budget = static_cast<size_t>(p->tune.chunk_bytes);
  const size_t per_field = T.n_ch * hvol * cs / (p->fast_h ? 2 : 1);
  size_t ch = std::max<size_t>(1, std::min<size_t>(B, budget / std::max<size_t>(per_field, 1)));
  // Batches of at least 8 fields on the fast path run as two concurrent lanes.
  p->lanes = 1;
  if (p->tune.lanes > 0) p->lanes = std::min(Plan::kMaxLanes, p->tune.lanes);
  else if (const char* ln = std::getenv("CFFT_LANES")) p->lanes = std::max(1, std::min(Plan::kMaxLanes, std::atoi(ln)));
  else if (p->fast_h && B >= 8) p->lanes = 2;
  if (p->lanes > 1) ch = std::min(ch, (B + p->lanes - 1) / p->lanes);
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
  p->w_lane_bytes = ((chunk * T.n_ch * hvol * cs + 255) / 256) * 256;
  if ((st = alloc(&p->d_work_T, p->lanes * p->w_lane_bytes, "channel workspace")) != Status::kOk) return st;
  if ((st = alloc(&p->d_work_F, B * T.spec.size() * cs, "spectrum workspace")) != Status::kOk) return st;
  if ((st = alloc(&p->d_work_E, B * mvol * rs, "interaction workspace")) != Status::kOk) return st;
  // Packed alias rows (spec+1 in 20 bits, conj, phase in 11 bits) for the quad gather.
  std::vector<uint32_t> inv_pk;
  p->reps_quad = p->fast_h && T.spec.size() < (1u << 20) - 1 && T.P <= 2048 && T.orbit_rep.size() < (1u << 21);
  if (p->reps_quad) {
    inv_pk.resize(T.inv_spec.size());
    for (size_t k = 0; k < inv_pk.size(); ++k) {
      const int sp = T.inv_spec[k];
      const uint32_t a = static_cast<uint32_t>(sp < 0 ? -sp : sp);
      inv_pk[k] = a | (sp < 0 ? (1u << 20) : 0u) | (static_cast<uint32_t>(T.inv_phase[k]) << 21);
    }
    if ((st = alloc(&p->d_inv_pk, inv_pk.size() * 4, "packed inverse table")) != Status::kOk) return st;
  }
  if (p->fast_h) {
    // The quad path reads the expansion entries packed in 32 bits (orbit | phase << 21).
    if ((st = alloc(&p->d_expand, expand.size() * (p->reps_quad ? 4 : sizeof(int2)), "expansion table")) != Status::kOk)
      return st;
    // Wide groups (16 FP32 / 8 FP64 fields per line) once a chunk fills one group; the
    // fused cluster kernels read the quad layout, so CFFT_CLUSTER keeps quads.
    const size_t gw = 128 / cs;
    const char* wide_env = std::getenv("CFFT_WIDE");
    const char* cl_env = std::getenv("CFFT_CLUSTER");
    const bool cluster_wanted = p->tune.cluster >= 0 ? p->tune.cluster > 0 : (cl_env && std::atoi(cl_env) > 0);
    const bool wide_wanted = p->tune.wide >= 0 ? p->tune.wide > 0 : !(wide_env && wide_env[0] == '0');
    p->reps_wide = p->reps_quad && chunk >= gw && wide_wanted && !cluster_wanted;
    const size_t chunk4 = p->reps_wide ? (chunk + gw - 1) / gw * gw : (chunk + 3) / 4 * 4;  // whole groups of fields
    p->g0r_lane_bytes = (((p->reps_quad ? chunk4 : chunk + 1) * T.orbit_rep.size() * cs + 255) / 256) * 256;
    if ((st = alloc(&p->d_g0r, p->lanes * p->g0r_lane_bytes, "representative workspace")) != Status::kOk) return st;
    if (p->reps_quad) {
      p->ft_lane_bytes = ((chunk4 * T.spec.size() * cs + 255) / 256) * 256;
      if ((st = alloc(&p->d_ft, p->lanes * p->ft_lane_bytes, "grouped spectra")) != Status::kOk) return st;
    }
  }
  // Q-matrix step (M2Q / M7): runs on the compile-time sized kernels only.
  if (p->qmode) {
    if (!p->fast_h) {
      *err = "the Q-matrix step needs a cubic channel grid of edge 4, 6, 8, 12, 16, 24, 32 (or 48 in FP32)";
      return Status::kUnsupported;
    }
    const size_t np = static_cast<size_t>(T.n_ch) * hvol;
    if ((st = alloc(&p->d_work_Q, p->lanes * p->w_lane_bytes, "Q workspace")) != Status::kOk) return st;
    // Separable Q-multiply (_is_pmmm_like, src/q_fused_krfft.jl:431-454): M2Q plan, d = 8,
    // L = (2, 2, 2), diagonal representatives listed in parity-class order with
    // translations 0 or N - 1, and an orthogonal cell (K factorises per axis).
    {
      bool sep = p->qmode == 3 && !T.centered && T.n_ch == 1 && T.d == 8 && p->fast_h == T.M[0] &&
                 T.M[0] == T.M[1] && T.M[1] == T.M[2] && T.L[0] == 2 && T.L[1] == 2 && T.L[2] == 2;
      for (int i = 0; i < 3 && sep; ++i)
        for (int j = 0; j < 3; ++j)
          if (i != j && std::fabs(p->lattice[3 * j + i]) > 1e-12 * std::fabs(p->lattice[4 * i])) sep = false;
      for (int a = 0; a < 8 && sep; ++a)
        for (int d = 0; d < 3 && sep; ++d) {
          for (int e = 0; e < 3; ++e)
            if (e != d && T.rep_ops[a].R[d][e] != 0) sep = false;
          const long tm = floor_mod(T.rep_ops[a].t[d], T.N[d]);
          if (tm != 0 && tm != T.N[d] - 1) sep = false;
          if ((tm != 0) != (((a >> d) & 1) != 0)) sep = false;
        }
      const char* qe = std::getenv("CFFT_QSEP");
      p->qsep = sep && !(qe && qe[0] == '0');
    }
    if (p->qsep) {
      if ((st = alloc(&p->d_qsep, static_cast<size_t>(9) * T.M[0] * cs, "separable Q factors")) != Status::kOk) return st;
    } else {
      if ((st = alloc(&p->d_qt, T.d * np * cs, "Q coefficients")) != Status::kOk) return st;
      if ((st = alloc(&p->d_gt, T.d * np * 4, "Q gather")) != Status::kOk) return st;
    }
    // Gather targets as indices into the z-fastest forward workspace WT[c][x][y][z].
    const int H = T.H[0];
    const long Mvol = static_cast<long>(T.M[0]) * T.M[1] * T.M[2];
    std::vector<int32_t> gt(static_cast<size_t>(T.d) * np);
    for (int b = 0; b < T.d; ++b)
      for (int c = 0; c < T.n_ch; ++c)
        for (int z = 0; z < H; ++z)
          for (int y = 0; y < H; ++y)
            for (int x = 0; x < H; ++x) {
              const size_t pos = ((static_cast<size_t>(c) * H + z) * H + y) * H + x;
              const long gq = p->q_gather[b * Mvol + q_of_channel_point(T, c, x, y, z)];
              const int gv[3] = {static_cast<int>(gq % T.M[0]), static_cast<int>((gq / T.M[0]) % T.M[1]),
                                 static_cast<int>(gq / (static_cast<long>(T.M[0]) * T.M[1]))};
              int cc = 0, k[3] = {gv[0], gv[1], gv[2]};
              if (T.centered) {
                cc = T.chan_of_parity[(gv[0] & 1) + 2 * (gv[1] & 1) + 4 * (gv[2] & 1)];
                for (int dd = 0; dd < 3; ++dd) k[dd] = gv[dd] >> 1;
              }
              gt[b * np + pos] = cc < 0 ? -1 : static_cast<int32_t>(cc * hvol + (static_cast<size_t>(k[0]) * H + k[1]) * H + k[2]);
            }
    if (p->d_gt) CFFT_CUDA(cudaMemcpy(p->d_gt, gt.data(), gt.size() * 4, cudaMemcpyHostToDevice), "upload Q gather");
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
  if (p->fast_h && p->reps_quad) {
    std::vector<uint32_t> epk(expand.size());
    for (size_t i = 0; i < expand.size(); ++i)
      epk[i] = static_cast<uint32_t>(expand[i].x) | (static_cast<uint32_t>(expand[i].y) << 21);
    CFFT_CUDA(cudaMemcpy(p->d_expand, epk.data(), epk.size() * 4, cudaMemcpyHostToDevice), "upload expansion");
  } else if (p->fast_h) {
    CFFT_CUDA(cudaMemcpy(p->d_expand, expand.data(), expand.size() * sizeof(int2), cudaMemcpyHostToDevice), "upload expansion");
  }
  if (p->reps_quad)
    CFFT_CUDA(cudaMemcpy(p->d_inv_pk, inv_pk.data(), inv_pk.size() * 4, cudaMemcpyHostToDevice), "upload packed table");
  if (p->fast_h && p->rep_diag8 && !p->qmode) {
    Status zs = build_zrecon_units(p, err);
    if (zs != Status::kOk) return zs;
  }
  // Orbit expansion writes only alive positions; channel positions never written stay zero.
  CFFT_CUDA(cudaMemset(p->d_work_T, 0, p->lanes * p->w_lane_bytes), "clear workspace");
  if (p->precision == 8) set_smem_attrs<double>();
  else set_smem_attrs<float>();
  CFFT_CUDA(cudaGetLastError(), "set shared-memory attributes");
  if (p->fast_h) {
    if (p->precision == 8) {
      if ((st = fast_init_planes_f64(err)) != Status::kOk) return st;
      if ((st = fast_init_other_f64(err)) != Status::kOk) return st;
    } else {
      if ((st = fast_init_planes_f32(err)) != Status::kOk) return st;
      if ((st = fast_init_other_f32(err)) != Status::kOk) return st;
    }
    // Fused cluster kernels (CFFT_CLUSTER = 8 or 16 CTAs per cluster) when the slot's
    // channel volume fits the CTAs of one cluster and at least one cluster can be
    // resident.  Off by default: on B200 at H = 32 the separate plane and z kernels are
    // faster (1.66 vs 1.90 / 2.07 us per Im-3m 128^3 field), because one slot per SM
    // group serialises the load, transform and exchange phases.
    const char* ce = std::getenv("CFFT_CLUSTER");
    const int want = p->tune.cluster >= 0 ? p->tune.cluster : (ce ? std::atoi(ce) : 0);
    p->cluster_ctas = want == 16 ? 16 : 8;
    p->cluster = want != 0 && !p->qmode && p->reps_quad && fast_cluster_fits(p->fast_h, T.n_ch, p->precision);
    if (p->cluster) {
      int mc = 0;
      st = p->precision == 8 ? fast_cluster_probe_f64(p->fast_h, p->cent_type, p->cluster_ctas, &mc, err)
                             : fast_cluster_probe_f32(p->fast_h, p->cent_type, p->cluster_ctas, &mc, err);
      if (st != Status::kOk) return st;
      if (mc < 1 && p->cluster_ctas == 16) {  // the device does not take 16-CTA clusters here
        p->cluster_ctas = 8;
        st = p->precision == 8 ? fast_cluster_probe_f64(p->fast_h, p->cent_type, 8, &mc, err)
                               : fast_cluster_probe_f32(p->fast_h, p->cent_type, 8, &mc, err);
        if (st != Status::kOk) return st;
      }
      p->cluster = mc >= 1;
    }
  }
  if (p->cluster) p->zrecon = false;  // the cluster forward writes the z-fastest workspace for stage 2
  {
    void* hs = nullptr;
    CFFT_CUDA(cudaHostAlloc(&hs, sizeof(int), cudaHostAllocMapped), "status word");
    p->h_status = static_cast<int*>(hs);
    *p->h_status = 0;
    void* ds = nullptr;
    CFFT_CUDA(cudaHostGetDevicePointer(&ds, hs, 0), "status word device address");
    p->d_status = static_cast<int*>(ds);
    if (const char* e = std::getenv("CFFT_WAIT_TIMEOUT_NS")) p->timeout_ns = std::strtoull(e, nullptr, 10);
  }
  cudaStream_t s;
  CFFT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "create stream");
  p->own_stream = s;
  if (p->lanes > 1) {
    cudaEvent_t e;
    CFFT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "create event");
    p->ev_fork = e;
    for (int l = 0; l < p->lanes; ++l) {
      cudaStream_t ls;
      CFFT_CUDA(cudaStreamCreateWithFlags(&ls, cudaStreamNonBlocking), "create lane stream");
      p->lane_stream[l] = ls;
      CFFT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "create event");
      p->ev_join[l] = e;
    }
  }
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
  if (p->qsep && p->d_qsep) {
    // 1-D twiddles e^{2 pi i q / N_d} (q < M) and kernel factors exp(-ds (2 pi h_c / a_d)^2)
    // (h < N_d, h_c = h - N_d for h >= N_d / 2) of the separable Q-multiply.
    const PlanTables& T = p->T;
    const int Mq = T.M[0];
    std::vector<double> qs(static_cast<size_t>(9) * Mq * 2, 0.0);
    for (int d = 0; d < 3; ++d) {
      for (int q = 0; q < Mq; ++q) {
        qs[(d * Mq + q) * 2] = std::cos(2.0 * M_PI * q / T.N[d]);
        qs[(d * Mq + q) * 2 + 1] = std::sin(2.0 * M_PI * q / T.N[d]);
      }
      const double ad = p->lattice[4 * d];
      for (int h = 0; h < T.N[d]; ++h) {
        const int hc = h >= T.N[d] / 2 ? h - T.N[d] : h;
        const double kk = 2.0 * M_PI * hc / ad;
        qs[(3 * Mq + d * T.N[d] + h) * 2] = std::exp(-p->ds * kk * kk);
      }
    }
    if (p->precision == 8) {
      CFFT_CUDA(cudaMemcpy(p->d_qsep, qs.data(), qs.size() * 8, cudaMemcpyHostToDevice), "upload separable Q");
    } else {
      std::vector<float> qf(qs.begin(), qs.end());
      CFFT_CUDA(cudaMemcpy(p->d_qsep, qf.data(), qf.size() * 4, cudaMemcpyHostToDevice), "upload separable Q");
    }
  }
  if (p->qmode && p->d_qt) {
    // Q first row in the order the Q-multiply kernel walks the channel points: [b][c][z][y][x].
    const PlanTables& T = p->T;
    const int H = T.H[0], d = T.d;
    const long Mvol = static_cast<long>(T.M[0]) * T.M[1] * T.M[2];
    const size_t np = static_cast<size_t>(T.n_ch) * H * H * H;
    std::vector<double> qt(static_cast<size_t>(d) * np * 2);
    for (int b = 0; b < d; ++b)
      for (int c = 0; c < T.n_ch; ++c)
        for (int z = 0; z < H; ++z)
          for (int y = 0; y < H; ++y)
            for (int x = 0; x < H; ++x) {
              const size_t pos = ((static_cast<size_t>(c) * H + z) * H + y) * H + x;
              const long q = q_of_channel_point(T, c, x, y, z);
              qt[(b * np + pos) * 2] = p->q_host[(b * Mvol + q) * 2];
              qt[(b * np + pos) * 2 + 1] = p->q_host[(b * Mvol + q) * 2 + 1];
            }
    if (p->precision == 8) {
      CFFT_CUDA(cudaMemcpy(p->d_qt, qt.data(), qt.size() * 8, cudaMemcpyHostToDevice), "upload Q");
    } else {
      std::vector<float> qf(qt.begin(), qt.end());
      CFFT_CUDA(cudaMemcpy(p->d_qt, qf.data(), qf.size() * 4, cudaMemcpyHostToDevice), "upload Q");
    }
  }
  return Status::kOk;
}

void plan_device_free(Plan* p) {
  void** bufs[] = {&p->d_geom, &p->d_tables, &p->d_spec_h, &p->d_K, &p->d_orbit_rep, &p->d_inv_spec,
                   &p->d_inv_phase, &p->d_img_mask, &p->d_fill_map, &p->d_work_T, &p->d_work_F,
                   &p->d_work_E, &p->d_stage_in, &p->d_stage_out, &p->d_expand, &p->d_g0r, &p->d_inv_pk, &p->d_ft,
                   &p->d_qt, &p->d_gt, &p->d_work_Q, &p->d_zr_units, &p->d_zr_pts, &p->d_qsep};
  for (void** b : bufs)
    if (*b) { cudaFree(*b); *b = nullptr; }
  if (p->h_status) { cudaFreeHost(p->h_status); p->h_status = nullptr; p->d_status = nullptr; }
  for (auto& gph : p->step_graphs) cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(gph.exec));
  p->step_graphs.clear();
  if (p->own_stream) { cudaStreamDestroy(static_cast<cudaStream_t>(p->own_stream)); p->own_stream = nullptr; }
  for (int l = 0; l < Plan::kMaxLanes; ++l) {
    if (p->lane_stream[l]) { cudaStreamDestroy(static_cast<cudaStream_t>(p->lane_stream[l])); p->lane_stream[l] = nullptr; }
    if (p->ev_join[l]) { cudaEventDestroy(static_cast<cudaEvent_t>(p->ev_join[l])); p->ev_join[l] = nullptr; }
  }
  if (p->ev_fork) { cudaEventDestroy(static_cast<cudaEvent_t>(p->ev_fork)); p->ev_fork = nullptr; }
  for (void** sp : {&p->h2d_stream, &p->d2h_stream})
    if (*sp) { cudaStreamDestroy(static_cast<cudaStream_t>(*sp)); *sp = nullptr; }
  for (int i = 0; i < Plan::kHostPieces; ++i)
    for (void** ep : {&p->ev_in[i], &p->ev_done[i]})
      if (*ep) { cudaEventDestroy(static_cast<cudaEvent_t>(*ep)); *ep = nullptr; }
}

Status plan_device_status(Plan* p, bool clear, std::string* err) {
  if (!p->h_status) { *err = "host-only plan: no device state"; return Status::kInvalid; }
  volatile int* hs = p->h_status;
  const int v = *hs;
  if (clear) *hs = 0;
  if (v != 0) { *err = "a bounded device wait gave up"; return Status::kTimeout; }
  return Status::kOk;
}

Status plan_wait_selftest(Plan* p, unsigned long long timeout_ns, void* stream, std::string* err) {
  if (!p->d_status) { *err = "host-only plan: no device state"; return Status::kInvalid; }
  return fast_wait_selftest(timeout_ns, p->d_status, stream, err);
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

// The n_steps contour steps (forward + K + backward with the interaction factors E on
// both sides) on field buffer q.
template <typename T>
Status contour_steps(Plan* p, T* q, int n_steps, int B, cudaStream_t s, std::string* err) {
  using C = typename Cx<T>::type;
  for (int i = 0; i < n_steps; ++i) {
    Status st = run_chunks<T>(p, true, true, q, static_cast<C*>(p->d_work_F), q, static_cast<const T*>(p->d_work_E),
                              true, B, s, err);
    if (st != Status::kOk) return st;
  }
  return Status::kOk;
}

// Contour loops of at least kGraphMinSteps steps run as a CUDA graph: captured on the
// plan's own stream the first time a (q, B, n_steps) combination is seen, then replayed
// on the caller's stream (one launch instead of ~7 per step and chunk).  The graph
// reads only plan-owned buffers besides q, so a new kernel (update_kernel) or new
// interaction factors are picked up on replay.  CFFT_STEP_GRAPH=0 launches directly.
constexpr int kGraphMinSteps = 4;
constexpr size_t kMaxStepGraphs = 8;

template <typename T>
Status step_graph_run(Plan* p, T* q, int n_steps, int B, cudaStream_t s, bool* done, std::string* err) {
  *done = false;
  for (auto& gph : p->step_graphs)
    if (gph.q == q && gph.batch == B && gph.n_steps == n_steps) {
      CFFT_CUDA(cudaGraphLaunch(static_cast<cudaGraphExec_t>(gph.exec), s), "step graph launch");
      gph.last_use = ++p->graph_clock;
      g_launches += gph.kernels;
      *done = true;
      return Status::kOk;
    }
  cudaStream_t cs = static_cast<cudaStream_t>(p->own_stream);
  const int64_t before = g_launches;
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return Status::kOk;  // not capturable here: the caller launches directly
  }
  std::string cerr;
  const Status st = contour_steps<T>(p, q, n_steps, B, cs, &cerr);
  cudaGraph_t graph = nullptr;
  const cudaError_t ee = cudaStreamEndCapture(cs, &graph);
  const int64_t kernels = g_launches - before;
  g_launches = before;  // captured, not launched
  cudaGraphExec_t exec = nullptr;
  if (st != Status::kOk || ee != cudaSuccess || !graph || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    return Status::kOk;  // direct launches instead
  }
  cudaGraphDestroy(graph);
  if (p->step_graphs.size() >= kMaxStepGraphs) {
    auto oldest = std::min_element(p->step_graphs.begin(), p->step_graphs.end(),
                                   [](const Plan::StepGraph& a, const Plan::StepGraph& b) { return a.last_use < b.last_use; });
    cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(oldest->exec));
    p->step_graphs.erase(oldest);
  }
  p->step_graphs.push_back({q, B, n_steps, exec, kernels, ++p->graph_clock});
  CFFT_CUDA(cudaGraphLaunch(exec, s), "step graph launch");
  g_launches += kernels;
  *done = true;
  return Status::kOk;
}

Status exec_step_diffusion(Plan* p, void* q, const void* w, double dt, int n_steps, int B, void* stream,
                           std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  if (!q || !w || n_steps < 0) { *err = "invalid argument"; return Status::kInvalid; }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t n = static_cast<size_t>(B) * p->T.M[0] * p->T.M[1] * p->T.M[2];
  const int grid = static_cast<int>(std::min<size_t>((n + 255) / 256, 148 * 16));
  const char* ge = std::getenv("CFFT_STEP_GRAPH");
  // Inside the caller's own stream capture the steps are recorded as plain launches:
  // a graph cannot be launched into (or captured beside) a capturing stream.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) cudaGetLastError();
  const bool graph = n_steps >= kGraphMinSteps && !(ge && ge[0] == '0') && cap == cudaStreamCaptureStatusNone;
  bool done = false;
  if (p->precision == 8) {
    k_interaction<double><<<grid, 256, 0, s>>>(static_cast<const double*>(w), static_cast<double*>(p->d_work_E), dt / 2, n);
    ++g_launches;
    if (graph && (st = step_graph_run<double>(p, static_cast<double*>(q), n_steps, B, s, &done, err)) != Status::kOk)
      return st;
    if (!done && (st = contour_steps<double>(p, static_cast<double*>(q), n_steps, B, s, err)) != Status::kOk) return st;
  } else {
    k_interaction<float><<<grid, 256, 0, s>>>(static_cast<const float*>(w), static_cast<float*>(p->d_work_E),
                                              static_cast<float>(dt / 2), n);
    ++g_launches;
    if (graph && (st = step_graph_run<float>(p, static_cast<float*>(q), n_steps, B, s, &done, err)) != Status::kOk)
      return st;
    if (!done && (st = contour_steps<float>(p, static_cast<float*>(q), n_steps, B, s, err)) != Status::kOk) return st;
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

// Legacy block plan: device block descriptors and a work buffer of the blocks' size.
Status block_plan_create(int n_blocks, const int32_t* dims, int precision, BlockPlan** out, std::string* err) {
  if (n_blocks < 1 || !dims || !out || (precision != 4 && precision != 8)) { *err = "invalid argument"; return Status::kInvalid; }
  std::vector<long long> off(n_blocks + 1, 0);
  for (int b = 0; b < n_blocks; ++b) {
    for (int d = 0; d < 3; ++d)
      if (dims[3 * b + d] < 1) { *err = "block dimensions must be positive"; return Status::kInvalid; }
    off[b + 1] = off[b] + static_cast<long long>(dims[3 * b]) * dims[3 * b + 1] * dims[3 * b + 2];
  }
  auto* bp = new (std::nothrow) BlockPlan();
  if (!bp) { *err = "host allocation failed"; return Status::kAlloc; }
  bp->n_blocks = n_blocks;
  bp->total = off[n_blocks];
  bp->precision = precision;
  // work items per axis: (block, first line, lines) with lines x length <= kBlockLineElems
  std::vector<int32_t> items;
  for (int a = 0; a < 3; ++a) {
    bp->item_off[a] = static_cast<int>(items.size() / 4);
    for (int b = 0; b < n_blocks; ++b) {
      const int n = dims[3 * b + a];
      if (n > kBlockMaxLen) { *err = "block edge above the supported length"; delete bp; return Status::kUnsupported; }
      const long long vol = static_cast<long long>(dims[3 * b]) * dims[3 * b + 1] * dims[3 * b + 2];
      const int lines = static_cast<int>(vol / n);
      const int per = std::max(1, std::min(lines, kBlockLineElems / n));
      for (int l = 0; l < lines; l += per) {
        items.push_back(b);
        items.push_back(l);
        items.push_back(std::min(per, lines - l));
        items.push_back(0);
      }
    }
    bp->n_items[a] = static_cast<int>(items.size() / 4) - bp->item_off[a];
    for (int b = 0; b < n_blocks; ++b) bp->max_len[a] = std::max(bp->max_len[a], dims[3 * b + a]);
  }
  cudaError_t e = cudaMalloc(&bp->d_dims, sizeof(int32_t) * 3 * n_blocks);
  if (e == cudaSuccess) e = cudaMalloc(&bp->d_off, sizeof(long long) * (n_blocks + 1));
  if (e == cudaSuccess) e = cudaMalloc(&bp->d_work, static_cast<size_t>(bp->total) * 2 * precision);
  if (e == cudaSuccess) e = cudaMalloc(&bp->d_items, sizeof(int32_t) * items.size());
  if (e == cudaSuccess) e = cudaMemcpy(bp->d_dims, dims, sizeof(int32_t) * 3 * n_blocks, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(bp->d_off, off.data(), sizeof(long long) * (n_blocks + 1), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(bp->d_items, items.data(), sizeof(int32_t) * items.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_block_fft_axis<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBlockSmemMax);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_block_fft_axis<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, kBlockSmemMax);
  if (e != cudaSuccess) {
    *err = cuda_msg(e, "block plan");
    block_plan_destroy(bp);
    return Status::kCuda;
  }
  *out = bp;
  return Status::kOk;
}

void block_plan_destroy(BlockPlan* bp) {
  if (!bp) return;
  for (void* q : {bp->d_dims, bp->d_off, bp->d_work, bp->d_items})
    if (q) cudaFree(q);
  delete bp;
}

// mul! (forward, unnormalised) / ldiv! (inverse, 1/n) over every block: x -> out -> work -> out.
template <typename T>
Status block_execute_t(BlockPlan* bp, const void* in, void* out, bool inverse, cudaStream_t s, std::string* err) {
  using C = typename Cx<T>::type;
  const int32_t* dims = static_cast<const int32_t*>(bp->d_dims);
  const long long* off = static_cast<const long long*>(bp->d_off);
  const int4* items = static_cast<const int4*>(bp->d_items);
  const C* src[3] = {static_cast<const C*>(in), static_cast<const C*>(out), static_cast<const C*>(bp->d_work)};
  C* dst[3] = {static_cast<C*>(out), static_cast<C*>(bp->d_work), static_cast<C*>(out)};
  for (int a = 0; a < 3; ++a) {
    if (bp->n_items[a] == 0) continue;
    // shared memory: two line buffers of up to max(kBlockLineElems, n) elements and n twiddles
    const size_t smem = static_cast<size_t>(2 * std::max(kBlockLineElems, bp->max_len[a]) + bp->max_len[a]) * sizeof(C);
    k_block_fft_axis<T><<<bp->n_items[a], 128, smem, s>>>(dims, off, items + bp->item_off[a], src[a], dst[a], a,
                                                         inverse ? 1 : 0);
    ++g_launches;
  }
  if (inverse) {
    const int grid = static_cast<int>(std::min<long long>((bp->total + 255) / 256, 148 * 16));
    k_block_scale<T><<<grid, 256, 0, s>>>(dims, off, bp->n_blocks, static_cast<C*>(out));
    ++g_launches;
  }
  CFFT_CUDA(cudaGetLastError(), "block transform launch");
  return Status::kOk;
}

Status block_execute(BlockPlan* bp, const void* in, void* out, bool inverse, void* stream, std::string* err) {
  if (!bp || !in || !out) { *err = "null argument"; return Status::kInvalid; }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  return bp->precision == 8 ? block_execute_t<double>(bp, in, out, inverse, s, err)
                            : block_execute_t<float>(bp, in, out, inverse, s, err);
}

// Subgrid spectrum G0 = FFT_M(f0) per field (the F000 of execute_staged!, the Y buffer
// of the M2Q path): forward fold + transforms of each chunk, then k_unpack_g0.
Status exec_subgrid_spectrum(Plan* p, const void* f0, void* G0, int B, void* stream, std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  if (!f0 || !G0) { *err = "null pointer"; return Status::kInvalid; }
  if (!p->fast_h) {
    *err = "the subgrid spectrum needs a cubic channel grid of edge 4, 6, 8, 12, 16, 24, 32 (or 48 in FP32)";
    return Status::kUnsupported;
  }
  const PlanTables& T = p->T;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t mvol = static_cast<size_t>(T.M[0]) * T.M[1] * T.M[2];
  const dim3 blk(256);
  for (int b0 = 0; b0 < B; b0 += p->chunk) {
    const int nb = std::min(p->chunk, B - b0);
    const dim3 grid(static_cast<unsigned>((mvol + 255) / 256), static_cast<unsigned>((nb + 1) / 2));
    if (p->precision == 8) {
      const double* fin = static_cast<const double*>(f0) + b0 * mvol;
      for (int stage = 0; stage < 2; ++stage)
        if ((st = launch_stage<double>(p, stage, fin, nullptr, nullptr, nullptr, nullptr, false, nb, s, err)) != Status::kOk)
          return st;
      k_unpack_g0<double><<<grid, blk, 0, s>>>(static_cast<const DevGeom*>(p->d_geom), static_cast<const double2*>(p->d_work_T),
                                               static_cast<double2*>(G0) + b0 * mvol, nb);
    } else {
      const float* fin = static_cast<const float*>(f0) + b0 * mvol;
      for (int stage = 0; stage < 2; ++stage)
        if ((st = launch_stage<float>(p, stage, fin, nullptr, nullptr, nullptr, nullptr, false, nb, s, err)) != Status::kOk)
          return st;
      k_unpack_g0<float><<<grid, blk, 0, s>>>(static_cast<const DevGeom*>(p->d_geom), static_cast<const float2*>(p->d_work_T),
                                              static_cast<float2*>(G0) + b0 * mvol, nb);
    }
    ++g_launches;
  }
  CFFT_CUDA(cudaGetLastError(), "subgrid spectrum launch");
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

// which: 0 forward, 1 backward, 2 scft step (in place on the host buffer `out`).
// The batch is cut into up to kHostPieces pieces of whole fields; piece i is copied in
// on h2d_stream, transformed on own_stream once its copy has landed, and copied out on
// d2h_stream, so the host<->device copies of different pieces (and the transforms)
// overlap.  The call returns when every output byte is in the host buffer.
Status exec_host(Plan* p, int which, const void* in, void* out, int B, std::string* err) {
  Status st = check_batch(p, B, err);
  if (st != Status::kOk) return st;
  const PlanTables& T = p->T;
  const size_t rs = p->precision, cs = 2 * rs;
  const size_t fvol = static_cast<size_t>(T.M[0]) * T.M[1] * T.M[2] * rs;   // bytes per field
  const size_t svol = T.spec.size() * cs;                                    // bytes per spectrum
  const size_t fmax = static_cast<size_t>(p->max_batch) * fvol;
  const size_t smax = static_cast<size_t>(p->max_batch) * svol;
  if (!p->d_stage_in) {
    CFFT_CUDA(cudaMalloc(&p->d_stage_in, std::max(fmax, smax)), "alloc staging");
    CFFT_CUDA(cudaMalloc(&p->d_stage_out, std::max(fmax, smax)), "alloc staging");
    p->workspace_bytes += 2 * std::max(fmax, smax);
  }
  if (!p->h2d_stream) {
    for (void** sp : {&p->h2d_stream, &p->d2h_stream}) {
      cudaStream_t cs_;
      CFFT_CUDA(cudaStreamCreateWithFlags(&cs_, cudaStreamNonBlocking), "create copy stream");
      *sp = cs_;
    }
    for (int i = 0; i < Plan::kHostPieces; ++i)
      for (void** ep : {&p->ev_in[i], &p->ev_done[i]}) {
        cudaEvent_t e;
        CFFT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "create copy event");
        *ep = e;
      }
  }
  cudaStream_t s = static_cast<cudaStream_t>(p->own_stream);
  cudaStream_t sin = static_cast<cudaStream_t>(p->h2d_stream);
  cudaStream_t sout = static_cast<cudaStream_t>(p->d2h_stream);
  const size_t in_per = which == 1 ? svol : fvol, out_per = which == 0 ? svol : fvol;
  // Pieces of at least 2 MiB of input, at most kHostPieces of them.
  const int by_bytes = static_cast<int>(std::max<size_t>(1, in_per * B / (2u << 20)));
  const int want = std::max(1, std::min({Plan::kHostPieces, B, by_bytes}));
  const int pb = (B + want - 1) / want;
  const int pieces = (B + pb - 1) / pb;
  const char* hin = static_cast<const char*>(which == 2 ? out : in);
  char* hout = static_cast<char*>(out);
  char* din = static_cast<char*>(p->d_stage_in);
  char* dout = static_cast<char*>(which == 2 ? p->d_stage_in : p->d_stage_out);
  Status res = Status::kOk;
  for (int i = 0; i < pieces && res == Status::kOk; ++i) {
    const int b0 = i * pb, nb = std::min(pb, B - b0);
    cudaEvent_t ein = static_cast<cudaEvent_t>(p->ev_in[i]), edone = static_cast<cudaEvent_t>(p->ev_done[i]);
    cudaError_t ce = cudaMemcpyAsync(din + b0 * in_per, hin + b0 * in_per, nb * in_per, cudaMemcpyHostToDevice, sin);
    if (ce == cudaSuccess) ce = cudaEventRecord(ein, sin);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(s, ein, 0);
    if (ce != cudaSuccess) {
      *err = std::string("host pipeline H2D: ") + cudaGetErrorString(ce);
      res = Status::kCuda;
      break;
    }
    if (which == 0) res = exec_forward(p, din + b0 * in_per, dout + b0 * out_per, nb, s, err);
    else if (which == 1) res = exec_backward(p, din + b0 * in_per, dout + b0 * out_per, nb, s, err);
    else res = exec_scft_step(p, din + b0 * in_per, nb, s, err);
    if (res != Status::kOk) break;
    ce = cudaEventRecord(edone, s);
    if (ce == cudaSuccess) ce = cudaStreamWaitEvent(sout, edone, 0);
    if (ce == cudaSuccess)
      ce = cudaMemcpyAsync(hout + b0 * out_per, dout + b0 * out_per, nb * out_per, cudaMemcpyDeviceToHost, sout);
    if (ce != cudaSuccess) {
      *err = std::string("host pipeline D2H: ") + cudaGetErrorString(ce);
      res = Status::kCuda;
    }
  }
  // Drain all three streams before returning (also on error: no copy may still touch
  // the caller's buffers after the call).
  cudaError_t e1 = cudaStreamSynchronize(sin), e2 = cudaStreamSynchronize(s), e3 = cudaStreamSynchronize(sout);
  if (res != Status::kOk) return res;
  for (cudaError_t e : {e1, e2, e3})
    if (e != cudaSuccess) {
      *err = std::string("host pipeline synchronize: ") + cudaGetErrorString(e);
      return Status::kCuda;
    }
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
// Per device: the context the set-up ran in and the array's device address there.  A
// new primary context (after cudaDeviceReset) gets the set-up again.
struct NoAllocSlot {
  void* ctx = nullptr;
  unsigned char* addr = nullptr;
};
NoAllocSlot g_noalloc_slot[kNoAllocMaxDevices];

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// The calling thread's current context (CUcontext), through the driver entry point so
// the library does not link libcuda; null when the entry point is unavailable.
void* current_context() {
  using GetCtx = int (*)(void**);
  static GetCtx fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<GetCtx>(p);
  }();
  void* ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

// Device address of the static scratch for the current device.  In host code the
// array's name is only a host-side stand-in, so the address is looked up with the
// device current, once per device and context, together with the kernels'
// shared-memory attributes.
Status noalloc_scratch_for_current_device(unsigned char** out, std::string* err) {
  int dev = 0;
  CFFT_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (dev < 0 || dev >= kNoAllocMaxDevices) { *err = "device ordinal above the supported range"; return Status::kUnsupported; }
  void* ctx = current_context();  // null before the device's first runtime call
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocSlot& slot = g_noalloc_slot[dev];
  if (!slot.addr || !ctx || slot.ctx != ctx) {
    void* ptr = nullptr;
    CFFT_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress(static scratch)");
    set_smem_attrs<float>();
    set_smem_attrs<double>();
    CFFT_CUDA(cudaGetLastError(), "set shared-memory attributes");
    slot.addr = static_cast<unsigned char*>(ptr);
    slot.ctx = current_context();
  }
  *out = slot.addr;
  return Status::kOk;
}

// Geometry, twiddle tables and spectral points reach the static array as kernel
// parameters: each launch carries up to kUploadWords words by value (parameter blocks
// up to 32,764 bytes are accepted on sm_70 and newer since CUDA 12.1), so no host
// buffer is referenced once the launch call has returned and nothing is staged
// through host memory the call would have to allocate.
constexpr int kUploadWords = 7680;
struct UploadBlock {
  uint32_t w[kUploadWords];
};
__global__ void k_noalloc_upload(uint32_t* __restrict__ dst, const __grid_constant__ UploadBlock blk, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = blk.w[i];
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
  // [geometry | tables | spectral points] at their 256-byte aligned offsets, as words.
  std::vector<uint32_t> blob(off_W / 4, 0u);
  std::memcpy(blob.data(), &g, sizeof(g));
  std::memcpy(blob.data() + off_tab / 4, tab.data(), tab.size());
  std::memcpy(blob.data() + off_spec / 4, hp.data(), hp.size() * 4);
  UploadBlock blk;
  for (size_t w0 = 0; w0 < blob.size(); w0 += kUploadWords) {
    const int n = static_cast<int>(std::min<size_t>(kUploadWords, blob.size() - w0));
    std::memcpy(blk.w, blob.data() + w0, static_cast<size_t>(n) * 4);
    k_noalloc_upload<<<(n + 255) / 256, 256, 0, st>>>(reinterpret_cast<uint32_t*>(base) + w0, blk, n);
    ++g_launches;
  }
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
