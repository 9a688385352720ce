// Compile-time sized fast-path kernels of libcfft_b200 (sm_100a).  Included by the four
// fast_*.cu translation units; each defines CFFT_FAST_T (float/double) and
// CFFT_FAST_GROUP (0: plane stages 0 and 5, 1: stages 1-4) before including it, so
// every unit instantiates only its own kernels.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include <cooperative_groups.h>

#include "device_common.cuh"
#include "fast_api.h"

namespace cfft {
namespace {

// ---------------------------------------------------------------- compile-time sized path
// For cubic channel grids with H in {4, 6, 8, 12, 16, 24, 32, 48} every line FFT is a
// fully unrolled mixed-radix Stockham in registers (one thread per line), with its
// twiddles in constant memory, so no runtime division or shared-memory pass remains
// inside an FFT.  Shared-memory rows are padded to an odd stride (H + 1 complex) so
// row and column accesses of a warp are bank-conflict free.

// Programmatic dependent launch: wait until the previous kernel of the stream has
// completed and its writes are visible (a no-op when the kernel was launched without
// the attribute), then let the next kernel of the stream start launching.  Called first
// in every kernel that launch_k starts, before any global memory access.
__device__ __forceinline__ void pdl_enter() {
  asm volatile("griddepcontrol.wait;\n" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

// Drop one 128-byte L2 line without writing it back (its contents become undefined).
// Used on channel-workspace lines that have been read for the last time, so the dirty
// intermediate never travels to HBM.
__device__ __forceinline__ void discard_l2_line(const void* p) {
  asm volatile("discard.global.L2 [%0], 128;\n" ::"l"(p) : "memory");
}

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

// Alive parity channels per centring (WHT index o = o0 + 2 o1 + 4 o2 of each channel),
// as compile-time data so channel loops unroll with constant register indices.
// CT: 0 plain (no fold), 1 I, 2 F, 3 C, 4 A (same order as the plan's offsets).
template <int CT> struct Cent {
  static constexpr int n = CT == 0 ? 1 : CT == 2 ? 2 : 4;
  static __host__ __device__ constexpr int off(int c) {
    return CT == 1 ? (c == 0 ? 0 : c == 1 ? 3 : c == 2 ? 5 : 6)
         : CT == 2 ? (c == 0 ? 0 : 7)
         : CT == 3 ? (c == 0 ? 0 : c == 1 ? 3 : c == 2 ? 4 : 7)
         : CT == 4 ? (c == 0 ? 0 : c == 1 ? 6 : c == 2 ? 1 : 7) : 0;
  }
};

// Two real fields share one complex transform on the fast path: slot s of the
// channel workspace holds g_a + i g_b for fields a = 2s and b = 2s + 1 (b may be
// absent at the end of a batch).  The forward gather separates them with
// G_a(p) = (X(p) + conj X(-p)) / 2 and G_b(p) = (X(p) - conj X(-p)) / 2i, the backward
// builds X = G_a + i G_b and the unfold reads field a from the real part and field b
// from the imaginary part.  This halves the FFT work and the workspace traffic.

// Row / column FFTs of nch padded planes for a group of threads (gtid of gnth).
template <typename C, bool INV, int H>
__device__ __forceinline__ void group_rows(C* buf, int nlines, int tid, int nth) {
  constexpr int S = H + 1;
  for (int l = tid; l < nlines; l += nth) {
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
__device__ __forceinline__ void group_cols(C* buf, int nlines, int tid, int nth) {
  constexpr int S = H + 1;
  for (int l = tid; l < nlines; l += nth) {
    C* p = buf + (l / H) * (H * S) + (l % H);
    C v[H];
#pragma unroll
    for (int i = 0; i < H; ++i) v[i] = p[i * S];
    reg_fft<C, INV, H>(v);
#pragma unroll
    for (int i = 0; i < H; ++i) p[i * S] = v[i];
  }
}

// Fold of VW consecutive x values (ix0 .. ix0 + VW - 1) of channel row iy: the eight
// octant values of fields a and b (va[k], vb[k], octant k = kx + 2 ky + 4 kz) go through
// the WHT8, each alive channel takes its fold twiddle, and the results land in the
// padded planes at buf.
template <typename T, int H, int CT, int VW>
__device__ __forceinline__ void fold_emit(const T (&va)[8][VW], const T (&vb)[8][VW], int ix0, int iy,
                                          const typename Cx<T>::type* __restrict__ ftx,
                                          typename Cx<T>::type ftz, typename Cx<T>::type* buf) {
  using C = typename Cx<T>::type;
  constexpr int S = H + 1;
  constexpr int PL = H * S;
  constexpr int nch = Cent<CT>::n;
  const T zero = static_cast<T>(0);
  const C ty = ftx[iy];
#pragma unroll
  for (int l = 0; l < VW; ++l) {
    C p8[8];  // field a in the real lane, field b in the imaginary lane
#pragma unroll
    for (int k = 0; k < 8; ++k) p8[k] = mk<C>(va[k][l], vb[k][l]);
    wht8c(p8);
    const int ix = ix0 + l;
    const C tx = ftx[ix];
#pragma unroll
    for (int c = 0; c < nch; ++c) {
      const int o = Cent<CT>::off(c);
      C w = mk<C>(static_cast<T>(1), zero);
      if (o & 1) w = tx;
      if (o & 2) w = cmul(w, ty);
      if (o & 4) w = cmul(w, ftz);
      buf[c * PL + iy * S + ix] = o ? cmul(p8[o], w) : p8[o];
    }
  }
}

// Fold (or plain load, CT = 0) of the two fields of one slot at channel z-plane iz into
// the nch padded planes at buf (channel c at buf + c * H * (H + 1)), with the fold
// twiddles e^{-2 pi i off.n / M} and the interaction factors E when given.  Work is
// spread over threads tid of nth.
template <typename T, int H, int CT>
__device__ __forceinline__ void fold_plane(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                                           const T* __restrict__ srca, const T* __restrict__ srcb,
                                           const T* __restrict__ Ea, const T* __restrict__ Eb, bool has_b, bool USE_E,
                                           int iz, typename Cx<T>::type* buf, int tid, int nth) {
  using C = typename Cx<T>::type;
  constexpr int S = H + 1;
  constexpr int PL = H * S;
  constexpr int nch = Cent<CT>::n;
  const T zero = static_cast<T>(0);
  if constexpr (CT == 0) {
    const size_t zoff = static_cast<size_t>(iz) * H * H;
    for (int e = tid; e < H * H; e += nth) {
      T va = srca[zoff + e];
      T vb = has_b ? srcb[zoff + e] : zero;
      if (USE_E) { va *= Ea[zoff + e]; if (has_b) vb *= Eb[zoff + e]; }
      buf[(e / H) * S + (e % H)] = mk<C>(va, vb);
    }
  } else {
    constexpr int M = 2 * H;
    constexpr int VW = 16 / static_cast<int>(sizeof(T));  // elements per 16-byte vector
    using V = typename Vec16<T>::type;
    const C* ftx = tables + g->ftw_off[0];
    const C ftz = tables[g->ftw_off[2] + iz];
    const bool vec = (H % VW == 0) && (reinterpret_cast<uintptr_t>(srca) % 16 == 0) &&
                     (!USE_E || reinterpret_cast<uintptr_t>(Ea) % 16 == 0);
    if (vec) {
      for (int e = tid; e < H * H / VW; e += nth) {
        const int ix0 = (e % (H / VW)) * VW, iy = e / (H / VW);
        T va[8][VW], vb[8][VW];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int idx = ((iz + ((k >> 2) & 1) * H) * M + iy + ((k >> 1) & 1) * H) * M + ix0 + (k & 1) * H;
          vload_stream<T>(va[k], srca + idx);
          if (has_b) vload_stream<T>(vb[k], srcb + idx);
          else {
#pragma unroll
            for (int l = 0; l < VW; ++l) vb[k][l] = zero;
          }
          if (USE_E) {
            T ea[VW];
            vload<T>(ea, Ea + idx);
#pragma unroll
            for (int l = 0; l < VW; ++l) va[k][l] *= ea[l];
            if (has_b) {
              vload<T>(ea, Eb + idx);
#pragma unroll
              for (int l = 0; l < VW; ++l) vb[k][l] *= ea[l];
            }
          }
        }
        fold_emit<T, H, CT, VW>(va, vb, ix0, iy, ftx, ftz, buf);
      }
    } else {
      for (int e = tid; e < H * H; e += nth) {
        const int ix = e % H, iy = e / H;
        T va[8], vb[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int idx = ((iz + ((k >> 2) & 1) * H) * M + iy + ((k >> 1) & 1) * H) * M + ix + (k & 1) * H;
          va[k] = srca[idx];
          vb[k] = has_b ? srcb[idx] : zero;
          if (USE_E) { va[k] *= Ea[idx]; if (has_b) vb[k] *= Eb[idx]; }
        }
        wht8(va);
        wht8(vb);
        const C tx = ftx[ix], ty = ftx[iy];  // cubic: the y fold twiddle table equals x's
#pragma unroll
        for (int c = 0; c < nch; ++c) {
          const int o = Cent<CT>::off(c);
          C w = mk<C>(static_cast<T>(1), zero);
          if (o & 1) w = tx;
          if (o & 2) w = cmul(w, ty);
          if (o & 4) w = cmul(w, ftz);
          buf[c * PL + iy * S + ix] = cmul(mk<C>(va[o], vb[o]), w);
        }
      }
    }
  }
}

// Unfold of the nch inverse-transformed planes at buf (channel z-plane iz) into the two
// fields of the slot: conjugate fold twiddle, inverse WHT8 / 8, real part -> field a,
// imaginary part -> field b, times E when given.
template <typename T, int H, int CT, bool VEC = false>
__device__ __forceinline__ void unfold_plane(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                                             const typename Cx<T>::type* buf, T* __restrict__ dsta, T* __restrict__ dstb,
                                             const T* __restrict__ Ea, const T* __restrict__ Eb, bool has_b, bool USE_E,
                                             int iz, int tid, int nth) {
  using C = typename Cx<T>::type;
  constexpr int S = H + 1;
  constexpr int PL = H * S;
  constexpr int nch = Cent<CT>::n;
  const size_t hvol = static_cast<size_t>(H) * H * H;
  const size_t mvol = static_cast<size_t>(g->M[0]) * g->M[1] * g->M[2];
  if constexpr (CT == 0) {
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
    constexpr int VW = 16 / static_cast<int>(sizeof(T));  // elements per 16-byte vector
    const bool vec = VEC && (H % VW == 0) && (reinterpret_cast<uintptr_t>(dsta) % 16 == 0) &&
                     (!has_b || reinterpret_cast<uintptr_t>(dstb) % 16 == 0) &&
                     (!USE_E || (reinterpret_cast<uintptr_t>(Ea) % 16 == 0 && (!has_b || reinterpret_cast<uintptr_t>(Eb) % 16 == 0)));
    if (vec) {
      // VW consecutive x values per thread; each octant row piece leaves as one 16-byte store.
      for (int e = tid; e < H * H / VW; e += nth) {
        const int ix0 = (e % (H / VW)) * VW, iy = e / (H / VW);
        const C ty = ftx[iy];
        T oa[8][VW], ob[8][VW];
#pragma unroll
        for (int l = 0; l < VW; ++l) {
          const int ix = ix0 + l;
          const C tx = ftx[ix];
          T va[8], vb[8];
#pragma unroll
          for (int k = 0; k < 8; ++k) { va[k] = static_cast<T>(0); vb[k] = static_cast<T>(0); }
#pragma unroll
          for (int c = 0; c < nch; ++c) {
            const int o = Cent<CT>::off(c);
            C w = mk<C>(static_cast<T>(1), static_cast<T>(0));
            if (o & 1) w = tx;
            if (o & 2) w = cmul(w, ty);
            if (o & 4) w = cmul(w, ftz);
            const C y = cmulc(buf[c * PL + iy * S + ix], w);
            va[o] = y.x;
            vb[o] = y.y;
          }
          wht8(va);
          wht8(vb);
#pragma unroll
          for (int k = 0; k < 8; ++k) { oa[k][l] = va[k] * scale; ob[k][l] = vb[k] * scale; }
        }
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int idx = ((iz + ((k >> 2) & 1) * H) * M + iy + ((k >> 1) & 1) * H) * M + ix0 + (k & 1) * H;
          if (USE_E) {
            T ea[VW];
            vload<T>(ea, Ea + idx);
#pragma unroll
            for (int l = 0; l < VW; ++l) oa[k][l] *= ea[l];
            if (has_b) {
              vload<T>(ea, Eb + idx);
#pragma unroll
              for (int l = 0; l < VW; ++l) ob[k][l] *= ea[l];
            }
          }
          vstore_stream<T>(dsta + idx, oa[k]);
          if (has_b) vstore_stream<T>(dstb + idx, ob[k]);
        }
      }
    } else {
      for (int e = tid; e < H * H; e += nth) {
        const int ix = e % H, iy = e / H;
        T va[8], vb[8];
#pragma unroll
        for (int k = 0; k < 8; ++k) { va[k] = static_cast<T>(0); vb[k] = static_cast<T>(0); }
        const C tx = ftx[ix], ty = ftx[iy];
#pragma unroll
        for (int c = 0; c < nch; ++c) {
          const int o = Cent<CT>::off(c);
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
          const int idx = ((iz + ((k >> 2) & 1) * H) * M + iy + ((k >> 1) & 1) * H) * M + ix + (k & 1) * H;
          T a = va[k] * scale, bq = vb[k] * scale;
          if (USE_E) { a *= Ea[idx]; if (has_b) bq *= Eb[idx]; }
          dsta[idx] = a;
          if (has_b) dstb[idx] = bq;
        }
      }
    }
  }
}

// y lines of the nch padded planes at buf: each thread owns the column (c, x),
// transforms it and stores it straight to the workspace plane dst0 (channel stride
// H^3, consecutive threads write consecutive x).
template <typename C, int H, int nch>
__device__ __forceinline__ void y_lines_to_workspace(const C* buf, C* __restrict__ dst0, int tid, int nth) {
  constexpr int S = H + 1;
  constexpr int PL = H * S;
  constexpr int HV = H * H * H;
  for (int l = tid; l < nch * H; l += nth) {
    const int c = l / H, x = l % H;
    const C* p = buf + c * PL + x;
    C v[H];
#pragma unroll
    for (int i = 0; i < H; ++i) v[i] = p[i * S];
    reg_fft<C, false, H>(v);
    C* d = dst0 + static_cast<size_t>(c) * HV + x;
#pragma unroll
    for (int i = 0; i < H; ++i) d[i * H] = v[i];
  }
}

// Forward plane kernel, cubic H: fold (or plain load) of two fields + x FFT + y FFT
// -> W[slot][c][z][y][x].
template <typename T, int H, int CT>
__global__ void k_plane_fwd_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                              const T* __restrict__ f0, const T* __restrict__ E, typename Cx<T>::type* __restrict__ W,
                              int nfields) {
  pdl_enter();
  using C = typename Cx<T>::type;
  constexpr int nch = Cent<CT>::n;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int iz = blockIdx.x, slot = blockIdx.y;
  const int fa = 2 * slot;
  const bool has_b = fa + 1 < nfields;
  const bool USE_E = E != nullptr;  // warp-uniform
  const int tid = threadIdx.x, nth = blockDim.x;
  const size_t mvol = static_cast<size_t>(g->M[0]) * g->M[1] * g->M[2];
  const T* srca = f0 + static_cast<size_t>(fa) * mvol;
  const T* Ea = USE_E ? E + static_cast<size_t>(fa) * mvol : nullptr;
  fold_plane<T, H, CT>(g, tables, srca, srca + mvol, Ea, USE_E ? Ea + mvol : nullptr, has_b, USE_E, iz, buf, tid, nth);
  __syncthreads();
  group_rows<C, false, H>(buf, nch * H, tid, nth);   // x lines
  __syncthreads();
  constexpr int HV = H * H * H;
  y_lines_to_workspace<C, H, nch>(buf, W + static_cast<size_t>(slot) * nch * HV + iz * H * H, tid, nth);
}

// Backward plane kernel, cubic H: inverse x/y FFT of W[slot][c][iz] + unfold of the two
// fields (real part -> field a, imaginary part -> field b).
template <typename T, int H, int CT, bool VEC>
__global__ void k_plane_bwd_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                              const typename Cx<T>::type* __restrict__ W, const T* __restrict__ E, T* __restrict__ f0,
                              int nfields) {
  pdl_enter();
  using C = typename Cx<T>::type;
  constexpr int S = H + 1;
  constexpr int PL = H * S;
  constexpr int nch = Cent<CT>::n;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int iz = blockIdx.x, slot = blockIdx.y;
  const int fa = 2 * slot;
  const bool has_b = fa + 1 < nfields;
  const bool USE_E = E != nullptr;  // warp-uniform
  const int tid = threadIdx.x, nth = blockDim.x;
  constexpr int HV = H * H * H;
  // y lines straight from the workspace into registers (coalesced across x), inverse
  // FFT, into shared memory; then the x lines there.
  const C* src0 = W + static_cast<size_t>(slot) * nch * HV + iz * H * H;
  for (int l = tid; l < nch * H; l += nth) {
    const int c = l / H, x = l % H;
    const C* q = src0 + static_cast<size_t>(c) * HV + x;
    C v[H];
#pragma unroll
    for (int i = 0; i < H; ++i) v[i] = q[i * H];
    reg_fft<C, true, H>(v);
    C* p = buf + c * PL + x;
#pragma unroll
    for (int i = 0; i < H; ++i) p[i * S] = v[i];
  }
  __syncthreads();
  // Last read of these workspace planes: drop their lines from L2 without a write-back.
  if constexpr ((H * H * sizeof(C)) % 128 == 0) {
    constexpr int LPP = static_cast<int>(H * H * sizeof(C) / 128);
    for (int i = tid; i < nch * LPP; i += nth)
      discard_l2_line(reinterpret_cast<const char*>(src0 + static_cast<size_t>(i / LPP) * HV) + (i % LPP) * 128);
  }
  group_rows<C, true, H>(buf, nch * H, tid, nth);
  __syncthreads();
  const size_t mvol = static_cast<size_t>(g->M[0]) * g->M[1] * g->M[2];
  T* dsta = f0 + static_cast<size_t>(fa) * mvol;
  const T* Ea = USE_E ? E + static_cast<size_t>(fa) * mvol : nullptr;
  unfold_plane<T, H, CT, VEC>(g, tables, buf, dsta, dsta + mvol, Ea, USE_E ? Ea + mvol : nullptr, has_b, USE_E, iz, tid, nth);
}

#include "tma_planes.cuh"

// ---------------------------------------------------------------- cluster kernels
// One thread-block cluster of KC CTAs holds the whole channel volume of one workspace
// slot (two fields) in distributed shared memory: CTA r owns the channel z-planes
// [ZPC r, ZPC r + ZPC), ZPC = H / KC, as padded nch x H x (H+1)
// planes.  The z transforms then read (forward) or write (backward) the peers' planes
// directly, so the channel workspace never makes the plane <-> z round trip through L2.
template <int H, int CT, int KC> struct ClusterShape {
  static constexpr int nch = Cent<CT>::n;
  static constexpr int zpc = H / KC;                    // channel z-planes per CTA
  static constexpr int threads = nch * zpc * H;         // one z line (c, y, x) per thread
  static constexpr int group = nch * H;                 // threads per plane in the x/y phase
};
// KC = 8 (portable) for H = 16, 24, 32; KC = 16 (non-portable, two CTAs per SM) for H = 32.
template <typename T, int H, int CT, int KC>
constexpr bool cluster_fits() {
  return H % KC == 0 && H >= 16 && H <= 32 && (KC == 8 || (KC == 16 && H == 32)) &&
         ClusterShape<H, CT, KC>::threads >= 32 && ClusterShape<H, CT, KC>::threads <= 1024 &&
         static_cast<long>(ClusterShape<H, CT, KC>::zpc) * Cent<CT>::n * H * (H + 1) * 2 * sizeof(T) <= 227 * 1024;
}
template <typename T, int H, int CT, int KC>
constexpr size_t cluster_smem() {
  return static_cast<size_t>(ClusterShape<H, CT, KC>::zpc) * Cent<CT>::n * H * (H + 1) * 2 * sizeof(T);
}

// Forward: fold + x/y FFT of the CTA's ZPC planes, cluster barrier, z FFT of the lines
// (c, y in the CTA's rows, x) gathered from the peers' planes, cluster barrier (every
// peer has finished reading), then the lines are transposed through the CTA's own
// shared memory and stored z-fastest: WT[slot][c][x][y][z].
template <typename T, int H, int CT, int KC>
__global__ void __launch_bounds__(ClusterShape<H, CT, KC>::threads)
k_fwd_cluster_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                const T* __restrict__ f0, const T* __restrict__ E, typename Cx<T>::type* __restrict__ WT, int nfields) {
  using C = typename Cx<T>::type;
  using CS = ClusterShape<H, CT, KC>;
  constexpr int S = H + 1, PL = H * S, NCH = CS::nch, ZPC = CS::zpc, HV = H * H * H;
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int r = static_cast<int>(cluster.block_rank());
  const int slot = blockIdx.y;
  const int fa = 2 * slot;
  const bool has_b = fa + 1 < nfields;
  const bool USE_E = E != nullptr;
  const int tid = threadIdx.x;
  const size_t mvol = static_cast<size_t>(g->M[0]) * g->M[1] * g->M[2];
  {
    const int grp = tid / CS::group, gtid = tid % CS::group;
    C* pbuf = buf + grp * NCH * PL;
    const T* srca = f0 + static_cast<size_t>(fa) * mvol;
    const T* Ea = USE_E ? E + static_cast<size_t>(fa) * mvol : nullptr;
    fold_plane<T, H, CT>(g, tables, srca, srca + mvol, Ea, USE_E ? Ea + mvol : nullptr, has_b, USE_E, ZPC * r + grp,
                         pbuf, gtid, CS::group);
    __syncthreads();
    group_rows<C, false, H>(pbuf, NCH * H, gtid, CS::group);
    __syncthreads();
    group_cols<C, false, H>(pbuf, NCH * H, gtid, CS::group);
  }
  cluster.sync();
  const int c = tid / (ZPC * H), yy = (tid / H) % ZPC, x = tid % H;
  const int y = ZPC * r + yy;
  C v[H];
#pragma unroll
  for (int z = 0; z < H; ++z) {
    const C* rb = cluster.map_shared_rank(buf, z / ZPC);
    v[z] = rb[((z % ZPC) * NCH + c) * PL + y * S + x];
  }
  reg_fft<C, false, H>(v);
  cluster.sync();
  constexpr int RUN = ZPC * H, PCX = RUN + 1;  // staging [c][x][yy][z], padded per (c, x)
#pragma unroll
  for (int z = 0; z < H; ++z) buf[(c * H + x) * PCX + yy * H + z] = v[z];
  __syncthreads();
  C* dst = WT + static_cast<size_t>(slot) * NCH * HV;
  for (int e = tid; e < NCH * H * RUN; e += CS::threads) {
    const int cx = e / RUN, rr = e % RUN;
    dst[static_cast<size_t>(cx / H) * HV + ((cx % H) * H + ZPC * r) * H + rr] = buf[cx * PCX + rr];
  }
}

// Backward: cluster barrier (every peer is running), orbit expansion + inverse z FFT of
// the CTA's lines (c, y, x) from the combined representatives G0P[slot / 2][o][slot & 1]
// and the packed expansion entries (orbit | phase << 21), written into the owning
// peers' planes; cluster barrier; inverse x/y FFT + unfold of the CTA's own planes.
template <typename T, int H, int CT, int KC>
__global__ void __launch_bounds__(ClusterShape<H, CT, KC>::threads)
k_bwd_cluster_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                const uint32_t* __restrict__ ETP, const typename Cx<T>::type* __restrict__ G0P,
                const T* __restrict__ E, T* __restrict__ f0, int nfields) {
  using C = typename Cx<T>::type;
  using CS = ClusterShape<H, CT, KC>;
  constexpr int S = H + 1, PL = H * S, NCH = CS::nch, ZPC = CS::zpc, HV = H * H * H;
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);
  const int r = static_cast<int>(cluster.block_rank());
  const int slot = blockIdx.y;
  const int tid = threadIdx.x;
  cluster.sync();
  {
    const int c = tid / (ZPC * H), yy = (tid / H) % ZPC, x = tid % H;
    const int y = ZPC * r + yy;
    const uint32_t* et = ETP + static_cast<size_t>(c) * HV + y * H + x;
    const C* rp = G0P + static_cast<size_t>(slot >> 1) * g->n_orbits * 2 + (slot & 1);
    const C* ph = tables + g->ph_off;
    C v[H];
#pragma unroll
    for (int z = 0; z < H; ++z) {
      const uint32_t t = __ldg(et + z * H * H);
      v[z] = cmulc(__ldg(rp + 2 * static_cast<size_t>(t & 0x1FFFFFu)), ph[t >> 21]);
    }
    reg_fft<C, true, H>(v);
#pragma unroll
    for (int z = 0; z < H; ++z) {
      C* rb = cluster.map_shared_rank(buf, z / ZPC);
      rb[((z % ZPC) * NCH + c) * PL + y * S + x] = v[z];
    }
  }
  cluster.sync();
  const int grp = tid / CS::group, gtid = tid % CS::group;
  C* pbuf = buf + grp * NCH * PL;
  group_rows<C, true, H>(pbuf, NCH * H, gtid, CS::group);
  __syncthreads();
  group_cols<C, true, H>(pbuf, NCH * H, gtid, CS::group);
  __syncthreads();
  const int fa = 2 * slot;
  const bool has_b = fa + 1 < nfields;
  const bool USE_E = E != nullptr;
  const size_t mvol = static_cast<size_t>(g->M[0]) * g->M[1] * g->M[2];
  T* dsta = f0 + static_cast<size_t>(fa) * mvol;
  const T* Ea = USE_E ? E + static_cast<size_t>(fa) * mvol : nullptr;
  unfold_plane<T, H, CT>(g, tables, pbuf, dsta, dsta + mvol, Ea, USE_E ? Ea + mvol : nullptr, has_b, USE_E,
                         ZPC * r + grp, gtid, CS::group);
}

constexpr int kZB = kFastZB;
// Threads of the z kernels that take one (y, x) line each: kZB y values x H lines, in
// whole warps, at least 64.
template <int H> constexpr int z_threads() { return ((kZB * H + 31) / 32) * 32 < 64 ? 64 : ((kZB * H + 31) / 32) * 32; }

// Forward z FFT, cubic H: W[slot][c][z][y][x] (in) -> WT[slot][c][x][y][z] (z fastest,
// out, same storage: each CTA reads and writes exactly the same addresses).  Thread
// (yy, x) loads its z line straight into registers (coalesced across x); the
// transposed store goes through shared memory.  Launched with z_threads<H>() threads;
// when kZB divides H every CTA holds kZB y values and the store loop's bounds and
// divisors are compile-time constants.
template <typename T, int H>
__global__ void k_fft_z_fwd_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* W,
                              typename Cx<T>::type* WT) {
  pdl_enter();
  using C = typename Cx<T>::type;
  constexpr int S = H + 1;
  constexpr int HV = H * H * H;
  constexpr int kThr = z_threads<H>();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);  // [yy][x][z] padded
  const int y0 = blockIdx.x * kZB, c = blockIdx.y, slot = blockIdx.z;
  const int ny = H % kZB == 0 ? kZB : min(kZB, H - y0);
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
  if constexpr (H % kZB == 0) {
    constexpr int run = kZB * H;  // contiguous (yy, z) run per x
#pragma unroll 4
    for (int e = tid; e < H * run; e += kThr) {
      const int xx = e / run, r = e % run;
      const int y2 = r / H, z = r % H;
      dst[(xx * H + y0) * H + r] = buf[(y2 * H + xx) * S + z];
    }
  } else {
    const int run = ny * H;
    for (int e = tid; e < H * run; e += kThr) {
      const int xx = e / run, r = e % run;
      const int y2 = r / H, z = r % H;
      dst[(xx * H + y0) * H + r] = buf[(y2 * H + xx) * S + z];
    }
  }
}

// Backward: expand G0 from orbit representatives (ET table) + inverse z FFT, cubic H:
// G0R[slot][o] -> W[slot][c][z][y][x].
template <typename T, int H>
__global__ void k_expand_ifft_z_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                                  const int2* __restrict__ ET, const typename Cx<T>::type* __restrict__ G0R,
                                  typename Cx<T>::type* __restrict__ W) {
  pdl_enter();
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


// Spectral-ASU gather from the z-fastest packed workspace, cubic M (= 2H centred,
// = H plain), D representative operations; separates the two fields of the slot on
// the fly.  The geometry is staged in shared memory once per CTA.
template <typename T, int M, int D, bool USE_K, bool PERM>
__global__ void k_recon_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                          const uint32_t* __restrict__ spec_h, const T* __restrict__ K,
                          const typename Cx<T>::type* __restrict__ WT, typename Cx<T>::type* __restrict__ F,
                          int nfields) {
  pdl_enter();
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
constexpr int kDiagSlots = 2;
template <typename T, int M, bool USE_K>
__global__ void k_recon_diag8(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                              const uint32_t* __restrict__ spec_h, const T* __restrict__ K,
                              const typename Cx<T>::type* __restrict__ WT, typename Cx<T>::type* __restrict__ F,
                              int nfields) {
  pdl_enter();
  using C = typename Cx<T>::type;
  __shared__ int sTP[8][3];  // indexed by sign pattern
  __shared__ int sCh[8];
  const int tid = threadIdx.x;
  if (tid < 24) sTP[tid / 3][tid % 3] = g->rep_tp[g->sign_op[tid / 3]][tid % 3];
  if (tid < 8) sCh[tid] = g->chan_of_parity[tid];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + tid;
  if (s >= g->n_spec) return;
  const int ns = g->n_spec;
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
  // This thread serves kDiagSlots consecutive slots (fields 2 slot, 2 slot + 1): the
  // indices and phases are shared, the gathers of all its slots are in flight together.
  const int slot0 = blockIdx.y * kDiagSlots;
  if (c < 0) {  // extinct parity class: every tap reads zero
    const C z = mk<C>(static_cast<T>(0), static_cast<T>(0));
    for (int f = 2 * slot0; f < min(nfields, 2 * (slot0 + kDiagSlots)); ++f) F[static_cast<size_t>(f) * ns + s] = z;
    return;
  }
  const int X0[2] = {(p0 >> ls) * Hc * Hc, (m0 >> ls) * Hc * Hc};
  const int X1[2] = {(p1 >> ls) * Hc, (m1 >> ls) * Hc};
  const int X2[2] = {p2 >> ls, m2 >> ls};
  C X[kDiagSlots][8];
#pragma unroll
  for (int k = 0; k < kDiagSlots; ++k) {
    const int slot = min(slot0 + k, (nfields - 1) / 2);  // clamped: beyond the batch the result is dropped
    const C* Wb = WT + (static_cast<size_t>(slot) * g->n_ch + c) * hvol;
#pragma unroll
    for (int sg = 0; sg < 8; ++sg) X[k][sg] = Wb[X0[sg & 1] + X1[(sg >> 1) & 1] + X2[(sg >> 2) & 1]];
  }
  const C* ph = tables + g->ph_off;
  const int P = g->P, pmask = g->pmask;
  C w[8];
#pragma unroll
  for (int sg = 0; sg < 8; ++sg) {
    int j = h0 * sTP[sg][0] + h1 * sTP[sg][1] + h2 * sTP[sg][2];
    j = pmask >= 0 ? (j & pmask) : ((j % P) + P) % P;
    w[sg] = ph[j];
  }
  // Taps sg and 7 - sg are Hermitian partners: with u = w[sg], v = w[7 - sg] and
  // 2 G = (a, b), G u + conj(G) v = (a Pw.x + b Qw.x, a Pw.y + b Qw.y) for
  // Pw = (u + v) / 2, Qw = ((v.y - u.y) / 2, (u.x - v.x) / 2), shared by every slot
  // and both fields.
  const T half = static_cast<T>(0.5);
  C Pw[4], Qw[4];
#pragma unroll
  for (int sg = 0; sg < 4; ++sg) {
    const C u = w[sg], v = w[7 - sg];
    Pw[sg] = mk<C>(half * (u.x + v.x), half * (u.y + v.y));
    Qw[sg] = mk<C>(half * (v.y - u.y), half * (u.x - v.x));
  }
  const T kk = USE_K ? K[s] : static_cast<T>(1);
#pragma unroll
  for (int k = 0; k < kDiagSlots; ++k) {
    const int fa = 2 * (slot0 + k);
    if (fa >= nfields) break;
    C acca = mk<C>(static_cast<T>(0), static_cast<T>(0));
    C accb = acca;
#pragma unroll
    for (int sg = 0; sg < 4; ++sg) {
      const C Xs = X[k][sg], Xn = X[k][7 - sg];
      const T a = Xs.x + Xn.x, b = Xs.y - Xn.y;    // 2 G_a
      const T a2 = Xs.y + Xn.y, b2 = Xn.x - Xs.x;  // 2 G_b
      acca.x = fma(a, Pw[sg].x, fma(b, Qw[sg].x, acca.x));
      acca.y = fma(a, Pw[sg].y, fma(b, Qw[sg].y, acca.y));
      accb.x = fma(a2, Pw[sg].x, fma(b2, Qw[sg].x, accb.x));
      accb.y = fma(a2, Pw[sg].y, fma(b2, Qw[sg].y, accb.y));
    }
    if (USE_K) { acca = cscale(acca, kk); accb = cscale(accb, kk); }
    F[static_cast<size_t>(fa) * ns + s] = acca;
    if (fa + 1 < nfields) F[static_cast<size_t>(fa + 1) * ns + s] = accb;
  }
}

// Forward z FFT fused with the spectral-ASU gather, for diagonal-sign representative
// operations (the taps of a spectral point h read G0 at the sign images of h, which lie
// in one channel c on the rows y = p1 >> ls and its mirror y' = m1 >> ls).  A CTA
// takes one unit (channel c and a mirrored pair of channel rows y_a, y_b; y_b < 0 when
// the unit has one row) and ZR_SLOTS workspace slots:
//   1. thread (slot, row, x) loads the z line W[slot][c][z][y_row][x] (coalesced across
//      x), transforms it in registers and keeps it in shared memory [slot][row][x][z];
//   2. the unit's spectral points (a list built at plan time) are gathered from shared
//      memory as in k_recon_diag8 and written to F.
// The transposed workspace of the separate z kernel is never written or read back.
// Unit entry: x = c | y_a << 8 | (y_b + 1) << 16, y = first point, z = point count.
template <int H> constexpr int zr_threads(int slots) { return slots * 2 * H < 32 ? 32 : ((slots * 2 * H + 31) / 32) * 32; }
template <typename T, int H, int SL, bool USE_K>
__global__ void k_fft_z_recon_diag8(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                                    const uint32_t* __restrict__ spec_h, const T* __restrict__ K,
                                    const uint4* __restrict__ units, const uint32_t* __restrict__ pts,
                                    const typename Cx<T>::type* __restrict__ W, typename Cx<T>::type* __restrict__ F,
                                    int nfields) {
  pdl_enter();
  using C = typename Cx<T>::type;
  constexpr int S = H + 1;
  constexpr int HV = H * H * H;
  constexpr int RS = H * S;  // one row of (x, z) lines
  extern __shared__ __align__(16) unsigned char smem_raw[];
  C* buf = reinterpret_cast<C*>(smem_raw);  // [slot][row][x][z] padded
  __shared__ int sTP[8][3];
  const int tid = threadIdx.x, nth = blockDim.x;
  if (tid < 24) sTP[tid / 3][tid % 3] = g->rep_tp[g->sign_op[tid / 3]][tid % 3];
  const uint4 un = units[blockIdx.x];
  const int c = static_cast<int>(un.x & 0xFFu), ya = static_cast<int>((un.x >> 8) & 0xFFu);
  const int yb = static_cast<int>((un.x >> 16) & 0xFFu) - 1;
  const int slot0 = blockIdx.y * SL;
  const int nslots = (nfields + 1) / 2;
  const int nch = g->n_ch;
  if (tid < SL * 2 * H) {
    const int k = tid / (2 * H), r = (tid / H) & 1, x = tid % H;
    const int slot = slot0 + k;
    const int y = r ? yb : ya;
    if (slot < nslots && y >= 0) {
      const C* src = W + (static_cast<size_t>(slot) * nch + c) * HV + y * H + x;
      C v[H];
#pragma unroll
      for (int z = 0; z < H; ++z) v[z] = src[static_cast<size_t>(z) * H * H];
      reg_fft<C, false, H>(v);
      C* row = buf + (k * 2 + r) * RS + x * S;
#pragma unroll
      for (int z = 0; z < H; ++z) row[z] = v[z];
    }
  }
  __syncthreads();
  // Every workspace row (slot, c, z, y) of this unit is read by this CTA alone and never
  // again: drop its lines from L2 (rows that fill whole 128-byte lines only).
  if constexpr ((H * sizeof(C)) % 128 == 0) {
    constexpr int LPR = static_cast<int>(H * sizeof(C) / 128);
    for (int i = tid; i < SL * 2 * H * LPR; i += nth) {
      const int li = i % LPR, z = (i / LPR) % H, r = (i / (LPR * H)) & 1, k = i / (LPR * H * 2);
      const int slot = slot0 + k, y = r ? yb : ya;
      if (slot < nslots && y >= 0)
        discard_l2_line(reinterpret_cast<const char*>(W + (static_cast<size_t>(slot) * nch + c) * HV +
                                                      static_cast<size_t>(z) * H * H + y * H) + li * 128);
    }
  }
  const bool cen = g->centered;
  const int M = cen ? 2 * H : H;
  const int ls = cen ? 1 : 0;
  const int ns = g->n_spec;
  const C* ph = tables + g->ph_off;
  const int P = g->P, pmask = g->pmask;
  const T half = static_cast<T>(0.5);
  const int nvalid = min(SL, nslots - slot0);
  for (int i = tid; i < static_cast<int>(un.z); i += nth) {
    const uint32_t sidx = __ldg(pts + un.y + i);
    const uint32_t hp = __ldg(spec_h + sidx);
    const int h0 = static_cast<int>(hp & 1023u), h1 = static_cast<int>((hp >> 10) & 1023u), h2 = static_cast<int>((hp >> 20) & 1023u);
    const int p0 = cen ? mod_m<2 * H>(h0) : mod_m<H>(h0);
    const int p1 = cen ? mod_m<2 * H>(h1) : mod_m<H>(h1);
    const int p2 = cen ? mod_m<2 * H>(h2) : mod_m<H>(h2);
    const int m0 = p0 ? M - p0 : 0, m1 = p1 ? M - p1 : 0, m2 = p2 ? M - p2 : 0;
    const int X0[2] = {(p0 >> ls) * S, (m0 >> ls) * S};
    const int X1[2] = {((p1 >> ls) != ya) * RS, ((m1 >> ls) != ya) * RS};
    const int X2[2] = {p2 >> ls, m2 >> ls};
    C Pw[4], Qw[4];
    {
      C w[8];
#pragma unroll
      for (int sg = 0; sg < 8; ++sg) {
        int j = h0 * sTP[sg][0] + h1 * sTP[sg][1] + h2 * sTP[sg][2];
        j = pmask >= 0 ? (j & pmask) : ((j % P) + P) % P;
        w[sg] = ph[j];
      }
      // Hermitian tap pairs (sg, 7 - sg), as in k_recon_diag8.
#pragma unroll
      for (int sg = 0; sg < 4; ++sg) {
        const C u = w[sg], v = w[7 - sg];
        Pw[sg] = mk<C>(half * (u.x + v.x), half * (u.y + v.y));
        Qw[sg] = mk<C>(half * (v.y - u.y), half * (u.x - v.x));
      }
    }
    const T kk = USE_K ? K[sidx] : static_cast<T>(1);
#pragma unroll
    for (int k = 0; k < SL; ++k) {
      if (k >= nvalid) break;
      const C* b = buf + k * 2 * RS;
      C X[8];
#pragma unroll
      for (int sg = 0; sg < 8; ++sg) X[sg] = b[X0[sg & 1] + X1[(sg >> 1) & 1] + X2[(sg >> 2) & 1]];
      C acca = mk<C>(static_cast<T>(0), static_cast<T>(0)), accb = acca;
#pragma unroll
      for (int sg = 0; sg < 4; ++sg) {
        const C Xs = X[sg], Xn = X[7 - sg];
        const T a = Xs.x + Xn.x, bq = Xs.y - Xn.y;
        const T a2 = Xs.y + Xn.y, b2 = Xn.x - Xs.x;
        acca.x = fma(a, Pw[sg].x, fma(bq, Qw[sg].x, acca.x));
        acca.y = fma(a, Pw[sg].y, fma(bq, Qw[sg].y, acca.y));
        accb.x = fma(a2, Pw[sg].x, fma(b2, Qw[sg].x, accb.x));
        accb.y = fma(a2, Pw[sg].y, fma(b2, Qw[sg].y, accb.y));
      }
      if (USE_K) { acca = cscale(acca, kk); accb = cscale(accb, kk); }
      const int fa = 2 * (slot0 + k);
      F[static_cast<size_t>(fa) * ns + sidx] = acca;
      if (fa + 1 < nfields) F[static_cast<size_t>(fa + 1) * ns + sidx] = accb;
    }
  }
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
  pdl_enter();
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

template <int D>
__device__ __forceinline__ void load_alias_row(const uint32_t* __restrict__ inv_pk, int o, uint32_t (&e)[D]) {
  if constexpr (D == 8) {
    const uint4* p4 = reinterpret_cast<const uint4*>(inv_pk + static_cast<size_t>(o) * 8);
    const uint4 u0 = __ldg(p4), u1 = __ldg(p4 + 1);
    e[0] = u0.x; e[1] = u0.y; e[2] = u0.z; e[3] = u0.w; e[4] = u1.x; e[5] = u1.y; e[6] = u1.z; e[7] = u1.w;
  } else if constexpr (D == 4) {
    const uint4 u0 = __ldg(reinterpret_cast<const uint4*>(inv_pk + static_cast<size_t>(o) * 4));
    e[0] = u0.x; e[1] = u0.y; e[2] = u0.z; e[3] = u0.w;
  } else {
#pragma unroll
    for (int a = 0; a < D; ++a) e[a] = __ldg(inv_pk + static_cast<size_t>(o) * D + a);
  }
}

// Four complex values (fields 4g .. 4g+3 of one spectral point or orbit) as 16-byte
// vector loads / stores: 32 bytes for float, 64 for double.
template <typename C>
__device__ __forceinline__ void load_quad(const C* __restrict__ p, C (&v)[4]) {
  if constexpr (sizeof(C) == 8) {
    const float4 u0 = __ldg(reinterpret_cast<const float4*>(p)), u1 = __ldg(reinterpret_cast<const float4*>(p) + 1);
    v[0] = mk<C>(u0.x, u0.y); v[1] = mk<C>(u0.z, u0.w); v[2] = mk<C>(u1.x, u1.y); v[3] = mk<C>(u1.z, u1.w);
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = __ldg(p + k);
  }
}
template <typename C>
__device__ __forceinline__ void store_quad(C* __restrict__ p, const C (&v)[4]) {
  if constexpr (sizeof(C) == 8) {
    reinterpret_cast<float4*>(p)[0] = make_float4(v[0].x, v[0].y, v[1].x, v[1].y);
    reinterpret_cast<float4*>(p)[1] = make_float4(v[2].x, v[2].y, v[3].x, v[3].y);
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) p[k] = v[k];
  }
}

// Regroup the spectra of nb fields into quads: FT[q][s][k] = F[4q + k][s] (zero past
// the last field), so one gather of a spectral point serves four fields with one
// fully used 32-byte sector (float).  Coalesced on both sides; two spectral points per
// thread, read as one 16-byte vector per field where the row allows it.
template <typename T>
__global__ void k_group_spectra(const typename Cx<T>::type* __restrict__ F, typename Cx<T>::type* __restrict__ FT,
                                int ns, int nb) {
  pdl_enter();
  using C = typename Cx<T>::type;
  const int s0 = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  if (s0 >= ns) return;
  const bool two = s0 + 1 < ns;
  const int q = blockIdx.y;
  const C z = mk<C>(static_cast<T>(0), static_cast<T>(0));
  C v[2][4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int f = 4 * q + k;
    const C* row = F + static_cast<size_t>(f) * ns + s0;
    bool done = f >= nb;
    if (done) { v[0][k] = z; v[1][k] = z; }
    if constexpr (sizeof(C) == 8) {
      if (!done && two && (reinterpret_cast<uintptr_t>(row) & 15u) == 0) {
        const float4 u = __ldg(reinterpret_cast<const float4*>(row));
        v[0][k] = make_float2(u.x, u.y);
        v[1][k] = make_float2(u.z, u.w);
        done = true;
      }
    }
    if (!done) {
      v[0][k] = __ldg(row);
      v[1][k] = two ? __ldg(row + 1) : z;
    }
  }
  store_quad(FT + (static_cast<size_t>(q) * ns + s0) * 4, v[0]);
  if (two) store_quad(FT + (static_cast<size_t>(q) * ns + s0 + 1) * 4, v[1]);
}

// Backward inverse reconstruction for a quad of fields:
//   G0(q_o) = (1/d) sum_a ph_a F(spec_a)   (F conjugated where flagged)
// from the packed alias rows (spec+1 in bits 0-19, conj in bit 20, phase numerator in
// bits 21-31; 0 = no alias).  Two consecutive lanes take one orbit: lane k reads fields
// 4q + 2k and 4q + 2k + 1, one 16-byte half (float) of the spectral point's 32-byte
// quad in FT, so every alias gather of a warp reads whole quads and the two fields of
// a workspace slot sit in the same lane.  The d loads of a lane are independent and in
// flight together.  Lane k stores the slot input X = G_a + i G_b of its pair as
// G0P[q][o][k] (pair 0: fields 4q, 4q+1; pair 1: fields 4q+2, 4q+3).
template <typename T, int D>
__global__ void __launch_bounds__(256)
k_inv_recon_quad(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                 const uint32_t* __restrict__ inv_pk, const typename Cx<T>::type* __restrict__ FT,
                 typename Cx<T>::type* __restrict__ G0P) {
  pdl_enter();
  using C = typename Cx<T>::type;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int no = g->n_orbits;
  const int o = t >> 1, k = t & 1;
  if (o >= no) return;
  const int q = blockIdx.y;
  const C* ft = FT + static_cast<size_t>(q) * g->n_spec * 4 + 2 * k;
  const C* ph = tables + g->ph_off;
  uint32_t e[D];
  load_alias_row<D>(inv_pk, o, e);
  C v[D][2];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const uint32_t sp = e[a] & 0xFFFFFu;
    const C* src = ft + static_cast<size_t>(sp ? sp - 1 : 0) * 4;
    if constexpr (sizeof(C) == 8) {
      const float4 u = __ldg(reinterpret_cast<const float4*>(src));
      v[a][0] = mk<C>(u.x, u.y);
      v[a][1] = mk<C>(u.z, u.w);
    } else {
      v[a][0] = __ldg(src);
      v[a][1] = __ldg(src + 1);
    }
  }
  const T zero = static_cast<T>(0);
  T re[2] = {zero, zero}, im[2] = {zero, zero};
#pragma unroll
  for (int a = 0; a < D; ++a) {
    // term = v conj(w), or conj(v) conj(w) when flagged: with s = -1 if flagged,
    // re = v.x w.x + v.y (s w.y), im = v.y (s w.x) - v.x w.y.
    C w = ph[e[a] >> 21];
    if ((e[a] & 0xFFFFFu) == 0) w = mk<C>(zero, zero);
    const T sg = ((e[a] >> 20) & 1u) ? static_cast<T>(-1) : static_cast<T>(1);
    const T cA = w.x, cB = sg * w.y, cC = sg * w.x, cD = -w.y;
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      re[f] = fma(v[a][f].x, cA, fma(v[a][f].y, cB, re[f]));
      im[f] = fma(v[a][f].y, cC, fma(v[a][f].x, cD, im[f]));
    }
  }
  const T inv_d = static_cast<T>(1.0 / static_cast<double>(D));
  // X = G_a + i G_b; fields past the batch were zero-filled.
  G0P[(static_cast<size_t>(q) * no + o) * 2 + k] = mk<C>(inv_d * (re[0] - im[1]), inv_d * (im[0] + re[1]));
}

// Backward orbit expansion + inverse z FFT for a quad of fields (two workspace
// slots): the two halves of the CTA build the z lines of slots 2q and 2q+1 at the same
// (y, x) positions, X_slot(R^T q) = X_slot(q_o) e^{+2 pi i j / P}, from the packed
// expansion entries (orbit in bits 0-20, phase numerator in bits 21-31) and the
// combined representatives G0P[q][o][pair]; both halves read the same entries and
// 16-byte pairs (the second read hits L1).  The line is transformed in registers and
// stored coalesced across x.  No shared memory.  A CTA covers YB y values.
template <typename T, int H, int YB>
__global__ void k_expand4_ifft_z_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                                   const uint32_t* __restrict__ ETP, const typename Cx<T>::type* __restrict__ G0P,
                                   typename Cx<T>::type* __restrict__ W, int nfields) {
  pdl_enter();
  using C = typename Cx<T>::type;
  constexpr int HV = H * H * H;
  constexpr int kHalf = ((YB * H + 31) / 32) * 32;
  const int y0 = blockIdx.x * YB, c = blockIdx.y, q = blockIdx.z;
  const int half = threadIdx.x / kHalf, r = threadIdx.x % kHalf;
  const int slot = 2 * q + half;
  if (2 * slot >= nfields) return;
  const int ny = min(YB, H - y0);
  const int yy = r / H, x = r % H;
  if (yy >= ny) return;
  const int y = y0 + yy;
  const uint32_t* et = ETP + static_cast<size_t>(c) * HV + y * H + x;
  const C* rp = G0P + static_cast<size_t>(q) * g->n_orbits * 2 + half;
  const C* ph = tables + g->ph_off;
  C v[H];
#pragma unroll
  for (int z = 0; z < H; ++z) {
    const uint32_t t = __ldg(et + z * H * H);
    v[z] = cmulc(__ldg(rp + 2 * static_cast<size_t>(t & 0x1FFFFFu)), ph[t >> 21]);
  }
  reg_fft<C, true, H>(v);
  C* dst = W + (static_cast<size_t>(slot) * g->n_ch + c) * HV + y * H + x;
#pragma unroll
  for (int z = 0; z < H; ++z) dst[z * H * H] = v[z];
}

// ---------------------------------------------------------------- wide backward gather
// Field groups of GW = 128 / sizeof(complex) fields (16 in FP32, 8 in FP64): the
// spectrum of a group keeps the GW values of one spectral point in one 128-byte line,
// FT[g][s][k] = F[GW g + k][s], and the orbit representatives of a group keep their
// GW / 2 workspace-slot inputs in one line, G0P[g][o][j] = X of slot GW/2 g + j.  Each
// random gather of a warp then fetches whole lines that serve GW fields, a quarter of
// the L1 wavefronts per useful byte of the quad layout.
template <typename C> constexpr int wide_fields() { return static_cast<int>(128 / sizeof(C)); }
constexpr int kWideTile = 128;  // spectral points per CTA of the regroup

// Regroup of the spectra of nb fields into groups of GW: a CTA moves a tile of
// kWideTile spectral points x GW fields through shared memory (row stride GW + 1, so
// both phases are free of bank conflicts); reads are coalesced along each field's
// row, writes are whole lines.  Fields past nb are zero.
template <typename T>
__global__ void __launch_bounds__(256) k_group_spectra_w(const typename Cx<T>::type* __restrict__ F,
                                                         typename Cx<T>::type* __restrict__ FT, int ns, int nb) {
  pdl_enter();
  using C = typename Cx<T>::type;
  constexpr int GW = wide_fields<C>(), SP = kWideTile, RS = GW + 1;
  __shared__ C tile[SP * RS];
  const int s0 = blockIdx.x * SP, gq = blockIdx.y;
  const int np = min(SP, ns - s0);
  const C z = mk<C>(static_cast<T>(0), static_cast<T>(0));
  for (int e = threadIdx.x; e < SP * GW; e += blockDim.x) {
    const int f = e / SP, i = e % SP;
    const int field = gq * GW + f;
    tile[i * RS + f] = (i < np && field < nb) ? __ldg(F + static_cast<size_t>(field) * ns + s0 + i) : z;
  }
  __syncthreads();
  C* out = FT + (static_cast<size_t>(gq) * ns + s0) * GW;
  for (int e = threadIdx.x; e < np * GW; e += blockDim.x) out[e] = tile[(e / GW) * RS + (e % GW)];
}

// Backward inverse reconstruction for a group of GW fields: as k_inv_recon_quad, with
// GW / 2 lanes per orbit; lane j reads fields GW g + 2j and GW g + 2j + 1 (two
// consecutive complex of the spectral point's line), so the lanes of an orbit read
// each tap's line whole, and stores the slot input X = G_a + i G_b as G0P[g][o][j].
template <typename T, int D>
__global__ void __launch_bounds__(256)
k_inv_recon_w(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
              const uint32_t* __restrict__ inv_pk, const typename Cx<T>::type* __restrict__ FT,
              typename Cx<T>::type* __restrict__ G0P) {
  pdl_enter();
  using C = typename Cx<T>::type;
  constexpr int GW = wide_fields<C>(), L = GW / 2;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int no = g->n_orbits;
  const int o = t / L, j = t % L;
  if (o >= no) return;
  const int gq = blockIdx.y;
  const C* ft = FT + static_cast<size_t>(gq) * g->n_spec * GW + 2 * j;
  const C* ph = tables + g->ph_off;
  uint32_t e[D];
  load_alias_row<D>(inv_pk, o, e);
  C v[D][2];
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const uint32_t sp = e[a] & 0xFFFFFu;
    const C* src = ft + static_cast<size_t>(sp ? sp - 1 : 0) * GW;
    if constexpr (sizeof(C) == 8) {
      const float4 u = __ldg(reinterpret_cast<const float4*>(src));
      v[a][0] = mk<C>(u.x, u.y);
      v[a][1] = mk<C>(u.z, u.w);
    } else {
      v[a][0] = __ldg(src);
      v[a][1] = __ldg(src + 1);
    }
  }
  const T zero = static_cast<T>(0);
  T re[2] = {zero, zero}, im[2] = {zero, zero};
#pragma unroll
  for (int a = 0; a < D; ++a) {
    C w = ph[e[a] >> 21];
    if ((e[a] & 0xFFFFFu) == 0) w = mk<C>(zero, zero);
    const T sg = ((e[a] >> 20) & 1u) ? static_cast<T>(-1) : static_cast<T>(1);
    const T cA = w.x, cB = sg * w.y, cC = sg * w.x, cD = -w.y;
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      re[f] = fma(v[a][f].x, cA, fma(v[a][f].y, cB, re[f]));
      im[f] = fma(v[a][f].y, cC, fma(v[a][f].x, cD, im[f]));
    }
  }
  const T inv_d = static_cast<T>(1.0 / static_cast<double>(D));
  G0P[(static_cast<size_t>(gq) * no + o) * L + j] = mk<C>(inv_d * (re[0] - im[1]), inv_d * (im[0] + re[1]));
}

// Backward orbit expansion + inverse z FFT for a group of GW fields (GW / 2 slots): a
// CTA takes one (y, c, group); thread (x, j) builds the z line of slot GW/2 g + j at
// (y, x) from the packed expansion entries and G0P[g][orbit][j] (the GW / 2 lanes of
// one x read one orbit's line), transforms it in registers and stores it to
// W[slot][c][z][y][x].  Launched with GW / 2 * H threads.
template <typename T, int H>
__global__ void __launch_bounds__(wide_fields<typename Cx<T>::type>() / 2 * H)
k_expand_w_ifft_z_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ tables,
                    const uint32_t* __restrict__ ETP, const typename Cx<T>::type* __restrict__ G0P,
                    typename Cx<T>::type* __restrict__ W, int nfields) {
  pdl_enter();
  using C = typename Cx<T>::type;
  constexpr int GW = wide_fields<C>(), L = GW / 2, HV = H * H * H;
  const int y = blockIdx.x, c = blockIdx.y, gq = blockIdx.z;
  const int j = threadIdx.x % L, x = threadIdx.x / L;
  const int slot = gq * L + j;
  if (2 * slot >= nfields) return;
  const uint32_t* et = ETP + static_cast<size_t>(c) * HV + y * H + x;
  const C* rp = G0P + static_cast<size_t>(gq) * g->n_orbits * L + j;
  const C* ph = tables + g->ph_off;
  C v[H];
#pragma unroll
  for (int z = 0; z < H; ++z) {
    const uint32_t t = __ldg(et + z * H * H);
    v[z] = cmulc(__ldg(rp + static_cast<size_t>(L) * (t & 0x1FFFFFu)), ph[t >> 21]);
  }
  reg_fft<C, true, H>(v);
  C* dst = W + (static_cast<size_t>(slot) * g->n_ch + c) * HV + y * H + x;
#pragma unroll
  for (int z = 0; z < H; ++z) dst[z * H * H] = v[z];
}

// Q-matrix diffusion step (execute_m2_q! / execute_m7_scft!, src/q_fused_krfft.jl:553-667,
// 870-895): for every channel point (c, x, y, z) of a slot, q its subgrid position,
//   Y'(q) = sum_b Q_b(q) G0(R_b^T q mod M)
// with G0 gathered from the forward workspace WT (z-fastest; index -1 marks a parity
// class without a channel, where G0 = 0), assembled as the z line of (c, y, x), inverse z
// FFT in registers, stored W2[slot][c][z][y][x] for the inverse plane kernel.  Both
// fields of the slot (G0_a + i G0_b) go through the same complex-linear map.
template <typename T, int H>
__global__ void k_qmul_ifft_z_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ QT,
                                const int32_t* __restrict__ GT, const typename Cx<T>::type* __restrict__ WT,
                                typename Cx<T>::type* __restrict__ W2) {
  pdl_enter();
  using C = typename Cx<T>::type;
  constexpr int HV = H * H * H;
  const int y0 = blockIdx.x * kZB, c = blockIdx.y, slot = blockIdx.z;
  const int ny = min(kZB, H - y0);
  const int yy = threadIdx.x / H, x = threadIdx.x % H;
  if (yy >= ny) return;
  const int y = y0 + yy;
  const int d = g->d;
  const size_t np = static_cast<size_t>(g->n_ch) * HV;
  const C* wt = WT + static_cast<size_t>(slot) * g->n_ch * HV;
  C v[H];
#pragma unroll
  for (int z = 0; z < H; ++z) {
    const size_t pos = static_cast<size_t>(c) * HV + (z * H + y) * H + x;
    C acc = mk<C>(static_cast<T>(0), static_cast<T>(0));
#pragma unroll
    for (int b = 0; b < 8; ++b) {
      if (b < d) {
        const int32_t gi = __ldg(GT + b * np + pos);
        if (gi >= 0) acc = cadd(acc, cmul(__ldg(QT + b * np + pos), __ldg(wt + gi)));
      }
    }
    v[z] = acc;
  }
  reg_fft<C, true, H>(v);
  C* dst = W2 + (static_cast<size_t>(slot) * g->n_ch + c) * HV + y * H + x;
#pragma unroll
  for (int z = 0; z < H; ++z) dst[z * H * H] = v[z];
}

// Separable Q-multiply of the M2Q step for Pmmm-like plans (_q_multiply_separable!,
// src/q_fused_krfft.jl:606-667; detection _is_pmmm_like, :431-454): d = 8, L = (2, 2, 2),
// the representatives diag(s) with translations 0 or -1, and an orthogonal cell.  Then
// B = WHT8 diag(tw^alpha) and the first row of Q = B^-1 diag(K) B gives
//   Y'(q) = (1/8) sum_m K(q + M alpha_m) [WHT8 (tw^alpha_a(q) Y(s_a q mod M))]_m,
// tw_d(q) = e^{2 pi i q_d / N_d}, K(h) = prod_d exp(-ds (2 pi h_c,d / a_d)^2).  Nothing is
// tabulated per point: QS holds the 1-D twiddles (3 x H complex) and the 1-D kernel
// factors (3 x 2H, real parts).  Same line structure as k_qmul_ifft_z_h (plain path,
// one channel, H = M): the z line of (y, x) is assembled, inverse z FFT, stored to W2.
template <typename T, int H>
__global__ void k_qsep_ifft_z_h(const DevGeom* __restrict__ g, const typename Cx<T>::type* __restrict__ QS,
                                const typename Cx<T>::type* __restrict__ WT, typename Cx<T>::type* __restrict__ W2) {
  pdl_enter();
  using C = typename Cx<T>::type;
  constexpr int HV = H * H * H;
  const int y0 = blockIdx.x * kZB, slot = blockIdx.z;
  const int ny = min(kZB, H - y0);
  const int yy = threadIdx.x / H, x = threadIdx.x % H;
  if (yy >= ny) return;
  const int y = y0 + yy;
  const C* wt = WT + static_cast<size_t>(slot) * HV;
  const C* tw = QS;              // tw[d * H + q]
  const C* kf = QS + 3 * H;      // kf[d * 2H + h].x
  int neg[8];                    // bit d: axis d negated by representative a
#pragma unroll
  for (int a = 0; a < 8; ++a)
    neg[a] = (g->rep_R[a][0] < 0 ? 1 : 0) | (g->rep_R[a][4] < 0 ? 2 : 0) | (g->rep_R[a][8] < 0 ? 4 : 0);
  const int xm = x ? H - x : 0, ym = y ? H - y : 0;
  const C twx = tw[x], twy = tw[H + y];
  const T kx0 = kf[x].x, kx1 = kf[x + H].x, ky0 = kf[2 * H + y].x, ky1 = kf[2 * H + y + H].x;
  const C txy = cmul(twx, twy);
  C v[H];
#pragma unroll
  for (int z = 0; z < H; ++z) {
    const int zm = z ? H - z : 0;
    const C twz = tw[2 * H + z];
    C p[8];
#pragma unroll
    for (int a = 0; a < 8; ++a) {
      const int gx = (neg[a] & 1) ? xm : x, gy = (neg[a] & 2) ? ym : y, gz = (neg[a] & 4) ? zm : z;
      p[a] = wt[(gx * H + gy) * H + gz];
    }
    p[1] = cmul(p[1], twx);
    p[2] = cmul(p[2], twy);
    p[3] = cmul(p[3], txy);
    p[4] = cmul(p[4], twz);
    p[5] = cmul(p[5], cmul(twx, twz));
    p[6] = cmul(p[6], cmul(twy, twz));
    p[7] = cmul(p[7], cmul(txy, twz));
    wht8c(p);
    const T kz0 = kf[4 * H + z].x, kz1 = kf[4 * H + z + H].x;
    const T k00 = kx0 * ky0, k10 = kx1 * ky0, k01 = kx0 * ky1, k11 = kx1 * ky1;
    const T km[8] = {k00 * kz0, k10 * kz0, k01 * kz0, k11 * kz0, k00 * kz1, k10 * kz1, k01 * kz1, k11 * kz1};
    C acc = cscale(p[0], km[0]);
#pragma unroll
    for (int m = 1; m < 8; ++m) acc = cadd(acc, cscale(p[m], km[m]));
    v[z] = cscale(acc, static_cast<T>(0.125));
  }
  reg_fft<C, true, H>(v);
  C* dst = W2 + static_cast<size_t>(slot) * HV + y * H + x;
#pragma unroll
  for (int z = 0; z < H; ++z) dst[z * H * H] = v[z];
}

constexpr int kMaxDynSmemFast = 227 * 1024;

// Programmatic dependent launch of the fast-path kernels (off with CFFT_PDL=0): each
// kernel of a lane may launch while its predecessor in the stream is finishing, and
// waits for it in hardware (griddepcontrol.wait, pdl_wait below) before touching memory.
inline bool pdl_enabled() {
  static const bool on = [] {
    const char* e = std::getenv("CFFT_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}
// First failure of a launch_k launch on this thread since fast_unit_launch last read it.
inline cudaError_t& launch_error() {
  static thread_local cudaError_t e = cudaSuccess;
  return e;
}
template <typename... KArgs, typename... Args>
inline void launch_k(void (*k)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args&&... args) {
  if (pdl_enabled()) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, k, std::forward<Args>(args)...);
    if (e != cudaSuccess && launch_error() == cudaSuccess) launch_error() = e;
  } else {
    k<<<grid, block, smem, st>>>(std::forward<Args>(args)...);
  }
}

// Persistent bulk-copy plane kernels (tma_planes.cuh).  They serve centred plans with
// H >= 16 whose per-group stage and buffer fit at least two groups into one CTA's
// shared memory.  CFFT_TMA selects them: "fwd" (the forward plane stage), "all" (both
// stages), unset or "0" (neither).  Measured on Im-3m 128^3 FP32 (B200): the forward
// one is 2-5% slower than the per-plane kernel and the backward one 30% slower -- with
// one 195 KB CTA per SM they run 8 and 12 warps per SM against the per-plane kernels'
// 20, and the FFT phases, not the loads, bound the stage -- so both are opt-in.
inline int tma_mode() {  // bit 0: forward, bit 1: backward
  static const int m = [] {
    const char* e = std::getenv("CFFT_TMA");
    if (!e) return 0;
    if (e[0] == '0') return 0;
    if (e[0] == 'a' || e[0] == '1') return 3;
    if (e[0] == 'b') return 2;
    return 1;
  }();
  return m;
}
inline bool tma_enabled() { return tma_mode() != 0; }
template <typename T, int H, int CT, bool USE_E>
constexpr bool fwd_tma_fits() {
  if constexpr (CT == 0 || H < 16 || H % (16 / static_cast<int>(sizeof(T))) != 0) return false;
  else return tma_groups<FwdTmaShape<T, H, CT, USE_E>>() >= 2;
}
template <typename T, int H, int CT>
constexpr bool bwd_tma_fits() {
  if constexpr (CT == 0 || H < 16 || H % (16 / static_cast<int>(sizeof(T))) != 0) return false;
  else return tma_groups<BwdTmaShape<T, H, CT>>() >= 2;
}
// Persistent grid of a bulk-copy plane kernel: every SM's resident CTAs, or fewer when
// the tasks run out.  The resident count is looked up once per kernel and device (the
// kernels of different H share a function type, so the cache is keyed by address) under
// a lock, since plans may be executed from several host threads.
template <typename K>
int tma_grid(K kernel, int threads, size_t smem, int ntasks, int ng) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, int> resident;
  int dev = 0;
  cudaGetDevice(&dev);
  int cap = 1;
  {
    std::lock_guard<std::mutex> lock(mu);
    const auto key = std::make_pair(reinterpret_cast<const void*>(kernel), dev);
    auto it = resident.find(key);
    if (it == resident.end()) {
      int occ = 0, sms = 0;
      if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) sms = 1;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem) != cudaSuccess) occ = 1;
      it = resident.emplace(key, std::max(1, occ) * std::max(1, sms)).first;
    }
    cap = it->second;
  }
  const int need = (ntasks + ng - 1) / ng;
  return std::max(1, std::min(need, cap));
}

// Workspace slots per CTA of the fused z FFT + gather: 4, or 2 with CFFT_ZR_SLOTS=2
// (measured on Im-3m 128^3 FP32: 4 slots slightly ahead).
inline int zr_slots() {
  static const int n = [] {
    const char* e = std::getenv("CFFT_ZR_SLOTS");
    return (e && e[0] == '2') ? 2 : 4;
  }();
  return n;
}


#define CFFT_FOR_H(H, ...)                                                        \
  switch (H) {                                                                    \
    case 4: { constexpr int HH = 4; __VA_ARGS__; } break;                         \
    case 6: { constexpr int HH = 6; __VA_ARGS__; } break;                         \
    case 8: { constexpr int HH = 8; __VA_ARGS__; } break;                         \
    case 12: { constexpr int HH = 12; __VA_ARGS__; } break;                       \
    case 16: { constexpr int HH = 16; __VA_ARGS__; } break;                       \
    case 24: { constexpr int HH = 24; __VA_ARGS__; } break;                       \
    case 32: { constexpr int HH = 32; __VA_ARGS__; } break;                       \
    default: { constexpr int HH = sizeof(T) == 4 ? 48 : 32; __VA_ARGS__; } break; \
  }

#define CFFT_FOR_M(M, ...)                                        \
  switch (M) {                                                     \
    case 4: { constexpr int MM = 4; __VA_ARGS__; } break;         \
    case 6: { constexpr int MM = 6; __VA_ARGS__; } break;         \
    case 8: { constexpr int MM = 8; __VA_ARGS__; } break;         \
    case 12: { constexpr int MM = 12; __VA_ARGS__; } break;       \
    case 16: { constexpr int MM = 16; __VA_ARGS__; } break;       \
    case 24: { constexpr int MM = 24; __VA_ARGS__; } break;       \
    case 32: { constexpr int MM = 32; __VA_ARGS__; } break;       \
    case 48: { constexpr int MM = 48; __VA_ARGS__; } break;       \
    case 64: { constexpr int MM = 64; __VA_ARGS__; } break;       \
    default: { constexpr int MM = 96; __VA_ARGS__; } break;       \
  }

#define CFFT_FOR_CT(CTV, ...)                                      \
  switch (CTV) {                                                   \
    case 1: { constexpr int CTT = 1; __VA_ARGS__; } break;         \
    case 2: { constexpr int CTT = 2; __VA_ARGS__; } break;         \
    case 3: { constexpr int CTT = 3; __VA_ARGS__; } break;         \
    case 4: { constexpr int CTT = 4; __VA_ARGS__; } break;         \
    default: { constexpr int CTT = 0; __VA_ARGS__; } break;        \
  }

inline Status fast_cuda(cudaError_t e, const char* what, std::string* err) {
  if (e == cudaSuccess) return Status::kOk;
  *err = std::string(what) + ": " + cudaGetErrorString(e);
  return Status::kCuda;
}

// Cluster kernels: attributes, launch (cluster size at run time, through
// cudaLaunchKernelEx) and occupancy, for the instantiations that fit.
template <typename T, int H, int CT, int KC>
void cluster_attrs() {
  if constexpr (cluster_fits<T, H, CT, KC>()) {
    const int smem = static_cast<int>(cluster_smem<T, H, CT, KC>());
    cudaFuncSetAttribute(k_fwd_cluster_h<T, H, CT, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaFuncSetAttribute(k_bwd_cluster_h<T, H, CT, KC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (KC > 8) {
      cudaFuncSetAttribute(k_fwd_cluster_h<T, H, CT, KC>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      cudaFuncSetAttribute(k_bwd_cluster_h<T, H, CT, KC>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    }
  }
}

template <typename T, int H, int CT, int KC>
cudaLaunchConfig_t cluster_config(int nslots, cudaStream_t st, cudaLaunchAttribute* attr) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(KC, static_cast<unsigned>(nslots), 1);
  cfg.blockDim = dim3(ClusterShape<H, CT, KC>::threads, 1, 1);
  cfg.dynamicSmemBytes = cluster_smem<T, H, CT, KC>();
  cfg.stream = st;
  attr->id = cudaLaunchAttributeClusterDimension;
  attr->val.clusterDim.x = KC;
  attr->val.clusterDim.y = 1;
  attr->val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cfg;
}

template <typename T, int H, int CT, int KC>
bool cluster_launch(int stage, int nslots, cudaStream_t st, const DevGeom* g, const typename Cx<T>::type* tab,
                    const T* f0, const T* E, typename Cx<T>::type* W, const uint32_t* ETP,
                    const typename Cx<T>::type* G0P, T* f0_out, int nb, cudaError_t* ce) {
  if constexpr (cluster_fits<T, H, CT, KC>()) {
    cudaLaunchAttribute attr;
    const cudaLaunchConfig_t cfg = cluster_config<T, H, CT, KC>(nslots, st, &attr);
    if (stage == 0) *ce = cudaLaunchKernelEx(&cfg, k_fwd_cluster_h<T, H, CT, KC>, g, tab, f0, E, W, nb);
    else *ce = cudaLaunchKernelEx(&cfg, k_bwd_cluster_h<T, H, CT, KC>, g, tab, ETP, G0P, E, f0_out, nb);
    return true;
  }
  return false;
}

template <typename T, int H, int CT, int KC>
cudaError_t cluster_occupancy(int* max_clusters) {
  if constexpr (cluster_fits<T, H, CT, KC>()) {
    cudaLaunchAttribute attr;
    const cudaLaunchConfig_t cfg = cluster_config<T, H, CT, KC>(1, nullptr, &attr);
    int nf = 0, nbk = 0;
    cudaError_t e = cudaOccupancyMaxActiveClusters(&nf, k_fwd_cluster_h<T, H, CT, KC>, &cfg);
    if (e == cudaSuccess) e = cudaOccupancyMaxActiveClusters(&nbk, k_bwd_cluster_h<T, H, CT, KC>, &cfg);
    if (e == cudaSuccess) *max_clusters = std::min(nf, nbk);
    return e;
  }
  *max_clusters = 0;
  return cudaSuccess;
}

// Per-device set-up of this unit: its own copy of the constant-memory twiddles
// e^{-2 pi i j / N} (FP64 values rounded) and the shared-memory limits of its kernels.
template <typename T, int GROUP>
Status fast_unit_init(std::string* err) {
  static std::mutex mu;
  static bool done[64] = {false};
  int dev = 0;
  Status s = fast_cuda(cudaGetDevice(&dev), "cudaGetDevice", err);
  if (s != Status::kOk) return s;
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
  if ((s = fast_cuda(cudaMemcpyToSymbol(c_tw_f, tf.data(), sizeof(float2) * kTwTotal), "upload twiddles", err)) != Status::kOk) return s;
  if ((s = fast_cuda(cudaMemcpyToSymbol(c_tw_d, td.data(), sizeof(double2) * kTwTotal), "upload twiddles", err)) != Status::kOk) return s;
  for (int H : {4, 6, 8, 12, 16, 24, 32, 48}) {
    if (!fast_size_ok(H, sizeof(T))) continue;
    CFFT_FOR_H(H, {
      if constexpr (GROUP == 0) {
        for (int ct = 0; ct < 5; ++ct) {
          CFFT_FOR_CT(ct, {
            cudaFuncSetAttribute(k_plane_fwd_h<T, HH, CTT>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemFast);
            cudaFuncSetAttribute(k_plane_bwd_h<T, HH, CTT, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemFast);
            // The bulk-copy kernels also hold a little static shared memory, so their
            // dynamic limit is their exact need; a refusal is reported.
            cudaError_t te = cudaSuccess;
            if constexpr (fwd_tma_fits<T, HH, CTT, false>()) {
              using SH = FwdTmaShape<T, HH, CTT, false>;
              constexpr int NG = tma_groups<SH>();
              te = cudaFuncSetAttribute(k_plane_fwd_tma<T, HH, CTT, NG, false>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(NG * SH::group));
            }
            if constexpr (fwd_tma_fits<T, HH, CTT, true>()) {
              using SH = FwdTmaShape<T, HH, CTT, true>;
              constexpr int NG = tma_groups<SH>();
              if (te == cudaSuccess)
                te = cudaFuncSetAttribute(k_plane_fwd_tma<T, HH, CTT, NG, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(NG * SH::group));
            }
            if constexpr (bwd_tma_fits<T, HH, CTT>()) {
              using SH = BwdTmaShape<T, HH, CTT>;
              constexpr int NG = tma_groups<SH>();
              if (te == cudaSuccess)
                te = cudaFuncSetAttribute(k_plane_bwd_tma<T, HH, CTT, NG>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(NG * SH::group));
            }
            if (te != cudaSuccess) return fast_cuda(te, "bulk-copy plane kernel shared-memory attribute", err);
            cluster_attrs<T, HH, CTT, 8>();
            cluster_attrs<T, HH, CTT, 16>();
          });
        }
      } else {
        cudaFuncSetAttribute(k_fft_z_fwd_h<T, HH>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemFast);
        // The fused kernel also holds 96 bytes of static shared memory; its dynamic
        // share above 48 KB (FP64, 4 slots) needs the attribute, so failures are reported.
        {
          constexpr int kZr = kMaxDynSmemFast - 1024;
          cudaError_t ze = cudaFuncSetAttribute(k_fft_z_recon_diag8<T, HH, 2, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kZr);
          if (ze == cudaSuccess) ze = cudaFuncSetAttribute(k_fft_z_recon_diag8<T, HH, 2, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kZr);
          if (ze == cudaSuccess) ze = cudaFuncSetAttribute(k_fft_z_recon_diag8<T, HH, 4, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kZr);
          if (ze == cudaSuccess) ze = cudaFuncSetAttribute(k_fft_z_recon_diag8<T, HH, 4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kZr);
          if (ze != cudaSuccess) return fast_cuda(ze, "fused z FFT + gather shared-memory attribute", err);
        }
        cudaFuncSetAttribute(k_expand_ifft_z_h<T, HH>, cudaFuncAttributeMaxDynamicSharedMemorySize, kMaxDynSmemFast);
      }
    });
  }
  if ((s = fast_cuda(cudaGetLastError(), "set shared-memory attributes", err)) != Status::kOk) return s;
  if (dev >= 0 && dev < 64) done[dev] = true;
  return Status::kOk;
}

// Occupancy of the fused cluster kernels with KC CTAs per cluster: resident clusters
// (the smaller of the forward and backward kernels), 0 when they do not fit.
template <typename T>
Status fast_unit_cluster_probe(int H, int ct, int kc, int* max_clusters, std::string* err) {
  *max_clusters = 0;
  Status s = fast_unit_init<T, 0>(err);
  if (s != Status::kOk) return s;
  cudaError_t e = cudaSuccess;
  CFFT_FOR_H(H, {
    CFFT_FOR_CT(ct, {
      if (kc == 16) e = cluster_occupancy<T, HH, CTT, 16>(max_clusters);
      else e = cluster_occupancy<T, HH, CTT, 8>(max_clusters);
    });
  });
  if (e != cudaSuccess) {  // e.g. a cluster size this device does not allow: not used
    cudaGetLastError();
    *max_clusters = 0;
  }
  return Status::kOk;
}

template <typename T>
void fast_unit_tma_planes(int H, int ct, int tma, bool* fwd, bool* fwd_e, bool* bwd) {
  *fwd = *fwd_e = *bwd = false;
  const int mode = tma >= 0 ? tma : tma_mode();
  if (!mode || !fast_size_ok(H, sizeof(T))) return;
  CFFT_FOR_H(H, {
    CFFT_FOR_CT(ct, {
      *fwd = (mode & 1) && fwd_tma_fits<T, HH, CTT, false>();
      *fwd_e = (mode & 1) && fwd_tma_fits<T, HH, CTT, true>();
      *bwd = (mode & 2) && bwd_tma_fits<T, HH, CTT>();
    });
  });
}

// One fast-path stage for `a.nb` fields (two per workspace slot).
template <typename T, int GROUP>
Status fast_unit_launch(const FastArgs& a, std::string* err) {
  using C = typename Cx<T>::type;
  const DevGeom* g = static_cast<const DevGeom*>(a.geom);
  const C* tab = static_cast<const C*>(a.tables);
  C* W = static_cast<C*>(a.W);
  C* G0R = static_cast<C*>(a.G0R);
  const T* f0 = static_cast<const T*>(a.f0);
  const T* E = static_cast<const T*>(a.E);
  C* F = static_cast<C*>(a.F);
  const C* Fin = static_cast<const C*>(a.Fin);
  T* f0_out = static_cast<T*>(a.f0_out);
  cudaStream_t st = static_cast<cudaStream_t>(a.stream);
  const int H = a.H, nb = a.nb, nch = a.n_ch;
  const int nslots = (nb + 1) / 2;
  const size_t cs = sizeof(C);
  if constexpr (GROUP == 0) {
    if (a.cluster) {
      bool launched = false;
      cudaError_t ce = cudaSuccess;
      CFFT_FOR_H(H, {
        CFFT_FOR_CT(a.cent_type, {
          if (a.cluster_ctas == 16) {
            launched = cluster_launch<T, HH, CTT, 16>(a.stage, nslots, st, g, tab, f0, E, W,
                                                      static_cast<const uint32_t*>(a.expand), G0R, f0_out, nb, &ce);
          } else {
            launched = cluster_launch<T, HH, CTT, 8>(a.stage, nslots, st, g, tab, f0, E, W,
                                                     static_cast<const uint32_t*>(a.expand), G0R, f0_out, nb, &ce);
          }
        });
      });
      if (!launched) {
        *err = "no fused cluster kernel for this channel grid";
        return Status::kUnsupported;
      }
      if (ce != cudaSuccess) return fast_cuda(ce, "fused cluster launch", err);
      return fast_cuda(cudaGetLastError(), "fused cluster launch", err);
    }
    const int thr_plane = std::max(128, ((nch * H + 31) / 32) * 32);
    const size_t smem_plane = static_cast<size_t>(nch) * H * (H + 1) * cs;
    const int ntasks = nslots * H;
    auto al16 = [](const void* p) { return p == nullptr || (reinterpret_cast<uintptr_t>(p) & 15u) == 0; };
    const int tmode = a.tma >= 0 ? a.tma : tma_mode();
    const bool tma = al16(f0) && al16(E) && al16(f0_out) && al16(W) && (tmode & (a.stage == 0 ? 1 : 2));
    if (a.stage == 0) {
      CFFT_FOR_H(H, {
        CFFT_FOR_CT(a.cent_type, {
          bool done = false;
          if (tma && E == nullptr) {
            if constexpr (fwd_tma_fits<T, HH, CTT, false>()) {
              using SH = FwdTmaShape<T, HH, CTT, false>;
              constexpr int NG = tma_groups<SH>();
              auto* k = k_plane_fwd_tma<T, HH, CTT, NG, false>;
              const int grid = tma_grid(k, NG * SH::threads, NG * SH::group, ntasks, NG);
              launch_k(k, dim3(grid), NG * SH::threads, NG * SH::group, st, g, tab, f0, E, W, nb, ntasks,
                       static_cast<uint64_t>(a.timeout_ns), a.status);
              done = true;
            }
          } else if (tma) {
            if constexpr (fwd_tma_fits<T, HH, CTT, true>()) {
              using SH = FwdTmaShape<T, HH, CTT, true>;
              constexpr int NG = tma_groups<SH>();
              auto* k = k_plane_fwd_tma<T, HH, CTT, NG, true>;
              const int grid = tma_grid(k, NG * SH::threads, NG * SH::group, ntasks, NG);
              launch_k(k, dim3(grid), NG * SH::threads, NG * SH::group, st, g, tab, f0, E, W, nb, ntasks,
                       static_cast<uint64_t>(a.timeout_ns), a.status);
              done = true;
            }
          }
          if (!done)
            launch_k(k_plane_fwd_h<T, HH, CTT>, dim3(H, nslots), thr_plane, smem_plane, st, g, tab, f0, E, W, nb);
        });
      });
    } else {
      CFFT_FOR_H(H, {
        CFFT_FOR_CT(a.cent_type, {
          bool done = false;
          if (tma) {
            if constexpr (bwd_tma_fits<T, HH, CTT>()) {
              using SH = BwdTmaShape<T, HH, CTT>;
              constexpr int NG = tma_groups<SH>();
              auto* k = k_plane_bwd_tma<T, HH, CTT, NG>;
              const int grid = tma_grid(k, NG * SH::threads, NG * SH::group, ntasks, NG);
              launch_k(k, dim3(grid), NG * SH::threads, NG * SH::group, st, g, tab, static_cast<const C*>(W), E, f0_out,
                       nb, ntasks, static_cast<uint64_t>(a.timeout_ns), a.status);
              done = true;
            }
          }
          if (!done)
            launch_k(k_plane_bwd_h<T, HH, CTT, true>, dim3(H, nslots), thr_plane, smem_plane, st, g, tab, W, E, f0_out, nb);
        });
      });
    }
  } else {
    const int thr_z = std::max(64, ((kZB * H + 31) / 32) * 32);
    const size_t smem_z = static_cast<size_t>(kZB) * H * (H + 1) * cs;
    const dim3 gz((H + kZB - 1) / kZB, nch, nslots);
    switch (a.stage) {
      case 1:
        CFFT_FOR_H(H, { launch_k(k_fft_z_fwd_h<T, HH>, gz, z_threads<HH>(), smem_z, st, g, W, W); });
        break;
      case 2: {
        const dim3 gr((a.n_spec + 255) / 256, nslots);
        const int M = a.centered ? 2 * H : H;
        const T* K = static_cast<const T*>(a.K);
        const uint32_t* sh = static_cast<const uint32_t*>(a.spec_h);
        const bool use_K = a.use_K, perm = a.rep_perm;
        if (a.rep_diag8) {
          const dim3 gd((a.n_spec + 255) / 256, (nslots + kDiagSlots - 1) / kDiagSlots);
          CFFT_FOR_M(M, {
            if (use_K) launch_k(k_recon_diag8<T, MM, true>, gd, 256, 0, st, g, tab, sh, K, W, F, nb);
            else launch_k(k_recon_diag8<T, MM, false>, gd, 256, 0, st, g, tab, sh, nullptr, W, F, nb);
          });
          break;
        }
#define CFFT_RECON_D(DD)                                                                                  \
  CFFT_FOR_M(M, {                                                                                         \
    if (use_K) {                                                                                          \
      if (perm) launch_k(k_recon_h<T, MM, DD, true, true>, gr, 256, 0, st, g, tab, sh, K, W, F, nb);            \
      else launch_k(k_recon_h<T, MM, DD, true, false>, gr, 256, 0, st, g, tab, sh, K, W, F, nb);                \
    } else {                                                                                              \
      if (perm) launch_k(k_recon_h<T, MM, DD, false, true>, gr, 256, 0, st, g, tab, sh, nullptr, W, F, nb);     \
      else launch_k(k_recon_h<T, MM, DD, false, false>, gr, 256, 0, st, g, tab, sh, nullptr, W, F, nb);         \
    }                                                                                                     \
  })
        switch (a.d) {
          case 1: CFFT_RECON_D(1); break;
          case 2: CFFT_RECON_D(2); break;
          case 4: CFFT_RECON_D(4); break;
          default: CFFT_RECON_D(8); break;
        }
#undef CFFT_RECON_D
        break;
      }
      case 6: {
        // fused z FFT + diagonal-sign gather, ZR_SLOTS workspace slots per CTA
        const int sl = a.zr_slots == 2 || a.zr_slots == 4 ? a.zr_slots : zr_slots();
        const T* K = static_cast<const T*>(a.K);
        const uint32_t* sh = static_cast<const uint32_t*>(a.spec_h);
        const uint4* un = static_cast<const uint4*>(a.zr_units);
        const uint32_t* pt = static_cast<const uint32_t*>(a.zr_pts);
        const C* Wc = W;
        CFFT_FOR_H(H, {
          const size_t sm = static_cast<size_t>(sl) * 2 * HH * (HH + 1) * cs;
          const dim3 gzr(a.zr_n_units, (nslots + sl - 1) / sl);
          if (sl == 4) {
            if (a.use_K) launch_k(k_fft_z_recon_diag8<T, HH, 4, true>, gzr, zr_threads<HH>(4), sm, st, g, tab, sh, K, un, pt, Wc, F, nb);
            else launch_k(k_fft_z_recon_diag8<T, HH, 4, false>, gzr, zr_threads<HH>(4), sm, st, g, tab, sh, nullptr, un, pt, Wc, F, nb);
          } else {
            if (a.use_K) launch_k(k_fft_z_recon_diag8<T, HH, 2, true>, gzr, zr_threads<HH>(2), sm, st, g, tab, sh, K, un, pt, Wc, F, nb);
            else launch_k(k_fft_z_recon_diag8<T, HH, 2, false>, gzr, zr_threads<HH>(2), sm, st, g, tab, sh, nullptr, un, pt, Wc, F, nb);
          }
        });
        break;
      }
      case 3: {
        const int no = a.n_orbits;
        if (a.reps_wide) {
          constexpr int GW = wide_fields<C>();
          const int ng = (nb + GW - 1) / GW;
          C* FT = static_cast<C*>(a.FT);
          launch_k(k_group_spectra_w<T>, dim3((a.n_spec + kWideTile - 1) / kWideTile, ng), 256, 0, st, Fin, FT,
                   a.n_spec, nb);
          const dim3 gw((GW / 2 * no + 255) / 256, ng);
          const uint32_t* pk = static_cast<const uint32_t*>(a.inv_pk);
          switch (a.d) {
            case 1: launch_k(k_inv_recon_w<T, 1>, gw, 256, 0, st, g, tab, pk, FT, G0R); break;
            case 2: launch_k(k_inv_recon_w<T, 2>, gw, 256, 0, st, g, tab, pk, FT, G0R); break;
            case 4: launch_k(k_inv_recon_w<T, 4>, gw, 256, 0, st, g, tab, pk, FT, G0R); break;
            default: launch_k(k_inv_recon_w<T, 8>, gw, 256, 0, st, g, tab, pk, FT, G0R); break;
          }
          break;
        }
        if (a.reps_quad) {
          const int nq = (nb + 3) / 4;
          C* FT = static_cast<C*>(a.FT);
          launch_k(k_group_spectra<T>, dim3((a.n_spec + 511) / 512, nq), 256, 0, st, Fin, FT, a.n_spec, nb);
          const dim3 gq((2 * no + 255) / 256, nq);
          const uint32_t* pk = static_cast<const uint32_t*>(a.inv_pk);
          switch (a.d) {
            case 1: launch_k(k_inv_recon_quad<T, 1>, gq, 256, 0, st, g, tab, pk, FT, G0R); break;
            case 2: launch_k(k_inv_recon_quad<T, 2>, gq, 256, 0, st, g, tab, pk, FT, G0R); break;
            case 4: launch_k(k_inv_recon_quad<T, 4>, gq, 256, 0, st, g, tab, pk, FT, G0R); break;
            default: launch_k(k_inv_recon_quad<T, 8>, gq, 256, 0, st, g, tab, pk, FT, G0R); break;
          }
          break;
        }
        launch_k(k_inv_recon_reps<T>, dim3((no + 127) / 128, (nslots + kRepSlots - 1) / kRepSlots), 128, 0, st, 
            g, tab, static_cast<const int32_t*>(a.inv_spec), static_cast<const int32_t*>(a.inv_phase), Fin, G0R, nb);
        break;
      }
      default:
        if (a.q_step && a.qsep) {
          CFFT_FOR_H(H, {
            launch_k(k_qsep_ifft_z_h<T, HH>, gz, thr_z, 0, st, g, static_cast<const C*>(a.QS), W,
                     static_cast<C*>(a.W2));
          });
          break;
        }
        if (a.q_step) {
          CFFT_FOR_H(H, {
            launch_k(k_qmul_ifft_z_h<T, HH>, gz, thr_z, 0, st, g, static_cast<const C*>(a.QT),
                                                         static_cast<const int32_t*>(a.GT), W,
                                                         static_cast<C*>(a.W2));
          });
          break;
        }
        CFFT_FOR_H(H, {
          if (a.reps_wide) {
            constexpr int GW = wide_fields<C>();
            launch_k(k_expand_w_ifft_z_h<T, HH>, dim3(HH, nch, (nb + GW - 1) / GW), GW / 2 * HH, 0, st, g, tab,
                     static_cast<const uint32_t*>(a.expand), G0R, W, nb);
          } else if (a.reps_quad) {
            // two y values per CTA (128 threads at H = 32): 5 CTAs per SM at this kernel's registers
            constexpr int half = ((2 * HH + 31) / 32) * 32;
            launch_k(k_expand4_ifft_z_h<T, HH, 2>, dim3((HH + 1) / 2, nch, (nb + 3) / 4), 2 * half, 0, st, 
                g, tab, static_cast<const uint32_t*>(a.expand), G0R, W, nb);
          } else
            launch_k(k_expand_ifft_z_h<T, HH>, gz, thr_z, smem_z, st, g, tab, static_cast<const int2*>(a.expand), G0R, W);
        });
        break;
    }
  }
  const cudaError_t le = launch_error();
  launch_error() = cudaSuccess;
  const cudaError_t ge = cudaGetLastError();
  return fast_cuda(le != cudaSuccess ? le : ge, "fast-path launch", err);
}

}  // namespace
}  // namespace cfft
