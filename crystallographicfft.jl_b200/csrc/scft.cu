// SCFT driver of libcfft_b200 (sm_100a): the self-consistent field iteration of an AB
// diblock melt built on the KRFFT contour step.  The reference stops at that step
// (step_diffusion!, src/diffusion_solver.jl:254-282; execute_m2_scft!,
// src/q_fused_krfft.jl:989-1026); the iteration itself is the textbook one:
//
//   q(r, 0) = 1, q_dagger(r, 1) = 1, each contour step
//   q <- e^{-w ds/2} IFFT(e^{-k^2 ds} FFT(e^{-w ds/2} q)) (the plan's step, ds = 1/Ns),
//   w = w_A on s < f, w_B after; Q = <q(r, 1)>; phi_A = (1/Q) int_0^f q q_dagger ds,
//   phi_B over [f, 1] (Simpson's rule, trapezoid for an odd block);
//   d_A = chiN (phi_B - 1/2) + (w_B - w_A)/2, d_B = chiN (phi_A - 1/2) + (w_A - w_B)/2;
//   err = sqrt(sum d^2 / sum w^2);
//   F = -ln Q + <w_-^2 / chiN - w_+> + chiN / 4 with w_+- = (w_B +- w_A) / 2, the
//   field-theoretic Hamiltonian: at the saddle point it equals the mean-field free energy
//   -ln Q + <chiN phi_A phi_B - w_A phi_A - w_B phi_B>, and it is stationary there
//   (dF/dw_+ = phi_A + phi_B - 1, dF/dw_- = phi_B - phi_A + 2 w_- / chiN), so its error
//   is second order in the residual and two solves converged to the same tolerance
//   agree on F far below that tolerance;
//   simple mixing (w += lam_s d) for the first min_simple iterations and while
//   err > anderson_start, then Anderson mixing over
//   the last `history` iterates (U c = V from the Gram matrix of the residuals).
//
// Fields live on the plan's stride-L subgrid (M-grid): for fields symmetric under the
// plan's operations every parity class of the full grid is an image of the subgrid, so
// grid means (Q, F, the dot products of the mixing) equal the subgrid means.
//
// Layout: w = [w_A | w_B] (2 x M-grid); the propagators run as one batch of two fields
// (q, q_dagger) -- the fast path packs them into one complex transform -- with history
// H2[i] = (q(i ds), q_dagger(1 - i ds)), i = 0..Ns, so step i maps H2[i] to H2[i+1].
// The Ns steps are captured once into a CUDA graph and replayed every iteration.
// Q, F, the residual norms, the Gram matrix and the least-squares solve are FP64 on
// the device; the fields and propagators are in the plan's precision.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "exec.h"
#include "scft.h"

namespace cfft {
namespace {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 296;  // 2 x 148 SMs

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x < 32) {
    t = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
  }
  return t;  // valid in thread 0
}

// E6 = [E_A, E_B, E_A, E_A, E_B, E_B] with E = exp(-w ds/2): every (q, q_dagger) pair of
// interaction factors a step needs is two consecutive fields of E6.
template <typename T>
__global__ void k_scft_exp(const T* __restrict__ w, T* __restrict__ E6, T half_ds, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const T ea = exp(-w[i] * half_ds), eb = exp(-w[n + i] * half_ds);
    E6[i] = ea;
    E6[n + i] = eb;
    E6[2 * n + i] = ea;
    E6[3 * n + i] = ea;
    E6[4 * n + i] = eb;
    E6[5 * n + i] = eb;
  }
}

template <typename T>
__global__ void k_scft_fill(T* __restrict__ x, T v, size_t n) {
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x)
    x[i] = v;
}

// Simpson weight of sample j of n intervals (trapezoid when n is odd).
__device__ __forceinline__ double quad_weight(int j, int n) {
  if (n % 2 == 0) return (j == 0 || j == n) ? 1.0 / 3.0 : ((j & 1) ? 4.0 / 3.0 : 2.0 / 3.0);
  return (j == 0 || j == n) ? 0.5 : 1.0;
}

// Unnormalised densities ds sum_j w_j q(j) q_dagger(j) over each block into phi, and the
// block sums of q(r, 1) (FP64) into part[block].
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_scft_density(const T* __restrict__ H2, T* __restrict__ phi,
                                                              double* __restrict__ part, int Ns, int NA, double ds,
                                                              size_t n) {
  __shared__ double sh[32];
  double qsum = 0.0;
  for (size_t r = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<size_t>(gridDim.x) * blockDim.x) {
    T a = static_cast<T>(0), b = static_cast<T>(0);
    for (int j = 0; j <= Ns; ++j) {
      const T qq = H2[(2 * static_cast<size_t>(j)) * n + r] * H2[(2 * static_cast<size_t>(Ns - j) + 1) * n + r];
      if (j <= NA) a += static_cast<T>(quad_weight(j, NA)) * qq;
      if (j >= NA) b += static_cast<T>(quad_weight(j - NA, Ns - NA)) * qq;
    }
    phi[r] = a * static_cast<T>(ds);
    phi[n + r] = b * static_cast<T>(ds);
    qsum += static_cast<double>(H2[(2 * static_cast<size_t>(Ns)) * n + r]);
  }
  const double t = block_sum(qsum, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// out[j] = scale * sum_b part[b * k + j], j < k (one block).
__global__ void k_scft_finalize(const double* __restrict__ part, int nblocks, int k, double scale,
                                double* __restrict__ out) {
  __shared__ double sh[32];
  for (int j = 0; j < k; ++j) {
    double v = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) v += part[static_cast<size_t>(b) * k + j];
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) out[j] = scale * t;
  }
}

// Normalised densities, residuals and the FP64 block sums of sum d^2, sum w^2 and
// sum (chiN phi_A phi_B - w_A phi_A - w_B phi_B).  Qm = <q(r, 1)>.
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_scft_residual(const T* __restrict__ w, T* __restrict__ phi,
                                                               T* __restrict__ d, const double* __restrict__ Qm,
                                                               double* __restrict__ part, double chiN, size_t n) {
  __shared__ double sh[32];
  const T invQ = static_cast<T>(1.0 / *Qm);
  const T cn = static_cast<T>(chiN), half = static_cast<T>(0.5);
  double sd = 0.0, sw = 0.0, sf = 0.0;
  for (size_t r = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; r < n;
       r += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const T pa = phi[r] * invQ, pb = phi[n + r] * invQ;
    phi[r] = pa;
    phi[n + r] = pb;
    const T wa = w[r], wb = w[n + r];
    const T da = cn * (pb - half) + half * (wb - wa), db = cn * (pa - half) + half * (wa - wb);
    d[r] = da;
    d[n + r] = db;
    sd += static_cast<double>(da) * da + static_cast<double>(db) * db;
    sw += static_cast<double>(wa) * wa + static_cast<double>(wb) * wb;
    const double wm = 0.5 * (static_cast<double>(wb) - static_cast<double>(wa));
    sf += wm * wm / chiN - 0.5 * (static_cast<double>(wa) + static_cast<double>(wb));
  }
  double t = block_sum(sd, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 3 + 0] = t;
  t = block_sum(sw, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 3 + 1] = t;
  t = block_sum(sf, sh);
  if (threadIdx.x == 0) part[blockIdx.x * 3 + 2] = t;
}

// Ring slots of the Anderson history passed by value: slot[0] = newest (k), slot[m] =
// k - m.
struct RingSlots {
  int slot[kScftMaxHistory + 1];
  int m;
};

// Block sums of x . ring[slot[j]] for j = 0..m (FP64): part[b * (m + 1) + j].
template <typename T>
__global__ void __launch_bounds__(kRedThreads) k_scft_dots(const T* __restrict__ x, const T* __restrict__ ring,
                                                           RingSlots rs, size_t n2, double* __restrict__ part) {
  __shared__ double sh[32];
  for (int j = 0; j <= rs.m; ++j) {
    const T* y = ring + static_cast<size_t>(rs.slot[j]) * n2;
    double v = 0.0;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n2;
         i += static_cast<size_t>(gridDim.x) * blockDim.x)
      v += static_cast<double>(x[i]) * static_cast<double>(y[i]);
    const double t = block_sum(v, sh);
    if (threadIdx.x == 0) part[static_cast<size_t>(blockIdx.x) * (rs.m + 1) + j] = t;
  }
}

// Gram row update and the least-squares solve (one thread, FP64): with G the Gram
// matrix of the residual ring (R x R, row-major by slot) and dots[j] = D_k . D_{slot[j]},
//   U_ab = G_kk - G_k,b - G_a,k + G_a,b,  V_a = G_kk - G_a,k   (a, b = k-1 .. k-m)
// solved by Gaussian elimination with partial pivoting; a vanishing pivot gives c = 0.
__global__ void k_scft_solve(double* __restrict__ G, int R, const double* __restrict__ dots, RingSlots rs,
                             double* __restrict__ c) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int k = rs.slot[0], m = rs.m;
  for (int j = 0; j <= m; ++j) {
    G[k * R + rs.slot[j]] = dots[j];
    G[rs.slot[j] * R + k] = dots[j];
  }
  double U[kScftMaxHistory][kScftMaxHistory + 1];
  const double gkk = G[k * R + k];
  for (int a = 0; a < m; ++a) {
    const int sa = rs.slot[a + 1];
    for (int b = 0; b < m; ++b) {
      const int sb = rs.slot[b + 1];
      U[a][b] = gkk - G[k * R + sb] - G[sa * R + k] + G[sa * R + sb];
    }
    U[a][m] = gkk - G[sa * R + k];
  }
  bool ok = true;
  for (int col = 0; col < m && ok; ++col) {
    int piv = col;
    for (int r = col + 1; r < m; ++r)
      if (fabs(U[r][col]) > fabs(U[piv][col])) piv = r;
    if (!(fabs(U[piv][col]) > 1e-300)) { ok = false; break; }
    if (piv != col)
      for (int q = col; q <= m; ++q) { const double t = U[col][q]; U[col][q] = U[piv][q]; U[piv][q] = t; }
    for (int r = col + 1; r < m; ++r) {
      const double fct = U[r][col] / U[col][col];
      for (int q = col; q <= m; ++q) U[r][q] -= fct * U[col][q];
    }
  }
  for (int a = m - 1; a >= 0; --a) {
    double v = ok ? U[a][m] : 0.0;
    if (ok) {
      for (int q = a + 1; q < m; ++q) v -= U[a][q] * c[q];
      v /= U[a][a];
    }
    c[a] = v;
  }
}

// w_next = W_k + sum_a c_a (W_a - W_k) + lam (D_k + sum_a c_a (D_a - D_k)); with m = 0
// simple mixing w_next = W_k + lam D_k.
template <typename T>
__global__ void k_scft_update(T* __restrict__ wnext, const T* __restrict__ Wr, const T* __restrict__ Dr, RingSlots rs,
                              const double* __restrict__ c, double lam, size_t n2) {
  const T* wk = Wr + static_cast<size_t>(rs.slot[0]) * n2;
  const T* dk = Dr + static_cast<size_t>(rs.slot[0]) * n2;
  for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n2;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const double w0 = wk[i], d0 = dk[i];
    double W = w0, D = d0;
    for (int a = 0; a < rs.m; ++a) {
      const size_t o = static_cast<size_t>(rs.slot[a + 1]) * n2 + i;
      W += c[a] * (static_cast<double>(Wr[o]) - w0);
      D += c[a] * (static_cast<double>(Dr[o]) - d0);
    }
    wnext[i] = static_cast<T>(W + lam * D);
  }
}

int red_grid(size_t n) { return static_cast<int>(std::max<size_t>(1, std::min<size_t>((n + kRedThreads - 1) / kRedThreads, kRedBlocks))); }

}  // namespace

struct Scft {
  Plan* plan = nullptr;
  ScftParams prm;
  int NA = 0;
  size_t n = 0;       // M-grid points
  int R = 0;          // ring depth (history + 1)
  int rs_bytes = 4;   // real size
  void* H2 = nullptr;
  void* E6 = nullptr;
  void* phi = nullptr;
  void* Wr = nullptr;  // R x 2n fields
  void* Dr = nullptr;  // R x 2n residuals
  double* part = nullptr;   // reduction partials
  double* red = nullptr;    // [Q, sum d^2, sum w^2, sum f, dots... ]
  double* G = nullptr;      // R x R Gram matrix
  double* c = nullptr;      // mixing coefficients
  double* h_red = nullptr;  // pinned copy of red[0..3]
  cudaGraphExec_t prop = nullptr;
  int64_t prop_kernels = 0;
  cudaStream_t cap = nullptr;
};

namespace {

Status cuda_status(cudaError_t e, const char* what, std::string* err) {
  if (e == cudaSuccess) return Status::kOk;
  *err = std::string(what) + ": " + cudaGetErrorString(e);
  return Status::kCuda;
}
#define SCFT_CUDA(call, what)                                          \
  do {                                                                 \
    const Status s_ = cuda_status((call), (what), err);                \
    if (s_ != Status::kOk) return s_;                                  \
  } while (0)

// The Ns propagator steps (H2[i] -> H2[i+1]) on stream st.
Status propagate_direct(Scft* S, cudaStream_t st, std::string* err) {
  const size_t n = S->n, rb = S->rs_bytes;
  char* H2 = static_cast<char*>(S->H2);
  const char* E6 = static_cast<const char*>(S->E6);
  const int Ns = S->prm.Ns, NA = S->NA;
  for (int i = 0; i < Ns; ++i) {
    const bool qa = i < NA, qda = Ns - 1 - i < NA;
    const int off = qa ? (qda ? 2 : 0) : (qda ? 1 : 4);  // (A,A) (A,B) (B,A) (B,B)
    Status s = exec_contour_step(S->plan, H2 + 2 * i * n * rb, H2 + 2 * (i + 1) * n * rb, E6 + off * n * rb, 2, st, err);
    if (s != Status::kOk) return s;
  }
  return Status::kOk;
}

// Replays the captured propagation (captured on first use; direct launches when the
// stream cannot be captured).
Status propagate(Scft* S, cudaStream_t st, std::string* err) {
  if (!S->prop) {
    const int64_t before = launch_count(false);
    if (cudaStreamBeginCapture(S->cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      std::string cerr;
      const Status s = propagate_direct(S, S->cap, &cerr);
      cudaGraph_t g = nullptr;
      const cudaError_t e = cudaStreamEndCapture(S->cap, &g);
      const int64_t k = launch_count(false) - before;
      add_launches(-k);  // captured, not launched
      if (s == Status::kOk && e == cudaSuccess && g && cudaGraphInstantiate(&S->prop, g, 0) == cudaSuccess)
        S->prop_kernels = k;
      else
        S->prop = nullptr;
      if (g) cudaGraphDestroy(g);
      cudaGetLastError();
    } else {
      cudaGetLastError();
    }
  }
  if (S->prop) {
    SCFT_CUDA(cudaGraphLaunch(S->prop, st), "propagator graph launch");
    add_launches(S->prop_kernels);
    return Status::kOk;
  }
  return propagate_direct(S, st, err);
}

template <typename T>
Status evaluate_t(Scft* S, const T* w, T* d, cudaStream_t st, std::string* err) {
  const size_t n = S->n;
  const int gr = red_grid(n);
  const int ge = static_cast<int>(std::min<size_t>((n + 255) / 256, 148 * 8));
  const double ds = 1.0 / S->prm.Ns;
  k_scft_exp<T><<<ge, 256, 0, st>>>(w, static_cast<T*>(S->E6), static_cast<T>(ds / 2), n);
  add_launches(1);
  Status s = propagate(S, st, err);
  if (s != Status::kOk) return s;
  k_scft_density<T><<<gr, kRedThreads, 0, st>>>(static_cast<const T*>(S->H2), static_cast<T*>(S->phi), S->part,
                                                S->prm.Ns, S->NA, ds, n);
  k_scft_finalize<<<1, 256, 0, st>>>(S->part, gr, 1, 1.0 / static_cast<double>(n), S->red);
  k_scft_residual<T><<<gr, kRedThreads, 0, st>>>(w, static_cast<T*>(S->phi), d, S->red, S->part, S->prm.chiN, n);
  k_scft_finalize<<<1, 256, 0, st>>>(S->part, gr, 3, 1.0, S->red + 1);
  add_launches(4);
  SCFT_CUDA(cudaGetLastError(), "scft evaluate launch");
  SCFT_CUDA(cudaMemcpyAsync(S->h_red, S->red, 4 * sizeof(double), cudaMemcpyDeviceToHost, st), "scft read back");
  SCFT_CUDA(cudaStreamSynchronize(st), "scft synchronise");
  return Status::kOk;
}

void fill_state(const Scft* S, ScftState* out) {
  const double* h = S->h_red;
  out->Q = h[0];
  out->err = std::sqrt(h[1] / std::max(h[2], 1e-300));
  out->F = -std::log(h[0]) + h[3] / static_cast<double>(S->n) + 0.25 * S->prm.chiN;
}

template <typename T>
Status solve_t(Scft* S, T* w, ScftState* out, cudaStream_t st, std::string* err) {
  const size_t n = S->n, n2 = 2 * n;
  const int R = S->R;
  T* Wr = static_cast<T*>(S->Wr);
  T* Dr = static_cast<T*>(S->Dr);
  const int gr = red_grid(n2);
  const int ge = static_cast<int>(std::min<size_t>((n2 + 255) / 256, 148 * 8));
  // The current iterate lives in ring slot k % R; the caller's w is copied in and out.
  SCFT_CUDA(cudaMemcpyAsync(Wr, w, n2 * sizeof(T), cudaMemcpyDeviceToDevice, st), "scft copy in");
  int hist = 0;  // valid Anderson entries before the newest
  int start = 0;  // iteration at which the current Anderson history began
  out->converged = 0;
  for (int it = 0; it < S->prm.max_iter; ++it) {
    const int k = it % R;
    T* wk = Wr + static_cast<size_t>(k) * n2;
    T* dk = Dr + static_cast<size_t>(k) * n2;
    Status s = evaluate_t<T>(S, wk, dk, st, err);
    if (s != Status::kOk) return s;
    fill_state(S, out);
    out->iterations = it;
    if (!(out->err == out->err)) { *err = "SCFT iteration diverged (NaN residual)"; return Status::kInvalid; }
    if (out->err < S->prm.tol) {
      out->converged = 1;
      SCFT_CUDA(cudaMemcpyAsync(w, wk, n2 * sizeof(T), cudaMemcpyDeviceToDevice, st), "scft copy out");
      return Status::kOk;
    }
    RingSlots rs;
    rs.slot[0] = k;
    T* wnext = Wr + static_cast<size_t>((it + 1) % R) * n2;
    double lam;
    if (out->err > S->prm.anderson_start || it < S->prm.min_simple) {
      hist = 0;
      start = it + 1;
      rs.m = 0;
      lam = S->prm.lam_simple;
    } else {
      rs.m = std::min(hist, S->prm.history);
      for (int a = 1; a <= rs.m; ++a) rs.slot[a] = (it - a) % R;
      k_scft_dots<T><<<gr, kRedThreads, 0, st>>>(dk, Dr, rs, n2, S->part);
      k_scft_finalize<<<1, 256, 0, st>>>(S->part, gr, rs.m + 1, 1.0, S->red + 4);
      k_scft_solve<<<1, 32, 0, st>>>(S->G, R, S->red + 4, rs, S->c);
      add_launches(3);
      hist = std::min(hist + 1, S->prm.history);
      lam = S->prm.lam_anderson;
    }
    (void)start;
    k_scft_update<T><<<ge, 256, 0, st>>>(wnext, Wr, Dr, rs, S->c, lam, n2);
    add_launches(1);
    SCFT_CUDA(cudaGetLastError(), "scft update launch");
  }
  const int k = S->prm.max_iter % R;
  Status s = evaluate_t<T>(S, Wr + static_cast<size_t>(k) * n2, Dr + static_cast<size_t>(k) * n2, st, err);
  if (s != Status::kOk) return s;
  fill_state(S, out);
  out->iterations = S->prm.max_iter;
  SCFT_CUDA(cudaMemcpyAsync(w, Wr + static_cast<size_t>(k) * n2, n2 * sizeof(T), cudaMemcpyDeviceToDevice, st),
            "scft copy out");
  return Status::kOk;
}

}  // namespace

Status scft_create(Plan* p, const ScftParams& prm, Scft** out, std::string* err) {
  if (!p->d_geom) { *err = "the SCFT driver needs a device plan"; return Status::kInvalid; }
  if (p->max_batch < 2) { *err = "the SCFT driver needs a plan with max_batch >= 2 (q and q_dagger)"; return Status::kInvalid; }
  if (prm.Ns < 2 || prm.f <= 0.0 || prm.f >= 1.0 || prm.history < 0 || prm.history > kScftMaxHistory ||
      prm.max_iter < 0 || !(prm.tol > 0.0) || prm.min_simple < 0) {
    *err = "invalid SCFT parameters (Ns >= 2, 0 < f < 1, 0 <= history <= 32, tol > 0, min_simple >= 0)";
    return Status::kInvalid;
  }
  const int NA = static_cast<int>(std::lround(prm.f * prm.Ns));
  if (NA < 1 || NA >= prm.Ns) { *err = "f * Ns must leave at least one step in each block"; return Status::kInvalid; }
  if (std::fabs(p->ds - 1.0 / prm.Ns) > 1e-12 * (1.0 / prm.Ns)) {
    *err = "the plan's ds must equal 1 / Ns";
    return Status::kInvalid;
  }
  auto* S = new Scft();
  S->plan = p;
  S->prm = prm;
  S->NA = NA;
  S->n = static_cast<size_t>(p->T.M[0]) * p->T.M[1] * p->T.M[2];
  S->R = prm.history + 1;
  S->rs_bytes = p->precision;
  const size_t rb = S->rs_bytes, n = S->n;
  auto al = [&](void** ptr, size_t bytes, const char* what) -> Status {
    const cudaError_t e = cudaMalloc(ptr, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) { *err = std::string(what) + ": " + cudaGetErrorString(e); return Status::kAlloc; }
    return Status::kOk;
  };
  Status s;
  if ((s = al(&S->H2, 2 * (prm.Ns + 1) * n * rb, "propagator history")) != Status::kOk ||
      (s = al(&S->E6, 6 * n * rb, "interaction factors")) != Status::kOk ||
      (s = al(&S->phi, 2 * n * rb, "densities")) != Status::kOk ||
      (s = al(&S->Wr, static_cast<size_t>(S->R) * 2 * n * rb, "field history")) != Status::kOk ||
      (s = al(&S->Dr, static_cast<size_t>(S->R) * 2 * n * rb, "residual history")) != Status::kOk ||
      (s = al(reinterpret_cast<void**>(&S->part), static_cast<size_t>(kRedBlocks) * (kScftMaxHistory + 1) * 8, "partials")) != Status::kOk ||
      (s = al(reinterpret_cast<void**>(&S->red), (5 + kScftMaxHistory) * 8, "reductions")) != Status::kOk ||
      (s = al(reinterpret_cast<void**>(&S->G), static_cast<size_t>(S->R) * S->R * 8, "Gram matrix")) != Status::kOk ||
      (s = al(reinterpret_cast<void**>(&S->c), (kScftMaxHistory + 1) * 8, "coefficients")) != Status::kOk) {
    scft_destroy(S);
    return s;
  }
  void* hr = nullptr;
  if (cudaHostAlloc(&hr, 8 * sizeof(double), cudaHostAllocDefault) != cudaSuccess) {
    *err = "pinned read-back buffer";
    scft_destroy(S);
    return Status::kAlloc;
  }
  S->h_red = static_cast<double*>(hr);
  if (cudaStreamCreateWithFlags(&S->cap, cudaStreamNonBlocking) != cudaSuccess) {
    *err = "capture stream";
    scft_destroy(S);
    return Status::kCuda;
  }
  // H2[0] = (q(0), q_dagger(1)) = (1, 1) once: the steps never write it.
  const int ge = static_cast<int>(std::min<size_t>((2 * n + 255) / 256, 148 * 8));
  if (p->precision == 8) k_scft_fill<double><<<ge, 256, 0, S->cap>>>(static_cast<double*>(S->H2), 1.0, 2 * n);
  else k_scft_fill<float><<<ge, 256, 0, S->cap>>>(static_cast<float*>(S->H2), 1.0f, 2 * n);
  cudaMemsetAsync(S->G, 0, static_cast<size_t>(S->R) * S->R * 8, S->cap);
  cudaMemsetAsync(S->c, 0, (kScftMaxHistory + 1) * 8, S->cap);
  const cudaError_t e = cudaStreamSynchronize(S->cap);
  if (e != cudaSuccess) {
    *err = std::string("SCFT set-up: ") + cudaGetErrorString(e);
    scft_destroy(S);
    return Status::kCuda;
  }
  add_launches(1);
  *out = S;
  return Status::kOk;
}

void scft_destroy(Scft* S) {
  if (!S) return;
  if (S->prop) cudaGraphExecDestroy(S->prop);
  for (void** b : {&S->H2, &S->E6, &S->phi, &S->Wr, &S->Dr, reinterpret_cast<void**>(&S->part),
                   reinterpret_cast<void**>(&S->red), reinterpret_cast<void**>(&S->G), reinterpret_cast<void**>(&S->c)})
    if (*b) cudaFree(*b);
  if (S->h_red) cudaFreeHost(S->h_red);
  if (S->cap) cudaStreamDestroy(S->cap);
  delete S;
}

Status scft_evaluate(Scft* S, const void* w, void* phi, void* d, ScftState* out, void* stream, std::string* err) {
  if (!w || !out) { *err = "null argument"; return Status::kInvalid; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t n2 = 2 * S->n, bytes = n2 * S->rs_bytes;
  void* dd = static_cast<char*>(S->Dr);  // scratch: ring slot 0 of the residuals
  Status s = S->rs_bytes == 8 ? evaluate_t<double>(S, static_cast<const double*>(w), static_cast<double*>(dd), st, err)
                              : evaluate_t<float>(S, static_cast<const float*>(w), static_cast<float*>(dd), st, err);
  if (s != Status::kOk) return s;
  fill_state(S, out);
  out->iterations = 0;
  out->converged = out->err < S->prm.tol ? 1 : 0;
  if (phi) SCFT_CUDA(cudaMemcpyAsync(phi, S->phi, bytes, cudaMemcpyDeviceToDevice, st), "copy densities");
  if (d) SCFT_CUDA(cudaMemcpyAsync(d, dd, bytes, cudaMemcpyDeviceToDevice, st), "copy residuals");
  SCFT_CUDA(cudaStreamSynchronize(st), "scft synchronise");
  return Status::kOk;
}

Status scft_solve(Scft* S, void* w, ScftState* out, void* stream, std::string* err) {
  if (!w || !out) { *err = "null argument"; return Status::kInvalid; }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  Status s = S->rs_bytes == 8 ? solve_t<double>(S, static_cast<double*>(w), out, st, err)
                              : solve_t<float>(S, static_cast<float*>(w), out, st, err);
  if (s != Status::kOk) return s;
  SCFT_CUDA(cudaStreamSynchronize(st), "scft synchronise");
  return Status::kOk;
}

Status scft_densities(const Scft* S, void* phi, void* stream, std::string* err) {
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  SCFT_CUDA(cudaMemcpyAsync(phi, S->phi, 2 * S->n * S->rs_bytes, cudaMemcpyDeviceToDevice, st), "copy densities");
  return Status::kOk;
}

}  // namespace cfft
