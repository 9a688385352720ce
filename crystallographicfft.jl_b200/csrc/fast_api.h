// Interface between the host execution layer (exec.cu) and the compile-time sized
// fast-path kernels, which are compiled in four translation units (plane stages /
// other stages x float / double) so the build runs in parallel.
#pragma once

#include <string>

#include "cfft_internal.h"

namespace cfft {

struct FastArgs {
  // plan state (device pointers)
  const void* geom = nullptr;
  const void* tables = nullptr;
  const void* spec_h = nullptr;
  const void* K = nullptr;
  const void* inv_spec = nullptr;
  const void* inv_phase = nullptr;
  const void* inv_pk = nullptr;
  const void* expand = nullptr;
  void* W = nullptr;      // channel workspace of this lane
  void* G0R = nullptr;    // representative workspace of this lane
  void* FT = nullptr;     // quad-grouped spectra of this lane (packed backward path)
  // call operands
  const void* f0 = nullptr;
  void* F = nullptr;
  const void* Fin = nullptr;
  void* f0_out = nullptr;
  const void* E = nullptr;
  // geometry / dispatch
  int stage = 0, nb = 0, H = 0, n_ch = 1, centered = 0, cent_type = 0, d = 1;
  int n_spec = 0, n_orbits = 0;
  bool use_K = false, rep_diag8 = false, rep_perm = false, reps_quad = false;
  bool reps_wide = false;  // backward gather in groups of 128 / sizeof(complex) fields
  // Stage 6 (fused z FFT + diagonal-sign gather): unit table and spectral points.
  const void* zr_units = nullptr;
  const void* zr_pts = nullptr;
  int zr_n_units = 0;
  bool cluster = false;   // fused cluster kernels for stages 0 (with 1) and 5 (with 4)
  int cluster_ctas = 8;   // CTAs per cluster (8, or 16 where the device allows it)
  // Q-matrix step: stage 4 reads W (forward G0, z-fastest) and writes W2
  bool q_step = false;
  const void* QT = nullptr;   // d x n_ch x H^3 coefficients
  const void* GT = nullptr;   // d x n_ch x H^3 int32 workspace indices (-1: extinct)
  void* W2 = nullptr;
  bool qsep = false;          // separable Q-multiply (Pmmm-like plans)
  const void* QS = nullptr;   // its 1-D twiddles and kernel factors
  void* stream = nullptr;
  // bounded device waits of the persistent bulk-copy kernels: limit, and the plan's
  // status word that a wait which runs out sets to CFFT_ERR_TIMEOUT
  unsigned long long timeout_ns = 1000000000ull;
  int* status = nullptr;
  // per-plan choices (0 / -1: the process default)
  int zr_slots = 0;
  int tma = -1;
};

// Stages 0 and 5 (plane kernels) and stages 1-4 (z FFTs, gathers).
Status fast_planes_f32(const FastArgs& a, std::string* err);
Status fast_planes_f64(const FastArgs& a, std::string* err);
Status fast_other_f32(const FastArgs& a, std::string* err);
Status fast_other_f64(const FastArgs& a, std::string* err);
// Largest number of concurrently resident kc-CTA clusters of the fused forward and
// backward kernels for channel edge H and centring type ct (0 if they cannot run).
Status fast_cluster_probe_f32(int H, int ct, int kc, int* max_clusters, std::string* err);
Status fast_cluster_probe_f64(int H, int ct, int kc, int* max_clusters, std::string* err);
// Whether the persistent bulk-copy plane kernels serve channel edge H and centring
// type ct (forward without / with interaction factors, backward).
void fast_tma_planes_f32(int H, int ct, int tma, bool* fwd, bool* fwd_e, bool* bwd);
void fast_tma_planes_f64(int H, int ct, int tma, bool* fwd, bool* fwd_e, bool* bwd);
// Launches the bounded-wait self-test kernel (k_wait_selftest) on `stream`.
Status fast_wait_selftest(unsigned long long timeout_ns, int* status, void* stream, std::string* err);
// Per-device set-up of each unit: constant-memory twiddles and shared-memory limits.
Status fast_init_planes_f32(std::string* err);
Status fast_init_planes_f64(std::string* err);
Status fast_init_other_f32(std::string* err);
Status fast_init_other_f64(std::string* err);

// Cubic channel edges with compile-time sized kernels for element size `real_bytes`.
inline bool fast_size_ok(int H, int real_bytes) {
  return H == 4 || H == 6 || H == 8 || H == 12 || H == 16 || H == 24 || H == 32 || (H == 48 && real_bytes == 4);
}
constexpr int kFastZB = 4;  // xz-planes (y values) per CTA in the z kernels

// The fused cluster kernels hold one slot's channel volume in the shared memory of 8
// CTAs (H / 8 z-planes of nch padded H x (H + 1) planes each, one z line per thread).
inline bool fast_cluster_fits(int H, int nch, int real_bytes) {
  if (H % 8 != 0 || H < 16 || H > 32) return false;
  const long threads = static_cast<long>(nch) * (H / 8) * H;
  const long smem = static_cast<long>(H / 8) * nch * H * (H + 1) * 2 * real_bytes;
  return threads >= 32 && threads <= 1024 && smem <= 227 * 1024;
}

}  // namespace cfft
