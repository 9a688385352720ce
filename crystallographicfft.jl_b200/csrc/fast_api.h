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
  void* stream = nullptr;
};

// Stages 0 and 5 (plane kernels) and stages 1-4 (z FFTs, gathers).
Status fast_planes_f32(const FastArgs& a, std::string* err);
Status fast_planes_f64(const FastArgs& a, std::string* err);
Status fast_other_f32(const FastArgs& a, std::string* err);
Status fast_other_f64(const FastArgs& a, std::string* err);
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

}  // namespace cfft
