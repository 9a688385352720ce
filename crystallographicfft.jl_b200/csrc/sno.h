// Spectral neural operator (learned SCFT warm start) on KRFFT plans: see sno.cu.
#pragma once

#include <cstdint>
#include <string>

#include "exec.h"

namespace cfft {

constexpr int kSnoWidth = 32;     // channels of the Fourier layers
constexpr int kSnoHidden = 64;    // hidden channels of the projection
constexpr int kSnoLayers = 4;
constexpr int kSnoModes = 12;     // retained modes per axis: |h_c,i| <= 11
constexpr int kSnoRefl = 8;       // reflections of the input plane-wave features
constexpr int kSnoCin = 5 + 2 * kSnoRefl;
constexpr int kSnoClasses = 364;  // (a, b, c), 11 >= a >= b >= c >= 0
constexpr int kSnoGroups = 3;     // one-hot slots: Im-3m, Ia-3d, Pm-3m

// Flattened parameter layout (FP32 master copy): lift W [32][21], lift b [32]; per layer
// W [32][32], b [32], spectral W [364][32][32]; projection W1 [64][32], b1 [64], W2 [2][64],
// b2 [2].
struct SnoLayout {
  static constexpr int64_t lift_W = 0;
  static constexpr int64_t lift_b = lift_W + kSnoWidth * kSnoCin;
  static constexpr int64_t layer0 = lift_b + kSnoWidth;
  static constexpr int64_t layer_W = 0;
  static constexpr int64_t layer_b = kSnoWidth * kSnoWidth;
  static constexpr int64_t layer_S = layer_b + kSnoWidth;
  static constexpr int64_t layer_size = layer_S + int64_t(kSnoClasses) * kSnoWidth * kSnoWidth;
  static constexpr int64_t p1_W = layer0 + kSnoLayers * layer_size;
  static constexpr int64_t p1_b = p1_W + kSnoHidden * kSnoWidth;
  static constexpr int64_t p2_W = p1_b + kSnoHidden;
  static constexpr int64_t p2_b = p2_W + 2 * kSnoHidden;
  static constexpr int64_t total = p2_b + 2;
};

struct SnoConfig {
  double lr = 1e-3, beta1 = 0.9, beta2 = 0.999, eps = 1e-8, weight_decay = 0.0;
};

struct SnoModel;
struct SnoCtx;

Status sno_model_create(const SnoConfig& cfg, SnoModel** out, std::string* err);
void sno_model_destroy(SnoModel* m);
Status sno_set_params(SnoModel* m, const float* host, std::string* err);
Status sno_get_params(const SnoModel* m, float* host, std::string* err);
Status sno_get_grads(const SnoModel* m, float* host, std::string* err);
Status sno_grads_device(const SnoModel* m, void* dst, void* stream, std::string* err);
Status sno_apply_grads(SnoModel* m, const void* grads, double lr, void* stream, std::string* err);

// A model bound to one FP32 KRFFT plan (cubic group, P = M^3 a multiple of 128) for up
// to max_samples samples per call; group_slot is the one-hot slot (0 Im-3m, 1 Ia-3d,
// 2 Pm-3m), shift the fractional origin shift of the plan's operations.  The plan's
// max_batch must be at least 32 * max_samples.
Status sno_bind(SnoModel* m, Plan* p, int group_slot, const double* shift, int max_samples, SnoCtx** out,
                std::string* err);
void sno_unbind(SnoCtx* c);
// Predicted fields [w_A | w_B] of each sample (S x 2 x M-grid, device, plan precision
// FP32) for the host parameters (chiN, f) of each sample.
Status sno_predict(SnoCtx* c, const double* params, int S, void* w_out, void* stream, std::string* err);
// Loss and parameter gradients (into the model's gradient buffer) for targets w
// (S x 2 x M-grid FP32, device); step > 0 also applies one Adam step with learning rate lr.
Status sno_train(SnoCtx* c, const double* params, int S, const void* w_target, double lr, int step, double* loss,
                 void* stream, std::string* err);

}  // namespace cfft
