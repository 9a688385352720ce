// Fast-path plane stages (0, 5), float precision.
#include "fast_kernels.cuh"

namespace cfft {

Status fast_planes_f32(const FastArgs& a, std::string* err) { return fast_unit_launch<float, 0>(a, err); }
Status fast_init_planes_f32(std::string* err) { return fast_unit_init<float, 0>(err); }
Status fast_cluster_probe_f32(int H, int ct, int kc, int* max_clusters, std::string* err) {
  return fast_unit_cluster_probe<float>(H, ct, kc, max_clusters, err);
}

}  // namespace cfft
