// Fast-path plane stages (0, 5), double precision.
#include "fast_kernels.cuh"

namespace cfft {

Status fast_planes_f64(const FastArgs& a, std::string* err) { return fast_unit_launch<double, 0>(a, err); }
Status fast_init_planes_f64(std::string* err) { return fast_unit_init<double, 0>(err); }
void fast_tma_planes_f64(int H, int ct, int tma, bool* fwd, bool* fwd_e, bool* bwd) {
  fast_unit_tma_planes<double>(H, ct, tma, fwd, fwd_e, bwd);
}
Status fast_cluster_probe_f64(int H, int ct, int kc, int* max_clusters, std::string* err) {
  return fast_unit_cluster_probe<double>(H, ct, kc, max_clusters, err);
}

}  // namespace cfft
