// Fast-path plane stages (0, 5), float precision.
#include "fast_kernels.cuh"

namespace cfft {

Status fast_planes_f32(const FastArgs& a, std::string* err) { return fast_unit_launch<float, 0>(a, err); }
Status fast_init_planes_f32(std::string* err) { return fast_unit_init<float, 0>(err); }
void fast_tma_planes_f32(int H, int ct, int tma, bool* fwd, bool* fwd_e, bool* bwd) {
  fast_unit_tma_planes<float>(H, ct, tma, fwd, fwd_e, bwd);
}
Status fast_cluster_probe_f32(int H, int ct, int kc, int* max_clusters, std::string* err) {
  return fast_unit_cluster_probe<float>(H, ct, kc, max_clusters, err);
}

Status fast_wait_selftest(unsigned long long timeout_ns, int* status, void* stream, std::string* err) {
  k_wait_selftest<<<1, 128, 0, static_cast<cudaStream_t>(stream)>>>(timeout_ns, status);
  return fast_cuda(cudaGetLastError(), "wait self-test launch", err);
}

}  // namespace cfft
