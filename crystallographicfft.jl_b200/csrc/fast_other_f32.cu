// Fast-path z-FFT and gather stages (1-4), float precision.
#include "fast_kernels.cuh"

namespace cfft {

Status fast_other_f32(const FastArgs& a, std::string* err) { return fast_unit_launch<float, 1>(a, err); }
Status fast_init_other_f32(std::string* err) { return fast_unit_init<float, 1>(err); }

}  // namespace cfft
