// Fast-path z-FFT and gather stages (1-4), double precision.
#include "fast_kernels.cuh"

namespace cfft {

Status fast_other_f64(const FastArgs& a, std::string* err) { return fast_unit_launch<double, 1>(a, err); }
Status fast_init_other_f64(std::string* err) { return fast_unit_init<double, 1>(err); }

}  // namespace cfft
