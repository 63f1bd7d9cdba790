// Instantiates the multi-pass kernels in float for orders 25..26.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_pass_f32_c(PassTable& t) { fill_pass_range<float, 25, kPassMaxP>(t); }
}  // namespace zlfft
