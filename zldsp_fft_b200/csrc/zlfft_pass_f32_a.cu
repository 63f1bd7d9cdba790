// Instantiates the multi-pass kernels in float for orders 14..18.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_pass_f32_a(PassTable& t) { fill_pass_range<float, 14, 18>(t); }
}  // namespace zlfft
