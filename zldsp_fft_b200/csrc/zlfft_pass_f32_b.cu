// Instantiates the multi-pass kernels in float for orders 19..24.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_pass_f32_b(PassTable& t) { fill_pass_range<float, 19, 24>(t); }
}  // namespace zlfft
