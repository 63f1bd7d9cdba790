// Instantiates the multi-pass kernels in double for orders 19..24.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_pass_f64_b(PassTable& t) { fill_pass_range<double, 19, 24>(t); }
}  // namespace zlfft
