// Instantiates the multi-pass kernels in double for orders 14..18.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_pass_f64_a(PassTable& t) { fill_pass_range<double, 14, 18>(t); }
}  // namespace zlfft
