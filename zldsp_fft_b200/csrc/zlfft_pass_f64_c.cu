// Instantiates the multi-pass kernels in double for orders 25..26.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_pass_f64_c(PassTable& t) { fill_pass_range<double, 25, kPassMaxP>(t); }
}  // namespace zlfft
