// Instantiates the tensor-core split-precision passes for orders 25..26.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_tc_pass_c(TcPassTable& t) { fill_tc_pass_range_impl<25>(t, std::make_integer_sequence<int, 2>{}); }
}  // namespace zlfft
