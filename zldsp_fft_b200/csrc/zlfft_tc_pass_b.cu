// Instantiates the tensor-core split-precision passes for orders 19..24.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_tc_pass_b(TcPassTable& t) { fill_tc_pass_range_impl<19>(t, std::make_integer_sequence<int, 6>{}); }
}  // namespace zlfft
