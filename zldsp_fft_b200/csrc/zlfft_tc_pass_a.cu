// Instantiates the tensor-core split-precision passes for orders 14..18.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_tc_pass_a(TcPassTable& t) { fill_tc_pass_range_impl<14>(t, std::make_integer_sequence<int, 5>{}); }
}  // namespace zlfft
