// Instantiates the two-pass scheme of orders 19 and 20 (pass scheme 1) in float and double.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_pass_split_f32(PassTable& t) {
    fill_pass_order<float, 19, 1>(t);
    fill_pass_order<float, 20, 1>(t);
}
void fill_pass_split_f64(PassTable& t) {
    fill_pass_order<double, 19, 1>(t);
    fill_pass_order<double, 20, 1>(t);
}
}  // namespace zlfft
