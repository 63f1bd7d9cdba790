// Instantiates the c2c tile kernels in double for every supported order.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_tile_c2c_f64(TileTable& t) {
    fill_c2c_orders<double>(t, std::make_integer_sequence<int, kTileMaxP_f64 + 1>{});
}
}  // namespace zlfft
