// Instantiates the c2c tile kernels in float for every supported order.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_tile_c2c_f32(TileTable& t) {
    fill_c2c_orders<float>(t, std::make_integer_sequence<int, kTileMaxP_f32 + 1>{});
}
}  // namespace zlfft
