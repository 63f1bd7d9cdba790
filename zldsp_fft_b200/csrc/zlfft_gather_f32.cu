// Instantiates the gathered (per-transform pointer) tile kernels in float for
// the AoS <-> AoS operations of mixed batches.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_gather_f32(GatherTable& t) {
    fill_gather_orders<float>(t, std::make_integer_sequence<int, kTileMaxP_f32 + 1>{});
}
}  // namespace zlfft
