// Instantiates the gathered (per-transform pointer) tile kernels in double for
// the AoS <-> AoS operations of mixed batches.
#include "zlfft_launch.cuh"

namespace zlfft {
void fill_gather_f64(GatherTable& t) {
    fill_gather_orders<double>(t, std::make_integer_sequence<int, kTileMaxP + 1>{});
}
}  // namespace zlfft
