// Instantiates the persistent mixed-order kernel in double.
#include "zlfft_mixed.cuh"

namespace zlfft {
cudaError_t launch_mixed_f64(const MixedGroup* groups, const MixedItem* items, int n_items, int* counter,
                             cudaStream_t stream, int num_sms) {
    return launch_mixed<double>(groups, items, n_items, counter, stream, num_sms);
}
}  // namespace zlfft
