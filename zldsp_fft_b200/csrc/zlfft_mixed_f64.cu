// Instantiates the persistent mixed-order kernels (both order classes) in double.
#include "zlfft_mixed.cuh"

namespace zlfft {
cudaError_t launch_mixed_f64(int cls, const MixedGroup* groups, const MixedItem* items, int n_items, int* counter,
                             cudaStream_t stream, int num_sms) {
    return launch_mixed<double>(cls, groups, items, n_items, counter, stream, num_sms);
}
}  // namespace zlfft
