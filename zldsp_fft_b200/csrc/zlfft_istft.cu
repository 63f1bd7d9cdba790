// Instantiates the inverse-STFT overlap-add kernels (zlfft_istft.cuh) in float
// and double, for bins in AoS and split-SoA layout.
#include "zlfft_istft.cuh"

namespace zlfft {
void fill_istft_f32(IstftTable& t) { fill_istft_orders<float>(t, std::make_integer_sequence<int, kTileMaxP + 1>{}); }
void fill_istft_f64(IstftTable& t) { fill_istft_orders<double>(t, std::make_integer_sequence<int, kTileMaxP + 1>{}); }
}  // namespace zlfft
