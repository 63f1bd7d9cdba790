// Instantiates the macro path's segment kernels (micro FFT + transposed store) in float.
#include "zlfft_macro.cuh"

namespace zlfft {
void fill_macro_seg_f32(MacroTable& t) { fill_macro_segs<float>(t); }
}  // namespace zlfft
