// Instantiates the macro path's segment kernels (micro FFT + transposed store) in double.
#include "zlfft_macro.cuh"

namespace zlfft {
void fill_macro_seg_f64(MacroTable& t) { fill_macro_segs<double>(t); }
}  // namespace zlfft
