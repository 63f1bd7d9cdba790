// Instantiates the macro path's DIF pass kernels in float.
#include "zlfft_macro.cuh"

namespace zlfft {
void fill_macro_dif_f32(MacroTable& t) { fill_macro_dif<float>(t); }
}  // namespace zlfft
