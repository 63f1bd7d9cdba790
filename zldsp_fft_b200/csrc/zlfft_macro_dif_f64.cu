// Instantiates the macro path's DIF pass kernels in double.
#include "zlfft_macro.cuh"

namespace zlfft {
void fill_macro_dif_f64(MacroTable& t) { fill_macro_dif<double>(t); }
}  // namespace zlfft
