// kernels_gf8_fixed2.cu -- the unrolled GF(2^8) kernels with a floor of 2
// resident CTAs per SM (see gf8_fixed.cuh).
#define RSGPU_FIXED_MINB 2
#include "gf8_fixed.cuh"

namespace rsgpu {
VecKernel fixed_kernel_minb2(int n_in, int G, int mode) { return fixed_for(n_in, G, mode); }
}  // namespace rsgpu
