// w2d_k32.cu -- FP32 kernels (state, slopes, fluxes and updates in float);
// the CFL reduction and the cooling source terms stay in FP64.
#define W2D_INST_NS k32
#define W2D_INST_REAL float
#include "w2d_kinst.cuh"

namespace w2d {
const Launchers& launchers32() { return k32::table; }
}  // namespace w2d
