// wos_kernels_mix32.cu -- the general sweeps instantiated in FP32 for
// mixed-radix (2^a 3^b 5^c) lines, compiled apart from the power-of-two ones.
#define WOS_DEFINE_MIX_LAUNCHERS
#include "wos_kernels_dev.cuh"

namespace wos {
WOS_MIX_INST(float, 2)
WOS_MIX_INST(float, 4)
WOS_MIX_INST(float, 8)
WOS_MIX_INST(float, 16)
}  // namespace wos
