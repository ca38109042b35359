// yee_fused.cu -- FP32 single-pass E+H step (placeholder until the fused
// kernel lands; the split kernels serve every configuration meanwhile).
#include "kernels.h"

namespace fdtd {

int fused_supported(int, int, int) { return 0; }
void launch_fused_step(const FusedArgs &, cudaStream_t) {}

}  // namespace fdtd
