// sqg_inst_f32_c.cu -- row and column pass kernels in float for log2(N) in {11, 12}.
#define SQG_LAUNCH_DEFS
#include "sqg_launch.cuh"

namespace sqg {
SQG_INSTANTIATE(float, 11)
SQG_INSTANTIATE(float, 12)
}  // namespace sqg
