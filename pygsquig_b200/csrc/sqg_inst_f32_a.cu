// sqg_inst_f32_a.cu -- row and column pass kernels in float for log2(N) in {3, 4, 5, 6, 7}.
#define SQG_LAUNCH_DEFS
#include "sqg_launch.cuh"

namespace sqg {
SQG_INSTANTIATE(float, 3)
SQG_INSTANTIATE(float, 4)
SQG_INSTANTIATE(float, 5)
SQG_INSTANTIATE(float, 6)
SQG_INSTANTIATE(float, 7)
}  // namespace sqg
