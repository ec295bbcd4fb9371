// sqg_inst_f32_b.cu -- row and column pass kernels in float for log2(N) in {8, 9, 10}.
#define SQG_LAUNCH_DEFS
#include "sqg_launch.cuh"

namespace sqg {
SQG_INSTANTIATE(float, 8)
SQG_INSTANTIATE(float, 9)
SQG_INSTANTIATE(float, 10)
}  // namespace sqg
