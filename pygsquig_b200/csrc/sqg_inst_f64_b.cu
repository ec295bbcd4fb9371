// sqg_inst_f64_b.cu -- row and column pass kernels in double for log2(N) in {8, 9, 10}.
#define SQG_LAUNCH_DEFS
#include "sqg_launch.cuh"

namespace sqg {
SQG_INSTANTIATE(double, 8)
SQG_INSTANTIATE(double, 9)
SQG_INSTANTIATE(double, 10)
}  // namespace sqg
