// sqg_inst_f64_c.cu -- row and column pass kernels in double for log2(N) in {11, 12}.
#define SQG_LAUNCH_DEFS
#include "sqg_launch.cuh"

namespace sqg {
SQG_INSTANTIATE(double, 11)
SQG_INSTANTIATE(double, 12)
}  // namespace sqg
