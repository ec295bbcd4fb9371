// sqg_inst_f64_a.cu -- row and column pass kernels in double for log2(N) in {3, 4, 5, 6, 7}.
#define SQG_LAUNCH_DEFS
#include "sqg_launch.cuh"

namespace sqg {
SQG_INSTANTIATE(double, 3)
SQG_INSTANTIATE(double, 4)
SQG_INSTANTIATE(double, 5)
SQG_INSTANTIATE(double, 6)
SQG_INSTANTIATE(double, 7)
}  // namespace sqg
