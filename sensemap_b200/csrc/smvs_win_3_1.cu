// smvs_win_3_1.cu — instantiates the PatchMatch kernels for window radius 3, step 1.
#include "smvs_sweep.cuh"

namespace smvs {
namespace detail {
template cudaError_t LaunchWindow<3, 1>(const Batch& b, int op, int colour, cudaStream_t stream);
template cudaError_t ConfigureWindow<3, 1>();
}  // namespace detail
}  // namespace smvs
