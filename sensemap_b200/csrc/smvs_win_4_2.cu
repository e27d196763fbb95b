// smvs_win_4_2.cu — instantiates the PatchMatch kernels for window radius 4, step 2.
#include "smvs_sweep.cuh"

namespace smvs {
namespace detail {
template cudaError_t LaunchWindow<4, 2>(const Batch& b, int op, int colour, cudaStream_t stream);
template cudaError_t ConfigureWindow<4, 2>();
}  // namespace detail
}  // namespace smvs
