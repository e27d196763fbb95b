// smvs_win_7_2.cu — instantiates the PatchMatch kernels for window radius 7, step 2.
#include "smvs_sweep.cuh"

namespace smvs {
namespace detail {
template cudaError_t LaunchWindow<7, 2>(const Batch& b, int op, int colour, cudaStream_t stream);
template cudaError_t ConfigureWindow<7, 2>();
}  // namespace detail
}  // namespace smvs
