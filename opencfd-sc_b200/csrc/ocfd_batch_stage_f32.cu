// Persistent batched stage kernels (ocfd_batch_stage.cuh), float arithmetic.
#include "ocfd_batch_stage.cuh"

namespace ocfd {
template cudaError_t launch_batch_stage<float>(bool, int, int, const StageTab<float>&, int, cudaStream_t, int*);
}  // namespace ocfd
