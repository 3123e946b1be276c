// Persistent batched stage kernels (ocfd_batch_stage.cuh), double arithmetic.
#include "ocfd_batch_stage.cuh"

namespace ocfd {
template cudaError_t launch_batch_stage<double>(bool, int, int, const StageTab<double>&, int, cudaStream_t, int*);
}  // namespace ocfd
