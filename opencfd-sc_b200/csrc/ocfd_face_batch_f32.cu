// Batched face-flux kernels (ocfd_face.cuh), float arithmetic: one launch per
// direction for all instances of a batch.
#include "ocfd_face.cuh"

namespace ocfd {
template cudaError_t launch_face_batch<float, float>(int, bool, int, int, const BatchTab<FaceArgs<float>>&, int,
                                                   cudaStream_t);
template dim3 face_batch_dims<float>(int, int, const FaceArgs<float>&);

// Sets the dynamic shared-memory limit of every batched float face kernel.
cudaError_t setup_face_batch_kernels_f32() {
  const int schemes[5] = {SCH_WENO5, SCH_WENO7, SCH_OMP6, SCH_UD7L, SCH_HYBRID};
  BatchTab<FaceArgs<float>> b;
  memset(&b, 0, sizeof(b));
  for (int d = 0; d < 3; d++)
    for (int c = 0; c < 2; c++)
      for (int s = 0; s < 5; s++)
        for (int v = 0; v < 2; v++) {
          cudaError_t e = launch_face_batch<float, float>(d, c == 1, schemes[s], v, b, 0, 0);
          if (e != cudaSuccess) return e;
        }
  return cudaSuccess;
}
}  // namespace ocfd
