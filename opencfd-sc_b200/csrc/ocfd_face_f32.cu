// FP32 (mixed-precision) instantiations of the face-flux kernels (ocfd_face.cuh).
#include "ocfd_face.cuh"

namespace ocfd {
template cudaError_t launch_face<float, float>(int, bool, int, const FaceArgs<float>&, cudaStream_t);

cudaError_t setup_face_kernels_f32() {
  const int schemes[5] = {SCH_WENO5, SCH_WENO7, SCH_OMP6, SCH_UD7L, SCH_HYBRID};
  FaceArgs<float> af;
  memset(&af, 0, sizeof(af));
  for (int per = 0; per < 2; per++)
    for (int d = 0; d < 3; d++)
      for (int c = 0; c < 2; c++)
        for (int s = 0; s < 5; s++) {
          af.ph.periodic[d] = per;
          cudaError_t e = launch_face<float, float>(d, c == 1, schemes[s], af, 0);
          if (e != cudaSuccess) return e;
        }
  return cudaSuccess;
}
}  // namespace ocfd
