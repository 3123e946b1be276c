// FP64 instantiations of the face-flux kernels (ocfd_face.cuh).
#include "ocfd_face.cuh"

namespace ocfd {
template cudaError_t launch_face<double, double>(int, bool, int, const FaceArgs<double>&, cudaStream_t);

// A FaceArgs with an empty grid asks launch_face_t to set the kernel's
// shared-memory attribute instead of launching it.
cudaError_t setup_face_kernels_f32();
cudaError_t setup_face_kernels() {
  const int schemes[5] = {SCH_WENO5, SCH_WENO7, SCH_OMP6, SCH_UD7L, SCH_HYBRID};
  FaceArgs<double> ad;
  memset(&ad, 0, sizeof(ad));
  for (int per = 0; per < 2; per++)
    for (int d = 0; d < 3; d++)
      for (int c = 0; c < 2; c++)
        for (int s = 0; s < 5; s++) {
          ad.ph.periodic[d] = per;
          cudaError_t e = launch_face<double, double>(d, c == 1, schemes[s], ad, 0);
          if (e != cudaSuccess) return e;
        }
  return setup_face_kernels_f32();
}
}  // namespace ocfd
