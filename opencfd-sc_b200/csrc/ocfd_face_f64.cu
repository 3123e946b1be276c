// FP64 instantiations of the face-flux kernels (ocfd_face.cuh).
#include "ocfd_face.cuh"

#include <cstdlib>

namespace ocfd {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda).
typedef CUresult (*TileEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static TileEncodeFn tile_encoder() {
  static TileEncodeFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<TileEncodeFn>(f);
  }
  return fn;
}

// TMA staging of the FP64 face sweeps: on unless OCFD_FACE_TMA=0 (or the
// driver offers no tensor-map encoder).
bool face_tma_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = std::getenv("OCFD_FACE_TMA");
    on = (e && e[0] == '0') ? 0 : (tile_encoder() != nullptr ? 1 : 0);
  }
  return on == 1;
}

// TMA staging of the FP32 face sweeps: off unless OCFD_FACE_TMA32=1 (and the
// driver offers a tensor-map encoder).  The FP32 sweeps compile to differently
// contracted arithmetic in the TMA kernels than in the batched kernels (plain
// loads), and a batched member must give the same bits as the same instance
// stepped alone; the staged and the plain sweeps agree to FP32 rounding.
bool face_tma32_enabled() {
  static int on = -1;
  if (on < 0) {
    const char* e = std::getenv("OCFD_FACE_TMA32");
    on = (e && e[0] == '1' && tile_encoder() != nullptr) ? 1 : 0;
  }
  return on == 1;
}

// Tiled 4-D map of the interleaved FP32 u,v,w,T copy (4 floats a haloed
// point): dimensions (4, nxh, nyh, nzh), box (4, bx, by, bz) -- the innermost
// box extent is the 16 bytes of one point, the point coordinates follow the
// scalar maps.
bool encode_tile_map4(CUtensorMap* map, const void* base, const Grid& g, int bx, int by, int bz) {
  TileEncodeFn fn = tile_encoder();
  if (!fn) return false;
  const cuuint64_t dims[4] = {4, (cuuint64_t)g.nxh, (cuuint64_t)g.nyh, (cuuint64_t)g.nzh};
  const cuuint64_t strides[3] = {16, (cuuint64_t)g.nxh * 16, (cuuint64_t)g.nxh * g.nyh * 16};
  const cuuint32_t box[4] = {4, (cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  return fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void*>(base), dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Tiled 3-D map of a haloed (nxh, nyh, nzh) array, box (bx, by, bz); tiles
// reaching past the array read zeros.
bool encode_tile_map(CUtensorMap* map, const void* base, bool f64, const Grid& g, int bx, int by, int bz) {
  TileEncodeFn fn = tile_encoder();
  if (!fn) return false;
  const cuuint64_t es = f64 ? 8 : 4;
  const cuuint64_t dims[3] = {(cuuint64_t)g.nxh, (cuuint64_t)g.nyh, (cuuint64_t)g.nzh};
  const cuuint64_t strides[2] = {(cuuint64_t)g.nxh * es, (cuuint64_t)g.nxh * g.nyh * es};
  const cuuint32_t box[3] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz};
  const cuuint32_t estr[3] = {1, 1, 1};
  return fn(map, f64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(base),
            dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

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
