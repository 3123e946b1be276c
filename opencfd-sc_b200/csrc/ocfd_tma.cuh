// ocfd_tma.cuh -- tensor-memory-accelerator (TMA) staging of the face sweeps'
// input tiles: the eight arrays a sweep reads (d, u, v, w, T and the three metric
// rows of its direction) are copied tile by tile from HBM into shared memory by
// cp.async.bulk.tensor, completion tracked by one mbarrier per block.
//
// Rules kept here: the innermost tile coordinate is rounded down to a 16-byte
// boundary (the tile is widened and the offset applied in shared memory), every
// tile slot starts on a 128-byte boundary, the global strides are multiples of
// 16 bytes (checked on the host before this path is chosen), no multicast, and
// every wait on the mbarrier is bounded: a block that gives up records an error
// (DevStatus::error = 4) and returns.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace ocfd {

// Tile geometry of one face sweep (NP pencils x TF faces, stencil TF + 7 points).
// A = elements per 16 bytes.  x is the innermost (i) dimension of the haloed array.
template <int DIR, int NP, int TF, typename S>
struct TmaBox {
  static constexpr int A = 16 / (int)sizeof(S);
  static constexpr int rup(int x) { return (x + A - 1) / A * A; }
  static constexpr int BX = DIR == 0 ? rup(TF + 7 + A - 1) : rup(NP + A - 1);
  static constexpr int BY = DIR == 0 ? NP : (DIR == 1 ? TF + 7 : 1);
  static constexpr int BZ = DIR == 2 ? TF + 7 : 1;
  static constexpr int ELEMS = BX * BY * BZ;
  static constexpr int BYTES = ELEMS * (int)sizeof(S);                // bytes one copy delivers
  static constexpr int SLOT = (BYTES + 127) / 128 * 128;              // shared-memory slot
  static constexpr int SLOT_ELEMS = SLOT / (int)sizeof(S);
  static_assert(BX * (int)sizeof(S) % 16 == 0, "TMA box inner extent must be a multiple of 16 bytes");
  static_assert(BX <= 256 && BY <= 256 && BZ <= 256, "TMA box dimensions are at most 256");
};

// Eight tensor maps (d, u, v, w, T, A1, A2, A3) of one sweep, passed as a
// __grid_constant__ kernel parameter.
struct FaceTmaMaps {
  CUtensorMap m[8];
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make the initialised mbarrier visible to the asynchronous (TMA) proxy
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// 3-D tiled copy global -> shared, completion counted on bar (no multicast)
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}

// 4-D tiled copy global -> shared (the FP32 u,v,w,T copies: four floats a point
// as the innermost dimension), completion counted on bar (no multicast)
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// Bounded wait for phase `parity` of bar: true when it completed.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t max_iter) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < max_iter; it++) {
    uint32_t done = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace ocfd
