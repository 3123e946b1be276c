// ocfd_batch_stage.cuh -- one persistent launch per RK stage for a whole batch
// of periodic instances (ragged grids): the three face sweeps, the viscous
// gradients, the stage tail and the negative-temperature repair of every
// member in a single kernel.
//
// The stage's work is one list of items (a block-sized tile of one kernel body
// for one member).  Resident blocks take items in list order from a counter in
// device memory and run the same device bodies as the single-instance
// launches (face_body, visc_grad_body, fused_body, negt_fix_body), so the
// results are the same bits.  Phase A of a member (its face and viscous tiles,
// which read the primitives and write the face and viscous fluxes) must finish
// before its tail tiles read those fluxes and overwrite the primitives, and the
// tail before the repair: each member counts its finished phase-A and tail
// items, and a tail (repair) item waits until its member's phase-A (tail) count
// is complete.  The list is ordered so that every item an item waits for comes
// before it -- phase A of member q+1 is listed before the tail of member q, and
// the repairs last -- so the items waited for were taken by running blocks
// that wait on nothing earlier: the waits end without any co-residency
// guarantee, and tails of one member overlap phase A of the next (no
// stage-wide barrier, no launch boundaries between the kernel bodies).  The
// waits are bounded (about a second); a block that gives up records error 5
// in its member's status word and skips the item, and the host reports the
// step as invalid.
//
// Reference: the stage body of NS_solver (OCFD_NS_Solver.f90:21-78) for each
// member -- du_inviscous[_Character], du_viscous, OCFD_time_adv_RK3,
// comput_duvwT + handle_NegativeT and the periodic boundary fill.
#pragma once

#include "ocfd_face.cuh"
#include "ocfd_update_body.cuh"

namespace ocfd {

// Bounded wait until *c >= need (thread 0 of a block): about a second at most,
// and none once an earlier wait of the same member has given up (error 5).
__device__ __forceinline__ bool stage_wait(const int* c, int need, const int* err) {
  const volatile int* vc = c;
  const volatile int* ve = err;
  for (unsigned it = 0; it < (1u << 22); it++) {
    if (*vc >= need) return true;
    if (*ve == 5) return false;
    __nanosleep(200);
  }
  return *vc >= need;
}

template <typename A>
__device__ __forceinline__ void stage_args(const A* src, unsigned char* dst) {
  static_assert(sizeof(A) % 4 == 0, "argument blocks are copied as 4-byte words");
  const int* s = reinterpret_cast<const int*>(src);
  int* d = reinterpret_cast<int*>(dst);
  for (int t = threadIdx.x; t < (int)(sizeof(A) / 4); t += blockDim.x) d[t] = __ldg(s + t);
}

template <typename R>
constexpr size_t stage_args_bytes() {
  size_t m = sizeof(FaceArgs<R>);
  m = sizeof(ViscArgs<R, R>) > m ? sizeof(ViscArgs<R, R>) : m;
  m = sizeof(UpdArgs<R>) > m ? sizeof(UpdArgs<R>) : m;
  m = sizeof(UpdArgs<double>) > m ? sizeof(UpdArgs<double>) : m;
  return (m + 15) & ~size_t(15);
}

// Dynamic shared memory of the persistent kernel: the largest face tile.
template <bool CHAR, int V, typename R>
constexpr size_t stage_smem() {
  constexpr size_t a = face_smem<0, CHAR, FaceTileV<0, V>::NP, FaceTileV<0, V>::TF, R>();
  constexpr size_t b = face_smem<1, CHAR, FaceTileV<1, V>::NP, FaceTileV<1, V>::TF, R>();
  constexpr size_t c = face_smem<2, CHAR, FaceTileV<2, V>::NP, FaceTileV<2, V>::TF, R>();
  return a > b ? (a > c ? a : c) : (b > c ? b : c);
}

template <int DIR, bool CHAR, int SCHEME, int V, typename R>
__device__ __forceinline__ void stage_face(const FaceArgs<R>& A, int bx, int by, int bz, R* sm) {
  constexpr int NP = FaceTileV<DIR, V>::NP, TF = FaceTileV<DIR, V>::TF;
  // the member's own sweep variant, as its single-instance launch chooses it
  if (OCFD_FEWER_DIVS && axis_aligned<DIR>(A.ph.metzero))
    face_body<DIR, CHAR, SCHEME, true, NP, TF, R, R, false, OCFD_FEWER_DIVS != 0>(A, bx, by, bz, sm);
  else
    face_body<DIR, CHAR, SCHEME, true, NP, TF, R, R>(A, bx, by, bz, sm);
}

// Minimum resident blocks per SM: those of the batched face kernels (the face
// bodies need the most registers).
template <bool CHAR, int SCHEME, int V, bool VISC, typename R>
__global__ void __launch_bounds__(256, OCFD_FACE_MINB) k_batch_stage(StageTab<R> t) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ __align__(16) unsigned char sa[stage_args_bytes<R>()];
  __shared__ int s_item, s_ok;
  R* const sm = reinterpret_cast<R*>(smem_raw);
  const int n = t.count;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(t.ctr, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= t.nitems) return;
    // the item's segment (binary search over the first items)
    int lo = 0, hi = t.nseg - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(&t.seg[mid].x) <= it)
        lo = mid;
      else
        hi = mid - 1;
    }
    const int4 e = __ldg(&t.seg[lo]);
    const int q = e.y >> 3, kind = e.y & 7;
    int l = it - e.x;
    const int bx = l % e.z;
    l /= e.z;
    const int by = l % e.w, bz = l / e.w;
    if (kind >= BW_TAIL) {
      if (threadIdx.x == 0) {
        const int2 nd = __ldg(&t.need[q]);
        int* const err = &t.negt[q].st->error;
        const bool ok = stage_wait(t.ctr + 1 + (kind == BW_TAIL ? q : n + q), kind == BW_TAIL ? nd.x : nd.y, err);
        if (!ok) atomicExch(err, 5);
        __threadfence();
        s_ok = ok;
      }
    }
    switch (kind) {
      case BW_FACE_X:
      case BW_FACE_Y:
      case BW_FACE_Z:
        stage_args(t.face[kind] + q, sa);
        break;
      case BW_VISC:
        stage_args(t.visc + q, sa);
        break;
      case BW_TAIL:
        stage_args(t.upd + q, sa);
        break;
      default:
        stage_args(t.negt + q, sa);
    }
    __syncthreads();
    if (kind < BW_TAIL || s_ok) {
      switch (kind) {
        case BW_FACE_X:
          stage_face<0, CHAR, SCHEME, V, R>(*reinterpret_cast<const FaceArgs<R>*>(sa), bx, by, bz, sm);
          break;
        case BW_FACE_Y:
          stage_face<1, CHAR, SCHEME, V, R>(*reinterpret_cast<const FaceArgs<R>*>(sa), bx, by, bz, sm);
          break;
        case BW_FACE_Z:
          stage_face<2, CHAR, SCHEME, V, R>(*reinterpret_cast<const FaceArgs<R>*>(sa), bx, by, bz, sm);
          break;
        case BW_VISC:
          if (VISC) {
            const ViscArgs<R, R>& A = *reinterpret_cast<const ViscArgs<R, R>*>(sa);
            if (OCFD_VISC_AXS && visc_axis_aligned(A.ph.metzero))
              visc_grad_body<R, R, OCFD_VISC_AXS != 0>(A, bx, by, bz);
            else
              visc_grad_body<R, R>(A, bx, by, bz);
          }
          break;
        case BW_TAIL:
          fused_body<CHAR, VISC, true, R>(*reinterpret_cast<const UpdArgs<R>*>(sa), bx, by, bz);
          break;
        default:
          if (threadIdx.x == 0) negt_fix_body(*reinterpret_cast<const UpdArgs<double>*>(sa));
      }
    }
    // every thread's stores are issued before thread 0 publishes the item
    // (the pattern of a grid barrier: block barrier, then one fence and the
    // count); the barrier also frees the shared memory for the next item
    __syncthreads();
    if (threadIdx.x == 0 && kind < BW_NEGT) {
      __threadfence();
      atomicAdd(t.ctr + 1 + (kind == BW_TAIL ? n + q : q), 1);
    }
  }
}

template <bool CHAR, int SCHEME, int V, typename R>
static cudaError_t launch_batch_stage_t(const StageTab<R>& t, int nblocks, cudaStream_t st, int* per_sm) {
  constexpr size_t smem = stage_smem<CHAR, V, R>();
  auto kern = k_batch_stage<CHAR, SCHEME, V, true, R>;
  if (nblocks == 0) {
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && per_sm) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kern, 256, smem);
    return e;
  }
  kern<<<nblocks, 256, smem, st>>>(t);
  return cudaGetLastError();
}

// One stage launch of nblocks persistent blocks.  nblocks == 0: sets the
// kernel's shared-memory limit and returns its resident blocks per SM in
// *per_sm (call outside graph capture).
template <typename R>
cudaError_t launch_batch_stage(bool chr, int scheme, int variant, const StageTab<R>& t, int nblocks, cudaStream_t st,
                               int* per_sm) {
  if (!chr && scheme == SCH_WENO7)
    return variant ? launch_batch_stage_t<false, SCH_WENO7, 1, R>(t, nblocks, st, per_sm)
                   : launch_batch_stage_t<false, SCH_WENO7, 0, R>(t, nblocks, st, per_sm);
  if (chr && scheme == SCH_OMP6)
    return variant ? launch_batch_stage_t<true, SCH_OMP6, 1, R>(t, nblocks, st, per_sm)
                   : launch_batch_stage_t<true, SCH_OMP6, 0, R>(t, nblocks, st, per_sm);
  return cudaErrorNotSupported;
}

}  // namespace ocfd
