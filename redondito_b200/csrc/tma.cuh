// tma.cuh -- 2D tensor-memory-accelerator (TMA) views of the physical grid
// and the tiled load that fills shared memory from them.
//
// A field's planes, (nz planes) x (nphi rows) x (nlat rings) in FP64, are
// seen as one 2D array of nlat columns and rows = nphi x planes; a box is
// `cols` consecutive rings of `rows` consecutive phi rows.  The loads are
// plain per-CTA copies of this GPU's own memory (no cluster multicast).
// A load's innermost coordinate (the ring) times the element size must be a
// multiple of 16 bytes: grid_map refuses boxes whose row is not, and callers
// pass ring indices that are multiples of the box width.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>
#include <stdint.h>

#include "tc05.cuh"

namespace tma {

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against the driver library)
static inline PFN_cuTensorMapEncodeTiled_v12000 encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }();
  return fn;
}

// 2D view [rows][nlat] of a grid array of FP64 or float values, box cols x
// box_rows; false when the encoder is missing, the base is not 16-byte
// aligned, or a grid row or a box row is not a multiple of 16 bytes (so that
// every ring index the callers use, a multiple of cols, is a multiple of 16
// bytes too).  With a swizzle mode of 2^B 16-byte chunks (64B: B = 2, 128B:
// B = 3) the box lands in shared memory with byte offset o moved to
// o ^ (((o >> 7) & (2^B - 1)) << 4): the 16-byte chunk index XORed with the
// 128-byte row index (destinations 1024-byte aligned).
template <typename T>
static inline bool grid_map(CUtensorMap* map, const T* base, int nlat, long long rows, int cols, int box_rows,
                            CUtensorMapL2promotion promo = CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                            CUtensorMapSwizzle swz = CU_TENSOR_MAP_SWIZZLE_NONE) {
  static_assert(sizeof(T) == 8 || sizeof(T) == 4, "FP64 or float grids");
  PFN_cuTensorMapEncodeTiled_v12000 enc = encoder();
  if (!enc || !base || rows < 1 || reinterpret_cast<uintptr_t>(base) % 16 || (nlat * sizeof(T)) % 16 ||
      (cols * sizeof(T)) % 16)
    return false;
  const cuuint64_t dims[2] = {(cuuint64_t)nlat, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)nlat * sizeof(T)};
  const cuuint32_t box[2] = {(cuuint32_t)cols, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  return enc(map, sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
             const_cast<T*>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, swz, promo,
             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// box at (ring x, row y) into this CTA's shared memory, completing on mbar
__device__ __forceinline__ void load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* mbar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
      "[%4];\n" ::"r"(tc05::smem_u32(dst)),
      "l"(map), "r"(x), "r"(y), "r"(tc05::smem_u32(mbar))
      : "memory");
}

__device__ __forceinline__ void expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}\n" ::"r"(
                   tc05::smem_u32(b)),
               "r"(bytes)
               : "memory");
}

}  // namespace tma
