// cluster.cuh -- thread-block cluster helpers: the CTA's rank, the cluster
// barrier, and loads from another CTA's shared memory (distributed shared
// memory) of the same cluster on this GPU.
#pragma once
#include <stdint.h>

#include "tc05.cuh"

namespace {

__device__ __forceinline__ uint32_t cluster_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;\n" : "=r"(r));
  return r;
}
__device__ __forceinline__ void cluster_sync_all() {
  asm volatile("barrier.cluster.arrive.release.aligned;\nbarrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// the cluster barrier with this warp's arrival either releasing (what the
// warp wrote or observed becomes visible to the cluster; its pending global
// stores drain first) or relaxed (no ordering: for warps whose only pending
// writes are global stores nobody in the cluster reads); `dep` is a value the
// arrival waits for (a result of loads that must have completed first)
__device__ __forceinline__ void cluster_sync_split(bool release, double dep = 0.0) {
  if (release)
    asm volatile("barrier.cluster.arrive.release.aligned;\n" ::"d"(dep) : "memory");
  else
    asm volatile("barrier.cluster.arrive.relaxed.aligned;\n" ::"d"(dep) : "memory");
  asm volatile("barrier.cluster.wait.acquire.aligned;\n" ::: "memory");
}
// shared::cluster address of `p` (a shared-memory location of this CTA) in CTA `rank`
__device__ __forceinline__ uint32_t cluster_map(const void* p, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;\n" : "=r"(r) : "r"(tc05::smem_u32(p)), "r"(rank));
  return r;
}
__device__ __forceinline__ double ld_cluster_f64(uint32_t addr) {
  double v;
  asm volatile("ld.shared::cluster.f64 %0, [%1];\n" : "=d"(v) : "r"(addr) : "memory");
  return v;
}
__device__ __forceinline__ int ld_cluster_s32(uint32_t addr) {
  int v;
  asm volatile("ld.shared::cluster.s32 %0, [%1];\n" : "=r"(v) : "r"(addr) : "memory");
  return v;
}

__host__ __device__ constexpr int largest_divisor_le(int n, int cap) {
  int d = cap < n ? cap : n;
  while (d > 1 && n % d) --d;
  return d;
}
__host__ __device__ constexpr size_t round_up(size_t x, size_t q) { return (x + q - 1) / q * q; }

}  // namespace
