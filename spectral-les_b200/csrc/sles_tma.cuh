// TMA tensor-tile staging for the strided-axis passes.
//
// A half-complex field set is addressed as a 4D tensor of 8-byte elements
// (complex64 = 1 element, complex128 = 2):
//   dim0: last-axis wavenumber columns (extent nk*EPC; columns past nk are
//         out of bounds and arrive zero-filled without touching DRAM)
//   dim1: the transformed axis (rows, the FFT line)
//   dim2: the slice index (the remaining axis)
//   dim3: the field slot
// A tile is one box [W columns x rows] of one slot/slice, i.e. W lines of the
// transform, landing densely in shared memory as [rows][W].  Boxes are at most
// 256 rows, so N = 512 / 1024 lines take 2 / 4 boxes.  The innermost
// coordinate is always chunk*W*EPC elements = chunk*64 bytes: 16-byte aligned.
//
// Tiles of a kernel's fixed per-item sequence are prefetched into a ring of
// NBUF buffers, each completed on its own mbarrier; consumers wait with a
// bounded spin (see sles_common.cuh).
#pragma once
#include <cuda.h>

#include "sles_common.cuh"

namespace sles {

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_load_5d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, "
      "%6}], [%7];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(smem_addr(bar))
      : "memory");
}

__device__ __forceinline__ void tma_prefetch_desc(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(map)) : "memory");
}

// Ring of NBUF tile buffers of TE complex elements each.
template <typename C, int NBUF, int TE>
struct TileRing {
  uint64_t* bar;
  C* buf;

  __device__ __forceinline__ void init(unsigned char* base, int tid) {
    bar = reinterpret_cast<uint64_t*>(base);
    buf = reinterpret_cast<C*>(base + 1024);  // tiles 1024-byte aligned
    if (tid == 0) {
      for (int i = 0; i < NBUF; ++i) mbar_init(&bar[i], 1);
      fence_mbar_init();
    }
  }
  static constexpr size_t bytes() { return 1024 + (size_t)NBUF * TE * sizeof(C); }
  __device__ __forceinline__ C* tile(long long t) { return buf + (int)(t % NBUF) * TE; }

  // thread 0: load sequence tile t = `nbox` boxes of `rows_per_box` rows of
  // (slot, slice, column chunk) into buffer t % NBUF
  __device__ __forceinline__ void issue(long long t, const CUtensorMap* map, int c0, int slice, int slot, int nbox,
                                        int rows_per_box, unsigned box_bytes) {
    uint64_t* b = &bar[t % NBUF];
    C* dst = tile(t);
    fence_proxy_async();
    mbar_arrive_expect_tx(b, box_bytes * nbox);
    for (int k = 0; k < nbox; ++k)
      tma_load_4d(dst + (long long)k * (TE / nbox), map, c0, k * rows_per_box, slice, slot, b);
  }
  // thread 0: the same with the box rows along the slice axis (dim 2) at the
  // fixed row `row` (dim 1): x-pass tiles [x][W] at one ky
  // (slice0: the first slice of the line, e.g. a batched member's offset)
  __device__ __forceinline__ void issue_rows(long long t, const CUtensorMap* map, int c0, int row, int slice0,
                                             int slot, int nbox, int rows_per_box, unsigned box_bytes) {
    uint64_t* b = &bar[t % NBUF];
    C* dst = tile(t);
    fence_proxy_async();
    mbar_arrive_expect_tx(b, box_bytes * nbox);
    for (int k = 0; k < nbox; ++k)
      tma_load_4d(dst + (long long)k * (TE / nbox), map, c0, row, slice0 + k * rows_per_box, slot, b);
  }
  // thread 0: one 5D box {cols, M rows, 1 slice, P blocks, 1 slot} holding a
  // whole line split in P blocks of M rows (the slab exchange buffer, where
  // the rows of a line arrive from P ranks); lands as [P][M][W] = [rows][W]
  __device__ __forceinline__ void issue_split(long long t, const CUtensorMap* map, int c0, int slice, int slot,
                                              unsigned bytes) {
    uint64_t* b = &bar[t % NBUF];
    fence_proxy_async();
    mbar_arrive_expect_tx(b, bytes);
    tma_load_5d(tile(t), map, c0, 0, slice, 0, slot, b);
  }
  __device__ __forceinline__ void wait(long long t, unsigned* err) {
    mbar_wait_bounded(&bar[t % NBUF], (unsigned)((t / NBUF) & 1), err);
  }
};

}  // namespace sles
