// Common device helpers for the spectral-LES B200 kernels.
//
// Complex numbers are float2/double2.  Field layouts (all row-major, C order):
//   half-complex 3D field:  [N][N][NKP] complex, kz fastest, NKP = round_up(N/2+1, 4)
//                           (padding keeps every row 32-byte aligned; columns
//                           N/2+1..NKP-1 are never read as data)
//   half-complex 2D field:  [N][NKP] complex
//   physical 3D field:      [N][N][N] real, z fastest;  2D: [N][N]
// Wavenumbers follow the reference (src/initialize_domain.py:76-79): on the
// c2c axes k = i for i < N/2 and i - N otherwise (index N/2 -> -N/2); on the
// r2c axis k = i for i in [0, N/2] (index N/2 -> +N/2).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace sles {

template <typename Tp> struct CT;
template <> struct CT<float> { using C = float2; };
template <> struct CT<double> { using C = double2; };

template <typename C> __device__ __forceinline__ C cmk(decltype(C::x) a, decltype(C::x) b) { C r; r.x = a; r.y = b; return r; }
template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return cmk<C>(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return cmk<C>(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) { return cmk<C>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// a * conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) { return cmk<C>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y); }
template <typename C> __device__ __forceinline__ C cconj(C a) { return cmk<C>(a.x, -a.y); }
// i * a
template <typename C> __device__ __forceinline__ C cmuli(C a) { return cmk<C>(-a.y, a.x); }
// -i * a
template <typename C> __device__ __forceinline__ C cmulmi(C a) { return cmk<C>(a.y, -a.x); }
template <typename C, typename S> __device__ __forceinline__ C cscale(C a, S s) { return cmk<C>(a.x * s, a.y * s); }
// i * s * a  (s real)
template <typename C, typename S> __device__ __forceinline__ C cmuli_s(C a, S s) { return cmk<C>(-a.y * s, a.x * s); }

// wavenumber of index i on a c2c axis of length n (numpy.fft.fftfreq * n)
__device__ __forceinline__ int kc2c(int i, int n) { return i < n / 2 ? i : i - n; }

// error flags written by kernels (bitwise OR into a device word)
enum : unsigned {
  SLES_ERRF_NONE = 0u,
  SLES_ERRF_WAIT_TIMEOUT = 1u,   // a bounded wait on an mbarrier gave up
  SLES_ERRF_NONFINITE = 2u,      // a reduction saw NaN/Inf
};

__device__ __forceinline__ void raise_flag(unsigned* flag, unsigned bit) {
  if (flag) atomicOr(flag, bit);
}

// ---------------------------------------------------------------------------
// TMA bulk copies (global -> shared) completed on an mbarrier.  Every wait is
// bounded: after MBAR_SPIN_LIMIT polls the wait raises SLES_ERRF_WAIT_TIMEOUT
// in the error word and returns false, so a kernel never spins forever.
// ---------------------------------------------------------------------------
constexpr long MBAR_SPIN_LIMIT = 1L << 21;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// order this thread's earlier generic-proxy shared accesses before later async-proxy ones
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, unsigned* flag,
                                                  long limit = MBAR_SPIN_LIMIT) {
  for (long it = 0; it < limit; ++it)
    if (mbar_try_wait(bar, parity)) return true;
  raise_flag(flag, SLES_ERRF_WAIT_TIMEOUT);
  return false;
}

// Self-test of the timeout path: waits on an mbarrier that nothing arrives
// at; the bounded wait gives up after `limit` polls and raises the flag.
// Rows of `w` 8-byte words from src (row pitch sp) to dst (row pitch dp),
// one warp per row (coalesced row segments): padded <-> contiguous fields.
static __global__ void k_copy_rows8(unsigned long long* __restrict__ dst, long long dp,
                                   const unsigned long long* __restrict__ src, long long sp, int w, long long h) {
  const long long row = (long long)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
  if (row >= h) return;
  const unsigned long long* s = src + row * sp;
  unsigned long long* d = dst + row * dp;
  for (int c = threadIdx.x & 31; c < w; c += 32) d[c] = s[c];
}

static __global__ void k_wait_selftest(unsigned* flag, long limit) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_wait_bounded(&bar, 0, flag, limit);
}

// bytes must be a multiple of 16; both addresses 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}

// Per-thread asynchronous copy of one complex element (8 or 16 bytes) from
// global to shared memory; pred = false zero-fills without reading.  A thread
// waits for its own groups only (cp.async.wait_group), so a buffer that each
// thread fills and later reads at the same positions needs no block barrier.
template <int BYTES>
__device__ __forceinline__ void cp_async_el(void* dst, const void* src, bool pred) {
  static_assert(BYTES == 8 || BYTES == 16, "8- or 16-byte elements");
  if (BYTES == 8)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(pred ? 8 : 0)
                 : "memory");
  else
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_addr(dst)), "l"(src), "r"(pred ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory"); }

// exp(sign * 2 pi i e / m) computed in float64 and rounded once to Tp
template <typename Tp>
__device__ __forceinline__ typename CT<Tp>::C twiddle(long long e, long long m, int sign) {
  double s, c;
  sincospi(2.0 * (double)(e % m) / (double)m, &s, &c);
  using C = typename CT<Tp>::C;
  return cmk<C>((Tp)c, (Tp)(sign * s));
}

}  // namespace sles
