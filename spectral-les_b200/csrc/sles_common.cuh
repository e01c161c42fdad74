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

// exp(sign * 2 pi i e / m) computed in float64 and rounded once to Tp
template <typename Tp>
__device__ __forceinline__ typename CT<Tp>::C twiddle(long long e, long long m, int sign) {
  double s, c;
  sincospi(2.0 * (double)(e % m) / (double)m, &s, &c);
  using C = typename CT<Tp>::C;
  return cmk<C>((Tp)c, (Tp)(sign * s));
}

}  // namespace sles
