// Standalone transform passes: batched c2c along a strided axis and r2c/c2r
// along the contiguous (last) axis.  A 3D rfftn is Zr2c -> Yc2c -> Xc2c, the
// inverse is Xc2c -> Yc2c -> Zc2r (c2c axes first, then c2r on the last axis,
// the order numpy.fft.irfftn and mpi4py-fft's PFFT.backward use, which fixes
// how the imaginary parts of the zero/Nyquist bins are discarded).
#pragma once
#include "sles_fft.cuh"

namespace sles {

// Twiddles exp(-2 pi i k/N), k < N/2, for the real<->half-complex step,
// filled cooperatively into shared memory (float64, rounded once).
template <typename Tp, int NR>
__device__ __forceinline__ void fill_twN(typename CT<Tp>::C* tw) {
  for (int k = threadIdx.x; k < NR / 2; k += blockDim.x) tw[k] = twiddle<Tp>(k, NR, -1);
}

// ---------------------------------------------------------------------------
// c2c along a strided axis.  Work item = (field f, slice a, column chunk c):
// W consecutive columns of the half-complex rows, each a line of N points
// spaced pstride elements apart.  Block = G items x W columns x T threads.
// ---------------------------------------------------------------------------
template <typename Tp, int N, int W, int G>
struct C2CAxis {
  using F = typename PlanFor<Tp, N>::F;
  using C = typename CT<Tp>::C;
  static constexpr int T = F::T;
  static constexpr int V = F::V;
  static constexpr int THREADS = G * W * T;
  static constexpr int SCR = F::XLEN * W;  // per item
  static constexpr size_t SMEM = (size_t)G * SCR * sizeof(C);
};

template <typename Tp, int N, int W, int G, int DIR>
__global__ void __launch_bounds__(C2CAxis<Tp, N, W, G>::THREADS)
k_c2c_axis(const typename CT<Tp>::C* src, typename CT<Tp>::C* dst,  // may alias (in place)
           long long fstride, int nfields, int na, long long astride, long long pstride,
           int ncols, int nchunks, Tp scale) {
  using K = C2CAxis<Tp, N, W, G>;
  using C = typename K::C;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  C* scr = reinterpret_cast<C*>(smem_raw);
  const int tid = threadIdx.x;
  const int l = tid % W, j = (tid / W) % K::T, g = tid / (W * K::T);
  typename K::F fft;
  fft.init(j);
  const long long items = (long long)nfields * na * nchunks;
  const long long nbi = (items + G - 1) / G;
  for (long long bi = blockIdx.x; bi < nbi; bi += gridDim.x) {  // persistent over work items
    const long long it = bi * G + g;
    const int chunk = (int)(it % nchunks);
    const long long rest = it / nchunks;
    const int a = (int)(rest % na);
    const int f = (int)(rest / na);
    const int col = chunk * W + l;
    const bool ok = (f < nfields) && (col < ncols);
    const long long base = ok ? (long long)f * fstride + (long long)a * astride + col : 0;
    C v[K::V];
#pragma unroll
    for (int m = 0; m < K::V; ++m)
      v[m] = ok ? src[base + (long long)(j + K::T * m) * pstride] : cmk<C>(0, 0);
    fft.template run<DIR>(v, j, scr + g * K::SCR + l, W);
    if (ok) {
#pragma unroll
      for (int m = 0; m < K::V; ++m) dst[base + (long long)(j + K::T * m) * pstride] = cscale(v[m], scale);
    }
  }
}

// ---------------------------------------------------------------------------
// r2c / c2r along the contiguous axis.  Work item = one line; block = LPB
// lines x T threads.  Real lines have NR points at stride NR, half-complex
// lines NR/2+1 bins at stride NKP.
// ---------------------------------------------------------------------------
template <typename Tp, int NR, int LPB>
struct RealAxis {
  using F = typename MirrorIf<typename PlanFor<Tp, NR / 2>::F>::type;  // mirrored where the plan allows
  using C = typename CT<Tp>::C;
  static constexpr int L = NR / 2;
  static constexpr int T = F::T;
  static constexpr int THREADS = LPB * T;
  static constexpr int LS = ((F::XLEN + 15) / 16) * 16 + 8;  // line stride of the scratch
  static constexpr size_t SMEM = ((size_t)LPB * LS + L) * sizeof(C);
  static constexpr int WS = (T <= 32 && 32 % T == 0) ? 1 : 0;  // a line's threads share one warp
};

template <typename Tp, int NR, int LPB>
__global__ void __launch_bounds__(RealAxis<Tp, NR, LPB>::THREADS)
k_r2c_line(const Tp* __restrict__ src, typename CT<Tp>::C* __restrict__ dst, long long nlines, int NKP) {
  using K = RealAxis<Tp, NR, LPB>;
  using C = typename K::C;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  C* twN = reinterpret_cast<C*>(smem_raw);
  C* scr = twN + K::L;
  fill_twN<Tp, NR>(twN);
  __syncthreads();  // twN is read by every line (its barriers may be line-level only)
  const int tid = threadIdx.x;
  const int j = tid % K::T, ln = tid / K::T;
  typename K::F fft;
  fft.init(j);
  const long long nbi = (nlines + LPB - 1) / LPB;
  for (long long bi = blockIdx.x; bi < nbi; bi += gridDim.x) {
    const long long line = bi * LPB + ln;
    const bool ok = line < nlines;
    const C* in = reinterpret_cast<const C*>(src + (ok ? line : 0) * NR);
    C* out = dst + (ok ? line : 0) * NKP;
    C v[K::F::V];
#pragma unroll
    for (int m = 0; m < K::F::V; ++m) v[m] = ok ? in[j + K::T * m] : cmk<C>(0, 0);
    fft.template run<-1, K::WS>(v, j, scr + ln * K::LS, 1);
    if constexpr (K::F::MIR) {
      r2c_post_mir<typename K::F>(v, j, twN, [&](int k, C x) {
        if (ok) out[k] = x;
      });
    } else {
      r2c_post<typename K::F, K::WS>(v, j, scr + ln * K::LS, 1, twN, [&](int k, C x) {
        if (ok) out[k] = x;
      });
    }
  }
}

template <typename Tp, int NR, int LPB>
__global__ void __launch_bounds__(RealAxis<Tp, NR, LPB>::THREADS)
k_c2r_line(const typename CT<Tp>::C* __restrict__ src, Tp* __restrict__ dst, long long nlines, int NKP,
           Tp scale) {
  using K = RealAxis<Tp, NR, LPB>;
  using C = typename K::C;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  C* twN = reinterpret_cast<C*>(smem_raw);
  C* scr = twN + K::L;
  fill_twN<Tp, NR>(twN);
  __syncthreads();
  const int tid = threadIdx.x;
  const int j = tid % K::T, ln = tid / K::T;
  typename K::F fft;
  fft.init(j);
  const long long nbi = (nlines + LPB - 1) / LPB;
  for (long long bi = blockIdx.x; bi < nbi; bi += gridDim.x) {
    const long long line = bi * LPB + ln;
    const bool ok = line < nlines;
    const C* in = src + (ok ? line : 0) * NKP;
    C* out = reinterpret_cast<C*>(dst + (ok ? line : 0) * NR);
    C v[K::F::V];
    c2r_pre<typename K::F>(v, j, twN, [&](int k) { return ok ? in[k] : cmk<C>(0, 0); });
    fft.template run<+1, K::WS>(v, j, scr + ln * K::LS, 1);
    if (ok) {
#pragma unroll
      for (int m = 0; m < K::F::V; ++m) out[K::F::pos(j, m)] = cscale(v[m], scale);
    }
  }
}

}  // namespace sles
