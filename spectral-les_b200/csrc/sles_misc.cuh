// Pointwise spectral kernels and float64 diagnostics.
#pragma once
#include "sles_common.cuh"

namespace sles {

// index -> (kx, ky, kz) wavenumbers of a half-complex element; returns false
// for padding columns.  3D layout [N][N][nkp], 2D [N][nkp].
template <int DIM>
__device__ __forceinline__ bool hc_k(long long e, int N, int nkp, int nk, int (&k)[3]) {
  const int col = (int)(e % nkp);
  if (col >= nk) return false;
  const long long row = e / nkp;
  if (DIM == 3) {
    k[0] = kc2c((int)(row / N), N);
    k[1] = kc2c((int)(row % N), N);
    k[2] = col;
  } else {
    k[0] = kc2c((int)row, N);
    k[1] = col;
    k[2] = 0;
  }
  return true;
}

// curl_hat = i k x U_hat (3 fields in 3D, 1 in 2D): math_formula.py:16-25
template <typename Tp, int DIM>
__global__ void k_curl_hat(const typename CT<Tp>::C* __restrict__ uh, typename CT<Tp>::C* __restrict__ out,
                           long long fs, int N, int nkp, int nk) {
  using C = typename CT<Tp>::C;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < fs; e += (long long)gridDim.x * blockDim.x) {
    int k[3];
    if (!hc_k<DIM>(e, N, nkp, nk, k)) continue;
    const Tp kx = (Tp)k[0], ky = (Tp)k[1], kz = (Tp)k[2];
    if (DIM == 3) {
      const C u = uh[e], v = uh[fs + e], w = uh[2 * fs + e];
      out[2 * fs + e] = cmuli(csub(cscale(v, kx), cscale(u, ky)));
      out[fs + e] = cmuli(csub(cscale(u, kz), cscale(w, kx)));
      out[e] = cmuli(csub(cscale(w, ky), cscale(v, kz)));
    } else {
      const C u = uh[e], v = uh[fs + e];
      out[e] = cmuli(csub(cscale(v, kx), cscale(u, ky)));
    }
  }
}

// out_j = i K_axis U_hat_j for j < DIM: one row of the velocity gradient
template <typename Tp, int DIM>
__global__ void k_deriv_hat(const typename CT<Tp>::C* __restrict__ uh, typename CT<Tp>::C* __restrict__ out,
                            long long fs, int N, int nkp, int nk, int axis) {
  using C = typename CT<Tp>::C;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < fs; e += (long long)gridDim.x * blockDim.x) {
    int k[3];
    if (!hc_k<DIM>(e, N, nkp, nk, k)) continue;
    const Tp ka = (Tp)k[axis];
#pragma unroll
    for (int c = 0; c < DIM; ++c) out[c * fs + e] = cmuli(cscale(uh[c * fs + e], ka));
  }
}

// y -= x over n complex elements (ETD2 bootstrap bookkeeping)
template <typename Tp>
__global__ void k_csub_inplace(typename CT<Tp>::C* __restrict__ y, const typename CT<Tp>::C* __restrict__ x,
                               long long n) {
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x)
    y[e] = csub(y[e], x[e]);
}

// Kahan-compensated accumulator in float64
struct KSum {
  double s = 0, c = 0;
  __device__ __forceinline__ void add(double x) {
    double y = x - c;
    double t = s + y;
    c = (t - s) - y;
    s = t;
  }
};

constexpr int DIAG_THREADS = 256;
constexpr int DIAG_BLOCKS = 592;  // 4 x 148 SMs

// Per-block partials of E and eps (and the shell spectrum) from U_hat.
// partial layout: [block][2 + nshell] doubles.
template <typename Tp, int DIM>
__global__ void __launch_bounds__(DIAG_THREADS)
k_diag_partial(const typename CT<Tp>::C* __restrict__ uh, long long fs, int N, int nkp, int nk, double* partial,
               int nshell) {
  extern __shared__ double sh[];  // nshell + 2*DIAG_THREADS
  double* hist = sh;
  double* red = sh + nshell;
  for (int i = threadIdx.x; i < nshell; i += blockDim.x) hist[i] = 0;
  __syncthreads();
  KSum e, d;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < fs; i += (long long)gridDim.x * blockDim.x) {
    int k[3];
    if (!hc_k<DIM>(i, N, nkp, nk, k)) continue;
    const int kl = (DIM == 3) ? k[2] : k[1];
    const double w = (kl > 0 && kl < N / 2) ? 2.0 : 1.0;
    double a = 0;
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      const double re = (double)uh[c * fs + i].x, im = (double)uh[c * fs + i].y;
      a += re * re + im * im;
    }
    const double k2 = (double)(k[0] * k[0] + k[1] * k[1] + k[2] * k[2]);
    e.add(w * a);
    d.add(w * a * k2);
    if (nshell > 0) {
      const int sidx = (int)rint(sqrt(k2));
      if (sidx < nshell) atomicAdd(&hist[sidx], w * a);
    }
  }
  red[threadIdx.x] = e.s;
  red[DIAG_THREADS + threadIdx.x] = d.s;
  __syncthreads();
  for (int s = DIAG_THREADS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      red[threadIdx.x] += red[threadIdx.x + s];
      red[DIAG_THREADS + threadIdx.x] += red[DIAG_THREADS + threadIdx.x + s];
    }
    __syncthreads();
  }
  double* out = partial + (long long)blockIdx.x * (2 + nshell);
  if (threadIdx.x == 0) {
    out[0] = red[0];
    out[1] = red[DIAG_THREADS];
  }
  for (int i = threadIdx.x; i < nshell; i += blockDim.x) out[2 + i] = hist[i];
}

// Signed max over nf real fields (find_max_velocity, SM_solver.py:245-255)
template <typename Tp>
__global__ void __launch_bounds__(DIAG_THREADS)
k_max_partial(const Tp* __restrict__ u, long long n, double* partial) {
  __shared__ double red[DIAG_THREADS];
  double m = -INFINITY;
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double x = (double)u[i];
    bad |= !isfinite(x);
    m = fmax(m, x);
  }
  red[threadIdx.x] = bad ? NAN : m;
  __syncthreads();
  for (int s = DIAG_THREADS / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      const double a = red[threadIdx.x], b = red[threadIdx.x + s];
      red[threadIdx.x] = (isnan(a) || isnan(b)) ? NAN : fmax(a, b);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Final ordered reduction of the partials: out[0]=E, out[1]=eps, out[2]=umax,
// out[3]=nonfinite flag; spectrum[i] (optional).
static __global__ void k_diag_final(const double* __restrict__ partial, int nblk, int nshell, const double* __restrict__ mpart,
                             int mblk, double norm, double nu, double* out, double* spectrum) {
  const int t = threadIdx.x;
  if (t == 0) {
    KSum e, d;
    for (int b = 0; b < nblk; ++b) {
      e.add(partial[(long long)b * (2 + nshell)]);
      d.add(partial[(long long)b * (2 + nshell) + 1]);
    }
    const double E = 0.5 * e.s * norm, eps = nu * d.s * norm;
    double m = -INFINITY;
    bool bad = !isfinite(E) || !isfinite(eps);
    for (int b = 0; b < mblk; ++b) {
      if (isnan(mpart[b])) bad = true;
      else m = fmax(m, mpart[b]);
    }
    out[0] = E;
    out[1] = eps;
    out[2] = mblk > 0 ? m : NAN;
    out[3] = bad ? 1.0 : 0.0;
  }
  if (spectrum) {
    for (int i = t; i < nshell; i += blockDim.x) {
      KSum s;
      for (int b = 0; b < nblk; ++b) s.add(partial[(long long)b * (2 + nshell) + 2 + i]);
      spectrum[i] = 0.5 * s.s * norm;
    }
  }
}

}  // namespace sles
