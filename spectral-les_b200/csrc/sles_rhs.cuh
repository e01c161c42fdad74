// Fused right-hand side + stage update (2D and 3D).
//
// One RHS evaluation in 3D is four kernels, each a single HBM pass:
//
//   Y1  inverse y-FFT      (x, ky, kz) -> (x, y, kz); applies i*ky where a
//                          y-derivative is needed
//   Z   fused z pass       per (x, y) line: c2r of the velocity and derivative
//                          lines, pointwise u x omega and the eddy-viscosity
//                          stress (Smagorinsky or Vreman), r2c of the products
//   Y2  forward y-FFT      adds the ky, kz parts of div(tau)
//   X   fused x pass       forward x-FFT, kx part of div(tau), 2/3 mask,
//                          projection, forcing, viscous term, the integrator's
//                          stage update, then the inverse x-FFT (and i*kx) of
//                          the new state, which primes the next evaluation
//
// In 2D the r2c axis is y (axis 1): X and Z(=y) passes only.
// Physical fields never touch HBM.  Derivatives along an axis are applied
// while that axis is still spectral, so the inverse passes carry 6 (LES) or
// 5 (no LES) fields rather than the 12 the reference transforms.
//
// Workspace slots (half-complex fields, updated in place pass to pass):
//  3D LES:   X -> [0..2] A_c = X^-1(u_c), [3..5] B_c = X^-1(i kx u_c)
//            Y1 -> [0..2] a_c, [3..5] dx_c, [6..8] dy_c
//            Z  -> [0..2] N_c = rfft(u x omega), [3..8] F_xx F_xy F_xz F_yy F_yz F_zz
//                  (F_ij = rfft(nu_t S_ij))
//            Y2 -> [0..2] G_c = N_c + 2i(ky F_cy + kz F_cz), [3..5] H_c = F_cx
//  3D plain: X -> [0..2] A_c, [3] X^-1(-i kx w), [4] X^-1(i kx v)
//            Y1 -> [0..2] a_c, [3] Oy, [4] Oz, [5] Ox (curl parts without kz)
//            Z  -> [0..2] N_c;  Y2 -> [0..2] in place
//  2D plain: X -> [0] A_u, [1] A_v, [2] X^-1(i kx v);  Z -> [0] rfft(v w), [1] rfft(-u w)
//  2D LES:   X -> [0] A_u, [1] A_v, [2] X^-1(i kx u), [3] X^-1(i kx v)
//            Z -> [0] N_0, [1] N_1, then F12, F22 (reference arithmetic) or
//                 F11, F12, F22 (corrected stress)
//
// Reference: computeRHS, src/RK4_method.py:38-71; U_cross_omega / del_cross_U /
// velocity_gradient / residue_stress, src/math_formula.py:5-146;
// calculate_nuR, src/smagorinsky.py:24-47 and src/vreman.py:30-147.
#pragma once
#include "sles_passes.cuh"
#include "sles_tma.cuh"

namespace sles {

enum StageKind { KX_RHS = 0, KX_RK4 = 1, KX_RK3P = 2, KX_SSP3 = 3, KX_ETD2P = 4, KX_ETD2C = 5, KX_RAW = 6 };
enum LesModel { M_NONE = 0, M_SMAG = 1, M_VREMAN = 2 };

template <typename Tp>
struct XArgs {
  using C = typename CT<Tp>::C;
  int need_uc, need_u0, need_u1;  // which state fields the stage reads (u0 aliasing ucur: need_u0 = 0)
  unsigned* err;
  C* ws;                 // workspace slot 0
  long long fs;          // elements per half-complex field
  int nkp, nk, nchunks;
  int nsl, ky0;          // 3D: ky slices held (N, or N/P on a slab) and the global index of the first
  int nmem;              // ensemble members batched in the plan (1: a single domain)
  long long mstride;     // elements between two members' parts of a field
  const double* mnu;     // per-member viscosity (device, nmem values) or null: nu_d for all
  int fwd;               // 1: forward part (RHS from the slots), 0: inverse only from uinv
  int prep;              // 1: inverse part (prime the slots for the next evaluation)
  const C* uinv;         // inverse-only source
  const C* ucur;         // state the RHS is evaluated at
  const C* u0;
  C* u1;
  C* uout;
  C* aux;                // ETD2: new F1; record_f1: recorded F1
  int kind, stage;
  int record_f1;         // 1: aux = projected term; 2: aux = projected term - aux
  Tp nu, forcing;
  double kmax;
  Tp c1, c2;             // stage coefficients (host-computed in float64)
  double nu_d, dt_d;     // ETD2 weights are evaluated in float64
  const double* dt_dev;  // non-null: dt read on the device (c1 = m1 dt, c2 = m2 dt, dt_d = dt)
  double m1, m2;
};

// The stage's coefficients: host-computed, or from a device-side dt (adaptive
// steps without host synchronisation; the products are the host's, in float64)
template <typename Tp>
struct StageCoef {
  Tp c1, c2;
  double dt;
};
template <typename Tp>
__device__ __forceinline__ StageCoef<Tp> stage_coef(const XArgs<Tp>& A) {
  if (!A.dt_dev) return StageCoef<Tp>{A.c1, A.c2, A.dt_d};
  const double dt = *A.dt_dev;
  return StageCoef<Tp>{(Tp)(A.m1 * dt), (Tp)(A.m2 * dt), dt};
}

// Per-position mask and projection for D velocity components (in place):
// R <- mask * R, then R <- R - k (k . R)/|k|^2 (src/RK4_method.py:48-57);
// KX_RAW keeps the masked term unprojected (the LES stress T_hat alone).
template <typename Tp, int D>
__device__ __forceinline__ void project(const XArgs<Tp>& A, typename CT<Tp>::C (&R)[D], const int (&k)[D]) {
  using C = typename CT<Tp>::C;
  int k2 = 0;
  bool in = true;
#pragma unroll
  for (int c = 0; c < D; ++c) {
    k2 += k[c] * k[c];
    in = in && fabs((double)k[c]) < A.kmax;  // initialize_domain.py:109-114
  }
  const double kk = (double)(k2 == 0 ? 1 : k2);  // K_over_K2, initialize_domain.py:163-165
  C P = cmk<C>(0, 0);
#pragma unroll
  for (int c = 0; c < D; ++c) {
    R[c] = in ? R[c] : cmk<C>(0, 0);
    P = cadd(P, cscale(R[c], (Tp)((double)k[c] / kk)));
  }
  if (A.kind == KX_RAW) return;
#pragma unroll
  for (int c = 0; c < D; ++c) R[c] = csub(R[c], cscale(P, (Tp)k[c]));
}

// Stage update of one component at one position.  R: projected term of
// component c; uc/u0/u1: state values at this position (u1: RK4 accumulator
// or ETD2's previous F1).  Writes uout/u1/aux and returns the new state.
// ETD = 0 drops the exponential schemes (their float64 weights) from the
// kernel, which keeps the Runge-Kutta kernels' register count down.
// nud: the member's viscosity (float64; the working precision rounds it once).
template <typename Tp, int ETD>
__device__ __forceinline__ typename CT<Tp>::C update_component(const XArgs<Tp>& A, const StageCoef<Tp>& K, int c,
                                                              typename CT<Tp>::C R,
                                                              typename CT<Tp>::C uc, typename CT<Tp>::C u0,
                                                              typename CT<Tp>::C u1, int k2, long long off,
                                                              double nud) {
  using C = typename CT<Tp>::C;
  const long long o = c * A.fs + off;
  if (A.kind == KX_RAW) {
    A.uout[o] = R;
    return R;
  }
  if (A.forcing > (Tp)0 && k2 != 0) R = cadd(R, cscale(uc, A.forcing));  // RK4_method.py:58-64
  if (A.record_f1) A.aux[o] = (A.record_f1 == 2) ? csub(R, A.aux[o]) : R;  // RK4_method.py:65-66
  C un;
  if (ETD && (A.kind == KX_ETD2P || A.kind == KX_ETD2C)) {
    // parity: src/ETD2_method.py:16-29; corrected: Cox & Matthews (2002) eq. 22
    const double z = K.dt * nud * (double)k2;
    const double E = exp(-K.dt * nud * (double)k2);
    double w1, w0;
    if (A.kind == KX_ETD2P) {
      const double nk2 = nud * (double)k2;
      const double den = (k2 == 0) ? 1.0 : K.dt * (nk2 * nk2);
      w1 = ((1.0 - z) + 2.0 * z) / den;
      w0 = (-E + 1.0 - z) / den;
    } else if (fabs(z) < 1e-2) {
      const double h = K.dt;
      w1 = h * (1.5 - 2.0 * z / 3.0 + z * z / 4.0 - z * z * z / 15.0);
      w0 = h * (-0.5 + z / 6.0 - z * z / 24.0 + z * z * z / 120.0);
    } else {
      const double h = K.dt;
      w1 = h * ((1.0 - z) * E - 1.0 + 2.0 * z) / (z * z);
      w0 = h * (-E + 1.0 - z) / (z * z);
    }
    un = cadd(cscale(uc, (Tp)E), cadd(cscale(R, (Tp)w1), cscale(u1, (Tp)w0)));
    // a paused step under device-side dt (dt = 0) passes the previous F1 through,
    // so the two-step history is the same when the run resumes
    A.aux[o] = (A.dt_dev && K.dt == 0.0) ? u1 : R;
    A.uout[o] = un;
    return un;
  }
  const C dU = csub(R, cscale(uc, (Tp)nud * (Tp)k2));  // (nu * K2) * U_hat, RK4_method.py:67-68
  switch (A.kind) {
    case KX_RK4:  // RK4_method.py:20-27
      if (A.stage < 3) {
        A.u1[o] = cadd(u1, cscale(dU, K.c1));
        un = cadd(u0, cscale(dU, K.c2));
      } else {
        un = cadd(u1, cscale(dU, K.c1));
        A.u1[o] = un;
      }
      break;
    case KX_RK3P:  // RK3_method.py:26-33
      if (A.stage == 0) {
        un = cadd(u0, cscale(dU, K.c2));
      } else if (A.stage == 1) {
        un = cadd(csub(u0, cscale(dU, K.c1)), cscale(dU, K.c2));
      } else {
        const C t = cadd(cadd(cscale(dU, (Tp)(1.0 / 6.0)), cscale(dU, (Tp)(2.0 / 3.0))), cscale(dU, (Tp)(1.0 / 6.0)));
        un = cadd(u0, cscale(t, K.c1));
      }
      break;
    case KX_SSP3:  // Shu & Osher (1988)
      if (A.stage == 0) {
        un = cadd(u0, cscale(dU, K.c1));
      } else if (A.stage == 1) {
        un = cadd(cscale(u0, (Tp)0.75), cscale(cadd(uc, cscale(dU, K.c1)), (Tp)0.25));
      } else {
        un = cadd(cscale(u0, (Tp)(1.0 / 3.0)), cscale(cadd(uc, cscale(dU, K.c1)), (Tp)(2.0 / 3.0)));
      }
      break;
    default:  // KX_RHS
      un = dU;
      break;
  }
  A.uout[o] = un;
  return un;
}

// ---------------------------------------------------------------------------
// Strided-axis pass geometry: one work item (W lines of N points) per block
// iteration; tiles arrive by TMA into a ring of NBUF buffers.
// ---------------------------------------------------------------------------
// WSET > 0 sets the tile width (the y-pass variant with the other width)
template <typename Tp, int N, class F, bool RING = true, int NBUF_SET = 0, int WIDE = 0, int WSET = 0>
struct TGeo {
  using C = typename CT<Tp>::C;
#ifndef SLES_Y_W
#define SLES_Y_W 0
#endif
#ifndef SLES_Y_NBUF
#define SLES_Y_NBUF 0
#endif
  // FP32: 64-byte tile rows; WIDE (the LES passes) at N = 512: 128-byte rows
  // (at 512^3, with the 32-thread inverse line plan, the LES y passes took
  // 1.75 + 2.01 ms against 2.21 + 2.06; the passes without LES and all passes
  // at 256^3 were slower with the wider rows); FP64: 64-byte rows
  static constexpr int W =
      WSET > 0 ? WSET : ((sizeof(Tp) == 4) ? (SLES_Y_W > 0 ? SLES_Y_W : ((N == 512 && WIDE) ? 16 : 8)) : 4);
  static constexpr int EPC = sizeof(C) / 8;                 // 8-byte tensor elements per complex
  static constexpr int T = F::T, V = F::V;
  static constexpr int THREADS = W * T;
  static constexpr int RB = N < 256 ? N : 256;              // rows per TMA box
  static constexpr int NBOX = N / RB;
  static constexpr int TE = N * W;                          // complex elements per tile
  static constexpr int NBUF =
      // 16 KB tiles: 4 buffers; larger tiles: 2 (at 512^3 a third 32 KB buffer made the y passes slower)
      NBUF_SET > 0 ? NBUF_SET : (SLES_Y_NBUF > 0 ? SLES_Y_NBUF : ((TE * sizeof(C) <= 16384) ? 4 : 2));
  static constexpr unsigned BOX_BYTES = RB * W * sizeof(C);
  static constexpr int SCR = F::XLEN * W;
  using Ring = TileRing<C, NBUF, TE>;
  static constexpr size_t RING_BYTES = RING ? Ring::bytes() : 0;
  static constexpr size_t SMEM = RING_BYTES + ((size_t)SCR + F::TAB) * sizeof(C);  // + twiddle tables
#ifndef SLES_T_MINB256
#define SLES_T_MINB256 2
#endif
  static constexpr int MINB = (sizeof(Tp) == 4) ? (THREADS >= 512 ? 1 : (THREADS >= 256 ? SLES_T_MINB256 : 4)) : 1;
};

// x-pass geometry: the projected components kept in a shared stash
// [D][N][W] between the forward and the per-component phase.  Variants XV
// (picked at run time, by default or by the autotuner):
//   0: W = 64-byte tile rows, direct loads, 16 warps per SM (FP32)
//   1: W = 64-byte rows, the item's tiles [N][W] prefetched one ahead into a
//      ring of 2 buffers with per-thread cp.async, 8 warps per SM
//   2: W = 32-byte rows, the same ring, 12 warps per SM
// A ring that does not fit the variant's shared-memory budget falls back to
// direct loads (NB = 0).  Variant 3 (sles_xtma.cuh) streams every tile through
// a TMA ring and keeps the projected components in registers.
constexpr int X_VARIANTS = 4;
template <typename Tp, int N, class F, int DIM, int XV>
struct XGeo {
  using C = typename CT<Tp>::C;
  static constexpr bool F32 = sizeof(Tp) == 4;
#ifndef SLES_X_W2
#define SLES_X_W2 4
#endif
#ifndef SLES_X_W0
#define SLES_X_W0 8
#endif
  static constexpr int W = (XV == 2) ? (F32 ? SLES_X_W2 : 2) : (F32 ? (XV == 0 ? SLES_X_W0 : 8) : 4);
  static constexpr int T = F::T, V = F::V;
  static constexpr int THREADS = W * T;
  static constexpr int TE = N * W;
  static constexpr int SCR = F::XLEN * W;
  static constexpr int WARPS = (THREADS + 31) / 32;
#ifndef SLES_X_T2
#define SLES_X_T2 12
#endif
#ifndef SLES_X_T0
#define SLES_X_T0 16
#endif
  static constexpr int TARGET = F32 ? (XV == 0 ? SLES_X_T0 : (XV == 1 ? 8 : SLES_X_T2)) : (XV == 2 ? 8 : WARPS);
  static constexpr int MINB0 = TARGET / WARPS;
  static constexpr int MINB = MINB0 < 1 ? 1 : (MINB0 > 16 ? 16 : MINB0);
  static constexpr size_t BASE = ((size_t)DIM * TE + SCR + F::LIN_LEN) * sizeof(C);  // + linear twiddle table
  // shared memory per block that keeps MINB blocks resident (228 KB per SM, 1 KB reserved per block)
  static constexpr size_t BUDGET = (228 / MINB - 1) * 1024;
#ifndef SLES_X_NB
#define SLES_X_NB 2
#endif
  static constexpr int NB =
      (XV == 0) ? 0 : ((BASE + (size_t)SLES_X_NB * TE * sizeof(C) <= BUDGET) ? SLES_X_NB : 0);
  // XV 0: the stage's state tiles (ucur, u0) of one component prefetched with
  // per-thread cp.async into two spare [N][W] buffers, while the item's
  // forward transforms (component 0) or the previous component's inverse
  // transforms run, where they fit the budget
#ifndef SLES_X_SB
#define SLES_X_SB 1
#endif
  static constexpr int SB = (SLES_X_SB && XV == 0 && BASE + (size_t)2 * TE * sizeof(C) <= BUDGET) ? 2 : 0;
  static constexpr size_t SMEM = BASE + (size_t)(NB + SB) * TE * sizeof(C);
};

// slot of tile `i` in a pass's per-item load sequence
template <int KIND>
__device__ __forceinline__ int seq_slot(int i) {
  // 0: y-inverse LES, 1: y-inverse plain, 2: y-forward LES, 3: y-forward plain / x plain 3D,
  // 4: x LES 3D, 5: identity (x 2D, inverse-only sources)
  if (KIND == 0) { const int s[6] = {0, 3, 1, 4, 2, 5}; return s[i]; }
  if (KIND == 1) { const int s[5] = {2, 0, 4, 1, 3}; return s[i]; }
  if (KIND == 2) { const int s[9] = {4, 5, 0, 3, 6, 7, 1, 8, 2}; return s[i]; }
  if (KIND == 4) { const int s[6] = {0, 3, 1, 4, 2, 5}; return s[i]; }
  // 6: adjoint y-inverse (two groups of 6 inputs at slot bases 0 and 9),
  // 7: adjoint y-forward (Z_j, A2_j, A1_j per component)
  if (KIND == 6) { const int s[6] = {0, 3, 1, 4, 2, 5}; return (i / 6) * 9 + s[i % 6]; }
  if (KIND == 7) { const int s[9] = {0, 6, 3, 1, 7, 4, 2, 8, 5}; return s[i]; }
  return i;
}

// ---------------------------------------------------------------------------
// X pass.  Work item = (ky slice [3D], column chunk of W last-axis wavenumbers);
// lines along x.  PAR2D selects the reference's 2D stress (1) or the corrected one.
// ---------------------------------------------------------------------------
template <typename Tp, int N, class F, int DIM, int LES, int PAR2D, int ETD, int XV>
__global__ void __launch_bounds__(XGeo<Tp, N, F, DIM, XV>::THREADS, XGeo<Tp, N, F, DIM, XV>::MINB)
k_xpass(const __grid_constant__ XArgs<Tp> A) {
  using K = XGeo<Tp, N, F, DIM, XV>;
  using C = typename CT<Tp>::C;
  constexpr int T = K::T, V = K::V, D = DIM, W = K::W, NB = K::NB;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  C* rst = reinterpret_cast<C*>(smem_raw);  // [D][N][W] projected components
  C* sm0 = rst + D * K::TE;                 // exchange scratch
  C* twt = sm0 + K::SCR;                    // twiddle table exp(-2 pi i e/N)
  C* ring = twt + F::LIN_LEN;               // NB tile buffers [N][W] (XV 0: SB state buffers)
  const StageCoef<Tp> SC = stage_coef<Tp>(A);
  const int tid = threadIdx.x;
  const int l = tid % W, j = tid / W;
  F::fill_table_lin(twt);
  __syncthreads();
  F fft;
  const int nsl = (DIM == 3) ? A.nsl : 1;
  const long long items = (long long)A.nmem * nsl * A.nchunks;
  const long long ps = (DIM == 3) ? (long long)nsl * A.nkp : (long long)A.nkp;  // x stride
  const long long fs = A.fs;
  C* sm = sm0 + l;
  C* ws = A.ws;
  auto kx_at = [&](int m) { return kc2c(j + T * m, N); };
  auto rpos = [&](int c, int m) { return c * K::TE + (j + T * m) * W + l; };
  // the item's tile sequence: forward tiles (slots), then per component the
  // state tiles the stage reads (ucur, u0, u1); inverse-only items: uinv
  constexpr int NTF = LES ? (DIM == 3 ? 6 : (PAR2D ? 4 : 5)) : D;
  const int nst = A.need_uc + A.need_u0 + A.need_u1;
  const int TPI = A.fwd ? NTF + D * nst : D;
  auto tile_src = [&](int k) -> const C* {
    if (!A.fwd) return A.uinv + k * fs;
    if (k < NTF) return ws + (LES && DIM == 3 ? seq_slot<4>(k) : k) * fs;
    k -= NTF;
    const int c = k / nst, r = k % nst;
    int q = 0;
    if (A.need_uc) { if (r == q) return A.ucur + c * fs; ++q; }
    if (A.need_u0) { if (r == q) return A.u0 + c * fs; ++q; }
    return A.u1 + c * fs;
  };
  long long tq = 0;  // next tile to consume
  auto issue = [&](long long t) {  // prefetch tile t of this block's sequence (every thread its own positions)
    if constexpr (NB > 0) {
      const long long it2 = blockIdx.x + (t / TPI) * (long long)gridDim.x;
      if (it2 < items) {
        const int col2 = (int)(it2 % A.nchunks) * W + l;
        const bool ok2 = col2 < A.nk;
        const long long r2 = it2 / A.nchunks;  // member * nsl + slice
        const C* src = tile_src((int)(t % TPI)) + (r2 / nsl) * A.mstride + (r2 % nsl) * A.nkp + (ok2 ? col2 : 0);
        C* dst = ring + (int)(t % NB) * K::TE + j * W + l;
#pragma unroll
        for (int m = 0; m < V; ++m) cp_async_el<sizeof(C)>(dst + T * m * W, src + (j + T * m) * ps, ok2);
      }
      cp_async_commit();
    }
  };
  if constexpr (NB > 0) {
    for (int t = 0; t < NB - 1; ++t) issue(t);
  }
  for (long long it = blockIdx.x; it < items; it += gridDim.x) {  // persistent over work items
    const int chunk = (int)(it % A.nchunks);
    const long long rest = it / A.nchunks;
    const int sl = (int)(rest % nsl);      // ky slice (3D); 0 in 2D
    const int mem = (int)(rest / nsl);     // ensemble member
    const int col = chunk * W + l;
    const bool ok = col < A.nk;
    const long long mbase = (long long)mem * A.mstride;
    const long long base = mbase + (long long)sl * A.nkp + col;
    const double nud = A.mnu ? A.mnu[mem] : A.nu_d;
    // next tile of the sequence (its source is implied by the sequence position)
    auto take = [&](C (&v)[V], const C* src, int slot) {
      if constexpr (NB > 0) {
        issue(tq + NB - 1);
        cp_async_wait<NB - 1>();
        const C* tl = ring + (int)(tq % NB) * K::TE + j * W + l;
#pragma unroll
        for (int m = 0; m < V; ++m) v[m] = tl[T * m * W];
        ++tq;
      } else {
#pragma unroll
        for (int m = 0; m < V; ++m) v[m] = ok ? src[slot * fs + base + (j + T * m) * ps] : cmk<C>(0, 0);
      }
    };
    auto ld = take;
    auto st = [&](int slot, const C (&v)[V]) {
      if (ok) {
#pragma unroll
        for (int m = 0; m < V; ++m) ws[slot * fs + base + (j + T * m) * ps] = v[m];
      }
    };
    // inverse x-transforms of component c of the new state: primes the next evaluation
    auto prep = [&](int c, C (&s)[V]) {
      if (LES) {
        C b[V];
#pragma unroll
        for (int m = 0; m < V; ++m) b[m] = cmuli_s(s[m], (Tp)kx_at(m));  // i kx u_c
        fft.template run_tab<+1, true>(b, j, sm, W, twt);
        st(D + c, b);
      } else if ((DIM == 3 && c >= 1) || (DIM == 2 && c == 1)) {
        C q[V];
        const Tp sg = (DIM == 3 && c == 2) ? (Tp)-1 : (Tp)1;  // 3D: -i kx w -> [3], i kx v -> [4]; 2D: i kx v -> [2]
#pragma unroll
        for (int m = 0; m < V; ++m) q[m] = cmuli_s(s[m], sg * (Tp)kx_at(m));
        fft.template run_tab<+1, true>(q, j, sm, W, twt);
        st(DIM == 3 ? (c == 2 ? 3 : 4) : 2, q);
      }
      fft.template run_tab<+1, true>(s, j, sm, W, twt);
      st(c, s);
    };
    if (!A.fwd) {
#pragma unroll 1
      for (int c = 0; c < D; ++c) {
        C v[V];
        ld(v, A.uinv, c);
        prep(c, v);
      }
      continue;
    }
    // XV 0: prefetch component c's state tiles into the two spare buffers (each
    // thread copies exactly the positions it later reads: no block barrier)
    auto sissue = [&](int c) {
      if constexpr (K::SB > 0) {
        const long long so = c * fs + mbase + (long long)sl * A.nkp + (ok ? col : 0);
        C* d0 = ring + j * W + l;
#pragma unroll
        for (int m = 0; m < V; ++m) {
          if (A.need_uc) cp_async_el<sizeof(C)>(d0 + T * m * W, A.ucur + so + (j + T * m) * ps, ok);
          if (A.need_u0) cp_async_el<sizeof(C)>(d0 + K::TE + T * m * W, A.u0 + so + (j + T * m) * ps, ok);
        }
        cp_async_commit();
      }
    };
    sissue(0);
    // forward x-transforms; the x part of div(tau) joins in spectral space
#pragma unroll 1
    for (int c = 0; c < D; ++c) {
      C v[V];
      ld(v, ws, c);
      fft.template run_tab<-1, true>(v, j, sm, W, twt);
      if (LES && DIM == 3) {  // + 2i kx F_cx
        C h[V];
        ld(h, ws, 3 + c);
        fft.template run_tab<-1, true>(h, j, sm, W, twt);
#pragma unroll
        for (int m = 0; m < V; ++m) v[m] = cadd(v[m], cmuli_s(h[m], (Tp)(2 * kx_at(m))));
      }
#pragma unroll
      for (int m = 0; m < V; ++m) rst[rpos(c, m)] = v[m];
    }
    if (LES && DIM == 2) {
      // reference (math_formula.py:128-146): T_0 = 2i(kx F12 + ky F22), T_1 = 0
      // corrected: T_0 = 2i(kx F11 + ky F12), T_1 = 2i(kx F12 + ky F22)
      const Tp ky2 = (Tp)(2 * col);
      C h[V];
      ld(h, ws, 2);
      fft.template run_tab<-1, true>(h, j, sm, W, twt);
#pragma unroll
      for (int m = 0; m < V; ++m) rst[rpos(0, m)] = cadd(rst[rpos(0, m)], cmuli_s(h[m], (Tp)(2 * kx_at(m))));
      ld(h, ws, 3);
      fft.template run_tab<-1, true>(h, j, sm, W, twt);
#pragma unroll
      for (int m = 0; m < V; ++m) {
        rst[rpos(0, m)] = cadd(rst[rpos(0, m)], cmuli_s(h[m], ky2));
        if (!PAR2D) rst[rpos(1, m)] = cadd(rst[rpos(1, m)], cmuli_s(h[m], (Tp)(2 * kx_at(m))));
      }
      if (!PAR2D) {
        ld(h, ws, 4);
        fft.template run_tab<-1, true>(h, j, sm, W, twt);
#pragma unroll
        for (int m = 0; m < V; ++m) rst[rpos(1, m)] = cadd(rst[rpos(1, m)], cmuli_s(h[m], ky2));
      }
    }
    // mask + projection (each thread revisits only its own stash positions)
#pragma unroll
    for (int m = 0; m < V; ++m) {
      C s[D];
      int kv[D];
#pragma unroll
      for (int c = 0; c < D; ++c) s[c] = rst[rpos(c, m)];
      kv[0] = kx_at(m);
      if (DIM == 3) { kv[1] = kc2c(A.ky0 + sl, N); kv[D - 1] = col; }
      else kv[1] = col;
      project<Tp, D>(A, s, kv);
#pragma unroll
      for (int c = 0; c < D; ++c) rst[rpos(c, m)] = s[c];
    }
    // per component: state update, then the inverse transforms of the new state
    const int kyv = (DIM == 3) ? kc2c(A.ky0 + sl, N) : 0;
#pragma unroll 1
    for (int c = 0; c < D; ++c) {
      C v[V];
      C ucv[NB > 0 || K::SB > 0 ? V : 1], u0v[NB > 0 || K::SB > 0 ? V : 1], u1v[NB > 0 ? V : 1];
      if constexpr (NB > 0) {
        if (A.need_uc) take(ucv, A.ucur, c);
        if (A.need_u0) take(u0v, A.u0, c);
        if (A.need_u1) take(u1v, A.u1, c);
      } else if constexpr (K::SB > 0) {
        cp_async_wait<0>();
        const C* s0 = ring + j * W + l;
#pragma unroll
        for (int m = 0; m < V; ++m) {
          ucv[m] = s0[T * m * W];
          u0v[m] = s0[K::TE + T * m * W];
        }
      }
      if (ok) {
#pragma unroll
        for (int m = 0; m < V; ++m) {
          const long long off = base + (j + T * m) * ps;
          const int kx = kx_at(m);
          const int k2 = kx * kx + kyv * kyv + col * col;
          C ucm, u0m, u1m;
          if constexpr (NB > 0) {
            ucm = A.need_uc ? ucv[m] : cmk<C>(0, 0);
            u0m = A.need_u0 ? u0v[m] : ucm;
            u1m = A.need_u1 ? u1v[m] : cmk<C>(0, 0);
          } else if constexpr (K::SB > 0) {
            ucm = A.need_uc ? ucv[m] : cmk<C>(0, 0);
            u0m = A.need_u0 ? u0v[m] : ucm;
            u1m = A.need_u1 ? A.u1[c * fs + off] : cmk<C>(0, 0);
          } else {
            ucm = A.need_uc ? A.ucur[c * fs + off] : cmk<C>(0, 0);
            u0m = A.need_u0 ? A.u0[c * fs + off] : ucm;
            u1m = A.need_u1 ? A.u1[c * fs + off] : cmk<C>(0, 0);
          }
          v[m] = update_component<Tp, ETD>(A, SC, c, rst[rpos(c, m)], ucm, u0m, u1m, k2, off, nud);
        }
      } else {
#pragma unroll
        for (int m = 0; m < V; ++m) v[m] = cmk<C>(0, 0);
      }
      if (c + 1 < D) sissue(c + 1);  // lands while this component's inverse transforms run
      if (A.prep) prep(c, v);
    }
  }
}

// ---------------------------------------------------------------------------
// Y passes (3D): work item = (x, kz chunk); lines along y (stride nkp)
// ---------------------------------------------------------------------------
template <typename Tp>
struct YArgs {
  using C = typename CT<Tp>::C;
  CUtensorMap tm;        // workspace slots as y-pass tiles (split loads: the 5D exchange-buffer map)
  unsigned* err;
  C* ws;
  C* out;                // where the pass stores (the workspace, or the slab exchange buffer)
  long long fs;
  int nkp, nk, nchunks;
  int nx;                // x planes held (N, or N/P on a slab)
  int split;             // slab exchange: 0 none; inverse pass: lines arrive split in P blocks of m rows
                         // (5D map); forward pass: outputs stored as [slot][P][nx][m][nkp] blocks
  int m;                 // rows per block (N/P)
};

// INV = 1: inverse (y1), 0: forward (y2).  ADJ = 1: the adjoint's passes
// (discrete adjoint of the RHS, see sles_adjoint.cuh): the inverse carries two
// groups (the recomputed state and the cotangent), the forward contracts
// Z_j - i ky A2_j.
// SPLIT = 1: the slab exchange layouts (A.split; see YArgs), compiled apart so
// the whole-grid kernels carry none of its addressing
template <typename Tp, int N, class F, int LES, int INV, int ADJ = 0, int SPLIT = 0, int YW = 0>
__global__ void __launch_bounds__(TGeo<Tp, N, F, true, 0, LES, YW>::THREADS, TGeo<Tp, N, F, true, 0, LES, YW>::MINB)
k_ypass(const __grid_constant__ YArgs<Tp> A) {
  using K = TGeo<Tp, N, F, true, 0, LES, YW>;
  using C = typename CT<Tp>::C;
  constexpr int T = K::T, V = K::V, W = K::W;
  constexpr int KIND = ADJ ? (INV ? 6 : 7) : (INV ? (LES ? 0 : 1) : (LES ? 2 : 3));
  constexpr int NT = ADJ ? (INV ? 12 : 9) : (INV ? (LES ? 6 : 5) : (LES ? 9 : 3));
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  typename K::Ring ring;
  const int tid = threadIdx.x;
  ring.init(smem_raw, tid);
  C* sm0 = reinterpret_cast<C*>(smem_raw + K::Ring::bytes());
  C* twt = sm0 + K::SCR;  // twiddle table exp(-2 pi i e/N)
  const int l = tid % W, j = tid / W;
  F fft;
  F::fill_table(twt);
  __syncthreads();
  const long long items = (long long)A.nx * A.nchunks;
  const long long mine = (blockIdx.x < items) ? (items - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  const long long ntiles = mine * NT;
  auto issue = [&](long long t) {
    const long long it = blockIdx.x + (t / NT) * (long long)gridDim.x;
    const int chunk = (int)(it % A.nchunks), x = (int)(it / A.nchunks);
    if (INV && SPLIT)
      ring.issue_split(t, &A.tm, chunk * W * K::EPC, x, seq_slot<KIND>((int)(t % NT)), K::NBOX * K::BOX_BYTES);
    else
      ring.issue(t, &A.tm, chunk * W * K::EPC, x, seq_slot<KIND>((int)(t % NT)), K::NBOX, K::RB, K::BOX_BYTES);
  };
  if (tid == 0) {
    tma_prefetch_desc(&A.tm);
    for (long long t = 0; t < K::NBUF && t < ntiles; ++t) issue(t);
  }
  long long t = 0;
  auto take = [&](C (&v)[V]) {
    ring.wait(t, A.err);
    const C* tl = ring.tile(t);
#pragma unroll
    for (int m = 0; m < V; ++m) v[m] = tl[(j + T * m) * W + l];
    __syncthreads();
    if (tid == 0 && t + K::NBUF < ntiles) issue(t + K::NBUF);
    ++t;
  };
  const long long ps = A.nkp, fs = A.fs;
  C* sm = sm0 + l;
  C* ws = A.ws;
  auto kyv = [&](int m) { return (Tp)kc2c(j + T * m, N); };
  for (long long k = 0; k < mine; ++k) {  // persistent over work items
    const long long it = blockIdx.x + k * (long long)gridDim.x;
    const int chunk = (int)(it % A.nchunks);
    const int x = (int)(it / A.nchunks);
    const int col = chunk * W + l;
    const bool ok = col < A.nk;
    const long long base = (long long)x * N * A.nkp + col;
    auto st = [&](int slot, const C (&v)[V]) {
      if (!ok) return;
      if (!INV && SPLIT) {  // row y = b*m + r goes to block b: [slot][b][x][r][kz]
        const long long bs = (long long)A.nx * A.m * A.nkp;
#pragma unroll
        for (int m = 0; m < V; ++m) {
          const int y = j + T * m, b = y / A.m, r = y - b * A.m;
          A.out[slot * fs + b * bs + ((long long)x * A.m + r) * A.nkp + col] = v[m];
        }
      } else {
#pragma unroll
        for (int m = 0; m < V; ++m) ws[slot * fs + base + (j + T * m) * ps] = v[m];
      }
    };
    if (ADJ && !INV) {
      C v[V], w[V];
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {  // Y_c = Y(Z_c) - i ky Y(A2_c);  A1_c passes through
        take(v);
        fft.template run_tab<-1, false, 0, false>(v, j, sm, W, twt);
        take(w);
        fft.template run_tab<-1, false, 0, false>(w, j, sm, W, twt);
#pragma unroll
        for (int m = 0; m < V; ++m) v[m] = cadd(v[m], cmuli_s(w[m], -kyv(m)));
        st(c, v);
        take(v);
        fft.template run_tab<-1, false, 0, false>(v, j, sm, W, twt);
        st(3 + c, v);
      }
      continue;
    }
    if (INV) {
      C v[V], w[V];
      if (LES) {
#pragma unroll 1
        for (int g = 0; g < (ADJ ? 2 : 1); ++g) {
          const int sb = 9 * g;
#pragma unroll 1
          for (int c = 0; c < 3; ++c) {  // a_c, dy_c = Y^-1(i ky A_c), dx_c = Y^-1(B_c)
            take(v);
#pragma unroll
            for (int m = 0; m < V; ++m) w[m] = cmuli_s(v[m], kyv(m));
            fft.template run_tab<+1, false, 0, false>(v, j, sm, W, twt);
            st(sb + c, v);
            fft.template run_tab<+1>(w, j, sm, W, twt);
            st(sb + 6 + c, w);
            take(v);
            fft.template run_tab<+1, false, 0, false>(v, j, sm, W, twt);
            st(sb + 3 + c, v);
          }
        }
      } else {
        take(v);  // A_w -> a_w and Ox = Y^-1(i ky A_w)
#pragma unroll
        for (int m = 0; m < V; ++m) w[m] = cmuli_s(v[m], kyv(m));
        fft.template run_tab<+1, false, 0, false>(v, j, sm, W, twt);
        st(2, v);
        fft.template run_tab<+1>(w, j, sm, W, twt);
        st(5, w);
        take(v);  // A_u -> a_u and Oz = Y^-1(Q_z - i ky A_u)
        take(w);
#pragma unroll
        for (int m = 0; m < V; ++m) w[m] = csub(w[m], cmuli_s(v[m], kyv(m)));
        fft.template run_tab<+1, false, 0, false>(v, j, sm, W, twt);
        st(0, v);
        fft.template run_tab<+1>(w, j, sm, W, twt);
        st(4, w);
        take(v);
        fft.template run_tab<+1, false, 0, false>(v, j, sm, W, twt);
        st(1, v);
        take(v);
        fft.template run_tab<+1, false, 0, false>(v, j, sm, W, twt);
        st(3, v);
      }
      continue;
    }
    if (!LES) {
      C v[V];
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        take(v);
        fft.template run_tab<-1, false, 0, false>(v, j, sm, W, twt);
        st(c, v);
      }
      continue;
    }
    const Tp kz2 = (Tp)(2 * col);
    C tt[V], acc[V], acc2[V];
    // G_x = N_x + 2i(ky F_xy + kz F_xz);  H_y = F_xy, H_z = F_xz, H_x = F_xx
    take(tt);
    fft.template run_tab<-1, false, 0, false>(tt, j, sm, W, twt);
    st(4, tt);
#pragma unroll
    for (int m = 0; m < V; ++m) acc[m] = cmuli_s(tt[m], (Tp)2 * kyv(m));
    take(tt);
    fft.template run_tab<-1, false, 0, false>(tt, j, sm, W, twt);
    st(5, tt);
#pragma unroll
    for (int m = 0; m < V; ++m) acc[m] = cadd(acc[m], cmuli_s(tt[m], kz2));
    take(tt);
    fft.template run_tab<-1, false, 0, false>(tt, j, sm, W, twt);
#pragma unroll
    for (int m = 0; m < V; ++m) tt[m] = cadd(tt[m], acc[m]);
    st(0, tt);
    take(tt);
    fft.template run_tab<-1, false, 0, false>(tt, j, sm, W, twt);
    st(3, tt);
    // G_y = N_y + 2i(ky F_yy + kz F_yz);  G_z = N_z + 2i(ky F_yz + kz F_zz)
    take(tt);
    fft.template run_tab<-1, false, 0, false>(tt, j, sm, W, twt);
#pragma unroll
    for (int m = 0; m < V; ++m) acc[m] = cmuli_s(tt[m], (Tp)2 * kyv(m));
    take(tt);
    fft.template run_tab<-1, false, 0, false>(tt, j, sm, W, twt);
#pragma unroll
    for (int m = 0; m < V; ++m) {
      acc[m] = cadd(acc[m], cmuli_s(tt[m], kz2));
      acc2[m] = cmuli_s(tt[m], (Tp)2 * kyv(m));
    }
    take(tt);
    fft.template run_tab<-1, false, 0, false>(tt, j, sm, W, twt);
#pragma unroll
    for (int m = 0; m < V; ++m) tt[m] = cadd(tt[m], acc[m]);
    st(1, tt);
    take(tt);
    fft.template run_tab<-1, false, 0, false>(tt, j, sm, W, twt);
#pragma unroll
    for (int m = 0; m < V; ++m) acc2[m] = cadd(acc2[m], cmuli_s(tt[m], kz2));
    take(tt);
    fft.template run_tab<-1, false, 0, false>(tt, j, sm, W, twt);
#pragma unroll
    for (int m = 0; m < V; ++m) tt[m] = cadd(tt[m], acc2[m]);
    st(2, tt);
  }
}

// ---------------------------------------------------------------------------
// Z pass (the r2c axis: z in 3D, y in 2D).  Per line: c2r of NG physical
// fields, pointwise products, r2c of NOUT products.  Threads: NG field groups
// x LPI lines x T threads per line.
// ---------------------------------------------------------------------------
template <typename Tp>
struct ZArgs {
  using C = typename CT<Tp>::C;
  C* ws;
  long long fs;
  int nkp;
  long long nlines;      // N^(DIM-1)
  Tp scale;              // 1/N^DIM
  Tp cdx2;               // (Cs dx)^2 (Smagorinsky) or 2.5 Cs^2 dx^2 (Vreman)
  const Tp* uphys;       // optional stored velocity (DIM real fields)
  const Tp* cphys;       // optional stored curl (3 real fields in 3D, 1 in 2D)
  long long rs;          // elements per real field
  int stress_only;       // 1: drop u x omega (evaluates the LES stress alone)
  unsigned* err;         // error word (bounded-wait timeouts)
  unsigned long long* umax;  // non-null: max over components and points of u (ordered encoding)
  const double* mcs;     // batched members: per-member C_s (device) or null: cdx2 for all
  long long lpm;         // lines per member
  double dx;             // grid spacing (with mcs: cdx2 = (Cs dx)^2, Vreman 2.5 Cs^2 dx^2)
  int vreman;
};

// order-preserving encoding of a double as an unsigned 64-bit integer (for atomicMax)
__device__ __forceinline__ unsigned long long ord_encode(double x) {
  const unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double ord_decode(unsigned long long e) {
  const unsigned long long u = (e >> 63) ? (e & 0x7fffffffffffffffull) : ~e;
  return __longlong_as_double((long long)u);
}

// One step of the driver loop's time-step logic (src/SM_solver.py:18-83,
// compute_dt :258-277) on the device; see sles_dtctl in include/sles.h.
static __global__ void k_dtctl(sles_dtctl* c, int parity) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const double umax = c->umax_bits[parity] ? ord_decode(c->umax_bits[parity]) : -INFINITY;
  c->umax_bits[parity ^ 1] = 0ull;  // the next step collects from scratch
  c->dt_step = 0.0;
  if (c->paused) return;
  const double cfl = (c->nsteps == 0) ? c->cfl_first : c->cfl;
  const double dt1 = cfl * c->dx / umax;
  const double dt2 = (c->nu > 0.0) ? 0.1 * c->dx * c->dx / c->nu : 1e6;
  const double dt = fmin(dt1, dt2);
  if (!(dt == dt)) { c->flags |= SLES_DT_NAN; c->paused = 1; return; }
  if (dt < 1e-6) { c->flags |= SLES_DT_TOO_SMALL; c->paused = 1; return; }
  c->dt = dt;
  if (c->nsteps == 0 && !c->t_init) { c->t = dt; c->t_init = 1; }
  if (c->t >= c->ek_next && !c->resumed) { c->flags |= SLES_DT_SNAPSHOT; c->paused = 1; return; }
  c->resumed = 0;
  if (c->t >= c->t_end || dt < 1e-8) { c->flags |= SLES_DT_DONE; c->paused = 1; return; }
  c->t += dt;
  c->dt_step = dt;
  c->nsteps += 1;
}

#ifndef SLES_Z_PADD
#define SLES_Z_PADD 0
#endif
template <typename Tp, int N, int DIM, int LES, int PAR2D, int LPI>
struct ZGeo {
  // the half-length plan, mirrored where it qualifies (the r2c post step
  // then pairs bins in registers)
  using F = typename MirrorIf<typename WithPad<typename PlanFor<Tp, N / 2>::F, SLES_Z_PADD>::F>::type;
  using C = typename CT<Tp>::C;
  static constexpr int L = N / 2, T = F::T, V = F::V;
  static constexpr int NG = (DIM == 3) ? (LES ? 12 : 6) : (LES ? 6 : 3);    // physical fields
  static constexpr int NIN = (DIM == 3) ? (LES ? 9 : 6) : (LES ? 4 : 3);    // input slots
  static constexpr int NOUT = (DIM == 3) ? (LES ? 9 : 3) : (LES ? (PAR2D ? 4 : 5) : 2);
  static constexpr int NKP = ((N / 2 + 1) + 3) / 4 * 4;
  static constexpr int THREADS = NG * LPI * T;
  // float32: 3 blocks per SM for one line per item (a 512 line's 192 threads
  // included), 2 for several lines up to 256 threads (their registers as one
  // line's), else 1
  static constexpr int MINB =
      (sizeof(Tp) == 4) ? ((THREADS <= 192 && LPI == 1) || THREADS <= 96 ? 3 : (THREADS <= 256 ? 2 : 1)) : 1;
  // per (field, line) region: the line's FFT exchange scratch (LS complex,
  // LS = 8 mod 16 keeps the autosort writes conflict-free) and, between the
  // transforms, the physical line itself (N reals)
  static constexpr int LS = ((F::XLEN + 15) / 16) * 16 + 8;
  static constexpr int RS = 2 * LS;
  static_assert(RS >= N, "region must hold a physical line");
  static_assert((size_t)NG * LPI * RS * sizeof(Tp) >= (size_t)THREADS * sizeof(double), "regions hold the u_max partials");
  // staging: NIN slot blocks of LPI lines; consecutive blocks start half the
  // bank space (64 bytes mod 128) apart, so the two line groups of a half warp
  // reading neighbouring slots hit disjoint banks
  static constexpr int SLOTS = LPI * NKP;
  static constexpr int SLOT_STRIDE =
      SLOTS + (int)(((64 - (long long)SLOTS * (long long)sizeof(C)) % 128 + 128) % 128 / (long long)sizeof(C));
  static_assert((SLOT_STRIDE * sizeof(C)) % 16 == 0, "bulk copies need 16-byte aligned slot blocks");
  static constexpr int STAGE = NIN * SLOT_STRIDE;  // complex elements per staging buffer
  static constexpr size_t OFF_TW = 16;
  static constexpr size_t OFF_STAGE = OFF_TW + (size_t)L * sizeof(C);
  static constexpr size_t OFF_REG = OFF_STAGE + 2 * (size_t)STAGE * sizeof(C);
  static constexpr size_t SMEM = OFF_REG + (size_t)NG * LPI * RS * sizeof(Tp);
};

template <typename Tp, int MODEL>
__device__ __forceinline__ Tp eddy_viscosity_3d(Tp a11, Tp a12, Tp a13, Tp a21, Tp a22, Tp a23, Tp a31, Tp a32,
                                                Tp a33, Tp cdx2) {
  if (MODEL == M_SMAG) {  // smagorinsky.py:31-39
    const Tp ss = a11 * a11 + ((Tp)0.5 * ((a12 + a21) * (a12 + a21))) + a22 * a22 +
                  ((Tp)0.5 * ((a13 + a31) * (a13 + a31))) + ((Tp)0.5 * ((a23 + a32) * (a23 + a32))) + a33 * a33;
    return sqrt((Tp)2 * ss) * cdx2;
  }
  // vreman.py:32-123: B_beta from b_pq = sum_m a_mp a_mq, gate on alpha:alpha
  const Tp b11 = a11 * a11 + a21 * a21 + a31 * a31;
  const Tp b22 = a12 * a12 + a22 * a22 + a32 * a32;
  const Tp b33 = a13 * a13 + a23 * a23 + a33 * a33;
  const Tp b12 = a11 * a12 + a21 * a22 + a31 * a32;
  const Tp b13 = a11 * a13 + a21 * a23 + a31 * a33;
  const Tp b23 = a12 * a13 + a22 * a23 + a32 * a33;
  const Tp B = (b11 * b22) - (b12 * b12) + (b11 * b33) - (b13 * b13) + (b22 * b33) - (b23 * b23);
  const Tp sb = sqrt(B);  // NaN for a round-off negative B, as in the reference
  const Tp aa = a11 * a11 + a12 * a12 + a13 * a13 + a21 * a21 + a22 * a22 + a23 * a23 + a31 * a31 + a32 * a32 +
                a33 * a33;
  const Tp gate = ((aa > (Tp)10e-5) && (sb > aa / (Tp)10e6)) ? sqrt((Tp)1 / aa) : (Tp)0;
  return sb * (gate * cdx2);
}

template <typename Tp, int MODEL>
__device__ __forceinline__ Tp eddy_viscosity_2d(Tp a11, Tp a12, Tp a21, Tp a22, Tp cdx2) {
  if (MODEL == M_SMAG) {  // smagorinsky.py:41-46
    const Tp ss = (a11 * a11) + ((Tp)0.5 * ((a12 + a21) * (a12 + a21))) + (a22 * a22);
    return sqrt((Tp)2 * ss) * cdx2;
  }
  // vreman.py:125-147
  const Tp b11 = a11 * a11 + a21 * a21, b22 = a12 * a12 + a22 * a22, b12 = a11 * a12 + a21 * a22;
  const Tp sb = sqrt((b11 * b22) - (b12 * b12));
  const Tp aa = a11 * a11 + a12 * a12 + a21 * a21 + a22 * a22;
  const Tp gate = ((aa > (Tp)10e-5) && (sb > aa / (Tp)10e6)) ? sqrt((Tp)1 / aa) : (Tp)0;
  return sb * (gate * cdx2);
}

// Pointwise products on the stash (field stride ps, point p).  uo/co: the
// stored physical velocity / curl at this point, or null.
template <typename Tp, int DIM, int LES, int MODEL, int PAR2D>
__device__ __forceinline__ void z_pointwise(Tp* st, int ps, int p, const Tp* uo, const Tp* co, Tp cdx2) {
  auto S = [&](int f) -> Tp& { return st[f * ps + p]; };
  if (DIM == 3) {
    Tp u = S(0), v = S(1), w = S(2);
    Tp ox, oy, oz;
    Tp a11 = 0, a12 = 0, a13 = 0, a21 = 0, a22 = 0, a23 = 0, a31 = 0, a32 = 0, a33 = 0;
    if (LES) {  // a[i][j] = d u_j / d x_i (math_formula.py:27-62)
      a11 = S(3); a12 = S(4); a13 = S(5);
      a21 = S(6); a22 = S(7); a23 = S(8);
      a31 = S(9); a32 = S(10); a33 = S(11);
      ox = a23 - a32; oy = a31 - a13; oz = a12 - a21;
    } else {
      ox = S(3); oy = S(4); oz = S(5);
    }
    if (uo) { u = uo[0]; v = uo[1]; w = uo[2]; }
    if (co) { ox = co[0]; oy = co[1]; oz = co[2]; }
    S(0) = v * oz - w * oy;  // math_formula.py:9-11
    S(1) = w * ox - u * oz;
    S(2) = u * oy - v * ox;
    if (LES) {
      const Tp nu = eddy_viscosity_3d<Tp, MODEL>(a11, a12, a13, a21, a22, a23, a31, a32, a33, cdx2);
      S(3) = a11 * nu;  // math_formula.py:76-127
      S(4) = ((Tp)0.5 * (a12 + a21)) * nu;
      S(5) = ((Tp)0.5 * (a13 + a31)) * nu;
      S(6) = a22 * nu;
      S(7) = ((Tp)0.5 * (a23 + a32)) * nu;
      S(8) = a33 * nu;
    }
  } else {
    Tp u = S(0), v = S(1);
    Tp om;
    Tp a11 = 0, a12 = 0, a21 = 0, a22 = 0;
    if (LES) {
      a11 = S(2); a12 = S(3); a21 = S(4); a22 = S(5);
      om = a12 - a21;
    } else {
      om = S(2);
    }
    if (uo) { u = uo[0]; v = uo[1]; }
    if (co) om = co[0];
    S(0) = v * om;  // math_formula.py:7-8
    S(1) = -u * om;
    if (LES) {
      const Tp nu = eddy_viscosity_2d<Tp, MODEL>(a11, a12, a21, a22, cdx2);
      const Tp f12 = ((Tp)0.5 * (a12 + a21)) * nu, f22 = a22 * nu;
      if (PAR2D) { S(2) = f12; S(3) = f22; }
      else { S(2) = a11 * nu; S(3) = f12; S(4) = f22; }
    }
  }
}

template <typename Tp, int N, int DIM, int LES, int MODEL, int PAR2D, int LPI>
__global__ void __launch_bounds__(ZGeo<Tp, N, DIM, LES, PAR2D, LPI>::THREADS, ZGeo<Tp, N, DIM, LES, PAR2D, LPI>::MINB)
k_zpass(const ZArgs<Tp> A) {
  using K = ZGeo<Tp, N, DIM, LES, PAR2D, LPI>;
  using F = typename K::F;
  using C = typename CT<Tp>::C;
  constexpr int T = K::T, V = K::V, NKP = K::NKP, SFS = LPI * K::RS;
  constexpr int WS = (T <= 32 && 32 % T == 0) ? 1 : 0;  // a line's threads share one warp
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
  C* twN = reinterpret_cast<C*>(smem_raw + K::OFF_TW);
  C* stage = reinterpret_cast<C*>(smem_raw + K::OFF_STAGE);   // [2][NIN][LPI][NKP]
  Tp* reg = reinterpret_cast<Tp*>(smem_raw + K::OFF_REG);     // [NG][LPI][RS]
  const int tid = threadIdx.x;
  fill_twN<Tp, N>(twN);
  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  const int j = tid % T, ln = (tid / T) % LPI, grp = tid / (T * LPI);
  F fft;
  fft.init(j);
  const long long fs = A.fs;
  Tp* myreg = reg + (grp * LPI + ln) * K::RS;
  C* sm = reinterpret_cast<C*>(myreg);
  // physical field `grp` = slot s1 + sgn * i k * slot s2  (k: r2c-axis wavenumber)
  int s1 = grp, s2 = -1;
  Tp sgn = 0;
  if (DIM == 3) {
    if (LES) {
      if (grp >= 9) { s1 = -1; s2 = grp - 9; sgn = 1; }      // d/dz u_c = i kz a_c
    } else {
      if (grp == 3) { s1 = 5; s2 = 1; sgn = -1; }             // omega_x = Ox - i kz v
      else if (grp == 4) { s1 = 3; s2 = 0; sgn = 1; }         // omega_y = Oy + i kz u
      else if (grp == 5) { s1 = 4; }                          // omega_z = Oz
    }
  } else {
    if (LES) {
      if (grp == 4) { s1 = -1; s2 = 0; sgn = 1; }             // a21 = du/dy
      else if (grp == 5) { s1 = -1; s2 = 1; sgn = 1; }        // a22 = dv/dy
    } else if (grp == 2) {
      s1 = 2; s2 = 0; sgn = -1;                               // omega = X^-1(i kx v) - i ky u
    }
  }
  // the same without branches that split a warp's groups: the first term is
  // (wr + i wk k) slot sa (wr, wk in {0, 1, sgn}); only the no-LES vorticity
  // groups add a second slot
  const int sa = (s1 >= 0) ? s1 : s2, s2b = (s1 >= 0) ? s2 : -1;
  const Tp wr = (s1 >= 0) ? (Tp)1 : (Tp)0, wk = (s1 >= 0) ? (Tp)0 : sgn;
  const long long nbi = (A.nlines + LPI - 1) / LPI;
  // thread 0 stages the NIN input slots of line group `b` into buffer `buf`
  auto issue = [&](long long b, int buf) {
    const long long l0 = b * LPI;
    const long long nl = (A.nlines - l0 < LPI) ? A.nlines - l0 : LPI;
    const unsigned bytes = (unsigned)(nl * A.nkp * (long long)sizeof(C));
    fence_proxy_async();
    mbar_arrive_expect_tx(&bar[buf], bytes * K::NIN);
    for (int s = 0; s < K::NIN; ++s)
      bulk_g2s(stage + buf * K::STAGE + s * K::SLOT_STRIDE, A.ws + s * fs + l0 * A.nkp, bytes, &bar[buf]);
  };
  if (tid == 0 && blockIdx.x < nbi) issue(blockIdx.x, 0);
  double lmax = -INFINITY;  // max of u over this thread's points (when A.umax)
  int iter = 0;
  for (long long bi = blockIdx.x; bi < nbi; bi += gridDim.x, ++iter) {  // persistent over line groups
    const int buf = iter & 1;
    if (tid == 0 && bi + gridDim.x < nbi) issue(bi + gridDim.x, buf ^ 1);
    mbar_wait_bounded(&bar[buf], (iter >> 1) & 1, A.err);
    const long long line0 = bi * LPI;
    const long long line = line0 + ln;
    const bool ok = line < A.nlines;
    const long long lo = (ok ? line : 0) * A.nkp;
    // ---- phase A: c2r of physical field `grp` from the staged slots
    {
      const C* sb = stage + buf * K::STAGE + ln * NKP;
      C v[V];
      c2r_pre<F>(v, j, twN, [&](int k) {
        if (!ok) return cmk<C>(0, 0);
        const C x = sb[sa * K::SLOT_STRIDE + k];
        const Tp kk = wk * (Tp)k;
        C r = cmk<C>(wr * x.x - kk * x.y, wr * x.y + kk * x.x);
        if (s2b >= 0) r = cadd(r, cmuli_s(sb[s2b * K::SLOT_STRIDE + k], sgn * (Tp)k));
        return r;
      });
      fft.template run<+1, WS>(v, j, sm, 1);
      F::template lsync<WS>();  // the region doubles as exchange scratch: all reads done
      C* dst = reinterpret_cast<C*>(myreg);
#pragma unroll
      for (int m = 0; m < V; ++m) dst[F::pos(j, m)] = cscale(v[m], A.scale);
    }
    __syncthreads();
    // ---- phase B: pointwise products, two neighbouring points per thread
    // (each field's pair moves as one 8/16-byte shared access)
    for (int p = tid; p < LPI * N / 2; p += K::THREADS) {
      const int pln = (2 * p) / N, z = (2 * p) % N;
      const long long pl = line0 + pln;
      if (pl >= A.nlines) continue;
      const long long o = pl * N + z;
      const int sp = pln * K::RS + z;
      Tp loc[2 * K::NG];  // [field][point]
#pragma unroll
      for (int f = 0; f < K::NG; ++f) {
        const C x = *reinterpret_cast<const C*>(reg + f * SFS + sp);
        loc[2 * f] = x.x;
        loc[2 * f + 1] = x.y;
      }
      Tp cdx2 = A.cdx2;
      if (LES && A.mcs) {  // the member's C_s (the host's float64 products, rounded once)
        const double cs = A.mcs[pl / A.lpm];
        cdx2 = A.vreman ? (Tp)(2.5 * cs * cs * A.dx * A.dx) : (Tp)((cs * A.dx) * (cs * A.dx));
      }
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        Tp ub[3], cb[3];
        const Tp* uo = nullptr;
        const Tp* co = nullptr;
        if (A.uphys) {
#pragma unroll
          for (int c = 0; c < DIM; ++c) ub[c] = A.uphys[c * A.rs + o + q];
          uo = ub;
        }
        if (A.cphys) {
#pragma unroll
          for (int c = 0; c < (DIM == 3 ? 3 : 1); ++c) cb[c] = A.cphys[c * A.rs + o + q];
          co = cb;
        }
        if (A.umax) {
#pragma unroll
          for (int c = 0; c < DIM; ++c) lmax = fmax(lmax, (double)(uo ? uo[c] : loc[2 * c + q]));
        }
        z_pointwise<Tp, DIM, LES, MODEL, PAR2D>(loc, 2, q, uo, co, cdx2);
        if (A.stress_only) {
#pragma unroll
          for (int c = 0; c < DIM; ++c) loc[2 * c + q] = (Tp)0;
        }
      }
#pragma unroll
      for (int f = 0; f < K::NOUT; ++f) *reinterpret_cast<C*>(reg + f * SFS + sp) = cmk<C>(loc[2 * f], loc[2 * f + 1]);
    }
    __syncthreads();
    // ---- phase C: r2c of product `grp` (with block-wide line barriers, groups
    // >= NOUT run idle for them; with line-level barriers they skip)
    if (!WS || grp < K::NOUT) {
      C v[V];
      const C* src = reinterpret_cast<const C*>(myreg);
#pragma unroll
      for (int m = 0; m < V; ++m) v[m] = src[j + T * m];
      fft.template run<-1, WS>(v, j, sm, 1);
      C* out = A.ws + (grp < K::NOUT ? grp : 0) * fs + lo;
      const bool wr = ok && grp < K::NOUT;
      if constexpr (F::MIR) {
        r2c_post_mir<F>(v, j, twN, [&](int k, C x) {
          if (wr) out[k] = x;
        });
      } else {
        r2c_post<F, WS>(v, j, sm, 1, twN, [&](int k, C x) {
          if (wr) out[k] = x;
        });
      }
    }
  }
  if (A.umax) {  // block maximum through the (now idle) line regions, one atomic per block
    __syncthreads();
    double* part = reinterpret_cast<double*>(reg);  // THREADS doubles fit in the regions
    part[tid] = lmax;
    __syncthreads();
    if (tid == 0) {
      double m = -INFINITY;
      for (int w = 0; w < K::THREADS; ++w) m = fmax(m, part[w]);
      atomicMax(A.umax, ord_encode(m));
    }
  }
}

}  // namespace sles
