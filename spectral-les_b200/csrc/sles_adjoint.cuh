// Discrete adjoint of the fused right-hand side and of the RK4 step (3D).
//
// The forward RHS at a state U (src/RK4_method.py:38-71 with the LES stress of
// src/math_formula.py:64-127) is
//   f(U) = P(mask rfft(u x w) + T) - nu K^2 U [+ c U, k != 0],
//   T_i  = 2i mask sum_j K_j rfft(nu_t S_ij),  u = irfft(U),  a_ij = irfft(i K_i U_j),
//   w    = (a23 - a32, a31 - a13, a12 - a21),  nu_t from a (Smagorinsky or Vreman).
// Its vector-Jacobian product g = J(U)^T lam, under the real inner product
// <x, y> = Re sum conj(x) y over the stored half-complex entries (the
// convention of torch's complex autograd), is assembled from the transposes
// of each piece:
//   rfft^T(G)  = N^3 c2r(h G)       h = 1/2 on bins 0 < kz < N/2, else 1
//   irfft^T(g) = (w / N^3) rfft(g)  w = 2 on bins 0 < kz < N/2, else 1
//   P^T = P (real symmetric per mode), mask^T = mask.
// With m = h mask P lam and n~ = N^3 c2r(m), D_ij = d_i n~_j (spectral):
//   nbar = n~,  sigbar_ii = -2 D_ii,  sigbar_ij = -2 (D_ij + D_ji)   (i < j)
//   ubar = w x nbar,  wbar = nbar x u
//   nubar = sum_{i<=j} sigbar_ij S_ij,  Sbar_ij = nu_t sigbar_ij + (d nu_t/d S_ij) nubar
//   abar from Sbar (S_ij = (a_ij + a_ji)/2) and wbar, plus d nu_t/d a for Vreman
//   g_j = (w/N^3) [rfft(ubar_j) - i sum_i K_i rfft(abar_ij)] - nu K^2 lam_j [+ c lam_j]
//   dL/dCs += (2/Cs) sum_x nubar nu_t                (nu_t is proportional to Cs^2)
//
// Passes (the forward's structure, run on two groups of fields):
//   AX prime   (x, ky, kz): from the state U and the cotangent lam: x-inverse of
//              U_c, i kx U_c (slots 0..5) and of m_c, i kx m_c (slots 9..14)
//   AY inverse y-inverse of both groups (k_ypass ADJ): slots 0..8 / 9..17 =
//              [a_c, dx_c, dy_c] of the state / of m
//   AZ         per z line: c2r of 24 physical lines (12 of the state, 12 of m),
//              the pointwise adjoint, r2c of ubar (3) and abar (9), then
//              Z_j = ubar_j - i kz abar_3j, A1_j, A2_j with the weights w/N^3
//   AY forward Y_j = Z_j - i ky A2_j, A1_j (k_ypass ADJ)
//   AX forward g_j = X(Y_j) - i kx X(A1_j) - nu K^2 lam_j [+ c lam_j]; the
//              adjoint RK4 update; then the AX prime of the next reverse stage
//
// Reverse RK4 stage s (forward stage s evaluated f at U_s; U_1 = U_0 + dt/2 k_0,
// U_2 = U_0 + dt/2 k_1, U_3 = U_0 + dt k_2, output U_0 + dt (k_0/6 + k_1/3 + k_2/3 + k_3/6)),
// with ubar = adjoint of the step output and acc = adjoint of the step input:
//   g = J(U_s)^T lam;  acc += g
//   s = 3: lam <- dt/3 ubar + dt g;   s = 2: lam <- dt/3 ubar + dt/2 g
//   s = 1: lam <- dt/6 ubar + dt/2 g; s = 0: ubar <- acc, lam <- dt/6 acc (next step back)
// Seed: acc = ubar, lam = dt/6 ubar.
//
// The corrected SSP-RK3 (U_1 = U_0 + dt k_0, U_2 = 3/4 U_0 + 1/4 (U_1 + dt k_1),
// output 1/3 U_0 + 2/3 (U_2 + dt k_2)) runs in Shu-Osher form, ubar carrying
// the cotangent of the latest stage state:
//   seed: acc = ubar/3, lam = 2/3 dt ubar
//   s = 2: w = 2/3 ubar + g; acc += 3/4 w; ubar <- w/4; lam <- dt/4 w
//   s = 1: w = ubar + g;     acc += w;                  lam <- dt w
//   s = 0: w = acc + g;      ubar <- w (gradient of the step input); acc <- w/3; lam <- 2/3 dt w
#pragma once
#include "sles_rhs.cuh"

namespace sles {

template <typename Tp>
struct AXArgs {
  using C = typename CT<Tp>::C;
  unsigned* err;
  C* ws;
  long long fs;
  int nkp, nk, nchunks;
  int fwd;             // 1: combine g from slots 0..5 and update acc / lam / ubar
  int prep;            // 1: x-inverse prime of (unext, lam) into slots 0..5, 9..14
  const C* unext;      // state of the next reverse stage
  C* ubar;
  C* acc;
  C* lam;
  Tp alpha, beta;      // lam <- alpha ubar + beta g;  last: ubar <- acc, lam <- alpha acc
  int last;
  // Shu-Osher form (SSP-RK3): w = pu ubar + g (last: w = acc + g); acc += pa w
  // (last: acc <- pa w); ubar <- pb w (last: ubar <- w); lam <- pl w
  int ssp;
  Tp pu, pa, pb, pl;
  Tp nu, forcing;
  double kmax;
  // corrected ETD2 (F excludes the viscous term, which E carries):
  // 1: w = E ubar + g; lam <- w1 w + w0 ubar; ubar <- w
  // 2: the step after the first (RK4) step: as 1 with lam <- w0 ubar (the
  //    cotangent of F(U_0), applied by mode 3 after the RK4 step's reverse)
  // 3: ubar <- ubar + g
  int etd;
  double dt_d, nu_d;
};

// Cox & Matthews (2002) ETD2 weights at z = dt nu k^2 (the forward's
// corrected branch, update_component in sles_rhs.cuh)
__device__ __forceinline__ void etd2_weights(double h, double z, double& E, double& w1, double& w0) {
  E = exp(-z);
  if (fabs(z) < 1e-2) {
    w1 = h * (1.5 - 2.0 * z / 3.0 + z * z / 4.0 - z * z * z / 15.0);
    w0 = h * (-0.5 + z / 6.0 - z * z / 24.0 + z * z * z / 120.0);
  } else {
    w1 = h * ((1.0 - z) * E - 1.0 + 2.0 * z) / (z * z);
    w0 = h * (-E + 1.0 - z) / (z * z);
  }
}

// m = h * mask * P(lam) at one mode (in place on s[3])
template <typename Tp>
__device__ __forceinline__ void adj_project(typename CT<Tp>::C (&s)[3], const int (&k)[3], double kmax, int n) {
  using C = typename CT<Tp>::C;
  const int k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
  const double kk = (double)(k2 == 0 ? 1 : k2);
  C P = cmk<C>(0, 0);
  bool in = true;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    P = cadd(P, cscale(s[c], (Tp)((double)k[c] / kk)));
    in = in && fabs((double)k[c]) < kmax;
  }
  const Tp h = in ? ((k[2] > 0 && k[2] < n / 2) ? (Tp)0.5 : (Tp)1) : (Tp)0;
#pragma unroll
  for (int c = 0; c < 3; ++c) s[c] = cscale(csub(s[c], cscale(P, (Tp)k[c])), h);
}

// ---------------------------------------------------------------------------
// AX pass.  Work item = (ky slice, chunk of W kz columns); lines along x.
// ---------------------------------------------------------------------------
// MODE (compile time, so each scheme's kernel carries only its own update):
// 0 the diagonal Runge-Kutta form (RK4, the reference's RK3), 1 Shu-Osher
// (SSP-RK3), 2 corrected ETD2.
template <typename Tp, int N, class F, int MODE>
__global__ void __launch_bounds__(XGeo<Tp, N, F, 3, 0>::THREADS, XGeo<Tp, N, F, 3, 0>::MINB)
k_adj_xpass(const __grid_constant__ AXArgs<Tp> A) {
  using K = XGeo<Tp, N, F, 3, 0>;
  using C = typename CT<Tp>::C;
  constexpr int T = K::T, V = K::V, W = K::W;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  C* rst = reinterpret_cast<C*>(smem_raw);  // [3][N][W] cotangent of the next stage
  C* sm0 = rst + 3 * K::TE;
  C* twt = sm0 + K::SCR;
  const int tid = threadIdx.x;
  const int l = tid % W, j = tid / W;
  F::fill_table_lin(twt);
  __syncthreads();
  F fft;
  const long long items = (long long)N * A.nchunks;
  const long long ps = (long long)N * A.nkp;
  const long long fs = A.fs;
  C* sm = sm0 + l;
  C* ws = A.ws;
  auto kx_at = [&](int m) { return kc2c(j + T * m, N); };
  auto rpos = [&](int c, int m) { return c * K::TE + (j + T * m) * W + l; };
  for (long long it = blockIdx.x; it < items; it += gridDim.x) {
    const int chunk = (int)(it % A.nchunks);
    const int sl = (int)(it / A.nchunks);
    const int col = chunk * W + l;
    const bool ok = col < A.nk;
    const long long base = (long long)sl * A.nkp + col;
    const int kyv = kc2c(sl, N);
    auto ld = [&](C (&v)[V], const C* src, int slot) {
#pragma unroll
      for (int m = 0; m < V; ++m) v[m] = ok ? src[slot * fs + base + (j + T * m) * ps] : cmk<C>(0, 0);
    };
    auto st = [&](int slot, const C (&v)[V]) {
      if (ok) {
#pragma unroll
        for (int m = 0; m < V; ++m) ws[slot * fs + base + (j + T * m) * ps] = v[m];
      }
    };
    // inverse x-transforms of a field and of i kx times it into slots s0, s0 + 3
    auto inv2 = [&](C (&v)[V], int s0) {
      C b[V];
#pragma unroll
      for (int m = 0; m < V; ++m) b[m] = cmuli_s(v[m], (Tp)kx_at(m));
      fft.template run_tab<+1, true>(b, j, sm, W, twt);
      st(s0 + 3, b);
      fft.template run_tab<+1, true>(v, j, sm, W, twt);
      st(s0, v);
    };
    if (A.fwd) {
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C v[V], h[V];
        ld(v, ws, c);
        fft.template run_tab<-1, true>(v, j, sm, W, twt);
        ld(h, ws, 3 + c);
        fft.template run_tab<-1, true>(h, j, sm, W, twt);
#pragma unroll
        for (int m = 0; m < V; ++m) {
          C g = cadd(v[m], cmuli_s(h[m], -(Tp)kx_at(m)));  // - i kx X(A1_c)
          C ln = cmk<C>(0, 0);
          if (ok) {
            const long long o = c * fs + base + (j + T * m) * ps;
            const int kx = kx_at(m);
            const int k2 = kx * kx + kyv * kyv + col * col;
            const C lc = A.lam[o];
            if constexpr (MODE != 2) g = csub(g, cscale(lc, A.nu * (Tp)k2));
            if (A.forcing > (Tp)0 && k2 != 0) g = cadd(g, cscale(lc, A.forcing));
            if constexpr (MODE == 2) {
              const C ub = A.ubar[o];
              if (A.etd == 3) {
                A.ubar[o] = cadd(ub, g);
                ln = lc;
              } else {
                double E, w1, w0;
                etd2_weights(A.dt_d, A.dt_d * A.nu_d * (double)k2, E, w1, w0);
                const C w = cadd(cscale(ub, (Tp)E), g);
                A.ubar[o] = w;
                ln = (A.etd == 1) ? cadd(cscale(w, (Tp)w1), cscale(ub, (Tp)w0)) : cscale(ub, (Tp)w0);
              }
            } else if constexpr (MODE == 1) {
              if (A.last) {
                const C w = cadd(A.acc[o], g);
                A.ubar[o] = w;
                A.acc[o] = cscale(w, A.pa);
                ln = cscale(w, A.pl);
              } else {
                const C w = cadd(cscale(A.ubar[o], A.pu), g);
                A.acc[o] = cadd(A.acc[o], cscale(w, A.pa));
                A.ubar[o] = cscale(w, A.pb);
                ln = cscale(w, A.pl);
              }
            } else {
              const C an = cadd(A.acc[o], g);
              A.acc[o] = an;
              if (A.last) {
                A.ubar[o] = an;
                ln = cscale(an, A.alpha);
              } else {
                ln = cadd(cscale(A.ubar[o], A.alpha), cscale(g, A.beta));
              }
            }
            A.lam[o] = ln;
          }
          rst[rpos(c, m)] = ln;
        }
      }
      if (!A.prep) continue;
    } else {
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C v[V];
        ld(v, A.lam, c);
#pragma unroll
        for (int m = 0; m < V; ++m) rst[rpos(c, m)] = v[m];
      }
    }
    // m = h mask P(lam) per mode (each thread revisits only its own positions)
#pragma unroll
    for (int m = 0; m < V; ++m) {
      C s[3];
      const int kv[3] = {kx_at(m), kyv, col};
#pragma unroll
      for (int c = 0; c < 3; ++c) s[c] = rst[rpos(c, m)];
      adj_project<Tp>(s, kv, A.kmax, N);
#pragma unroll
      for (int c = 0; c < 3; ++c) rst[rpos(c, m)] = s[c];
    }
#pragma unroll 1
    for (int c = 0; c < 3; ++c) {
      C v[V];
      ld(v, A.unext, c);
      inv2(v, c);
#pragma unroll
      for (int m = 0; m < V; ++m) v[m] = rst[rpos(c, m)];
      inv2(v, 9 + c);
    }
  }
}

// ---------------------------------------------------------------------------
// AZ pass: per z line, 12 thread groups; group g transforms physical lines g
// (state) and 12 + g (cotangent), then one adjoint product line.
// ---------------------------------------------------------------------------
template <typename Tp>
struct AZArgs {
  using C = typename CT<Tp>::C;
  C* ws;
  long long fs;
  int nkp;
  long long nlines;     // N^2
  Tp scale;             // 1/N^3 (state lines)
  Tp cdx2;              // (Cs dx)^2 (Smagorinsky) or 2.5 Cs^2 dx^2 (Vreman)
  double csfac;         // 2/Cs (0 when Cs == 0)
  double* csgrad;       // accumulates dL/dCs (device)
  unsigned* err;
};

template <typename Tp, int N, int LPI>
struct AZGeo {
  using F = typename MirrorIf<typename PlanFor<Tp, N / 2>::F>::type;  // as the forward z pass
  using C = typename CT<Tp>::C;
  static constexpr int L = N / 2, T = F::T, V = F::V;
  static constexpr int NGT = 12;                  // thread groups
  static constexpr int NPH = 24;                  // physical lines per z line
  static constexpr int NIN = 18;                  // input slots
  static constexpr int NKP = ((N / 2 + 1) + 3) / 4 * 4;
  static constexpr int THREADS = NGT * LPI * T;
  static constexpr int MINB = 1;
  static constexpr int LS = ((F::XLEN + 15) / 16) * 16 + 8;
  static constexpr int RS = 2 * LS;
  static_assert(RS >= N, "region must hold a physical line");
  static_assert(LS >= NKP, "region must hold a half-complex line");
  static constexpr int STAGE = NIN * LPI * NKP;
  static constexpr size_t OFF_TW = 16;
  static constexpr size_t OFF_RED = OFF_TW + (size_t)L * sizeof(C);
  static constexpr size_t OFF_STAGE = (OFF_RED + 32 * sizeof(double) + 127) / 128 * 128;
  static constexpr size_t OFF_REG = OFF_STAGE + 2 * (size_t)STAGE * sizeof(C);
  static constexpr size_t SMEM = OFF_REG + (size_t)NPH * LPI * RS * sizeof(Tp);
};

// d nu_t / d a for the Vreman model, scaled: out[m][p] += f * dnu/da_mp / nu
// = f * [dB/da_mp / (2B) - a_mp / aa] (gate held fixed; vreman.py:30-123)
template <typename Tp>
__device__ __forceinline__ void vreman_dnu(const Tp (&a)[3][3], Tp f, Tp (&ab)[3][3]) {
  Tp b[3][3];
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) b[p][q] = a[0][p] * a[0][q] + a[1][p] * a[1][q] + a[2][p] * a[2][q];
  const Tp B = (b[0][0] * b[1][1]) - (b[0][1] * b[0][1]) + (b[0][0] * b[2][2]) - (b[0][2] * b[0][2]) +
               (b[1][1] * b[2][2]) - (b[1][2] * b[1][2]);
  Tp aa = 0;
#pragma unroll
  for (int p = 0; p < 3; ++p)
#pragma unroll
    for (int q = 0; q < 3; ++q) aa += a[p][q] * a[p][q];
  const Tp tr = b[0][0] + b[1][1] + b[2][2];
  const Tp iB = (Tp)1 / B, ia = (Tp)1 / aa;
#pragma unroll
  for (int m = 0; m < 3; ++m)
#pragma unroll
    for (int p = 0; p < 3; ++p) {
      Tp s = a[m][p] * (tr - b[p][p]);
#pragma unroll
      for (int q = 0; q < 3; ++q)
        if (q != p) s -= b[p][q] * a[m][q];
      ab[m][p] += f * (s * iB - a[m][p] * ia);  // dB/da = 2 s
    }
}

// Pointwise adjoint at one point.  st(f): physical line value f of the 24
// (0..2 u_c, 3+3(i-1)+c: a_ic = d_i u_c; 12 + same for n~); writes ubar_c to
// line c and abar_ic to line 3 + 3(i-1) + c.  Returns nubar * nu_t.
template <typename Tp, int MODEL, class Acc>
__device__ __forceinline__ double adj_pointwise(Acc st, Tp cdx2) {
  Tp u[3], a[3][3], nb[3], D[3][3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    u[c] = st(c);
    nb[c] = st(12 + c);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      a[i][c] = st(3 + 3 * i + c);
      D[i][c] = st(15 + 3 * i + c);
    }
  const Tp w0 = a[1][2] - a[2][1], w1 = a[2][0] - a[0][2], w2 = a[0][1] - a[1][0];
  Tp ab[3][3];
  // wbar = nbar x u  -> a
  const Tp wb0 = nb[1] * u[2] - nb[2] * u[1], wb1 = nb[2] * u[0] - nb[0] * u[2], wb2 = nb[0] * u[1] - nb[1] * u[0];
  ab[0][0] = 0; ab[1][1] = 0; ab[2][2] = 0;
  ab[1][2] = wb0; ab[2][1] = -wb0;
  ab[2][0] = wb1; ab[0][2] = -wb1;
  ab[0][1] = wb2; ab[1][0] = -wb2;
  // ubar = w x nbar
  st(0) = w1 * nb[2] - w2 * nb[1];
  st(1) = w2 * nb[0] - w0 * nb[2];
  st(2) = w0 * nb[1] - w1 * nb[0];
  double red = 0.0;
  if (MODEL != M_NONE) {
    const Tp nu = eddy_viscosity_3d<Tp, MODEL>(a[0][0], a[0][1], a[0][2], a[1][0], a[1][1], a[1][2], a[2][0],
                                               a[2][1], a[2][2], cdx2);
    Tp S[3][3], sb[3][3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = i; j < 3; ++j) {
        S[i][j] = (i == j) ? a[i][i] : (Tp)0.5 * (a[i][j] + a[j][i]);
        sb[i][j] = (i == j) ? (Tp)-2 * D[i][i] : (Tp)-2 * (D[i][j] + D[j][i]);
      }
    Tp nub = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = i; j < 3; ++j) nub += sb[i][j] * S[i][j];
    red = (double)nub * (double)nu;
    Tp gS = 0;  // Smagorinsky: d nu / d S_ij = (c^2/nu) (2 S_ii | 4 S_ij), c = cdx2
    if (MODEL == M_SMAG && nu > (Tp)0) gS = nub * (cdx2 * cdx2 / nu);
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = i; j < 3; ++j) {
        const Tp Sb = nu * sb[i][j] + gS * (i == j ? (Tp)2 : (Tp)4) * S[i][j];
        if (i == j) {
          ab[i][i] += Sb;
        } else {
          ab[i][j] += (Tp)0.5 * Sb;
          ab[j][i] += (Tp)0.5 * Sb;
        }
      }
    if (MODEL == M_VREMAN && nu > (Tp)0) vreman_dnu<Tp>(a, nub * nu, ab);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int c = 0; c < 3; ++c) st(3 + 3 * i + c) = ab[i][c];
  return red;
}

template <typename Tp, int N, int MODEL, int LPI>
__global__ void __launch_bounds__(AZGeo<Tp, N, LPI>::THREADS, AZGeo<Tp, N, LPI>::MINB)
k_adj_zpass(const AZArgs<Tp> A) {
  using K = AZGeo<Tp, N, LPI>;
  using F = typename K::F;
  using C = typename CT<Tp>::C;
  constexpr int T = K::T, V = K::V, NKP = K::NKP, SFS = LPI * K::RS;
  constexpr int WS = (T <= 32 && 32 % T == 0) ? 1 : 0;  // a line's threads share one warp
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
  C* twN = reinterpret_cast<C*>(smem_raw + K::OFF_TW);
  double* red = reinterpret_cast<double*>(smem_raw + K::OFF_RED);
  C* stage = reinterpret_cast<C*>(smem_raw + K::OFF_STAGE);   // [2][NIN][LPI][NKP]
  Tp* reg = reinterpret_cast<Tp*>(smem_raw + K::OFF_REG);     // [NPH][LPI][RS]
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
  const long long nbi = (A.nlines + LPI - 1) / LPI;
  auto issue = [&](long long b, int buf) {
    const long long l0 = b * LPI;
    const long long nl = (A.nlines - l0 < LPI) ? A.nlines - l0 : LPI;
    const unsigned bytes = (unsigned)(nl * A.nkp * (long long)sizeof(C));
    fence_proxy_async();
    mbar_arrive_expect_tx(&bar[buf], bytes * K::NIN);
    for (int s = 0; s < K::NIN; ++s)
      bulk_g2s(stage + buf * K::STAGE + s * LPI * NKP, A.ws + s * fs + l0 * A.nkp, bytes, &bar[buf]);
  };
  if (tid == 0 && blockIdx.x < nbi) issue(blockIdx.x, 0);
  double racc = 0.0;
  int iter = 0;
  for (long long bi = blockIdx.x; bi < nbi; bi += gridDim.x, ++iter) {
    const int buf = iter & 1;
    if (tid == 0 && bi + gridDim.x < nbi) issue(bi + gridDim.x, buf ^ 1);
    mbar_wait_bounded(&bar[buf], (iter >> 1) & 1, A.err);
    const long long line0 = bi * LPI;
    const long long line = line0 + ln;
    const bool ok = line < A.nlines;
    // ---- phase A: c2r of physical lines grp (state) and 12 + grp (cotangent)
#pragma unroll 1
    for (int r = 0; r < 2; ++r) {
      const int f = grp + 12 * r;
      const int sbase = 9 * r, g = grp;  // slot base of the group; line index within it
      // slot g, or for g >= 9 i kz times slot g - 9 (d/dz a_c), without
      // branches that would split a warp's groups
      const int sl = (g < 9) ? sbase + g : sbase + g - 9;
      const Tp wr = (g < 9) ? (Tp)1 : (Tp)0, wk = (g < 9) ? (Tp)0 : (Tp)1;
      const C* sb = stage + buf * K::STAGE + ln * NKP;
      Tp* myreg = reg + (f * LPI + ln) * K::RS;
      C* sm = reinterpret_cast<C*>(myreg);
      C v[V];
      c2r_pre<F>(v, j, twN, [&](int k) {
        if (!ok) return cmk<C>(0, 0);
        const C x = sb[sl * LPI * NKP + k];
        const Tp kk = wk * (Tp)k;
        return cmk<C>(wr * x.x - kk * x.y, wr * x.y + kk * x.x);
      });
      fft.template run<+1, WS>(v, j, sm, 1);
      F::template lsync<WS>();
      const Tp sc = r == 0 ? A.scale : (Tp)1;
#pragma unroll
      for (int m = 0; m < V; ++m) sm[F::pos(j, m)] = cscale(v[m], sc);
    }
    __syncthreads();
    // ---- phase B: pointwise adjoint
    for (int p = tid; p < LPI * N; p += K::THREADS) {
      const int pln = p / N, z = p % N;
      if (line0 + pln >= A.nlines) continue;
      const int sp = pln * K::RS + z;
      racc += adj_pointwise<Tp, MODEL>([&](int f) -> Tp& { return reg[f * SFS + sp]; }, A.cdx2);
    }
    __syncthreads();
    // ---- phase C: r2c of adjoint product `grp` into region 12 + grp (as a half-complex line)
    {
      Tp* myreg = reg + (grp * LPI + ln) * K::RS;
      C* sm = reinterpret_cast<C*>(myreg);
      C* spec = reinterpret_cast<C*>(reg + ((12 + grp) * LPI + ln) * K::RS);
      C v[V];
#pragma unroll
      for (int m = 0; m < V; ++m) v[m] = sm[j + T * m];
      fft.template run<-1, WS>(v, j, sm, 1);
      if constexpr (F::MIR) r2c_post_mir<F>(v, j, twN, [&](int k, C x) { spec[k] = x; });
      else r2c_post<F, WS>(v, j, sm, 1, twN, [&](int k, C x) { spec[k] = x; });
    }
    __syncthreads();
    // ---- phase D: Z_c = ubar_c - i kz abar_3c, A1_c, A2_c with weights w/N^3
    const int nk = N / 2 + 1;
    for (int e = tid; e < 9 * LPI * nk; e += K::THREADS) {
      const int k = e % nk, rest = e / nk;
      const int pln = rest % LPI, o = rest / LPI;
      const long long pl = line0 + pln;
      if (pl >= A.nlines) continue;
      auto spec = [&](int q) { return reinterpret_cast<const C*>(reg + ((12 + q) * LPI + pln) * K::RS)[k]; };
      const Tp wgt = ((k > 0 && k < N / 2) ? (Tp)2 : (Tp)1) * A.scale;
      C x;
      if (o < 3) x = cadd(spec(o), cmuli_s(spec(9 + o), -(Tp)k));
      else x = spec(o);
      A.ws[o * fs + pl * A.nkp + k] = cscale(x, wgt);
    }
    __syncthreads();  // the regions are rewritten by the next line group's phase A
  }
  if (MODEL != M_NONE) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) racc += __shfl_down_sync(0xffffffffu, racc, o);
    if ((tid & 31) == 0) red[tid >> 5] = racc;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int w = 0; w < (K::THREADS + 31) / 32; ++w) s += red[w];
      atomicAdd(A.csgrad, s * A.csfac);
    }
  }
}

// lam = w1(k) ubar on every stored mode of the 3 half-complex fields (the
// corrected ETD2 seed; w1 the step's F_n weight at z = dt nu k^2)
template <typename Tp>
__global__ void k_adj_seed_etd(const typename CT<Tp>::C* __restrict__ ubar, typename CT<Tp>::C* __restrict__ lam,
                               long long fs, int n, int nkp, int nk, double dt, double nu) {
  const long long tot = 3LL * fs;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
    const long long e = i % fs;
    const int kz = (int)(e % nkp);
    const long long r = e / nkp;
    const int y = (int)(r % n);
    const long long x = r / n;
    if (kz >= nk || x >= n) {
      lam[i] = cmk<typename CT<Tp>::C>(0, 0);
      continue;
    }
    const int kx = kc2c((int)x, n), ky = kc2c(y, n);
    double E, w1, w0;
    etd2_weights(dt, dt * nu * (double)(kx * kx + ky * ky + kz * kz), E, w1, w0);
    lam[i] = cscale(ubar[i], (Tp)w1);
  }
}

// acc = sacc ubar, lam = alpha ubar over n complex elements (adjoint seed)
template <typename Tp>
__global__ void k_adj_seed(const typename CT<Tp>::C* __restrict__ ubar, typename CT<Tp>::C* __restrict__ acc,
                           typename CT<Tp>::C* __restrict__ lam, long long n, Tp alpha, Tp sacc) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const auto v = ubar[i];
    acc[i] = cscale(v, sacc);
    lam[i] = cscale(v, alpha);
  }
}

}  // namespace sles
