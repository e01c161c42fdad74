// Register-resident Stockham line FFT for sm_100a.
//
// A line of L complex points is owned by T cooperating threads; thread j holds
// the V = L/T points x[j + T*m] ("cyclic" distribution) in registers.  The
// transform runs as up to three Stockham radix stages R0, R1, R2
// (L = R0*R1*R2).  Every stage reads the cyclic distribution and performs
// L/(R*T) radix-R butterflies per thread in registers (twiddle first, then the
// DFT_R, Stockham autosort indexing idxD = (b/Ns)*Ns*R + b%Ns).  Between
// stages the values are exchanged through a padded shared-memory line (one
// pad slot every 16 points keeps the strided writes of the autosort free of
// bank conflicts); the last stage writes its outputs straight back into the
// cyclic registers, so input and output of a transform share the same
// distribution and forward/inverse transforms and pointwise products chain in
// registers without any shared-memory traffic.
//
// Stage twiddles are generated once per thread in float64 (sincospi) and
// rounded once to the working precision.  Forward = exp(-2 pi i nk/L),
// inverse = exp(+2 pi i nk/L), both unscaled.
#pragma once
#include "sles_common.cuh"

namespace sles {

// ---------------------------------------------------------------------------
// small DFTs on registers, natural order in and out; DIR = -1 forward, +1 inverse
// ---------------------------------------------------------------------------
template <typename C, typename Tp>
__device__ __forceinline__ C rot(C a, Tp c, Tp s) {  // a * (c + i s)
  return cmk<C>(a.x * c - a.y * s, a.x * s + a.y * c);
}

template <int DIR, typename C>
__device__ __forceinline__ void dft2(C& a, C& b) {
  C t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <int DIR, typename C>
__device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3) {
  C t0 = cadd(a0, a2), t1 = csub(a0, a2), t2 = cadd(a1, a3), t3 = csub(a1, a3);
  a0 = cadd(t0, t2);
  a2 = csub(t0, t2);
  if (DIR < 0) {
    a1 = cadd(t1, cmulmi(t3));
    a3 = cadd(t1, cmuli(t3));
  } else {
    a1 = cadd(t1, cmuli(t3));
    a3 = cadd(t1, cmulmi(t3));
  }
}

template <int DIR, typename C>
__device__ __forceinline__ void dft3(C& a0, C& a1, C& a2) {
  using Tp = decltype(C::x);
  const Tp h = (Tp)0.86602540378443864676;  // sin(2 pi / 3)
  C s = cadd(a1, a2), d = csub(a1, a2);
  C m = cmk<C>(a0.x - (Tp)0.5 * s.x, a0.y - (Tp)0.5 * s.y);
  a0 = cadd(a0, s);
  C id = cmk<C>(-d.y * h, d.x * h);  // i h d
  if (DIR < 0) {
    a1 = csub(m, id);
    a2 = cadd(m, id);
  } else {
    a1 = cadd(m, id);
    a2 = csub(m, id);
  }
}

template <int R, int DIR, typename C>
__device__ __forceinline__ void dft(C (&u)[R]) {
  using Tp = decltype(C::x);
  if constexpr (R == 1) {
  } else if constexpr (R == 2) {
    dft2<DIR>(u[0], u[1]);
  } else if constexpr (R == 3) {
    dft3<DIR>(u[0], u[1], u[2]);
  } else if constexpr (R == 4) {
    dft4<DIR>(u[0], u[1], u[2], u[3]);
  } else if constexpr (R == 6) {
    // 6 = 2 (inner, stride 3) x 3 (outer); X[k1 + 2 k2]
    C y[3][2];
#pragma unroll
    for (int n2 = 0; n2 < 3; ++n2) {
      y[n2][0] = u[n2];
      y[n2][1] = u[n2 + 3];
      dft2<DIR>(y[n2][0], y[n2][1]);
    }
    const Tp c = (Tp)0.5, s = (Tp)0.86602540378443864676;  // w6^1
    y[1][1] = rot(y[1][1], c, (Tp)DIR * s);
    y[2][1] = rot(y[2][1], -c, (Tp)DIR * s);  // w6^2
#pragma unroll
    for (int k1 = 0; k1 < 2; ++k1) {
      dft3<DIR>(y[0][k1], y[1][k1], y[2][k1]);
      u[k1] = y[0][k1];
      u[k1 + 2] = y[1][k1];
      u[k1 + 4] = y[2][k1];
    }
  } else if constexpr (R == 8) {
    C e0 = u[0], e1 = u[2], e2 = u[4], e3 = u[6];
    C o0 = u[1], o1 = u[3], o2 = u[5], o3 = u[7];
    dft4<DIR>(e0, e1, e2, e3);
    dft4<DIR>(o0, o1, o2, o3);
    const Tp r = (Tp)0.70710678118654752440;
    o1 = rot(o1, r, (Tp)DIR * r);
    o2 = (DIR < 0) ? cmulmi(o2) : cmuli(o2);
    o3 = rot(o3, -r, (Tp)DIR * r);
    u[0] = cadd(e0, o0); u[4] = csub(e0, o0);
    u[1] = cadd(e1, o1); u[5] = csub(e1, o1);
    u[2] = cadd(e2, o2); u[6] = csub(e2, o2);
    u[3] = cadd(e3, o3); u[7] = csub(e3, o3);
  } else if constexpr (R == 16) {
    // 16 = 4 (inner over n1, stride 4) x 4 (outer over n2); X[k1 + 4 k2]
    C y[4][4];
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) {
      y[n2][0] = u[n2];
      y[n2][1] = u[n2 + 4];
      y[n2][2] = u[n2 + 8];
      y[n2][3] = u[n2 + 12];
      dft4<DIR>(y[n2][0], y[n2][1], y[n2][2], y[n2][3]);
    }
    const Tp c1 = (Tp)0.92387953251128675613, s1 = (Tp)0.38268343236508977173;
    const Tp r = (Tp)0.70710678118654752440;
    const Tp d = (Tp)DIR;
    y[1][1] = rot(y[1][1], c1, d * s1);   // w^1
    y[1][2] = rot(y[1][2], r, d * r);     // w^2
    y[1][3] = rot(y[1][3], s1, d * c1);   // w^3
    y[2][1] = rot(y[2][1], r, d * r);     // w^2
    y[2][2] = (DIR < 0) ? cmulmi(y[2][2]) : cmuli(y[2][2]);  // w^4
    y[2][3] = rot(y[2][3], -r, d * r);    // w^6
    y[3][1] = rot(y[3][1], s1, d * c1);   // w^3
    y[3][2] = rot(y[3][2], -r, d * r);    // w^6
    y[3][3] = rot(y[3][3], -c1, -d * s1); // w^9
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
      dft4<DIR>(y[0][k1], y[1][k1], y[2][k1], y[3][k1]);
      u[k1] = y[0][k1];
      u[k1 + 4] = y[1][k1];
      u[k1 + 8] = y[2][k1];
      u[k1 + 12] = y[3][k1];
    }
  } else {
    static_assert(R == 0, "unsupported radix");
  }
}


// ---------------------------------------------------------------------------
// Stockham line engine
// ---------------------------------------------------------------------------
// PADD: one exchange pad slot after every PADD points (0: PADD = R0, which
// keeps the first stage's autosort writes, stride R0, on distinct banks)
template <typename Tp, int L_, int R0, int R1, int R2, int T_, int PADD_ = 0>
struct LineFFT {
  using C = typename CT<Tp>::C;
  static constexpr int L = L_;
  static constexpr int T = T_;
  static constexpr int V = L / T;
  static constexpr int S = (R1 == 1) ? 1 : ((R2 == 1) ? 2 : 3);
  static_assert(R0 * R1 * R2 == L, "radix plan does not multiply to L");
  static_assert((L / R0) % T == 0 && (L / R1) % T == 0 && (L / R2) % T == 0,
                "threads per line must divide the butterfly count of every stage");
  static constexpr int NB1 = (S >= 2) ? (L / R1) / T : 0;
  static constexpr int NB2 = (S >= 3) ? (L / R2) / T : 0;
  static constexpr int TW1 = (S >= 2) ? NB1 * (R1 - 1) : 1;
  static constexpr int TW2 = (S >= 3) ? NB2 * (R2 - 1) : 1;
  static constexpr int PADD = PADD_ > 0 ? PADD_ : R0;
  static constexpr int RAD0 = R0, RAD1 = R1, RAD2 = R2;
  static constexpr int XLEN = L + L / PADD + 1;  // exchange line length (slots)
  // output bin of register m of thread j (the cyclic distribution)
  static constexpr bool MIR = false;
  __device__ __forceinline__ static int pos(int j, int m) { return j + T * m; }
  __device__ __forceinline__ static int pad(int p) { return p + (int)((unsigned)p / (unsigned)PADD); }
  // per-stage twiddle tables, [r][k] so a warp reads consecutive entries:
  // stage 1: W_{R0 R1}^{k r}, k < R0; stage 2: W_L^{k r}, k < R0 R1
  static constexpr int TAB1 = (S >= 2) ? (R1 - 1) * R0 : 0;
  static constexpr int TAB = TAB1 + ((S >= 3) ? (R2 - 1) * R0 * R1 : 0) + 1;

  C tw1[TW1];
  C tw2[TW2];

  // forward twiddles of stage s for thread j (float64, rounded once)
  __device__ __forceinline__ void init(int j) {
    if constexpr (S >= 2) {
#pragma unroll
      for (int q = 0; q < NB1; ++q) {
        int k = (j + T * q) % R0;
#pragma unroll
        for (int r = 1; r < R1; ++r) tw1[q * (R1 - 1) + r - 1] = twiddle<Tp>((long long)k * r, R0 * R1, -1);
      }
    }
    if constexpr (S >= 3) {
#pragma unroll
      for (int q = 0; q < NB2; ++q) {
        int k = (j + T * q) % (R0 * R1);
#pragma unroll
        for (int r = 1; r < R2; ++r) tw2[q * (R2 - 1) + r - 1] = twiddle<Tp>((long long)k * r, L, -1);
      }
    }
  }

  template <int R, int DIR, bool LAST, bool TWID, int NTW>
  __device__ __forceinline__ void stage(C (&v)[V], const C (&tw)[NTW], int Ns, int j, C* sm, int ws) {
    constexpr int NB = (L / R) / T;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      C u[R];
#pragma unroll
      for (int r = 0; r < R; ++r) u[r] = v[q + r * NB];
      if constexpr (TWID) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          C w = tw[q * (R - 1) + r - 1];
          u[r] = (DIR < 0) ? cmul(u[r], w) : cmulc(u[r], w);
        }
      }
      dft<R, DIR>(u);
      if constexpr (LAST) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[q + r * NB] = u[r];
      } else {
        const unsigned b = (unsigned)(j + T * q), ns = (unsigned)Ns;
        const int idxD = (int)((b / ns) * ns * R + b % ns);
#pragma unroll
        for (int r = 0; r < R; ++r) sm[pad(idxD + r * Ns) * ws] = u[r];
      }
    }
  }

  // Same stage with twiddles read from a shared table tab[e] = exp(-2 pi i e/L)
  // (threads of one line share j, so a warp reads few distinct entries).
  // LIN: tab is the linear table W_L^e (e < L) instead of the per-stage [r][k] tables
  template <int R, int DIR, bool LAST, bool LIN>
  __device__ __forceinline__ void stage_tab(C (&v)[V], const C* tab, int Ns, int j, C* sm, int ws) {
    constexpr int NB = (L / R) / T;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      C u[R];
#pragma unroll
      for (int r = 0; r < R; ++r) u[r] = v[q + r * NB];
      const unsigned b = (unsigned)(j + T * q), ns = (unsigned)Ns;
      const int k = (int)(b % ns);
      if (Ns > 1) {  // tab points at this stage's [r-1][k] table (Ns entries per r)
#pragma unroll
        for (int r = 1; r < R; ++r) {
          const C w = LIN ? tab[lin_pad(k * r * (L / (Ns * R)))] : tab[(r - 1) * Ns + k];
          u[r] = (DIR < 0) ? cmul(u[r], w) : cmulc(u[r], w);
        }
      }
      dft<R, DIR>(u);
      if constexpr (LAST) {
#pragma unroll
        for (int r = 0; r < R; ++r) v[q + r * NB] = u[r];
      } else {
        const int idxD = (int)((b / ns) * ns * R) + k;
#pragma unroll
        for (int r = 0; r < R; ++r) sm[pad(idxD + r * Ns) * ws] = u[r];
      }
    }
  }

  // Barrier among the threads that share a line's exchange scratch: the whole
  // block (WS = 0, lines spread over warps) or only the line's own T
  // consecutive lanes of one warp (WS = 1).
  template <int WS>
  __device__ __forceinline__ static void lsync() {
    if constexpr (WS) {
      static_assert(T <= 32 && 32 % T == 0, "a line's threads must lie in one warp");
      const unsigned lane = threadIdx.x & 31u;
      const unsigned m = (T == 32) ? 0xffffffffu : (((1u << T) - 1u) << (lane / T * T));
      __syncwarp(m);
    } else {
      __syncthreads();
    }
  }

  // Transform with twiddles from `tab` (L entries, see fill_table); needs no init().
  // LEAD = false drops the leading barrier (the guard of the scratch against
  // the previous transform's last reads) where the caller has just passed one.
  template <int DIR, bool LIN = false, int WS = 0, bool LEAD = true>
  __device__ __forceinline__ void run_tab(C (&v)[V], int j, C* sm, int ws, const C* tab) {
    if constexpr (S >= 2 && LEAD) lsync<WS>();
    stage_tab<R0, DIR, S == 1, LIN>(v, tab, 1, j, sm, ws);
    if constexpr (S >= 2) {
      exchange<WS>(v, j, sm, ws);
      if constexpr (S >= 3) lsync<WS>();
      stage_tab<R1, DIR, S == 2, LIN>(v, tab, R0, j, sm, ws);
    }
    if constexpr (S >= 3) {
      exchange<WS>(v, j, sm, ws);
      stage_tab<R2, DIR, true, LIN>(v, LIN ? tab : tab + TAB1, R0 * R1, j, sm, ws);
    }
  }

  // linear table W_L^e, e < L (float64, rounded once)
  __device__ __forceinline__ static void fill_table_lin(C* tab) {
    for (int e = threadIdx.x; e < L; e += blockDim.x) tab[lin_pad(e)] = twiddle<Tp>(e, L, -1);
  }
  // The linear table is read at strides k*r*L/(Ns*R); one pad slot per 16
  // entries spreads the indices a warp reads over the shared-memory banks.
  static constexpr int LIN_LEN = L + L / 16 + 1;  // slots of the padded linear table
  __device__ __forceinline__ static int lin_pad(int e) { return e + (int)((unsigned)e / 16u); }

  // cooperative fill of the per-stage twiddle tables (TAB entries; float64, rounded once)
  __device__ __forceinline__ static void fill_table(C* tab) {
    for (int e = threadIdx.x; e < TAB; e += blockDim.x) {
      if (e < TAB1) {
        const int r = e / R0 + 1, k = e % R0;
        tab[e] = twiddle<Tp>((long long)k * r, R0 * R1, -1);
      } else if (e < TAB - 1) {
        const int f = e - TAB1, r = f / (R0 * R1) + 1, k = f % (R0 * R1);
        tab[e] = twiddle<Tp>((long long)k * r, L, -1);
      }
    }
  }

  template <int WS = 0>
  __device__ __forceinline__ void exchange(C (&v)[V], int j, C* sm, int ws) {
    lsync<WS>();
#pragma unroll
    for (int m = 0; m < V; ++m) v[m] = sm[pad(j + T * m) * ws];
  }

  // In-place transform of the cyclic registers.  sm: this line's exchange
  // scratch (XLEN slots of stride ws).  With WS = 0 all threads of the block
  // must call this uniformly (it contains __syncthreads when S > 1); with
  // WS = 1 only the line's own lanes.  Convention shared by every user of an
  // exchange scratch: a barrier precedes each write phase, so back-to-back
  // transforms on one scratch are safe.
  template <int DIR, int WS = 0>
  __device__ __forceinline__ void run(C (&v)[V], int j, C* sm, int ws) {
    if constexpr (S >= 2) lsync<WS>();
    stage<R0, DIR, S == 1, false>(v, tw1, 1, j, sm, ws);
    if constexpr (S >= 2) {
      exchange<WS>(v, j, sm, ws);
      if constexpr (S >= 3) lsync<WS>();
      stage<R1, DIR, S == 2, true>(v, tw1, R0, j, sm, ws);
    }
    if constexpr (S >= 3) {
      exchange<WS>(v, j, sm, ws);
      stage<R2, DIR, true, true>(v, tw2, R0 * R1, j, sm, ws);
    }
  }
};

// ---------------------------------------------------------------------------
// radix plans per line length (complex points).  T = threads per line.
// ---------------------------------------------------------------------------
template <typename Tp, int L> struct PlanFor;
template <typename Tp> struct PlanFor<Tp, 4>    { using F = LineFFT<Tp, 4, 4, 1, 1, 1>; };
template <typename Tp> struct PlanFor<Tp, 6>    { using F = LineFFT<Tp, 6, 6, 1, 1, 1>; };
template <typename Tp> struct PlanFor<Tp, 8>    { using F = LineFFT<Tp, 8, 8, 1, 1, 1>; };
template <typename Tp> struct PlanFor<Tp, 12>   { using F = LineFFT<Tp, 12, 4, 3, 1, 1>; };
template <typename Tp> struct PlanFor<Tp, 16>   { using F = LineFFT<Tp, 16, 4, 4, 1, 4>; };
template <typename Tp> struct PlanFor<Tp, 24>   { using F = LineFFT<Tp, 24, 2, 4, 3, 2>; };
template <typename Tp> struct PlanFor<Tp, 32>   { using F = LineFFT<Tp, 32, 8, 4, 1, 4>; };
template <typename Tp> struct PlanFor<Tp, 48>   { using F = LineFFT<Tp, 48, 4, 4, 3, 4>; };
template <typename Tp> struct PlanFor<Tp, 64>   { using F = LineFFT<Tp, 64, 8, 8, 1, 8>; };
template <typename Tp> struct PlanFor<Tp, 96>   { using F = LineFFT<Tp, 96, 4, 4, 6, 8>; };
template <typename Tp> struct PlanFor<Tp, 128>  { using F = LineFFT<Tp, 128, 16, 8, 1, 8>; };
template <typename Tp> struct PlanFor<Tp, 256>  { using F = LineFFT<Tp, 256, 16, 16, 1, 16>; };
template <typename Tp> struct PlanFor<Tp, 512>  { using F = LineFFT<Tp, 512, 16, 16, 2, 32>; };
template <typename Tp> struct PlanFor<Tp, 1024> { using F = LineFFT<Tp, 1024, 16, 16, 4, 64>; };

// the same plan with another exchange padding divisor
template <class F, int P> struct WithPad;
template <typename Tp, int L, int R0, int R1, int R2, int T, int P0, int P>
struct WithPad<LineFFT<Tp, L, R0, R1, R2, T, P0>, P> {
  using F = LineFFT<Tp, L, R0, R1, R2, T, P>;
};

// The plan with the second butterfly of its last stage mirrored: thread j runs
// the last-stage butterflies j and 2T - j (thread 0: 0 and T) in place of j
// and j + T, so its outputs are the bins b_q + 2T r (q = register m mod 2,
// r = m / 2) and every bin k has its mirror L - k in the same thread: the
// real<->half-complex post step (r2c_post_mir) needs no exchange.  For plans
// of two stages with two last-stage butterflies per thread (R0 = 2T).  Inputs
// stay cyclic; only the outputs are permuted (pos).
template <class B>
struct MirrorFFT : B {
  using C = typename B::C;
  using Tp = decltype(C::x);
  static constexpr int L = B::L, T = B::T, V = B::V, R0 = B::RAD0, R1 = B::RAD1;
  static_assert(B::S == 2 && B::NB1 == 2 && R0 == 2 * T, "mirrored plans have two stages, two last butterflies");
  static constexpr bool MIR = true;
  __device__ __forceinline__ static int bfly1(int j) { return j ? 2 * T - j : T; }
  __device__ __forceinline__ static int pos(int j, int m) { return ((m & 1) ? bfly1(j) : j) + R0 * (m >> 1); }
  // register holding the mirror bin (L - k) mod L of register m (j != 0, j == 0)
  static constexpr int mirror_reg(int m, bool j0) {
    return !j0 ? (1 - (m & 1)) + 2 * (R1 - 1 - (m >> 1))
               : ((m & 1) ? 1 + 2 * (R1 - 1 - (m >> 1)) : ((m >> 1) == 0 ? 0 : 2 * (R1 - (m >> 1))));
  }
  __device__ __forceinline__ void init(int j) {
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      const int k = q ? bfly1(j) : j;  // < R0
#pragma unroll
      for (int r = 1; r < R1; ++r) this->tw1[q * (R1 - 1) + r - 1] = twiddle<Tp>((long long)k * r, R0 * R1, -1);
    }
  }
  template <int DIR, int WS = 0>
  __device__ __forceinline__ void run(C (&v)[V], int j, C* sm, int ws) {
    B::template lsync<WS>();
    this->template stage<R0, DIR, false, false>(v, this->tw1, 1, j, sm, ws);
    B::template lsync<WS>();
    const int b1 = bfly1(j);
#pragma unroll
    for (int m = 0; m < V; ++m) v[m] = sm[B::pad(((m & 1) ? b1 : j) + R0 * (m >> 1)) * ws];
    this->template stage<R1, DIR, true, true>(v, this->tw1, R0, j, sm, ws);
  }
};

// MirrorFFT<F> where F qualifies (and SLES_MIRROR != 0), else F
#ifndef SLES_MIRROR
#define SLES_MIRROR 1
#endif
template <class F, bool OK = (SLES_MIRROR != 0 && F::S == 2 && F::NB1 == 2 && F::RAD0 == 2 * F::T)>
struct MirrorIf { using type = F; };
template <class F> struct MirrorIf<F, true> { using type = MirrorFFT<F>; };

// Plans with at most 8-12 points per thread, for passes that keep several
// transformed lines live in registers at once (one more exchange per line).
template <typename Tp, int L> struct PlanLo { using F = typename PlanFor<Tp, L>::F; };
template <typename Tp> struct PlanLo<Tp, 128> { using F = LineFFT<Tp, 128, 8, 4, 4, 16>; };
template <typename Tp> struct PlanLo<Tp, 256> { using F = LineFFT<Tp, 256, 8, 8, 4, 32>; };
template <typename Tp> struct PlanLo<Tp, 512> { using F = LineFFT<Tp, 512, 8, 8, 8, 64>; };

// ---------------------------------------------------------------------------
// real <-> half-complex via a half-length complex FFT (N = 2L real points)
// ---------------------------------------------------------------------------
// c2r pre-processing.  X(k) returns the half-complex input bin k in [0, L].
// The imaginary parts of bins 0 and L are discarded (pocketfft/numpy irfft
// semantics).  Produces Z'[k] = (X_k + conj X_{L-k}) + i (X_k - conj X_{L-k}) W_N^{-k}
// in the cyclic registers; the unscaled inverse L-point FFT of Z' then yields
// z'[n] = N*(x[2n] + i x[2n+1]).  twN[k] = exp(-2 pi i k/N), k < L.
template <class F, class Src>
__device__ __forceinline__ void c2r_pre(typename F::C (&v)[F::V], int j, const typename F::C* twN, Src X) {
  using C = typename F::C;
#pragma unroll
  for (int m = 0; m < F::V; ++m) {
    int k = j + F::T * m;
    C a = X(k), b = X(F::L - k);
    if (k == 0) { a.y = 0; b.y = 0; }
    C e = cadd(a, cconj(b));
    C o = cmulc(csub(a, cconj(b)), twN[k]);
    v[m] = cadd(e, cmuli(o));
  }
}

// r2c post-processing.  v holds Z = FFT_L(z) with z[n] = x[2n] + i x[2n+1];
// emits out(k, X_k) for k in [0, L] (bin L by thread j == 0).  Uses the line's
// exchange scratch; all threads of the block (WS = 0) or the line's lanes
// (WS = 1) must call it uniformly.
template <class F, int WS = 0, class Dst>
__device__ __forceinline__ void r2c_post(typename F::C (&v)[F::V], int j, typename F::C* sm, int ws,
                                         const typename F::C* twN, Dst out) {
  using C = typename F::C;
  using Tp = decltype(C::x);
  F::template lsync<WS>();
#pragma unroll
  for (int m = 0; m < F::V; ++m) sm[F::pad(j + F::T * m) * ws] = v[m];
  F::template lsync<WS>();
#pragma unroll
  for (int m = 0; m < F::V; ++m) {
    int k = j + F::T * m;
    C z = v[m];
    C zc = cconj(sm[F::pad((int)((unsigned)(F::L - k) % (unsigned)F::L)) * ws]);
    C s = cadd(z, zc), d = csub(z, zc);
    C t = cmulmi(cmul(twN[k], d));
    out(k, cmk<C>((Tp)0.5 * (s.x + t.x), (Tp)0.5 * (s.y + t.y)));
    if (k == 0) out(F::L, cmk<C>(z.x - z.y, (Tp)0));
  }
}

// r2c post-processing on a mirrored plan's outputs (MirrorFFT): each bin's
// mirror is in the thread's own registers, so no exchange and no barrier.
// Emits out(k, X_k) for the thread's bins (k = F::pos(j, m)) and bin L by j == 0.
template <class F, class Dst>
__device__ __forceinline__ void r2c_post_mir(typename F::C (&v)[F::V], int j, const typename F::C* twN, Dst out) {
  using C = typename F::C;
  using Tp = decltype(C::x);
  const bool j0 = (j == 0);
#pragma unroll
  for (int m = 0; m < F::V; ++m) {
    const int k = F::pos(j, m);
    const C z = v[m];
    const C zc = cconj(j0 ? v[F::mirror_reg(m, true)] : v[F::mirror_reg(m, false)]);
    C s = cadd(z, zc), d = csub(z, zc);
    C t = cmulmi(cmul(twN[k], d));
    out(k, cmk<C>((Tp)0.5 * (s.x + t.x), (Tp)0.5 * (s.y + t.y)));
    if (m == 0 && j0) out(F::L, cmk<C>(z.x - z.y, (Tp)0));
  }
}

}  // namespace sles
