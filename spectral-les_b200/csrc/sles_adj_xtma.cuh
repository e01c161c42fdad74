// Adjoint x pass streamed through a TMA tile ring (3D; the adjoint's form of
// the forward's x-pass variant 3, sles_xtma.cuh).
//
// Same arithmetic as k_adj_xpass (sles_adjoint.cuh): per work item (ky slice,
// chunk of W kz columns), the reverse stage's combine g_j = X(Y_j) - i kx
// X(A1_j) - nu K^2 lam_j [+ c lam_j], the scheme's update of acc / lam / ubar,
// then m = h mask P(lam) and the x-inverse priming of the next reverse stage.
// Every tile the item reads is one TMA box [x][W] at fixed ky, in the item's
// sequence
//   combine (fwd): per component c: Y_c, A1_c, lam_c [, ubar_c] [, acc_c]
//   prime only   : lam_0, lam_1, lam_2
//   priming      : unext_0, unext_1, unext_2
// prefetched NBUF tiles ahead into an mbarrier-completed ring (one elected
// thread issues; bounded waits); the state values of a component are read
// from the ring inside the update loop and their tiles released together.
// The cotangent of the next stage waits in a shared stash [3][N][W].
#pragma once
#include "sles_adjoint.cuh"
#include "sles_xtma.cuh"

namespace sles {

template <typename Tp>
struct AXTArgs {
  AXArgs<Tp> a;
  int need_ubar, need_acc;  // state tiles the update reads besides lam
  CUtensorMap tws;          // adjoint workspace slots
  CUtensorMap tlam, tubar, tacc, tunext;
};

template <typename Tp, int N, class F, int MODE>
__global__ void __launch_bounds__(XTGeo<Tp, N, F>::THREADS, XTGeo<Tp, N, F>::MINB)
k_adj_xpass_tma(const __grid_constant__ AXTArgs<Tp> P) {
  using K = XTGeo<Tp, N, F>;
  using C = typename CT<Tp>::C;
  constexpr int T = K::T, V = K::V, W = K::W;
  const AXArgs<Tp>& A = P.a;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  typename K::Ring ring;
  const int tid = threadIdx.x;
  ring.init(smem_raw, tid);
  C* rst = reinterpret_cast<C*>(smem_raw + K::Ring::bytes());  // [3][N][W] cotangent of the next stage
  C* sm0 = rst + K::STASH;
  C* twt = sm0 + K::SCR;
  F::fill_table_lin(twt);
  __syncthreads();
  const int l = tid % W, j = tid / W;
  F fft;
  const long long items = (long long)N * A.nchunks;
  const long long mine = (blockIdx.x < items) ? (items - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  const int nst = 1 + P.need_ubar + P.need_acc;  // lam [, ubar] [, acc]
  const int TPC = A.fwd ? 2 + nst : 1;             // tiles per component before the priming
  const int TPI = 3 * TPC + (A.prep ? 3 : 0);
  const long long ntiles = mine * TPI;
  auto issue = [&](long long t) {
    const long long it = blockIdx.x + (t / TPI) * (long long)gridDim.x;
    const int chunk = (int)(it % A.nchunks), sl = (int)(it / A.nchunks);
    const int k = (int)(t % TPI);
    const CUtensorMap* m;
    int slot;
    if (k >= 3 * TPC) {
      m = &P.tunext;
      slot = k - 3 * TPC;
    } else if (!A.fwd) {
      m = &P.tlam;
      slot = k;
    } else {
      const int c = k / TPC, r = k % TPC;
      slot = c;
      if (r == 0) m = &P.tws;
      else if (r == 1) { m = &P.tws; slot = 3 + c; }
      else if (r == 2) m = &P.tlam;
      else if (r == 3 && P.need_ubar) m = &P.tubar;
      else m = &P.tacc;
    }
    ring.issue_rows(t, m, chunk * W * K::EPC, sl, 0, slot, K::NBOX, K::RB, K::BOX_BYTES);
  };
  if (tid == 0) {
    tma_prefetch_desc(&P.tws);
    for (long long t = 0; t < K::NBUF && t < ntiles; ++t) issue(t);
  }
  long long t = 0;
  auto wait_at = [&](long long tt) -> const C* {
    ring.wait(tt, A.err);
    return ring.tile(tt) + j * W + l;
  };
  auto release = [&](int n) {
    __syncthreads();
    if (tid == 0)
      for (int i = 0; i < n; ++i)
        if (t + i + K::NBUF < ntiles) issue(t + i + K::NBUF);
    t += n;
  };
  auto take = [&](C (&v)[V]) {
    const C* p = wait_at(t);
#pragma unroll
    for (int m = 0; m < V; ++m) v[m] = p[T * m * W];
    release(1);
  };
  const long long ps = (long long)N * A.nkp, fs = A.fs;
  C* sm = sm0 + l;
  C* ws = A.ws;
  auto kx_at = [&](int m) { return kc2c(j + T * m, N); };
  auto rpos = [&](int c, int m) { return c * K::TE + (j + T * m) * W + l; };
  for (long long k = 0; k < mine; ++k) {  // persistent over work items
    const long long it = blockIdx.x + k * (long long)gridDim.x;
    const int chunk = (int)(it % A.nchunks);
    const int sl = (int)(it / A.nchunks);
    const int col = chunk * W + l;
    const bool ok = col < A.nk;
    const long long base = (long long)sl * A.nkp + col;
    const int kyv = kc2c(sl, N);
    auto st = [&](int slot, const C (&v)[V]) {
      if (ok) {
#pragma unroll
        for (int m = 0; m < V; ++m) ws[slot * fs + base + (j + T * m) * ps] = v[m];
      }
    };
    // inverse x-transforms of a field and of i kx times it into slots s0, s0 + 3
    // (after_release: a block barrier was just passed, the first transform
    // skips its leading one)
    auto inv2 = [&](C (&v)[V], int s0, bool after_release) {
      C b[V];
#pragma unroll
      for (int m = 0; m < V; ++m) b[m] = cmuli_s(v[m], (Tp)kx_at(m));
      if (after_release) fft.template run_tab<+1, true, 0, false>(b, j, sm, W, twt);
      else fft.template run_tab<+1, true>(b, j, sm, W, twt);
      st(s0 + 3, b);
      fft.template run_tab<+1, true>(v, j, sm, W, twt);
      st(s0, v);
    };
    if (A.fwd) {
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C v[V], h[V];
        take(v);
        fft.template run_tab<-1, true, 0, false>(v, j, sm, W, twt);
        take(h);
        fft.template run_tab<-1, true, 0, false>(h, j, sm, W, twt);
        const C* pl = wait_at(t);
        const C* pu = P.need_ubar ? wait_at(t + 1) : nullptr;
        const C* pa = P.need_acc ? wait_at(t + 1 + P.need_ubar) : nullptr;
#pragma unroll
        for (int m = 0; m < V; ++m) {
          C g = cadd(v[m], cmuli_s(h[m], -(Tp)kx_at(m)));  // - i kx X(A1_c)
          C ln = cmk<C>(0, 0);
          if (ok) {
            const long long o = c * fs + base + (j + T * m) * ps;
            const int kx = kx_at(m);
            const int k2 = kx * kx + kyv * kyv + col * col;
            const C lc = pl[T * m * W];
            if constexpr (MODE != 2) g = csub(g, cscale(lc, A.nu * (Tp)k2));
            if (A.forcing > (Tp)0 && k2 != 0) g = cadd(g, cscale(lc, A.forcing));
            if constexpr (MODE == 2) {
              const C ub = pu[T * m * W];
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
              const C ac = pa[T * m * W];
              if (A.last) {
                const C w = cadd(ac, g);
                A.ubar[o] = w;
                A.acc[o] = cscale(w, A.pa);
                ln = cscale(w, A.pl);
              } else {
                const C w = cadd(cscale(pu[T * m * W], A.pu), g);
                A.acc[o] = cadd(ac, cscale(w, A.pa));
                A.ubar[o] = cscale(w, A.pb);
                ln = cscale(w, A.pl);
              }
            } else {
              const C an = cadd(pa[T * m * W], g);
              A.acc[o] = an;
              if (A.last) {
                A.ubar[o] = an;
                ln = cscale(an, A.alpha);
              } else {
                ln = cadd(cscale(pu[T * m * W], A.alpha), cscale(g, A.beta));
              }
            }
            A.lam[o] = ln;
          }
          rst[rpos(c, m)] = ln;
        }
        release(nst);
      }
      if (!A.prep) continue;
    } else {
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        C v[V];
        take(v);
#pragma unroll
        for (int m = 0; m < V; ++m) rst[rpos(c, m)] = ok ? v[m] : cmk<C>(0, 0);
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
      take(v);
      inv2(v, c, true);
#pragma unroll
      for (int m = 0; m < V; ++m) v[m] = rst[rpos(c, m)];
      inv2(v, 9 + c, false);
    }
  }
}

}  // namespace sles
