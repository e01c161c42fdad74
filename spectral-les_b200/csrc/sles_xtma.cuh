// X pass streamed through a TMA tile ring (3D; x-pass variant XV_TMA).
//
// Same arithmetic as k_xpass (sles_rhs.cuh): per work item (ky slice, chunk of
// W last-axis columns) the forward x-transforms of the slot fields, the kx
// part of div(tau), mask and projection, the integrator's stage update and the
// inverse x-transforms that prime the next evaluation.  What differs is how
// the data moves:
//  * every tile the item reads -- the slot fields, then per component the
//    state fields the stage needs (u_cur, u0, u1) -- is one TMA box
//    [x rows][W columns] at fixed ky, prefetched NBUF tiles ahead into a ring
//    of shared buffers completed on mbarriers (one elected thread issues,
//    bounded waits), as the y passes stream theirs;
//  * the three projected components wait in a shared stash [3][N][W] between
//    the forward transforms and the per-component update (kept in registers
//    they spill: the update and inverse transforms of one component run while
//    the other two wait);
//  * the state tiles of a component are read straight from the ring inside
//    the update loop, then released together.
// Stores (new state, primed slots) are plain 8/16-byte global stores, each
// warp writing whole 64-byte row segments.
//
// Tensor maps (4D, 8-byte elements): {nk*EPC columns, nsl ky rows, N x slices,
// slots}; box {W*EPC, 1, RB, 1}, so a box lands as [RB x][W] in shared memory
// (nsl = N, or N/P ky rows on a slab of a P-rank decomposition).
// The innermost coordinate is chunk*W*EPC elements = a multiple of 64 bytes.
#pragma once
#include "sles_rhs.cuh"

namespace sles {

template <typename Tp>
struct XTArgs {
  XArgs<Tp> a;
  CUtensorMap tws;   // workspace slots
  CUtensorMap tcur;  // u_cur (inverse-only items: the source u_inv)
  CUtensorMap t0;    // u0
  CUtensorMap t1;    // u1 (RK4 accumulator, ETD2 previous F1)
};

template <typename Tp, int N, class F>
struct XTGeo {
  using C = typename CT<Tp>::C;
  static constexpr int W = (sizeof(Tp) == 4) ? 4 : 2;  // 32-byte tile rows
  static constexpr int EPC = sizeof(C) / 8;
  static constexpr int T = F::T, V = F::V;
  static constexpr int THREADS = W * T;
  static constexpr int RB = N < 256 ? N : 256;  // rows per TMA box
  static constexpr int NBOX = N / RB;
  static constexpr int TE = N * W;
  static constexpr unsigned BOX_BYTES = RB * W * sizeof(C);
  static constexpr int SCR = F::XLEN * W;
  static constexpr int STASH = 3 * TE;  // projected components [3][N][W]
  static constexpr long long FIXED = 1024 + ((long long)STASH + SCR + F::LIN_LEN) * (long long)sizeof(C);
  // tile buffers that fit next to the scratch when `minb` blocks share an SM
  // (228 KB of shared memory per SM, 1 KB reserved per block)
  static constexpr long long nbuf_for(int minb) {
    return ((228LL / minb - 1) * 1024 - FIXED) / ((long long)TE * (long long)sizeof(C));
  }
  // blocks per SM: the most (4, 3, 2, 1) that keep at least 4 ring buffers
  static constexpr int MINB = (THREADS * 4 <= 1024 && nbuf_for(4) >= 4) ? 4
                              : ((THREADS * 3 <= 1024 && nbuf_for(3) >= 4) ? 3
                                 : ((THREADS * 2 <= 1024 && nbuf_for(2) >= 4) ? 2 : 1));
  static constexpr int NBUF = nbuf_for(MINB) > 6 ? 6 : (int)nbuf_for(MINB);
  static_assert(NBUF >= 4, "the ring must hold a component's state tiles plus lookahead");
  using Ring = TileRing<C, NBUF, TE>;
  static constexpr size_t SMEM = Ring::bytes() + ((size_t)STASH + SCR + F::LIN_LEN) * sizeof(C);
};

template <typename Tp, int N, class F, int LES, int ETD>
__global__ void __launch_bounds__(XTGeo<Tp, N, F>::THREADS, XTGeo<Tp, N, F>::MINB)
k_xpass_tma(const __grid_constant__ XTArgs<Tp> P) {
  using K = XTGeo<Tp, N, F>;
  using C = typename CT<Tp>::C;
  constexpr int T = K::T, V = K::V, W = K::W, D = 3;
  const XArgs<Tp>& A = P.a;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  typename K::Ring ring;
  const int tid = threadIdx.x;
  ring.init(smem_raw, tid);
  C* rst = reinterpret_cast<C*>(smem_raw + K::Ring::bytes());  // projected components [3][N][W]
  C* sm0 = rst + K::STASH;                                       // exchange scratch
  C* twt = sm0 + K::SCR;                                         // linear twiddle table
  F::fill_table_lin(twt);
  __syncthreads();
  const int l = tid % W, j = tid / W;
  F fft;
  const long long items = (long long)A.nmem * A.nsl * A.nchunks;
  const long long mine = (blockIdx.x < items) ? (items - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  constexpr int NTF = LES ? 6 : D;
  const int nst = A.need_uc + A.need_u0 + A.need_u1;
  const int TPI = A.fwd ? NTF + D * nst : D;
  const long long ntiles = mine * TPI;
  // tile `k` of an item's sequence: forward slots, then per component the state tiles
  auto issue = [&](long long t) {
    const long long it = blockIdx.x + (t / TPI) * (long long)gridDim.x;
    const int chunk = (int)(it % A.nchunks);
    const long long rest = it / A.nchunks;
    const int sl = (int)(rest % A.nsl), mem = (int)(rest / A.nsl);
    int k = (int)(t % TPI);
    const CUtensorMap* m = &P.tcur;
    int slot = k;
    if (A.fwd) {
      if (k < NTF) {
        m = &P.tws;
        slot = LES ? seq_slot<4>(k) : k;
      } else {
        k -= NTF;
        const int r = k % nst;
        slot = k / nst;
        int q = 0;
        m = &P.t1;
        if (A.need_uc) { if (r == q) m = &P.tcur; ++q; }
        if (A.need_u0 && m == &P.t1) { if (r == q) m = &P.t0; ++q; }
      }
    }
    // members follow one another along the x-slice axis of the maps
    ring.issue_rows(t, m, chunk * W * K::EPC, sl, mem * N, slot, K::NBOX, K::RB, K::BOX_BYTES);
  };
  if (tid == 0) {
    tma_prefetch_desc(&P.tws);
    tma_prefetch_desc(&P.tcur);
    for (long long t = 0; t < K::NBUF && t < ntiles; ++t) issue(t);
  }
  long long t = 0;
  // this thread's position in tile tt once it has landed
  auto wait_at = [&](long long tt) -> const C* {
    ring.wait(tt, A.err);
    return ring.tile(tt) + j * W + l;
  };
  // every thread is done with the next n tiles: refill their buffers
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
  const long long ps = (long long)A.nsl * A.nkp, fs = A.fs;  // x stride
  C* sm = sm0 + l;
  C* ws = A.ws;
  const StageCoef<Tp> SC = stage_coef<Tp>(A);
  auto kx_at = [&](int m) { return kc2c(j + T * m, N); };
  for (long long k = 0; k < mine; ++k) {  // persistent over work items
    const long long it = blockIdx.x + k * (long long)gridDim.x;
    const int chunk = (int)(it % A.nchunks);
    const long long rest = it / A.nchunks;
    const int sl = (int)(rest % A.nsl), mem = (int)(rest / A.nsl);
    const int col = chunk * W + l;
    const bool ok = col < A.nk;
    const long long base = (long long)mem * A.mstride + (long long)sl * A.nkp + col;
    const double nud = A.mnu ? A.mnu[mem] : A.nu_d;
    auto st = [&](int slot, const C (&v)[V]) {
      if (ok) {
#pragma unroll
        for (int m = 0; m < V; ++m) ws[slot * fs + base + (j + T * m) * ps] = v[m];
      }
    };
    // inverse x-transforms of component c of the new state (primes the next
    // evaluation); callers have just passed a block barrier (a tile release),
    // so the first transform skips its leading one
    auto prep = [&](int c, C (&s)[V]) {
      if (LES) {
        C b[V];
#pragma unroll
        for (int m = 0; m < V; ++m) b[m] = cmuli_s(s[m], (Tp)kx_at(m));  // i kx u_c
        fft.template run_tab<+1, true, 0, false>(b, j, sm, W, twt);
        st(D + c, b);
        fft.template run_tab<+1, true>(s, j, sm, W, twt);
      } else if (c >= 1) {
        C q[V];
        const Tp sg = (c == 2) ? (Tp)-1 : (Tp)1;  // -i kx w -> [3], i kx v -> [4]
#pragma unroll
        for (int m = 0; m < V; ++m) q[m] = cmuli_s(s[m], sg * (Tp)kx_at(m));
        fft.template run_tab<+1, true, 0, false>(q, j, sm, W, twt);
        st(c == 2 ? 3 : 4, q);
        fft.template run_tab<+1, true>(s, j, sm, W, twt);
      } else {
        fft.template run_tab<+1, true, 0, false>(s, j, sm, W, twt);
      }
      st(c, s);
    };
    if (!A.fwd) {
#pragma unroll 1
      for (int c = 0; c < D; ++c) {
        C v[V];
        take(v);
        prep(c, v);
      }
      continue;
    }
    // forward x-transforms; the x part of div(tau) joins in spectral space
    // (component loops not unrolled: each transform's code exists once)
    auto rpos = [&](int c, int m) { return c * K::TE + (j + T * m) * W + l; };
#pragma unroll 1
    for (int c = 0; c < D; ++c) {
      C v[V];
      take(v);
      fft.template run_tab<-1, true, 0, false>(v, j, sm, W, twt);
      if (LES) {  // + 2i kx F_cx
        C h[V];
        take(h);
        fft.template run_tab<-1, true, 0, false>(h, j, sm, W, twt);
#pragma unroll
        for (int m = 0; m < V; ++m) v[m] = cadd(v[m], cmuli_s(h[m], (Tp)(2 * kx_at(m))));
      }
#pragma unroll
      for (int m = 0; m < V; ++m) rst[rpos(c, m)] = v[m];
    }
    // mask + projection (each thread revisits only its own stash positions)
    const int kyv = kc2c(A.ky0 + sl, N);
#pragma unroll
    for (int m = 0; m < V; ++m) {
      C s3[D];
      int kv[D];
#pragma unroll
      for (int c = 0; c < D; ++c) s3[c] = rst[rpos(c, m)];
      kv[0] = kx_at(m);
      kv[1] = kyv;
      kv[2] = col;
      project<Tp, D>(A, s3, kv);
#pragma unroll
      for (int c = 0; c < D; ++c) rst[rpos(c, m)] = s3[c];
    }
    // per component: the stage update from the state tiles in the ring, then
    // the inverse transforms of the new state
#pragma unroll 1
    for (int c = 0; c < D; ++c) {
      const C* pu = nullptr;
      const C* p0 = nullptr;
      const C* p1 = nullptr;
      {
        long long tt = t;
        if (A.need_uc) pu = wait_at(tt++);
        if (A.need_u0) p0 = wait_at(tt++);
        if (A.need_u1) p1 = wait_at(tt++);
      }
      C v[V];
      if (ok) {
#pragma unroll
        for (int m = 0; m < V; ++m) {
          const long long off = base + (j + T * m) * ps;
          const int kx = kx_at(m);
          const int k2 = kx * kx + kyv * kyv + col * col;
          const C ucm = pu ? pu[T * m * W] : cmk<C>(0, 0);
          const C u0m = p0 ? p0[T * m * W] : ucm;
          const C u1m = p1 ? p1[T * m * W] : cmk<C>(0, 0);
          v[m] = update_component<Tp, ETD>(A, SC, c, rst[rpos(c, m)], ucm, u0m, u1m, k2, off, nud);
        }
      } else {
#pragma unroll
        for (int m = 0; m < V; ++m) v[m] = cmk<C>(0, 0);
      }
      release(nst);
      if (A.prep) prep(c, v);
    }
  }
}

}  // namespace sles
