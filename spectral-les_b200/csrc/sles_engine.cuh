// Host-side engine: launch sequences for one (precision, N, dim) triple.
// One instantiation per grid size lives in sles_n<N>.cu so the sizes compile
// in parallel; sles_api.cu dispatches to them through the Engine interface.
#pragma once
#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <mutex>
#include <type_traits>
#include <unordered_map>
#include <unordered_set>

#include "../../include/sles.h"
#include "sles_misc.cuh"
#include "sles_passes.cuh"
#include "sles_rhs.cuh"
#include "sles_xtma.cuh"
#include "sles_adjoint.cuh"
#include "sles_adj_xtma.cuh"

namespace sles {

struct PlanInfo {
  sles_plan_desc d;
  int nkp, nk;
  long long hc_elems, real_elems;
  size_t elem_bytes;     // bytes of one complex element
  void* ws;              // workspace base (device)
  size_t ws_bytes;
  int ws_fields;         // half-complex field slots in the workspace
  unsigned* flags;       // device error word inside the workspace
  double* scal;          // device scalar scratch inside the workspace (64 doubles)
  int xvar;              // x-pass variant (XGeo), set by default or by the autotuner
  int yvar, zvar;        // y- and z-pass variants (tile width, lines per work item)
  int axvar;             // adjoint x pass: 0 direct loads, 1 TMA tile ring
  // slab decomposition over P ranks (3D): this rank holds ky rows [r*m, (r+1)*m)
  // of spectral fields and x planes [r*m, (r+1)*m) of physical ones (m = N/P);
  // P = 1, m = N: the whole grid
  int slab_p, slab_r, slab_m;
  int slab_n1, slab_n2;  // fields of the two exchanges (x-inverse outputs, y-forward outputs)
  // ensemble batch: nmem members of this plan's grid stepped together; every
  // field holds the members one after another (hc_elems counts all of them)
  int nmem;
  const double* mnu;     // per-member nu (device), or null
  const double* mcs;     // per-member C_s (device), or null
};

// workspace header: error word + scalar scratch, then the diagnostics area,
// then the field slots (256-byte aligned)
constexpr size_t WS_HEADER = 4096;
inline int max_shell(int dim, int n) { return (int)(0.5 * n * (dim == 3 ? 1.7320508075688772 : 1.4142135623730951)) + 3; }
inline size_t diag_area_bytes(int dim, int n) {
  return ((size_t)DIAG_BLOCKS * (2 + max_shell(dim, n)) + DIAG_BLOCKS) * sizeof(double);
}
inline size_t slots_offset(int dim, int n) { return ((WS_HEADER + diag_area_bytes(dim, n)) + 255) / 256 * 256; }

struct Engine {
  virtual ~Engine() {}
  virtual int ws_fields_needed(const PlanInfo& p) const = 0;
  virtual int default_xvar() const = 0;
  virtual int variant_count(int pass) const = 0;  // SLES_PASS_X / _Y / _Z / _AX
  virtual int fft_r2c(PlanInfo& p, const void* in, void* out, int nf, cudaStream_t st) = 0;
  virtual int fft_c2r(PlanInfo& p, const void* in, void* out, int nf, cudaStream_t st) = 0;
  virtual int velocity_curl(PlanInfo& p, const void* uh, void* u, void* curl, cudaStream_t st) = 0;
  virtual int velocity_gradient(PlanInfo& p, const void* uh, void* grad, cudaStream_t st) = 0;
  virtual int rhs(PlanInfo& p, const void* uh, const void* uphys, const void* cphys, void* du, void* f1,
                  cudaStream_t st) = 0;
  virtual int stage(PlanInfo& p, int stage, double dt, const void* ucur, const void* u0, void* u1,
                    void* uout, void* aux, const void* uphys, const void* cphys, int flags,
                    cudaStream_t st, sles_dtctl* ctl = nullptr, int parity = 0) = 0;
  virtual int diag(PlanInfo& p, const void* uh, const void* uphys, double* out, double* spec, int nshell,
                   cudaStream_t st) = 0;
  virtual int profile_rhs(PlanInfo& p, const void* uh, void* du, int iters, double* ms, cudaStream_t st) = 0;
  // discrete adjoint (3D): workspace slots, seed, prime, one reverse RK4 stage
  virtual int adjoint_fields() const = 0;
  virtual int adjoint_seed(PlanInfo& pa, double dt, const void* ubar, void* acc, void* lam, cudaStream_t st) = 0;
  virtual int adjoint_prime(PlanInfo& pa, const void* u_state, const void* lam, cudaStream_t st) = 0;
  virtual int adjoint_stage(PlanInfo& pa, int s, double dt, const void* unext, void* ubar, void* acc, void* lam,
                            double* csgrad, cudaStream_t st) = 0;
  // slab decomposition (3D): exchange field counts, and the three pass groups
  // around the two exchanges of one RHS evaluation
  virtual int slab_counts(const PlanInfo& p, int* n1, int* n2) const = 0;
  virtual int slab_prime(PlanInfo& p, const void* u, cudaStream_t st) = 0;
  virtual int slab_middle(PlanInfo& p, unsigned long long* umax, cudaStream_t st) = 0;
  virtual int slab_stage(PlanInfo& p, int stage, double dt, const void* ucur, const void* u0, void* u1, void* uout,
                         void* aux, int flags, cudaStream_t st) = 0;
};

inline int cuda_status(cudaError_t e) { return e == cudaSuccess ? SLES_OK : SLES_ERR_CUDA; }

// Raise the dynamic shared-memory limit of a kernel once, then launch.
template <typename... KArgs, typename... Args>
inline int launch(void (*kern)(KArgs...), long long grid, int block, size_t smem, cudaStream_t st,
                  Args... args) {
  if (grid <= 0) return SLES_OK;
  if (grid > 0x7fffffffLL) return SLES_ERR_UNSUPPORTED;
  if (smem > 48 * 1024) {
    static std::mutex mu;
    static std::unordered_set<const void*> done;
    std::lock_guard<std::mutex> g(mu);
    if (!done.count((const void*)kern)) {
      cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return SLES_ERR_CUDA;
      done.insert((const void*)kern);
    }
  }
  kern<<<(unsigned)grid, block, smem, st>>>(static_cast<KArgs>(args)...);
  return cuda_status(cudaGetLastError());
}

// Persistent launch: `work` block-sized work units, grid capped at the number
// of blocks that can be resident at once (kernels loop over their units).
template <typename... KArgs, typename... Args>
inline int launch_persistent(void (*kern)(KArgs...), long long work, int block, size_t smem, cudaStream_t st,
                             Args... args) {
  if (work <= 0) return SLES_OK;
  static std::mutex mu;
  static std::unordered_map<const void*, int> cache;
  int resident = 0;
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find((const void*)kern);
    if (it != cache.end()) {
      resident = it->second;
    } else {
      if (smem > 48 * 1024 &&
          cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return SLES_ERR_CUDA;
      int dev = 0, nsm = 0, per = 0;
      if (cudaGetDevice(&dev) != cudaSuccess) return SLES_ERR_CUDA;
      if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return SLES_ERR_CUDA;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, block, smem) != cudaSuccess) return SLES_ERR_CUDA;
      if (per < 1) return SLES_ERR_UNSUPPORTED;
      resident = per * nsm;
      cache[(const void*)kern] = resident;
    }
  }
  const long long grid = work < resident ? work : resident;
  kern<<<(unsigned)grid, block, smem, st>>>(static_cast<KArgs>(args)...);
  return cuda_status(cudaGetLastError());
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
inline PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  });
  return fn;
}

// 4D tile map over half-complex fields as 8-byte elements:
// {nk*epc columns, rows, slices, slots}; box {box_cols*epc, box_rows, 1, 1}
inline int make_tmap(CUtensorMap* m, const void* base, int epc, int nk, long long rows, long long row_stride_b,
                     long long slices, long long slice_stride_b, long long nslot, long long slot_stride_b,
                     int box_cols, int box_rows) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = tmap_encoder();
  if (!fn) return SLES_ERR_CUDA;
  cuuint64_t dims[4] = {(cuuint64_t)nk * epc, (cuuint64_t)rows, (cuuint64_t)slices, (cuuint64_t)nslot};
  cuuint64_t strides[3] = {(cuuint64_t)row_stride_b, (cuuint64_t)slice_stride_b, (cuuint64_t)slot_stride_b};
  cuuint32_t box[4] = {(cuuint32_t)(box_cols * epc), (cuuint32_t)box_rows, 1, 1};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? SLES_OK : SLES_ERR_CUDA;
}

// the same map with box {box_cols*epc, box1, box2, 1}
inline int make_tmap_box(CUtensorMap* m, const void* base, int epc, int nk, long long rows, long long row_stride_b,
                         long long slices, long long slice_stride_b, long long nslot, long long slot_stride_b,
                         int box_cols, int box1, int box2) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = tmap_encoder();
  if (!fn) return SLES_ERR_CUDA;
  cuuint64_t dims[4] = {(cuuint64_t)nk * epc, (cuuint64_t)rows, (cuuint64_t)slices, (cuuint64_t)nslot};
  cuuint64_t strides[3] = {(cuuint64_t)row_stride_b, (cuuint64_t)slice_stride_b, (cuuint64_t)slot_stride_b};
  cuuint32_t box[4] = {(cuuint32_t)(box_cols * epc), (cuuint32_t)box1, (cuuint32_t)box2, 1};
  cuuint32_t es[4] = {1, 1, 1, 1};
  CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4, const_cast<void*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? SLES_OK : SLES_ERR_CUDA;
}

// 5D map over a slab exchange buffer [fields][P blocks][m x planes][m rows][nkp]:
// dims {nk*epc, m rows, m planes, P blocks, fields}; box {box_cols*epc, m, 1, P, 1}
// (one whole line of N = P*m rows, landing as [P][m][cols] = [rows][cols])
inline int make_tmap_split(CUtensorMap* mp, const void* base, int epc, int nk, int nkp, long long m, long long P,
                           long long nfields, long long field_stride_b, int elem_b, int box_cols) {
  PFN_cuTensorMapEncodeTiled_v12000 fn = tmap_encoder();
  if (!fn) return SLES_ERR_CUDA;
  const long long row_b = (long long)nkp * elem_b;
  cuuint64_t dims[5] = {(cuuint64_t)nk * epc, (cuuint64_t)m, (cuuint64_t)m, (cuuint64_t)P, (cuuint64_t)nfields};
  cuuint64_t strides[4] = {(cuuint64_t)row_b, (cuuint64_t)(m * row_b), (cuuint64_t)(m * m * row_b),
                           (cuuint64_t)field_stride_b};
  cuuint32_t box[5] = {(cuuint32_t)(box_cols * epc), (cuuint32_t)m, 1, (cuuint32_t)P, 1};
  cuuint32_t es[5] = {1, 1, 1, 1, 1};
  CUresult r = fn(mp, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 5, const_cast<void*>(base), dims, strides, box, es,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? SLES_OK : SLES_ERR_CUDA;
}

#define SLES_TRY(x)              \
  do {                           \
    int _s = (x);                \
    if (_s != SLES_OK) return _s; \
  } while (0)

// columns per c2c work item: 64-byte row segments
template <typename Tp> struct Cols { static constexpr int W = (sizeof(Tp) == 4) ? 8 : 4; };

template <typename Tp, int N>
struct Geo {
  static constexpr int W = Cols<Tp>::W;
  static constexpr int T = PlanFor<Tp, N>::F::T;
  static constexpr int G = (W * T >= 256) ? 1 : 256 / (W * T);
  static constexpr int TR = PlanFor<Tp, N / 2>::F::T;
  static constexpr int LPB = (TR >= 128) ? 1 : 128 / TR;
};

// ---------------------------------------------------------------------------
// standalone transforms
// ---------------------------------------------------------------------------
template <typename Tp, int N, int DIM>
struct Transforms {
  using C = typename CT<Tp>::C;
  using G = Geo<Tp, N>;

  // c2c along axis `ax` (0 = x, 1 = y; 2D: ax 0 only) of nf fields
  template <int DIR>
  static int c2c(const PlanInfo& p, const C* src, C* dst, int nf, int ax, Tp scale, cudaStream_t st) {
    using K = C2CAxis<Tp, N, G::W, G::G>;
    const long long fs = p.hc_elems;
    const int nchunks = (p.nk + G::W - 1) / G::W;
    int na;
    long long astride, pstride;
    if (DIM == 3) {
      na = N;
      if (ax == 0) { astride = p.nkp; pstride = (long long)N * p.nkp; }
      else { astride = (long long)N * p.nkp; pstride = p.nkp; }
    } else {
      na = 1; astride = 0; pstride = p.nkp;
    }
    const long long items = (long long)nf * na * nchunks;
    return launch_persistent(k_c2c_axis<Tp, N, G::W, G::G, DIR>, (items + G::G - 1) / G::G, K::THREADS, K::SMEM, st,
                  src, dst, fs, nf, na, astride, pstride, p.nk, nchunks, scale);
  }

  static int r2c_lines(const PlanInfo& p, const Tp* src, C* dst, int nf, cudaStream_t st) {
    using K = RealAxis<Tp, N, G::LPB>;
    const long long nlines = (long long)nf * (DIM == 3 ? (long long)N * N : N);
    return launch_persistent(k_r2c_line<Tp, N, G::LPB>, (nlines + G::LPB - 1) / G::LPB, K::THREADS, K::SMEM, st, src,
                  dst, nlines, p.nkp);
  }

  static int c2r_lines(const PlanInfo& p, const C* src, Tp* dst, int nf, Tp scale, cudaStream_t st) {
    using K = RealAxis<Tp, N, G::LPB>;
    const long long nlines = (long long)nf * (DIM == 3 ? (long long)N * N : N);
    return launch_persistent(k_c2r_line<Tp, N, G::LPB>, (nlines + G::LPB - 1) / G::LPB, K::THREADS, K::SMEM, st, src,
                  dst, nlines, p.nkp, scale);
  }

  static int r2c(const PlanInfo& p, const Tp* in, C* out, int nf, cudaStream_t st) {
    SLES_TRY(r2c_lines(p, in, out, nf, st));
    if (DIM == 3) SLES_TRY(c2c<-1>(p, out, out, nf, 1, (Tp)1, st));
    return c2c<-1>(p, out, out, nf, 0, (Tp)1, st);
  }

  // c2r of nf fields through `tmp` (nf half-complex slots); `in` is preserved
  static int c2r(const PlanInfo& p, const C* in, Tp* out, int nf, C* tmp, cudaStream_t st) {
    const Tp scale = (Tp)(1.0 / ((DIM == 3) ? (double)N * N * N : (double)N * N));
    SLES_TRY(c2c<+1>(p, in, tmp, nf, 0, (Tp)1, st));
    if (DIM == 3) SLES_TRY(c2c<+1>(p, tmp, tmp, nf, 1, (Tp)1, st));
    return c2r_lines(p, tmp, out, nf, scale, st);
  }
};

}  // namespace sles

namespace sles {

enum { STAGE_RECORD_F1 = 1, STAGE_PRIMED = 2, STAGE_NO_PREPARE = 4, STAGE_RK4 = 8 };

constexpr int cmax(int a, int b) { return a > b ? a : b; }

template <typename Tp, int N, int DIM>
struct EngineImpl final : Engine {
  using C = typename CT<Tp>::C;
  using TR = Transforms<Tp, N, DIM>;
#ifndef SLES_X_PADD
#define SLES_X_PADD 16
#endif
  // x pass: exchange padding divisor SLES_X_PADD (0: the plan's first radix)
  using FX = typename WithPad<typename PlanLo<Tp, N>::F, SLES_X_PADD>::F;
  // per x-pass variant: the 32-byte-row tiles (XV 2) pad the exchange every 8 points
  template <int XV>
  using FXV = typename WithPad<typename PlanLo<Tp, N>::F, XV == 2 ? 8 : SLES_X_PADD>::F;
  // y-pass FFT plans per direction: PlanFor (more points per thread) or PlanLo.
  // At N = 512 in FP32 the LES inverse pass (6 inputs, 128-byte rows) runs
  // fastest on PlanFor (32 threads per line), the LES forward pass (9 inputs)
  // and the passes without LES on PlanLo (64).
#ifndef SLES_YI_PLANFOR
#define SLES_YI_PLANFOR -1
#endif
#ifndef SLES_YF_PLANFOR
#define SLES_YF_PLANFOR 0
#endif
  template <int LES>
  using FYI = typename std::conditional<(SLES_YI_PLANFOR >= 0 ? SLES_YI_PLANFOR != 0
                                                              : (N == 512 && sizeof(Tp) == 4 && LES != 0)),
                                        typename PlanFor<Tp, N>::F, typename PlanLo<Tp, N>::F>::type;
  using FYF = typename std::conditional<SLES_YF_PLANFOR != 0, typename PlanFor<Tp, N>::F,
                                        typename PlanLo<Tp, N>::F>::type;
  template <int LES>
  using YGeoI = TGeo<Tp, N, FYI<LES>, true, 0, LES>;
  template <int LES>
  using YGeoF = TGeo<Tp, N, FYF, true, 0, LES>;
  static constexpr int TZ = PlanFor<Tp, N / 2>::F::T;
#ifndef SLES_Z_LPI
#define SLES_Z_LPI 0
#endif
  // z lines per work item: 8 threads' worth of lines (one line of 8 or more
  // threads); at 256^3 one line per item ran the z pass 13% faster than two,
  // at 128^3 7%, at 64^3 two and four were equal.  SLES_Z_LPI > 0 overrides.
  static constexpr int LPI = SLES_Z_LPI > 0 ? SLES_Z_LPI : cmax(1, 8 / TZ);

  static C* slot(const PlanInfo& p, int i) {
    return reinterpret_cast<C*>(reinterpret_cast<char*>(p.ws) + slots_offset(DIM, N)) + (long long)i * p.hc_elems;
  }
  template <int XV>
  static int xchunks(const PlanInfo& p) {  // x-pass column chunks of variant XV
    constexpr int WX = XGeo<Tp, N, FXV<XV>, DIM, XV>::W;
    return (p.nk + WX - 1) / WX;
  }
  // x-pass variant used until a caller (the autotuner) sets another: the
  // fastest in a timing sweep of every size on a B200 (RK3 Smagorinsky and
  // RK4 without LES; see sles/autotune.py)
  int variant_count(int pass) const override {
    if (pass == 0) return X_VARIANTS;
    if (pass == 1) return HAS_YVAR ? 2 : 1;
    if (pass == 2) return HAS_ZVAR ? 2 : 1;
    if (pass == 3) return HAS_XTMA ? 2 : 1;
    return 0;
  }
  int default_xvar() const override {
    if (sizeof(Tp) == 8) return (DIM == 2 && N >= 1024) ? 0 : (DIM == 2 ? 2 : 1);
    if (DIM == 2) return 2;
    if (N <= 64) return 1;
    if (N == 256 || N == 512) return 3;  // the TMA-ring x pass: 4.28 vs 4.72 ms/step at 256^3, 39.0 vs 43.2 at 512^3
    return N == 128 ? 2 : 0;
  }
  template <int LES>
  static int ychunks(const PlanInfo& p) {                                 // y-pass column chunks
    constexpr int WY = YGeoI<LES>::W;
    static_assert(YGeoF<LES>::W == WY, "one tile width for both y directions");
    return (p.nk + WY - 1) / WY;
  }

  int ws_fields_needed(const PlanInfo& p) const override {
    const bool les = p.d.les_model != SLES_LES_NONE;
    if (DIM == 3) return les ? 9 : 6;
    return les ? 5 : 3;
  }

  // ---------------- standalone transforms ----------------
  int fft_r2c(PlanInfo& p, const void* in, void* out, int nf, cudaStream_t st) override {
    return TR::r2c(p, (const Tp*)in, (C*)out, nf, st);
  }
  int fft_c2r(PlanInfo& p, const void* in, void* out, int nf, cudaStream_t st) override {
    const int cap = p.ws_fields;
    for (int f0 = 0; f0 < nf; f0 += cap) {
      const int n = (nf - f0 < cap) ? nf - f0 : cap;
      SLES_TRY(TR::c2r(p, (const C*)in + (long long)f0 * p.hc_elems, (Tp*)out + (long long)f0 * p.real_elems, n,
                       slot(p, 0), st));
    }
    return SLES_OK;
  }
  int velocity_curl(PlanInfo& p, const void* uh, void* u, void* curl, cudaStream_t st) override {
    if (u) SLES_TRY(fft_c2r(p, uh, u, DIM, st));
    if (curl) {
      const int nc = DIM == 3 ? 3 : 1;
      SLES_TRY(launch(k_curl_hat<Tp, DIM>, 1184, 256, 0, st, (const C*)uh, slot(p, 0), p.hc_elems, N, p.nkp, p.nk));
      SLES_TRY(TR::c2r(p, slot(p, 0), (Tp*)curl, nc, slot(p, 0), st));
    }
    return SLES_OK;
  }
  int velocity_gradient(PlanInfo& p, const void* uh, void* grad, cudaStream_t st) override {
    for (int i = 0; i < DIM; ++i) {
      SLES_TRY(launch(k_deriv_hat<Tp, DIM>, 1184, 256, 0, st, (const C*)uh, slot(p, 0), p.hc_elems, N, p.nkp, p.nk, i));
      SLES_TRY(TR::c2r(p, slot(p, 0), (Tp*)grad + (long long)i * DIM * p.real_elems, DIM, slot(p, 0), st));
    }
    return SLES_OK;
  }

  // ---------------- fused passes ----------------
  XArgs<Tp> xbase(const PlanInfo& p) const {
    XArgs<Tp> a{};
    a.ws = slot(p, 0);
    a.fs = p.hc_elems;
    a.nkp = p.nkp;
    a.nk = p.nk;
    a.nu = (Tp)p.d.nu;
    a.forcing = (Tp)p.d.forcing;
    a.kmax = 2.0 / 3.0 * (double)(N / 2 + 1);  // initialize_domain.py:79
    a.nu_d = p.d.nu;
    a.nsl = p.slab_m;
    a.ky0 = p.slab_r * p.slab_m;
    a.nmem = p.nmem;
    a.mstride = p.hc_elems / p.nmem;
    a.mnu = p.mnu;
    return a;
  }

  template <int LES, int PAR2D>
  int xpass(const PlanInfo& p, XArgs<Tp> a, cudaStream_t st) {
    switch (p.xvar) {
      case 1: return xpass_v<LES, PAR2D, 1>(p, a, st);
      case 2: return xpass_v<LES, PAR2D, 2>(p, a, st);
      case 3: return xpass_tma<LES, PAR2D>(p, a, st);
      default: return xpass_v<LES, PAR2D, 0>(p, a, st);
    }
  }
  // state tiles a stage reads (u_cur for viscous/forcing/update; u0 when
  // distinct from u_cur; u1 = RK4 accumulator or ETD2's previous F1)
  static void set_needs(XArgs<Tp>& a) {
    a.need_uc = a.need_u0 = a.need_u1 = 0;
    if (a.fwd && a.kind != KX_RAW) {
      a.need_uc = 1;
      const bool uses_u0 = a.kind == KX_RK4 ? a.stage < 3 : (a.kind == KX_RK3P || a.kind == KX_SSP3);
      a.need_u0 = (uses_u0 && a.u0 != a.ucur) ? 1 : 0;
      a.need_u1 = (a.kind == KX_RK4 || a.kind == KX_ETD2P || a.kind == KX_ETD2C) ? 1 : 0;
    }
  }
  // x-pass variant XV_TMA (sles_xtma.cuh): compiled for the 3D grids 128, 256
  // and 512; elsewhere the variant runs as variant 0
  static constexpr bool HAS_XTMA = DIM == 3 && (N == 128 || N == 256 || N == 512);
  template <int LES, int PAR2D>
  int xpass_tma(const PlanInfo& p, XArgs<Tp> a, cudaStream_t st) {
    if constexpr (!HAS_XTMA) {
      return xpass_v<LES, PAR2D, 0>(p, a, st);
    } else {
      using F = FXV<2>;  // 32-byte tile rows: the exchange padded every 8 points, as variant 2
      using K = XTGeo<Tp, N, F>;
      XTArgs<Tp> P{};
      a.nchunks = (p.nk + K::W - 1) / K::W;
      set_needs(a);
      a.err = p.flags;
      P.a = a;
      const long long cb = sizeof(C), row = (long long)p.nkp * cb, slice = (long long)a.nsl * p.nkp * cb;
      const long long fsb = p.hc_elems * cb;
      // {columns, ky rows, x slices, slots}; box {W columns, 1 ky row, RB x rows, 1 slot}
      auto mk = [&](CUtensorMap* m, const void* base, long long nslot) {
        return make_tmap_box(m, base, K::EPC, p.nk, a.nsl, row, (long long)p.nmem * N, slice, nslot, fsb, K::W, 1,
                             K::RB);
      };
      SLES_TRY(mk(&P.tws, slot(p, 0), p.ws_fields));
      const void* cur = a.fwd ? (const void*)a.ucur : (const void*)a.uinv;
      SLES_TRY(mk(&P.tcur, cur ? cur : slot(p, 0), 3));
      SLES_TRY(mk(&P.t0, a.need_u0 ? (const void*)a.u0 : slot(p, 0), 3));
      SLES_TRY(mk(&P.t1, a.need_u1 ? (const void*)a.u1 : slot(p, 0), 3));
      const long long items = (long long)a.nmem * a.nsl * a.nchunks;
      if (a.kind == KX_ETD2P || a.kind == KX_ETD2C) {
        if (LES) return launch_persistent(k_xpass_tma<Tp, N, F, 1, 1>, items, K::THREADS, K::SMEM, st, P);
        return launch_persistent(k_xpass_tma<Tp, N, F, 0, 1>, items, K::THREADS, K::SMEM, st, P);
      }
      if (LES) return launch_persistent(k_xpass_tma<Tp, N, F, 1, 0>, items, K::THREADS, K::SMEM, st, P);
      return launch_persistent(k_xpass_tma<Tp, N, F, 0, 0>, items, K::THREADS, K::SMEM, st, P);
    }
  }
  template <int LES, int PAR2D, int XV>
  int xpass_v(const PlanInfo& p, XArgs<Tp> a, cudaStream_t st) {
    using K = XGeo<Tp, N, FXV<XV>, DIM, XV>;
    a.nchunks = xchunks<XV>(p);
    set_needs(a);
    a.err = p.flags;
    const long long items = (long long)a.nmem * (DIM == 3 ? a.nsl : 1) * a.nchunks;
    if (a.kind == KX_ETD2P || a.kind == KX_ETD2C)
      return launch_persistent(k_xpass<Tp, N, FXV<XV>, DIM, LES, PAR2D, 1, XV>, items, K::THREADS, K::SMEM, st, a);
    return launch_persistent(k_xpass<Tp, N, FXV<XV>, DIM, LES, PAR2D, 0, XV>, items, K::THREADS, K::SMEM, st, a);
  }
  int xpass_rt(const PlanInfo& p, const XArgs<Tp>& a, int les, int par2d, cudaStream_t st) {
    if (!les) return xpass<0, 0>(p, a, st);
    if (DIM == 2 && par2d) return xpass<1, 1>(p, a, st);
    return xpass<1, 0>(p, a, st);
  }

  // slab exchange buffers inside the workspace (after the pass slots): the
  // x-inverse outputs go out from slots [0, n1) and arrive in `recv1`; the
  // y-forward outputs go out from `send2` and arrive in slots [0, n2)
  static int pass_slots(const PlanInfo& p) { return p.ws_fields - p.slab_n1 - p.slab_n2; }
  static C* slab_recv1(const PlanInfo& p) { return slot(p, pass_slots(p)); }
  static C* slab_send2(const PlanInfo& p) { return slot(p, pass_slots(p) + p.slab_n1); }

  // y-pass variant 1 (float32 3D grids 128, 256, 512): the other tile width
  // (8 <-> 16 columns); elsewhere one variant
  static constexpr bool HAS_YVAR = sizeof(Tp) == 4 && DIM == 3 && (N == 128 || N == 256 || N == 512);
  template <int LES>
  static constexpr int yw_alt() { return YGeoI<LES>::W == 8 ? 16 : 8; }

  // split: on a slab (P > 1 or an explicit exchange), the inverse pass reads the
  // exchange buffer and the forward pass stores into the outgoing one
  template <int LES>
  int ypass(const PlanInfo& p, int inv, cudaStream_t st, bool split = false) {
    if constexpr (DIM != 3) {
      return SLES_OK;
    } else {
      if constexpr (HAS_YVAR) {
        if (p.yvar == 1 && !split) return ypass_w<LES, yw_alt<LES>()>(p, inv, st, false);
      }
      return ypass_w<LES, 0>(p, inv, st, split);
    }
  }
  template <int LES, int YW>
  int ypass_w(const PlanInfo& p, int inv, cudaStream_t st, bool split) {
    using K = TGeo<Tp, N, FYI<LES>, true, 0, LES, YW>;  // tile geometry (the tensor map) shared by both plans
    using KF = TGeo<Tp, N, FYF, true, 0, LES, YW>;
    static_assert(K::W == KF::W, "one tile width for both y directions");
    YArgs<Tp> a{};
    const long long cb = sizeof(C);
    const int M = p.slab_m * p.nmem;  // x planes held: a slab's, or every batched member's
    if (split && inv) {
      SLES_TRY(make_tmap_split(&a.tm, slab_recv1(p), K::EPC, p.nk, p.nkp, M, p.slab_p, p.slab_n1, p.hc_elems * cb,
                               (int)cb, K::W));
    } else {
      SLES_TRY(make_tmap(&a.tm, slot(p, 0), K::EPC, p.nk, N, (long long)p.nkp * cb, M, (long long)N * p.nkp * cb,
                         pass_slots(p), p.hc_elems * cb, K::W, K::RB));
    }
    a.err = p.flags;
    a.ws = slot(p, 0);
    a.out = (split && !inv) ? slab_send2(p) : slot(p, 0);
    a.split = split ? 1 : 0;
    a.m = M;
    a.nx = M;
    a.fs = p.hc_elems;
    a.nkp = p.nkp;
    a.nk = p.nk;
    a.nchunks = (p.nk + K::W - 1) / K::W;
    const long long items = (long long)M * a.nchunks;
    if (split) {
      if (inv) return launch_persistent(k_ypass<Tp, N, FYI<LES>, LES, 1, 0, 1, YW>, items, K::THREADS, K::SMEM, st, a);
      return launch_persistent(k_ypass<Tp, N, FYF, LES, 0, 0, 1, YW>, items, KF::THREADS, KF::SMEM, st, a);
    }
    if (inv) return launch_persistent(k_ypass<Tp, N, FYI<LES>, LES, 1, 0, 0, YW>, items, K::THREADS, K::SMEM, st, a);
    return launch_persistent(k_ypass<Tp, N, FYF, LES, 0, 0, 0, YW>, items, KF::THREADS, KF::SMEM, st, a);
  }

  // z-pass variant 1 (float32 3D grids 128, 256, 512): twice the z lines per work item
  static constexpr bool HAS_ZVAR = sizeof(Tp) == 4 && DIM == 3 && (N == 128 || N == 256 || N == 512);
  template <int LES, int MODEL, int PAR2D>
  int zpass(const PlanInfo& p, const Tp* uphys, const Tp* cphys, int stress_only, cudaStream_t st,
            unsigned long long* umax) {
    if constexpr (HAS_ZVAR) {
      if (p.zvar == 1) return zpass_l<LES, MODEL, PAR2D, 2 * LPI>(p, uphys, cphys, stress_only, st, umax);
    }
    return zpass_l<LES, MODEL, PAR2D, LPI>(p, uphys, cphys, stress_only, st, umax);
  }

  template <int LES, int MODEL, int PAR2D, int ZL>
  int zpass_l(const PlanInfo& p, const Tp* uphys, const Tp* cphys, int stress_only, cudaStream_t st,
              unsigned long long* umax) {
    using K = ZGeo<Tp, N, DIM, LES, PAR2D, ZL>;
    ZArgs<Tp> a{};
    a.ws = slot(p, 0);
    a.fs = p.hc_elems;
    a.nkp = p.nkp;
    a.lpm = (DIM == 3) ? (long long)p.slab_m * N : N;
    a.nlines = a.lpm * p.nmem;
    a.mcs = p.mcs;
    a.dx = 2.0 * 3.141592653589793 / N;
    a.vreman = MODEL == M_VREMAN ? 1 : 0;
    a.scale = (Tp)(1.0 / (DIM == 3 ? (double)N * N * N : (double)N * N));
    const double dx = 2.0 * 3.141592653589793 / N;  // initialize_domain.py:42
    if (MODEL == M_SMAG) a.cdx2 = (Tp)((p.d.cs * dx) * (p.d.cs * dx));
    else a.cdx2 = (Tp)(2.5 * p.d.cs * p.d.cs * dx * dx);
    a.uphys = uphys;
    a.cphys = cphys;
    a.rs = p.real_elems;
    a.stress_only = stress_only;
    a.err = p.flags;
    a.umax = umax;
    if (p.nkp != K::NKP) return SLES_ERR_INVALID_ARG;
    return launch_persistent(k_zpass<Tp, N, DIM, LES, MODEL, PAR2D, ZL>, (a.nlines + ZL - 1) / ZL, K::THREADS, K::SMEM,
                             st, a);
  }
  int zpass_rt(const PlanInfo& p, int les, int model, int par2d, const Tp* uphys, const Tp* cphys, int so,
               cudaStream_t st, unsigned long long* umax = nullptr) {
    if (!les) return zpass<0, M_NONE, 0>(p, uphys, cphys, so, st, umax);
    const int pz = (DIM == 2) ? par2d : 0;
    if (model == SLES_LES_SMAGORINSKY) {
      return pz ? zpass<1, M_SMAG, 1>(p, uphys, cphys, so, st, umax)
                : zpass<1, M_SMAG, 0>(p, uphys, cphys, so, st, umax);
    }
    return pz ? zpass<1, M_VREMAN, 1>(p, uphys, cphys, so, st, umax)
              : zpass<1, M_VREMAN, 0>(p, uphys, cphys, so, st, umax);
  }

  // One RHS evaluation ending in the X pass described by `fin`.  ctl_step:
  // the z pass collects max u into ctl_step->umax_bits[parity] and the
  // time-step kernel runs before the X pass (stage 0 under device-side dt).
  int pipeline(const PlanInfo& p, int les, const C* ucur, bool primed, const Tp* uphys, const Tp* cphys,
               int stress_only, XArgs<Tp> fin, cudaStream_t st, sles_dtctl* ctl_step = nullptr, int parity = 0) {
    const int model = p.d.les_model, par2d = p.d.parity;
    if (!primed) {
      XArgs<Tp> a0 = xbase(p);
      a0.fwd = 0;
      a0.prep = 1;
      a0.uinv = ucur;
      SLES_TRY(xpass_rt(p, a0, les, par2d, st));
    }
    SLES_TRY(les ? ypass<1>(p, 1, st) : ypass<0>(p, 1, st));
    SLES_TRY(zpass_rt(p, les, model, par2d, uphys, cphys, stress_only, st,
                      ctl_step ? &ctl_step->umax_bits[parity & 1] : nullptr));
    SLES_TRY(les ? ypass<1>(p, 0, st) : ypass<0>(p, 0, st));
    if (ctl_step) SLES_TRY(launch(k_dtctl, 1, 32, 0, st, ctl_step, parity & 1));
    fin.fwd = 1;
    return xpass_rt(p, fin, les, par2d, st);
  }

  // LES stress alone (masked, unprojected) into `out`: the T_hat the
  // reference adds after recording F1 (RK4_method.py:65-70).
  int stress_raw(const PlanInfo& p, const C* ucur, C* out, cudaStream_t st) {
    XArgs<Tp> a = xbase(p);
    a.kind = KX_RAW;
    a.prep = 0;
    a.ucur = ucur;
    a.uout = out;
    return pipeline(p, 1, ucur, false, nullptr, nullptr, 1, a, st);
  }

  int rhs(PlanInfo& p, const void* uh, const void* uphys, const void* cphys, void* du, void* f1,
          cudaStream_t st) override {
    const int les = p.d.les_model != SLES_LES_NONE;
    XArgs<Tp> a = xbase(p);
    a.kind = KX_RHS;
    a.prep = 0;
    a.ucur = (const C*)uh;
    a.uout = (C*)du;
    a.aux = (C*)f1;
    if (f1) {
      a.record_f1 = 1;
      if (les && p.d.parity) {  // F1 = P(mask N + T) - T  (the reference records F1 before adding T back)
        SLES_TRY(stress_raw(p, (const C*)uh, (C*)f1, st));
        a.record_f1 = 2;
      }
    }
    return pipeline(p, les, (const C*)uh, false, (const Tp*)uphys, (const Tp*)cphys, 0, a, st);
  }

  // The x-pass arguments of one integrator stage (kind, coefficients, state
  // pointers).  les / primed may be cleared (the reference's ETD2 drops LES).
  int stage_args(const PlanInfo& p, int s, double dt, const void* ucur, const void* u0, void* u1, void* uout,
                 void* aux, int flags, XArgs<Tp>& a, int& les, bool& primed) {
    const auto& d = p.d;
    les = d.les_model != SLES_LES_NONE;
    a = xbase(p);
    a.ucur = (const C*)ucur;
    a.u0 = (const C*)u0;
    a.u1 = (C*)u1;
    a.uout = (C*)uout;
    a.aux = (C*)aux;
    a.stage = s;
    a.prep = (flags & STAGE_NO_PREPARE) ? 0 : 1;
    primed = (flags & STAGE_PRIMED) != 0;
    const int scheme = (flags & STAGE_RK4) ? SLES_RK4 : d.scheme;
    static const double rk4a[4] = {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0};  // initialize_domain.py:166
    static const double rk4b[3] = {0.5, 0.5, 1.0};                              // initialize_domain.py:167
    switch (scheme) {
      case SLES_RK4:
        if (s < 0 || s > 3) return SLES_ERR_INVALID_ARG;
        a.kind = KX_RK4;
        a.m1 = rk4a[s];
        a.m2 = s < 3 ? rk4b[s] : 0.0;
        break;
      case SLES_RK3:
        if (s < 0 || s > 2) return SLES_ERR_INVALID_ARG;
        if (d.parity) {
          a.kind = KX_RK3P;
          if (s == 0) a.m2 = 0.5;
          if (s == 1) { a.m1 = 1.0; a.m2 = 2.0; }
          if (s == 2) a.m1 = 1.0;
        } else {
          a.kind = KX_SSP3;
          a.m1 = 1.0;
        }
        break;
      case SLES_ETD2:
        if (s != 0 || !aux || !u1) return SLES_ERR_INVALID_ARG;
        a.kind = d.parity ? KX_ETD2P : KX_ETD2C;
        a.dt_d = dt;
        if (d.parity && les) {  // ETD2_method.py:39-46 evaluates u x omega only
          les = 0;
          primed = false;  // the slots hold the LES pipeline's transforms
        }
        break;
      default:
        return SLES_ERR_INVALID_ARG;
    }
    // stage coefficients: the dt multiples, in float64 then rounded (device dt: the same products in-kernel)
    a.c1 = (Tp)(a.m1 * dt);
    a.c2 = (Tp)(a.m2 * dt);
    return SLES_OK;
  }

  int stage(PlanInfo& p, int s, double dt, const void* ucur, const void* u0, void* u1, void* uout, void* aux,
            const void* uphys, const void* cphys, int flags, cudaStream_t st, sles_dtctl* ctl = nullptr,
            int parity = 0) override {
    const auto& d = p.d;
    XArgs<Tp> a;
    int les = 0;
    bool primed = false;
    SLES_TRY(stage_args(p, s, dt, ucur, u0, u1, uout, aux, flags, a, les, primed));
    if (ctl) a.dt_dev = &ctl->dt_step;
    if (flags & STAGE_RECORD_F1) {
      if (!aux) return SLES_ERR_INVALID_ARG;
      a.record_f1 = 1;
      if (les && d.parity) {
        SLES_TRY(stress_raw(p, (const C*)ucur, (C*)aux, st));
        a.record_f1 = 2;
        primed = false;
      }
    }
    return pipeline(p, les, (const C*)ucur, primed, (const Tp*)uphys, (const Tp*)cphys, 0, a, st,
                    (ctl && s == 0) ? ctl : nullptr, parity);
  }

  // ---------------- slab decomposition (3D) ----------------
  int slab_counts(const PlanInfo& p, int* n1, int* n2) const override {
    const bool les = p.d.les_model != SLES_LES_NONE;
    *n1 = les ? 6 : 5;  // x-inverse outputs (A_c, B_c; no LES: A_c and the two kx curl parts)
    *n2 = les ? 6 : 3;  // y-forward outputs (G_c, H_c; no LES: N_c)
    return DIM == 3 ? SLES_OK : SLES_ERR_UNSUPPORTED;
  }
  // inverse x-transforms of the state on this rank's ky rows -> slots [0, n1)
  int slab_prime(PlanInfo& p, const void* u, cudaStream_t st) override {
    XArgs<Tp> a0 = xbase(p);
    a0.fwd = 0;
    a0.prep = 1;
    a0.uinv = (const C*)u;
    return xpass_rt(p, a0, p.d.les_model != SLES_LES_NONE, p.d.parity, st);
  }
  // after exchange 1: y inverse (from the exchange buffer), z, y forward (into
  // the outgoing buffer) on this rank's x planes
  int slab_middle(PlanInfo& p, unsigned long long* umax, cudaStream_t st) override {
    const int les = p.d.les_model != SLES_LES_NONE;
    SLES_TRY(les ? ypass<1>(p, 1, st, true) : ypass<0>(p, 1, st, true));
    SLES_TRY(zpass_rt(p, les, p.d.les_model, p.d.parity, nullptr, nullptr, 0, st, umax));
    return les ? ypass<1>(p, 0, st, true) : ypass<0>(p, 0, st, true);
  }
  // after exchange 2: the x forward, combine, projection and stage update on
  // this rank's ky rows, then (unless NO_PREPARE) the x-inverse priming
  int slab_stage(PlanInfo& p, int s, double dt, const void* ucur, const void* u0, void* u1, void* uout, void* aux,
                 int flags, cudaStream_t st) override {
    if (flags & (STAGE_RECORD_F1 | STAGE_PRIMED)) return SLES_ERR_UNSUPPORTED;
    XArgs<Tp> a;
    int les = 0;
    bool primed = false;
    SLES_TRY(stage_args(p, s, dt, ucur, u0, u1, uout, aux, flags, a, les, primed));
    if (les != (p.d.les_model != SLES_LES_NONE)) return SLES_ERR_UNSUPPORTED;  // the reference's ETD2 with LES
    a.fwd = 1;
    return xpass_rt(p, a, les, p.d.parity, st);
  }

  int profile_rhs(PlanInfo& p, const void* uh, void* du, int iters, double* ms, cudaStream_t st) override {
    const int les = p.d.les_model != SLES_LES_NONE;
    const int model = p.d.les_model, par2d = p.d.parity;
    cudaEvent_t ev[6];
    for (int i = 0; i < 6; ++i)
      if (cudaEventCreate(&ev[i]) != cudaSuccess) return SLES_ERR_CUDA;
    double acc[5] = {0, 0, 0, 0, 0};
    int status = SLES_OK;
    for (int it = 0; it < iters && status == SLES_OK; ++it) {
      XArgs<Tp> a0 = xbase(p);
      a0.fwd = 0;
      a0.prep = 1;
      a0.uinv = (const C*)uh;
      XArgs<Tp> a = xbase(p);
      a.kind = KX_RHS;
      a.prep = 1;
      a.fwd = 1;
      a.ucur = (const C*)uh;
      a.uout = (C*)du;
      cudaEventRecord(ev[0], st);
      status = xpass_rt(p, a0, les, par2d, st);
      cudaEventRecord(ev[1], st);
      if (status == SLES_OK) status = les ? ypass<1>(p, 1, st) : ypass<0>(p, 1, st);
      cudaEventRecord(ev[2], st);
      if (status == SLES_OK) status = zpass_rt(p, les, model, par2d, nullptr, nullptr, 0, st);
      cudaEventRecord(ev[3], st);
      if (status == SLES_OK) status = les ? ypass<1>(p, 0, st) : ypass<0>(p, 0, st);
      cudaEventRecord(ev[4], st);
      if (status == SLES_OK) status = xpass_rt(p, a, les, par2d, st);
      cudaEventRecord(ev[5], st);
      if (cudaEventSynchronize(ev[5]) != cudaSuccess) status = SLES_ERR_CUDA;
      for (int k = 0; k < 5 && status == SLES_OK; ++k) {
        float t = 0;
        cudaEventElapsedTime(&t, ev[k], ev[k + 1]);
        acc[k] += t;
      }
    }
    for (int i = 0; i < 6; ++i) cudaEventDestroy(ev[i]);
    for (int k = 0; k < 5; ++k) ms[k] = iters > 0 ? acc[k] / iters : 0.0;
    return status;
  }

  // ---------------- discrete adjoint (sles_adjoint.cuh) ----------------
  static constexpr int ADJ_FIELDS = 18;
  // lines per AZ work item: halved (keeping whole warps) when the staging
  // buffers and 24 line regions would not fit in shared memory
#ifndef SLES_AZ_LPI
#define SLES_AZ_LPI 0
#endif
  // the adjoint's z lines per item: 8 threads' worth as the forward's (12
  // groups x 8 threads keep whole warps; at 128^3 one line per item made the
  // backward 7% faster than two).  SLES_AZ_LPI > 0 overrides.
  static constexpr int LPI_ADJ = SLES_AZ_LPI > 0 ? SLES_AZ_LPI : cmax(1, 8 / TZ);
  static constexpr int ALPI = (AZGeo<Tp, N, LPI_ADJ>::SMEM > 227 * 1024 && LPI_ADJ > 1) ? LPI_ADJ / 2 : LPI_ADJ;
  int adjoint_fields() const override { return DIM == 3 ? ADJ_FIELDS : 0; }

  AXArgs<Tp> axbase(const PlanInfo& pa) const {
    AXArgs<Tp> a{};
    a.err = pa.flags;
    a.ws = slot(pa, 0);
    a.fs = pa.hc_elems;
    a.nkp = pa.nkp;
    a.nk = pa.nk;
    a.nchunks = xchunks<0>(pa);
    a.nu = (Tp)pa.d.nu;
    a.forcing = (Tp)pa.d.forcing;
    a.kmax = 2.0 / 3.0 * (double)(N / 2 + 1);  // initialize_domain.py:79
    return a;
  }
  // adjoint x-pass variant 1: the TMA tile ring (sles_adj_xtma.cuh) for the
  // Runge-Kutta reverse stages; at 128^3 RK4 Smagorinsky it ran 19% (float32)
  // and 27% (float64) faster than the direct loads of variant 0.  The ETD2
  // reverse steps keep the direct loads (the ring ran them 14% slower).
  int axpass(const PlanInfo& pa, const AXArgs<Tp>& a, cudaStream_t st) {
    if constexpr (HAS_XTMA) {
      if (pa.axvar == 1 && !a.etd) return axpass_tma(pa, a, st);
    }
    using K = XGeo<Tp, N, FX, 3, 0>;
    const long long items = (long long)N * xchunks<0>(pa);
    if (a.etd) return launch_persistent(k_adj_xpass<Tp, N, FX, 2>, items, K::THREADS, K::SMEM, st, a);
    if (a.ssp) return launch_persistent(k_adj_xpass<Tp, N, FX, 1>, items, K::THREADS, K::SMEM, st, a);
    return launch_persistent(k_adj_xpass<Tp, N, FX, 0>, items, K::THREADS, K::SMEM, st, a);
  }
  int axpass_tma(const PlanInfo& pa, const AXArgs<Tp>& a0, cudaStream_t st) {
    if constexpr (!HAS_XTMA) {
      return SLES_ERR_UNSUPPORTED;
    } else {
      using F = FXV<2>;
      using K = XTGeo<Tp, N, F>;
      AXTArgs<Tp> P{};
      P.a = a0;
      P.a.nchunks = (pa.nk + K::W - 1) / K::W;
      P.need_ubar = (a0.fwd && (a0.etd || !a0.last)) ? 1 : 0;
      P.need_acc = (a0.fwd && !a0.etd) ? 1 : 0;
      const long long cb = sizeof(C), row = (long long)pa.nkp * cb, slice = (long long)N * pa.nkp * cb;
      const long long fsb = pa.hc_elems * cb;
      // {columns, ky rows, x slices, components}; box {W columns, 1 ky row, RB x rows, 1}
      auto mk = [&](CUtensorMap* m, const void* base, long long nslot) {
        return make_tmap_box(m, base ? base : (const void*)slot(pa, 0), K::EPC, pa.nk, N, row, N, slice, nslot, fsb,
                             K::W, 1, K::RB);
      };
      SLES_TRY(mk(&P.tws, slot(pa, 0), pa.ws_fields));
      SLES_TRY(mk(&P.tlam, a0.lam, 3));
      SLES_TRY(mk(&P.tubar, P.need_ubar ? (const void*)a0.ubar : nullptr, 3));
      SLES_TRY(mk(&P.tacc, P.need_acc ? (const void*)a0.acc : nullptr, 3));
      SLES_TRY(mk(&P.tunext, a0.prep ? (const void*)a0.unext : nullptr, 3));
      const long long items = (long long)N * P.a.nchunks;
      if (a0.etd) return launch_persistent(k_adj_xpass_tma<Tp, N, F, 2>, items, K::THREADS, K::SMEM, st, P);
      if (a0.ssp) return launch_persistent(k_adj_xpass_tma<Tp, N, F, 1>, items, K::THREADS, K::SMEM, st, P);
      return launch_persistent(k_adj_xpass_tma<Tp, N, F, 0>, items, K::THREADS, K::SMEM, st, P);
    }
  }
  template <int MODEL>
  int azpass(const PlanInfo& pa, double* csgrad, cudaStream_t st) {
    using K = AZGeo<Tp, N, ALPI>;
    static_assert(K::THREADS % 32 == 0, "whole warps");
    if (K::SMEM > 227 * 1024) return SLES_ERR_UNSUPPORTED;
    if (pa.nkp != K::NKP) return SLES_ERR_INVALID_ARG;
    AZArgs<Tp> a{};
    a.ws = slot(pa, 0);
    a.fs = pa.hc_elems;
    a.nkp = pa.nkp;
    a.nlines = (long long)N * N;
    a.scale = (Tp)(1.0 / ((double)N * N * N));
    const double dx = 2.0 * 3.141592653589793 / N;  // initialize_domain.py:42
    const double cs = pa.d.cs;
    a.cdx2 = (MODEL == M_SMAG) ? (Tp)((cs * dx) * (cs * dx)) : (Tp)(2.5 * cs * cs * dx * dx);
    a.csfac = cs != 0.0 ? 2.0 / cs : 0.0;
    a.csgrad = csgrad;
    a.err = pa.flags;
    return launch_persistent(k_adj_zpass<Tp, N, MODEL, ALPI>, (a.nlines + ALPI - 1) / ALPI, K::THREADS, K::SMEM, st,
                             a);
  }
  int aypass(const PlanInfo& pa, int inv, cudaStream_t st) {
    using K = YGeoI<1>;
    using KF = YGeoF<1>;
    YArgs<Tp> a{};
    const long long cb = sizeof(C);
    SLES_TRY(make_tmap(&a.tm, slot(pa, 0), K::EPC, pa.nk, N, (long long)pa.nkp * cb, N, (long long)N * pa.nkp * cb,
                       pa.ws_fields, pa.hc_elems * cb, K::W, K::RB));
    a.err = pa.flags;
    a.ws = slot(pa, 0);
    a.out = slot(pa, 0);
    a.nx = N;
    a.m = N;
    a.fs = pa.hc_elems;
    a.nkp = pa.nkp;
    a.nk = pa.nk;
    a.nchunks = ychunks<1>(pa);
    const long long items = (long long)N * ychunks<1>(pa);
    if (inv) return launch_persistent(k_ypass<Tp, N, FYI<1>, 1, 1, 1>, items, K::THREADS, K::SMEM, st, a);
    return launch_persistent(k_ypass<Tp, N, FYF, 1, 0, 1>, items, KF::THREADS, KF::SMEM, st, a);
  }

  // Reverse-stage coefficients of the plan's scheme.  The step output is
  // U_0 + dt sum_s b_s k_s and stage s > 0 evaluates the RHS at U_0 + dt c_s k_{s-1}:
  //   RK4 (src/RK4_method.py:20-35): b = (1/6, 1/3, 1/3, 1/6), c = (-, 1/2, 1/2, 1)
  //   the reference's RK3 (src/RK3_method.py:20-41, parity = 1): the stages
  //   U_0 + dt/2 k_0, U_0 - dt k_1 + 2 dt k_1 and the output U_0 + dt (k_2/6 + 2 k_2/3 + k_2/6)
  //   give b = (0, 0, 1), c = (-, 1/2, 1).
  // The corrected SSP-RK3 (parity = 0) runs in Shu-Osher form (ssp = 1) and
  // the corrected ETD2 in its two-step form (etd = 1; stage 0: a reverse
  // step, 1: the step after the first RK4 step, 2: the cotangent of F(U_0)),
  // see sles_adjoint.cuh.  The reference's ETD2 (parity = 1) is not covered.
  struct AdjScheme {
    int ns, ssp;
    double b[4], c[4];
    int etd;
  };
  static int adj_scheme(const PlanInfo& pa, AdjScheme* o) {
    if (pa.d.scheme == SLES_RK4) {
      *o = AdjScheme{4, 0, {1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0}, {0.0, 0.5, 0.5, 1.0}, 0};
      return SLES_OK;
    }
    if (pa.d.scheme == SLES_RK3 && pa.d.parity) {
      *o = AdjScheme{3, 0, {0.0, 0.0, 1.0 / 6.0 + 2.0 / 3.0 + 1.0 / 6.0, 0.0}, {0.0, 0.5, 1.0, 0.0}, 0};
      return SLES_OK;
    }
    if (pa.d.scheme == SLES_RK3) {  // SSP-RK3, Shu & Osher (1988)
      *o = AdjScheme{3, 1, {0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}, 0};
      return SLES_OK;
    }
    if (pa.d.scheme == SLES_ETD2 && !pa.d.parity) {  // Cox & Matthews (2002)
      *o = AdjScheme{3, 0, {0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}, 1};
      return SLES_OK;
    }
    return SLES_ERR_UNSUPPORTED;
  }
  int adjoint_seed(PlanInfo& pa, double dt, const void* ubar, void* acc, void* lam, cudaStream_t st) override {
    if constexpr (DIM != 3) {
      return SLES_ERR_UNSUPPORTED;
    } else {
      AdjScheme sc;
      SLES_TRY(adj_scheme(pa, &sc));
      if (sc.etd)  // lam = w1(k) ubar
        return launch(k_adj_seed_etd<Tp>, 1184, 256, 0, st, (const C*)ubar, (C*)lam, pa.hc_elems, N, pa.nkp, pa.nk,
                      dt, pa.d.nu);
      if (sc.ssp)  // acc = ubar/3, lam = 2/3 dt ubar
        return launch(k_adj_seed<Tp>, 1184, 256, 0, st, (const C*)ubar, (C*)acc, (C*)lam, 3 * pa.hc_elems,
                      (Tp)(2.0 / 3.0 * dt), (Tp)(1.0 / 3.0));
      return launch(k_adj_seed<Tp>, 1184, 256, 0, st, (const C*)ubar, (C*)acc, (C*)lam, 3 * pa.hc_elems,
                    (Tp)(sc.b[sc.ns - 1] * dt), (Tp)1);
    }
  }
  int adjoint_prime(PlanInfo& pa, const void* u_state, const void* lam, cudaStream_t st) override {
    if constexpr (DIM != 3) {
      return SLES_ERR_UNSUPPORTED;
    } else {
      if (pa.ws_fields < ADJ_FIELDS) return SLES_ERR_WORKSPACE;
      AXArgs<Tp> a = axbase(pa);
      a.fwd = 0;
      a.prep = 1;
      a.unext = (const C*)u_state;
      a.lam = (C*)lam;
      return axpass(pa, a, st);
    }
  }
  int adjoint_stage(PlanInfo& pa, int s, double dt, const void* unext, void* ubar, void* acc, void* lam,
                    double* csgrad, cudaStream_t st) override {
    if constexpr (DIM != 3) {
      return SLES_ERR_UNSUPPORTED;
    } else {
      if (pa.ws_fields < ADJ_FIELDS) return SLES_ERR_WORKSPACE;
      AdjScheme sc;
      SLES_TRY(adj_scheme(pa, &sc));
      if (s < 0 || s >= sc.ns) return SLES_ERR_INVALID_ARG;
      SLES_TRY(aypass(pa, 1, st));
      switch (pa.d.les_model) {
        case SLES_LES_SMAGORINSKY: SLES_TRY(azpass<M_SMAG>(pa, csgrad, st)); break;
        case SLES_LES_VREMAN: SLES_TRY(azpass<M_VREMAN>(pa, csgrad, st)); break;
        default: SLES_TRY(azpass<M_NONE>(pa, csgrad, st)); break;
      }
      SLES_TRY(aypass(pa, 0, st));
      AXArgs<Tp> a = axbase(pa);
      a.fwd = 1;
      a.prep = unext ? 1 : 0;
      a.unext = (const C*)unext;
      a.ubar = (C*)ubar;
      a.acc = (C*)acc;
      a.lam = (C*)lam;
      // reverse stage s: lam <- b_{s-1} dt ubar + c_s dt g;  s = 0: ubar <- acc, lam <- b_last dt acc
      a.alpha = (Tp)((s > 0 ? sc.b[s - 1] : sc.b[sc.ns - 1]) * dt);
      a.beta = (Tp)(sc.c[s] * dt);
      a.last = (s == 0) ? 1 : 0;
      a.ssp = sc.ssp;
      a.etd = sc.etd ? s + 1 : 0;
      a.dt_d = dt;
      a.nu_d = pa.d.nu;
      if (sc.ssp) {  // Shu-Osher reverse stages of SSP-RK3 (sles_adjoint.cuh)
        static const double pu[3] = {0.0, 1.0, 2.0 / 3.0}, pa3[3] = {1.0 / 3.0, 1.0, 0.75},
                            pb[3] = {1.0, 1.0, 0.25}, pl[3] = {2.0 / 3.0, 1.0, 0.25};
        a.pu = (Tp)pu[s];
        a.pa = (Tp)pa3[s];
        a.pb = (Tp)pb[s];
        a.pl = (Tp)(pl[s] * dt);
      }
      return axpass(pa, a, st);
    }
  }

  int diag(PlanInfo& p, const void* uh, const void* uphys, double* out, double* spec, int nshell,
           cudaStream_t st) override {
    if (nshell > max_shell(DIM, N)) nshell = max_shell(DIM, N);
    if (!spec) nshell = 0;
    double* part = reinterpret_cast<double*>(reinterpret_cast<char*>(p.ws) + WS_HEADER);
    double* mpart = part + (size_t)DIAG_BLOCKS * (2 + max_shell(DIM, N));
    const size_t smem = (nshell + 2 * DIAG_THREADS) * sizeof(double);
    SLES_TRY(launch(k_diag_partial<Tp, DIM>, DIAG_BLOCKS, DIAG_THREADS, smem, st, (const C*)uh, p.hc_elems, N,
                    p.nkp, p.nk, part, nshell));
    int mblk = 0;
    if (uphys) {
      mblk = DIAG_BLOCKS;
      SLES_TRY(launch(k_max_partial<Tp>, DIAG_BLOCKS, DIAG_THREADS, 0, st, (const Tp*)uphys,
                      (long long)DIM * p.real_elems, mpart));
    }
    const double nd = (DIM == 3) ? (double)N * N * N : (double)N * N;
    return launch(k_diag_final, 1, 256, 0, st, (const double*)part, DIAG_BLOCKS, nshell, (const double*)mpart, mblk,
                  1.0 / (nd * nd), p.d.nu, out, spec);
  }
};

// factories, defined in sles_n<N>.cu
Engine* make_engine(int dtype, int dim, int n);

}  // namespace sles

#define SLES_DEFINE_ENGINES(NN)                                                   \
  namespace sles {                                                               \
  Engine* make_engine_##NN(int dtype, int dim) {                                 \
    if (dtype == SLES_F32 && dim == 3) return new EngineImpl<float, NN, 3>();    \
    if (dtype == SLES_F64 && dim == 3) return new EngineImpl<double, NN, 3>();   \
    if (dtype == SLES_F32 && dim == 2) return new EngineImpl<float, NN, 2>();    \
    if (dtype == SLES_F64 && dim == 2) return new EngineImpl<double, NN, 2>();   \
    return nullptr;                                                              \
  }                                                                              \
  }
