// C ABI of libsles_b200.so (declarations and reference citations: include/sles.h).
#include <cstdio>
#include <new>

#include "sles_engine.cuh"

namespace sles {
#define SLES_DECL(NN) Engine* make_engine_##NN(int dtype, int dim);
SLES_DECL(16) SLES_DECL(24) SLES_DECL(32) SLES_DECL(48) SLES_DECL(64) SLES_DECL(96) SLES_DECL(128)
SLES_DECL(256) SLES_DECL(512) SLES_DECL(1024)
#undef SLES_DECL

Engine* make_engine(int dtype, int dim, int n) {
  switch (n) {
    case 16: return make_engine_16(dtype, dim);
    case 24: return make_engine_24(dtype, dim);
    case 32: return make_engine_32(dtype, dim);
    case 48: return make_engine_48(dtype, dim);
    case 64: return make_engine_64(dtype, dim);
    case 96: return make_engine_96(dtype, dim);
    case 128: return make_engine_128(dtype, dim);
    case 256: return make_engine_256(dtype, dim);
    case 512: return make_engine_512(dtype, dim);
    case 1024: return make_engine_1024(dtype, dim);
    default: return nullptr;
  }
}
}  // namespace sles

struct sles_plan {
  sles::PlanInfo info;
  sles::Engine* eng;
};



extern "C" {

int sles_version(void) { return SLES_VERSION; }

const char* sles_status_string(int s) {
  switch (s) {
    case SLES_OK: return "ok";
    case SLES_ERR_INVALID_ARG: return "invalid argument";
    case SLES_ERR_UNSUPPORTED: return "unsupported grid size or combination";
    case SLES_ERR_CUDA: return "CUDA runtime error";
    case SLES_ERR_WORKSPACE: return "workspace missing or too small";
    case SLES_ERR_TIMEOUT: return "bounded device wait timed out";
    case SLES_ERR_NONFINITE: return "non-finite value";
    case SLES_ERR_STATE: return "call out of order";
    default: return "unknown status";
  }
}

int sles_plan_create(const sles_plan_desc* d, sles_plan** out) {
  if (!d || !out) return SLES_ERR_INVALID_ARG;
  *out = nullptr;
  if ((d->dim != 2 && d->dim != 3) || (d->dtype != SLES_F32 && d->dtype != SLES_F64)) return SLES_ERR_INVALID_ARG;
  if (d->les_model < SLES_LES_NONE || d->les_model > SLES_LES_VREMAN) return SLES_ERR_INVALID_ARG;
  if (d->scheme < SLES_RK4 || d->scheme > SLES_ETD2) return SLES_ERR_INVALID_ARG;
  if (d->parity != 0 && d->parity != 1) return SLES_ERR_INVALID_ARG;
  if (!(d->nu >= 0.0) || !(d->forcing >= 0.0)) return SLES_ERR_INVALID_ARG;
  sles::Engine* eng = sles::make_engine(d->dtype, d->dim, d->n);
  if (!eng) return SLES_ERR_UNSUPPORTED;
  sles_plan* p = new (std::nothrow) sles_plan();
  if (!p) {
    delete eng;
    return SLES_ERR_INVALID_ARG;
  }
  p->eng = eng;
  sles::PlanInfo& I = p->info;
  I.d = *d;
  I.nk = d->n / 2 + 1;
  I.nkp = (I.nk + 3) / 4 * 4;
  I.hc_elems = (long long)(d->dim == 3 ? d->n * d->n : d->n) * I.nkp;
  I.real_elems = (long long)d->n * d->n * (d->dim == 3 ? d->n : 1);
  I.elem_bytes = d->dtype == SLES_F32 ? 8 : 16;
  I.ws = nullptr;
  I.ws_bytes = 0;
  I.ws_fields = eng->ws_fields_needed(I);
  I.flags = nullptr;
  I.scal = nullptr;
  I.xvar = eng->default_xvar();
  I.yvar = I.zvar = 0;
  I.axvar = eng->variant_count(SLES_PASS_AX) - 1;
  I.slab_p = 1;
  I.slab_r = 0;
  I.slab_m = d->n;
  I.slab_n1 = I.slab_n2 = 0;
  I.nmem = 1;
  I.mnu = I.mcs = nullptr;
  *out = p;
  return SLES_OK;
}

int sles_plan_set_batch(sles_plan* p, int nmembers, const double* nu_dev, const double* cs_dev) {
  if (!p) return SLES_ERR_INVALID_ARG;
  sles::PlanInfo& I = p->info;
  if (I.ws || I.slab_n1 || I.nmem != 1) return SLES_ERR_STATE;  // before the workspace; not on a slab; once
  if (nmembers < 1 || nmembers > 4096) return SLES_ERR_INVALID_ARG;
  I.nmem = nmembers;
  I.mnu = nu_dev;
  I.mcs = cs_dev;
  I.hc_elems *= nmembers;
  I.real_elems *= nmembers;
  return SLES_OK;
}

int sles_plan_set_slab(sles_plan* p, int nranks, int rank) {
  if (!p) return SLES_ERR_INVALID_ARG;
  sles::PlanInfo& I = p->info;
  if (I.ws || I.nmem != 1) return SLES_ERR_STATE;  // before the workspace; not on a member batch
  if (I.d.dim != 3) return SLES_ERR_UNSUPPORTED;
  if (nranks < 1 || rank < 0 || rank >= nranks || I.d.n % nranks != 0) return SLES_ERR_INVALID_ARG;
  const int m = I.d.n / nranks;
  if (m > 256) return SLES_ERR_UNSUPPORTED;  // a line's P blocks of m rows arrive as one TMA box
  int n1 = 0, n2 = 0;
  if (int s = p->eng->slab_counts(I, &n1, &n2)) return s;
  I.slab_p = nranks;
  I.slab_r = rank;
  I.slab_m = m;
  I.slab_n1 = n1;
  I.slab_n2 = n2;
  I.hc_elems = (long long)I.d.n * m * I.nkp;
  I.real_elems = (long long)m * I.d.n * I.d.n;
  I.ws_fields = p->eng->ws_fields_needed(I) + n1 + n2;
  return SLES_OK;
}

int sles_slab_info(const sles_plan* p, sles_slab_layout* out) {
  if (!p || !out) return SLES_ERR_INVALID_ARG;
  const sles::PlanInfo& I = p->info;
  out->nranks = I.slab_p;
  out->rank = I.slab_r;
  out->m = I.slab_m;
  out->n_exchange1 = I.slab_n1;
  out->n_exchange2 = I.slab_n2;
  out->block_elems = (int64_t)I.slab_m * I.slab_m * I.nkp;
  out->field_elems = I.hc_elems;
  return SLES_OK;
}

int sles_plan_variant_count(const sles_plan* p, int pass) {
  if (!p) return 0;
  return p->eng->variant_count(pass);
}

int sles_plan_get_variant(const sles_plan* p, int pass) {
  if (!p) return -1;
  switch (pass) {
    case SLES_PASS_X: return p->info.xvar;
    case SLES_PASS_Y: return p->info.yvar;
    case SLES_PASS_Z: return p->info.zvar;
    case SLES_PASS_AX: return p->info.axvar;
    default: return -1;
  }
}

int sles_plan_set_variant(sles_plan* p, int pass, int variant) {
  if (!p) return SLES_ERR_INVALID_ARG;
  if (variant < 0 || variant >= p->eng->variant_count(pass)) return SLES_ERR_INVALID_ARG;
  switch (pass) {
    case SLES_PASS_X: p->info.xvar = variant; break;
    case SLES_PASS_Y: p->info.yvar = variant; break;
    case SLES_PASS_Z: p->info.zvar = variant; break;
    case SLES_PASS_AX: p->info.axvar = variant; break;
    default: return SLES_ERR_INVALID_ARG;
  }
  return SLES_OK;
}

int sles_plan_destroy(sles_plan* p) {
  if (!p) return SLES_ERR_INVALID_ARG;
  delete p->eng;
  delete p;
  return SLES_OK;
}

int sles_plan_layout(const sles_plan* p, sles_layout* out) {
  if (!p || !out) return SLES_ERR_INVALID_ARG;
  out->hc_elems = p->info.hc_elems;
  out->real_elems = p->info.real_elems;
  out->nkp = p->info.nkp;
  out->nk = p->info.nk;
  return SLES_OK;
}

size_t sles_plan_workspace_bytes(const sles_plan* p) {
  if (!p) return 0;
  const sles::PlanInfo& I = p->info;
  return sles::slots_offset(I.d.dim, I.d.n) + (size_t)I.ws_fields * I.hc_elems * I.elem_bytes;
}

int sles_plan_set_workspace(sles_plan* p, void* ws, size_t bytes) {
  if (!p) return SLES_ERR_INVALID_ARG;
  if (!ws || bytes < sles_plan_workspace_bytes(p)) return SLES_ERR_WORKSPACE;
  if (((uintptr_t)ws) % 256 != 0) return SLES_ERR_INVALID_ARG;
  p->info.ws = ws;
  p->info.ws_bytes = bytes;
  p->info.flags = reinterpret_cast<unsigned*>(ws);
  p->info.scal = reinterpret_cast<double*>(reinterpret_cast<char*>(ws) + 256);
  return SLES_OK;
}

int sles_plan_set_params(sles_plan* p, double nu, double cs, double forcing) {
  if (!p || !(nu >= 0.0) || !(forcing >= 0.0)) return SLES_ERR_INVALID_ARG;
  p->info.d.nu = nu;
  p->info.d.cs = cs;
  p->info.d.forcing = forcing;
  return SLES_OK;
}

static int ready(sles_plan* p) {
  if (!p) return SLES_ERR_INVALID_ARG;
  if (!p->info.ws) return SLES_ERR_WORKSPACE;
  return SLES_OK;
}

// entry points that work on the whole grid: not on a plan set to a slab, nor
// (except the stage and RHS calls) on a batch of ensemble members
static int ready_full(sles_plan* p) {
  if (int s = ready(p)) return s;
  if (p->info.slab_n1 != 0 || p->info.nmem != 1) return SLES_ERR_STATE;
  return SLES_OK;
}
static int ready_batch(sles_plan* p, const void* uphys, const void* cphys) {
  if (int s = ready(p)) return s;
  if (p->info.slab_n1 != 0) return SLES_ERR_STATE;
  if (p->info.nmem != 1 && (uphys || cphys)) return SLES_ERR_UNSUPPORTED;  // stored fields are per domain
  return SLES_OK;
}

int sles_fft_r2c(sles_plan* p, const void* in, void* out, int nf, void* stream) {
  if (int s = ready_full(p)) return s;
  if (!in || !out || nf < 0) return SLES_ERR_INVALID_ARG;
  return p->eng->fft_r2c(p->info, in, out, nf, (cudaStream_t)stream);
}

int sles_fft_c2r(sles_plan* p, const void* in, void* out, int nf, void* stream) {
  if (int s = ready_full(p)) return s;
  if (!in || !out || nf < 0) return SLES_ERR_INVALID_ARG;
  return p->eng->fft_c2r(p->info, in, out, nf, (cudaStream_t)stream);
}

int sles_velocity_curl(sles_plan* p, const void* uh, void* u, void* curl, void* stream) {
  if (int s = ready_full(p)) return s;
  if (!uh) return SLES_ERR_INVALID_ARG;
  return p->eng->velocity_curl(p->info, uh, u, curl, (cudaStream_t)stream);
}

int sles_velocity_gradient(sles_plan* p, const void* uh, void* grad, void* stream) {
  if (int s = ready_full(p)) return s;
  if (!uh || !grad) return SLES_ERR_INVALID_ARG;
  return p->eng->velocity_gradient(p->info, uh, grad, (cudaStream_t)stream);
}

int sles_rhs(sles_plan* p, const void* uh, const void* uphys, const void* cphys, void* du, void* f1, void* stream) {
  if (int s = ready_batch(p, uphys, cphys)) return s;
  if (!uh || !du) return SLES_ERR_INVALID_ARG;
  if (p->info.d.dim == 2 && p->info.d.les_model == SLES_LES_VREMAN && p->info.d.parity) return SLES_ERR_UNSUPPORTED;
  return p->eng->rhs(p->info, uh, uphys, cphys, du, f1, (cudaStream_t)stream);
}

int sles_stage(sles_plan* p, int stage, double dt, const void* ucur, const void* u0, void* u1, void* uout, void* aux,
               const void* uphys, const void* cphys, int flags, void* stream) {
  if (int s = ready_batch(p, uphys, cphys)) return s;
  if (!ucur || !uout || !(dt == dt)) return SLES_ERR_INVALID_ARG;
  if (p->info.d.dim == 2 && p->info.d.les_model == SLES_LES_VREMAN && p->info.d.parity) return SLES_ERR_UNSUPPORTED;
  const int scheme = (flags & sles::STAGE_RK4) ? SLES_RK4 : p->info.d.scheme;
  if ((scheme == SLES_RK4 && (!u0 || !u1)) || (scheme == SLES_RK3 && !u0)) return SLES_ERR_INVALID_ARG;
  return p->eng->stage(p->info, stage, dt, ucur, u0, u1, uout, aux, uphys, cphys, flags, (cudaStream_t)stream);
}

int sles_stage_ctl(sles_plan* p, int stage, void* dtctl, int parity, const void* ucur, const void* u0, void* u1,
                   void* uout, void* aux, const void* uphys, const void* cphys, int flags, void* stream) {
  if (int s = ready_full(p)) return s;
  if (!dtctl || !ucur || !uout || (parity != 0 && parity != 1)) return SLES_ERR_INVALID_ARG;
  if (p->info.d.dim == 2 && p->info.d.les_model == SLES_LES_VREMAN && p->info.d.parity) return SLES_ERR_UNSUPPORTED;
  const int scheme = (flags & sles::STAGE_RK4) ? SLES_RK4 : p->info.d.scheme;
  if ((scheme == SLES_RK4 && (!u0 || !u1)) || (scheme == SLES_RK3 && !u0)) return SLES_ERR_INVALID_ARG;
  return p->eng->stage(p->info, stage, 0.0, ucur, u0, u1, uout, aux, uphys, cphys, flags, (cudaStream_t)stream,
                       reinterpret_cast<sles_dtctl*>(dtctl), parity);
}

}  // extern "C"

namespace {
// Copy a device error word to the host, clear it and map its bits to a status.
int read_clear_flags(unsigned* word, unsigned* flags_out, cudaStream_t st) {
  unsigned w = 0;
  if (cudaMemcpyAsync(&w, word, sizeof(unsigned), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return SLES_ERR_CUDA;
  if (flags_out) *flags_out = w;
  if (w && cudaMemsetAsync(word, 0, sizeof(unsigned), st) != cudaSuccess) return SLES_ERR_CUDA;
  if (w & sles::SLES_ERRF_WAIT_TIMEOUT) return SLES_ERR_TIMEOUT;
  if (w & sles::SLES_ERRF_NONFINITE) return SLES_ERR_NONFINITE;
  return SLES_OK;
}
}  // namespace

extern "C" {

int sles_plan_check(sles_plan* p, unsigned* flags_out, void* stream) {
  if (int s = ready(p)) return s;
  return read_clear_flags(p->info.flags, flags_out, (cudaStream_t)stream);
}

int sles_selftest_wait_timeout(sles_plan* p, void* stream) {
  if (int s = ready(p)) return s;
  return sles::launch(sles::k_wait_selftest, 1, 32, 0, (cudaStream_t)stream, p->info.flags, 4096L);
}

static int slab_ready(sles_plan* p) {
  if (int s = ready(p)) return s;  // (a slab plan is never ready_full)
  if (p->info.slab_n1 == 0) return SLES_ERR_STATE;  // sles_plan_set_slab was not called
  return SLES_OK;
}

int sles_slab_buffers(sles_plan* p, void** send1, void** recv1, void** send2, void** recv2) {
  if (int s = slab_ready(p)) return s;
  const sles::PlanInfo& I = p->info;
  char* slots = reinterpret_cast<char*>(I.ws) + sles::slots_offset(I.d.dim, I.d.n);
  const size_t fb = (size_t)I.hc_elems * I.elem_bytes;
  const int base = I.ws_fields - I.slab_n1 - I.slab_n2;
  if (send1) *send1 = slots;
  if (recv2) *recv2 = slots;
  if (recv1) *recv1 = slots + (size_t)base * fb;
  if (send2) *send2 = slots + (size_t)(base + I.slab_n1) * fb;
  return SLES_OK;
}

int sles_slab_prime(sles_plan* p, const void* u_state, void* stream) {
  if (int s = slab_ready(p)) return s;
  if (!u_state) return SLES_ERR_INVALID_ARG;
  return p->eng->slab_prime(p->info, u_state, (cudaStream_t)stream);
}

int sles_slab_middle(sles_plan* p, unsigned long long* umax_bits, void* stream) {
  if (int s = slab_ready(p)) return s;
  return p->eng->slab_middle(p->info, umax_bits, (cudaStream_t)stream);
}

int sles_slab_stage(sles_plan* p, int stage, double dt, const void* ucur, const void* u0, void* u1, void* uout,
                    void* aux, int flags, void* stream) {
  if (int s = slab_ready(p)) return s;
  if (!ucur || !uout || !(dt == dt)) return SLES_ERR_INVALID_ARG;
  const int scheme = (flags & sles::STAGE_RK4) ? SLES_RK4 : p->info.d.scheme;
  if ((scheme == SLES_RK4 && (!u0 || !u1)) || (scheme == SLES_RK3 && !u0)) return SLES_ERR_INVALID_ARG;
  return p->eng->slab_stage(p->info, stage, dt, ucur, u0, u1, uout, aux, flags, (cudaStream_t)stream);
}

int sles_copy_rows(void* dst, size_t dst_pitch, const void* src, size_t src_pitch, size_t width, size_t height,
                   void* stream) {
  if (!dst || !src || width > dst_pitch || width > src_pitch) return SLES_ERR_INVALID_ARG;
  if ((dst_pitch | src_pitch | width) % 8 != 0 || ((uintptr_t)dst | (uintptr_t)src) % 8 != 0)
    return SLES_ERR_INVALID_ARG;
  if (width == 0 || height == 0) return SLES_OK;
  if (width / 8 > 0x7fffffffULL) return SLES_ERR_UNSUPPORTED;
  constexpr int ROWS = 8;  // rows (warps) per block
  return sles::launch(sles::k_copy_rows8, (long long)((height + ROWS - 1) / ROWS), 32 * ROWS, 0,
                      (cudaStream_t)stream, reinterpret_cast<unsigned long long*>(dst), (long long)(dst_pitch / 8),
                      reinterpret_cast<const unsigned long long*>(src), (long long)(src_pitch / 8), (int)(width / 8),
                      (long long)height);
}

int sles_selftest_wait_timeout_word(void* word, void* stream) {
  if (!word || ((uintptr_t)word) % sizeof(unsigned) != 0) return SLES_ERR_INVALID_ARG;
  return sles::launch(sles::k_wait_selftest, 1, 32, 0, (cudaStream_t)stream, reinterpret_cast<unsigned*>(word),
                      4096L);
}

int sles_diag(sles_plan* p, const void* uh, const void* uphys, double* out, double* spectrum, int nshell,
              void* stream) {
  if (int s = ready_full(p)) return s;
  if (!uh || !out || nshell < 0) return SLES_ERR_INVALID_ARG;
  return p->eng->diag(p->info, uh, uphys, out, spectrum, nshell, (cudaStream_t)stream);
}

int sles_profile_rhs(sles_plan* p, const void* uh, void* du, int iters, double* ms, void* stream) {
  if (int s = ready_full(p)) return s;
  if (!uh || !du || !ms || iters < 1) return SLES_ERR_INVALID_ARG;
  return p->eng->profile_rhs(p->info, uh, du, iters, ms, (cudaStream_t)stream);
}

size_t sles_adjoint_workspace_bytes(const sles_plan* p) {
  if (!p || p->info.d.dim != 3) return 0;
  const sles::PlanInfo& I = p->info;
  return sles::slots_offset(I.d.dim, I.d.n) + (size_t)p->eng->adjoint_fields() * I.hc_elems * I.elem_bytes;
}

// the plan's descriptor with the adjoint workspace in place of its own
static int adjoint_info(sles_plan* p, void* adj_ws, sles::PlanInfo* out) {
  if (!p || !adj_ws) return SLES_ERR_INVALID_ARG;
  if (p->info.d.dim != 3) return SLES_ERR_UNSUPPORTED;
  if (p->info.slab_n1 != 0 || p->info.nmem != 1) return SLES_ERR_STATE;
  if (((uintptr_t)adj_ws) % 256 != 0) return SLES_ERR_INVALID_ARG;
  *out = p->info;
  out->ws = adj_ws;
  out->ws_bytes = sles_adjoint_workspace_bytes(p);
  out->ws_fields = p->eng->adjoint_fields();
  out->flags = reinterpret_cast<unsigned*>(adj_ws);
  out->scal = reinterpret_cast<double*>(reinterpret_cast<char*>(adj_ws) + 256);
  return SLES_OK;
}

int sles_adjoint_check(sles_plan* p, void* adj_ws, unsigned* flags_out, void* stream) {
  sles::PlanInfo I;
  if (int s = adjoint_info(p, adj_ws, &I)) return s;
  return read_clear_flags(I.flags, flags_out, (cudaStream_t)stream);
}

int sles_adjoint_seed(sles_plan* p, void* adj_ws, double dt, const void* ubar, void* acc, void* lam, void* stream) {
  sles::PlanInfo I;
  if (int s = adjoint_info(p, adj_ws, &I)) return s;
  if (!ubar || !acc || !lam || !(dt == dt)) return SLES_ERR_INVALID_ARG;
  return p->eng->adjoint_seed(I, dt, ubar, acc, lam, (cudaStream_t)stream);
}

int sles_adjoint_prime(sles_plan* p, void* adj_ws, const void* u_state, const void* lam, void* stream) {
  sles::PlanInfo I;
  if (int s = adjoint_info(p, adj_ws, &I)) return s;
  if (!u_state || !lam) return SLES_ERR_INVALID_ARG;
  return p->eng->adjoint_prime(I, u_state, lam, (cudaStream_t)stream);
}

int sles_adjoint_stage(sles_plan* p, void* adj_ws, int stage, double dt, const void* u_next, void* ubar, void* acc,
                       void* lam, double* cs_grad, void* stream) {
  sles::PlanInfo I;
  if (int s = adjoint_info(p, adj_ws, &I)) return s;
  if (!ubar || !acc || !lam || !(dt == dt) || stage < 0 || stage > 3) return SLES_ERR_INVALID_ARG;
  if (p->info.d.les_model != SLES_LES_NONE && !cs_grad) return SLES_ERR_INVALID_ARG;
  return p->eng->adjoint_stage(I, stage, dt, u_next, ubar, acc, lam, cs_grad, (cudaStream_t)stream);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// sles_rhs_static_workspace: the fused RHS evaluation for callers that cannot
// allocate device memory (no counterpart in the reference).  Its scratch is
// this file-scope device array instead of a caller-provided workspace, so the
// call makes no cudaMalloc/cudaFree and no allocating library call.  Every GPU
// that loads this library holds the array (SLES_STATIC_WORKSPACE_BYTES) until
// the process exits.  All calls on a device share it and it keeps the previous
// call's contents; the only part that must start at zero (the error word) is
// cleared by each call.  Calls whose work overlaps on the GPU (two streams, two
// threads) race on the array and must be serialized by the caller.
// ---------------------------------------------------------------------------
static __device__ __align__(256) unsigned char g_sles_static_ws[SLES_STATIC_WORKSPACE_BYTES];

namespace {
std::mutex g_static_ws_mu;
constexpr int kMaxDevices = 64;
// device address of g_sles_static_ws per device ordinal, with the CUDA context
// it was looked up in: after a device reset (or in another context) the
// address is looked up again
struct StaticAddr {
  void* ctx;
  void* addr;
};
StaticAddr g_static_ws_addr[kMaxDevices] = {};

using CtxGetCurrentFn = CUresult (*)(CUcontext*);
CtxGetCurrentFn ctx_get_current() {
  static CtxGetCurrentFn fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrentFn>(f);
  });
  return fn;
}

// The array's device address on the current device (in host code the array's
// name is only a host-side stand-in, so it is looked up with the device
// current).  Makes no allocation.
int static_ws_address(void** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return SLES_ERR_CUDA;
  if (dev < 0 || dev >= kMaxDevices) return SLES_ERR_UNSUPPORTED;
  CtxGetCurrentFn getctx = ctx_get_current();
  if (!getctx) return SLES_ERR_CUDA;
  CUcontext ctx = nullptr;
  if (getctx(&ctx) != CUDA_SUCCESS) return SLES_ERR_CUDA;
  std::lock_guard<std::mutex> g(g_static_ws_mu);
  StaticAddr& e = g_static_ws_addr[dev];
  if (!e.addr || !ctx || e.ctx != (void*)ctx) {
    void* a = nullptr;
    if (cudaGetSymbolAddress(&a, g_sles_static_ws) != cudaSuccess || !a) return SLES_ERR_CUDA;
    // the lookup makes the device's context current if none was
    if (getctx(&ctx) != CUDA_SUCCESS || !ctx) return SLES_ERR_CUDA;
    e.addr = a;
    e.ctx = (void*)ctx;
  }
  *out = e.addr;
  return SLES_OK;
}
}  // namespace

extern "C" int sles_rhs_static_workspace(sles_plan* p, const void* uh, const void* uphys, const void* cphys,
                                         void* du, void* f1, void* stream) {
  if (!p || !uh || !du) return SLES_ERR_INVALID_ARG;
  if (p->info.slab_n1 != 0 || p->info.nmem != 1) return SLES_ERR_STATE;
  if (sles_plan_workspace_bytes(p) > (size_t)SLES_STATIC_WORKSPACE_BYTES) return SLES_ERR_WORKSPACE;
  if (p->info.d.dim == 2 && p->info.d.les_model == SLES_LES_VREMAN && p->info.d.parity) return SLES_ERR_UNSUPPORTED;
  void* ws = nullptr;
  if (int s = static_ws_address(&ws)) return s;
  sles::PlanInfo info = p->info;  // the plan's own workspace (if any) is left untouched
  info.ws = ws;
  info.ws_bytes = SLES_STATIC_WORKSPACE_BYTES;
  info.flags = reinterpret_cast<unsigned*>(ws);
  info.scal = reinterpret_cast<double*>(reinterpret_cast<char*>(ws) + 256);
  if (cudaMemsetAsync(info.flags, 0, sizeof(unsigned), (cudaStream_t)stream) != cudaSuccess) return SLES_ERR_CUDA;
  return p->eng->rhs(info, uh, uphys, cphys, du, f1, (cudaStream_t)stream);
}

extern "C" int sles_static_workspace_check(unsigned* flags_out, void* stream) {
  void* ws = nullptr;
  if (int s = static_ws_address(&ws)) return s;
  return read_clear_flags(reinterpret_cast<unsigned*>(ws), flags_out, (cudaStream_t)stream);
}

extern "C" int sles_static_workspace_selftest_timeout(void* stream) {
  void* ws = nullptr;
  if (int s = static_ws_address(&ws)) return s;
  return sles::launch(sles::k_wait_selftest, 1, 32, 0, (cudaStream_t)stream, reinterpret_cast<unsigned*>(ws), 4096L);
}
