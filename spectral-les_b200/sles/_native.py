"""ctypes binding of libsles_b200.so (the C ABI declared in include/sles.h).

Only plain pointers, sizes and a CUDA stream handle cross the boundary; torch
is used for device memory and streams.  There is no CPU fallback: loading
fails loudly if the library is missing or no CUDA device is present.
"""
from __future__ import annotations

import ctypes
import os

import torch

LIB_NAME = "libsles_b200.so"
# SLES_LIB_PATH selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("SLES_LIB_PATH") or os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

SLES_F32, SLES_F64 = 0, 1
LES_NONE, LES_SMAGORINSKY, LES_VREMAN = 0, 1, 2
SCHEME_RK4, SCHEME_RK3, SCHEME_ETD2 = 0, 1, 2
STAGE_RECORD_F1, STAGE_PRIMED, STAGE_NO_PREPARE, STAGE_RK4 = 1, 2, 4, 8

EXPORTED = [
    "sles_plan_create", "sles_plan_destroy", "sles_plan_layout", "sles_plan_workspace_bytes",
    "sles_plan_set_workspace", "sles_plan_set_params", "sles_fft_r2c", "sles_fft_c2r",
    "sles_velocity_curl", "sles_velocity_gradient", "sles_rhs", "sles_stage", "sles_diag",
    "sles_status_string", "sles_version", "sles_profile_rhs", "sles_rhs_static_workspace",
    "sles_adjoint_workspace_bytes", "sles_adjoint_seed", "sles_adjoint_prime", "sles_adjoint_stage",
    "sles_plan_variant_count", "sles_plan_get_variant", "sles_plan_set_variant", "sles_stage_ctl",
    "sles_plan_check", "sles_selftest_wait_timeout", "sles_selftest_wait_timeout_word", "sles_adjoint_check",
    "sles_static_workspace_check", "sles_static_workspace_selftest_timeout",
    "sles_plan_set_slab", "sles_plan_set_batch", "sles_slab_info", "sles_slab_buffers", "sles_slab_prime", "sles_slab_middle",
    "sles_slab_stage", "sles_copy_rows",
]
DT_DONE, DT_SNAPSHOT, DT_NAN, DT_TOO_SMALL = 1, 2, 4, 8


class DtCtl(ctypes.Structure):
    """sles_dtctl (include/sles.h): device-side time-step control."""
    _fields_ = [("dt_step", ctypes.c_double), ("dt", ctypes.c_double), ("t", ctypes.c_double),
                ("t_end", ctypes.c_double), ("ek_next", ctypes.c_double), ("cfl_first", ctypes.c_double),
                ("cfl", ctypes.c_double), ("dx", ctypes.c_double), ("nu", ctypes.c_double),
                ("umax_bits", ctypes.c_uint64 * 2), ("flags", ctypes.c_uint32), ("paused", ctypes.c_uint32),
                ("nsteps", ctypes.c_uint32), ("t_init", ctypes.c_uint32), ("resumed", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32)]
PASS_X, PASS_Y, PASS_Z = 0, 1, 2
PASS_AX = 3  # the adjoint x pass (not timed by the forward autotuner)
PASSES = (PASS_X, PASS_Y, PASS_Z)


class PlanDesc(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("n", ctypes.c_int), ("dtype", ctypes.c_int),
                ("les_model", ctypes.c_int), ("scheme", ctypes.c_int), ("parity", ctypes.c_int),
                ("nu", ctypes.c_double), ("cs", ctypes.c_double), ("forcing", ctypes.c_double)]


class SlabLayout(ctypes.Structure):
    """sles_slab_layout (include/sles.h)."""
    _fields_ = [("nranks", ctypes.c_int32), ("rank", ctypes.c_int32), ("m", ctypes.c_int32),
                ("n_exchange1", ctypes.c_int32), ("n_exchange2", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("block_elems", ctypes.c_int64), ("field_elems", ctypes.c_int64)]


class Layout(ctypes.Structure):
    _fields_ = [("hc_elems", ctypes.c_int64), ("real_elems", ctypes.c_int64),
                ("nkp", ctypes.c_int32), ("nk", ctypes.c_int32)]


class SlesError(RuntimeError):
    def __init__(self, status, where):
        self.status = status
        msg = _lib.sles_status_string(status).decode() if _lib else str(status)
        super().__init__("%s failed: %s (status %d)" % (where, msg, status))


_lib = None


def load_library(path: str = LIB_PATH):
    """Load the shared library and declare every entry point's signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise RuntimeError("%s is not built (run `make -C spectral-les_b200/csrc -j8` or "
                           "`python -c 'import __graft_entry__ as g; g.build()'`)" % path)
    L = ctypes.CDLL(path)
    vp, i, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    sig = {
        "sles_plan_create": (i, [ctypes.POINTER(PlanDesc), ctypes.POINTER(vp)]),
        "sles_plan_destroy": (i, [vp]),
        "sles_plan_layout": (i, [vp, ctypes.POINTER(Layout)]),
        "sles_plan_workspace_bytes": (ctypes.c_size_t, [vp]),
        "sles_plan_set_workspace": (i, [vp, vp, ctypes.c_size_t]),
        "sles_plan_set_params": (i, [vp, d, d, d]),
        "sles_fft_r2c": (i, [vp, vp, vp, i, vp]),
        "sles_fft_c2r": (i, [vp, vp, vp, i, vp]),
        "sles_velocity_curl": (i, [vp, vp, vp, vp, vp]),
        "sles_velocity_gradient": (i, [vp, vp, vp, vp]),
        "sles_rhs": (i, [vp, vp, vp, vp, vp, vp, vp]),
        "sles_stage": (i, [vp, i, d, vp, vp, vp, vp, vp, vp, vp, i, vp]),
        "sles_diag": (i, [vp, vp, vp, vp, vp, i, vp]),
        "sles_status_string": (ctypes.c_char_p, [i]),
        "sles_profile_rhs": (i, [vp, vp, vp, i, vp, vp]),
        "sles_rhs_static_workspace": (i, [vp, vp, vp, vp, vp, vp, vp]),
        "sles_version": (i, []),
        "sles_stage_ctl": (i, [vp, i, vp, i, vp, vp, vp, vp, vp, vp, vp, i, vp]),
        "sles_plan_check": (i, [vp, ctypes.POINTER(ctypes.c_uint), vp]),
        "sles_selftest_wait_timeout": (i, [vp, vp]),
        "sles_selftest_wait_timeout_word": (i, [vp, vp]),
        "sles_adjoint_check": (i, [vp, vp, ctypes.POINTER(ctypes.c_uint), vp]),
        "sles_static_workspace_check": (i, [ctypes.POINTER(ctypes.c_uint), vp]),
        "sles_static_workspace_selftest_timeout": (i, [vp]),
        "sles_plan_variant_count": (i, [vp, i]),
        "sles_plan_get_variant": (i, [vp, i]),
        "sles_plan_set_variant": (i, [vp, i, i]),
        "sles_plan_set_slab": (i, [vp, i, i]),
        "sles_plan_set_batch": (i, [vp, i, vp, vp]),
        "sles_slab_info": (i, [vp, ctypes.POINTER(SlabLayout)]),
        "sles_slab_buffers": (i, [vp, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp),
                                  ctypes.POINTER(vp)]),
        "sles_slab_prime": (i, [vp, vp, vp]),
        "sles_slab_middle": (i, [vp, vp, vp]),
        "sles_slab_stage": (i, [vp, i, d, vp, vp, vp, vp, vp, i, vp]),
        "sles_copy_rows": (i, [vp, ctypes.c_size_t, vp, ctypes.c_size_t, ctypes.c_size_t, ctypes.c_size_t, vp]),
        "sles_adjoint_workspace_bytes": (ctypes.c_size_t, [vp]),
        "sles_adjoint_seed": (i, [vp, vp, d, vp, vp, vp, vp]),
        "sles_adjoint_prime": (i, [vp, vp, vp, vp, vp]),
        "sles_adjoint_stage": (i, [vp, vp, i, d, vp, vp, vp, vp, vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def check(status, where):
    if status != 0:
        raise SlesError(status, where)


def copy_rows(dst, src, width, height, dst_pitch, src_pitch, stream=None):
    """sles_copy_rows: ``height`` rows of ``width`` bytes between device
    tensors, rows ``dst_pitch`` / ``src_pitch`` bytes apart (padded <->
    contiguous fields), on ``stream`` (default: the current stream)."""
    L = load_library()
    s = stream if stream is not None else torch.cuda.current_stream(dst.device)
    check(L.sles_copy_rows(ctypes.c_void_p(dst.data_ptr()), int(dst_pitch), ctypes.c_void_p(src.data_ptr()),
                           int(src_pitch), int(width), int(height), ctypes.c_void_p(s.cuda_stream)),
          "sles_copy_rows")


def ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_handle(device=None):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


class Plan:
    """Owns a ``sles_plan`` and its workspace (from torch's caching allocator)."""

    def __init__(self, dim, n, dtype, les_model, scheme, parity, nu, cs, forcing, device, slab=None, batch=None):
        if not torch.cuda.is_available():
            raise RuntimeError("the spectral-LES B200 path needs a CUDA device; there is no CPU fallback")
        L = load_library()
        self.L = L
        self.device = torch.device(device)
        self.desc = PlanDesc(dim, n, SLES_F64 if dtype == torch.float64 else SLES_F32, les_model, scheme,
                             1 if parity else 0, float(nu), float(cs), float(forcing))
        h = ctypes.c_void_p()
        check(L.sles_plan_create(ctypes.byref(self.desc), ctypes.byref(h)), "sles_plan_create")
        self.h = h
        if slab is not None:  # (nranks, rank): this rank's slab of a decomposed domain
            check(L.sles_plan_set_slab(h, int(slab[0]), int(slab[1])), "sles_plan_set_slab")
        if batch is not None:  # (nu per member, Cs per member): an ensemble batch of this grid
            nus, css = batch
            self.member_nu = torch.tensor([float(x) for x in nus], dtype=torch.float64, device=device)
            self.member_cs = torch.tensor([float(x) for x in css], dtype=torch.float64, device=device)
            check(L.sles_plan_set_batch(h, len(nus), ptr(self.member_nu), ptr(self.member_cs)), "sles_plan_set_batch")
        lay = Layout()
        check(L.sles_plan_layout(h, ctypes.byref(lay)), "sles_plan_layout")
        self.hc_elems, self.real_elems, self.nkp, self.nk = lay.hc_elems, lay.real_elems, lay.nkp, lay.nk
        nbytes = int(L.sles_plan_workspace_bytes(h))
        with torch.cuda.device(self.device):
            # zeroed: the header's error word must start clear (the caching
            # allocator may hand back memory holding another tensor's bytes)
            self.workspace = torch.zeros(nbytes + 256, dtype=torch.uint8, device=self.device)
        off = (-self.workspace.data_ptr()) % 256
        self._ws_ptr = self.workspace.data_ptr() + off
        check(L.sles_plan_set_workspace(h, ctypes.c_void_p(self._ws_ptr), ctypes.c_size_t(nbytes)),
              "sles_plan_set_workspace")

    # slab decomposition (include/sles.h): layout, exchange buffers, the three pass groups
    def slab_info(self):
        lay = SlabLayout()
        check(self.L.sles_slab_info(self.h, ctypes.byref(lay)), "sles_slab_info")
        return lay

    def slab_buffers(self):
        """Device addresses (send1, recv1, send2, recv2) inside the workspace."""
        p = [ctypes.c_void_p() for _ in range(4)]
        check(self.L.sles_slab_buffers(self.h, *[ctypes.byref(x) for x in p]), "sles_slab_buffers")
        return [int(x.value) for x in p]

    def slab_prime(self, u):
        check(self.L.sles_slab_prime(self.h, ptr(u), stream_handle(self.device)), "sles_slab_prime")

    def slab_middle(self, umax_bits=None):
        check(self.L.sles_slab_middle(self.h, ptr(umax_bits), stream_handle(self.device)), "sles_slab_middle")

    def slab_stage(self, stage, dt, ucur, u0, u1, uout, aux=None, flags=0):
        check(self.L.sles_slab_stage(self.h, int(stage), float(dt), ptr(ucur), ptr(u0), ptr(u1), ptr(uout), ptr(aux),
                                     int(flags), stream_handle(self.device)), "sles_slab_stage")

    def variant_count(self, pass_=PASS_X):
        return int(self.L.sles_plan_variant_count(self.h, int(pass_)))

    def get_variant(self, pass_=PASS_X):
        return int(self.L.sles_plan_get_variant(self.h, int(pass_)))

    def set_variant(self, variant, pass_=PASS_X):
        check(self.L.sles_plan_set_variant(self.h, int(pass_), int(variant)), "sles_plan_set_variant")

    def set_params(self, nu, cs, forcing):
        check(self.L.sles_plan_set_params(self.h, float(nu), float(cs), float(forcing)), "sles_plan_set_params")

    def close(self):
        if getattr(self, "h", None):
            self.L.sles_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # thin wrappers; tensors must be contiguous padded storage of this plan
    def fft_r2c(self, real, hc, nf):
        check(self.L.sles_fft_r2c(self.h, ptr(real), ptr(hc), nf, stream_handle(self.device)), "sles_fft_r2c")

    def fft_c2r(self, hc, real, nf):
        check(self.L.sles_fft_c2r(self.h, ptr(hc), ptr(real), nf, stream_handle(self.device)), "sles_fft_c2r")

    def velocity_curl(self, uh, u, curl):
        check(self.L.sles_velocity_curl(self.h, ptr(uh), ptr(u), ptr(curl), stream_handle(self.device)),
              "sles_velocity_curl")

    def velocity_gradient(self, uh, grad):
        check(self.L.sles_velocity_gradient(self.h, ptr(uh), ptr(grad), stream_handle(self.device)),
              "sles_velocity_gradient")

    def rhs(self, uh, du, f1=None, uphys=None, cphys=None):
        check(self.L.sles_rhs(self.h, ptr(uh), ptr(uphys), ptr(cphys), ptr(du), ptr(f1),
                              stream_handle(self.device)), "sles_rhs")

    def stage(self, stage, dt, ucur, u0, u1, uout, aux=None, uphys=None, cphys=None, flags=0):
        check(self.L.sles_stage(self.h, int(stage), float(dt), ptr(ucur), ptr(u0), ptr(u1), ptr(uout), ptr(aux),
                                ptr(uphys), ptr(cphys), int(flags), stream_handle(self.device)), "sles_stage")

    def stage_ctl(self, stage, ctl, parity, ucur, u0, u1, uout, aux=None, uphys=None, cphys=None, flags=0):
        """As stage(), with dt from the device-side controller ``ctl`` (a uint8
        device tensor holding a DtCtl)."""
        check(self.L.sles_stage_ctl(self.h, int(stage), ptr(ctl), int(parity), ptr(ucur), ptr(u0), ptr(u1), ptr(uout),
                                    ptr(aux), ptr(uphys), ptr(cphys), int(flags), stream_handle(self.device)),
              "sles_stage_ctl")

    def check(self):
        """Synchronise this plan's stream and raise SlesError if a kernel's
        bounded wait gave up (the device error word is cleared)."""
        w = ctypes.c_uint(0)
        check(self.L.sles_plan_check(self.h, ctypes.byref(w), stream_handle(self.device)), "sles_plan_check")
        return int(w.value)

    def selftest_wait_timeout(self):
        check(self.L.sles_selftest_wait_timeout(self.h, stream_handle(self.device)), "sles_selftest_wait_timeout")

    def profile_rhs(self, uh, du, iters):
        """Mean ms per launch of {x-inverse, y-inverse, z, y-forward, x-forward}."""
        ms = (ctypes.c_double * 5)()
        check(self.L.sles_profile_rhs(self.h, ptr(uh), ptr(du), int(iters), ms, stream_handle(self.device)),
              "sles_profile_rhs")
        return list(ms)

    # discrete adjoint (include/sles.h); ws: the adjoint workspace (uint8 tensor)
    def adjoint_workspace(self):
        """A zeroed, 256-byte aligned adjoint workspace: (owner tensor, aligned pointer)."""
        nbytes = int(self.L.sles_adjoint_workspace_bytes(self.h))
        if nbytes == 0:
            raise SlesError(2, "sles_adjoint_workspace_bytes")
        with torch.cuda.device(self.device):
            t = torch.zeros(nbytes + 256, dtype=torch.uint8, device=self.device)
        return t, t.data_ptr() + (-t.data_ptr()) % 256

    def adjoint_check(self, ws_ptr):
        """As check(), for the adjoint workspace's error word: raises SlesError
        if a reverse pass's bounded wait gave up or saw a non-finite value."""
        w = ctypes.c_uint(0)
        check(self.L.sles_adjoint_check(self.h, ctypes.c_void_p(ws_ptr), ctypes.byref(w), stream_handle(self.device)),
              "sles_adjoint_check")
        return int(w.value)

    def adjoint_seed(self, ws_ptr, dt, ubar, acc, lam):
        check(self.L.sles_adjoint_seed(self.h, ctypes.c_void_p(ws_ptr), float(dt), ptr(ubar), ptr(acc), ptr(lam),
                                       stream_handle(self.device)), "sles_adjoint_seed")

    def adjoint_prime(self, ws_ptr, u_state, lam):
        check(self.L.sles_adjoint_prime(self.h, ctypes.c_void_p(ws_ptr), ptr(u_state), ptr(lam),
                                        stream_handle(self.device)), "sles_adjoint_prime")

    def adjoint_stage(self, ws_ptr, stage, dt, u_next, ubar, acc, lam, cs_grad):
        check(self.L.sles_adjoint_stage(self.h, ctypes.c_void_p(ws_ptr), int(stage), float(dt), ptr(u_next),
                                        ptr(ubar), ptr(acc), ptr(lam), ptr(cs_grad), stream_handle(self.device)),
              "sles_adjoint_stage")

    def diag(self, uh, out, uphys=None, spectrum=None):
        ns = 0 if spectrum is None else spectrum.numel()
        check(self.L.sles_diag(self.h, ptr(uh), ptr(uphys), ptr(out), ptr(spectrum), ns,
                               stream_handle(self.device)), "sles_diag")
