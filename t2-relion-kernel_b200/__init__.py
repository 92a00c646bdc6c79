"""Python mirror of the coarse-pass diff2 C ABI (include/b200d2.h).

The compute path is libb200d2.so (hand-written CUDA for sm_100a); this module
only binds it with ctypes and converts torch tensors to device pointers.  There
is no CPU fallback: importing works without a GPU, but every compute call needs
the library and a CUDA device and raises B200D2Error otherwise.

Names follow the reference harness (Edgarrrrrr/T2-RELION-kernel):
`Projector` is AccProjector (src/acc_projector.h), `Projector.view()` is
AccProjectorKernel::makeKernel (src/acc_projectorkernel_impl.h:410),
`run_diff2_kernel_coarse` is runDiff2KernelCoarse
(src/acc_helper_functions_impl.h:15) and `run_diff2_kernel_coarse_double` is
runDiff2KernelCoarseDouble (src/acc_helper_functions_impl.h:503).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libb200d2.so")

INTERP_TEXTURE = 0
INTERP_LINEAR = 1
PREC_FP32 = 0
PREC_TF32 = 1
PREC_TF32X3 = 2
PREC_BF16X3 = 3
PREC_FP64 = 4
PREC_FP16 = 5  # scaled FP16, one product
PREC_FP16X3 = 6  # scaled FP16 hi/lo split, three products

_STATUS = {0: "ok", 1: "invalid argument", 2: "unsupported", 3: "CUDA error", 4: "out of memory",
           5: "device wait timed out", 6: "no device", 7: "request exceeds a fixed capacity"}
STATIC_SCRATCH_BYTES = 64 << 20  # B200D2_STATIC_SCRATCH_BYTES


class B200D2Error(RuntimeError):
    def __init__(self, code: int, where: str):
        super().__init__(f"{where}: {_STATUS.get(code, 'status %d' % code)} ({code})")
        self.code = code


class View(C.Structure):
    """b200d2_view: kernel-side projector view (mirrors AccProjectorKernel)."""

    _fields_ = [(n, C.c_int) for n in ("mdlX", "mdlXY", "mdlZ", "imgX", "imgY", "imgZ", "mdlInitY",
                                         "mdlInitZ", "maxR", "maxR2", "maxR2_padded")] + [
        ("padding_factor", C.c_float), ("tex_re", C.c_ulonglong), ("tex_im", C.c_ulonglong),
        ("lin_re", C.c_void_p), ("lin_im", C.c_void_p), ("interp", C.c_int), ("tex_c", C.c_ulonglong)]


class Batch(C.Structure):
    """b200d2_batch: P particles sharing orientations and translations."""

    _fields_ = [("d_eulers", C.c_void_p), ("O", C.c_int), ("d_trans_x", C.c_void_p), ("d_trans_y", C.c_void_p),
                ("T", C.c_int), ("P", C.c_int), ("N_img", C.c_int), ("d_real", C.c_void_p),
                ("d_imag", C.c_void_p), ("d_corr", C.c_void_p), ("img_stride", C.c_longlong),
                ("d_diff2", C.c_void_p), ("accumulate", C.c_int), ("d_min", C.c_void_p),
                ("d_argmin", C.c_void_p), ("d_coor_xy", C.c_void_p), ("n_listed", C.c_int),
                ("score", C.c_int)]


SCORE_DIFF2 = 0
SCORE_CC = 1


class ParticleDesc(C.Structure):
    """b200d2_particle_desc: one particle of an uneven plan."""

    _fields_ = [("d_real", C.c_void_p), ("d_imag", C.c_void_p), ("d_corr", C.c_void_p), ("d_diff2", C.c_void_p),
                ("h_orient", C.c_void_p), ("O", C.c_int), ("h_trans_x", C.c_void_p), ("h_trans_y", C.c_void_p),
                ("T", C.c_int)]


class CTF(C.Structure):
    """b200d2_ctf: one particle's CTF parameters."""

    _fields_ = [(n, C.c_float) for n in ("defocus_u_A", "defocus_v_A", "defocus_angle_deg", "voltage_kV", "cs_mm",
                                         "amp_contrast", "phase_shift_deg", "bfactor", "scale")]


PLAN_MAX_VARIANTS = 16


class PlanInfo(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("P", "O_all", "rows", "tiles", "tiles_dense", "row_bytes", "graph",
                                         "stages")] + [
        ("evals", C.c_longlong), ("workspace_bytes", C.c_size_t), ("tile_n", C.c_int), ("split", C.c_int),
        ("pair", C.c_int), ("tiles_n128", C.c_int), ("tiles_pair", C.c_int), ("n_tuned", C.c_int),
        ("tuned_variant", (C.c_int * 4) * PLAN_MAX_VARIANTS),
        ("tuned_ms", C.c_double * PLAN_MAX_VARIANTS), ("norm_tiles", C.c_int * 3), ("norm_tile_p", C.c_int),
        ("norm_tuned_ms", C.c_double * 3)]


class Request(C.Structure):
    """b200d2_request: one serving request (host buffers)."""

    _fields_ = [("ref", C.c_int), ("P", C.c_int), ("h_real", C.c_void_p), ("h_imag", C.c_void_p),
                ("h_corr", C.c_void_p), ("h_orient", C.c_void_p), ("O", C.c_int), ("h_trans_x", C.c_void_p),
                ("h_trans_y", C.c_void_p), ("T", C.c_int), ("h_diff2", C.c_void_p), ("h_min", C.c_void_p),
                ("h_argmin", C.c_void_p)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_longlong), ("completed", C.c_longlong), ("rejected", C.c_longlong),
                ("evals", C.c_longlong), ("in_flight", C.c_int), ("queued", C.c_int), ("max_in_flight", C.c_int),
                ("bytes_in_use", C.c_size_t), ("peak_bytes", C.c_size_t), ("admit_host_s", C.c_double),
                ("cancelled", C.c_longlong), ("merged_admissions", C.c_longlong), ("merged_requests", C.c_longlong),
                ("stream_s", C.c_double), ("admit_host_max_s", C.c_double), ("admit_grow_max_s", C.c_double),
                ("admit_launch_max_s", C.c_double), ("queue_wait_max_s", C.c_double), ("done_lag_max_s", C.c_double)]


# status codes (b200d2_status)
OK, ERR_INVALID, ERR_UNSUPPORTED, ERR_CUDA, ERR_OOM, ERR_TIMEOUT, ERR_NO_DEVICE, ERR_TOO_LARGE, ERR_CANCELLED = range(9)

PLAN_AUTOTUNE = 1
PLAN_GRAPH = 2
PLAN_ACCUMULATE = 4
PLAN_REORDER = 8

_lib = None


def library_path() -> str:
    return LIB_PATH


def lib():
    """Load libb200d2.so (fails loudly if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise B200D2Error(6, f"libb200d2.so not built ({LIB_PATH}); run t2-relion-kernel_b200/build.py")
        L = C.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def _declare(L):
    P, I, F, Z = C.c_void_p, C.c_int, C.c_float, C.c_size_t
    sig = {
        "b200d2_projector_create": [I, I, I, I, I, I, F, P, P, I, C.POINTER(P)],
        "b200d2_projector_load_dat": [C.c_char_p, I, C.POINTER(P)],
        "b200d2_projector_destroy": [P],
        "b200d2_projector_dims": [P, P, P],
        "b200d2_projector_view": [P, I, I, I, I, I, C.POINTER(View)],
        "b200d2_diff2_coarse": [C.POINTER(View), P, P, P, P, P, P, P, Z, Z, Z, P, I],
        "b200d2_diff2_coarse_f64": [C.POINTER(View), P, P, P, P, P, P, P, Z, Z, Z, I, P],
        "b200d2_diff2_coarse_cc": [C.POINTER(View), P, P, P, P, P, P, P, Z, Z, Z, P, I],
        "b200d2_diff2_coarse_cc_f64": [C.POINTER(View), P, P, P, P, P, P, P, Z, Z, Z, P],
        "b200d2_diff2_coarse_batch": [C.POINTER(View), C.POINTER(Batch), I, P, Z, P],
        "b200d2_minloc": [P, C.c_longlong, I, P, P, P],
        "b200d2_project_pixels": [C.POINTER(View), P, I, P, P, I, P, P, P],
        "b200d2_diff2_coarse_batch_static": [C.POINTER(View), C.POINTER(Batch), I, P],
        "b200d2_plan_create": [C.POINTER(View), P, I, I, C.POINTER(ParticleDesc), I, I, I, P, P, C.POINTER(P)],
        "b200d2_plan_run": [P, P],
        "b200d2_plan_get_info": [P, C.POINTER(PlanInfo)],
        "b200d2_plan_destroy": [P],
        "b200d2_server_create": [I, Z, I, C.POINTER(P)],
        "b200d2_server_add_reference": [P, C.POINTER(View), P, I, I, C.POINTER(I)],
        "b200d2_server_submit": [P, C.POINTER(Request), C.POINTER(C.c_longlong)],
        "b200d2_server_wait": [P, C.c_longlong, C.c_double, C.POINTER(C.c_double), C.POINTER(C.c_double)],
        "b200d2_server_get_stats": [P, C.POINTER(ServerStats)],
        "b200d2_server_cancel": [P, C.c_longlong],
        "b200d2_server_set_merging": [P, I, I, I],
        "b200d2_server_destroy": [P],
        "b200d2_coarse_weights": [P, I, I, I, P, P, P, I, P, P, P, Z, P],
        "b200d2_significance": [P, I, C.c_longlong, P, C.c_double, C.c_longlong, P, P, P, P, Z, P],
        "b200d2_pack_mask": [P, I, C.c_longlong, P, P],
        "b200d2_set_gemm_variant": [I, I, I, I],
        "b200d2_set_combine": [I],
        "b200d2_set_wait_limit_ns": [C.c_ulonglong],
        "b200d2_set_operand_gen": [I],
        "b200d2_set_projection_cache": [I],
        "b200d2_set_batch_graphs": [I],
        "b200d2_diff2_fine": [C.POINTER(View), P, P, P, P, P, P, P, Z, F, Z, P, P, P, P, P],
        "b200d2_diff2_fine_cc": [C.POINTER(View), P, P, P, P, P, P, P, Z, Z, P, P, P, P, P],
        "b200d2_ctf_fold": [P, P, C.c_longlong, I, I, I, I, I, I, F, P, P, C.c_longlong, P, P, P, P],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.b200d2_diff2_coarse_batch_workspace.argtypes = [C.POINTER(View), C.POINTER(Batch), I]
    L.b200d2_diff2_coarse_batch_workspace.restype = C.c_size_t
    L.b200d2_diff2_coarse_batch_stage.argtypes = [C.POINTER(View), C.POINTER(Batch), I, I, P, Z, P]
    L.b200d2_diff2_coarse_batch_stage.restype = C.c_int
    L.b200d2_stage_name.argtypes = [I, I]
    L.b200d2_stage_name.restype = C.c_char_p
    L.b200d2_workspace_status.argtypes = [P, P, C.POINTER(C.c_int)]
    L.b200d2_workspace_status.restype = C.c_int
    L.b200d2_coarse_weights_workspace.argtypes = [I, C.c_longlong]
    L.b200d2_coarse_weights_workspace.restype = C.c_size_t
    L.b200d2_significance_workspace.argtypes = [I, C.c_longlong]
    L.b200d2_significance_workspace.restype = C.c_size_t
    L.b200d2_launch_count.argtypes = []
    L.b200d2_launch_count.restype = C.c_ulonglong
    # optional entry points declared by later modules of the library
    for name, (args, res) in _EXTRA.items():
        if hasattr(L, name):
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res


_EXTRA: dict = {}


def _check(code: int, where: str) -> None:
    if code != 0:
        raise B200D2Error(code, where)


def _ptr(t) -> int:
    """Device pointer of a torch CUDA tensor (or an int address)."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if not t.is_cuda:
        raise B200D2Error(1, "expected a CUDA tensor")
    if not t.is_contiguous():
        raise B200D2Error(1, "expected a contiguous tensor")
    return t.data_ptr()


def _stream(stream) -> int:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    if isinstance(stream, int):
        return stream
    return stream.cuda_stream


class Projector:
    """Resident padded Fourier volume (AccProjector).  use_texture: 1 texture,
    0 linear arrays, 2 both."""

    def __init__(self, pv=None, use_texture: int = 2, *, dat_path: str | None = None):
        self._h = C.c_void_p()
        if dat_path is not None:
            _check(lib().b200d2_projector_load_dat(dat_path.encode(), use_texture, C.byref(self._h)),
                   "projector_load_dat")
        else:
            re = np.ascontiguousarray(pv.re, np.float32)
            im = np.ascontiguousarray(pv.im, np.float32)
            _check(lib().b200d2_projector_create(pv.mdlX, pv.mdlY, pv.mdlZ, pv.mdlInitY, pv.mdlInitZ,
                                                 pv.mdlMaxR, float(pv.padding_factor),
                                                 re.ctypes.data_as(C.c_void_p), im.ctypes.data_as(C.c_void_p),
                                                 use_texture, C.byref(self._h)), "projector_create")

    @property
    def handle(self):
        return self._h

    def dims(self):
        d = (C.c_int * 6)()
        pf = C.c_float()
        _check(lib().b200d2_projector_dims(self._h, d, C.byref(pf)), "projector_dims")
        return tuple(d), pf.value

    def view(self, imgX: int, imgY: int, imgMaxR: int, imgZ: int = 1, interp: int = INTERP_TEXTURE) -> View:
        v = View()
        _check(lib().b200d2_projector_view(self._h, imgX, imgY, imgZ, imgMaxR, interp, C.byref(v)),
               "projector_view")
        return v

    def close(self):
        if self._h and self._h.value:
            lib().b200d2_projector_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def project_pixels(view: View, eulers, px, py, out_re, out_im, O: int, K: int, stream=None):
    """Projections of O orientations at K pixels: out[o*K + k] (project3Dmodel)."""
    _check(lib().b200d2_project_pixels(C.byref(view), _ptr(eulers), O, _ptr(px), _ptr(py), K, _ptr(out_re),
                                       _ptr(out_im), _stream(stream)), "project_pixels")


def run_diff2_kernel_coarse(view: View, trans_x, trans_y, corr, real, imag, eulers, diff2s,
                            O: int, T: int, N_img: int, stream=None, precision: int = PREC_FP32):
    """runDiff2KernelCoarse: diff2s[o*T+t] += diff2 (FP32 CUDA cores)."""
    _check(lib().b200d2_diff2_coarse(C.byref(view), _ptr(trans_x), _ptr(trans_y), _ptr(corr), _ptr(real),
                                     _ptr(imag), _ptr(eulers), _ptr(diff2s), O, T, N_img, _stream(stream),
                                     precision), "diff2_coarse")


def run_diff2_kernel_coarse_double(view: View, trans_x, trans_y, corr, real, imag, eulers, diff2s,
                                   O: int, T: int, N_img: int, filter_img: bool = False, stream=None):
    """runDiff2KernelCoarseDouble: diff2s (double) += FP64 diff2."""
    _check(lib().b200d2_diff2_coarse_f64(C.byref(view), _ptr(trans_x), _ptr(trans_y), _ptr(corr), _ptr(real),
                                         _ptr(imag), _ptr(eulers), _ptr(diff2s), O, T, N_img,
                                         1 if filter_img else 0, _stream(stream)), "diff2_coarse_f64")


def run_diff2_kernel_coarse_cc(view: View, trans_x, trans_y, corr, real, imag, eulers, diff2s,
                               O: int, T: int, N_img: int, stream=None, precision: int = PREC_FP32):
    """runDiff2KernelCoarse with do_CC: diff2s[o*T+t] = -cross / sqrt(norm) (written)."""
    _check(lib().b200d2_diff2_coarse_cc(C.byref(view), _ptr(trans_x), _ptr(trans_y), _ptr(corr), _ptr(real),
                                        _ptr(imag), _ptr(eulers), _ptr(diff2s), O, T, N_img, _stream(stream),
                                        precision), "diff2_coarse_cc")


def run_diff2_kernel_coarse_cc_double(view: View, trans_x, trans_y, corr, real, imag, eulers, diff2s,
                                      O: int, T: int, N_img: int, stream=None):
    """The CC score summed in FP64 (diff2s double, written)."""
    _check(lib().b200d2_diff2_coarse_cc_f64(C.byref(view), _ptr(trans_x), _ptr(trans_y), _ptr(corr), _ptr(real),
                                            _ptr(imag), _ptr(eulers), _ptr(diff2s), O, T, N_img, _stream(stream)),
           "diff2_coarse_cc_f64")


def launch_count() -> int:
    """Kernels launched by libb200d2 in this process so far."""
    return int(lib().b200d2_launch_count())


def make_batch(eulers, trans_x, trans_y, real, imag, corr, diff2, *, O: int, T: int, P: int, N_img: int,
               img_stride: int | None = None, accumulate: bool = False, out_min=None, out_argmin=None,
               coor_xy=None, n_listed: int = 0, score: int = SCORE_DIFF2) -> Batch:
    b = Batch()
    b.score = score
    b.d_coor_xy = _ptr(coor_xy)
    b.n_listed = n_listed if coor_xy is not None else 0
    b.d_eulers, b.O = _ptr(eulers), O
    b.d_trans_x, b.d_trans_y, b.T = _ptr(trans_x), _ptr(trans_y), T
    b.P, b.N_img = P, N_img
    b.d_real, b.d_imag, b.d_corr = _ptr(real), _ptr(imag), _ptr(corr)
    b.img_stride = N_img if img_stride is None else img_stride
    b.d_diff2 = _ptr(diff2)
    b.accumulate = 1 if accumulate else 0
    b.d_min = _ptr(out_min)
    b.d_argmin = _ptr(out_argmin)
    return b


def batch_workspace_bytes(view: View, batch: Batch, precision: int) -> int:
    return int(lib().b200d2_diff2_coarse_batch_workspace(C.byref(view), C.byref(batch), precision))


def diff2_coarse_batch(view: View, batch: Batch, precision: int = PREC_BF16X3, workspace=None, stream=None):
    """Score P particles against O orientations x T translations -> diff2[p][o][t]."""
    ws = _ptr(workspace) if workspace is not None else None
    nbytes = workspace.numel() * workspace.element_size() if workspace is not None and not isinstance(
        workspace, int) else 0
    _check(lib().b200d2_diff2_coarse_batch(C.byref(view), C.byref(batch), precision, ws, nbytes,
                                           _stream(stream)), "diff2_coarse_batch")


class Plan:
    """Uneven batch in one persistent contraction launch (b200d2_plan_*).

    `particles`: list of dicts with device tensors real, imag, corr, diff2
    ([O_p*T_p]) and host numpy arrays orient (int32, or None), trans_x,
    trans_y (float32)."""

    def __init__(self, view: View, eulers, O_all: int, N_img: int, particles: list, precision: int = PREC_BF16X3,
                 flags: int = PLAN_AUTOTUNE | PLAN_GRAPH | PLAN_REORDER, out_min=None, out_argmin=None):
        self._keep = []
        descs = (ParticleDesc * len(particles))()
        for i, pt in enumerate(particles):
            d = descs[i]
            d.d_real, d.d_imag, d.d_corr, d.d_diff2 = (_ptr(pt[k]) for k in ("real", "imag", "corr", "diff2"))
            orient = pt.get("orient")
            if orient is not None:
                orient = np.ascontiguousarray(orient, np.int32)
                self._keep.append(orient)
                d.h_orient = orient.ctypes.data_as(C.c_void_p)
                d.O = int(orient.size)
            else:
                d.h_orient = None
                d.O = int(pt["O"])
            tx = np.ascontiguousarray(pt["trans_x"], np.float32)
            ty = np.ascontiguousarray(pt["trans_y"], np.float32)
            self._keep += [tx, ty]
            d.h_trans_x = tx.ctypes.data_as(C.c_void_p)
            d.h_trans_y = ty.ctypes.data_as(C.c_void_p)
            d.T = int(tx.size)
        self._h = C.c_void_p()
        _check(lib().b200d2_plan_create(C.byref(view), _ptr(eulers), O_all, N_img, descs, len(particles), precision,
                                        flags, _ptr(out_min), _ptr(out_argmin), C.byref(self._h)), "plan_create")

    def run(self, stream=None):
        _check(lib().b200d2_plan_run(self._h, _stream(stream)), "plan_run")

    def info(self) -> dict:
        inf = PlanInfo()
        _check(lib().b200d2_plan_get_info(self._h, C.byref(inf)), "plan_get_info")
        d = {n: getattr(inf, n) for n, _ in PlanInfo._fields_
             if n not in ("tuned_ms", "tuned_variant", "norm_tiles", "norm_tuned_ms")}
        d["norm_tiles"] = list(inf.norm_tiles)
        d["norm_tuned_ms"] = list(inf.norm_tuned_ms)
        # autotuner record: ((row_bytes, tile_n, split), ms) per variant timed
        d["tuned"] = [(tuple(inf.tuned_variant[i]), inf.tuned_ms[i]) for i in range(inf.n_tuned)]
        return d

    def close(self):
        if self._h and self._h.value:
            lib().b200d2_plan_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _host_ptr(a):
    """Address of a host buffer: C-contiguous numpy array or CPU torch tensor."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise B200D2Error(1, "expected a C-contiguous host array")
        return a.ctypes.data
    if getattr(a, "is_cuda", False):
        raise B200D2Error(1, "expected a host buffer")
    return a.data_ptr()


class Server:
    """Request loop with continuous batching over resident references
    (b200d2_server_*).  Host buffers of a request are kept alive until wait()."""

    def __init__(self, slots: int = 4, hbm_budget: int = 32 << 30, precision: int = PREC_TF32):
        self._h = C.c_void_p()
        _check(lib().b200d2_server_create(slots, hbm_budget, precision, C.byref(self._h)), "server_create")
        self._keep: dict = {}

    def add_reference(self, view: View, eulers: np.ndarray, N_img: int) -> int:
        eul = np.ascontiguousarray(eulers, np.float32).reshape(-1, 9)
        rid = C.c_int()
        _check(lib().b200d2_server_add_reference(self._h, C.byref(view), eul.ctypes.data_as(C.c_void_p),
                                                 eul.shape[0], N_img, C.byref(rid)), "server_add_reference")
        return rid.value

    def submit(self, ref: int, real, imag, corr, orient, trans_x, trans_y, out_diff2=None, out_min=None,
               out_argmin=None) -> int:
        orient = np.ascontiguousarray(orient, np.int32)
        tx = np.ascontiguousarray(trans_x, np.float32)
        ty = np.ascontiguousarray(trans_y, np.float32)
        r = Request()
        r.ref, r.P = ref, int(real.shape[0])
        r.h_real, r.h_imag, r.h_corr = _host_ptr(real), _host_ptr(imag), _host_ptr(corr)
        r.h_orient, r.O = orient.ctypes.data, int(orient.size)
        r.h_trans_x, r.h_trans_y, r.T = tx.ctypes.data, ty.ctypes.data, int(tx.size)
        r.h_diff2, r.h_min, r.h_argmin = _host_ptr(out_diff2), _host_ptr(out_min), _host_ptr(out_argmin)
        t = C.c_longlong()
        _check(lib().b200d2_server_submit(self._h, C.byref(r), C.byref(t)), "server_submit")
        self._keep[t.value] = (real, imag, corr, orient, tx, ty, out_diff2, out_min, out_argmin)
        return t.value

    def wait(self, ticket: int, timeout: float = 120.0):
        """Returns (status, latency_s, device_s) of the request."""
        lat, dev = C.c_double(), C.c_double()
        st = lib().b200d2_server_wait(self._h, ticket, timeout, C.byref(lat), C.byref(dev))
        self._keep.pop(ticket, None)
        return st, lat.value, dev.value

    def set_merging(self, max_requests: int = 8, max_particles: int = 512, max_request_particles: int = 128):
        """Merged admissions (b200d2_server_set_merging): queued requests on one
        reference run as one block-diagonal batch; max_requests=1 turns it off."""
        _check(lib().b200d2_server_set_merging(self._h, max_requests, max_particles, max_request_particles),
               "server_set_merging")

    def cancel(self, ticket: int) -> int:
        """Cancel a queued request (b200d2_server_cancel): 0, or the status code
        (ERR_UNSUPPORTED once it has been admitted, ERR_INVALID if unknown)."""
        return int(lib().b200d2_server_cancel(self._h, ticket))

    def stats(self) -> dict:
        s = ServerStats()
        _check(lib().b200d2_server_get_stats(self._h, C.byref(s)), "server_get_stats")
        return {n: getattr(s, n) for n, _ in ServerStats._fields_}

    def close(self):
        if self._h and self._h.value:
            lib().b200d2_server_destroy(self._h)
            self._h = C.c_void_p()
        self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def diff2_coarse_batch_static(view: View, batch: Batch, precision: int = PREC_BF16X3, stream=None):
    """The tensor-core batch on the library's fixed scratch (no device allocation).

    For callers that cannot allocate device memory.  This path never splits
    the contraction over k, so it needs the batch's workspace without the
    split-K partial-sum buffer, which can be less than
    batch_workspace_bytes() reports; a batch whose need exceeds
    STATIC_SCRATCH_BYTES is rejected (B200D2Error code 7).  Calls share the
    scratch, so they must not overlap on the GPU."""
    _check(lib().b200d2_diff2_coarse_batch_static(C.byref(view), C.byref(batch), precision, _stream(stream)),
           "diff2_coarse_batch_static")


def minloc(diff2, n: int, P: int, out_min=None, out_argmin=None, stream=None):
    _check(lib().b200d2_minloc(_ptr(diff2), n, P, _ptr(out_min), _ptr(out_argmin), _stream(stream)), "minloc")


def diff2_fine(view: View, eulers, real, imag, trans_x, trans_y, corr, diff2s, *, rot_idx, trans_idx, job_idx,
               job_num, image_size: int, sum_init: float = 0.0, stream=None):
    """Fine-pass diff2 over a job list (b200d2_diff2_fine); index tensors are
    CUDA int64 [jobs] (rot_idx / trans_idx indexed by job_idx)."""
    _check(lib().b200d2_diff2_fine(C.byref(view), _ptr(eulers), _ptr(real), _ptr(imag), _ptr(trans_x),
                                   _ptr(trans_y), _ptr(corr), _ptr(diff2s), image_size, sum_init,
                                   int(job_idx.numel()), _ptr(rot_idx), _ptr(trans_idx), _ptr(job_idx),
                                   _ptr(job_num), _stream(stream)), "diff2_fine")


def diff2_fine_cc(view: View, eulers, real, imag, trans_x, trans_y, corr, diff2s, *, rot_idx, trans_idx, job_idx,
                  job_num, image_size: int, stream=None):
    """CC form of the fine pass (b200d2_diff2_fine_cc): -cross / sqrt(norm)
    per (job, translation), written."""
    _check(lib().b200d2_diff2_fine_cc(C.byref(view), _ptr(eulers), _ptr(real), _ptr(imag), _ptr(trans_x),
                                      _ptr(trans_y), _ptr(corr), _ptr(diff2s), image_size, int(job_idx.numel()),
                                      _ptr(rot_idx), _ptr(trans_idx), _ptr(job_idx), _ptr(job_num),
                                      _stream(stream)), "diff2_fine_cc")


def coarse_weights(diff2, P: int, O: int, T: int, out_min=None, pdf_orient=None, pdf_offset=None,
                   normalize: bool = True, weights=None, sums=None, workspace=None, stream=None):
    """FP64 coarse weights pdf_o * pdf_t * exp(-(diff2 - min)) per particle
    (b200d2_coarse_weights).  diff2: CUDA float32 [P*O*T]; returns
    (weights [P, O, T] float64, sums [P] float64), normalised by the sums
    unless normalize is False."""
    import torch
    dev = diff2.device
    if weights is None:
        weights = torch.empty((P, O, T), dtype=torch.float64, device=dev)
    if sums is None:
        sums = torch.empty(P, dtype=torch.float64, device=dev)
    nb = lib().b200d2_coarse_weights_workspace(P, O * T)
    if workspace is None or workspace.numel() < nb:
        workspace = torch.empty(max(nb, 1), dtype=torch.uint8, device=dev)
    _check(lib().b200d2_coarse_weights(_ptr(diff2), P, O, T, _ptr(out_min), _ptr(pdf_orient), _ptr(pdf_offset),
                                       1 if normalize else 0, _ptr(weights), _ptr(sums), _ptr(workspace), nb,
                                       _stream(stream)), "coarse_weights")
    return weights, sums


def significance(weights, sums, adaptive_fraction: float, max_significants: int = 0, *, passed=True,
                 sig_weight=None, nsig=None, workspace=None, stream=None):
    """Significant samples per particle (b200d2_significance).  weights: CUDA
    float64 [P, n] (any shape with P rows); sums: CUDA float64 [P].  Returns
    (sig_weight [P] float64, nsig [P] int64, passed [P, n] uint8 or None):
    the threshold weight sorted[idx] of the positive weights in ascending
    order, the number of significant samples, and the mask w >= sig_weight."""
    import torch
    P = int(weights.shape[0])
    n = int(weights.numel() // max(P, 1))
    dev = weights.device
    if sig_weight is None:
        sig_weight = torch.empty(P, dtype=torch.float64, device=dev)
    if nsig is None:
        nsig = torch.empty(P, dtype=torch.int64, device=dev)
    mask = None
    if passed is True:
        mask = torch.empty((P, n), dtype=torch.uint8, device=dev)
    elif passed is not None and passed is not False:
        mask = passed
    nb = lib().b200d2_significance_workspace(P, n)
    if workspace is None or workspace.numel() < nb:
        workspace = torch.empty(max(nb, 1), dtype=torch.uint8, device=dev)
    _check(lib().b200d2_significance(_ptr(weights), P, n, _ptr(sums), float(adaptive_fraction), int(max_significants),
                                     _ptr(sig_weight), _ptr(nsig), _ptr(mask), _ptr(workspace), nb, _stream(stream)),
           "significance")
    return sig_weight, nsig, mask


def pack_mask(mask, out=None, stream=None):
    """Byte mask [P, n] (CUDA uint8) packed to bits (b200d2_pack_mask):
    returns CUDA int32 [P, (n + 31) // 32], sample 32 j + i of a row in bit i
    of its word j."""
    import torch
    P = int(mask.shape[0])
    n = int(mask.numel() // max(P, 1))
    if out is None:
        out = torch.empty((P, (n + 31) // 32), dtype=torch.int32, device=mask.device)
    _check(lib().b200d2_pack_mask(_ptr(mask), P, n, _ptr(out), _stream(stream)), "pack_mask")
    return out


def ctf_fold(real, imag, ctf_params: list, minvsigma2, *, imgX: int, imgY: int, maxR: int, ori_size: int,
             pixel_A: float, out_real=None, out_imag=None, out_corr=None, stream=None):
    """Fold each particle's CTF into its image and weights on the device
    (b200d2_ctf_fold).  real/imag: CUDA float32 [P, N_img]; ctf_params: P
    dicts of CTF fields; minvsigma2: CUDA float32 [N_img] (shared) or
    [P, N_img].  Returns (Fimg_real, Fimg_imag, corr)."""
    import torch
    P, N = int(real.shape[0]), int(real.shape[1])
    arr = (CTF * max(P, 1))()
    for i, c in enumerate(ctf_params):
        for k, v in c.items():
            setattr(arr[i], k, float(v))
    d_ctf = torch.frombuffer(bytearray(bytes(arr)), dtype=torch.uint8).to(real.device)
    out_real = torch.empty_like(real) if out_real is None else out_real
    out_imag = torch.empty_like(imag) if out_imag is None else out_imag
    out_corr = torch.empty_like(real) if out_corr is None else out_corr
    ms = 0 if minvsigma2.dim() == 1 else int(minvsigma2.stride(0))
    _check(lib().b200d2_ctf_fold(_ptr(real), _ptr(imag), int(real.stride(0)), P, N, imgX, imgY, maxR, ori_size,
                                 pixel_A, _ptr(d_ctf), _ptr(minvsigma2), ms, _ptr(out_real), _ptr(out_imag),
                                 _ptr(out_corr), _stream(stream)), "ctf_fold")
    if stream is None:
        torch.cuda.current_stream().synchronize()  # d_ctf is a temporary
    else:
        stream.synchronize()
    return out_real, out_imag, out_corr


COMBINE_DF32 = 0
COMBINE_FP64 = 1


def set_combine(mode: int) -> None:
    """Final combination of the tensor-core forms: COMBINE_DF32 (default,
    double-float) or COMBINE_FP64."""
    _check(lib().b200d2_set_combine(mode), "set_combine")


def set_batch_graphs(enable: bool) -> None:
    """CUDA graphs of the batch entry point (on by default): the second call
    with the same arguments captures the pipeline, later ones launch it."""
    _check(lib().b200d2_set_batch_graphs(1 if enable else 0), "set_batch_graphs")


def set_operand_gen(mode: int) -> None:
    """A operand of the contraction: 0 (default) materialised in the workspace
    by its own kernel, 1 generated in shared memory inside the contraction
    (bit-identical results).  Query workspace sizes after setting it."""
    _check(lib().b200d2_set_operand_gen(int(mode)), "set_operand_gen")


def set_projection_cache(enable: bool) -> None:
    """Projection cache of the single-particle tensor-core call (on by
    default): calls whose Euler matrices equal the last projected ones (bit
    for bit, checked on the device) reuse those projections."""
    _check(lib().b200d2_set_projection_cache(1 if enable else 0), "set_projection_cache")


def set_wait_limit_ns(ns: int) -> None:
    """Test hook: limit (ns) of the single-CTA contraction's pipeline waits;
    0 restores the default (4 s).  A short limit makes correct runs give up
    with B200D2_ERR_TIMEOUT in the workspace status word."""
    _check(lib().b200d2_set_wait_limit_ns(int(ns)), "set_wait_limit_ns")


def set_gemm_variant(row_bytes: int = 0, tile_n: int = 0, split: int = 0, pair: int = 0) -> None:
    """Contraction variant of the batch entry points (0 = default; pair: 1 =
    CTA-pair 256 x 256 tiles, 2 = single-CTA tiles)."""
    _check(lib().b200d2_set_gemm_variant(row_bytes, tile_n, split, pair), "set_gemm_variant")


def stage_names(precision: int) -> list[str]:
    out, i = [], 0
    while True:
        n = lib().b200d2_stage_name(precision, i)
        if not n:
            return out
        out.append(n.decode())
        i += 1


def kernel_breakdown(view: View, batch: Batch, precision: int, workspace=None, stream=None, reps: int = 3) -> dict:
    """Time each pipeline stage (one kernel each) with CUDA events on `stream`.

    Runs every stage in order `reps` times (the outputs accumulate; callers
    reset them afterwards if they need the values)."""
    import torch
    st = stream if stream is not None else torch.cuda.current_stream()
    names = stage_names(precision)
    ws = _ptr(workspace) if workspace is not None else None
    nbytes = workspace.numel() * workspace.element_size() if workspace is not None else 0
    acc = {n: 0.0 for n in names}
    for _ in range(reps):
        for i, n in enumerate(names):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(st)
            _check(lib().b200d2_diff2_coarse_batch_stage(C.byref(view), C.byref(batch), precision, i, ws, nbytes,
                                                         _stream(st)), "batch_stage")
            b.record(st)
            b.synchronize()
            acc[n] += a.elapsed_time(b)
    per = {n: v / reps for n, v in acc.items()}
    dom = max(per, key=per.get) if per else None
    return {"per_kernel_ms": per, "dominant": dom, "dominant_ms": per.get(dom) if dom else None, "traffic": None}


def workspace_status(workspace, stream=None) -> int:
    """0, or B200D2_ERR_TIMEOUT if a bounded device wait of the last tensor-core run gave up."""
    st = C.c_int(-1)
    _check(lib().b200d2_workspace_status(_ptr(workspace), _stream(stream), C.byref(st)), "workspace_status")
    return st.value
