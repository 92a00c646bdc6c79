"""ctypes front end of the C oracle (oracle/diff2_oracle.c).

TEST INFRASTRUCTURE ONLY: used by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py as the checker.  The product library never
imports this module.

Also exposes, when present, the reference project's own CUDA kernels compiled
into oracle/_ref/libref_diff2.so (see oracle/ref_shim.cu) for GPU-side
parity tests.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref_diff2.so")

INTERP_EXACT = 0
INTERP_TEX_ROUND = 1
INTERP_TEX_TRUNC = 2


class OrcProjector(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("mdlX", "mdlY", "mdlZ", "mdlInitY", "mdlInitZ", "mdlMaxR")] + [
        ("padding_factor", C.c_float)] + [
        (n, C.c_int) for n in ("imgX", "imgY", "imgZ", "maxR", "maxR2", "maxR2_padded")] + [
        ("re", C.c_void_p), ("im", C.c_void_p)]


_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, os.path.join(HERE, "liboracle.so")], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.c_void_p
        L.orc_projector_init.argtypes = [C.POINTER(OrcProjector)] + [C.c_int] * 6 + [C.c_float, P, P] + [C.c_int] * 4
        L.orc_project_pixels.argtypes = [C.POINTER(OrcProjector), P, C.c_long, P, P, C.c_long, C.c_int, P, P, C.c_int]
        L.orc_diff2_coarse_f64.argtypes = [C.POINTER(OrcProjector), P, C.c_long, P, P, C.c_long, P, P, P,
                                           C.c_long, C.c_int, P, C.c_int]
        L.orc_diff2_coarse_f32.argtypes = [C.POINTER(OrcProjector), P, C.c_long, P, P, C.c_long, P, P, P,
                                           C.c_long, P, C.c_int]
        L.orc_filter_image.argtypes = [C.POINTER(OrcProjector), P, P, P, C.c_long, P, P, P, P]
        L.orc_filter_image.restype = C.c_long
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


class Projector:
    """Oracle-side projector: keeps the volume arrays alive for the C struct."""

    def __init__(self, pv, imgX: int, imgY: int, imgMaxR: int, imgZ: int = 1):
        self.re = np.ascontiguousarray(pv.re, dtype=np.float32)
        self.im = np.ascontiguousarray(pv.im, dtype=np.float32)
        self.s = OrcProjector()
        lib().orc_projector_init(C.byref(self.s), pv.mdlX, pv.mdlY, pv.mdlZ, pv.mdlInitY, pv.mdlInitZ,
                                 pv.mdlMaxR, pv.padding_factor, _p(self.re), _p(self.im),
                                 imgX, imgY, imgZ, imgMaxR)

    @property
    def maxR(self) -> int:
        return self.s.maxR

    @property
    def maxR2_padded(self) -> int:
        return self.s.maxR2_padded


def projector_for(prob) -> Projector:
    return Projector(prob.projector, prob.imgX, prob.imgY, prob.imgMaxR)


def project_pixels(proj: Projector, eulers: np.ndarray, px: np.ndarray, py: np.ndarray,
                   mode: int = INTERP_TEX_ROUND, nthreads: int = 0):
    eulers = np.ascontiguousarray(eulers, np.float32)
    px = np.ascontiguousarray(px, np.int32)
    py = np.ascontiguousarray(py, np.int32)
    O, K = eulers.shape[0], px.size
    re = np.zeros((O, K), np.float64)
    im = np.zeros((O, K), np.float64)
    lib().orc_project_pixels(C.byref(proj.s), _p(eulers), O, _p(px), _p(py), K, mode, _p(re), _p(im), nthreads)
    return re, im


def diff2_coarse_f64(proj: Projector, eulers, trans_x, trans_y, fre, fim, corr,
                     mode: int = INTERP_TEX_ROUND, diff2_init=None, nthreads: int = 0) -> np.ndarray:
    """FP64 restatement of cuda_kernel_diff2_coarse for one particle -> [O, T]."""
    eulers = np.ascontiguousarray(eulers, np.float32)
    tx = np.ascontiguousarray(trans_x, np.float32)
    ty = np.ascontiguousarray(trans_y, np.float32)
    fre = np.ascontiguousarray(fre, np.float32)
    fim = np.ascontiguousarray(fim, np.float32)
    corr = np.ascontiguousarray(corr, np.float32)
    O, T, N = eulers.shape[0], tx.size, fre.size
    out = np.zeros((O, T), np.float64) if diff2_init is None else np.array(diff2_init, np.float64).reshape(O, T)
    lib().orc_diff2_coarse_f64(C.byref(proj.s), _p(eulers), O, _p(tx), _p(ty), T, _p(fre), _p(fim), _p(corr),
                               N, mode, _p(out), nthreads)
    return out


def diff2_from_projections(proj: Projector, prj_re, prj_im, trans_x, trans_y, fre, fim, corr,
                           nthreads: int = 0) -> np.ndarray:
    """FP64 coarse diff2 with given projections prj[o][i] over all image pixels -> [O, T]."""
    L = lib()
    P_ = C.c_void_p
    L.orc_diff2_from_projections.argtypes = [C.POINTER(OrcProjector), P_, P_, C.c_long, P_, P_, C.c_long, P_, P_,
                                             P_, C.c_long, P_, C.c_int]
    prj_re = np.ascontiguousarray(prj_re, np.float32)
    prj_im = np.ascontiguousarray(prj_im, np.float32)
    tx = np.ascontiguousarray(trans_x, np.float32)
    ty = np.ascontiguousarray(trans_y, np.float32)
    fre = np.ascontiguousarray(fre, np.float32)
    fim = np.ascontiguousarray(fim, np.float32)
    corr = np.ascontiguousarray(corr, np.float32)
    O, T, N = prj_re.shape[0], tx.size, fre.size
    out = np.zeros((O, T), np.float64)
    L.orc_diff2_from_projections(C.byref(proj.s), _p(prj_re), _p(prj_im), O, _p(tx), _p(ty), T, _p(fre), _p(fim),
                                 _p(corr), N, _p(out), nthreads)
    return out


def diff2_coarse_f32(proj: Projector, eulers, trans_x, trans_y, fre, fim, corr,
                     diff2_init=None, nthreads: int = 0) -> np.ndarray:
    """FP32 port of cuda_kernel_diff2_coarse (the CPU baseline) -> [O, T] float32."""
    eulers = np.ascontiguousarray(eulers, np.float32)
    tx = np.ascontiguousarray(trans_x, np.float32)
    ty = np.ascontiguousarray(trans_y, np.float32)
    fre = np.ascontiguousarray(fre, np.float32)
    fim = np.ascontiguousarray(fim, np.float32)
    corr = np.ascontiguousarray(corr, np.float32)
    O, T, N = eulers.shape[0], tx.size, fre.size
    out = np.zeros((O, T), np.float32) if diff2_init is None else np.array(diff2_init, np.float32).reshape(O, T)
    lib().orc_diff2_coarse_f32(C.byref(proj.s), _p(eulers), O, _p(tx), _p(ty), T, _p(fre), _p(fim), _p(corr),
                               N, _p(out), nthreads)
    return out


def cc_coarse_f64(proj: Projector, eulers, trans_x, trans_y, fre, fim, corr, projections=None) -> np.ndarray:
    """FP64 restatement of cuda_kernel_diff2_CC_coarse (src/diff2.cuh:691-809)
    for one particle: cc[o][t] = -sum corr Re(conj(A_o) S_t) / sqrt(sum corr
    |A_o|^2) over the pixels inside the projector radius (elsewhere A = 0).
    Projections are the oracle's (project3Dmodel restatement); the phase shift
    is translatePixel's (src/cuda_device_utils.cuh:110-129) in FP64.
    projections: optional (re, im) [O][N_img] samples to use instead (e.g.
    the texture unit's own, to compare arithmetic without the texture-weight
    model)."""
    v = proj.s
    n = fre.size
    x = np.arange(n) % v.imgX
    y = np.arange(n) // v.imgX
    y = np.where(y > v.maxR, y - v.imgY, y)
    # every pixel is projected (0 outside the radius), so the sums are exact
    inside = np.ones(n, bool)
    px, py = x.astype(np.int32), y.astype(np.int32)
    O = eulers.reshape(-1, 9).shape[0]
    ar, ai = project_pixels(proj, eulers, px, py) if projections is None else projections
    ar = ar.reshape(O, -1).astype(np.float64)
    ai = ai.reshape(O, -1).astype(np.float64)
    w = np.asarray(corr, np.float64)[inside]
    xr = np.asarray(fre, np.float64)[inside]
    xi = np.asarray(fim, np.float64)[inside]
    ph = np.outer(np.asarray(trans_x, np.float64), px) + np.outer(np.asarray(trans_y, np.float64), py)
    c, s = np.cos(ph), np.sin(ph)
    sr = c * xr - s * xi  # [T][K]
    si = c * xi + s * xr
    cross = (ar * w) @ sr.T + (ai * w) @ si.T  # [O][T]
    norm = (ar * ar + ai * ai) @ w
    return -cross / np.sqrt(norm)[:, None]


def filter_image(proj: Projector, fre, fim, corr):
    """FilterCoarseParamImage restatement -> (re, im, corr, coor_xy, n_inside)."""
    N = fre.size
    fre = np.ascontiguousarray(fre, np.float32)
    fim = np.ascontiguousarray(fim, np.float32)
    corr = np.ascontiguousarray(corr, np.float32)
    ore, oim, oc = np.zeros(N, np.float32), np.zeros(N, np.float32), np.zeros(N, np.float32)
    oxy = np.zeros(2 * N, np.float32)
    n = lib().orc_filter_image(C.byref(proj.s), _p(fre), _p(fim), _p(corr), N, _p(ore), _p(oim), _p(oc), _p(oxy))
    return ore, oim, oc, oxy, int(n)


# --------------------------------------------------------------------------
# error statistics (restatement of ErrorComparator / check_array_equal,
# reference src/check.cuh:11-148: |ref| <= 1e-12 skipped for relative error)
# --------------------------------------------------------------------------
def error_stats(test: np.ndarray, ref: np.ndarray) -> dict:
    a = np.asarray(test, np.float64).ravel()
    b = np.asarray(ref, np.float64).ravel()
    ae = np.abs(a - b)
    m = np.abs(b) > 1e-12
    re = ae[m] / np.abs(b[m])
    return dict(count=int(a.size), count_rel=int(m.sum()),
                sum_abs=float(ae.sum()), max_abs=float(ae.max(initial=0.0)),
                avg_abs=float(ae.mean()) if a.size else 0.0,
                sum_rel=float(re.sum()), max_rel=float(re.max(initial=0.0)),
                avg_rel=float(re.mean()) if re.size else 0.0)


def weights_from_diff2(d: np.ndarray) -> tuple[float, np.ndarray]:
    """Per-particle minimum and normalised exp(-(diff2 - min)) weights in FP64."""
    d = np.asarray(d, np.float64).ravel()
    mn = float(d.min())
    w = np.exp(-(d - mn))
    return mn, w / w.sum()


def significance(w: np.ndarray, total: float, adaptive_fraction: float, max_significants: int = 0):
    """Significant samples of one particle's weights, RELION's pass-0 steps
    around the reference's cuda_kernel_find_threshold_idx_in_cumulative and
    cuda_kernel_array_over_threshold (src/cuda_device_utils.cuh:238-266):
    keep the weights > 0 (finite), sort them ascending, take inclusive
    cumulative sums c_k, idx = i + 1 for the i with c_i <= thr < c_{i+1}
    (else 0) at thr = (1 - adaptive_fraction) * total, nsig = count - idx
    capped at max_significants (idx = count - nsig), threshold weight
    sorted[idx], mask w >= threshold.

    The cumulative sums are exact: every double is an integer multiple of a
    common power of two, added as Python integers.  Returns (sig_weight,
    nsig, passed, margin), margin = min |c_k - thr| / max(|c_k|, |thr|) over
    the two sums either side of the crossing (how far the decision is from a
    tie)."""
    import bisect
    import itertools
    w = np.asarray(w, np.float64).ravel()
    pos = np.sort(w[(w > 0) & np.isfinite(w)])
    cnt = int(pos.size)
    if cnt == 0:
        return float("inf"), 0, np.zeros(w.size, np.uint8), float("inf")
    thr = float(np.float64(1.0 - adaptive_fraction) * np.float64(total))
    mant, expo = np.frexp(pos)
    M = (mant * 2.0 ** 53).astype(np.int64)
    E = expo.astype(np.int64) - 53
    tm, te = np.frexp(thr)
    tM, tE = int(tm * 2.0 ** 53), int(te) - 53
    base = int(min(E.min(), tE))
    vals = [int(m) << int(e - base) for m, e in zip(M.tolist(), E.tolist())]
    cum = list(itertools.accumulate(vals))
    thr_i = tM << (tE - base) if tM >= 0 else -((-tM) << (tE - base))
    k = bisect.bisect_right(cum, thr_i)  # number of c_i <= thr
    idx = k if 1 <= k <= cnt - 1 else 0
    # distance of the decision from a tie, relative to the sums compared
    margin = min((abs(cum[j] - thr_i) / max(abs(cum[j]), abs(thr_i)) for j in (k - 1, k) if 0 <= j < cnt),
                 default=float("inf"))
    nsig = cnt - idx
    if max_significants > 0 and nsig > max_significants:
        nsig = int(max_significants)
        idx = cnt - nsig
    sig = float(pos[idx])
    return sig, nsig, (w >= sig).astype(np.uint8), margin


# --------------------------------------------------------------------------
# the reference project's own kernels (GPU), compiled into oracle/_ref
# --------------------------------------------------------------------------
_ref = None


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


def ref_lib():
    global _ref
    if _ref is None:
        L = C.CDLL(REF_PATH)
        P = C.c_void_p
        L.refshim_projector_create.argtypes = [C.c_int] * 6 + [C.c_float, P, P]
        L.refshim_projector_create.restype = P
        L.refshim_projector_destroy.argtypes = [P]
        L.refshim_diff2_coarse.argtypes = [P] + [C.c_int] * 4 + [P] * 7 + [C.c_long] * 3 + [P]
        if hasattr(L, "refshim_diff2_coarse_cc"):
            L.refshim_diff2_coarse_cc.argtypes = [P] + [C.c_int] * 4 + [P] * 7 + [C.c_long] * 3 + [P]
        L.refshim_diff2_coarse_double.argtypes = [P] + [C.c_int] * 4 + [P] * 7 + [C.c_long] * 3 + [C.c_int, P]
        L.refshim_variant_workspace_bytes.argtypes = [C.c_int] * 6
        L.refshim_variant_workspace_bytes.restype = C.c_size_t
        L.refshim_variant_run.argtypes = [C.c_int, P] + [C.c_int] * 4 + [P] * 9 + [C.c_int] * 5 + [P]
        if hasattr(L, "refshim_find_threshold_idx"):
            L.refshim_find_threshold_idx.argtypes = [P, C.c_double, C.c_long, P, P]
            L.refshim_array_over_threshold.argtypes = [P, P, C.c_double, C.c_long, P]
        if hasattr(L, "refshim_diff2_fine"):
            L.refshim_diff2_fine.argtypes = ([P] + [C.c_int] * 4 + [P] * 7 + [C.c_long, C.c_float] + [C.c_long] * 3 +
                                             [P] * 4 + [P])
        if hasattr(L, "refshim_diff2_fine_cc"):
            L.refshim_diff2_fine_cc.argtypes = ([P] + [C.c_int] * 4 + [P] * 7 + [C.c_long] * 4 + [P] * 4 + [P])
        _ref = L
    return _ref


def tex_sample(vol: np.ndarray, uvw: np.ndarray, mode: int = INTERP_TEX_ROUND) -> np.ndarray:
    """Emulated tex3D (linear filter, clamp, unnormalised) of vol [Z][Y][X] at uvw [n, 3]."""
    L = lib()
    L.orc_tex_sample.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_long, C.c_int, C.c_void_p]
    vol = np.ascontiguousarray(vol, np.float32)
    uvw = np.ascontiguousarray(uvw, np.float32)
    out = np.zeros(uvw.shape[0], np.float64)
    Z, Y, X = vol.shape
    L.orc_tex_sample(_p(vol), X, Y, Z, _p(uvw), uvw.shape[0], mode, _p(out))
    return out
