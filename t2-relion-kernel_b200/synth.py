"""Seeded synthetic coarse-pass workloads.

The reference benchmarks replay RELION dumps (Zenodo record 15283628) that are
not available here; these generators stand in for them with the shapes, sizes
and value distributions of the five workloads this library is measured on:

  c1  64^3 volume, image 32 (N_img 544, ~418 in-radius), HEALPix order 1 x 12 psi
      = 576 orientations, 21 translations (x^2+y^2 <= 5), 8 particles, SNR 0.1, no CTF
  c2  128^3 volume, image 64 (N_img 2112, ~1640 in-radius), order 2 x 24 psi = 4608,
      113 translations (radius 6), 256 particles, SNR 0.05, per-particle CTF
  c3  256^3 volume, image 96, order 3 x 48 psi = 36864, 49 translations (radius 4),
      64 particles, SNR 0.02, CTF
  c4  the c2 setup with 1024 particles, each with a contiguous HEALPix
      neighbourhood of 10-100 % of the 4608 orientations and a translation radius
      drawn from {2..8} (13..197 translations)

Physical model.  The reference volume is a sum of 20 Gaussian blobs (centres
uniform in a ball of radius 20 px at box 64, sigma U(2,5) px, amplitude
U(0.5,1); radii scale with the box).  It is zero-padded by the padding factor,
Fourier transformed, and stored as RELION's padded Hermitian-half projector
array: pad_size = 2*(pf*r_max + 1) + 1, x dimension pad_size//2 + 1 starting at
0, y and z dimensions pad_size centred (init = -(pf*r_max + 1)), coefficients
beyond radius pf*r_max zeroed.  Particles are central slices at a grid
orientation, shifted by a grid translation, multiplied by a CTF and corrupted by
complex Gaussian noise of variance sigma^2(r) = c*exp(-r/8), with c set by the
SNR.  The kernel inputs are then folded the way RELION folds them before the
coarse kernel: Fimg = X / CTF where |CTF| > 1e-8, corr = Minvsigma2 * CTF^2,
Minvsigma2 = 1/sigma^2(r).  Translations are phase slopes
trans = -2*pi*shift/ori_size.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

try:  # package-relative when loaded as a package, plain when on sys.path
    from . import healpix
except ImportError:  # pragma: no cover
    import healpix  # type: ignore


# --------------------------------------------------------------------------
# data containers
# --------------------------------------------------------------------------
@dataclass
class ProjectorVolume:
    """Padded Hermitian-half Fourier volume, arrays [mdlZ][mdlY][mdlX] float32."""

    re: np.ndarray
    im: np.ndarray
    mdlX: int
    mdlY: int
    mdlZ: int
    mdlInitY: int
    mdlInitZ: int
    mdlMaxR: int
    padding_factor: float
    ori_size: int


@dataclass
class CoarseProblem:
    name: str
    projector: ProjectorVolume
    img_size: int  # coarse box size S
    imgX: int
    imgY: int
    imgMaxR: int
    eulers: np.ndarray  # [O, 9] float32
    trans_x: np.ndarray  # [T] float32 phase slopes
    trans_y: np.ndarray
    shifts: np.ndarray  # [T, 2] pixel shifts
    fimg_re: np.ndarray  # [P, N_img] float32 (CTF-folded)
    fimg_im: np.ndarray
    corr: np.ndarray  # [P, N_img] float32 (Minvsigma2 * CTF^2)
    true_orient: np.ndarray  # [P]
    true_trans: np.ndarray  # [P]
    # uneven batches: per-particle orientation index lists and translation lists
    orient_lists: list | None = None
    trans_lists: list | None = None
    meta: dict = field(default_factory=dict)

    @property
    def N_img(self) -> int:
        return self.imgX * self.imgY

    @property
    def O(self) -> int:
        return int(self.eulers.shape[0])

    @property
    def T(self) -> int:
        return int(self.trans_x.shape[0])

    @property
    def P(self) -> int:
        return int(self.fimg_re.shape[0])

    def evals(self) -> int:
        if self.orient_lists is not None:
            return int(sum(len(o) * len(t) for o, t in zip(self.orient_lists, self.trans_lists)))
        return self.P * self.O * self.T


CONFIGS = {
    # small fixture-sized case (box 16, 72 orientations, 9 translations, CTF on)
    "g0": dict(box=16, img=16, pf=2, order=0, n_psi=6, r2_trans=2, P=2, snr=0.1, ctf=True),
    "tiny": dict(box=32, img=16, pf=2, order=0, n_psi=6, r2_trans=2, P=3, snr=0.1, ctf=False),
    "c1": dict(box=64, img=32, pf=2, order=1, n_psi=12, r2_trans=5, P=8, snr=0.1, ctf=False),
    "c2": dict(box=128, img=64, pf=2, order=2, n_psi=24, r2_trans=36, P=256, snr=0.05, ctf=True),
    "c3": dict(box=256, img=96, pf=2, order=3, n_psi=48, r2_trans=16, P=64, snr=0.02, ctf=True),
    "c4": dict(box=128, img=64, pf=2, order=2, n_psi=24, r2_trans=64, P=1024, snr=0.05, ctf=True,
               uneven=True),
    # serving: three resident references (coarse sizes 48 / 64 / 96 from 96^3,
    # 128^3, 192^3 volumes), a 512-particle pool each; requests take subsets
    "c5s": dict(box=96, img=48, pf=2, order=2, n_psi=24, r2_trans=36, P=512, snr=0.05, ctf=True),
    "c5m": dict(box=128, img=64, pf=2, order=2, n_psi=24, r2_trans=36, P=512, snr=0.05, ctf=True),
    "c5l": dict(box=192, img=96, pf=2, order=2, n_psi=24, r2_trans=36, P=512, snr=0.05, ctf=True),
}


# --------------------------------------------------------------------------
# reference volume and projector
# --------------------------------------------------------------------------
def blob_volume(box: int, rng: np.random.Generator, n_blobs: int = 20) -> np.ndarray:
    scale = box / 64.0
    vol = np.zeros((box, box, box), dtype=np.float64)
    ax = np.arange(box, dtype=np.float64) - box / 2
    for _ in range(n_blobs):
        while True:  # uniform in a ball of radius 20 px (at box 64)
            c = rng.uniform(-1, 1, 3)
            if c @ c <= 1:
                break
        c = c * 20.0 * scale
        sig = rng.uniform(2.0, 5.0) * scale
        amp = rng.uniform(0.5, 1.0)
        gz = np.exp(-((ax - c[2]) ** 2) / (2 * sig * sig))
        gy = np.exp(-((ax - c[1]) ** 2) / (2 * sig * sig))
        gx = np.exp(-((ax - c[0]) ** 2) / (2 * sig * sig))
        vol += amp * gz[:, None, None] * gy[None, :, None] * gx[None, None, :]
    return vol


def projector_from_volume(vol: np.ndarray, pf: int, coarse_r: int) -> ProjectorVolume:
    n = vol.shape[0]
    m = pf * n
    padded = np.zeros((m, m, m), dtype=np.float64)
    o = (m - n) // 2
    padded[o:o + n, o:o + n, o:o + n] = vol
    f = np.fft.rfftn(np.fft.ifftshift(padded)) / float(m) ** 3  # [kz, ky, kx]
    r_max = n // 2
    pr = pf * r_max
    pad_size = 2 * (pr + 1) + 1
    mdlX = pad_size // 2 + 1
    mdlY = mdlZ = pad_size
    init = -(pr + 1)
    kx = np.arange(mdlX)
    ky = np.arange(mdlY) + init
    kz = np.arange(mdlZ) + init
    data = f[np.mod(kz, m)[:, None, None], np.mod(ky, m)[None, :, None],
             np.minimum(kx, m // 2)[None, None, :]]
    r2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    data = np.where(r2 <= pr * pr, data, 0)
    # scale so the RMS of the coefficients inside the coarse radius is 1
    sel = r2 <= (pf * coarse_r) ** 2
    rms = math.sqrt(float(np.mean(np.abs(data[sel]) ** 2)))
    data = data / rms
    return ProjectorVolume(
        re=np.ascontiguousarray(data.real.astype(np.float32)),
        im=np.ascontiguousarray(data.imag.astype(np.float32)),
        mdlX=mdlX, mdlY=mdlY, mdlZ=mdlZ, mdlInitY=init, mdlInitZ=init,
        mdlMaxR=r_max, padding_factor=float(pf), ori_size=n)


def pixel_coords(imgX: int, imgY: int, maxR: int) -> tuple[np.ndarray, np.ndarray]:
    """pixel_index2coor for all half-plane pixels (reference src/diff2.cuh:182-188)."""
    idx = np.arange(imgX * imgY)
    x = idx % imgX
    y = idx // imgX
    y = np.where(y > maxR, y - imgY, y)
    return x.astype(np.int32), y.astype(np.int32)


def _trilinear(vol: np.ndarray, u: np.ndarray, v: np.ndarray, w: np.ndarray) -> np.ndarray:
    x0 = np.floor(u).astype(np.int64)
    y0 = np.floor(v).astype(np.int64)
    z0 = np.floor(w).astype(np.int64)
    fx, fy, fz = u - x0, v - y0, w - z0
    nz, ny, nx = vol.shape

    def g(z, y, x):
        return vol[np.clip(z, 0, nz - 1), np.clip(y, 0, ny - 1), np.clip(x, 0, nx - 1)].astype(np.float64)

    c00 = g(z0, y0, x0) * (1 - fx) + g(z0, y0, x0 + 1) * fx
    c10 = g(z0, y0 + 1, x0) * (1 - fx) + g(z0, y0 + 1, x0 + 1) * fx
    c01 = g(z0 + 1, y0, x0) * (1 - fx) + g(z0 + 1, y0, x0 + 1) * fx
    c11 = g(z0 + 1, y0 + 1, x0) * (1 - fx) + g(z0 + 1, y0 + 1, x0 + 1) * fx
    c0 = c00 * (1 - fy) + c10 * fy
    c1 = c01 * (1 - fy) + c11 * fy
    return c0 * (1 - fz) + c1 * fz


def project_exact(pv: ProjectorVolume, euler9: np.ndarray, x: np.ndarray, y: np.ndarray,
                  maxR: int) -> np.ndarray:
    """Central slice by exact trilinear interpolation in float64 (generator only)."""
    e = euler9.astype(np.float64)
    pf = pv.padding_factor
    xp = (e[0] * x + e[1] * y) * pf
    yp = (e[3] * x + e[4] * y) * pf
    zp = (e[6] * x + e[7] * y) * pf
    inside = (xp * xp + yp * yp + zp * zp) <= (maxR * pf) ** 2
    neg = xp < 0
    sgn = np.where(neg, -1.0, 1.0)
    xp, yp, zp = xp * sgn, yp * sgn, zp * sgn
    re = _trilinear(pv.re, xp, yp - pv.mdlInitY, zp - pv.mdlInitZ)
    im = _trilinear(pv.im, xp, yp - pv.mdlInitY, zp - pv.mdlInitZ) * sgn
    out = (re + 1j * im)
    return np.where(inside, out, 0)


def translation_grid(r2max: int) -> np.ndarray:
    r = int(math.isqrt(r2max))
    pts = [(sx, sy) for sy in range(-r, r + 1) for sx in range(-r, r + 1) if sx * sx + sy * sy <= r2max]
    return np.array(pts, dtype=np.float64)


def ctf_values(x: np.ndarray, y: np.ndarray, ori_size: int, defocus_A: float,
               pixel_A: float = 1.5, kv: float = 300.0, cs_mm: float = 2.7,
               amp_contrast: float = 0.1) -> np.ndarray:
    volt = kv * 1e3
    lam = 12.2643247 / math.sqrt(volt * (1.0 + volt * 0.978466e-6))
    cs = cs_mm * 1e7
    k2 = (x.astype(np.float64) ** 2 + y.astype(np.float64) ** 2) / (ori_size * pixel_A) ** 2
    chi = math.pi * lam * defocus_A * k2 - 0.5 * math.pi * cs * lam ** 3 * k2 * k2
    q = amp_contrast
    return -(math.sqrt(1 - q * q) * np.sin(chi) + q * np.cos(chi))


def _noise_model(x, y, snr, signal_pow):
    r = np.sqrt(x.astype(np.float64) ** 2 + y.astype(np.float64) ** 2)
    shape = np.exp(-r / 8.0)
    c = signal_pow / (snr * shape.sum())
    return c * shape


def write_projector_dat(path: str, pv: ProjectorVolume) -> None:
    """projector_proc_*.dat: int32 {mdlX, mdlY, mdlZ, mdlInitY, mdlInitZ, mdlMaxR},
    float32 padding_factor, float32 real[mdlX*mdlY*mdlZ], imag[...] (x fastest)
    (reference reader: src/acc_projector_impl.h:300-334)."""
    with open(path, "wb") as f:
        np.array([pv.mdlX, pv.mdlY, pv.mdlZ, pv.mdlInitY, pv.mdlInitZ, pv.mdlMaxR], np.int32).tofile(f)
        np.array([pv.padding_factor], np.float32).tofile(f)
        np.ascontiguousarray(pv.re, np.float32).tofile(f)
        np.ascontiguousarray(pv.im, np.float32).tofile(f)


def write_coarse_dat(path: str, prob: CoarseProblem, p: int, diff2_init: np.ndarray | None = None) -> None:
    """coarse_data*.dat for particle p: int32 {xdim, ydim, zdim, rmax, T, O, image_size},
    float32 eulers[9*O], trans[2*T] (x block then y block), fimg[2*N] (real block
    then imag block), corr[N], diff2s[O*T] (reference reader: src/main.cu:153-191)."""
    N = prob.N_img
    d2 = np.zeros(prob.O * prob.T, np.float32) if diff2_init is None else np.asarray(diff2_init, np.float32)
    with open(path, "wb") as f:
        np.array([prob.imgX, prob.imgY, 1, prob.imgMaxR, prob.T, prob.O, N], np.int32).tofile(f)
        np.ascontiguousarray(prob.eulers, np.float32).tofile(f)
        np.concatenate([prob.trans_x, prob.trans_y]).astype(np.float32).tofile(f)
        np.concatenate([prob.fimg_re[p], prob.fimg_im[p]]).astype(np.float32).tofile(f)
        np.ascontiguousarray(prob.corr[p], np.float32).tofile(f)
        d2.reshape(-1).tofile(f)


def read_coarse_dat(path: str) -> dict:
    """Inverse of write_coarse_dat (same layout as the reference's replay files)."""
    with open(path, "rb") as f:
        hdr = np.fromfile(f, np.int32, 7)
        xdim, ydim, zdim, rmax, T, O, N = (int(v) for v in hdr)
        eul = np.fromfile(f, np.float32, 9 * O).reshape(O, 9)
        tr = np.fromfile(f, np.float32, 2 * T)
        fimg = np.fromfile(f, np.float32, 2 * N)
        corr = np.fromfile(f, np.float32, N)
        d2 = np.fromfile(f, np.float32, O * T)
    return dict(xdim=xdim, ydim=ydim, zdim=zdim, rmax=rmax, T=T, O=O, image_size=N, eulers=eul,
                trans_x=tr[:T], trans_y=tr[T:], fimg_re=fimg[:N], fimg_im=fimg[N:], corr=corr, diff2s=d2)


def make_problem(name: str = "c1", seed: int = 20251203, P: int | None = None,
                 orient_limit: int | None = None) -> CoarseProblem:
    """Build a seeded synthetic coarse-pass problem.

    `P` overrides the particle count and `orient_limit` keeps only the first
    orientations (used for bounded CPU samples and small parity cases).
    """
    cfg = dict(CONFIGS[name])
    rng = np.random.default_rng(seed)
    box, S, pf = cfg["box"], cfg["img"], cfg["pf"]
    vol = blob_volume(box, rng)
    pv = projector_from_volume(vol, pf, S // 2)
    eulers, _ = healpix.orientation_grid(cfg["order"], cfg["n_psi"])
    if orient_limit is not None:
        eulers = eulers[:orient_limit]
    shifts = translation_grid(cfg["r2_trans"])
    imgX, imgY, imgMaxR = S // 2 + 1, S, S // 2
    maxR = min(pv.mdlMaxR, imgMaxR)
    x, y = pixel_coords(imgX, imgY, maxR)
    nP = cfg["P"] if P is None else P
    O, T, N = eulers.shape[0], shifts.shape[0], imgX * imgY
    tx = (-2.0 * math.pi * shifts[:, 0] / pv.ori_size).astype(np.float32)
    ty = (-2.0 * math.pi * shifts[:, 1] / pv.ori_size).astype(np.float32)

    orient_lists = trans_lists = None
    if cfg.get("uneven"):
        dirs = healpix.direction_vectors(cfg["order"])
        n_psi = cfg["n_psi"]
        orient_lists, trans_lists = [], []

    fre = np.zeros((nP, N), np.float32)
    fim = np.zeros((nP, N), np.float32)
    corr = np.zeros((nP, N), np.float32)
    true_o = np.zeros(nP, np.int64)
    true_t = np.zeros(nP, np.int64)
    for p in range(nP):
        if orient_lists is not None:
            frac = rng.uniform(0.1, 1.0)
            centre = dirs[rng.integers(dirs.shape[0])]
            nd = max(1, int(round(frac * dirs.shape[0])))
            near = np.sort(np.argsort(-(dirs @ centre), kind="stable")[:nd])
            olist = (near[:, None] * n_psi + np.arange(n_psi)[None, :]).reshape(-1)
            rad = int(rng.integers(2, 9))
            tl = translation_grid(rad * rad)
            orient_lists.append(olist.astype(np.int32))
            trans_lists.append(np.stack([-2.0 * math.pi * tl[:, 0] / pv.ori_size,
                                         -2.0 * math.pi * tl[:, 1] / pv.ori_size], 1).astype(np.float32))
            o_t = int(olist[rng.integers(olist.size)])
            sh = tl[rng.integers(tl.shape[0])]
            true_t[p] = -1
        else:
            o_t = int(rng.integers(O))
            it = int(rng.integers(T))
            sh = shifts[it]
            true_t[p] = it
        true_o[p] = o_t
        a = project_exact(pv, eulers[o_t], x, y, maxR)
        # particle = shifted projection: X = A * exp(-i (x*tx + y*ty))
        ph = -2.0 * math.pi * (x * sh[0] + y * sh[1]) / pv.ori_size
        xim = a * np.exp(-1j * ph)
        if cfg["ctf"]:
            ctf = ctf_values(x, y, pv.ori_size, rng.uniform(1e4, 3e4))
        else:
            ctf = np.ones(N)
        xim = xim * ctf
        inside = (x.astype(np.int64) ** 2 + y.astype(np.int64) ** 2) <= maxR * maxR
        sig_pow = float(np.sum(np.abs(xim[inside]) ** 2))
        s2 = _noise_model(x, y, cfg["snr"], sig_pow)
        noise = (rng.standard_normal(N) + 1j * rng.standard_normal(N)) * np.sqrt(s2 / 2.0)
        xim = xim + noise
        minv = 1.0 / s2
        ok = np.abs(ctf) > 1e-8
        folded = np.where(ok, xim / np.where(ok, ctf, 1.0), xim)
        fre[p] = folded.real.astype(np.float32)
        fim[p] = folded.imag.astype(np.float32)
        corr[p] = (minv * ctf * ctf).astype(np.float32)

    return CoarseProblem(
        name=name, projector=pv, img_size=S, imgX=imgX, imgY=imgY, imgMaxR=imgMaxR,
        eulers=np.ascontiguousarray(eulers), trans_x=tx, trans_y=ty, shifts=shifts,
        fimg_re=fre, fimg_im=fim, corr=corr, true_orient=true_o, true_trans=true_t,
        orient_lists=orient_lists, trans_lists=trans_lists,
        meta=dict(cfg=cfg, seed=seed, maxR=maxR))
