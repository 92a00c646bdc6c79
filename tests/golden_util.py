"""Loading the golden fixtures of tests/golden/ (written by
tests/golden/make_golden.py from the reference's own kernels).

Two layouts:
- self-contained (ref_g0.npz): the projector volume and every input array are
  stored in the file;
- regenerated (ref_c1s.npz): the file names a seeded problem of
  relion_b200.synth, the particles and the orientation stride it used, and the
  SHA-256 of every input array; the inputs are rebuilt from the generator and
  checked against those digests before use, so the file holds only the
  reference's outputs and the texture unit's projections.
"""
from __future__ import annotations

import hashlib
from types import SimpleNamespace

import numpy as np

INPUT_KEYS = ("vol_re", "vol_im", "eulers", "trans_x", "trans_y", "fimg_re", "fimg_im", "corr")


def digest(a) -> str:
    a = np.ascontiguousarray(a)
    return hashlib.sha256(a.dtype.str.encode() + str(a.shape).encode() + a.tobytes()).hexdigest()


def inputs_of(pr, particles, o_stride):
    """The fixture's inputs taken from a synthetic problem."""
    pv = pr.projector
    sl = slice(0, particles)
    return dict(vol_re=pv.re, vol_im=pv.im, eulers=np.ascontiguousarray(pr.eulers[::o_stride]),
                trans_x=pr.trans_x, trans_y=pr.trans_y, fimg_re=pr.fimg_re[sl], fimg_im=pr.fimg_im[sl],
                corr=pr.corr[sl])


def load(path, synth=None) -> SimpleNamespace:
    """Fixture as a namespace: projector geometry (pv), image geometry, the
    input arrays of INPUT_KEYS and the stored outputs."""
    g = np.load(path)
    d = {k: g[k] for k in g.files}
    if "problem" in d:
        if synth is None:
            raise ValueError(f"{path} regenerates its inputs: pass the synth module")
        pr = synth.make_problem(str(d["problem"]), seed=int(d["seed"]))
        ins = inputs_of(pr, int(d["particles"]), int(d["o_stride"]))
        for k in INPUT_KEYS:
            got = digest(ins[k])
            if got != str(d["sha256_" + k]):
                raise AssertionError(f"{path}: regenerated input {k} differs from the one the reference saw")
        d.update(ins)
        pv = pr.projector
        d.update(mdlX=pv.mdlX, mdlY=pv.mdlY, mdlZ=pv.mdlZ, mdlInitY=pv.mdlInitY, mdlInitZ=pv.mdlInitZ,
                 mdlMaxR=pv.mdlMaxR, pf=pv.padding_factor, imgX=pr.imgX, imgY=pr.imgY, imgMaxR=pr.imgMaxR)
    geo = {k: int(d[k]) for k in ("mdlX", "mdlY", "mdlZ", "mdlInitY", "mdlInitZ", "mdlMaxR")}
    pv = SimpleNamespace(re=d["vol_re"], im=d["vol_im"], padding_factor=float(d["pf"]), **geo)
    ns = SimpleNamespace(**{k: v for k, v in d.items() if k not in ("vol_re", "vol_im")})
    ns.pv = pv
    ns.imgX, ns.imgY, ns.imgMaxR = int(d["imgX"]), int(d["imgY"]), int(d["imgMaxR"])
    ns.P, ns.O, ns.T = d["fimg_re"].shape[0], d["eulers"].shape[0], d["trans_x"].size
    ns.N_img = d["fimg_re"].shape[1]
    return ns
