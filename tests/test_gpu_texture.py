"""Texture-unit linear filtering vs the oracle's CPU emulation, sample by
sample.  The projector's texture objects (cudaFilterModeLinear, clamp,
unnormalised coordinates) are sampled at chosen coordinates through a probe
kernel (oracle/tex_probe.cu).  With B200D2_REPORT_DIR set, the raw samples are
saved for inspection."""
from __future__ import annotations

import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _probe_lib():
    L = C.CDLL(os.path.join(os.path.dirname(HERE), "oracle", "libtexprobe.so"))
    L.texprobe_sample.argtypes = [C.c_ulonglong, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    return L


def _sample(pkg, torch, vol, uvw):
    from types import SimpleNamespace
    Z, Y, X = vol.shape
    pv = SimpleNamespace(re=vol, im=vol, mdlX=X, mdlY=Y, mdlZ=Z, mdlInitY=0, mdlInitZ=0, mdlMaxR=3,
                         padding_factor=1.0)
    proj = pkg.Projector(pv, use_texture=1)
    view = proj.view(X, Y, 3)
    d_uvw = torch.as_tensor(uvw.reshape(-1), device="cuda")
    out = torch.empty(uvw.shape[0], device="cuda")
    assert _probe_lib().texprobe_sample(view.tex_re, d_uvw.data_ptr(), uvw.shape[0], out.data_ptr(),
                                        torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    proj.close()
    return out.cpu().numpy()


def test_texture_weight_structure(pkg, cuda, oracle):
    """Constant, linear and one-hot volumes expose the effective per-axis
    weights of the texture unit at random interior points."""
    torch = cuda
    rng = np.random.default_rng(11)
    X = Y = Z = 8
    uvw = rng.uniform(1.0, 6.5, (2048, 3)).astype(np.float32)
    z, y, x = np.meshgrid(np.arange(Z), np.arange(Y), np.arange(X), indexing="ij")
    vols = {"const": np.ones((Z, Y, X)), "x": x, "y": y, "z": z, "xy": x * y, "xyz": x * y * z}
    for c in [(3, 3, 3), (2, 4, 5)]:
        v = np.zeros((Z, Y, X))
        v[c] = 1.0
        vols["hot%d%d%d" % c] = v
    res = {k: _sample(pkg, torch, np.ascontiguousarray(v, np.float32), uvw) for k, v in vols.items()}
    d = os.environ.get("B200D2_REPORT_DIR")
    if d:
        np.savez(os.path.join(d, "tex_probe_structure.npz"), uvw=uvw, **res)
    # the weights of a linear filter sum to one
    assert np.abs(res["const"] - 1.0).max() < 1e-5


def test_texture_filtering_samples(pkg, cuda, oracle):
    """1D sweeps match the 1/256 weight model to FP32 rounding; 3D samples
    deviate by the hardware's joint weight rounding (bounded here)."""
    torch = cuda
    rng = np.random.default_rng(7)
    X = Y = Z = 8
    vol = rng.uniform(-1, 1, (Z, Y, X)).astype(np.float32)
    from types import SimpleNamespace
    pv = SimpleNamespace(re=vol, im=vol, mdlX=X, mdlY=Y, mdlZ=Z, mdlInitY=0, mdlInitZ=0, mdlMaxR=3,
                         padding_factor=1.0)
    proj = pkg.Projector(pv, use_texture=1)
    view = proj.view(8, 8, 3)
    pts = []
    # 1D sweeps of the fractional coordinate (other axes at texel centres)
    for k in range(1024):
        f = k / 1024.0
        pts.append((2.5 + f, 3.5, 4.5))
        pts.append((2.5, 3.5 + f, 4.5))
        pts.append((2.5, 3.5, 4.5 + f))
    # random interior points
    for _ in range(4096):
        pts.append(tuple(rng.uniform(1.0, 6.5, 3)))
    uvw = np.array(pts, np.float32)
    d_uvw = torch.as_tensor(uvw.reshape(-1), device="cuda")
    out = torch.empty(len(pts), device="cuda")
    L = _probe_lib()
    assert L.texprobe_sample(view.tex_re, d_uvw.data_ptr(), len(pts), out.data_ptr(),
                             torch.cuda.current_stream().cuda_stream) == 0
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    d = os.environ.get("B200D2_REPORT_DIR")
    if d:
        os.makedirs(d, exist_ok=True)
        np.savez(os.path.join(d, "tex_probe.npz"), vol=vol, uvw=uvw, out=got)
    em = oracle.tex_sample(vol, uvw)
    err = np.abs(em - got)
    print("texture emulation max abs err", err.max(), "mean", err.mean())
    assert err[:3072].max() < 1e-6  # single-axis sweeps: exact 1/256 weights
    assert err.max() < 2e-2  # 3D: joint corner-weight rounding, |values| <= 1
    proj.close()


def test_float2_texture_equals_two_textures(pkg, synth, cuda):
    """The interleaved (re, im) texture gives bit-identical projections to the
    two single-channel textures the reference uses (one fetch instead of
    two; the filtering weights belong to the fetch, not the channel)."""
    torch = cuda
    pr = synth.make_problem("c1", P=1)
    proj = pkg.Projector(pr.projector, use_texture=1)
    both = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    assert both.tex_c != 0
    split = pkg.View.from_buffer_copy(both)
    split.tex_c = 0
    x, y = synth.pixel_coords(pr.imgX, pr.imgY, both.maxR)
    px = torch.as_tensor(np.asarray(x, np.int32), device="cuda")
    py = torch.as_tensor(np.asarray(y, np.int32), device="cuda")
    eul = torch.as_tensor(pr.eulers.reshape(-1), device="cuda")
    outs = []
    for v in (both, split):
        re = torch.empty(pr.O * pr.N_img, device="cuda")
        im = torch.empty(pr.O * pr.N_img, device="cuda")
        pkg.project_pixels(v, eul, px, py, re, im, pr.O, pr.N_img)
        outs.append((re, im))
    torch.cuda.synchronize()
    assert torch.equal(outs[0][0], outs[1][0]) and torch.equal(outs[0][1], outs[1][1])
    assert float(outs[0][0].abs().max()) > 0
    proj.close()
