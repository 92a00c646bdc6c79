"""Batched CTF folding (b200d2_ctf_fold) against a float64 numpy restatement
of the same weak-phase CTF, and the coarse pass on device-folded inputs
against the same pass on host-folded inputs."""
from __future__ import annotations

import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def ctf_ref(x, y, ori_size, pixel_A, c):
    c = {k: float(np.float32(v)) for k, v in c.items()}  # the device receives FP32 parameters
    volt = c["voltage_kV"] * 1e3
    lam = 12.2643247 / math.sqrt(volt * (1.0 + volt * 0.978466e-6))
    kx = x.astype(np.float64) / (ori_size * pixel_A)
    ky = y.astype(np.float64) / (ori_size * pixel_A)
    k2 = kx * kx + ky * ky
    du, dv = c["defocus_u_A"], c["defocus_v_A"]
    ang = math.radians(c.get("defocus_angle_deg", 0.0))
    dz = 0.5 * (du + dv) + 0.5 * (du - dv) * np.cos(2.0 * (np.arctan2(ky, kx) - ang))
    chi = math.pi * lam * dz * k2 - 0.5 * math.pi * c["cs_mm"] * 1e7 * lam ** 3 * k2 * k2
    chi = chi + math.radians(c.get("phase_shift_deg", 0.0))
    q = c["amp_contrast"]
    v = -(math.sqrt(1 - q * q) * np.sin(chi) + q * np.cos(chi)) * (c.get("scale", 1.0) or 1.0)
    return v * np.exp(-0.25 * c.get("bfactor", 0.0) * k2)


def host_fold(re, im, v, minv):
    ok = np.abs(v) > 1e-8
    fre = np.where(ok, re.astype(np.float64) / np.where(ok, v, 1.0), re).astype(np.float32)
    fim = np.where(ok, im.astype(np.float64) / np.where(ok, v, 1.0), im).astype(np.float32)
    return fre, fim, (minv.astype(np.float64) * v * v).astype(np.float32)


def _params(rng, P):
    out = []
    for p in range(P):
        du = rng.uniform(1e4, 3e4)
        out.append(dict(defocus_u_A=du, defocus_v_A=du - rng.uniform(0, 800) * (p % 2), defocus_angle_deg=rng.uniform(0, 180),
                        voltage_kV=300.0, cs_mm=2.7, amp_contrast=0.1, phase_shift_deg=0.0,
                        bfactor=(0.0 if p % 3 else 50.0), scale=1.0))
    return out


def test_ctf_fold_matches_reference(pkg, synth, cuda):
    torch = cuda
    pr = synth.make_problem("c1", P=6)
    rng = np.random.default_rng(11)
    x, y = synth.pixel_coords(pr.imgX, pr.imgY, pr.imgMaxR)
    params = _params(rng, pr.P)
    minv = rng.uniform(0.5, 2.0, pr.N_img).astype(np.float32)
    re = torch.as_tensor(pr.fimg_re, device="cuda")
    im = torch.as_tensor(pr.fimg_im, device="cuda")
    fr, fi, co = pkg.ctf_fold(re, im, params, torch.as_tensor(minv, device="cuda"), imgX=pr.imgX, imgY=pr.imgY,
                              maxR=pr.imgMaxR, ori_size=pr.projector.ori_size, pixel_A=1.5)
    torch.cuda.synchronize()
    for p in range(pr.P):
        v = ctf_ref(x, y, pr.projector.ori_size, 1.5, params[p])
        hr, hi, hc = host_fold(pr.fimg_re[p], pr.fimg_im[p], v, minv)
        sel = np.abs(v) > 1e-5  # away from the zeros of the CTF, where 1/CTF amplifies the last bit
        np.testing.assert_allclose(fr[p].cpu().numpy()[sel], hr[sel], rtol=2e-6)
        np.testing.assert_allclose(fi[p].cpu().numpy()[sel], hi[sel], rtol=2e-6)
        np.testing.assert_allclose(co[p].cpu().numpy(), hc, rtol=2e-6, atol=1e-30)


def test_coarse_pass_on_device_folded_inputs(pkg, synth, oracle, cuda):
    torch = cuda
    from gpu_util import DeviceProblem
    pr = synth.make_problem("c1", P=4)
    rng = np.random.default_rng(5)
    x, y = synth.pixel_coords(pr.imgX, pr.imgY, pr.imgMaxR)
    params = _params(rng, pr.P)
    minv = np.stack([rng.uniform(0.5, 2.0, pr.N_img) for _ in range(pr.P)]).astype(np.float32)
    dp = DeviceProblem(torch, pr)
    fr, fi, co = pkg.ctf_fold(dp.re, dp.im, params, torch.as_tensor(minv, device="cuda"), imgX=pr.imgX,
                              imgY=pr.imgY, maxR=pr.imgMaxR, ori_size=pr.projector.ori_size, pixel_A=1.5)
    hr, hi, hc = zip(*[host_fold(pr.fimg_re[p], pr.fimg_im[p],
                                 ctf_ref(x, y, pr.projector.ori_size, 1.5, params[p]), minv[p]) for p in range(pr.P)])
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)

    def run(re_, im_, co_):
        out = torch.zeros(pr.P * pr.O * pr.T, device="cuda")
        b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, re_, im_, co_, out, O=pr.O, T=pr.T, P=pr.P, N_img=pr.N_img)
        ws = torch.empty(pkg.batch_workspace_bytes(view, b, pkg.PREC_BF16X3), device="cuda", dtype=torch.uint8)
        pkg.diff2_coarse_batch(view, b, pkg.PREC_BF16X3, ws)
        torch.cuda.synchronize()
        return out.cpu().numpy()

    dev = run(fr, fi, co)
    host = run(*(torch.as_tensor(np.stack(a), device="cuda") for a in (hr, hi, hc)))
    assert oracle.error_stats(dev, host)["max_rel"] <= 1e-5
    proj.close()
