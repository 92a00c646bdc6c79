"""This library's kernels against the committed golden fixtures: outputs of the
reference's own runDiff2KernelCoarse (FP32) and runDiff2KernelCoarseDouble
(FP64), stored by tests/golden/make_golden.py, with no reference code run
here.

- projections at every pixel: bit-identical to the stored texture-unit
  samples (same positions, same texture unit);
- FP64 kernel vs the reference FP64 kernel: 1e-6;
- FP32 drop-in vs the reference FP32 kernel and vs its FP64 kernel: 1e-5;
- BF16x3 and TF32x3 tensor-core batches vs the reference FP64 kernel: 1e-5,
  with the argmin equal wherever the FP64 best-to-second gap exceeds twice
  that.
"""
from __future__ import annotations

import glob
import os

import numpy as np
import pytest

import golden_util
from gpu_util import argmin_consistent, dev

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz"))))
def test_library_against_reference_golden(pkg, synth, oracle, cuda, path):
    torch = cuda
    g = golden_util.load(path, synth)
    proj = pkg.Projector(g.pv, use_texture=1)
    view = proj.view(g.imgX, g.imgY, g.imgMaxR)
    eul, tx, ty = dev(torch, g.eulers.reshape(-1)), dev(torch, g.trans_x), dev(torch, g.trans_y)
    re, im, corr = dev(torch, g.fimg_re), dev(torch, g.fimg_im), dev(torch, g.corr)

    x, y = synth.pixel_coords(g.imgX, g.imgY, view.maxR)
    pre = torch.empty(g.O * g.N_img, device="cuda")
    pim = torch.empty(g.O * g.N_img, device="cuda")
    pkg.project_pixels(view, eul, dev(torch, x), dev(torch, y), pre, pim, g.O, g.N_img)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(pre.cpu().numpy().reshape(g.O, g.N_img), g.prj_re)
    np.testing.assert_array_equal(pim.cpu().numpy().reshape(g.O, g.N_img), g.prj_im)

    for p in range(g.P):
        o64 = torch.zeros(g.O * g.T, device="cuda", dtype=torch.float64)
        pkg.run_diff2_kernel_coarse_double(view, tx, ty, corr[p], re[p], im[p], eul, o64, g.O, g.T, g.N_img)
        o32 = torch.zeros(g.O * g.T, device="cuda")
        pkg.run_diff2_kernel_coarse(view, tx, ty, corr[p], re[p], im[p], eul, o32, g.O, g.T, g.N_img)
        torch.cuda.synchronize()
        d64 = o64.cpu().numpy().reshape(g.O, g.T)
        d32 = o32.cpu().numpy().reshape(g.O, g.T)
        assert oracle.error_stats(d64, g.ref_f64[p])["max_rel"] <= 1e-6
        assert oracle.error_stats(d32, g.ref_f32[p])["max_rel"] <= 1e-5
        assert oracle.error_stats(d32, g.ref_f64[p])["max_rel"] <= 1e-5

    for prec in (pkg.PREC_BF16X3, pkg.PREC_TF32X3):
        out = torch.zeros(g.P * g.O * g.T, device="cuda")
        mn = torch.empty(g.P, device="cuda", dtype=torch.float64)
        am = torch.empty(g.P, device="cuda", dtype=torch.int64)
        b = pkg.make_batch(eul, tx, ty, re, im, corr, out, O=g.O, T=g.T, P=g.P, N_img=g.N_img, out_min=mn,
                           out_argmin=am)
        ws = torch.empty(pkg.batch_workspace_bytes(view, b, prec), device="cuda", dtype=torch.uint8)
        pkg.diff2_coarse_batch(view, b, prec, ws)
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(g.P, g.O, g.T)
        assert oracle.error_stats(got, g.ref_f64)["max_rel"] <= 1e-5
        for p in range(g.P):
            assert am[p].item() == int(np.argmin(got[p]))
            ok, gap = argmin_consistent(got[p], g.ref_f64[p], 1e-5)
            assert ok, (prec, p, gap)
    proj.close()
