"""Every tensor-core form against the reference's own FP64 kernel, at the
precision-study shape (C3: image 96, 36864 orientations, 49 translations) and
the production shape (C2: image 64, 4608 orientations, 113 translations, 32
particles).

The reference is runDiff2KernelCoarseDouble (src/acc_helper_functions_impl.h:
503-854, kernel src/diff2.cuh:205-365), compiled from the reference sources
into oracle/_ref and run on the same device buffers (projector volume,
orientations, translations, images) as this library.  Both sample the
projector through the texture unit, so the FP64 kernel's output is the
reference value of every diff2 here.

Checked per form, with the stated tolerances (max relative diff2 error):
  BF16x3, TF32x3, FP16x3   1e-5        TF32, FP16 (single product)   1e-3
- every diff2 (max relative error over all evaluations);
- the per-particle minimum and argmin fused into the contraction epilogue:
  the minimum equals the smallest stored diff2 and lies within the tolerance
  of the FP64 minimum; the argmin is the stored block's argmin and equals the
  FP64 argmin wherever the FP64 best-to-second gap exceeds twice the
  tolerance;
- the normalised weights exp(-(diff2 - min)) / sum, computed on the device in
  FP64 by b200d2_coarse_weights from the form's FP32 diff2, against the same
  weights computed in numpy from the FP64 diff2.  A relative diff2 error e
  moves each exponent d - min of a weight that matters (d - min < 50) by at
  most Delta = e (2 |min| + 50), so every weight moves by a factor within
  exp(+-2 Delta): max abs and L1 errors are bounded by exp(2 Delta) - 1 with
  e the measured max relative error.
"""
from __future__ import annotations

import math

import numpy as np
import pytest

from gpu_util import DeviceProblem, RefKernels, argmin_consistent

pytestmark = pytest.mark.gpu
TOL = {"bf16x3": 1e-5, "tf32x3": 1e-5, "tf32": 1e-3, "fp16x3": 1e-5, "fp16": 1e-3}
ALL = ["bf16x3", "tf32x3", "tf32", "fp16x3", "fp16"]


def prec_code(pkg, name):
    return {"bf16x3": pkg.PREC_BF16X3, "tf32x3": pkg.PREC_TF32X3, "tf32": pkg.PREC_TF32,
            "fp16x3": pkg.PREC_FP16X3, "fp16": pkg.PREC_FP16}[name]


class Case:
    def __init__(self, pkg, synth, oracle, torch, name, P):
        self.pr = synth.make_problem(name, P=P)
        self.proj = pkg.Projector(self.pr.projector, use_texture=1)
        self.view = self.proj.view(self.pr.imgX, self.pr.imgY, self.pr.imgMaxR)
        self.dp = DeviceProblem(torch, self.pr)
        ref = RefKernels(oracle, self.pr)
        try:
            self.f64 = np.stack([ref.f64(self.dp, p) for p in range(self.pr.P)])
        finally:
            ref.close()

    def close(self):
        self.proj.close()


@pytest.fixture(scope="module")
def c3(pkg, synth, oracle, cuda):
    c = Case(pkg, synth, oracle, cuda, "c3", 6)
    yield c
    c.close()


@pytest.fixture(scope="module")
def c2_32(pkg, synth, oracle, cuda):
    c = Case(pkg, synth, oracle, cuda, "c2", 32)
    yield c
    c.close()


def _weights_fp64(d):
    """exp(-(d - min)) / sum per particle, FP64, d [P, O, T]."""
    d = np.asarray(d, np.float64).reshape(d.shape[0], -1)
    w = np.exp(-(d - d.min(axis=1, keepdims=True)))
    return w / w.sum(axis=1, keepdims=True)


def _run_and_check(pkg, oracle, torch, case, name):
    pr, dp, view, ref = case.pr, case.dp, case.view, case.f64
    prec = prec_code(pkg, name)
    out = torch.zeros(pr.P * pr.O * pr.T, device="cuda")
    mn = torch.empty(pr.P, device="cuda", dtype=torch.float64)
    am = torch.empty(pr.P, device="cuda", dtype=torch.int64)
    b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, out, O=pr.O, T=pr.T, P=pr.P,
                       N_img=pr.N_img, out_min=mn, out_argmin=am)
    ws = torch.empty(pkg.batch_workspace_bytes(view, b, prec), device="cuda", dtype=torch.uint8)
    pkg.diff2_coarse_batch(view, b, prec, ws)
    torch.cuda.synchronize()
    assert pkg.workspace_status(ws) == 0
    # device FP64 weights from this form's FP32 diff2
    w_dev, _ = pkg.coarse_weights(out, pr.P, pr.O, pr.T)
    got = out.cpu().numpy().reshape(pr.P, pr.O, pr.T)
    mn, am = mn.cpu().numpy(), am.cpu().numpy()
    w_got = w_dev.cpu().numpy().reshape(pr.P, -1)
    del w_dev, out, ws

    s = oracle.error_stats(got, ref)
    e = s["max_rel"]
    assert e <= TOL[name], (name, s)
    w_ref = _weights_fp64(ref)
    report = {"max_rel": e, "avg_rel": s["avg_rel"], "min_rel": 0.0, "w_max_abs": 0.0, "w_l1": 0.0}
    for p in range(pr.P):
        gp, rp = got[p].ravel(), ref[p].ravel()
        # fused min / argmin against the stored block
        assert am[p] == int(np.argmin(gp))
        assert mn[p] == float(gp.min())
        # against FP64
        rmin = float(rp.min())
        report["min_rel"] = max(report["min_rel"], abs(mn[p] - rmin) / abs(rmin))
        assert abs(mn[p] - rmin) <= TOL[name] * abs(rmin)
        ok, gap = argmin_consistent(gp, rp, TOL[name])
        assert ok, (name, p, gap)
        # weights
        delta = e * (2.0 * abs(rmin) + 50.0)
        bound = math.expm1(2.0 * delta) * 1.01 + 1e-12
        dw = np.abs(w_got[p] - w_ref[p])
        report["w_max_abs"] = max(report["w_max_abs"], float(dw.max()))
        report["w_l1"] = max(report["w_l1"], float(dw.sum()))
        assert float(dw.max()) <= bound, (name, p, float(dw.max()), bound)
        assert float(dw.sum()) <= bound, (name, p, float(dw.sum()), bound)
    print(pr.name, name, " ".join(f"{k} {v:.3g}" for k, v in report.items()))
    return report


@pytest.mark.parametrize("name", ALL)
def test_tc_c3_vs_reference_fp64(pkg, oracle, cuda, c3, name):
    _run_and_check(pkg, oracle, cuda, c3, name)


@pytest.mark.parametrize("name", ALL)
def test_tc_c2_32_particles_vs_reference_fp64(pkg, oracle, cuda, c2_32, name):
    _run_and_check(pkg, oracle, cuda, c2_32, name)


def test_fp32_dropin_c3_vs_reference_fp64(pkg, oracle, cuda, c3):
    """The FP32 CUDA-core drop-in (runDiff2KernelCoarse's replacement) at C3,
    one particle, against the reference's FP64 kernel: within 1e-5."""
    pr, dp, view = c3.pr, c3.dp, c3.view
    out = cuda.zeros(pr.O * pr.T, device="cuda")
    pkg.run_diff2_kernel_coarse(view, dp.tx, dp.ty, dp.corr[0], dp.re[0], dp.im[0], dp.eulers, out, pr.O, pr.T,
                                pr.N_img)
    cuda.cuda.synchronize()
    s = oracle.error_stats(out.cpu().numpy().reshape(pr.O, pr.T), c3.f64[0])
    assert s["max_rel"] <= 1e-5, s
