"""Cross-correlation coarse score (runDiff2KernelCoarse with do_CC,
cuda_kernel_diff2_CC_coarse, src/diff2.cuh:691-809):
  cc[o][t] = -sum corr Re(conj(A_o) S_t) / sqrt(sum corr |A_o|^2).

Checked against the oracle's FP64 restatement (oracle.cc_coarse_f64, itself
pinned to the C oracle's diff2 on the CPU), against the reference's own CC
kernel (compiled into oracle/_ref, same device buffers), and across this
library's forms: the FP32 and FP64 CUDA-core kernels and the tensor-core
batch (score B200D2_SCORE_CC).

Bar: CC values change sign and pass through zero, so the error is measured
relative to the particle's largest score magnitude: 1e-5 for the FP32
CUDA-core sums; 3e-5 for the three-term tensor-core splits, whose cross term
is accumulated in FP32 over all pixels in TMEM (unlike diff2, the score has no
large norm offset that hides that rounding; measured 1.3-1.4e-5 at C2 for both
BF16x3 and TF32x3); 1e-3 for the single TF32 / FP16 products; the argmin
agrees wherever the best-to-second gap exceeds the tolerance."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import DeviceProblem, argmin_consistent

pytestmark = pytest.mark.gpu
TOL = {"fp32": 1e-5, "bf16x3": 3e-5, "tf32x3": 3e-5, "fp16x3": 3e-5, "tf32": 1e-3, "fp16": 1e-3}


def scaled_err(got, ref):
    got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
    return float(np.abs(got - ref).max() / np.abs(ref).max())


def cc64(pkg, torch, view, dp, p):
    pr = dp.pr
    out = torch.zeros(pr.O * pr.T, device="cuda", dtype=torch.float64)
    pkg.run_diff2_kernel_coarse_cc_double(view, dp.tx, dp.ty, dp.corr[p], dp.re[p], dp.im[p], dp.eulers, out,
                                          pr.O, pr.T, pr.N_img)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(pr.O, pr.T)


@pytest.fixture(scope="module", params=["tiny", "c1"])
def case(request, pkg, synth, cuda):
    pr = synth.make_problem(request.param, P=3)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(cuda, pr)
    ref = np.stack([cc64(pkg, cuda, view, dp, p) for p in range(pr.P)])
    yield pr, proj, view, dp, ref
    proj.close()


def test_cc_fp64_matches_oracle(pkg, synth, oracle, cuda, case):
    """FP64 GPU CC vs the oracle fed the texture unit's own projections
    (1e-9), and vs the oracle's texture-weight model (2e-3: the model's
    weight rounding, as for diff2)."""
    torch = cuda
    pr, _, view, dp, ref = case
    proj = oracle.projector_for(pr)
    n = pr.N_img
    x = np.arange(n) % pr.imgX
    y = np.arange(n) // pr.imgX
    y = np.where(y > proj.maxR, y - pr.imgY, y)
    pre = torch.empty(pr.O * n, device="cuda")
    pim = torch.empty(pr.O * n, device="cuda")
    pkg.project_pixels(view, dp.eulers, torch.as_tensor(x.astype(np.int32), device="cuda"),
                       torch.as_tensor(y.astype(np.int32), device="cuda"), pre, pim, pr.O, n)
    torch.cuda.synchronize()
    given = (pre.cpu().numpy().reshape(pr.O, n).astype(np.float64), pim.cpu().numpy().reshape(pr.O, n).astype(np.float64))
    for p in range(pr.P):
        args = (proj, pr.eulers, pr.trans_x, pr.trans_y, pr.fimg_re[p], pr.fimg_im[p], pr.corr[p])
        assert scaled_err(ref[p], oracle.cc_coarse_f64(*args, projections=given)) <= 1e-9
        assert scaled_err(ref[p], oracle.cc_coarse_f64(*args)) <= 2e-3


def test_cc_fp32_matches_reference_kernel(pkg, oracle, cuda, case):
    """The drop-in (b200d2_diff2_coarse_cc) and the reference's CC kernel on
    the same buffers; both write (a garbage initial value must not leak)."""
    torch = cuda
    pr, _, view, dp, ref = case
    L = oracle.ref_lib()
    pv = pr.projector
    h = L.refshim_projector_create(pv.mdlX, pv.mdlY, pv.mdlZ, pv.mdlInitY, pv.mdlInitZ, pv.mdlMaxR,
                                   pv.padding_factor, np.ascontiguousarray(pv.re, np.float32).ctypes.data,
                                   np.ascontiguousarray(pv.im, np.float32).ctypes.data)
    assert h
    for p in range(pr.P):
        ours = torch.full((pr.O * pr.T,), 123.0, device="cuda")
        theirs = torch.full((pr.O * pr.T,), -7.0, device="cuda")
        pkg.run_diff2_kernel_coarse_cc(view, dp.tx, dp.ty, dp.corr[p], dp.re[p], dp.im[p], dp.eulers, ours,
                                       pr.O, pr.T, pr.N_img)
        assert L.refshim_diff2_coarse_cc(h, pr.imgX, pr.imgY, 1, pr.imgMaxR, dp.eulers.data_ptr(), dp.tx.data_ptr(),
                                         dp.ty.data_ptr(), dp.corr[p].data_ptr(), dp.re[p].data_ptr(),
                                         dp.im[p].data_ptr(), theirs.data_ptr(), pr.O, pr.T, pr.N_img, None) == 0
        torch.cuda.synchronize()
        o = ours.cpu().numpy().reshape(pr.O, pr.T)
        t = theirs.cpu().numpy().reshape(pr.O, pr.T)
        assert scaled_err(o, t) <= TOL["fp32"]
        assert scaled_err(t, ref[p]) <= TOL["fp32"]  # the reference itself against FP64
        assert scaled_err(o, ref[p]) <= TOL["fp32"]
    L.refshim_projector_destroy(h)


@pytest.mark.parametrize("name", ["fp32", "bf16x3", "tf32x3", "fp16x3", "tf32", "fp16"])
def test_cc_batch_forms(pkg, cuda, case, name):
    """The batch with score CC, every precision, with per-particle min/argmin."""
    torch = cuda
    pr, _, view, dp, ref = case
    prec = {"fp32": pkg.PREC_FP32, "bf16x3": pkg.PREC_BF16X3, "tf32x3": pkg.PREC_TF32X3,
            "fp16x3": pkg.PREC_FP16X3, "tf32": pkg.PREC_TF32, "fp16": pkg.PREC_FP16}[name]
    out = torch.full((pr.P * pr.O * pr.T,), 55.0, device="cuda")
    mn = torch.empty(pr.P, device="cuda", dtype=torch.float64)
    am = torch.empty(pr.P, device="cuda", dtype=torch.int64)
    b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, out, O=pr.O, T=pr.T, P=pr.P, N_img=pr.N_img,
                       out_min=mn, out_argmin=am, score=pkg.SCORE_CC)
    nb = pkg.batch_workspace_bytes(view, b, prec)
    ws = torch.empty(max(nb, 1), device="cuda", dtype=torch.uint8)
    pkg.diff2_coarse_batch(view, b, prec, ws)
    torch.cuda.synchronize()
    got = out.cpu().numpy().reshape(pr.P, pr.O, pr.T)
    mn, am = mn.cpu().numpy(), am.cpu().numpy()
    for p in range(pr.P):
        assert scaled_err(got[p], ref[p]) <= TOL[name], (p, scaled_err(got[p], ref[p]))
        ok, gap = argmin_consistent(got[p], ref[p], TOL[name])
        assert ok, (p, gap)
        assert mn[p] == pytest.approx(float(got[p].min()), rel=1e-7)
        assert int(am[p]) == int(np.argmin(got[p].ravel()))


def test_cc_batch_accumulates(pkg, cuda, case):
    torch = cuda
    pr, _, view, dp, ref = case
    init = np.random.default_rng(3).uniform(-1, 1, (pr.P, pr.O, pr.T)).astype(np.float32)
    for prec in (pkg.PREC_FP32, pkg.PREC_BF16X3):
        out = torch.as_tensor(init.reshape(-1).copy(), device="cuda")
        b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, out, O=pr.O, T=pr.T, P=pr.P,
                           N_img=pr.N_img, accumulate=True, score=pkg.SCORE_CC)
        ws = torch.empty(max(pkg.batch_workspace_bytes(view, b, prec), 1), device="cuda", dtype=torch.uint8)
        pkg.diff2_coarse_batch(view, b, prec, ws)
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(pr.P, pr.O, pr.T) - init
        for p in range(pr.P):
            assert np.abs(got[p] - ref[p]).max() <= 2e-5 * (np.abs(ref[p]).max() + 1.0)


def test_cc_score_rejected_when_invalid(pkg, cuda, case):
    torch = cuda
    pr, _, view, dp, _ = case
    out = torch.zeros(pr.P * pr.O * pr.T, device="cuda")
    b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, out, O=pr.O, T=pr.T, P=pr.P, N_img=pr.N_img,
                       score=7)
    with pytest.raises(pkg.B200D2Error):
        pkg.diff2_coarse_batch(view, b, pkg.PREC_BF16X3, torch.empty(1, device="cuda", dtype=torch.uint8))
