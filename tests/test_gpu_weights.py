"""Coarse weights (b200d2_coarse_weights) against a float64 numpy restatement
of w = pdf_o * pdf_t * exp(-(diff2 - min)) on the same FP32 diff2 block.
Tolerance: 1e-12 relative (the device uses the same FP64 formula; only the
summation order and the last bit of exp differ)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def ref_weights(d, mn=None, po=None, pt=None, normalize=True):
    d = d.astype(np.float64)
    P = d.shape[0]
    if mn is None:
        mn = d.reshape(P, -1).min(axis=1)
    w = np.exp(-(d - mn[:, None, None]))
    if po is not None:
        w = w * po[None, :, None]
    if pt is not None:
        w = w * pt[None, None, :]
    s = w.reshape(P, -1).sum(axis=1)
    return (w / s[:, None, None] if normalize else w), s


@pytest.mark.parametrize("P,O,T", [(1, 1, 1), (3, 37, 5), (2, 7001, 9), (4, 576, 21)])
def test_weights_match_reference(pkg, cuda, P, O, T):
    torch = cuda
    rng = np.random.default_rng(P * 1000 + O)
    # diff2-like values: a large common offset and a spread of tens of units,
    # so that exp() spans from 1 down to underflow
    d = (5000.0 + rng.exponential(40.0, (P, O, T))).astype(np.float32)
    dd = torch.as_tensor(d.reshape(-1), device="cuda")
    w, s = pkg.coarse_weights(dd, P, O, T)
    torch.cuda.synchronize()
    rw, rs = ref_weights(d)
    np.testing.assert_allclose(s.cpu().numpy(), rs, rtol=1e-12)
    np.testing.assert_allclose(w.cpu().numpy(), rw, rtol=1e-12, atol=1e-300)
    assert abs(float(w.sum()) - P) < 1e-9 * P


def test_weights_priors_min_and_determinism(pkg, cuda):
    torch = cuda
    P, O, T = 3, 4099, 13  # two chunks per particle
    rng = np.random.default_rng(5)
    d = (100.0 + rng.exponential(10.0, (P, O, T))).astype(np.float32)
    po = rng.uniform(0, 1, O)
    po[::7] = 0.0  # zero orientation priors give zero weights
    pt = rng.uniform(0.5, 1.5, T)
    dd = torch.as_tensor(d.reshape(-1), device="cuda")
    mn = torch.as_tensor(d.reshape(P, -1).min(axis=1).astype(np.float64), device="cuda")
    tpo, tpt = torch.as_tensor(po, device="cuda"), torch.as_tensor(pt, device="cuda")
    w1, s1 = pkg.coarse_weights(dd, P, O, T, out_min=mn, pdf_orient=tpo, pdf_offset=tpt)
    w2, s2 = pkg.coarse_weights(dd, P, O, T, pdf_orient=tpo, pdf_offset=tpt)  # min computed on the device
    torch.cuda.synchronize()
    assert torch.equal(w1, w2) and torch.equal(s1, s2)  # bit-reproducible
    rw, rs = ref_weights(d, po=po, pt=pt)
    np.testing.assert_allclose(w1.cpu().numpy(), rw, rtol=1e-12, atol=1e-300)
    assert (w1.cpu().numpy()[:, ::7, :] == 0).all()
    # unnormalised weights and sums only
    w3, s3 = pkg.coarse_weights(dd, P, O, T, pdf_orient=tpo, pdf_offset=tpt, normalize=False)
    torch.cuda.synchronize()
    np.testing.assert_allclose(w3.cpu().numpy(), ref_weights(d, po=po, pt=pt, normalize=False)[0], rtol=1e-12,
                               atol=1e-300)
    assert torch.equal(s3, s1)


def test_weights_after_tensor_core_batch(pkg, synth, oracle, cuda):
    """The batch's per-particle minimum feeds the weights; their error against
    weights from the FP64 kernel's diff2 is bounded by the diff2 error."""
    from gpu_util import DeviceProblem, ours_f64
    torch = cuda
    pr = synth.make_problem("c1", P=3)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(cuda, pr)
    out = torch.zeros(pr.P * pr.O * pr.T, device="cuda")
    mn = torch.empty(pr.P, device="cuda", dtype=torch.float64)
    b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, out, O=pr.O, T=pr.T, P=pr.P,
                       N_img=pr.N_img, out_min=mn)
    ws = torch.empty(pkg.batch_workspace_bytes(view, b, pkg.PREC_BF16X3), device="cuda", dtype=torch.uint8)
    pkg.diff2_coarse_batch(view, b, pkg.PREC_BF16X3, ws)
    w, s = pkg.coarse_weights(out, pr.P, pr.O, pr.T, out_min=mn)
    torch.cuda.synchronize()
    ref = np.stack([ours_f64(pkg, view, dp, p) for p in range(pr.P)])
    rw, _ = ref_weights(ref)
    got = w.cpu().numpy()
    # with |diff2 error| <= e, (d - min) moves by at most 2e and the
    # normalising sum by a factor within exp(+-2e): log ratio within 4e
    err = float(np.abs(out.cpu().numpy().reshape(ref.shape) - ref).max())
    big = rw > 1e-6
    assert np.all(np.abs(np.log(got[big] / rw[big])) <= 4 * err + 1e-9), err
    proj.close()
