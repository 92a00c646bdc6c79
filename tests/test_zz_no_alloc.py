"""The allocation-free tensor-core entry point (b200d2_diff2_coarse_batch_static).

It exists for callers that cannot call cudaMalloc: a host whose device memory
belongs to another allocator, a request path that must not pay cudaMalloc's
device synchronisation, or a plug-in that only receives its input and output
buffers.  It runs the batch pipeline on a fixed scratch area compiled into the
library.  Here it must give the same diff2, minimum and argmin as the
allocating entry point (b200d2_diff2_coarse_batch with a caller workspace),
within the tolerance the other tensor-core tests use, on two calls in a row
(the scratch keeps the previous call's contents, so the second call checks
that everything that must start at zero is reset).  Collected last on
purpose, and independent of the other tests' state."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import DeviceProblem

pytestmark = pytest.mark.gpu
TOL = 1e-5  # max relative diff2 difference, as in tests/test_gpu_tc.py


def _outputs(torch, pr):
    d = torch.zeros(pr.P * pr.O * pr.T, device="cuda")
    mn = torch.empty(pr.P, device="cuda", dtype=torch.float64)
    am = torch.empty(pr.P, device="cuda", dtype=torch.int64)
    return d, mn, am


def _listed_inputs(torch, oracle, pr):
    """The reference's filtered layout (FilterCoarseParamImage): in-radius
    pixels first with their coordinates, shared by all particles."""
    op = oracle.projector_for(pr)
    cols = [oracle.filter_image(op, pr.fimg_re[p], pr.fimg_im[p], pr.corr[p]) for p in range(pr.P)]
    n = cols[0][4]
    assert all(c[4] == n for c in cols)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(np.stack(a)), device="cuda")  # noqa: E731
    return t([c[0] for c in cols]), t([c[1] for c in cols]), t([c[2] for c in cols]), \
        torch.as_tensor(cols[0][3], device="cuda"), n


@pytest.mark.parametrize("form", ["diff2", "listed", "cc", "accumulate"])
def test_static_scratch_matches_allocating_entry_point(pkg, synth, oracle, cuda, form):
    """Two calls in a row on the fixed scratch give the allocating entry
    point's outputs, for the plain diff2 batch, caller-listed pixels (whose
    first stage takes another branch), the CC score and accumulation onto the
    caller's buffer.  Between the two calls a batch of another shape runs on
    the same scratch, so the second call starts from different leftovers."""
    torch = cuda
    pr = synth.make_problem("c1")
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(torch, pr)
    re, im, corr = dp.re, dp.im, dp.corr
    coor, n_listed = None, 0
    if form == "listed":
        re, im, corr, coor, n_listed = _listed_inputs(torch, oracle, pr)
    score = pkg.SCORE_CC if form == "cc" else pkg.SCORE_DIFF2
    accumulate = form == "accumulate"
    init = np.random.default_rng(7).uniform(0, 50, pr.P * pr.O * pr.T).astype(np.float32)

    def batch(out):
        d, mn, am = out
        if accumulate:
            d.copy_(torch.as_tensor(init, device="cuda"))
        return pkg.make_batch(dp.eulers, dp.tx, dp.ty, re, im, corr, d, O=pr.O, T=pr.T, P=pr.P,
                              N_img=pr.N_img, out_min=mn, out_argmin=am, coor_xy=coor, n_listed=n_listed,
                              score=score, accumulate=accumulate)

    ref = _outputs(torch, pr)
    b = batch(ref)
    need = pkg.batch_workspace_bytes(view, b, pkg.PREC_BF16X3)
    assert 0 < need <= pkg.STATIC_SCRATCH_BYTES
    ws = torch.empty(need, device="cuda", dtype=torch.uint8)
    pkg.diff2_coarse_batch(view, b, pkg.PREC_BF16X3, ws)
    torch.cuda.synchronize()
    assert pkg.workspace_status(ws) == 0
    r_d, r_mn, r_am = (t.cpu().numpy() for t in ref)
    if form == "cc":  # CC scores pass through zero: errors relative to the largest magnitude
        scale = np.abs(r_d).max()

    other = synth.make_problem("tiny")
    oproj = pkg.Projector(other.projector, use_texture=1)
    oview = oproj.view(other.imgX, other.imgY, other.imgMaxR)
    odp = DeviceProblem(torch, other)
    for call in range(2):
        out = _outputs(torch, pr)
        pkg.diff2_coarse_batch_static(view, batch(out), pkg.PREC_BF16X3)
        torch.cuda.synchronize()
        d, mn, am = (t.cpu().numpy() for t in out)
        if form == "cc":
            assert np.abs(d.astype(np.float64) - r_d).max() <= TOL * scale, call
        else:
            s = oracle.error_stats(d, r_d)
            assert s["max_rel"] <= TOL, (call, s)
        np.testing.assert_allclose(mn, r_mn, rtol=TOL, atol=TOL * abs(r_mn).max())
        np.testing.assert_array_equal(am, r_am)
        if call == 0:  # another shape on the same scratch before the second call
            od = _outputs(torch, other)
            pkg.diff2_coarse_batch_static(oview, pkg.make_batch(
                odp.eulers, odp.tx, odp.ty, odp.re, odp.im, odp.corr, od[0], O=other.O, T=other.T, P=other.P,
                N_img=other.N_img, out_min=od[1], out_argmin=od[2]), pkg.PREC_BF16X3)
            torch.cuda.synchronize()
    oproj.close()
    proj.close()


def test_static_scratch_rejects_oversized_batches(pkg, synth, cuda):
    """A production-size batch (4608 orientations at image 64) needs more than
    the fixed scratch and is refused before anything runs; the header's
    example sizes fit."""
    torch = cuda
    pr = synth.make_problem("c2", P=2)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(torch, pr)
    d, mn, am = _outputs(torch, pr)
    d.fill_(-1.0)
    b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, d, O=pr.O, T=pr.T, P=pr.P,
                       N_img=pr.N_img, out_min=mn, out_argmin=am)
    assert pkg.batch_workspace_bytes(view, b, pkg.PREC_BF16X3) > pkg.STATIC_SCRATCH_BYTES
    with pytest.raises(pkg.B200D2Error) as e:
        pkg.diff2_coarse_batch_static(view, b, pkg.PREC_BF16X3)
    assert e.value.code == 7
    torch.cuda.synchronize()
    assert float(d.max().item()) == -1.0  # nothing ran
    # the header's example shape fits: 16 particles x 1024 orientations x
    # 113 translations at image 64 (the scratch holds the contraction without
    # k-splits, so its need can be below the allocating entry point's query)
    P16 = 16
    re16 = dp.re[:1].expand(P16, -1).contiguous()
    im16 = dp.im[:1].expand(P16, -1).contiguous()
    co16 = dp.corr[:1].expand(P16, -1).contiguous()
    d16 = torch.full((P16 * 1024 * pr.T,), -1.0, device="cuda")
    small = pkg.make_batch(dp.eulers, dp.tx, dp.ty, re16, im16, co16, d16, O=1024, T=pr.T, P=P16,
                           N_img=pr.N_img)
    pkg.diff2_coarse_batch_static(view, small, pkg.PREC_BF16X3)
    torch.cuda.synchronize()
    got = d16.view(P16, -1)
    assert float(got.min()) > 0.0
    assert torch.equal(got[0], got[P16 - 1])  # identical particles, identical rows
    proj.close()
