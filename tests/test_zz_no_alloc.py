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


def test_static_scratch_matches_allocating_entry_point(pkg, synth, oracle, cuda):
    torch = cuda
    pr = synth.make_problem("c1")
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(torch, pr)

    def batch(out):
        d, mn, am = out
        return pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, d, O=pr.O, T=pr.T, P=pr.P,
                              N_img=pr.N_img, out_min=mn, out_argmin=am)

    ref = _outputs(torch, pr)
    b = batch(ref)
    need = pkg.batch_workspace_bytes(view, b, pkg.PREC_BF16X3)
    assert 0 < need <= pkg.STATIC_SCRATCH_BYTES
    ws = torch.empty(need, device="cuda", dtype=torch.uint8)
    pkg.diff2_coarse_batch(view, b, pkg.PREC_BF16X3, ws)
    torch.cuda.synchronize()
    r_d, r_mn, r_am = (t.cpu().numpy() for t in ref)

    for call in range(2):
        out = _outputs(torch, pr)
        pkg.diff2_coarse_batch_static(view, batch(out), pkg.PREC_BF16X3)
        torch.cuda.synchronize()
        d, mn, am = (t.cpu().numpy() for t in out)
        s = oracle.error_stats(d, r_d)
        assert s["max_rel"] <= TOL, (call, s)
        np.testing.assert_allclose(mn, r_mn, rtol=TOL)
        np.testing.assert_array_equal(am, r_am)
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
