"""Tensor-core batch path (tcgen05) against the FP64 GPU kernel on the same
projections, and against the FP32 drop-in.

Stated tolerances (max relative diff2 error vs FP64, over every evaluation):
  BF16x3 (hi*hi + hi*lo + lo*hi)  1e-5
  TF32x3                          1e-5
  TF32 (single product)           1e-3
  FP16x3 (scaled hi/lo split)     1e-5
  FP16 (scaled, single product)   1e-3
The argmin (o, t) must equal the FP64 argmin wherever the FP64 best-to-second
gap exceeds twice the tolerance."""
from __future__ import annotations

import math

import numpy as np
import pytest

from gpu_util import DeviceProblem, argmin_consistent, ours_f64

pytestmark = pytest.mark.gpu
TOL = {"bf16x3": 1e-5, "tf32x3": 1e-5, "tf32": 1e-3, "fp16x3": 1e-5, "fp16": 1e-3}
ALL = ["bf16x3", "tf32x3", "tf32", "fp16x3", "fp16"]


def prec_code(pkg, name):
    return {"bf16x3": pkg.PREC_BF16X3, "tf32x3": pkg.PREC_TF32X3, "tf32": pkg.PREC_TF32,
            "fp16x3": pkg.PREC_FP16X3, "fp16": pkg.PREC_FP16}[name]


def run_tc(pkg, torch, view, dp, prec, accumulate=False, init=None, stages=False):
    pr = dp.pr
    out = torch.zeros(pr.P * pr.O * pr.T, device="cuda")
    if init is not None:
        out.copy_(torch.as_tensor(np.asarray(init, np.float32).reshape(-1), device="cuda"))
    mn = torch.empty(pr.P, device="cuda", dtype=torch.float64)
    am = torch.empty(pr.P, device="cuda", dtype=torch.int64)
    b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, out, O=pr.O, T=pr.T, P=pr.P,
                       N_img=pr.N_img, accumulate=accumulate, out_min=mn, out_argmin=am)
    nb = pkg.batch_workspace_bytes(view, b, prec)
    ws = torch.empty(nb, device="cuda", dtype=torch.uint8)
    if stages:
        pkg.kernel_breakdown(view, b, prec, ws, reps=1)
    else:
        pkg.diff2_coarse_batch(view, b, prec, ws)
    torch.cuda.synchronize()
    assert pkg.workspace_status(ws) == 0
    return out.cpu().numpy().reshape(pr.P, pr.O, pr.T), mn.cpu().numpy(), am.cpu().numpy()


def fp64_all(pkg, view, dp):
    return np.stack([ours_f64(pkg, view, dp, p) for p in range(dp.pr.P)])


@pytest.fixture(scope="module")
def tiny(pkg, synth, cuda):
    pr = synth.make_problem("tiny")
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(cuda, pr)
    yield pr, view, dp, fp64_all(pkg, view, dp)
    proj.close()


@pytest.fixture(scope="module")
def c1(pkg, synth, cuda):
    pr = synth.make_problem("c1")
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(cuda, pr)
    yield pr, view, dp, fp64_all(pkg, view, dp)
    proj.close()


def _check(pkg, oracle, cuda, case, name):
    pr, view, dp, ref = case
    got, mn, am = run_tc(pkg, cuda, view, dp, prec_code(pkg, name))
    s = oracle.error_stats(got, ref)
    print(name, pr.name, "max rel %.3g avg rel %.3g" % (s["max_rel"], s["avg_rel"]))
    assert s["max_rel"] <= TOL[name], s
    for p in range(pr.P):
        ok, gap = argmin_consistent(got[p], ref[p], TOL[name])
        assert ok, (p, gap)
        assert am[p] == int(np.argmin(got[p].ravel()))
        assert mn[p] == pytest.approx(float(got[p].min()), rel=1e-7)
    return s


@pytest.mark.parametrize("name", ALL)
def test_tc_tiny(pkg, oracle, cuda, tiny, name):
    _check(pkg, oracle, cuda, tiny, name)


@pytest.mark.parametrize("name", ALL)
def test_tc_c1(pkg, oracle, cuda, c1, name):
    _check(pkg, oracle, cuda, c1, name)


@pytest.mark.parametrize("P", [32, 40, 128])
def test_tc_norm_tile_shapes(pkg, synth, oracle, cuda, P):
    """The FP64 norm kernel picks its particle x orientation tile by batch
    size: with 4608 orientations, 32 particles take 16 x 32 tiles, 40 take
    16 x 64 and 128 take 32 x 64 (C2's 256 take 64 x 64, C1 16 x 16).  Every
    shape gives the same diff2, min and argmin as the FP64 kernel within the
    BF16x3 tolerance.  Five of the 113 translations keep the FP64 reference
    short; the tile choice depends only on particles and orientations."""
    import dataclasses
    pr = synth.make_problem("c2", P=P)
    pr = dataclasses.replace(pr, trans_x=pr.trans_x[:5].copy(), trans_y=pr.trans_y[:5].copy(),
                             shifts=pr.shifts[:5].copy())
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(cuda, pr)
    try:
        _check(pkg, oracle, cuda, (pr, view, dp, fp64_all(pkg, view, dp)), "bf16x3")
    finally:
        proj.close()


def test_tc_c2_subset(pkg, synth, oracle, cuda):
    pr = synth.make_problem("c2", P=6)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(cuda, pr)
    ref = fp64_all(pkg, view, dp)
    for name in ("bf16x3", "tf32x3", "fp16x3"):
        _check(pkg, oracle, cuda, (pr, view, dp, ref), name)
    proj.close()


def test_tc_accumulate_and_stages(pkg, oracle, cuda, tiny):
    pr, view, dp, ref = tiny
    init = np.random.default_rng(3).uniform(0, 50, (pr.P, pr.O, pr.T)).astype(np.float32)
    got, _, _ = run_tc(pkg, cuda, view, dp, pkg.PREC_BF16X3, accumulate=True, init=init)
    assert oracle.error_stats(got - init, ref)["max_rel"] <= 1e-5
    got2, _, _ = run_tc(pkg, cuda, view, dp, pkg.PREC_BF16X3, stages=True)
    np.testing.assert_array_equal(got2, run_tc(pkg, cuda, view, dp, pkg.PREC_BF16X3)[0])


@pytest.mark.parametrize("o_lim,r2,P", [(37, 5, 1), (300, 0, 3), (257, 64, 2)])
def test_tc_ragged(pkg, synth, oracle, cuda, o_lim, r2, P):
    """O not a multiple of 256, P*T not a multiple of 128, T = 1 and T = 197."""
    pr = synth.make_problem("c1", P=P, orient_limit=o_lim)
    sh = synth.translation_grid(r2)
    pr.shifts = sh
    pr.trans_x = (-2 * math.pi * sh[:, 0] / pr.projector.ori_size).astype(np.float32)
    pr.trans_y = (-2 * math.pi * sh[:, 1] / pr.projector.ori_size).astype(np.float32)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(cuda, pr)
    ref = fp64_all(pkg, view, dp)
    for prec in (pkg.PREC_BF16X3, pkg.PREC_FP16X3):
        got, mn, am = run_tc(pkg, cuda, view, dp, prec)
        assert got.shape == (P, o_lim, sh.shape[0])
        assert oracle.error_stats(got, ref)["max_rel"] <= 1e-5
    proj.close()


def test_tc_deterministic(pkg, cuda, tiny):
    pr, view, dp, ref = tiny
    a = run_tc(pkg, cuda, view, dp, pkg.PREC_BF16X3)
    b = run_tc(pkg, cuda, view, dp, pkg.PREC_BF16X3)
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[2], b[2])


@pytest.mark.parametrize("rb,tn,split,pair", [(64, 256, 1, 2), (64, 256, 2, 2), (64, 256, 4, 2), (128, 256, 2, 2),
                                              (64, 128, 1, 2), (64, 128, 4, 2), (128, 128, 1, 2),
                                              (64, 256, 1, 1), (128, 256, 1, 1)])
def test_tc_gemm_variants(pkg, oracle, cuda, c1, rb, tn, split, pair):
    """Every contraction variant (k-block row width, tile width, k-splits with
    FP64 addition of the partials, CTA-pair tiles) meets the same tolerance,
    and a run is reproducible bit for bit."""
    pr, view, dp, ref = c1
    pkg.set_gemm_variant(rb, tn, split, pair)
    try:
        got, mn, am = run_tc(pkg, cuda, view, dp, pkg.PREC_BF16X3)
        again, _, _ = run_tc(pkg, cuda, view, dp, pkg.PREC_BF16X3)
    finally:
        pkg.set_gemm_variant(0, 0, 0, 0)
    np.testing.assert_array_equal(got, again)
    s = oracle.error_stats(got, ref)
    assert s["max_rel"] <= TOL["bf16x3"], s
    for p in range(pr.P):
        assert am[p] == int(np.argmin(got[p].ravel()))
        ok, gap = argmin_consistent(got[p], ref[p], TOL["bf16x3"])
        assert ok, (p, gap)


@pytest.mark.parametrize("name", ["bf16x3", "tf32", "fp16x3"])
def test_tc_pair_tiles_c2_subset(pkg, synth, oracle, cuda, name):
    """CTA-pair tiles (cta_group::2) on a C2 subset: several 256 x 256 tiles
    per pair, O not a multiple of 256 handled by the epilogue."""
    pr = synth.make_problem("c2", P=5, orient_limit=1000)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(cuda, pr)
    ref = fp64_all(pkg, view, dp)
    pkg.set_gemm_variant(0, 0, 1, 1)
    try:
        _check(pkg, oracle, cuda, (pr, view, dp, ref), name)
    finally:
        pkg.set_gemm_variant(0, 0, 0, 0)
    proj.close()


@pytest.mark.parametrize("case,variant", [("c1", (0, 0, 0, 0)), ("c1", (64, 256, 4, 2)), ("c1", (64, 256, 1, 2)),
                                          ("c2", (0, 0, 1, 1))])
def test_combine_df32_matches_fp64_combine(pkg, synth, oracle, cuda, case, variant):
    """The double-float combine (nA as hi + lo floats, one FMA and one add)
    stays within 2 ulp of the FP64 combine rounded to FP32, on the default
    small-batch choice (128-wide tiles), a 4-way k-split, single-CTA
    256-wide and CTA-pair contractions."""
    pr = synth.make_problem(case, P=5 if case == "c2" else None, orient_limit=700 if case == "c2" else None)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(cuda, pr)
    pkg.set_gemm_variant(*variant)
    try:
        pkg.set_combine(pkg.COMBINE_FP64)
        d64, mn64, am64 = run_tc(pkg, cuda, view, dp, pkg.PREC_BF16X3)
        pkg.set_combine(pkg.COMBINE_DF32)
        d32, mn32, am32 = run_tc(pkg, cuda, view, dp, pkg.PREC_BF16X3)
    finally:
        pkg.set_combine(pkg.COMBINE_DF32)
        pkg.set_gemm_variant(0, 0, 0, 0)
    ulp = np.spacing(np.abs(d64).astype(np.float32))
    assert np.all(np.abs(d32.astype(np.float64) - d64) <= 2 * ulp)
    ref = fp64_all(pkg, view, dp)
    assert oracle.error_stats(d32, ref)["max_rel"] <= TOL["bf16x3"]
    proj.close()



@pytest.mark.parametrize("bad", [(600.0, 0.0), (-1.0, 3.0), (2.0, -513.0), (2.5, 1.0)])
def test_listed_coordinate_out_of_range_reported(pkg, synth, oracle, cuda, bad):
    """Caller-listed pixel coordinates are device data: one that lies outside
    x in [0, 512], y in [-512, 512], or is not an integer, sets the workspace
    status word to B200D2_ERR_INVALID; the same batch with valid coordinates
    reports 0."""
    torch = cuda
    pr = synth.make_problem("tiny")
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(torch, pr)
    op = oracle.projector_for(pr)
    cols = [oracle.filter_image(op, pr.fimg_re[p], pr.fimg_im[p], pr.corr[p]) for p in range(pr.P)]
    t = lambda a: torch.as_tensor(np.ascontiguousarray(np.stack(a)), device="cuda")  # noqa: E731
    re, im, corr = t([c[0] for c in cols]), t([c[1] for c in cols]), t([c[2] for c in cols])
    n_listed = cols[0][4]
    for corrupt in (False, True):
        xy = cols[0][3].copy()
        if corrupt:
            xy[2 * (n_listed // 2)], xy[2 * (n_listed // 2) + 1] = bad
        coor = torch.as_tensor(xy, device="cuda")
        out = torch.zeros(pr.P * pr.O * pr.T, device="cuda")
        b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, re, im, corr, out, O=pr.O, T=pr.T, P=pr.P, N_img=pr.N_img,
                           coor_xy=coor, n_listed=n_listed)
        ws = torch.empty(pkg.batch_workspace_bytes(view, b, pkg.PREC_BF16X3), device="cuda", dtype=torch.uint8)
        pkg.diff2_coarse_batch(view, b, pkg.PREC_BF16X3, ws)
        torch.cuda.synchronize()
        assert pkg.workspace_status(ws) == (1 if corrupt else 0)
    proj.close()


def test_bounded_wait_gives_up_and_context_stays_usable(pkg, synth, oracle, cuda):
    """The contraction's device-side waits are bounded.  With the pipeline-wait
    limit of the single-CTA contraction cut to 1 us (a test hook), its waits
    for an accumulator run out before the first tile's MMAs finish: the kernel
    raises its abort flag, lets its copies and MMAs in flight finish, frees
    its tensor memory and returns, and the workspace status reads
    B200D2_ERR_TIMEOUT.  The call returns, the context stays usable, and the
    next call with the default limit gives correct results in the same
    workspace."""
    torch = cuda
    pr = synth.make_problem("c1")
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(torch, pr)
    ref = fp64_all(pkg, view, dp)
    out = torch.zeros(pr.P * pr.O * pr.T, device="cuda")
    b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, out, O=pr.O, T=pr.T, P=pr.P,
                       N_img=pr.N_img)
    ws = torch.empty(pkg.batch_workspace_bytes(view, b, pkg.PREC_BF16X3), device="cuda", dtype=torch.uint8)
    pkg.set_gemm_variant(64, 256, 1, 2)  # single-CTA tiles: the kernel the hook applies to
    try:
        pkg.set_wait_limit_ns(1000)
        try:
            pkg.diff2_coarse_batch(view, b, pkg.PREC_BF16X3, ws)
            torch.cuda.synchronize()
        finally:
            pkg.set_wait_limit_ns(0)
        assert pkg.workspace_status(ws) == 5  # B200D2_ERR_TIMEOUT
        out.zero_()
        pkg.diff2_coarse_batch(view, b, pkg.PREC_BF16X3, ws)
        torch.cuda.synchronize()
        assert pkg.workspace_status(ws) == 0
    finally:
        pkg.set_gemm_variant(0, 0, 0, 0)
    got = out.cpu().numpy().reshape(pr.P, pr.O, pr.T)
    assert oracle.error_stats(got, ref)["max_rel"] <= TOL["bf16x3"]
    proj.close()


def test_batch_graphs_match_direct_launches(pkg, oracle, cuda, c1):
    """The batch entry point's cached graphs: calls 2.. with the same
    arguments launch a captured graph of the pipeline.  Outputs are bit
    identical to direct launches, inputs refilled in place are picked up, a
    different output buffer is a new signature, the launch count stays the
    number of kernels, and a caller's own capture of the call still works."""
    torch = cuda
    pr, view, dp, ref = c1
    prec = pkg.PREC_BF16X3

    def run(out, mn, am, stream=None):
        b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, out, O=pr.O, T=pr.T, P=pr.P,
                           N_img=pr.N_img, out_min=mn, out_argmin=am)
        pkg.diff2_coarse_batch(view, b, prec, ws, stream)

    mk = lambda: (torch.zeros(pr.P * pr.O * pr.T, device="cuda"),  # noqa: E731
                  torch.empty(pr.P, device="cuda", dtype=torch.float64),
                  torch.empty(pr.P, device="cuda", dtype=torch.int64))
    o = mk()
    b0 = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, o[0], O=pr.O, T=pr.T, P=pr.P, N_img=pr.N_img)
    ws = torch.empty(pkg.batch_workspace_bytes(view, b0, prec), device="cuda", dtype=torch.uint8)
    pkg.set_batch_graphs(False)
    try:
        run(*o)
        torch.cuda.synchronize()
        direct = [t.clone() for t in o]
        n0 = pkg.launch_count()
        run(*o)
        torch.cuda.synchronize()
        per_call = pkg.launch_count() - n0
    finally:
        pkg.set_batch_graphs(True)
    outs = []
    for k in range(4):  # direct, capture + launch, launch, launch
        n0 = pkg.launch_count()
        o[0].fill_(-1.0)
        run(*o)
        torch.cuda.synchronize()
        assert pkg.launch_count() - n0 == per_call
        outs.append(o[0].clone())
        for a, b in zip(o, direct):
            assert torch.equal(a, b), k
    # inputs refilled in place: the graph reads the new values
    saved = dp.re.clone()
    dp.re.mul_(0.5)
    run(*o)
    torch.cuda.synchronize()
    changed = o[0].clone()
    pkg.set_batch_graphs(False)
    try:
        run(*o)
        torch.cuda.synchronize()
        assert torch.equal(o[0], changed)
    finally:
        pkg.set_batch_graphs(True)
        dp.re.copy_(saved)
    assert not torch.equal(changed, direct[0])
    # a new output buffer is a new signature
    o2 = mk()
    for _ in range(3):
        run(*o2)
    torch.cuda.synchronize()
    assert torch.equal(o2[0], direct[0])
    # the caller captures the call into its own graph
    o3 = mk()
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        run(*o3, stream=s)  # warm (attributes set outside the capture)
    torch.cuda.synchronize()
    o3[0].fill_(-1.0)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=s):
        run(*o3, stream=s)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(o3[0], direct[0])
    del g
