"""Plans: particles with uneven orientation subsets and translation sets in one
persistent contraction launch, autotuned and captured in a CUDA graph.
Each particle's diff2 is checked against the FP64 CUDA-core kernel run on
that particle's own orientation subset and translations (tolerance 1e-5, as
for the uniform BF16x3 batch)."""
from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _plan_case(pkg, synth, torch, P, name="c4", seed=7):
    pr = synth.make_problem(name, P=P, seed=seed)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    eul = dev(pr.eulers.reshape(-1))
    parts = []
    for p in range(P):
        ol, tl = pr.orient_lists[p], pr.trans_lists[p]
        parts.append(dict(real=dev(pr.fimg_re[p]), imag=dev(pr.fimg_im[p]), corr=dev(pr.corr[p]),
                          diff2=torch.zeros(len(ol) * len(tl), device="cuda"), orient=ol,
                          trans_x=tl[:, 0].copy(), trans_y=tl[:, 1].copy()))
    return pr, proj, view, eul, parts


def _fp64_particle(pkg, torch, view, pr, part, p):
    ol = part["orient"]
    eul = torch.as_tensor(np.ascontiguousarray(pr.eulers[ol].reshape(-1)), device="cuda")
    tx = torch.as_tensor(part["trans_x"], device="cuda")
    ty = torch.as_tensor(part["trans_y"], device="cuda")
    out = torch.zeros(len(ol) * tx.numel(), device="cuda", dtype=torch.float64)
    pkg.run_diff2_kernel_coarse_double(view, tx, ty, part["corr"], part["real"], part["imag"], eul, out, len(ol),
                                       tx.numel(), pr.N_img)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("reorder", [False, True])
def test_uneven_plan_matches_fp64(pkg, synth, oracle, cuda, reorder):
    torch = cuda
    P = 6
    pr, proj, view, eul, parts = _plan_case(pkg, synth, torch, P)
    mn = torch.empty(P, device="cuda", dtype=torch.float64)
    am = torch.empty(P, device="cuda", dtype=torch.int64)
    flags = pkg.PLAN_AUTOTUNE | pkg.PLAN_GRAPH | (pkg.PLAN_REORDER if reorder else 0)
    plan = pkg.Plan(view, eul, pr.O, pr.N_img, parts, pkg.PREC_BF16X3, flags=flags, out_min=mn, out_argmin=am)
    info = plan.info()
    print(info)
    assert info["graph"] == 1 and info["row_bytes"] in (64, 128)
    assert info["tile_n"] in (128, 256) and info["split"] >= 1
    # the autotuner timed every variant and kept the fastest (a plan with the
    # same problem signature as an earlier one reuses its choice untimed)
    if info["n_tuned"]:
        assert info["n_tuned"] >= 4
        best = min(info["tuned"], key=lambda x: x[1])[0]
        assert best == (info["row_bytes"], info["tile_n"], info["split"], 1 if info["pair"] else 2)
    assert 0 < info["tiles_n128"] <= 2 * info["tiles"]
    assert info["evals"] == sum(len(p["orient"]) * len(p["trans_x"]) for p in parts)
    assert 0 < info["tiles"] <= info["tiles_dense"]
    for rep in range(2):  # the graph replays on the same buffers
        for pt in parts:
            pt["diff2"].fill_(-7.0)
        plan.run()
        torch.cuda.synchronize()
        for p, pt in enumerate(parts):
            got = pt["diff2"].cpu().numpy()
            ref = _fp64_particle(pkg, torch, view, pr, pt, p)
            s = oracle.error_stats(got, ref)
            assert s["max_rel"] <= TOL, (rep, p, s)
            assert am[p].item() == int(np.argmin(got))
            assert mn[p].item() == pytest.approx(float(got.min()), rel=1e-7)
    # refill one image in place: the replay sees the new data
    parts[2]["real"].mul_(1.5)
    parts[2]["imag"].mul_(0.5)
    plan.run()
    torch.cuda.synchronize()
    got = parts[2]["diff2"].cpu().numpy()
    ref = _fp64_particle(pkg, torch, view, pr, parts[2], 2)
    assert oracle.error_stats(got, ref)["max_rel"] <= TOL
    plan.close()
    proj.close()


def test_plan_uniform_matches_batch_api(pkg, synth, oracle, cuda):
    """Particles sharing all orientations and translations through a plan give
    the batch API's result (same kernels, tabled indexing)."""
    torch = cuda
    pr = synth.make_problem("c1", P=4)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    eul, tx, ty = dev(pr.eulers.reshape(-1)), dev(pr.trans_x), dev(pr.trans_y)
    re, im, corr = dev(pr.fimg_re), dev(pr.fimg_im), dev(pr.corr)
    out = torch.zeros(pr.P * pr.O * pr.T, device="cuda")
    b = pkg.make_batch(eul, tx, ty, re, im, corr, out, O=pr.O, T=pr.T, P=pr.P, N_img=pr.N_img)
    ws = torch.empty(pkg.batch_workspace_bytes(view, b, pkg.PREC_BF16X3), device="cuda", dtype=torch.uint8)
    pkg.diff2_coarse_batch(view, b, pkg.PREC_BF16X3, ws)
    parts = [dict(real=re[p], imag=im[p], corr=corr[p], diff2=torch.zeros(pr.O * pr.T, device="cuda"),
                  orient=None, O=pr.O, trans_x=pr.trans_x, trans_y=pr.trans_y) for p in range(pr.P)]
    plan = pkg.Plan(view, eul, pr.O, pr.N_img, parts, pkg.PREC_BF16X3, flags=pkg.PLAN_GRAPH)
    plan.run()
    torch.cuda.synchronize()
    ref = out.cpu().numpy().reshape(pr.P, -1)
    for p in range(pr.P):
        assert oracle.error_stats(parts[p]["diff2"].cpu().numpy(), ref[p])["max_rel"] <= 1e-6
    plan.close()
    proj.close()


@pytest.mark.parametrize("variant", [(128, 256, 1, 1), (64, 128, 1, 2)])
def test_uneven_plan_fixed_variants(pkg, synth, oracle, cuda, variant):
    """Plans without the autotuner take the process-wide contraction variant:
    CTA-pair 256 x 256 tiles and 128-wide single-CTA tiles on uneven work lists."""
    torch = cuda
    P = 5
    pr, proj, view, eul, parts = _plan_case(pkg, synth, torch, P)
    mn = torch.empty(P, device="cuda", dtype=torch.float64)
    am = torch.empty(P, device="cuda", dtype=torch.int64)
    pkg.set_gemm_variant(*variant)
    try:
        plan = pkg.Plan(view, eul, pr.O, pr.N_img, parts, pkg.PREC_BF16X3, flags=pkg.PLAN_GRAPH | pkg.PLAN_REORDER,
                        out_min=mn, out_argmin=am)
    finally:
        pkg.set_gemm_variant(0, 0, 0, 0)
    info = plan.info()
    assert info["pair"] == (1 if variant[3] == 1 else 0) and info["tile_n"] == variant[1]
    assert info["tiles_pair"] > 0
    for pt in parts:
        pt["diff2"].fill_(-7.0)
    plan.run()
    torch.cuda.synchronize()
    for p, pt in enumerate(parts):
        got = pt["diff2"].cpu().numpy()
        ref = _fp64_particle(pkg, torch, view, pr, pt, p)
        assert oracle.error_stats(got, ref)["max_rel"] <= TOL, p
        assert am[p].item() == int(np.argmin(got))
    plan.close()
    proj.close()

