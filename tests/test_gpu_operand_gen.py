"""The A operand generated inside the contraction (shared memory) against the
materialised one (the default: written to the workspace by its own kernel and
read back by TMA): both compute every element with the same roundings, so
diff2, the per-particle minimum and the argmin must be bit-identical, for

- every contraction kernel: single-CTA 128- and 256-wide tiles with 64- and
  128-byte k-rows, k-splits, CTA-pair tiles with both row widths;
- every tensor-core precision (the FP16 forms with their particle scales);
- caller-listed pixels (the reference's filtered layout);
- translations whose distinct values do not fit the shared phase rows (the
  kernel then reads the (translation, pixel) products from global memory);
- uneven batches (plans), and the CC score.
Accuracy against FP64 is covered by the other tensor-core tests, which run
the materialised form."""
from __future__ import annotations

import math

import numpy as np
import pytest

from gpu_util import DeviceProblem

pytestmark = pytest.mark.gpu


def _run(pkg, torch, view, dp, prec, gen, variant=(0, 0, 0, 0), T=None, tx=None, ty=None, coor=None, n_listed=0,
         re=None, im=None, corr=None, score=0):
    pr = dp.pr
    T = pr.T if T is None else T
    pkg.set_operand_gen(gen)
    pkg.set_gemm_variant(*variant)
    try:
        out = torch.zeros(pr.P * pr.O * T, device="cuda")
        mn = torch.empty(pr.P, device="cuda", dtype=torch.float64)
        am = torch.empty(pr.P, device="cuda", dtype=torch.int64)
        b = pkg.make_batch(dp.eulers, dp.tx if tx is None else tx, dp.ty if ty is None else ty,
                           dp.re if re is None else re, dp.im if im is None else im,
                           dp.corr if corr is None else corr, out, O=pr.O, T=T, P=pr.P, N_img=pr.N_img,
                           out_min=mn, out_argmin=am, coor_xy=coor, n_listed=n_listed, score=score)
        ws = torch.empty(pkg.batch_workspace_bytes(view, b, prec), device="cuda", dtype=torch.uint8)
        pkg.diff2_coarse_batch(view, b, prec, ws)
        torch.cuda.synchronize()
        assert pkg.workspace_status(ws) == 0
        return out.cpu().numpy(), mn.cpu().numpy(), am.cpu().numpy(), ws.numel()
    finally:
        pkg.set_operand_gen(0)
        pkg.set_gemm_variant(0, 0, 0, 0)


def _same(a, b):
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])
    np.testing.assert_array_equal(a[2], b[2])


@pytest.fixture(scope="module")
def c1(pkg, synth, cuda):
    pr = synth.make_problem("c1")
    proj = pkg.Projector(pr.projector, use_texture=1)
    yield pr, proj.view(pr.imgX, pr.imgY, pr.imgMaxR), DeviceProblem(cuda, pr)
    proj.close()


@pytest.fixture(scope="module")
def c2s(pkg, synth, cuda):
    pr = synth.make_problem("c2", P=5, orient_limit=1000)
    proj = pkg.Projector(pr.projector, use_texture=1)
    yield pr, proj.view(pr.imgX, pr.imgY, pr.imgMaxR), DeviceProblem(cuda, pr)
    proj.close()


@pytest.mark.parametrize("variant", [(0, 0, 0, 0), (64, 256, 1, 2), (128, 256, 1, 2), (64, 128, 1, 2),
                                     (128, 128, 1, 2), (64, 256, 4, 2), (64, 256, 1, 1), (128, 256, 1, 1)])
def test_generated_operand_bit_identical_kernels(pkg, cuda, c1, variant):
    pr, view, dp = c1
    a = _run(pkg, cuda, view, dp, pkg.PREC_BF16X3, 1, variant)
    b = _run(pkg, cuda, view, dp, pkg.PREC_BF16X3, 0, variant)
    _same(a, b)
    assert a[3] < b[3]  # no A planes in the workspace


@pytest.mark.parametrize("prec", ["tf32", "tf32x3", "fp16", "fp16x3", "bf16x3"])
@pytest.mark.parametrize("variant", [(0, 0, 1, 1), (64, 256, 1, 1)])
def test_generated_operand_bit_identical_precisions_pairs(pkg, cuda, c2s, prec, variant):
    pr, view, dp = c2s
    code = {"tf32": pkg.PREC_TF32, "tf32x3": pkg.PREC_TF32X3, "fp16": pkg.PREC_FP16, "fp16x3": pkg.PREC_FP16X3,
            "bf16x3": pkg.PREC_BF16X3}[prec]
    _same(_run(pkg, cuda, view, dp, code, 1, variant), _run(pkg, cuda, view, dp, code, 0, variant))


def test_generated_operand_cc_score(pkg, cuda, c1):
    pr, view, dp = c1
    _same(_run(pkg, cuda, view, dp, pkg.PREC_BF16X3, 1, score=pkg.SCORE_CC),
          _run(pkg, cuda, view, dp, pkg.PREC_BF16X3, 0, score=pkg.SCORE_CC))


def test_generated_operand_listed_pixels(pkg, oracle, cuda, c1):
    pr, view, dp = c1
    torch = cuda
    op = oracle.projector_for(pr)
    cols = [oracle.filter_image(op, pr.fimg_re[p], pr.fimg_im[p], pr.corr[p]) for p in range(pr.P)]
    t = lambda a: torch.as_tensor(np.ascontiguousarray(np.stack(a)), device="cuda")  # noqa: E731
    kw = dict(re=t([c[0] for c in cols]), im=t([c[1] for c in cols]), corr=t([c[2] for c in cols]),
              coor=torch.as_tensor(cols[0][3], device="cuda"), n_listed=cols[0][4])
    _same(_run(pkg, cuda, view, dp, pkg.PREC_BF16X3, 1, **kw), _run(pkg, cuda, view, dp, pkg.PREC_BF16X3, 0, **kw))


def test_generated_operand_phase_rows_in_global_memory(pkg, cuda, c1):
    """300 translations with distinct non-integer shifts: their deduplicated
    phase rows (300 x 17 + 300 x 33 entries) exceed the shared-memory table,
    so the generator reads the (translation, pixel) products from global
    memory; the operand stays bit-identical."""
    pr, view, dp = c1
    torch = cuda
    rng = np.random.default_rng(11)
    sh = rng.uniform(-3.0, 3.0, (300, 2))
    tx = torch.as_tensor((-2 * math.pi * sh[:, 0] / pr.projector.ori_size).astype(np.float32), device="cuda")
    ty = torch.as_tensor((-2 * math.pi * sh[:, 1] / pr.projector.ori_size).astype(np.float32), device="cuda")
    for variant in ((0, 0, 0, 0), (128, 256, 1, 1)):
        _same(_run(pkg, cuda, view, dp, pkg.PREC_BF16X3, 1, variant, T=300, tx=tx, ty=ty),
              _run(pkg, cuda, view, dp, pkg.PREC_BF16X3, 0, variant, T=300, tx=tx, ty=ty))


@pytest.mark.parametrize("variant", [(128, 256, 1, 1), (64, 128, 1, 2), (64, 256, 2, 2)])
def test_generated_operand_plans(pkg, synth, cuda, variant):
    torch = cuda
    P = 6
    pr = synth.make_problem("c4", P=P, seed=7)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dev = lambda a: torch.as_tensor(np.ascontiguousarray(a), device="cuda")  # noqa: E731
    eul = dev(pr.eulers.reshape(-1))
    outs = []
    for gen in (1, 0):
        parts = []
        for p in range(P):
            ol, tl = pr.orient_lists[p], pr.trans_lists[p]
            parts.append(dict(real=dev(pr.fimg_re[p]), imag=dev(pr.fimg_im[p]), corr=dev(pr.corr[p]),
                              diff2=torch.zeros(len(ol) * len(tl), device="cuda"), orient=ol,
                              trans_x=tl[:, 0].copy(), trans_y=tl[:, 1].copy()))
        mn = torch.empty(P, device="cuda", dtype=torch.float64)
        am = torch.empty(P, device="cuda", dtype=torch.int64)
        pkg.set_operand_gen(gen)
        pkg.set_gemm_variant(*variant)
        try:
            plan = pkg.Plan(view, eul, pr.O, pr.N_img, parts, pkg.PREC_BF16X3, flags=pkg.PLAN_GRAPH | pkg.PLAN_REORDER,
                            out_min=mn, out_argmin=am)
        finally:
            pkg.set_operand_gen(0)
            pkg.set_gemm_variant(0, 0, 0, 0)
        plan.run()
        torch.cuda.synchronize()
        outs.append(([pt["diff2"].cpu().numpy() for pt in parts], mn.cpu().numpy(), am.cpu().numpy()))
        plan.close()
    for a, b in zip(outs[0][0], outs[1][0]):
        np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    np.testing.assert_array_equal(outs[0][2], outs[1][2])
    proj.close()
