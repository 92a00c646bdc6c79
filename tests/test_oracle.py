"""CPU tests of the oracle (restatement of the reference's coarse diff2), the
synthetic workload generator and the HEALPix grid.  No GPU needed."""
from __future__ import annotations

import glob
import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def test_oracle_projector_view(oracle, synth):
    pr = synth.make_problem("c1", P=1)
    op = oracle.projector_for(pr)
    # makeKernel: maxR = min(mdlMaxR=32, imgMaxR=16); maxR2_padded = int(16^2 * 2 * 2)
    assert op.maxR == 16
    assert op.maxR2_padded == 1024
    assert pr.N_img == 544


def test_filter_image_partition(oracle, synth):
    """FilterCoarseParamImage: inside pixels first in index order, outside from the back."""
    pr = synth.make_problem("c1", P=1)
    op = oracle.projector_for(pr)
    re, im, corr, xy, n = oracle.filter_image(op, pr.fimg_re[0], pr.fimg_im[0], pr.corr[0])
    x, y = synth.pixel_coords(pr.imgX, pr.imgY, op.maxR)
    inside = (x.astype(np.int64) ** 2 + y.astype(np.int64) ** 2) * 4 <= op.maxR2_padded
    assert n == int(inside.sum()) == 414
    np.testing.assert_array_equal(re[:n], pr.fimg_re[0][inside])
    np.testing.assert_array_equal(re[n:][::-1], pr.fimg_re[0][~inside])
    np.testing.assert_array_equal(xy[0:2 * n:2], x[inside].astype(np.float32))


def test_oracle_f32_port_matches_f64(oracle, synth):
    pr = synth.make_problem("c1", P=2)
    op = oracle.projector_for(pr)
    for p in range(2):
        d64 = oracle.diff2_coarse_f64(op, pr.eulers, pr.trans_x, pr.trans_y, pr.fimg_re[p], pr.fimg_im[p], pr.corr[p])
        d32 = oracle.diff2_coarse_f32(op, pr.eulers, pr.trans_x, pr.trans_y, pr.fimg_re[p], pr.fimg_im[p], pr.corr[p])
        assert oracle.error_stats(d32, d64)["max_rel"] < 1e-5


def test_oracle_accumulates_onto_initial_buffer(oracle, synth):
    pr = synth.make_problem("g0", P=1)
    op = oracle.projector_for(pr)
    args = (op, pr.eulers, pr.trans_x, pr.trans_y, pr.fimg_re[0], pr.fimg_im[0], pr.corr[0])
    init = np.arange(pr.O * pr.T, dtype=np.float64).reshape(pr.O, pr.T)
    a = oracle.diff2_coarse_f64(*args)
    b = oracle.diff2_coarse_f64(*args, diff2_init=init)
    np.testing.assert_allclose(b - init, a, rtol=0, atol=1e-9)


def test_texture_weights_differ_from_exact(oracle, synth):
    """The 8-bit texture weights move diff2 by ~1e-5..1e-4 relative: the reason
    the FP32 drop-in keeps the texture path (parity at 1e-5)."""
    pr = synth.make_problem("c1", P=1)
    op = oracle.projector_for(pr)
    args = (op, pr.eulers, pr.trans_x, pr.trans_y, pr.fimg_re[0], pr.fimg_im[0], pr.corr[0])
    tex = oracle.diff2_coarse_f64(*args, mode=oracle.INTERP_TEX_ROUND)
    ex = oracle.diff2_coarse_f64(*args, mode=oracle.INTERP_EXACT)
    r = oracle.error_stats(tex, ex)["max_rel"]
    assert 1e-7 < r < 1e-3


def test_high_snr_recovers_true_pose(oracle, synth):
    pr = synth.make_problem("c1", P=3)
    op = oracle.projector_for(pr)
    # noiseless version of the particles: argmin must be the true pose
    import math
    x, y = synth.pixel_coords(pr.imgX, pr.imgY, op.maxR)
    for p in range(3):
        a = synth.project_exact(pr.projector, pr.eulers[pr.true_orient[p]], x, y, op.maxR)
        sh = pr.shifts[pr.true_trans[p]]
        ph = -2.0 * math.pi * (x * sh[0] + y * sh[1]) / pr.projector.ori_size
        xim = a * np.exp(-1j * ph)
        d = oracle.diff2_coarse_f64(op, pr.eulers, pr.trans_x, pr.trans_y, xim.real.astype(np.float32),
                                    xim.imag.astype(np.float32), np.ones(pr.N_img, np.float32),
                                    mode=oracle.INTERP_EXACT)
        o, t = np.unravel_index(np.argmin(d), d.shape)
        assert (o, t) == (pr.true_orient[p], pr.true_trans[p])


def test_error_stats_restatement(oracle):
    ref = np.array([1.0, 2.0, 0.0, 4.0])
    test = np.array([1.1, 2.0, 1e-3, 3.0])
    s = oracle.error_stats(test, ref)
    assert s["count"] == 4 and s["count_rel"] == 3  # |ref| <= 1e-12 skipped
    assert s["max_abs"] == pytest.approx(1.0)
    assert s["max_rel"] == pytest.approx(0.25)


def test_weights_normalised(oracle):
    mn, w = oracle.weights_from_diff2(np.array([3.0, 1.0, 2.0]))
    assert mn == 1.0 and w.sum() == pytest.approx(1.0) and np.argmax(w) == 1


def _naive_significance(w, total, frac, maxsig):
    """The same steps with a floating-point cumulative sum (numpy, sequential)."""
    pos = np.sort(w[(w > 0) & np.isfinite(w)])
    if pos.size == 0:
        return float("inf"), 0
    c = np.cumsum(pos)
    k = int(np.searchsorted(c, (1.0 - frac) * total, side="right"))
    idx = k if 1 <= k <= pos.size - 1 else 0
    nsig = pos.size - idx
    if maxsig > 0 and nsig > maxsig:
        nsig, idx = maxsig, pos.size - maxsig
    return float(pos[idx]), nsig


@pytest.mark.parametrize("seed", range(6))
def test_significance_oracle_matches_sorted_scan(oracle, seed):
    """Away from ties the exact-sum restatement equals a sort + FP64 scan."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 20000))
    w = np.exp(-rng.exponential(rng.uniform(1, 200), n))
    w[rng.random(n) < 0.2] = 0.0
    frac = float(rng.choice([0.999, 0.99, 0.5, 1.0, 0.0]))
    maxsig = int(rng.choice([0, 5, 1000]))
    sig, nsig, passed, margin = oracle.significance(w, w.sum(), frac, maxsig)
    if margin > 1e-9:
        assert (sig, nsig) == _naive_significance(w, w.sum(), frac, maxsig)
    assert passed.sum() >= nsig and (passed == (w >= sig)).all()


def test_significance_oracle_edge_cases(oracle):
    inf = float("inf")
    # no positive weight: nothing significant
    assert oracle.significance(np.zeros(5), 0.0, 0.999)[:2] == (inf, 0)
    # fraction 0: thr equals the total, no crossing, idx 0, every positive weight
    w = np.array([0.0, 1.0, 2.0, 3.0])
    assert oracle.significance(w, 6.0, 0.0)[:2] == (1.0, 3)
    # fraction 1: thr = 0 < c_0, idx 0
    assert oracle.significance(w, 6.0, 1.0)[:2] == (1.0, 3)
    # thr = 1.5: c = 1, 3, 6 -> idx 1, threshold 2, two significant
    assert oracle.significance(w, 6.0, 0.75)[:2] == (2.0, 2)
    # a cumulative sum equal to thr counts as below it (c_i <= thr)
    assert oracle.significance(w, 6.0, 0.5)[:2] == (3.0, 1)
    # ties: [1, 1, 1, 1], thr = 2.5 -> c = 1, 2, 3, 4, idx 2, threshold 1, nsig 2,
    # but all four pass the mask (w >= 1)
    sig, nsig, passed, _ = oracle.significance(np.ones(4), 4.0, 0.375)
    assert (sig, nsig, int(passed.sum())) == (1.0, 2, 4)
    # cap at two: idx = 3 - 2 = 1
    assert oracle.significance(w, 6.0, 1.0, 2)[:2] == (2.0, 2)
    # negative, NaN and infinite weights take no part in the sums
    w2 = np.array([-1.0, np.nan, np.inf, 1.0, 2.0])
    sig, nsig, passed, _ = oracle.significance(w2, 3.0, 0.5)
    assert (sig, nsig) == (2.0, 1) and passed.tolist() == [0, 0, 1, 0, 1]


@pytest.mark.parametrize("case", ["tiny", "c1"])
def test_cc_restatement_consistent_with_diff2(oracle, synth, case):
    """sum corr/2 |A - S|^2 = (normA + normX)/2 - cross, so the CC
    restatement's cross term (-cc sqrt(normA)) must equal the C oracle's FP64
    diff2 rearranged."""
    pr = synth.make_problem(case, P=1)
    proj = oracle.projector_for(pr)
    cc = oracle.cc_coarse_f64(proj, pr.eulers, pr.trans_x, pr.trans_y, pr.fimg_re[0], pr.fimg_im[0], pr.corr[0])
    d2 = np.asarray(oracle.diff2_coarse_f64(proj, pr.eulers, pr.trans_x, pr.trans_y, pr.fimg_re[0], pr.fimg_im[0],
                                            pr.corr[0]), np.float64).reshape(cc.shape)
    n = pr.N_img
    x = np.arange(n) % pr.imgX
    y = np.arange(n) // pr.imgX
    y = np.where(y > proj.maxR, y - pr.imgY, y)
    ar, ai = oracle.project_pixels(proj, pr.eulers, x.astype(np.int32), y.astype(np.int32))
    w = pr.corr[0].astype(np.float64)
    norm_a = (ar * ar + ai * ai) @ w
    norm_x = float((pr.fimg_re[0].astype(np.float64) ** 2 + pr.fimg_im[0].astype(np.float64) ** 2) @ w)
    cross_cc = -cc * np.sqrt(norm_a)[:, None]
    cross_d2 = 0.5 * (norm_a[:, None] + norm_x) - d2
    assert np.abs(cross_cc - cross_d2).max() <= 1e-9 * np.abs(cross_d2).max() + 1e-9 * norm_x
    assert np.unravel_index(cc.argmin(), cc.shape) == np.unravel_index(d2.argmin(), cc.shape)


def test_healpix_grid(synth):
    import importlib
    hp = importlib.import_module("relion_b200.healpix")
    for order in range(4):
        th, ph = hp.pix2ang_ring(2 ** order)
        assert th.size == 12 * 4 ** order
        z = np.cos(th)
        assert np.all(np.diff(z) <= 1e-12)  # RING order runs north to south
        assert abs(z.sum()) < 1e-9  # equal-area: symmetric about the equator
    eul, _ = hp.orientation_grid(1, 12)
    assert eul.shape == (576, 9)
    r = eul.reshape(-1, 3, 3).astype(np.float64)
    np.testing.assert_allclose(r @ np.swapaxes(r, 1, 2), np.broadcast_to(np.eye(3), r.shape), atol=1e-6)
    np.testing.assert_allclose(np.linalg.det(r), 1.0, atol=1e-5)


def test_config_shapes(synth):
    pr = synth.make_problem("c1")
    assert (pr.P, pr.O, pr.T, pr.N_img) == (8, 576, 21, 544)
    assert synth.translation_grid(36).shape[0] == 113
    assert synth.translation_grid(16).shape[0] == 49
    assert synth.translation_grid(4).shape[0] == 13
    assert synth.translation_grid(64).shape[0] == 197


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "ref_*.npz"))))
def test_oracle_against_reference_golden(oracle, synth, path):
    """Golden vectors written by the reference's own kernels (runDiff2KernelCoarse
    and runDiff2KernelCoarseDouble, compiled from the reference sources and run
    on a B200 by tests/golden/make_golden.py), with the texture unit's
    projections at every pixel stored beside them: the box-16 problem g0 and
    a C1-sized slice (image 32, radius 16, 21 translations, every 9th of the
    576 orientations, 2 particles) whose inputs are rebuilt from the seeded
    generator and checked by digest.

    * Given the hardware projections, the oracle's FP64 arithmetic (phase
      shift, corr/2 weighting, sum, accumulation) reproduces the reference's
      FP64 kernel to 1e-9 on at least 90 % of the orientations (all of g0's)
      and to 1e-6 on every one, and its FP32 kernel to 1e-5.  The stored
      projections sample at FP32 positions, as the reference's FP32 kernel
      does; its FP64 kernel forms the positions in FP64
      (project3DmodelDouble), so at the few orientations where a sample lies
      next to a 1/256 weight step of the texture unit it reads a slightly
      different value (3 of the 64 C1 orientations here).
    * With its own texture-weight model the oracle is within 5e-4: the B200
      texture unit rounds the eight corner weights jointly to 1/256 in a way
      the model approximates but does not reproduce exactly."""
    import golden_util
    g = golden_util.load(path, synth)
    op = oracle.Projector(g.pv, g.imgX, g.imgY, g.imgMaxR)
    for p in range(g.P):
        d = oracle.diff2_from_projections(op, g.prj_re, g.prj_im, g.trans_x, g.trans_y, g.fimg_re[p], g.fimg_im[p],
                                          g.corr[p])
        s_d = oracle.error_stats(d, g.ref_f64[p])
        s_f = oracle.error_stats(d, g.ref_f32[p])
        rel = np.abs(d - g.ref_f64[p]) / np.abs(g.ref_f64[p])
        exact = int((rel.max(axis=1) < 1e-9).sum())
        assert exact >= 0.9 * g.O, (exact, g.O)
        assert s_d["max_rel"] < 1e-6, s_d
        assert s_f["max_rel"] < 1e-5, s_f
        d = oracle.diff2_coarse_f64(op, g.eulers, g.trans_x, g.trans_y, g.fimg_re[p], g.fimg_im[p], g.corr[p],
                                    mode=oracle.INTERP_TEX_ROUND)
        assert oracle.error_stats(d, g.ref_f64[p])["max_rel"] < 5e-4
