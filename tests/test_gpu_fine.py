"""Fine-pass diff2 over a job list (b200d2_diff2_fine) against the
reference's own cuda_kernel_diff2_fine (src/diff2.cuh:540-682, compiled into
oracle/_ref) on the same device buffers and job lists, and against this
library's FP64 coarse kernel (every (orientation, translation) pair scored
over all pixels, plus sum_init).  The CC form (b200d2_diff2_fine_cc) is
checked the same way against cuda_kernel_diff2_CC_fine (src/diff2.cuh:811-960)
and the FP64 CC coarse kernel.  Tolerance: 1e-5 relative (both FP32 sums,
different summation orders); CC scores change sign, so their error is taken
relative to the largest score magnitude of the job list."""
from __future__ import annotations

import numpy as np
import pytest

from gpu_util import DeviceProblem

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _err(oracle, got, ref, cc):
    if cc:
        got, ref = np.asarray(got, np.float64), np.asarray(ref, np.float64)
        return float(np.abs(got - ref).max() / np.abs(ref).max())
    return oracle.error_stats(got, ref)["max_rel"]


def _jobs(rng, O, T, n_jobs, max_chunk):
    """Random significant samples grouped the way RELION's fine scheduler
    does: one orientation and a run of consecutive translations per job."""
    rot, trans, jidx, jnum = [], [], [], []
    pos = 0
    for _ in range(n_jobs):
        o = int(rng.integers(O))
        n = int(rng.integers(1, max_chunk + 1))
        t0 = int(rng.integers(0, T - n + 1))
        for i in range(n):  # per-sample tables, indexed by the job's first sample
            rot.append(o)
            trans.append(t0 + i)
        jidx.append(pos)
        jnum.append(n)
        pos += n
    return (np.array(rot, np.uint64), np.array(trans, np.uint64), np.array(jidx, np.uint64),
            np.array(jnum, np.uint64))


def _check_fine(pkg, oracle, torch, pr, view, imgX, imgY, imgMaxR, N, eulers, tx, ty, re, im, corr, max_chunk,
                seed=7, cc=False):
    """Score 37 random jobs through b200d2_diff2_fine (b200d2_diff2_fine_cc
    with cc) and compare with the FP64 coarse kernel of the same score and,
    for jobs of at most 16 translations, with the reference's fine kernel.
    Returns the largest relative difference seen."""
    O, T = eulers.numel() // 9, tx.numel()
    rng = np.random.default_rng(seed)
    rot, trans, jidx, jnum = _jobs(rng, O, T, 37, min(max_chunk, T))
    dev = lambda a: torch.as_tensor(a.astype(np.int64), device="cuda")  # noqa: E731
    d_rot, d_trans, d_jidx, d_jnum = dev(rot), dev(trans), dev(jidx), dev(jnum)
    n_out = int(jnum.sum())
    sum_init = 0.0 if cc else 3.25
    out = torch.full((n_out,), -1.0, device="cuda")
    jobs = dict(rot_idx=d_rot, trans_idx=d_trans, job_idx=d_jidx, job_num=d_jnum, image_size=N)
    if cc:
        pkg.diff2_fine_cc(view, eulers, re, im, tx, ty, corr, out, **jobs)
    else:
        pkg.diff2_fine(view, eulers, re, im, tx, ty, corr, out, sum_init=sum_init, **jobs)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    # FP64 coarse scores of every (o, t), then picked per sample
    f64 = torch.zeros(O * T, device="cuda", dtype=torch.float64)
    if cc:
        pkg.run_diff2_kernel_coarse_cc_double(view, tx, ty, corr, re, im, eulers, f64, O, T, N)
    else:
        pkg.run_diff2_kernel_coarse_double(view, tx, ty, corr, re, im, eulers, f64, O, T, N)
    torch.cuda.synchronize()
    ref64 = f64.cpu().numpy().reshape(O, T)[rot.astype(np.int64), trans.astype(np.int64)] + sum_init
    worst = _err(oracle, got, ref64, cc)
    assert worst <= TOL
    if max_chunk <= 16:  # the reference kernel holds at most 16 translations per job
        L = oracle.ref_lib()
        h = L.refshim_projector_create(pr.projector.mdlX, pr.projector.mdlY, pr.projector.mdlZ,
                                       pr.projector.mdlInitY, pr.projector.mdlInitZ, pr.projector.mdlMaxR,
                                       pr.projector.padding_factor,
                                       np.ascontiguousarray(pr.projector.re, np.float32).ctypes.data,
                                       np.ascontiguousarray(pr.projector.im, np.float32).ctypes.data)
        assert h
        rout = torch.full((n_out,), -1.0, device="cuda")
        ptrs = (eulers.data_ptr(), re.data_ptr(), im.data_ptr(), tx.data_ptr(), ty.data_ptr(), corr.data_ptr(),
                rout.data_ptr(), N)
        idx = (len(jidx), d_rot.data_ptr(), d_trans.data_ptr(), d_jidx.data_ptr(), d_jnum.data_ptr(), None)
        if cc:
            st = L.refshim_diff2_fine_cc(h, imgX, imgY, 1, imgMaxR, *ptrs, O, T, *idx)
        else:
            st = L.refshim_diff2_fine(h, imgX, imgY, 1, imgMaxR, *ptrs, sum_init, O, T, *idx)
        torch.cuda.synchronize()
        L.refshim_projector_destroy(h)
        assert st == 0
        d = _err(oracle, got, rout.cpu().numpy(), cc)
        assert d <= TOL
        worst = max(worst, d)
    return worst


@pytest.mark.parametrize("cc", [False, True], ids=["diff2", "cc"])
@pytest.mark.parametrize("case,max_chunk", [("c1", 16), ("tiny", 16), ("c1", 40)])
def test_fine_matches_reference_and_fp64(pkg, synth, oracle, cuda, case, max_chunk, cc):
    """Coarse-sized images: the phase shifts come from the per-pass tables."""
    torch = cuda
    pr = synth.make_problem(case, P=2)
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(torch, pr)
    for p in range(pr.P):
        _check_fine(pkg, oracle, torch, pr, view, pr.imgX, pr.imgY, pr.imgMaxR, pr.N_img, dp.eulers, dp.tx, dp.ty,
                    dp.re[p], dp.im[p], dp.corr[p], max_chunk, cc=cc)
    proj.close()


@pytest.mark.parametrize("cc", [False, True], ids=["diff2", "cc"])
@pytest.mark.parametrize("imgX,imgY,imgMaxR", [(65, 128, 64), (129, 256, 128), (257, 512, 256)])
def test_fine_images_beyond_projector_radius(pkg, synth, oracle, cuda, imgX, imgY, imgMaxR, cc):
    """Images larger than the c1 projector's radius (16): the view's maxR is
    the projector's, so rows between maxR and imgY - maxR take the fine
    kernel's x = maxR mapping.  At 128 pixels the column form runs (tables
    and the shared q fit); at 256 only the tables fit and the per-pixel table
    form runs; at 512 (257 x 512 half-transform) the tables would exceed the
    shared-memory area and the kernel takes sincos per pixel.  Random image data; pixels beyond the
    projector's radius score against a zero projection."""
    torch = cuda
    pr = synth.make_problem("c1", P=1, orient_limit=64)
    N = imgX * imgY
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(imgX, imgY, imgMaxR)
    rng = np.random.default_rng(11)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")  # noqa: E731
    re, im = t(rng.normal(0, 1e-3, N)), t(rng.normal(0, 1e-3, N))
    corr = t(rng.uniform(0.5, 2.0, N))
    _check_fine(pkg, oracle, torch, pr, view, imgX, imgY, imgMaxR, N, t(pr.eulers.reshape(-1)), t(pr.trans_x),
                t(pr.trans_y), re, im, corr, 16, seed=3, cc=cc)
    proj.close()


def test_fine_rejects_bad_arguments(pkg, cuda):
    import ctypes as C
    v = pkg.View()
    assert pkg.lib().b200d2_diff2_fine(C.byref(v), None, None, None, None, None, None, None, 10, 0.0, 3,
                                       None, None, None, None, None) == 1
    assert pkg.lib().b200d2_diff2_fine(C.byref(v), None, None, None, None, None, None, None, 10, 0.0, 0,
                                       None, None, None, None, None) == 0
    assert pkg.lib().b200d2_diff2_fine_cc(C.byref(v), None, None, None, None, None, None, None, 10, 3,
                                          None, None, None, None, None) == 1
    assert pkg.lib().b200d2_diff2_fine_cc(C.byref(v), None, None, None, None, None, None, None, 10, 0,
                                          None, None, None, None, None) == 0
