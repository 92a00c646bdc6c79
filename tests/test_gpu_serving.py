"""Serving loop (b200d2_server_*): requests over two resident references,
admitted as stream slots and HBM budget free up, overlapping on the GPU.
Each request's result must be the same alone and in the mix (the kernels are
deterministic, so within 1e-6 relative), and agree with the FP64 CUDA-core
kernel within the TF32 tolerance (1e-3)."""
from __future__ import annotations

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(synth, rng, prob, ref, n):
    reqs = []
    for _ in range(n):
        P = int(rng.integers(1, prob.P + 1))
        ps = np.sort(rng.choice(prob.P, P, replace=False))
        O = int(rng.integers(prob.O // 4, prob.O + 1))
        orient = np.sort(rng.choice(prob.O, O, replace=False)).astype(np.int32)
        sh = synth.translation_grid(int(rng.choice([1, 2, 4, 5])))
        tx = (-2 * np.pi * sh[:, 0] / prob.projector.ori_size).astype(np.float32)
        ty = (-2 * np.pi * sh[:, 1] / prob.projector.ori_size).astype(np.float32)
        reqs.append(dict(ref=ref, prob=prob, ps=ps, real=np.ascontiguousarray(prob.fimg_re[ps]),
                         imag=np.ascontiguousarray(prob.fimg_im[ps]), corr=np.ascontiguousarray(prob.corr[ps]),
                         orient=orient, tx=tx, ty=ty))
    return reqs


def _submit(srv, rq):
    out = np.zeros((len(rq["ps"]), rq["orient"].size, rq["tx"].size), np.float32)
    mn = np.zeros(len(rq["ps"]), np.float64)
    am = np.zeros(len(rq["ps"]), np.int64)
    t = srv.submit(rq["ref"], rq["real"], rq["imag"], rq["corr"], rq["orient"], rq["tx"], rq["ty"], out, mn, am)
    return t, out, mn, am


def test_serving_alone_and_in_the_mix(pkg, synth, oracle, cuda):
    torch = cuda
    rng = np.random.default_rng(17)
    probs = [synth.make_problem("tiny", P=6), synth.make_problem("c1", P=6)]
    projs = [pkg.Projector(p.projector, use_texture=1) for p in probs]
    views = [pj.view(p.imgX, p.imgY, p.imgMaxR) for pj, p in zip(projs, probs)]
    srv = pkg.Server(slots=4, hbm_budget=4 << 30, precision=pkg.PREC_TF32)
    refs = [srv.add_reference(v, p.eulers, p.N_img) for v, p in zip(views, probs)]
    reqs = _requests(synth, rng, probs[0], refs[0], 6) + _requests(synth, rng, probs[1], refs[1], 6)
    rng.shuffle(reqs)

    # in the mix: everything submitted at once
    mix = [_submit(srv, rq) for rq in reqs]
    for t, *_ in mix:
        st, lat, dev = srv.wait(t)
        assert st == 0 and lat > 0 and dev > 0
    stats = srv.stats()
    assert stats["completed"] == len(reqs) and stats["in_flight"] == 0
    assert stats["max_in_flight"] >= 2  # requests overlapped on the device

    # alone: one at a time
    for rq, (t0, out_mix, mn_mix, am_mix) in zip(reqs, mix):
        t, out, mn, am = _submit(srv, rq)
        assert srv.wait(t)[0] == 0
        assert oracle.error_stats(out_mix, out)["max_rel"] <= 1e-6
        np.testing.assert_array_equal(am_mix, am)

    # against the FP64 kernel on the same subset
    for rq, (_, out_mix, _, _) in zip(reqs[:4], mix[:4]):
        prob = rq["prob"]
        v = views[rq["ref"]]
        eul = torch.as_tensor(np.ascontiguousarray(prob.eulers[rq["orient"]].reshape(-1)), device="cuda")
        tx, ty = torch.as_tensor(rq["tx"], device="cuda"), torch.as_tensor(rq["ty"], device="cuda")
        for i in range(len(rq["ps"])):
            d = torch.zeros(rq["orient"].size * rq["tx"].size, device="cuda", dtype=torch.float64)
            pkg.run_diff2_kernel_coarse_double(v, tx, ty, torch.as_tensor(rq["corr"][i], device="cuda"),
                                               torch.as_tensor(rq["real"][i], device="cuda"),
                                               torch.as_tensor(rq["imag"][i], device="cuda"), eul, d,
                                               rq["orient"].size, rq["tx"].size, prob.N_img)
            torch.cuda.synchronize()
            assert oracle.error_stats(out_mix[i].ravel(), d.cpu().numpy())["max_rel"] <= 1e-3
    srv.close()
    for pj in projs:
        pj.close()


def test_serving_admission_by_budget(pkg, synth, cuda):
    prob = synth.make_problem("c1", P=4)
    proj = pkg.Projector(prob.projector, use_texture=1)
    view = proj.view(prob.imgX, prob.imgY, prob.imgMaxR)
    budget = 4 << 20  # 4 MiB: one small request (~2.5 MiB with its workspace) at a time
    srv = pkg.Server(slots=2, hbm_budget=budget, precision=pkg.PREC_TF32)
    srv.set_merging(1)  # one request per admission: the budget alone bounds what runs together
    ref = srv.add_reference(view, prob.eulers, prob.N_img)
    tx = np.zeros(1, np.float32)
    big = np.arange(prob.O, dtype=np.int32)
    with pytest.raises(pkg.B200D2Error) as e:  # 4 particles x 576 orientations x 21 t: ~8 MiB
        srv.submit(ref, prob.fimg_re, prob.fimg_im, prob.corr, big,
                   np.zeros(21, np.float32), np.zeros(21, np.float32))
    assert e.value.code == 7
    small = np.arange(64, dtype=np.int32)
    outs = []
    for _ in range(6):  # each fits; together they exceed the budget and queue
        o = np.zeros((1, 64, 1), np.float32)
        outs.append((srv.submit(ref, prob.fimg_re[:1].copy(), prob.fimg_im[:1].copy(), prob.corr[:1].copy(),
                                small, tx, tx, o), o))
    for t, o in outs:
        assert srv.wait(t)[0] == 0
        assert np.isfinite(o).all() and (o > 0).all()
    st = srv.stats()
    assert st["rejected"] == 1 and st["completed"] == 6 and st["peak_bytes"] <= budget
    assert st["max_in_flight"] == 1  # the budget, not the two slots, limited concurrency
    srv.close()
    proj.close()


def test_serving_page_locked_and_pageable_buffers(pkg, synth, cuda):
    """Host buffers that are not page-locked go through the server's staging
    buffers (so the scheduler thread never waits for the GPU); page-locked
    ones are copied directly.  Every combination gives the same results, and
    the staging buffers are reused across requests of different sizes."""
    torch = cuda
    rng = np.random.default_rng(23)
    prob = synth.make_problem("c1", P=6)
    proj = pkg.Projector(prob.projector, use_texture=1)
    view = proj.view(prob.imgX, prob.imgY, prob.imgMaxR)
    srv = pkg.Server(slots=2, hbm_budget=2 << 30, precision=pkg.PREC_BF16X3)
    ref = srv.add_reference(view, prob.eulers, prob.N_img)
    reqs = _requests(synth, rng, prob, ref, 4)

    def run(rq, pinned_in, pinned_out):
        n, O, T = len(rq["ps"]), rq["orient"].size, rq["tx"].size
        host = (lambda a: torch.as_tensor(a).pin_memory()) if pinned_in else (lambda a: a)  # noqa: E731
        mk = (lambda *s, dt: torch.zeros(s, dtype=dt).pin_memory()) if pinned_out else \
            (lambda *s, dt: torch.zeros(s, dtype=dt))  # noqa: E731
        out, mn, am = mk(n, O, T, dt=torch.float32), mk(n, dt=torch.float64), mk(n, dt=torch.int64)
        if not pinned_out:
            assert not out.is_pinned()
        t = srv.submit(ref, host(rq["real"]), host(rq["imag"]), host(rq["corr"]), rq["orient"], rq["tx"], rq["ty"],
                       out, mn, am)
        assert srv.wait(t)[0] == 0
        return out.numpy().copy(), mn.numpy().copy(), am.numpy().copy()

    for rq in reqs:
        base = run(rq, False, False)
        for pin_in, pin_out in ((True, True), (True, False), (False, True)):
            got = run(rq, pin_in, pin_out)
            for a, b in zip(got, base):
                np.testing.assert_array_equal(a, b)
        assert np.all(base[1] == base[0].reshape(len(rq["ps"]), -1).min(axis=1))
    srv.close()
    proj.close()


def test_serving_cancel_queued_request(pkg, synth, cuda):
    """A queued request can be cancelled: it never runs and its wait returns
    ERR_CANCELLED; an admitted one cannot (ERR_UNSUPPORTED) and completes; an
    unknown ticket is ERR_INVALID.  One slot held by a C2 batch of 256
    particles on the FP32 CUDA cores (about 57 ms) keeps the queue waiting
    while the test cancels."""
    prob = synth.make_problem("c2")
    proj = pkg.Projector(prob.projector, use_texture=1)
    view = proj.view(prob.imgX, prob.imgY, prob.imgMaxR)
    srv = pkg.Server(slots=1, hbm_budget=8 << 30, precision=pkg.PREC_FP32)
    ref = srv.add_reference(view, prob.eulers, prob.N_img)
    allo = np.arange(prob.O, dtype=np.int32)
    mn_a, am_a = np.zeros(prob.P), np.zeros(prob.P, np.int64)
    long_t = srv.submit(ref, prob.fimg_re, prob.fimg_im, prob.corr, allo, prob.trans_x, prob.trans_y, None, mn_a, am_a)
    t0 = time.monotonic()
    while srv.stats()["in_flight"] < 1:  # admitted: the slot is busy from here on
        assert time.monotonic() - t0 < 30.0
        time.sleep(0.0005)
    small = [srv.submit(ref, prob.fimg_re[:1].copy(), prob.fimg_im[:1].copy(), prob.corr[:1].copy(), allo[:64],
                        prob.trans_x, prob.trans_y, None, np.zeros(1), np.zeros(1, np.int64)) for _ in range(3)]
    assert srv.cancel(long_t) == pkg.ERR_UNSUPPORTED  # running: not interrupted
    assert srv.cancel(small[1]) == pkg.OK
    assert srv.cancel(small[1]) == pkg.OK  # again: still cancelled
    st_long = srv.wait(long_t)[0]
    assert st_long == pkg.OK and np.isfinite(mn_a).all()
    assert srv.cancel(long_t) == pkg.ERR_INVALID  # waited for: the ticket is gone
    assert srv.wait(small[0])[0] == pkg.OK
    assert srv.wait(small[1])[0] == pkg.ERR_CANCELLED
    assert srv.wait(small[2])[0] == pkg.OK
    st = srv.stats()
    assert st["cancelled"] == 1 and st["completed"] == 3
    srv.close()
    proj.close()


def test_serving_allocation_failure_is_reported(pkg, synth, cuda):
    """A request whose device footprint cannot be allocated (its output alone
    is about 400 GB, more than the GPU holds, within a 1 TB budget) fails with
    ERR_OOM before anything is launched, and the server goes on serving: the
    next request's minima and argmins equal those of a server that never saw
    the failure (the kernels are deterministic)."""
    prob = synth.make_problem("c1", P=8)
    proj = pkg.Projector(prob.projector, use_texture=1)
    view = proj.view(prob.imgX, prob.imgY, prob.imgMaxR)
    srv = pkg.Server(slots=2, hbm_budget=1 << 40, precision=pkg.PREC_FP32)
    ref = srv.add_reference(view, prob.eulers, prob.N_img)
    allo = np.arange(prob.O, dtype=np.int32)
    T = 22_000_000  # 8 x 576 x 2.2e7 x 4 B = 405 GB of diff2
    tx = np.zeros(T, np.float32)
    t_big = srv.submit(ref, prob.fimg_re, prob.fimg_im, prob.corr, allo, tx, tx, None, np.zeros(prob.P),
                       np.zeros(prob.P, np.int64))
    assert srv.wait(t_big, timeout=120.0)[0] == pkg.ERR_OOM
    mn, am = np.zeros(prob.P), np.zeros(prob.P, np.int64)
    t_ok = srv.submit(ref, prob.fimg_re, prob.fimg_im, prob.corr, allo, prob.trans_x, prob.trans_y, None, mn, am)
    assert srv.wait(t_ok)[0] == pkg.OK
    assert np.isfinite(mn).all() and (am >= 0).all()
    assert srv.stats()["completed"] == 2
    srv.close()
    fresh = pkg.Server(slots=2, hbm_budget=1 << 40, precision=pkg.PREC_FP32)
    ref2 = fresh.add_reference(view, prob.eulers, prob.N_img)
    mn2, am2 = np.zeros(prob.P), np.zeros(prob.P, np.int64)
    t2 = fresh.submit(ref2, prob.fimg_re, prob.fimg_im, prob.corr, allo, prob.trans_x, prob.trans_y, None, mn2, am2)
    assert fresh.wait(t2)[0] == pkg.OK
    np.testing.assert_array_equal(am, am2)
    np.testing.assert_array_equal(mn, mn2)
    fresh.close()
    proj.close()


@pytest.mark.parametrize("precision,tol", [("PREC_TF32", 1e-3), ("PREC_BF16X3", 1e-5)])
def test_serving_merged_requests(pkg, synth, oracle, cuda, precision, tol):
    """Queued requests on one reference run as one merged, block-diagonal
    batch (b200d2_server_set_merging): each request's particles against its
    own orientation subset at its own translations.  One slot, held by a
    long request on another reference, makes the small requests queue; they
    are then admitted together.  Each merged result equals the same request
    run alone with merging off (same kernels, same sums: within 1e-6 and the
    same argmin), and agrees with the FP64 CUDA-core kernel within the
    precision's tolerance."""
    torch = cuda
    prec = getattr(pkg, precision)
    rng = np.random.default_rng(29)
    blk = synth.make_problem("c2", P=64)
    prob = synth.make_problem("c1", P=8)
    projs = [pkg.Projector(p.projector, use_texture=1) for p in (blk, prob)]
    vb, view = (pj.view(p.imgX, p.imgY, p.imgMaxR) for pj, p in zip(projs, (blk, prob)))
    srv = pkg.Server(slots=1, hbm_budget=8 << 30, precision=prec)
    rb = srv.add_reference(vb, blk.eulers, blk.N_img)
    ref = srv.add_reference(view, prob.eulers, prob.N_img)
    reqs = _requests(synth, rng, prob, ref, 7)
    reqs[0]["orient"] = np.arange(3, 300, dtype=np.int32)  # 297 columns: a gap to the next request's
    # the blocker: 64 C2 particles with their 133 MB diff2 copied back through
    # the staging buffer (tens of ms), so that the small requests queue
    blk_out = np.zeros((blk.P, blk.O, blk.T), np.float32)
    t_blk = srv.submit(rb, blk.fimg_re, blk.fimg_im, blk.corr, np.arange(blk.O, dtype=np.int32), blk.trans_x,
                       blk.trans_y, blk_out, np.zeros(blk.P), np.zeros(blk.P, np.int64))
    mix = [_submit(srv, rq) for rq in reqs]
    assert srv.wait(t_blk)[0] == 0
    for t, *_ in mix:
        assert srv.wait(t)[0] == 0
    st = srv.stats()
    assert st["completed"] == len(reqs) + 1
    assert st["merged_admissions"] >= 1 and st["merged_requests"] >= 2

    srv.set_merging(1)  # off: every request alone
    for rq, (_, out_mix, mn_mix, am_mix) in zip(reqs, mix):
        t, out, mn, am = _submit(srv, rq)
        assert srv.wait(t)[0] == 0
        assert oracle.error_stats(out_mix, out)["max_rel"] <= 1e-6
        np.testing.assert_array_equal(am_mix, am)
        assert np.all(mn_mix == out_mix.reshape(len(rq["ps"]), -1).min(axis=1))
    assert srv.stats()["merged_admissions"] == st["merged_admissions"]

    eul_all = prob.eulers.reshape(-1, 9)
    for rq, (_, out_mix, _, _) in zip(reqs, mix):
        eul = torch.as_tensor(np.ascontiguousarray(eul_all[rq["orient"]].reshape(-1)), device="cuda")
        tx, ty = torch.as_tensor(rq["tx"], device="cuda"), torch.as_tensor(rq["ty"], device="cuda")
        for i in range(len(rq["ps"])):
            d = torch.zeros(rq["orient"].size * rq["tx"].size, device="cuda", dtype=torch.float64)
            pkg.run_diff2_kernel_coarse_double(view, tx, ty, torch.as_tensor(rq["corr"][i], device="cuda"),
                                               torch.as_tensor(rq["real"][i], device="cuda"),
                                               torch.as_tensor(rq["imag"][i], device="cuda"), eul, d,
                                               rq["orient"].size, rq["tx"].size, prob.N_img)
            torch.cuda.synchronize()
            assert oracle.error_stats(out_mix[i].ravel(), d.cpu().numpy())["max_rel"] <= tol
    srv.close()
    for pj in projs:
        pj.close()


def test_serving_c5_shapes(pkg, synth, oracle, cuda):
    """The serving workload's own shapes: three resident references at
    coarse image sizes 48, 64 and 96 (all 4608 orientations), requests of
    4-24 particles against random 10-100 % orientation subsets at
    translation radii 2-6 px, TF32 with FP64 norms.  Submitted together on
    two slots (so that requests queue, overlap and merge), each result equals
    the request run alone with merging off (1e-6, same argmin), and one
    particle of every request agrees with the FP64 CUDA-core kernel (1e-3)."""
    torch = cuda
    rng = np.random.default_rng(31)
    probs = [synth.make_problem(n, seed=20251203 + i, P=24) for i, n in enumerate(("c5s", "c5m", "c5l"))]
    projs = [pkg.Projector(p.projector, use_texture=1) for p in probs]
    views = [pj.view(p.imgX, p.imgY, p.imgMaxR) for pj, p in zip(projs, probs)]
    srv = pkg.Server(slots=2, hbm_budget=16 << 30, precision=pkg.PREC_TF32)
    refs = [srv.add_reference(v, p.eulers, p.N_img) for v, p in zip(views, probs)]
    reqs = []
    for k in range(9):
        r = k % 3
        prob = probs[r]
        P = int(rng.integers(4, 25))
        ps = np.sort(rng.choice(prob.P, P, replace=False))
        O = max(1, int(round(rng.uniform(0.1, 1.0) * prob.O)))
        orient = np.sort(rng.choice(prob.O, O, replace=False)).astype(np.int32)
        rad = int(rng.integers(2, 7))
        sh = synth.translation_grid(rad * rad)
        tx = (-2 * np.pi * sh[:, 0] / prob.projector.ori_size).astype(np.float32)
        ty = (-2 * np.pi * sh[:, 1] / prob.projector.ori_size).astype(np.float32)
        reqs.append(dict(ref=refs[r], r=r, prob=prob, ps=ps, real=np.ascontiguousarray(prob.fimg_re[ps]),
                         imag=np.ascontiguousarray(prob.fimg_im[ps]), corr=np.ascontiguousarray(prob.corr[ps]),
                         orient=orient, tx=tx, ty=ty))
    mix = [_submit(srv, rq) for rq in reqs]
    for t, *_ in mix:
        assert srv.wait(t, timeout=300.0)[0] == 0
    st = srv.stats()
    assert st["completed"] == len(reqs) and st["max_in_flight"] >= 2

    srv.set_merging(1)
    for rq, (_, out_mix, mn_mix, am_mix) in zip(reqs, mix):
        t, out, mn, am = _submit(srv, rq)
        assert srv.wait(t, timeout=300.0)[0] == 0
        assert oracle.error_stats(out_mix, out)["max_rel"] <= 1e-6
        np.testing.assert_array_equal(am_mix, am)

    for rq, (_, out_mix, _, _) in zip(reqs, mix):
        prob = rq["prob"]
        eul = torch.as_tensor(np.ascontiguousarray(prob.eulers.reshape(-1, 9)[rq["orient"]].reshape(-1)),
                              device="cuda")
        tx, ty = torch.as_tensor(rq["tx"], device="cuda"), torch.as_tensor(rq["ty"], device="cuda")
        i = len(rq["ps"]) // 2
        d = torch.zeros(rq["orient"].size * rq["tx"].size, device="cuda", dtype=torch.float64)
        pkg.run_diff2_kernel_coarse_double(views[rq["r"]], tx, ty, torch.as_tensor(rq["corr"][i], device="cuda"),
                                           torch.as_tensor(rq["real"][i], device="cuda"),
                                           torch.as_tensor(rq["imag"][i], device="cuda"), eul, d,
                                           rq["orient"].size, rq["tx"].size, prob.N_img)
        torch.cuda.synchronize()
        assert oracle.error_stats(out_mix[i].ravel(), d.cpu().numpy())["max_rel"] <= 1e-3
    srv.close()
    for pj in projs:
        pj.close()
