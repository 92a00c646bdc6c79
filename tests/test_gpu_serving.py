"""Serving loop (b200d2_server_*): requests over two resident references,
admitted as stream slots and HBM budget free up, overlapping on the GPU.
Each request's result must be the same alone and in the mix (the kernels are
deterministic, so within 1e-6 relative), and agree with the FP64 CUDA-core
kernel within the TF32 tolerance (1e-3)."""
from __future__ import annotations

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
