"""Significant samples per particle (b200d2_significance) against the oracle's
restatement of RELION's pass-0 steps with exact cumulative sums
(oracle.significance), and against the reference's own
cuda_kernel_find_threshold_idx_in_cumulative / cuda_kernel_array_over_threshold
(src/cuda_device_utils.cuh:238-266, compiled into oracle/_ref) fed a sort and
an FP64 scan of the same weights.

Bar: the threshold weight, the count and the mask are identical (integer and
index results).  The oracle's sums are exact, so the comparison with it is
unconditional except where a cumulative sum lies within 1e-20 (relative) of
thr (the device truncates the far tail below 2^-64 thr to a fixed point of
2^-100 thr and carries its sums in double-double: about 2^-72 of thr); the
comparison with the FP64 scan skips particles whose crossing lies within the
scan's own rounding (n * 2^-52, relative) of thr."""
from __future__ import annotations

import zlib

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(rng, P, n, kind):
    w = np.zeros((P, n))
    for p in range(P):
        if kind == "exp":  # exp(-(diff2 - min)) shapes: a few strong samples, a long tail
            w[p] = np.exp(-rng.exponential(rng.uniform(2, 300), n))
            w[p, rng.random(n) < 0.3] = 0.0
        elif kind == "ties":
            w[p] = rng.choice([0.0, 0.125, 0.3, 0.7, 1.0], n)
        elif kind == "wide":  # binades from 2^-1070 (subnormal) to 1
            w[p] = np.ldexp(rng.uniform(1, 2, n), -rng.integers(0, 1070, n))
        elif kind == "flat":
            w[p] = rng.uniform(0.9, 1.1, n)
    return w


def _check(torch, pkg, oracle, w, frac, maxsig, sums=None):
    P, n = w.shape
    if sums is None:
        sums = np.array([float(np.sum(r[(r > 0) & np.isfinite(r)])) for r in w])
    dw = torch.as_tensor(w, device="cuda")
    ds = torch.as_tensor(sums, device="cuda")
    sig, nsig, passed = pkg.significance(dw, ds, frac, maxsig)
    torch.cuda.synchronize()
    sig, nsig, passed = sig.cpu().numpy(), nsig.cpu().numpy(), passed.cpu().numpy()
    checked = 0
    for p in range(P):
        osig, onsig, opassed, margin = oracle.significance(w[p], sums[p], frac, maxsig)
        if margin < 1e-20:
            continue
        checked += 1
        assert sig[p] == osig, (p, sig[p], osig)
        assert nsig[p] == onsig, (p, nsig[p], onsig)
        assert np.array_equal(passed[p], opassed), p
    assert checked >= max(1, P - 1)
    return sig, nsig, passed


@pytest.mark.parametrize("kind", ["exp", "ties", "wide", "flat"])
@pytest.mark.parametrize("frac,maxsig", [(0.999, 0), (0.99, 50), (0.5, 0), (0.0, 0), (1.0, 7)])
def test_significance_matches_oracle(pkg, oracle, cuda, kind, frac, maxsig):
    rng = np.random.default_rng(zlib.crc32(repr((kind, frac, maxsig)).encode()))
    w = _rows(rng, 5, 30011, kind)
    _check(cuda, pkg, oracle, w, frac, maxsig)


def test_significance_edge_rows(pkg, oracle, cuda):
    """A row of zeros (nothing significant, threshold +inf), a single positive
    weight, negative / NaN / infinite entries, and a total that the caller
    gives larger than the weights' sum (no crossing: every positive weight)."""
    torch = cuda
    n = 1000
    w = np.zeros((5, n))
    w[1, 17] = 0.25
    rng = np.random.default_rng(5)
    w[2] = rng.random(n)
    w[2, :10] = [-1.0, np.nan, np.inf, -np.inf, -0.0, 0.0, 1e-310, 5e-324, 2.0, 3.0]
    w[3] = rng.random(n)
    w[4] = rng.random(n)
    # row 3: the given total is 2000x the weights' sum, so thr = 2 x their sum
    # is never reached: idx = 0 and every positive weight is significant.
    # row 4: a total 1e-25 of the weights' sum puts thr 2^-90 below them,
    # beyond the 128 binades histogrammed from 2^-64 thr: the crossing is the
    # smallest weight
    sums = np.array([0.0, 0.25, float(np.sum(w[2][np.isfinite(w[2]) & (w[2] > 0)])), 2000 * w[3].sum(),
                     1e-25 * w[4].sum()])
    sig, nsig, passed = _check(torch, pkg, oracle, w, 0.999, 0, sums)
    assert sig[0] == np.inf and nsig[0] == 0 and passed[0].sum() == 0
    assert sig[1] == 0.25 and nsig[1] == 1
    assert nsig[3] == np.count_nonzero(w[3] > 0) and sig[3] == w[3][w[3] > 0].min()
    assert nsig[4] == n and sig[4] == w[4].min()
    # one weight per particle
    one = np.array([[0.5], [0.0]])
    s1, n1, _ = _check(torch, pkg, oracle, one, 0.999, 0, np.array([0.5, 0.0]))
    assert (s1[0], n1[0], n1[1]) == (0.5, 1, 0)


def test_significance_repeatable_and_cap_mix(pkg, oracle, cuda):
    """Two calls on one workspace give identical results; in one batch some
    particles hit the cap (rank phase) and others do not."""
    torch = cuda
    rng = np.random.default_rng(9)
    w = np.zeros((6, 20000))
    w[::2] = _rows(rng, 3, 20000, "flat")  # flat rows: thousands significant, capped at 100
    for p in (1, 3, 5):  # a few strong weights over a faint floor: fewer than 100 significant
        w[p] = 1e-12 * rng.random(20000)
        w[p, rng.choice(20000, 30, replace=False)] = rng.uniform(0.5, 1.0, 30)
    dw = torch.as_tensor(w, device="cuda")
    ds = torch.as_tensor(w.sum(axis=1), device="cuda")
    ws = torch.empty(pkg.lib().b200d2_significance_workspace(6, 20000), dtype=torch.uint8, device="cuda")
    a = [t.cpu().numpy() for t in pkg.significance(dw, ds, 0.999, 100, workspace=ws)]
    b = [t.cpu().numpy() for t in pkg.significance(dw, ds, 0.999, 100, workspace=ws)]
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
    assert (a[1][::2] == 100).all() and (a[1][1::2] < 100).any()
    _check(torch, pkg, oracle, w, 0.999, 100)


def test_significance_at_c2_row_size(pkg, oracle, cuda):
    """Rows of 4608 x 113 = 520704 samples, the C2 coarse block per particle."""
    rng = np.random.default_rng(13)
    w = _rows(rng, 3, 4608 * 113, "exp")
    _check(cuda, pkg, oracle, w, 0.999, 0)


def test_significance_of_coarse_weights(pkg, synth, oracle, cuda):
    """The E-step chain on device: tensor-core coarse batch -> FP64 weights ->
    significance, against the oracle on the same weights."""
    from gpu_util import DeviceProblem
    torch = cuda
    pr = synth.make_problem("c1")
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    dp = DeviceProblem(torch, pr)
    d2 = torch.zeros(pr.P * pr.O * pr.T, device="cuda")
    b = pkg.make_batch(dp.eulers, dp.tx, dp.ty, dp.re, dp.im, dp.corr, d2, O=pr.O, T=pr.T, P=pr.P, N_img=pr.N_img)
    ws = torch.empty(pkg.batch_workspace_bytes(view, b, pkg.PREC_BF16X3), device="cuda", dtype=torch.uint8)
    pkg.diff2_coarse_batch(view, b, pkg.PREC_BF16X3, ws)
    w, sums = pkg.coarse_weights(d2, pr.P, pr.O, pr.T, normalize=True)
    wn = w.reshape(pr.P, -1).cpu().numpy()
    sig, nsig, passed = pkg.significance(w.reshape(pr.P, -1), torch.ones_like(sums), 0.999, 0)
    torch.cuda.synchronize()
    for p in range(pr.P):
        osig, onsig, opassed, margin = oracle.significance(wn[p], 1.0, 0.999, 0)
        assert margin > 1e-20
        assert (sig[p].item(), nsig[p].item()) == (osig, onsig)
        assert np.array_equal(passed[p].cpu().numpy(), opassed)
    assert (nsig.cpu().numpy() >= 1).all()
    proj.close()


def test_significance_matches_reference_kernels(pkg, oracle, cuda):
    """RELION's device sequence with the reference's own kernels: positive
    weights sorted (torch), inclusive FP64 scan (torch), the reference's
    find-threshold kernel, the cap, then its over-threshold mask."""
    torch = cuda
    L = oracle.ref_lib()
    rng = np.random.default_rng(21)
    for kind, frac, maxsig in [("exp", 0.999, 0), ("exp", 0.99, 40), ("ties", 0.7, 0), ("wide", 0.999, 0)]:
        w = _rows(rng, 4, 25000, kind)
        sums = np.array([float(np.sum(r[r > 0])) for r in w])
        dw = torch.as_tensor(w, device="cuda")
        sig, nsig, passed = pkg.significance(dw, torch.as_tensor(sums, device="cuda"), frac, maxsig)
        torch.cuda.synchronize()
        for p in range(4):
            pos = torch.sort(dw[p][dw[p] > 0]).values.contiguous()
            cum = torch.cumsum(pos, 0).contiguous()
            thr = (1.0 - frac) * sums[p]
            d_idx = torch.zeros(1, dtype=torch.int64, device="cuda")
            assert L.refshim_find_threshold_idx(cum.data_ptr(), thr, pos.numel(), d_idx.data_ptr(), None) == 0
            torch.cuda.synchronize()
            idx = int(d_idx.item())
            cnt = pos.numel()
            ref_nsig = cnt - idx
            if maxsig > 0 and ref_nsig > maxsig:
                ref_nsig, idx = maxsig, cnt - maxsig
            ref_sig = float(pos[idx].item())
            ref_mask = torch.zeros(w.shape[1], dtype=torch.bool, device="cuda")
            assert L.refshim_array_over_threshold(dw[p].data_ptr(), ref_mask.data_ptr(), ref_sig, w.shape[1],
                                                  None) == 0
            torch.cuda.synchronize()
            margin = oracle.significance(w[p], sums[p], frac, maxsig)[3]
            if margin < cnt * 2.0 ** -52:
                continue  # the FP64 scan's rounding reaches the threshold
            assert sig[p].item() == ref_sig and nsig[p].item() == ref_nsig
            assert torch.equal(passed[p].bool(), ref_mask)


def _packbits_ref(m):
    """numpy reference of b200d2_pack_mask: rows of bits, little-endian words."""
    P, n = m.shape
    w = (n + 31) // 32
    out = np.zeros((P, w * 4), np.uint8)
    for p in range(P):
        b = np.packbits(m[p] != 0, bitorder="little")
        out[p, :b.size] = b
    return out.view("<u4")


@pytest.mark.parametrize("P,n,offset", [(3, 100, 0), (2, 64, 0), (4, 1000, 1), (1, 1, 0), (5, 4096, 0),
                                        (2, 4096, 3), (3, 31, 0)])
def test_pack_mask(pkg, cuda, P, n, offset):
    """Byte masks packed to bits: aligned rows (16-byte loads), unaligned
    bases and ragged rows (byte loads), arbitrary non-zero bytes."""
    torch = cuda
    rng = np.random.default_rng(P * 1000 + n + offset)
    m = (rng.integers(0, 2, (P, n)) * rng.integers(1, 256, (P, n))).astype(np.uint8)
    flat = torch.zeros(P * n + offset, dtype=torch.uint8, device="cuda")
    flat[offset:] = torch.as_tensor(m.reshape(-1), device="cuda")
    got = pkg.pack_mask(flat[offset:].view(P, n))
    torch.cuda.synchronize()
    np.testing.assert_array_equal(got.cpu().numpy().view(np.uint32), _packbits_ref(m))


def test_pack_mask_of_significance(pkg, oracle, cuda):
    """The packed form of a significance mask unpacks to the byte mask (with
    no tied weights, as here, it holds exactly nsig set bits per particle;
    weights equal to the threshold weight all pass)."""
    torch = cuda
    rng = np.random.default_rng(5)
    P, n = 4, 20000
    w = torch.as_tensor(rng.exponential(1.0, (P, n)) ** 4, device="cuda")
    sums = w.sum(dim=1)
    _, nsig, mask = pkg.significance(w, sums, 0.999)
    bits = pkg.pack_mask(mask)
    torch.cuda.synchronize()
    b = bits.cpu().numpy().view(np.uint32)
    unpacked = np.unpackbits(b.view(np.uint8), axis=1, bitorder="little")[:, :n]
    np.testing.assert_array_equal(unpacked, mask.cpu().numpy())
    assert [int(np.unpackbits(b[p].view(np.uint8)).sum()) for p in range(P)] == nsig.cpu().tolist()
