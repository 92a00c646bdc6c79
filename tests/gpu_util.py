"""Helpers shared by the GPU tests: device copies of a synthetic problem and
runners for this library's kernels and for the reference's own kernels
(oracle/_ref, compiled from the reference sources)."""
from __future__ import annotations

import ctypes as C

import numpy as np


def dev(torch, x, dtype=None):
    t = torch.as_tensor(np.ascontiguousarray(x), device="cuda")
    return t if dtype is None else t.to(dtype)


class DeviceProblem:
    def __init__(self, torch, pr):
        self.torch = torch
        self.pr = pr
        self.eulers = dev(torch, pr.eulers.reshape(-1))
        self.tx = dev(torch, pr.trans_x)
        self.ty = dev(torch, pr.trans_y)
        self.re = dev(torch, pr.fimg_re)
        self.im = dev(torch, pr.fimg_im)
        self.corr = dev(torch, pr.corr)


def ours_f32(pkg, view, dp, p, init=None):
    pr, torch = dp.pr, dp.torch
    out = torch.zeros(pr.O * pr.T, device="cuda", dtype=torch.float32)
    if init is not None:
        out.copy_(dev(torch, np.asarray(init, np.float32).reshape(-1)))
    pkg.run_diff2_kernel_coarse(view, dp.tx, dp.ty, dp.corr[p], dp.re[p], dp.im[p], dp.eulers, out,
                                pr.O, pr.T, pr.N_img)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(pr.O, pr.T)


def ours_f64(pkg, view, dp, p, filter_img=False):
    pr, torch = dp.pr, dp.torch
    out = torch.zeros(pr.O * pr.T, device="cuda", dtype=torch.float64)
    pkg.run_diff2_kernel_coarse_double(view, dp.tx, dp.ty, dp.corr[p], dp.re[p], dp.im[p], dp.eulers, out,
                                       pr.O, pr.T, pr.N_img, filter_img=filter_img)
    torch.cuda.synchronize()
    return out.cpu().numpy().reshape(pr.O, pr.T)


class RefKernels:
    """The reference project's runDiff2KernelCoarse / runDiff2KernelCoarseDouble."""

    def __init__(self, oracle, pr):
        self.L = oracle.ref_lib()
        pv = pr.projector
        re = np.ascontiguousarray(pv.re, np.float32)
        im = np.ascontiguousarray(pv.im, np.float32)
        self.h = self.L.refshim_projector_create(pv.mdlX, pv.mdlY, pv.mdlZ, pv.mdlInitY, pv.mdlInitZ,
                                                 pv.mdlMaxR, pv.padding_factor,
                                                 re.ctypes.data_as(C.c_void_p), im.ctypes.data_as(C.c_void_p))
        assert self.h
        self.pr = pr

    def f32(self, dp, p, init=None):
        pr, torch = self.pr, dp.torch
        out = torch.zeros(pr.O * pr.T, device="cuda", dtype=torch.float32)
        if init is not None:
            out.copy_(dev(torch, np.asarray(init, np.float32).reshape(-1)))
        st = self.L.refshim_diff2_coarse(self.h, pr.imgX, pr.imgY, 1, pr.imgMaxR, dp.eulers.data_ptr(),
                                         dp.tx.data_ptr(), dp.ty.data_ptr(), dp.corr[p].data_ptr(),
                                         dp.re[p].data_ptr(), dp.im[p].data_ptr(), out.data_ptr(),
                                         pr.O, pr.T, pr.N_img, torch.cuda.current_stream().cuda_stream)
        assert st == 0
        torch.cuda.synchronize()
        return out.cpu().numpy().reshape(pr.O, pr.T)

    def f64(self, dp, p, filter_img=False):
        pr, torch = self.pr, dp.torch
        out = torch.zeros(pr.O * pr.T, device="cuda", dtype=torch.float64)
        st = self.L.refshim_diff2_coarse_double(self.h, pr.imgX, pr.imgY, 1, pr.imgMaxR, dp.eulers.data_ptr(),
                                                dp.tx.data_ptr(), dp.ty.data_ptr(), dp.corr[p].data_ptr(),
                                                dp.re[p].data_ptr(), dp.im[p].data_ptr(), out.data_ptr(),
                                                pr.O, pr.T, pr.N_img, 1 if filter_img else 0,
                                                torch.cuda.current_stream().cuda_stream)
        assert st == 0
        torch.cuda.synchronize()
        return out.cpu().numpy().reshape(pr.O, pr.T)

    def close(self):
        if self.h:
            self.L.refshim_projector_destroy(self.h)
            self.h = None


def argmin_consistent(test, ref, rel_tol):
    """The argmin (o, t) must agree wherever the best-to-second gap of the
    reference exceeds the tolerance; returns (agree, gap_rel)."""
    r = np.asarray(ref, np.float64).ravel()
    t = np.asarray(test, np.float64).ravel()
    order = np.argsort(r)
    gap = (r[order[1]] - r[order[0]]) / abs(r[order[0]])
    if gap <= 2 * rel_tol:
        return True, gap
    return int(np.argmin(t)) == int(order[0]), gap
