"""Generate golden vectors from the reference's own kernels.

Runs on a machine with a CUDA GPU and the reference kernels compiled into
oracle/_ref/libref_diff2.so (oracle/Makefile builds them from the reference
sources).  For the small seeded problem "g0" (box 16, 72 orientations, 9
translations, 2 particles with CTF) it stores the inputs and the outputs of
runDiff2KernelCoarse (FP32) and runDiff2KernelCoarseDouble (FP64):

    python tests/golden/make_golden.py [out_dir]      # default tests/golden
"""
from __future__ import annotations

import ctypes as C
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def main(out_dir: str) -> str:
    import torch

    from conftest import load_package
    import oracle
    from gpu_util import DeviceProblem, RefKernels

    load_package()
    import importlib
    synth = importlib.import_module("relion_b200.synth")
    pr = synth.make_problem("g0")
    ref = RefKernels(oracle, pr)
    dp = DeviceProblem(torch, pr)
    f32 = np.stack([ref.f32(dp, p) for p in range(pr.P)])
    f64 = np.stack([ref.f64(dp, p) for p in range(pr.P)])
    ref.close()
    # this library's texture projections at every image pixel (same sample
    # positions as the reference kernels, sampled by the same texture unit)
    import relion_b200 as pkg
    proj = pkg.Projector(pr.projector, use_texture=1)
    view = proj.view(pr.imgX, pr.imgY, pr.imgMaxR)
    x, y = synth.pixel_coords(pr.imgX, pr.imgY, view.maxR)
    d_x = torch.as_tensor(x, device="cuda")
    d_y = torch.as_tensor(y, device="cuda")
    pre = torch.empty(pr.O * pr.N_img, device="cuda")
    pim = torch.empty(pr.O * pr.N_img, device="cuda")
    pkg.project_pixels(view, dp.eulers, d_x, d_y, pre, pim, pr.O, pr.N_img)
    torch.cuda.synchronize()
    prj_re = pre.cpu().numpy().reshape(pr.O, pr.N_img)
    prj_im = pim.cpu().numpy().reshape(pr.O, pr.N_img)
    proj.close()
    pv = pr.projector
    os.makedirs(out_dir, exist_ok=True)
    path = os.path.join(out_dir, "ref_g0.npz")
    np.savez_compressed(
        path, vol_re=pv.re, vol_im=pv.im, mdlX=pv.mdlX, mdlY=pv.mdlY, mdlZ=pv.mdlZ, mdlInitY=pv.mdlInitY,
        mdlInitZ=pv.mdlInitZ, mdlMaxR=pv.mdlMaxR, pf=pv.padding_factor, imgX=pr.imgX, imgY=pr.imgY,
        imgMaxR=pr.imgMaxR, eulers=pr.eulers, trans_x=pr.trans_x, trans_y=pr.trans_y, fimg_re=pr.fimg_re,
        fimg_im=pr.fimg_im, corr=pr.corr, ref_f32=f32, ref_f64=f64, prj_re=prj_re, prj_im=prj_im,
        gpu=np.array(torch.cuda.get_device_name(0)))
    return path


if __name__ == "__main__":
    print(main(sys.argv[1] if len(sys.argv) > 1 else HERE))
