"""Generate golden vectors from the reference's own kernels.

Runs on a machine with a CUDA GPU and the reference kernels compiled into
oracle/_ref/libref_diff2.so (oracle/Makefile builds them from the reference
sources).  For each fixture it stores the outputs of runDiff2KernelCoarse
(FP32) and runDiff2KernelCoarseDouble (FP64) and this library's texture-unit
projections at every image pixel (the same sample positions, sampled by the
same texture unit):

- ref_g0.npz: the small seeded problem "g0" (box 16, 72 orientations, 9
  translations, 2 particles with CTF), every input stored in the file;
- ref_c1s.npz: the C1 problem (image 32, 544 half-plane pixels of which those
  within radius 16 meet the projector, 21 translations), its first 2
  particles and every 9th of its 576 orientations; the inputs are rebuilt from
  the seeded generator and checked by SHA-256 (tests/golden_util.py), so the
  file holds only outputs and projections.

    python tests/golden/make_golden.py [out_dir]      # default tests/golden
"""
from __future__ import annotations

import dataclasses
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def reference_outputs(torch, pkg, synth, oracle, pr):
    """(f32 [P,O,T], f64 [P,O,T], prj_re [O,N], prj_im [O,N]) for problem pr."""
    from gpu_util import DeviceProblem, RefKernels
    ref = RefKernels(oracle, pr)
    dp = DeviceProblem(torch, pr)
    f32 = np.stack([ref.f32(dp, p) for p in range(pr.P)])
    f64 = np.stack([ref.f64(dp, p) for p in range(pr.P)])
    ref.close()
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
    return f32, f64, prj_re, prj_im


def main(out_dir: str) -> list[str]:
    import torch

    from conftest import load_package
    import golden_util
    import oracle

    pkg = load_package()
    import importlib
    synth = importlib.import_module("relion_b200.synth")
    os.makedirs(out_dir, exist_ok=True)
    paths = []

    # g0: self-contained
    pr = synth.make_problem("g0")
    f32, f64, prj_re, prj_im = reference_outputs(torch, pkg, synth, oracle, pr)
    pv = pr.projector
    path = os.path.join(out_dir, "ref_g0.npz")
    np.savez_compressed(
        path, vol_re=pv.re, vol_im=pv.im, mdlX=pv.mdlX, mdlY=pv.mdlY, mdlZ=pv.mdlZ, mdlInitY=pv.mdlInitY,
        mdlInitZ=pv.mdlInitZ, mdlMaxR=pv.mdlMaxR, pf=pv.padding_factor, imgX=pr.imgX, imgY=pr.imgY,
        imgMaxR=pr.imgMaxR, eulers=pr.eulers, trans_x=pr.trans_x, trans_y=pr.trans_y, fimg_re=pr.fimg_re,
        fimg_im=pr.fimg_im, corr=pr.corr, ref_f32=f32, ref_f64=f64, prj_re=prj_re, prj_im=prj_im,
        gpu=np.array(torch.cuda.get_device_name(0)))
    paths.append(path)

    # c1s: regenerated inputs, C1 image and translations
    seed, particles, o_stride = 20251203, 2, 9
    full = synth.make_problem("c1", seed=seed)
    ins = golden_util.inputs_of(full, particles, o_stride)
    pr = dataclasses.replace(full, eulers=ins["eulers"], fimg_re=ins["fimg_re"], fimg_im=ins["fimg_im"],
                             corr=ins["corr"], true_orient=full.true_orient[:particles],
                             true_trans=full.true_trans[:particles])
    f32, f64, prj_re, prj_im = reference_outputs(torch, pkg, synth, oracle, pr)
    path = os.path.join(out_dir, "ref_c1s.npz")
    np.savez_compressed(
        path, problem=np.array("c1"), seed=seed, particles=particles, o_stride=o_stride,
        **{"sha256_" + k: np.array(golden_util.digest(v)) for k, v in ins.items()},
        ref_f32=f32, ref_f64=f64, prj_re=prj_re, prj_im=prj_im, gpu=np.array(torch.cuda.get_device_name(0)))
    paths.append(path)
    return paths


if __name__ == "__main__":
    for p in main(sys.argv[1] if len(sys.argv) > 1 else HERE):
        print(p)
