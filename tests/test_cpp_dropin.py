"""The reference harness's C++ API (include/b200d2_relion.hpp) over the C ABI:
compile a C++ caller against it (CPU), and run it on the GPU on .dat files in
the reference's replay formats."""
from __future__ import annotations

import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cpp", "relion_dropin.cpp")
LIBDIR = os.path.join(ROOT, "t2-relion-kernel_b200", "lib")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def build(out_dir: str) -> str:
    exe = os.path.join(out_dir, "relion_dropin")
    cmd = ["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), "-I",
           os.path.join(CUDA, "include"), SRC, "-o", exe, "-L", LIBDIR, "-lb200d2",
           f"-Wl,-rpath,{LIBDIR}", "-L", os.path.join(CUDA, "lib64"), "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_caller_compiles(pkg, tmp_path):
    pkg.lib()  # the library must exist (built by __graft_entry__.build)
    assert os.path.exists(build(str(tmp_path)))


@pytest.mark.gpu
def test_cpp_caller_runs_on_dat_files(pkg, synth, cuda, tmp_path):
    pr = synth.make_problem("c1", P=1)
    pj = os.path.join(tmp_path, "projector_proc_1_1.dat")
    cd = os.path.join(tmp_path, "coarse_data100_1.dat")
    synth.write_projector_dat(pj, pr.projector)
    import numpy as np
    init = np.random.default_rng(5).uniform(0, 10, pr.O * pr.T)
    synth.write_coarse_dat(cd, pr, 0, diff2_init=init)
    back = synth.read_coarse_dat(cd)
    assert back["O"] == pr.O and back["T"] == pr.T and back["image_size"] == pr.N_img
    exe = build(str(tmp_path))
    r = subprocess.run([exe, pj, cd], capture_output=True, text=True, timeout=300)
    print(r.stdout, r.stderr)
    assert r.returncode == 0, r.stderr
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["fp32_vs_fp64_max_rel"] <= 1e-5
    assert res["functor_vs_fp64_max_rel"] <= 1e-5
    assert res["bf16x3_dropin_vs_fp64_max_rel"] <= 1e-5  # runDiff2KernelCoarse on the tensor cores
    assert res["cc_fp32_vs_fp64_max_rel"] <= 1e-5  # runDiff2KernelCoarse with do_CC
