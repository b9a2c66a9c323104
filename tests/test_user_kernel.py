"""The device-side API (include/pd/vector_dist_ker.cuh): user __global__ kernels
written against vd.toKernel() / cl.toKernel() with GET_PARTICLE,
GET_PARTICLE_SORT, getCell, getNNIteratorBox, get() and get_sort(), compiled by
nvcc for sm_100a into a program linked with libpdgpu.so, give the oracle's
cell-list walk within the reference's 3e-4 (FP32)
(Vector/cuda/vector_dist_gpu_unit_tests.cu:259-423, functor at :46-119)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
F32 = np.float32


def _nvcc():
    for c in (os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc"), shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    pytest.skip("nvcc not found")


def _compile(tmpdir):
    exe = os.path.join(tmpdir, "nn_user_kernel")
    lib = os.path.join(ROOT, "openfpm_pdata_b200")
    subprocess.run([_nvcc(), "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", os.path.join(ROOT, "include"), os.path.join(ROOT, "tests", "cpp", "nn_user_kernel.cu"),
                    "-L", lib, "-lpdgpu", "-Xlinker", "-rpath," + lib, "-o", exe], check=True)
    return exe


def test_user_kernel_compiles(tmp_path):
    """The device header compiles into user kernels and links with the library (no GPU call)."""
    assert os.path.exists(_compile(str(tmp_path)))


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["unsorted", "sorted"])
def test_user_kernel_matches_oracle(tmp_path, orc, variant):
    exe = _compile(str(tmp_path))
    rng = np.random.default_rng(55067)
    pos = rng.random((10000, 3)).astype(F32)
    inp = f"{pos.shape[0]}\n" + "\n".join(f"{a!r} {b!r} {c!r}" for a, b, c in pos.tolist())
    r = subprocess.run([exe, variant], input=inp, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    n_all, n_dom = (int(t) for t in lines[0].split()[1:3])
    assert n_dom == 10000
    xa = np.array([[float(t) for t in ln.split()] for ln in lines[1:1 + n_all]], dtype=F32)
    got = np.array([[float(t) for t in ln.split()] for ln in lines[1 + n_all:1 + n_all + n_dom]], dtype=F32)
    allp, p0 = np.ascontiguousarray(xa[:, :3]), np.ascontiguousarray(xa[:, 3])
    # the initialising user kernel wrote prop0 = x + y + z on the device
    np.testing.assert_allclose(p0[:n_dom], allp[:n_dom].sum(axis=1), rtol=1e-6)
    lo, hi = np.zeros(3, F32), np.ones(3, F32)
    G = orc.cl_geometry(lo, hi, F32(0.1), F32(0.1), dtype=F32)
    exp = orc.test_force(allp, p0, n_dom, G)
    assert np.max(np.abs(got - exp)) < 3e-4
    assert np.abs(exp).sum() > 1000  # the walk found neighbours
