"""The C++ host API (include/pd/vector_dist_gpu.hpp) drives the CUDA path: a
compiled C++ program runs the reference-style loop and the integrator, and its
results equal the oracle's."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _compile(tmpdir):
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else shutil.which("g++")
    exe = os.path.join(tmpdir, "lj_host")
    lib = os.path.join(ROOT, "openfpm_pdata_b200")
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "lj_host.cpp"), "-L", lib, "-lpdgpu",
                    "-Wl,-rpath," + lib, "-o", exe], check=True)
    return exe


def test_cpp_host_compiles(tmp_path):
    """The header and the C ABI compile and link into a C++ program (no GPU call)."""
    assert os.path.exists(_compile(str(tmp_path)))


@pytest.mark.gpu
def test_cpp_host_lj_matches_oracle(tmp_path, orc):
    from openfpm_pdata_b200 import workloads
    exe = _compile(str(tmp_path))
    x, v, L = workloads.lj_lattice(9, 1.1, 0.05, seed=21)
    inp = f"{x.shape[0]} {L!r}\n" + "\n".join(" ".join(repr(float(t)) for t in np.concatenate([x[i], v[i]]))
                                              for i in range(x.shape[0]))
    r = subprocess.run([exe, "15"], input=inp, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    lines = r.stdout.strip().splitlines()
    pairs = int(lines[0].split()[1])
    E = np.array([[float(t) for t in ln.split()[1:]] for ln in lines[1:]])
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)
    img, _, _ = orc.ghost_get(orc.wrap(x, lo, hi, bc), lo, hi, bc, 2.8)
    allp = np.concatenate([orc.wrap(x, lo, hi, bc), img])
    G = orc.cl_geometry(lo, hi, 2.8, 2.8, verlet=True)
    off, _ = orc.verlet(allp, x.shape[0], G, 2.8)
    assert pairs == off[-1]
    _, _, Eo = orc.md_lj(x, v, lo, hi, bc, 2.8, 2.5, 0.3, 1.0, 1.0, 0.005, 1.0, 15)
    np.testing.assert_allclose(E[:, :3], Eo[1:, :3], rtol=1e-9, atol=1e-9)
