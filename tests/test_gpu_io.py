"""Checkpoint / restart and particle writers through the C ABI.

save / load mirror Vector/tests/vector_dist_HDF5_chckpnt_restart_test.cpp:24-117
(a 32^3 grid, non-periodic, float positions, float[3] property 0.51234 + x + y + z:
after load the sizes, positions and properties are equal); the format is this
library's own checksummed binary file.  An MD run restarted from a checkpoint
follows the uninterrupted run.  write / write_frame emit VTK XML PolyData
(ASCII and base64 binary) and CSV, parsed back here.
"""
import base64
import os
import xml.etree.ElementTree as ET

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

F32, F64 = np.float32, np.float64


@pytest.fixture(scope="module")
def pd():
    from openfpm_pdata_b200 import pd as _pd
    _pd.lib()
    return _pd


def _grid_vd(pd, ng=32):
    k = np.arange(ng)
    z, y, x = np.meshgrid(k, k, k, indexing="ij")
    sp = F32(1.0) / F32(ng)
    pos = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1).astype(F32) * sp
    vd = pd.VectorDist(pos.shape[0], np.zeros(3), np.ones(3), np.zeros(3, np.int32), 1.0 / (ng - 2), dtype=F32,
                       props=[(pd.PD_F32, 3)])
    vd.hostToDevicePos(pos)
    vd.map()
    p = vd.deviceToHostPos(with_ghost=False)
    f = np.repeat((F32(0.51234) + p[:, 0] + p[:, 1] + p[:, 2]).astype(F32)[:, None], 3, axis=1)
    vd.hostToDeviceProp(0, f)
    return vd


def test_save_load_reference_case(pd, tmp_path):
    vd = _grid_vd(pd)
    path = str(tmp_path / "vector_dist1.pdv")
    vd.save(path)
    vd2 = pd.VectorDist(0, np.zeros(3), np.ones(3), np.zeros(3, np.int32), 1.0 / 30, dtype=F32,
                        props=[(pd.PD_F32, 3)])
    vd2.load(path)
    assert vd2.size_local() == vd.size_local() == 32 ** 3
    assert np.array_equal(vd2.deviceToHostPos(), vd.deviceToHostPos(with_ghost=False))
    assert np.array_equal(vd2.deviceToHostProp(0), vd.deviceToHostProp(0, with_ghost=False))
    assert np.array_equal(vd2.gid(), vd.gid(with_ghost=False))
    # a vector without properties receives the file's
    vd3 = pd.VectorDist(0, np.zeros(3), np.ones(3), np.zeros(3, np.int32), 1.0 / 30, dtype=F32)
    vd3.load(path)
    assert vd3.props == [(pd.PD_F32, 3)]
    assert np.array_equal(vd3.deviceToHostProp(0), vd.deviceToHostProp(0, with_ghost=False))


def test_load_rejects_bad_files(pd, tmp_path):
    vd = _grid_vd(pd, 8)
    path = str(tmp_path / "c.pdv")
    vd.save(path)
    raw = bytearray(open(path, "rb").read())
    bad = str(tmp_path / "bad.pdv")
    raw2 = bytearray(raw)
    raw2[200] ^= 0x40                      # a flipped bit in the positions
    open(bad, "wb").write(raw2)
    tgt = pd.VectorDist(0, np.zeros(3), np.ones(3), np.zeros(3, np.int32), 0.1, dtype=F32, props=[(pd.PD_F32, 3)])
    with pytest.raises(pd.PdError) as e:
        tgt.load(bad)
    assert e.value.code == -8
    open(bad, "wb").write(raw[: len(raw) - 20])   # truncated
    with pytest.raises(pd.PdError) as e:
        tgt.load(bad)
    assert e.value.code == -8
    open(bad, "wb").write(b"not a checkpoint at all" * 10)
    with pytest.raises(pd.PdError):
        tgt.load(bad)
    wrong_t = pd.VectorDist(0, np.zeros(3), np.ones(3), np.zeros(3, np.int32), 0.1, dtype=F64,
                            props=[(pd.PD_F32, 3)])
    with pytest.raises(pd.PdError) as e:
        wrong_t.load(path)
    assert e.value.code == -1
    wrong_p = pd.VectorDist(0, np.zeros(3), np.ones(3), np.zeros(3, np.int32), 0.1, dtype=F32,
                            props=[(pd.PD_F64, 3)])
    with pytest.raises(pd.PdError):
        wrong_p.load(path)
    tgt.load(path)                                   # the good file still loads
    assert tgt.size_local() == 512


def test_md_restart_follows_uninterrupted_run(pd, orc, tmp_path):
    """60 LJ steps in one go against 30 steps, save, load into a new vector and a
    new driver, 30 more: energies within 1e-10 relative, positions within 1e-9."""
    from openfpm_pdata_b200 import workloads
    x, v, L = workloads.lj_lattice(10, 1.1, 0.05, seed=8)
    lo, hi, bc = np.zeros(3), np.full(3, L), np.ones(3, np.int32)

    def system():
        vd = pd.VectorDist(x.shape[0], lo, hi, bc, 2.8, dtype=F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
        vd.hostToDevicePos(x)
        vd.hostToDeviceProp(0, v)
        return vd
    a = system()
    Ea = pd.MD(a, 0, 1, dt=0.005, skin=0.3).run(60)
    b = system()
    mb = pd.MD(b, 0, 1, dt=0.005, skin=0.3)
    Eb1 = mb.run(30)
    path = str(tmp_path / "md.pdv")
    b.save(path)
    del mb
    c = pd.VectorDist(0, lo, hi, bc, 2.8, dtype=F64, props=[(pd.PD_F64, 3), (pd.PD_F64, 3)])
    c.load(path)
    Eb2 = pd.MD(c, 0, 1, dt=0.005, skin=0.3).run(30)
    Eb = np.concatenate([Eb1, Eb2])
    assert np.all(np.abs(Eb[:, :3] - Ea[:, :3]) <= 1e-10 * np.abs(Ea[:, :3]).max(axis=0))
    xa = np.zeros_like(x)
    xa[a.gid(with_ghost=False)] = a.deviceToHostPos(with_ghost=False)
    xc = np.zeros_like(x)
    xc[c.gid(with_ghost=False)] = c.deviceToHostPos(with_ghost=False)
    assert np.abs(xa - xc).max() <= 1e-9


def _arrays(path):
    root = ET.parse(path).getroot()
    piece = root.find("PolyData/Piece")
    out = {}
    for da in root.iter("DataArray"):
        t = {"Float32": F32, "Float64": F64, "Int32": np.int32, "UInt32": np.uint32, "Int64": np.int64}[da.get("type")]
        nc = int(da.get("NumberOfComponents", "1"))
        if da.get("format") == "binary":
            raw = base64.b64decode(da.text.strip())
            nb = int(np.frombuffer(raw[:4], np.uint32)[0])
            a = np.frombuffer(raw[4:4 + nb], t)
        else:
            a = np.array(da.text.split(), dtype=F64 if np.issubdtype(t, np.floating) else np.int64).astype(t)
        out[da.get("Name")] = a.reshape(-1, nc) if nc > 1 else a
    return int(piece.get("NumberOfPoints")), out


@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("dtype", [F32, F64])
def test_write_vtp(pd, tmp_path, binary, dtype):
    rng = np.random.default_rng(2)
    n = 777
    vd = pd.VectorDist(n, np.zeros(3), np.ones(3), np.ones(3, np.int32), 0.1, dtype=dtype,
                       props=[(pd.PD_F64, 3), (pd.PD_I32, 1), (pd.PD_F32, 2)])
    x = rng.random((n, 3)).astype(dtype)
    a = rng.normal(size=(n, 3))
    b = rng.integers(-5, 5, size=n).astype(np.int32)
    c = rng.normal(size=(n, 2)).astype(F32)
    vd.hostToDevicePos(x)
    for p, arr in enumerate([a, b, c]):
        vd.hostToDeviceProp(p, arr)
    vd.map()
    vd.ghost_get()                               # ghosts exist but are not written
    out = str(tmp_path / "particles")
    vd.write(out, "time = 1.25", opt=pd.FORMAT_BINARY if binary else pd.VTK_WRITER)
    npts, arrs = _arrays(out + "_0.vtp")
    assert npts == n
    assert np.array_equal(arrs["Points"], x)
    assert np.array_equal(arrs["attr0"], a) and np.array_equal(arrs["attr1"], b) and np.array_equal(arrs["attr2"], c)
    assert np.array_equal(arrs["connectivity"], np.arange(n)) and np.array_equal(arrs["offsets"], np.arange(1, n + 1))
    assert float(arrs["time"][0]) == 1.25
    vd.write_frame(out, 7)
    assert os.path.exists(out + "_0_7.vtp")


def test_write_csv(pd, tmp_path):
    rng = np.random.default_rng(3)
    n = 321
    vd = pd.VectorDist(n, np.zeros(3), np.ones(3), np.ones(3, np.int32), 0.1, dtype=F64,
                       props=[(pd.PD_F64, 1), (pd.PD_F32, 3)])
    x = rng.random((n, 3))
    a = rng.normal(size=n)
    c = rng.normal(size=(n, 3)).astype(F32)
    vd.hostToDevicePos(x)
    vd.hostToDeviceProp(0, a)
    vd.hostToDeviceProp(1, c)
    out = str(tmp_path / "parts")
    vd.write(out, opt=pd.CSV_WRITER)
    lines = open(out + "_0.csv").read().splitlines()
    assert lines[0] == "x[0],x[1],x[2],attr0,attr1[0],attr1[1],attr1[2]"
    t = np.array([[float(v) for v in ln.split(",")] for ln in lines[1:]])
    assert t.shape == (n, 7)
    assert np.array_equal(t[:, :3], x) and np.array_equal(t[:, 3], a)
    assert np.array_equal(t[:, 4:].astype(F32), c)
    vd.write_frame(out, 3, opt=pd.CSV_WRITER)
    assert os.path.exists(out + "_0_3.csv")
