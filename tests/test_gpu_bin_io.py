"""The reference's BIN output (src/output.f90:39-67) and warm start
(src/basegrid.f90:167-251) through the library's driver.

- the files the device run writes equal the oracle's after the same steps:
  the pointers file byte for byte, the blocks file on every cell the block
  update defines (the 16 corner ghost cells of a block are undefined on the
  device, as they are unused by the reference);
- a warm start continues the run bit for bit (AMR Sedov in FP64 through the
  step graphs; the jet, whose boundary depends on the run time);
- a warm start from the oracle's files with the reference's four admesh
  passes equals the oracle doing the same;
- an FP32 run's files start an FP64 run with the same values.
"""
import numpy as np
import pytest

from helpers import noncorner_mask

pytestmark = pytest.mark.gpu

W = 20


def _files(tmp_path, tag):
    return str(tmp_path / f"pointers_{tag}.bin"), str(tmp_path / f"blocks_{tag}.bin")


def _leaf_blocks(path, nleaf, neq):
    u = np.fromfile(path, dtype="<f8").reshape(nleaf, W, W, neq)
    return u.transpose(0, 3, 1, 2)


def test_device_files_equal_the_oracle_files(oracle_lib, tmp_path):
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config("sedov_amr_small")
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    s = Simulation(p, ic)
    o.run(12)
    s.run(12)
    fo, fd = _files(tmp_path, "orc"), _files(tmp_path, "dev")
    o.write_bin(*fo)
    s.write_bin(*fd)
    assert open(fo[0], "rb").read() == open(fd[0], "rb").read()
    n = o.nbleafs
    a, b = _leaf_blocks(fo[1], n, p.neq), _leaf_blocks(fd[1], n, p.neq)
    m = noncorner_mask()
    assert np.array_equal(a[:, :, m], b[:, :, m])


@pytest.mark.parametrize("name,graphs", [("sedov_amr_small", True), ("jet_small", False)])
def test_warm_start_continues_bit_for_bit(tmp_path, name, graphs):
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config(name)
    a = Simulation(p, ic)
    if graphs:
        a.ctx.set_graphs(True)
    a.run(8)
    f = _files(tmp_path, name)
    a.write_bin(*f)
    sa = a.status()
    b = Simulation(p, ic)
    if graphs:
        b.ctx.set_graphs(True)
    b.read_bin(*f, time=sa["time"])
    assert b.status()["nleaf"] == sa["nleaf"] and b.status()["time"] == sa["time"]
    for _ in range(8):
        a.run(1)
        b.run(1)
        assert a.status()["dt"] == b.status()["dt"]
    ta, tb = a.tree(), b.tree()
    for x, y in zip(ta, tb):
        assert np.array_equal(x, y)
    ids, ua = a.blocks()
    ids2, ub = b.blocks()
    assert np.array_equal(ids, ids2)
    m = noncorner_mask()
    assert np.array_equal(ua[:, :, m], ub[:, :, m])
    assert a.status()["time"] == b.status()["time"]


def test_warm_start_from_oracle_files_with_admesh(oracle_lib, tmp_path):
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config("sedov_amr_small")
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    o.run(10)
    f = _files(tmp_path, "orc")
    o.write_bin(*f, true_value=1)          # gfortran's encoding of .true.
    t0 = o.time
    o2 = oracle_lib.Oracle(p, ic, threads=8)
    o2.read_bin(*f, t0)
    for _ in range(4):                     # src/main.f90:59-62
        o2.admesh()
    s = Simulation(p, ic)
    s.read_bin(*f, time=t0, nadmesh=4)
    ids = o2.leaves()
    assert np.array_equal(np.nonzero(s.tree()[1])[0], ids)
    for _ in range(6):
        dt = o2.run(1)
        s.run(1)
        assert s.status()["dt"] == dt
    ids = o2.leaves()
    lp, lf, icd, _ = s.tree()
    assert np.array_equal(np.nonzero(lf)[0], ids)
    assert np.array_equal(lp[1:o2.nbmax + 1], o2.lp[1:o2.nbmax + 1])
    m = noncorner_mask()
    u = s.ctx.get_blocks(ids)
    assert np.array_equal(u[:, :, m], o2.u[ids][:, :, m])


def test_fp32_files_start_an_fp64_run(tmp_path):
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config("sedov_amr_small")
    p32 = p.copy()
    p32.precision = 32
    a = Simulation(p32, ic)
    a.run(10)
    f = _files(tmp_path, "fp32")
    a.write_bin(*f)
    ids, ua = a.blocks()
    b = Simulation(p, ic)
    b.read_bin(*f, time=a.status()["time"])
    ids2, ub = b.blocks()
    assert np.array_equal(ids, ids2)
    m = noncorner_mask()
    assert np.array_equal(ua[:, :, m], ub[:, :, m])
    assert np.array_equal(ub[:, :, m], ub[:, :, m].astype(np.float32).astype(np.float64))
    b.run(5)
