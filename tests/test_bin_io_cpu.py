"""The reference's BIN output and warm start on the CPU oracle.

The file layout (src/output.f90:39-67, read back by src/basegrid.f90:167-251
and by the reference's py/walicxe2d_utils.py read_mesh/read_blocks) is
decoded here independently with numpy: four 4-byte integers (nbmin, nbmax,
nbleafs, nblocks), lp(nbmin:nbmax,1:8), leaf(nbmin:nbmax) and
icoord(nbmin:nbmax,1:2) column-major; then, in the blocks file, u(nb,:,:,:)
of every leaf in ascending ID with the equation index fastest, then i, then
j, as 8-byte reals.  A warm start from the files continues the run bit for
bit.
"""
import os

import numpy as np
import pytest

W = 20


def _decode(pointers, blocks, neq):
    head = np.fromfile(pointers, dtype="<i4", count=4)
    nbmin, nbmax, nbleafs, nblocks = (int(x) for x in head)
    n = nbmax - nbmin + 1
    body = np.fromfile(pointers, dtype="<i4", offset=16)
    assert body.size == 11 * n
    lp = body[: 8 * n].reshape(8, n).T
    leaf = body[8 * n: 9 * n]
    icoord = body[9 * n:].reshape(2, n).T
    u = np.fromfile(blocks, dtype="<f8")
    assert u.size == nbleafs * neq * W * W
    # per leaf: [j][i][eq] in file order -> [eq][j][i]
    u = u.reshape(nbleafs, W, W, neq).transpose(0, 3, 1, 2)
    return (nbmin, nbmax, nbleafs, nblocks), lp, leaf, icoord, u


@pytest.mark.parametrize("true_value", [-1, 1])
def test_oracle_bin_layout(oracle_lib, tmp_path, true_value):
    from walicxe2d_b200.params import config
    p, ic = config("sedov_amr_small")
    o = oracle_lib.Oracle(p, ic, threads=4)
    o.startup()
    o.run(10)
    fp, fb = str(tmp_path / "pointers000.bin"), str(tmp_path / "blocks000.bin")
    o.write_bin(fp, fb, true_value)
    head, lp, leaf, icoord, u = _decode(fp, fb, p.neq)
    nbmax = o.nbmax
    assert head == (1, nbmax, o.nbleafs, p.nblocks)
    assert np.array_equal(lp, o.lp[1: nbmax + 1])
    assert np.array_equal(leaf, np.where(o.leaf[1: nbmax + 1] != 0, true_value, 0))
    assert np.array_equal(icoord, o.icoord[1: nbmax + 1])
    ids = o.leaves()
    assert np.array_equal(u, o.u[ids])


def test_oracle_warm_start_continues_bit_for_bit(oracle_lib, tmp_path):
    from walicxe2d_b200.params import config
    p, ic = config("sedov_amr_small")
    a = oracle_lib.Oracle(p, ic, threads=4)
    a.startup()
    a.run(8)
    fp, fb = str(tmp_path / "p.bin"), str(tmp_path / "b.bin")
    a.write_bin(fp, fb)
    b = oracle_lib.Oracle(p, ic, threads=4)
    b.read_bin(fp, fb, a.time)
    assert b.nbmax == a.nbmax and b.nbleafs == a.nbleafs
    for _ in range(8):
        assert a.run(1) == b.run(1)
    assert np.array_equal(a.lp, b.lp) and np.array_equal(a.leaf, b.leaf)
    ids = a.leaves()
    assert np.array_equal(ids, b.leaves())
    assert np.array_equal(a.u[ids], b.u[ids])


def test_oracle_reader_refuses_bad_files(oracle_lib, tmp_path):
    from walicxe2d_b200.params import config
    p, ic = config("sedov_amr_small")
    o = oracle_lib.Oracle(p, ic, threads=2)
    o.startup()
    fp, fb = str(tmp_path / "p.bin"), str(tmp_path / "b.bin")
    o.write_bin(fp, fb)
    raw = open(fb, "rb").read()
    short = str(tmp_path / "short.bin")
    open(short, "wb").write(raw[:-8])
    longer = str(tmp_path / "long.bin")
    open(longer, "wb").write(raw + b"\0" * 8)
    for bad in (short, longer):
        q = oracle_lib.Oracle(p, ic, threads=2)
        with pytest.raises(RuntimeError):
            q.read_bin(fp, bad, 0.0)
    # a tree larger than the pool
    small = p.copy()
    small.nblocks = o.nbmax - 1
    q = oracle_lib.Oracle(small, ic, threads=2)
    with pytest.raises(RuntimeError):
        q.read_bin(fp, fb, 0.0)
    assert os.path.getsize(fp) == 16 + 44 * o.nbmax
