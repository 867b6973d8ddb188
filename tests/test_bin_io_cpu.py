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


def test_reference_reader_sees_the_oracle_state(oracle_lib, tmp_path):
    """tests/golden/bin_reader_sedov.json holds what the reference's own
    reader (py/walicxe2d_utils.py, run by tests/golden/make_bin_golden.py)
    made of the oracle's BIN files after 12 steps of the small AMR blast:
    the mesh table (corners and level of every leaf), per-leaf sums of the
    decoded blocks, and the sum of the density map at the finest
    resolution.  The oracle's state gives the same, so the files carry
    that state as the reference's post-processing reads it."""
    import json

    from scipy import ndimage

    from walicxe2d_b200.params import config
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "bin_reader_sedov.json")))
    p, ic = config("sedov_amr_small")
    o = oracle_lib.Oracle(p, ic, threads=4)
    o.startup()
    o.run(12)
    ids = o.leaves()
    assert len(ids) == g["nleaf"]
    lp, icd = o.lp, o.icoord
    mesh = []
    for nb in ids:
        lev = int(lp[nb, 0])
        dx = p.xmax / p.nbroot_x / p.nx / (2.0 ** (lev - 1))
        dy = p.ymax / p.nbroot_y / p.ny / (2.0 ** (lev - 1))
        mesh.append([icd[nb, 0] * dx, icd[nb, 1] * dy, (icd[nb, 0] + p.nx) * dx, (icd[nb, 1] + p.ny) * dy,
                     float(lev), 0.0])
    assert mesh == g["mesh"]
    # the reader's blocks[a, b, eq, leaf] is u(leaf, eq, i=a, j=b)
    blk = np.zeros((W, W, p.neq, len(ids)))
    for q, nb in enumerate(ids):
        for k in range(p.neq):
            blk[:, :, k, q] = o.u[nb, k].T
    sums = [[float(blk[:, :, k, q].sum()) for k in range(p.neq)] for q in range(len(ids))]
    assert sums == g["block_sums"]
    # density at the finest resolution, coarser leaves zoomed (order 1)
    nxt, nyt = p.nbroot_x * p.nx * 2 ** (p.nlevs - 1), p.nbroot_y * p.ny * 2 ** (p.nlevs - 1)
    rho = np.zeros((nxt, nyt))
    for q, nb in enumerate(ids):
        f = 2 ** (p.nlevs - int(lp[nb, 0]))
        x0, y0 = int(icd[nb, 0]) * f, int(icd[nb, 1]) * f
        a = blk[2:p.ny + 2, 2:p.nx + 2, 0, q]
        rho[x0:x0 + f * p.nx, y0:y0 + f * p.ny] = a if f == 1 else ndimage.zoom(a, f, order=1)
    assert list(rho.T.shape) == g["map_shape"]
    assert abs(rho.sum() - g["map_sum"]) <= 1e-12 * abs(g["map_sum"])
