"""The device's rules for the block tree's integer work (walicxe2d_b200/csrc/
w2d_mark.cu), restated here in numpy and checked on the CPU against the
oracle's restatement of the reference's own loops, at many tree states:

- locatebounds (src/locatebounds.f90:29-540): each leaf's entries follow
  from its links (a box wall always; a same-level leaf only from the lower
  ID of the pair; a same-level block with sons always, toward its facing
  son of lower ID; a coarser neighbour never) -- the same list, in the same
  order, as the oracle's sequential walk with bnd flags;
- one admesh pass (src/admesh.f90:23-105): markref, the closure of
  critneighup, critneighdown as the tree stands after the pass's refines,
  and the families coarsened -- the same refines and coarsenings as the
  oracle's admesh.
"""
import os

import numpy as np
import pytest

from oracle import oracle as orc

SAME, REST, SON_OFF = (1, 4, 7, 10), (2, 5, 8, 11), (1, 0, 2, 0)


def locate_by_owner(lp, leaf, nbmax):
    out = []
    for nb in range(1, nbmax + 1):
        if not leaf[nb]:
            continue
        for s in range(4):
            m = int(lp[nb, 4 + s])
            if m == -1:
                out.append((nb, 0, -(s + 1)))
            elif lp[m, 0] < lp[nb, 0]:
                continue                                   # coarser: its entry
            elif leaf[m]:
                if nb < m:
                    out.append((nb, m, SAME[s]))
            else:
                out.append((nb, int(lp[m, 2]) + SON_OFF[s], REST[s]))
    return np.array(out, np.int64).reshape(-1, 3)


def flags_by_rule(lp, leaf, nbmax, grad, tol, tol2, nlevs):
    lev = lp[:, 0]
    up = np.zeros(nbmax + 1, bool)
    down = np.zeros(nbmax + 1, bool)
    for nb in range(1, nbmax + 1):
        if not leaf[nb] or lev[nb] < 1:
            continue
        g = grad[nb - 1]
        if g >= tol:
            up[nb] = lev[nb] < nlevs
        elif g <= tol2:
            down[nb] = True
    stack = list(np.nonzero(up)[0])                        # critneighup: the closure
    while stack:
        x = stack.pop()
        for m in lp[x, 4:8]:
            if m != -1 and lev[m] < lev[x] and not up[m]:
                up[m] = True
                stack.append(int(m))
    refined = up & (lev[: nbmax + 1] >= 1) & (lev[: nbmax + 1] <= nlevs - 1)
    down2 = down & ~refined                                # critneighdown after the refines
    for nb in np.nonzero(down2)[0]:
        for m in lp[nb, 4:8]:
            if m == -1:
                continue
            if refined[m] and lev[m] < lev[nb]:
                continue                                   # now a new son, a leaf
            if not leaf[m] or refined[m]:
                down2[nb] = False
    first = []
    for nb in np.nonzero(down2)[0]:
        if lp[nb, 3] != 1 or not (2 <= lev[nb] <= nlevs):
            continue
        s2, s3 = lp[nb, 5], lp[nb, 7]
        s4 = lp[s2, 7]
        if down2[s2] and down2[s3] and down2[s4]:
            first.append(int(nb))
    ref = sorted(np.nonzero(refined)[0].tolist(), key=lambda b: (lev[b], b))
    first = sorted(first, key=lambda b: (-lev[b], b))
    return ref, first


def _oracle(name, **over):
    from walicxe2d_b200.params import COOLINGDMC, config
    p, ic = config(name)
    for k, v in over.items():
        setattr(p, k, v)
    o = orc.Oracle(p, ic, threads=4)
    if p.cooling == COOLINGDMC:
        rows = np.loadtxt(os.path.join(os.path.dirname(__file__), "golden", "coolingDMC.tab"))
        o.set_cooltab(rows[:, 0], rows[:, 1])
    o.startup()
    return p, o


def _check_state(p, o):
    """Both rules at the oracle's current state, then one admesh pass."""
    lp, leaf, nbmax = o.lp.copy(), o.leaf.copy(), o.nbmax
    o.locatebounds()
    assert np.array_equal(o.innerbounds.astype(np.int64), locate_by_owner(lp, leaf, nbmax))
    ref, first = flags_by_rule(lp, leaf, nbmax, o.criteria(), p.tol, p.tol2, p.nlevs)
    dads = [int(lp[b, 1]) for b in first]
    o.admesh()
    leaf2 = o.leaf
    # a coarsened parent becomes a leaf and its sons (leaves before) stop
    # being leaves; a refine may reuse four slots of an old family, which
    # become leaves without being parents of leaves
    coarsened = [b for b in range(1, nbmax + 1)
                 if not leaf[b] and leaf2[b] and lp[b, 2] > 0 and leaf[lp[b, 2]]]
    sons = {int(lp[d, 2]) + q for d in coarsened for q in range(4)}
    refined = [b for b in range(1, nbmax + 1) if leaf[b] and not leaf2[b] and b not in sons]
    assert sorted(ref) == refined
    assert sorted(dads) == coarsened
    return len(ref), len(first)


@pytest.mark.parametrize("name,steps", [("sedov_amr_small", 120), ("jet_small", 200), ("snr_small", 100),
                                        ("jet_cyl_small", 60)])
def test_rules_equal_the_oracle_loops(name, steps):
    p, o = _oracle(name)
    nref = ncoar = 0
    for _ in range(steps):
        o.run(1, amr=False)               # a step, then its own admesh pass, checked
        r, c = _check_state(p, o)
        nref += r
        ncoar += c
    assert nref + ncoar > 0               # the passes did change the mesh


@pytest.mark.parametrize("mode", ["refine_all", "coarsen_all"])
def test_rules_on_passes_that_change_every_block(mode):
    from walicxe2d_b200.params import sedov
    p, ic = sedov(nbroot=12, nlevs=3, tol=0.1, nblocks=12 * 12 * 21 + 16, startup_admesh=0)
    if mode == "refine_all":
        p.tol = -1.0
    else:
        p.tol, p.tol2 = 1e30, 1e30
        ic.init_levels = 3
    o = orc.Oracle(p, ic, threads=4)
    o.basegrid()
    counts = [_check_state(p, o) for _ in range(3)]
    if mode == "refine_all":
        assert counts[0][0] == 144 and counts[1][0] == 576, counts
    else:
        assert counts[0][1] == 576 and counts[1][1] == 144, counts
