"""The coolingh surrogate on the tensor cores.

- gradients of the device training kernel against the CPU restatement of
  the network (oracle/nn_oracle.py) with the same BF16 operand rounding:
  relative L2 difference per parameter group <= 2e-2 (accumulation order
  and single BF16 ulp flips of intermediate operands);
- the forward pass against the same restatement: |difference| <= 2e-2;
- training on samples the exact routine labels reduces the loss, and the
  exact routine judges the trained network on fresh samples.
"""
import numpy as np
import pytest

from oracle import nn_oracle as nno

pytestmark = pytest.mark.gpu


def _net(seed=5):
    from walicxe2d_b200.api import Surrogate
    s = Surrogate(seed)
    rng = np.random.default_rng(seed)
    p = rng.normal(0.0, 0.25, nno.NPARAM).astype(np.float32)
    s.set_params(p)
    return s, p


@pytest.mark.parametrize("n", [128, 384, 1000])
def test_gradient_against_cpu(n):
    s, p = _net()
    rng = np.random.default_rng(n)
    X = rng.uniform(-1, 1, (n, 4)).astype(np.float32)
    Y = rng.uniform(-1, 1, (n, 2)).astype(np.float32)
    loss_d, g_d = s.grad(X, Y)
    loss_c, g_c = nno.loss_grad(p, X.astype(np.float64), Y.astype(np.float64), bf=True)
    assert abs(loss_d - loss_c) <= 1e-3 * abs(loss_c), (loss_d, loss_c)
    for name, sl in nno.groups():
        a, b = g_d[sl].astype(np.float64), g_c[sl]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel <= 2e-2, (name, rel)


def test_forward_against_cpu():
    s, p = _net(9)
    rng = np.random.default_rng(1)
    X = rng.uniform(-1, 1, (777, 4)).astype(np.float32)
    o_d = s.forward(X)
    o_c, _ = nno.forward(p, X.astype(np.float64), bf=True)
    assert np.abs(o_d - o_c).max() <= 2e-2, np.abs(o_d - o_c).max()


def test_training_reduces_loss_and_is_judged():
    from walicxe2d_b200.api import Surrogate
    s = Surrogate(20261203)
    s.samples(1 << 18, seed=20261203)
    first = s.train(1, batch=4096, lr=2e-3, lr_end=2e-3)
    last = s.train(4, batch=4096, lr=2e-3, lr_end=1e-4)
    assert np.isfinite(last) and last < first, (first, last)
    j = s.judge(1 << 16, seed=11)
    assert 0.0 < j["served"] <= 1.0
    assert j["t_err_median"] < 0.05, j


@pytest.fixture(scope="module")
def trained():
    from walicxe2d_b200.api import Surrogate
    s = Surrogate(20261203)
    s.samples(10_000_000, seed=20261203)
    s.train(100, batch=8192, lr=2e-3, lr_end=2e-5)
    return s


def test_surrogate_in_fp32_remnant_against_fp64_oracle(oracle_lib, trained):
    """FP32 path with the surrogate on the remnant set-up (coolingh, AMR):
    density L1 against the FP64 oracle <= 1e-3; the network serves most
    cells and the exact routine the rest."""
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config("snr_small")
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.startup()
    p32 = p.copy()
    p32.precision = 32
    s = Simulation(p32, ic)
    s.ctx.set_surrogate(trained)
    for _ in range(40):
        o.run(1)
        s.run(1)
    served, exact = s.ctx.surrogate_counts()
    assert served > 0 and exact >= 0
    assert served / (served + exact) > 0.3, (served, exact)
    ids = o.leaves()
    lp, lf, icd, ib = s.tree()
    if np.array_equal(np.nonzero(lf)[0], ids):
        rho = s.ctx.get_blocks(ids)[:, 0, 2:18, 2:18]
        ro = o.u[ids, 0, 2:18, 2:18]
        l1 = np.abs(rho - ro).sum() / np.abs(ro).sum()
        assert l1 <= 1e-3, l1


def test_surrogate_gain_over_exact_cooling(trained):
    """What the trained network gains: the same FP32 ensemble step with and
    without it (cooling kernels' device time), and the share it serves."""
    from walicxe2d_b200.api import Ensemble
    from walicxe2d_b200.params import ensemble_members
    mem = ensemble_members(count=24, precision=32)
    for p, ic in mem:
        p.nblocks = min(p.nblocks, 4000)
    t = {}
    for use in (False, True):
        ens = Ensemble(mem, threads=0)
        if use:
            ens.ctx.set_surrogate(trained)
        ens.run(5)
        ens.ctx.profile(True)
        ens.run(10)
        prof = ens.ctx.profile_read()
        ens.ctx.profile(False)
        t[use] = sum(v[1] for k, v in prof.items() if k in ("cooling", "cooling_nn", "calcprim"))
        if use:
            sv, ex = ens.ctx.surrogate_counts()
        ens.close()
    gain = t[False] / t[True]
    print(f"cooling ms: exact {t[False]:.3f}, surrogate {t[True]:.3f}, gain {gain:.2f}x, "
          f"served {sv / (sv + ex):.2f}")
    assert sv / (sv + ex) > 0.5
    assert gain > 1.0, gain
