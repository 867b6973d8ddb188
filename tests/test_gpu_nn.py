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
    j = s.judge(1 << 16, seed=11, tol=0.1)
    assert 0.0 < j["served"] <= 1.0
    assert j["t_err_median"] < 0.05, j


def test_judge_at_the_serve_tolerance(trained):
    """The exact routine rates the trained network at the cooling kernel's
    own serve test (tolerance 0.2%: predicted changes of T, of the thermal
    pressure and of the neutral fraction): among the samples it would
    serve, the errors of T and of the neutral fraction stay small."""
    import json
    import os
    j = trained.judge(1 << 20, seed=13, tol=0.002)
    path = os.environ.get("W2D_PARITY_LOG")
    if path:
        with open(path, "a") as f:
            f.write(json.dumps({"test": "surrogate_judge_tol_0.002", **j}) + "\n")
    assert j["served"] > 0.05, j
    assert j["y_err_max"] <= 0.05, j
    assert j["t_err_p99"] <= 0.01, j


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


def test_surrogate_tiny_tolerance_follows_the_exact_fp32_run(trained):
    """With a serve tolerance of 1e-6 the surrogate path leaves nearly every
    cell to the exact routine and so follows the exact FP32 run (same tree;
    density L1 <= 1e-6 from the few cells whose predicted change is below
    1e-6)."""
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config("snr_small")
    p.precision = 32
    out = {}
    for tol in (None, 1e-6):
        s = Simulation(p, ic)
        if tol is not None:
            s.ctx.set_surrogate(trained)
            s.ctx.set_surrogate_tol(tol)
        s.run(30)
        ids = np.nonzero(s.tree()[1])[0]
        out[tol] = (ids, s.ctx.get_blocks(ids)[:, 0, 2:18, 2:18])
        s.close()
    assert np.array_equal(out[None][0], out[1e-6][0])
    a, b = out[None][1], out[1e-6][1]
    l1 = float(np.abs(b - a).sum() / np.abs(a).sum())
    print("remnant density L1, tolerance 1e-6 against the exact FP32 run:", l1)
    assert l1 <= 1e-6, l1


def test_surrogate_gain_over_exact_cooling(trained):
    """What the trained network gains: the same FP32 ensemble step with and
    without it (the cooling kernels' device time: the network, the exact
    routine on the cells it leaves and the statistics pass, against the
    exact routine with the statistics in one kernel), and the share it
    serves.  Since the exact coolingh routine evaluates its powers through
    one shared logarithm and takes one cell per thread, it costs about what
    the network alone does, and the network's path, which adds the fallback
    and a separate statistics pass, is the slower one (measured 0.79x on
    this workload).  The gain is recorded (W2D_PARITY_LOG) and held above
    0.5 as a regression bound; the network must serve most cells."""
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
    from parity_log import record_value
    record_value("surrogate_gain_over_exact_cooling", gain=gain, served=sv / (sv + ex),
                 exact_ms=t[False], surrogate_ms=t[True])
    assert sv / (sv + ex) > 0.5
    assert gain > 0.5, gain


def test_dmc_surrogate_in_fp32_blast_against_fp64_oracle(oracle_lib):
    """The coolingdmc mode: samples labelled with the DMC table; the FP32
    64x64 blast with DMC cooling and the network against the FP64 oracle
    (density L1 <= 1e-3), the exact FP32 path beside it."""
    import os
    from walicxe2d_b200.api import Simulation, Surrogate
    from walicxe2d_b200.params import COOLINGDMC, config, scalings
    rows = np.loadtxt(os.path.join(os.path.dirname(__file__), "golden", "coolingDMC.tab"))
    p, ic = config("sedov64")
    p.cooling = COOLINGDMC
    sc = scalings(3.0e17, p.xmax, p.cv)
    p.tempsc, p.psc, p.tsc, p.rsc = sc["tempsc"], sc["psc"], sc["tsc"], sc["rsc"]
    nn = Surrogate(3)
    nn.samples_dmc(4_000_000, rows[:, 0], rows[:, 1], p, seed=11)
    assert nn.L.w2d_nn_kind(nn.h) == 2
    nn.train(60, batch=8192, lr=2e-3, lr_end=2e-5)
    o = oracle_lib.Oracle(p, ic, threads=8)
    o.set_cooltab(rows[:, 0], rows[:, 1])
    o.startup()
    l1 = {}
    for use in (False, True):
        p32 = p.copy()
        p32.precision = 32
        s = Simulation(p32, ic)
        s.set_cooltab(rows[:, 0], rows[:, 1])
        if use:
            s.ctx.set_surrogate(nn)
        s.run(60)
        if use:
            served, exact = s.ctx.surrogate_counts()
            assert served > 0, (served, exact)
        ids = np.nonzero(s.tree()[1])[0]
        l1[use] = s.ctx.get_blocks(ids)[:, 0, 2:18, 2:18]
    o.run(60, amr=False)
    ids = o.leaves()
    ro = o.u[ids, 0, 2:18, 2:18]
    e = {k: float(np.abs(v - ro).sum() / np.abs(ro).sum()) for k, v in l1.items()}
    print("DMC blast density L1: FP32", e[False], "FP32 + network", e[True])
    assert e[True] <= 1e-3, e


def test_dmc_surrogate_keeps_the_jet():
    """The jet with coolingdmc through the network: boundaryI's impose_jet
    on the interiors still precedes cooling.  With a serve tolerance of 1e-6
    (nearly every cooling cell takes the exact routine) the run equals the
    exact FP32 run to rounding; with the default tolerance it runs on and
    the network serves cells."""
    import os
    from walicxe2d_b200.api import Simulation, Surrogate
    from walicxe2d_b200.params import config
    rows = np.loadtxt(os.path.join(os.path.dirname(__file__), "golden", "coolingDMC.tab"))
    p, ic = config("jet_small_dmc")
    nn = Surrogate(4)
    nn.samples_dmc(1_000_000, rows[:, 0], rows[:, 1], p, seed=13)
    nn.train(20, batch=8192, lr=2e-3, lr_end=2e-5)
    rho, served = {}, {}
    for tol in (None, 1e-6, 0.01):
        p32 = p.copy()
        p32.precision = 32
        s = Simulation(p32, ic)
        s.set_cooltab(rows[:, 0], rows[:, 1])
        if tol is not None:
            s.ctx.set_surrogate(nn)
            s.ctx.set_surrogate_tol(tol)
        s.run(60)
        if tol is not None:
            served[tol] = s.ctx.surrogate_counts()
        lf = s.tree()[1]
        ids = np.nonzero(lf)[0]
        rho[tol] = (ids, s.ctx.get_blocks(ids)[:, 0, 2:18, 2:18])
        s.close()

    def l1(a, b):
        assert np.array_equal(a[0], b[0]), "different trees"
        return float(np.abs(b[1] - a[1]).sum() / np.abs(a[1]).sum())

    e_tight, e_def = l1(rho[None], rho[1e-6]), l1(rho[None], rho[0.01])
    print("jet DMC density L1 against the exact FP32 run: tol 1e-6", e_tight, "tol 0.01", e_def,
          "served/exact", served)
    assert e_tight <= 1e-6, e_tight
    assert served[0.01][0] > 0, served


def test_surrogate_refuses_the_wrong_cooling(trained):
    from walicxe2d_b200.api import Simulation
    from walicxe2d_b200.params import config
    p, ic = config("jet_small_dmc")
    p.precision = 32
    s = Simulation(p, ic)
    with pytest.raises(Exception):
        s.ctx.set_surrogate(trained)      # a coolingh network on a coolingdmc run
