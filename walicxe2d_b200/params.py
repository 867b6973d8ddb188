"""Runtime parameters of the block update (ctypes mirror of ``include/w2d.h``).

The reference fixes all of these at compile time (``src/parameters.f90`` and
the ``-D`` flags of ``JET/Makefile:27-62``); here they are fields of
``W2dParams`` so one build serves every configuration.  ``W2dInit`` selects
the initial conditions of the whole-run driver.
"""
from __future__ import annotations

import ctypes as C
import math

# method selectors (JET/Makefile:27-62)
HLLC, HLL, HLL_HLLC = 0, 1, 2
ADIABATIC, COOLINGH, COOLINGDMC = 0, 1, 2
BC_OUTFLOW, BC_REFLECTIVE = 0, 1
USERBC_NONE, USERBC_JET = 0, 1
GEOM_CARTESIAN, GEOM_CYLINDRICAL = 0, 1   # JET/Makefile:39 CYLINDRICAL
COMPAT_HLLC_STAR = 1   # src/hllcfluxes.f90:157
COMPAT_OUTFYB = 2      # src/boundaryI.f90:87
IC_SEDOV, IC_SNR, IC_JET = 0, 1, 2

# physical constants of src/parameters.f90:28-34 (cgs)
PC = 3.0857e18
AU = 1.496e13
MSUN = 1.99e33
AMH = 1.66e-24
KB = 1.38e-16
RG = 8.3145e7
YR = 3.156e7


class W2dParams(C.Structure):
    _fields_ = [
        ("neq", C.c_int32), ("npas", C.c_int32), ("nx", C.c_int32), ("ny", C.c_int32),
        ("nlevs", C.c_int32), ("nbroot_x", C.c_int32), ("nbroot_y", C.c_int32),
        ("nblocks", C.c_int32), ("solver", C.c_int32), ("limiter", C.c_int32),
        ("cooling", C.c_int32), ("bc_left", C.c_int32), ("bc_right", C.c_int32),
        ("bc_bottom", C.c_int32), ("bc_top", C.c_int32), ("otherb", C.c_int32),
        ("compat", C.c_int32), ("precision", C.c_int32), ("geometry", C.c_int32),
        ("cv", C.c_double), ("gamma", C.c_double), ("cfl", C.c_double), ("eta", C.c_double),
        ("xmax", C.c_double), ("ymax", C.c_double),
        ("tempsc", C.c_double), ("psc", C.c_double), ("tsc", C.c_double), ("rsc", C.c_double),
        ("tol", C.c_double), ("tol2", C.c_double),
        ("jet_rj", C.c_double), ("jet_lj", C.c_double), ("jet_posx", C.c_double),
        ("jet_posy", C.c_double), ("jet_den", C.c_double), ("jet_temp", C.c_double),
        ("jet_v0", C.c_double), ("jet_dv", C.c_double), ("jet_tau", C.c_double),
    ]

    def copy(self) -> "W2dParams":
        q = W2dParams()
        C.pointer(q)[0] = self
        return q

    def as_dict(self) -> dict:
        return {f[0]: getattr(self, f[0]) for f in self._fields_ if f[0] != "pad_"}


class W2dInit(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("init_levels", C.c_int32), ("startup_admesh", C.c_int32),
        ("pad_", C.c_int32),
        ("rho0", C.c_double), ("p0", C.c_double), ("e_dep", C.c_double),
        ("xc", C.c_double), ("yc", C.c_double), ("rb", C.c_double), ("xh0", C.c_double),
        ("extra", C.c_double * 8),
    ]


class W2dError(C.Structure):
    _fields_ = [("code", C.c_int32), ("block", C.c_int32), ("i", C.c_int32),
                ("j", C.c_int32), ("message", C.c_char * 240)]


def scalings(xphys: float, xmax: float, cv: float = 1.5, t0: float = 1.0e4,
             amol: float = 0.6) -> dict:
    """Scaling factors of src/parameters.f90:39-54, evaluated left to right."""
    gamma = (cv + 1.0) / cv
    rsc = xphys / xmax
    tempsc = t0 * gamma
    psc = gamma * AMH * RG * t0
    vsc2 = gamma * t0 * RG / amol
    tsc = rsc / math.sqrt(vsc2)
    return dict(gamma=gamma, rsc=rsc, rhosc=AMH * amol, tempsc=tempsc, psc=psc,
                vsc2=vsc2, tsc=tsc)


def base_params(**kw) -> W2dParams:
    """Defaults of src/parameters.f90 with the serial build's flag set."""
    p = W2dParams()
    p.neq, p.npas, p.nx, p.ny = 4, 0, 16, 16
    p.nlevs, p.nbroot_x, p.nbroot_y, p.nblocks = 1, 4, 4, 64
    p.solver, p.limiter, p.cooling = HLLC, 1, ADIABATIC
    p.bc_left = p.bc_right = p.bc_bottom = p.bc_top = BC_OUTFLOW
    p.otherb = USERBC_NONE
    p.compat = COMPAT_HLLC_STAR | COMPAT_OUTFYB
    p.precision = 64
    p.geometry = GEOM_CARTESIAN
    p.cv = 1.5
    sc = scalings(3.0e17, 1.0, p.cv)
    p.gamma = sc["gamma"]
    p.cfl, p.eta = 0.4, 0.001
    p.xmax, p.ymax = 1.0, 1.0
    p.tempsc, p.psc, p.tsc, p.rsc = sc["tempsc"], sc["psc"], sc["tsc"], sc["rsc"]
    p.tol, p.tol2 = 0.05, 1.0          # src/criteria.f90:11
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def sedov(nbroot: int = 4, nlevs: int = 1, tol: float = 0.1, nblocks: int | None = None,
          rb_cells: float = 3.0, e0: float = 1.0, p0: float = 1.0e-5, rho0: float = 1.0,
          startup_admesh: int | None = None, **kw):
    """2D Sedov blast: ambient rho0, p0 and energy e0 deposited as a uniform
    energy density in the cells (of the root level) whose centres lie within
    rb_cells root cells of the domain centre.

    nbroot=4, nlevs=1 is the CPU-runnable 4x4-block case; nbroot=8, nlevs=5,
    tol=0.1 is the AMR case (about 1,500-4,000 leaves once the blast grows).
    """
    if nblocks is None:
        nblocks = nbroot * nbroot if nlevs == 1 else 40000
    p = base_params(nlevs=nlevs, nbroot_x=nbroot, nbroot_y=nbroot, nblocks=nblocks,
                    tol=tol, **kw)
    dx1 = p.xmax / p.nx / nbroot
    dy1 = p.ymax / p.ny / nbroot
    # count of root-level cell centres inside the deposit radius (32 for 3 cells)
    n_in = 0
    half = int(rb_cells) + 2
    for a in range(-half, half):
        for b in range(-half, half):
            if (a + 0.5) ** 2 + (b + 0.5) ** 2 < rb_cells ** 2:
                n_in += 1
    ic = W2dInit()
    ic.kind = IC_SEDOV
    ic.init_levels = 1
    ic.startup_admesh = 4 if (startup_admesh is None and nlevs > 1) else (startup_admesh or 0)
    ic.rho0, ic.p0 = rho0, p0
    ic.xc, ic.yc = 0.5 * p.xmax, 0.5 * p.ymax
    ic.rb = rb_cells * dx1
    ic.e_dep = e0 / (n_in * dx1 * dy1)
    ic.xh0 = 0.0
    return p, ic


def jet(nbroot_x: int = 32, nbroot_y: int = 8, nlevs: int = 7, cooling: int = COOLINGDMC,
        nblocks: int | None = None, tol: float = 0.1, rj_cm: float = 1.0e15, **kw):
    """Planar variable-velocity jet (the reference's OTHERB set-up with
    impose_jet, src/jet.f90): box 4e17 x 1e17 cm (xmax 1, ymax 0.25), ambient
    1 cm^-3 at 1e3 K, jet 100 cm^-3 at 1e3 K of radius rj_cm entering at
    x = 0, mid-height, with v = 200 (1 + 0.25 sin(2 pi t / 20 yr)) km/s;
    reflective left wall, outflow elsewhere; neq = 6 (neutral density and a
    tracer, as the jet state writes both)."""
    if nblocks is None:
        nblocks = 200000 if nlevs >= 6 else 20000
    p = base_params(neq=6, npas=2, nlevs=nlevs, nbroot_x=nbroot_x, nbroot_y=nbroot_y,
                    nblocks=nblocks, cooling=cooling, otherb=USERBC_JET, tol=tol, **kw)
    p.xmax, p.ymax = 1.0, 0.25
    p.bc_left = BC_REFLECTIVE
    sc = scalings(4.0e17, p.xmax, p.cv)
    p.tempsc, p.psc, p.tsc, p.rsc = sc["tempsc"], sc["psc"], sc["tsc"], sc["rsc"]
    vsc = math.sqrt(sc["vsc2"])
    p.jet_rj = rj_cm / sc["rsc"]
    p.jet_lj = rj_cm / sc["rsc"]
    p.jet_posx, p.jet_posy = 0.0, 0.5 * p.ymax
    p.jet_den = 100.0
    p.jet_temp = 1.0e3 / sc["tempsc"]
    p.jet_v0 = 200.0e5 / vsc
    p.jet_dv = 50.0e5 / vsc
    p.jet_tau = 20.0 * YR / sc["tsc"]
    ic = W2dInit()
    ic.kind = IC_JET
    ic.init_levels = 1
    ic.startup_admesh = min(nlevs - 1, 6) if nlevs > 1 else 0
    ic.rho0, ic.p0 = 1.0, 1.0e3      # ambient n and T (initial_conditions)
    return p, ic


def jet_cyl(nlevs: int = 7, nbroot_x: int = 4, nbroot_y: int = 1, cooling: int = COOLINGDMC,
            nblocks: int | None = None, rj_cm: float = 1.0e15, **kw):
    """The reference's shipped jet set-up in cylindrical coordinates
    (JET/Makefile:27-62, src/parameters.f90, src/jet.f90:16-33,
    src/user_mod.f90:39-62): x -> z, y -> r; box 3e17 x 0.75e17 cm (xmax 1,
    ymax 0.25) of 4 x 1 roots; HLLC, limiter 2, cfl 0.7, DMC cooling,
    passives (neutral density, tracer); reflective left wall and axis,
    outflow right and top; ambient 15 cm^-3 at 1e3 K; the jet, 5000 cm^-3 at
    1e3 K with radius and length rj_cm, on the axis at z = 0 with
    v = 250 + 30 sin(2 pi t / 30 yr) km/s."""
    p, ic = jet(nbroot_x=nbroot_x, nbroot_y=nbroot_y, nlevs=nlevs, cooling=cooling, nblocks=nblocks,
                rj_cm=rj_cm, **kw)
    p.geometry = GEOM_CYLINDRICAL
    p.limiter = 2
    p.cfl = 0.7
    p.bc_left = p.bc_bottom = BC_REFLECTIVE
    p.bc_right = p.bc_top = BC_OUTFLOW
    sc = scalings(3.0e17, p.xmax, p.cv)
    p.tempsc, p.psc, p.tsc, p.rsc = sc["tempsc"], sc["psc"], sc["tsc"], sc["rsc"]
    vsc = math.sqrt(sc["vsc2"])
    p.jet_rj = rj_cm / sc["rsc"]
    p.jet_lj = rj_cm / sc["rsc"]
    p.jet_posx, p.jet_posy = 0.0, 0.0
    p.jet_den = 5000.0
    p.jet_temp = 1.0e3 / sc["tempsc"]
    p.jet_v0 = 250.0e5 / vsc
    p.jet_dv = 30.0e5 / vsc
    p.jet_tau = 30.0 * YR / sc["tsc"]
    ic.rho0, ic.p0 = 15.0, 1.0e3
    # the jet (1e15 cm) is narrower than a root cell: start from the finest
    # level everywhere (the reference's basegrid forces refinement along the
    # axis, src/basegrid.f90:113-160) and let the four startup admesh passes
    # of src/main.f90:59-62 coarsen the rest
    ic.init_levels = nlevs
    ic.startup_admesh = 4 if nlevs > 1 else 0
    return p, ic


def snr(nbroot: int = 10, nlevs: int = 6, n_amb: float = 1.0, t_amb: float = 1.0e4, xh: float = 0.9,
        e_sn: float = 1.0e51, m_sn: float = 4.0 * MSUN, r_sn: float = 1.0 * PC, chi: float = 0.5,
        size_pc: float = 40.0, nblocks: int | None = None, tol: float = 0.1, precision: int = 64, **kw):
    """Supernova remnant with coolingh (src/sn.f90 parameterized): a
    size_pc x size_pc box of nbroot x nbroot roots, ambient n_amb cm^-3 at
    t_amb K with neutral fraction xh, and impose_sn at the centre: ejecta of
    mass m_sn (g) spread over radius r_sn (cm) with density (3/4pi) M/R^3 *
    1.3/2.1, linear velocity profile holding a fraction chi of e_sn (erg) as
    kinetic energy and the rest as uniform thermal energy.  m_sn = 0 (with
    chi = 0) leaves the ambient density and deposits e_sn as heat only: a
    Sedov blast in physical units.  neq = 6 (neutral density, tracer)."""
    if nblocks is None:
        nblocks = 200000
    p = base_params(neq=6, npas=2, nlevs=nlevs, nbroot_x=nbroot, nbroot_y=nbroot, nblocks=nblocks,
                    cooling=COOLINGH, tol=tol, precision=precision, **kw)
    sc = scalings(size_pc * PC, p.xmax, p.cv)
    p.tempsc, p.psc, p.tsc, p.rsc = sc["tempsc"], sc["psc"], sc["tsc"], sc["rsc"]
    ic = W2dInit()
    ic.kind = IC_SNR
    ic.init_levels = 1
    ic.startup_admesh = nlevs - 1 if nlevs > 1 else 0
    ic.rho0 = n_amb
    ic.p0 = (2.0 - xh) * n_amb * t_amb / sc["tempsc"]
    ic.xh0 = xh
    ic.xc = 0.5 * p.xmax * sc["rsc"]
    ic.yc = 0.5 * p.ymax * sc["rsc"]
    ic.rb = r_sn
    pi = math.pi
    r3 = r_sn * r_sn * r_sn
    if m_sn > 0.0:
        dens = 3.0 / 4.0 / pi * m_sn / r3 * 1.3 / 2.1 / sc["rhosc"]
        s1 = math.sqrt(10.0 * chi * e_sn / (3.0 * m_sn))
    else:
        dens, s1 = n_amb, 0.0
    ic.e_dep = 3.0 / 4.0 / pi * e_sn * (1.0 - chi) / r3 / sc["psc"]
    dxn = p.xmax / p.nx / (2.0 ** (nlevs - 1)) / nbroot
    for k, v in enumerate([dens, s1, math.sqrt(sc["vsc2"]), sc["rsc"], 0.1 * dxn * sc["rsc"]]):
        ic.extra[k] = v
    return p, ic


def ensemble_members(count: int = 256, seed: int = 20261203, precision: int = 32, size_pc: float = 40.0):
    """Independent Sedov-with-coolingh runs of uneven size, run r drawn with
    seed + r: roots k x k with k uniform in 2..16, levels uniform in 3..6,
    ambient n log-uniform in [0.1, 10] cm^-3, E log-uniform in [1e50, 1e51]
    erg deposited as heat within 1 pc; T = 1e4 K, neutral fraction 0.9."""
    import numpy as np
    out = []
    for r in range(count):
        g = np.random.default_rng(seed + r)
        k = int(g.integers(2, 17))
        nl = int(g.integers(3, 7))
        n = float(10.0 ** g.uniform(-1.0, 1.0))
        e = float(10.0 ** g.uniform(50.0, 51.0))
        cap = max(4 * k * k * (1 << (2 * (nl - 1))) // 6, 4 * k * k + 64)
        out.append(snr(nbroot=k, nlevs=nl, n_amb=n, e_sn=e, m_sn=0.0, chi=0.0, size_pc=size_pc,
                       nblocks=min(cap, 40000), precision=precision))
    return out


def config(name: str):
    """Named workloads: 'sedov64' (4x4 roots, no AMR), 'sedov_amr' (8x8
    roots, 5 levels, tol 0.1) and small test variants."""
    if name == "sedov64":
        return sedov(nbroot=4, nlevs=1)
    if name == "sedov_amr":
        return sedov(nbroot=8, nlevs=5, tol=0.1)
    if name == "sedov_amr_small":
        return sedov(nbroot=4, nlevs=3, tol=0.1, nblocks=4000)
    if name == "jet_small":
        return jet(nbroot_x=8, nbroot_y=2, nlevs=3, cooling=ADIABATIC, nblocks=4000, rj_cm=8.0e15)
    if name == "jet_small_dmc":
        return jet(nbroot_x=8, nbroot_y=2, nlevs=3, cooling=COOLINGDMC, nblocks=4000, rj_cm=8.0e15)
    if name == "jet_dmc":
        return jet()
    if name == "jet_cyl":
        return jet_cyl()
    if name == "jet_cyl_small":
        return jet_cyl(nlevs=5, nblocks=4000)
    if name == "sedov_cyl_small":
        p, ic = sedov(nbroot=4, nlevs=3, tol=0.1, nblocks=4000)
        p.geometry = GEOM_CYLINDRICAL
        p.bc_bottom = BC_REFLECTIVE
        return p, ic
    if name == "snr":
        return snr()
    if name == "snr_small":
        return snr(nbroot=4, nlevs=3, nblocks=4000, size_pc=10.0)
    raise KeyError(name)
