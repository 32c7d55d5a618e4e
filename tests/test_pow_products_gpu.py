"""CAPAZ_FLAG_POW_PRODUCTS: the FP64 forms with lambda == 2 take the relative
permeabilities as products and square roots instead of pow (two-phase.cpp:
10-13, three-phase.cpp:146-186 with A = 2).  Each value moves by a few ulps;
the bar is unchanged: P and S within 1e-12 (normwise relative) of the
reference's fixtures and of the oracle after N steps."""
import numpy as np
import pytest

from conftest import load_golden, rel_err
from capaz_b200 import Simulation, native
from capaz_b200.configs import config0, config2
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


def _run(p, state, m, nsteps, K=None):
    q = p.copy()
    q.flags |= native.FLAG_POW_PRODUCTS
    with Simulation(q) as s:
        s.set_field("m", m)
        if K is not None:
            s.set_field("K", K)
        for k, v in state.items():
            s.set_field(k, v)
        s.step(nsteps)
        return {k: s.get_field(k) for k in state}


@pytest.mark.parametrize("name", ["g2_3d_pd0_12x10x7", "g2_planar_17x13x1", "g2_min_3x3x3"])
def test_two_phase_golden(name):
    p, g = load_golden(name)
    assert p.lambda_ == 2.0
    if "in_P_w" in g:
        state, m = {"P_w": g["in_P_w"], "S_n": g["in_S_n"]}, g["in_m"]
    else:
        st = O.init(p)
        state, m = {"P_w": st["P_w"], "S_n": st["S_n"]}, st["m"]
    out = _run(p, state, m, int(g["nsteps"]))
    for k in ("P_w", "S_n"):
        assert rel_err(out[k], g["out_" + k]) <= TOL, k


def test_three_phase_golden():
    p, g = load_golden("g3_3d_9x8x6")
    assert p.lambda_ == 2.0
    keys = ("P_w", "S_w", "S_n", "P_n", "P_g")
    out = _run(p, {k: g["in_" + k] for k in keys}, g["in_m"], int(g["nsteps"]))
    for k in keys:
        assert rel_err(out[k], g["out_" + k]) <= TOL, k


def test_config0_as_defined():
    w = config0()
    p = w.params
    st = O.init(p, w.m)
    ref = O.step(p, {"P_w": st["P_w"], "S_n": st["S_n"]}, w.steps, w.m)
    out = _run(p, {"P_w": st["P_w"], "S_n": st["S_n"]}, w.m, w.steps)
    for k in ("P_w", "S_n"):
        assert rel_err(out[k], ref[k]) <= TOL, k


def test_config2_grid_three_steps():
    w = config2()
    p = w.params
    keys = ("P_w", "S_w", "S_n", "P_n", "P_g")
    st = O.init(p, w.m)
    ref = O.step(p, {k: st[k] for k in keys}, 3, w.m, w.K)
    out = _run(p, {k: st[k] for k in keys}, w.m, 3, w.K)
    for k in keys:
        assert rel_err(out[k], ref[k]) <= TOL, k
