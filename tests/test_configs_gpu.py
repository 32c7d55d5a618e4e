"""Parity at the benchmark configurations themselves, against the oracle.

The oracle (oracle/capaz_oracle.cpp) is bit-identical to the reference's own
CPU step (cpu.cpp:52-104 over Two-phase/two-phase.cpp and
Three-phase/three-phase.cpp) on every golden fixture.  Here the GPU runs the
configurations the benchmark measures, from the GPU's own initial state
(data_initialization on the device), and is compared with the oracle from the
oracle's initial state:

* the 64x64x32 two-phase workload exactly as defined (100 steps, i.i.d.
  porosity, uniform K), FP64, bar 1e-12;
* the 256x256x128 two-phase workload (lognormal K) for a few steps, FP64 bar
  1e-12, and the precision form (FP32 storage, FP64 Newton) bar 1e-6 in
  relative L2 of P and S;
* the 192x192x96 three-phase workload (lognormal K, 3x3 NAPL source) for a
  few steps, FP64 bar 1e-12, and its precision form bar 1e-6.

The bar for FP64 is the normwise relative error max|gpu - ref| / max|ref|.
"""
import numpy as np
import pytest

from conftest import rel_err
from capaz_b200 import Simulation, native
from capaz_b200.configs import config0, config1, config2
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL64 = 1e-12
TOL32 = 1e-6


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def gpu_run(p, m, K, nsteps, fields, form=native.FORM_FP64):
    q = p.copy()
    q.form = form
    with Simulation(q) as s:
        s.set_field("m", m)
        if K is not None:
            s.set_field("K", K)
        s.init_state()
        init = {k: s.get_field(k) for k in fields}
        s.step(nsteps)
        out = {k: s.get_field(k) for k in fields}
    return init, out


def test_config0_as_defined_fp64():
    w = config0()
    p = w.params
    assert (p.nx, p.ny, p.nz) == (64, 32, 64) and w.steps == 100 and w.K is None
    st = O.init(p, w.m)
    ref = O.step(p, {"P_w": st["P_w"], "S_n": st["S_n"]}, w.steps, w.m)
    init, out = gpu_run(p, w.m, None, w.steps, ("P_w", "S_n"))
    for k in ("P_w", "S_n"):
        assert np.array_equal(init[k], st[k]), f"initial {k}"
        assert rel_err(out[k], ref[k]) <= TOL64, k
    assert np.mean(out["P_w"] == ref["P_w"]) > 0.5
    # the run moved the state (the comparison is not of an idle grid)
    assert np.abs(ref["S_n"] - st["S_n"]).max() > 1e-6


@pytest.fixture(scope="module")
def cfg1():
    return config1()


@pytest.fixture(scope="module")
def cfg1_ref(cfg1):
    p = cfg1.params
    st = O.init(p, cfg1.m)
    ref = O.step(p, {"P_w": st["P_w"], "S_n": st["S_n"]}, 3, cfg1.m, cfg1.K)
    return st, ref


def test_config1_grid_fp64(cfg1, cfg1_ref):
    st, ref = cfg1_ref
    p = cfg1.params
    assert (p.nx, p.ny, p.nz) == (256, 128, 256)
    init, out = gpu_run(p, cfg1.m, cfg1.K, 3, ("P_w", "S_n"))
    for k in ("P_w", "S_n"):
        assert rel_err(init[k], st[k]) <= TOL64, f"initial {k}"
        assert rel_err(out[k], ref[k]) <= TOL64, k


def test_config1_grid_precision_form(cfg1, cfg1_ref):
    st, ref = cfg1_ref
    _, out = gpu_run(cfg1.params, cfg1.m, cfg1.K, 3, ("P_w", "S_n"), form=native.FORM_FP32C)
    for k in ("P_w", "S_n"):
        assert rel_l2(out[k], ref[k]) <= TOL32, k
    # the three steps' increments are resolved, not rounded away
    dS = np.abs(ref["S_n"] - st["S_n"]).max()
    assert dS > 0 and np.abs(out["S_n"] - ref["S_n"]).max() < 0.05 * dS


STATE3 = ("P_w", "S_w", "S_n", "P_n", "P_g")


@pytest.fixture(scope="module")
def cfg2():
    w = config2()
    p = w.params
    st = O.init(p, w.m)
    ref = O.step(p, {k: st[k] for k in STATE3}, 3, w.m, w.K)
    return w, st, ref


def test_config2_grid_fp64(cfg2):
    w, st, ref = cfg2
    p = w.params
    assert (p.nx, p.ny, p.nz) == (192, 96, 192) and p.phases == 3
    init, out = gpu_run(p, w.m, w.K, 3, STATE3)
    for k in STATE3:
        assert rel_err(init[k], st[k]) <= TOL64, f"initial {k}"
        assert rel_err(out[k], ref[k]) <= TOL64, k


def test_config2_grid_precision_form(cfg2):
    w, st, ref = cfg2
    _, out = gpu_run(w.params, w.m, w.K, 3, ("P_w", "S_w", "S_n"), form=native.FORM_FP32C)
    for k in ("P_w", "S_w", "S_n"):
        assert rel_l2(out[k], ref[k]) <= TOL32, k
