"""Three-phase FP64 step on the GPU against the reference and the oracle
(normwise relative error of every state field at most 1e-12)."""
import numpy as np
import pytest

from conftest import GOLDEN_3PH, interior, load_golden, rel_err
from capaz_b200 import Simulation, native
from capaz_b200.simulation import default_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12
STATE = ["P_w", "S_w", "S_n", "P_n", "P_g"]
DERIVED = ["S_g", "ro_w", "ro_n", "ro_g", "Xi_w", "Xi_n", "Xi_g", "ux_w", "uy_w", "uz_w", "ux_n", "uy_n", "uz_n",
           "ux_g", "uy_g", "uz_g", "roS_w", "roS_n", "roS_g", "roS_w_old", "roS_n_old", "roS_g_old"]


def run3(p, state, m, nsteps, K=None, derived=(), diag=False):
    q = p.copy()
    if diag:
        q.flags |= native.FLAG_DIAGNOSTICS
    with Simulation(q) as s:
        s.set_field("m", m)
        if K is not None:
            s.set_field("K", K)
        for k in STATE:
            s.set_field(k, state[k])
        s.step(nsteps)
        out = {k: s.get_field(k) for k in STATE}
        out["derived"] = {f: s.get_field(f) for f in derived}
        if diag:
            out["diag"] = s.diag()
    return out


def params3(**kw):
    base = dict(phases=3, newton_iterations=7, lambda_=2.0, S_wr=0.1, S_nr=0.05, S_gr=0.02, ro0_w=1000.0,
                ro0_n=850.0, ro0_g=1.2, mu_w=1e-3, mu_n=3e-3, mu_g=1.8e-5, beta_w=1e-9, beta_n=1e-9,
                beta_g=9.2e-6, S_w_gr=0.25, S_n_gr=0.7, S_w_init=0.2, S_n_init=0.3, source=1, porosity=0.3,
                K0=1e-12, hx=1.0, hy=1.0, hz=1.0, dt=0.01, g_const=9.81, P_d=0.0)
    base.update(kw)
    return default_params(**base)


def random_state3(p, seed):
    rng = np.random.default_rng(seed)
    m = np.clip(0.3 + 0.03 * rng.standard_normal((p.nz, p.ny, p.nx)), 0.15, 0.45)
    st = O.init(p, m)
    st["S_w"] = np.clip(0.3 + 0.1 * rng.standard_normal(st["S_w"].shape), 0.12, 0.6)
    st["S_n"] = np.clip(0.3 + 0.1 * rng.standard_normal(st["S_n"].shape), 0.07, 0.35)
    return {k: st[k] for k in STATE}, m


@pytest.mark.parametrize("name", GOLDEN_3PH)
def test_gpu3_matches_reference_golden(name):
    p, g = load_golden(name)
    if "in_P_w" in g:
        state, m = {k: g["in_" + k] for k in STATE}, g["in_m"]
    else:
        st = O.init(p)
        state, m = {k: st[k] for k in STATE}, st["m"]
    out = run3(p, state, m, int(g["nsteps"]), derived=DERIVED)
    for k in STATE:
        assert rel_err(out[k], g["out_" + k]) <= TOL, k
    for f in DERIVED:
        a, b = out["derived"][f], g["der_" + f]
        if f.startswith("roS"):
            a, b = interior(a), interior(b)
        assert rel_err(a, b) <= TOL, f


@pytest.mark.parametrize("shape,nsteps,seed", [((45, 21, 19), 10, 1), ((70, 13, 1), 15, 2), ((1, 40, 1), 30, 3),
                                               ((3, 3, 3), 5, 4)])
def test_gpu3_matches_oracle_random(shape, nsteps, seed):
    nx, ny, nz = shape
    p = params3(nx=nx, ny=ny, nz=nz, dt=0.002)
    state, m = random_state3(p, seed)
    ref = O.step(p, state, nsteps, m)
    out = run3(p, state, m, nsteps)
    for k in STATE:
        assert rel_err(out[k], ref[k]) <= TOL, k


def test_gpu3_percell_k_window_source_and_diag():
    p = params3(nx=40, ny=18, nz=22, dt=0.002, source=1)
    p.flags = native.FLAG_PERCELL_K | native.FLAG_SOURCE_WINDOW
    state, m = random_state3(p, 9)
    rng = np.random.default_rng(9)
    K = np.exp(np.log(1e-12) + 0.5 * rng.standard_normal(m.shape))
    ref = O.step(p, state, 8, m, K, diag=True)
    out = run3(p, state, m, 8, K=K, diag=True)
    for k in STATE:
        assert rel_err(out[k], ref[k]) <= TOL, k
    for i in range(3):
        assert abs(out["diag"]["mass"][i] - ref["diag"]["mass"][i]) <= 1e-12 * abs(ref["diag"]["mass"][i])


def test_gpu3_config2_workload_shape():
    """The config-2 setup (per-cell K and porosity fields, 3x3 NAPL window,
    the workload's stable dt) on a reduced grid, 30 steps from
    capaz_init_state's state, against the oracle."""
    from capaz_b200.configs import config2
    w = config2(grid=(40, 40, 20))
    p = w.params
    st = O.init(p, w.m)
    state = {k: st[k] for k in STATE}
    ref = O.step(p, state, 30, w.m, w.K)
    with Simulation(p) as s:
        s.set_field("m", w.m)
        s.set_field("K", w.K)
        s.init_state()
        for k in STATE:
            assert np.array_equal(s.get_field(k), st[k]), k
        s.step(30)
        out = {k: s.get_field(k) for k in STATE}
    for k in STATE:
        assert rel_err(out[k], ref[k]) <= TOL, k
