"""Three-phase precision form (FP32 storage and stencil, Kahan-summed flux
divergence, FP64 Newton) against the plain FP64 three-phase step, which
matches the reference CPU step to 1e-12.

Bar: relative L2 error of P_w, S_w and S_n at most 1e-6 after the steps (the
precision form's state is rounded to FP32 deviations once per step);
boundary values, the decoded state and the derived fields follow the FP64
step within the same bound."""
import numpy as np
import pytest

from capaz_b200 import Simulation, native
from capaz_b200.configs import heterogeneous_fields, stable_dt, three_phase_params

pytestmark = pytest.mark.gpu
TOL = 1e-6
STATE = ["P_w", "S_w", "S_n", "P_n", "P_g"]


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run(p, form, m, K, nsteps, state=None, derived=(), diag=False):
    q = p.copy()
    q.form = form
    if diag:
        q.flags |= native.FLAG_DIAGNOSTICS
    with Simulation(q) as s:
        s.set_field("m", m)
        s.set_field("K", K)
        if state is None:
            s.init_state()
        else:
            for k in STATE:
                s.set_field(k, state[k])
        s.step(nsteps)
        out = {k: s.get_field(k) for k in STATE}
        out["derived"] = {f: s.get_field(f) for f in derived}
        if diag:
            out["diag"] = s.diag()
    return out


def case(shape, seed):
    nx, ny, nz = shape
    p = three_phase_params(nx, ny, nz)
    m, K = heterogeneous_fields((nz, ny, nx), 1.0, 8.0, seed)
    p.dt = stable_dt(p, m, K)
    return p, m, K


@pytest.mark.parametrize("shape,nsteps,no_tma", [
    ((48, 24, 40), 300, False),  # TMA-staged sweep (nx a multiple of 4)
    ((48, 24, 40), 300, True),   # the plain-load sweep on the same grid
    ((44, 37, 19), 200, False),  # TMA, ragged tiles in x and y (the bottom row inside a tile)
    ((32, 20, 1), 300, False),   # TMA, planar
    ((33, 20, 1), 300, False),   # plain-load sweep (nx not a multiple of 4), planar
    ((1, 40, 1), 300, False),    # column
])
def test_fp32c3_tracks_fp64(shape, nsteps, no_tma):
    """Config-2 physics (3x3 top NAPL source, lognormal K) from the
    reference's initial state; planar and column grids as well."""
    p, m, K = case(shape, sum(shape))
    if no_tma:
        p.flags |= native.FLAG_NO_TMA
    ref = run(p, native.FORM_FP64, m, K, nsteps)
    got = run(p, native.FORM_FP32C, m, K, nsteps)
    for k in ("P_w", "S_w", "S_n"):
        assert np.isfinite(got[k]).all(), k
        assert rel_l2(got[k], ref[k]) <= TOL, (k, rel_l2(got[k], ref[k]))
    for k in ("P_n", "P_g"):
        assert rel_l2(got[k], ref[k]) <= TOL, (k, rel_l2(got[k], ref[k]))


def test_fp32c3_random_state_derived_and_diagnostics():
    p, m, K = case((24, 16, 20), 7)
    rng = np.random.default_rng(7)
    with Simulation(p) as s:
        s.set_field("m", m)
        s.set_field("K", K)
        s.init_state()
        state = {k: s.get_field(k) for k in STATE}
    state["S_w"] = np.clip(0.3 + 0.05 * rng.standard_normal(state["S_w"].shape), 0.15, 0.5)
    state["S_n"] = np.clip(0.3 + 0.05 * rng.standard_normal(state["S_n"].shape), 0.1, 0.4)
    der = ["S_g", "ro_w", "ro_g", "Xi_n", "uy_w", "roS_w", "roS_g_old"]
    ref = run(p, native.FORM_FP64, m, K, 50, state, der, diag=True)
    got = run(p, native.FORM_FP32C, m, K, 50, state, der, diag=True)
    for k in ("P_w", "S_w", "S_n"):
        assert rel_l2(got[k], ref[k]) <= TOL, (k, rel_l2(got[k], ref[k]))
    for f in der:
        assert rel_l2(got["derived"][f], ref["derived"][f]) <= 1e-5, f
    for q in range(3):
        a, b = got["diag"]["mass"][q], ref["diag"]["mass"][q]
        assert abs(a - b) <= 1e-6 * abs(b), q
    assert got["diag"]["nonfinite_cells"] == 0
