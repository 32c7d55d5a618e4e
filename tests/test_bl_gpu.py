"""Buckley-Leverett task (the reference's B_L build) on the GPU against the
reference's golden vectors and the oracle.

Bar: normwise relative error max|gpu - ref| / max|ref| of P_w and S_n (and
every derived field) at most 1e-12 after N steps, as for the two-phase FP64
step: the kernels keep the reference's operation order without FMA
contraction; CUDA's pow (in the production well's relative permeability)
may round differently from the host libm's.
"""
import numpy as np
import pytest

from conftest import GOLDEN_BL, interior, load_golden, rel_err
from capaz_b200 import Simulation, native
from capaz_b200.simulation import buckley_leverett_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12

DERIVED = ["S_w", "P_n", "ro_w", "ro_n", "Xi_w", "Xi_n", "ux_w", "uy_w", "uz_w", "ux_n", "uy_n", "uz_n",
           "roS_w", "roS_n", "roS_w_old", "roS_n_old"]


def _percell(p):
    q = p.copy()
    q.flags |= native.FLAG_PERCELL_K
    return q


@pytest.mark.parametrize("name", GOLDEN_BL)
def test_gpu_bl_matches_reference_golden(name):
    """data_initialization on the context, then N steps, against the
    reference's B_L program run on the same K."""
    p, g = load_golden(name)
    q = _percell(p)
    nsteps = int(g["nsteps"])
    with Simulation(q) as s:
        s.set_field("K", g["K"])
        s.init_state()
        l0 = s.launch_count
        s.step(nsteps)
        assert s.launch_count - l0 == 2 * nsteps  # interior update + boundary/wells
        out = {k: s.get_field(k) for k in ("P_w", "S_n")}
    for k in ("P_w", "S_n"):
        assert rel_err(out[k], g["out_" + k]) <= TOL, k


@pytest.mark.parametrize("name", GOLDEN_BL)
def test_gpu_bl_derived_fields_match_oracle(name):
    p, g = load_golden(name)
    q = _percell(p)
    nsteps = int(g["nsteps"])
    st = O.init(q)
    want = O.step(q, {"P_w": st["P_w"], "S_n": st["S_n"]}, nsteps, st["m"], g["K"], derived=True)
    with Simulation(q) as s:
        s.set_field("K", g["K"])
        s.init_state()
        s.step(nsteps)
        got = {f: s.get_field(f) for f in DERIVED}
    for f in DERIVED:
        a, b = got[f], want["derived"][f]
        if f.startswith("roS"):
            a, b = interior(a), interior(b)
        assert rel_err(a, b) <= TOL, f


@pytest.mark.parametrize("shape,g,dt,seed", [
    ((16, 12, 1), 0.0, 500.0, 1),      # planar, the reference's g = 0
    ((9, 7, 5), 9.81, 30.0, 2),        # 3-D with gravity
    ((33, 5, 3), 0.0, 1000.0, 3),      # thin in y: wells two rows apart
])
def test_gpu_bl_random_states_match_oracle(shape, g, dt, seed):
    """Random saturations across every branch of the relative permeability
    (S_w below S_sv, between S_1 and S_zv, above S_zv) and random K."""
    nx, ny, nz = shape
    p = buckley_leverett_params(nx=nx, ny=ny, nz=nz, g_const=g, dt=dt)
    rng = np.random.default_rng(seed)
    K = 6.64e-11 * np.exp(0.5 * rng.standard_normal((nz, ny, nx)))
    st = O.init(p)
    S = rng.choice([0.05, 0.15, 0.25, 0.27, 0.5, 0.75, 0.95], size=st["S_n"].shape)
    S = S + 0.01 * rng.standard_normal(S.shape)
    P = st["P_w"] + 2e3 * rng.standard_normal(S.shape)
    nsteps = 12
    want = O.step(p, {"P_w": P, "S_n": S}, nsteps, st["m"], K)
    with Simulation(p) as s:
        s.set_field("K", K)
        s.set_field("P_w", P)
        s.set_field("S_n", S)
        s.step(nsteps)
        got = {k: s.get_field(k) for k in ("P_w", "S_n")}
    for k in ("P_w", "S_n"):
        assert rel_err(got[k], want[k]) <= TOL, k


def test_gpu_bl_wells_and_boundary_rules():
    """After a step the injection and production blocks hold the wells'
    pressures in every z-plane, and S_n on boundary cells equals its basic
    coordinate's value."""
    p = buckley_leverett_params(nx=10, ny=8, nz=5, g_const=9.81, dt=500.0)
    with Simulation(p) as s:
        s.set_field("K", np.full((p.nz, p.ny, p.nx), p.K0))
        s.init_state()
        s.step(3)
        P, S = s.get_field("P_w"), s.get_field("S_n")
    assert np.all(P[:, 0:2, 0:2] == p.injwell_Pw)
    assert np.all(P[:, -2:, -2:] == p.outwell_Pw)
    assert np.array_equal(S[0], S[1]) and np.array_equal(S[-1], S[-2])
    assert np.array_equal(S[1:-1, 0, 1:-1], S[1:-1, 1, 1:-1])
    assert np.array_equal(S[1:-1, 1:-1, 0], S[1:-1, 1:-1, 1])


def test_gpu_bl_mass_noalloc_matches_oracle():
    """The allocation-free mass balance on a B-L state uses P_n = P_w."""
    import ctypes as C

    import torch
    p = buckley_leverett_params(nx=12, ny=9, nz=4, g_const=9.81, dt=200.0)
    rng = np.random.default_rng(5)
    st = O.init(p)
    S = np.clip(0.6 + 0.1 * rng.standard_normal(st["S_n"].shape), 0.2, 0.9)
    q = p.copy()
    q.flags |= native.FLAG_DIAGNOSTICS
    want = O.step(q, {"P_w": st["P_w"], "S_n": S}, 0, st["m"], np.full(S.shape, p.K0), diag=True)["diag"]
    dev = torch.device("cuda:0")
    Pd, Sd, md = (torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in (st["P_w"], S, st["m"]))
    out = torch.zeros(5, dtype=torch.float64, device=dev)  # mass[3], max residual, non-finite cells
    lib = native.load()
    rc = lib.capaz_mass_noalloc(C.byref(p), Pd.data_ptr(), Sd.data_ptr(), md.data_ptr(), out.data_ptr(), None)
    assert rc == native.OK
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for i in range(2):
        assert abs(got[i] - want["mass"][i]) <= 1e-12 * abs(want["mass"][i])
