"""Two-phase FP64 step on the GPU against the reference and the oracle.

Bar: the normwise relative error max|gpu - ref| / max|ref| of P_w and S_n
(and every derived field) is at most 1e-12 after N steps.  The FP64 kernels
keep the reference's operation order without FMA contraction, so most cells
match to the last bit; the rest differ where CUDA's pow and the host libm's
pow round differently.
"""
import numpy as np
import pytest

from conftest import GOLDEN_2PH, interior, load_golden, rel_err
from capaz_b200 import Simulation, native
from capaz_b200.simulation import default_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu
TOL = 1e-12


def run_gpu(p, state, m, nsteps, K=None, derived=(), diag=False):
    q = p.copy()
    if diag:
        q.flags |= native.FLAG_DIAGNOSTICS
    with Simulation(q) as s:
        s.set_field("m", m)
        if K is not None:
            s.set_field("K", K)
        for k, v in state.items():
            s.set_field(k, v)
        l0 = s.launch_count
        s.step(nsteps)
        launched = s.launch_count - l0
        out = {k: s.get_field(k) for k in ("P_w", "S_n")}
        out["derived"] = {f: s.get_field(f) for f in derived}
        if diag:
            out["diag"] = s.diag()
        out["launches"] = launched
    return out


def cfg_params(**kw):
    base = dict(hx=1.0, hy=1.0, hz=1.0, mu_w=1e-3, mu_n=5e-3, ro0_w=1000.0, ro0_n=850.0, beta_w=1e-9,
                beta_n=1e-9, lambda_=2.0, S_wr=0.1, P_d=0.0, g_const=9.81, P_atm=1e5, K0=1e-12,
                porosity=0.3, newton_iterations=10, dt=0.02)
    base.update(kw)
    return default_params(**base)


def random_case(p, seed, s_mean=0.5):
    rng = np.random.default_rng(seed)
    m = np.clip(0.3 + 0.03 * rng.standard_normal((p.nz, p.ny, p.nx)), 0.15, 0.45)
    st = O.init(p, m)
    S = np.clip(s_mean + 0.2 * rng.standard_normal(st["S_n"].shape), 0.05, 0.85)
    return {"P_w": st["P_w"], "S_n": S}, m


DERIVED = ["S_w", "P_n", "ro_w", "ro_n", "Xi_w", "Xi_n", "ux_w", "uy_w", "uz_w", "ux_n", "uy_n", "uz_n",
           "roS_w", "roS_n", "roS_w_old", "roS_n_old"]


@pytest.mark.parametrize("name", GOLDEN_2PH)
def test_gpu_matches_reference_golden(name):
    p, g = load_golden(name)
    if "in_P_w" in g:
        state, m = {"P_w": g["in_P_w"], "S_n": g["in_S_n"]}, g["in_m"]
    else:
        st = O.init(p)
        state, m = {"P_w": st["P_w"], "S_n": st["S_n"]}, st["m"]
    out = run_gpu(p, state, m, int(g["nsteps"]), derived=DERIVED)
    for k in ("P_w", "S_n"):
        assert rel_err(out[k], g["out_" + k]) <= TOL, k
    for f in DERIVED:
        a, b = out["derived"][f], g["der_" + f]
        if f.startswith("roS"):
            a, b = interior(a), interior(b)
        assert rel_err(a, b) <= TOL, f


@pytest.mark.parametrize("shape,nsteps,seed", [
    ((67, 35, 29), 20, 1),    # several tiles and z-chunks, ragged edges
    ((130, 70, 1), 30, 2),    # planar
    ((3, 3, 3), 10, 3),       # minimum grid
    ((34, 10, 40), 15, 4),    # exactly one tile wide + 2, many z-chunks
    ((5, 200, 3), 10, 5),     # tall and thin
])
def test_gpu_matches_oracle_random(shape, nsteps, seed):
    nx, ny, nz = shape
    p = cfg_params(nx=nx, ny=ny, nz=nz, source=3, S_n_gr=0.1)
    state, m = random_case(p, seed)
    ref = O.step(p, state, nsteps, m)
    out = run_gpu(p, state, m, nsteps)
    for k in ("P_w", "S_n"):
        assert rel_err(out[k], ref[k]) <= TOL, k
    same = np.mean(out["P_w"] == ref["P_w"])
    assert same > 0.5, f"only {same:.3f} of cells bit-identical"
    assert out["launches"] == nsteps


def test_gpu_capillary_pressure_path():
    """P_d != 0 takes the general pow path of two-phase.cpp:36-40."""
    p = cfg_params(nx=40, ny=24, nz=11, source=2, S_n_gr=0.3, P_d=755.0, lambda_=2.7)
    state, m = random_case(p, 7)
    ref = O.step(p, state, 25, m)
    out = run_gpu(p, state, m, 25)
    for k in ("P_w", "S_n"):
        assert rel_err(out[k], ref[k]) <= TOL, k


def test_gpu_percell_permeability_and_extensions():
    """Per-cell K, top-pressure offset and background saturation (extensions)
    against the oracle, from capaz_init_state's initial state."""
    p = cfg_params(nx=48, ny=20, nz=17, source=48, S_n_gr=0.1, P_top_offset=1e4, S_n_background=0.85)
    p.flags = native.FLAG_PERCELL_K
    rng = np.random.default_rng(11)
    m = np.clip(0.25 + 0.02 * rng.standard_normal((p.nz, p.ny, p.nx)), 0.1, 0.4)
    K = np.exp(np.log(1e-12) + 0.5 * rng.standard_normal(m.shape))
    st = O.init(p, m)
    with Simulation(p) as s:
        s.set_field("m", m)
        s.set_field("K", K)
        s.init_state()
        assert np.array_equal(s.get_field("P_w"), st["P_w"])
        assert np.array_equal(s.get_field("S_n"), st["S_n"])
        s.step(30)
        P, S = s.get_field("P_w"), s.get_field("S_n")
    ref = O.step(p, {"P_w": st["P_w"], "S_n": st["S_n"]}, 30, m, K)
    assert rel_err(P, ref["P_w"]) <= TOL
    assert rel_err(S, ref["S_n"]) <= TOL


def test_gpu_diagnostics_match_oracle():
    p = cfg_params(nx=70, ny=30, nz=21, source=5, S_n_gr=0.1)
    state, m = random_case(p, 13)
    ref = O.step(p, state, 12, m, diag=True)
    out = run_gpu(p, state, m, 12, diag=True)
    d, r = out["diag"], ref["diag"]
    for i in range(2):
        assert abs(d["mass"][i] - r["mass"][i]) <= 1e-12 * abs(r["mass"][i])
    assert d["mass"][2] == 0.0
    assert abs(d["max_residual"] - r["max_residual"]) <= 1e-9 * max(r["max_residual"], 1e-300) + 1e-30
    assert d["nonfinite_cells"] == 0


@pytest.mark.parametrize("form", [native.FORM_FP64, native.FORM_FP32C])
def test_gpu_pipelined_diagnostics_equal_synchronous_reads(form):
    """post_diag after step i and wait_diag for step i - 1 return, step by
    step, what read_diag returns right after each step."""
    p = cfg_params(nx=64, ny=32, nz=19, source=4, S_n_gr=0.1)
    p.form = form
    p.flags |= native.FLAG_DIAGNOSTICS
    state, m = random_case(p, 17)
    nsteps = 7

    def fresh(s):
        s.set_field("m", m)
        for k, v in state.items():
            s.set_field(k, v)

    with Simulation(p) as s:
        fresh(s)
        want = []
        for _ in range(nsteps):
            s.step(1)
            want.append(s.diag())
    with Simulation(p) as s:
        fresh(s)
        got = []
        for i in range(nsteps):
            s.step(1)
            s.post_diag(i % native.DIAG_SLOTS)
            if i > 0:
                got.append(s.wait_diag((i - 1) % native.DIAG_SLOTS))
        got.append(s.wait_diag((nsteps - 1) % native.DIAG_SLOTS))
        with pytest.raises(native.CapazError) as e:
            s.wait_diag(0)  # nothing posted since its last wait
        assert e.value.code == native.ERR_INVALID_ARGUMENT
    # The step and the post in one call (the precision form's sweep writes
    # the slot itself).
    with Simulation(p) as s:
        fresh(s)
        fused = []
        for i in range(nsteps):
            s.step_post_diag(1, i % native.DIAG_SLOTS)
            if i > 0:
                fused.append(s.wait_diag((i - 1) % native.DIAG_SLOTS))
        fused.append(s.wait_diag((nsteps - 1) % native.DIAG_SLOTS))
    for seq in (got, fused):
        if form == native.FORM_FP64:
            assert seq == want
        else:
            # The precision form's sweep may hand out tiles from a work
            # counter, so its per-CTA partial sums (and their FP64 rounding)
            # may vary from run to run; the state itself does not.
            for a, b in zip(seq, want):
                for i in range(2):
                    assert abs(a["mass"][i] - b["mass"][i]) <= 1e-13 * abs(b["mass"][i])
                assert a["max_residual"] == b["max_residual"] and a["nonfinite_cells"] == b["nonfinite_cells"]
    assert len({d["mass"][0] for d in got}) > 1  # the steps differ


def test_gpu_nonfinite_state_is_reported():
    """S_n above 1 - S_wr makes S_e < 0 and P_k NaN, as in the reference;
    the step reports CAPAZ_ERR_NONFINITE instead of returning silently."""
    p = cfg_params(nx=12, ny=10, nz=7, source=1)
    state, m = random_case(p, 3)
    state["S_n"][3, 4, 5] = 0.97
    with Simulation(p) as s:
        s.set_field("m", m)
        for k, v in state.items():
            s.set_field(k, v)
        s.step(3)
        with pytest.raises(native.CapazError) as e:
            s.get_field("P_w")
        assert e.value.code == native.ERR_NONFINITE


def test_gpu_rejects_bad_porosity():
    p = cfg_params(nx=8, ny=8, nz=8)
    with Simulation(p) as s:
        m = np.full((8, 8, 8), 0.3)
        m[1, 2, 3] = 0.0
        with pytest.raises(native.CapazError) as e:
            s.set_field("m", m)
        assert e.value.code == native.ERR_BAD_STATE


def test_gpu_step_is_deterministic():
    p = cfg_params(nx=64, ny=32, nz=33, source=3, S_n_gr=0.1)
    state, m = random_case(p, 21)
    a = run_gpu(p, state, m, 10)
    b = run_gpu(p, state, m, 10)
    assert np.array_equal(a["P_w"], b["P_w"]) and np.array_equal(a["S_n"], b["S_n"])
