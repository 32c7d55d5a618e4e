"""Precision form (FP32 storage, compensated FP32 stencil, FP64 Newton).

Bar (BASELINE): relative L2 error in S of at most 1e-6 after 1000 steps at
the 256x256x128 workload against the FP64 path, which itself matches the
reference CPU step to 1e-12.  The per-field max-abs and relative-L2 errors of
P and S are asserted here and reported by bench.py.
"""
import numpy as np
import pytest

from conftest import rel_err
from capaz_b200 import Simulation, native
from capaz_b200.configs import config1, heterogeneous_fields, stable_dt, two_phase_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    return float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel()))


def run(p, m, K, nsteps, init=True, state=None, diag=False):
    q = p.copy()
    if diag:
        q.flags |= native.FLAG_DIAGNOSTICS
    with Simulation(q) as s:
        s.set_field("m", m)
        if K is not None:
            s.set_field("K", K)
        if state is None:
            s.init_state()
        else:
            for k, v in state.items():
                s.set_field(k, v)
        s.step(nsteps)
        out = {"P_w": s.get_field("P_w"), "S_n": s.get_field("S_n")}
        if diag:
            out["diag"] = s.diag()
    return out


def test_encode_decode_round_trip():
    p = two_phase_params(40, 20, 30, form=native.FORM_FP32C)
    m, K = heterogeneous_fields((p.nz, p.ny, p.nx), 1.0, 4.0, 3)
    st = O.init(p, m)
    with Simulation(p) as s:
        s.set_field("m", m)
        s.set_field("K", K)
        s.set_field("P_w", st["P_w"])
        s.set_field("S_n", st["S_n"])
        P, S = s.get_field("P_w"), s.get_field("S_n")
        mm, KK = s.get_field("m"), s.get_field("K")
    # Deviations from the row profile are small: far better than FP32 of P.
    assert np.abs(P - st["P_w"]).max() <= 1e-3
    assert np.abs(S - st["S_n"]).max() <= 1e-7
    assert np.abs(mm - m).max() <= 1e-7 and rel_err(KK, K) <= 1e-7


def test_fp32c_against_oracle_heterogeneous():
    """100 steps on a 96x40x64 grid with a lognormal K field, from the
    reference initial state, against the FP64 oracle."""
    p64 = two_phase_params(96, 40, 64)
    m, K = heterogeneous_fields((p64.nz, p64.ny, p64.nx), 1.0, 8.0, 5)
    p64.dt = stable_dt(p64, m, K)
    st = O.init(p64, m)
    ref = O.step(p64, {"P_w": st["P_w"], "S_n": st["S_n"]}, 100, m, K)
    p32 = p64.copy()
    p32.form = native.FORM_FP32C
    out = run(p32, m, K, 100)
    eS = rel_l2(out["S_n"], ref["S_n"])
    eP = rel_l2(out["P_w"], ref["P_w"])
    dS = np.abs(ref["S_n"] - st["S_n"]).max()
    assert eS <= 1e-6, eS
    assert eP <= 1e-6, eP
    # The increments are resolved: the error is far below the change itself.
    assert np.abs(out["S_n"] - ref["S_n"]).max() < 0.05 * dS


def test_fp32c_full_workload_1000_steps_vs_fp64():
    """The precision bar at the full workload: 256x256x128, 1000 steps."""
    w64 = config1(form=native.FORM_FP64)
    out64 = run(w64.params, w64.m, w64.K, 1000, diag=True)
    p32 = w64.params.copy()
    p32.form = native.FORM_FP32C
    out32 = run(p32, w64.m, w64.K, 1000, diag=True)
    eS = rel_l2(out32["S_n"], out64["S_n"])
    eP = rel_l2(out32["P_w"], out64["P_w"])
    assert eS <= 1e-6, eS
    assert eP <= 1e-6, eP
    m64, m32 = out64["diag"]["mass"], out32["diag"]["mass"]
    for i in range(2):
        assert abs(m32[i] - m64[i]) <= 1e-6 * abs(m64[i])
    assert out32["diag"]["max_residual"] < 1e-9


def test_diagnostics_leave_the_state_unchanged():
    """A precision-form step that reduces the diagnostics computes the same
    state as one that does not (both refine the reciprocal of the Newton
    determinant once), and the diagnostics of every step agree with those of
    a run that reduces them only at its end."""
    p = two_phase_params(64, 40, 48, form=native.FORM_FP32C)
    m, K = heterogeneous_fields((p.nz, p.ny, p.nx), 1.0, 4.0, 11)
    p.dt = stable_dt(p, m, K)
    plain = run(p, m, K, 6)
    q = p.copy()
    q.flags |= native.FLAG_DIAGNOSTICS
    with Simulation(q) as s:
        s.set_field("m", m)
        s.set_field("K", K)
        s.init_state()
        for _ in range(6):
            s.step(1)
        every = {"P_w": s.get_field("P_w"), "S_n": s.get_field("S_n"), "diag": s.diag()}
    last = run(p, m, K, 6, diag=True)
    for k in ("P_w", "S_n"):
        assert np.array_equal(every[k], plain[k]), k
        assert np.array_equal(last[k], plain[k]), k
    assert every["diag"]["mass"] == last["diag"]["mass"]
    assert every["diag"]["max_residual"] == last["diag"]["max_residual"]
    assert every["diag"]["nonfinite_cells"] == 0


def test_fp32c_planar_and_capillary():
    p = two_phase_params(70, 33, 1, form=native.FORM_FP32C)
    p.P_d, p.lambda_ = 755.0, 2.7
    p.flags = 0
    rng = np.random.default_rng(2)
    m = np.clip(0.3 + 0.03 * rng.standard_normal((1, 33, 70)), 0.15, 0.45)
    p.dt = stable_dt(p, m, None)
    st = O.init(p, m)
    p64 = p.copy()
    p64.form = native.FORM_FP64
    ref = O.step(p64, {"P_w": st["P_w"], "S_n": st["S_n"]}, 50, m)
    out = run(p, m, None, 50)
    assert rel_l2(out["S_n"], ref["S_n"]) <= 1e-6
    assert rel_l2(out["P_w"], ref["P_w"]) <= 1e-6


def test_fp32c_derived_fields_decode():
    p = two_phase_params(40, 20, 30, form=native.FORM_FP32C)
    m, K = heterogeneous_fields((p.nz, p.ny, p.nx), 1.0, 4.0, 9)
    p.dt = stable_dt(p, m, K)
    st = O.init(p, m)
    p64 = p.copy()
    p64.form = native.FORM_FP64
    ref = O.step(p64, {"P_w": st["P_w"], "S_n": st["S_n"]}, 5, m, K, derived=True)
    with Simulation(p) as s:
        s.set_field("m", m)
        s.set_field("K", K)
        s.init_state()
        s.step(5)
        for f in ("ro_w", "ro_n", "Xi_w", "Xi_n", "uy_w"):
            a = s.get_field(f)
            assert rel_l2(a, ref["derived"][f]) <= 1e-5, f


@pytest.mark.parametrize("shape,steps,h", [((68, 21, 19), 40, (1.0, 1.0, 1.0)), ((256, 30, 20), 20, (1.0, 1.0, 1.0)),
                                            ((36, 9, 1), 30, (1.0, 1.0, 1.0)), ((44, 19, 13), 30, (0.5, 2.0, 1.5))])
def test_fp32c_tma_path_matches_plain_load_path(shape, steps, h):
    """The TMA-staged kernel (nx a multiple of 4) against the plain-load
    kernel and the FP64 oracle, on ragged tiles, several z-chunks, a planar
    grid and a non-unit spacing."""
    nx, ny, nz = shape
    p = two_phase_params(nx, ny, nz, form=native.FORM_FP32C)
    p.hx, p.hy, p.hz = h
    m, K = heterogeneous_fields((nz, ny, nx), 1.0, 4.0, 17)
    p.dt = stable_dt(p, m, K)
    st = O.init(p, m)
    p64 = p.copy()
    p64.form = native.FORM_FP64
    ref = O.step(p64, {"P_w": st["P_w"], "S_n": st["S_n"]}, steps, m, K)
    tma = run(p, m, K, steps)
    q = p.copy()
    q.flags |= native.FLAG_NO_TMA
    plain = run(q, m, K, steps)
    for f in ("S_n", "P_w"):
        assert rel_l2(tma[f], ref[f]) <= 1e-6, f
        assert rel_l2(tma[f], plain[f]) <= 1e-6, f


def test_tma_wait_timeout_stops_the_step_and_the_process_carries_on():
    """The TMA-staged sweep's bounded waits: with CAPAZ_FLAG_TEST_WAIT_TIMEOUT
    each stage announces more bytes than its copies bring, so every CTA's
    first wait runs out after about a second.  The CTA stops (no stage is
    consumed or re-armed), lets its copies land, and leaves; the step
    reports CAPAZ_ERR_CUDA.  Nothing faults or hangs: a fresh context on the
    same device then steps normally."""
    import time

    from capaz_b200.native import CapazError
    p = two_phase_params(64, 40, 48, form=native.FORM_FP32C)
    m, K = heterogeneous_fields((p.nz, p.ny, p.nx), 1.0, 4.0, 9)
    p.dt = stable_dt(p, m, K)
    q = p.copy()
    q.flags |= native.FLAG_TEST_WAIT_TIMEOUT
    t0 = time.time()
    with Simulation(q) as s:
        s.set_field("m", m)
        s.set_field("K", K)
        s.init_state()
        with pytest.raises(CapazError) as e:
            s.step(1)
            s.sync()
        assert e.value.code == native.ERR_CUDA
        assert "bounded wait" in str(e.value)
    assert time.time() - t0 < 60
    ref = run(p, m, K, 5)
    st = O.init(p, m)
    exp = O.step(p, {"P_w": st["P_w"], "S_n": st["S_n"]}, 5, m, K)
    assert rel_l2(ref["S_n"], exp["S_n"]) <= 1e-6 and rel_l2(ref["P_w"], exp["P_w"]) <= 1e-6
