"""Discrete adjoint of the two-phase FP64 step (capaz_forward_checkpointed /
capaz_backward) against the oracle's forward-mode (dual-number) derivative of
the same misfit, and against central finite differences of the GPU forward.

Both the adjoint and the forward mode are exact derivatives of the discrete
step; they differ by the Newton iterations (implicit-function transpose at
the final iterate vs. the unrolled iterations) and by summation order.
"""
import numpy as np
import pytest

from capaz_b200 import Adjoint, Simulation, native
from capaz_b200.configs import heterogeneous_fields, observe, stable_dt, two_phase_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu

TOL_TANGENT = 1e-9   # adjoint <g, d> vs forward-mode dJ, relative
TOL_J = 1e-12        # misfit, GPU forward vs oracle


def _case(nx, ny, nz, steps, every, seed, cols, **kw):
    p = two_phase_params(nx, ny, nz)
    for k, v in kw.items():
        setattr(p, k, v)
    sh = (nz, ny, nx)
    m_t, K_t = heterogeneous_fields(sh, 1.0, 4.0, seed)
    m_p, K_p = heterogeneous_fields(sh, 0.5, 3.0, seed + 100)
    p.dt = min(stable_dt(p, m_t, K_t), stable_dt(p, m_p, K_p))
    obs = np.array([i + j * nx + k * nx * ny for (i, k) in cols for j in range(ny)], dtype=np.int64)
    data = observe(p, m_t, K_t, obs, every, steps)
    return p, m_p, K_p, obs, data


def _gradient(p, m, K, obs, data, steps, every, cp, init_from_m=True, pre_steps=0):
    with Simulation(p) as sim:
        sim.set_field("m", m)
        sim.set_field("K", K)
        sim.init_state()
        state = None
        if pre_steps:
            sim.step(pre_steps)
            state = (sim.get_field("P_w"), sim.get_field("S_n"))
        with Adjoint(sim, steps, obs, every, cp, init_from_m=init_from_m) as adj:
            adj.set_observations(data)
            J = adj.forward()
            gK, gm = adj.backward()
    return J, gK, gm, state


def _directions(p, obs, seed):
    rng = np.random.default_rng(seed)
    sh = (p.nz, p.ny, p.nx)
    dirs = [(rng.standard_normal(sh), 0.01 * rng.standard_normal(sh)) for _ in range(2)]
    for q in range(2):  # single cells next to observed columns
        l = int(obs[len(obs) // 3 + 5 * q]) + 1
        e = np.zeros(p.nx * p.ny * p.nz)
        e[l] = 1.0
        dirs.append((e.reshape(sh), None))
        dirs.append((None, e.reshape(sh)))
    return dirs


def _check_against_tangent(p, m, K, obs, data, steps, every, J, gK, gm, init_from_m=True, state=None):
    P0, S0 = state if state is not None else (None, None)
    J_o, _ = O.tangent(p, steps, m, K, obs, every, data, init_from_m=init_from_m, P0=P0, S0=S0)
    assert abs(J - J_o) <= TOL_J * abs(J_o), (J, J_o)
    nonzero = 0
    for dl, dm in _directions(p, obs, 7):
        _, dJ = O.tangent(p, steps, m, K, obs, every, data, dlnK=dl, dm=dm, init_from_m=init_from_m, P0=P0, S0=S0)
        terms = []
        if dl is not None:
            terms.append((gK * dl).ravel())
        if dm is not None:
            terms.append((gm * dm).ravel())
        terms = np.concatenate(terms)
        g = float(np.sum(terms))
        # Relative to the magnitude of the inner product's terms: a direction
        # the misfit does not depend on (dJ == 0) needs a zero gradient there.
        scale = float(np.sum(np.abs(terms)))
        assert abs(g - dJ) <= TOL_TANGENT * max(abs(dJ), scale), (g, dJ)
        nonzero += dJ != 0.0
    assert nonzero >= 3


def test_adjoint_matches_forward_mode_3d():
    steps, every = 60, 10
    p, m, K, obs, data = _case(20, 12, 14, steps, every, 11, [(5, 4), (14, 9)])
    J, gK, gm, _ = _gradient(p, m, K, obs, data, steps, every, cp=25)
    _check_against_tangent(p, m, K, obs, data, steps, every, J, gK, gm)


def test_adjoint_capillary_general_lambda():
    """P_d != 0 and lambda = 2.7: P_n = P_w + P_k(S) in fluxes, densities and Newton."""
    steps, every = 40, 8
    p, m, K, obs, data = _case(16, 10, 9, steps, every, 21, [(4, 3), (11, 5)], P_d=755.0, lambda_=2.7)
    J, gK, gm, _ = _gradient(p, m, K, obs, data, steps, every, cp=16)
    _check_against_tangent(p, m, K, obs, data, steps, every, J, gK, gm)


def test_adjoint_planar_window_from_given_state():
    """nz = 1, an injection window narrower than the top face (constant S
    cells and copied S cells on the top row), start state not a function of m."""
    steps, every = 50, 5
    p, m, K, obs, data = _case(23, 13, 1, steps, every, 31, [(3, 0), (11, 0), (20, 0)], source=3)
    J, gK, gm, state = _gradient(p, m, K, obs, data, steps, every, cp=12, init_from_m=False, pre_steps=7)
    _check_against_tangent(p, m, K, obs, data, steps, every, J, gK, gm, init_from_m=False, state=state)


def test_adjoint_checkpoint_interval_does_not_change_the_gradient():
    steps, every = 30, 6
    p, m, K, obs, data = _case(12, 9, 8, steps, every, 41, [(3, 3), (8, 5)])
    J1, gK1, gm1, _ = _gradient(p, m, K, obs, data, steps, every, cp=7)
    J2, gK2, gm2, _ = _gradient(p, m, K, obs, data, steps, every, cp=steps)
    assert J1 == J2
    assert np.array_equal(gK1, gK2) and np.array_equal(gm1, gm2)


def test_adjoint_central_differences():
    """Central differences of the GPU forward at the cells of largest
    sensitivity.  The misfit's rounding noise (the FP64 state carries about
    1e-16 absolute in S while the signal is h * dS/dtheta) limits how small
    the step can be at this short horizon, hence h = 1e-4 and 1e-3 relative
    tolerance; exactness is checked against the forward mode above."""
    steps, every = 60, 10
    p, m, K, obs, data = _case(20, 12, 14, steps, every, 51, [(5, 4), (14, 9)])
    J, gK, gm, _ = _gradient(p, m, K, obs, data, steps, every, cp=30)
    h = 1e-4

    def misfit(mm, KK):
        with Simulation(p) as sim:
            sim.set_field("m", mm)
            sim.set_field("K", KK)
            with Adjoint(sim, steps, obs, every, steps) as adj:
                adj.set_observations(data)
                return adj.forward()

    for which, g in (("K", gK), ("m", gm)):
        cells = np.argsort(-np.abs(g).ravel())[:5]
        fd, ad = [], []
        for l in cells:
            mp, mq = m.copy().reshape(-1), m.copy().reshape(-1)
            Kp, Kq = K.copy().reshape(-1), K.copy().reshape(-1)
            if which == "K":
                Kp[l] *= np.exp(h)
                Kq[l] *= np.exp(-h)
            else:
                mp[l] += h
                mq[l] -= h
            fd.append((misfit(mp.reshape(m.shape), Kp.reshape(K.shape)) -
                       misfit(mq.reshape(m.shape), Kq.reshape(K.shape))) / (2 * h))
            ad.append(g.reshape(-1)[l])
        fd, ad = np.array(fd), np.array(ad)
        assert np.linalg.norm(fd - ad) <= 1e-3 * np.linalg.norm(fd), (which, fd, ad)
