"""Generates tests/golden/*.npz from the reference's own CPU implementation.

    python tests/golden/make_golden.py        # every fixture
    python tests/golden/make_golden.py bl     # the Buckley-Leverett ones only
    python tests/golden/make_golden.py energy # the energy-equation ones only

Each fixture holds the parameter set, the input state (or none: the
reference's data_initialization), and the reference's outputs after N steps:
the state and, where asked, every other per-cell array the reference keeps
(S_w, P_n, rho, Xi, u, roS, roS_old ...).  The reference binaries come from
oracle/Makefile (compiled from the reference sources, which must be present
where the fixtures are generated); the fixtures need nothing at test time.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from capaz_b200.simulation import default_params  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cfg_fluids(**kw):
    """Config-0 fluids in the reference model (lambda 2, S_wr 0.1, no P_d)."""
    base = dict(hx=1.0, hy=1.0, hz=1.0, mu_w=1e-3, mu_n=5e-3, ro0_w=1000.0, ro0_n=850.0, beta_w=1e-9,
                beta_n=1e-9, lambda_=2.0, S_wr=0.1, P_d=0.0, g_const=9.81, P_atm=1e5, K0=1e-12,
                porosity=0.3, newton_iterations=10)
    base.update(kw)
    return default_params(**base)


def random_state2(p, rng, s_mean=0.5):
    m = np.clip(0.3 + 0.03 * rng.standard_normal((p.nz, p.ny, p.nx)), 0.15, 0.45)
    st = O.init(p, m)
    S = np.clip(s_mean + 0.2 * rng.standard_normal(st["S_n"].shape), 0.05, 0.85)
    return {"P_w": st["P_w"], "S_n": S}, m


def save(name, p, nsteps, state, m, with_derived):
    r = O.ref_run(p, nsteps, state, m if state is not None else None, derived=with_derived)
    out = {"params": np.array(json.dumps(p.as_dict())), "nsteps": np.array(nsteps)}
    if state is not None:
        for k, v in state.items():
            out["in_" + k] = v
        out["in_m"] = m
    for k in ("P_w", "S_w", "S_n", "P_n", "P_g", "T"):
        if k in r:
            out["out_" + k] = r[k]
    if with_derived:
        for k, v in r["derived"].items():
            out["der_" + k] = v
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print(f"{path}: {os.path.getsize(path)} bytes, ref {r['info']}")


def main():
    if not (O.ref_available(2) and O.ref_available(3)):
        raise SystemExit("build the reference binaries first: make -C oracle REF=<reference tree> ref")
    rng = np.random.default_rng(20261203)

    # The reference's own Two-phase/defines.ini values, its own initial state.
    save("g2_default_15x15x1", default_params(), 100, None, None, True)
    # data_initialization on a 3-D grid with a source window (0 steps).
    save("g2_init_10x9x7", default_params(nx=10, ny=9, nz=7, source=2), 0, None, None, False)
    # Random states on 3-D grids, with and without capillary pressure.
    p = cfg_fluids(nx=12, ny=10, nz=7, dt=0.02, source=2, S_n_gr=0.1)
    st, m = random_state2(p, rng)
    save("g2_3d_pd0_12x10x7", p, 30, st, m, True)
    p = cfg_fluids(nx=12, ny=10, nz=7, dt=0.02, source=1, S_n_gr=0.3, P_d=755.0, lambda_=2.7)
    st, m = random_state2(p, rng)
    save("g2_3d_pd_12x10x7", p, 30, st, m, True)
    # Planar grid (NZ = 1), the reference's default geometry, odd sizes.
    p = cfg_fluids(nx=17, ny=13, nz=1, dt=0.02, source=3, S_n_gr=0.1)
    st, m = random_state2(p, rng)
    save("g2_planar_17x13x1", p, 40, st, m, True)
    # Smallest 3-D grid (every interior cell touches the boundary).
    p = cfg_fluids(nx=3, ny=3, nz=3, dt=0.02, source=0)
    st, m = random_state2(p, rng)
    save("g2_min_3x3x3", p, 10, st, m, True)

    # Three-phase: the reference's Three-phase/defines.ini column case.
    p3 = default_params(phases=3, nx=1, ny=15, nz=1, newton_iterations=7, lambda_=3.25, S_wr=0.0,
                        ro0_n=850.0, ro0_g=1.4, mu_n=1e-3, mu_g=1.84e-5, beta_g=9.2e-6, S_w_gr=0.4,
                        S_n_gr=0.3, S_w_init=0.4, S_n_init=0.3, source=0, porosity=0.4, K0=6.64e-11,
                        timeX=1000.0)
    save("g3_column_1x15x1", p3, 200, None, None, True)
    p3 = default_params(phases=3, nx=9, ny=8, nz=6, newton_iterations=7, lambda_=2.0, S_wr=0.1, S_nr=0.05,
                        S_gr=0.02, ro0_w=1000.0, ro0_n=850.0, ro0_g=1.2, mu_w=1e-3, mu_n=3e-3, mu_g=1.8e-5,
                        beta_w=1e-9, beta_n=1e-9, beta_g=9.2e-6, S_w_gr=0.25, S_n_gr=0.7, S_w_init=0.2,
                        S_n_init=0.3, source=1, porosity=0.3, K0=1e-12, hx=1.0, hy=1.0, hz=1.0, dt=0.01,
                        g_const=9.81)
    m = np.clip(0.3 + 0.03 * rng.standard_normal((p3.nz, p3.ny, p3.nx)), 0.15, 0.45)
    st = O.init(p3, m)
    st["S_w"] = np.clip(0.3 + 0.1 * rng.standard_normal(st["S_w"].shape), 0.12, 0.6)
    st["S_n"] = np.clip(0.3 + 0.1 * rng.standard_normal(st["S_n"].shape), 0.07, 0.35)
    state = {k: st[k] for k in ("P_w", "S_w", "S_n", "P_n", "P_g")}
    save("g3_3d_9x8x6", p3, 30, state, m, True)


def energy_3d_params(nx, ny, nz):
    """Three-phase fluids of the random 3-D case, with the energy equation."""
    return default_params(phases=3, nx=nx, ny=ny, nz=nz, newton_iterations=7, lambda_=2.0, S_wr=0.1, S_nr=0.05,
                          S_gr=0.02, ro0_w=1000.0, ro0_n=850.0, ro0_g=1.2, mu_w=1e-3, mu_n=3e-3, mu_g=1.8e-5,
                          beta_w=1e-9, beta_n=1e-9, beta_g=9.2e-6, S_w_gr=0.25, S_n_gr=0.7, S_w_init=0.2,
                          S_n_init=0.3, source=1, porosity=0.3, K0=1e-12, hx=1.0, hy=1.0, hz=1.0, dt=0.01,
                          g_const=9.81, model=2)


def main_energy():
    """The THREE_PHASE + ENERGY build: the reference's Three-phase/defines.ini
    column case from its own initial state, and random 3-D states with a
    random temperature field."""
    if not os.path.exists(O.ref_binary(3, 2)):
        raise SystemExit("build the reference binaries first: make -C oracle REF=<reference tree> ref")
    rng = np.random.default_rng(20261204)
    p3 = default_params(phases=3, nx=1, ny=15, nz=1, newton_iterations=7, lambda_=3.25, S_wr=0.0,
                        ro0_n=850.0, ro0_g=1.4, mu_n=1e-3, mu_g=1.84e-5, beta_g=9.2e-6, S_w_gr=0.4,
                        S_n_gr=0.3, S_w_init=0.4, S_n_init=0.3, source=0, porosity=0.4, K0=6.64e-11,
                        timeX=1000.0, model=2)
    save("ge_column_1x15x1", p3, 200, None, None, True)
    for shape, nsteps in (((9, 8, 6), 20), ((11, 7, 1), 25)):
        p = energy_3d_params(*shape)
        m = np.clip(0.3 + 0.03 * rng.standard_normal((p.nz, p.ny, p.nx)), 0.15, 0.45)
        st = O.init(p, m)
        st["S_w"] = np.clip(0.3 + 0.1 * rng.standard_normal(st["S_w"].shape), 0.12, 0.6)
        st["S_n"] = np.clip(0.3 + 0.1 * rng.standard_normal(st["S_n"].shape), 0.07, 0.35)
        st["T"] = 285 + 5 * rng.standard_normal(st["S_w"].shape)
        state = {k: st[k] for k in ("P_w", "S_w", "S_n", "P_n", "P_g", "T")}
        save("ge_%dx%dx%d" % shape, p, nsteps, state, m, True)


def bl_params(nx, ny, nz, g, dt):
    """The reference's Backley-Leverett/defines.ini fluids and wells."""
    return default_params(nx=nx, ny=ny, nz=nz, dt=dt, model=1, Q=3.5e-6, background_Pw=3e5,
                          background_Sn=0.7, injwell_Pw=2e5, outwell_Pw=0.9e5, beta_w=4.35e-5, beta_n=1e-5,
                          mu_w=1.2e-3, mu_n=6e-3, ro0_n=848.978559, porosity=0.2, K0=6.64e-11, g_const=g,
                          hx=15.0, hy=15.0, hz=10.0, newton_iterations=10, source=0, P_d=755.0, lambda_=2.7)


def save_bl(name, p, nsteps, seed):
    """A Buckley-Leverett case from the reference's data_initialization with
    K from a permeability file written here (K itself as the reference's
    loader reads it, through oracle/_ref/capaz_ref_loadk)."""
    import tempfile
    import make_media_golden as mg
    with tempfile.TemporaryDirectory() as d:
        noise = os.path.join(d, "noise.dat")
        vals = np.random.default_rng(seed).normal(-1.5, 0.6, size=(p.ny, p.nx))
        mg.write_noise(noise, vals)
        if p.nz > 1:
            text = open(noise, "rb").read().split(b"\r\n", 1)
            open(noise, "wb").write(f"{p.nx} {p.ny} {p.nz}".encode() + b"\r\n" + text[1])
        K = mg.reference_K(noise, p.nx, p.ny, p.nz)
        r = O.ref_run(p, nsteps, noise=noise)
    out = {"params": np.array(json.dumps(p.as_dict())), "nsteps": np.array(nsteps), "K": K,
           "out_P_w": r["P_w"], "out_S_n": r["S_n"]}
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **out)
    print(f"{path}: {os.path.getsize(path)} bytes, ref {r['info']}")


def main_bl():
    if not os.path.exists(O.ref_binary(2, 1)):
        raise SystemExit("build the reference binaries first: make -C oracle REF=<reference tree> ref")
    save_bl("gbl_planar_20x15x1", bl_params(20, 15, 1, 0.0, 2000.0), 40, 20)
    save_bl("gbl_3d_gravity_12x10x6", bl_params(12, 10, 6, 9.81, 200.0), 30, 12)


if __name__ == "__main__":
    if sys.argv[1:] == ["bl"]:
        main_bl()
    elif sys.argv[1:] == ["energy"]:
        main_energy()
    else:
        main()
        main_bl()
        main_energy()
