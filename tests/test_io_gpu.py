"""Files in the reference's formats: the Tecplot plot file (capaz_write_plot,
print_plots main.cpp:549-781) against the plot files the reference's own
whole program writes, and save.dat (capaz_save / capaz_restore,
main.cpp:1035-1145)."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT
from capaz_b200 import Simulation, native
from capaz_b200.simulation import buckley_leverett_params, default_params
from oracle import oracle as O

pytestmark = pytest.mark.gpu

MAIN_REF = {2: os.path.join(ROOT, "oracle", "_ref", "capaz_ref_main_2ph"),
            3: os.path.join(ROOT, "oracle", "_ref", "capaz_ref_main_3ph"),
            "bl": os.path.join(ROOT, "oracle", "_ref", "capaz_ref_main_bl"),
            "energy": os.path.join(ROOT, "oracle", "_ref", "capaz_ref_main_3phe")}


def params3(**kw):
    base = dict(phases=3, newton_iterations=7, lambda_=2.0, S_wr=0.1, S_nr=0.05, S_gr=0.02, ro0_w=1000.0,
                ro0_n=850.0, ro0_g=1.2, mu_w=1e-3, mu_n=3e-3, mu_g=1.8e-5, beta_w=1e-9, beta_n=1e-9,
                beta_g=9.2e-6, S_w_gr=0.25, S_n_gr=0.7, S_w_init=0.2, S_n_init=0.3, source=1, porosity=0.3,
                K0=1e-12, hx=1.0, hy=1.0, hz=1.0, g_const=9.81, P_d=0.0)
    base.update(kw)
    return default_params(**base)


def reference_plots(p, tmp_path, save_every, noise=None):
    """Runs the reference's whole program (its own main and CPU backend) and
    returns its plot files.  `noise`: the permeability file of the B_L build
    (read from ../noise.dat)."""
    exe = MAIN_REF[{native.MODEL_BUCKLEY_LEVERETT: "bl", native.MODEL_ENERGY: "energy"}.get(p.model, p.phases)]
    if not os.path.exists(exe):
        pytest.skip("reference whole-program binaries not built (make -C oracle REF=<reference tree> ref)")
    ini = O.ref_ini_text(p).replace("SAVE_PLOTS=1000000", f"SAVE_PLOTS={save_every}")
    wd = tmp_path / "ref"
    (wd / "run").mkdir(parents=True)
    (wd / "defines.ini").write_text(ini)
    if noise is not None:
        (wd / "noise.dat").write_bytes(open(noise, "rb").read())
    res = subprocess.run([exe], cwd=wd / "run", capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
    d = wd / "run" / "plots"
    return {f: (d / f).read_text().splitlines() for f in sorted(os.listdir(d))}


def our_plots(p, tmp_path, save_every, nsave, noise=None):
    d = tmp_path / "ours"
    with Simulation(p) as s:
        if noise is not None:
            s.load_permeability(noise)
        s.init_state()
        s.write_plot(str(d), 0.0)
        for q in range(1, nsave + 1):
            s.step(save_every)
            s.write_plot(str(d), q * save_every * p.dt)
    return {f: (d / f).read_text().splitlines() for f in sorted(os.listdir(d))}


def compare(ref, ours):
    assert ref.keys() == ours.keys()
    exact = total = 0
    for f, lines in ref.items():
        other = ours[f]
        assert len(lines) == len(other), f
        assert lines[:3] == other[:3], f  # TITLE, VARIABLES, ZONE
        for a, b in zip(lines[3:], other[3:]):
            total += 1
            if a == b:
                exact += 1
                continue
            va = np.array([float(x) for x in a.split()])
            vb = np.array([float(x) for x in b.split()])
            # a value on a rounding boundary of the printed digits
            assert np.allclose(va, vb, rtol=2e-3, atol=1e-30), (f, a, b)
    assert exact / total > 0.999, f"{exact}/{total} plot rows identical"


@pytest.mark.parametrize("shape", [(31, 21, 9), (25, 17, 1)])
def test_plot_file_matches_reference_program_two_phase(tmp_path, shape):
    nx, ny, nz = shape
    p = default_params(nx=nx, ny=ny, nz=nz, dt=1e-3, source=3, timeX=0.2)
    compare(reference_plots(p, tmp_path, 100), our_plots(p, tmp_path, 100, 2))


@pytest.mark.parametrize("shape", [(9, 8, 6), (1, 15, 1)])
def test_plot_file_matches_reference_program_three_phase(tmp_path, shape):
    nx, ny, nz = shape
    p = params3(nx=nx, ny=ny, nz=nz, dt=1e-3, timeX=0.06)
    compare(reference_plots(p, tmp_path, 30), our_plots(p, tmp_path, 30, 2))


@pytest.mark.parametrize("shape,g,dt", [((20, 15, 1), 0.0, 2000.0), ((12, 10, 6), 9.81, 50.0)])
def test_plot_file_matches_reference_program_buckley_leverett(tmp_path, shape, g, dt):
    """The B_L build's plot rows (S_w, P_w, u, K) with K from a noise.dat."""
    nx, ny, nz = shape
    p = buckley_leverett_params(nx=nx, ny=ny, nz=nz, g_const=g, dt=dt, timeX=40 * dt)
    noise = str(tmp_path / "noise.dat")
    write_noise(noise, np.random.default_rng(nx).normal(-1.5, 0.6, size=(ny, nx)), nz)
    compare(reference_plots(p, tmp_path, 20, noise), our_plots(p, tmp_path, 20, 2, noise))


@pytest.mark.parametrize("shape", [(9, 8, 6), (1, 15, 1), (11, 7, 1)])
def test_plot_file_matches_reference_program_energy(tmp_path, shape):
    """The THREE_PHASE + ENERGY build's plot rows (T after P_w)."""
    nx, ny, nz = shape
    p = params3(nx=nx, ny=ny, nz=nz, dt=1e-3, timeX=0.06, model=native.MODEL_ENERGY)
    compare(reference_plots(p, tmp_path, 30), our_plots(p, tmp_path, 30, 2))


def write_noise(path, values, nz=1):
    """A permeability file: header "Nx Ny" (or "Nx Ny Nz"), then Ny rows of
    values, CRLF line ends as the reference's sample file has them."""
    ny, nx = values.shape
    head = f"{nx} {ny}" if nz < 2 else f"{nx} {ny} {nz}"
    with open(path, "wb") as f:
        f.write((head + "\r\n").encode())
        for row in values:
            f.write(("".join(f"{v:.6f} " for v in row) + "\r\n").encode())


def _state(s, phases):
    names = ["P_w", "S_n"] + (["S_w", "P_n", "P_g"] if phases == 3 else [])
    return {k: s.get_field(k) for k in names}


@pytest.mark.parametrize("phases", [2, 3])
def test_save_restore_continues_bit_identically(tmp_path, phases):
    p = default_params(nx=20, ny=14, nz=9, dt=1e-3, source=3) if phases == 2 else \
        params3(nx=9, ny=12, nz=7, dt=1e-3)
    rng = np.random.default_rng(phases)
    m = np.clip(0.3 + 0.02 * rng.standard_normal((p.nz, p.ny, p.nx)), 0.2, 0.4)
    path = str(tmp_path / "save.dat")
    with Simulation(p) as a:
        a.set_field("m", m)
        a.init_state()
        a.step(7)
        a.save(path, 7)
        saved = _state(a, phases)
        a.step(5)
        want = _state(a, phases)
    n = p.nx * p.ny * p.nz
    nf = 7 if phases == 3 else 5
    assert os.path.getsize(path) == 4 + 8 * n * nf
    raw = np.fromfile(path, dtype=np.float64, offset=4).reshape(nf, p.nz, p.ny, p.nx)
    assert int(np.fromfile(path, dtype=np.int32, count=1)[0]) == 7
    off = 1 if phases == 3 else 0
    assert np.array_equal(raw[off], saved["P_w"]) and np.array_equal(raw[off + 1], saved["S_n"])
    assert np.array_equal(raw[-1], m)
    if phases == 3:
        assert np.array_equal(raw[0], saved["S_w"])
    with Simulation(p) as b:
        assert b.restore(path) == 7
        if phases == 3:
            # P_n, P_g as the reference restores them: equal to P_w
            b.set_field("P_n", saved["P_n"])
            b.set_field("P_g", saved["P_g"])
        b.step(5)
        got = _state(b, phases)
    for k in want:
        assert np.array_equal(got[k], want[k]), k


def test_restore_rejects_a_file_of_another_grid(tmp_path):
    p = default_params(nx=10, ny=8, nz=5, dt=1e-3)
    path = str(tmp_path / "save.dat")
    with Simulation(p) as a:
        a.init_state()
        a.save(path, 1)
    q = default_params(nx=10, ny=8, nz=6, dt=1e-3)
    with Simulation(q) as b:
        with pytest.raises(native.CapazError, match="size does not match"):
            b.restore(path)
