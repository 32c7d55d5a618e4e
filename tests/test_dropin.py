"""Link-level drop-in (include/capaz_refabi.h, libcapaz_dropin_2ph.so and
libcapaz_dropin_3ph.so).

The reference's own host objects (main.cpp, no_communication.cpp,
shared_test.cpp, gauss.cpp), compiled from its sources by oracle/Makefile,
are linked against this library in place of the reference's GPU backend.
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

from conftest import GOLDEN_2PH, GOLDEN_3PH, ROOT, interior, load_golden, rel_err
from oracle import oracle as O

DROPIN = os.path.join(ROOT, "capaz_b200", "lib", "libcapaz_dropin_2ph.so")
HARNESS = os.path.join(ROOT, "oracle", "_ref", "capaz_dropin_harness_2ph")
MAIN_DROPIN = os.path.join(ROOT, "oracle", "_ref", "capaz_dropin_main_2ph")
MAIN_REF = os.path.join(ROOT, "oracle", "_ref", "capaz_ref_main_2ph")
DROPIN3 = os.path.join(ROOT, "capaz_b200", "lib", "libcapaz_dropin_3ph.so")
HARNESS3 = os.path.join(ROOT, "oracle", "_ref", "capaz_dropin_harness_3ph")
MAIN_DROPIN3 = os.path.join(ROOT, "oracle", "_ref", "capaz_dropin_main_3ph")
MAIN_REF3 = os.path.join(ROOT, "oracle", "_ref", "capaz_ref_main_3ph")


def declared_refabi_functions():
    text = open(os.path.join(ROOT, "include", "capaz_refabi.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^void\s+([A-Za-z_0-9]+)\s*\(", text, flags=re.M)))


@pytest.mark.parametrize("lib", [DROPIN, DROPIN3])
def test_dropin_exports_every_declared_function(lib):
    names = declared_refabi_functions()
    assert len(names) == 27  # 6 stages, 5 memory, 2 device, init, 12 halo, checkErrors
    out = subprocess.run(["nm", "-D", "--defined-only", "-C", lib], capture_output=True, text=True,
                         check=True).stdout
    for n in names:
        assert re.search(r"\s" + re.escape(n) + r"\(", out), n


@pytest.mark.parametrize("exe,lib", [(MAIN_DROPIN, "libcapaz_dropin_2ph.so"),
                                     (MAIN_DROPIN3, "libcapaz_dropin_3ph.so")])
def test_dropin_covers_what_the_reference_host_program_needs(exe, lib):
    """Every symbol the reference's main.cpp takes from its arch backend is
    among those the drop-in exports (checked on the linked test binary)."""
    if not os.path.exists(exe):
        pytest.skip("drop-in link binaries not built (make -C oracle REF=<reference tree> all)")
    res = subprocess.run(["ldd", exe], capture_output=True, text=True)
    assert "not found" not in res.stdout
    assert lib in res.stdout


def _plots(dirpath):
    out = {}
    for f in sorted(os.listdir(dirpath)):
        with open(os.path.join(dirpath, f)) as fh:
            out[f] = fh.read().splitlines()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", GOLDEN_2PH)
def test_dropin_harness_matches_reference(name):
    """The reference's step loop driven through the drop-in reproduces the
    reference CPU results (state and every derived array)."""
    p, g = load_golden(name)
    if "in_P_w" in g:
        state, m = {"P_w": g["in_P_w"], "S_n": g["in_S_n"]}, g["in_m"]
    else:
        state, m = None, None
    r = O.ref_run(p, int(g["nsteps"]), state, m, binary=HARNESS, derived=True)
    for k in ("P_w", "S_n"):
        assert rel_err(r[k], g["out_" + k]) <= 1e-12, k
    for f, v in r["derived"].items():
        a, b = v, g["der_" + f]
        if f.startswith("roS"):
            a, b = interior(a), interior(b)
        assert rel_err(a, b) <= 1e-12, f


@pytest.mark.gpu
def test_reference_program_runs_unmodified_on_the_dropin(tmp_path):
    """The reference's whole program (its own main and defines.ini handling,
    plot output every SAVE_PLOTS steps) produces the same plot files with
    this library as with the reference's CPU backend."""
    from capaz_b200.simulation import default_params
    p = default_params(nx=31, ny=21, nz=9, dt=1e-3, source=3, timeX=0.2)
    ini = O.ref_ini_text(p).replace("SAVE_PLOTS=1000000", "SAVE_PLOTS=100")
    results = {}
    for tag, exe in (("ref", MAIN_REF), ("dropin", MAIN_DROPIN)):
        wd = tmp_path / tag
        (wd / "run").mkdir(parents=True)
        (wd / "defines.ini").write_text(ini)
        res = subprocess.run([exe], cwd=wd / "run", capture_output=True, text=True, timeout=600)
        assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
        results[tag] = _plots(wd / "run" / "plots")
    assert results["ref"].keys() == results["dropin"].keys()
    assert len(results["ref"]) == 3  # t = 0, 0.1, 0.2
    exact = total = 0
    for f, lines in results["ref"].items():
        other = results["dropin"][f]
        assert len(lines) == len(other)
        for a, b in zip(lines, other):
            total += 1
            if a == b:
                exact += 1
                continue
            va = np.array([float(x) for x in a.split()])
            vb = np.array([float(x) for x in b.split()])
            assert np.allclose(va, vb, rtol=2e-3, atol=1e-30), (f, a, b)
    assert exact / total > 0.999, f"{exact}/{total} plot lines identical"


@pytest.mark.gpu
@pytest.mark.parametrize("name", GOLDEN_3PH)
def test_dropin3_harness_matches_reference(name):
    """The reference's three-phase step loop driven through
    libcapaz_dropin_3ph reproduces the reference CPU results."""
    if not os.path.exists(HARNESS3):
        pytest.skip("drop-in link binaries not built (make -C oracle REF=<reference tree> all)")
    p, g = load_golden(name)
    names = ["P_w", "S_w", "S_n", "P_n", "P_g"]
    if "in_P_w" in g:
        state, m = {k: g["in_" + k] for k in names}, g["in_m"]
    else:
        state, m = None, None
    r = O.ref_run(p, int(g["nsteps"]), state, m, binary=HARNESS3, derived=True)
    for k in names:
        assert rel_err(r[k], g["out_" + k]) <= 1e-12, k
    for f, v in r["derived"].items():
        a, b = v, g["der_" + f]
        if f.startswith("roS"):
            a, b = interior(a), interior(b)
        assert rel_err(a, b) <= 1e-12, f


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(9, 8, 6), (1, 15, 1)])
def test_reference_three_phase_program_runs_unmodified_on_the_dropin(tmp_path, shape):
    """The reference's whole THREE_PHASE program with libcapaz_dropin_3ph in
    place of its backend writes the plot files its CPU backend writes, except
    the S_g column: save_data_plots downloads S_w, S_n, P_w and the
    velocities but not S_g (main.cpp:475-491), so with any device backend
    (the reference's own gpu.o too) the plot shows the host copy that
    data_initialization left, while the CPU backend updates it in place."""
    from capaz_b200.simulation import default_params
    if not os.path.exists(MAIN_DROPIN3):
        pytest.skip("drop-in link binaries not built (make -C oracle REF=<reference tree> all)")
    nx, ny, nz = shape
    p = default_params(phases=3, nx=nx, ny=ny, nz=nz, newton_iterations=7, lambda_=2.0, S_wr=0.1, S_nr=0.05,
                       S_gr=0.02, ro0_w=1000.0, ro0_n=850.0, ro0_g=1.2, mu_w=1e-3, mu_n=3e-3, mu_g=1.8e-5,
                       beta_w=1e-9, beta_n=1e-9, beta_g=9.2e-6, S_w_gr=0.25, S_n_gr=0.7, S_w_init=0.2,
                       S_n_init=0.3, source=1, porosity=0.3, K0=1e-12, hx=1.0, hy=1.0, hz=1.0, dt=1e-3,
                       g_const=9.81, P_d=0.0, timeX=0.06)
    ini = O.ref_ini_text(p).replace("SAVE_PLOTS=1000000", "SAVE_PLOTS=30")
    sg_col = 3 if nx == 1 and nz == 1 else 5  # "Y",S_w,S_n,S_g... / "X","Y","Z",S_w,S_n,S_g...
    results = {}
    for tag, exe in (("ref", MAIN_REF3), ("dropin", MAIN_DROPIN3)):
        wd = tmp_path / tag
        (wd / "run").mkdir(parents=True)
        (wd / "defines.ini").write_text(ini)
        res = subprocess.run([exe], cwd=wd / "run", capture_output=True, text=True, timeout=600)
        assert res.returncode == 0, res.stdout[-2000:] + res.stderr[-2000:]
        results[tag] = _plots(wd / "run" / "plots")
    assert results["ref"].keys() == results["dropin"].keys()
    assert len(results["ref"]) == 3
    exact = total = 0
    for f, lines in results["ref"].items():
        other = results["dropin"][f]
        assert len(lines) == len(other)
        for q, (a, b) in enumerate(zip(lines, other)):
            if q < 3:  # TITLE, VARIABLES, ZONE
                assert a == b
                continue
            ta, tb = a.split(), b.split()
            del ta[sg_col], tb[sg_col]
            total += 1
            if ta == tb:
                exact += 1
                continue
            va = np.array([float(x) for x in ta])
            vb = np.array([float(x) for x in tb])
            assert np.allclose(va, vb, rtol=2e-3, atol=1e-30), (f, a, b)
    assert exact / total > 0.999, f"{exact}/{total} plot lines identical"


@pytest.mark.gpu
def test_dropin_rejects_out_of_order_stages(tmp_path):
    """A stage out of time_step_function's order is an error (exit 1 with
    the reference's error format), not a silently different result."""
    src = tmp_path / "bad.cpp"
    src.write_text(
        '#include "capaz_refabi.h"\n#include <string.h>\n'
        "int main(){ consts d; memset(&d,0,sizeof d); d.locNx=d.Nx=5; d.locNy=d.Ny=5; d.locNz=d.Nz=1;"
        "d.size=d.sizex=d.sizey=d.sizez=1; d.hx=d.hy=d.hz=1; d.dt=1e-3; d.mu_w=d.mu_n=1e-3; d.P_atm=1e5;"
        "d.lambda[0]=2; d.K[0]=1e-12; d.porosity[0]=0.3; d.newton_iterations=1; device_initialization(&d);"
        "ptr_Arrays H, D; P_S_calculation(H, D, d); return 0; }\n")
    exe = tmp_path / "bad"
    subprocess.run(["g++", "-I" + os.path.join(ROOT, "include"), str(src), "-o", str(exe), DROPIN,
                    "-Wl,-rpath," + os.path.dirname(DROPIN)], check=True)
    res = subprocess.run([str(exe)], capture_output=True, text=True)
    assert res.returncode == 1
    assert "Error:" in res.stdout and "out of the order" in res.stdout
