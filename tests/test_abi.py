"""The C-ABI library on the CPU: it loads, exports every declared symbol,
and its host-only entry points (parameters, defines.ini) behave."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, gpu_present
import capaz_b200
from capaz_b200 import native
from capaz_b200.simulation import default_params, params_from_ini, write_ini


def declared_c_symbols(header):
    text = open(os.path.join(ROOT, "include", header)).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(capaz_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = native.load()
    names = declared_c_symbols("capaz_b200.h")
    assert len(names) >= 18
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(native.PROTOTYPES), "bindings and header disagree"


def test_struct_layouts():
    lib = native.load()
    assert lib.capaz_params_size() == C.sizeof(native.Params)
    assert lib.capaz_diag_size() == C.sizeof(native.Diag)
    assert lib.capaz_abi_version() == 6


def test_defaults_are_reference_two_phase_ini():
    p = default_params()
    assert (p.nx, p.ny, p.nz, p.source, p.newton_iterations) == (15, 15, 1, 30, 10)
    assert (p.lambda_, p.S_wr, p.P_d, p.K0, p.porosity) == (2.7, 0.09, 755.0, 6.64e-11, 0.4)


def test_ini_round_trip(tmp_path):
    p = default_params(nx=33, ny=17, nz=9, dt=0.125, lambda_=2.0, P_d=0.0, source=4, S_n_gr=0.1,
                       P_top_offset=1e4, S_n_background=0.85)
    path = str(tmp_path / "defines.ini")
    write_ini(p, path)
    q = params_from_ini(path, base=default_params())
    for k, v in p.as_dict().items():
        assert getattr(q, k) == v, k


def test_ini_parsing_rules(tmp_path):
    """read_defines rules: '#' lines skipped, value ends at the first space,
    unknown keys ignored, atoi truncation (main.cpp:1299-1323)."""
    path = tmp_path / "defines.ini"
    path.write_text("# comment NX=99\nNX=21    trailing words\nHX=5e-2\nUNKNOWN=1\nNZ=3.7\n"
                    "SOURCE=30           \nDT=1e-3")
    q = params_from_ini(str(path), base=default_params())
    assert q.nx == 21 and q.hx == 5e-2 and q.nz == 3 and q.source == 30 and q.dt == 1e-3


def test_validate_rejects_unsupported_grids():
    lib = native.load()
    for nx, ny, nz in [(2, 5, 5), (5, 2, 5), (5, 5, 2), (5, 5, 0)]:
        p = default_params(nx=nx, ny=ny, nz=nz)
        assert lib.capaz_params_validate(C.byref(p)) == native.ERR_UNSUPPORTED_GRID
    p = default_params(nx=1, phases=3)
    assert lib.capaz_params_validate(C.byref(p)) == native.OK
    p = default_params(dt=0.0)
    assert lib.capaz_params_validate(C.byref(p)) == native.ERR_INVALID_ARGUMENT


def test_validate_buckley_leverett_model():
    """The B-L task is the two-phase FP64 step with its own wells and
    boundary; its well blocks need nx, ny >= 4."""
    lib = native.load()
    ok = dict(model=native.MODEL_BUCKLEY_LEVERETT, nx=8, ny=6, nz=1)
    assert lib.capaz_params_validate(C.byref(default_params(**ok))) == native.OK
    assert lib.capaz_params_validate(C.byref(default_params(**dict(ok, nz=5)))) == native.OK
    for bad, code in [(dict(nx=3), native.ERR_UNSUPPORTED_GRID), (dict(ny=3), native.ERR_UNSUPPORTED_GRID),
                      (dict(phases=3), native.ERR_UNSUPPORTED), (dict(form=native.FORM_FP32C), native.ERR_UNSUPPORTED),
                      (dict(flags=native.FLAG_DIAGNOSTICS), native.ERR_UNSUPPORTED),
                      (dict(model=7), native.ERR_INVALID_ARGUMENT)]:
        p = default_params(**dict(ok, **bad))
        assert lib.capaz_params_validate(C.byref(p)) == code, bad


def test_validate_energy_model():
    """The energy equation is the three-phase FP64 step with T; no
    diagnostics, no z-slab placement (its stencil reaches two cells)."""
    lib = native.load()
    ok = dict(model=native.MODEL_ENERGY, phases=3, nx=9, ny=8, nz=6)
    assert lib.capaz_params_validate(C.byref(default_params(**ok))) == native.OK
    assert lib.capaz_params_validate(C.byref(default_params(**dict(ok, nx=1, nz=1)))) == native.OK
    for bad, code in [(dict(phases=2), native.ERR_UNSUPPORTED), (dict(form=native.FORM_FP32C), native.ERR_UNSUPPORTED),
                      (dict(flags=native.FLAG_DIAGNOSTICS), native.ERR_UNSUPPORTED),
                      (dict(z_offset=1, nz_global=8), native.ERR_UNSUPPORTED)]:
        p = default_params(**dict(ok, **bad))
        assert lib.capaz_params_validate(C.byref(p)) == code, bad


def test_ini_round_trip_buckley_leverett(tmp_path):
    p = default_params(nx=20, ny=15, model=native.MODEL_BUCKLEY_LEVERETT, Q=3.5e-6, background_Pw=3e5,
                       background_Sn=0.7, injwell_Pw=2e5, outwell_Pw=0.9e5)
    path = str(tmp_path / "defines.ini")
    write_ini(p, path)
    q = params_from_ini(path, base=default_params())
    for k, v in p.as_dict().items():
        assert getattr(q, k) == v, k


def test_missing_ini_is_an_error():
    with pytest.raises(native.CapazError) as e:
        params_from_ini("/nonexistent/defines.ini")
    assert e.value.code == native.ERR_INI


@pytest.mark.skipif(gpu_present(), reason="checks the no-GPU error path")
def test_create_without_gpu_fails_cleanly():
    with pytest.raises(native.CapazError) as e:
        capaz_b200.Simulation(default_params())
    assert e.value.code == native.ERR_NO_DEVICE


def test_null_arguments_return_errors():
    lib = native.load()
    assert lib.capaz_step(None, 1, None) == native.ERR_INVALID_ARGUMENT
    assert lib.capaz_destroy(None) == native.ERR_INVALID_ARGUMENT
    assert lib.capaz_params_default(None) == native.ERR_INVALID_ARGUMENT
    assert lib.capaz_post_diag(None, 0, None) == native.ERR_INVALID_ARGUMENT
    assert lib.capaz_wait_diag(None, 0, None) == native.ERR_INVALID_ARGUMENT


def test_diag_slot_count_matches_header():
    text = open(os.path.join(ROOT, "include", "capaz_b200.h")).read()
    assert re.search(r"#define CAPAZ_DIAG_SLOTS (\d+)", text).group(1) == str(native.DIAG_SLOTS)
