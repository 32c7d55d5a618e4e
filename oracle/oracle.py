"""Python access to the oracle — TEST INFRASTRUCTURE.

Two CPU implementations used as the parity reference:
  - the restatement libcapaz_oracle.so (oracle/capaz_oracle.cpp), OpenMP;
  - the reference's own CPU step, compiled from its sources into
    oracle/_ref/capaz_ref_{2ph,3ph} by oracle/Makefile, driven through
    oracle/ref_harness.cpp.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use
this module.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import json
import os
import subprocess
import tempfile

import numpy as np

from capaz_b200.native import FIELD_COUNT, Diag, Params

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libcapaz_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            subprocess.run(["make", "-C", HERE, "oracle"], check=True, capture_output=True)
        lib = C.CDLL(LIB)
        P = C.POINTER(C.c_double)
        lib.oracle_reverse_matrix.argtypes = [P, C.c_int]
        lib.oracle_reverse_matrix.restype = C.c_int
        lib.oracle_init.argtypes = [C.POINTER(Params), P, P, P, P, P, P, P]
        lib.oracle_init.restype = C.c_int
        lib.oracle_step.argtypes = [C.POINTER(Params), C.c_int, P, P, P, P, P, P, P,
                                    C.POINTER(P), C.POINTER(Diag), C.c_int]
        lib.oracle_step.restype = C.c_int
        lib.oracle_max_threads.restype = C.c_int
        lib.oracle_init_temperature.argtypes = [C.POINTER(Params), P]
        lib.oracle_init_temperature.restype = C.c_int
        lib.oracle_step_energy.argtypes = [C.POINTER(Params), C.c_int, P, P, P, P, P, P, P, P, C.POINTER(P),
                                           C.c_int]
        lib.oracle_step_energy.restype = C.c_int
        lib.oracle_tangent.argtypes = [C.POINTER(Params), C.c_int, P, P, P, P, C.c_int, P, P,
                                       C.POINTER(C.c_long), C.c_int, C.c_int, P, P, P, C.c_int]
        lib.oracle_tangent.restype = C.c_int
        _lib = lib
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _shape(p: Params):
    return (p.nz, p.ny, p.nx)


def reverse_matrix(a: np.ndarray) -> tuple[int, np.ndarray]:
    a = np.ascontiguousarray(a, dtype=np.float64).copy()
    rc = load().oracle_reverse_matrix(_ptr(a), a.shape[0])
    return rc, a


def init(p: Params, m: np.ndarray | None = None) -> dict:
    """data_initialization (two-phase.cpp:113-172 / three-phase.cpp:438-500)."""
    sh = _shape(p)
    out = {k: np.zeros(sh) for k in ("m", "P_w", "S_w", "S_n", "P_n", "P_g")}
    m_in = None if m is None else np.ascontiguousarray(m, dtype=np.float64)
    rc = load().oracle_init(C.byref(p), _ptr(m_in), _ptr(out["m"]), _ptr(out["P_w"]), _ptr(out["S_w"]),
                            _ptr(out["S_n"]), _ptr(out["P_n"]), _ptr(out["P_g"]))
    if rc:
        raise RuntimeError(f"oracle_init failed: {rc}")
    if p.phases == 2:
        for k in ("S_w", "P_n", "P_g"):
            out.pop(k)
    if p.model == 2:
        out["T"] = np.zeros(sh)
        rc = load().oracle_init_temperature(C.byref(p), _ptr(out["T"]))
        if rc:
            raise RuntimeError(f"oracle_init_temperature failed: {rc}")
    return out


def step(p: Params, state: dict, nsteps: int, m: np.ndarray, K: np.ndarray | None = None,
         derived: bool = False, diag: bool = False, nthreads: int = 0) -> dict:
    """Advances a copy of `state` by nsteps with the restated reference step.
    Returns the new state (and 'derived' / 'diag' when asked)."""
    sh = _shape(p)
    st = {k: np.ascontiguousarray(v, dtype=np.float64).copy() for k, v in state.items()}
    for k in ("S_w", "P_n", "P_g"):
        if p.phases == 3 and k not in st:
            raise ValueError(f"three-phase state needs {k}")
    m = np.ascontiguousarray(m, dtype=np.float64)
    K = None if K is None else np.ascontiguousarray(K, dtype=np.float64)
    dptrs = None
    dout = {}
    if derived:
        arr = (C.POINTER(C.c_double) * FIELD_COUNT)()
        from capaz_b200.native import ENERGY_FIELDS, FIELDS
        for name, idx in FIELDS.items():
            if name in ("P_w", "S_n", "m", "K") or (p.phases == 3 and name in ("S_w", "P_n", "P_g")):
                continue
            if name in ENERGY_FIELDS and (p.model != 2 or name == "T"):
                continue
            if p.phases == 2 and name.endswith("_g") or name == "P_g":
                continue
            dout[name] = np.zeros(sh)
            arr[idx] = _ptr(dout[name])
        dptrs = arr
    if p.model == 2:
        if "T" not in st:
            raise ValueError("the energy model's state needs T")
        rc = load().oracle_step_energy(C.byref(p), int(nsteps), _ptr(st["P_w"]), _ptr(st["S_w"]), _ptr(st["S_n"]),
                                       _ptr(st["P_n"]), _ptr(st["P_g"]), _ptr(st["T"]), _ptr(m), _ptr(K), dptrs,
                                       int(nthreads))
        if rc:
            raise RuntimeError(f"oracle_step_energy failed: {rc}")
        if derived:
            st["derived"] = dout
        return st
    d = Diag()
    rc = load().oracle_step(C.byref(p), int(nsteps), _ptr(st["P_w"]), _ptr(st.get("S_w")), _ptr(st["S_n"]),
                            _ptr(st.get("P_n")), _ptr(st.get("P_g")), _ptr(m), _ptr(K), dptrs,
                            C.byref(d) if diag else None, int(nthreads))
    if rc:
        raise RuntimeError(f"oracle_step failed: {rc}")
    if derived:
        st["derived"] = dout
    if diag:
        st["diag"] = {"mass": list(d.mass), "max_residual": d.max_residual,
                      "nonfinite_cells": d.nonfinite_cells}
    return st


def max_threads() -> int:
    return int(load().oracle_max_threads())


# ---------------------------------------------------------------------------
# The reference's own CPU step (oracle/_ref).

REF_KEYS_2PH = ["NX", "NY", "NZ", "HX", "HY", "HZ", "DT", "TAU", "L", "C_W", "C_N", "BETA_W", "BETA_N",
                "RO_W", "RO_N", "MU_W", "MU_N", "G_CONST", "P_ATM", "LAMBDA_0", "LAMBDA_1", "M_0", "M_1",
                "S_WR_0", "S_WR_1", "K_0", "K_1", "P_D_0", "P_D_1", "S_N_GR", "SOURCE", "ITERATIONS",
                "TIMEX", "SAVE_PLOTS", "PRINT_SCREEN"]


def ref_ini_text(p: Params) -> str:
    """defines.ini text for the reference (KEY=value, main.cpp:1299-1627)."""
    vals = {
        "NX": p.nx, "NY": p.ny, "NZ": p.nz, "HX": p.hx, "HY": p.hy, "HZ": p.hz, "DT": p.dt,
        "TAU": 1e-7, "L": 1e-4, "C_W": 1500, "C_N": 1000, "C_G": 330,
        "BETA_W": p.beta_w, "BETA_N": p.beta_n, "BETA_G": p.beta_g,
        "RO_W": p.ro0_w, "RO_N": p.ro0_n, "RO_G": p.ro0_g,
        "MU_W": p.mu_w, "MU_N": p.mu_n, "MU_G": p.mu_g, "G_CONST": p.g_const, "P_ATM": p.P_atm,
        "LAMBDA_0": p.lambda_, "LAMBDA_1": p.lambda_, "M_0": p.porosity, "M_1": p.porosity,
        "S_WR_0": p.S_wr, "S_WR_1": p.S_wr, "S_NR_0": p.S_nr, "S_NR_1": p.S_nr,
        "S_GR_0": p.S_gr, "S_GR_1": p.S_gr, "K_0": p.K0, "K_1": p.K0, "P_D_0": p.P_d, "P_D_1": p.P_d,
        "P_D_NW_0": 0.0, "P_D_NW_1": 0.0, "P_D_GN_0": 0.0, "P_D_GN_1": 0.0,
        "S_N_GR": p.S_n_gr, "S_W_GR": p.S_w_gr, "S_W_INIT": p.S_w_init, "S_N_INIT": p.S_n_init,
        "SOURCE": p.source, "ITERATIONS": p.newton_iterations, "TIMEX": p.timeX,
        "SAVE_PLOTS": 1000000, "PRINT_SCREEN": 1000000,
        "Q": p.Q, "BACKGROUND_Pw": p.background_Pw, "BACKGROUND_Sn": p.background_Sn,
        "INJECTION_WELL_Pw": p.injwell_Pw, "INJECTION_WELL_Sn": 0.0,
        "OUTPUT_WELL_Pw": p.outwell_Pw, "OUTPUT_WELL_Sn": 0.0,
    }
    lines = ["# defines.ini for the reference harness"]
    for k, v in vals.items():
        lines.append(f"{k}={v!r}" if isinstance(v, float) else f"{k}={v}")
    return "\n".join(lines) + "\n"


def ref_binary(phases: int, model: int = 0) -> str:
    if model == 1:
        return os.path.join(REF_DIR, "capaz_ref_bl")
    if model == 2:
        return os.path.join(REF_DIR, "capaz_ref_3phe")
    return os.path.join(REF_DIR, "capaz_ref_2ph" if phases == 2 else "capaz_ref_3ph")


def ref_available(phases: int = 2) -> bool:
    return os.path.exists(ref_binary(phases))


REF_DERIVED_2PH = ["S_w", "P_n", "ro_w", "ro_n", "ux_w", "uy_w", "uz_w", "ux_n", "uy_n", "uz_n",
                   "Xi_w", "Xi_n", "roS_w", "roS_w_old", "roS_n", "roS_n_old"]
REF_DERIVED_3PH = REF_DERIVED_2PH + ["S_g", "ro_g", "ux_g", "uy_g", "uz_g", "Xi_g", "roS_g", "roS_g_old"]
REF_DERIVED_3PHE = REF_DERIVED_3PH + ["H_w", "H_n", "H_g", "H_r", "E", "E_new"]


def ref_run(p: Params, nsteps: int, state: dict | None = None, m: np.ndarray | None = None,
            binary: str | None = None, env: dict | None = None, derived: bool = False,
            noise: str | None = None) -> dict:
    """Runs the reference's own CPU time step (or, with `binary`, the same
    harness linked to another backend) for nsteps from `state` (None: the
    reference's data_initialization).  Returns the final state and timing.
    The Buckley-Leverett build reads its permeability from `noise` (a file in
    load_permeability's format; K_0 everywhere without one)."""
    bl = p.model == 1
    if p.P_top_offset != 0.0 or (p.phases == 2 and p.S_n_background != 0.0) or ((p.flags & 1) and not bl):
        raise ValueError("the reference has no P_top_offset / S_n_background / per-cell K")
    exe = binary or ref_binary(p.phases, p.model)
    sh = _shape(p)
    n = p.nx * p.ny * p.nz
    with tempfile.TemporaryDirectory() as wd:
        with open(os.path.join(wd, "defines.ini"), "w") as f:
            f.write(ref_ini_text(p))
        if noise is not None:
            with open(noise, "rb") as src, open(os.path.join(wd, "noise.dat"), "wb") as dst:
                dst.write(src.read())
        in_path = "-"
        if state is not None:
            in_path = os.path.join(wd, "in.bin")
            if p.phases == 2:
                fields = [state["P_w"], state["S_n"], m]
            else:
                fields = [state["P_w"], state["S_w"], state["S_n"], state["P_n"], state["P_g"], m]
                if p.model == 2:
                    fields.append(state["T"])
            np.concatenate([np.ascontiguousarray(a, dtype=np.float64).ravel() for a in fields]).tofile(in_path)
        out_path = os.path.join(wd, "out.bin")
        cmd = [exe, wd, str(nsteps), in_path, out_path]
        der_path = os.path.join(wd, "derived.bin")
        if derived:
            cmd.append(der_path)
        res = subprocess.run(cmd, capture_output=True, text=True, env=env)
        if res.returncode != 0:
            raise RuntimeError(f"{exe} failed ({res.returncode}): {res.stdout[-2000:]} {res.stderr[-2000:]}")
        line = [ln for ln in res.stdout.splitlines() if ln.startswith("RESULT ")][-1]
        info = json.loads(line[len("RESULT "):])
        raw = np.fromfile(out_path, dtype=np.float64)
        draw = np.fromfile(der_path, dtype=np.float64) if derived else None
    names = ["P_w", "S_n"] if p.phases == 2 else ["P_w", "S_w", "S_n", "P_n", "P_g"]
    if p.model == 2:
        names.append("T")
    out = {k: raw[a * n:(a + 1) * n].reshape(sh) for a, k in enumerate(names)}
    out["info"] = info
    if derived:
        dn = REF_DERIVED_2PH if p.phases == 2 else REF_DERIVED_3PHE if p.model == 2 else REF_DERIVED_3PH
        out["derived"] = {k: draw[a * n:(a + 1) * n].reshape(sh) for a, k in enumerate(dn)}
    return out


def tangent(p: Params, nsteps: int, m, K, obs, every: int, data=None, dlnK=None, dm=None,
            init_from_m: bool = True, P0=None, S0=None, nthreads: int = 0) -> tuple[float, float]:
    """(J, dJ): the observation misfit after `nsteps` two-phase steps and its
    forward-mode derivative along (dlnK, dm) (oracle_tangent)."""
    sh = _shape(p)
    f = lambda a: None if a is None else np.ascontiguousarray(np.broadcast_to(a, sh), dtype=np.float64)
    m, K, dlnK, dm, P0, S0 = f(m), f(K), f(dlnK), f(dm), f(P0), f(S0)
    obs = np.ascontiguousarray(obs, dtype=np.int64)
    data = None if data is None else np.ascontiguousarray(data, dtype=np.float64)
    J, dJ = C.c_double(), C.c_double()
    rc = load().oracle_tangent(C.byref(p), nsteps, _ptr(m), _ptr(K), _ptr(dlnK), _ptr(dm), int(init_from_m),
                               _ptr(P0), _ptr(S0), obs.ctypes.data_as(C.POINTER(C.c_long)), len(obs), every,
                               _ptr(data), C.byref(J), C.byref(dJ), nthreads)
    if rc:
        raise RuntimeError(f"oracle_tangent failed: {rc}")
    return J.value, dJ.value
