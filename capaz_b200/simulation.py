"""Python host mirror of the C ABI: one `Simulation` per capaz_ctx.

Arrays are numpy float64 of shape (nz, ny, nx) in C order, i.e. the
reference's index i + j*nx + k*nx*ny (main.cpp:695) with y vertical
(j = 0 is the top face).  Device-resident variants take raw device pointers
(e.g. torch tensors' data_ptr()) and a stream handle.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import native
from .native import FIELDS, Diag, Params, check


def default_params(**overrides) -> Params:
    """The reference's Two-phase/defines.ini values, then `overrides`."""
    lib = native.load()
    p = Params()
    check(lib.capaz_params_default(C.byref(p)))
    for k, v in overrides.items():
        setattr(p, "lambda_" if k == "lambda" else k, v)
    return p


def buckley_leverett_params(**overrides) -> Params:
    """The reference's Backley-Leverett/defines.ini (its B_L build): the
    Buckley-Leverett model, fluids, wells and 100 x 100 grid, then
    `overrides`.  K per cell comes from a permeability file
    (Simulation.load_permeability, with FLAG_PERCELL_K)."""
    base = dict(model=native.MODEL_BUCKLEY_LEVERETT, nx=100, ny=100, nz=1, hx=15.0, hy=15.0, hz=10.0,
                dt=86400.0, timeX=1.5e6, source=0, Q=3.5e-6, injwell_Pw=2e5, outwell_Pw=0.9e5,
                background_Pw=3e5, background_Sn=0.7, beta_w=4.35e-5, beta_n=1.0e-5, K0=6.64e-11,
                mu_w=1.2e-3, mu_n=6e-3, ro0_w=1e3, ro0_n=0.848978559e3, lambda_=2.7, S_wr=0.2, S_n_gr=0.4,
                porosity=0.2, P_d=755.0, P_atm=100000.0, g_const=0.0, newton_iterations=10,
                flags=native.FLAG_PERCELL_K)
    base.update(overrides)
    return default_params(**base)


def params_from_ini(path: str, base: Params | None = None) -> Params:
    """Parses a defines.ini the way the reference's read_defines does."""
    lib = native.load()
    p = base.copy() if base is not None else default_params()
    check(lib.capaz_params_from_ini(path.encode(), C.byref(p)))
    return p


def write_ini(p: Params, path: str, extensions: bool = True) -> None:
    """Writes `p` as a defines.ini the reference reads (KEY=value lines)."""
    keys = [
        ("NX", p.nx), ("NY", p.ny), ("NZ", p.nz), ("HX", p.hx), ("HY", p.hy), ("HZ", p.hz),
        ("DT", p.dt), ("TAU", 1e-7), ("L", 1e-4), ("C_W", 1500), ("C_N", 1000), ("C_G", 330),
        ("BETA_W", p.beta_w), ("BETA_N", p.beta_n), ("BETA_G", p.beta_g),
        ("RO_W", p.ro0_w), ("RO_N", p.ro0_n), ("RO_G", p.ro0_g),
        ("MU_W", p.mu_w), ("MU_N", p.mu_n), ("MU_G", p.mu_g),
        ("G_CONST", p.g_const), ("P_ATM", p.P_atm), ("LAMBDA_0", p.lambda_), ("LAMBDA_1", p.lambda_),
        ("M_0", p.porosity), ("M_1", p.porosity), ("S_WR_0", p.S_wr), ("S_WR_1", p.S_wr),
        ("S_NR_0", p.S_nr), ("S_NR_1", p.S_nr), ("S_GR_0", p.S_gr), ("S_GR_1", p.S_gr),
        ("K_0", p.K0), ("K_1", p.K0), ("P_D_0", p.P_d), ("P_D_1", p.P_d),
        ("P_D_NW_0", 0.0), ("P_D_NW_1", 0.0), ("P_D_GN_0", 0.0), ("P_D_GN_1", 0.0),
        ("S_N_GR", p.S_n_gr), ("S_W_GR", p.S_w_gr), ("S_W_INIT", p.S_w_init), ("S_N_INIT", p.S_n_init),
        ("SOURCE", p.source), ("ITERATIONS", p.newton_iterations), ("TIMEX", p.timeX),
        ("SAVE_PLOTS", 1000000), ("PRINT_SCREEN", 1000000),
        ("Q", p.Q), ("BACKGROUND_Pw", p.background_Pw), ("BACKGROUND_Sn", p.background_Sn),
        ("INJECTION_WELL_Pw", p.injwell_Pw), ("INJECTION_WELL_Sn", 0.0),
        ("OUTPUT_WELL_Pw", p.outwell_Pw), ("OUTPUT_WELL_Sn", 0.0),
    ]
    if extensions:
        keys += [("P_TOP_OFFSET", p.P_top_offset), ("S_N_BACKGROUND", p.S_n_background),
                 ("PERCELL_K", 1 if p.flags & native.FLAG_PERCELL_K else 0), ("PHASES", p.phases),
                 ("MODEL", p.model)]
    with open(path, "w") as f:
        f.write("# written by capaz_b200.simulation.write_ini\n")
        for k, v in keys:
            f.write(f"{k}={v!r}\n" if isinstance(v, float) else f"{k}={v}\n")


class Simulation:
    """A context of the C ABI (capaz_create ... capaz_destroy)."""

    def __init__(self, params: Params, device: int = 0, _ctx=None):
        self.lib = native.load()
        self.params = params.copy()
        self._owned = _ctx is None
        if _ctx is None:
            st = C.c_int(0)
            self.ctx = self.lib.capaz_create(C.byref(self.params), device, C.byref(st))
            if not self.ctx:
                msg = self.lib.capaz_last_error(None)
                raise native.CapazError(st.value, msg.decode() if msg else "")
        else:
            self.ctx = _ctx
        self.shape = (params.nz, params.ny, params.nx)

    # -- lifetime --------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "ctx", None):
            if self._owned:
                self.lib.capaz_destroy(self.ctx)
            self.ctx = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- fields ----------------------------------------------------------
    def set_field(self, name: str, arr, stream: int = 0) -> None:
        a = np.ascontiguousarray(np.asarray(arr, dtype=np.float64).reshape(self.shape))
        check(self.lib.capaz_set_field(self.ctx, FIELDS[name], a.ctypes.data, stream or None), self.ctx)

    def get_field(self, name: str, stream: int = 0) -> np.ndarray:
        out = np.empty(self.shape, dtype=np.float64)
        check(self.lib.capaz_get_field(self.ctx, FIELDS[name], out.ctypes.data, stream or None), self.ctx)
        return out

    def set_field_device(self, name: str, dev_ptr: int, stream: int = 0) -> None:
        check(self.lib.capaz_set_field_device(self.ctx, FIELDS[name], dev_ptr, stream or None), self.ctx)

    def get_field_device(self, name: str, dev_ptr: int, stream: int = 0) -> None:
        check(self.lib.capaz_get_field_device(self.ctx, FIELDS[name], dev_ptr, stream or None), self.ctx)

    # -- stepping --------------------------------------------------------
    def init_state(self, stream: int = 0) -> None:
        check(self.lib.capaz_init_state(self.ctx, stream or None), self.ctx)

    def step(self, nsteps: int = 1, stream: int = 0) -> None:
        check(self.lib.capaz_step(self.ctx, int(nsteps), stream or None), self.ctx)

    def set_dt(self, dt: float) -> None:
        check(self.lib.capaz_set_dt(self.ctx, float(dt)), self.ctx)

    def set_sweep_tile(self, tile_y: int) -> None:
        check(self.lib.capaz_set_sweep_tile(self.ctx, int(tile_y)), self.ctx)

    def diag(self, stream: int = 0) -> dict:
        d = Diag()
        check(self.lib.capaz_read_diag(self.ctx, C.byref(d), stream or None), self.ctx)
        return {"mass": list(d.mass), "max_residual": d.max_residual, "nonfinite_cells": d.nonfinite_cells}

    def post_diag(self, slot: int, stream: int = 0) -> None:
        """Queues the copy of the last step's diagnostics into pinned slot
        `slot` (< native.DIAG_SLOTS) without waiting."""
        check(self.lib.capaz_post_diag(self.ctx, int(slot), stream or None), self.ctx)

    def step_post_diag(self, nsteps: int, slot: int, stream: int = 0) -> None:
        """step(nsteps) and post_diag(slot) in one call: the precision form's
        sweep writes the last step's diagnostics into the slot itself."""
        check(self.lib.capaz_step_post_diag(self.ctx, int(nsteps), int(slot), stream or None), self.ctx)

    def wait_diag(self, slot: int) -> dict:
        """Waits for the copy posted to `slot` and returns it (the form of diag())."""
        d = Diag()
        check(self.lib.capaz_wait_diag(self.ctx, int(slot), C.byref(d)), self.ctx)
        return {"mass": list(d.mass), "max_residual": d.max_residual, "nonfinite_cells": d.nonfinite_cells}

    def sync(self) -> None:
        check(self.lib.capaz_sync(self.ctx), self.ctx)

    # -- z-planes of the state (slab halo exchange) -----------------------
    def get_plane(self, name: str, k: int, dev_ptr: int, stream: int = 0) -> None:
        check(self.lib.capaz_get_plane(self.ctx, FIELDS[name], int(k), dev_ptr, stream or None), self.ctx)

    def get_plane_raw(self, name: str, k: int, dev_ptr: int, stream: int = 0) -> None:
        check(self.lib.capaz_get_plane_raw(self.ctx, FIELDS[name], int(k), dev_ptr, stream or None), self.ctx)

    def set_plane_raw(self, name: str, k: int, dev_ptr: int, stream: int = 0) -> None:
        check(self.lib.capaz_set_plane_raw(self.ctx, FIELDS[name], int(k), dev_ptr, stream or None), self.ctx)

    def get_reference(self):
        Pref = np.empty(self.params.ny, dtype=np.float64)
        S = C.c_double(0.0)
        check(self.lib.capaz_get_reference(self.ctx, Pref.ctypes.data_as(C.POINTER(C.c_double)), C.byref(S)),
              self.ctx)
        return Pref, S.value

    def set_reference(self, Pref, S_ref: float) -> None:
        Pref = np.ascontiguousarray(Pref, dtype=np.float64)
        check(self.lib.capaz_set_reference(self.ctx, Pref.ctypes.data_as(C.POINTER(C.c_double)), float(S_ref)),
              self.ctx)

    def step_split(self, edge_stream: int, interior_stream: int) -> None:
        check(self.lib.capaz_step_split(self.ctx, edge_stream, interior_stream), self.ctx)

    def set_plane(self, name: str, k: int, dev_ptr: int, stream: int = 0) -> None:
        check(self.lib.capaz_set_plane(self.ctx, FIELDS[name], int(k), dev_ptr, stream or None), self.ctx)

    # -- heterogeneous media ----------------------------------------------
    def load_permeability(self, path: str) -> None:
        """K per cell from a permeability file (load_permeability's format)."""
        check(self.lib.capaz_load_permeability(self.ctx, os.fsencode(path)), self.ctx)

    def generate_media(self, seed: int, sigma: float = 1.0, ell: float = 8.0, K_mean: float = 1e-12,
                       phi0: float = 0.25, dphi: float = 0.02, nmodes: int = 1024) -> None:
        """Seeded Gaussian field on the device: K = K_mean exp(sigma G),
        porosity = clip(phi0 + dphi G, 0.1, 0.4), covariance exp(-r/ell)."""
        check(self.lib.capaz_generate_media(self.ctx, int(seed), float(sigma), float(ell), float(K_mean),
                                            float(phi0), float(dphi), int(nmodes)), self.ctx)

    # -- files in the reference's formats ---------------------------------
    def write_plot(self, dirpath: str, t: float) -> str:
        """Tecplot plot file <dirpath>/S=%012.4f.dat; returns its path."""
        check(self.lib.capaz_write_plot(self.ctx, os.fsencode(dirpath), float(t)), self.ctx)
        return os.path.join(dirpath, "S=%012.4f.dat" % t)

    def save(self, path: str, time_counter: int = 0) -> None:
        check(self.lib.capaz_save(self.ctx, os.fsencode(path), int(time_counter)), self.ctx)

    def restore(self, path: str) -> int:
        tc = C.c_int(0)
        check(self.lib.capaz_restore(self.ctx, os.fsencode(path), C.byref(tc)), self.ctx)
        return tc.value

    @property
    def launch_count(self) -> int:
        return int(self.lib.capaz_launch_count(self.ctx))


class Ensemble:
    """A batch of instances stepped by one persistent launch per step
    (capaz_batch_* in include/capaz_b200.h)."""

    def __init__(self, params_list, device: int = 0):
        self.lib = native.load()
        n = len(params_list)
        arr = (Params * n)(*[p.copy() for p in params_list])
        st = C.c_int(0)
        self.b = self.lib.capaz_batch_create(arr, n, device, C.byref(st))
        if not self.b:
            msg = self.lib.capaz_last_error(None)
            raise native.CapazError(st.value, msg.decode() if msg else "")
        self.instances = [Simulation(params_list[q], device, _ctx=self.lib.capaz_batch_instance(self.b, q))
                          for q in range(n)]

    def step(self, nsteps: int = 1, stream: int = 0) -> None:
        check(self.lib.capaz_batch_step(self.b, int(nsteps), stream or None))

    def autotune(self, stream: int = 0) -> dict:
        check(self.lib.capaz_batch_autotune(self.b, stream or None, None, None))
        return self.tuning()

    def tuning(self) -> dict:
        zc, per, ty = C.c_int(0), C.c_int(0), C.c_int(0)
        check(self.lib.capaz_batch_get_tuning(self.b, C.byref(zc), C.byref(per), C.byref(ty)))
        return {"zchunk": zc.value, "ctas_per_sm": per.value, "tile": [32, ty.value] if ty.value else None}

    def set_tuning(self, zchunk: int, ctas_per_sm: int = 0, tile_y: int = 16) -> None:
        check(self.lib.capaz_batch_set_tuning(self.b, int(zchunk), int(ctas_per_sm), int(tile_y)))

    @property
    def launch_count(self) -> int:
        return int(self.lib.capaz_batch_launch_count(self.b))

    def close(self) -> None:
        if getattr(self, "b", None):
            for s in self.instances:
                s.ctx = None
            self.lib.capaz_batch_destroy(self.b)
            self.b = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Adjoint:
    """Misfit gradient of a two-phase FP64 context (capaz_adjoint_create ...
    capaz_backward): J = sum over observation times and cells of
    (S_w - data)^2, gradients with respect to ln K and porosity per cell."""

    def __init__(self, sim: Simulation, nsteps: int, obs_cells, obs_every: int, checkpoint_every: int = 50,
                 init_from_m: bool = True):
        self.sim = sim
        self.lib = sim.lib
        self.obs = np.ascontiguousarray(obs_cells, dtype=np.int64)
        self.nsteps, self.obs_every = int(nsteps), int(obs_every)
        self.ntimes = self.nsteps // self.obs_every
        st = C.c_int(0)
        flags = native.ADJ_INIT_FROM_M if init_from_m else 0
        self.adj = self.lib.capaz_adjoint_create(sim.ctx, self.nsteps, int(checkpoint_every), self.obs.ctypes.data,
                                                 len(self.obs), self.obs_every, flags, C.byref(st))
        if not self.adj:
            msg = self.lib.capaz_last_error(None)
            raise native.CapazError(st.value, msg.decode() if msg else "")

    def set_observations(self, data) -> None:
        d = np.ascontiguousarray(np.asarray(data, dtype=np.float64).reshape(self.ntimes, len(self.obs)))
        check(self.lib.capaz_adjoint_set_observations(self.adj, d.ctypes.data, 0, None), self.sim.ctx)

    def forward(self, stream: int = 0) -> float:
        J = C.c_double(0.0)
        check(self.lib.capaz_forward_checkpointed(self.adj, C.byref(J), stream or None), self.sim.ctx)
        return J.value

    def backward(self, stream: int = 0):
        gK = np.empty(self.sim.shape, dtype=np.float64)
        gm = np.empty(self.sim.shape, dtype=np.float64)
        check(self.lib.capaz_backward(self.adj, gK.ctypes.data, gm.ctypes.data, 0, stream or None), self.sim.ctx)
        return gK, gm

    def close(self) -> None:
        if getattr(self, "adj", None):
            self.lib.capaz_adjoint_destroy(self.adj)
            self.adj = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_permeability_file(path: str, nx: int, ny: int, nz: int) -> np.ndarray:
    """K (nz, ny, nx) from a permeability file in load_permeability's format."""
    lib = native.load()
    K = np.empty((nz, ny, nx), dtype=np.float64)
    st = lib.capaz_read_permeability_file(os.fsencode(path), nx, ny, nz, K.ctypes.data)
    if st:
        msg = lib.capaz_last_error(None)
        raise native.CapazError(st, msg.decode() if msg else "")
    return K
