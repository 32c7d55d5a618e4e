"""The benchmark workloads as parameter sets and seeded synthetic inputs.

Axes.  The workloads are stated with gravity on z; the reference's vertical
axis is y with j = 0 at the top (cpu.cpp:699-705, main.cpp:255-267).  A
workload grid (Nx, Ny, Nz) with gravity on z maps to the reference grid
NX = Nx, NY = Nz (vertical), NZ = Ny.  Arrays here are (NZ, NY, NX).

Physics mapping (two-phase, the reference's Brooks-Corey/Burdine model,
two-phase.cpp:8-13): lambda = 2 gives k_w = S_e^4, k_n = (1-S_e)^2 (1-S_e^2);
S_wr = 0.1; no capillary pressure (P_d = 0); S_or is not part of the
reference model and is not represented.  Water enters through the whole top
face at S_w = 0.9 (S_n = S_N_GR = 0.1, SOURCE covering the face) with the
top pressure raised by 1e4 Pa (extension P_top_offset).  Other faces keep
the reference's rules (zero-gradient sides, hydrostatic bottom).  Initial
S_w = 0.15 (S_n_background = 0.85) and the reference's hydrostatic initial
pressure recurrence (two-phase.cpp:138-145).

Time step.  The scheme is explicit; its stability limit is set by pressure
diffusion, D = K k_r / (mu m beta).  dt = cfl * min over cells of
h^2 m mu_w beta_w / (6 K), with cfl = 0.4.  (A dt of 1 s diverges at the
64x64x32 workload in the reference scheme itself.)

Random fields.  Log-permeability is a Gaussian random field with exponential
covariance exp(-r/ell) (r in cells), generated by FFT circulant embedding on
a grid padded to twice the size, standardised to zero mean and unit variance
(G); ln K = ln 1e-12 + sigma G.  Porosity phi = 0.25 + 0.02 G clipped to
[0.1, 0.4].  Everything is seeded (numpy default_rng).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import native
from .native import Params


@dataclass
class Workload:
    name: str
    params: Params
    steps: int
    m: np.ndarray                 # porosity (NZ, NY, NX)
    K: np.ndarray | None          # permeability or None (uniform K0)
    notes: dict = field(default_factory=dict)

    @property
    def cells(self) -> int:
        return self.params.ncell


def grf(shape, ell: float, seed: int) -> np.ndarray:
    """Standardised Gaussian random field, exponential covariance, by FFT."""
    rng = np.random.default_rng(seed)
    pad = tuple(2 * s for s in shape)
    axes = [np.minimum(np.arange(n), n - np.arange(n)).astype(np.float64) for n in pad]
    r2 = np.zeros(pad, dtype=np.float64)
    for ax, a in enumerate(axes):
        sh = [1] * len(pad)
        sh[ax] = -1
        r2 = r2 + (a.reshape(sh)) ** 2
    cov = np.exp(-np.sqrt(r2) / ell)
    axes_all = tuple(range(len(pad)))
    lam = np.fft.rfftn(cov, axes=axes_all).real
    np.maximum(lam, 0.0, out=lam)
    del cov, r2
    noise = rng.standard_normal(pad)
    f = np.fft.irfftn(np.sqrt(lam) * np.fft.rfftn(noise, axes=axes_all), s=pad, axes=axes_all)
    g = f[tuple(slice(0, s) for s in shape)]
    g = (g - g.mean()) / g.std()
    return np.ascontiguousarray(g)


def stable_dt(p: Params, m: np.ndarray, K: np.ndarray | None, cfl: float = 0.4) -> float:
    h2 = min(p.hx, p.hy, p.hz if p.nz > 1 else p.hx) ** 2
    Kmax_ratio = (K / m).max() if K is not None else p.K0 / m.min()
    return float(cfl * h2 * p.mu_w * p.beta_w / (6.0 * Kmax_ratio))


def two_phase_params(nx_ref: int, ny_ref: int, nz_ref: int, form: int = native.FORM_FP64,
                     percell_k: bool = True) -> Params:
    """Workload fluids (config 0): mu 1e-3/5e-3, rho 1000/850, beta 1e-9,
    Brooks-Corey lambda = 2, S_wr = 0.1, no capillarity, h = 1 m."""
    from .simulation import default_params
    p = default_params()
    p.nx, p.ny, p.nz = nx_ref, ny_ref, nz_ref
    p.phases = 2
    p.form = form
    p.hx = p.hy = p.hz = 1.0
    p.mu_w, p.mu_n = 1e-3, 5e-3
    p.ro0_w, p.ro0_n = 1000.0, 850.0
    p.beta_w = p.beta_n = 1e-9
    p.lambda_ = 2.0
    p.S_wr = 0.1
    p.P_d = 0.0
    p.g_const = 9.81
    p.P_atm = 1e5
    p.K0 = 1e-12
    p.porosity = 0.3
    p.S_n_gr = 0.1                       # S_w = 0.9 injected at the top
    p.source = max(nx_ref, nz_ref)       # window covers the whole top face
    p.S_n_background = 0.85              # initial S_w = 0.15
    p.P_top_offset = 1e4
    p.newton_iterations = 10
    p.flags = native.FLAG_PERCELL_K if percell_k else 0
    return p


def config0(seed: int = 0) -> Workload:
    """64x64x32 (gravity on z), 100 steps, phi ~ N(0.3, 0.03^2) clipped to
    [0.15, 0.45] i.i.d., K = 1e-12 uniform."""
    nx, ny, nz = 64, 32, 64  # reference axes: NY = workload Nz (vertical)
    p = two_phase_params(nx, ny, nz, percell_k=False)
    rng = np.random.default_rng(seed)
    m = np.clip(0.3 + 0.03 * rng.standard_normal((nz, ny, nx)), 0.15, 0.45)
    p.dt = stable_dt(p, m, None)
    return Workload("cfg0 two-phase 64x64x32 fp64", p, 100, m, None,
                    {"workload_grid": [64, 64, 32], "ref_grid": [nx, ny, nz], "dt": p.dt})


def heterogeneous_fields(shape, sigma: float, ell: float, seed: int):
    g = grf(shape, ell, seed)
    lnk = math.log(1e-12) + sigma * g
    K = np.exp(lnk)
    m = np.clip(0.25 + 0.02 * g, 0.1, 0.4)
    return m, K


def config1(form: int = native.FORM_FP64, seed: int = 1, grid=(256, 256, 128), steps: int = 1000) -> Workload:
    """256x256x128 (gravity on z), 1000 steps, lognormal K (sigma 1, ell 8)."""
    Nx, Ny, Nz = grid
    nx, ny, nz = Nx, Nz, Ny
    p = two_phase_params(nx, ny, nz, form=form, percell_k=True)
    m, K = heterogeneous_fields((nz, ny, nx), 1.0, 8.0, seed)
    p.dt = stable_dt(p, m, K)
    return Workload(f"cfg1 two-phase {Nx}x{Ny}x{Nz} " + ("fp64" if form == native.FORM_FP64 else "fp32c"),
                    p, steps, m, K, {"workload_grid": list(grid), "ref_grid": [nx, ny, nz], "dt": p.dt,
                                     "sigma": 1.0, "ell": 8.0, "seed": seed})


def config3(form: int = native.FORM_FP32C, seed: int = 3, count: int = 64, dims=(32, 48, 64, 96, 128),
            steps: int = 300) -> list:
    """Ensemble: `count` two-phase instances, grid sizes drawn uniformly per
    axis from `dims`, each with its own seeded lognormal K (sigma in
    [0.5, 1.5], correlation length in [4, 16] cells), config-0 fluids and its
    own stable dt; 300 steps each."""
    rng = np.random.default_rng(seed)
    out = []
    for q in range(count):
        Nx, Ny, Nz = (int(v) for v in rng.choice(dims, 3))
        sigma = float(rng.uniform(0.5, 1.5))
        ell = float(rng.uniform(4.0, 16.0))
        nx, ny, nz = Nx, Nz, Ny
        p = two_phase_params(nx, ny, nz, form=form, percell_k=True)
        m, K = heterogeneous_fields((nz, ny, nx), sigma, ell, seed * 1000 + q)
        p.dt = stable_dt(p, m, K)
        out.append(Workload(f"cfg3[{q}] {Nx}x{Ny}x{Nz}", p, steps, m, K,
                            {"workload_grid": [Nx, Ny, Nz], "sigma": sigma, "ell": ell, "dt": p.dt}))
    return out


def config4(seed: int = 4, grid=(128, 128, 64), steps: int = 500, obs_every: int = 25,
            checkpoint_every: int = 50) -> Workload:
    """Inverse problem, 128x128x64 (gravity on z), FP64, 500 steps.  Truth:
    lognormal K (sigma 1, ell 8) and its porosity field (seeded).  Prior
    (the point where the gradient is taken): ln K = ln 1e-12, phi = 0.25.
    S_w observed on a 4x4 lattice of vertical columns (every vertical cell)
    every 25 steps: 16 x 64 x 20 = 20,480 observations; checkpoints every 50
    steps.  `m`/`K` hold the prior; notes hold the truth and the observation
    layout."""
    Nx, Ny, Nz = grid
    nx, ny, nz = Nx, Nz, Ny
    p = two_phase_params(nx, ny, nz, form=native.FORM_FP64, percell_k=True)
    m_true, K_true = heterogeneous_fields((nz, ny, nx), 1.0, 8.0, seed)
    m0 = np.full((nz, ny, nx), 0.25)
    K0 = np.full((nz, ny, nx), 1e-12)
    p.dt = min(stable_dt(p, m_true, K_true), stable_dt(p, m0, K0))
    ci = [nx // 8 + q * nx // 4 for q in range(4)]
    ck = [nz // 8 + q * nz // 4 for q in range(4)]
    obs = np.array([i + j * nx + k * nx * ny for i in ci for k in ck for j in range(ny)], dtype=np.int64)
    return Workload(f"cfg4 two-phase adjoint {Nx}x{Ny}x{Nz}", p, steps, m0, K0,
                    {"workload_grid": list(grid), "ref_grid": [nx, ny, nz], "dt": p.dt, "seed": seed,
                     "m_true": m_true, "K_true": K_true, "obs": obs, "obs_every": obs_every,
                     "checkpoint_every": checkpoint_every, "columns_i": ci, "columns_k": ck})


def observe(params: Params, m: np.ndarray, K: np.ndarray, obs: np.ndarray, obs_every: int, steps: int,
            device: int = 0) -> np.ndarray:
    """S_w at the observed cells every `obs_every` steps of a run from the
    reference initial state for porosity m (synthetic data of the truth)."""
    from .simulation import Simulation
    out = []
    with Simulation(params, device=device) as s:
        s.set_field("m", m)
        s.set_field("K", K)
        s.init_state()
        for _ in range(steps // obs_every):
            s.step(obs_every)
            out.append(1.0 - s.get_field("S_n").reshape(-1)[obs])
    return np.array(out)


def three_phase_params(nx_ref: int, ny_ref: int, nz_ref: int, percell_k: bool = True) -> Params:
    """Three-phase fluids (config 2): water / NAPL / gas densities 1000 / 850 /
    1.2 (ideal gas, rho_g = rho_0g P / P_atm), viscosities 1e-3 / 3e-3 /
    1.8e-5, residual saturations 0.1 / 0.05 / 0.02, the reference CPU
    relative permeabilities with A = 2 and no capillarity (three-phase.cpp:
    11-186), 7 Newton iterations; initial S_w = 0.2, S_n = 0.3; NAPL enters
    through a 3x3 window of the top face at S_n = 0.7 (S_w = 0.2)."""
    from .simulation import default_params
    p = default_params()
    p.nx, p.ny, p.nz = nx_ref, ny_ref, nz_ref
    p.phases = 3
    p.form = native.FORM_FP64
    p.hx = p.hy = p.hz = 1.0
    p.ro0_w, p.ro0_n, p.ro0_g = 1000.0, 850.0, 1.2
    p.mu_w, p.mu_n, p.mu_g = 1e-3, 3e-3, 1.8e-5
    p.beta_w = p.beta_n = 1e-9
    p.lambda_ = 2.0
    p.S_wr, p.S_nr, p.S_gr = 0.1, 0.05, 0.02
    p.S_w_init, p.S_n_init = 0.2, 0.3
    p.S_w_gr, p.S_n_gr = 0.2, 0.7
    p.source = 1                          # 3x3 window with CAPAZ_FLAG_SOURCE_WINDOW
    p.P_d = 0.0
    p.g_const = 9.81
    p.P_atm = 1e5
    p.K0 = 1e-12
    p.porosity = 0.25
    p.newton_iterations = 7
    p.flags = native.FLAG_SOURCE_WINDOW | (native.FLAG_PERCELL_K if percell_k else 0)
    return p


def config2(seed: int = 2, grid=(192, 192, 96), steps: int = 500) -> Workload:
    """192x192x96 (gravity on z) three-phase, 500 steps, FP64, lognormal K
    (sigma 1, ell 8) and its porosity field, 3x3 NAPL source on the top face."""
    Nx, Ny, Nz = grid
    nx, ny, nz = Nx, Nz, Ny
    p = three_phase_params(nx, ny, nz)
    m, K = heterogeneous_fields((nz, ny, nx), 1.0, 8.0, seed)
    p.dt = stable_dt(p, m, K)
    return Workload(f"cfg2 three-phase {Nx}x{Ny}x{Nz} fp64", p, steps, m, K,
                    {"workload_grid": list(grid), "ref_grid": [nx, ny, nz], "dt": p.dt, "sigma": 1.0, "ell": 8.0,
                     "seed": seed})
