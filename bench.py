"""Benchmark of the two-phase time step (cell-steps/s) on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form fp64|fp32c]
                    [--impl capaz|reference] [--grid NX NY NZ]

Workload: the 256x256x128 two-phase problem with gravity on z (reference axes
NX=256, NY=128 vertical, NZ=256; 8,388,608 cells), lognormal permeability
(sigma 1, correlation length 8 cells, seeded FFT field), porosity tied to it,
the workload fluids and boundary setup (capaz_b200/configs.py).  A step is
one time step of the whole grid.  With N GPUs every rank steps its own
replica of the grid (weak scaling; the step needs no data-path collective).

One JSON line on rank 0:
  value   cell-steps/s of the precision form (FP32 storage and stencil,
          FP64 Newton) over exactly K steps, state resident in HBM, CUDA
          events on the launching stream, max over ranks, summed over ranks;
          the plain FP64 path is timed the same way (`forms`), and both forms
          are run for the workload's 1000 steps from the same initial state to
          report the precision form's error against FP64 (`precision`);
  e2e     the same metric through the C ABI with host buffers: pinned-host
          float64 upload of the state (P_w, S_n, m, K), K steps each followed
          by a device->host read of that step's diagnostics (mass balance,
          Newton residual; posted after the step, waited for one step later),
          then download of (P_w, S_n), all timed, after one untimed pass of
          the same with W steps;
  roofline  algorithmic HBM bytes of one step divided by the step's time
          (CUDA events around the K steps; the precision form's step is its
          sweep kernel plus the small boundary kernel, the sweep taking ~90 %),
          against the measured copy bandwidth; `traffic`: the sweep's DRAM
          bytes per launch from the committed ncu summary;
  cpu_baseline  the OpenMP oracle (all host threads) on a bounded sample.
`--impl reference` times the reference's own CPU step (oracle/_ref) instead.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

# Algorithmic HBM bytes per cell-step of the fused step kernels: read the
# state and the media, write the state, with perfect halo reuse.
ALGO_BYTES = {
    ("fp64", True): 48,   # P_w, S_n, m, K read (32) + P_w, S_n written (16)
    ("fp64", False): 40,  # uniform K
    ("fp32c", True): 24,  # the same fields at 4 bytes
    ("fp32c", False): 20,
}
PUBLISHED_1GPU = 44.9e6  # reference's published 1-GPU two-phase step, 250^3, cell-steps/s


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="capaz", choices=["capaz", "reference"])
    ap.add_argument("--form", default=None, choices=[None, "fp64", "fp32c"])
    ap.add_argument("--grid", type=int, nargs=3, default=[256, 256, 128],
                    help="workload grid Nx Ny Nz, gravity on z")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-precision", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--forward-mode-fd-cells", type=int, default=0,
                    help="also run the FP64 forward mode along the first N central-difference cells of each field "
                         "(about 50 s of host time per cell)")
    ap.add_argument("--no-three-phase", action="store_true")
    ap.add_argument("--no-physics", action="store_true", help="skip the Buckley-Leverett and energy legs")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--decompose", action="store_true",
                    help="split the one grid into z-slabs over the N GPUs (strong scaling, NCCL halo "
                         "exchange every step) instead of one replica per GPU")
    return ap.parse_args()


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []
        self.proc = None
        self.t0 = self.t1 = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.samples.append((time.perf_counter(), line.strip()))

    def mark(self, begin: bool):
        if begin:
            self.t0 = time.perf_counter()
        else:
            self.t1 = time.perf_counter()

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for t, line in self.samples:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            rows.append((t, f))
        inside = [r for r in rows if self.t0 is not None and self.t0 - 0.15 <= r[0] <= (self.t1 or 1e30) + 0.15]
        use = inside if inside else rows
        sm = [float(f[1]) for _, f in use if f[1].replace(".", "").isdigit()]
        mx = [float(f[2]) for _, f in use if f[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, f in use for i in range(4) if f[5 + i].lower().startswith("active")})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples_in_region": len(inside), "samples": len(rows)}


# ---------------------------------------------------------------------------
def dist_setup():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime

        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        backend = "nccl"
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws, local=0):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier(device_ids=[local])


def reduce_max(x: float, ws: int) -> float:
    if ws == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def load_traffic(kernel: str, workload: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            d = json.load(f)
        e = d.get(kernel, {}).get(workload)
        return None if e is None else e
    except Exception:
        return None


def fp64_flops_per_cell(kernel: str):
    """FP64 operations per cell-step of an FP64 step kernel (DADD + DMUL +
    2 DFMA thread-instructions per launch / cells, from the committed ncu
    counts), keyed by kernel and relative-permeability form."""
    try:
        with open(os.path.join(ROOT, "profiles", "fp64_ops.json")) as f:
            return json.load(f).get(kernel)
    except Exception:
        return None


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ---------------------------------------------------------------------------
def cpu_baseline_port(w, nsteps: int = 2) -> dict:
    """The OpenMP oracle on the workload's full grid for a few steps."""
    from oracle import oracle as O
    p = w.params
    st = O.init(p, w.m)
    state = {"P_w": st["P_w"], "S_n": st["S_n"]}
    O.step(p, state, 1, w.m, w.K)  # page in, thread pool up
    t0 = time.perf_counter()
    O.step(p, state, nsteps, w.m, w.K)
    dt = time.perf_counter() - t0
    return {"value": p.ncell * nsteps / dt, "unit": "cell-steps/s", "cores": O.max_threads(), "kind": "port",
            "sample": f"{nsteps} steps of the full {p.nx}x{p.ny}x{p.nz} grid (FP64, bit-identical to the "
                      f"reference CPU step), {dt:.1f} s"}


def workload_config(grid, ws: int) -> dict:
    """The `config` object both arms print for the two-phase workload: the
    grid and what one step is.  What differs between the arms (the storage
    form, the media fields, dt) is reported beside it, not in it."""
    Nx, Ny, Nz = grid
    cells = Nx * Ny * Nz
    return {"workload": f"two-phase time step, {Nx}x{Ny}x{Nz} grid with gravity on z ({cells} cells); "
                        "one step = one time step of the whole grid",
            "grid_ref": [Nx, Nz, Ny], "cells": cells, "parallelism": f"replicas x{ws}",
            "l2": ("inputs larger than L2" if 24 * cells > 126e6 else "inputs smaller than L2 (not a roofline size)")
                  + f": every step reads and writes the whole state ({24 * cells / 1e6:.0f} MB in the "
                    f"FP32-storage form, {48 * cells / 1e6:.0f} MB in FP64; the GPU's L2 is 126 MB)"}


# The reference's CPU build, run as a subprocess: the harness that the oracle
# recipe (oracle/Makefile) links from the reference's own main.cpp, cpu.cpp and
# two-phase.cpp.  The arm writes its defines.ini itself so that nothing of this
# repository's package or oracle library is loaded into the process.
REF_BINARY_2PH = os.path.join(ROOT, "oracle", "_ref", "capaz_ref_2ph")
REF_MAX_STEPS = 12


def reference_ini(nx: int, ny: int, nz: int, dt: float) -> str:
    """defines.ini (KEY=value, the reference's read_defines format) for the
    workload's fluids on the reference model: mu 1e-3/5e-3 Pa s, rho
    1000/850 kg/m^3, beta 1e-9 1/Pa, Brooks-Corey lambda 2, S_wr 0.1, no
    capillary pressure, h = 1 m, K = 1e-12 m^2 and porosity 0.3 uniform (the
    reference model reads K_0 and M_0 only), S_n = 0.1 injected over the whole
    top face, 10 Newton iterations."""
    vals = [("NX", nx), ("NY", ny), ("NZ", nz), ("HX", 1.0), ("HY", 1.0), ("HZ", 1.0), ("DT", dt),
            ("TAU", 1e-7), ("L", 1e-4), ("C_W", 1500), ("C_N", 1000), ("C_G", 330),
            ("BETA_W", 1e-9), ("BETA_N", 1e-9), ("BETA_G", 9.2e-6), ("RO_W", 1000.0), ("RO_N", 850.0),
            ("RO_G", 1.4), ("MU_W", 1e-3), ("MU_N", 5e-3), ("MU_G", 1.84e-5), ("G_CONST", 9.81),
            ("P_ATM", 1e5), ("LAMBDA_0", 2.0), ("LAMBDA_1", 2.0), ("M_0", 0.3), ("M_1", 0.3),
            ("S_WR_0", 0.1), ("S_WR_1", 0.1), ("S_NR_0", 0.0), ("S_NR_1", 0.0), ("S_GR_0", 0.0),
            ("S_GR_1", 0.0), ("K_0", 1e-12), ("K_1", 1e-12), ("P_D_0", 0.0), ("P_D_1", 0.0),
            ("P_D_NW_0", 0.0), ("P_D_NW_1", 0.0), ("P_D_GN_0", 0.0), ("P_D_GN_1", 0.0),
            ("S_N_GR", 0.1), ("S_W_GR", 0.4), ("S_W_INIT", 0.4), ("S_N_INIT", 0.3),
            ("SOURCE", max(nx, nz)), ("ITERATIONS", 10), ("TIMEX", 100.0),
            ("SAVE_PLOTS", 1000000), ("PRINT_SCREEN", 1000000)]
    return "".join(f"{k}={v!r}\n" if isinstance(v, float) else f"{k}={v}\n" for k, v in vals)


def reference_cpu_step(grid, nsteps: int) -> dict:
    """Runs the reference's own CPU time step (single-threaded, as written) on
    the workload grid for `nsteps` steps from its data_initialization state.
    dt is 0.4 x the explicit scheme's stability bound for the uniform media,
    0.4 h^2 m mu_w beta / (6 K) = 0.02 s; the work per cell-step does not
    depend on it.  Returns the harness's own timing of the step loop."""
    import tempfile
    Nx, Ny, Nz = grid
    nx, ny, nz = Nx, Nz, Ny                       # reference axes: NY vertical
    dt = 0.4 * 1.0 * 0.3 * 1e-3 * 1e-9 / (6.0 * 1e-12)
    with tempfile.TemporaryDirectory() as wd:
        with open(os.path.join(wd, "defines.ini"), "w") as f:
            f.write(reference_ini(nx, ny, nz, dt))
        out = os.path.join(wd, "out.bin")
        t0 = time.perf_counter()
        res = subprocess.run([REF_BINARY_2PH, wd, str(nsteps), "-", out], capture_output=True, text=True)
        wall = time.perf_counter() - t0
        if res.returncode != 0:
            raise RuntimeError(f"reference step failed ({res.returncode}): {res.stderr[-500:]}")
        info = json.loads([ln for ln in res.stdout.splitlines() if ln.startswith("RESULT ")][-1][7:])
        S = np.fromfile(out, dtype=np.float64)[nx * ny * nz:]
    return {"cells": nx * ny * nz, "steps": nsteps, "seconds": info["seconds"], "wall": wall, "dt": dt,
            "finite": bool(np.isfinite(S).all())}


def run_reference(args) -> None:
    """The reference arm: the reference's own CPU time step on the workload's
    full grid, through its own code path (main.cpp's time_step_function over
    cpu.cpp and two-phase.cpp).  Rank 0 only; other ranks exit."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    K, W = args.steps, args.warmup
    line = {"impl": "reference", "metric": "cell-steps/s", "unit": "cell-steps/s", "higher_is_better": True,
            "n_gpus": args.gpus, "steps": K, "warmup": W, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic", "config": workload_config(args.grid, args.gpus)}
    if not os.path.exists(REF_BINARY_2PH):
        line["unavailable"] = "reference CPU binaries (oracle/_ref) were not built"
        print(json.dumps(line), flush=True)
        return
    # One step of the full grid takes seconds on one core: the run steps the
    # whole grid K + W times, at most REF_MAX_STEPS, and times every step.
    n = max(1, min(K + W, REF_MAX_STEPS))
    r = reference_cpu_step(args.grid, n)
    val = r["cells"] * n / r["seconds"]
    line.update({
        "value": val, "ms_per_step": 1e3 * r["seconds"] / n,
        "form": "f64 (the reference's CPU step, single-threaded as written)",
        "media": "uniform K 1e-12 and porosity 0.3 (the reference model has no per-cell K); the work per "
                 "cell-step does not depend on the values",
        "dt": r["dt"], "finite": r["finite"],
        "cpu_baseline": {"value": val, "unit": "cell-steps/s", "cores": 1, "kind": "reference",
                         "sample": f"{n} steps of the full {args.grid[0]}x{args.grid[1]}x{args.grid[2]} grid "
                                   f"with the reference's own CPU step, {r['seconds']:.1f} s step loop "
                                   f"({r['wall']:.1f} s with set-up)"},
        "e2e": {"value": val, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    })
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
def time_form(sim, K, W, stream, ws, local, clocks=None, repeats=0):
    """W untimed steps, then exactly K steps between two CUDA events on the
    launching stream; barrier + synchronize on both sides.  A step is the
    form's kernels for one time step (the precision form: the sweep and its
    boundary kernel), so the per-step time is also the kernels' time.  With
    `repeats`, that many more blocks of K steps are timed the same way
    afterwards (reported beside the measurement, with their median)."""
    import torch
    sh = stream.cuda_stream
    with torch.cuda.stream(stream):
        sim.step(W, stream=sh)
        stream.synchronize()
        barrier(ws, local)
        torch.cuda.synchronize()
        l0 = sim.launch_count
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if clocks:
            clocks.mark(True)
        start.record(stream)
        sim.step(K, stream=sh)
        end.record(stream)
        torch.cuda.synchronize()
        if clocks:
            clocks.mark(False)
        barrier(ws, local)
        launches = sim.launch_count - l0
        total_ms = start.elapsed_time(end)
        reps = []
        for _ in range(repeats):
            barrier(ws, local)
            torch.cuda.synchronize()
            start.record(stream)
            sim.step(K, stream=sh)
            end.record(stream)
            torch.cuda.synchronize()
            reps.append(reduce_max(start.elapsed_time(end), ws) / K)
    sim.sync()
    return {"total_ms": reduce_max(total_ms, ws), "kern_ms": total_ms / K, "launches": launches,
            "repeat_ms_per_step": reps}


def tma_applies(p) -> bool:
    """Whether the precision form of `p` runs the TMA-staged kernel (two-phase,
    nx % 4 == 0, no capillary pressure, lambda == 2, TMA not disabled)."""
    from capaz_b200 import native
    return (p.phases == 2 and p.nx % 4 == 0 and p.P_d == 0.0 and p.lambda_ == 2.0
            and not (p.flags & native.FLAG_NO_TMA))


def make_sim(w, form, dev, diag=False, flags=0):
    from capaz_b200 import Simulation, native
    p = w.params.copy()
    p.form = form
    p.flags |= flags
    if diag:
        p.flags |= native.FLAG_DIAGNOSTICS
    sim = Simulation(p, device=dev)
    sim.set_field("m", w.m)
    if w.K is not None:
        sim.set_field("K", w.K)
    sim.init_state()
    sim.sync()
    return sim


def precision_check(w, dev, steps):
    """Both forms from the same initial state for `steps` steps: per-field
    max-abs and relative-L2 error of the precision form against FP64."""
    from capaz_b200 import native
    out = {}
    init = None
    for name, form in (("fp64", native.FORM_FP64), ("fp32c", native.FORM_FP32C)):
        sim = make_sim(w, form, dev, diag=True)
        if init is None:
            init = {"P_w": sim.get_field("P_w"), "S_n": sim.get_field("S_n")}
        sim.step(steps)
        out[name] = {"P_w": sim.get_field("P_w"), "S_n": sim.get_field("S_n"), "diag": sim.diag()}
        sim.close()
    r = {"steps": steps, "against": "FP64 path (matches the reference CPU step to 1e-12)"}
    for f in ("S_n", "P_w"):
        a, b = out["fp32c"][f], out["fp64"][f]
        r[f] = {"max_abs": float(np.abs(a - b).max()),
                "rel_l2": float(np.linalg.norm((a - b).ravel()) / np.linalg.norm(b.ravel())),
                "max_change_over_run": float(np.abs(b - init[f]).max())}
    ds = [float(out["fp32c"]["diag"]["mass"][i] / out["fp64"]["diag"]["mass"][i] - 1.0) for i in range(2)]
    r["mass_rel_diff"] = ds
    r["newton_residual_fp32c"] = out["fp32c"]["diag"]["max_residual"]
    return r


def three_phase_leg(dev, steps: int = 200, warmup: int = 5) -> dict:
    """Three-phase step on the config-2 workload (192x192x96, gravity on z,
    lognormal K, 3x3 NAPL source): cell-steps/s of the plain FP64 path and of
    the precision form (FP32 storage and stencil, FP64 Newton) over `steps`
    steps with the state in HBM (CUDA events), the kernels' algorithmic HBM
    bytes (FP64: 64 B/cell-step, P_w, S_w, S_n, m, K read and P_w, S_w, S_n
    written; FP32: 32 B), and the precision form's error against the FP64
    path after the workload's 500 steps from the same initial state."""
    import torch

    from capaz_b200 import Simulation, native
    from capaz_b200.configs import config2
    w = config2()
    p = w.params
    peak, _ = measured_peaks()
    out = {"workload": f"cfg2 three-phase {w.notes['workload_grid']} (reference axes {w.notes['ref_grid']}), "
                       f"dt {p.dt:.3g} s, per-cell K, 3x3 top source"}
    final = {}
    for form, name, nbytes in ((native.FORM_FP64, "fp64", 64), (native.FORM_FP32C, "fp32c", 32),
                               (native.FORM_FP64, "fp64_products", 64)):
        q = p.copy()
        q.form = form
        if name == "fp64_products":
            q.flags |= native.FLAG_POW_PRODUCTS
        with Simulation(q, device=dev) as sim:
            sim.set_field("m", w.m)
            sim.set_field("K", w.K)
            sim.init_state()
            st = torch.cuda.Stream(device=dev)
            sim.step(warmup, st.cuda_stream)
            torch.cuda.synchronize()
            l0 = sim.launch_count
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            sim.step(steps, st.cuda_stream)
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / steps
            launches = sim.launch_count - l0
            # the workload's run from the initial state, for the precision comparison
            sim.init_state()
            sim.step(w.steps, st.cuda_stream)
            torch.cuda.synchronize()
            final[name] = {k: sim.get_field(k) for k in ("P_w", "S_w", "S_n")}
        gbs = nbytes * p.ncell / (ms * 1e-3) / 1e9
        out[name] = {"value": p.ncell / (ms * 1e-3), "unit": "cell-steps/s", "ms_per_step": ms, "steps": steps,
                     "launches": launches, "algorithmic_bytes_per_cell": nbytes, "achieved_gbs": gbs,
                     "hbm_frac": gbs / peak, "finite": bool(np.isfinite(final[name]["S_n"]).all())}
        fl = fp64_flops_per_cell("step3_fp64_kernel") if form == native.FORM_FP64 else None
        if fl:
            per = fl["products" if name == "fp64_products" else "pow"]
            out[name]["fp64_flops_per_cell"] = per
            out[name]["fp64_gflops"] = per * p.ncell / (ms * 1e-3) / 1e9
    out["value"], out["unit"], out["ms_per_step"] = out["fp64"]["value"], "cell-steps/s", out["fp64"]["ms_per_step"]
    out["speedup_fp32c_vs_fp64"] = out["fp32c"]["value"] / out["fp64"]["value"]
    prec = {"steps": w.steps, "against": "FP64 three-phase path (matches the reference CPU step to 1e-12)"}
    for k in ("P_w", "S_w", "S_n"):
        a, b = final["fp32c"][k], final["fp64"][k]
        prec[k] = {"max_abs": float(np.abs(a - b).max()),
                   "rel_l2": float(np.linalg.norm(a - b) / np.linalg.norm(b))}
    out["precision"] = prec
    for k in ("P_w", "S_w", "S_n"):
        a, b = final["fp64_products"][k], final["fp64"][k]
        out["fp64_products"][f"{k}_max_rel_vs_pow"] = float(np.abs(a - b).max() / np.abs(b).max())
    out["speedup_products_vs_pow"] = out["fp64_products"]["value"] / out["fp64"]["value"]
    out["kernel"] = ("step3_fp64_kernel (FP64: 13 pow per cell, or products and 4 sqrt with "
                     "CAPAZ_FLAG_POW_PRODUCTS; 7 Newton iterations with Gauss-Jordan); step3_fp32c_tma_kernel + "
                     "boundary3_kernel (TMA-staged FP32 stencil, one FP64 Newton step, Cramer's rule)")
    return out


def _leg_timing(sim, dev, steps: int, warmup: int):
    """ms per step of `sim` over `steps` steps after `warmup` (CUDA events on
    one stream) and the launches counted inside."""
    import torch
    st = torch.cuda.Stream(device=dev)
    sim.step(warmup, st.cuda_stream)
    torch.cuda.synchronize()
    l0 = sim.launch_count
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    sim.step(steps, st.cuda_stream)
    e1.record(st)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps, sim.launch_count - l0


def bl_leg(dev, steps: int = 200, warmup: int = 5) -> dict:
    """Buckley-Leverett task (the reference's B_L build) on a 1000x1000 plane
    (100 times the reference's 100x100), dt 2000 s, K = 1e-10 exp(v) with v a
    seeded Gaussian field (mean -1.5, sd 0.6, correlation 8 cells) standing in
    for the reference's noise.dat; the reference's fluids and wells.  GPU
    cell-steps/s with the state in HBM; cpu_baseline: the oracle (the
    restatement pinned to the reference) on a 200x200 sample, all host
    threads."""
    from capaz_b200 import Simulation
    from capaz_b200.configs import grf
    from capaz_b200.simulation import buckley_leverett_params
    p = buckley_leverett_params(nx=1000, ny=1000, nz=1, dt=2000.0)
    K = (1e-10 * np.exp(-1.5 + 0.6 * grf((p.ny, p.nx), 8.0, 7)))[None]
    with Simulation(p, device=dev) as sim:
        sim.set_field("K", K)
        sim.init_state()
        ms, launches = _leg_timing(sim, dev, steps, warmup)
        S = sim.get_field("S_n")
    out = {"workload": "Buckley-Leverett 1000x1000x1, dt 2000 s, lognormal K, reference wells and fluids, FP64",
           "value": p.ncell / (ms * 1e-3), "unit": "cell-steps/s", "ms_per_step": ms, "steps": steps,
           "launches": launches, "finite": bool(np.isfinite(S).all()),
           "kernel": "step_bl_tile_kernel + step_bl_boundary_kernel"}
    try:
        from oracle import oracle as O
        q = buckley_leverett_params(nx=200, ny=200, nz=1, dt=2000.0)
        Kq = (1e-10 * np.exp(-1.5 + 0.6 * grf((q.ny, q.nx), 8.0, 7)))[None]
        st = O.init(q)
        n = 100
        t0 = time.perf_counter()
        O.step(q, {"P_w": st["P_w"], "S_n": st["S_n"]}, n, st["m"], Kq)
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": q.ncell * n / sec, "unit": "cell-steps/s", "cores": O.max_threads(),
                               "kind": "port", "sample": f"200x200x1, {n} steps"}
    except Exception as e:  # the CPU figure is optional
        out["cpu_baseline"] = {"unavailable": str(e)}
    return out


def energy_leg(dev, steps: int = 100, warmup: int = 3) -> dict:
    """Three-phase with the energy equation (the reference's THREE_PHASE +
    ENERGY build) on the config-2 grid (192x192x96, gravity on z, lognormal
    K, 3x3 NAPL source), T = 285 K initially with 400 K / 273 K top and
    bottom rows.  GPU cell-steps/s; cpu_baseline: the oracle on a 32x24x32
    sample, all host threads (the reference has this build on the CPU only)."""
    from capaz_b200 import Simulation, native
    from capaz_b200.configs import config2, heterogeneous_fields, stable_dt, three_phase_params
    w = config2()
    p = w.params.copy()
    p.model = native.MODEL_ENERGY
    with Simulation(p, device=dev) as sim:
        sim.set_field("m", w.m)
        sim.set_field("K", w.K)
        sim.init_state()
        ms, launches = _leg_timing(sim, dev, steps, warmup)
        T = sim.get_field("T")
    out = {"workload": f"energy equation, cfg2 grid {w.notes['workload_grid']}, FP64, dt {p.dt:.3g} s",
           "value": p.ncell / (ms * 1e-3), "unit": "cell-steps/s", "ms_per_step": ms, "steps": steps,
           "launches": launches, "finite": bool(np.isfinite(T).all()),
           "kernel": "energy_{derive,velocity,balance,newton,boundary}_kernel"}
    try:
        from oracle import oracle as O
        q = three_phase_params(32, 24, 32)
        q.model = native.MODEL_ENERGY
        mq, Kq = heterogeneous_fields((q.nz, q.ny, q.nx), 1.0, 8.0, 2)
        q.dt = stable_dt(q, mq, Kq)
        st = O.init(q, mq)
        n = 50
        t0 = time.perf_counter()
        O.step(q, {k: st[k] for k in ("P_w", "S_w", "S_n", "P_n", "P_g", "T")}, n, mq, Kq)
        sec = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": q.ncell * n / sec, "unit": "cell-steps/s", "cores": O.max_threads(),
                               "kind": "port", "sample": f"32x24x32, {n} steps"}
    except Exception as e:  # the CPU figure is optional
        out["cpu_baseline"] = {"unavailable": str(e)}
    return out


def ensemble_leg(dev, steps: int = 300, warmup: int = 3) -> dict:
    """Batching form on the config-3 ensemble (64 two-phase instances, dims
    per axis from {32, 48, 64, 96, 128}, own lognormal K and dt each, 300
    steps): one persistent launch per step over all instances, the step
    pair replayed as a CUDA graph, tile shape, z-chunk and CTAs per SM autotuned;
    against the same 64 instances stepped one after another as separate
    contexts (precision form, and the plain FP64 path).  GPU time by CUDA
    events on one stream; aggregate cell-steps/s."""
    import torch

    from capaz_b200 import Ensemble, Simulation, native
    from capaz_b200.configs import config3
    ws = config3(form=native.FORM_FP32C)
    cells = sum(w.params.ncell for w in ws)
    st = torch.cuda.Stream(device=dev)

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    with Ensemble([w.params for w in ws], device=dev) as ens:
        for sim, w in zip(ens.instances, ws):
            sim.set_field("m", w.m)
            sim.set_field("K", w.K)
            sim.init_state()
        tune = ens.autotune(st.cuda_stream)
        ens.step(warmup, st.cuda_stream)
        torch.cuda.synchronize()
        l0 = ens.launch_count
        batch_ms = timed(lambda: ens.step(steps, st.cuda_stream))
        launches = ens.launch_count - l0
        finite = all(bool(np.isfinite(s.get_field("S_n")).all()) for s in ens.instances)

    def sequential(form):
        total = 0.0
        for w in ws:
            q = w.params.copy()
            q.form = form
            with Simulation(q, device=dev) as sim:
                sim.set_field("m", w.m)
                sim.set_field("K", w.K)
                sim.init_state()
                sim.step(warmup, st.cuda_stream)
                torch.cuda.synchronize()
                total += timed(lambda: sim.step(steps, st.cuda_stream))
        return total

    seq32 = sequential(native.FORM_FP32C)
    seq64 = sequential(native.FORM_FP64)
    rate = lambda ms: cells * steps / (ms * 1e-3)  # noqa: E731
    return {"workload": f"cfg3 ensemble, {len(ws)} instances, {cells} cells, {steps} steps, precision form",
            "value": rate(batch_ms), "unit": "cell-steps/s", "ms_per_step": batch_ms / steps,
            "launches": launches, "autotune": tune, "finite": finite,
            "sequential_fp32c": {"value": rate(seq32), "ms_per_step": seq32 / steps},
            "sequential_fp64": {"value": rate(seq64), "ms_per_step": seq64 / steps},
            "speedup_vs_sequential_fp32c": seq32 / batch_ms, "speedup_vs_sequential_fp64": seq64 / batch_ms}


def adjoint_leg(dev, fm_cells: int = 0) -> dict:
    """Differentiation form on the config-4 inverse problem (128x128x64,
    FP64, 500 steps, checkpoints every 50): time of one forward solve vs. one
    gradient (checkpointed forward + backward), and central differences of
    the misfit (steps 1e-6 and 1e-4 in ln K and in porosity) at 32 seeded
    random cells among those whose gradient is at least 1% of the largest.
    With fm_cells > 0 the FP64 forward mode also runs along the first fm_cells
    of those cells in each field, beside their central differences."""
    import torch

    from capaz_b200 import Adjoint, Simulation
    from capaz_b200.configs import config4, observe
    w = config4()
    p, obs, every = w.params, w.notes["obs"], w.notes["obs_every"]
    steps, cp = w.steps, w.notes["checkpoint_every"]
    data = observe(p, w.notes["m_true"], w.notes["K_true"], obs, every, steps, device=dev)

    def best_of(fn, reps=3):
        best, out = float("inf"), None
        for _ in range(reps):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            best = min(best, time.perf_counter() - t0)
        return best, out

    with Simulation(p, device=dev) as sim:
        sim.set_field("m", w.m)
        sim.set_field("K", w.K)

        def forward_solve():
            sim.init_state()
            sim.step(steps)
            sim.sync()
        t_fwd, _ = best_of(forward_solve)
        with Adjoint(sim, steps, obs, every, cp) as adj:
            adj.set_observations(data)
            t_grad, (J, (gK, gm)) = best_of(lambda: (adj.forward(), adj.backward()))

    def misfit(m, K):
        with Simulation(p, device=dev) as sim:
            sim.set_field("m", m)
            sim.set_field("K", K)
            with Adjoint(sim, steps, obs, every, steps) as adj:
                adj.set_observations(data)
                return adj.forward()

    # Central differences at the specified step 1e-6 and at 1e-4: at 1e-6 the
    # difference of two misfits (~1.6e-9, S moving ~1e-6 over the horizon) sits
    # near the rounding noise of the forward solves; 1e-4 lifts the signal 100x
    # while the truncation error stays O(h^2) ~ 1e-8 relative.
    steps_fd = (1e-6, 1e-4)
    rng = np.random.default_rng(32)
    fd_out = {}
    fd_cells = {}
    for which, g in (("lnK", gK), ("porosity", gm)):
        flat = np.abs(g).ravel()
        pool = np.flatnonzero(flat >= 1e-2 * flat.max())
        cells = rng.choice(pool, min(32, len(pool)), replace=False)
        ad = np.array([float(g.ravel()[l]) for l in cells])
        for h in steps_fd:
            fd = []
            for l in cells:
                mp, mq = w.m.copy().reshape(-1), w.m.copy().reshape(-1)
                Kp, Kq = w.K.copy().reshape(-1), w.K.copy().reshape(-1)
                if which == "lnK":
                    Kp[l] *= math.exp(h)
                    Kq[l] *= math.exp(-h)
                else:
                    mp[l] += h
                    mq[l] -= h
                fd.append((misfit(mp.reshape(w.m.shape), Kp.reshape(w.K.shape)) -
                           misfit(mq.reshape(w.m.shape), Kq.reshape(w.K.shape))) / (2 * h))
            fd = np.array(fd)
            for l, v in zip(cells[:fm_cells], fd[:fm_cells]):
                fd_cells.setdefault(which, {}).setdefault(int(l), {})[f"fd_h{h:g}"] = float(v)
            key = which if h == steps_fd[0] else f"{which}_h{h:g}"
            fd_out[key] = {"cells": len(cells), "step": h,
                           "rel_l2": float(np.linalg.norm(fd - ad) / np.linalg.norm(fd)),
                           "max_rel": float(np.max(np.abs(fd - ad) / np.abs(fd))), "pool_cells": int(len(pool))}
    # Forward mode at the full size: the oracle's FP64 tangent-linear run (the
    # restated reference step on dual numbers, through every Newton
    # iteration) along two of the central-difference directions, the cells
    # of the largest ln K and porosity gradients among the ones drawn, and
    # along one dense seeded direction in both fields.
    fwd = {}
    try:
        from oracle import oracle as O
        t0 = time.perf_counter()
        dirs = []
        for which, g in (("lnK", gK), ("porosity", gm)):
            flat = np.abs(g).ravel()
            l = int(np.argmax(flat))
            d = np.zeros(w.m.shape)
            d.reshape(-1)[l] = 1.0
            dirs.append((f"{which}_cell_{l}", d if which == "lnK" else None, d if which == "porosity" else None))
        rng_d = np.random.default_rng(44)
        dirs.append(("dense_both_fields", rng_d.standard_normal(w.m.shape), 0.01 * rng_d.standard_normal(w.m.shape)))
        for name, dl, dm in dirs:
            J_o, dJ = O.tangent(p, steps, w.m, w.K, obs, every, data, dlnK=dl, dm=dm)
            fwd["misfit_oracle"] = J_o
            fwd["misfit_rel_diff"] = abs(J - J_o) / abs(J_o)
            terms = np.concatenate([(gK * dl).ravel() if dl is not None else np.zeros(0),
                                    (gm * dm).ravel() if dm is not None else np.zeros(0)])
            ad = float(np.sum(terms))
            fwd[name] = {"adjoint": ad, "forward_mode": dJ, "rel_diff": abs(ad - dJ) / abs(dJ) if dJ else None}
        fwd["rel_diff_max"] = max(v["rel_diff"] for v in fwd.values() if isinstance(v, dict) and v["rel_diff"] is not None)
        # The central-difference cells themselves, each a unit direction.
        if fd_cells:
            per = {}
            for which, g in (("lnK", gK), ("porosity", gm)):
                for l, row in fd_cells.get(which, {}).items():
                    d = np.zeros(w.m.shape)
                    d.reshape(-1)[l] = 1.0
                    _, dJ = O.tangent(p, steps, w.m, w.K, obs, every, data, dlnK=d if which == "lnK" else None,
                                      dm=d if which == "porosity" else None)
                    ad = float(g.ravel()[l])
                    row.update({"adjoint": ad, "forward_mode": dJ, "rel_diff": abs(ad - dJ) / abs(dJ) if dJ else None})
                    per[f"{which}_cell_{l}"] = row
            fwd["fd_cells"] = per
            fwd["fd_cells_rel_diff_max"] = max(v["rel_diff"] for v in per.values() if v["rel_diff"] is not None)
        fwd["cpu_seconds"] = time.perf_counter() - t0
        fwd["threads"] = O.max_threads()
    except Exception as e:  # reported, never fatal
        fwd = {"failed": str(e)}
    h = steps_fd[0]
    return {"workload": f"cfg4 two-phase inverse problem {w.notes['workload_grid']}, FP64, {steps} steps, "
                        f"{len(obs)} observed cells every {every} steps, checkpoints every {cp}",
            "forward_ms": t_fwd * 1e3, "gradient_ms": t_grad * 1e3, "adjoint_over_forward": t_grad / t_fwd,
            "misfit": J, "fd_step": h, "fd": fd_out, "forward_mode": fwd,
            "timing": "wall clock around synchronised calls, best of 3; forward = data_initialization + "
                      "500 steps; gradient = checkpointed forward (misfit) + backward (recompute + reverse sweep)"}


def run_decomposed(args) -> None:
    """The workload's one grid split into z-slabs over the N ranks: every
    step is the slab step on each GPU plus one NCCL exchange of the boundary
    planes with the neighbours (capaz_b200/slabs.py).  value = cells of the
    whole grid x K / the slowest rank's time for the K steps."""
    import torch

    from capaz_b200 import native
    from capaz_b200.configs import config1
    from capaz_b200.slabs import SlabSimulation

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    form = args.form or "fp32c"
    w = config1(form=native.FORM_FP64, grid=tuple(args.grid))
    p = w.params.copy()
    p.form = {"fp64": native.FORM_FP64, "fp32c": native.FORM_FP32C}[form]
    group = None
    if ws == 1:
        import torch.distributed as dist
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        os.environ.setdefault("MASTER_PORT", "29533")
        dist.init_process_group("nccl", rank=0, world_size=1)
    slab = SlabSimulation(p, local, group)
    slab.set_global_field("m", w.m)
    slab.set_global_field("K", w.K)
    slab.init_state()
    slab.step(args.warmup)
    torch.cuda.synchronize()
    barrier(ws, local)
    l0 = slab.sim.launch_count
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    cs = torch.cuda.current_stream()
    e0.record()
    if slab.overlap:  # the split steps run on the slab's edge and interior streams
        slab.edge.wait_stream(cs)
        slab.interior.wait_stream(cs)
    slab.step(args.steps)
    if slab.overlap:
        cs.wait_stream(slab.edge)
        cs.wait_stream(slab.interior)
    e1.record()
    torch.cuda.synchronize()
    barrier(ws, local)
    ms = reduce_max(e0.elapsed_time(e1), ws)
    launches = slab.sim.launch_count - l0
    value = p.ncell * args.steps / (ms * 1e-3)
    S = slab.gather("S_n")
    if rank == 0:
        line = {"metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
                "higher_is_better": True, "scaling": "strong", "vs_baseline": value / PUBLISHED_1GPU,
                "dtype": "f64" if form == "fp64" else "f32 storage+stencil (compensated), f64 Newton",
                "data": "synthetic (seeded lognormal K and porosity fields)",
                "config": {"workload": f"two-phase {args.grid[0]}x{args.grid[1]}x{args.grid[2]} gravity on z, "
                                       f"lognormal K sigma 1 ell 8, form {form}, one grid in z-slabs",
                           "grid_ref": [p.nx, p.ny, p.nz], "cells": p.ncell, "form": form,
                           "parallelism": f"z-slabs x{ws} (one halo plane per neighbour; NCCL point-to-point "
                                          "exchange of P_w, S_n every step" +
                                          (", float32 planes on an edge stream while the interior sweep runs)"
                                           if slab.overlap else ")")},
                "gpu_launches": launches, "finite": bool(np.isfinite(S).all())}
        print(json.dumps(line), flush=True)
    slab.close()
    import torch.distributed as dist
    dist.destroy_process_group()


def run_capaz(args) -> None:
    import torch

    from capaz_b200 import Simulation, native
    from capaz_b200.configs import config1

    ws, rank, local = dist_setup()
    torch.cuda.set_device(local)
    dev = local
    forms = [args.form] if args.form else ["fp32c", "fp64"]
    head = forms[0]
    form_id = {"fp64": native.FORM_FP64, "fp32c": native.FORM_FP32C}
    K, W = args.steps, args.warmup
    w = config1(form=native.FORM_FP64, grid=tuple(args.grid))
    p = w.params
    ncell = p.ncell
    percell = w.K is not None
    stream = torch.cuda.Stream(device=dev)
    sh = stream.cuda_stream

    # ---- device-resident timing of each form --------------------------------
    timing = {}
    clk = None
    for f in forms:
        sim = make_sim(w, form_id[f], dev)
        clocks = None
        if f == head:
            clocks = Clocks(dev)
            clocks.start()
            time.sleep(0.3)
        timing[f] = time_form(sim, K, W, stream, ws, local, clocks, repeats=5 if f == head else 0)
        if clocks:
            clk = clocks.stop()
        sim.close()
    t = timing[head]
    value = ncell * K * ws / (t["total_ms"] * 1e-3)
    # The plain FP64 path with the lambda = 2 relative permeabilities as
    # products (CAPAZ_FLAG_POW_PRODUCTS), timed the same way.
    prod = None
    if "fp64" in forms:
        simq = make_sim(w, form_id["fp64"], dev, flags=native.FLAG_POW_PRODUCTS)
        tq = time_form(simq, K, W, stream, ws, local)
        simq.close()
        prod = {"value": ncell * K * ws / (tq["total_ms"] * 1e-3), "ms_per_step": tq["total_ms"] / K,
                "launches": tq["launches"]}
        fl = fp64_flops_per_cell("step2_fp64_kernel")
        if fl:
            prod["fp64_flops_per_cell"] = fl["products"]
            prod["fp64_gflops"] = fl["products"] * ncell / (tq["kern_ms"] * 1e-3) / 1e9

    # ---- precision of the precision form (1000 steps of the workload) -------
    prec = None
    if not args.no_precision and "fp32c" in forms and "fp64" in forms:
        prec = precision_check(w, dev, w.steps)

    # ---- three-phase form (config 2) -----------------------------------------
    three = None
    if not args.no_three_phase and ws == 1:
        try:
            three = three_phase_leg(dev)
        except Exception as e:  # reported, never fatal to the headline line
            three = {"failed": str(e)}

    # ---- Buckley-Leverett task and energy equation ---------------------------
    bl = energy = None
    if not args.no_physics and ws == 1:
        for name, fn in (("bl", bl_leg), ("energy", energy_leg)):
            try:
                r = fn(dev)
            except Exception as e:  # reported, never fatal to the headline line
                r = {"failed": str(e)}
            if name == "bl":
                bl = r
            else:
                energy = r

    # ---- batching form (config 3) --------------------------------------------
    ens = None
    if not args.no_ensemble and ws == 1:
        try:
            ens = ensemble_leg(dev)
        except Exception as e:  # reported, never fatal to the headline line
            ens = {"failed": str(e)}

    # ---- differentiation form (config 4) ------------------------------------
    adj = None
    if not args.no_adjoint and ws == 1:
        try:
            adj = adjoint_leg(dev, args.forward_mode_fd_cells)
        except Exception as e:  # reported, never fatal to the headline line
            adj = {"failed": str(e)}

    # ---- end to end through the C ABI with host buffers ---------------------
    e2e = None
    if not args.no_e2e:
        q = p.copy()
        q.form = form_id[head]
        q.flags |= native.FLAG_DIAGNOSTICS
        init = make_sim(w, native.FORM_FP64, dev)
        host = {k: torch.empty(w.m.shape, dtype=torch.float64, pin_memory=True) for k in ("P_w", "S_n", "m", "K")}
        host["P_w"].numpy()[...] = init.get_field("P_w")
        host["S_n"].numpy()[...] = init.get_field("S_n")
        host["m"].numpy()[...] = w.m
        host["K"].numpy()[...] = w.K
        init.close()
        out_P = torch.empty(w.m.shape, dtype=torch.float64, pin_memory=True)
        out_S = torch.empty(w.m.shape, dtype=torch.float64, pin_memory=True)
        sim2 = Simulation(q, device=dev)
        slots = native.DIAG_SLOTS

        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]

        def e2e_pass(nsteps):
            """Upload, nsteps steps with their diagnostics, download.  Each
            step's diagnostics are read one step behind: capaz_step_post_diag
            steps and posts them into a pinned ring slot (the sweep writes the
            slot itself), and the host waits for step i after step i + 1 has
            been queued, so the device never idles while the host reads.
            Events on the stream split the pass into upload, steps and
            download."""
            ev[0].record(stream)
            for name in ("m", "K", "P_w", "S_n"):
                native.check(sim2.lib.capaz_set_field(sim2.ctx, native.FIELDS[name], host[name].data_ptr(), sh),
                             sim2.ctx)
            ev[1].record(stream)
            for i in range(nsteps):
                sim2.step_post_diag(1, i % slots, stream=sh)
                if i > 0:
                    sim2.wait_diag((i - 1) % slots)
            ev[2].record(stream)
            sim2.wait_diag((nsteps - 1) % slots)
            native.check(sim2.lib.capaz_get_field(sim2.ctx, native.FIELDS["P_w"], out_P.data_ptr(), sh), sim2.ctx)
            native.check(sim2.lib.capaz_get_field(sim2.ctx, native.FIELDS["S_n"], out_S.data_ptr(), sh), sim2.ctx)
            ev[3].record(stream)

        # Warm-up pass (W steps): the context's first download allocates its
        # FP64 decode buffers; the timed pass starts from the same upload.
        e2e_pass(max(W, 1))
        torch.cuda.synchronize()
        barrier(ws, local)
        t0 = time.perf_counter()
        e2e_pass(K)
        e2e_s = time.perf_counter() - t0
        barrier(ws, local)
        e2e_s = reduce_max(e2e_s, ws)
        torch.cuda.synchronize()
        up_ms, loop_ms, down_ms = (ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]),
                                   ev[2].elapsed_time(ev[3]))
        h2d = 4 * ncell * 8
        d2h = 2 * ncell * 8 + K * 40
        e2e = {"value": ncell * K * ws / e2e_s, "unit": "cell-steps/s",
               "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
               "upload_ms": up_ms, "download_ms": down_ms, "step_with_diag_ms": loop_ms / K,
               "per_step_value": ncell * ws / (loop_ms * 1e-3 / K),
               "breakdown": "device-stream events: upload (4 float64 fields, encoded on the device) and download "
                            "(2 fields, decoded) once per pass; step_with_diag_ms = a step plus its posted "
                            "diagnostics read, what every further step costs; per_step_value = cells / that",
               "definition": "float64 pinned-host upload of P_w, S_n, m, K; K steps each followed by a "
                             "device-to-host read of that step's diagnostics (mass balance, Newton residual, "
                             "40 B into a pinned ring, waited for one step behind); float64 download of P_w, "
                             "S_n; wall clock around all of it"}
        sim2.close()

    # ---- roofline of the headline kernel -------------------------------------
    peak, peak_kind = measured_peaks()
    abytes = ALGO_BYTES[(head, percell)] * ncell
    achieved = abytes / (t["kern_ms"] * 1e-3) / 1e9
    kname = "step2_fp64_kernel" if head == "fp64" else (
        "step2_fp32c_tma_kernel + boundary_fp32c_kernel" if tma_applies(p) else "step2_fp32c_kernel")
    wl_key = f"{args.grid[0]}x{args.grid[1]}x{args.grid[2]}"
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": load_traffic(kname.split(" + ")[0], wl_key), "kernel": kname,
            "algorithmic_bytes_per_launch": abytes,
            "algorithmic_bytes_per_cell": ALGO_BYTES[(head, percell)],
            "kernel_ms": t["kern_ms"], "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"}

    # ---- CPU baselines: the reference's own step (one core, as written) and
    # the OpenMP oracle (all host threads), both on the full workload grid --
    cpu = cpu_port = None
    if rank == 0 and not args.no_cpu_baseline:
        try:
            r = reference_cpu_step(args.grid, 2)
            cpu = {"value": r["cells"] * r["steps"] / r["seconds"], "unit": "cell-steps/s", "cores": 1,
                   "kind": "reference",
                   "sample": f"{r['steps']} steps of the full {args.grid[0]}x{args.grid[1]}x{args.grid[2]} grid "
                             f"with the reference's own CPU step (oracle/_ref, uniform K), "
                             f"{r['seconds']:.1f} s step loop"}
        except Exception as e:  # the baseline is informative, never fatal
            cpu = {"value": None, "unit": "cell-steps/s", "cores": 1, "kind": "reference",
                   "sample": f"failed: {e}"}
        try:
            cpu_port = cpu_baseline_port(w)
        except Exception as e:  # the baseline is informative, never fatal
            cpu_port = {"value": None, "unit": "cell-steps/s", "cores": 0, "kind": "port",
                        "sample": f"failed: {e}"}

    if rank == 0:
        forms_out = {}
        for f, tt in timing.items():
            ab = ALGO_BYTES[(f, percell)] * ncell
            forms_out[f] = {"value": ncell * K * ws / (tt["total_ms"] * 1e-3), "ms_per_step": tt["total_ms"] / K,
                            "kernel_ms": tt["kern_ms"], "hbm_frac": ab / (tt["kern_ms"] * 1e-3) / 1e9 / peak,
                            "launches": tt["launches"]}
            fl = fp64_flops_per_cell("step2_fp64_kernel") if f == "fp64" else None
            if fl:
                rate = ncell / (tt["kern_ms"] * 1e-3)
                forms_out[f]["fp64_gflops"] = fl["pow"] * rate / 1e9
                forms_out[f]["fp64_flops_per_cell"] = fl["pow"]
                forms_out[f]["fp64_flops_source"] = "ncu DADD + DMUL + 2 DFMA per launch / cells (profiles/fp64_ops.json)"
        line = {
            "metric": "cell-steps/s", "value": value, "unit": "cell-steps/s", "n_gpus": ws, "steps": K,
            "warmup": W, "ms_per_step": t["total_ms"] / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": value / PUBLISHED_1GPU,
            "vs_baseline_source": "reference's published 1-GPU two-phase step, 250^3 grid, 44.9e6 cell-steps/s "
                                  "(Fermi-era GPU)",
            "dtype": "f64" if head == "fp64" else "f32 storage+stencil (compensated), f64 Newton",
            "data": "synthetic (seeded lognormal K and porosity fields)",
            "config": workload_config(args.grid, ws),
            "form": head, "dt": p.dt,
            "media": "lognormal K (sigma 1, correlation length 8 cells, seeded FFT field), porosity "
                     "0.25 + 0.02 G clipped to [0.1, 0.4]",
            "repeats": {"count": len(t["repeat_ms_per_step"]), "steps_each": K,
                        "ms_per_step": t["repeat_ms_per_step"],
                        "median_ms_per_step": (statistics.median(t["repeat_ms_per_step"])
                                               if t["repeat_ms_per_step"] else None),
                        "note": "further blocks of K steps timed the same way after the measurement"},
            "forms": forms_out,
            "speedup_fp32c_vs_fp64": (forms_out["fp32c"]["value"] / forms_out["fp64"]["value"]
                                      if "fp32c" in forms_out and "fp64" in forms_out else None),
            "fp64_products": prod,
            "precision": prec,
            "adjoint": adj,
            "three_phase": three,
            "ensemble": ens,
            "buckley_leverett": bl,
            "energy": energy,
            "roofline": roof, "cpu_baseline": cpu, "cpu_baseline_port": cpu_port,
            "e2e": e2e, "clocks": clk, "gpu_launches": t["launches"],
        }
        ref_v = cpu["value"] if cpu else None
        if ref_v:
            # Speed-ups over the reference's own CPU step timed in this run
            # (one core, as the reference is written): the headline form, the
            # plain FP64 form (the like-for-like arithmetic), and end to end.
            line["speedup_vs_reference_cpu"] = {
                "form_" + f: forms_out[f]["value"] / ref_v for f in forms_out}
            if e2e:
                line["speedup_vs_reference_cpu"]["e2e"] = e2e["value"] / ref_v
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.decompose:
        run_decomposed(args)
    else:
        run_capaz(args)


if __name__ == "__main__":
    main()
