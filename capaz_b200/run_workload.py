"""Runs one of the benchmark workloads for a few steps: a small, fixed
command line to time or profile a single step kernel (ncu, nvidia-smi).

    python -m capaz_b200.run_workload WORKLOAD [--steps N] [--warmup W]
                                      [--pow-products] [--no-tma] [--tile 16|32] [--diag]

Workloads (gravity on z, the workloads of capaz_b200.configs):
  two-phase-fp32c    256x256x128 two-phase, precision form
  two-phase-fp64     256x256x128 two-phase, plain FP64
  three-phase-fp32c  192x192x96 three-phase, precision form
  three-phase-fp64   192x192x96 three-phase, plain FP64
Each run sets the media, builds the initial state on the device, steps
`warmup` steps, synchronises, steps `steps` steps and prints the time of the
latter (CUDA events) and the kernel launches it made.  With --diag every
step reduces the step diagnostics (CAPAZ_FLAG_DIAGNOSTICS, one step per call).
"""
from __future__ import annotations

import argparse
import json

from . import native
from .configs import config1, config2
from .simulation import Simulation

WORKLOADS = {
    "two-phase-fp32c": (config1, native.FORM_FP32C),
    "two-phase-fp64": (config1, native.FORM_FP64),
    "three-phase-fp32c": (config2, native.FORM_FP32C),
    "three-phase-fp64": (config2, native.FORM_FP64),
}


def main(argv=None) -> dict:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("workload", choices=sorted(WORKLOADS))
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--pow-products", action="store_true", help="CAPAZ_FLAG_POW_PRODUCTS (FP64 forms)")
    ap.add_argument("--no-tma", action="store_true", help="CAPAZ_FLAG_NO_TMA (precision forms)")
    ap.add_argument("--tile", type=int, default=16, help="rows of the two-phase precision sweep's tile")
    ap.add_argument("--diag", action="store_true", help="diagnostics reduced on every step")
    a = ap.parse_args(argv)
    import torch

    make, form = WORKLOADS[a.workload]
    w = make()
    p = w.params.copy()
    p.form = form
    if a.pow_products:
        p.flags |= native.FLAG_POW_PRODUCTS
    if a.no_tma:
        p.flags |= native.FLAG_NO_TMA
    if a.diag:
        p.flags |= native.FLAG_DIAGNOSTICS

    def run(n):
        if a.diag:
            for _ in range(n):
                s.step(1)
        else:
            s.step(n)

    with Simulation(p) as s:
        s.set_field("m", w.m)
        if w.K is not None:
            s.set_field("K", w.K)
        if a.tile != 16:
            s.set_sweep_tile(a.tile)
        s.init_state()
        run(a.warmup)
        s.sync()
        l0 = s.launch_count
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        run(a.steps)
        e1.record()
        s.sync()
        out = {"workload": a.workload, "cells": p.ncell, "steps": a.steps, "ms_per_step": e0.elapsed_time(e1) / max(a.steps, 1),
               "launches": s.launch_count - l0, "flags": p.flags}
    print(json.dumps(out), flush=True)
    return out


if __name__ == "__main__":
    main()
