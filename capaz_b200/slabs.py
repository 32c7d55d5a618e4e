"""z-slab decomposition of one grid over several GPUs (one process per GPU).

The reference splits its grid over MPI ranks (global_to_local_vars,
main.cpp; exchanges in mpi.cpp:113-294).  Here each rank owns a contiguous
range of z-planes (the reference's split: Nz/size planes each, the first
Nz % size ranks one more) plus one halo plane towards each neighbour.  Every
rank steps its slab with the ordinary single-GPU step (the injection window
placed by capaz_params.z_offset / nz_global); after each step the first and
last owned planes of the state go to the neighbours and theirs come into the
halo planes (one grouped point-to-point exchange per step through
torch.distributed: NCCL over NVLink between GPUs, gloo between CPU
processes).  Everything the step derives (P_n, rho, Xi, velocities) is
recomputed from the state in the halo, so the state is the only thing that
crosses.

The stepping object only needs step(n), get_plane(name, k, dst) and
set_plane(name, k, src) on tensors of nx*ny float64: `SlabSimulation` wraps a
GPU context; tests drive the same layout and exchange with other steppers.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .native import Params


def partition(nz: int, nranks: int) -> list[tuple[int, int]]:
    """Owned global planes [k0, k1) of each rank."""
    if nranks < 1 or nz < nranks:
        raise ValueError(f"cannot split {nz} planes over {nranks} ranks")
    base, rem = divmod(nz, nranks)
    out, k = [], 0
    for r in range(nranks):
        n = base + (1 if r < rem else 0)
        out.append((k, k + n))
        k += n
    return out


@dataclass
class SlabLayout:
    """Local grid of one rank: owned planes plus a halo plane towards each
    neighbour.  Local plane q is global plane z_offset + q."""
    nz_global: int
    rank: int
    nranks: int

    def __post_init__(self):
        self.k0, self.k1 = partition(self.nz_global, self.nranks)[self.rank]
        self.lo = self.rank > 0                 # halo plane below
        self.hi = self.rank < self.nranks - 1   # halo plane above
        self.z_offset = self.k0 - (1 if self.lo else 0)
        self.nz_local = (self.k1 - self.k0) + int(self.lo) + int(self.hi)
        self.own_lo = 1 if self.lo else 0                 # local index of the first owned plane
        self.own_hi = self.own_lo + (self.k1 - self.k0) - 1
        if self.nz_local < 3:
            raise ValueError(f"rank {self.rank}: a slab needs at least 3 local planes (has {self.nz_local})")

    def local_params(self, p: Params) -> Params:
        q = p.copy()
        q.nz = self.nz_local
        q.z_offset = self.z_offset
        q.nz_global = p.nz
        return q

    def local(self, a: np.ndarray) -> np.ndarray:
        """The slab (with halos) of a global (nz, ny, nx) array."""
        return np.ascontiguousarray(a[self.z_offset:self.z_offset + self.nz_local])

    def owned(self, a_local: np.ndarray) -> np.ndarray:
        """The owned planes of a local (nz_local, ny, nx) array."""
        return a_local[self.own_lo:self.own_hi + 1]


class HaloExchange:
    """After a step: send the first / last owned plane of every state field
    to the rank below / above and receive theirs into the halo planes, as one
    grouped batch of point-to-point operations."""

    def __init__(self, layout: SlabLayout, plane_size: int, fields, device, group=None):
        import torch
        self.layout, self.fields, self.group = layout, list(fields), group
        mk = lambda: torch.empty(plane_size, dtype=torch.float64, device=device)  # noqa: E731
        self.send = {(f, side): mk() for f in self.fields for side in ("lo", "hi")}
        self.recv = {(f, side): mk() for f in self.fields for side in ("lo", "hi")}

    def exchange(self, get_plane, set_plane) -> None:
        import torch.distributed as dist
        L = self.layout
        ops = []
        for f in self.fields:
            if L.lo:
                get_plane(f, L.own_lo, self.send[(f, "lo")])
                ops.append(dist.P2POp(dist.isend, self.send[(f, "lo")], L.rank - 1, self.group))
                ops.append(dist.P2POp(dist.irecv, self.recv[(f, "lo")], L.rank - 1, self.group))
            if L.hi:
                get_plane(f, L.own_hi, self.send[(f, "hi")])
                ops.append(dist.P2POp(dist.isend, self.send[(f, "hi")], L.rank + 1, self.group))
                ops.append(dist.P2POp(dist.irecv, self.recv[(f, "hi")], L.rank + 1, self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for f in self.fields:
            if L.lo:
                set_plane(f, 0, self.recv[(f, "lo")])
            if L.hi:
                set_plane(f, L.nz_local - 1, self.recv[(f, "hi")])


def reduce_diag(d: dict, device, group=None) -> dict:
    """Diagnostics of the whole grid from each rank's slab diagnostics (the
    reference's global checks after its MPI exchanges): one all-reduce of the
    phase masses and non-finite counts (sum) and one of the largest Newton
    residual (max).  A slab's diagnostics cover its local interior cells,
    which are exactly its owned interior cells (halo planes are local
    boundary planes), so the sums count every interior cell of the grid once."""
    import torch
    import torch.distributed as dist
    sums = torch.tensor(list(d["mass"]) + [d["nonfinite_cells"]], dtype=torch.float64, device=device)
    mx = torch.tensor([d["max_residual"]], dtype=torch.float64, device=device)
    dist.all_reduce(sums, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(mx, op=dist.ReduceOp.MAX, group=group)
    v = sums.cpu().tolist()
    return {"mass": v[:3], "max_residual": float(mx.cpu().item()), "nonfinite_cells": v[3]}


def state_fields(p: Params) -> list[str]:
    return ["P_w", "S_n"] + (["S_w", "P_n", "P_g"] if p.phases == 3 else [])


def overlap_applies(p: Params) -> bool:
    """Whether a slab of `p` steps with capaz_step_split and exchanges its
    halo while the interior sweep runs (the two-phase precision form with
    the TMA-staged sweep, no diagnostics)."""
    from . import native
    return (p.phases == 2 and p.form == native.FORM_FP32C and p.nx % 4 == 0 and p.P_d == 0.0 and
            p.lambda_ == 2.0 and not (p.flags & (native.FLAG_NO_TMA | native.FLAG_DIAGNOSTICS)))


def shared_reference(P_owned: np.ndarray, S_owned: np.ndarray, device, group=None):
    """The precision form's reference state of the whole grid from every
    rank's owned planes (nz_own, ny, nx): per-row means of P_w and the mean of
    S_n, by all-reduces of sums and counts, so every rank holds the same."""
    import torch
    import torch.distributed as dist
    rows = torch.from_numpy(np.ascontiguousarray(P_owned.sum(axis=(0, 2)))).to(device)
    tot = torch.tensor([float(S_owned.sum()), float(S_owned.size), float(P_owned.shape[0] * P_owned.shape[2])],
                       dtype=torch.float64, device=device)
    dist.all_reduce(rows, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(tot, op=dist.ReduceOp.SUM, group=group)
    t = tot.cpu().tolist()
    return rows.cpu().numpy() / t[2], t[0] / t[1]


class SlabSimulation:
    """One rank's slab of a decomposed grid on its GPU (torch.distributed
    initialised with the NCCL backend, one process per GPU).

    In the two-phase precision form every step is capaz_step_split: the
    slab's edge planes are swept on one stream and sent to the neighbours
    (float32 deviations, grouped NCCL send/recv) while the interior planes
    are swept on another; the received planes land in the halo planes before
    the next step reads them.  All ranks share one reference state, so the
    planes cross unchanged.  Other forms step, then exchange float64 planes."""

    def __init__(self, params: Params, device: int, group=None, overlap=None):
        import torch
        import torch.distributed as dist

        from .simulation import Simulation
        self.rank, self.nranks = dist.get_rank(group), dist.get_world_size(group)
        self.global_params = params.copy()
        self.layout = SlabLayout(params.nz, self.rank, self.nranks)
        self.params = self.layout.local_params(params)
        self.sim = Simulation(self.params, device=device)
        self.device = torch.device("cuda", device)
        self.stream = torch.cuda.current_stream(self.device).cuda_stream
        self.fields = state_fields(params)
        self.group = group
        self.overlap = overlap_applies(params) if overlap is None else bool(overlap)
        if self.overlap:
            n = params.nx * params.ny
            self.edge = torch.cuda.Stream(self.device)
            self.interior = torch.cuda.Stream(self.device)
            mk = lambda: torch.empty(n, dtype=torch.float32, device=self.device)  # noqa: E731
            self.send = {(f, side): mk() for f in self.fields for side in ("lo", "hi")}
            self.recv = {(f, side): mk() for f in self.fields for side in ("lo", "hi")}
        else:
            self.halo = HaloExchange(self.layout, params.nx * params.ny, self.fields, self.device, group)

    def _get(self, f, k, t):
        self.sim.get_plane(f, k, t.data_ptr(), self.stream)

    def _set(self, f, k, t):
        self.sim.set_plane(f, k, t.data_ptr(), self.stream)

    def set_global_field(self, name: str, a: np.ndarray) -> None:
        self.sim.set_field(name, self.layout.local(np.asarray(a, dtype=np.float64)))

    def init_state(self) -> None:
        self.sim.init_state()
        if self.overlap:
            self.share_reference()

    def share_reference(self) -> None:
        """Gives every rank the whole grid's reference state (collective)."""
        Pref, S_ref = shared_reference(self.owned_field("P_w"), self.owned_field("S_n"), self.device, self.group)
        self.sim.set_reference(Pref, S_ref)

    def _exchange_raw(self) -> None:
        """The halo exchange of one split step, queued on the edge stream."""
        import torch
        import torch.distributed as dist
        L, es = self.layout, self.edge.cuda_stream
        with torch.cuda.stream(self.edge):
            ops = []
            for f in self.fields:
                if L.lo:
                    self.sim.get_plane_raw(f, L.own_lo, self.send[(f, "lo")].data_ptr(), es)
                    ops.append(dist.P2POp(dist.isend, self.send[(f, "lo")], L.rank - 1, self.group))
                    ops.append(dist.P2POp(dist.irecv, self.recv[(f, "lo")], L.rank - 1, self.group))
                if L.hi:
                    self.sim.get_plane_raw(f, L.own_hi, self.send[(f, "hi")].data_ptr(), es)
                    ops.append(dist.P2POp(dist.isend, self.send[(f, "hi")], L.rank + 1, self.group))
                    ops.append(dist.P2POp(dist.irecv, self.recv[(f, "hi")], L.rank + 1, self.group))
            if ops:
                for req in dist.batch_isend_irecv(ops):
                    req.wait()  # the edge stream waits; the host does not
            for f in self.fields:
                if L.lo:
                    self.sim.set_plane_raw(f, 0, self.recv[(f, "lo")].data_ptr(), es)
                if L.hi:
                    self.sim.set_plane_raw(f, L.nz_local - 1, self.recv[(f, "hi")].data_ptr(), es)

    def step(self, nsteps: int = 1) -> None:
        for _ in range(nsteps):
            if self.overlap:
                self.sim.step_split(self.edge.cuda_stream, self.interior.cuda_stream)
                self._exchange_raw()
            else:
                self.sim.step(1, self.stream)
                self.halo.exchange(self._get, self._set)

    def synchronize(self) -> None:
        import torch
        torch.cuda.synchronize(self.device)

    def diag(self) -> dict:
        """Diagnostics of the last step over the whole grid (needs
        FLAG_DIAGNOSTICS; every rank calls it)."""
        return reduce_diag(self.sim.diag(self.stream), self.device, self.group)

    def owned_field(self, name: str) -> np.ndarray:
        if self.overlap:
            self.synchronize()
        return self.layout.owned(self.sim.get_field(name))

    def gather(self, name: str):
        """The global field on rank 0 (None elsewhere): each rank sends its
        owned planes to rank 0."""
        import torch
        import torch.distributed as dist
        parts = partition(self.global_params.nz, self.nranks)
        shape = (self.global_params.ny, self.global_params.nx)
        mine = torch.from_numpy(np.ascontiguousarray(self.owned_field(name))).to(self.device)
        if self.rank != 0:
            dist.send(mine, 0, group=self.group)
            return None
        out = [mine]
        for r in range(1, self.nranks):
            k0, k1 = parts[r]
            buf = torch.empty((k1 - k0,) + shape, dtype=torch.float64, device=self.device)
            dist.recv(buf, r, group=self.group)
            out.append(buf)
        return torch.cat(out).cpu().numpy()

    def close(self) -> None:
        self.sim.close()
