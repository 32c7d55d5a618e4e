"""z-slab decomposition (capaz_b200/slabs.py): the partition and local
layout, the halo exchange over torch.distributed point-to-point, and the
stepped result against the undecomposed grid.

On the CPU the ranks are gloo processes whose slabs step with the oracle
(world sizes 2 and 3); on the GPU the slabs are contexts of one process whose
halo planes are exchanged by device copies (a run here has one GPU, and NCCL
needs one GPU per rank)."""
import os
import socket

import numpy as np
import pytest

from capaz_b200 import native
from capaz_b200.native import FORM_FP32C, FORM_FP64
from capaz_b200.slabs import HaloExchange, SlabLayout, partition, reduce_diag, state_fields
from capaz_b200.simulation import default_params


def test_partition_matches_the_reference_split():
    assert partition(10, 3) == [(0, 4), (4, 7), (7, 10)]
    assert partition(9, 3) == [(0, 3), (3, 6), (6, 9)]
    L = SlabLayout(10, 1, 3)
    assert (L.z_offset, L.nz_local, L.own_lo, L.own_hi) == (3, 5, 1, 3)
    L0, L2 = SlabLayout(10, 0, 3), SlabLayout(10, 2, 3)
    assert (L0.z_offset, L0.nz_local, L0.own_lo, L0.own_hi) == (0, 5, 0, 3)
    assert (L2.z_offset, L2.nz_local, L2.own_lo, L2.own_hi) == (6, 4, 1, 3)
    with pytest.raises(ValueError):
        SlabLayout(4, 0, 4)  # one owned plane and one halo: too thin


def _params(nz):
    # a 5x5 injection window centred in the global grid: slabs must place it
    return default_params(nx=11, ny=9, nz=nz, dt=2e-3, source=2, S_n_gr=0.3, P_top_offset=5e3,
                          S_n_background=0.1)


def _porosity(p, seed):
    return np.clip(0.3 + 0.02 * np.random.default_rng(seed).standard_normal((p.nz, p.ny, p.nx)), 0.2, 0.4)


class OracleSlab:
    """A slab stepped by the oracle (FP64 restatement of the reference)."""

    def __init__(self, p, layout, m):
        from oracle import oracle as O
        self.O, self.p, self.m = O, layout.local_params(p), layout.local(m)
        st = O.init(self.p, self.m)
        self.state = {"P_w": st["P_w"], "S_n": st["S_n"]}

    def step(self):
        self.state = self.O.step(self.p, self.state, 1, self.m)

    def get_plane(self, f, k, t):
        import torch
        t.copy_(torch.from_numpy(self.state[f][k].reshape(-1).copy()))

    def set_plane(self, f, k, t):
        self.state[f][k] = t.numpy().reshape(self.state[f][k].shape)


def _gloo_rank(rank, world, port, nz, nsteps, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = _params(nz)
        m = _porosity(p, 3)
        L = SlabLayout(nz, rank, world)
        slab = OracleSlab(p, L, m)
        halo = HaloExchange(L, p.nx * p.ny, state_fields(p), "cpu")
        for t in range(nsteps):
            if t == nsteps - 1:
                # the last step with diagnostics, reduced over the ranks
                q = slab.p.copy()
                q.flags |= native.FLAG_DIAGNOSTICS
                r = slab.O.step(q, slab.state, 1, slab.m, diag=True)
                slab.state = {k: r[k] for k in slab.state}
                d = reduce_diag(r["diag"], "cpu")
            else:
                slab.step()
            halo.exchange(slab.get_plane, slab.set_plane)
        np.savez(os.path.join(out, f"r{rank}.npz"), P=L.owned(slab.state["P_w"]), S=L.owned(slab.state["S_n"]),
                 mass=np.array(d["mass"]), rmax=d["max_residual"], nonfinite=d["nonfinite_cells"])
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_decomposed_oracle_equals_whole_grid(tmp_path, world):
    import torch.multiprocessing as mp
    from oracle import oracle as O
    nz, nsteps = 14, 12
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    mp.start_processes(_gloo_rank, args=(world, port, nz, nsteps, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    p = _params(nz)
    m = _porosity(p, 3)
    st = O.init(p, m)
    ref = O.step(p, {"P_w": st["P_w"], "S_n": st["S_n"]}, nsteps, m)
    parts = [np.load(os.path.join(tmp_path, f"r{r}.npz")) for r in range(world)]
    P = np.concatenate([q["P"] for q in parts])
    S = np.concatenate([q["S"] for q in parts])
    assert np.array_equal(P, ref["P_w"]) and np.array_equal(S, ref["S_n"])
    # global diagnostics: every rank holds the same reduction, equal to the
    # whole grid's up to the order of the sums
    q = p.copy()
    q.flags |= native.FLAG_DIAGNOSTICS
    whole = O.step(q, {"P_w": st["P_w"], "S_n": st["S_n"]}, nsteps, m, diag=True)["diag"]
    for part in parts:
        for a in range(2):
            assert abs(part["mass"][a] - whole["mass"][a]) <= 1e-12 * abs(whole["mass"][a])
        assert float(part["rmax"]) == whole["max_residual"]
        assert float(part["nonfinite"]) == whole["nonfinite_cells"] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("form,world", [(FORM_FP64, 3), (FORM_FP32C, 2)])
def test_decomposed_gpu_slabs_equal_whole_grid(form, world):
    """Slab contexts of one process, halo planes moved by device copies
    through capaz_get_plane / capaz_set_plane, against one context on the
    whole grid: bit-identical in FP64; within the precision form's storage
    rounding for FP32C (each slab has its own reference state)."""
    import torch
    from capaz_b200 import Simulation
    nz, nsteps = 22, 15
    p = _params(nz)
    p.nx = 12  # the precision form's TMA path needs nx % 4 == 0
    p.form = form
    m = _porosity(p, 4)
    with Simulation(p) as whole:
        whole.set_field("m", m)
        whole.init_state()
        whole.step(nsteps)
        want = {f: whole.get_field(f) for f in ("P_w", "S_n")}
    layouts = [SlabLayout(nz, r, world) for r in range(world)]
    sims = [Simulation(L.local_params(p)) for L in layouts]
    buf = torch.empty(p.nx * p.ny, dtype=torch.float64, device="cuda:0")
    try:
        for L, s in zip(layouts, sims):
            s.set_field("m", L.local(m))
            s.init_state()
        for _ in range(nsteps):
            for s in sims:
                s.step(1)
            for r in range(world - 1):  # plane exchange between ranks r and r+1
                a, b, La, Lb = sims[r], sims[r + 1], layouts[r], layouts[r + 1]
                for f in ("P_w", "S_n"):
                    a.get_plane(f, La.own_hi, buf.data_ptr())
                    b.set_plane(f, 0, buf.data_ptr())
                    b.get_plane(f, Lb.own_lo, buf.data_ptr())
                    a.set_plane(f, La.nz_local - 1, buf.data_ptr())
        got = {f: np.concatenate([L.owned(s.get_field(f)) for L, s in zip(layouts, sims)]) for f in ("P_w", "S_n")}
    finally:
        for s in sims:
            s.close()
    for f in ("P_w", "S_n"):
        if form == FORM_FP64:
            assert np.array_equal(got[f], want[f]), f
        else:
            assert np.linalg.norm(got[f] - want[f]) <= 1e-7 * np.linalg.norm(want[f]), f
