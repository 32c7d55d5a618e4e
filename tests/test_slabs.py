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


@pytest.mark.gpu
@pytest.mark.parametrize("world", [2, 3])
def test_split_step_slabs_equal_whole_grid(world):
    """The overlapped slab step (capaz_step_split: edge planes and interior
    planes on two streams, float32 planes exchanged on the edge side while
    the interior sweep runs) with every slab holding the whole grid's
    reference state: bit-identical to one context stepping the whole grid."""
    import torch
    from capaz_b200 import Simulation
    nz, nsteps = 29, 17
    p = _params(nz)
    p.nx, p.form = 12, FORM_FP32C
    p.lambda_, p.P_d = 2.0, 0.0  # the TMA-staged sweep's model
    m = _porosity(p, 6)
    with Simulation(p) as whole:
        whole.set_field("m", m)
        whole.init_state()
        Pref, S_ref = whole.get_reference()
        whole.step(nsteps)
        want = {f: whole.get_field(f) for f in ("P_w", "S_n")}
    layouts = [SlabLayout(nz, r, world) for r in range(world)]
    sims = [Simulation(L.local_params(p)) for L in layouts]
    edge = [torch.cuda.Stream() for _ in sims]
    inner = [torch.cuda.Stream() for _ in sims]
    xchg = torch.cuda.Stream()
    n = p.nx * p.ny
    buf = {(r, f, side): torch.empty(n, dtype=torch.float32, device="cuda:0")
           for r in range(world) for f in ("P_w", "S_n") for side in ("lo", "hi")}
    try:
        for L, s in zip(layouts, sims):
            s.set_field("m", L.local(m))
            s.set_reference(Pref, S_ref)  # fixed before the state is encoded
            s.init_state()
        torch.cuda.synchronize()
        for _ in range(nsteps):
            for s, e, i in zip(sims, edge, inner):
                s.step_split(e.cuda_stream, i.cuda_stream)
            # the exchange: after every slab's edge sweep, before its next step
            for e in edge:
                xchg.wait_stream(e)
            xs = xchg.cuda_stream
            for r in range(world):
                L, s = layouts[r], sims[r]
                for f in ("P_w", "S_n"):
                    if L.lo:
                        s.get_plane_raw(f, L.own_lo, buf[(r, f, "lo")].data_ptr(), xs)
                    if L.hi:
                        s.get_plane_raw(f, L.own_hi, buf[(r, f, "hi")].data_ptr(), xs)
            for r in range(world):
                L, s = layouts[r], sims[r]
                for f in ("P_w", "S_n"):
                    if L.lo:
                        s.set_plane_raw(f, 0, buf[(r - 1, f, "hi")].data_ptr(), xs)
                    if L.hi:
                        s.set_plane_raw(f, L.nz_local - 1, buf[(r + 1, f, "lo")].data_ptr(), xs)
            for e in edge:
                e.wait_stream(xchg)
        torch.cuda.synchronize()
        got = {f: np.concatenate([L.owned(s.get_field(f)) for L, s in zip(layouts, sims)]) for f in ("P_w", "S_n")}
    finally:
        for s in sims:
            s.close()
    for f in ("P_w", "S_n"):
        assert np.array_equal(got[f], want[f]), f


@pytest.mark.gpu
def test_split_step_of_one_grid_matches_single_launch_steps():
    """capaz_step_split on an undivided grid (nothing to exchange), mixed
    with ordinary steps, reproduces ordinary steps bit for bit."""
    import torch
    from capaz_b200 import Simulation
    p = _params(21)
    p.nx, p.form = 16, FORM_FP32C
    p.lambda_, p.P_d = 2.0, 0.0
    m = _porosity(p, 7)
    out = []
    for plan in ("ssssss", "pppppp", "psspps"):
        with Simulation(p) as s:
            s.set_field("m", m)
            s.init_state()
            e, i = torch.cuda.Stream(), torch.cuda.Stream()
            for c in plan:
                if c == "s":
                    s.step(1)
                else:
                    torch.cuda.synchronize()
                    s.step_split(e.cuda_stream, i.cuda_stream)
                    torch.cuda.synchronize()
            out.append((s.get_field("P_w"), s.get_field("S_n")))
    for P, S in out[1:]:
        assert np.array_equal(P, out[0][0]) and np.array_equal(S, out[0][1])


def _reference_worker(rank, world, port, tmp):
    import torch.distributed as dist
    from capaz_b200.slabs import SlabLayout, shared_reference
    os.environ["MASTER_ADDR"], os.environ["MASTER_PORT"] = "127.0.0.1", str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    rng = np.random.default_rng(5)
    P = 1e5 + 1e3 * rng.standard_normal((19, 7, 8))
    S = rng.uniform(0.1, 0.9, (19, 7, 8))
    L = SlabLayout(19, rank, world)
    k0, k1 = L.k0, L.k1
    Pref, S_ref = shared_reference(P[k0:k1], S[k0:k1], "cpu")
    np.savez(os.path.join(tmp, f"ref{rank}.npz"), Pref=Pref, S_ref=S_ref, want=P.mean(axis=(0, 2)), wantS=S.mean())
    dist.destroy_process_group()


def test_shared_reference_is_the_whole_grids_on_every_rank(tmp_path):
    """The overlapped slabs' common reference state: every rank gets the
    same per-row mean pressure and mean saturation of the whole grid."""
    import torch.multiprocessing as mp
    world = 3
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    mp.start_processes(_reference_worker, args=(world, port, str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    parts = [np.load(os.path.join(tmp_path, f"ref{r}.npz")) for r in range(world)]
    for q in parts:
        assert np.array_equal(q["Pref"], parts[0]["Pref"]) and float(q["S_ref"]) == float(parts[0]["S_ref"])
        assert np.allclose(q["Pref"], q["want"], rtol=1e-13) and abs(float(q["S_ref"]) - float(q["wantS"])) < 1e-13
