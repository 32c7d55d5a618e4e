"""Ensembles: one persistent launch per step over uneven instances, graph
replay and autotuning, against each instance stepped on its own."""
import numpy as np
import pytest

from capaz_b200 import Ensemble, Simulation, native
from capaz_b200.configs import config3

pytestmark = pytest.mark.gpu


def setup(sim, w):
    sim.set_field("m", w.m)
    sim.set_field("K", w.K)
    sim.init_state()


@pytest.mark.parametrize("form", [native.FORM_FP64, native.FORM_FP32C])
def test_batch_matches_individual_runs(form):
    ws = config3(form=form, seed=5, count=7, dims=(32, 36, 48), steps=25)
    with Ensemble([w.params for w in ws]) as ens:
        for sim, w in zip(ens.instances, ws):
            setup(sim, w)
        l0 = ens.launch_count
        ens.step(25)  # odd: graph pairs plus one plain launch
        # the precision form's step is the sweep plus its boundary kernel
        assert ens.launch_count - l0 == 25 * (2 if form == native.FORM_FP32C else 1)
        got = [(s.get_field("P_w"), s.get_field("S_n")) for s in ens.instances]
    for w, (P, S) in zip(ws, got):
        with Simulation(w.params) as s:
            setup(s, w)
            s.step(25)
            assert np.array_equal(s.get_field("P_w"), P)
            assert np.array_equal(s.get_field("S_n"), S)


def test_batch_autotune_keeps_state():
    ws = config3(form=native.FORM_FP32C, seed=6, count=5, dims=(32, 64), steps=10)
    with Ensemble([w.params for w in ws]) as ens:
        for sim, w in zip(ens.instances, ws):
            setup(sim, w)
        before = [s.get_field("S_n") for s in ens.instances]
        choice = ens.autotune()
        assert choice["zchunk"] in (8, 16, 32, 64) and choice["ctas_per_sm"] >= 1
        assert choice["tile"] in ([32, 16], [32, 32])
        after = [s.get_field("S_n") for s in ens.instances]
        for a, b in zip(before, after):
            assert np.array_equal(a, b)
        ens.step(10)
        got = [s.get_field("S_n") for s in ens.instances]
    for w, S in zip(ws, got):
        with Simulation(w.params) as s:
            setup(s, w)
            s.step(10)
            assert np.array_equal(s.get_field("S_n"), S)


@pytest.mark.parametrize("tile_y,zchunk,per", [(16, 16, 0), (32, 16, 0), (32, 8, 1), (16, 64, 2)])
def test_batch_tile_shapes_match_individual_runs(tile_y, zchunk, per):
    """Every sweep tile shape the autotuner chooses among (32 x 16 and
    32 x 32 cells) gives each instance exactly its own run's result."""
    ws = config3(form=native.FORM_FP32C, seed=8, count=6, dims=(32, 40, 68), steps=9)
    with Ensemble([w.params for w in ws]) as ens:
        for sim, w in zip(ens.instances, ws):
            setup(sim, w)
        ens.set_tuning(zchunk, per, tile_y)
        assert ens.tuning() == {"zchunk": zchunk, "ctas_per_sm": per, "tile": [32, tile_y]}
        ens.step(9)
        got = [(s.get_field("P_w"), s.get_field("S_n")) for s in ens.instances]
    for w, (P, S) in zip(ws, got):
        with Simulation(w.params) as s:
            setup(s, w)
            s.step(9)
            assert np.array_equal(s.get_field("P_w"), P)
            assert np.array_equal(s.get_field("S_n"), S)


def test_sweep_tile_of_one_grid_is_bit_identical():
    """The precision form's single-grid sweep with 32 x 32 tiles, switched
    between steps, reproduces the 32 x 16 run bit for bit (ragged tiles in
    both directions)."""
    ws = config3(form=native.FORM_FP32C, seed=9, count=1, dims=(100,), steps=6)
    w = ws[0]
    out = {}
    for tiles in ((16, 16, 16), (32, 32, 32), (16, 32, 16)):
        with Simulation(w.params) as s:
            setup(s, w)
            for t in tiles:
                s.set_sweep_tile(t)
                s.step(2)
            out[tiles] = (s.get_field("P_w"), s.get_field("S_n"))
    ref = out[(16, 16, 16)]
    for k, (P, S) in out.items():
        assert np.array_equal(P, ref[0]) and np.array_equal(S, ref[1]), k
    with Simulation(w.params) as s:
        with pytest.raises(native.CapazError):
            s.set_sweep_tile(24)
