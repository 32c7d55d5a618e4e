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
