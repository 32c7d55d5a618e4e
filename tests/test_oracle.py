"""The oracle restatement against the reference's golden vectors (CPU)."""
import numpy as np
import pytest

from conftest import ENERGY_STATE, GOLDEN_2PH, GOLDEN_3PH, GOLDEN_BL, GOLDEN_ENERGY, interior, load_golden
from oracle import oracle as O


def _state_names(p):
    return ["P_w", "S_n"] if p.phases == 2 else ["P_w", "S_w", "S_n", "P_n", "P_g"]


@pytest.mark.parametrize("name", GOLDEN_2PH + GOLDEN_3PH)
def test_oracle_matches_reference_bitwise(name):
    """oracle/capaz_oracle.cpp reproduces the reference CPU step bit for bit."""
    p, g = load_golden(name)
    if "in_P_w" in g:
        state = {k: g["in_" + k] for k in _state_names(p)}
        m = g["in_m"]
    else:
        st = O.init(p)
        state = {k: st[k] for k in _state_names(p)}
        m = st["m"]
    out = O.step(p, state, int(g["nsteps"]), m, derived=True)
    for k in _state_names(p):
        assert np.array_equal(out[k], g["out_" + k]), k
    for key in [k for k in g if k.startswith("der_")]:
        f = key[4:]
        if f in _state_names(p):  # three-phase S_w, P_n are state arrays
            assert np.array_equal(out[f], g[key]), f
        elif f.startswith("roS"):  # the reference writes roS on interior cells only
            assert np.array_equal(interior(out["derived"][f]), interior(g[key])), f
        else:
            assert np.array_equal(out["derived"][f], g[key]), f


@pytest.mark.parametrize("name", GOLDEN_BL)
def test_oracle_buckley_leverett_matches_reference_bitwise(name):
    """The Buckley-Leverett task (B_L build of the reference: b-l.cpp with
    cpu.cpp): data_initialization, then the steps, with K as the reference's
    permeability-file loader produced it."""
    from capaz_b200 import native
    p, g = load_golden(name)
    q = p.copy()
    q.flags |= native.FLAG_PERCELL_K
    st = O.init(q)
    out = O.step(q, {"P_w": st["P_w"], "S_n": st["S_n"]}, int(g["nsteps"]), st["m"], g["K"])
    assert np.array_equal(out["P_w"], g["out_P_w"])
    assert np.array_equal(out["S_n"], g["out_S_n"])


@pytest.mark.parametrize("name", GOLDEN_ENERGY)
def test_oracle_energy_matches_reference_bitwise(name):
    """The energy equation (THREE_PHASE + ENERGY build: energy.cpp with the
    three-phase module): the state with T and every array the reference
    keeps, bit for bit (E_new and roS exist on interior cells only)."""
    p, g = load_golden(name)
    if "in_P_w" in g:
        state, m = {k: g["in_" + k] for k in ENERGY_STATE}, g["in_m"]
    else:
        st = O.init(p)
        state, m = {k: st[k] for k in ENERGY_STATE}, st["m"]
    out = O.step(p, state, int(g["nsteps"]), m, derived=True)
    for k in ENERGY_STATE:
        assert np.array_equal(out[k], g["out_" + k]), k
    for key in [k for k in g if k.startswith("der_")]:
        f = key[4:]
        a = out[f] if f in ENERGY_STATE else out["derived"][f]
        if f.startswith("roS") or f == "E_new":
            assert np.array_equal(interior(a), interior(g[key])), f
        else:
            assert np.array_equal(a, g[key]), f


def test_oracle_init_matches_reference():
    """data_initialization (two-phase.cpp:113-172) on a 3-D grid."""
    p, g = load_golden("g2_init_10x9x7")
    st = O.init(p)
    assert np.array_equal(st["P_w"], g["out_P_w"])
    assert np.array_equal(st["S_n"], g["out_S_n"])


@pytest.mark.parametrize("nthreads", [1, 3, 8])
def test_oracle_thread_count_independent(nthreads):
    p, g = load_golden("g2_3d_pd_12x10x7")
    state = {"P_w": g["in_P_w"], "S_n": g["in_S_n"]}
    out = O.step(p, state, int(g["nsteps"]), g["in_m"], nthreads=nthreads)
    assert np.array_equal(out["P_w"], g["out_P_w"])
    assert np.array_equal(out["S_n"], g["out_S_n"])


# Known-answer vectors of the reference's 3x3 inverse test
# (Three-phase/Test/test_main.cpp:53-66), checked to 1e-10 as there.
KAT = [
    ([1, 0, 0, 0, 1, 0, 0, 0, 1], [1, 0, 0, 0, 1, 0, 0, 0, 1]),
    ([-4 / 19, 7 / 38, 5 / 38, 3 / 19, 9 / 38, 1 / 38, 2 / 19, -13 / 38, 7 / 38],
     [-2, 3, 1, 1, 2, -1, 3, 2, 3]),
    ([3, 0, 0, 2, 2, 1, 1, 0, 1], [1 / 3, 0, 0, -1 / 6, 0.5, -0.5, -1 / 3, 0, 1]),
]


@pytest.mark.parametrize("a,b", KAT)
def test_reverse_matrix_kat(a, b):
    rc, inv = O.reverse_matrix(np.array(a, dtype=np.float64).reshape(3, 3))
    assert rc == 0
    assert np.all(np.abs(inv.ravel() - np.array(b)) < 1e-10)


def test_reverse_matrix_singular_and_pivot():
    rc, _ = O.reverse_matrix(np.zeros((3, 3)))
    assert rc == -1
    # A zero leading pivot forces the row exchange of gauss.cpp:43-58.
    a = np.array([[0.0, 1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 2.0]])
    rc, inv = O.reverse_matrix(a)
    assert rc == 0
    assert np.allclose(inv @ a, np.eye(3))


@pytest.mark.skipif(not O.ref_available(2), reason="reference binaries not built (make -C oracle REF=<reference tree> ref)")
@pytest.mark.parametrize("seed", [1, 2])
def test_oracle_vs_reference_binary_random(seed):
    """Fresh random cases straight against the compiled reference."""
    from capaz_b200.simulation import default_params
    rng = np.random.default_rng(seed)
    nx, ny, nz = rng.integers(3, 14), rng.integers(3, 12), int(rng.choice([1, 3, 5, 9]))
    p = default_params(nx=int(nx), ny=int(ny), nz=nz, dt=0.01, hx=1.0, hy=1.0, hz=1.0, beta_w=1e-9,
                       beta_n=1e-9, K0=1e-12, mu_n=5e-3, ro0_n=850.0, source=int(rng.integers(0, 4)))
    m = np.clip(0.3 + 0.03 * rng.standard_normal((nz, ny, nx)), 0.15, 0.45)
    st = O.init(p, m)
    st["S_n"] = np.clip(0.4 + 0.2 * rng.standard_normal(st["S_n"].shape), 0.05, 0.8)
    state = {"P_w": st["P_w"], "S_n": st["S_n"]}
    r = O.ref_run(p, 15, state, m)
    o = O.step(p, state, 15, m)
    assert np.array_equal(o["P_w"], r["P_w"]) and np.array_equal(o["S_n"], r["S_n"])
