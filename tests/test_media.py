"""Heterogeneous-media inputs: the permeability-file reader against the
reference's load_permeability (golden fixture made by
tests/golden/make_media_golden.py, and live when oracle/_ref is built), and
the on-device Gaussian field generator."""
import os
import sys

import numpy as np
import pytest

from conftest import ROOT
from capaz_b200 import Simulation, native
from capaz_b200.simulation import default_params, read_permeability_file

GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)
import make_media_golden as mg  # noqa: E402


def test_reader_matches_reference_golden():
    g = np.load(os.path.join(GOLDEN, "media_K_13x9.npz"))
    K = read_permeability_file(os.path.join(GOLDEN, "media_noise_13x9.dat"), 13, 9, 1)
    assert np.array_equal(K, g["K"])


@pytest.mark.skipif(not os.path.exists(mg.LOADK), reason="reference harness not built (make -C oracle REF=<reference tree> ref)")
@pytest.mark.parametrize("shape,seed", [((17, 11, 1), 1), ((8, 6, 5), 2)])
def test_reader_matches_reference_live(tmp_path, shape, seed):
    """Any field, any z depth: every z layer takes the file's (i, j) value."""
    nx, ny, nz = shape
    vals = np.random.default_rng(seed).normal(0.0, 2.0, size=(ny, nx))
    path = str(tmp_path / "noise.dat")
    mg.write_noise(path, vals)
    if nz > 1:  # the 3-D header has three numbers
        text = open(path, "rb").read().split(b"\r\n", 1)
        open(path, "wb").write(f"{nx} {ny} {nz}".encode() + b"\r\n" + text[1])
    ref = mg.reference_K(path, nx, ny, nz)
    assert np.array_equal(read_permeability_file(path, nx, ny, nz), ref)


def test_reader_rejects_bad_files(tmp_path):
    path = str(tmp_path / "noise.dat")
    mg.write_noise(path, np.zeros((4, 5)))
    with pytest.raises(native.CapazError, match="does not match"):
        read_permeability_file(path, 5, 5, 1)
    with open(path, "wb") as f:
        f.write(b"5 4\r\n 1.0 2.0 \r\n")
    with pytest.raises(native.CapazError, match="missing"):
        read_permeability_file(path, 5, 4, 1)
    with pytest.raises(native.CapazError, match="cannot open"):
        read_permeability_file(str(tmp_path / "absent.dat"), 5, 4, 1)


@pytest.mark.gpu
def test_load_permeability_into_a_context():
    p = default_params(nx=13, ny=9, nz=4, dt=1e-3, flags=native.FLAG_PERCELL_K)
    path = os.path.join(GOLDEN, "media_noise_13x9.dat")
    g = np.load(os.path.join(GOLDEN, "media_K_13x9.npz"))["K"]
    text = open(path, "rb").read().split(b"\r\n", 1)
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        f3 = os.path.join(d, "noise.dat")
        open(f3, "wb").write(b"13 9 4\r\n" + text[1])
        with Simulation(p) as s:
            s.load_permeability(f3)
            K = s.get_field("K")
    assert np.array_equal(K, np.broadcast_to(g, K.shape))


@pytest.mark.gpu
@pytest.mark.parametrize("form", [native.FORM_FP64, native.FORM_FP32C])
def test_generated_media_statistics_and_determinism(form):
    nx, ny, nz, ell, sigma = 96, 64, 80, 6.0, 1.0
    p = default_params(nx=nx, ny=ny, nz=nz, dt=1e-3, flags=native.FLAG_PERCELL_K, form=form)
    with Simulation(p) as s:
        s.generate_media(seed=7, sigma=sigma, ell=ell)
        K1, m1 = s.get_field("K"), s.get_field("m")
        s.generate_media(seed=7, sigma=sigma, ell=ell)
        K2 = s.get_field("K")
        s.generate_media(seed=8, sigma=sigma, ell=ell)
        K3 = s.get_field("K")
    assert np.array_equal(K1, K2) and not np.array_equal(K1, K3)
    G = (np.log(K1) - np.log(1e-12)) / sigma
    tol = 1e-6 if form == native.FORM_FP32C else 1e-12  # K stored as float32 in the precision form
    assert abs(G.mean()) < 0.25 and abs(G.std() - 1.0) < 0.25
    # correlation at lag ell along x, against exp(-1)
    c = np.mean((G[:, :, :-6] - G.mean()) * (G[:, :, 6:] - G.mean())) / G.var()
    assert abs(c - np.exp(-1.0)) < 0.12, c
    assert m1.min() >= 0.1 - tol and m1.max() <= 0.4 + tol
    assert np.allclose(m1, np.clip(0.25 + 0.02 * G, 0.1, 0.4), atol=1e-6)
