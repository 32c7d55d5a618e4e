"""capaz_mass_noalloc, the allocation-free mass balance, through the C ABI.

It reduces the same per-cell quantities as a context's step diagnostics
(CAPAZ_FLAG_DIAGNOSTICS) over a state in caller-owned device memory, with its
scratch in a fixed device array of the library.  The GPU tests compare two
calls in a row with the diagnostics of the step that produced the state;
only the summation order differs, hence the 1e-12 relative tolerance.
"""
import ctypes as C

import numpy as np
import pytest

from capaz_b200 import Simulation, native
from capaz_b200.configs import two_phase_params

TOL = 1e-12


def _case(nx, ny, nz, P_d, seed):
    p = two_phase_params(nx, ny, nz)
    p.flags |= native.FLAG_DIAGNOSTICS
    p.dt = 0.02
    if P_d:
        p.P_d = P_d
        p.lambda_ = 2.7
        p.dt = 0.005
    rng = np.random.default_rng(seed)
    m = np.clip(0.25 + 0.02 * rng.standard_normal((p.nz, p.ny, p.nx)), 0.1, 0.4)
    K = np.exp(np.log(1e-12) + 0.5 * rng.standard_normal(m.shape))
    return p, m, K


def _noalloc(lib, p, P, S, m, out):
    st = lib.capaz_mass_noalloc(C.byref(p), P.data_ptr(), S.data_ptr(), m.data_ptr(), out.data_ptr(), None)
    assert st == native.OK, lib.capaz_last_error(None)
    return out.cpu().numpy().copy()


def _check(diag, got):
    for q in range(2):
        ref = diag["mass"][q]
        assert abs(got[q] - ref) <= TOL * abs(ref), (q, got[q], ref)
    assert got[2] == 0.0 and got[3] == 0.0
    assert got[4] == diag["nonfinite_cells"]


@pytest.mark.gpu
@pytest.mark.parametrize("shape,P_d", [((40, 24, 17), 0.0), ((37, 29, 1), 0.0), ((24, 13, 9), 755.0)])
def test_noalloc_mass_matches_step_diagnostics(shape, P_d):
    import torch

    p, m, K = _case(*shape, P_d, seed=sum(shape))
    lib = native.load()
    n = p.nx * p.ny * p.nz
    dev = torch.device("cuda:0")
    torch.cuda.set_device(0)
    P = torch.empty(n, dtype=torch.float64, device=dev)
    S = torch.empty_like(P)
    M = torch.empty_like(P)
    out = torch.full((5,), -1.0, dtype=torch.float64, device=dev)
    with Simulation(p) as sim:
        sim.set_field("m", m)
        sim.set_field("K", K)
        sim.init_state()
        for nsteps in (5, 3):
            sim.step(nsteps)
            diag = sim.diag()
            sim.get_field_device("P_w", P.data_ptr())
            sim.get_field_device("S_n", S.data_ptr())
            sim.get_field_device("m", M.data_ptr())
            sim.sync()
            first = _noalloc(lib, p, P, S, M, out)
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info(0)[0]
            second = _noalloc(lib, p, P, S, M, out)
            for _ in range(4):
                _noalloc(lib, p, P, S, M, out)
            torch.cuda.synchronize()
            # the property the entry point exists for: calls allocate nothing
            assert torch.cuda.mem_get_info(0)[0] == free0, "device free memory changed across the calls"
            _check(diag, first)
            _check(diag, second)
            assert np.array_equal(first, second), "two calls in a row differ"


@pytest.mark.gpu
def test_noalloc_rejects_host_pointers():
    lib = native.load()
    p, _, _ = _case(8, 8, 3, 0.0, 0)
    host = np.zeros(p.nx * p.ny * p.nz)
    ptr = host.ctypes.data
    st = lib.capaz_mass_noalloc(C.byref(p), ptr, ptr, ptr, ptr, None)
    assert st == native.ERR_INVALID_ARGUMENT
    assert b"device memory" in lib.capaz_last_error(None)


def test_noalloc_rejects_grids_beyond_fixed_scratch():
    """Rejected from the sizes alone, before any pointer is touched."""
    lib = native.load()
    p, _, _ = _case(8, 8, 3, 0.0, 0)
    p.ny = native.NOALLOC_MAX_ROWS + 3  # (ny-2)*(nz-2) = max + 1
    fake = 0x1000
    st = lib.capaz_mass_noalloc(C.byref(p), fake, fake, fake, fake, None)
    assert st == native.ERR_UNSUPPORTED_GRID
    assert b"exceed the fixed scratch" in lib.capaz_last_error(None)


@pytest.mark.parametrize("model", [native.MODEL_ENERGY, 7])
def test_noalloc_rejects_other_models(model):
    """Only the isothermal two-phase and Buckley-Leverett models are summed;
    anything else is rejected from the parameters alone, before any pointer
    is touched."""
    lib = native.load()
    p, _, _ = _case(8, 8, 3, 0.0, 0)
    p.model = model
    fake = 0x1000
    st = lib.capaz_mass_noalloc(C.byref(p), fake, fake, fake, fake, None)
    assert st == native.ERR_UNSUPPORTED
    assert b"models only" in lib.capaz_last_error(None)
