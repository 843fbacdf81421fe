"""amdk_fft_sphere_noalloc: the density-sphere FFT for callers that cannot
allocate device memory (their allocations all go through their own pool, or
an OpenACC/OpenMP runtime owns the device memory).  The caller passes device
input and output buffers; the library's fixed scratch array does the rest.

It must give the same transform as the allocating entry amdk_fft_sphere, on
consecutive calls (the shared scratch keeps the previous call's contents),
equal numpy.fft's transform, read inputs that the caller wrote on another
stream without synchronising, work on a grid close to its limit (90^3, 89% of
the scratch), and refuse grids whose transform does not fit its scratch.
This file runs last so that a failure here leaves every other test run."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12   # relative, as the other FFT parity tests


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _bind(lib):
    f = lib.amdk_fft_sphere_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _numpy_grid(e, coef):
    """The backward transform of the +G half sphere (and -G = conj) by numpy."""
    g = e.gvectors()
    n1, n2, n3 = e.nr
    nh = np.array([n1 // 2 + 1, n2 // 2 + 1, n3 // 2 + 1])
    mil = g["inyh"] - nh[None, :]
    full = np.zeros((n3, n2, n1), complex)
    full[mil[:, 2] % n3, mil[:, 1] % n2, mil[:, 0] % n1] = coef
    full[(-mil[:, 2]) % n3, (-mil[:, 1]) % n2, (-mil[:, 0]) % n1] = np.conj(coef)
    full[0, 0, 0] = coef[0]
    return np.fft.ifftn(full) * full.size


def test_noalloc_matches_allocating_entry_on_consecutive_calls():
    import torch

    from amdkiit_b200 import configs
    from amdkiit_b200.engine import FP64, Engine

    e = Engine(configs.water1(), FP64)          # 64^3 grid: fits the fixed scratch
    noalloc = _bind(e.lib)
    n1, n2, n3 = e.nr
    hg = e.gvectors()["hg"]
    rng = np.random.default_rng(11)
    for call in range(2):
        coef = (rng.standard_normal(e.ngrho) + 1j * rng.standard_normal(e.ngrho)) / (1.0 + hg)
        coef[0] = coef[0].real
        # backward: sphere -> grid
        _, grid_ref = e.fft_sphere(-1, coef=coef)
        d_coef = torch.from_numpy(coef.copy()).to("cuda")
        d_grid = torch.empty((n3, n2, n1), dtype=torch.complex128, device="cuda")
        torch.cuda.synchronize()
        assert noalloc(e.h, -1, d_coef.data_ptr(), d_grid.data_ptr()) == 0, e.lib.amdk_last_error()
        assert rel(d_grid.cpu().numpy(), grid_ref) < TOL, f"backward, call {call}"
        assert rel(d_grid.cpu().numpy(), _numpy_grid(e, coef)) < TOL, f"numpy, call {call}"
        # forward: grid -> sphere
        coef_ref, _ = e.fft_sphere(+1, grid=grid_ref)
        d_out = torch.empty(e.ngrho, dtype=torch.complex128, device="cuda")
        assert noalloc(e.h, +1, d_out.data_ptr(), d_grid.data_ptr()) == 0, e.lib.amdk_last_error()
        assert rel(d_out.cpu().numpy(), coef_ref) < TOL, f"forward, call {call}"
        assert rel(d_out.cpu().numpy(), coef) < TOL
    e.close()


def test_noalloc_refuses_grids_beyond_its_scratch():
    import torch

    from amdkiit_b200 import configs
    from amdkiit_b200.engine import FP64, Engine

    e = Engine(configs.water32(), FP64)         # 100^3: the transform needs ~30 MB
    noalloc = _bind(e.lib)
    n1, n2, n3 = e.nr
    d_coef = torch.zeros(e.ngrho, dtype=torch.complex128, device="cuda")
    d_grid = torch.zeros((n3, n2, n1), dtype=torch.complex128, device="cuda")
    rc = noalloc(e.h, -1, d_coef.data_ptr(), d_grid.data_ptr())
    assert rc != 0
    assert b"maximum" in e.lib.amdk_last_error()
    e.close()


def test_noalloc_near_its_limit():
    """The 90^3 H2 cell (tests/H2_upf) needs 22.3 MB of the 24 MiB scratch:
    it runs, and matches the allocating entry both ways."""
    import torch

    from amdkiit_b200.engine import FP64, Engine
    from tests.helpers import load_fixture

    e = Engine(load_fixture("h2_upf"), FP64)
    assert e.nr == (90, 90, 90)
    noalloc = _bind(e.lib)
    n1, n2, n3 = e.nr
    hg = e.gvectors()["hg"]
    rng = np.random.default_rng(13)
    coef = (rng.standard_normal(e.ngrho) + 1j * rng.standard_normal(e.ngrho)) / (1.0 + hg)
    coef[0] = coef[0].real
    _, grid_ref = e.fft_sphere(-1, coef=coef)
    d_coef = torch.from_numpy(coef.copy()).to("cuda")
    d_grid = torch.empty((n3, n2, n1), dtype=torch.complex128, device="cuda")
    torch.cuda.synchronize()
    assert noalloc(e.h, -1, d_coef.data_ptr(), d_grid.data_ptr()) == 0, e.lib.amdk_last_error()
    assert rel(d_grid.cpu().numpy(), grid_ref) < TOL
    d_out = torch.empty(e.ngrho, dtype=torch.complex128, device="cuda")
    assert noalloc(e.h, +1, d_out.data_ptr(), d_grid.data_ptr()) == 0, e.lib.amdk_last_error()
    assert rel(d_out.cpu().numpy(), coef) < TOL
    e.close()


def test_noalloc_reads_inputs_written_on_another_stream():
    """A caller that writes the input on its own stream (behind a long
    kernel) and calls at once, with no synchronisation, gets the transform of
    what it wrote: the entry waits for the device before reading."""
    import torch

    from amdkiit_b200 import configs
    from amdkiit_b200.engine import FP64, Engine

    e = Engine(configs.water1(), FP64)
    noalloc = _bind(e.lib)
    n1, n2, n3 = e.nr
    hg = e.gvectors()["hg"]
    rng = np.random.default_rng(17)
    coef = (rng.standard_normal(e.ngrho) + 1j * rng.standard_normal(e.ngrho)) / (1.0 + hg)
    coef[0] = coef[0].real
    _, grid_ref = e.fft_sphere(-1, coef=coef)
    host = torch.from_numpy(coef.copy()).pin_memory()
    d_coef = torch.zeros(e.ngrho, dtype=torch.complex128, device="cuda")
    d_grid = torch.empty((n3, n2, n1), dtype=torch.complex128, device="cuda")
    a = torch.randn(4096, 4096, device="cuda")
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        for _ in range(8):
            a = a @ a.T * 1e-3           # keeps the stream busy before the copy
        d_coef.copy_(host, non_blocking=True)
    assert noalloc(e.h, -1, d_coef.data_ptr(), d_grid.data_ptr()) == 0, e.lib.amdk_last_error()
    assert rel(d_grid.cpu().numpy(), grid_ref) < TOL
    torch.cuda.synchronize()
    e.close()
