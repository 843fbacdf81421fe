"""amdk_fft_sphere_noalloc: the density-sphere FFT for callers that cannot
allocate device memory (their allocations all go through their own pool, or
an OpenACC/OpenMP runtime owns the device memory).  The caller passes device
input and output buffers; the library's fixed scratch array does the rest.

It must give the same transform as the allocating entry amdk_fft_sphere, on
consecutive calls (the shared scratch keeps the previous call's contents),
and must refuse grids whose transform does not fit its fixed scratch.
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
