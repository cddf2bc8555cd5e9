"""The allocation-free MHE entry point (piv_mhe_process_noalloc) against the allocating one.

Callers that cannot allocate device memory where they enhance a frame (real-time
acquisition callbacks that must not wait on the allocator, applications whose own pool owns
all device memory) use piv_mhe_process_noalloc, which keeps its tile histograms in a fixed
array of the library.  This checks, through the C-ABI, that calls in a row -- a full
6600x4400 frame, then a smaller frame with a different tile grid, then a mid-size frame whose
tile grid is larger than the previous call's, so each call starts from the previous call's
leftovers in the shared array -- give exactly the output of piv_mhe_process (MHE is integer
arithmetic: bit-exact), and that requests larger than the array are refused.
Collected last (file name) so that a stop-at-first-failure run has already run the rest.
"""
import ctypes as C

import numpy as np
import pytest

import piv_b200 as P

pytestmark = pytest.mark.gpu


def allocating(d_in, Nx, Ny, ws, thresh):
    import torch

    h = C.c_void_p()
    assert P.lib().piv_mhe_create(Nx, Ny, ws, thresh, C.byref(h)) == 0
    out = torch.full((Ny, Nx), 7, dtype=torch.uint8, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    assert P.lib().piv_mhe_process(h, C.c_void_p(d_in.data_ptr()), C.c_void_p(out.data_ptr()), s) == 0
    torch.cuda.synchronize()
    assert P.lib().piv_mhe_destroy(h) == 0
    return out.cpu().numpy()


def no_alloc(d_in, Nx, Ny, ws, thresh):
    import torch

    out = torch.full((Ny, Nx), 7, dtype=torch.uint8, device="cuda")
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = P.lib().piv_mhe_process_noalloc(C.c_void_p(d_in.data_ptr()), C.c_void_p(out.data_ptr()), Nx, Ny, ws,
                                         thresh, s)
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


def test_no_alloc_mhe_matches_allocating_entry_point(cuda):
    import torch

    cases = [(6600, 4400, 40, 0.91, 1), (333, 251, 16, 0.5, 2), (2048, 1536, 24, 0.8, 3)]
    for Nx, Ny, ws, th, seed in cases:
        f, _ = P.synth_pair(P.synth_params(Nx, Ny, ppp=0.04, seed=seed))
        d = torch.from_numpy(np.ascontiguousarray(f)).cuda()
        want = allocating(d, Nx, Ny, ws, th)
        rc, got = no_alloc(d, Nx, Ny, ws, th)
        assert rc == P.PIV_OK
        assert np.array_equal(got, want), f"{Nx}x{Ny} ws {ws}"
        assert got.any()


def test_no_alloc_mhe_refuses_oversized_request(cuda):
    import torch

    Nx, Ny, ws = 8192, 8192, 16  # (512+2)^2 tiles > PIV_MHE_NOALLOC_MAX_TILES
    d = torch.zeros((Ny, Nx), dtype=torch.uint8, device="cuda")
    rc, _ = no_alloc(d, Nx, Ny, ws, 0.9)
    assert rc == P.PIV_ERR_ARG
