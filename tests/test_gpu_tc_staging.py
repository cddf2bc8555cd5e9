"""TMA staging of the square tensor-core kernel's window rows (16 and 32 px windows).

A tile whose 128/WS windows lie in one row of the window grid is copied into shared memory
by one 2D tensor-map copy per frame; other tiles, and engines created with PIV_TC_STAGING=0,
load their rows directly from global memory.  Both read the same pixels, so the outputs must
be bit-identical: correlation planes, peak lists and displacements, on the undeformed and the
deformed pass, over sectioned launches (Nsec_cc > 1, window ranges starting inside a tile),
a plane dump starting at an odd window, and grids whose rows are not a multiple of the tile.
"""
import os

import numpy as np
import pytest

import piv_b200 as P

pytestmark = pytest.mark.gpu

# (window, spacing, Nx, Ny): staged boxes of 80-112 bytes; rows of 13-40 windows
CASES = [(32, 16, 660, 440), (32, 8, 500, 300), (16, 8, 408, 256), (16, 4, 260, 200)]
PATHS = [("split-bf16", P.PIV_XCORR_TC_SPLIT), ("split-fp16", P.PIV_XCORR_TC_SPLIT_F16),
         ("bf16", P.PIV_XCORR_TC_BF16)]


def _run(p, f1, f2, path, staging):
    old = os.environ.get("PIV_TC_STAGING")
    os.environ["PIV_TC_STAGING"] = "1" if staging else "0"
    try:
        with P.Engine(p) as e:
            e.set_xcorr_path(0, path)
            e.set_images(f1, f2)
            e.prep()
            nt = e.geom["Nt_vec"][0]
            nxv, nyv = e.geom["Nx_vec"][0], e.geom["Ny_vec"][0]
            out = []
            for j in (0, 1):
                if j == 1:
                    yy, xx = np.mgrid[0:nyv, 0:nxv]
                    dx = (1.7 * np.sin(xx / 4.0) + 0.03 * yy).astype(np.float32).ravel()
                    dy = (-1.2 * np.cos(yy / 3.0)).astype(np.float32).ravel()
                    e.set_field(0, dx, dy, np.ones(nt, np.uint8))
                e.pass_grid1(j)
                e.synchronize()
                out.append((e.peaks(0), e.field(0), e.cc_planes(0, 5, nt - 9)))
            return out
    finally:
        if old is None:
            del os.environ["PIV_TC_STAGING"]
        else:
            os.environ["PIV_TC_STAGING"] = old


@pytest.mark.parametrize("ws,sp,Nx,Ny", CASES, ids=[f"{c[0]}px-sp{c[1]}" for c in CASES])
@pytest.mark.parametrize("name,path", PATHS, ids=[n for n, _ in PATHS])
def test_staged_rows_match_direct_rows(cuda, ws, sp, Nx, Ny, name, path):
    p = P.default_params(Nx=Nx, Ny=Ny, ws_x1=ws, ws_y1=ws, spacing_x1=sp, spacing_y1=sp, Npass1=2, Npass2=0,
                         Nsec_cc=3, max_dispx_win_percent1=0.25, max_dispy_win_percent1=0.25)
    f1, f2 = P.synth_pair(P.synth_params(Nx, Ny, ppp=0.05, field=P.PIV_FIELD_FOURIER, a=150.0, b=900.0, c=4.0,
                                         seed=ws + sp))
    staged = _run(p, f1, f2, path, True)
    direct = _run(p, f1, f2, path, False)
    for j, ((pk_s, fd_s, pl_s), (pk_d, fd_d, pl_d)) in enumerate(zip(staged, direct)):
        assert np.array_equal(pl_s, pl_d), f"pass {j}: planes differ"
        for a, b in zip(pk_s, pk_d):
            assert np.array_equal(a, b), f"pass {j}: peaks differ"
        for a, b in zip(fd_s, fd_d):
            assert np.array_equal(a, b, equal_nan=True), f"pass {j}: field differs"
