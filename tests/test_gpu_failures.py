"""Failure detection, with the failures made on the host (no GPU fault, trap or hang).

The reference reports failure as a bool plus a printed message, and the driver stops its
pair loop (X/main.cpp:292-325); its hole fill loops on the host until nothing changes
(X/xcorr2d_multi_grid.cu:1515-1528).  The engine returns a status from every call, caps
the device-side hole fill, and frees what it allocated when piv_create fails.  Two
injection knobs, read at piv_create and off by default, make those paths run:
  PIV_TEST_FILL_CAP=n    the hole fill stops after n iterations and sets the status word;
  PIV_TEST_FAIL_ALLOC=k  the engine's k-th device allocation fails.
"""
import numpy as np
import pytest

import piv_b200 as P

pytestmark = pytest.mark.gpu


def _holed_candidates(nx, ny, nps, hole):
    """A smooth field with every candidate valid except in a hole x hole block."""
    yy, xx = np.mgrid[0:ny, 0:nx]
    bx = (1.5 + 0.05 * xx + 0.02 * yy).ravel().astype(np.float32)
    by = (-0.7 + 0.03 * xx).ravel().astype(np.float32)
    dx = np.repeat(bx[:, None], nps, 1)
    dy = np.repeat(by[:, None], nps, 1)
    valid = np.ones((nx * ny, nps), np.uint8)
    x0, y0 = (nx - hole) // 2, (ny - hole) // 2
    block = ((xx >= x0) & (xx < x0 + hole) & (yy >= y0) & (yy < y0 + hole)).ravel()
    valid[block] = 0
    dx[block] = 0
    dy[block] = 0
    return dx, dy, valid, block


def _engine_params():
    return P.default_params(Nx=24 * 16 + 8, Ny=20 * 16 + 8, ws_x1=32, ws_y1=32, spacing_x1=16, spacing_y1=16,
                            Npass1=1, Npass2=0)


def test_fill_iteration_cap_reports_and_recovers(cuda, monkeypatch):
    p = _engine_params()
    with P.Engine(p) as e:
        nx, ny = e.geom["Nx_vec"][0], e.geom["Ny_vec"][0]
        dx, dy, valid, block = _holed_candidates(nx, ny, p.Npeak_save, hole=12)
        e.set_candidates(0, dx, dy, valid)
        e.validate_grid1(2, 5, 2.0, 2.0, 0)
        e.synchronize()
        _, _, fx, fy, fv = e.field(1)
        assert fv.all(), "the default cap fills the whole hole"
    monkeypatch.setenv("PIV_TEST_FILL_CAP", "2")  # a 12x12 hole needs 6 iterations
    with P.Engine(p) as e:
        e.set_candidates(0, dx, dy, valid)
        e.validate_grid1(2, 5, 2.0, 2.0, 0)
        with pytest.raises(P.PivError) as err:
            e.synchronize()
        assert err.value.status == P.PIV_ERR_DEVICE
        assert "iteration cap" in str(err.value)
        _, _, gx, gy, gv = e.field(1)
        assert not gv[block].all(), "the capped fill left part of the hole"
        assert gv[~block].all()
        # the status word was cleared: the engine keeps working
        e.synchronize()
        e.set_candidates(0, dx, dy, np.ones_like(valid))
        e.validate_grid1(2, 5, 2.0, 2.0, 0)
        e.synchronize()


def test_allocation_failure_in_create_frees_everything(cuda, monkeypatch):
    import torch

    p = P.default_params(Nx=1536, Ny=1024, if_mhe=1, ws_x1=64, ws_y1=64, spacing_x1=32, spacing_y1=32, Npass1=2,
                         ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=2)
    with P.Engine(p):  # one-time costs (context, modules) before the baseline
        pass
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    failed = 0
    for k in range(1, 80):
        monkeypatch.setenv("PIV_TEST_FAIL_ALLOC", str(k))
        try:
            e = P.Engine(p)
        except P.PivError as err:
            assert err.status == P.PIV_ERR_ALLOC, err
            failed += 1
            torch.cuda.synchronize()
            assert torch.cuda.mem_get_info()[0] == free0, f"allocation {k} failed and device memory leaked"
            continue
        e.close()  # past the last allocation of piv_create
        break
    assert failed >= 30, f"only {failed} allocations were exercised"
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
