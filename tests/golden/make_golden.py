"""Records the reference engine's own outputs as golden fixtures (needs a GPU).

The reference (xinzhixue/PIV_xcorr2d_V1.0: xcorr2d_V1.0/xcorr2d_multi_grid.cu and
MHE7_4_gpu.cu, compiled unmodified for sm_100a into oracle/_ref/ by `make -C oracle ref`)
is driven through its public methods in the order of X/main.cpp:263-376 on seeded
synthetic inputs.  Inputs are not stored: they are regenerated from the recorded seed by
piv_synth_pair and pinned by their SHA-256.  Before a case runs on the GPU, the CPU
oracle checks that the reference's unchecked deformation reads stay inside its padded
buffers for that input (a case that would read outside is skipped, not run).

    python tests/golden/make_golden.py [outdir]
"""
import hashlib
import importlib.util
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
_spec = importlib.util.spec_from_file_location("piv_b200", ROOT / "piv_xcorr2d_v1.0_b200" / "__init__.py",
                                               submodule_search_locations=[str(ROOT / "piv_xcorr2d_v1.0_b200")])
P = importlib.util.module_from_spec(_spec)
sys.modules["piv_b200"] = P
_spec.loader.exec_module(P)
from oracle import oracle as O  # noqa: E402
from oracle import ref as R  # noqa: E402

# name -> (synthetic-input kwargs, engine parameter overrides)
CASES = {
    # the 1024^2 single-grid case: uniform (3.3, -1.7), 32x32 windows at 50 %, 1 pass, top-4, pct 0.25, threshold 2
    "c0": (dict(Nx=1024, Ny=1024, ppp=0.05, field=P.PIV_FIELD_UNIFORM, a=3.3, b=-1.7, seed=1),
           dict(Nx=1024, Ny=1024, ws_x1=32, ws_y1=32, spacing_x1=16, spacing_y1=16, Npass1=1,
                ws_x2=32, ws_y2=32, spacing_x2=16, spacing_y2=16, Npass2=0,
                max_dispx_win_percent1=0.25, max_dispy_win_percent1=0.25, max_dispx_win_percent2=0.25,
                max_dispy_win_percent2=0.25, insert_threshold_p1=2.0, insert_threshold_p2=2.0)),
    # a small form of the 6600x4400 multigrid case: Lamb-Oseen vortex + shear, MHE (40 px, 0.91, non-divisible crop), 64->32
    "multigrid": (dict(Nx=520, Ny=392, ppp=0.04, field=P.PIV_FIELD_VORTEX, a=6.0, b=120.0, c=0.002, seed=2),
                  dict(Nx=520, Ny=392, if_mhe=1, mhe_ws=40, mhe_thresh=0.91, Npass1=2, Npass2=3,
                       insert_threshold_p1=2.0, insert_threshold_p2=2.0, max_dispx_win_percent1=0.25,
                       max_dispy_win_percent1=0.25, max_dispx_win_percent2=0.25, max_dispy_win_percent2=0.25)),
    # non-square windows, 75 % overlap on grid 2, random Fourier field, no MHE
    "nonsquare": (dict(Nx=384, Ny=320, ppp=0.06, field=P.PIV_FIELD_FOURIER, a=150.0, b=600.0, c=5.0, seed=3),
                  dict(Nx=384, Ny=320, ws_x1=48, ws_y1=24, spacing_x1=24, spacing_y1=12, Npass1=2,
                       ws_x2=24, ws_y2=24, spacing_x2=8, spacing_y2=8, Npass2=2, insert_threshold_p1=2.0,
                       insert_threshold_p2=2.0, max_dispx_win_percent1=0.3, max_dispy_win_percent1=0.3,
                       max_dispx_win_percent2=0.3, max_dispy_win_percent2=0.3, Npeak_save=4)),
}

MHE_CASES = {"mhe_640x480": (640, 480, 40, 0.91, 4), "mhe_333x251": (333, 251, 40, 0.91, 5),
             "mhe_300x200_16": (300, 200, 16, 0.5, 6)}


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def make_case(name, sk, pk, outdir):
    s = P.synth_params(**sk)
    f1, f2 = P.synth_pair(s)
    p = P.default_params(**pk)
    chk = O.run_pair(O.mhe(f1, p.mhe_ws, p.mhe_thresh) if p.if_mhe else f1,
                     O.mhe(f2, p.mhe_ws, p.mhe_thresh) if p.if_mhe else f2, p)
    if chk["deform_oob"]:
        print(f"{name}: skipped, the reference would read outside its buffers ({chk['deform_oob']} taps)")
        return
    g = chk["geom"]
    out = dict(synth=np.array([repr(sk)]), params=np.array([repr(pk)]), f1_sha=np.array([sha(f1)]),
               f2_sha=np.array([sha(f2)]))
    with R.RefEngine(p) as r:
        if p.if_mhe:
            out["f1_mhe"] = r.mhe(f1)
            out["f2_mhe"] = r.mhe(f2)
        pred = r.run_pair_recording(f1, f2, g["Nt_vec"][0], g["Nt_vec"][1])
        # the filtered field each grid's last pass started from (predictor + deformation field)
        if p.Npass1 > 1:
            out["pred0_dx"], out["pred0_dy"] = pred["p1x"], pred["p1y"]
        if p.Npass2 > 0:
            out["pred1_dx"], out["pred1_dy"] = pred["p2x"], pred["p2y"]
        for k in range(2 if p.Npass2 > 0 else 1):
            nt = g["Nt_vec"][k]
            dx, dy, v = r.raw(k, nt)
            out[f"raw{k}_dx"], out[f"raw{k}_dy"], out[f"raw{k}_valid"] = dx, dy, v
            cnt, idx, val = r.peaks(k, nt)
            out[f"peaks{k}_count"], out[f"peaks{k}_index"], out[f"peaks{k}_value"] = cnt, idx, val
            fx, fy, fv = r.filtered(k, nt)
            out[f"filt{k}_dx"], out[f"filt{k}_dy"], out[f"filt{k}_valid"] = fx, fy, fv
        if name in ("c0", "multigrid"):
            # write_vec_data_general's own files, to pin the Tecplot format byte for byte
            import tempfile

            with tempfile.TemporaryDirectory() as td:
                for sel in range(4 if p.Npass2 > 0 else 2):
                    fn = Path(td) / f"sel{sel}.dat"
                    r.write_tecplot(fn, sel)
                    out[f"tecplot_sel{sel}"] = np.frombuffer(fn.read_bytes(), np.uint8)
        last = 1 if p.Npass2 > 0 else 0
        wsx = p.ws_x2 if last else p.ws_x1
        wsy = p.ws_y2 if last else p.ws_y1
        out["cc_last"] = r.cc(last, 0, 48, wsx, wsy)
        if p.Npass2 > 0:
            out["deformed1_rows"] = r.deformed(1, g["Ny_aug"][1], g["Nx_aug"][1])[::16]
            r.median_only()
            mx, my, mv = r.filtered(1, g["Nt_vec"][1])
            out["median2_dx"], out["median2_dy"], out["median2_valid"] = mx, my, mv
    np.savez_compressed(outdir / f"golden_{name}.npz", **out)
    print(f"{name}: written")


def make_mhe(name, Nx, Ny, ws, th, seed, outdir):
    s = P.synth_params(Nx, Ny, ppp=0.04, seed=seed)
    f1, _ = P.synth_pair(s)
    p = P.default_params(Nx=Nx, Ny=Ny, if_mhe=1, mhe_ws=ws, mhe_thresh=th, Npass1=1, Npass2=0,
                         ws_x1=16, ws_y1=16, spacing_x1=8, spacing_y1=8, ws_x2=16, ws_y2=16, spacing_x2=8,
                         spacing_y2=8)
    with R.RefEngine(p) as r:
        got = r.mhe(f1)
    np.savez_compressed(outdir / f"golden_{name}.npz", synth=np.array([repr(dict(Nx=Nx, Ny=Ny, ppp=0.04, seed=seed))]),
                        f1_sha=np.array([sha(f1)]), ws=ws, thresh=th, out=got)
    print(f"{name}: written")


def main():
    outdir = Path(sys.argv[1]) if len(sys.argv) > 1 else Path(__file__).resolve().parent
    outdir.mkdir(parents=True, exist_ok=True)
    for name, (sk, pk) in CASES.items():
        make_case(name, sk, pk, outdir)
    for name, a in MHE_CASES.items():
        make_mhe(name, *a, outdir)


if __name__ == "__main__":
    main()
