#!/usr/bin/env python
"""Trains the learned grid-1 predictor and writes its weights.

  python piv_xcorr2d_v1.0_b200/train_predictor.py --pairs 20000 --epochs 30 \\
      --out piv_xcorr2d_v1.0_b200/weights/predictor.bin

Generates the labelled pairs on the GPU (see learned.py), trains with the hand-written
kernels and prints one JSON line with the training history and the held-out errors
(against the labels and against the generator's true field, and of the zero predictor
for comparison).
"""
import argparse
import importlib.util
import json
import math
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent


def load_pkg():
    if "piv_b200" in sys.modules:
        return sys.modules["piv_b200"]
    spec = importlib.util.spec_from_file_location("piv_b200", HERE / "__init__.py",
                                                  submodule_search_locations=[str(HERE)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["piv_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=20000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--out", default=str(HERE / "weights" / "predictor.bin"))
    ap.add_argument("--init", default=None, help="start from these weights")
    a = ap.parse_args()
    P = load_pkg()
    import piv_b200.learned as LN
    import numpy as np

    log = lambda m: print(m, file=sys.stderr, flush=True)
    t0 = time.time()
    data = LN.make_dataset(a.pairs, seed=a.seed, log=log)
    t_data = time.time() - t0
    log(f"dataset: {a.pairs} pairs in {t_data:.1f} s")
    net = P.PredictorNet(seed=a.seed)
    if a.init:
        net.load(a.init)
    n = a.pairs
    val = np.arange(n - max(1, int(round(n * 0.05))), n)
    # the zero predictor on the held-out pairs, for comparison
    lab, tru, m = data["label"][val], data["truth"][val], data["mask"][val]
    zero_label = math.sqrt(float(((lab[:, 0] ** 2 + lab[:, 1] ** 2) * m).sum() / m.sum())) * LN.DOWN
    label_vs_truth = math.sqrt(float((((lab - tru)[:, 0] ** 2 + (lab - tru)[:, 1] ** 2) * m).sum() / m.sum())) * LN.DOWN
    t1 = time.time()
    hist = LN.train(net, data, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed + 1, log=log)
    t_train = time.time() - t1
    Path(a.out).parent.mkdir(parents=True, exist_ok=True)
    net.save(a.out)
    print(json.dumps({"pairs": a.pairs, "size": LN.TRAIN_SIZE, "epochs": a.epochs, "batch": a.batch, "lr": a.lr,
                      "params": net.n_params, "data_seconds": round(t_data, 1), "train_seconds": round(t_train, 1),
                      "held_out_pairs": len(val), "zero_predictor_rms_px": round(zero_label, 4),
                      "label_vs_truth_rms_px": round(label_vs_truth, 4),
                      "final": hist[-1], "history": hist, "weights": a.out}))


if __name__ == "__main__":
    main()
