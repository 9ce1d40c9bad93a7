"""Build the learned parameter predictor (predictor.npz beside this script).

    python make_predictor.py generate N SEED OUT.npz [reduced MAX_SECONDS MIN_NODES MAX_NODES]
                                                          # sweep N random tangles (GPU)
    python make_predictor.py train OUT.npz DS.npz [...]   # train on the GPU with the library's MLP kernels
    python make_predictor.py evaluate MODEL.npz N SEED OUT.json   # held-out tangles: predictor vs default rule

`generate` draws tangles from learned.random_configuration, sweeps tuning's parameter grid in the
mixed form against the FP64 reference and keeps, per tangle, the features and the cheapest
parameters within 0.6 rtol.  `evaluate` runs, per held-out tangle, the predicted parameters
(with the FP64 check and its default-rule fallback) and the default rule alone, and reports
times and errors.
"""

from __future__ import annotations

import importlib.util
import json
import math
import sys
import time
from pathlib import Path

import numpy as np

PKG = Path(__file__).resolve().parents[1]


def load_package():
    name = "vortexpasta_b200"
    if name in sys.modules:
        return sys.modules[name]
    spec = importlib.util.spec_from_file_location(name, PKG / "__init__.py", submodule_search_locations=[str(PKG)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def generate(n, seed, out, reduced=False, max_seconds=None, min_nodes=5_000, max_nodes=1_200_000):
    load_package()
    from vortexpasta_b200 import learned
    t0 = time.time()
    d = learned.generate_dataset(n, seed, log=lambda s: print(f"[{time.time() - t0:7.1f}s] {s}", flush=True),
                                 reduced=reduced, deadline=t0 + max_seconds if max_seconds else None,
                                 checkpoint=lambda ds: np.savez(out, **ds), min_nodes=min_nodes, max_nodes=max_nodes)
    np.savez(out, **d)
    print(f"{len(d['X'])} configurations in {time.time() - t0:.0f} s", flush=True)


def train(out, paths, steps=6000, lr=3e-3, seed=0):
    load_package()
    from vortexpasta_b200 import learned
    ds = [np.load(p) for p in paths]
    X = np.concatenate([d["X"] for d in ds])
    Y = np.concatenate([d["Y"] for d in ds])
    rtol = float(ds[0]["rtol"])
    pred = learned.train(X, Y, rtol, steps=steps, lr=lr, seed=seed)
    pred.save(out)
    Yp = pred.outputs(X)
    rms = np.sqrt(((Yp - Y) ** 2).mean(0))
    print(f"trained on {len(X)} configurations; rms error per output {np.round(rms, 4).tolist()}")


def evaluate(model, n, seed, out):
    load_package()
    from vortexpasta_b200 import learned, tuning
    L = 2 * math.pi
    pred = learned.Predictor.load(model)
    rng = np.random.default_rng(seed)
    rows = []
    for k in range(n):
        fs = learned.random_configuration(rng, L)
        N = sum(len(f) for f in fs)
        vref = learned.reference_velocity(fs, L)
        ch, info = learned.choose_parameters(fs, L, pred.rtol, pred, kaiser_bessel=False)
        ms_p, v_p = tuning.measure(fs, ch, L, "mixed")
        d = tuning.default_rule(L, pred.rtol, learned.FEATURE_RCUT * L)
        ms_d, v_d = tuning.measure(fs, d, L, "mixed")
        row = {"nodes": N, "pred_ms": ms_p, "pred_err": tuning.rel_errors(v_p, vref)[0], "fallback": info["fallback"],
               "default_ms": ms_d, "default_err": tuning.rel_errors(v_d, vref)[0],
               "pred_rcut_over_L": ch.rcut / L, "pred_fft": ch.fft_size(), "pred_m": ch.m, "pred_sigma": ch.sigma}
        rows.append(row)
        print(json.dumps(row), flush=True)
    r = pred.rtol
    summ = {"n": n, "rtol": r,
            "pred_meets_rtol": sum(x["pred_err"] <= r for x in rows),
            "default_meets_rtol": sum(x["default_err"] <= r for x in rows),
            "fallbacks": sum(x["fallback"] for x in rows),
            "geomean_speedup_vs_default": float(np.exp(np.mean([math.log(x["default_ms"] / x["pred_ms"]) for x in rows]))),
            "total_ms_pred": sum(x["pred_ms"] for x in rows), "total_ms_default": sum(x["default_ms"] for x in rows)}
    Path(out).write_text(json.dumps({"summary": summ, "rows": rows}, indent=1))
    print(json.dumps(summ))


if __name__ == "__main__":
    cmd = sys.argv[1]
    if cmd == "generate":
        # optional: reduced  MAX_SECONDS  MIN_NODES  MAX_NODES
        extra = sys.argv[5:]
        generate(int(sys.argv[2]), int(sys.argv[3]), sys.argv[4], reduced=bool(extra and extra[0] == "reduced"),
                 max_seconds=float(extra[1]) if len(extra) > 1 else None,
                 min_nodes=int(extra[2]) if len(extra) > 2 else 5_000,
                 max_nodes=int(extra[3]) if len(extra) > 3 else 1_200_000)
    elif cmd == "train":
        train(sys.argv[2], sys.argv[3:])
    elif cmd == "evaluate":
        evaluate(sys.argv[2], int(sys.argv[3]), int(sys.argv[4]), sys.argv[5])
    else:
        raise SystemExit(__doc__)
