"""Learned Ewald/NUFFT parameter predictor.

A 16 -> 64 -> 64 -> 5 GELU perceptron (hand-written CUDA forward, backward and Adam kernels in
csrc/mlp.cu, reached through the C ABI) maps cheap configuration features (csrc/features.cu) to
the parameters of the cheapest evaluation that met the accuracy target in the library's own
sweeps (tuning.sweep against an FP64 reference):

    outputs = (log alpha L, r_cut / L, log2 Ns, sigma, m)   (standardised for training)

``predict_choice`` turns the outputs into a valid ``EwaldChoice`` (sigma snapped to the
allowed set, m rounded, the grid rounded up to a brick-friendly FFT size) and
``choose_parameters`` checks the prediction against a plain FP64 evaluation and falls back to
the reference's default rule (tuning.default_rule) when the target is missed.  The reference
has no counterpart (it removed its alpha autotuner).
"""

from __future__ import annotations

import ctypes as ct
import math
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from . import _lib, curves, tuning
from .params import GaussianSplitting, GaussLegendre, NonuniformFFTsBackend, ParamsBiotSavart

DATA_DIR = Path(__file__).resolve().parent / "data"
DEFAULT_MODEL = DATA_DIR / "predictor.npz"
FEATURE_RCUT = 1.0 / 16  # r_cut / L of the cell lists the feature search runs on


class MLP:
    """The predictor network on the GPU (vpbs_mlp_*)."""

    def __init__(self, max_batch: int = 1024, device: int = 0, params: np.ndarray | None = None, seed: int = 0):
        self._lib = _lib.load()
        h = ct.c_void_p()
        rc = self._lib.vpbs_mlp_create(int(device), int(max_batch), ct.byref(h))
        if rc != 0:
            raise _lib.VpbsError(f"vpbs_mlp_create failed ({rc})")
        self._h = h
        self.max_batch = int(max_batch)
        self.set_params(init_params(seed) if params is None else params)

    def _check(self, rc, what):
        if rc != 0:
            msg = self._lib.vpbs_mlp_last_error(self._h)
            raise _lib.VpbsError(f"{what} failed ({rc}): {msg.decode() if msg else ''}")

    def close(self):
        if getattr(self, "_h", None):
            self._lib.vpbs_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self._lib.vpbs_mlp_set_params(self._h, _lib.fptr(p), p.size), "mlp set_params")

    def get_params(self) -> np.ndarray:
        p = np.zeros(_lib.MLP_NPARAMS, dtype=np.float32)
        self._check(self._lib.vpbs_mlp_get_params(self._h, _lib.fptr(p), p.size), "mlp get_params")
        return p

    def set_loss_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        self._check(self._lib.vpbs_mlp_set_loss_weights(self._h, _lib.fptr(w)), "mlp set_loss_weights")

    def forward(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.zeros((X.shape[0], _lib.MLP_OUT), dtype=np.float32)
        for a in range(0, X.shape[0], self.max_batch):
            Xa = np.ascontiguousarray(X[a:a + self.max_batch])
            Ya = np.zeros((Xa.shape[0], _lib.MLP_OUT), dtype=np.float32)
            self._check(self._lib.vpbs_mlp_forward(self._h, _lib.fptr(Xa), Xa.shape[0], _lib.fptr(Ya)), "mlp forward")
            Y[a:a + self.max_batch] = Ya
        return Y

    def gradient(self, X, T):
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        g = np.zeros(_lib.MLP_NPARAMS, dtype=np.float32)
        loss = ct.c_float()
        self._check(self._lib.vpbs_mlp_gradient(self._h, _lib.fptr(X), _lib.fptr(T), X.shape[0], _lib.fptr(g),
                                                ct.byref(loss)), "mlp gradient")
        return float(loss.value), g

    def train_step(self, X, T, lr: float) -> float:
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        loss = ct.c_float()
        self._check(self._lib.vpbs_mlp_train_step(self._h, _lib.fptr(X), _lib.fptr(T), X.shape[0], float(lr),
                                                  ct.byref(loss)), "mlp train_step")
        return float(loss.value)


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases, in the flat layout of csrc/mlp.cu."""
    rng = np.random.default_rng(seed)
    I, H, O = _lib.MLP_IN, _lib.MLP_HIDDEN, _lib.MLP_OUT
    parts = [rng.normal(0, math.sqrt(2.0 / I), (H, I)), np.zeros(H), rng.normal(0, math.sqrt(2.0 / H), (H, H)),
             np.zeros(H), rng.normal(0, math.sqrt(1.0 / H), (O, H)), np.zeros(O)]
    return np.concatenate([p.ravel() for p in parts]).astype(np.float32)


def targets_of(choice: tuning.EwaldChoice, L: float) -> np.ndarray:
    """Network outputs of a parameter choice: (beta_short, log(r_cut / L), beta_long, sigma, m).
    alpha = beta_short / r_cut and the grid (through k_max = 2 alpha beta_long) follow from them;
    the betas, which set the accuracy, are predicted directly so that errors in alpha and r_cut
    do not compound."""
    return np.array([choice.beta_short, math.log(choice.rcut / L), choice.beta_long(L), choice.sigma, choice.m],
                    dtype=np.float64)


BETA_SHIFT = 0.15   # added to both predicted betas (conservative side of the regression noise)
RETRY_SHIFT = 0.45  # second attempt when the FP64 check rejects the first


def choice_of(y, L: float, shift: float = 0.0) -> tuning.EwaldChoice:
    """Valid parameters from (de-standardised) network outputs, the betas raised by `shift`."""
    rcut = min(max(math.exp(float(y[1])), 1 / 64), 0.35) * L
    beta_s = float(y[0]) + shift
    beta_l = float(y[2]) + shift
    sigma = min(tuning.SIGMAS, key=lambda s: abs(s - float(y[3])))
    m = int(min(max(round(float(y[4])), 2), 8))
    return tuning.choice_from(L, rcut, beta_s, beta_l, sigma, m)


@dataclass
class Predictor:
    """Trained network weights with the feature and output standardisation."""
    params: np.ndarray
    x_mean: np.ndarray
    x_std: np.ndarray
    y_mean: np.ndarray
    y_std: np.ndarray
    rtol: float

    def save(self, path):
        np.savez(path, params=self.params, x_mean=self.x_mean, x_std=self.x_std, y_mean=self.y_mean,
                 y_std=self.y_std, rtol=np.array(self.rtol))

    @classmethod
    def load(cls, path=DEFAULT_MODEL) -> "Predictor":
        z = np.load(path)
        return cls(params=z["params"].astype(np.float32), x_mean=z["x_mean"], x_std=z["x_std"], y_mean=z["y_mean"],
                   y_std=z["y_std"], rtol=float(z["rtol"]))

    def outputs(self, features, net: MLP | None = None) -> np.ndarray:
        X = ((np.atleast_2d(features) - self.x_mean) / self.x_std).astype(np.float32)
        own = net is None
        net = net or MLP(max_batch=max(1, X.shape[0]), params=self.params)
        try:
            if not own:
                net.set_params(self.params)
            Y = net.forward(X)
        finally:
            if own:
                net.close()
        return Y * self.y_std + self.y_mean

    def predict_choice(self, features, L: float, shift: float = BETA_SHIFT) -> tuning.EwaldChoice:
        return choice_of(self.outputs(features)[0], L, shift)


def feature_params(L: float, device: int = 0):
    """Parameters of the cache the features are computed on (its cell lists bound the nearest-
    distance search; its Fourier grid is never used)."""
    rcut = FEATURE_RCUT * L
    return ParamsBiotSavart(Gamma=1.0, a=1e-8, Delta=0.25,
                            splitting=GaussianSplitting(Ls=L, alpha=3.0 / rcut, rcut=rcut, Ns=16),
                            quadrature=GaussLegendre(3), backend_long=NonuniformFFTsBackend(1.5, 2), device=device)


def features_of(fs, L: float, device: int = 0) -> np.ndarray:
    from .biotsavart import init_cache
    c = init_cache(feature_params(L, device))
    try:
        c.set_filaments(fs)
        return c.features()
    finally:
        c.close()


def reference_choice(L: float) -> tuning.EwaldChoice:
    """Parameters of the FP64 reference the sweeps and the check compare against (beta = 4 in both
    ranges, r_cut = L/16, NUFFT m = 6): about 1e-8 relative error, far below the targets."""
    alpha = 4.0 / (L / 16)
    return tuning.EwaldChoice(alpha=alpha, rcut=L / 16, Ns=tuning.grid_for(
        tuning.kmax_to_gridsize(2 * alpha * 4.0, L), 1.5, 6), sigma=1.5, m=6)


def reference_velocity(fs, L: float, device: int = 0) -> np.ndarray:
    return tuning.measure(fs, reference_choice(L), L, precision="fp64", reps=1, device=device)[1]


def random_configuration(rng: np.random.Generator, L: float = 2 * math.pi, min_nodes: int = 5_000,
                         max_nodes: int = 1_200_000):
    """A random tangle of the benchmark's ring family: node count log-uniform in
    [min_nodes, max_nodes], random ring resolution (32-400 nodes per ring, at most 8000 rings) and
    radii (the training and held-out configurations)."""
    target = 10 ** rng.uniform(math.log10(min_nodes), math.log10(max_nodes))
    npr = int(rng.choice([32, 48, 64, 96, 128, 200, 256, 400]))
    nrings = int(min(max(1, round(target / npr)), 8000))
    rmin = L * rng.uniform(0.04, 0.14)
    rmax = min(rmin * rng.uniform(1.2, 2.5), L / 4)
    return curves.random_tangle(nrings, npr, L=L, rmin=rmin, rmax=rmax, seed=int(rng.integers(1 << 31)))


LABEL_MARGIN = 0.6  # labels are the cheapest sweep point with error <= LABEL_MARGIN * rtol


def sweep_configuration(fs, L: float, choices, rtol: float = 1e-5):
    """Features, sweep records and label (cheapest choice within LABEL_MARGIN * rtol) of one
    configuration, plus the cost of the default rule at rtol."""
    feats = features_of(fs, L)
    vref = reference_velocity(fs, L)
    recs = tuning.sweep(fs, L, vref, choices, "mixed")
    best = tuning.cheapest(recs, LABEL_MARGIN * rtol)
    d = tuning.sweep(fs, L, vref, [tuning.default_rule(L, rtol, FEATURE_RCUT * L)], "mixed")[0]
    return feats, recs, best, d


RCUT_FRACS = (1 / 12, 1 / 16, 1 / 20, 1 / 24, 1 / 32, 1 / 40, 1 / 48, 1 / 56)


def training_choices(L: float, reduced: bool = False):
    """The sweep grid: 8 cut-offs x 3 betas x 3 NUFFT (sigma, m) (72 sets), or with `reduced` the
    32 sets of the betas and NUFFTs that won most often on the full grid (betas 3.15 and 3.35;
    (sigma, m) = (1.5, 3) and (1.25, 4): 90 % of the 150 labels of the first data set)."""
    if reduced:
        return tuning.candidate_grid(L, rcut_fracs=RCUT_FRACS, betas=(3.15, 3.35), sigma_m=((1.25, 4), (1.5, 3)))
    return tuning.candidate_grid(L, rcut_fracs=RCUT_FRACS, betas=(2.95, 3.15, 3.35),
                                 sigma_m=((1.25, 4), (1.5, 3), (2.0, 3)))


def generate_dataset(n: int, seed: int, L: float = 2 * math.pi, rtol: float = 1e-5, min_nodes: int = 5_000,
                     max_nodes: int = 1_200_000, log=None, reduced: bool = False, deadline: float | None = None,
                     checkpoint=None, checkpoint_every: int = 25) -> dict:
    """(features, label) pairs of `n` random configurations from parameter sweeps against the
    FP64 reference, with the default rule's cost and error for comparison.  Stops early at the
    wall-clock `deadline` (time.time() value); `checkpoint(dataset)` is called every
    `checkpoint_every` configurations."""
    import time as _time
    rng = np.random.default_rng(seed)
    choices = training_choices(L, reduced)
    X, Y, nodes, best_ms, default_ms, default_err = [], [], [], [], [], []

    def pack():
        return {"X": np.array(X, dtype=np.float32), "Y": np.array(Y), "nodes": np.array(nodes),
                "best_ms": np.array(best_ms), "default_ms": np.array(default_ms),
                "default_err": np.array(default_err), "rtol": rtol, "L": L}

    for k in range(n):
        if deadline is not None and _time.time() > deadline:
            break
        if checkpoint is not None and k > 0 and k % checkpoint_every == 0:
            checkpoint(pack())
        fs = random_configuration(rng, L, min_nodes, max_nodes)
        feats, recs, best, d = sweep_configuration(fs, L, choices, rtol)
        if best is None:
            continue
        ch = tuning.EwaldChoice(alpha=best["alpha"], rcut=best["rcut"], Ns=best["Ns"], sigma=best["sigma"], m=best["m"])
        X.append(feats)
        Y.append(targets_of(ch, L))
        nodes.append(sum(len(f) for f in fs))
        best_ms.append(best["ms"])
        default_ms.append(d["ms"])
        default_err.append(d["rel_l2"])
        if log:
            log(f"{k}: N={nodes[-1]} best {best['ms']:.2f} ms (rcut L/{L / best['rcut']:.0f}, fft {best['fft']}, "
                f"m {best['m']}) default {d['ms']:.2f} ms err {d['rel_l2']:.1e}")
    return pack()


def train(X, Y, rtol: float, steps: int = 1000, lr: float = 1e-3, weight_decay: float = 1e-2, seed: int = 0,
          device: int = 0) -> Predictor:
    """Full-batch Adam with an L2 term on the GPU (the library's MLP kernels) on standardised
    inputs/outputs.  The defaults were chosen by 5-fold cross-validation on the sweep data (the
    labels are noisy argmins, so a short, regularised fit generalises best)."""
    X = np.asarray(X, dtype=np.float64)
    Y = np.asarray(Y, dtype=np.float64)
    x_mean, x_std = X.mean(0), X.std(0) + 1e-6
    y_mean, y_std = Y.mean(0), Y.std(0) + 1e-6
    Xs = ((X - x_mean) / x_std).astype(np.float32)
    Ys = ((Y - y_mean) / y_std).astype(np.float32)
    net = MLP(max_batch=len(Xs), device=device, seed=seed)
    net._check(net._lib.vpbs_mlp_set_weight_decay(net._h, float(weight_decay)), "mlp set_weight_decay")
    try:
        for s in range(steps):
            net.train_step(Xs, Ys, lr if s < steps // 2 else lr / 4)
        params = net.get_params()
    finally:
        net.close()
    return Predictor(params=params, x_mean=x_mean, x_std=x_std, y_mean=y_mean, y_std=y_std, rtol=rtol)


KB_MARGIN = 4.0  # Kaiser-Bessel beta from the reference's rule rtol = C exp(-beta) at rtol / KB_MARGIN


KB_NUFFT = ((1.5, 3), (2.0, 3))  # NUFFT (sigma, m) tried besides the predicted one


def kaiser_bessel_variants(ch: tuning.EwaldChoice, L: float, rtol: float) -> list[tuning.KBChoice]:
    """Kaiser-Bessel splits at the predicted cut-off: beta from the reference's accuracy rule
    (kaiser_bessel.jl:104-109) at rtol / KB_MARGIN, grid resolving k_max = beta / r_cut (rounded
    as for the Gaussian choices), with the predicted NUFFT (sigma, m) and the narrower kernels of
    KB_NUFFT (cheaper spreading; the smaller Kaiser-Bessel grid makes the wider oversampling
    affordable).  Compact support needs a much smaller grid than the Gaussian at the same
    cut-off (about (21.6 / 13.4)^3 = 4x fewer modes at rtol 1e-6)."""
    from .params import C_RTOL_KB
    beta = -math.log(rtol / KB_MARGIN / C_RTOL_KB)
    out = []
    for sigma, m in ((ch.sigma, ch.m),) + KB_NUFFT:
        kb = tuning.kb_choice_from(L, ch.rcut, beta, sigma, m)
        if kb not in out:
            out.append(kb)
    return out


def class_features(fs, L: float) -> np.ndarray:
    """Host-side summary of a configuration for ChoiceCache (numpy, no GPU): log10 N,
    log10(line length / L^2), log10 of the mean and the minimum chord / L (closing chords included;
    an unclosed filament's closing chord runs to its first node plus the end-to-end offset)."""
    n, total, cmin = 0, 0.0, math.inf
    for f in fs:
        x = np.asarray(f, dtype=np.float64)
        nxt = np.roll(x, -1, axis=0)
        nxt[-1] = nxt[-1] + curves.end_to_end_offset(f)
        d = np.linalg.norm(nxt - x, axis=1)
        n += len(x)
        total += float(d.sum())
        cmin = min(cmin, float(d.min()))
    return np.array([math.log10(n), math.log10(total / L ** 2), math.log10(total / n / L), math.log10(cmin / L)])


class ChoiceCache:
    """Checked parameter choices per configuration class, so that a solver meeting similar
    configurations again (the steps of one simulation, an ensemble of similar tangles) pays the FP64
    check once per class instead of once per call; a lookup costs a numpy pass over the nodes.

    The class of a configuration: L, rtol and its ``class_features`` rounded -- log10 N and
    log10(line length / L^2) to 1/8 (steps of 33 %), log10 of the mean and minimum chord / L to 1/4.
    With `path`, entries are read from and written to that JSON file."""

    def __init__(self, path: str | Path | None = None):
        import json
        self.path = Path(path) if path else None
        self.entries: dict[str, dict] = {}
        if self.path and self.path.exists():
            self.entries = json.loads(self.path.read_text())

    @staticmethod
    def key(cf, L: float, rtol: float) -> str:
        f = np.asarray(cf, dtype=np.float64).ravel()
        parts = [round(L, 9), float(f"{rtol:.3e}"), int(round(8 * f[0])), int(round(8 * f[1])),
                 int(round(4 * f[2])), int(round(4 * f[3]))]
        return "/".join(str(x) for x in parts)

    def get(self, feats, L: float, rtol: float):
        e = self.entries.get(self.key(feats, L, rtol))
        if e is None:
            return None
        d = dict(e["choice"])
        if d.pop("splitting", "gaussian") == "kaiser_bessel":
            return tuning.KBChoice(**d), e
        return tuning.EwaldChoice(**d), e

    def put(self, feats, L: float, rtol: float, choice, rel_l2, fallback: bool) -> None:
        import json
        self.entries[self.key(feats, L, rtol)] = {"choice": choice.as_dict(), "rel_l2": rel_l2,
                                                  "fallback": bool(fallback)}
        if self.path:
            self.path.write_text(json.dumps(self.entries, indent=1))


def choose_parameters(fs, L: float, rtol: float = 1e-5, predictor: Predictor | None = None, check: bool = True,
                      device: int = 0, kaiser_bessel: bool = True, cache: ChoiceCache | None = None):
    """Predicted parameters for `fs` at tolerance `rtol`.  With `check`, a plain FP64 evaluation
    judges the prediction (mixed form); a rejected prediction is retried once with larger betas,
    and the default rule replaces it when that also misses rtol.  With `kaiser_bessel`, the
    Kaiser-Bessel splits at the accepted cut-off (``kaiser_bessel_variants``) are judged the same
    way and the fastest choice meeting rtol is kept.  With `cache`, a checked choice of the same
    configuration class is returned without a new check (info["cached"]), and a new checked
    choice is stored.  Returns (choice, info)."""
    cf = class_features(fs, L) if cache is not None else None
    if cache is not None and check:
        hit = cache.get(cf, L, rtol)
        if hit is not None:
            ch, e = hit
            return ch, {"features": None, "predicted": None, "attempts": [], "fallback": e["fallback"],
                        "rel_l2": e["rel_l2"], "cached": True}
    pred = predictor or Predictor.load()
    feats = features_of(fs, L, device)
    y = pred.outputs(feats)[0]
    ch = choice_of(y, L, BETA_SHIFT)
    info = {"features": feats, "outputs": y, "predicted": ch, "attempts": [], "fallback": False, "cached": False}
    if not check:
        return ch, info
    vref = reference_velocity(fs, L, device)
    accepted = None
    for shift in (BETA_SHIFT, RETRY_SHIFT):
        ch = choice_of(y, L, shift)
        ms, v = tuning.measure(fs, ch, L, "mixed", reps=2, device=device)
        err = tuning.rel_errors(v, vref)[0]
        info["attempts"].append({"shift": shift, "rel_l2": err, "ms": ms, **ch.as_dict()})
        if err <= rtol:
            accepted = (ch, err, ms)
            break
    if accepted is None:
        info["fallback"] = True
        ch = tuning.default_rule(L, rtol, FEATURE_RCUT * L)
        if cache is not None:
            cache.put(cf, L, rtol, ch, None, True)
        return ch, info
    if kaiser_bessel:
        for kb in kaiser_bessel_variants(accepted[0], L, rtol):
            ms, v = tuning.measure(fs, kb, L, "mixed", reps=2, device=device)
            err = tuning.rel_errors(v, vref)[0]
            info["attempts"].append({"rel_l2": err, "ms": ms, **kb.as_dict()})
            if err <= rtol and ms < accepted[2]:
                accepted = (kb, err, ms)
    info["rel_l2"] = accepted[1]
    if cache is not None:
        cache.put(cf, L, rtol, accepted[0], accepted[1], False)
    return accepted[0], info
