"""Learned warm start of the parquet loop.

No counterpart in the reference, whose loop starts from Sigma = 0 and
F_r = Gamma_r = Lambda_r on the (l=1, l=1) nu-block (preprocessing.f90:100-116).
Here a small network maps (U, beta, n, t', Sigma after two plain iterations)
to the converged Sigma and to one constant per channel for the (l=1, l=1)
block of Gamma_r; the library rebuilds F_r from that Gamma_r with one BSE
solve in LU form (``Solver.warm_start``).  The plain iteration then runs to
the same convergence threshold as a cold start.  When the first iteration
after the warm start moves Sigma further than the last cold iteration did
(or fails), the state saved before the warm start is restored and the run
continues cold: at most one iteration is lost.

Pieces:

* ``MLP``: FP32 network with SiLU hidden layers, forward/backward/Adam in
  the library's own CUDA kernels (``tups_mlp_*``).
* ``reduce_sigma`` / ``expand_sigma``: Sigma on the irreducible k wedge and
  back (C4v point group of the square lattice).
* ``run_cold`` / ``run_warm``: one loop to ``conv_abs`` each.
* ``WarmStart``: feature scaling + network; ``fit`` and ``predict``.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import asdict, dataclass, replace

import numpy as np

from . import _lib
from ._lib import TupsError
from .parquet import Params, Solver


# --------------------------------------------------------------------------
# network
# --------------------------------------------------------------------------
def mlp_widths(n_in: int, n_out: int, hidden: int = 512, layers: int = 3) -> list[int]:
    return [n_in] + [hidden] * layers + [n_out]


def mlp_init_params(widths, seed: int) -> np.ndarray:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights, zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for fin, fout in zip(widths[:-1], widths[1:]):
        lim = 1.0 / np.sqrt(fin)
        parts.append(rng.uniform(-lim, lim, fin * fout).astype(np.float32))
        parts.append(np.zeros(fout, dtype=np.float32))
    return np.concatenate(parts)


def _f32(a, cols: int) -> np.ndarray:
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim == 1:
        a = a.reshape(1, -1)
    assert a.shape[1] == cols, (a.shape, cols)
    return a


def _fp(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data)


class MLP:
    """FP32 multilayer perceptron trained and evaluated by the library's kernels."""

    def __init__(self, n_in: int, n_out: int, hidden: int = 512, layers: int = 3, max_batch: int = 256,
                 device: int = 0, seed: int = 0):
        self.lib = _lib.load()
        self.widths = mlp_widths(n_in, n_out, hidden, layers)
        self.n_in, self.n_out, self.max_batch = n_in, n_out, max_batch
        h = C.c_void_p()
        rc = self.lib.tups_mlp_create(n_in, hidden, layers, n_out, max_batch, device, C.byref(h))
        if rc:
            raise TupsError(rc, "tups_mlp_create failed")
        self.h = h
        self.n_params = int(self.lib.tups_mlp_num_params(h))
        self.set_params(mlp_init_params(self.widths, seed))

    def _call(self, name, *args):
        rc = getattr(self.lib, name)(self.h, *args)
        if rc:
            raise TupsError(rc, self.lib.tups_mlp_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.tups_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.tups_mlp_kernel_launches(self.h))

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.n_params
        self._call("tups_mlp_set_params", _fp(p))

    def get_params(self) -> np.ndarray:
        p = np.empty(self.n_params, dtype=np.float32)
        self._call("tups_mlp_get_params", _fp(p))
        return p

    def forward(self, x) -> np.ndarray:
        x = _f32(x, self.n_in)
        out = []
        for i in range(0, x.shape[0], self.max_batch):
            xb = np.ascontiguousarray(x[i:i + self.max_batch])
            y = np.empty((xb.shape[0], self.n_out), dtype=np.float32)
            self._call("tups_mlp_forward", _fp(xb), xb.shape[0], _fp(y))
            out.append(y)
        return np.concatenate(out)

    def gradients(self, x, t) -> tuple[float, np.ndarray]:
        x = _f32(x, self.n_in)
        t = _f32(t, self.n_out)
        g = np.empty(self.n_params, dtype=np.float32)
        loss = C.c_double()
        self._call("tups_mlp_gradients", _fp(x), _fp(t), x.shape[0], _fp(g), C.byref(loss))
        return loss.value, g

    def train(self, x, t, batch: int = 32, epochs: int = 100, lr: float = 1e-3, weight_decay: float = 0.0,
              seed: int = 0) -> np.ndarray:
        x = _f32(x, self.n_in)
        t = _f32(t, self.n_out)
        hist = np.zeros(max(epochs, 1))
        self._call("tups_mlp_train", _fp(x), _fp(t), x.shape[0], int(batch), int(epochs), C.c_float(lr),
                   C.c_float(weight_decay), C.c_ulonglong(seed), _fp(hist))
        return hist[:epochs]


# --------------------------------------------------------------------------
# Sigma on the irreducible wedge
# --------------------------------------------------------------------------
def wedge_points(Nx: int) -> list[tuple[int, int]]:
    """0 <= ky <= kx <= Nx/2, in the order of the features."""
    return [(kx, ky) for kx in range(Nx // 2 + 1) for ky in range(kx + 1)]


def _wedge_index(Nx: int) -> np.ndarray:
    """For every (ix, iy) of the full grid, its wedge point's position."""
    pos = {k: i for i, k in enumerate(wedge_points(Nx))}
    out = np.empty((Nx, Nx), dtype=np.int64)
    for ix in range(Nx):
        for iy in range(Nx):
            fx, fy = min(ix, Nx - ix), min(iy, Nx - iy)
            out[ix, iy] = pos[(max(fx, fy), min(fx, fy))]
    return out


def reduce_sigma(sigma: np.ndarray, Nx: int, Nf: int) -> np.ndarray:
    """Sigma (Nx*Nx*Nf, layout (ix, iy, nu) row-major) -> (wedge points, Nf).

    All Nf frequencies are kept: the truncated frequency box breaks
    Sigma(k, -nu) = conj Sigma(k, nu) at the 1e-4 level."""
    s = np.asarray(sigma).reshape(Nx, Nx, Nf)
    return np.array([s[kx, ky, :] for kx, ky in wedge_points(Nx)])


def expand_sigma(red: np.ndarray, Nx: int, Nf: int) -> np.ndarray:
    """Inverse of ``reduce_sigma`` for a C4v-symmetric Sigma."""
    return np.asarray(red)[_wedge_index(Nx)].reshape(-1)


# --------------------------------------------------------------------------
# one loop, cold or warm
# --------------------------------------------------------------------------
@dataclass
class RunResult:
    iterations: int
    seconds: float
    converged: bool
    sigma2: np.ndarray | None = None      # Sigma after two iterations
    sigma: np.ndarray | None = None       # final Sigma
    gamma_l1: np.ndarray | None = None    # mean of Gamma_r over its (l=1, l=1) block, 4 channels
    history: list | None = None           # max |Delta Sigma| per iteration
    fallback: bool = False


N_PLAIN = 2  # plain iterations before the warm start


def _gamma_l1(sol: Solver) -> np.ndarray:
    Nf = sol.Nf
    return np.array([sol.G(r)[:Nf, :Nf, :].mean() for r in range(4)])


def run_cold(params: Params, max_iter: int = 2000, device: int = 0, summary: bool = True) -> RunResult:
    """The plain loop from the reference's initial state until conv_abs.

    A run that stops with a library error (NaN, mu bisection) is returned
    as not converged."""
    sol = Solver(params, device=device)
    try:
        hist, sig2, ok = [], None, False
        t0 = time.perf_counter()
        ite = 0
        try:
            while ite < max_iter:
                ci = sol.iteration(ite)
                hist.append(ci["dsigma_inf"])
                ite += 1
                if ite == N_PLAIN:
                    sig2 = sol.Sigma
                if ci["converged"]:
                    ok = True
                    break
        except TupsError:
            ok = False
        secs = time.perf_counter() - t0
        res = RunResult(ite, secs, ok, sigma2=sig2, history=hist)
        if summary and ok:
            res.sigma = sol.Sigma
            res.gamma_l1 = _gamma_l1(sol)
        return res
    finally:
        sol.close()


def run_warm(params: Params, predictor, max_iter: int = 2000, device: int = 0, accept: float = 1.0) -> RunResult:
    """Two plain iterations, the predicted warm start, then the plain loop.

    ``predictor(params, sigma2) -> (sigma, gamma_l1)``.  The warm start is
    kept when the first iteration after it changes Sigma by less than
    ``accept`` times the last plain iteration did; otherwise the saved state
    is restored and the plain loop continues.  ``iterations`` counts every
    iteration run, the rejected one included."""
    sol = Solver(params, device=device)
    try:
        hist, ok, fell_back = [], False, False
        t0 = time.perf_counter()
        ite = 0
        while ite < N_PLAIN:
            ci = sol.iteration(ite)
            hist.append(ci["dsigma_inf"])
            ite += 1
            if ci["converged"]:
                return RunResult(ite, time.perf_counter() - t0, True, history=hist, sigma=sol.Sigma)
        sig2 = sol.Sigma
        last = hist[-1]
        sol.checkpoint(True)
        try:
            sigma, gamma = predictor(params, sig2)
            sol.warm_start(sigma, gamma)
            ci = sol.iteration(ite)
            good = bool(np.isfinite(ci["dsigma_inf"]) and ci["dsigma_inf"] < accept * last)
        except TupsError:
            good = False
        extra = 0
        if not good:
            fell_back, extra = True, 1
            sol.checkpoint(False)
            ci = sol.iteration(ite)
        hist.append(ci["dsigma_inf"])
        ite += 1
        ok = ci["converged"]
        try:
            while not ok and ite < max_iter:
                ci = sol.iteration(ite)
                hist.append(ci["dsigma_inf"])
                ite += 1
                ok = ci["converged"]
        except TupsError:
            ok = False
        secs = time.perf_counter() - t0
        return RunResult(ite + extra, secs, ok, history=hist, sigma=sol.Sigma, fallback=fell_back)
    finally:
        sol.close()


# --------------------------------------------------------------------------
# features and the trained predictor
# --------------------------------------------------------------------------
PARAM_KEYS = ("U", "beta", "nParticle", "tprime")


def features(params: Params, sigma2: np.ndarray) -> np.ndarray:
    red = reduce_sigma(sigma2, params.Nx, params.Nf).reshape(-1)
    return np.concatenate([[getattr(params, k) for k in PARAM_KEYS], red.real, red.imag]).astype(np.float64)


def targets(params: Params, sigma2: np.ndarray, sigma: np.ndarray, gamma_l1: np.ndarray) -> np.ndarray:
    d = (reduce_sigma(sigma, params.Nx, params.Nf) - reduce_sigma(sigma2, params.Nx, params.Nf)).reshape(-1)
    g = np.asarray(gamma_l1).reshape(4)
    return np.concatenate([d.real, d.imag, g.real, g.imag]).astype(np.float64)


class WarmStart:
    """Feature scaling + ``MLP``; ``predict`` has the signature ``run_warm`` wants."""

    def __init__(self, Nx: int, Nf: int, hidden: int = 512, layers: int = 3, device: int = 0, seed: int = 0):
        self.Nx, self.Nf = Nx, Nf
        self.nw = len(wedge_points(Nx)) * Nf
        self.n_in = len(PARAM_KEYS) + 2 * self.nw
        self.n_out = 2 * self.nw + 8
        self.net = MLP(self.n_in, self.n_out, hidden, layers, max_batch=256, device=device, seed=seed)
        self.xm = self.xs = self.ym = self.ys = None

    @staticmethod
    def _scale(a):
        m = a.mean(axis=0)
        s = a.std(axis=0)
        s[s < 1e-12 * max(1.0, float(np.abs(m).max()))] = 1.0
        return m, s

    def fit(self, X: np.ndarray, Y: np.ndarray, epochs: int = 2000, batch: int = 32, lr: float = 1e-3,
            weight_decay: float = 1e-4, seed: int = 0) -> np.ndarray:
        self.xm, self.xs = self._scale(X)
        self.ym, self.ys = self._scale(Y)
        xn = (X - self.xm) / self.xs
        yn = (Y - self.ym) / self.ys
        # step decay of the learning rate: half the epochs at lr, then lr/4, lr/16
        hist = []
        for k, frac in enumerate((0.5, 0.25, 0.25)):
            hist.append(self.net.train(xn, yn, batch=batch, epochs=max(1, int(epochs * frac)), lr=lr / 4 ** k,
                                       weight_decay=weight_decay, seed=seed + k))
        return np.concatenate(hist)

    def predict_raw(self, X: np.ndarray) -> np.ndarray:
        xn = (np.atleast_2d(X) - self.xm) / self.xs
        return self.net.forward(xn).astype(np.float64) * self.ys + self.ym

    def predict(self, params: Params, sigma2: np.ndarray):
        y = self.predict_raw(features(params, sigma2))[0]
        nw = self.nw
        d = (y[:nw] + 1j * y[nw:2 * nw]).reshape(-1, self.Nf)
        red = reduce_sigma(sigma2, self.Nx, self.Nf) + d
        gamma = y[2 * nw:2 * nw + 4] + 1j * y[2 * nw + 4:2 * nw + 8]
        return expand_sigma(red, self.Nx, self.Nf), gamma

    def close(self) -> None:
        self.net.close()


# --------------------------------------------------------------------------
# the parameter sweep: data, training, evaluation
# --------------------------------------------------------------------------
SWEEP = dict(U=(1.0, 4.0), beta=(2.0, 10.0), nParticle=(0.8, 1.0), tprime=(-0.3, 0.0))


def sweep_params(n: int, seed: int, base: Params) -> list[Params]:
    """n parameter sets drawn uniformly from SWEEP (one generator, fixed order)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        kw = {k: float(rng.uniform(lo, hi)) for k, (lo, hi) in SWEEP.items()}
        out.append(replace(base, **kw))
    return out


def sweep(base: Params, runs: int = 200, n_train: int = 160, seed: int = 0, max_iter: int = 2000,
          epochs: int = 3000, batch: int = 32, lr: float = 1e-3, weight_decay: float = 1e-4, device: int = 0,
          log=print) -> dict:
    """Cold runs for every parameter set; train on the first n_train converged
    ones; warm vs cold on the rest.  Returns a summary and per-run records."""
    params = sweep_params(runs, seed, base)
    cold = []
    for i, p in enumerate(params):
        r = run_cold(p, max_iter=max_iter, device=device)
        cold.append(r)
        log(f"cold {i:3d} U={p.U:.3f} beta={p.beta:.3f} n={p.nParticle:.3f} t'={p.tprime:.3f}: "
            f"{r.iterations} it {r.seconds:.3f} s converged={r.converged}")
    idx_train = [i for i in range(min(n_train, runs)) if cold[i].converged]
    idx_test = [i for i in range(n_train, runs) if cold[i].converged]
    X = np.array([features(params[i], cold[i].sigma2) for i in idx_train])
    Y = np.array([targets(params[i], cold[i].sigma2, cold[i].sigma, cold[i].gamma_l1) for i in idx_train])
    ws = WarmStart(base.Nx, base.Nf, device=device, seed=seed)
    t0 = time.perf_counter()
    hist = ws.fit(X, Y, epochs=epochs, batch=batch, lr=lr, weight_decay=weight_decay, seed=seed)
    t_train = time.perf_counter() - t0
    log(f"trained on {len(idx_train)} runs: loss {hist[0]:.3e} -> {hist[-1]:.3e} in {t_train:.1f} s")
    rec = []
    for i in idx_test:
        p = params[i]
        ref = run_cold(p, max_iter=max_iter, device=device, summary=False)
        w = run_warm(p, ws.predict, max_iter=max_iter, device=device)
        forced = run_warm(p, ws.predict, max_iter=max_iter, device=device, accept=np.inf)
        y = ws.predict_raw(features(p, cold[i].sigma2))[0]
        t = targets(p, cold[i].sigma2, cold[i].sigma, cold[i].gamma_l1)
        nw = ws.nw
        err_pred = float(np.max(np.abs(y[:2 * nw] - t[:2 * nw])) / np.max(np.abs(t[:2 * nw])))
        sig_scale = float(np.max(np.abs(cold[i].sigma)))
        rec.append(dict(run=i, U=p.U, beta=p.beta, n=p.nParticle, tprime=p.tprime,
                        cold_iterations=ref.iterations, cold_seconds=ref.seconds,
                        warm_iterations=w.iterations, warm_seconds=w.seconds, fallback=w.fallback,
                        warm_converged=w.converged, forced_iterations=forced.iterations,
                        forced_converged=forced.converged,
                        forced_final_sigma_rel_diff=float(np.max(np.abs(forced.sigma - cold[i].sigma)) / sig_scale),
                        sigma_pred_rel_err=float(np.max(np.abs(ws.predict(p, cold[i].sigma2)[0] - cold[i].sigma))
                                                 / sig_scale),
                        sigma2_rel_err=float(np.max(np.abs(cold[i].sigma2 - cold[i].sigma)) / sig_scale),
                        delta_pred_rel_err=err_pred,
                        final_sigma_rel_diff=float(np.max(np.abs(w.sigma - cold[i].sigma)) / sig_scale)))
        r = rec[-1]
        log(f"test {i:3d}: cold {r['cold_iterations']} it {r['cold_seconds']:.3f} s | warm {r['warm_iterations']} it "
            f"{r['warm_seconds']:.3f} s fallback={r['fallback']} | Sigma err pred {r['sigma_pred_rel_err']:.2e} "
            f"vs after 2 it {r['sigma2_rel_err']:.2e}")
    ws.close()
    ci = np.array([r["cold_iterations"] for r in rec], dtype=float)
    wi = np.array([r["warm_iterations"] for r in rec], dtype=float)
    cs = np.array([r["cold_seconds"] for r in rec])
    wsec = np.array([r["warm_seconds"] for r in rec])
    summary = dict(runs=runs, converged=sum(r.converged for r in cold), n_train=len(idx_train), n_test=len(rec),
                   train_seconds=t_train, loss_first=float(hist[0]), loss_last=float(hist[-1]),
                   cold_iterations_mean=float(ci.mean()) if len(rec) else None,
                   warm_iterations_mean=float(wi.mean()) if len(rec) else None,
                   cold_seconds_total=float(cs.sum()), warm_seconds_total=float(wsec.sum()),
                   fallbacks=int(sum(r["fallback"] for r in rec)),
                   forced_iterations_mean=float(np.mean([r["forced_iterations"] for r in rec])) if rec else None,
                   forced_all_converged=bool(all(r["forced_converged"] for r in rec)),
                   all_warm_converged=bool(all(r["warm_converged"] for r in rec)),
                   max_final_sigma_rel_diff=float(max((r["final_sigma_rel_diff"] for r in rec), default=0.0)),
                   sigma_pred_rel_err_median=float(np.median([r["sigma_pred_rel_err"] for r in rec]))
                   if rec else None,
                   sigma2_rel_err_median=float(np.median([r["sigma2_rel_err"] for r in rec])) if rec else None)
    return dict(summary=summary, tests=rec,
                cold=[dict(run=i, iterations=c.iterations, seconds=c.seconds, converged=c.converged)
                      for i, c in enumerate(cold)],
                loss=[float(v) for v in hist])


def restart_study(params: Params, max_iter: int = 2000, device: int = 0) -> dict:
    """How much an ideal warm start could save: converge cold, then restart
    from the state after N_PLAIN plain iterations with parts of it replaced by
    the converged ones (Sigma only, vertices only, both on the (l=1, l=1)
    block only, everything), or moved a fraction a of the way back from the
    converged state towards the 2-iteration state.  Returns iterations to
    conv_abs per variant (N_PLAIN included)."""
    sol = Solver(params, device=device)
    n_cold = 0
    while n_cold < max_iter and not sol.iteration(n_cold)["converged"]:
        n_cold += 1
    n_cold += 1
    S = sol.Sigma
    F = [sol.F(r) for r in range(4)]
    G = [sol.G(r) for r in range(4)]
    sol.close()
    Nf = params.Nf
    sol = Solver(params, device=device)
    for ite in range(N_PLAIN):
        sol.iteration(ite)
    S2 = sol.Sigma
    F2 = [sol.F(r) for r in range(4)]
    G2 = [sol.G(r) for r in range(4)]
    sol.checkpoint(True)

    def put(sig, f, g):
        sol.Sigma = sig
        for r in range(4):
            sol.set_vertex(r, 0, f[r])
            sol.set_vertex(r, 1, g[r])

    def l1(conv, two):
        out = [x.copy() for x in two]
        for r in range(4):
            out[r][:Nf, :Nf] = conv[r][:Nf, :Nf]
        return out

    variants = {
        "plain": None,
        "sigma_converged": (S, F2, G2),
        "vertices_converged": (S2, F, G),
        "sigma_and_l1_block_converged": (S, l1(F, F2), l1(G, G2)),
        "all_converged": (S, F, G),
    }
    for a in (0.01, 0.1, 0.5):
        variants[f"converged+{a}*(2-iteration - converged)"] = (
            S + a * (S2 - S), [x + a * (y - x) for x, y in zip(F, F2)], [x + a * (y - x) for x, y in zip(G, G2)])
    out = {"cold_iterations": n_cold}
    for name, st in variants.items():
        sol.checkpoint(False)
        if st is not None:
            put(*st)
        n = N_PLAIN
        while n < max_iter and not sol.iteration(n)["converged"]:
            n += 1
        out[name] = n + 1
    sol.close()
    return out


def main(argv=None) -> None:
    import argparse
    import json
    ap = argparse.ArgumentParser(description="learned warm start over a seeded parameter sweep")
    ap.add_argument("--runs", type=int, default=200)
    ap.add_argument("--train", type=int, default=160)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--Nx", type=int, default=8)
    ap.add_argument("--Nf", type=int, default=32)
    ap.add_argument("--neighbours", type=int, default=2)
    ap.add_argument("--max-iter", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--conv-abs", type=float, default=1e-10)
    ap.add_argument("--out", default=None, help="JSON file for the summary and per-run records")
    ap.add_argument("--restart-study", action="store_true",
                    help="only the ideal-restart study at U=2, beta=5, n=1 and U=3.5, beta=8, n=0.85, t'=-0.2")
    a = ap.parse_args(argv)
    base = Params(Nx=a.Nx, Nf=a.Nf, neighbours=a.neighbours, f_damping=0.5, use_U2=True, ite_max=10 ** 6,
                  conv_abs=a.conv_abs)
    if a.restart_study:
        res = {}
        for kw in (dict(U=2.0, beta=5.0, nParticle=1.0, tprime=0.0),
                   dict(U=3.5, beta=8.0, nParticle=0.85, tprime=-0.2)):
            res[json.dumps(kw)] = restart_study(replace(base, **kw), max_iter=a.max_iter)
            print(json.dumps({"params": kw, **res[json.dumps(kw)]}), flush=True)
        if a.out:
            with open(a.out, "w") as f:
                json.dump(res, f, indent=1)
        return
    res = sweep(base, runs=a.runs, n_train=a.train, seed=a.seed, max_iter=a.max_iter, epochs=a.epochs)
    print(json.dumps(res["summary"]))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
