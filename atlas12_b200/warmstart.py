"""Learned warm start for the ATLAS12 iteration.

A small MLP (4 -> 256 -> 256 -> 216, FP32, tanh) maps the stellar parameters
(Teff, log g, [M/H], vturb) to a starting structure on the standard Rosseland
grid: log10 T, log10 P and log10 Ne at each of the 72 depths.  It is trained on
converged models that this library's own ATLAS12 iteration produces, with the
library's forward / backward / Adam kernels (csrc/mlp.cu).  The plain grey
start stays the fallback, and the unmodified iteration still judges
convergence, so the network can only shorten the iteration.

    ws = WarmStart.load(path, ctx)
    start = ws.start(teff, logg, mh, vturb)      # dict t, p, rhox, tauros, xne
    model.set_params(teff, logg, vturb, mh); model.set_structure(start["t"], start["p"], start["rhox"])
"""
import ctypes

import numpy as np

from . import _lib, surrogate
from ._lib import ptr

NRHOX = 72
TAUSTD = 10.0 ** (-6.875 + 0.125 * np.arange(NRHOX))
SHAPE = (4, 256, 256, 3 * NRHOX)
# parameter box of the training grid: Teff, log g, [M/H], vturb (km/s)
BOX = np.array([[3500.0, 8000.0], [1.0, 5.0], [-2.0, 0.5], [0.5, 3.0]])


def sample_params(n, seed, box=BOX):
    """n parameter sets uniform in the box (seeded)."""
    rng = np.random.default_rng(seed)
    return box[:, 0] + (box[:, 1] - box[:, 0]) * rng.uniform(size=(n, 4))


def encode_inputs(params, box=BOX):
    """Parameters to [-1, 1] over the box."""
    p = np.atleast_2d(np.asarray(params, dtype=np.float64))
    return (2.0 * (p - box[:, 0]) / (box[:, 1] - box[:, 0]) - 1.0).astype(np.float32)


class MLP:
    """The device network (csrc/mlp.cu) on one context."""

    def __init__(self, ctx, shape=SHAPE, seed=1):
        self.ctx = ctx
        self.shape = tuple(shape)
        self._h = ctypes.c_void_p()
        ctx.call("atlasgpu_mlp_create", *[int(s) for s in self.shape], ctypes.c_uint64(seed), ctypes.byref(self._h))
        self.nparam = int(_lib.lib().atlasgpu_mlp_nparam(self._h))

    def params(self):
        out = np.zeros(self.nparam, np.float32)
        self.ctx.call("atlasgpu_mlp_get_params", self._h, ptr(out))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.nparam
        self.ctx.call("atlasgpu_mlp_set_params", self._h, ptr(p))

    def forward(self, x):
        x = np.ascontiguousarray(np.atleast_2d(x), np.float32)
        y = np.zeros((x.shape[0], self.shape[3]), np.float32)
        self.ctx.call("atlasgpu_mlp_forward", self._h, ptr(x), x.shape[0], ptr(y))
        return y

    def loss_grad(self, x, t):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        g = np.zeros(self.nparam, np.float32)
        loss = ctypes.c_float(0.0)
        self.ctx.call("atlasgpu_mlp_loss_grad", self._h, ptr(x), ptr(t), x.shape[0], ptr(g), ctypes.byref(loss))
        return float(loss.value), g

    def train(self, x, t, epochs, batch=64, lr=1e-3, seed=7):
        x = np.ascontiguousarray(x, np.float32)
        t = np.ascontiguousarray(t, np.float32)
        hist = np.zeros(max(epochs, 1), np.float32)
        self.ctx.call("atlasgpu_mlp_train", self._h, ptr(x), ptr(t), x.shape[0], int(epochs), int(batch),
                      ctypes.c_float(lr), ctypes.c_uint64(seed), ptr(hist))
        return hist[:epochs]

    def close(self):
        if self._h:
            _lib.lib().atlasgpu_mlp_destroy(self.ctx.handle, self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def structure_targets(t, p, xne):
    """[n, 216] = log10 T, log10 P, log10 Ne per depth."""
    return np.concatenate([np.log10(t), np.log10(p), np.log10(np.maximum(xne, 1.0))], axis=1)


class WarmStart:
    """Trained network plus the output standardisation.

    With residual = True (the default for training) the network predicts
    log10 T and log10 P relative to the plain grey start of the same
    parameters, which already carries most of their variation across the box;
    log10 Ne is predicted absolute (the iteration recomputes it anyway)."""

    def __init__(self, mlp, ymean, ystd, residual=False):
        self.mlp = mlp
        self.ymean = np.asarray(ymean, np.float64)
        self.ystd = np.asarray(ystd, np.float64)
        self.residual = bool(residual)

    @staticmethod
    def _grey_logs(params):
        g = [grey_start(teff, logg, mh) for teff, logg, mh, _ in np.atleast_2d(params)]
        return np.array([np.log10(x["t"]) for x in g]), np.array([np.log10(x["p"]) for x in g])

    @classmethod
    def fit(cls, ctx, params, t, p, xne, epochs=2000, batch=64, lr=1e-3, seed=1, residual=True, lr_tail=None,
            tail_epochs=0):
        """Train on converged structures (each [n, 72]); returns (WarmStart, loss history).
        A second phase of tail_epochs at lr_tail follows when given."""
        y = structure_targets(t, p, xne)
        if residual:
            gt, gp = cls._grey_logs(params)
            y[:, :NRHOX] -= gt
            y[:, NRHOX:2 * NRHOX] -= gp
        ymean, ystd = y.mean(0), np.maximum(y.std(0), 1e-3)
        mlp = MLP(ctx, seed=seed)
        x = encode_inputs(params)
        yn = ((y - ymean) / ystd).astype(np.float32)
        hist = mlp.train(x, yn, epochs, batch, lr, seed + 1)
        if tail_epochs and lr_tail:
            hist = np.concatenate([hist, mlp.train(x, yn, tail_epochs, batch, lr_tail, seed + 2)])
        return cls(mlp, ymean, ystd, residual), hist

    def predict(self, params, grey=None):
        """T, P, XNE [n, 72] for params [n, 4] from one forward pass; grey:
        the plain grey starts of the same parameters, when the caller has
        them (the residual network adds to their log T and log P)."""
        params = np.atleast_2d(params)
        return self.destandardise(self.mlp.forward(encode_inputs(params)), params, grey)

    def destandardise(self, yn, params, grey=None):
        """T, P, XNE [n, 72] from the network's standardised outputs yn [n, 216]."""
        params = np.atleast_2d(params)
        y = np.asarray(yn, np.float64) * self.ystd + self.ymean
        n = NRHOX
        if self.residual:
            if grey is None:
                gt, gp = self._grey_logs(params)
            else:
                gt = np.array([np.log10(g["t"]) for g in grey])
                gp = np.array([np.log10(g["p"]) for g in grey])
            y[:, :n] += gt
            y[:, n:2 * n] += gp
        return 10.0 ** y[:, :n], 10.0 ** y[:, n:2 * n], 10.0 ** y[:, 2 * n:]

    def starts(self, params, grey=None):
        """Starting structures on TAUSTD for every parameter set: T, P from
        the network, RHOX = P / g (one forward pass for all of them)."""
        params = np.atleast_2d(params)
        return structures(params, *self.predict(params, grey))

    def start(self, teff, logg, mh, vturb):
        """Starting structure on TAUSTD for one parameter set."""
        return self.starts([[teff, logg, mh, vturb]])[0]

    def save(self, path):
        np.savez(path, params=self.mlp.params(), shape=np.array(self.mlp.shape), ymean=self.ymean,
                 ystd=self.ystd, box=BOX, residual=np.array(self.residual))

    @classmethod
    def load(cls, path, ctx):
        d = np.load(path)
        mlp = MLP(ctx, shape=tuple(int(s) for s in d["shape"]))
        mlp.set_params(d["params"])
        return cls(mlp, d["ymean"], d["ystd"], bool(d["residual"]) if "residual" in d.files else False)


def structures(params, t, p, xne):
    """Starting structures on TAUSTD from predicted T, P, XNE [n, 72]: T made
    monotone (each depth at least 1 K below the next, the iteration's own
    rule) and floored at 1200 K, RHOX = P / g."""
    out = []
    for i, (teff, logg, mh, vturb) in enumerate(np.atleast_2d(params)):
        ti = t[i].copy()
        for j in range(NRHOX - 2, -1, -1):
            ti[j] = min(ti[j], ti[j + 1] - 1.0)
        out.append(dict(t=np.maximum(ti, 1200.0), p=p[i], rhox=p[i] / 10.0 ** logg, tauros=TAUSTD.copy(),
                        xne=xne[i]))
    return out


_ross_cache = {}


def grey_start(teff, logg, mh, nrhox=NRHOX):
    """The plain grey start at [M/H] (Rosseland tables cached per 0.1 dex)."""
    key = round(float(mh), 1)
    if key not in _ross_cache:
        _ross_cache[key] = surrogate.RossTable(mh=key, nwave=600)
    return surrogate.grey_model(teff, logg, nrhox=nrhox, ross=_ross_cache[key])


def run_models(batch, params, starts=None, max_iter=80, tol=0.1):
    """Iterate every parameter set ([n, 4]: Teff, log g, [M/H], vturb) on an
    AtlasBatch (shared line list and grid) from its grey start (or
    starts[i]).  Returns per-model iterations, final max |FLXERR| (inf when
    the model did not converge) and the final T, P, XNE [n, 72]."""
    n = len(params)
    if starts is None:
        starts = [grey_start(teff, logg, mh, batch.nrhox) for teff, logg, mh, _ in params]
    res = batch.run_queue(params, starts, max_iter=max_iter, tol_percent=tol)
    iters = np.array([r["iters"] for r in res], np.int32)
    err = np.array([r["maxerr"] if r["status"] == _lib.SLOT_CONVERGED else np.inf for r in res])
    T, P, NE = (np.array([r[k] for r in res]) for k in ("t", "p", "xne"))
    return iters, err, T, P, NE


def workload_batch(ctx, tables, nslots=64, numnu=30000, nlines=500000, seed=2):
    """An AtlasBatch on the 30,000-frequency, 500,000-line opacity-sampling
    workload (every model shares the line list and the grid)."""
    from . import atlas, synthetic
    ws, rc = synthetic.geometric_waveset(9.0, 160000.0, numnu)
    lines = synthetic.atlas_lines(nlines, ws[2], ws[-3], seed=seed)
    return atlas.AtlasBatch(ctx, tables, nslots=nslots, linedata=lines, waveset=ws, rcoset=rc)


def compare_starts(batch, ws, params, max_iter=80, tol=0.1):
    """Iterations to max |FLXERR| <= tol from the grey start and from the
    network's start, per parameter set (the unmodified iteration judges both).
    Returns dict of arrays: iters/err for 'grey' and 'mlp'."""
    out = {}
    for name, starts in (("grey", None), ("mlp", ws.starts(params))):
        it, er, _, _, _ = run_models(batch, params, starts, max_iter=max_iter, tol=tol)
        out[name] = dict(iters=it, err=er)
    return out


def main(argv=None):
    """generate: converged models over the parameter box; train: fit the
    network; evaluate: held-out iterations from the grey and the learned start.

    python -m atlas12_b200.warmstart generate --n 2000 --seed 11 --out models.npz
    python -m atlas12_b200.warmstart train --data models.npz[,more.npz] --out warmstart.npz
    python -m atlas12_b200.warmstart evaluate --weights warmstart.npz --n 200 --seed 12 --out heldout.npz
    """
    import argparse
    import time

    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["generate", "train", "evaluate"])
    ap.add_argument("--n", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--max-iter", type=int, default=80)
    ap.add_argument("--slots", type=int, default=64)
    ap.add_argument("--data", default=None)
    ap.add_argument("--weights", default=None)
    ap.add_argument("--out", required=True)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=1e-3)
    a = ap.parse_args(argv)
    from . import operators
    tables = operators.load()
    ctx = _lib.Context(0, _lib.PREC_MIXED)
    t0 = time.time()
    if a.cmd == "generate":
        batch = workload_batch(ctx, tables, a.slots)
        params = sample_params(a.n, a.seed)
        it, er, T, P, NE = run_models(batch, params, max_iter=a.max_iter)
        np.savez(a.out, params=params, iters=it, err=er, t=T, p=P, xne=NE)
        conv = np.isfinite(er)
        print(f"{a.n} models, {int(conv.sum())} converged (mean {it[conv].mean():.1f} iterations), "
              f"{time.time() - t0:.0f} s", flush=True)
        batch.close()
    elif a.cmd == "train":
        parts = [np.load(f) for f in a.data.split(",")]
        d = {k: np.concatenate([q[k] for q in parts]) for k in ("params", "iters", "err", "t", "p", "xne")}
        # converged models with a physical structure (the surface P of a remapped model can dip below 0)
        ok = (np.isfinite(d["err"]) & (d["err"] <= 0.1) & np.all(d["t"] > 0, axis=1) & np.all(d["p"] > 0, axis=1)
              & np.all(np.isfinite(d["xne"]), axis=1))
        idx = np.where(ok)[0]
        rng = np.random.default_rng(a.seed)
        val = rng.permutation(idx)[: max(1, idx.size // 10)]
        trn = np.setdiff1d(idx, val)
        for name, use in (("validation split", trn), ("all", idx)):
            ws, hist = WarmStart.fit(ctx, d["params"][use], d["t"][use], d["p"][use], d["xne"][use],
                                     epochs=a.epochs, lr=a.lr, lr_tail=a.lr / 4, tail_epochs=a.epochs // 2)
            tv, _, _ = ws.predict(d["params"][val])
            dex = np.abs(np.log10(tv) - np.log10(d["t"][val]))
            print(f"{name}: trained on {use.size} converged models, loss {hist[0]:.4g} -> {hist[-1]:.4g}; "
                  f"held-out {val.size}: median max|dlog T| {np.median(dex.max(1)):.4f} dex", flush=True)
        ws.save(a.out)
        print(f"{time.time() - t0:.0f} s", flush=True)
    else:
        ws = WarmStart.load(a.weights, ctx)
        batch = workload_batch(ctx, tables, a.slots)
        params = sample_params(a.n, a.seed)
        r = compare_starts(batch, ws, params, max_iter=a.max_iter)
        np.savez(a.out, params=params, **{f"{k}_{q}": r[k][q] for k in r for q in r[k]})
        for k in r:
            c = np.isfinite(r[k]["err"])
            it = r[k]["iters"]
            print(f"{k}: {int(c.sum())}/{a.n} converged, mean iterations {it[c].mean():.2f}, total iterations "
                  f"{int(it.sum())}; within 30 iterations {int(np.sum(c & (it <= 30)))}, "
                  f"iterations spent with a 30 cap {int(np.minimum(it, 30).sum())}", flush=True)
        batch.close()
    ctx.close()


if __name__ == "__main__":
    main()
