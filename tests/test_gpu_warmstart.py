"""What the trained warm start gains over the plain grey start.

The network (atlas12_b200/data/warmstart_c2.npz, trained on converged
models of this library's own ATLAS12 iteration over Teff 3500-8000 K,
log g 1-5, [M/H] -2..+0.5, vturb 0.5-3 km/s) gives the starting structure;
the unmodified iteration judges convergence (max |FLXERR| <= 0.1 %).  On 32
held-out parameter sets (a seed the training never saw), on the
30,000-frequency, 500,000-line workload and within the 30-iteration budget
of the reference's default NUMITS, the learned start must converge more
models than the grey start while spending no more iterations in total.
"""
import os

import numpy as np
import pytest

from atlas12_b200 import _lib, warmstart

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "atlas12_b200", "data",
                       "warmstart_c2.npz")


def test_learned_start_converges_more_models_in_the_budget(gpu_ctx, tables):
    if not os.path.exists(WEIGHTS):
        pytest.fail("trained warm-start weights are missing")
    params = warmstart.sample_params(32, seed=12)
    ws = warmstart.WarmStart.load(WEIGHTS, gpu_ctx)
    # one forward pass for many models, with or without the caller's grey starts, = one model at a time
    grey = [warmstart.grey_start(teff, logg, mh) for teff, logg, mh, _ in params[:4]]
    for a, b, c in zip(ws.starts(params[:4]), ws.starts(params[:4], grey), [ws.start(*p) for p in params[:4]]):
        for k in ("t", "p", "rhox"):
            np.testing.assert_allclose(a[k], c[k], rtol=1e-12)
            np.testing.assert_array_equal(a[k], b[k])
    batch = warmstart.workload_batch(gpu_ctx, tables, nslots=32)
    r = warmstart.compare_starts(batch, ws, params, max_iter=30, tol=0.1)
    batch.close()
    ws.mlp.close()
    conv = {k: int(np.sum(np.isfinite(r[k]["err"]))) for k in r}
    spent = {k: int(np.sum(r[k]["iters"])) for k in r}
    print("converged within 30 iterations", conv, "iterations spent", spent)
    assert conv["mlp"] > conv["grey"], conv
    assert spent["mlp"] <= spent["grey"], spent
