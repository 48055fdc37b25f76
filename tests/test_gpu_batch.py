"""Batched ATLAS12 models (atlasgpu_batch_*) against the single-model path.

Every slot of a batch must follow exactly the iteration a lone model follows
from the same start: the batch only changes how the work is launched (one
graph for all slots) and how the frequency sums are grouped before their
fixed-order reduction.  Tolerance: relative 1e-8 on T, P, RHOX and on each
iteration's max |FLXERR| after 5 iterations (the frequency-sum grouping
differs, the rest is the same FP64 arithmetic).
"""
import os

import numpy as np
import pytest

from atlas12_b200 import _lib, atlas, surrogate, synthetic

pytestmark = pytest.mark.gpu

PARAMS = [(5777.0, 4.44, 0.0, 1.5), (6200.0, 4.2, -0.5, 2.0), (5400.0, 4.6, 0.3, 1.0)]
NIT = 5


@pytest.fixture(scope="module")
def small_grid():
    ws, rc = synthetic.geometric_waveset(9.0, 160000.0, 2000)
    lines = synthetic.atlas_lines(5000, ws[2], ws[-3], seed=3)
    return ws, rc, lines


def _start(teff, logg, mh):
    return surrogate.grey_model(teff, logg, ross=surrogate.RossTable(mh=mh, nwave=600))


@pytest.fixture(scope="module")
def singles(gpu_ctx, tables, small_grid):
    ws, rc, lines = small_grid
    out = []
    m = atlas.AtlasModel(gpu_ctx, tables, linedata=lines, waveset=ws, rcoset=rc)
    for teff, logg, mh, vt in PARAMS:
        s = _start(teff, logg, mh)
        m.set_params(teff, logg, vt, mh)
        m.set_structure(s["t"], s["p"], s["rhox"])
        n, hist = m.iterate(max_iter=NIT, tol_percent=0.0, graph=True)
        assert n == NIT
        out.append(dict(m.structure(), hist=hist))
    m.close()
    return out


def test_batch_queue_matches_single_models(gpu_ctx, tables, small_grid, singles):
    ws, rc, lines = small_grid
    b = atlas.AtlasBatch(gpu_ctx, tables, nslots=2, linedata=lines, waveset=ws, rcoset=rc)
    starts = [_start(teff, logg, mh) for teff, logg, mh, _ in PARAMS]
    # three models through two slots: the third reuses a slot that held another model
    res = b.run_queue(PARAMS, starts, max_iter=NIT, tol_percent=0.0, poll_every=2)
    for i, (r, s) in enumerate(zip(res, singles)):
        assert r["status"] == _lib.SLOT_CAPPED and r["iters"] == NIT, (i, r["status"], r["iters"])
        for k in ("t", "p", "rhox"):
            np.testing.assert_allclose(r[k], s[k], rtol=1e-8, err_msg=f"model {i} {k}")
        np.testing.assert_allclose(r["hist"], s["hist"], rtol=1e-8, err_msg=f"model {i} history")
        np.testing.assert_allclose(r["hsurf"], s["hsurf"], rtol=1e-8, err_msg=f"model {i} HNU(1)")
    b.close()


def test_batch_slots_stop_by_themselves(gpu_ctx, tables, small_grid):
    """A converged slot (tol above its error) stops; the others keep their cap;
    idle slots never run; extra graph replays change nothing."""
    ws, rc, lines = small_grid
    b = atlas.AtlasBatch(gpu_ctx, tables, nslots=4, linedata=lines, waveset=ws, rcoset=rc)
    teff, logg, mh, vt = PARAMS[0]
    s = _start(teff, logg, mh)
    b.load(0, teff, logg, vt, mh, s, max_iter=6, tol_percent=1e9)  # converges at its first iteration
    b.load(1, teff, logg, vt, mh, s, max_iter=3, tol_percent=0.0)
    b.load(3, teff, logg, vt, mh, s, max_iter=4, tol_percent=0.0)
    st, it, er = b.run(poll_every=3)
    assert list(st) == [_lib.SLOT_CONVERGED, _lib.SLOT_CAPPED, _lib.SLOT_IDLE, _lib.SLOT_CAPPED]
    assert list(it) == [1, 3, 0, 4]
    t3 = b.structure(3)["t"].copy()
    b.step(3)
    st2, it2, _, run = b.poll()
    assert run == 0 and list(it2) == list(it)
    np.testing.assert_array_equal(b.structure(3)["t"], t3)
    b.close()


def test_batch_rejects_bad_arguments(gpu_ctx, tables, small_grid):
    ws, rc, lines = small_grid
    b = atlas.AtlasBatch(gpu_ctx, tables, nslots=2, linedata=lines[:100], waveset=ws, rcoset=rc)
    s = _start(5777.0, 4.44, 0.0)
    with pytest.raises(_lib.AtlasGPUError, match="bad argument"):
        b.load(2, 5777.0, 4.44, 1.5, 0.0, s)
    with pytest.raises(_lib.AtlasGPUError, match="bad argument"):
        b.load(0, 5777.0, 4.44, 1.5, 0.0, s, max_iter=_lib.BATCH_MAX_ITER + 1)
    bad = dict(s, t=np.where(np.arange(s["t"].size) == 7, -1.0, s["t"]))
    with pytest.raises(_lib.AtlasGPUError, match="depth 8"):
        b.load(0, 5777.0, 4.44, 1.5, 0.0, bad)
    b.close()


def test_launch_shape_and_autotuner(gpu_ctx, tables, small_grid, singles, tmp_path, monkeypatch):
    """Every launch shape gives the lone model's iteration (relative 1e-8);
    the autotuner picks one of its candidates and caches it per workload, and
    later batches of that workload start from the cached shape."""
    from atlas12_b200 import autotune
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    ws, rc, lines = small_grid
    b = atlas.AtlasBatch(gpu_ctx, tables, nslots=2, linedata=lines, waveset=ws, rcoset=rc)
    starts = [_start(teff, logg, mh) for teff, logg, mh, _ in PARAMS]
    for shape in ((8, 8), (32, 64), (1, 1)):
        b.set_shape(*shape)
        assert b.shape() == shape
        res = b.run_queue(PARAMS, starts, max_iter=NIT, tol_percent=0.0)
        for i, (r, s) in enumerate(zip(res, singles)):
            np.testing.assert_allclose(r["t"], s["t"], rtol=1e-8, err_msg=f"shape {shape} model {i}")
    lc, rw, entry = autotune.tune_batch(b, PARAMS, starts)
    assert lc in autotune.LINOP_CANDIDATES and rw in autotune.RT_CANDIDATES and b.shape() == (lc, rw)
    assert os.path.exists(autotune.cache_path())
    b.set_shape(16, 32)
    assert autotune.tune_batch(b, PARAMS, starts)[:2] == (lc, rw)  # from the cache
    with pytest.raises(_lib.AtlasGPUError, match="RT waves"):
        b.set_shape(16, 0)
    default = atlas.AtlasBatch(gpu_ctx, tables, nslots=2, linedata=lines, waveset=ws, rcoset=rc, shape=None).shape()
    b2 = atlas.AtlasBatch(gpu_ctx, tables, nslots=2, linedata=lines, waveset=ws, rcoset=rc)
    assert b2.shape() == (lc, rw)  # a new batch of this workload starts from the cached shape
    b2.close()
    b3 = atlas.AtlasBatch(gpu_ctx, tables, nslots=3, linedata=lines, waveset=ws, rcoset=rc)
    assert b3.shape() == default  # another workload: nothing cached
    b3.close()
    b.close()


def test_batch_runs_are_bit_identical(gpu_ctx, tables, small_grid):
    """Two runs of the same models give the same bits: LINOP1's sums are
    exact (order-free) and every other reduction has a fixed order, so
    convergence no longer depends on the run."""
    ws, rc, lines = small_grid
    starts = [_start(teff, logg, mh) for teff, logg, mh, _ in PARAMS]
    b = atlas.AtlasBatch(gpu_ctx, tables, nslots=3, linedata=lines, waveset=ws, rcoset=rc, shape=None)
    r1 = b.run_queue(PARAMS, starts, max_iter=NIT, tol_percent=0.0, poll_every=1)
    r2 = b.run_queue(PARAMS, starts, max_iter=NIT, tol_percent=0.0, poll_every=1)
    b.close()
    for a, c in zip(r1, r2):
        for k in ("t", "p", "rhox", "flxerr", "hist"):
            assert np.array_equal(np.asarray(a[k]).view(np.uint64), np.asarray(c[k]).view(np.uint64)), k


def test_timed_iteration_counts_without_changing_results(gpu_ctx, tables, small_grid):
    """A timed iteration also runs LINOP1's counting pass (the same walks,
    counting the atomics the exact sums issue, adding nothing): the counts are
    consistent (1-3 atomics per wing point) and the models' structure is the
    same bits as an untimed iteration's."""
    ws, rc, lines = small_grid
    starts = [_start(teff, logg, mh) for teff, logg, mh, _ in PARAMS]
    out = []
    for timed in (False, True):
        b = atlas.AtlasBatch(gpu_ctx, tables, nslots=3, linedata=lines, waveset=ws, rcoset=rc, shape=None)
        for s, (teff, logg, mh, vt) in enumerate(PARAMS):
            b.load(s, teff, logg, vt, mh, starts[s], max_iter=4, tol_percent=0.0)
        b.step(1)
        gpu_ctx.enable_timing(timed)
        b.step(1)
        if timed:
            pts = gpu_ctx.kernel_work("batch_linop_points")
            atoms = gpu_ctx.kernel_work("batch_linop_atomics")
            assert pts > 0 and pts <= atoms <= 3 * pts, (pts, atoms)
        gpu_ctx.enable_timing(False)
        b.step(2)
        out.append([b.structure(s) for s in range(3)])
        b.close()
    for a, c in zip(*out):
        for k in ("t", "p", "rhox", "flxerr"):
            assert np.array_equal(np.asarray(a[k]).view(np.uint64), np.asarray(c[k]).view(np.uint64)), k


def test_atomic_peak_probe(gpu_ctx):
    """The denominator of LINOP1's roofline: a positive rate of 64-bit atomics."""
    rate = float(_lib.lib().atlasgpu_u64_atomic_peak(gpu_ctx.handle))
    assert rate > 10.0, rate  # billions per second
