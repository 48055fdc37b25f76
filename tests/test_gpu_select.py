"""SELECTLINES on the device (atlasgpu_atlas_selectlines / _dev) against the
oracle (oracle.c orc_atlas_selectlines): bit-exact LINEDATA records in file
order, the same count and the same loop state (NU, FREQ, IGR), for every
database kind, on sorted and shuffled records, in chunks, at tile edges, in
the reference's fatal cases, and on records planted next to the rounding
boundaries the host decides (atlas12_modules.f90:19171-19781).
"""
import math

import numpy as np
import pytest

from atlas12_b200 import _lib, atlas, linelists, synthetic

pytestmark = pytest.mark.gpu

CLIGHT_NMS = 2.99792458e17
RATIOLG = math.log(1.0 + 1.0 / 2000000.0)
KINDS = range(1, 8)


@pytest.fixture(scope="module")
def sel(tables, po, gpu_ctx):
    wt = tables["wavetab"]
    xn, hckt, tc = synthetic.selectlines_tables(wt)
    iwt = atlas.iwavetab(wt)
    dev = linelists.SelectLines(gpu_ctx, 72, xn, hckt, tc, iwt, wt)
    return dict(wt=wt, iwt=iwt, xn=xn, tc=tc, xmax=po.xnfdopmax(72, xn, tc), hckt=hckt, dev=dev,
                tb={k: tables[k] for k in ("molcodes", "isox", "tio_isocorr", "h2o_isocorr")})


def oracle(po, sel, kind, recs, state, cap=None, xmax=None):
    st = dict(state)
    out, err, bad = po.selectlines(sel["tb"], kind, recs, st, sel["xmax"] if xmax is None else xmax,
                                   sel["hckt"][-1], sel["iwt"], sel["wt"], cap=cap)
    return out, err, bad, st


def start(sel, igr=5):
    return {"nu": 1, "freq": CLIGHT_NMS / sel["wt"][-1], "igr": igr}


def check(sel, po, kind, recs, state=None, dev=None):
    state = start(sel) if state is None else state
    want, err, bad, wst = oracle(po, sel, kind, recs, state)
    assert err == 0, (err, bad)
    st = dict(state)
    got = (dev or sel["dev"]).select(kind, recs, st)
    np.testing.assert_array_equal(got, want)
    assert st == wst, (st, wst)
    return got


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("n,shuffle", [(2_000_000, 0.0), (300_000, 0.02)])
def test_selectlines_matches_oracle(sel, po, kind, n, shuffle):
    recs = synthetic.selectlines_records(kind, n, sel["wt"], seed=100 + kind, shuffle_frac=shuffle)
    got = check(sel, po, kind, recs)
    assert got.shape[0] > 100


@pytest.mark.parametrize("kind", [1, 5, 6])
@pytest.mark.parametrize("n", [1, 2, 2047, 2048, 2049, 4096, 6145])
def test_tile_edges(sel, po, kind, n):
    recs = synthetic.selectlines_records(kind, n, sel["wt"], seed=7 + n)
    check(sel, po, kind, recs)


def test_empty_input_leaves_state(sel):
    st = {"nu": 17, "freq": 1.25e15, "igr": -4}
    out = sel["dev"].select(1, np.zeros((0, 4), np.int32), st)
    assert out.shape == (0, 4) and st == {"nu": 17, "freq": 1.25e15, "igr": -4}


@pytest.mark.parametrize("kind", KINDS)
def test_chunks_and_device_entry(sel, po, kind):
    """Chunks carry the loop state; the device entry point gives the same records."""
    import torch
    recs = synthetic.selectlines_records(kind, 50_000, sel["wt"], seed=300 + kind, shuffle_frac=0.01)
    st0 = start(sel, igr=-11)
    want, err, _, wst = oracle(po, sel, kind, recs, st0)
    st = dict(st0)
    parts = [sel["dev"].select(kind, recs[a:b], st) for a, b in ((0, 1), (1, 20_001), (20_001, 20_001),
                                                                  (20_001, 50_000))]
    np.testing.assert_array_equal(np.concatenate(parts), want)
    assert st == wst
    raw = np.ascontiguousarray(recs).view(np.uint8).reshape(len(recs), -1)
    d_in = torch.from_numpy(raw.copy()).cuda()
    d_out = torch.zeros((len(recs), 4), dtype=torch.int32, device="cuda")
    st = dict(st0)
    m = sel["dev"].select_dev(kind, d_in, len(recs), st, d_out, len(recs))
    np.testing.assert_array_equal(d_out[:m].cpu().numpy(), want)
    assert st == wst


def test_reference_fatal_cases(sel, po):
    dev = sel["dev"]
    recs = synthetic.selectlines_records(2, 40_000, sel["wt"], seed=5, bad_frac=0.001)
    _, err, bad, _ = oracle(po, sel, 2, recs, start(sel))
    assert err == -1
    with pytest.raises(_lib.AtlasGPUError, match=rf"record {bad}: NELION"):
        dev.select(2, recs, start(sel))
    check(sel, po, 1, recs)  # LOWPRED skips the same records
    recs = synthetic.selectlines_records(4, 9000, sel["wt"], seed=2)
    recs[7001, 1] = (recs[7001, 1] & ~0xFFFF) | 8420
    recs[8500, 1] = (recs[8500, 1] & ~0xFFFF) | 8421
    with pytest.raises(_lib.AtlasGPUError, match=r"record 7001: diatomic MOLCODE"):
        dev.select(4, recs, start(sel))
    recs = synthetic.selectlines_records(3, 9000, sel["wt"], seed=3)
    recs[4444:, 0] = 2 ** 30 + 5
    with pytest.raises(_lib.AtlasGPUError, match=r"record 4444: IWL at or past"):
        dev.select(3, recs, start(sel))
    recs = synthetic.selectlines_records(7, 9000, sel["wt"], seed=4)
    n = oracle(po, sel, 7, recs, start(sel))[0].shape[0]
    with pytest.raises(_lib.AtlasGPUError, match="LINEDATA overflow"):
        dev.select(7, recs, start(sel), cap=n - 1)
    assert dev.select(7, recs, start(sel), cap=n).shape[0] == n


def _tio_border_records(rng, n_want=40):
    """MOL2 records whose IWL argument LOG(W)/RATIOLG + 0.5 lies within 5e-7 of an
    integer, or whose IELO / IGR argument does."""
    k = np.arange(int(np.log(300.0) / RATIOLG), int(np.log(5000.0) / RATIOLG), dtype=np.int64)
    w = np.exp((k - 0.5) * RATIOLG).astype(np.float32)
    x = np.log(w.astype(np.float64)) / RATIOLG + 0.5
    near = w[np.abs(x - np.rint(x)) < 5e-7][:n_want]
    m = np.arange(16384 - 3000, 16384 + 4600)
    e = (10.0 ** ((m - 16384.5) / 1000.0)).astype(np.float32)
    xe = np.log10(e.astype(np.float64)) * 1000.0 + 16384.5
    e_near = e[np.abs(xe - np.rint(xe)) < 5e-7]
    mg = np.arange(22340, 24770)  # IGR = INT(LOG10(2.223E13/W**2)*1000 + 16384.5) for W in 300-5000 nm
    wg = np.sqrt(2.223e13 / 10.0 ** ((mg - 16384.5) / 1000.0)).astype(np.float32)
    xg = np.log10(2.223e13 / wg.astype(np.float64) ** 2) * 1000.0 + 16384.5
    w_gnear = wg[np.abs(xg - np.rint(xg)) < 5e-7]
    assert near.size >= 5 and e_near.size >= 20 and w_gnear.size >= 5, (near.size, e_near.size, w_gnear.size)
    wl = np.concatenate([near, rng.choice(w, 300).astype(np.float32), w_gnear])
    r = np.zeros(wl.size, _lib.MOL2_REC)
    r["wl"] = wl
    r["gflog"] = np.float32(-1.0)
    r["e1"] = rng.choice(e_near, wl.size)
    r["e2"] = np.float32(40000.0)
    r["code"] = 822
    r["iso"] = rng.integers(46, 51, wl.size)
    r["gr"] = np.where(np.isin(wl, w_gnear), 0, rng.integers(700, 900, wl.size))
    return r


def test_tio_rounding_boundaries(sel, po):
    """TiO records whose IWL, IELO or IGR argument sits next to an integer: the
    host decides them with the C library, bit-exact with the oracle.  (H2O's
    IELO argument, LOG10 of an INTEGER(2), comes no closer than 1e-6 to an
    integer for any value, so H2O has no such record.)"""
    rng = np.random.default_rng(77)
    base = synthetic.selectlines_records(5, 200_000, sel["wt"], seed=8)
    r = np.concatenate([base, _tio_border_records(rng)])
    r = r[np.argsort(r["wl"], kind="stable")]
    check(sel, po, 5, r)
    x = np.log10(np.arange(1, 32768, dtype=np.float64)) * 1000.0 + 16384.5
    assert not np.any(np.abs(x - np.rint(x)) < 1e-6)


def test_boltzmann_test_at_one(sel, po, gpu_ctx):
    """Lines tuned so that CENRATIO * exp(-E*HCKT(NRHOX)) is 1 to a few ulps: the
    host's C-library exp decides keep or drop, and dropped records close up."""
    wt, iwt, hl = sel["wt"], sel["iwt"], sel["hckt"][-1]
    rng = np.random.default_rng(5)
    xn, tc = sel["xn"].copy(), sel["tc"]
    species = np.arange(100, 140)
    bins = np.sort(rng.choice(np.arange(20, 340), species.size, replace=False))
    recs = synthetic.selectlines_records(3, 20_000, wt, seed=6)
    rows = []
    for e, nu in zip(species, bins):
        iwl = (int(iwt[nu - 2]) + int(iwt[nu - 1])) // 2  # inside bin nu
        igf = int(rng.integers(14000, 16000))
        ielo = int(rng.integers(18000, 20000))
        freq = CLIGHT_NMS / wt[nu - 2]
        boltz = math.exp(-math.pow(10.0, (ielo - 16384) * 0.001) * hl)
        target = freq / (0.026538 / 1.7724538509055159 * math.pow(10.0, (igf - 16384) * 0.001) * boltz)
        xn[e, :] = 0.0
        j = int(rng.integers(0, 72))
        xn[e, j] = target * tc[nu - 1, j] * (1.0 + float(rng.integers(-3, 4)) * 2.0 ** -52)
        rows.append(synthetic.pack_linedata(np.array([iwl]), np.array([10 * (e + 1)], np.int16),
                                            np.array([ielo], np.int16), np.array([igf], np.int16),
                                            np.array([16000], np.int16), np.array([1], np.int16),
                                            np.array([9384], np.int16))[0])
    recs = np.concatenate([recs, np.array(rows)])
    recs = recs[np.argsort(recs[:, 0], kind="stable")]
    xmax = po.xnfdopmax(72, xn, tc)
    want, err, _, wst = oracle(po, sel, 3, recs, start(sel), xmax=xmax)
    assert err == 0
    kept = sum(1 for r in rows if (want == r).all(axis=1).any())
    assert 0 < kept < len(rows), kept  # both outcomes occur
    try:
        dev = linelists.SelectLines(gpu_ctx, 72, xn, sel["hckt"], tc, iwt, wt)
        st = start(sel)
        got = dev.select(3, recs, st)
        np.testing.assert_array_equal(got, want)
        assert st == wst
    finally:
        sel["dev"] = linelists.SelectLines(gpu_ctx, 72, sel["xn"], sel["hckt"], sel["tc"], iwt, wt)


def test_driver_order_matches_oracle(sel, po):
    """select_all: NU restarts per database except LOWOBS after LOWPRED; FREQ and
    IGR carry; TiO and H2O are skipped above 8000 K."""
    dbs = {k: synthetic.selectlines_records(k, 30_000, sel["wt"], seed=500 + k) for k in KINDS}
    for teff in (5000.0, 9000.0):
        got, counts, st = sel["dev"].select_all(dbs, teff)
        state = linelists.initial_state(sel["wt"])
        parts = []
        for kind, _ in linelists.DATABASES:
            if kind in (5, 6) and teff > 8000.0:
                continue
            if kind != 2:
                state["nu"] = 1
            out, err, _, state = oracle(po, sel, kind, dbs[kind], state)
            parts.append(out)
        np.testing.assert_array_equal(got, np.concatenate(parts))
        assert st == state
        assert (counts[5] == 0) == (teff > 8000.0)
