"""The oracle's SELECTLINES (oracle.c orc_atlas_selectlines) against a second,
independent restatement in plain Python loops, on small seeded databases of
every kind, and the loop's state rules (atlas12_modules.f90:19171-19781).

The reference has no tests or golden vectors for this path and cannot be
built here; the pins are its own constant tables (MOLCODES, ISOX,
TIO_ISOCORR, H2O_ISOCORR, WAVETAB extracted from the source by
tests/golden/make_golden.py) and agreement of two restatements written from
the source separately.
"""
import math
import struct

import numpy as np
import pytest

from atlas12_b200 import atlas, synthetic

CLIGHT_NMS = 2.99792458e17
CEN_PREFAC = 0.026538 / 1.7724538509055159
RATIOLG = math.log(1.0 + 1.0 / 2000000.0)
KINDS = range(1, 8)


def fint(x):
    """INT() as x86-64 converts a REAL(8): truncation, -2**31 for NaN / out of range."""
    if not (-2147483649.0 < x < 2147483648.0):
        return -2147483648
    return int(x)


def i16(v):
    v &= 0xFFFF
    return v - 0x10000 if v >= 0x8000 else v


def nint(x):
    """NINT: nearest, halves away from zero."""
    a = abs(x)
    r = math.floor(a)
    r += 1 if a - r >= 0.5 else 0
    return int(math.copysign(r, x))


def tablog(i):
    return math.pow(10.0, (i - 16384) * 0.001)


def py_select(tb, kind, recs, st, xmax, hckt_last, iwt, wavetab):
    """Plain-loop SELECTLINES database loop (returns records, error, record)."""
    nwave = len(wavetab)
    nspec = xmax.shape[1]
    nu, freq, igr = st["nu"], st["freq"], st["igr"]
    out = []
    molcodes = [int(x) for x in tb["molcodes"]]

    def advance(iwl, h2o=False):
        nonlocal nu, freq, igr
        while iwl >= iwt[nu - 1]:
            if nu == nwave + 1:
                raise IndexError
            freq = CLIGHT_NMS / wavetab[nu - 1]
            if h2o:
                gammar = 2.474e-22 * (freq * freq) * float(np.float32(0.001))
                igr = i16(fint(math.log10(gammar) * 1000.0 + 16384.5))
            nu += 1

    for i in range(len(recs)):
        try:
            if kind == 5:
                r = recs[i]
                if int(r["code"]) != 822:
                    continue
                iso = int(r["iso"]) - 45
                if iso < 1 or iso > 5:
                    continue
                w = float(r["wl"])
                if w <= 0.0:
                    continue
                iwl = fint(math.log(w) / RATIOLG + 0.5)
                advance(iwl)
                kg = nint(float(r["gflog"]) * 1000.0) + 16384
                igf = i16(max(kg + int(tb["tio_isocorr"][iso - 1]), 1))
                xm = xmax[nu - 1, 894]
                if xm == 0.0:
                    continue
                cen = CEN_PREFAC * tablog(igf) * xm / freq
                if cen < 1.0:
                    continue
                elo = min(abs(float(r["e1"])), abs(float(r["e2"])))
                if cen * math.exp(-elo * hckt_last) < 1.0:
                    continue
                g = 2.223e13 / (w * w) if int(r["gr"]) == 0 else math.pow(10.0, float(int(r["gr"])) * 0.01)
                igr = i16(fint(math.log10(g) * 1000.0 + 16384.5))
                f = [8949 + iso, i16(fint(math.log10(max(elo, 1e-10)) * 1000.0 + 16384.5)), igf, igr, 1, 9384]
            elif kind == 6:
                r = recs[i]
                iwl = int(r["iwl"])
                advance(iwl, h2o=True)
                ie, ig = int(r["ielo"]), int(r["igflog"])
                iso = 1 if (ie > 0 and ig > 0) else 2 if ie > 0 else 3 if ig > 0 else 4
                elo = float(abs(ie))
                igf = i16(max(abs(ig) + int(tb["h2o_isocorr"][iso - 1]), 1))
                xm = xmax[nu - 1, 939]
                if xm == 0.0:
                    continue
                cen = CEN_PREFAC * tablog(igf) * xm / freq
                if cen < 1.0 or cen * math.exp(-elo * hckt_last) < 1.0:
                    continue
                f = [-(9399 + iso), i16(fint(math.log10(elo) * 1000.0 + 16384.5)), igf, igr, 1, 9384]
            else:
                w = [int(x) for x in recs[i]]
                iwl = w[0]
                f = [i16(w[1]), i16(w[1] >> 16), i16(w[2]), i16(w[2] >> 16), i16(w[3]), i16(w[3] >> 16)]
                igr = f[3]
                advance(iwl)
                if kind == 4:
                    if f[0] not in molcodes:
                        return None, -2, i
                    f[2] = i16(max(f[2] + int(tb["isox"][molcodes.index(f[0])]), 1))
                if kind == 7:
                    f[2] = i16(max(f[2] - 1272, 1))
                    f[4], f[5] = 1, 9384
                nelion = 895 if kind == 7 else abs(int(f[0] / 10))
                if nelion < 1 or nelion > nspec:
                    if kind == 1:
                        continue
                    return None, -1, i
                xm = xmax[nu - 1, nelion - 1]
                if (xm <= 1e-37) if kind in (1, 2) else (xm == 0.0):
                    continue
                cen = CEN_PREFAC * tablog(f[2]) * xm / freq
                if cen < 1.0 or cen * math.exp(-tablog(f[1]) * hckt_last) < 1.0:
                    continue
        except IndexError:
            return None, -3, i
        out.append([iwl] + [struct.unpack("<i", struct.pack("<hh", f[2 * k], f[2 * k + 1]))[0] for k in range(3)])
    st.update(nu=nu, freq=freq, igr=igr)
    return np.array(out, np.int32).reshape(-1, 4), 0, -1


@pytest.fixture(scope="module")
def sel(tables, po):
    wt = tables["wavetab"]
    xn, hckt, tc = synthetic.selectlines_tables(wt)
    return dict(wt=wt, iwt=atlas.iwavetab(wt), xmax=po.xnfdopmax(72, xn, tc), hckt=hckt,
                tb={k: tables[k] for k in ("molcodes", "isox", "tio_isocorr", "h2o_isocorr")})


def test_xnfdopmax_is_the_depth_maximum(po):
    rng = np.random.default_rng(3)
    xn = rng.uniform(0.0, 2.0, (5, 9))
    tc = rng.uniform(0.5, 1.5, (4, 9))
    got = po.xnfdopmax(7, xn, tc)
    want = np.max(xn[None, :, :7] / tc[:, None, :7], axis=2)
    np.testing.assert_array_equal(got, np.maximum(want, 0.0))


@pytest.mark.parametrize("kind", KINDS)
@pytest.mark.parametrize("shuffle", [0.0, 0.05])
def test_oracle_matches_plain_loop_restatement(sel, po, kind, shuffle):
    recs = synthetic.selectlines_records(kind, 3000, sel["wt"], seed=20 + kind, shuffle_frac=shuffle)
    if kind == 5:
        # log gf with an exact half in millidex: NINT rounds it away from zero
        recs["gflog"][::7] = np.float32(-3.9375)
        recs["gflog"][3::7] = np.float32(0.0625)
    st0 = {"nu": 1, "freq": CLIGHT_NMS / sel["wt"][-1], "igr": 7}
    s1, s2 = dict(st0), dict(st0)
    got, e1, b1 = po.selectlines(sel["tb"], kind, recs, s1, sel["xmax"], sel["hckt"][-1], sel["iwt"], sel["wt"])
    want, e2, b2 = py_select(sel["tb"], kind, recs, s2, sel["xmax"], sel["hckt"][-1], sel["iwt"], sel["wt"])
    assert (e1, b1) == (e2, b2)
    assert got.shape[0] > 0
    np.testing.assert_array_equal(got, want)
    assert s1 == s2


@pytest.mark.parametrize("kind", [2, 3])
def test_out_of_range_species_stop_the_loop(sel, po, kind):
    """LOWOBS and HILINES index XNFDOPMAX with any NELION: the oracle stops at the
    first such record; LOWPRED skips them."""
    recs = synthetic.selectlines_records(kind, 2000, sel["wt"], seed=5, bad_frac=0.01)
    bad_rows = [i for i in range(len(recs)) if not 1 <= abs(int(int(np.int16(recs[i, 1] & 0xFFFF)) / 10)) <= 1006]
    st = {"nu": 1, "freq": 1.0, "igr": 0}
    out, err, bad = po.selectlines(sel["tb"], kind, recs, st, sel["xmax"], sel["hckt"][-1], sel["iwt"], sel["wt"])
    assert err == -1 and bad == bad_rows[0]
    st = {"nu": 1, "freq": 1.0, "igr": 0}
    out, err, bad = po.selectlines(sel["tb"], 1, recs, st, sel["xmax"], sel["hckt"][-1], sel["iwt"], sel["wt"])
    assert err == 0


def test_chunks_continue_the_loop(sel, po):
    """The state (NU, FREQ, IGR) carries a loop across calls: chunks = one call."""
    for kind in KINDS:
        recs = synthetic.selectlines_records(kind, 5000, sel["wt"], seed=40 + kind, shuffle_frac=0.01)
        st = {"nu": 1, "freq": 3.0e15, "igr": -3}
        whole, _, _ = po.selectlines(sel["tb"], kind, recs, st, sel["xmax"], sel["hckt"][-1], sel["iwt"], sel["wt"])
        st2 = {"nu": 1, "freq": 3.0e15, "igr": -3}
        parts = [po.selectlines(sel["tb"], kind, recs[a:b], st2, sel["xmax"], sel["hckt"][-1], sel["iwt"],
                                sel["wt"])[0] for a, b in ((0, 1), (1, 1777), (1777, 1777), (1777, 5000))]
        np.testing.assert_array_equal(np.concatenate(parts), whole)
        assert st == st2


def test_sentinel_and_overflow(sel, po):
    recs = synthetic.selectlines_records(1, 100, sel["wt"], seed=9)
    recs[60, 0] = 2 ** 30
    st = {"nu": 1, "freq": 1.0, "igr": 0}
    assert po.selectlines(sel["tb"], 1, recs, st, sel["xmax"], sel["hckt"][-1], sel["iwt"], sel["wt"])[1:] == (-3, 60)
    recs = synthetic.selectlines_records(7, 1000, sel["wt"], seed=9)
    st = {"nu": 1, "freq": 1.0, "igr": 0}
    n = po.selectlines(sel["tb"], 7, recs, st, sel["xmax"], sel["hckt"][-1], sel["iwt"], sel["wt"])[0].shape[0]
    st = {"nu": 1, "freq": 1.0, "igr": 0}
    assert po.selectlines(sel["tb"], 7, recs, st, sel["xmax"], sel["hckt"][-1], sel["iwt"], sel["wt"],
                          cap=n - 1)[1] == -4


def test_unknown_molcode_stops(sel, po):
    recs = synthetic.selectlines_records(4, 300, sel["wt"], seed=2)
    recs[123, 1] = (recs[123, 1] & ~0xFFFF) | 8420  # not a MOLCODE
    st = {"nu": 1, "freq": 1.0, "igr": 0}
    assert po.selectlines(sel["tb"], 4, recs, st, sel["xmax"], sel["hckt"][-1], sel["iwt"], sel["wt"])[1:] == (-2, 123)


def test_host_record_conversion():
    """LINEREC kinds go to the library as int32 [n, 4]; MOL2 / H2O keep their layout."""
    from atlas12_b200 import _lib, linelists
    r = linelists.SelectLines._records(1, np.arange(40, dtype=np.int64).reshape(10, 4))
    assert r.dtype == np.int32 and r.shape == (10, 4) and r.flags["C_CONTIGUOUS"]
    t = np.zeros(3, _lib.MOL2_REC)
    assert linelists.SelectLines._records(5, t).nbytes == 96
    with pytest.raises(ValueError):
        linelists.SelectLines._records(6, t)
    with pytest.raises(ValueError):
        linelists.SelectLines._records(2, np.zeros((5, 3), np.int32))


def test_binary_readers_roundtrip(tmp_path, tables):
    """The MOL2 (header + 32-byte records), H2O (8-byte) and LINEREC readers
    return the bytes written, memory-mapped; a file without the MOL2 magic is
    refused; the header count caps the records read (no GPU)."""
    from atlas12_b200 import linelists
    wt = tables["wavetab"]
    mol = synthetic.selectlines_records(5, 1000, wt, seed=1)
    p = tmp_path / "toto.bin"
    linelists.write_mol2(str(p), mol)
    assert linelists.read_mol2(str(p)).tobytes() == mol.tobytes()
    with open(p, "ab") as f:  # trailing records beyond the header's count are not read
        f.write(mol[:3].tobytes())
    assert len(linelists.read_mol2(str(p))) == 1000
    h = synthetic.selectlines_records(6, 500, wt, seed=2)
    q = tmp_path / "h2o.bin"
    h.tofile(str(q))
    assert linelists.read_h2o(str(q)).tobytes() == h.tobytes()
    with pytest.raises(ValueError, match="MOL2"):
        linelists.read_mol2(str(q))
    ld = synthetic.selectlines_records(1, 700, wt, seed=3)
    r = tmp_path / "gfpred.bin"
    ld.tofile(str(r))
    np.testing.assert_array_equal(linelists.read_linerec(str(r)), ld)


def test_driver_order_rules():
    """SELECTLINES's database order and entry state (no GPU)."""
    from atlas12_b200 import _lib, linelists
    kinds = [k for k, _ in linelists.DATABASES]
    assert kinds == [_lib.SEL_LOWPRED, _lib.SEL_LOWOBS, _lib.SEL_HI, _lib.SEL_DIATOMIC, _lib.SEL_TIO, _lib.SEL_H2O,
                     _lib.SEL_H3PLUS]
    st = linelists.initial_state(np.array([9.09, 160000.0]))
    assert st["nu"] == 1 and st["freq"] == CLIGHT_NMS / 160000.0 and st["igr"] == 0


def test_select_all_threads_the_state(monkeypatch):
    """select_all on a stub database loop: NU restarts at 1 for every database
    but LOWOBS, FREQ and IGR carry from one to the next, TiO and H2O are
    skipped above 8000 K (no GPU)."""
    from atlas12_b200 import _lib, linelists
    calls = []

    def fake_select(self, kind, recs, state, cap=None):
        calls.append((kind, dict(state)))
        state.update(nu=state["nu"] + 10 * kind, freq=state["freq"] * 2.0, igr=kind)
        return np.full((len(recs), 4), kind, np.int32)

    monkeypatch.setattr(linelists.SelectLines, "select", fake_select)
    S = object.__new__(linelists.SelectLines)
    S.wavetab = np.array([10.0, 20.0])
    dbs = {k: np.zeros((k, 4), np.int32) for k in range(1, 8)}
    out, counts, st = S.select_all(dbs, teff=5000.0)
    assert [c[0] for c in calls] == [1, 2, 3, 4, 5, 6, 7]
    assert calls[0][1]["nu"] == 1 and calls[1][1]["nu"] == 11  # LOWOBS continues from LOWPRED
    assert all(c[1]["nu"] == 1 for c in calls[2:])
    assert calls[0][1]["freq"] == CLIGHT_NMS / 20.0 and calls[3][1]["freq"] == 8.0 * CLIGHT_NMS / 20.0
    assert [c[1]["igr"] for c in calls] == [0, 1, 2, 3, 4, 5, 6]
    assert counts == {k: k for k in range(1, 8)} and out.shape == (28, 4)
    calls.clear()
    out, counts, st = S.select_all(dbs, teff=9000.0)
    assert [c[0] for c in calls] == [1, 2, 3, 4, 7] and counts[_lib.SEL_TIO] == 0 and counts[_lib.SEL_H2O] == 0


def test_autotune_cache_lookup(tmp_path, monkeypatch):
    """autotune.cached_shape reads the per-GPU, per-workload entry tune_batch
    writes, and nothing for another workload (no GPU)."""
    import json
    from atlas12_b200 import autotune
    monkeypatch.setenv("XDG_CACHE_HOME", str(tmp_path))
    monkeypatch.setattr(autotune, "_device_name", lambda device: "B200")

    class Fake:
        class ctx:
            device = 0
        waveset = np.zeros(30000)
        nlines, nrhox, nslots = 500000, 72, 32

    assert autotune.cached_shape(Fake) is None
    path = autotune.cache_path()
    import os
    os.makedirs(os.path.dirname(path))
    with open(path, "w") as f:
        json.dump({autotune._key(Fake, "B200"): {"shape": [32, 64]}}, f)
    assert autotune.cached_shape(Fake) == (32, 64)
    Fake.nslots = 16
    assert autotune.cached_shape(Fake) is None
