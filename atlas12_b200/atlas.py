"""Host-side mirror of ATLAS12's hot path (atlas12c.f90 + RUN_RT_PASS), on the C ABI.

Reference names and meanings:

* ``waveset_rcoset``  -- WAVESET and the RCOSET trapezoid weights (atlas12c.f90:451-491)
* ``tabvoigt``        -- H0/H1/H2 tables at 200 steps per Doppler width (TABVOIGT)
* ``Atlas.linop1``    -- XLINES(J,NU) from LINEDATA (LINOP1)
* ``Atlas.rt_pass``   -- the frequency loop with JOSH and the mode-2 sums (RUN_RT_PASS)
* ``Atlas.finish``    -- ROSS(3), RADIAP(3), TCORR(3) on one model
* ``AtlasModel``      -- one atmosphere iterated on the device (the ITERAT loop,
                         atlas12c.f90:496-606) with the synthetic surrogate physics

Arrays follow the reference layouts seen from C: XLINES(kw, numnu) is
[numnu, kw], XNFDOP(kw, mion) is [mion, kw].
"""
import ctypes

import numpy as np

from . import _lib, surrogate, synthetic
from ._lib import Accum, Context, FinishState, ModelDesc, ptr

LINE_CUTOFF = 1.0e-3
RATIOLG_LINES = np.log(1.0 + 1.0 / 2000000.0)
ACC_NAMES = ("rjmins", "rdabh", "rdiagj", "flxrad", "raden", "h_total", "accrad", "abross")


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def tabvoigt(operators, vsteps=200.0, n=2001):
    """TABVOIGT (atlas12_modules.f90:19796-19851): H0, H1, H2 at vsteps points per
    Doppler width, H1 mapped (MAP1) from the reference's TABVI/TABH1 table
    (operators["tabvi"], operators["tabh1"]), computed by the library."""
    tv = np.ascontiguousarray(operators["tabvi"], np.float64)
    th = np.ascontiguousarray(operators["tabh1"], np.float64)
    h0, h1, h2 = np.zeros(n), np.zeros(n), np.zeros(n)
    rc = _lib.lib().atlasgpu_atlas_tabvoigt(float(vsteps), int(n), ptr(tv), ptr(th), tv.size, ptr(h0), ptr(h1),
                                           ptr(h2))
    if rc != _lib.OK:
        raise _lib.AtlasGPUError(rc, "atlasgpu_atlas_tabvoigt: bad table")
    return h0, h1, h2


def cutoff_grid(n=361, lo=9.0, hi=400000.0):
    """KAPCONT's continuum-cutoff wavelengths (nm): a log-spaced stand-in for WAVETAB."""
    return np.geomspace(lo, hi, n)


def iwavetab(cutwave):
    """IWAVETAB = INT(LOG(WAVE)/RATIOLG + 0.5) plus the 2**30 sentinel (KAPCONT :19096)."""
    iw = np.empty(cutwave.size + 1, dtype=np.int32)
    iw[:-1] = (np.log(cutwave) / RATIOLG_LINES + 0.5).astype(np.int64)
    iw[-1] = 2 ** 30
    return iw


class Atlas:
    """The ATLAS12 kernels on one context (parity-level entry points)."""

    def __init__(self, ctx: Context, operators, h0=None, h1=None, h2=None):
        self.ctx = ctx
        ctx.set_operators(operators["xtau8"], operators["coefj"], operators["coefh"], operators["ch_j"],
                          operators["ck_j"])
        if h0 is None:
            h0, h1, h2 = tabvoigt(operators)
        self.tables = [np.ascontiguousarray(x, np.float64) for x in (h0, h1, h2)]
        ctx.call("atlasgpu_atlas_set_voigt_tables", *[ptr(x) for x in self.tables], 2001)

    def linop1(self, linedata, nrhox, xnfdop, dopple, xne, txnxn, hckt, tabcont, iwt, waveset):
        ld = np.ascontiguousarray(linedata, np.int32)
        xd = np.ascontiguousarray(xnfdop, np.float64)
        dp = np.ascontiguousarray(dopple, np.float64)
        nspec, kw = xd.shape
        vec = [np.ascontiguousarray(v, np.float64) for v in (xne, txnxn, hckt)]
        tc = np.ascontiguousarray(tabcont, np.float64)
        iw = np.ascontiguousarray(iwt, np.int32)
        ws = np.ascontiguousarray(waveset, np.float64)
        out = np.zeros((ws.size, kw))
        used = ctypes.c_int64(0)
        self.ctx.call("atlasgpu_atlas_linop", ptr(ld), ld.shape[0], int(nrhox), kw, ptr(xd), ptr(dp), nspec,
                      *[ptr(v) for v in vec], ptr(tc), ptr(iw), iw.size - 1, ptr(ws), ws.size, ptr(out),
                      ctypes.byref(used))
        return out, used.value

    def set_hydrogen_tables(self, tables):
        """The hydrogen line profile's tables (arrays h_* as the fixture
        extracted from the reference holds them) for XLINOP's hydrogen lines."""
        self._htab = _lib.HydrogenTables.from_tables(tables)
        self.ctx.call("atlasgpu_atlas_set_hydrogen_tables", ctypes.byref(self._htab))

    def set_kapp_tables(self, tables):
        """KAPP's hydrogen continuum tables (arrays k_* as the fixture
        extracted from the reference's data files and source holds them)."""
        self._ktab = _lib.KappTables.from_tables(tables)
        self.ctx.call("atlasgpu_atlas_set_kapp_tables", ctypes.byref(self._ktab))

    def kapp_hydrogen(self, waveset, t, xne, rho, xnfp1, xnfp2, bhyd=None, bmin=None, kw=None, parts=False):
        """KAPP with its hydrogen, H-, H2+, Rayleigh and electron-scattering
        sources at every (frequency, depth): (acont, sigmac, scont) [numnu, kw],
        and with parts=True also [numnu, 7, kw] (AHYD, SHYD, AH2P, AHMIN,
        SHMIN, SIGH, SIGEL).  bhyd [6, kw] and bmin [kw]: None for LTE."""
        ws = np.ascontiguousarray(waveset, np.float64)
        vec = [np.ascontiguousarray(v, np.float64) for v in (t, xne, rho, xnfp1, xnfp2)]
        nrhox = vec[0].size
        kw = nrhox if kw is None else int(kw)
        bh = None if bhyd is None else np.ascontiguousarray(bhyd, np.float64)
        if bh is not None and bh.shape != (6, kw):
            raise ValueError("bhyd must be [6, kw]")
        bm = None if bmin is None else np.ascontiguousarray(bmin, np.float64)
        out = [np.zeros((ws.size, kw)) for _ in range(3)]
        pt = np.zeros((ws.size, 7, kw)) if parts else None
        self.ctx.call("atlasgpu_atlas_kapp_hydrogen", ws.size, ptr(ws), nrhox, kw, *[ptr(v) for v in vec], ptr(bh),
                      ptr(bm), *[ptr(o) for o in out], ptr(pt))
        return (*out, pt) if parts else tuple(out)

    def set_kapp_h2_tables(self, tables, use_pair=(1, 1, 1, 1)):
        """Keep KAPP's H2 tables (H2MINOP, PARTFNH2, H2COLLOP's CIA grid) on the
        context; use_pair = USE_CIA_PAIR for H2-H2, H2-He, H2-H, H-He."""
        t = _lib.KappH2Tables.from_tables(tables, use_pair)
        self.ctx.call("atlasgpu_atlas_set_kapp_h2_tables", ctypes.byref(t))

    def set_stehle_tables(self, stehle):
        """The four Stehle series STARK_MMM reads (4 dicts as read_stehle or
        synthetic.stehle_tables give, None entries not loaded); None: STARK's
        analytic profile throughout."""
        st, keep = (None, []) if stehle is None else _lib.stehle_array(stehle)
        self.ctx.call("atlasgpu_atlas_set_stehle_tables", st)
        del keep  # the library copied the tables

    def hlinop(self, waveset, t, xne, rho, xnfp1, bhyd=None, kw=None):
        """HLINOP's hydrogen line pseudo-continuum at every (frequency, depth):
        (AHLINE, SHLINE) [numnu, kw].  bhyd [6, kw]: None for LTE."""
        ws = np.ascontiguousarray(waveset, np.float64)
        vec = [np.ascontiguousarray(v, np.float64) for v in (t, xne, rho, xnfp1)]
        nrhox = vec[0].size
        kw = nrhox if kw is None else int(kw)
        bh = None if bhyd is None else np.ascontiguousarray(bhyd, np.float64)
        if bh is not None and bh.shape != (6, kw):
            raise ValueError("bhyd must be [6, kw]")
        out = [np.zeros((ws.size, kw)) for _ in range(2)]
        self.ctx.call("atlasgpu_atlas_hlinop", ws.size, ptr(ws), nrhox, kw, *[ptr(v) for v in vec], ptr(bh),
                      *[ptr(o) for o in out])
        return tuple(out)

    def kapp(self, waveset, t, xne, rho, xnfp1, xnfp2, xnfp3, xnfp4, xnfp5, xnf4, bhyd=None, bmin=None, kw=None,
             parts=False, xnf3=None):
        """KAPP with the hydrogen sources of kapp_hydrogen and the helium ones
        (HE1OP, HE2OP, HEMIOP, HERAOP): (acont, sigmac, scont) [numnu, kw], and
        with parts=True also [numnu, 11, kw] (AHYD, SHYD, AH2P, AHMIN, SHMIN,
        SIGH, SIGEL, AHE1, AHE2, AHEMIN, SIGHE).  xnfp1..5 = XNFP(J,1..5),
        xnf4 = XNF(J,4) (He II number density), each [nrhox].  With xnf3 =
        XNF(J,3) (He I number density; set_kapp_h2_tables first) also the H2
        sources (H2MINOP, H2COLLOP, H2RAOP), and parts [numnu, 14, kw] with
        AH2MIN, AH2COLL, SIGH2 appended."""
        ws = np.ascontiguousarray(waveset, np.float64)
        vec = [np.ascontiguousarray(v, np.float64) for v in (t, xne, rho, xnfp1, xnfp2, xnfp3, xnfp4, xnfp5, xnf4)]
        x3 = None if xnf3 is None else np.ascontiguousarray(xnf3, np.float64)
        nrhox = vec[0].size
        kw = nrhox if kw is None else int(kw)
        bh = None if bhyd is None else np.ascontiguousarray(bhyd, np.float64)
        if bh is not None and bh.shape != (6, kw):
            raise ValueError("bhyd must be [6, kw]")
        bm = None if bmin is None else np.ascontiguousarray(bmin, np.float64)
        pops = _lib.KappPops(*[v.ctypes.data for v in vec], None if bh is None else bh.ctypes.data,
                             None if bm is None else bm.ctypes.data, None if x3 is None else x3.ctypes.data)
        out = [np.zeros((ws.size, kw)) for _ in range(3)]
        pt = np.zeros((ws.size, 11 if x3 is None else 14, kw)) if parts else None
        self.ctx.call("atlasgpu_atlas_kapp", ws.size, ptr(ws), nrhox, kw, ctypes.byref(pops),
                      *[ptr(o) for o in out], ptr(pt))
        return (*out, pt) if parts else tuple(out)

    def xlinop(self, records, nrhox, xnfdop, dopple, xne, txnxn, hckt, tabcont, iwt, waveset, contx, xlines=None,
               xnfp=None, rho=None, hydrogen=None):
        """XLINOP on unit-19 records (NLTE_LINE array, sorted by wavelength),
        added into a copy of xlines [numnu, kw] (zeros when None).  contx:
        CONTX(25,16) as [16, 25].  With xnfp [nspec, kw] and rho [kw] also the
        autoionizing and merged-continuum records; with hydrogen = dict(t,
        xnf1, xnf2, xnh2) [nrhox] (and xnfp, and set_hydrogen_tables) also the
        hydrogen lines.  Returns (xlines, number of records of the types not
        handled)."""
        rec = np.ascontiguousarray(records, _lib.NLTE_LINE)
        xd = np.ascontiguousarray(xnfdop, np.float64)
        dp = np.ascontiguousarray(dopple, np.float64)
        nspec, kw = xd.shape
        vec = [np.ascontiguousarray(v, np.float64) for v in (xne, txnxn, hckt)]
        tc = np.ascontiguousarray(tabcont, np.float64)
        iw = np.ascontiguousarray(iwt, np.int32)
        ws = np.ascontiguousarray(waveset, np.float64)
        cx = np.ascontiguousarray(contx, np.float64)
        out = np.zeros((ws.size, kw)) if xlines is None else np.array(xlines, np.float64, copy=True, order="C")
        other = ctypes.c_int64(0)
        xp = None if xnfp is None else np.ascontiguousarray(xnfp, np.float64)
        rh = None if rho is None else np.ascontiguousarray(rho, np.float64)
        hy = None
        if hydrogen is not None:
            hv = [np.ascontiguousarray(hydrogen[k], np.float64) for k in ("t", "xnf1", "xnf2", "xnh2")]
            hs = _lib.XlinopHydrogen(*[v.ctypes.data for v in hv])
            hy = ctypes.byref(hs)
        self.ctx.call("atlasgpu_atlas_xlinop", ptr(rec), rec.shape[0], int(nrhox), kw, ptr(xd), ptr(dp), nspec,
                      *[ptr(v) for v in vec], ptr(tc), ptr(iw), iw.size - 1, ptr(ws), ws.size, ptr(cx), ptr(xp),
                      ptr(rh), hy, ptr(out), ctypes.byref(other))
        return out, other.value

    def rt_pass(self, waveset, rcoset, acont, sigmac, xlines, rhox, t, hkt, teff, scont=None):
        ws, rc = (np.ascontiguousarray(v, np.float64) for v in (waveset, rcoset))
        ac, sg, xl = (np.ascontiguousarray(v, np.float64) for v in (acont, sigmac, xlines))
        sc = None if scont is None else np.ascontiguousarray(scont, np.float64)
        numnu, kw = ac.shape
        rx, tt, hk = (np.ascontiguousarray(v, np.float64) for v in (rhox, t, hkt))
        nrhox = rx.size
        acc = {k: np.zeros(nrhox) for k in ACC_NAMES}
        A = Accum(*[_dp(acc[k]) for k in ACC_NAMES], 0.0)
        hs = np.zeros(numnu)
        self.ctx.call("atlasgpu_atlas_rt_pass", numnu, ptr(ws), ptr(rc), ptr(ac), ptr(sg), ptr(sc), kw, ptr(xl),
                      nrhox, ptr(rx), ptr(tt), ptr(hk), float(teff), ctypes.byref(A), ptr(hs))
        acc["pradk0"] = A.pradk0
        return acc, hs

    def finish(self, model, acc, iteration, store):
        """model: dict of [nrhox] arrays (t, rhox, p, xne, abross, prad, vturb, pturb, tauros, accrad,
        raden, oldt1) updated in place; store: RossStore (ROSSTAB history, updated).
        Returns (max |FLXERR|, dict of the .iter columns)."""
        n = model["t"].size
        out = {k: np.zeros(n) for k in ("flxerr", "dtflux", "dtlamb", "dtsurf", "t1")}
        names = ("t", "rhox", "p", "xne", "abross", "prad", "vturb", "pturb", "tauros", "accrad", "raden", "oldt1")
        for k in names:
            model[k] = np.ascontiguousarray(model[k], np.float64)
        st = FinishState(n, int(iteration), float(model["teff"]), float(model["grav"]), float(acc["pradk0"]),
                         *[_dp(model[k]) for k in names], *[_dp(out[k]) for k in out],
                         store.n, store.maxtab, *store.norm, _dp(store.t), _dp(store.p), _dp(store.k))
        a = {k: np.ascontiguousarray(acc[k], np.float64).copy() for k in ACC_NAMES}
        A = Accum(*[_dp(a[k]) for k in ACC_NAMES], float(acc["pradk0"]))
        err = ctypes.c_double(0)
        self.ctx.call("atlasgpu_atlas_finish", ctypes.byref(st), ctypes.byref(A), ctypes.byref(err))
        model["pradk0"] = st.pradk0
        store.n = st.ross_n
        store.norm = [st.ross_zerot, st.ross_slopet, st.ross_zerop, st.ross_slopep]
        return err.value, out


class RossStore:
    """ROSSTAB's growing table of the model's own (log T, log P, log kappa_R)
    points (ROSSTAB_MAXTAB = kw*60 with kw = 80)."""

    def __init__(self, maxtab=80 * 60):
        self.n = 0
        self.maxtab = maxtab
        self.norm = [0.0, 1.0, 0.0, 1.0]
        self.t = np.zeros(maxtab)
        self.p = np.zeros(maxtab)
        self.k = np.zeros(maxtab)

    def copy(self):
        c = RossStore(self.maxtab)
        c.n, c.norm = self.n, list(self.norm)
        c.t, c.p, c.k = self.t.copy(), self.p.copy(), self.k.copy()
        return c


class AtlasModel:
    """One ATLAS12 atmosphere iterated entirely on the device.

    The starting structure is the Eddington grey model on TAUSTD (or a given
    structure); populations and continuum come from atlas12_b200.surrogate.
    """

    def __init__(self, ctx: Context, operators, teff=5777.0, logg=4.44, vturb=1.5, linedata=None,
                 waveset=None, rcoset=None, nrhox=72, ross=None, start=None, h_tables=None, mh=0.0):
        self.ctx = ctx
        ctx.set_operators(operators["xtau8"], operators["coefj"], operators["coefh"], operators["ch_j"],
                          operators["ck_j"])
        if start is None:
            ross = ross or surrogate.RossTable(mh=mh)
            start = surrogate.grey_model(teff, logg, nrhox=nrhox, ross=ross)
        m = start
        if waveset is None:
            waveset, rcoset = synthetic.geometric_waveset()
        self.waveset = np.ascontiguousarray(waveset, np.float64)
        self.rcoset = np.ascontiguousarray(rcoset, np.float64)
        self.cutwave = cutoff_grid()
        ld = np.zeros((0, 4), np.int32) if linedata is None else np.ascontiguousarray(linedata, np.int32)
        h0, h1, h2 = h_tables or tabvoigt(operators)
        self._keep = [np.ascontiguousarray(x, np.float64) for x in (m["t"], m["p"], m["rhox"], m["tauros"])]
        self._keep += [np.ascontiguousarray(x, np.float64) for x in (h0, h1, h2)]
        self._keep += [ld]
        t, p, rx, tau, h0, h1, h2, ld = self._keep
        self.nrhox = t.size
        self.teff = teff
        d = ModelDesc(teff, logg, vturb, self.nrhox, _dp(t), _dp(p), _dp(rx), _dp(tau), _dp(self.waveset),
                      _dp(self.rcoset), self.waveset.size, _dp(self.cutwave), self.cutwave.size,
                      ld.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ld.shape[0], _dp(h0), _dp(h1), _dp(h2),
                      float(mh))
        self._h = ctypes.c_void_p()
        ctx.call("atlasgpu_model_create", ctypes.byref(d), ctypes.byref(self._h))

    def iterate(self, max_iter=30, tol_percent=0.1, graph=True):
        """Iterate until max |FLXERR| <= tol_percent (percent) or max_iter.
        Returns (iterations run, per-iteration max |FLXERR|)."""
        hist = np.zeros(max(max_iter, 1))
        done = ctypes.c_int(0)
        self.ctx.call("atlasgpu_model_iterate", self._h, int(max_iter), float(tol_percent), 1 if graph else 0,
                      ctypes.byref(done), ptr(hist))
        return done.value, hist[:done.value]

    def structure(self):
        n = self.nrhox
        out = {k: np.zeros(n) for k in ("t", "rhox", "p", "xne", "flxerr")}
        hs = np.zeros(self.waveset.size)
        self.ctx.call("atlasgpu_model_get", self._h, *[ptr(out[k]) for k in ("t", "rhox", "p", "xne", "flxerr")],
                      ptr(hs))
        out["hsurf"] = hs
        return out

    def tables(self):
        """The last iteration's TABCONT [nwave+1, nrhox], XLINES, ACONT and
        SIGMAC [numnu, nrhox] (KAPCONT's cutoff table, LINOP1's output and
        the RT pass's continuum)."""
        kw, nn = self.nrhox, self.waveset.size
        tc = np.zeros((self.cutwave.size + 1, kw))
        xl, ac, sg = np.zeros((nn, kw)), np.zeros((nn, kw)), np.zeros((nn, kw))
        self.ctx.call("atlasgpu_model_get_tables", self._h, ptr(tc), ptr(xl), ptr(ac), ptr(sg))
        return dict(tabcont=tc, xlines=xl, acont=ac, sigmac=sg)

    def set_params(self, teff, logg, vturb, mh=0.0):
        """New stellar parameters on the same line list and grid; follow with set_structure."""
        self.teff = teff
        self.ctx.call("atlasgpu_model_set_params", self._h, float(teff), float(logg), float(vturb), float(mh))

    def set_structure(self, t, p, rhox):
        arrs = [np.ascontiguousarray(x, np.float64) for x in (t, p, rhox)]
        self.ctx.call("atlasgpu_model_set_structure", self._h, *[ptr(a) for a in arrs])

    def set_shard(self, nu_first, nu_last):
        """Restrict LINOP1 and the RT pass to frequencies nu_first..nu_last (1-based, inclusive)."""
        self.ctx.call("atlasgpu_model_set_shard", self._h, int(nu_first), int(nu_last))

    def set_sums_buffer(self, d_sums):
        """Frequency sums [8*nrhox + 1] in a caller-owned device buffer (torch tensor; None: internal)."""
        self._sums_ref = d_sums
        self.ctx.call("atlasgpu_model_set_sums_buffer", self._h, ptr(d_sums))

    def iterate_begin(self):
        """Enqueue one iteration up to the (shard's) frequency sums."""
        self.ctx.call("atlasgpu_model_iterate_begin", self._h)

    def iterate_end(self):
        """Enqueue the finish from the sums, wait; returns max |FLXERR| (percent)."""
        e = ctypes.c_double(0.0)
        self.ctx.call("atlasgpu_model_iterate_end", self._h, ctypes.byref(e))
        return e.value

    def close(self):
        if self._h:
            _lib.lib().atlasgpu_model_destroy(self.ctx.handle, self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class AtlasBatch:
    """Many ATLAS12 atmospheres iterated together on the device
    (atlasgpu_batch_*): they share one frequency grid, line list and Voigt
    tables; each slot has its own parameters and structure.

        b = AtlasBatch(ctx, operators, nslots=32, linedata=lines, waveset=ws, rcoset=rc)
        results = b.run_queue(params, starts)     # work queue over all models

    The reference runs the same models as one process each
    (scripts/runat12_grid.slurm:1-16).
    """

    def __init__(self, ctx: Context, operators, nslots, linedata=None, waveset=None, rcoset=None, nrhox=72,
                 h_tables=None, shape="cached"):
        """shape: "cached" applies the launch shape the autotuner cached for
        this GPU and workload (autotune.tune_batch), if any; None keeps the
        library's default; or a (linop_ctas_per_sm, rt_waves) pair."""
        self.ctx = ctx
        ctx.set_operators(operators["xtau8"], operators["coefj"], operators["coefh"], operators["ch_j"],
                          operators["ck_j"])
        if waveset is None:
            waveset, rcoset = synthetic.geometric_waveset()
        self.waveset = np.ascontiguousarray(waveset, np.float64)
        self.rcoset = np.ascontiguousarray(rcoset, np.float64)
        self.cutwave = cutoff_grid()
        ld = np.zeros((0, 4), np.int32) if linedata is None else np.ascontiguousarray(linedata, np.int32)
        h0, h1, h2 = h_tables or tabvoigt(operators)
        dummy = np.ones(nrhox)
        keep = [np.ascontiguousarray(x, np.float64) for x in (dummy, dummy, dummy, dummy, h0, h1, h2)] + [ld]
        t, p, rx, tau, h0, h1, h2, ld = keep
        self.nrhox = nrhox
        self.nslots = int(nslots)
        self.nlines = int(ld.shape[0])
        d = ModelDesc(5777.0, 4.44, 1.5, nrhox, _dp(t), _dp(p), _dp(rx), _dp(tau), _dp(self.waveset),
                      _dp(self.rcoset), self.waveset.size, _dp(self.cutwave), self.cutwave.size,
                      ld.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ld.shape[0], _dp(h0), _dp(h1), _dp(h2), 0.0)
        self._h = ctypes.c_void_p()
        ctx.call("atlasgpu_batch_create", ctypes.byref(d), self.nslots, ctypes.byref(self._h))
        if shape == "cached":
            from .autotune import cached_shape
            shape = cached_shape(self)
        if shape is not None:
            self.set_shape(*shape)

    def load(self, slot, teff, logg, vturb, mh, start, max_iter=60, tol_percent=0.1):
        """Start a model in `slot` from start = dict(t, p, rhox) on TAUSTD."""
        arrs = [np.ascontiguousarray(start[k], np.float64) for k in ("t", "p", "rhox")]
        self.ctx.call("atlasgpu_batch_load", self._h, int(slot), float(teff), float(logg), float(vturb), float(mh),
                      *[ptr(a) for a in arrs], int(max_iter), float(tol_percent))

    def step(self, n=1):
        self.ctx.call("atlasgpu_batch_step", self._h, int(n))

    def set_shape(self, linop_ctas_per_sm, rt_waves):
        """Launch shape of the batched LINOP1 and RT kernels (see atlas12_b200.autotune)."""
        self.ctx.call("atlasgpu_batch_set_shape", self._h, int(linop_ctas_per_sm), int(rt_waves))

    def shape(self):
        a, b = ctypes.c_int(0), ctypes.c_int(0)
        self.ctx.call("atlasgpu_batch_get_shape", self._h, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def poll(self):
        """(status, iterations done, last max |FLXERR|) per slot, and the number running."""
        st = np.zeros(self.nslots, np.int32)
        it = np.zeros(self.nslots, np.int32)
        er = np.zeros(self.nslots)
        run = ctypes.c_int(0)
        self.ctx.call("atlasgpu_batch_poll", self._h, ptr(st), ptr(it), ptr(er), ctypes.byref(run))
        return st, it, er, run.value

    def run(self, poll_every=4):
        st = np.zeros(self.nslots, np.int32)
        it = np.zeros(self.nslots, np.int32)
        er = np.zeros(self.nslots)
        self.ctx.call("atlasgpu_batch_run", self._h, int(poll_every), ptr(st), ptr(it), ptr(er))
        return st, it, er

    def structure(self, slot, iters=None):
        n = self.nrhox
        out = {k: np.zeros(n) for k in ("t", "rhox", "p", "xne", "flxerr")}
        hs = np.zeros(self.waveset.size)
        hist = np.zeros(_lib.BATCH_MAX_ITER)
        self.ctx.call("atlasgpu_batch_get", self._h, int(slot), *[ptr(out[k]) for k in ("t", "rhox", "p", "xne",
                                                                                        "flxerr")], ptr(hs),
                      ptr(hist))
        out["hsurf"] = hs
        if iters is not None:
            out["hist"] = hist[:iters]
        return out

    def run_queue(self, params, starts, max_iter=60, tol_percent=0.1, poll_every=2, keep=True, fallback=None,
                  first_max_iter=None):
        """Iterate every model of `params` ([n, 4]: Teff, log g, [M/H], vturb)
        from starts[i] (dict t, p, rhox), keeping all slots busy: a slot that
        finishes is read back and loaded with the next model.  With
        `fallback` (a second list of starts, e.g. the grey models), a model
        whose first attempt ends without converging (non-finite, or capped
        at first_max_iter iterations) is run again from fallback[i] with
        max_iter.  Returns a list of dicts (status, iters = iterations of
        all attempts, maxerr, attempts, and the structure when keep)."""
        n = len(params)
        res = [None] * n
        spent = [0] * n
        slot_of = [-1] * self.nslots
        attempt = [0] * self.nslots
        queue = [(i, 0) for i in range(n)]  # (model, attempt)
        cap0 = max_iter if (fallback is None or first_max_iter is None) else first_max_iter

        def load(s, i, k):
            teff, logg, mh, vt = params[i]
            st = starts[i] if k == 0 else fallback[i]
            self.load(s, teff, logg, vt, mh, st, cap0 if k == 0 else max_iter, tol_percent)
            slot_of[s] = i
            attempt[s] = k

        for s in range(min(self.nslots, n)):
            load(s, *queue.pop(0))
        while any(k >= 0 for k in slot_of):
            self.step(poll_every)
            st, it, er, _ = self.poll()
            for s in range(self.nslots):
                i = slot_of[s]
                if i < 0 or st[s] == _lib.SLOT_RUNNING:
                    continue
                spent[i] += int(it[s])
                slot_of[s] = -1
                if st[s] != _lib.SLOT_CONVERGED and fallback is not None and attempt[s] == 0:
                    queue.insert(0, (i, 1))
                else:
                    r = {"status": int(st[s]), "iters": spent[i], "maxerr": float(er[s]), "attempts": attempt[s] + 1}
                    if keep:
                        r.update(self.structure(s, int(it[s])))
                    res[i] = r
                if queue:
                    load(s, *queue.pop(0))
        return res

    def close(self):
        if self._h:
            _lib.lib().atlasgpu_batch_destroy(self.ctx.handle, self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
