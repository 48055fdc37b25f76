"""ctypes wrapper around the CPU oracle (oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The product (atlas12_b200)
never imports this module.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int32)
NXTAU = 51
REF32, FP64 = 0, 1


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = ctypes.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


def _declare(L):
    L.orc_integ.argtypes = [_dp, _dp, _dp, ctypes.c_int, ctypes.c_double]
    L.orc_parcoe.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_int]
    L.orc_deriv.argtypes = [_dp, _dp, _dp, ctypes.c_int]
    L.orc_map1.argtypes = [_dp, _dp, ctypes.c_int, _dp, _dp, ctypes.c_int]
    L.orc_map1.restype = ctypes.c_int
    L.orc_solvit.argtypes = [_dp, ctypes.c_int, _dp, _ip]
    L.orc_expi.argtypes = [ctypes.c_int, ctypes.c_double]
    L.orc_expi.restype = ctypes.c_double
    L.orc_voigt_weideman.argtypes = [ctypes.c_double, ctypes.c_double]
    L.orc_voigt_weideman.restype = ctypes.c_double
    L.orc_voigt_profile.argtypes = [ctypes.c_float, ctypes.c_float]
    L.orc_voigt_profile.restype = ctypes.c_float
    L.orc_tabvoigt.argtypes = [ctypes.c_double, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp, _dp]
    L.orc_voigt_kurucz.argtypes = [ctypes.c_double, ctypes.c_double, _dp, _dp, _dp]
    L.orc_voigt_kurucz.restype = ctypes.c_double
    L.orc_synthe_nbuff.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_int32]
    L.orc_synthe_nbuff.restype = ctypes.c_int32
    L.orc_build_tablog.argtypes = [_dp]


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a, t=_dp):
    return a.ctypes.data_as(t)


# ---------------------------------------------------------------- numerics
def integ(x, f, start):
    x, f = _d(x), _d(f)
    out = np.zeros_like(x)
    lib().orc_integ(_ptr(x), _ptr(f), _ptr(out), x.size, float(start))
    return out


def deriv(x, f):
    x, f = _d(x), _d(f)
    out = np.zeros_like(x)
    lib().orc_deriv(_ptr(x), _ptr(f), _ptr(out), x.size)
    return out


def map1(xold, fold, xnew):
    xold, fold, xnew = _d(xold), _d(fold), _d(xnew)
    out = np.zeros_like(xnew)
    r = lib().orc_map1(_ptr(xold), _ptr(fold), xold.size, _ptr(xnew), _ptr(out), xnew.size)
    return out, r


def solvit(A, b):
    n = A.shape[0]
    a = np.asfortranarray(A, dtype=np.float64).copy(order="F")
    x = _d(b).copy()
    piv = np.zeros(n, dtype=np.int32)
    lib().orc_solvit(a.ctypes.data_as(_dp), n, _ptr(x), _ptr(piv, _ip))
    return x


def expi(n, x):
    return lib().orc_expi(int(n), float(x))


def voigt_weideman(v, a):
    return lib().orc_voigt_weideman(float(v), float(a))


def voigt_profile(v, a):
    return lib().orc_voigt_profile(float(v), float(a))


def tabvoigt(tabvi, tabh1, vsteps=200.0, n=2001):
    tabvi, tabh1 = _d(tabvi), _d(tabh1)
    h0, h1, h2 = (np.zeros(n) for _ in range(3))
    lib().orc_tabvoigt(vsteps, n, _ptr(tabvi), _ptr(tabh1), tabvi.size, _ptr(h0), _ptr(h1), _ptr(h2))
    return h0, h1, h2


def voigt_kurucz(v, a, h0, h1, h2):
    return lib().orc_voigt_kurucz(float(v), float(a), _ptr(h0), _ptr(h1), _ptr(h2))


def build_tablog():
    out = np.zeros(65536)
    lib().orc_build_tablog(_ptr(out))
    return out


def nbuff(wlvac, ratiolg, ixwlbeg):
    return lib().orc_synthe_nbuff(float(wlvac), float(ratiolg), int(ixwlbeg))


# ---------------------------------------------------------------- structs
class _Grid(ctypes.Structure):
    _fields_ = [("ratio", ctypes.c_double), ("ratiolg", ctypes.c_double), ("wbegin", ctypes.c_double),
                ("length", ctypes.c_int32), ("ixwlbeg", ctypes.c_int32)]


class Ops(ctypes.Structure):
    _fields_ = [("xtau", ctypes.c_double * NXTAU), ("coefj", ctypes.c_double * (NXTAU * NXTAU)),
                ("coefh", ctypes.c_double * (NXTAU * NXTAU)), ("ch", ctypes.c_double * NXTAU),
                ("ck", ctypes.c_double * NXTAU)]

    @classmethod
    def from_tables(cls, t):
        o = cls()
        o.xtau[:] = list(t["xtau8"])
        o.coefj[:] = list(np.asarray(t["coefj"]).ravel(order="F"))
        o.coefh[:] = list(np.asarray(t["coefh"]).ravel(order="F"))
        o.ch[:] = list(t["ch_j"])
        o.ck[:] = list(t["ck_j"])
        return o


class _Lines(ctypes.Structure):
    _fields_ = [("nbuff", _ip), ("cgf", _fp), ("nelion", _ip), ("elo", _fp), ("gamrf", _fp),
                ("gamsf", _fp), ("gamwf", _fp), ("n", ctypes.c_int64)]


class _Josh(ctypes.Structure):
    _fields_ = [(n, _dp) for n in ("rhox", "acont", "aline", "sigmac", "sigmal", "scont", "sline", "bnu")] + \
               [("nrhox", ctypes.c_int)] + \
               [(n, _dp) for n in ("abtot", "alpha", "taunu", "snu", "jnu", "hnu", "jmins")] + \
               [("knu1", ctypes.c_double), ("maxj", ctypes.c_int), ("edd_iters", ctypes.c_int)]


class _Accum(ctypes.Structure):
    _fields_ = [(n, _dp) for n in ("rjmins", "rdabh", "rdiagj", "flxrad", "raden", "h_total",
                                     "accrad", "abross")] + [("pradk0", ctypes.c_double)]


class _AtlasTables(ctypes.Structure):
    _fields_ = [("h0tab", _dp), ("h1tab", _dp), ("h2tab", _dp), ("tablog", _dp)]


def _declare2(L):
    L.orc_synthe_grid.argtypes = [ctypes.c_double] * 3 + [ctypes.POINTER(_Grid)]
    L.orc_synthe_continuum.argtypes = [ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_void_p]
    L.orc_synthe_line_opacity.argtypes = [ctypes.c_int, ctypes.POINTER(_Lines), ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_void_p, _dp, _dp, ctypes.c_int, _dp, _dp,
                                          _dp, ctypes.c_int, _dp, _fp]
    L.orc_josh.argtypes = [ctypes.POINTER(Ops), ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Josh)]
    L.orc_synthe_spectrum.argtypes = [ctypes.POINTER(Ops), _dp, ctypes.c_int, _dp, _dp, ctypes.c_int,
                                      ctypes.c_int, _dp, _dp, ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                      _fp, ctypes.c_int, ctypes.c_int, _dp, _dp]
    L.orc_atlas_linop1.argtypes = [ctypes.POINTER(_AtlasTables), _ip, ctypes.c_int64, ctypes.c_int,
                                   ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp, _dp, _dp, _ip,
                                   ctypes.c_int, _dp, ctypes.c_int, _dp]
    L.orc_atlas_linop1.restype = ctypes.c_int64
    L.orc_atlas_xlinop.argtypes = [ctypes.POINTER(_AtlasTables), ctypes.c_void_p, ctypes.c_int64, ctypes.c_int,
                                   ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp, _dp, _dp, _ip,
                                   ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp, ctypes.c_void_p,
                                   ctypes.c_void_p, _dp]
    L.orc_stark_profile.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_int]
    L.orc_stark_profile.restype = ctypes.c_double
    L.orc_hfnm.argtypes = [ctypes.c_int, ctypes.c_int]
    L.orc_hfnm.restype = ctypes.c_double
    L.orc_hprof4_point.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 9
    L.orc_hprof4_point.restype = ctypes.c_double
    L.orc_atlas_xlinop.restype = ctypes.c_int64
    L.orc_synthe_nlte_opacity.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                          ctypes.POINTER(ctypes.c_float), _dp, _dp, _dp, ctypes.c_int, _dp, _dp,
                                          _dp, _dp, _dp]
    L.orc_synthe_nlte_opacity.restype = None
    L.orc_atlas_rt_pass.argtypes = [ctypes.POINTER(Ops), ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_void_p,
                                    ctypes.c_int, _dp, ctypes.c_int, _dp, _dp, _dp, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Accum), _dp]


_declared2 = False


def _lib2():
    global _declared2
    L = lib()
    if not _declared2:
        _declare2(L)
        _declared2 = True
    return L


# ---------------------------------------------------------------- SYNTHE
def synthe_grid(wlbeg, wlend, resolu):
    g = _Grid()
    _lib2().orc_synthe_grid(wlbeg, wlend, resolu, ctypes.byref(g))
    return dict(ratio=g.ratio, ratiolg=g.ratiolg, wbegin=g.wbegin, length=g.length, ixwlbeg=g.ixwlbeg)


def synthe_continuum(mode, wledge, continall, wbegin, ratio, length):
    wledge, continall = _d(wledge), _d(continall)
    nrhox, stride = continall.shape
    out = np.zeros((nrhox, length), dtype=np.float32 if mode == REF32 else np.float64)
    _lib2().orc_synthe_continuum(mode, _ptr(wledge), wledge.size, _ptr(continall), stride, nrhox,
                                 wbegin, ratio, length, out.ctypes.data_as(ctypes.c_void_p))
    return out


def synthe_line_opacity(mode, lines, length, atm, continuum, resolu, maxprof=1000000):
    """lines: dict of SoA arrays; atm: dict(xnfdop[nrhox,nspec], dopple, xne, txnxn, hckt)."""
    arrs = dict(nbuff=np.ascontiguousarray(lines["nbuff"], np.int32),
                cgf=np.ascontiguousarray(lines["cgf"], np.float32),
                nelion=np.ascontiguousarray(lines["nelion"], np.int32),
                elo=np.ascontiguousarray(lines["elo"], np.float32),
                gamrf=np.ascontiguousarray(lines["gamrf"], np.float32),
                gamsf=np.ascontiguousarray(lines["gamsf"], np.float32),
                gamwf=np.ascontiguousarray(lines["gamwf"], np.float32))
    L = _Lines(_ptr(arrs["nbuff"], _ip), _ptr(arrs["cgf"], _fp), _ptr(arrs["nelion"], _ip),
               _ptr(arrs["elo"], _fp), _ptr(arrs["gamrf"], _fp), _ptr(arrs["gamsf"], _fp),
               _ptr(arrs["gamwf"], _fp), arrs["nbuff"].size)
    xnfdop, dopple = _d(atm["xnfdop"]), _d(atm["dopple"])
    nrhox, nspec = xnfdop.shape
    xne, txnxn, hckt = _d(atm["xne"]), _d(atm["txnxn"]), _d(atm["hckt"])
    cont = np.ascontiguousarray(continuum)
    out64 = np.zeros((nrhox, length))
    out32 = np.zeros((nrhox, length), dtype=np.float32)
    _lib2().orc_synthe_line_opacity(mode, ctypes.byref(L), length, nrhox, resolu,
                                    cont.ctypes.data_as(ctypes.c_void_p), _ptr(xnfdop), _ptr(dopple), nspec,
                                    _ptr(xne), _ptr(txnxn), _ptr(hckt), maxprof, _ptr(out64), _ptr(out32, _fp))
    return out32, out64


def josh(ops, ifscat, ifsurf, rhox, acont, aline, sigmac, sigmal, scont, sline, bnu):
    ins = [_d(v) for v in (rhox, acont, aline, sigmac, sigmal, scont, sline, bnu)]
    nr = ins[0].size
    outs = [np.zeros(nr) for _ in range(7)]
    st = _Josh(*[_ptr(v) for v in ins], nr, *[_ptr(v) for v in outs], 0.0, 0, 0)
    _lib2().orc_josh(ctypes.byref(ops), ifscat, ifsurf, ctypes.byref(st))
    names = ("abtot", "alpha", "taunu", "snu", "jnu", "hnu", "jmins")
    r = dict(zip(names, outs))
    r.update(knu1=st.knu1, maxj=st.maxj, edd_iters=st.edd_iters)
    return r


def synthe_spectrum(ops, wledge, contabs, contscat, rhox, hkt, wbegin, ratio, opacity, iw0=1, iw1=None):
    wledge, contabs, contscat, rhox, hkt = (_d(v) for v in (wledge, contabs, contscat, rhox, hkt))
    op = np.ascontiguousarray(opacity, np.float32)
    nrhox, length = op.shape
    iw1 = length if iw1 is None else iw1
    n = iw1 - iw0 + 1
    flux, cont = np.zeros(n), np.zeros(n)
    _lib2().orc_synthe_spectrum(ctypes.byref(ops), _ptr(wledge), wledge.size, _ptr(contabs), _ptr(contscat),
                                contabs.shape[1], nrhox, _ptr(rhox), _ptr(hkt), wbegin, ratio, length,
                                _ptr(op, _fp), iw0, iw1, _ptr(flux), _ptr(cont))
    return flux, cont


# ---------------------------------------------------------------- ATLAS
def atlas_linop1(h0, h1, h2, tablog, linedata, atm, tabcont, iwavetab, waveset):
    """atm: dict(xnfdop[nspec,kw], dopple[nspec,kw], xne[kw], txnxn[kw], hckt[kw]) -> xlines[numnu,kw]."""
    h0, h1, h2, tablog = (_d(v) for v in (h0, h1, h2, tablog))
    tb = _AtlasTables(_ptr(h0), _ptr(h1), _ptr(h2), _ptr(tablog))
    ld = np.ascontiguousarray(linedata, np.int32)
    xnfdop, dopple = _d(atm["xnfdop"]), _d(atm["dopple"])
    nspec, kw = xnfdop.shape
    nrhox = int(atm.get("nrhox", kw))
    xne, txnxn, hckt = _d(atm["xne"]), _d(atm["txnxn"]), _d(atm["hckt"])
    tabcont = _d(tabcont)
    iw = np.ascontiguousarray(iwavetab, np.int32)
    waveset = _d(waveset)
    xl = np.zeros((waveset.size, kw))
    used = _lib2().orc_atlas_linop1(ctypes.byref(tb), _ptr(ld, _ip), ld.shape[0], nrhox, kw, _ptr(xnfdop),
                                    _ptr(dopple), nspec, _ptr(xne), _ptr(txnxn), _ptr(hckt), _ptr(tabcont),
                                    _ptr(iw, _ip), iw.size - 1, _ptr(waveset), waveset.size, _ptr(xl))
    return xl, used


def atlas_rt_pass(ops, waveset, rcoset, acont, sigmac, xlines, rhox, t, hkt, teff, scont=None, nu0=1, nu1=None):
    waveset, rcoset, acont, sigmac, xlines, rhox, t, hkt = (
        _d(v) for v in (waveset, rcoset, acont, sigmac, xlines, rhox, t, hkt))
    numnu, kw = acont.shape
    nrhox = rhox.size
    nu1 = numnu if nu1 is None else nu1
    acc = {k: np.zeros(nrhox) for k in ("rjmins", "rdabh", "rdiagj", "flxrad", "raden", "h_total",
                                         "accrad", "abross")}
    A = _Accum(*[_ptr(acc[k]) for k in ("rjmins", "rdabh", "rdiagj", "flxrad", "raden", "h_total",
                                        "accrad", "abross")], 0.0)
    hs = np.zeros(nu1 - nu0 + 1)
    sc = None if scont is None else _d(scont)
    _lib2().orc_atlas_rt_pass(ctypes.byref(ops), numnu, _ptr(waveset), _ptr(rcoset), _ptr(acont), _ptr(sigmac),
                              None if sc is None else sc.ctypes.data_as(ctypes.c_void_p), kw, _ptr(xlines), nrhox,
                              _ptr(rhox), _ptr(t), _ptr(hkt), teff, nu0, nu1, ctypes.byref(A), _ptr(hs))
    acc["pradk0"] = A.pradk0
    return acc, hs


# ---------------------------------------------------------------- ATLAS finish
_DPp = ctypes.POINTER(ctypes.c_double)


class _Tcorr(ctypes.Structure):
    _fields_ = [("nrhox", ctypes.c_int), ("iter", ctypes.c_int), ("teff", ctypes.c_double),
                ("grav", ctypes.c_double), ("pradk0", ctypes.c_double)] + \
               [(n, _DPp) for n in ("t", "rhox", "p", "xne", "abross", "prad", "vturb", "pturb", "tauros",
                                    "accrad", "raden", "oldt1", "rjmins", "rdabh", "rdiagj", "flxrad", "h_total",
                                    "flxerr", "dtflux", "dtlamb", "dtsurf", "t1")] + \
               [("nross", ctypes.c_int), ("maxtab", ctypes.c_int), ("zerot", ctypes.c_double),
                ("slopet", ctypes.c_double), ("zerop", ctypes.c_double), ("slopep", ctypes.c_double),
                ("tabt", _DPp), ("tabp", _DPp), ("tabk", _DPp)]


class RossStore:
    """ROSSTAB's growing (log T, log P, log kappa_R) table (KW*60 entries, KW = 80)."""

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


def atlas_finish(model, acc, iteration, store):
    """ROSS(3)/ROSSTAB store/RADIAP(3)/TCORR(3) restatement; model dict and the
    RossStore updated in place."""
    L = lib()
    L.orc_atlas_finish.argtypes = [ctypes.POINTER(_Tcorr)]
    L.orc_atlas_finish.restype = ctypes.c_double
    n = model["t"].size
    names = ("t", "rhox", "p", "xne", "abross", "prad", "vturb", "pturb", "tauros", "accrad", "raden", "oldt1")
    for k in names:
        model[k] = np.ascontiguousarray(model[k], np.float64)
    a = {k: np.ascontiguousarray(acc[k], np.float64).copy() for k in ("rjmins", "rdabh", "rdiagj", "flxrad",
                                                                      "h_total", "raden", "accrad", "abross")}
    # ROSS/RADIAP mode 3 turn the accumulated sums into the model quantities in place
    model["abross"] = a["abross"]
    model["raden"] = a["raden"]
    model["accrad"] = a["accrad"]
    out = {k: np.zeros(n) for k in ("flxerr", "dtflux", "dtlamb", "dtsurf", "t1")}
    s = _Tcorr(n, int(iteration), float(model["teff"]), float(model["grav"]), float(acc["pradk0"]),
               *[_ptr(model[k]) for k in names], *[_ptr(a[k]) for k in ("rjmins", "rdabh", "rdiagj", "flxrad",
                                                                         "h_total")],
               *[_ptr(out[k]) for k in out], store.n, store.maxtab, *store.norm, _ptr(store.t), _ptr(store.p),
               _ptr(store.k))
    err = L.orc_atlas_finish(ctypes.byref(s))
    store.n = s.nross
    store.norm = [s.zerot, s.slopet, s.zerop, s.slopep]
    model["pradk0"] = s.pradk0
    return err, out


def _tcorr_for(store, t, p, abross, grav, keep):
    """A _Tcorr over (t, p, abross) carrying the ROSSTAB store; arrays kept alive in keep."""
    n = np.asarray(t).size
    cols = {k: np.zeros(n) for k in ("t", "rhox", "p", "xne", "abross", "prad", "vturb", "pturb", "tauros",
                                     "accrad", "raden", "oldt1", "rjmins", "rdabh", "rdiagj", "flxrad",
                                     "h_total", "flxerr", "dtflux", "dtlamb", "dtsurf", "t1")}
    cols["t"][:], cols["p"][:], cols["abross"][:] = t, p, abross
    keep.append(cols)
    return _Tcorr(n, 1, 0.0, float(grav), 0.0, *[_ptr(cols[k]) for k in cols], store.n, store.maxtab,
                  *store.norm, _ptr(store.t), _ptr(store.p), _ptr(store.k))


def rosstab_store(store, t, p, abross):
    """ROSSTAB store (IROSSTAB = 1) of one model's (T, P, ABROSS) into store."""
    keep = []
    s = _tcorr_for(store, t, p, abross, 0.0, keep)
    L = lib()
    L.orc_rosstab_store.argtypes = [ctypes.POINTER(_Tcorr)]
    L.orc_rosstab_store(ctypes.byref(s))
    store.n = s.nross
    store.norm = [s.zerot, s.slopet, s.zerop, s.slopep]


def ttaup(store, t, tau, grav, prad):
    """TTAUP: hydrostatic P(tau) for T(tau) with kappa_R from the ROSSTAB store.
    Returns (abstd, ptotal, p)."""
    keep = []
    n = np.asarray(t).size
    s = _tcorr_for(store, t, np.zeros(n), np.zeros(n), grav, keep)
    t, tau, prad = _d(t), _d(tau), _d(prad)
    ab, pt, po = np.zeros(n), np.zeros(n), np.zeros(n)
    L = lib()
    L.orc_ttaup.argtypes = [ctypes.POINTER(_Tcorr)] + [ctypes.c_void_p] * 6 + [ctypes.c_int]
    L.orc_ttaup(ctypes.byref(s), _ptr(t), _ptr(tau), _ptr(ab), _ptr(pt), _ptr(po), _ptr(prad), n)
    return ab, pt, po


# unit-19 NLTE / complex-profile record (nlte_line_t, mod_mklinelist.f90:43-63), padded to 64 bytes
NLTE_LINE = np.dtype([("wlvac", "<f8"), ("elo", "<f4"), ("gf", "<f4"), ("nblo", "<i4"), ("nbup", "<i4"),
                      ("nelion", "<i4"), ("itype", "<i4"), ("ncon", "<i4"), ("nelionx", "<i4"), ("gammar", "<f4"),
                      ("gammas", "<f4"), ("gammaw", "<f4"), ("nbuff", "<i4"), ("lim", "<i4"), ("pad", "<i4")])
assert NLTE_LINE.itemsize == 64


class HTab(ctypes.Structure):
    """orc_htab_t: HPROF4's and STARK_PROFILE's tables and XLINOP's hydrogen level energies."""
    _fields_ = [("xknmtb", ctypes.c_double * 12), ("y1wtm", ctypes.c_double * 4), ("stalph", ctypes.c_double * 34),
                ("stwtal", ctypes.c_double * 34), ("istal", ctypes.c_int32 * 4), ("lnghal", ctypes.c_int32 * 4),
                ("stcomp", ctypes.c_double * 20), ("stcpwt", ctypes.c_double * 20), ("lncomp", ctypes.c_int32 * 4),
                ("cutoffh2plus", ctypes.c_double * 111), ("cutoffh2", ctypes.c_double * 91),
                ("asum", ctypes.c_double * 100), ("asumlyman", ctypes.c_double * 100),
                ("betagrid", ctypes.c_double * 15), ("pp", ctypes.c_double * 5), ("propbm", ctypes.c_double * 525),
                ("c", ctypes.c_double * 35), ("d", ctypes.c_double * 35), ("eh", ctypes.c_double * 10),
                ("elim", ctypes.c_double)]

    @classmethod
    def from_tables(cls, t, prefix="h_"):
        """prefix "h_": ATLAS12's HPROF4 tables; "s_": SYNTHE's hydrogen_line_profile ones."""
        h = cls()
        for name in ("xknmtb", "y1wtm", "stalph", "stwtal", "stcomp", "stcpwt", "cutoffh2plus", "cutoffh2", "asum",
                     "asumlyman", "betagrid", "pp", "propbm", "c", "d", "eh"):
            v = np.ascontiguousarray(t[prefix + name], np.float64).ravel()  # C order: [first-1][second-1]
            getattr(h, name)[:] = v.tolist()
        for name in ("istal", "lnghal", "lncomp"):
            getattr(h, name)[:] = [int(x) for x in t[prefix + name]]
        h.elim = float(t[prefix + "elim"][0])
        return h


class _HAtm(ctypes.Structure):
    _fields_ = [("t", _dp), ("xnf1", _dp), ("xnf2", _dp), ("xnh2", _dp)]


def stark_profile(htab, b, p, n, m):
    return _lib2().orc_stark_profile(ctypes.byref(htab), float(b), float(p), int(n), int(m))


def hfnm(n, m):
    return _lib2().orc_hfnm(int(n), int(m))


def hprof4(htab, n, m, xne, t, xnfp3, xnh2, xnf1, xnf2, xnfp1, dop1, delw):
    return _lib2().orc_hprof4_point(ctypes.byref(htab), int(n), int(m), *[float(v) for v in
                                                                         (xne, t, xnfp3, xnh2, xnf1, xnf2, xnfp1,
                                                                          dop1, delw)])


def atlas_xlinop(h0, h1, h2, tablog, recs, atm, tabcont, iwavetab, waveset, contx, xlines=None):
    """XLINOP; adds into a copy of xlines [numnu, kw] (zeros when None).  contx: CONTX(25,16) as a
    numpy [16, 25] array (column-major view).  With atm["xnfp"] [nspec, kw] and atm["rho"] [kw] also
    the autoionizing and merged-continuum records; with atm["htab"] (HTab) and atm["t"], atm["xnf1"],
    atm["xnf2"], atm["xnh2"] [kw] also the hydrogen lines.  Returns (xlines, records read)."""
    h0, h1, h2, tablog = (_d(v) for v in (h0, h1, h2, tablog))
    tb = _AtlasTables(_ptr(h0), _ptr(h1), _ptr(h2), _ptr(tablog))
    rec = np.ascontiguousarray(recs, NLTE_LINE)
    xnfdop, dopple = _d(atm["xnfdop"]), _d(atm["dopple"])
    nspec, kw = xnfdop.shape
    nrhox = int(atm.get("nrhox", kw))
    xne, txnxn, hckt = _d(atm["xne"]), _d(atm["txnxn"]), _d(atm["hckt"])
    tabcont, waveset, cx = _d(tabcont), _d(waveset), _d(contx)
    iw = np.ascontiguousarray(iwavetab, np.int32)
    xl = np.zeros((waveset.size, kw)) if xlines is None else _d(xlines).copy()
    xp = rh = None
    if atm.get("xnfp") is not None:
        xnfp_a, rho_a = _d(atm["xnfp"]), _d(atm["rho"])
        xp, rh = _ptr(xnfp_a), _ptr(rho_a)
    ht = ha = None
    if atm.get("htab") is not None:
        hv = [_d(atm[k]) for k in ("t", "xnf1", "xnf2", "xnh2")]
        hatm = _HAtm(*[_ptr(v) for v in hv])
        ht, ha = ctypes.byref(atm["htab"]), ctypes.byref(hatm)
    nread = _lib2().orc_atlas_xlinop(ctypes.byref(tb), rec.ctypes.data_as(ctypes.c_void_p), rec.shape[0], nrhox, kw,
                                     _ptr(xnfdop), _ptr(dopple), nspec, _ptr(xne), _ptr(txnxn), _ptr(hckt),
                                     _ptr(tabcont), _ptr(iw, _ip), iw.size - 1, _ptr(waveset), waveset.size, _ptr(cx),
                                     xp, rh, ht, ha, _ptr(xl))
    return xl, nread


def synthe_nlte_opacity(recs, length, wbegin, ratio, wlend, velshift_kms, continuum, atm, contx):
    """compute_line_opacity's normal-metal branch (and, with atm["xnfpel"] [nrhox, nspec], the Shore
    lines) in FP64: the contribution [nrhox, length] (double).  continuum [nrhox, length] float;
    atm: xnfdop, dopple [nrhox, nspec], xne, txnxn, hckt; contx [17, 26]."""
    rec = np.ascontiguousarray(recs, NLTE_LINE)
    cont = np.ascontiguousarray(continuum, np.float32)
    xnfdop, dopple = _d(atm["xnfdop"]), _d(atm["dopple"])
    xp = None if atm.get("xnfpel") is None else _d(atm["xnfpel"])
    nrhox, nspec = xnfdop.shape
    out = np.zeros((nrhox, length))
    _lib2().orc_synthe_nlte_opacity(rec.ctypes.data_as(ctypes.c_void_p), rec.shape[0], length, nrhox, wbegin, ratio,
                                    wlend, velshift_kms, cont.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                    _ptr(xnfdop), _ptr(dopple), None if xp is None else _ptr(xp), nspec,
                                    _ptr(_d(atm["xne"])), _ptr(_d(atm["txnxn"])), _ptr(_d(atm["hckt"])),
                                    _ptr(_d(contx)), _ptr(out))
    return out


# ------------------------------------------------------------- SELECTLINES
SEL_LOWPRED, SEL_LOWOBS, SEL_HI, SEL_DIATOMIC, SEL_TIO, SEL_H2O, SEL_H3PLUS = range(1, 8)
SEL_ERRORS = {-1: "NELION out of range", -2: "unknown MOLCODE", -3: "IWL past the IWAVETAB sentinel",
              -4: "LINEDATA overflow"}
MOL2_REC = np.dtype([("wl", "<f4"), ("gflog", "<f4"), ("e1", "<f4"), ("e2", "<f4"), ("code", "<i4"),
                     ("iso", "<i4"), ("gr", "<i4"), ("label", "<i4")])
H2O_REC = np.dtype([("iwl", "<i4"), ("ielo", "<i2"), ("igflog", "<i2")])
CLIGHT_NMS = 2.99792458e17


class _SelState(ctypes.Structure):
    _fields_ = [("nu", ctypes.c_int32), ("igr", ctypes.c_int32), ("freq", ctypes.c_double)]


class _SelTables(ctypes.Structure):
    _fields_ = [("molcodes", _ip), ("isox", _ip), ("nmol", ctypes.c_int), ("tio_isocorr", _ip),
                ("h2o_isocorr", _ip)]


def xnfdopmax(nrhox, xnfdop, tabcont):
    """XNFDOPMAX [nwave+1, nspec] from xnfdop [nspec, kw] and tabcont [nwave+1, kw]."""
    xnfdop, tabcont = _d(xnfdop), _d(tabcont)
    nspec, kw = xnfdop.shape
    out = np.zeros((tabcont.shape[0], nspec))
    L = _lib2()
    L.orc_xnfdopmax.argtypes = [ctypes.c_int, ctypes.c_int, _dp, ctypes.c_int, _dp, ctypes.c_int, _dp]
    L.orc_xnfdopmax(nrhox, kw, _ptr(xnfdop), nspec, _ptr(tabcont), tabcont.shape[0] - 1, _ptr(out))
    return out


def selectlines(tables, kind, recs, state, xmax, hckt_last, iwavetab, wavetab, cap=None):
    """One SELECTLINES database loop.  tables: dict with molcodes, isox, tio_isocorr, h2o_isocorr;
    state: dict(nu, freq, igr), updated in place.  Returns (linedata [m, 4] int32, error code, record)."""
    recs = np.ascontiguousarray(recs)
    n = recs.shape[0]
    cap = n if cap is None else cap
    mc, ix, ti, hi = (np.ascontiguousarray(tables[k], np.int32)
                      for k in ("molcodes", "isox", "tio_isocorr", "h2o_isocorr"))
    tb = _SelTables(_ptr(mc, _ip), _ptr(ix, _ip), mc.size, _ptr(ti, _ip), _ptr(hi, _ip))
    st = _SelState(int(state["nu"]), int(state["igr"]), float(state["freq"]))
    xmax = _d(xmax)
    iw = np.ascontiguousarray(iwavetab, np.int32)
    wt = _d(wavetab)
    out = np.zeros((max(cap, 1), 4), np.int32)
    bad = ctypes.c_int64(-1)
    L = _lib2()
    L.orc_atlas_selectlines.argtypes = [ctypes.POINTER(_SelTables), ctypes.c_int, ctypes.c_void_p, ctypes.c_int64,
                                        ctypes.POINTER(_SelState), _dp, ctypes.c_int, ctypes.c_double, _ip, _dp,
                                        ctypes.c_int, _ip, ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]
    L.orc_atlas_selectlines.restype = ctypes.c_int64
    r = L.orc_atlas_selectlines(ctypes.byref(tb), kind, recs.ctypes.data_as(ctypes.c_void_p), n, ctypes.byref(st),
                                _ptr(xmax), xmax.shape[1], float(hckt_last), _ptr(iw, _ip), _ptr(wt), wt.size,
                                _ptr(out, _ip), cap, ctypes.byref(bad))
    if r < 0:
        return None, int(r), int(bad.value)
    state.update(nu=st.nu, igr=st.igr, freq=st.freq)
    return out[:r].copy(), 0, -1


# ------------------------------------------------------------- SYNTHE hydrogen lines
class Stehle(ctypes.Structure):
    """orc_stehle_t: one Stehle series (n_dens = 0: not loaded)."""
    _fields_ = [("n_lower", ctypes.c_int32), ("n_upper_min", ctypes.c_int32), ("n_upper_max", ctypes.c_int32),
                ("n_dens", ctypes.c_int32), ("density_grid", ctypes.c_double * 20), ("temp_grid", ctypes.c_double * 10),
                ("log_dalpha_grid", ctypes.c_double * 60), ("max_dens_idx", ctypes.c_void_p),
                ("k_alpha", ctypes.c_void_p), ("profiles", ctypes.c_void_p)]


def stehle_structs(series):
    """series: 4 dicts (or None) with n_lower, n_upper_min, n_upper_max, density_grid, temp_grid,
    log_dalpha_grid, max_dens_idx, k_alpha, profiles [n_trans, n_dens, 10, 60].  Returns the ctypes
    array and the arrays it points into (keep both alive)."""
    arr, keep = (Stehle * 4)(), []
    for i, s in enumerate(series):
        if s is None:
            continue
        mdi = np.ascontiguousarray(s["max_dens_idx"], np.int32)
        ka = np.ascontiguousarray(s["k_alpha"], np.float64)
        pr = np.ascontiguousarray(s["profiles"], np.float64)
        keep += [mdi, ka, pr]
        a = arr[i]
        a.n_lower, a.n_upper_min, a.n_upper_max = int(s["n_lower"]), int(s["n_upper_min"]), int(s["n_upper_max"])
        a.n_dens = len(s["density_grid"])
        a.density_grid[:a.n_dens] = [float(x) for x in s["density_grid"]]
        a.temp_grid[:] = [float(x) for x in s["temp_grid"]]
        a.log_dalpha_grid[:] = [float(x) for x in s["log_dalpha_grid"]]
        a.max_dens_idx, a.k_alpha, a.profiles = mdi.ctypes.data, ka.ctypes.data, pr.ctypes.data
    return arr, keep


class _SHAtm(ctypes.Structure):
    _fields_ = [("t", _dp), ("xnfph1", _dp), ("xnfph2", _dp), ("xnfhe1", _dp), ("xnfh2", _dp)]


def synthe_hprof_kp(htab, n, m, xne, t, xnfph1, xnfph2, xnfhe1, xnfh2, dopph, delw):
    """hydrogen_line_profile's K-P path at one depth (SYNTHE's tables in htab)."""
    f = _lib2().orc_synthe_hprof_kp
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 8
    return f(ctypes.byref(htab), n, m, xne, t, xnfph1, xnfph2, xnfhe1, xnfh2, dopph, delw)


def synthe_hprof_stehle(htab, stehle, n, m, xne, t, xnfph1, xnfph2, xnfhe1, xnfh2, dopph_conv, dopph, delw):
    """hydrogen_line_profile on the Stehle path at one depth (the analytic one where no series covers the
    line): the convolution built with dopph_conv, evaluated with dopph.  stehle: 4 series dicts."""
    st, keep = stehle_structs(stehle)
    f = _lib2().orc_synthe_hprof_stehle
    f.restype = ctypes.c_double
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 9
    return f(ctypes.byref(htab), st, n, m, xne, t, xnfph1, xnfph2, xnfhe1, xnfh2, dopph_conv, dopph, delw)


def synthe_hydrogen_opacity(recs, length, wbegin, ratio, wlend, velshift_kms, continuum, atm, htab, stehle=None):
    """compute_line_opacity's hydrogen and deuterium lines in FP64: the contribution [nrhox, length].
    atm: xnfdop, dopple [nrhox, nspec], xne, hckt, t, xnfph1, xnfph2, xnfhe1, xnfh2 [nrhox]; htab: HTab of
    SYNTHE's tables; stehle: 4 series dicts (None entries: not loaded) or None for the K-P path."""
    rec = np.ascontiguousarray(recs, NLTE_LINE)
    cont = np.ascontiguousarray(continuum, np.float32)
    xnfdop, dopple = _d(atm["xnfdop"]), _d(atm["dopple"])
    nrhox, nspec = xnfdop.shape
    hv = [_d(atm[k]) for k in ("t", "xnfph1", "xnfph2", "xnfhe1", "xnfh2")]
    sa = _SHAtm(*[_ptr(v) for v in hv])
    st, keep = (None, None) if stehle is None else stehle_structs(stehle)
    out = np.zeros((nrhox, length))
    f = _lib2().orc_synthe_hydrogen_opacity
    f.restype = ctypes.c_int
    rc = f(rec.ctypes.data_as(ctypes.c_void_p), ctypes.c_int64(rec.shape[0]), length, nrhox, ctypes.c_double(wbegin),
           ctypes.c_double(ratio), ctypes.c_double(wlend), ctypes.c_double(velshift_kms),
           cont.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _ptr(xnfdop), _ptr(dopple), nspec,
           _ptr(_d(atm["xne"])), _ptr(_d(atm["hckt"])), ctypes.byref(htab), st, ctypes.byref(sa), _ptr(out))
    if rc != 0:
        raise ValueError("hydrogen record NBLO/NBUP/NCON outside EHYD/ALPHAHYD/CONTH")
    return out


# ---------------------------------------------------------------- KAPP (hydrogen sources)
KAPP_NAMES = ("ahyd", "shyd", "ah2p", "ahmin", "shmin", "sigh", "sigel", "acont", "scont", "sigmac")
KAPP_NAMES_HE = KAPP_NAMES + ("ahe1", "ahe2", "ahemin", "sighe")
KAPP_NAMES_H2 = KAPP_NAMES_HE + ("ah2min", "ah2coll", "sigh2")
_KAPP_HE_TABLES = ("he1_chi", "he1_freq", "he1_g", "he_x505", "he_x50", "he_x20", "he_x10", "he2s1s_f", "he2s1s_x",
                   "he2s3s_f", "he2s3s_x", "he2p1p_f", "he2p1p_x", "he2p3p_f", "he2p3p_x", "hem_w", "hem_t", "hem_k",
                   "gf_lyman", "gf_balmer", "gf_paschen", "gf_brackett", "stark_knm", "stark_f")


class KappTables(ctypes.Structure):
    """orc_kapp_tables; keeps its arrays alive (built by kapp_tables)."""
    _fields_ = [(k, _fp) for k in ("freqn", "xn", "xl", "ekarzas")] + \
               [(k, _dp) for k in ("gff_logtab", "q_holtsmark", "hop_elev", "hmin_wbf", "hmin_bf", "hmin_thetaff",
                                   "hmin_wavek", "hmin_ff", "h2p_fr", "h2p_es", "ray_m", "ray_ab", "ray_bc", "ray_cd",
                                   "ray_ly", "ray_fly") + _KAPP_HE_TABLES]


class KappH2Tables(ctypes.Structure):
    """orc_kapp_h2_tables; keeps its arrays alive (built by kapp_h2_tables)."""
    _ip = ctypes.POINTER(ctypes.c_int)
    _fields_ = [("h2m_w", _dp), ("h2m_t", _dp), ("h2m_k", _dp), ("pf_n", ctypes.c_int), ("pf_tstart", ctypes.c_double),
                ("pf_tstep", ctypes.c_double), ("pf", _dp), ("cia_nnu", ctypes.c_int), ("cia_ntmax", ctypes.c_int),
                ("cia_nt", _ip), ("use_pair", _ip), ("cia_nu0", ctypes.c_double), ("cia_dnu", ctypes.c_double),
                ("cia_temp", _dp), ("cia_tab", _dp)]


def _lib_kapp():
    L = lib()
    if not getattr(L, "_kapp_declared", False):
        L.orc_log10_array.argtypes = [_dp, _dp, ctypes.c_int]
        L.orc_occupation_prob.argtypes = [ctypes.POINTER(KappTables), ctypes.c_int, ctypes.c_double]
        L.orc_occupation_prob.restype = ctypes.c_double
        L.orc_xkarzas.argtypes = [ctypes.POINTER(KappTables), ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                  ctypes.c_int]
        L.orc_xkarzas.restype = ctypes.c_double
        L.orc_kapp_hydrogen.argtypes = [ctypes.POINTER(KappTables), ctypes.c_double, ctypes.c_int] + [_dp] * 8
        L.orc_kapp.argtypes = [ctypes.POINTER(KappTables), ctypes.c_double, ctypes.c_int] + [_dp] * 12
        L.orc_crosshe.argtypes = [ctypes.POINTER(KappTables), ctypes.c_double]
        L.orc_crosshe.restype = ctypes.c_double
        L.orc_kapp_h2.argtypes = [ctypes.POINTER(KappTables), ctypes.POINTER(KappH2Tables), ctypes.c_double,
                                  ctypes.c_int] + [_dp] * 13
        L.orc_hlinop.argtypes = [ctypes.POINTER(KappTables), ctypes.c_void_p, ctypes.c_double, ctypes.c_int] + \
            [_dp] * 7
        L.orc_stark_mmm.argtypes = [ctypes.POINTER(KappTables), ctypes.c_void_p, ctypes.c_int, ctypes.c_int] + \
            [ctypes.c_double] * 3
        L.orc_stark_mmm.restype = ctypes.c_double
        for f in (L.orc_partfnh2, L.orc_equilh2):
            f.argtypes = [ctypes.POINTER(KappH2Tables), ctypes.c_double]
            f.restype = ctypes.c_double
        L._kapp_declared = True
    return L


def kapp_tables(tables):
    """KappTables from the k_* entries of the reference tables (GFF as its
    reader stores it: log10 by the C library)."""
    L = _lib_kapp()
    keep = {}
    for k in ("freqn", "xn", "xl", "ekarzas"):
        keep[k] = np.ascontiguousarray(tables["k_" + k], np.float32)
    gff = _d(tables["k_gff"])
    keep["gff_logtab"] = np.empty_like(gff)
    L.orc_log10_array(_ptr(gff), _ptr(keep["gff_logtab"]), gff.size)
    for k in ("q_holtsmark", "hop_elev", "hmin_wbf", "hmin_bf", "hmin_thetaff", "hmin_wavek", "hmin_ff", "h2p_fr",
              "h2p_es", "ray_m", "ray_ab", "ray_bc", "ray_cd", "ray_ly", "ray_fly") + _KAPP_HE_TABLES:
        keep[k] = _d(tables["k_" + k])
    kt = KappTables(*[_ptr(keep[n], _fp if t is _fp else _dp) for n, t in KappTables._fields_])
    kt._keep = keep
    return kt


def kapp_hydrogen(kt, wave, t, xne, rho, xnfp1, xnfp2, bhyd=None, bmin=None):
    """KAPP's hydrogen sources and totals at one wavelength (nm): dict of [nrhox] arrays (KAPP_NAMES)."""
    L = _lib_kapp()
    nr = len(t)
    out = np.zeros((len(KAPP_NAMES), nr))
    v = [_d(a) for a in (t, xne, rho, xnfp1, xnfp2)]
    bh = None if bhyd is None else _d(bhyd)
    bm = None if bmin is None else _d(bmin)
    L.orc_kapp_hydrogen(ctypes.byref(kt), float(wave), nr, *[_ptr(a) for a in v],
                        _ptr(bh) if bh is not None else None, _ptr(bm) if bm is not None else None, _ptr(out))
    return dict(zip(KAPP_NAMES, out))


def kapp(kt, wave, t, xne, rho, xnfp1, xnfp2, xnfp3, xnfp4, xnfp5, xnf4, bhyd=None, bmin=None):
    """KAPP's hydrogen and helium sources and totals at one wavelength (nm):
    dict of [nrhox] arrays (KAPP_NAMES_HE)."""
    L = _lib_kapp()
    nr = len(t)
    out = np.zeros((len(KAPP_NAMES_HE), nr))
    v = [_d(a) for a in (t, xne, rho, xnfp1, xnfp2, xnfp3, xnfp4, xnfp5, xnf4)]
    bh = None if bhyd is None else _d(bhyd)
    bm = None if bmin is None else _d(bmin)
    L.orc_kapp(ctypes.byref(kt), float(wave), nr, *[_ptr(a) for a in v],
               _ptr(bh) if bh is not None else None, _ptr(bm) if bm is not None else None, _ptr(out))
    return dict(zip(KAPP_NAMES_HE, out))


def kapp_h2_tables(tables, use_pair=(1, 1, 1, 1)):
    """KappH2Tables from the k_h2m_*, k_pf_h2*, k_cia_* entries of the reference tables."""
    _lib_kapp()
    keep = dict(h2m_w=_d(tables["k_h2m_w"]), h2m_t=_d(tables["k_h2m_t"]), h2m_k=_d(tables["k_h2m_k"]),
                pf=_d(tables["k_pf_h2"]), cia_temp=_d(tables["k_cia_temp"]), cia_tab=_d(tables["k_cia_tab"]),
                cia_nt=np.ascontiguousarray(tables["k_cia_nt"], np.int32),
                use_pair=np.ascontiguousarray(use_pair, np.int32))
    tpf = np.asarray(tables["k_pf_h2_t"], np.float64)
    grid = np.asarray(tables["k_cia_grid"], np.float64)
    assert 3 <= keep["pf"].size <= 512
    ip = ctypes.POINTER(ctypes.c_int)
    h = KappH2Tables(_ptr(keep["h2m_w"]), _ptr(keep["h2m_t"]), _ptr(keep["h2m_k"]), keep["pf"].size, float(tpf[0]),
                     float(tpf[1] - tpf[0]), _ptr(keep["pf"]), int(grid[0]), keep["cia_temp"].shape[1],
                     keep["cia_nt"].ctypes.data_as(ip), keep["use_pair"].ctypes.data_as(ip), float(grid[1]),
                     float(grid[2]), _ptr(keep["cia_temp"]), _ptr(keep["cia_tab"]))
    h._keep = keep
    return h


def kapp_h2(kt, h2, wave, t, xne, rho, xnfp1, xnfp2, xnfp3, xnfp4, xnfp5, xnf4, xnf3, bhyd=None, bmin=None):
    """KAPP's hydrogen, helium and H2 sources and totals at one wavelength
    (nm): dict of [nrhox] arrays (KAPP_NAMES_H2)."""
    L = _lib_kapp()
    nr = len(t)
    out = np.zeros((len(KAPP_NAMES_H2), nr))
    v = [_d(a) for a in (t, xne, rho, xnfp1, xnfp2, xnfp3, xnfp4, xnfp5, xnf4, xnf3)]
    bh = None if bhyd is None else _d(bhyd)
    bm = None if bmin is None else _d(bmin)
    L.orc_kapp_h2(ctypes.byref(kt), ctypes.byref(h2), float(wave), nr, *[_ptr(a) for a in v],
                  _ptr(bh) if bh is not None else None, _ptr(bm) if bm is not None else None, _ptr(out))
    return dict(zip(KAPP_NAMES_H2, out))


def hlinop(kt, wave, t, xne, rho, xnfp1, bhyd=None, stehle=None):
    """HLINOP at one wavelength (nm): (ahline, shline) [nrhox].  stehle: the
    ctypes array of stehle_structs, or None (STARK throughout)."""
    L = _lib_kapp()
    nr = len(t)
    ah, sh = np.zeros(nr), np.zeros(nr)
    v = [_d(a) for a in (t, xne, rho, xnfp1)]
    bh = None if bhyd is None else _d(bhyd)
    L.orc_hlinop(ctypes.byref(kt), None if stehle is None else ctypes.addressof(stehle), float(wave), nr,
                 *[_ptr(a) for a in v], _ptr(bh) if bh is not None else None, _ptr(ah), _ptr(sh))
    return ah, sh


def stark_mmm(kt, n, m, freq, t, xne, stehle=None):
    """STARK_MMM(N, M, J) at one (frequency, T, XNE)."""
    return _lib_kapp().orc_stark_mmm(ctypes.byref(kt), None if stehle is None else ctypes.addressof(stehle), n, m,
                                     float(freq), float(t), float(xne))


def partfnh2(h2, t):
    return _lib_kapp().orc_partfnh2(ctypes.byref(h2), float(t))


def equilh2(h2, t):
    return _lib_kapp().orc_equilh2(ctypes.byref(h2), float(t))


def crosshe(kt, freq):
    """CROSSHE(FREQ): He I ground-state cross-section (cm^2)."""
    return _lib_kapp().orc_crosshe(ctypes.byref(kt), float(freq))
