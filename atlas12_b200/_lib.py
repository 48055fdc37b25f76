"""ctypes binding of libatlasgpu.so (include/atlasgpu.h).

The library is built in-tree (atlas12_b200/libatlasgpu.so).  There is no CPU
fallback: if the library cannot be loaded every entry point raises.
"""
import atexit
import ctypes
import os
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# ATLASGPU_LIB selects another build of the same library (e.g. an instrumented one)
LIB_PATH = os.environ.get("ATLASGPU_LIB") or os.path.join(HERE, "libatlasgpu.so")

OK, EINVAL, ENOMEM, ECUDA, ETIMEOUT, ENONFINITE, ESTATE = 0, -1, -2, -3, -4, -5, -6
PREC_FP64, PREC_MIXED = 0, 1
NXTAU = 51


class AtlasGPUError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"atlasgpu status {code}: {msg}")
        self.code = code


class Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int), ("stream", ctypes.c_void_p)]


class Grid(ctypes.Structure):
    _fields_ = [("ratio", ctypes.c_double), ("ratiolg", ctypes.c_double), ("wbegin", ctypes.c_double),
                ("length", ctypes.c_int32), ("ixwlbeg", ctypes.c_int32)]


class Accum(ctypes.Structure):
    _fields_ = [(n, ctypes.POINTER(ctypes.c_double)) for n in
                ("rjmins", "rdabh", "rdiagj", "flxrad", "raden", "h_total", "accrad", "abross")] + \
               [("pradk0", ctypes.c_double)]


LTE_LINE = np.dtype([("nbuff", "<i4"), ("cgf", "<f4"), ("nelion", "<i4"), ("elo", "<f4"),
                     ("gamrf", "<f4"), ("gamsf", "<f4"), ("gamwf", "<f4"), ("code", "<f4")])
assert LTE_LINE.itemsize == 32
# unit-19 NLTE / complex-profile record (atlasgpu_nlte_line), 64 bytes
NLTE_LINE = np.dtype([("wlvac", "<f8"), ("elo", "<f4"), ("gf", "<f4"), ("nblo", "<i4"), ("nbup", "<i4"),
                      ("nelion", "<i4"), ("itype", "<i4"), ("ncon", "<i4"), ("nelionx", "<i4"), ("gammar", "<f4"),
                      ("gammas", "<f4"), ("gammaw", "<f4"), ("nbuff", "<i4"), ("lim", "<i4"), ("pad", "<i4")])
assert NLTE_LINE.itemsize == 64

_P = ctypes.c_void_p
_I = ctypes.c_int
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "atlasgpu_device_count": (_I, []),
    "atlasgpu_create": (_I, [ctypes.POINTER(_P), ctypes.POINTER(Opts)]),
    "atlasgpu_destroy": (_I, [_P]),
    "atlasgpu_last_error": (ctypes.c_char_p, [_P]),
    "atlasgpu_set_precision": (_I, [_P, _I]),
    "atlasgpu_set_stream": (_I, [_P, _P]),
    "atlasgpu_synchronize": (_I, [_P]),
    "atlasgpu_launch_count": (_I64, [_P]),
    "atlasgpu_enable_timing": (_I, [_P, _I]),
    "atlasgpu_kernel_ms": (_D, [_P, ctypes.c_char_p]),
    "atlasgpu_kernel_work": (_D, [_P, ctypes.c_char_p]),
    "atlasgpu_set_operators": (_I, [_P, _P, _P, _P, _P, _P]),
    "atlasgpu_synthe_grid": (_I, [_D, _D, _D, ctypes.POINTER(Grid)]),
    "atlasgpu_synthe_bin": (_I, [_P, _P, _I64, _D, _I32, _P]),
    "atlasgpu_synthe_bin_dev": (_I, [_P, _P, _I64, _D, _I32, _P, ctypes.POINTER(_I64)]),
    "atlasgpu_synthe_continuum": (_I, [_P, _P, _I, _P, _I, _I, _D, _D, _I, _P]),
    "atlasgpu_synthe_line_opacity": (_I, [_P, _P, _I64, _I, _I, _D, _P, _P, _P, _I, _P, _P, _P, _I, _P]),
    "atlasgpu_synthe_line_opacity_dev": (_I, [_P, _P, _I64, _I, _I, _D, _P, _P, _P, _I, _P, _P, _P, _I, _P]),
    "atlasgpu_synthe_spectrum": (_I, [_P, _P, _I, _P, _P, _I, _I, _P, _P, _D, _D, _I, _P, _P, _P]),
    "atlasgpu_synthe_spectrum_dev": (_I, [_P, _P, _I, _P, _P, _I, _I, _P, _P, _D, _D, _I, _P, _P, _P]),
    "atlasgpu_atlas_set_voigt_tables": (_I, [_P, _P, _P, _P, _I]),
    "atlasgpu_atlas_tabvoigt": (_I, [_D, _I, _P, _P, _I, _P, _P, _P]),
    "atlasgpu_atlas_linop": (_I, [_P, _P, _I64, _I, _I, _P, _P, _I, _P, _P, _P, _P, _P, _I, _P, _I, _P,
                                  ctypes.POINTER(_I64)]),
    "atlasgpu_synthe_nlte_opacity": (_I, [_P, _P, _I64, _I, _I, _D, _D, _D, _D, _P, _P, _P, _P, _I, _P, _P, _P,
                                          _P, _P, _P]),
    "atlasgpu_synthe_set_hydrogen_tables": (_I, [_P, _P, _P]),
    "atlasgpu_atlas_xlinop": (_I, [_P, _P, _I64, _I, _I, _P, _P, _I, _P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _P,
                                   _P, _P, ctypes.POINTER(_I64)]),
    "atlasgpu_atlas_set_hydrogen_tables": (_I, [_P, _P]),
    "atlasgpu_atlas_set_kapp_tables": (_I, [_P, _P]),
    "atlasgpu_atlas_kapp_hydrogen": (_I, [_P, _I, _P, _I, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P]),
    "atlasgpu_atlas_kapp": (_I, [_P, _I, _P, _I, _I, _P, _P, _P, _P, _P]),
    "atlasgpu_atlas_set_kapp_h2_tables": (_I, [_P, _P]),
    "atlasgpu_atlas_set_stehle_tables": (_I, [_P, _P]),
    "atlasgpu_atlas_hlinop": (_I, [_P, _I, _P, _I, _I, _P, _P, _P, _P, _P, _P, _P]),
    "atlasgpu_atlas_rt_pass": (_I, [_P, _I, _P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _P, _D,
                                    ctypes.POINTER(Accum), _P]),
    "atlasgpu_atlas_finish": (_I, [_P, ctypes.c_void_p, ctypes.POINTER(Accum), ctypes.POINTER(_D)]),
    "atlasgpu_model_create": (_I, [_P, ctypes.c_void_p, ctypes.POINTER(_P)]),
    "atlasgpu_model_iterate": (_I, [_P, _P, _I, _D, _I, ctypes.POINTER(_I), _P]),
    "atlasgpu_model_get": (_I, [_P, _P, _P, _P, _P, _P, _P, _P]),
    "atlasgpu_model_get_tables": (_I, [_P, _P, _P, _P, _P, _P]),
    "atlasgpu_model_set_structure": (_I, [_P, _P, _P, _P, _P]),
    "atlasgpu_model_destroy": (_I, [_P, _P]),
    "atlasgpu_model_set_params": (_I, [_P, _P, _D, _D, _D, _D]),
    "atlasgpu_model_set_shard": (_I, [_P, _P, _I, _I]),
    "atlasgpu_model_set_sums_buffer": (_I, [_P, _P, _P]),
    "atlasgpu_model_iterate_begin": (_I, [_P, _P]),
    "atlasgpu_model_iterate_end": (_I, [_P, _P, ctypes.POINTER(_D)]),
    "atlasgpu_surrogate_eval": (_I, [_P, _I, _P, _P, _D, _I, _P, _P, _P, _P, _P]),
    "atlasgpu_fp64_peak_tflops": (_D, [_P]),
    "atlasgpu_u64_atomic_peak": (_D, [_P]),
    "atlasgpu_mlp_create": (_I, [_P, _I, _I, _I, _I, ctypes.c_uint64, ctypes.POINTER(_P)]),
    "atlasgpu_mlp_destroy": (_I, [_P, _P]),
    "atlasgpu_mlp_nparam": (_I64, [_P]),
    "atlasgpu_mlp_get_params": (_I, [_P, _P, _P]),
    "atlasgpu_mlp_set_params": (_I, [_P, _P, _P]),
    "atlasgpu_mlp_forward": (_I, [_P, _P, _P, _I, _P]),
    "atlasgpu_mlp_loss_grad": (_I, [_P, _P, _P, _P, _I, _P, _P]),
    "atlasgpu_mlp_train": (_I, [_P, _P, _P, _P, _I, _I, _I, ctypes.c_float, ctypes.c_uint64, _P]),
    "atlasgpu_atlas_rt_pass_noalloc": (_I, [_P, _I, _P, _P, _P, _P, _P, _I, _P, _I, _P, _P, _P, _D, _P, _P]),
    "atlasgpu_batch_create": (_I, [_P, ctypes.c_void_p, _I, ctypes.POINTER(_P)]),
    "atlasgpu_batch_load": (_I, [_P, _P, _I, _D, _D, _D, _D, _P, _P, _P, _I, _D]),
    "atlasgpu_batch_step": (_I, [_P, _P, _I]),
    "atlasgpu_batch_poll": (_I, [_P, _P, _P, _P, _P, ctypes.POINTER(_I)]),
    "atlasgpu_batch_run": (_I, [_P, _P, _I, _P, _P, _P]),
    "atlasgpu_batch_get": (_I, [_P, _P, _I, _P, _P, _P, _P, _P, _P, _P]),
    "atlasgpu_batch_nslots": (_I, [_P]),
    "atlasgpu_batch_set_shape": (_I, [_P, _P, _I, _I]),
    "atlasgpu_batch_get_shape": (_I, [_P, _P, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "atlasgpu_batch_destroy": (_I, [_P, _P]),
    "atlasgpu_atlas_select_tables": (_I, [_P, _I, _I, _P, _I, _P, _P, _P, _P, _I]),
    "atlasgpu_atlas_selectlines": (_I, [_P, _I, _P, _I64, ctypes.c_void_p, _P, _I64, ctypes.POINTER(_I64)]),
    "atlasgpu_atlas_selectlines_dev": (_I, [_P, _I, _P, _I64, ctypes.c_void_p, _P, _I64, ctypes.POINTER(_I64)]),
}

SLOT_IDLE, SLOT_RUNNING, SLOT_CONVERGED, SLOT_NONFINITE, SLOT_CAPPED = 0, 1, 2, 3, 4

# SELECTLINES database kinds (ATLASGPU_SEL_*) and their record formats
SEL_LOWPRED, SEL_LOWOBS, SEL_HI, SEL_DIATOMIC, SEL_TIO, SEL_H2O, SEL_H3PLUS = range(1, 8)
MOL2_REC = np.dtype([("wl", "<f4"), ("gflog", "<f4"), ("e1", "<f4"), ("e2", "<f4"), ("code", "<i4"),
                     ("iso", "<i4"), ("gr", "<i4"), ("label", "<i4")])
assert MOL2_REC.itemsize == 32
H2O_REC = np.dtype([("iwl", "<i4"), ("ielo", "<i2"), ("igflog", "<i2")])
assert H2O_REC.itemsize == 8


class HydrogenTables(ctypes.Structure):
    """atlasgpu_hydrogen_tables (include/atlasgpu.h): HPROF4's and STARK_PROFILE's
    tables and XLINOP's hydrogen level energies."""
    _fields_ = [("xknmtb", _D * 12), ("y1wtm", _D * 4), ("stalph", _D * 34), ("stwtal", _D * 34),
                ("istal", ctypes.c_int32 * 4), ("lnghal", ctypes.c_int32 * 4), ("stcomp", _D * 20),
                ("stcpwt", _D * 20), ("lncomp", ctypes.c_int32 * 4), ("cutoffh2plus", _D * 111),
                ("cutoffh2", _D * 91), ("asum", _D * 100), ("asumlyman", _D * 100), ("betagrid", _D * 15),
                ("pp", _D * 5), ("propbm", _D * 525), ("c", _D * 35), ("d", _D * 35), ("eh", _D * 10), ("elim", _D)]

    @classmethod
    def from_tables(cls, t, prefix="h_"):
        """From arrays named <prefix><field> (first index slowest, as the header
        lays them out): "h_" ATLAS12's HPROF4 tables, "s_" SYNTHE's own."""
        h = cls()
        for name, typ in cls._fields_:
            v = np.asarray(t[prefix + name]).ravel()
            if name == "elim":
                h.elim = float(v[0])
            elif name in ("istal", "lnghal", "lncomp"):
                getattr(h, name)[:] = [int(x) for x in v]
            else:
                getattr(h, name)[:] = [float(x) for x in v]
        return h


class KappTables(ctypes.Structure):
    """atlasgpu_kapp_tables (include/atlasgpu.h): KAPP's hydrogen continuum
    tables (Karzas-Latter, van Hoof g_ff, Holtsmark Q, HOP's level energies,
    HMINOP's, H2PLOP's and HRAYOP's tables) and the helium ones (HE1OP's
    levels, CROSSHE, the 2s/2p fits, HEMIOP's table)."""
    _F = ctypes.c_float
    _fields_ = [("freqn", _F * 435), ("xn", _F * 435), ("xl", _F * 1044), ("ekarzas", _F * 29),
                ("gff", _D * 11826), ("q_holtsmark", _D * 150), ("hop_elev", _D * 15), ("hmin_wbf", _D * 116),
                ("hmin_bf", _D * 116), ("hmin_thetaff", _D * 11), ("hmin_wavek", _D * 22), ("hmin_ff", _D * 242),
                ("h2p_fr", _D * 5), ("h2p_es", _D * 6), ("ray_m", _D * 74), ("ray_ab", _D * 27), ("ray_bc", _D * 24),
                ("ray_cd", _D * 22), ("ray_ly", _D * 64), ("ray_fly", _D * 64),
                ("he1_chi", _D * 10), ("he1_freq", _D * 10), ("he1_g", _D * 10), ("he_x505", _D * 92),
                ("he_x50", _D * 16), ("he_x20", _D * 11), ("he_x10", _D * 21)] + \
        [(k, _D * 16) for k in ("he2s1s_f", "he2s1s_x", "he2s3s_f", "he2s3s_x", "he2p1p_f", "he2p1p_x",
                                "he2p3p_f", "he2p3p_x")] + \
        [("hem_w", _D * 17), ("hem_t", _D * 12), ("hem_k", _D * 204), ("gf_lyman", _D * 29),
         ("gf_balmer", _D * 28), ("gf_paschen", _D * 27), ("gf_brackett", _D * 3), ("stark_knm", _D * 20),
         ("stark_f", _D * 40)]

    @classmethod
    def from_tables(cls, t):
        """From the arrays k_<field> of the reference tables, each flattened in
        Fortran (column-major) order, which is the header's layout."""
        k = cls()
        for name, typ in cls._fields_:
            v = np.asarray(t["k_" + name]).ravel()
            arr = getattr(k, name)
            if len(arr) != v.size:
                raise ValueError(f"kapp table {name}: {v.size} values, expected {len(arr)}")
            arr[:] = [float(x) for x in v]
        return k


class KappPops(ctypes.Structure):
    """atlasgpu_kapp_pops: the depth vectors of atlasgpu_atlas_kapp (addresses)."""
    _fields_ = [(k, ctypes.c_void_p) for k in ("t", "xne", "rho", "xnfp_h1", "xnfp_h2", "xnfp_he1", "xnfp_he2",
                                               "xnfp_he3", "xnf_he2", "bhyd", "bmin", "xnf_he1")]


class KappH2Tables(ctypes.Structure):
    """atlasgpu_kapp_h2_tables: H2MINOP's table, PARTFNH2's values, H2COLLOP's
    CIA grid (the two large arrays by address; from_tables keeps them alive)."""
    _I32 = ctypes.c_int32
    _fields_ = [("h2m_w", _D * 10), ("h2m_t", _D * 7), ("h2m_k", _D * 70), ("pf_n", _I32), ("pf_tstart", _D),
                ("pf_tstep", _D), ("pf", ctypes.c_void_p), ("cia_nnu", _I32), ("cia_ntmax", _I32),
                ("cia_nt", _I32 * 4), ("use_pair", _I32 * 4), ("cia_nu0", _D), ("cia_dnu", _D),
                ("cia_temp", ctypes.c_void_p), ("cia_tab", ctypes.c_void_p)]

    @classmethod
    def from_tables(cls, t, use_pair=(1, 1, 1, 1)):
        """From the k_h2m_*, k_pf_h2*, k_cia_* arrays of the reference tables."""
        k = cls()
        k.h2m_w[:] = [float(x) for x in np.asarray(t["k_h2m_w"]).ravel()]
        k.h2m_t[:] = [float(x) for x in np.asarray(t["k_h2m_t"]).ravel()]
        k.h2m_k[:] = [float(x) for x in np.asarray(t["k_h2m_k"]).ravel()]
        pf = np.ascontiguousarray(t["k_pf_h2"], np.float64)
        tpf = np.asarray(t["k_pf_h2_t"], np.float64)
        temp = np.ascontiguousarray(t["k_cia_temp"], np.float64)
        tab = np.ascontiguousarray(t["k_cia_tab"], np.float64)
        grid = np.asarray(t["k_cia_grid"], np.float64)
        k.pf_n, k.pf_tstart, k.pf_tstep, k.pf = pf.size, float(tpf[0]), float(tpf[1] - tpf[0]), pf.ctypes.data
        k.cia_nnu, k.cia_ntmax = int(grid[0]), temp.shape[1]
        k.cia_nt[:] = [int(x) for x in np.asarray(t["k_cia_nt"]).ravel()]
        k.use_pair[:] = [int(bool(x)) for x in use_pair]
        k.cia_nu0, k.cia_dnu = float(grid[1]), float(grid[2])
        k.cia_temp, k.cia_tab = temp.ctypes.data, tab.ctypes.data
        k._keep = (pf, temp, tab)
        return k


class StehleSeries(ctypes.Structure):
    """atlasgpu_stehle_series: one Stehle Stark-profile series (n_dens 0: not loaded)."""
    _fields_ = [("n_lower", ctypes.c_int32), ("n_upper_min", ctypes.c_int32), ("n_upper_max", ctypes.c_int32),
                ("n_dens", ctypes.c_int32), ("density_grid", _D * 20), ("temp_grid", _D * 10),
                ("log_dalpha_grid", _D * 60), ("max_dens_idx", ctypes.c_void_p), ("k_alpha", ctypes.c_void_p),
                ("profiles", ctypes.c_void_p)]


def stehle_array(stehle):
    """(StehleSeries * 4) from 4 dicts as read_stehle / synthetic.stehle_tables
    give them (None entries: not loaded), and the arrays it points into (keep
    both alive while the library reads them)."""
    st, keep = (StehleSeries * 4)(), []
    for q, ser in enumerate(stehle):
        if ser is None:
            continue
        arrs = [np.ascontiguousarray(ser["max_dens_idx"], np.int32), np.ascontiguousarray(ser["k_alpha"], np.float64),
                np.ascontiguousarray(ser["profiles"], np.float64)]
        keep += arrs
        a = st[q]
        a.n_lower, a.n_upper_min, a.n_upper_max = (int(ser[k]) for k in ("n_lower", "n_upper_min", "n_upper_max"))
        a.n_dens = len(ser["density_grid"])
        a.density_grid[:a.n_dens] = [float(x) for x in ser["density_grid"]]
        a.temp_grid[:] = [float(x) for x in ser["temp_grid"]]
        a.log_dalpha_grid[:] = [float(x) for x in ser["log_dalpha_grid"]]
        a.max_dens_idx, a.k_alpha, a.profiles = (v.ctypes.data for v in arrs)
    return st, keep


class SyntheHydrogen(ctypes.Structure):
    """atlasgpu_synthe_hydrogen: T, XNFPH(J,1), XNFPH(J,2), XNFHE(J,1), XNFH2 [nrhox]."""
    _fields_ = [("t", ctypes.c_void_p), ("xnfph1", ctypes.c_void_p), ("xnfph2", ctypes.c_void_p),
                ("xnfhe1", ctypes.c_void_p), ("xnfh2", ctypes.c_void_p)]


class XlinopHydrogen(ctypes.Structure):
    """atlasgpu_xlinop_hydrogen: T, XNF(J,1), XNF(J,2), XNH2 [nrhox]."""
    _fields_ = [("t", ctypes.c_void_p), ("xnf1", ctypes.c_void_p), ("xnf2", ctypes.c_void_p),
                ("xnh2", ctypes.c_void_p)]


class SelectState(ctypes.Structure):
    """atlasgpu_select_state (include/atlasgpu.h)."""
    _fields_ = [("nu", ctypes.c_int32), ("igr", ctypes.c_int32), ("freq", ctypes.c_double)]
BATCH_MAX_ITER = 256

_DP = ctypes.POINTER(ctypes.c_double)


class FinishState(ctypes.Structure):
    """atlasgpu_finish_state (include/atlasgpu.h)."""
    _fields_ = [("nrhox", _I), ("iter", _I), ("teff", _D), ("grav", _D), ("pradk0", _D)] + \
               [(n, _DP) for n in ("t", "rhox", "p", "xne", "abross", "prad", "vturb", "pturb", "tauros",
                                   "accrad", "raden", "oldt1", "flxerr", "dtflux", "dtlamb", "dtsurf", "t1")] + \
               [("ross_n", _I), ("ross_max", _I), ("ross_zerot", _D), ("ross_slopet", _D), ("ross_zerop", _D),
                ("ross_slopep", _D), ("ross_t", _DP), ("ross_p", _DP), ("ross_k", _DP)]


class ModelDesc(ctypes.Structure):
    """atlasgpu_model_desc (include/atlasgpu.h)."""
    _fields_ = [("teff", _D), ("logg", _D), ("vturb_kms", _D), ("nrhox", _I),
                ("t", _DP), ("p", _DP), ("rhox", _DP), ("tauros", _DP),
                ("waveset", _DP), ("rcoset", _DP), ("numnu", _I),
                ("cutoff_wave", _DP), ("nwave", _I),
                ("linedata", ctypes.POINTER(ctypes.c_int32)), ("nlines", _I64),
                ("h0tab", _DP), ("h1tab", _DP), ("h2tab", _DP), ("mh", _D)]

_lib = None


def lib():
    """Load libatlasgpu.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise AtlasGPUError(ESTATE, f"{LIB_PATH} not built (run __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name, None)
            if f is None:
                continue
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    L = lib()
    return {n for n in SIGNATURES if hasattr(L, n)}


def ptr(a):
    """Data pointer of a numpy array (contiguous) or a torch tensor."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return ctypes.c_void_p(a.data_ptr())
    assert a.flags["C_CONTIGUOUS"], "arrays must be C-contiguous"
    return ctypes.c_void_p(a.ctypes.data)


def device_count():
    return int(lib().atlasgpu_device_count())


_live = weakref.WeakSet()


@atexit.register
def _close_all():
    # release device memory before the interpreter (and the CUDA runtime) shut down
    for c in list(_live):
        try:
            c.close()
        except Exception:
            pass


class Context:
    """Owns one atlasgpu_ctx (one CUDA stream on one device)."""

    def __init__(self, device=0, precision=PREC_MIXED, stream=None):
        self._h = _P()
        o = Opts(device, precision, stream)
        rc = lib().atlasgpu_create(ctypes.byref(self._h), ctypes.byref(o))
        if rc != OK:
            raise AtlasGPUError(rc, "atlasgpu_create failed (device %d)" % device)
        self.device = device
        _live.add(self)

    @property
    def handle(self):
        return self._h

    def check(self, rc):
        if rc != OK:
            raise AtlasGPUError(rc, lib().atlasgpu_last_error(self._h).decode())
        return rc

    def call(self, name, *args):
        return self.check(getattr(lib(), name)(self._h, *args))

    def close(self):
        if self._h:
            lib().atlasgpu_destroy(self._h)
            self._h = _P()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_precision(self, p):
        self.call("atlasgpu_set_precision", int(p))

    def set_stream(self, stream):
        self.call("atlasgpu_set_stream", stream)

    def synchronize(self):
        self.call("atlasgpu_synchronize")

    def launches(self):
        return int(lib().atlasgpu_launch_count(self._h))

    def enable_timing(self, on=True):
        self.call("atlasgpu_enable_timing", 1 if on else 0)

    def kernel_ms(self, name):
        return float(lib().atlasgpu_kernel_ms(self._h, name.encode()))

    def kernel_work(self, name):
        """Work units the last timed launch of `name` counted (-1 if none)."""
        return float(lib().atlasgpu_kernel_work(self._h, name.encode()))

    def set_operators(self, xtau8, coefj, coefh, ch_j, ck_j):
        """coefj/coefh as 2-D arrays COEF[L-1, M-1]; passed column-major."""
        self._ops = [np.ascontiguousarray(xtau8, np.float64),
                     np.ascontiguousarray(np.asarray(coefj, np.float64).ravel(order="F")),
                     np.ascontiguousarray(np.asarray(coefh, np.float64).ravel(order="F")),
                     np.ascontiguousarray(ch_j, np.float64), np.ascontiguousarray(ck_j, np.float64)]
        self.call("atlasgpu_set_operators", *[ptr(a) for a in self._ops])
