"""SELECTLINES (atlas12_modules.f90:19171-19781): the line databases filtered
into LINEDATA on the device, and readers for their binary record formats.

The reference opens each database with ACCESS='STREAM' (little endian):

  LINEREC   [4] int32: IWL | IELION, IELO int16 | IGFLOG, IGR int16 | IGS, IGW
            int16 (UNPACK_LINEDATA, :1950-1963) -- gfpred29dec2014.bin,
            lowobsat12.bin, hilines.bin, h3plus.dat
  MOL2      one header record (int32 magic 'MOL2', int32 count, 6 more int32)
            then 32-byte records: real32 wavelength (nm), log gf, E, E';
            int32 molecule, isotope, 100*log10(gamma_r), label (:19531-19575)
  H2O       8-byte records: int32 IWL, INTEGER(2) IELO, IGFLOG (READ(51) IWL,
            IELO, IGFLOG with the module's INTEGER(2) IELO / IGFLOG, :1373-1374,
            :19664)

The diatomic lists are ASCII files the reference reads, sorts and packs on
the host (read_diatomics_for_atlas, :19427-19475); `select` takes their
packed LINEREC records (kind SEL_DIATOMIC, IGFLOG before the isotopologue
correction).
"""
import os

import numpy as np

from . import _lib
from ._lib import Context, ptr, SEL_LOWPRED, SEL_LOWOBS, SEL_HI, SEL_DIATOMIC, SEL_TIO, SEL_H2O, SEL_H3PLUS

MOL2_MAGIC = 0x4D4F4C32
CLIGHT_NMS = 2.99792458e17
LINEREC_KINDS = (SEL_LOWPRED, SEL_LOWOBS, SEL_HI, SEL_DIATOMIC, SEL_H3PLUS)
# the reference's database order and file names (:19262-19767); TiO's path comes from lines.list
DATABASES = [(SEL_LOWPRED, "gfpred29dec2014.bin"), (SEL_LOWOBS, "lowobsat12.bin"), (SEL_HI, "hilines.bin"),
             (SEL_DIATOMIC, None), (SEL_TIO, None), (SEL_H2O, "h2opokazatel.bin"), (SEL_H3PLUS, "h3plus.dat")]
TEFF_COOL_LIMIT = 8000.0  # TiO and H2O are skipped above it (:19553, :19655)


def read_linerec(path):
    """LINEREC records of a LINEDATA-format database as int32 [n, 4] (memory-mapped)."""
    n = os.path.getsize(path) // 16
    return np.memmap(path, dtype="<i4", mode="r", shape=(n, 4)) if n else np.zeros((0, 4), np.int32)


def read_mol2(path):
    """The records of a MOL2 list after its header (magic 'MOL2', count), memory-mapped."""
    hdr = np.fromfile(path, dtype="<i4", count=8)
    if hdr.size < 8 or int(hdr[0]) != MOL2_MAGIC:
        raise ValueError(f"not a MOL2 binary line list: {path}")
    n = int(hdr[1])
    avail = (os.path.getsize(path) - 32) // 32
    # the reference stops at the first short read
    return np.memmap(path, dtype=_lib.MOL2_REC, mode="r", offset=32, shape=(min(n, avail),))


def read_h2o(path):
    """8-byte H2O records (IWL, IELO, IGFLOG), memory-mapped."""
    n = os.path.getsize(path) // 8
    return np.memmap(path, dtype=_lib.H2O_REC, mode="r", shape=(n,))


def write_mol2(path, recs):
    hdr = np.zeros(8, "<i4")
    hdr[0], hdr[1] = MOL2_MAGIC, len(recs)
    with open(path, "wb") as f:
        f.write(hdr.tobytes())
        f.write(np.ascontiguousarray(recs, _lib.MOL2_REC).tobytes())


def initial_state(wavetab, igr=0):
    """The module variables at SELECTLINES's entry: NU = 1, FREQ as KAPCONT
    (called just before it, atlas12c.f90:562-563) leaves it, IGR as given."""
    return {"nu": 1, "freq": CLIGHT_NMS / float(wavetab[-1]), "igr": int(igr)}


class SelectLines:
    """SELECTLINES's tables on one context and its database loops.

    xnfdop [nspec, kw] (XNFDOP(J, NELION)), hckt [nrhox], tabcont [nwave+1, kw],
    iwavetab [nwave+1] (sentinel last), wavetab [nwave] (nm)."""

    def __init__(self, ctx: Context, nrhox, xnfdop, hckt, tabcont, iwavetab, wavetab):
        self.ctx = ctx
        xnfdop = np.ascontiguousarray(xnfdop, np.float64)
        tabcont = np.ascontiguousarray(tabcont, np.float64)
        self.wavetab = np.ascontiguousarray(wavetab, np.float64)
        iw = np.ascontiguousarray(iwavetab, np.int32)
        hckt = np.ascontiguousarray(hckt, np.float64)
        nspec, kw = xnfdop.shape
        if tabcont.shape != (self.wavetab.size + 1, kw) or iw.size != self.wavetab.size + 1:
            raise ValueError("tabcont [nwave+1, kw] and iwavetab [nwave+1] must match wavetab [nwave]")
        self.nspec = nspec
        ctx.call("atlasgpu_atlas_select_tables", int(nrhox), kw, ptr(xnfdop), nspec, ptr(hckt), ptr(tabcont),
                 ptr(iw), ptr(self.wavetab), self.wavetab.size)

    @staticmethod
    def _records(kind, recs):
        if kind in LINEREC_KINDS:
            recs = np.ascontiguousarray(recs, np.int32)
            if recs.ndim != 2 or recs.shape[1] != 4:
                raise ValueError("LINEREC records are int32 [n, 4]")
            return recs
        dt = _lib.MOL2_REC if kind == SEL_TIO else _lib.H2O_REC if kind == SEL_H2O else None
        if dt is None:
            raise ValueError(f"unknown database kind {kind}")
        recs = np.ascontiguousarray(recs)
        if recs.dtype != dt:
            raise ValueError(f"records of kind {kind} must have dtype {dt}")
        return recs

    @staticmethod
    def _state(state):
        return _lib.SelectState(int(state["nu"]), int(state["igr"]), float(state["freq"]))

    def select(self, kind, recs, state, cap=None):
        """One database loop over host records (file order).  state (dict nu,
        freq, igr) is updated in place.  Returns LINEDATA [m, 4] int32."""
        recs = self._records(kind, recs)
        n = recs.shape[0]
        cap = n if cap is None else int(cap)
        out = np.empty((max(cap, 1), 4), np.int32)
        st = self._state(state)
        nout = _lib.ctypes.c_int64(0)
        self.ctx.call("atlasgpu_atlas_selectlines", int(kind), ptr(recs) if n else None, n,
                      _lib.ctypes.byref(st), ptr(out), cap, _lib.ctypes.byref(nout))
        state.update(nu=st.nu, freq=st.freq, igr=st.igr)
        return out[:nout.value].copy()

    def select_dev(self, kind, d_recs, n, state, d_out, cap):
        """The same on device buffers (torch tensors or raw pointers); returns the count."""
        st = self._state(state)
        nout = _lib.ctypes.c_int64(0)
        p_in = d_recs.data_ptr() if hasattr(d_recs, "data_ptr") else d_recs
        p_out = d_out.data_ptr() if hasattr(d_out, "data_ptr") else d_out
        self.ctx.call("atlasgpu_atlas_selectlines_dev", int(kind), p_in, int(n), _lib.ctypes.byref(st), p_out,
                      int(cap), _lib.ctypes.byref(nout))
        state.update(nu=st.nu, freq=st.freq, igr=st.igr)
        return int(nout.value)

    def select_all(self, databases, teff, state=None):
        """SELECTLINES's driver order over {kind: records}: NU restarts at 1 for
        every database but the observed low lines, which continue from the
        predicted ones (:19270-19330); FREQ and IGR carry through; TiO and H2O
        are skipped above Teff 8000 K.  Returns (LINEDATA, {kind: count}, the
        state the last loop leaves)."""
        state = dict(initial_state(self.wavetab)) if state is None else dict(state)
        parts, counts = [], {}
        for kind, _name in DATABASES:
            if kind not in databases:
                continue
            if kind in (SEL_TIO, SEL_H2O) and teff > TEFF_COOL_LIMIT:
                counts[kind] = 0
                continue
            if kind != SEL_LOWOBS:
                state["nu"] = 1
            ld = self.select(kind, databases[kind], state)
            parts.append(ld)
            counts[kind] = ld.shape[0]
        out = np.concatenate(parts) if parts else np.zeros((0, 4), np.int32)
        return out, counts, state


STEHLE_FILES = ("stehle_lyman.bin", "stehle_balmer.bin", "stehle_paschen.bin", "stehle_brackett.bin")


def _fortran_records(buf):
    """The records of a sequential unformatted file (4-byte length markers)."""
    out, o = [], 0
    while o < len(buf):
        n = int(np.frombuffer(buf, "<i4", 1, o)[0])
        if o + 8 + n > len(buf) or int(np.frombuffer(buf, "<i4", 1, o + 4 + n)[0]) != n:
            raise ValueError("record markers do not match at byte %d" % o)
        out.append(buf[o + 4:o + 4 + n])
        o += 8 + n
    return out


def read_stehle(path):
    """One Stehle MMM Stark-profile series as INIT_STARK_TABLES reads it
    (atlas12_modules.f90:17682-17746): record 1 the dimensions (n_lower,
    n_upper_min, n_upper_max, n_dens, n_temps, n_dalpha), then the density,
    temperature and log Delta-alpha grids, the per-transition highest valid
    density index and wing constant, and PROFILES(n_dalpha, n_temps, n_dens,
    n_trans).  Returns a dict with profiles as [n_trans, n_dens, n_temps,
    n_dalpha]."""
    r = _fortran_records(open(path, "rb").read())
    if len(r) != 7:
        raise ValueError("%s: %d records, expected 7" % (path, len(r)))
    n_lower, n_min, n_max, n_dens, n_temps, n_da = (int(x) for x in np.frombuffer(r[0], "<i4", 6))
    n_trans = n_max - n_min + 1
    if n_temps != 10 or n_da != 60 or not 2 <= n_dens <= 20 or n_trans < 1:
        raise ValueError("%s: unexpected dimensions %s" % (path, (n_dens, n_temps, n_da, n_trans)))
    prof = np.frombuffer(r[6], "<f8", n_da * n_temps * n_dens * n_trans)
    return dict(n_lower=n_lower, n_upper_min=n_min, n_upper_max=n_max,
                density_grid=np.frombuffer(r[1], "<f8", n_dens).copy(),
                temp_grid=np.frombuffer(r[2], "<f8", n_temps).copy(),
                log_dalpha_grid=np.frombuffer(r[3], "<f8", n_da).copy(),
                max_dens_idx=np.frombuffer(r[4], "<i4", n_trans).copy(),
                k_alpha=np.frombuffer(r[5], "<f8", n_trans).copy(),
                profiles=prof.reshape(n_trans, n_dens, n_temps, n_da).copy())


def read_stehle_dir(datadir):
    """The four series from DATADIR; a missing file leaves its entry None (the
    reference marks that series not loaded and uses the analytic profile)."""
    out = []
    for name in STEHLE_FILES:
        p = os.path.join(datadir, name)
        out.append(read_stehle(p) if os.path.exists(p) else None)
    return out
