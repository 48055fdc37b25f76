"""The operator data a caller passes to the library.

The reference reads these at start-up: JOSH's 51x51 J and H operators from
data/blockj.dat and data/blockh.dat (BLOCKJ/BLOCKH,
atlas12_modules.f90:18792-18860), its tau grid and surface weights XTAU8,
CH_J, CK_J (:18409-18451), TABVOIGT's H1 table (:19805-19835), KAPCONT's
WAVETAB (:1811-1857), SELECTLINES's species and isotope tables
(:19182-19207) and the hydrogen profiles' tables of both programs.  A
Fortran driver passes what it holds; Python callers load the same values
from ``data/operators.npz`` (written from the reference's files by the
fixture script beside the tests).
"""
import os

import numpy as np

PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "operators.npz")


def load(path=PATH):
    """dict of name -> array (coefj, coefh, xtau8, ch_j, ck_j, tabvi, tabh1,
    wavetab, molcodes, isox, tio_isocorr, h2o_isocorr, h_*, s_*)."""
    t = np.load(path)
    return {k: t[k] for k in t.files}
