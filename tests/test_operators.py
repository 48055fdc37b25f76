"""The operator data shipped with the package equals the reference's values
held in the test fixture (both written from the reference's files by
tests/golden/make_golden.py)."""
import numpy as np

from atlas12_b200 import operators


def test_package_operators_match_fixture(tables):
    ops = operators.load()
    for k in ("coefj", "coefh", "xtau8", "ch_j", "ck_j", "tabvi", "tabh1", "wavetab", "molcodes", "isox",
              "tio_isocorr", "h2o_isocorr", "h_propbm", "s_asum"):
        assert k in ops, k
    for k, v in ops.items():
        np.testing.assert_array_equal(v, tables[k], err_msg=k)
    # test-only entries are not shipped
    assert "deck" not in ops and "awei" not in ops
