"""List-directed REAL(8) records as gfortran writes them (host code of the
library; no GPU needed): one blank then a G25.17 field per item."""
import numpy as np
import pytest


@pytest.mark.parametrize("x,field", [
    (1.0, "  1.0000000000000000     "),
    (0.1, " 0.10000000000000001     "),
    (1.0 / 3.0, " 0.33333333333333331     "),
    (-2.5, " -2.5000000000000000     "),
    (0.0, "  0.0000000000000000     "),
    (12345.678, "  12345.678000000000     "),
    (1e-5, "  1.0000000000000001E-005"),
    (-3.0e-20, " -3.0000000000000003E-020"),
    (6.02e23, "  6.0200000000000000E+023"),
    (1e16, "  10000000000000000.     "),
])
def test_g_fields(tara, x, field):
    assert len(field) == 25
    assert tara.format_list_directed([x]) == " " + field


def test_record_and_round_trip(tara):
    rng = np.random.default_rng(0)
    v = np.concatenate([rng.standard_normal(50) * 10.0 ** rng.integers(-30, 30, 50), [0.0, 1.0]])
    s = tara.format_list_directed(v)
    assert len(s) == 26 * v.size
    back = np.array([float(s[26 * k:26 * (k + 1)].replace("E", "e")) for k in range(v.size)])
    assert np.array_equal(back, v)  # 17 significant digits round-trip every double
