"""The reference's compressed-coefficient and Mur-configuration unit tests
(src/fdtd/compressed.rs:296-436, src/extensions/mur_abc.rs:504-610),
replayed on this project's host routines (CPU, no GPU): the coefficient
deduplication the engine's compressed storage uses
(oems_compress_coefficients) and the Mur configuration.

The reference keeps (vv, vi, ii, iv) per direction, so its unique sets are
per component; the engine keeps the 12 coefficients of a cell as one set.
For the reference's test fields (the same values in every direction) both
count the same sets."""
import numpy as np
import pytest

import openems_b200 as oe
from openems_b200.constants import C0


def _fields(n, vv, vi, ii, iv):
    """12 arrays (ca0..2 = vv, cb0..2 = vi, da0..2 = ii, db0..2 = iv) of an
    n^3 grid, from per-cell value functions or scalars."""
    shape = (n, n, n)
    out = np.empty((12,) + shape, dtype=np.float32)
    for d in range(3):
        for base, v in ((0, vv), (3, vi), (6, ii), (9, iv)):
            out[base + d] = v(d) if callable(v) else v
    return out


def test_coefficient_set_round_trip():
    """test_coefficient_set: a set keeps vv = 1.0 and vi = 0.5."""
    ids, table = oe.compress_coefficients(_fields(2, 1.0, 0.5, 1.0, 0.5))
    assert table.shape == (1, 12)
    assert np.all(table[0, 0:3] == 1.0) and np.all(table[0, 3:6] == 0.5)
    assert np.all(ids == 0)


def test_compression_uniform():
    """test_compression_uniform: a uniform 10^3 field compresses to one set."""
    ids, table = oe.compress_coefficients(_fields(10, 1.0, 0.5, 1.0, 0.5))
    assert len(table) == 1 and ids.shape == (10, 10, 10)


def test_compression_varied():
    """test_compression_varied: value 1.0 for i < 5, 0.5 beyond (vi, iv half
    of it): two sets."""
    i = np.arange(10)[:, None, None] * np.ones((1, 10, 10))
    val = np.where(i < 5, 1.0, 0.5).astype(np.float32)
    ids, table = oe.compress_coefficients(_fields(10, lambda d: val, lambda d: val * 0.5,
                                                  lambda d: val, lambda d: val * 0.5))
    assert len(table) == 2
    assert np.array_equal(ids[:5], np.zeros((5, 10, 10))) and np.array_equal(ids[5:], np.ones((5, 10, 10)))


def test_coefficient_access():
    """test_coefficient_access: one cell with vv_x = 1.5, vi_x = 0.75 reads
    back through its set."""
    f = _fields(5, 1.0, 0.5, 1.0, 0.5)
    f[0, 2, 2, 2] = 1.5
    f[3, 2, 2, 2] = 0.75
    ids, table = oe.compress_coefficients(f)
    assert len(table) == 2
    s = table[ids[2, 2, 2]]
    assert s[0] == pytest.approx(1.5, abs=1e-6) and s[3] == pytest.approx(0.75, abs=1e-6)
    assert table[ids[0, 0, 0]][0] == 1.0
    # every cell decodes to its own coefficients
    assert np.array_equal(table[ids].transpose(3, 0, 1, 2), f)


def test_stats():
    """test_stats: 10^3 cells x 3 components = 3000 points, one set."""
    f = _fields(10, 1.0, 0.5, 1.0, 0.5)
    ids, table = oe.compress_coefficients(f)
    assert ids.size * 3 == 3000 and len(table) == 1


def test_operator_materials_give_one_set_each():
    """An operator with a dielectric box and a PEC sheet: vacuum, the box and
    the sheet are three sets, and the table decodes the operator exactly."""
    op = oe.Operator(oe.Grid.uniform(12, 10, 8, 1e-3), oe.BoundaryConditions.all_pec())
    op.set_material(4.0, 1.0, 0.01, 0.0, (2, 6, 2, 6, 2, 6))
    op.set_pec((8, 9, 0, 10, 0, 8))
    c = op.coefficients()
    ids, table = oe.compress_coefficients(c)
    assert len(table) == 3
    assert np.array_equal(table[ids].transpose(3, 0, 1, 2), c)


def test_mur_config_all_none_partial():
    """test_mur_config / test_mur_partial_boundaries: all faces, none, and
    all but the two x faces (4 faces)."""
    assert all(oe.MurAbcConfig.all().enabled) and oe.MurAbcConfig.all().num_faces() == 6
    assert not any(oe.MurAbcConfig.none().enabled)
    c = oe.MurAbcConfig.all()
    c.set_enabled(0, False)
    c.set_enabled(1, False)
    assert c.num_faces() == 4 and c.enabled == (False, False, True, True, True, True)


def test_mur_coefficient_negative():
    """test_mur_coefficient: (c dt - d) / (c dt + d) < 0 at dt = 1 ps, 1 mm."""
    dt, d = 1e-12, 1e-3
    assert (C0 * dt - d) / (C0 * dt + d) < 0.0
