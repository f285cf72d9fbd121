"""Host side of the scattering scene and set_material_cells (no GPU)."""
import numpy as np

import openems_b200 as oe
from openems_b200.scene import ScatterScene


def test_set_material_cells_equals_box():
    a = oe.Operator(oe.Grid.uniform(9, 8, 7, 1e-3))
    b = oe.Operator(oe.Grid.uniform(9, 8, 7, 1e-3))
    a.set_material(3.5, 1.2, 0.01, 2.0, (2, 6, 1, 5, 3, 7))
    cells = np.mgrid[2:6, 1:5, 3:7].reshape(3, -1).T
    b.set_material_cells(3.5, 1.2, 0.01, 2.0, cells)
    assert np.array_equal(a.coefficients(), b.coefficients())


def test_set_material_cells_rejects_outside():
    op = oe.Operator(oe.Grid.uniform(4, 4, 4, 1e-3))
    try:
        op.set_material_cells(2.0, 1.0, 0.0, 0.0, [(4, 0, 0)])
    except oe.MaterialError:
        return
    raise AssertionError("expected MaterialError")


def test_scene_geometry():
    sc = ScatterScene(n=384)
    assert sc.radius == 96 and sc.shell == 8 and sc.box == ((18,) * 3, (365,) * 3)
    small = ScatterScene(n=48, layers=4)
    sphere, shell = small.cells()
    c = small.center
    d = lambda p: np.sqrt(((p + 0.5 - c) ** 2).sum(1))  # noqa: E731
    assert d(sphere.astype(float)).max() <= small.radius
    assert d(shell.astype(float)).min() > small.radius
    lo, hi = small.box
    assert lo[0] < small.port[0] < hi[0]  # the source lies inside the NF2FF box
    assert small.port[0] - 0 > small.layers
