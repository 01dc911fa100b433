"""Seeded grid generators: determinants and validity of the synthetic grids
the tests and the bench workloads use."""

from __future__ import annotations

import numpy as np

from egg_b200 import configs


def test_grid_mindet_2d_and_3d_on_uniform_grids():
    g2 = configs.unit_square(9, frac=0.0)
    np.testing.assert_allclose(configs.grid_mindet(g2.blocks, g2.X, 2), (1 / 8) ** 2)
    g3 = configs.unit_cube(5, frac=0.0)
    np.testing.assert_allclose(configs.grid_mindet(g3.blocks, g3.X, 3), (1 / 4) ** 3)


def test_sphere_in_cube_is_valid_without_noise():
    g = configs.sphere_in_cube(17, frac=0.0)
    assert configs.grid_mindet(g.blocks, g.X, 3).min() > 0


def test_tangled_square_reaches_its_target():
    g = configs.tangled_square(65, target=0.05, seed=1)
    md = configs.grid_mindet(g.blocks, g.X, 2).reshape(-1, 4)
    assert (md <= 0).any(axis=1).mean() >= 0.05
