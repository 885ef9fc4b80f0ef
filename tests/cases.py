"""Seeded parity cases shared by the tests (small enough for the oracle)."""
import numpy as np

from dendro_b200 import inputs as I

CASES = {
    # name: (points generator, maxDepth, maxNumPts)
    "gauss2k_d8": (lambda: I.clamp_unit(I.gaussian_cloud(2000, 0), 8), 8, 1),
    "gauss20k_d10": (lambda: I.clamp_unit(I.gaussian_cloud(20000, 0), 10), 10, 1),
    "lognormal20k_d12": (lambda: I.clamp_unit(I.lognormal_cloud(20000, 2), 12), 12, 1),
    "uniform8k_d9_m4": (lambda: I.clamp_unit(I.uniform_cloud(8000, 5), 9), 9, 4),
    "dup_points_d6": (lambda: np.repeat(I.clamp_unit(I.uniform_cloud(50, 7), 6), 5, axis=0), 6, 1),
    "single_point": (lambda: np.array([[0.3, 0.6, 0.9]]), 7, 1),
    "corner_points_d5": (lambda: np.array([[0, 0, 0], [1 - 2.0 ** -6, 1 - 2.0 ** -6, 1 - 2.0 ** -6],
                                           [0.5, 0.5, 0.5], [0.49, 0.51, 0.5]]), 5, 1),
}


def points(name):
    gen, d, m = CASES[name]
    return gen(), d, m
