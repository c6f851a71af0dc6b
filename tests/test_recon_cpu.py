"""CPU checks of the reconstruction driver's data generation."""

import numpy as np


def test_voxelize_boxes_matches_dense_voxelization():
    from adaptivetensordf_b200 import synthetic as syn
    from adaptivetensordf_b200.recon import voxelize_boxes

    ph = syn.ellipsoid_phantom(20, 1001)
    a = syn.voxelize(ph, 40)
    b = voxelize_boxes(ph, 40)
    assert np.array_equal(a, b)
    assert 0 < a.mean() < 1
