"""The transmural coordinate (hrdayapy_b200.coordinates.
generate_transmural_coordinate) against the upstream function's own output
on a truncated ellipsoidal shell (tests/golden/transmural.npz, made by
running coordinates/functions/generate_transmural_coordinate.py at
tol 1e-8): the same Laplace problem (Dirichlet voxels +1 / -1, zero-flux
faces elsewhere), solved here to 1e-8 as well.  Tolerance 1e-5 in phi (both
are FP32 CG solutions of the same system)."""
import numpy as np
import pytest

from tests.conftest import has_gpu


def _check(device, golden):
    from hrdayapy_b200.coordinates import generate_transmural_coordinate
    g = golden("transmural.npz")
    phi = generate_transmural_coordinate(g["S"], g["surface_label"], device=device, tol=1e-8,
                                         maxiter=20000)
    ref = g["phi"]
    inside = g["S"] == 1
    assert np.isnan(phi[~inside]).all()
    assert np.abs(phi[inside] - ref[inside]).max() <= 1e-5
    assert (phi[g["surface_label"] == 1] == 1.0).all()
    assert (phi[g["surface_label"] == -1] == 0.0).all()


def test_transmural_coordinate_vs_upstream(golden):
    _check("cpu", golden)


@pytest.mark.gpu
def test_transmural_coordinate_on_the_device_vs_upstream(golden):
    _check("cuda", golden)


def test_shape_mismatch_is_rejected():
    from hrdayapy_b200.coordinates import generate_transmural_coordinate
    with pytest.raises(ValueError):
        generate_transmural_coordinate(np.ones((3, 3, 3), np.uint8), np.zeros((3, 3, 2), np.int8),
                                       device="cpu")
