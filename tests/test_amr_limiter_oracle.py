"""Mesh-level and limiter checkers, CPU: the library's generated projector tables against the
reference's own (the compiled GaussLegendreBasis snippet's fineGridProjector and the limiter
solver's runtime projectors, oracle/_ref/libexaref_amrlim3d.so), the compiled reference kernels
against the reference's limiter known-answer vectors (tests/golden/limiter_3d.npz, from
ExaHyPE/exahype/tests/kernels/testdata/limiter_testdata.cpp), and the reference's own mesh-level
test (GenericEulerKernelTest3D.cpp:706-851: constants are prolongated exactly and restored by
restricting all children). No GPU: the library is only asked for its host tables.
"""
import os

import numpy as np
import pytest

from conftest import REPO
from pyoracle import RefAmrLimiter

ref_missing = not os.path.exists(os.path.join(REPO, "oracle", "_ref", "libexaref_amrlim3d.so"))
pytestmark = pytest.mark.skipif(ref_missing, reason="oracle/_ref not built")
GOLD = os.path.join(REPO, "tests", "golden")


@pytest.mark.parametrize("order", range(1, 10))
def test_projector_tables_match_reference(order):
    import exa_aderdg
    ours = exa_aderdg.amr_limiter_projectors(order)
    ref = RefAmrLimiter.tables(order)
    # fineGridProjector: both rounded from the exact values
    assert np.array_equal(ours["fine"], ref["fine"])
    # the reference computes dg2fv, fv2dg (a Gauss-Jordan inverse) and leg2lob in double at run time
    for k in ("dg2fv", "fv2dg", "leg2lob"):
        assert np.abs(ours[k] - ref[k]).max() <= 1e-14 * max(1.0, np.abs(ref[k]).max()), k


def test_reference_limiter_kernels_reproduce_known_answers():
    """N = 3, nVar = 5, no ghost layers: the reference's known-answer vectors through its kernels,
    node-major layout ([node][variable]). This pins the checker the GPU tests use."""
    g = np.load(os.path.join(GOLD, "limiter_3d.npz"))
    ref = RefAmrLimiter(3, 5, 0)
    _, lim, _, _ = ref.limiter(0, g["testFromLuhConversion.luh_in"], ghost=0, out=np.zeros(343 * 5))
    assert np.abs(lim - g["testFromLuhConversion.lim_out"]).max() <= 1e-13 * np.abs(g["testFromLuhConversion.lim_out"]).max()
    _, luh, _, _ = ref.limiter(1, g["testToLuhConversion.lim_in"], ghost=0, out=np.zeros(64 * 5))
    assert np.abs(luh - g["testToLuhConversion.luh_out"]).max() <= 1e-13 * np.abs(g["testToLuhConversion.luh_out"]).max()
    # Gauss-Lobatto values: the leg2lob projector applied along each axis
    L = RefAmrLimiter.tables(3)["leg2lob"]
    U = g["testFromLuhConversion.luh_in"].reshape(4, 4, 4, 5)
    lob = np.einsum("zyxv,za,yb,xc->abcv", U, L, L, L).reshape(-1)
    assert np.abs(lob - g["testFromLuhConversion.lob_out"]).max() <= 1e-13 * np.abs(lob).max()


@pytest.mark.parametrize("level_delta", [1, 2])
def test_reference_amr_known_answer_constants(level_delta):
    """The reference's own test: a constant coarse cell prolongates to the same constant in every
    child, and restricting every child of a constant field restores it."""
    ref = RefAmrLimiter(3, 5, 1)
    nb, D = 64, 6
    ones = np.ones(nb * D)
    k = 3 ** level_delta
    coarse = np.zeros(nb * D)
    for i3 in range(k):
        for i2 in range(k):
            for i1 in range(k):
                fine = ref.volume(0, np.zeros(nb * D), ones, 0, level_delta, (i1, i2, i3))
                assert np.abs(fine - 1.0).max() < 1e-12
                coarse = ref.volume(1, coarse, ones, 0, level_delta, (i1, i2, i3))
    assert np.abs(coarse - 1.0).max() < 1e-10
