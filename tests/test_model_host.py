"""Host functions of the library that build the benchmark model (no GPU): genZ! with the Z
refinement of NZ = 30 m and the XY pitch round(1.2e-3 / N, digits=8), bit-identical to the
oracle; an NZ the refinement does not cover is rejected by both."""
import numpy as np
import pytest

import h2_b200


def test_zgrid_bit_exact(oracle):
    from h2_b200 import model
    for nz in (30, 60, 90, 120, 240):
        for a, b in zip(model.zgrid(nz), oracle.genz(nz)):
            assert np.array_equal(a, b)


def test_zgrid_rejects_other_nz(oracle):
    from h2_b200 import model
    for nz in (0, 29, 31, 45):
        with pytest.raises(h2_b200.H2GError):
            model.zgrid(nz)
        with pytest.raises(ValueError):
            oracle.genz(nz)


def test_pitch_bit_exact(oracle):
    from h2_b200 import model
    for n in range(1, 2001):
        assert model.pitch(n) == oracle.pitch(n), n
