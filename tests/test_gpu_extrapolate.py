"""GPU tests of the state snapshots behind the refined solver's extrapolation
(piks_snapshot_slot / _gram / _combine): a snapshot holds everything the next iteration
reads (put back, the iteration retraces its path bit for bit), combinations are evaluated
exactly as written, and the Gram matrix is that of the slot differences."""
import numpy as np
import pytest

import piks3d_b200 as pk
from conftest import base_params
from piks3d_b200 import images

pytestmark = pytest.mark.gpu


def _solver(prec=pk.PREC_FP64):
    img = images.sphere_pack(16, 0.5, 1.5, 3.5, seed=3)
    s = pk.Solver(base_params(16, wallExtOrder=1, Kn=0.7), device=0)
    s.set_precision(prec)
    s.setup_physical_grid(img)
    return s


def test_restored_snapshot_retraces_the_iteration():
    s = _solver()
    s.iterate(10)
    s.snapshot_slot(0, 3)
    s.iterate(10)
    f20, m20 = s.get_f()[0].copy(), s.chk_converge()
    s.snapshot_slot(1, 3)
    s.iterate(10)
    s.snapshot_slot(2, 3)
    # back to the state after 10 iterations, then 10 more: the same state as at 20
    s.snapshot_combine([1.0, 0.0, 0.0])
    s.iterate(10)
    assert np.array_equal(s.get_f()[0], f20)
    s.close()


def test_combination_and_gram_of_slots():
    s = _solver()
    fs = []
    for j in range(3):
        s.iterate(10)
        s.snapshot_slot(j, 3)
        fs.append(s.get_f()[0].copy())
    g = s.snapshot_gram(3)
    assert g.shape == (2, 2) and np.allclose(g, g.T)
    u0, u1 = fs[1] - fs[0], fs[2] - fs[1]
    # the state also holds fw, the moments and the ghost planes: the f part alone is a lower
    # bound of each diagonal entry, and the matrix is positive semidefinite
    assert g[0, 0] >= u0 @ u0 * (1 - 1e-12) and g[1, 1] >= u1 @ u1 * (1 - 1e-12)
    assert np.linalg.eigvalsh(g).min() >= -1e-12 * abs(g).max()
    s.snapshot_combine([2.0, -1.0])
    assert np.array_equal(s.get_f()[0], 2.0 * fs[0] - fs[1])
    # slots are used up by a combination
    with pytest.raises(pk.PiksError):
        s.snapshot_combine([1.0])
    s.close()


def test_slots_must_lie_an_even_number_of_iterations_away():
    s = _solver(pk.PREC_FP32)
    s.iterate(10)
    s.snapshot_slot(0, 2)
    s.iterate(1)
    with pytest.raises(pk.PiksError):
        s.snapshot_combine([1.0])
    s.close()
