"""The reference scheme's known instability, shown with the oracle (CPU).

With second-order wall extrapolation (wallExtOrder = 2, the default), a wall one voxel
away from the inlet or outlet plane (x = 2 with fluid at x = 1, or x = Nx - 1 with fluid at
x = Nx) extrapolates its incoming distribution through the periodic ghost plane, and the
source iteration diverges (mass flux and permeability grow without bound). Two fluid layers
at inlet and outlet (fluidlayer = 2) keep every such wall away from the ghost planes, but on
larger packs walls facing each other across one-voxel channels extrapolate from each
other's re-emitted values with gain 2 and diverge as well. The reference's shipped
tutorials use wallExtOrder = 1, and so do the benchmark workloads.
"""
import numpy as np
import pytest

from piks3d_b200 import images
from conftest import base_params
from oracle import Oracle


def _trace(img, steps, **kw):
    nz, ny, nx = img.shape
    p = base_params(nx, Ny=ny, Nz=nz, Nc_fundamental=2, Kn=0.5, **kw)
    o = Oracle(p, img.tobytes(), nthreads=4)
    out = []
    for _ in range(steps // 10):
        o.iterate(10)
        out.append(o.chk_converge()[1])
    o.close()
    return np.array(out)


def test_walls_next_to_inlet_diverge_with_second_order_extrapolation():
    img = images.sphere_pack(16, 0.5, 2.0, 4.0, seed=7)
    k = _trace(img, 100, fluidlayer=1)
    assert not np.all(np.abs(k) < 1.0), k


def test_two_fluid_layers_keep_the_iteration_bounded():
    img = images.sphere_pack(16, 0.5, 2.0, 4.0, seed=7)
    k = _trace(img, 100, fluidlayer=2)
    assert np.all(np.isfinite(k)) and np.all(np.abs(k) < 0.1), k
    assert k[-1] > 0
