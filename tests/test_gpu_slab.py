"""GPU tests of the x-slab decomposition of one box (mpiParams.F90:120-240 with mpi_xdim
ranks; halos of solver.F90:146-170, :535-612): the ranks run as contexts on one GPU
(piks3d_b200.slab.LocalSlabs, halos moved by device copies between iterations, no kernel
of one rank waits on another's), FP64 bit for bit against the oracle's ranks moved the same
way (SlabOracle), under the launch schedules; FP32 slabs within the FP32 tolerance; the
single-rank SlabSolver equal to a plain context."""
import numpy as np
import pytest

import piks3d_b200 as pk
from conftest import base_params
from oracle import SlabOracle
from piks3d_b200 import images
from piks3d_b200.slab import LocalSlabs, SlabSolver

pytestmark = pytest.mark.gpu

CASES = [
    ("pack14_ext1", lambda: images.sphere_pack(14, 0.5, 1.5, 3.5, seed=1), dict(wallExtOrder=1, Kn=0.7)),
    ("pack16_ext2_nv512", lambda: images.sphere_pack(16, 0.45, 1.2, 3.0, seed=2), dict(wallExtOrder=2, Nc_fundamental=4)),
    ("pack13_ext3_fl1", lambda: images.sphere_pack(13, 0.4, 1.2, 3.0, seed=3), dict(wallExtOrder=3, fluidlayer=1)),
]
SCHEDULES = {"diagonals": (None, None), "dataflow": ((4, 4, 4), pk.SCHED_TILE_DATAFLOW),
             "hyperplanes": ((0, 0, 0), None), "columns": ((4, 4, 4), pk.SCHED_TILE_COLUMNS)}


def _owned_rows_equal(ls, so):
    for s in ls.solvers:
        sl = s.slab()
        inf = s.info()
        gx, gy = inf["Nx"] + 4, inf["Ny"] + 4
        g = s.geometry_array("node_g").astype(np.int64)
        i, j, k = g % gx - 1, (g // gx) % gy - 1, g // (gx * gy) - 1
        own = np.nonzero((i >= sl["xl"]) & (i <= sl["xu"]))[0].astype(np.int32)
        fs = s.get_f_nodes(own)
        fo = so.f_at_global(i[own], j[own], k[own])
        assert np.array_equal(fs, fo), (sl, np.abs(fs - fo).max())


@pytest.mark.parametrize("schedule", list(SCHEDULES))
@pytest.mark.parametrize("n", [2, 3])
@pytest.mark.parametrize("name,make,kw", CASES, ids=[c[0] for c in CASES])
def test_slabs_equal_slab_oracle(name, make, kw, n, schedule):
    img = make()
    p = base_params(img.shape[2], **kw)
    tiles, sched = SCHEDULES[schedule]
    ls = LocalSlabs(p, img, n, tiles=tiles, schedule=sched)
    so = SlabOracle(p, img.tobytes(), n, nthreads=8)
    for it in range(3):
        ls.iterate(1)
        so.iterate(1)
    for a, b in zip(so.macro(), ls.macro()):
        assert np.array_equal(a, b)
    assert ls.chk_converge() == so.chk_converge()
    _owned_rows_equal(ls, so)
    ls.close()
    so.close()


def test_bench_workload_on_two_slabs_equals_oracle():
    """The benchmark's 128^3 pack (512 velocities, Kn 0.5, wallExtOrder 1) as two x slabs:
    two FP64 iterations, full-box moments and the check triple bit for bit."""
    import bench
    img = bench.workload_image()
    p = bench.workload_params(pk)
    ls = LocalSlabs(p, img, 2)
    so = SlabOracle(p, img.tobytes(), 2, nthreads=0)
    ls.iterate(2)
    so.iterate(2)
    for a, b in zip(so.macro(), ls.macro()):
        assert np.array_equal(a, b)
    assert ls.chk_converge() == so.chk_converge()
    ls.close()
    so.close()


def test_fp32_slabs_track_fp64_oracle():
    img = images.sphere_pack(16, 0.5, 1.5, 3.5, seed=5)
    p = base_params(16, wallExtOrder=1, Kn=0.8)
    ls = LocalSlabs(p, img, 2, precision="fp32")
    so = SlabOracle(p, img.tobytes(), 2, nthreads=8)
    for _ in range(3):
        ls.iterate(10)
        so.iterate(10)
        m32, _, _ = ls.chk_converge()
        m64, _, _ = so.chk_converge()
        assert abs(m32 - m64) <= 1e-4 * abs(m64)
    # switching every rank to FP64 keeps the state (and its in-flight halo buffers) usable
    ls.set_precision(pk.PREC_FP64)
    ls.iterate(10)
    so.iterate(10)
    assert abs(ls.chk_converge()[0] - so.chk_converge()[0]) <= 1e-4 * abs(so.chk_converge()[0])
    ls.close()
    so.close()


def test_slab_context_iterates_one_step_per_call():
    img = images.sphere_pack(12, 0.5, 1.5, 3.0, seed=4)
    p = base_params(12, wallExtOrder=1)
    ls = LocalSlabs(p, img, 2)
    with pytest.raises(pk.PiksError):
        ls.solvers[0].iterate(2)
    with pytest.raises(pk.PiksError):
        ls.solvers[0].run()
    ls.close()


def test_single_rank_slab_solver_equals_plain_context():
    img = images.sphere_pack(14, 0.5, 1.5, 3.5, seed=6)
    p = base_params(14, wallExtOrder=1)
    a = pk.Solver(p, device=0)
    a.setup_physical_grid(img)
    b = SlabSolver(p, img, device=0)
    a.iterate(4)
    b.iterate(4)
    assert a.chk_converge() == b.chk_converge()
    for x, y in zip(a.get_macro(), b.owned_macro()[2]):
        assert np.array_equal(x, y)
    a.close()
    b.close()
