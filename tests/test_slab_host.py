"""x-slab decomposition of one box (mpiParams.F90:120-240 with mpi_xdim ranks; halos of
solver.F90:146-170, :535-612), on the CPU: the library's slab geometry (host-only contexts)
replayed by the numpy model of the device data flow, rank by rank with the halo buffers
moved between iterations, against the oracle's ranks moved the same way; the partition;
the halo lists of neighbouring ranks; and the single-rank case against the undecomposed
context. Multi-process (gloo) exchange: tests/test_slab_dist.py."""
import numpy as np
import pytest

import device_model as dm
import piks3d_b200 as pk
from conftest import base_params
from oracle import Oracle, SlabOracle
from piks3d_b200 import images


def _slab_contexts(p, img, n):
    out = []
    for r in range(n):
        s = pk.Solver(p, device=-1)
        s.set_decomposition(n, r)
        s.setup_physical_grid(img)
        out.append(s)
    return out


@pytest.mark.parametrize("nx,n", [(16, 2), (16, 3), (17, 4), (9, 4), (30, 7)])
def test_partition_matches_the_reference_formula(nx, n):
    p = base_params(nx, Ny=6, Nz=6)
    img = np.zeros((6, 6, nx), np.uint8)
    for r in range(n):
        s = pk.Solver(p, device=-1)
        s.set_decomposition(n, r)
        o = Oracle(p, img.tobytes(), 1, n, r)
        so, ss = o.slab(), s.slab()
        assert (ss["xl"], ss["xu"]) == (so["xl"], so["xu"])
        o.close()
        s.close()


def test_too_many_ranks_and_late_decomposition_are_refused():
    p = base_params(8)
    s = pk.Solver(p, device=-1)
    with pytest.raises(pk.PiksError):
        s.set_decomposition(5, 0)     # 7 plane gaps over 5 ranks: a rank with one plane
    with pytest.raises(pk.PiksError):
        s.set_decomposition(2, 2)
    s.set_decomposition(2, 1)
    s.setup_physical_grid(images.centred_sphere(8, 2.5))
    with pytest.raises(pk.PiksError):
        s.set_decomposition(2, 0)
    s.close()


def test_single_rank_decomposition_is_the_plain_geometry():
    p = base_params(14, wallExtOrder=3)
    img = images.sphere_pack(14, 0.5, 1.5, 3.5, seed=1)
    a = pk.Solver(p, device=-1)
    a.setup_physical_grid(img)
    b = _slab_contexts(p, img, 1)[0]
    for name in ("nodemap", "node_g", "tasks", "hyper_start", "wall_node", "wall_e", "wall_nb", "roles", "commit",
                 "plane_x1", "plane_xN", "sym_node", "flux_list", "flux_groups", "tile_rows", "tile_tasks"):
        assert np.array_equal(a.geometry_array(name), b.geometry_array(name)), name
    for name in ("halo_send_w", "halo_send_e", "halo_recv_w", "halo_recv_e"):
        assert len(b.geometry_array(name)) == 0
    a.close()
    b.close()


def _coords(s, nodes):
    inf = s.info()
    gx, gy = inf["Nx"] + 4, inf["Ny"] + 4
    g = s.geometry_array("node_g")[nodes].astype(np.int64)
    return np.stack([g % gx - 1, (g // gx) % gy - 1, g // (gx * gy) - 1], axis=1)


@pytest.mark.parametrize("n", [2, 3])
def test_halo_lists_of_neighbours_pair_up(n):
    p = base_params(15, wallExtOrder=1)
    img = images.sphere_pack(15, 0.5, 1.5, 3.5, seed=7)
    ctx = _slab_contexts(p, img, n)
    for r in range(n):
        e = (r + 1) % n
        if r == n - 1:
            # the box's edge: the pair exchanges the inlet / outlet planes, not node lists
            assert len(ctx[r].geometry_array("halo_send_e")) == 0
            continue
        se = _coords(ctx[r], ctx[r].geometry_array("halo_send_e"))
        rw = _coords(ctx[e], ctx[e].geometry_array("halo_recv_w"))
        sw = _coords(ctx[e], ctx[e].geometry_array("halo_send_w"))
        re = _coords(ctx[r], ctx[r].geometry_array("halo_recv_e"))
        assert np.array_equal(se, rw) and np.array_equal(sw, re)
        xu = ctx[r].slab()["xu"]
        assert set(se[:, 0]) <= {xu - 1, xu} and set(sw[:, 0]) <= {xu + 1, xu + 2}
    for s in ctx:
        s.close()


SLAB_CASES = [
    ("pack14_ext1", lambda: images.sphere_pack(14, 0.5, 1.5, 3.5, seed=1), dict(wallExtOrder=1, Kn=0.7)),
    ("pack14_ext2", lambda: images.sphere_pack(14, 0.45, 1.2, 3.0, seed=2), dict(wallExtOrder=2, Kn=0.5)),
    ("pack13_ext3_fl1", lambda: images.sphere_pack(13, 0.4, 1.2, 3.0, seed=3), dict(wallExtOrder=3, fluidlayer=1)),
]


@pytest.mark.parametrize("n", [2, 3])
@pytest.mark.parametrize("name,make,kw", SLAB_CASES, ids=[c[0] for c in SLAB_CASES])
def test_slab_model_equals_slab_oracle(name, make, kw, n):
    img = make()
    nx = img.shape[2]
    p = base_params(nx, **kw)
    so = SlabOracle(p, img.tobytes(), n, nthreads=2)
    ctx = _slab_contexts(p, img, n)
    models = [dm.DeviceModel(s, p) for s in ctx]
    for it in range(3):
        so.iterate(1)
        dm.iterate_slabs(models, 1)
    mo = so.macro()
    for s, m in zip(ctx, models):
        c = _coords(s, np.arange(m.NF))
        for q in range(4):
            assert np.array_equal(mo[q][c[:, 2] - 1, c[:, 1] - 1, c[:, 0] - 1], m.mom[q]), (q, s.slab())
        # every owned node's rows (fluid and solid) equal the oracle's at that voxel
        own = np.nonzero((lambda cc: (cc[:, 0] >= s.slab()["xl"]) & (cc[:, 0] <= s.slab()["xu"]))(
            _coords(s, np.arange(m.nn))))[0]
        cc = _coords(s, own)
        fo = so.f_at_global(cc[:, 0], cc[:, 1], cc[:, 2])
        assert np.array_equal(fo, m.h[own]), s.slab()
    assert so.chk_converge()[0] == models[0].mass_flux()
    so.close()
    for s in ctx:
        s.close()


@pytest.mark.parametrize("form,tiles,sched", [("tiles", (4, 4, 4), pk.SCHED_TILE_DIAGONALS),
                                              ("tiles", (5, 2, 3), pk.SCHED_TILE_DATAFLOW),
                                              ("columns", (4, 4, 4), pk.SCHED_TILE_COLUMNS)])
def test_slab_tile_schedules_equal_slab_oracle(form, tiles, sched):
    """The tile jobs and column lists built on a slab, replayed job by job."""
    img = images.sphere_pack(14, 0.5, 1.5, 3.5, seed=1)
    p = base_params(14, wallExtOrder=1, Kn=0.7)
    n = 3
    so = SlabOracle(p, img.tobytes(), n, nthreads=2)
    ctx = []
    for r in range(n):
        s = pk.Solver(p, device=-1)
        s.set_decomposition(n, r)
        s.set_tiles(*tiles)
        s.set_schedule(sched)
        s.setup_physical_grid(img)
        ctx.append(s)
    models = [dm.DeviceModel(s, p) for s in ctx]
    for _ in range(3):
        so.iterate(1)
        dm.exchange(models)
        for m, s in zip(models, ctx):
            m.iterate(1, schedule=form, solver=s)
    mo = so.macro()
    for s, m in zip(ctx, models):
        c = _coords(s, np.arange(m.NF))
        for q in range(4):
            assert np.array_equal(mo[q][c[:, 2] - 1, c[:, 1] - 1, c[:, 0] - 1], m.mom[q])
    assert so.chk_converge()[0] == models[0].mass_flux()
    so.close()
    for s in ctx:
        s.close()
