"""Voxel classification on the device (piks_set_preprocessing, preprocess.cu) against the
host's: wall labels, the node map of the voxels the solver reads, 3-fold corner numbers
and wall records come from CUDA kernels, and every geometry array the setup derives from
them (wall levels, switch roles, commits, sweep tasks, tile jobs, planes, flux list) must
equal the host path's exactly, on the parity images and on the benchmark's 128^3 pack
(physicalGrid.F90:546-936)."""
import numpy as np
import pytest

import piks3d_b200 as pk
from piks3d_b200 import images
from conftest import base_params

pytestmark = pytest.mark.gpu

ARRAYS = ("label", "nodemap", "node_g", "bcorner", "wall_node", "wall_label", "wall_corner", "wall_e", "wall_nb",
          "wall_order", "level_start", "roles", "commit", "tasks", "hyper_start", "plane_x1", "plane_xN",
          "sym_node", "sym_flag", "flux_list", "flux_groups", "tile_rows", "tile_row_begin", "tile_tasks",
          "tile_task_begin", "tile_steps", "tile_up")

CASES = [
    ("sphere16", lambda: images.centred_sphere(16, 5.0), dict(Nc_fundamental=2)),
    ("pack14_ext2", lambda: images.sphere_pack(14, 0.5, 1.5, 3.5, seed=1), dict(Nc_fundamental=2)),
    ("pack12_ext3_fl1", lambda: images.sphere_pack(12, 0.4, 1.2, 3.0, seed=3),
     dict(Nc_fundamental=2, wallExtOrder=3, fluidlayer=1)),
    ("aniso_13x9x11", lambda: images.sphere_pack(13, 0.5, 1.2, 2.5, seed=5)[:11, :9, :13].copy(),
     dict(Nx=13, Ny=9, Nz=11)),
    ("rep2x1x1", lambda: images.sphere_pack(10, 0.5, 1.2, 2.5, seed=6), dict(block_repx=2)),
]


def _compare(p, img):
    with pk.Solver(p, device=0) as d, pk.Solver(p, device=-1) as h:
        d.setup_physical_grid(img)
        h.setup_physical_grid(img)
        for key in ("Nfluid", "nWall", "nCorner", "nNodes", "nWallLevels"):
            assert d.info()[key] == h.info()[key], key
        for name in ARRAYS:
            a, b = d.geometry_array(name), h.geometry_array(name)
            assert a.shape == b.shape and np.array_equal(a, b), name
        return d.setup_seconds()


@pytest.mark.parametrize("name,make,kw", CASES, ids=[c[0] for c in CASES])
def test_device_classification_equals_host(name, make, kw):
    img = make()
    nz, ny, nx = img.shape
    p = base_params(nx, **{k: v for k, v in kw.items() if k not in ("Nx", "Ny", "Nz")})
    p.Ny, p.Nz = kw.get("Ny", ny), kw.get("Nz", nz)
    if "block_repx" in kw:
        p.Nx = nx
    _compare(p, img)


def test_device_classification_equals_host_bench_pack():
    import bench
    img = bench.workload_image()
    secs = _compare(bench.workload_params(pk), img)
    print("setup stages (box, device classification, rest, whole call): %.3f %.3f %.3f %.3f s" % secs)
