"""GPU tests of the FP32 sweep and its FP64 refinement, against the FP64 oracle.

The FP32 path stores and sweeps f in FP32 while the moments, wall densities, mass flux and
convergence test stay FP64. Tolerances, relative to the oracle's FP64 values:
- converged permeability of the FP32 solve: 1e-4; velocity field (L2 over fluid voxels): 1e-4;
- converged permeability of the refined solve (FP32, then FP64 to eps): 1e-6;
- a few iterations from rest: f within 1e-5 of max|f|.
Every test prints the measured relative errors.
"""
import numpy as np
import pytest

import piks3d_b200 as pk
from piks3d_b200 import images
from conftest import base_params
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return abs(a - b) / abs(b)


def _velocity_rel_l2(macro_a, macro_b):
    num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(macro_a[1:], macro_b[1:]))
    den = sum(float(np.sum(b ** 2)) for b in macro_b[1:])
    return (num / den) ** 0.5


@pytest.fixture(scope="module")
def sphere32_oracle():
    img = images.centred_sphere(32, 12.0)
    p = base_params(32, Nc_fundamental=2, Kn=1.0, eps=1e-8, maxStep=2000)
    o = Oracle(p, img.tobytes(), nthreads=8)
    steps, k, _ = o.run()
    macro = tuple(m[2:-2, 2:-2, 2:-2] for m in o.macro())
    return img, p, steps, k, macro


def test_fp32_solve_sphere32(sphere32_oracle):
    img, p, steps_o, k_o, macro_o = sphere32_oracle
    with pk.Solver(p, device=0) as s:
        s.set_precision(pk.PREC_FP32)
        s.setup_physical_grid(img)
        assert s.precision == pk.PREC_FP32
        steps, k, _ = s.run()
        ek = _rel(k, k_o)
        eu = _velocity_rel_l2(s.get_macro(), macro_o)
        print("fp32 sphere32: steps %d (oracle %d) perm rel err %.3e velocity rel L2 err %.3e" % (steps, steps_o, ek, eu))
        assert ek <= 1e-4
        assert eu <= 1e-4


def test_refined_solve_sphere32(sphere32_oracle):
    img, p, steps_o, k_o, macro_o = sphere32_oracle
    with pk.Solver(p, device=0) as s:
        s.setup_physical_grid(img)
        n32, steps, k, _ = s.run_refined(switch_eps=1e-6)
        assert s.precision == pk.PREC_FP64
        ek = _rel(k, k_o)
        eu = _velocity_rel_l2(s.get_macro(), macro_o)
        print("refined sphere32: %d FP32 + %d FP64 steps (oracle %d) perm rel err %.3e velocity rel L2 err %.3e"
              % (n32, steps - n32, steps_o, ek, eu))
        assert 0 < n32 < steps
        assert ek <= 1e-6
        assert eu <= 1e-6


def test_refined_solve_pack_nv512():
    # two fluid layers at inlet and outlet: without them the walls next to x = 1 / Nx
    # extrapolate through the periodic ghost planes and the iteration diverges
    img = images.sphere_pack(12, 0.5, 1.5, 3.0, seed=7)
    p = base_params(12, Nc_fundamental=4, Kn=0.5, eps=1e-8, maxStep=3000, fluidlayer=2)
    o = Oracle(p, img.tobytes(), nthreads=8)
    _, k_o, _ = o.run()
    with pk.Solver(p, device=0) as s:
        s.setup_physical_grid(img)
        n32, steps, k, _ = s.run_refined(switch_eps=1e-6)
        print("refined pack12 nv512: %d FP32 + %d FP64 steps, perm rel err %.3e" % (n32, steps - n32, _rel(k, k_o)))
        assert _rel(k, k_o) <= 1e-6


def test_fp32_iterations_track_fp64():
    img = images.sphere_pack(10, 0.55, 1.2, 2.5, seed=4)
    p = base_params(10, Nc_fundamental=4, Kn=0.3, pressDrop=0.1)
    o = Oracle(p, img.tobytes(), nthreads=4)
    with pk.Solver(p, device=0) as s:
        s.set_precision(pk.PREC_FP32)
        s.setup_physical_grid(img)
        nodes = s.geometry_array("node_g")
        for _ in range(5):
            o.iterate(1)
            s.iterate(1)
        nc8 = s.info()["Nc8"]
        fo = o.f().reshape(8, nc8, -1)[:, :, nodes]
        fs = s.get_f()[0].reshape(8, nc8, -1)[:, :, nodes]
        err = np.abs(fs - fo).max() / np.abs(fo).max()
        print("fp32 after 5 iterations: max |f32 - f64| / max |f64| = %.3e" % err)
        assert err <= 1e-5
        mo, _, _ = o.chk_converge()
        ms, _, _ = s.chk_converge()
        assert _rel(ms, mo) <= 1e-5


def test_precision_switch_round_trip():
    img = images.sphere_pack(10, 0.55, 1.2, 2.5, seed=4)
    p = base_params(10, Nc_fundamental=4, Kn=0.3, pressDrop=0.1)
    with pk.Solver(p, device=0) as s:
        s.setup_physical_grid(img)
        s.iterate(4)
        f64, fw64 = s.get_f()
        s.set_precision(pk.PREC_FP32)
        f32, fw32 = s.get_f()
        assert np.array_equal(f32, f64.astype(np.float32).astype(np.float64))
        assert np.array_equal(fw32, fw64.astype(np.float32).astype(np.float64))
        s.set_precision(pk.PREC_FP64)
        fb, _ = s.get_f()
        assert np.array_equal(fb, f32)  # widening is exact
        s.iterate(1)


def test_fp32_footprint_is_smaller():
    img = images.sphere_pack(16, 0.5, 1.5, 3.5, seed=1)
    p = base_params(16, Nc_fundamental=4)
    with pk.Solver(p, device=0) as a, pk.Solver(p, device=0) as b:
        a.setup_physical_grid(img)
        b.set_precision(pk.PREC_FP32)
        b.setup_physical_grid(img)
        inf = a.info()
        f_bytes = inf["nNodes"] * 8 * inf["Nc8"] * 8
        assert a.info()["device_bytes"] - b.info()["device_bytes"] >= f_bytes // 2


def test_fp32_tile_and_hyperplane_schedules_agree():
    img = images.sphere_pack(16, 0.5, 1.5, 3.5, seed=1)
    p = base_params(16, Nc_fundamental=4, Kn=0.5, fluidlayer=2)
    out = []
    for tiles in ((8, 8, 8), (0, 0, 0)):
        with pk.Solver(p, device=0) as s:
            s.set_tiles(*tiles)
            s.set_precision(pk.PREC_FP32)
            s.setup_physical_grid(img)
            s.iterate(20)
            out.append((s.get_f()[0], s.chk_converge()[0]))
    (fa, ma), (fb, mb) = out
    err = np.abs(fa - fb).max() / np.abs(fb).max()
    print("fp32 tiles vs hyperplanes after 20 iterations: max rel diff %.3e, mass rel diff %.3e" % (err, _rel(ma, mb)))
    assert err <= 1e-5 and _rel(ma, mb) <= 1e-5


def test_switch_to_fp64_takes_the_fp64_tile_shape():
    """An FP32 state built with the default tiles (4x4x4) moves to the FP64 default shape
    (8x4x4, built on a host thread meanwhile) when it switches to FP64; the FP64 values do
    not depend on the schedule, so they equal those of a state that keeps 4x4x4 tiles."""
    img = images.sphere_pack(16, 0.5, 1.5, 3.5, seed=1)
    p = base_params(16, Nc_fundamental=4, Kn=0.5, fluidlayer=2)
    out = []
    for explicit in (False, True):
        with pk.Solver(p, device=0) as s:
            if explicit:
                s.set_tiles(4, 4, 4)
            s.set_precision(pk.PREC_FP32)
            s.setup_physical_grid(img)
            assert s.schedule()["TX"] == 4
            s.iterate(6)
            s.set_precision(pk.PREC_FP64)
            assert s.schedule()["TX"] == (4 if explicit else 8)
            s.iterate(5)
            out.append((s.get_f()[0], s.chk_converge()))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]


def test_fp32_dataflow_216_velocities_matches_diagonals():
    img = images.sphere_pack(10, 0.5, 1.2, 2.5, seed=8)
    p = base_params(10, Nc_fundamental=6, Kn=0.5)
    out = []
    for sched in (pk.SCHED_TILE_DATAFLOW, pk.SCHED_TILE_DIAGONALS):
        with pk.Solver(p, device=0) as s:
            s.set_precision(pk.PREC_FP32)
            s.set_schedule(sched)
            s.setup_physical_grid(img)
            s.iterate(5)
            out.append((s.get_f()[0], s.chk_converge()))
    assert np.array_equal(out[0][0], out[1][0]) and out[0][1] == out[1][1]


@pytest.mark.parametrize("nf", [2, 4, 6])
def test_fp32_columns_match_diagonals(nf):
    """The column-march and pipelined FP32 sweeps evaluate each update with the tile
    kernel's operations, so their values equal the tile-diagonal sweep's bit for bit (64,
    512 and 1728 velocities: rows of 8, 32 and 8 FP32 velocities per chunk)."""
    img = images.sphere_pack(14, 0.5, 1.2, 3.0, seed=31)
    p = base_params(14, Nc_fundamental=nf, Kn=0.5, fluidlayer=1)
    out = []
    for sched in (pk.SCHED_TILE_COLUMNS, pk.SCHED_TILE_PIPELINED, pk.SCHED_TILE_DIAGONALS):
        with pk.Solver(p, device=0) as s:
            s.set_tiles(4, 4, 4)
            s.set_precision(pk.PREC_FP32)
            s.set_schedule(sched)
            s.setup_physical_grid(img)
            s.iterate(6)
            out.append((s.get_f()[0], s.chk_converge()))
    for f, m in out[:2]:
        assert np.array_equal(f, out[2][0]) and m == out[2][1]
