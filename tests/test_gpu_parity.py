"""GPU parity: the CUDA library through its C ABI against the CPU oracle.

The FP64 path evaluates every value with the oracle's operation order and rounding, so
the distribution function, the moments and the mass flux must match the oracle bit for
bit after each iteration (tolerance 0). Converged permeability must match within a
relative 1e-8 (and is in fact identical).
"""
import numpy as np
import pytest

import piks3d_b200 as pk
from piks3d_b200 import images
from conftest import base_params
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _compare_state(o, s, nodes):
    fo = o.f()
    fs, fws = s.get_f()
    inf = s.info()
    nc8 = inf["Nc8"]
    fo = fo.reshape(8, nc8, -1)[:, :, nodes]
    fs = fs.reshape(8, nc8, -1)[:, :, nodes]
    assert np.array_equal(fo, fs), "f differs: max %g" % np.abs(fo - fs).max()
    fwo = o.fw()
    assert np.array_equal(fwo, fws), "fw differs"
    mo = o.macro()
    rho, ux, uy, uz = s.get_macro()
    for a, b in zip(mo, (rho, ux, uy, uz)):
        assert np.array_equal(a[2:-2, 2:-2, 2:-2], b)


CASES = [
    # (image builder, params) — small images that exercise every wall type
    ("sphere16", lambda: images.centred_sphere(16, 5.0), dict(Nc_fundamental=2, Kn=1.0)),
    ("pack14_ext2", lambda: images.sphere_pack(14, 0.5, 1.5, 3.5, seed=1), dict(Nc_fundamental=2, Kn=0.7)),
    ("pack12_ext1", lambda: images.sphere_pack(12, 0.45, 1.2, 3.0, seed=2), dict(Nc_fundamental=2, wallExtOrder=1, accom=0.8)),
    ("pack12_ext3_fl1", lambda: images.sphere_pack(12, 0.4, 1.2, 3.0, seed=3), dict(Nc_fundamental=2, wallExtOrder=3, fluidlayer=1)),
    ("pack10_nv512", lambda: images.sphere_pack(10, 0.55, 1.2, 2.5, seed=4), dict(Nc_fundamental=4, Kn=0.3, pressDrop=0.1)),
    ("aniso_13x9x11", lambda: images.sphere_pack(13, 0.5, 1.2, 2.5, seed=5)[:11, :9, :13].copy(), dict(Nx=13, Ny=9, Nz=11)),
]


SCHEDULES = {"tiles844_dataflow": ((8, 4, 4), pk.SCHED_TILE_DATAFLOW),
             "tiles435_dataflow": ((4, 3, 5), pk.SCHED_TILE_DATAFLOW),
             "tiles8_diagonals": ((8, 8, 8), pk.SCHED_TILE_DIAGONALS),
             "hyperplanes": ((0, 0, 0), pk.SCHED_TILE_DATAFLOW),
             "columns444": ((4, 4, 4), pk.SCHED_TILE_COLUMNS),
             "columns523": ((5, 2, 3), pk.SCHED_TILE_COLUMNS),
             "pipelined444": ((4, 4, 4), pk.SCHED_TILE_PIPELINED),
             "pipelined523": ((5, 2, 3), pk.SCHED_TILE_PIPELINED)}


@pytest.mark.parametrize("schedule", list(SCHEDULES))
@pytest.mark.parametrize("name,make,kw", CASES, ids=[c[0] for c in CASES])
def test_iterations_bit_exact(name, make, kw, schedule):
    img = make()
    nz, ny, nx = img.shape
    p = base_params(nx, Ny=ny, Nz=nz, **{k: v for k, v in kw.items() if k not in ("Nx", "Ny", "Nz")})
    o = Oracle(p, img.tobytes(), nthreads=4)
    s = pk.Solver(p, device=0)
    tiles, launch = SCHEDULES[schedule]
    s.set_tiles(*tiles)
    s.set_schedule(launch)
    s.setup_physical_grid(img)
    assert s.schedule()["tiles"] == (tiles[0] > 0)
    assert np.array_equal(o.labels(), s.get_labels())
    nodes = s.geometry_array("node_g")
    for it in range(5):
        o.iterate(1)
        s.iterate(1)
        _compare_state(o, s, nodes)
        mo, ko, eo = o.chk_converge()
        ms, ks, es = s.chk_converge()
        assert (mo, ko, eo) == (ms, ks, es)
    s.close()


def test_graph_replay_equals_plain_launches():
    """Iterations replayed from the per-parity CUDA graphs (the default) give the values of
    plain launches (per-kernel timing on forces those), across a precision switch, which
    re-captures the graphs, for the tile-diagonal and the per-node hyperplane schedules."""
    img = images.sphere_pack(14, 0.5, 1.5, 3.5, seed=1)
    p = base_params(14, Nc_fundamental=4, Kn=0.5, fluidlayer=2)
    for tiles in ((4, 4, 4), (0, 0, 0)):
        out = []
        for timing in (True, False):
            with pk.Solver(p, device=0) as s:
                s.enable_timing(timing)
                s.set_tiles(*tiles)
                s.set_precision(pk.PREC_FP32)
                s.setup_physical_grid(img)
                s.iterate(7)
                m32 = s.chk_converge()
                s.set_precision(pk.PREC_FP64)
                s.iterate(6)
                out.append((s.get_f()[0], m32, s.chk_converge()))
        (fa, m32a, ma), (fb, m32b, mb) = out
        assert np.array_equal(fa, fb) and m32a == m32b and ma == mb, tiles


def test_converged_permeability_sphere32():
    """32^3 box with a centred sphere of radius 12, 64 velocities, Kn = 1: the solve
    converges to the same permeability and step count as the oracle."""
    img = images.centred_sphere(32, 12.0)
    p = base_params(32, Nc_fundamental=2, Kn=1.0, eps=1e-8, maxStep=2000)
    o = Oracle(p, img.tobytes(), nthreads=8)
    so, ko, _ = o.run()
    s = pk.Solver(p, device=0)
    s.setup_physical_grid(img)
    ss, ks, _ = s.run()
    assert ss == so
    assert abs(ks - ko) <= 1e-8 * abs(ko)
    assert ks == ko
    s.close()


def test_run_writes_reference_files(tmp_path):
    img = images.sphere_pack(12, 0.5, 1.5, 3.0, seed=9)
    p = base_params(12, maxStep=30, chkConvergeStep=10, saveFormat=1)
    o = Oracle(p, img.tobytes(), nthreads=2)
    odir = tmp_path / "oracle"
    sdir = tmp_path / "gpu"
    odir.mkdir()
    sdir.mkdir()
    o.run(results_path=str(odir / "Results.dat"))
    s = pk.Solver(p, device=0)
    s.setup_physical_grid(img)
    s.run(results_path=str(sdir / "Results.dat"), out_dir=str(sdir))
    assert (odir / "Results.dat").read_text() == (sdir / "Results.dat").read_text()
    for fmt, names in ((1, ("Field_000.vti", "Field.pvti")), (2, ("Field_000.dat",)), (3, ("Field_000.vtk",))):
        o.save(str(odir), fmt)
        s.save_fields(str(sdir), fmt)
        for nm in names:
            assert (odir / nm).read_text() == (sdir / nm).read_text(), nm
    s.close()


def test_sweep_division_matches_ieee():
    """The sweep divides with a correctly rounded reciprocal and one fused correction
    (Markstein); it must return exactly the IEEE quotient."""
    import ctypes
    lib = pk.load_library()
    lib.piks_selftest_division.argtypes = [ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int64)]
    bad = ctypes.c_int64(-1)
    assert lib.piks_selftest_division(0, 1 << 28, 12345, ctypes.byref(bad)) == 0
    assert bad.value == 0


def test_tutorial_case_trace_matches_golden():
    """The reference's shipped tutorial (tutorials/cubicSpherePacking: 100^3 quarter
    sphere, 512 velocities, Kn = 0.1, first-order wall extrapolation, 100 steps) run
    through the C ABI reproduces the oracle's committed chkConverge trace exactly."""
    import json
    import os
    from conftest import ROOT
    tr = json.load(open(os.path.join(ROOT, "tests", "golden", "oracle_traces.json")))["tutorial_cubicSpherePacking"]
    p = pk.default_params(**{k: v for k, v in tr["params"].items()})
    s = pk.Solver(p, device=0)
    s.setup_physical_grid(images.quarter_sphere(100, 0.75))
    for step, mass, perm, err in tr["checks"]:
        s.iterate(p.chkConvergeStep)
        m, k, e = s.chk_converge()
        assert (repr(m), repr(k), repr(e)) == (mass, perm, err), step
    s.close()


def test_autotune_then_bit_exact():
    """The autotuner's trial sweeps leave no trace: after it, iterations equal the oracle's."""
    img = images.sphere_pack(10, 0.55, 1.2, 2.5, seed=4)
    p = base_params(10, Nc_fundamental=4, Kn=0.3, pressDrop=0.1)
    o = Oracle(p, img.tobytes(), nthreads=4)
    s = pk.Solver(p, device=0)
    s.setup_physical_grid(img)
    cands = [(8, 4, 4, pk.SCHED_TILE_DIAGONALS), (4, 4, 4, pk.SCHED_TILE_DATAFLOW), (2, 3, 2, pk.SCHED_TILE_DIAGONALS)]
    chosen, ms = s.autotune(cands, sweeps=2)
    assert chosen in cands and all(m > 0 for m in ms)
    sch = s.schedule()
    assert (sch["TX"], sch["TY"], sch["TZ"], sch["launch"]) == chosen
    nodes = s.geometry_array("node_g")
    for _ in range(3):
        o.iterate(1)
        s.iterate(1)
    _compare_state(o, s, nodes)
    assert o.chk_converge() == s.chk_converge()
    s.close()


@pytest.mark.parametrize("nf", [6, 8])
def test_larger_velocity_sets_bit_exact(nf):
    """6 and 8 abscissae per axis (216 and 512 velocities per octant): the sweep on rows of
    other widths and the wall and moment kernels that loop over several velocity chunks,
    for both schedules; FP64 bit for bit against the oracle, FP32 within 1e-5 of it."""
    img = images.sphere_pack(10, 0.55, 1.2, 2.5, seed=4)
    p = base_params(10, Nc_fundamental=nf, Kn=0.3, pressDrop=0.1, fluidlayer=1)
    o = Oracle(p, img.tobytes(), nthreads=8)
    o.iterate(3)
    mo = o.chk_converge()
    for tiles in ((4, 4, 4), (0, 0, 0)):
        with pk.Solver(p, device=0) as s:
            s.set_tiles(*tiles)
            s.setup_physical_grid(img)
            s.iterate(3)
            nodes = s.geometry_array("node_g")
            _compare_state(o, s, nodes)
            assert s.chk_converge() == mo
    with pk.Solver(p, device=0) as s:
        s.set_precision(pk.PREC_FP32)
        s.setup_physical_grid(img)
        s.iterate(3)
        m32 = s.chk_converge()[0]
        nc8 = s.info()["Nc8"]
        nodes = s.geometry_array("node_g")
        fo = o.f().reshape(8, nc8, -1)[:, :, nodes]
        fs = s.get_f()[0].reshape(8, nc8, -1)[:, :, nodes]
        err = np.abs(fs - fo).max() / np.abs(fo).max()
        print("Nc_fundamental %d: FP32 after 3 iterations max |f32 - f64| / max |f64| = %.3e" % (nf, err))
        assert err <= 1e-5 and abs(m32 - mo[0]) / abs(mo[0]) <= 1e-5


def test_bench_workload_fp64_iterations_equal_oracle():
    """The benchmark's own configuration (128^3 sphere pack, porosity 0.40, radii 4-8, seed
    12345, 512 velocities, Kn = 0.5, wallExtOrder 1), two FP64 iterations through the C ABI
    against two oracle iterations: the chkConverge triple and the full-box Rho and U equal
    bit for bit, and so do f at 4096 seeded nodes (fluid and wall rows, all octants and
    velocities) and every 3-fold corner slot. The refined solver's errors in the bench are
    stated against this FP64 path."""
    import os
    import bench
    img = bench.workload_image()
    p = bench.workload_params(pk)
    o = Oracle(p, img.tobytes(), nthreads=os.cpu_count() or 8)
    s = pk.Solver(p, device=0)
    s.setup_physical_grid(img)
    assert np.array_equal(o.labels(), s.get_labels())
    o.iterate(2)
    s.iterate(2)
    assert o.chk_converge() == s.chk_converge()
    mo = o.macro()
    for a, b in zip(mo, s.get_macro()):
        assert np.array_equal(a[2:-2, 2:-2, 2:-2], b)
    inf = s.info()
    rng = np.random.default_rng(20261203)
    nodes = np.sort(rng.choice(inf["nNodes"], size=4096, replace=False)).astype(np.int32)
    gidx = s.geometry_array("node_g")[nodes]
    fs = s.get_f_nodes(nodes)
    fo = o.f_at(gidx)
    assert np.array_equal(fo, fs), "f differs: max %g" % np.abs(fo - fs).max()
    assert np.array_equal(o.fw(), s.get_fw())
    s.close()
    o.close()


@pytest.mark.parametrize("nf", [12, 16])
def test_velocity_sets_beyond_512_bit_exact(nf):
    """12 and 16 abscissae per axis (1728 and 4096 velocities per octant, 13,824 and 32,768
    in all; velocityGrid.F90:130-154), as CPC Table 3 uses at Kn >= 1, on a 6^3 pack: every
    kernel loops over 108 / 256 FP64 chunks; FP64 bit for bit against the oracle after two
    iterations, for the tile and the per-node schedules."""
    img = images.sphere_pack(6, 0.6, 1.0, 1.8, seed=21)
    p = base_params(6, Nc_fundamental=nf, Kn=2.0, pressDrop=0.1)
    o = Oracle(p, img.tobytes(), nthreads=8)
    o.iterate(2)
    mo = o.chk_converge()
    for tiles in ((2, 2, 2), (0, 0, 0)):
        with pk.Solver(p, device=0) as s:
            s.set_tiles(*tiles)
            s.setup_physical_grid(img)
            assert s.info()["Nc8"] == nf ** 3
            s.iterate(2)
            _compare_state(o, s, s.geometry_array("node_g"))
            assert s.chk_converge() == mo


@pytest.mark.parametrize("nf", [2, 4, 8])
def test_full_range_gauss_hermite_bit_exact(nf):
    """halfRange = F: the full-range Gauss-Hermite abscissae and weights
    (velocityGrid.F90:102-127) drive the sweep, walls and moments; FP64 bit for bit
    against the oracle after three iterations on a pack with every wall type."""
    img = images.sphere_pack(12, 0.5, 1.5, 3.0, seed=23)
    p = base_params(12, Nc_fundamental=nf, halfRange=0, Kn=0.8, pressDrop=0.5)
    o = Oracle(p, img.tobytes(), nthreads=8)
    s = pk.Solver(p, device=0)
    s.setup_physical_grid(img)
    cx = s.geometry_array("cx")
    assert np.array_equal(cx, o.velocity()[0])
    nodes = s.geometry_array("node_g")
    for _ in range(3):
        o.iterate(1)
        s.iterate(1)
        _compare_state(o, s, nodes)
        assert o.chk_converge() == s.chk_converge()
    s.close()
