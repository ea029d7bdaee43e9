"""CPU tests of the product's host side: C ABI exports, parameter reading, error codes,
image preprocessing (labels identical to the oracle) and the device data flow (numpy
model over the library's exported geometry, bit-identical to the oracle)."""
import ctypes
import os
import re

import numpy as np
import pytest

import piks3d_b200 as pk
from piks3d_b200 import images
from conftest import ROOT, base_params
from device_model import DeviceModel
from oracle import Oracle


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(ROOT, "include", "piks3d_gpu.h")).read()
    names = set(re.findall(r"^\s*(?:piks_status|const char \*)\s*(piks_\w+)\s*\(", hdr, re.M))
    assert len(names) >= 20
    lib = ctypes.CDLL(pk.LIB_PATH)
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_read_params_reference_format(tmp_path):
    txt = """&physicalNml
imageFileName = 'singleSphere100^3.raw'
Nx = 100
Ny = 100
Nz = 100
wallExtOrder = 1
fluidLayer = 0
Ref_L = 1.d0
/

&velocityNml
Nc_fundamental = 4
halfRange = T
/

&mpiNml
mpi_xdim = 2
mpi_ydim = 2
mpi_zdim = 1
/

&solverNml
maxStep = 100
chkConvergeStep = 10
saveStep = 50
eps = 1.0d-7
saveLast = T
saveFormat = 1
/

&flowNml
Kn = 1.0d-1
pressDrop = 1.0d-1
accom = 1.d0
/
"""
    f = tmp_path / "para.in"
    f.write_text(txt)
    p, image = pk.read_params(str(f))
    assert image == "singleSphere100^3.raw"
    assert (p.Nx, p.Ny, p.Nz, p.wallExtOrder, p.fluidlayer) == (100, 100, 100, 1, 0)
    assert p.Nc_fundamental == 4 and p.halfRange == 1 and p.mpi_xdim == 2
    assert (p.maxStep, p.chkConvergeStep, p.saveStep, p.saveLast, p.saveFormat) == (100, 10, 50, 1, 1)
    assert p.eps == 1.0e-7 and p.Kn == 0.1 and p.pressDrop == 0.1 and p.accom == 1.0
    assert p.block_repx == 1 and p.Ref_L == 1.0


def test_error_codes(tmp_path):
    with pytest.raises(pk.PiksError) as e:
        pk.read_params(str(tmp_path / "missing.in"))
    assert e.value.status == 7
    with pytest.raises(pk.PiksError) as e:
        pk.Solver(base_params(8, Nc_fundamental=3), device=-1)
    assert e.value.status == 2
    s = pk.Solver(base_params(8), device=-1)
    bad = np.zeros((8, 8, 8), np.uint8)
    bad[3, 3, 3] = 7
    with pytest.raises(pk.PiksError) as e:
        s.setup_physical_grid(bad)
    assert e.value.status == 3
    with pytest.raises(pk.PiksError) as e:
        s.setup_physical_grid(np.zeros(100, np.uint8))
    assert e.value.status == 3
    s.setup_physical_grid(np.zeros((8, 8, 8), np.uint8))
    with pytest.raises(pk.PiksError) as e:
        s.iterate(1)
    assert e.value.status == 8


@pytest.mark.parametrize("n,por,seed,kw", [
    (24, 0.5, 1, {}), (20, 0.35, 2, dict(fluidlayer=2)), (18, 0.6, 3, dict(block_repx=2, block_repz=2)),
    (16, 0.45, 4, dict(wallExtOrder=3)),
])
def test_preprocessing_matches_oracle(n, por, seed, kw):
    img = images.sphere_pack(n, por, 1.2, 4.0, seed=seed)
    p = base_params(n, **kw)
    o = Oracle(p, img.tobytes(), nthreads=2)
    s = pk.Solver(p, device=-1)
    s.setup_physical_grid(img)
    assert np.array_equal(o.labels(), s.get_labels())
    d, inf = o.dims(), s.info()
    assert (d["Nfluid"], d["nWall"], d["nCorner"]) == (inf["Nfluid"], inf["nWall"], inf["nCorner"])
    # vecWall order and extrapolation coefficients
    wn = s.geometry_array("wall_node")
    ng = s.geometry_array("node_g")
    assert np.array_equal(o.vecwall() - 1, ng[wn])
    assert np.array_equal(o.extcoef().T.reshape(-1), s.geometry_array("wall_e"))


def test_velocity_grid_matches_oracle():
    for nc in (2, 4, 6, 8, 12, 16):
        for half in (1, 0):
            p = base_params(6, Nc_fundamental=nc, halfRange=half)
            s = pk.Solver(p, device=-1)
            o = Oracle(p, np.zeros(216, np.uint8).tobytes(), nthreads=1)
            for a, name in zip(o.velocity(), ("cx", "cy", "cz", "w")):
                assert np.array_equal(a, s.geometry_array(name)), (nc, half, name)


@pytest.mark.parametrize("n,por,seed,kw", [
    (12, 0.5, 11, dict(Kn=0.7)), (12, 0.4, 12, dict(wallExtOrder=1, accom=0.8)),
    (11, 0.45, 13, dict(wallExtOrder=3, fluidlayer=1)), (9, 0.6, 14, dict(Nc_fundamental=4, Kn=0.3, pressDrop=0.1)),
])
def test_device_model_bit_exact(n, por, seed, kw):
    img = images.sphere_pack(n, por, 1.2, 3.0, seed=seed)
    p = base_params(n, **kw)
    o = Oracle(p, img.tobytes(), nthreads=1)
    s = pk.Solver(p, device=-1)
    s.setup_physical_grid(img)
    m = DeviceModel(s, p)
    nodes = m.node_g
    for _ in range(3):
        o.iterate(1)
        m.iterate(1)
        fo = o.f().reshape(8, m.Nc8, -1)[:, :, nodes]
        fm = m.f_reference_layout().reshape(8, m.Nc8, -1)[:, :, nodes]
        assert np.array_equal(fo, fm)
        assert o.chk_converge()[0] == m.mass_flux()


@pytest.mark.parametrize("n,por,seed,tiles,kw", [
    (12, 0.5, 11, (8, 8, 8), dict(Kn=0.7)),
    (13, 0.45, 21, (4, 3, 5), dict(wallExtOrder=1)),
    (11, 0.45, 13, (2, 2, 2), dict(wallExtOrder=3, fluidlayer=1)),
    (9, 0.6, 14, (5, 4, 3), dict(Nc_fundamental=4, Kn=0.3, pressDrop=0.1)),
])
def test_tile_schedule_bit_exact(n, por, seed, tiles, kw):
    """The tile-wavefront schedule (rows copied per job at the start of its diagonal, local
    hyperplanes on the copies) gives the oracle's values bit for bit."""
    img = images.sphere_pack(n, por, 1.2, 3.0, seed=seed)
    p = base_params(n, **kw)
    o = Oracle(p, img.tobytes(), nthreads=1)
    s = pk.Solver(p, device=-1)
    s.set_tiles(*tiles)
    s.setup_physical_grid(img)
    sch = s.schedule()
    assert sch["tiles"] and (sch["TX"], sch["TY"], sch["TZ"]) == tiles
    m = DeviceModel(s, p)
    nodes = m.node_g
    for _ in range(2):
        o.iterate(1)
        m.iterate(1, schedule="tiles", solver=s)
        fo = o.f().reshape(8, m.Nc8, -1)[:, :, nodes]
        fm = m.f_reference_layout().reshape(8, m.Nc8, -1)[:, :, nodes]
        assert np.array_equal(fo, fm)
        assert o.chk_converge()[0] == m.mass_flux()


@pytest.mark.parametrize("schedule", ["columns", "pipelined"])
@pytest.mark.parametrize("n,por,seed,tiles,kw,arena", [
    (12, 0.5, 11, (4, 4, 4), dict(Kn=0.7), 1.0),
    (13, 0.45, 21, (4, 3, 5), dict(wallExtOrder=1), 1.5),
    (11, 0.45, 13, (2, 2, 2), dict(wallExtOrder=3, fluidlayer=1), 1.0),
    (9, 0.6, 14, (5, 4, 3), dict(Nc_fundamental=4, Kn=0.3, pressDrop=0.1), 2.0),
    (14, 0.5, 15, (8, 4, 4), dict(Kn=0.5, fluidlayer=2), 1.2),
])
def test_column_schedule_bit_exact(n, por, seed, tiles, kw, arena, schedule):
    """The split forms of the tile schedule, run as the producer / consumer kernel runs them
    (column march: rows carried between the tiles of a column; pipelined: every upwind row
    staged; regions in an arena of `arena` times the largest region, dependent rows read
    after their jobs), give the oracle's values bit for bit, and every slot, cell and count
    stays inside the kernel's shared-memory bounds."""
    img = images.sphere_pack(n, por, 1.2, 3.0, seed=seed)
    p = base_params(n, **kw)
    o = Oracle(p, img.tobytes(), nthreads=1)
    s = pk.Solver(p, device=-1)
    s.set_tiles(*tiles)
    s.set_schedule(pk.SCHED_TILE_COLUMNS if schedule == "columns" else pk.SCHED_TILE_PIPELINED)
    s.setup_physical_grid(img)
    info = s.geometry_array("tile_column_info")
    if schedule == "columns":
        assert info[0] == 1 and info[1] == 2 * tiles[0] * tiles[1]
    else:
        assert info[0] == 2 and info[1] == 0
    m = DeviceModel(s, p)
    nodes = m.node_g
    for _ in range(2):
        o.iterate(1)
        m.iterate(1, schedule="columns", solver=s, arena_rows=int(arena * info[2]))
        fo = o.f().reshape(8, m.Nc8, -1)[:, :, nodes]
        fm = m.f_reference_layout().reshape(8, m.Nc8, -1)[:, :, nodes]
        assert np.array_equal(fo, fm)
        assert o.chk_converge()[0] == m.mass_flux()


def test_tile_jobs_cover_every_task_once():
    img = images.sphere_pack(16, 0.45, 1.5, 3.5, seed=3)
    p = base_params(16)
    s = pk.Solver(p, device=-1)
    s.setup_physical_grid(img)
    t = s.geometry_array("tasks").reshape(-1, 8)
    tt = s.geometry_array("tile_tasks").reshape(-1, 4)
    rows, rbeg, tbeg = s.geometry_array("tile_rows"), s.geometry_array("tile_row_begin"), s.geometry_array("tile_task_begin")
    own = []
    for j in range(len(tbeg) - 1):
        own.extend(rows[rbeg[j]:rbeg[j] + (tbeg[j + 1] - tbeg[j])])
    assert sorted(own) == sorted((t[:, 0] * 8 + (t[:, 1] & 7)).tolist())
    assert len(tt) == len(t)
    rows_per_job = s.geometry_array("tile_row_count") + 1
    assert np.all(rbeg % 4 == 0) and np.all(np.diff(rbeg) >= rows_per_job - 1)
    # launch plan: every job once, one diagonal per launch, launch sized for its jobs
    jl = s.geometry_array("tile_job_list")
    L = s.geometry_array("tile_launches").reshape(-1, 4)
    dbeg = s.geometry_array("tile_diag_begin")
    assert sorted(jl.tolist()) == list(range(len(rbeg) - 1))
    ntask = np.diff(tbeg)
    for first, count, slots, tmax in L:
        jobs = jl[first:first + count]
        diag = np.searchsorted(dbeg, jobs, side="right") - 1
        assert count > 0 and np.all(diag == diag[0])
        assert slots >= rows_per_job[jobs].max() and tmax >= ntask[jobs].max()
    assert s.schedule()["max_slots"] == rows_per_job.max()


def test_wall_programs_read_no_slot_an_earlier_write_stores():
    """The wall kernels load the sources of up to four re-emission writes before storing
    them; that is only valid because no write of a program reads a slot that an earlier
    write of the same program stores."""
    from device_model import wall_programs
    for lab, (faces, writes) in wall_programs().items():
        stored = set()
        for dst_st, dst_o, fi, src_st, src_o in writes:
            assert (src_st, src_o) not in stored, lab
            stored.add((dst_st, dst_o))


INCOMING = [(2, 3, 6, 7), (1, 4, 5, 8), (3, 4, 7, 8), (1, 2, 5, 6), (5, 6, 7, 8), (1, 2, 3, 4)]


def test_wall_program_sources_are_face_values():
    """The on-chip wall kernels take every re-emission source from the wall's own face
    extrapolations and store a face value only where no write replaces it. Valid because,
    in every program, each source (store, octant) is produced by exactly one face, and no
    two writes share a destination."""
    from device_model import wall_programs
    progs = wall_programs()
    assert len(progs) == 26
    for lab, (faces, writes) in progs.items():
        produced = {}
        for fi, (d, st) in enumerate(faces):
            for m, o in enumerate(INCOMING[d]):
                produced.setdefault((st, o), []).append(fi * 4 + m)
        dsts = [(w[0], w[1]) for w in writes]
        assert len(set(dsts)) == len(dsts), lab
        for dst_st, dst_o, fi, src_st, src_o in writes:
            assert len(produced.get((src_st, src_o), [])) == 1, (lab, src_st, src_o)
            assert dst_st != 1, lab  # writes go to the slots or the corner array


def _tile_jobs_model(s, TX, TY, TZ):
    """The tile schedule restated in Python from its contract: jobs are the non-empty
    (tile, octant) pairs ordered by (tile diagonal of the octant's frame, octant, tile index);
    a job's tasks are ordered by local hyperplane (step), then by their index in the per-node
    task list; its rows are its own rows in task order, then every other row in the order
    its tasks first read them (slot = 1 + position, 0 = the zero row); each job's row list is
    padded with zeros to a multiple of 4; steps hold the task offset of each local
    hyperplane; up holds the jobs of the upwind neighbour tiles (same octant) or -1."""
    inf = s.info()
    Nx, Ny, Nz = inf["Nx"], inf["Ny"], inf["Nz"]
    GX, GY = Nx + 4, Ny + 4
    t = s.geometry_array("tasks").reshape(-1, 8).astype(np.int64)
    node_g = s.geometry_array("node_g").astype(np.int64)
    nrows_h = inf["nNodes"] * 8
    nTx, nTy, nTz = -(-Nx // TX), -(-Ny // TY), -(-Nz // TZ)
    sx = lambda o: 1 if o in (0, 3, 4, 7) else -1
    sy = lambda o: 1 if o in (0, 1, 4, 5) else -1
    sz = lambda o: 1 if o < 4 else -1
    keys = []
    for i, r in enumerate(t):
        o = int(r[1]) & 7
        gi = int(node_g[r[0]])
        x, y, z = gi % GX - 2, (gi // GX) % GY - 2, gi // (GX * GY) - 2
        a, b, c = x // TX, y // TY, z // TZ
        diag = (a if sx(o) > 0 else nTx - 1 - a) + (b if sy(o) > 0 else nTy - 1 - b) + (c if sz(o) > 0 else nTz - 1 - c)
        u = x - a * TX if sx(o) > 0 else min((a + 1) * TX, Nx) - 1 - x
        v = y - b * TY if sy(o) > 0 else min((b + 1) * TY, Ny) - 1 - y
        w = z - c * TZ if sz(o) > 0 else min((c + 1) * TZ, Nz) - 1 - z
        keys.append((diag * 8 + o, a + nTx * (b + nTy * c), u + v + w, i))
    keys.sort()
    nsteps = TX + TY + TZ - 2
    stride = (nsteps + 1 + 7) // 8 * 8
    ndiag = nTx + nTy + nTz - 2
    rows, row_begin, row_count, tasks, task_begin, steps = [], [], [], [], [], []
    diag_begin = [0] * (ndiag + 1)
    job_of, job_key = {}, []
    q = 0
    while q < len(keys):
        e = q
        while e < len(keys) and keys[e][:2] == keys[q][:2]:
            e += 1
        j = len(row_begin)
        dio, tile = keys[q][:2]
        job_of[(tile, dio % 8)] = j
        job_key.append((tile, dio % 8))
        row_begin.append(len(rows))
        task_begin.append(len(tasks) // 4)
        slot, mine = {}, []
        for k in range(q, e):
            r = t[keys[k][3]]
            own = int(r[0]) * 8 + (int(r[1]) & 7)
            slot[own] = len(mine) + 1
            mine.append(own)
        for k in range(q, e):
            r = t[keys[k][3]]
            sl = []
            for code in (int(x) for x in r[2:8]):
                if code < 0:
                    sl.append(0)
                    continue
                idx = nrows_h + (code & ~(1 << 30)) if code & (1 << 30) else code
                if idx not in slot:
                    slot[idx] = len(mine) + 1
                    mine.append(code)
                sl.append(slot[idx])
            fl = int(r[1])
            tasks += [int(r[0]) | (1 << 27 if fl & 8 else 0) | (1 << 28 if fl & 16 else 0) | (1 << 29 if fl & 32 else 0),
                      sl[0] | sl[1] << 16, sl[2] | sl[3] << 16, sl[4] | sl[5] << 16]
        row_count.append(len(mine))
        rows += mine + [0] * (-len(mine) % 4)
        st = [0] * stride
        for k in range(q, e):
            st[keys[k][2] + 1] += 1
        for h in range(nsteps):
            st[h + 1] += st[h]
        steps += st
        diag_begin[dio // 8 + 1] = j + 1
        q = e
    row_begin.append(len(rows))
    task_begin.append(len(tasks) // 4)
    for d in range(ndiag):
        diag_begin[d + 1] = max(diag_begin[d + 1], diag_begin[d])
    up = []
    for tile, o in job_key:
        a, b, c = tile % nTx, (tile // nTx) % nTy, tile // (nTx * nTy)
        for na, nb, nc in ((a - sx(o), b, c), (a, b - sy(o), c), (a, b, c - sz(o))):
            ok = 0 <= na < nTx and 0 <= nb < nTy and 0 <= nc < nTz
            up.append(job_of.get((na + nTx * (nb + nTy * nc), o), -1) if ok else -1)
        up.append(-1)
    return dict(tile_rows=rows, tile_row_begin=row_begin, tile_row_count=row_count, tile_tasks=tasks,
                tile_task_begin=task_begin, tile_steps=steps, tile_diag_begin=diag_begin, tile_up=up)


@pytest.mark.parametrize("tiles,kw", [((4, 4, 4), {}), ((8, 4, 4), dict(fluidlayer=2)), ((4, 3, 5), dict(wallExtOrder=1))])
def test_tile_jobs_match_their_contract(tiles, kw):
    img = images.sphere_pack(14, 0.45, 1.5, 3.5, seed=5)
    p = base_params(14, **kw)
    s = pk.Solver(p, device=-1)
    s.set_tiles(*tiles)
    s.setup_physical_grid(img)
    model = _tile_jobs_model(s, *tiles)
    for name, want in model.items():
        got = s.geometry_array(name)
        assert np.array_equal(got.astype(np.int64), np.array(want, dtype=np.int64)), name


@pytest.mark.parametrize("n,kw", [(14, {}), (12, dict(fluidlayer=2)), (13, dict(block_repx=2))])
def test_sweep_tasks_follow_their_order(n, kw):
    """The per-node sweep tasks (generated one thread per octant) are ordered by the
    hyperplane index u+v+w of their octant's frame, then by octant, then by voxel in raster
    order; hyper_start gives each hyperplane's first task; every swept (fluid node, octant)
    appears once."""
    img = images.sphere_pack(n, 0.45, 1.5, 3.5, seed=11)
    p = base_params(n, **kw)
    s = pk.Solver(p, device=-1)
    s.setup_physical_grid(img)
    inf = s.info()
    Nx, Ny, Nz = inf["Nx"], inf["Ny"], inf["Nz"]
    GX, GY = Nx + 4, Ny + 4
    t = s.geometry_array("tasks").reshape(-1, 8).astype(np.int64)
    hs = s.geometry_array("hyper_start").astype(np.int64)
    gi = s.geometry_array("node_g").astype(np.int64)[t[:, 0]]
    i, j, k = gi % GX - 1, (gi // GX) % GY - 1, gi // (GX * GY) - 1   # 1-based voxel indices
    o = t[:, 1] & 7
    sx = np.where(np.isin(o, (0, 3, 4, 7)), 1, -1)
    sy = np.where(np.isin(o, (0, 1, 4, 5)), 1, -1)
    sz = np.where(o < 4, 1, -1)
    u = np.where(sx > 0, i - 1, Nx - i)
    v = np.where(sy > 0, j - 1, Ny - j)
    w = np.where(sz > 0, k - 1, Nz - k)
    assert np.all((u >= 1) & (v >= 1) & (w >= 1))     # inflow planes are not swept
    h = u + v + w - 3
    key = np.stack([h, o, gi], axis=1)
    assert np.all(np.diff(key[:, 0]) >= 0)
    same_h = np.diff(key[:, 0]) == 0
    assert np.all(np.diff(key[:, 1])[same_h] >= 0)
    same_ho = same_h & (np.diff(key[:, 1]) == 0)
    assert np.all(np.diff(key[:, 2])[same_ho] > 0)
    assert np.array_equal(hs[:-1], np.searchsorted(h, np.arange(len(hs) - 1)))
    assert hs[-1] == len(t)
    assert len(np.unique(t[:, 0] * 8 + o)) == len(t)


@pytest.mark.timeout(120)
def test_oversized_tiles_fall_back_to_the_node_schedule():
    """A tile shape whose jobs need more shared-memory rows than a block holds (here 16^3
    tiles, whose own rows alone exceed the row set's capacity) is rejected while the jobs are
    built, and the context falls back to the per-node hyperplane schedule."""
    img = images.sphere_pack(20, 0.45, 1.5, 3.0, seed=8)
    s = pk.Solver(base_params(20, wallExtOrder=1), device=-1)
    s.set_tiles(16, 16, 16)
    s.setup_physical_grid(img)
    assert s.schedule()["tiles"] is False
    s.close()
