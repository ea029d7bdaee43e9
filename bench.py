#!/usr/bin/env python
"""Benchmark of the B200 source-iteration solver (one JSON line on rank 0).

Workload (per rank): the 128^3 Boolean sphere pack (porosity 0.40, radii uniform in 4-8
voxels, seed 12345), 512 discrete velocities (Nc_fundamental = 4, half-range Gauss-Hermite),
Kn = 0.5, first-order wall extrapolation (wallExtOrder = 1, as in the reference's shipped
tutorials: with second-order extrapolation the scheme diverges on packs with one-voxel
channels). A step is one source iteration (8 octant sweeps, halo, walls, inlet/outlet,
symmetry, moments).

value: fluid voxel-velocity updates per second of the plain FP64 iteration (the reference's
arithmetic, operation for operation), whole job; the same for the refined solver's iteration
(FP32 sweep, FP64 moments / wall densities / flux) is in "fp32". "solve": both solvers run to
convergence at a 1e-4 permeability tolerance (solves/s, iterations, permeability difference,
velocity-field difference); "e2e" is the plain FP64 solve through the public API, host image
in to fields out ("solve.e2e_refined" the same for the refined solve).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-solve]

--impl reference times the CPU restatement of PIKS3D's own OpenMP solver (oracle/;
the reference itself is Fortran + MPI and cannot be built here) on the same workload
with all host threads, on rank 0 only. Under torchrun with N > 1 every rank solves its
own copy of the workload (independent solves, no collective on the data path) and the
time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import tempfile
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(n=128, porosity=0.40, rmin=4.0, rmax=8.0, seed=12345, Nc_fundamental=4, Kn=0.5, wallExtOrder=1)
METRIC = "solves/s + p99 latency vs plain FP64 GPU at 1e-4 perm error; Gvoxel-vel upd/s"
UNIT = "Gupd/s"
TOL = 1e-4


# the large single solve: a 256^3 Gaussian random field (correlation length 6 voxels)
# thresholded at porosity 0.20, x-percolating pore cluster kept, 512 velocities, Kn = 0.1
LARGE = dict(kind="grf", n=256, porosity=0.20, corr=6.0, seed=2024, Nc_fundamental=4, Kn=0.1, wallExtOrder=1)


def workload_image():
    from piks3d_b200 import images
    w = WORKLOAD
    if w.get("kind") == "grf":
        return images.gaussian_field(w["n"], w["porosity"], corr=w["corr"], seed=w["seed"])
    return images.sphere_pack(w["n"], w["porosity"], w["rmin"], w["rmax"], seed=w["seed"])


def workload_overrides():
    w = WORKLOAD
    return dict(Nx=w["n"], Ny=w["n"], Nz=w["n"], Nc_fundamental=w["Nc_fundamental"], Kn=w["Kn"], pressDrop=1.0,
                eps=1e-8, chkConvergeStep=10, maxStep=20000, wallExtOrder=w["wallExtOrder"])


def workload_params(pk):
    return pk.default_params(**workload_overrides())


# initParams' defaults (parameters.F90:91-98), as plain values: the reference arm hands these
# to the oracle without loading the product library
PARAM_DEFAULTS = dict(Nx=0, Ny=0, Nz=0, wallExtOrder=2, fluidlayer=0, Ref_L=1.0, Nc_fundamental=0, halfRange=1,
                      mpi_xdim=1, mpi_ydim=1, mpi_zdim=1, block_repx=1, block_repy=1, block_repz=1, maxStep=1000,
                      chkConvergeStep=10, saveStep=1 << 30, eps=1e-8, saveLast=1, saveFormat=1, Kn=0.0,
                      pressDrop=0.0, accom=1.0)


def workload_param_dict():
    d = dict(PARAM_DEFAULTS)
    d.update(workload_overrides())
    return d


def config_dict():
    w = WORKLOAD
    if w.get("kind") == "grf":
        name = "Gaussian random field %d^3 corr %g porosity %.2f (x-percolating cluster) seed %d, Nv=%d, Kn=%g, " \
               "wallExtOrder %d" % (w["n"], w["corr"], w["porosity"], w["seed"], 8 * w["Nc_fundamental"] ** 3, w["Kn"],
                                    w["wallExtOrder"])
    else:
        name = "sphere-pack %d^3 porosity %.2f radii %g-%g seed %d, Nv=%d, Kn=%g, wallExtOrder %d" % (
            w["n"], w["porosity"], w["rmin"], w["rmax"], w["seed"], 8 * w["Nc_fundamental"] ** 3, w["Kn"],
            w["wallExtOrder"])
    d = {"workload": name,
         "image": "%dx%dx%d uint8" % (w["n"], w["n"], w["n"]), "velocities": 8 * w["Nc_fundamental"] ** 3,
         "Kn": w["Kn"], "l2": "inputs larger than L2 (distribution function > 4 GB per rank)",
         "parallelism": "replicas (one independent solve per GPU)"}
    return d


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        # raw samples go to $PIKS_CLOCKS_DIR (default: the temporary directory); the JSON line
        # carries their summary
        out = os.environ.get("PIKS_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(out, "clocks_rank%d.csv" % gpu_index)

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "50"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        # wait (at most 5 s) until nvidia-smi writes, so that the timed region is sampled from
        # its start; stop() reads only the lines written after this point
        t0 = time.time()
        while time.time() - t0 < 5.0 and os.path.getsize(self.path) == 0 and self.proc.poll() is None:
            time.sleep(0.01)
        self.offset = os.path.getsize(self.path)

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            fh.seek(getattr(self, "offset", 0))
            lines = fh.read().splitlines()
        for line in lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        backend = "nccl" if args.impl == "ours" else "gloo"
        dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def reduce_max(value, world, device=None):
    if world == 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world, device=None):
    if world > 1:
        import torch.distributed as dist
        if device is not None:
            dist.barrier(device_ids=[device.index])
        else:
            dist.barrier()


def cpu_baseline(p, img, iters):
    """The oracle (CPU restatement of the reference's OpenMP solver) on this workload."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Oracle, build as obuild
    obuild()
    threads = os.cpu_count() or 1
    os.environ.setdefault("OMP_PROC_BIND", "close")
    o = Oracle(p, img.tobytes(), nthreads=threads)
    nf = o.dims()["Nfluid"]
    nv = 8 * o.dims()["Nc8"]
    o.iterate(1)  # warm-up (page faults of the 9 GB f array)
    t0 = time.perf_counter()
    o.iterate(iters)
    dt = time.perf_counter() - t0
    o.close()
    return {"value": nf * nv * iters / dt / 1e9, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "%d source iterations of the full workload after 1 warm-up (%.1f s)" % (iters, dt),
            "seconds_per_iteration": dt / iters}


def run_reference(args, world, rank):
    """The reference's algorithm on the host cores: the oracle (a line-by-line C++/OpenMP
    restatement of the Fortran solver, which cannot be built here) on this workload, in
    FP64. Loads only oracle/liboracle.so."""
    if rank != 0:
        return 0
    img = workload_image()
    p = workload_param_dict()
    iters = max(1, min(args.steps, 3))
    warm = 1
    cb = cpu_baseline(p, img, iters)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": iters,
            "warmup": warm, "ms_per_step": cb["seconds_per_iteration"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict(),
            "sample": "each step is a bounded sample: the CPU run times %d source iterations of the full "
                      "workload after 1 warm-up" % iters,
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": 0}
    print(json.dumps(line))
    return 0


def swept_updates(s):
    """Swept (node, octant) pairs per iteration: fluid nodes outside each octant's inflow planes."""
    fluid = s.get_labels() == 0
    swept = 0
    for sx in (1, -1):
        for sy in (1, -1):
            for sz in (1, -1):
                f = fluid[1:, :, :] if sz > 0 else fluid[:-1, :, :]
                f = f[:, 1:, :] if sy > 0 else f[:, :-1, :]
                f = f[:, :, 1:] if sx > 0 else f[:, :, :-1]
                swept += int(f.sum())
    return swept


def measure_iterations(pk, p, img, prec, args, world, local, device, clocks=None):
    """K timed iterations (after W warm-up) of one precision, as a user runs them (iteration
    graphs replayed), timed with CUDA events on the launching stream; then K more with the
    library's per-kernel events for the breakdown and the sweep's own duration."""
    import torch
    s = pk.Solver(p, device=local)
    s.set_precision(prec)
    s.setup_physical_grid(img)
    info = s.info()
    stream = torch.cuda.Stream(device=device)
    s.set_stream(stream.cuda_stream)
    esz = 4 if prec == pk.PREC_FP32 else 8
    nf, nc8 = info["Nfluid"], info["Nc8"]
    swept = swept_updates(s)
    sweep_bytes = 2 * esz * nc8 * swept + 32 * nf     # f read + write per swept update, moments read once
    s.iterate(args.warmup)
    s.synchronize()
    barrier(world, device)
    torch.cuda.synchronize()
    if clocks:
        clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    s.iterate(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop() if clocks else None
    s.synchronize()
    ms_local = ev0.elapsed_time(ev1)
    # per-kernel breakdown (plain launches with an event pair around each kernel group)
    s.enable_timing(True)
    s.kernel_times(reset=True)
    s.iterate(args.steps)
    s.synchronize()
    kt = s.kernel_times(reset=True)
    s.enable_timing(False)
    launches = s.launches_per_iteration() * args.steps
    sched = s.schedule()
    s.close()
    ms = reduce_max(ms_local, world, device)
    sweep_ms = kt["sweep"][0] / max(1, kt["sweep"][1])
    return {"info": info, "ms": ms, "kt": kt, "launches": launches, "clocks": clk, "swept": swept,
            "sweep_bytes": sweep_bytes, "sweep_ms": sweep_ms, "schedule": sched,
            "gupd": nf * 8 * nc8 * args.steps * world / (ms * 1e-3) / 1e9}


def traffic_per_update(precision):
    """DRAM bytes per swept voxel-velocity update of the sweep kernel, from the committed
    summary of an ncu capture (profiles/), or None."""
    try:
        d = json.load(open(os.path.join(ROOT, "profiles", "tile_sweep_traffic.json")))
        return d[precision]["dram_bytes_per_swept_update"]
    except Exception:
        return None


def roofline_of(m, hbm, peaks, tpu, nc8, kernel):
    achieved = m["sweep_bytes"] / (m["sweep_ms"] * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": (tpu * m["swept"] * nc8) if tpu else None,
            "kernel": kernel, "alg_bytes_per_iteration": m["sweep_bytes"],
            "sweep_ms_per_iteration": m["sweep_ms"],
            "peak_source": ("MEASURED_PEAKS.json hbm_gbs (of measured)" if "hbm_gbs" in peaks
                            else "fallback 6650 (of fallback)")}


def run_ours(args, world, rank, local):
    import numpy as np
    import torch
    import piks3d_b200 as pk
    from piks3d_b200.solve import solve_one

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    img = workload_image()
    p = workload_params(pk)

    # --- device-resident iterations: value (plain FP64 iteration, the reference's arithmetic),
    #     fp32 (the refined solver's FP32 iteration), rooflines of both sweeps
    clocks = ClockSampler(local)
    m64 = measure_iterations(pk, p, img, pk.PREC_FP64, args, world, local, device, clocks)
    m32 = measure_iterations(pk, p, img, pk.PREC_FP32, args, world, local, device)
    info = m64["info"]
    nf, nc8 = info["Nfluid"], info["Nc8"]
    nv = 8 * nc8

    # --- full solves through the public API (host image in, fields out) ------------------------
    solve = None
    e2e = None
    if not args.no_solve:
        torch.cuda.synchronize()
        barrier(world, device)
        t0 = time.perf_counter()
        r64 = solve_one(img, p, device=local, precision="fp64", tol=TOL, keep_fields=True)
        t64 = reduce_max(time.perf_counter() - t0, world, device)
        barrier(world, device)
        t0 = time.perf_counter()
        rrf = solve_one(img, p, device=local, precision="refined", tol=TOL, keep_fields=True)
        trf = reduce_max(time.perf_counter() - t0, world, device)
        u64, urf = r64.pop("macro"), rrf.pop("macro")
        num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(urf[1:], u64[1:]))
        den = sum(float(np.sum(b ** 2)) for b in u64[1:])
        solve = {
            "tolerance": TOL, "rule": "estimated distance of k to the iteration's limit <= tol/2, two checks in a row",
            "fp64": {**r64, "seconds": t64, "solves_per_s": world / t64},
            "refined": {**rrf, "seconds": trf, "solves_per_s": world / trf},
            "speedup_solves_per_s": t64 / trf,
            "errors_measured_against": "the plain FP64 GPU solve of the same image and parameters, whose "
                                       "iterations are bit-identical to the oracle's on this workload "
                                       "(tests/test_gpu_parity.py::test_bench_workload_fp64_iterations_equal_oracle)",
            "perm_rel_diff_refined_vs_fp64": abs(rrf["permeability"] - r64["permeability"]) / abs(r64["permeability"]),
            "velocity_rel_l2_diff_refined_vs_fp64": (num / den) ** 0.5,
        }
        box = info["Nx"] * info["Ny"] * info["Nz"]

        def e2e_of(r, t, what):
            st = r["steps"]
            return {"value": nf * nv * st * world / t / 1e9, "unit": UNIT,
                    "h2d_bytes_per_step": img.nbytes / st,
                    "d2h_bytes_per_step": (8 * st / p.chkConvergeStep + 4 * box * 8) / st, "seconds": t,
                    "setup_seconds": {"box_and_drill_thin": r["setup_seconds"][0],
                                      "voxel_classification_on_device": r["setup_seconds"][1],
                                      "rest_of_geometry": r["setup_seconds"][2],
                                      "whole_setup_call": r["setup_seconds"][3]},
                    "what": what + " solve through the public API: create + setup_physical_grid(host image) + "
                            "%d iterations with a check every %d + get_macro, wall clock" % (st, p.chkConvergeStep)}
        e2e = e2e_of(r64, t64, "plain FP64")
        solve["e2e_refined"] = e2e_of(rrf, trf, "refined (FP32 sweep, FP64 refinement)")

    batch = None
    if args.batch_images > 0:
        batch = small_batch(args, world, rank, local, device)

    if rank != 0:
        return 0
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    per_it = lambda m: {k: v[0] / max(1, args.steps) for k, v in m["kt"].items()}
    line = {
        "metric": METRIC, "value": m64["gupd"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": m64["ms"] / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": config_dict(),
        "workload_info": {"Nfluid": nf, "nWall": info["nWall"], "replicas": world, "schedule_fp64": m64["schedule"],
                          "schedule_fp32": m32["schedule"]},
        "roofline": roofline_of(m64, hbm, peaks, traffic_per_update("fp64"), nc8,
                                "FP64 octant sweep (all launches of one iteration's sweep)"),
        "kernel_ms_per_iteration": per_it(m64),
        "fp32": {"value": m32["gupd"], "unit": UNIT, "ms_per_step": m32["ms"] / args.steps,
                 "what": "the refined solver's iteration: FP32 sweep, FP64 moments, wall densities and flux",
                 "kernel_ms_per_iteration": per_it(m32),
                 "roofline": roofline_of(m32, hbm, peaks, traffic_per_update("fp32"), nc8,
                                         "FP32 octant sweep (all launches of one iteration's sweep)")},
        "solve": solve,
        "batch": batch,
        "e2e": e2e,
        "gpu_launches": m64["launches"],
        "clocks": m64["clocks"],
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(workload_param_dict(), img, args.cpu_iters)
    print(json.dumps(line))
    return 0


def batch_jobs(pk, count, seed, max_step, edges=(32, 48, 64, 80, 96), kn_range=(0.01, 10.0)):
    """The batching workload: seeded sphere packs, edges from {32, 48, 64, 80, 96}, porosity
    U[0.3, 0.6], Kn log-uniform in [0.01, 10], 64 or 512 velocities per sample."""
    import numpy as np
    from piks3d_b200 import images
    from piks3d_b200.solve import Job
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(count):
        n = int(rng.choice(list(edges)))
        por = float(rng.uniform(0.3, 0.6))
        kn = float(np.exp(rng.uniform(np.log(kn_range[0]), np.log(kn_range[1]))))
        ncf = int(rng.choice([2, 4]))
        img = images.sphere_pack(n, por, 4.0, 8.0, seed=seed * 1000 + i)
        p = pk.default_params(Nx=n, Ny=n, Nz=n, Nc_fundamental=ncf, Kn=kn, pressDrop=1.0, wallExtOrder=1,
                              maxStep=max_step, chkConvergeStep=10, eps=1e-8)
        jobs.append(Job(img, p, name="img%d" % i))
    return jobs


SMALL_BATCH = dict(edges=(32, 48, 64), kn_range=(0.3, 10.0), seed=77)


def small_batch(args, world, rank, local, device):
    """The reduced batching workload of the default line: `--batch-images` seeded sphere
    packs (edges 32-64, porosity U[0.3, 0.6], Kn log-uniform in [0.3, 10], 64 or 512
    velocities) solved to the 1e-4 permeability tolerance, plain FP64 one after another
    against the refined solver's batch runner (all images in flight together)."""
    import numpy as np
    import piks3d_b200 as pk
    from piks3d_b200.solve import BatchRunner, solve_one
    from piks3d_b200 import images
    from piks3d_b200.solve import Job
    sb = SMALL_BATCH
    # untimed warm-up of both arms: 20 iterations of a small pack per velocity set, plain and
    # batched in both precisions, so that neither timed arm pays the first use of a kernel
    warm = []
    for ncf in (2, 4):
        p = pk.default_params(Nx=24, Ny=24, Nz=24, Nc_fundamental=ncf, Kn=1.0, pressDrop=1.0, wallExtOrder=1,
                              maxStep=20, chkConvergeStep=10, eps=1e-8)
        warm.append((images.sphere_pack(24, 0.45, 4.0, 8.0, seed=4242 + ncf), p))
    for img, p in warm:
        solve_one(img, p, device=local, precision="fp64", tol=TOL)
    for prec in ("fp64", "fp32"):
        wr = BatchRunner(device=local, precision=prec, tol=TOL, max_members=2, autotune=False)
        wr.run([Job(img, p, name="warm%d" % i) for i, (img, p) in enumerate(warm)])
        wr.close()
    jobs = batch_jobs(pk, args.batch_images, sb["seed"] + rank, args.max_step, sb["edges"], sb["kn_range"])
    barrier(world, device)
    t0 = time.perf_counter()
    plain = [solve_one(j.image, j.params, device=local, precision="fp64", tol=TOL) for j in jobs]
    t_plain = reduce_max(time.perf_counter() - t0, world, device)
    runner = BatchRunner(device=local, precision="refined", tol=TOL, max_members=args.batch_images)
    barrier(world, device)
    t0 = time.perf_counter()
    done = runner.run(batch_jobs(pk, args.batch_images, sb["seed"] + rank, args.max_step, sb["edges"],
                                 sb["kn_range"]))
    t_batch = reduce_max(time.perf_counter() - t0, world, device)
    runner.close()
    by = {j.name: j.result for j in done}
    diffs = [abs(by[j.name]["permeability"] - p["permeability"]) / abs(p["permeability"]) for j, p in zip(jobs, plain)]
    return {"workload": "%d seeded sphere packs, edges %s, porosity U[0.3,0.6], Kn log-U[%g,%g], 64 or 512 velocities, "
                        "wallExtOrder 1, tolerance %g on k" % (args.batch_images, list(sb["edges"]), sb["kn_range"][0],
                                                              sb["kn_range"][1], TOL),
            "plain_fp64_sequential": {"seconds": t_plain, "solves_per_s": args.batch_images * world / t_plain,
                                      "iterations": sum(p["steps"] for p in plain)},
            "refined_batched": {"seconds": t_batch, "solves_per_s": args.batch_images * world / t_batch,
                                "iterations": sum(r["steps"] for r in by.values()),
                                "converged": sum(1 for r in by.values() if r["converged"])},
            "speedup_solves_per_s": t_plain / t_batch,
            "perm_rel_diff_refined_vs_fp64": {"max": max(diffs), "median": float(np.median(diffs))},
            "autotuned_tiles": sorted({str(r.get("tiles")) for r in by.values()})}


def run_batch_workload(args, world, rank, local):
    """Many images: plain FP64 solves one after another vs the refined solver's batch runner,
    both to the 1e-4 permeability tolerance; solves/s of each and the permeability
    differences per image."""
    import numpy as np
    import torch
    import piks3d_b200 as pk
    from piks3d_b200.solve import BatchRunner, solve_one
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    jobs = batch_jobs(pk, args.images, args.seed + rank, args.max_step)
    barrier(world, device)
    t0 = time.perf_counter()
    plain = [solve_one(j.image, j.params, device=local, precision="fp64", tol=TOL) for j in jobs]
    t_plain = reduce_max(time.perf_counter() - t0, world, device)
    runner = BatchRunner(device=local, precision="refined", tol=TOL, max_members=args.images)
    barrier(world, device)
    t0 = time.perf_counter()
    done = runner.run(batch_jobs(pk, args.images, args.seed + rank, args.max_step))
    t_batch = reduce_max(time.perf_counter() - t0, world, device)
    runner.close()
    if rank != 0:
        return 0
    by = {j.name: j.result for j in done}
    diffs = [abs(by[j.name]["permeability"] - p["permeability"]) / abs(p["permeability"]) for j, p in zip(jobs, plain)]
    steps_plain = sum(p["steps"] for p in plain)
    line = {
        "metric": METRIC, "workload": "batch", "value": args.images * world / t_batch, "unit": "solves/s",
        "n_gpus": world, "higher_is_better": True, "scaling": "weak", "data": "synthetic",
        "config": {"workload": "%d seeded sphere packs, edges {32..96}, porosity U[0.3,0.6], Kn log-U[0.01,10], "
                               "64 or 512 velocities, wallExtOrder 1, tolerance %g on k" % (args.images, TOL)},
        "plain_fp64_sequential": {"seconds": t_plain, "solves_per_s": args.images * world / t_plain,
                                  "iterations": steps_plain,
                                  "converged": sum(1 for p in plain if p["converged"])},
        "refined_batched": {"seconds": t_batch, "solves_per_s": args.images * world / t_batch,
                            "iterations": sum(r["steps"] for r in by.values()),
                            "fp32_iterations": sum(r["steps32"] for r in by.values()),
                            "converged": sum(1 for r in by.values() if r["converged"])},
        "speedup_solves_per_s": t_plain / t_batch,
        "perm_rel_diff_refined_vs_fp64": {"max": max(diffs), "median": float(np.median(diffs))},
        "images": [{"name": j.name, "n": int(j.image.shape[0]), "velocities": 8 * j.params.Nc_fundamental ** 3,
                    "Kn": j.params.Kn, "porosity": float((j.image == 0).mean()),
                    "fp64_steps": p["steps"], "fp64_k": p["permeability"],
                    "refined_steps": by[j.name]["steps"], "refined_fp32_steps": by[j.name]["steps32"],
                    "refined_k": by[j.name]["permeability"]} for j, p in zip(jobs, plain)],
    }
    print(json.dumps(line))
    return 0


def run_slab_workload(args, world, rank, local):
    """One image over `world` GPUs as x slabs (strong scaling; the reference's MPI
    decomposition with mpi_xdim = world): the 128^3 workload's FP64 and FP32 iterations,
    each rank a SlabSolver, the halos moved by NCCL point-to-point calls on the context's
    stream between iterations; value = the whole box's voxel-velocity updates/s (time =
    max over ranks, CUDA events on the launching stream). On one GPU it also times the same
    box cut into 2 and 4 slab contexts sharing the device (block-Jacobi in x: the slabs'
    sweeps run concurrently, the halos one iteration behind)."""
    import torch
    import torch.distributed as dist
    import piks3d_b200 as pk
    from piks3d_b200.slab import LocalSlabs, SlabSolver
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    img = workload_image()
    p = workload_params(pk)
    out = {}
    for prec in ("fp64", "fp32"):
        ss = SlabSolver(p, img, device=local, precision=prec)
        nf = ss.solver.info()["Nfluid"]
        if world > 1:
            t = torch.tensor([nf], dtype=torch.int64, device=device)
            dist.all_reduce(t)
            nf = int(t.item())
        nv = 8 * ss.solver.info()["Nc8"]
        ss.iterate(args.warmup)
        torch.cuda.synchronize()
        barrier(world, device)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(ss.stream)
        ss.iterate(args.steps)
        ev1.record(ss.stream)
        torch.cuda.synchronize()
        ms = reduce_max(ev0.elapsed_time(ev1), world, device)
        m, k, e = ss.chk_converge()
        sl = ss.solver.slab()
        ss.close()
        out[prec] = {"value": nf * nv * args.steps / (ms * 1e-3) / 1e9, "unit": UNIT,
                     "ms_per_step": ms / args.steps, "mass_after": m, "slab_of_rank0": [sl["xl"], sl["xu"]]}
    emulated = None
    if world == 1:
        emulated = {}
        for n in (1, 2, 4):
            row = {}
            for prec in ("fp64", "fp32"):
                ls = LocalSlabs(p, img, n, devices=(local,), precision=prec)
                ls.iterate(args.warmup)
                torch.cuda.synchronize()
                t0 = time.perf_counter()
                ls.iterate(args.steps)
                for s_ in ls.solvers:
                    s_.synchronize()
                row[prec + "_ms_per_step"] = (time.perf_counter() - t0) * 1e3 / args.steps
                ls.close()
            emulated["%d_slabs" % n] = row
    if rank != 0:
        return 0
    line = {"metric": METRIC, "workload": "slab", "value": out["fp64"]["value"], "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": out["fp64"]["ms_per_step"],
            "higher_is_better": True, "scaling": "strong", "dtype": "f64", "data": "synthetic",
            "config": {**config_dict(), "parallelism": "x slabs, one per GPU (halo exchange by NCCL send / recv)"},
            "fp32": out["fp32"], "fp64": out["fp64"],
            "emulated_ranks_one_gpu": emulated}
    print(json.dumps(line))
    return 0


def run_serve_workload(args, world, rank, local):
    """The serving workload: a seeded Poisson request stream through the server."""
    import torch
    import piks3d_b200 as pk
    from piks3d_b200.serve import Server, make_stream
    from piks3d_b200.solve import BatchRunner
    torch.cuda.set_device(local)

    def params(n, kn):
        return pk.default_params(Nx=n, Ny=n, Nz=n, Nc_fundamental=4, Kn=kn, pressDrop=1.0, wallExtOrder=1,
                                 maxStep=args.max_step, chkConvergeStep=10, eps=1e-8)

    jobs = make_stream(args.rate, args.duration, args.seed + rank, params,
                       edge_range=(args.edge_min, args.edge_max))
    runner = BatchRunner(device=local, precision="refined", tol=TOL, max_members=64)
    rep = Server(runner, horizon=args.horizon).run(jobs)
    runner.close()
    if rank != 0:
        return 0
    rep.pop("jobs")
    line = {"metric": METRIC, "workload": "serve", "value": rep["solves_per_s"], "unit": "solves/s",
            "n_gpus": world, "higher_is_better": True, "data": "synthetic",
            "config": {"workload": "Poisson %g req/s for %g s, sphere packs edges %d-%d, porosity U[0.25,0.6], "
                                   "Kn log-U[0.01,10], 512 velocities, tolerance %g on k, horizon %g s" % (
                                       args.rate, args.duration, args.edge_min, args.edge_max, TOL, args.horizon)},
            **rep}
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-iters", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-solve", action="store_true", help="skip the full solves (solve / e2e blocks)")
    ap.add_argument("--batch-images", type=int, default=12,
                    help="images of the reduced batching workload in the default line (0: skip)")
    ap.add_argument("--workload", default="precision", choices=["precision", "batch", "serve", "large", "slab"],
                    help="precision: the 128^3 pack (default); batch: many images; serve: request stream; "
                         "large: the 256^3 Gaussian random field (add --solve-large for the full solves); "
                         "slab: the 128^3 pack decomposed over the GPUs as x slabs (strong scaling)")
    ap.add_argument("--solve-large", action="store_true")
    ap.add_argument("--images", type=int, default=64)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--max-step", type=int, default=20000)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--duration", type=float, default=60.0)
    ap.add_argument("--horizon", type=float, default=240.0)
    ap.add_argument("--edge-min", type=int, default=48)
    ap.add_argument("--edge-max", type=int, default=160)
    ap.add_argument("--edge", "--n", dest="n", type=int, default=None,
                    help="image edge (default 128); smaller edges are for profiling captures, not bench lines")
    args = ap.parse_args()
    if args.workload == "large":
        WORKLOAD.clear()
        WORKLOAD.update(LARGE)
        args.no_solve = args.no_solve or not args.solve_large
        args.workload = "precision"
    if args.no_solve:
        args.batch_images = 0
    if args.n:
        WORKLOAD["n"] = args.n
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            rc = run_reference(args, world, rank)
        elif args.workload == "batch":
            rc = run_batch_workload(args, world, rank, local)
        elif args.workload == "serve":
            rc = run_serve_workload(args, world, rank, local)
        elif args.workload == "slab":
            rc = run_slab_workload(args, world, rank, local)
        else:
            rc = run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
