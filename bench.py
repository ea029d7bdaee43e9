#!/usr/bin/env python
"""Benchmark of the B200 source-iteration solver (one JSON line on rank 0).

Workload (N = 1, per rank): the 128^3 Boolean sphere pack (porosity 0.40, radii uniform
in 4-8 voxels, seed 12345) with two fluid layers at inlet and outlet (fluidlayer = 2: with
walls next to the periodic inlet/outlet planes the scheme's second-order wall
extrapolation diverges), 512 discrete velocities (Nc_fundamental = 4, half-range
Gauss-Hermite), Kn = 0.5, plain FP64 solve (--precision fp32: FP32 sweep). A step is one source iteration (8 octant
sweeps, halo, wall, inlet/outlet and symmetry boundary conditions, moments). The metric
is fluid voxel-velocity updates per second (N_fluid * Nv per iteration), whole job.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the CPU restatement of PIKS3D's own OpenMP solver (oracle/,
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
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = dict(n=128, porosity=0.40, rmin=4.0, rmax=8.0, seed=12345, Nc_fundamental=4, Kn=0.5, fluidlayer=2)
METRIC = "fluid voxel-velocity updates/s (plain FP64 source iteration)"
UNIT = "Gupd/s"


def workload_image():
    from piks3d_b200 import images
    w = WORKLOAD
    return images.sphere_pack(w["n"], w["porosity"], w["rmin"], w["rmax"], seed=w["seed"])


def workload_params(pk):
    w = WORKLOAD
    return pk.default_params(Nx=w["n"], Ny=w["n"], Nz=w["n"], Nc_fundamental=w["Nc_fundamental"],
                             Kn=w["Kn"], pressDrop=1.0, eps=1e-8, chkConvergeStep=10, maxStep=100000,
                             fluidlayer=w["fluidlayer"])


def config_dict(extra=None):
    w = WORKLOAD
    d = {"workload": "sphere-pack %d^3 porosity %.2f radii %g-%g seed %d, fluidlayer %d, Nv=%d, Kn=%g" % (
        w["n"], w["porosity"], w["rmin"], w["rmax"], w["seed"], w["fluidlayer"], 8 * w["Nc_fundamental"] ** 3, w["Kn"]),
         "image": "%dx%dx%d uint8" % (w["n"], w["n"], w["n"]), "velocities": 8 * w["Nc_fundamental"] ** 3,
         "Kn": w["Kn"], "l2": "inputs larger than L2 (distribution function > 4 GB per rank)"}
    if extra:
        d.update(extra)
    return d


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", "clocks_rank%d.csv" % gpu_index)

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

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
        for line in open(self.path):
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
    import piks3d_b200 as pk
    if rank != 0:
        return 0
    img = workload_image()
    p = workload_params(pk)
    iters = max(1, min(args.steps, 3))
    warm = 1
    cb = cpu_baseline(p, img, iters)
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": args.gpus, "steps": iters,
            "warmup": warm, "ms_per_step": cb["seconds_per_iteration"] * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": config_dict({"note": "each step is a bounded sample: the CPU run times %d iterations" % iters}),
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "gpu_launches": 0}
    print(json.dumps(line))
    return 0


def run_ours(args, world, rank, local):
    import torch
    import piks3d_b200 as pk

    torch.cuda.set_device(local)
    device = torch.device("cuda", local)
    img = workload_image()
    p = workload_params(pk)

    # --- device-resident run: value, roofline ---------------------------------------------
    prec = pk.PREC_FP32 if args.precision == "fp32" else pk.PREC_FP64
    esz = 4 if prec == pk.PREC_FP32 else 8
    s = pk.Solver(p, device=local)
    s.set_precision(prec)
    s.setup_physical_grid(img)
    info = s.info()
    stream = torch.cuda.Stream(device=device)
    s.set_stream(stream.cuda_stream)
    nf, nc8 = info["Nfluid"], info["Nc8"]
    nv = 8 * nc8
    sw = s.geometry_array("node_g")  # noqa: F841 (keeps the call path warm)
    # swept updates per iteration: fluid nodes outside each octant's inflow planes
    lab = s.get_labels()
    fluid = lab == 0
    swept = 0
    for sx in (1, -1):
        for sy in (1, -1):
            for sz in (1, -1):
                f = fluid[1:, :, :] if sz > 0 else fluid[:-1, :, :]
                f = f[:, 1:, :] if sy > 0 else f[:, :-1, :]
                f = f[:, :, 1:] if sx > 0 else f[:, :, :-1]
                swept += int(f.sum())
    sweep_bytes = 2 * esz * nc8 * swept + 32 * nf     # h read + write per swept update, moments read once
    iter_bytes = 2 * esz * nv * (nf + info["nWall"]) + 2 * 32 * nf

    s.iterate(args.warmup)
    s.synchronize()
    s.enable_timing(True)
    s.kernel_times(reset=True)
    clocks = ClockSampler(local)
    barrier(world, device)
    torch.cuda.synchronize()
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    s.iterate(args.steps)
    ev1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_local = ev0.elapsed_time(ev1)
    kt = s.kernel_times(reset=True)
    s.enable_timing(False)
    launches = s.launches_per_iteration() * args.steps
    s.close()
    ms = reduce_max(ms_local, world, device)
    barrier(world, device)

    # --- end to end through the C ABI with host buffers ---------------------------------------
    box = info["Nx"] * info["Ny"] * info["Nz"]
    torch.cuda.synchronize()
    barrier(world, device)
    t0 = time.perf_counter()
    s2 = pk.Solver(p, device=local)
    s2.set_precision(prec)
    s2.setup_physical_grid(img)                 # H2D: image -> geometry tables + zeroed state
    s2.iterate(args.steps)
    mass, perm, err = s2.chk_converge()          # D2H: mass flux
    rho, ux, uy, uz = s2.get_macro()             # D2H: fields
    s2.close()
    e2e_local = time.perf_counter() - t0
    e2e_s = reduce_max(e2e_local, world, device)

    if rank != 0:
        return 0
    upd = nf * nv * args.steps * world
    value = upd / (ms * 1e-3) / 1e9
    sweep_ms, sweep_groups = kt["sweep"]
    per_iter_sweep_ms = sweep_ms / max(1, sweep_groups)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = peaks.get("hbm_gbs", 6650.0)
    achieved = sweep_bytes / (per_iter_sweep_ms * 1e-3) / 1e9
    h2d = img.nbytes
    d2h = 4 * box * 8 + 8
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if esz == 8 else "f32 (moments, wall densities, flux f64)",
        "data": "synthetic",
        "config": config_dict({"Nfluid": nf, "nWall": info["nWall"], "parallelism": "replicas x%d" % world,
                               "precision": args.precision}),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None,
                     "kernel": "k_sweep (all tile-diagonal launches of one iteration)",
                     "alg_bytes_per_iteration": sweep_bytes,
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650"},
        "iteration_bandwidth_gbs": iter_bytes / (ms / args.steps * 1e-3) / 1e9,
        "kernel_ms_per_iteration": {k: v[0] / max(1, args.steps) for k, v in kt.items()},
        "e2e": {"value": upd / e2e_s / 1e9, "unit": UNIT, "h2d_bytes_per_step": h2d / args.steps,
                "d2h_bytes_per_step": d2h / args.steps, "seconds": e2e_s,
                "what": "create + setup_physical_grid(host image) + %d iterations + chk_converge + get_macro, wall clock" % args.steps},
        "gpu_launches": launches,
        "clocks": clk,
        "permeability_after_steps": perm,
    }
    if not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(p, img, args.cpu_iters)
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-iters", type=int, default=2)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp32"],
                    help="fp32: FP32 f and sweep, FP64 moments / wall densities / flux")
    ap.add_argument("--n", type=int, default=None,
                    help="image edge (default 128); smaller edges are for profiling captures, not bench lines")
    args = ap.parse_args()
    if args.n:
        WORKLOAD["n"] = args.n
    world, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            rc = run_reference(args, world, rank)
        else:
            rc = run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    return rc


if __name__ == "__main__":
    sys.exit(main())
