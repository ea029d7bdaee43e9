"""Continuous-batching request server for permeability solves on one GPU.

Requests arrive over time (for the benchmark: a seeded Poisson stream). The loop keeps a
FIFO queue; at every convergence check of the running batch it admits queued requests
whose estimated HBM footprint (FP32 f plus FP64 moments per fluid voxel, and the FP64 copy
made when a refined solve switches precision) fits the memory left, preprocesses them on
host threads while the GPU keeps iterating, and lets them join the batch, where their
sweeps share the dataflow launches of the solves already running. A solve's state stays on
the device until it converges; it then leaves the batch and frees its memory. Latency is
measured from arrival to the end of the check that found the solve converged.
"""
import collections
import time

import numpy as np

from .solve import BatchRunner, Job


def poisson_arrivals(rate, duration, seed):
    """Arrival times (s) of a Poisson process of `rate` per second over [0, duration)."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return out
        out.append(t)


def percentile(values, q):
    return float(np.percentile(np.asarray(values, dtype=np.float64), q)) if len(values) else None


class Server:
    """Runs a request stream through a BatchRunner (continuous batching)."""

    def __init__(self, runner: BatchRunner, horizon=None, clock=time.perf_counter, sleep=time.sleep):
        self.runner, self.horizon, self.clock, self.sleep = runner, horizon, clock, sleep

    def run(self, jobs):
        """jobs: Job objects with `arrival` set (seconds from the start). Returns a report."""
        jobs = sorted(jobs, key=lambda j: j.arrival)
        t0 = self.clock()
        incoming = collections.deque(jobs)
        queue = collections.deque()
        done = []
        busy = 0.0
        def ended():  # jobs the runner finished without running them (refused, failed to prepare)
            return bool(getattr(self.runner, "refused", ()))

        while incoming or queue or self.runner.active or self.runner.preparing or ended():
            now = self.clock() - t0
            if self.horizon is not None and now > self.horizon:
                break
            while incoming and incoming[0].arrival <= now:
                queue.append(incoming.popleft())
            while queue and self.runner.try_admit(queue[0], now):
                queue.popleft()
            if not self.runner.active and not self.runner.preparing and not ended():
                if incoming:
                    self.sleep(max(0.0, min(0.05, incoming[0].arrival - now)))
                continue
            t1 = self.clock()
            for job in self.runner.step():
                job.latency = job.finished - (t0 + job.arrival)
                done.append(job)
            busy += self.clock() - t1
        wall = self.clock() - t0
        failed = [j for j in done if j.result is not None and ("refused" in j.result or "failed" in j.result)]
        done = [j for j in done if j not in failed]
        lat = [j.latency for j in done]
        return {
            "requests": len(jobs), "completed": len(done), "refused_or_failed": len(failed),
            "unfinished": len(jobs) - len(done) - len(failed),
            "wall_s": wall, "busy_s": busy, "solves_per_s": len(done) / wall if wall > 0 else 0.0,
            "latency_p50_s": percentile(lat, 50), "latency_p99_s": percentile(lat, 99),
            "latency_max_s": max(lat) if lat else None, "jobs": done,
        }


def make_stream(rate, duration, seed, make_params, edge_range=(48, 160), porosity_range=(0.25, 0.6),
                kn_range=(0.01, 10.0)):
    """A seeded request stream of sphere-pack images (the serving workload): edges uniform in
    edge_range, porosity uniform, Kn log-uniform; make_params(n, Kn) builds the parameters."""
    from . import images
    rng = np.random.default_rng(seed)
    jobs = []
    for i, t in enumerate(poisson_arrivals(rate, duration, seed)):
        n = int(rng.integers(edge_range[0], edge_range[1] + 1))
        por = float(rng.uniform(*porosity_range))
        kn = float(np.exp(rng.uniform(np.log(kn_range[0]), np.log(kn_range[1]))))
        def make(n=n, por=por, sd=int(seed * 1000 + i)):
            return images.sphere_pack(n, por, 4.0, 8.0, seed=sd)
        jobs.append(Job(None, make_params(n, kn), name="req%d" % i, arrival=t, make_image=make, porosity=por))
    return jobs
