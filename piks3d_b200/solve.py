"""Host-side drivers above the C ABI: convergence control for one solve, batched solves of
many images, and a continuous-batching request server.

Convergence (main.F90:98-121 keeps iterating until chkConverge's error <= eps). Besides
that rule, a solve can stop at a permeability tolerance: chkConverge runs every
chkConvergeStep iterations; with d_k the relative change of the mass flux between two
checks and r the observed contraction per check, the distance of the current
permeability to the limit of the iteration is estimated as d_k * r / (1 - r) (geometric
tail, as in Aitken's extrapolation); see Convergence for the exact rule.

Precision: a "refined" solve runs the FP32 sweep (FP64 moments, wall densities, flux and
convergence test) until it meets the stopping rule or its mass flux changes by less than
`switch_change` (relative) per check twice in a row (the FP32 iterate then sits near its
rounding floor); it then widens its state to FP64 on the device and continues in FP64
until the rule holds there. The FP64 phase runs the same iteration, so its rule starts from
the contraction per check fitted in the FP32 phase instead of waiting for checks of its own.
"""
import concurrent.futures as cf
import math
import time

import numpy as np

from . import Batch, PREC_FP32, PREC_FP64, SCHED_TILE_DATAFLOW, Solver


class Convergence:
    """Per-solve stopping rule over the sequence of chkConverge results.

    With `tol` set: d_i is the relative change of the mass flux between consecutive checks.
    Over the last `window` values a straight line is fitted to log d_i; its slope gives the
    contraction per check r, and the remaining relative distance of the permeability to the
    limit of the iteration is estimated as d * r / (1 - r), with d the fitted last change.
    The solve stops once that estimate is below safety * tol at `consec` checks in a row,
    provided r < 1 and the points lie close to the line (residual below `maxres` in log),
    and the last `gate_run` changes were each at most gate * tol. Fitting over several
    checks, rather than taking one ratio of two changes, keeps the rule from being fooled by
    the early transient of the source iteration or by rounding noise in the FP32 phase of a
    refined solve; the gate on the size of the changes keeps it from stopping where a fast
    mode and a slow mode of opposite sign cancel for a few checks (the mass flux passing
    through a turning point looks converged there). A watchdog flags divergence (`diverged`)."""

    def __init__(self, eps=1e-8, tol=None, stall_checks=5, window=6, min_checks=8, consec=2, safety=0.5,
                 maxres=0.35, gate=0.02, gate_run=3, blowup=1e6, prior_r=None):
        self.eps, self.tol, self.stall_checks = eps, tol, stall_checks
        # contraction per check already measured on the same iteration (the FP32 phase of a
        # refined solve): until enough checks exist for a fit of its own, the estimate uses it
        self.prior_r = prior_r
        self.last_r = None            # contraction of the last fit that met the residual bound
        self.r_now = None             # contraction of this check's fit (None: no fit, or a poor one)
        # watchdog: a non-finite mass flux or error, or a mass flux `blowup` times the largest
        # of the first checks, marks the iteration as diverged (the reference would run on to
        # maxStep)
        self.blowup = blowup
        self.diverged = False
        self.window, self.min_checks, self.consec, self.safety, self.maxres = window, min_checks, consec, safety, maxres
        self.gate, self.gate_run = gate, gate_run
        self._gate_ok = 0
        self.masses = []
        self.best = math.inf
        self.since_best = 0
        self.estimate = math.inf     # estimated relative distance of the permeability to its limit
        self._ok_run = 0
        self._small_run = 0

    def last_change(self):
        """Relative change of the mass flux between the last two checks."""
        if len(self.masses) < 2:
            return math.inf
        return abs(self.masses[-1] - self.masses[-2]) / max(abs(self.masses[-1]), 1e-300)

    def update(self, mass, error):
        """Records one check; returns True when the solve has converged."""
        if not (math.isfinite(mass) and math.isfinite(error)):
            self.diverged = True
        elif self.masses and abs(mass) > self.blowup * max(abs(m) for m in self.masses[:self.window]):
            self.diverged = True
        self.masses.append(mass)
        if error < self.best:
            self.best, self.since_best = error, 0
        else:
            self.since_best += 1
        if self.tol is None:
            return error <= self.eps
        w = self.window
        self.r_now = None
        if len(self.masses) < max(w + 1, self.min_checks):
            if self.prior_r is None or len(self.masses) < 2:
                return False
            r = self.prior_r
            self.estimate = self.last_change() * r / (1.0 - r)
            self._ok_run = self._ok_run + 1 if self.estimate <= self.safety * self.tol else 0
            self._gate_ok = self._gate_ok + 1 if self.last_change() <= self.gate * self.tol else 0
            return self._ok_run >= self.consec and self._gate_ok >= self.gate_run
        m = self.masses
        d = np.array([abs(m[-w + i] - m[-w + i - 1]) / max(abs(m[-w + i]), 1e-300) for i in range(w)])
        if d[-1] == 0.0:
            self.estimate = 0.0
        elif np.any(d <= 0.0):
            self.estimate = math.inf
        else:
            x = np.arange(w, dtype=np.float64)
            y = np.log(d)
            b, a = np.polyfit(x, y, 1)
            res = float(np.std(y - (a + b * x)))
            r = math.exp(b)
            good = r < 1.0 and res <= self.maxres
            if good:
                self.last_r = r
                self.r_now = r
            self.estimate = math.exp(a + b * (w - 1)) * r / (1.0 - r) if good else math.inf
        self._ok_run = self._ok_run + 1 if self.estimate <= self.safety * self.tol else 0
        self._gate_ok = self._gate_ok + 1 if self.last_change() <= self.gate * self.tol else 0
        return self._ok_run >= self.consec and self._gate_ok >= self.gate_run

    def small_changes(self, threshold, checks=2):
        """True once the last `checks` relative changes were all at most `threshold`."""
        self._small_run = self._small_run + 1 if self.last_change() <= threshold else 0
        return self._small_run >= checks

    def stalled(self):
        return self.since_best >= self.stall_checks


class Extrapolator:
    """Moves a refined solve's state toward the iteration's limit by minimal polynomial
    extrapolation (MPE) of its checks.

    The source iteration is affine (f_{n+1} = M f_n + b), so its error is soon a few slow
    modes of M. After `burn` checks from the start or from the last jump, the states of
    k + 2 consecutive checks x_0 .. x_{k+1} go to snapshot slots on the device; with the
    differences u_j = x_{j+1} - x_j, c minimises |U c + u_k| over the first k differences
    (from their Gram matrix), c_k = 1, and the state becomes sum_j g_j x_j (j <= k) with
    g = c / sum(c): the combination that cancels k modes (k = 1: Aitken's extrapolation of
    the whole state). The caller then starts a fresh stopping rule (the trace restarts from
    the new state). Once the rule's estimate is below `quiet` times its tolerance, or after
    `max_jumps` jumps, the solve is left to finish. Used in the FP32 phase of refined solves
    only; the plain FP64 solve stays the reference's iteration. Measured on the oracle (FP64,
    checks every 10 iterations, to the 1e-4 rule; 32^3 Kn 0.5 / 32^3 Kn 2 / 40^3 Kn 0.3):
    k = 4, burn 6: 220 / 220 / 340 iterations; k = 3: 270 / 440 / 320; k = 2: 480 / 1000 /
    470; none: 970 / 1180 / 920."""

    def __init__(self, k=4, burn=6, quiet=1.0, max_jumps=8):
        self.k, self.burn, self.quiet, self.max_jumps = k, burn, quiet, max_jumps
        self.since = 0
        self.n = 0                    # slots filled in this round
        self.jumps = 0

    def slots(self):
        return self.k + 2

    def after_check(self, solver, conv):
        """Call after each check with the solve's stopping rule; True when the state jumped."""
        self.since += 1
        if (math.isfinite(conv.estimate) and conv.tol is not None and conv.estimate < self.quiet * conv.tol) \
                or self.jumps >= self.max_jumps:
            self.n = 0
            return False
        if self.since <= self.burn:
            return False
        k = self.k
        solver.snapshot_slot(self.n, k + 2)
        self.n += 1
        if self.n < k + 2:
            return False
        self.n = 0
        G = solver.snapshot_gram(k + 2)
        c = np.linalg.lstsq(G[:k, :k], -G[:k, k], rcond=None)[0]
        c = np.append(c, 1.0)
        total = float(c.sum())
        if not np.all(np.isfinite(c)) or abs(total) < 1e-12:
            return False
        g = c / total
        if np.max(np.abs(g)) > 1e4:   # ill-conditioned: the differences are noise
            return False
        solver.snapshot_combine(g)
        self.jumps += 1
        self.since = 0
        return True


class Job:
    """One solve request: an image (uint8, z-y-x) and its piks_params."""

    def __init__(self, image, params, name=None, arrival=0.0, make_image=None, porosity=None):
        # image may be None with make_image (a callable) given: it is then generated when the
        # job is prepared, and `porosity` sizes the footprint estimate before that
        self.image, self.params, self.name, self.arrival = image, params, name, arrival
        self.make_image, self.porosity = make_image, porosity
        self.solver = None
        self.tuned = None             # (TX, TY, TZ, schedule) chosen by the batch runner's autotuner
        self.conv = None
        self.ex = None                # Extrapolator of a refined job's FP32 phase
        self.phase = None             # "fp32" / "fp64"
        self.steps32 = 0
        self.steps = 0
        self.result = None
        self.admitted = None
        self.finished = None
        self.footprint = None


def footprint_bytes(image, params, precision="refined", slots=None):
    """HBM needed by a solve, estimated from the image before preprocessing: per fluid voxel
    the distribution function (8 octants x Nc8 velocities, FP32 or FP64) and its FP64 moments,
    plus the solid voxels next to fluid (walls) and a fixed overhead for tables. A refined
    solve holds the extrapolator's snapshot slots of its FP32 state (`slots`, default the
    Extrapolator's) during its FP32 phase, and FP32 and FP64 copies of f for the instant of
    the switch (the slots are freed first)."""
    nc8 = params.Nc_fundamental ** 3
    if isinstance(image, tuple):      # (n voxels, porosity) before the image exists
        fluid = int(image[0] * image[1])
        face = int(round(image[0] ** (2.0 / 3.0)))
    else:
        fluid = int(np.count_nonzero(np.asarray(image) == 0))
        face = image.shape[0] * image.shape[1]
    nodes = int(fluid * 1.7) + 2 * params.fluidlayer * face
    f32 = nodes * 8 * nc8 * 4
    f64 = nodes * 8 * nc8 * 8
    moments = fluid * 32
    tables = nodes * 8 * 48 + (64 << 20)
    if precision == "fp64":
        return f64 + moments + tables
    if precision == "fp32":
        return f32 + moments + tables
    if slots is None:
        slots = Extrapolator().slots()
    return max((f32 + moments) * (1 + slots), f32 + f64 + moments) + tables


# Tile shapes the batch runner's autotuner times on each job (the batch sweeps every member
# with its own tile jobs in one dataflow launch, so candidates use the dataflow schedule).
TUNE_CANDIDATES = ((4, 4, 4, SCHED_TILE_DATAFLOW), (8, 4, 4, SCHED_TILE_DATAFLOW), (4, 4, 8, SCHED_TILE_DATAFLOW))


def _prepare(job, device, precision, autotune=False):
    if job.image is None:
        job.image = job.make_image()
    s = Solver(job.params, device=device)
    try:
        if precision in ("fp32", "refined"):
            s.set_precision(PREC_FP32)
        s.setup_physical_grid(job.image)
        if autotune:
            # times one sweep of each candidate on this image (its own stream: the batch's
            # iterations may run meanwhile), keeps the fastest, resets the state
            job.tuned = s.autotune(TUNE_CANDIDATES, sweeps=1)[0]
    except Exception:
        s.close()
        raise
    return s


class BatchRunner:
    """Solves many jobs on one GPU as a continuously refilled batch: jobs are admitted while
    their estimated footprint fits the HBM budget and the batch has a free slot, preprocessed
    (and, with `autotune`, their tile shape timed on the image) on host threads while the GPU
    iterates, iterated together (piks_batch_*), checked every
    chkConvergeStep iterations, switched from FP32 to FP64 when their FP32 phase ends, and
    retired (state freed) as soon as they converge."""

    def __init__(self, device=0, precision="refined", tol=1e-4, eps=None, switch_eps=1e-6, switch_change=1e-6,
                 max_members=64, hbm_budget=None, prep_threads=4, keep_fields=False, autotune=True, extrapolate=True):
        import torch  # noqa: F401  (device memory query only)
        self.device, self.precision, self.tol, self.eps = device, precision, tol, eps
        self.switch_eps, self.max_members, self.keep_fields = switch_eps, max_members, keep_fields
        self.switch_change = switch_change
        self.autotune = autotune
        self.extrapolate = extrapolate
        if hbm_budget is None:
            import torch
            free, _total = torch.cuda.mem_get_info(device)
            hbm_budget = int(free * 0.85)
        self.hbm_budget = hbm_budget
        self.pool = cf.ThreadPoolExecutor(max_workers=prep_threads)
        self.batch = Batch(device=device)
        self.active = []
        self.preparing = []           # (job, future)
        self.refused = []             # jobs finished without running (refused or failed to prepare)
        self.reserved = 0

    def close(self):
        for j in self.active:
            j.solver.close()
        self.active = []
        for j, fut in self.preparing:
            try:
                fut.result().close()
            except Exception:
                pass
        self.preparing = []
        self.batch.close()
        self.pool.shutdown(wait=True)

    def _chk_step(self):
        return self.active[0].params.chkConvergeStep if self.active else 10

    def try_admit(self, job, now):
        """Starts preprocessing `job` if its footprint fits; returns False when it must wait."""
        if job.image is None:
            p = job.params
            img = (p.Nx * p.Ny * p.Nz, job.porosity if job.porosity is not None else 1.0)
        else:
            img = job.image
        fp = footprint_bytes(img, job.params, self.precision, slots=None if self.extrapolate else 0)
        if fp > self.hbm_budget:
            # can never fit, not even alone: refused rather than left to fail on allocation
            job.footprint = 0
            job.admitted = now
            job.result = {"refused": "footprint %d bytes exceeds the HBM budget %d" % (fp, self.hbm_budget),
                          "converged": False}
            self.refused.append(job)
            return True
        slots = len(self.active) + len(self.preparing)
        if slots >= self.max_members or (self.reserved + fp > self.hbm_budget and slots > 0):
            return False
        job.footprint = fp
        job.admitted = now
        self.reserved += fp
        self.preparing.append((job, self.pool.submit(_prepare, job, self.device, self.precision, self.autotune)))
        return True

    def _join_ready(self, block=False):
        still = []
        for job, fut in self.preparing:
            if block or fut.done():
                try:
                    job.solver = fut.result()
                except Exception as e:  # bad image, allocation failure: the job ends with the error
                    job.result = {"failed": "%s: %s" % (type(e).__name__, e), "converged": False}
                    self.reserved -= job.footprint
                    self.refused.append(job)
                    continue
                job.phase = "fp64" if self.precision == "fp64" else "fp32"
                job.conv = self._new_conv(job)
                job.ex = Extrapolator() if (self.extrapolate and self.precision == "refined" and self.tol is not None) \
                    else None
                self.batch.add(job.solver)
                self.active.append(job)
            else:
                still.append((job, fut))
        self.preparing = still

    def _new_conv(self, job):
        eps = self.eps if self.eps is not None else job.params.eps
        if job.phase == "fp32" and self.precision == "refined":
            return Convergence(eps=max(eps, self.switch_eps), tol=self.tol)
        return Convergence(eps=eps, tol=self.tol)

    def step(self):
        """Admitted jobs that finished preprocessing join; one chkConvergeStep of iterations;
        one check; finished jobs leave. Returns the jobs that finished (refused and failed
        jobs included, with the reason in their result)."""
        self._join_ready(block=not self.active and bool(self.preparing))
        ended, self.refused = self.refused, []
        for job in ended:
            job.finished = time.perf_counter()
        if not self.active:
            return ended
        chk = self._chk_step()
        self.batch.iterate(chk)
        mass, perm, err = self.batch.chk_converge()
        done = []
        for i, job in enumerate(list(self.active)):
            job.steps += chk
            if job.phase == "fp32":
                job.steps32 += chk
            conv = job.conv.update(mass[i], err[i])
            small = job.conv.small_changes(self.switch_change)
            if job.phase == "fp32" and self.precision == "refined" and (conv or small):
                # the FP64 phase continues from the widened FP32 iterate
                job.solver.set_precision(PREC_FP64)
                job.phase = "fp64"
                prior = job.conv.last_r
                job.conv = self._new_conv(job)
                job.conv.prior_r = prior
                job.conv.masses = [mass[i]]
                continue
            if conv or job.conv.diverged or job.steps >= job.params.maxStep:
                job.result = {"steps": job.steps, "steps32": job.steps32, "mass": float(mass[i]),
                              "permeability": float(perm[i]), "error": float(err[i]),
                              "converged": bool(conv), "diverged": job.conv.diverged,
                              "estimate": job.conv.estimate, "tiles": job.tuned,
                              "jumps": job.ex.jumps if job.ex else 0}
                if self.keep_fields:
                    job.result["macro"] = job.solver.get_macro()
                done.append(job)
                continue
            if job.ex is not None and job.phase == "fp32" and job.ex.after_check(job.solver, job.conv):
                job.conv = self._new_conv(job)
        done_solved = list(done)
        done = ended + done
        for job in done_solved:
            self.batch.remove(job.solver)
            self.active.remove(job)
            job.solver.close()
            job.solver = None
            self.reserved -= job.footprint
            job.finished = time.perf_counter()
        return done

    def run(self, jobs):
        """Solves `jobs` (all available at once) and returns them with results."""
        t0 = time.perf_counter()
        pending = list(jobs)
        finished = []
        while pending or self.active or self.preparing or self.refused:
            now = time.perf_counter() - t0
            while pending and self.try_admit(pending[0], now):
                pending.pop(0)
            finished.extend(self.step())
        return finished


def solve_one(image, params, device=0, precision="fp64", tol=None, eps=None, switch_eps=1e-6, switch_change=1e-6,
              tiles=None, keep_fields=False, extrapolate=True):
    """One solve through a context of its own (no batch): the reference's loop with the same
    stopping rule as the batch runner. With a tolerance, the FP32 phase of a refined solve
    also extrapolates its state along its slowest mode (Extrapolator; `extrapolate`).
    Returns a result dict."""
    s = Solver(params, device=device)
    if tiles is not None:
        s.set_tiles(*tiles)
    if precision in ("fp32", "refined"):
        s.set_precision(PREC_FP32)
    s.setup_physical_grid(image)
    setup_seconds = list(s.setup_seconds())
    chk = params.chkConvergeStep
    phase = "fp64" if precision == "fp64" else "fp32"
    base_eps = eps if eps is not None else params.eps
    conv = Convergence(eps=max(base_eps, switch_eps) if precision == "refined" else base_eps, tol=tol)
    ex = Extrapolator() if (extrapolate and precision == "refined" and tol is not None) else None
    steps = steps32 = 0
    while True:
        s.iterate(chk)
        steps += chk
        if phase == "fp32":
            steps32 += chk
        m, k, e = s.chk_converge()
        ok = conv.update(m, e)
        small = conv.small_changes(switch_change)
        if phase == "fp32" and precision == "refined" and (ok or small):
            s.set_precision(PREC_FP64)
            phase = "fp64"
            conv = Convergence(eps=base_eps, tol=tol, prior_r=conv.last_r)
            conv.masses = [m]
            continue
        if ok or conv.diverged or steps >= params.maxStep:
            res = {"steps": steps, "steps32": steps32, "mass": m, "permeability": k, "error": e,
                   "converged": bool(ok), "diverged": conv.diverged, "estimate": conv.estimate,
                   "setup_seconds": setup_seconds, "jumps": ex.jumps if ex else 0}
            if keep_fields:
                res["macro"] = s.get_macro()
            s.close()
            return res
        if ex is not None and phase == "fp32" and ex.after_check(s, conv):
            conv = Convergence(eps=max(base_eps, switch_eps), tol=tol)
