"""Host logic of the drivers (no GPU): the permeability-tolerance stopping rule, the HBM
footprint estimate, and the request server's queueing, admission and latency accounting
(driven by a stand-in runner and a simulated clock)."""
import math

import numpy as np

import piks3d_b200 as pk
from piks3d_b200.solve import Convergence, Job, footprint_bytes
from piks3d_b200.serve import Server, percentile, poisson_arrivals


def test_tolerance_rule_on_geometric_sequence():
    for r in (0.3, 0.7, 0.95):
        c = Convergence(tol=1e-4)
        for k in range(1, 2000):
            m = 2.0 * (1.0 - 0.5 * r ** k)
            if c.update(m, 0.1):
                break
        limit = 2.0
        assert abs(m - limit) / limit <= 1e-4, (r, k)
        assert abs(m - limit) / limit >= 1e-9, "stopped far later than needed"


def test_tolerance_rule_waits_on_non_contracting_changes():
    c = Convergence(tol=1e-4)
    out = [c.update(1.0 + 0.01 * ((-1) ** k), 0.1) for k in range(20)]
    assert not any(out) and math.isinf(c.estimate)


def test_eps_rule_and_stall():
    c = Convergence(eps=1e-8)
    assert not c.update(1.0, 1e-7) and c.update(1.0, 1e-9)
    c = Convergence(eps=1e-12, stall_checks=3)
    for e in (1e-6, 2e-6, 3e-6, 4e-6):
        c.update(1.0, e)
    assert c.stalled()


def test_footprint_orders():
    p = pk.default_params(Nx=32, Ny=32, Nz=32, Nc_fundamental=4)
    img = np.zeros((32, 32, 32), np.uint8)
    f32 = footprint_bytes(img, p, "fp32")
    f64 = footprint_bytes(img, p, "fp64")
    ref = footprint_bytes(img, p, "refined")
    assert f32 < f64 < ref
    assert f64 - f32 >= 32 ** 3 * 8 * 64 * 4


def test_poisson_arrivals_rate():
    t = poisson_arrivals(20.0, 60.0, seed=1)
    assert 1000 < len(t) < 1400 and all(0 <= a < 60 for a in t) and t == sorted(t)


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += max(dt, 1e-3)


class FakeRunner:
    """Stand-in for BatchRunner: each job needs `work` checks; a check takes 0.1 s; at most
    `slots` jobs at once."""

    def __init__(self, clock, slots=2):
        self.clock, self.slots = clock, slots
        self.active, self.preparing = [], []

    def try_admit(self, job, now):
        if len(self.active) >= self.slots:
            return False
        job.left = job.work
        self.active.append(job)
        return True

    def step(self):
        self.clock.t += 0.1
        done = []
        for j in list(self.active):
            j.left -= 1
            if j.left == 0:
                j.finished = self.clock.t
                self.active.remove(j)
                done.append(j)
        return done


def test_server_fifo_admission_and_latency():
    clock = FakeClock()
    runner = FakeRunner(clock, slots=2)
    jobs = []
    for i, (arr, work) in enumerate([(0.0, 3), (0.05, 1), (0.06, 2), (1.0, 1)]):
        j = Job(None, None, name=str(i), arrival=arr)
        j.work = work
        jobs.append(j)
    rep = Server(runner, clock=clock, sleep=clock.sleep).run(jobs)
    assert rep["completed"] == 4 and rep["unfinished"] == 0
    lat = {j.name: round(j.latency, 6) for j in rep["jobs"]}
    # job 0 and 1 start at t=0 (job 1 only arrives at 0.05: admitted at the next check), job 2 waits for a slot
    assert lat["0"] == 0.3
    assert lat["1"] == round(0.2 - 0.05, 6)
    assert lat["2"] == round(0.4 - 0.06, 6)
    assert lat["3"] < 0.2
    assert abs(rep["latency_p50_s"] - percentile(list(lat.values()), 50)) < 1e-9


def test_server_horizon_stops_with_unfinished():
    clock = FakeClock()
    runner = FakeRunner(clock, slots=1)
    jobs = []
    for i in range(5):
        j = Job(None, None, name=str(i), arrival=0.0)
        j.work = 10
        jobs.append(j)
    rep = Server(runner, horizon=1.5, clock=clock, sleep=clock.sleep).run(jobs)
    assert rep["completed"] == 1 and rep["unfinished"] == 4


def test_tolerance_rule_on_oracle_traces():
    """The rule applied to the oracle's own mass-flux trace stops within the tolerance of
    the converged value (pack with an early transient, and a single sphere)."""
    from piks3d_b200 import images
    from conftest import base_params
    from oracle import Oracle
    cases = [(images.sphere_pack(18, 0.45, 2.0, 4.0, seed=3), base_params(18, Nc_fundamental=2, Kn=2.0, fluidlayer=2)),
             (images.centred_sphere(20, 7.0), base_params(20, Nc_fundamental=2, Kn=1.0))]
    for img, p in cases:
        o = Oracle(p, img.tobytes(), nthreads=4)
        ms = []
        for _ in range(100):
            o.iterate(10)
            m, _, e = o.chk_converge()
            ms.append(m)
            if e < 1e-12:
                break
        o.close()
        c = Convergence(tol=1e-4)
        stop = next(k for k, m in enumerate(ms) if c.update(m, 1.0))
        assert abs(ms[stop] - ms[-1]) / abs(ms[-1]) <= 1e-4


def test_tolerance_rule_waits_past_a_turning_point():
    """A trace whose mass flux falls, turns near iteration 600 and then rises slowly (fast
    and slow modes of opposite sign): the rule must not stop at the turning point."""
    import json
    import os
    ms = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mass_trace_turning.json")))["masses"]
    c = Convergence(tol=1e-4)
    stop = next(k for k, m in enumerate(ms) if c.update(m, 1.0))
    assert abs(ms[stop] - ms[-1]) / abs(ms[-1]) <= 1e-4
    assert stop * 10 > 1000


def test_prior_contraction_does_not_stop_at_a_turning_point():
    """The FP64 phase of a refined solve starts with the contraction fitted in its FP32 phase
    (prior_r). Fed the turning-point trace from anywhere before the turn, with that fit or a
    too-fast or too-slow one, the rule still waits for the gate on the size of the changes
    and stops within tolerance of the limit."""
    import json
    import os
    ms = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "mass_trace_turning.json")))["masses"]
    fp32 = Convergence(tol=1e-4)
    for m in ms[:50]:
        fp32.update(m, 1.0)
    assert fp32.last_r is not None
    for start in (30, 45, 55, 60, 65):
        for r in (fp32.last_r, 0.5, 0.95):
            c = Convergence(tol=1e-4, prior_r=r)
            stop = next(start + k for k, m in enumerate(ms[start:]) if c.update(m, 1.0))
            assert stop * 10 > 1000
            assert abs(ms[stop] - ms[-1]) / abs(ms[-1]) <= 1e-4


class _OracleStates:
    """The snapshot-slot calls of a Solver, on an oracle's iteration state (numpy)."""

    def __init__(self, o):
        self.o, self.slots = o, {}

    @staticmethod
    def _flat(st):
        f, fw, mac, (w, e) = st
        return np.concatenate([f, fw, np.concatenate([m.reshape(-1) for m in mac]), w, e])

    def snapshot_slot(self, slot, nslots):
        self.slots[slot] = self._flat(self.o.state())

    def snapshot_gram(self, n):
        X = np.stack([self.slots[j] for j in range(n)], axis=1)
        U = np.diff(X, axis=1)
        return U.T @ U

    def snapshot_combine(self, coef):
        st = self.o.state()
        v = sum(c * self.slots[j] for j, c in enumerate(coef))
        f, fw, mac, (w, e) = st
        out, o = [], 0
        for a in [f, fw] + list(mac) + [w, e]:
            out.append(v[o:o + a.size].reshape(a.shape))
            o += a.size
        self.o.set_state((out[0], out[1], out[2:6], (out[6], out[7])))
        self.slots = {}


def _solve_oracle(p, img, tol, extrapolate, max_iter=20000):
    from oracle import Oracle
    from piks3d_b200.solve import Extrapolator
    o = Oracle(p, img.tobytes(), nthreads=4)
    conv = Convergence(tol=tol)
    ex = Extrapolator() if extrapolate else None
    states = _OracleStates(o)
    n = 0
    while n < max_iter:
        o.iterate(10)
        n += 10
        m, k, e = o.chk_converge()
        if conv.update(m, e):
            break
        if ex is not None and ex.after_check(states, conv):
            conv = Convergence(tol=tol)
    o.close()
    return n, k, (ex.jumps if ex else 0)


def test_extrapolation_cuts_iterations_within_tolerance():
    """The refined solver's extrapolation of its state (Extrapolator: MPE over snapshot
    slots), driven on the oracle's FP64 state: fewer iterations to the 1e-4 rule,
    permeability still within 1e-4 of the iteration's limit (a run to a 1e-7 estimate)."""
    from piks3d_b200 import images
    img = images.sphere_pack(20, 0.45, 2.5, 5.0, seed=8)
    p = pk.default_params(Nx=20, Ny=20, Nz=20, Nc_fundamental=2, Kn=1.0, pressDrop=1.0, wallExtOrder=1)
    _, kref, _ = _solve_oracle(p, img, 1e-7, False)
    n1, k1, _ = _solve_oracle(p, img, 1e-4, False)
    n2, k2, jumps = _solve_oracle(p, img, 1e-4, True)
    assert jumps >= 1 and n2 < n1
    assert abs(k2 - kref) / kref <= 1e-4 and abs(k1 - kref) / kref <= 1e-4


def test_watchdog_flags_non_finite_and_blowup():
    c = Convergence(tol=1e-4)
    for m in (1.0, 0.9, 0.85):
        c.update(m, 0.1)
    assert not c.diverged
    c.update(float("nan"), float("nan"))
    assert c.diverged
    c = Convergence(eps=1e-8)
    c.update(1e-2, 1.0)
    c.update(5e-2, 1.0)
    assert not c.diverged
    c.update(1e5, 1.0)  # 1e7 times the first checks
    assert c.diverged
    c = Convergence(tol=1e-4)
    for k in range(1, 200):
        c.update(2.0 * (1.0 - 0.5 * 0.9 ** k), 0.1)
    assert not c.diverged


def _runner_without_gpu(budget):
    """A BatchRunner whose admission and bookkeeping run without a device."""
    from piks3d_b200.solve import BatchRunner
    r = object.__new__(BatchRunner)
    r.device, r.precision, r.tol, r.eps = 0, "refined", 1e-4, None
    r.switch_eps, r.switch_change, r.max_members, r.keep_fields = 1e-6, 1e-6, 4, False
    r.hbm_budget = budget
    r.autotune, r.extrapolate = False, True
    r.active, r.preparing, r.refused, r.reserved = [], [], [], 0
    return r


def test_admission_refuses_a_job_that_can_never_fit():
    p = pk.default_params(Nx=64, Ny=64, Nz=64, Nc_fundamental=4)
    img = np.zeros((64, 64, 64), np.uint8)
    r = _runner_without_gpu(budget=footprint_bytes(img, p) // 2)
    j = Job(img, p, name="big")
    assert r.try_admit(j, 0.0)             # consumed from the queue ...
    assert r.reserved == 0 and not r.preparing
    assert "refused" in j.result and not j.result["converged"]
    out = r.step()                         # ... and handed back as finished
    assert out == [j] and j.finished is not None and r.refused == []


def test_failed_preparation_ends_the_job_with_its_error():
    import concurrent.futures as cf
    p = pk.default_params(Nx=16, Ny=16, Nz=16, Nc_fundamental=2)
    img = np.zeros((16, 16, 16), np.uint8)
    r = _runner_without_gpu(budget=1 << 40)
    j = Job(img, p, name="bad")
    j.footprint = footprint_bytes(img, p)
    r.reserved = j.footprint
    fut = cf.Future()
    fut.set_exception(pk.PiksError(3, "invalid image data file"))
    r.preparing.append((j, fut))
    out = r.step()
    assert out == [j] and "failed" in j.result and r.reserved == 0 and not r.active


def test_server_reports_refused_jobs_apart():
    clock = FakeClock()

    class RefusingRunner(FakeRunner):
        def __init__(self, clock):
            super().__init__(clock, slots=2)
            self.refused = []

        def try_admit(self, job, now):
            if job.name == "huge":
                job.result = {"refused": "footprint", "converged": False}
                self.refused.append(job)
                return True
            return super().try_admit(job, now)

        def step(self):
            ended, self.refused = self.refused, []
            for j in ended:
                j.finished = self.clock.t
            return ended + super().step()

    jobs = []
    for i, name in enumerate(["a", "huge", "b"]):
        j = Job(None, None, name=name, arrival=0.01 * i)
        j.work = 2
        jobs.append(j)
    for j in jobs:  # solved jobs carry the reference's error value in their result
        j.result = {"error": 1e-9, "converged": True} if j.name != "huge" else None
    rep = Server(RefusingRunner(clock), clock=clock, sleep=clock.sleep).run(jobs)
    assert rep["completed"] == 2 and rep["refused_or_failed"] == 1 and rep["unfinished"] == 0
    assert sorted(j.name for j in rep["jobs"]) == ["a", "b"]


def test_refinement_phase_uses_the_measured_contraction():
    """After a switch (the FP32 iterate as the starting mass, a small jump, then the same
    contraction), a rule given the contraction of the first phase stops within the tolerance,
    and checks earlier than a rule that has to fit it again."""
    r, tol = 0.8, 1e-4
    limit = 2.0
    first = Convergence(tol=tol)
    k = 0
    while True:
        k += 1
        m = limit * (1.0 + 3e-4 * r ** k)
        if first.update(m, 0.1):
            break
    assert first.last_r is not None and abs(first.last_r - r) < 0.02
    m32 = m * (1.0 + 1e-5)                  # the FP32 phase ends slightly off the FP64 limit path

    def run(prior):
        c = Convergence(tol=tol, prior_r=prior)
        c.masses = [m32]
        for j in range(1, 200):
            mj = limit * (1.0 + 2e-5 * r ** j)
            if c.update(mj, 0.1):
                return j, mj
    j_prior, m_prior = run(first.last_r)
    j_fresh, m_fresh = run(None)
    assert abs(m_prior - limit) / limit <= tol and abs(m_fresh - limit) / limit <= tol
    assert j_prior < j_fresh
