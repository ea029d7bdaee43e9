"""GPU tests of batches: solves iterated together (merged dataflow sweep launches, CUDA
graph replay, members joining and leaving between iterations) give every member exactly
the values of the same solve run alone - FP64 and FP32 members alike (tolerance 0)."""
import numpy as np
import pytest

import piks3d_b200 as pk
from piks3d_b200 import images
from conftest import base_params

pytestmark = pytest.mark.gpu

MEMBERS = [
    # (image, params, precision)
    (lambda: images.centred_sphere(16, 5.0), dict(Nc_fundamental=2, Kn=1.0), pk.PREC_FP64),
    (lambda: images.sphere_pack(12, 0.5, 1.5, 3.0, seed=7), dict(Nc_fundamental=4, Kn=0.5, fluidlayer=2), pk.PREC_FP64),
    (lambda: images.sphere_pack(14, 0.5, 1.5, 3.5, seed=1), dict(Nc_fundamental=2, Kn=0.7), pk.PREC_FP32),
    (lambda: images.sphere_pack(10, 0.55, 1.2, 2.5, seed=4), dict(Nc_fundamental=4, Kn=0.3, pressDrop=0.1), pk.PREC_FP32),
    (lambda: images.sphere_pack(16, 0.45, 1.5, 3.0, seed=9), dict(Nc_fundamental=2, Kn=0.05, wallExtOrder=1), pk.PREC_FP64),
]


def _solver(k):
    make, kw, prec = MEMBERS[k]
    img = make()
    n = img.shape[0]
    s = pk.Solver(base_params(n, **kw), device=0)
    s.set_precision(prec)
    s.setup_physical_grid(img)
    return s


def _alone(k, steps):
    s = _solver(k)
    out = {}
    for it in range(1, max(steps) + 1):
        s.iterate(1)
        if it in steps:
            out[it] = (s.get_f()[0].copy(), s.chk_converge())
    s.close()
    return out


def test_batch_members_equal_alone_runs():
    # member k joins at iteration join[k] (of the batch) and leaves at leave[k]
    join = [0, 0, 0, 3, 5]
    leave = [12, 9, 12, 12, 12]
    total = 12
    ref = {}
    for k in range(len(MEMBERS)):
        n = leave[k] - join[k]
        ref[k] = _alone(k, {n, max(1, n // 2)})
    solvers = {}
    with pk.Batch(device=0) as b:
        for t in range(total):
            for k in range(len(MEMBERS)):
                if join[k] == t:
                    solvers[k] = _solver(k)
                    b.add(solvers[k])
            b.iterate(1)
            for k in list(solvers):
                done = t + 1 - join[k]
                if done == max(1, (leave[k] - join[k]) // 2) or t + 1 == leave[k]:
                    b.synchronize()
                    f = solvers[k].get_f()[0]
                    assert np.array_equal(f, ref[k][done][0]), "member %d differs at its iteration %d" % (k, done)
                if t + 1 == leave[k]:
                    b.remove(solvers[k])
                    m = solvers[k].chk_converge()
                    assert m[:2] == ref[k][done][1][:2]  # mass flux and permeability
                    solvers.pop(k).close()
        assert len(b) == 0


def test_batch_chk_converge_matches_members():
    with pk.Batch(device=0) as b:
        ss = [_solver(k) for k in (0, 2, 4)]
        for s in ss:
            b.add(s)
        b.iterate(10)
        mass, perm, err = b.chk_converge()
        alone = [_alone(k, {10})[10][1] for k in (0, 2, 4)]
        for i, a in enumerate(alone):
            assert (mass[i], perm[i], err[i]) == a
        for s in ss:
            b.remove(s)
            s.close()


def test_batch_with_216_velocity_members_equals_alone():
    """Members with 216 velocities per octant (narrower sweep CTAs, several velocity chunks)
    batched with 8- and 64-velocity members, FP32 and FP64: each equals its solo run."""
    extra = [
        (lambda: images.sphere_pack(10, 0.55, 1.2, 2.5, seed=4), dict(Nc_fundamental=6, Kn=0.3, pressDrop=0.1), pk.PREC_FP64),
        (lambda: images.sphere_pack(10, 0.5, 1.2, 2.5, seed=8), dict(Nc_fundamental=6, Kn=0.5), pk.PREC_FP32),
    ]

    def solver(make, kw, prec):
        img = make()
        s = pk.Solver(base_params(img.shape[0], **kw), device=0)
        s.set_precision(prec)
        s.setup_physical_grid(img)
        return s

    members = [MEMBERS[0], MEMBERS[2]] + extra
    alone = []
    for m in members:
        s = solver(*m)
        s.iterate(6)
        alone.append((s.get_f()[0], s.chk_converge()))
        s.close()
    with pk.Batch(device=0) as b:
        ss = [solver(*m) for m in members]
        for s in ss:
            b.add(s)
        b.iterate(6)
        b.synchronize()
        for k, s in enumerate(ss):
            assert np.array_equal(s.get_f()[0], alone[k][0]), "member %d differs" % k
            assert s.chk_converge()[:2] == alone[k][1][:2]
        for s in ss:
            b.remove(s)
            s.close()
