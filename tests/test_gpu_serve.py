"""GPU tests of the batch runner and the continuous-batching server: every solve's result
in the mix (batched with others, joining while others run) equals the same solve run alone
(steps and permeability identical: tolerance 0), and the refined FP32 solve stopped at a
1e-4 permeability tolerance is within 1e-4 of the FP64 oracle's converged permeability."""
import numpy as np
import pytest

import piks3d_b200 as pk
from piks3d_b200 import images
from piks3d_b200.serve import Server
from piks3d_b200.solve import BatchRunner, Job, solve_one
from conftest import base_params
from oracle import Oracle

pytestmark = pytest.mark.gpu


def _jobs():
    specs = [
        (images.centred_sphere(20, 7.0), base_params(20, Nc_fundamental=2, Kn=1.0, maxStep=3000)),
        (images.sphere_pack(16, 0.5, 2.0, 4.0, seed=7), base_params(16, Nc_fundamental=2, Kn=0.5, fluidlayer=2, maxStep=3000)),
        (images.sphere_pack(12, 0.5, 1.5, 3.0, seed=7), base_params(12, Nc_fundamental=4, Kn=0.5, fluidlayer=2, maxStep=3000)),
        (images.sphere_pack(18, 0.45, 2.0, 4.0, seed=3), base_params(18, Nc_fundamental=2, Kn=2.0, fluidlayer=2, maxStep=3000)),
        (images.centred_sphere(14, 4.0), base_params(14, Nc_fundamental=4, Kn=0.3, maxStep=3000)),
    ]
    return [Job(img, p, name="j%d" % i, arrival=0.05 * i) for i, (img, p) in enumerate(specs)]


@pytest.mark.parametrize("precision", ["refined", "fp64"])
def test_batch_runner_equals_alone(precision):
    jobs = _jobs()
    alone = [solve_one(j.image, j.params, precision=precision, tol=1e-4) for j in jobs]
    r = BatchRunner(device=0, precision=precision, tol=1e-4, max_members=3)
    try:
        done = r.run(jobs)
    finally:
        r.close()
    assert len(done) == len(jobs)
    for j in jobs:
        a = alone[int(j.name[1:])]
        print(j.name, precision, j.result["steps"], j.result["steps32"], j.result["permeability"])
        assert j.result["converged"] and a["converged"]
        assert j.result["steps"] == a["steps"] and j.result["steps32"] == a["steps32"]
        assert j.result["permeability"] == a["permeability"]


def test_server_results_equal_alone():
    jobs = _jobs()
    alone = [solve_one(j.image, j.params, precision="refined", tol=1e-4) for j in jobs]
    r = BatchRunner(device=0, precision="refined", tol=1e-4, max_members=4)
    try:
        rep = Server(r).run(jobs)
    finally:
        r.close()
    assert rep["completed"] == len(jobs)
    print({k: v for k, v in rep.items() if k != "jobs"})
    for j in rep["jobs"]:
        assert j.result["permeability"] == alone[int(j.name[1:])]["permeability"]
        assert j.latency > 0


def test_refined_tolerance_solve_vs_oracle():
    img = images.centred_sphere(32, 12.0)
    p = base_params(32, Nc_fundamental=2, Kn=1.0, eps=1e-8, maxStep=2000)
    _, k_o, _ = Oracle(p, img.tobytes(), nthreads=8).run()
    res = solve_one(img, p, precision="refined", tol=1e-4)
    err = abs(res["permeability"] - k_o) / abs(k_o)
    print("refined, tol 1e-4: steps %d (%d FP32), perm rel err vs FP64 oracle %.3e" % (res["steps"], res["steps32"], err))
    assert err <= 1e-4
