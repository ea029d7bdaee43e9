"""Makes mass_trace_turning.json (needs a GPU): the chkConverge mass-flux trace, every 10
iterations for 2500 iterations, of image 2 of the batching workload (96^3 sphere pack,
porosity 0.35, 64 velocities, Kn 0.12, FP64). Its mass flux falls, passes a turning point
near iteration 600 and rises slowly: a stopping rule must not stop at the turning point.

    python tests/golden/make_trace_turning.py
"""
import json
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import bench  # noqa: E402
import piks3d_b200 as pk  # noqa: E402


def main():
    job = bench.batch_jobs(pk, 16, 2024, 20000)[2]
    s = pk.Solver(job.params, device=0)
    s.setup_physical_grid(job.image)
    masses = []
    for _ in range(250):
        s.iterate(10)
        masses.append(s.chk_converge()[0])
    s.close()
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "mass_trace_turning.json")
    json.dump({"what": "mass flux every 10 iterations, batching workload image 2 (FP64)", "masses": masses},
              open(out, "w"))


if __name__ == "__main__":
    main()
