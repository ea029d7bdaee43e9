"""GPU test of the bounded waits of the dataflow sweep, without a fault, trap or hang: one job
waits on a flag that nothing sets; its wait gives up after its iteration limit (about a
second), sets the sweep's error flag, and every job finishes. The context stays usable: set
up again, it iterates exactly as a fresh context does."""
import numpy as np
import pytest

import piks3d_b200 as pk
from piks3d_b200 import images
from conftest import base_params

pytestmark = pytest.mark.gpu


def test_dataflow_wait_gives_up_and_context_stays_usable():
    img = images.sphere_pack(12, 0.5, 1.5, 3.0, seed=7)
    p = base_params(12, Nc_fundamental=2, Kn=1.0)
    with pk.Solver(p, device=0) as s:
        s.set_tiles(4, 4, 4)
        s.setup_physical_grid(img)
        sec = s.selftest_wait_timeout()
        print("dataflow sweep with a wait on a flag nothing sets: %.3f s" % sec)
        assert 0.05 < sec < 10.0
        s.setup_physical_grid(img)
        s.set_schedule(pk.SCHED_TILE_DATAFLOW)
        s.iterate(4)
        a = (s.get_f()[0], s.chk_converge())
    with pk.Solver(p, device=0) as r:
        r.set_tiles(4, 4, 4)
        r.setup_physical_grid(img)
        r.iterate(4)
        b = (r.get_f()[0], r.chk_converge())
    assert np.array_equal(a[0], b[0]) and a[1] == b[1]
