"""The x-slab halo exchange over torch.distributed on CPU (gloo; world sizes 2 and 3): each
process runs one oracle rank and moves its x messages with piks3d_b200.slab.exchange, the
same point-to-point pattern the GPU ranks use with NCCL; the result equals the oracle's
ranks moved in one process (SlabOracle) bit for bit, and chkConverge's triple is rank 0's."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _case():
    from piks3d_b200 import images
    from conftest import base_params
    img = images.sphere_pack(14, 0.5, 1.5, 3.5, seed=11)
    return img, base_params(14, wallExtOrder=1, Kn=0.6)


def _worker(rank, world, port, iters, out):
    import datetime
    import torch
    import torch.distributed as dist
    for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")):
        sys.path.insert(0, p)
    from oracle import Oracle
    from piks3d_b200 import slab
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    img, p = _case()
    o = Oracle(p, img.tobytes(), 1, world, rank)
    for _ in range(iters):
        w, e = o.halo_send()
        send = (torch.from_numpy(w), torch.from_numpy(e))
        recv = (torch.zeros_like(send[0]), torch.zeros_like(send[1]))
        slab.exchange(send, recv, rank, world)
        o.halo_recv(recv[0].numpy(), recv[1].numpy())
        o.iterate(1)
    m, k, err = o.chk_converge()
    t = torch.tensor([m, k, err], dtype=torch.float64)
    dist.broadcast(t, src=0)
    sl = o.slab()
    mac = o.macro()
    lo = sl["xl"] - sl["xlg"]
    own = [a[2:-2, 2:-2, lo:lo + sl["xu"] - sl["xl"] + 1].copy() for a in mac]
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, sl["xl"], own, t.tolist()))


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_exchange_equals_in_process_ranks(world):
    from oracle import SlabOracle
    iters = 4
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, iters, q)) for r in range(world)]
    for pr in procs:
        pr.start()
    res = sorted((q.get(timeout=300) for _ in procs), key=lambda r: r[0])
    for pr in procs:
        pr.join(timeout=60)
        assert pr.exitcode == 0
    img, p = _case()
    so = SlabOracle(p, img.tobytes(), world, nthreads=1)
    so.iterate(iters)
    ref = so.macro()
    got = [np.concatenate([r[2][qq] for r in res], axis=2) for qq in range(4)]
    for a, b in zip(ref, got):
        assert np.array_equal(a, b)
    trip = so.chk_converge()
    for r in res:
        assert tuple(r[3]) == trip     # every rank holds rank 0's check after the broadcast
    so.close()
