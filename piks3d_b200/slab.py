"""One box over several GPUs: x slabs, one per rank.

The reference decomposes its box with MPI over a Cartesian grid (mpiParams.F90:120-240); with
mpi_xdim = ranks and mpi_ydim = mpi_zdim = 1 every rank owns the x planes [xl, xu] of its
partition and receives two planes of each neighbour (periodic in x) one iteration behind
(solver.F90:146-170 sends at the start of an iteration what the previous one packed,
:535-612 packs and unpacks after the sweeps). The library does the packing and unpacking
inside each iteration (piks_set_decomposition, piks_halo_buffers); this module moves the
buffers between iterations:

- `SlabSolver`: one rank per process and GPU, the buffers moved by torch.distributed
  point-to-point calls (NCCL over NVLink between GPUs; gloo for CPU tensors), ordered on
  the context's stream;
- `LocalSlabs`: all ranks in one process (one GPU or several), the buffers moved by device
  copies between iterations.

Only the west-most rank holds the plane x = 2 of chkConverge (output.F90:89); its
(mass, k, error) is broadcast to the others (output.F90:162).
"""
import numpy as np

from . import PREC_FP32, PREC_FP64, Solver


class _DeviceBytes:
    """A device buffer (pointer, byte count) as a __cuda_array_interface__ object."""

    def __init__(self, ptr, nbytes):
        self.__cuda_array_interface__ = {"shape": (int(nbytes),), "typestr": "|u1", "data": (int(ptr), False),
                                         "version": 3}


def device_bytes(ptr, nbytes, device):
    """A torch uint8 tensor viewing `nbytes` of device memory at `ptr` (no copy)."""
    import torch
    if not nbytes:
        return torch.empty(0, dtype=torch.uint8, device=device)
    return torch.as_tensor(_DeviceBytes(ptr, nbytes), device=device)


def neighbours(rank, world):
    """(west, east) ranks of an x-periodic ring."""
    return (rank - 1) % world, (rank + 1) % world


def exchange(send, recv, rank, world, group=None):
    """Moves this rank's halo buffers: send = (to_west, to_east), recv = (from_west,
    from_east), torch tensors on the process group's device kind. Rank r's from_west
    receives rank r-1's to_east and its from_east rank r+1's to_west. The calls are
    posted in the same order on every rank (to the west, from the east, to the east, from
    the west), so two ranks, each other's west and east neighbour, pair them correctly;
    empty buffers are skipped on both sides of a pair alike (their sizes agree)."""
    import torch.distributed as dist
    if world == 1:
        return
    west, east = neighbours(rank, world)
    ops = []
    if send[0].numel():
        ops.append(dist.P2POp(dist.isend, send[0], west, group))
    if recv[1].numel():
        ops.append(dist.P2POp(dist.irecv, recv[1], east, group))
    if send[1].numel():
        ops.append(dist.P2POp(dist.isend, send[1], east, group))
    if recv[0].numel():
        ops.append(dist.P2POp(dist.irecv, recv[0], west, group))
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()


class SlabSolver:
    """Rank `rank` of `world` x slabs of one box, one process per GPU (torch.distributed
    initialised, NCCL backend). Every rank passes the whole image."""

    def __init__(self, params, image, device=0, group=None, precision="fp64"):
        import torch
        import torch.distributed as dist
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.device = torch.device("cuda", device)
        self.solver = Solver(params, device=device)
        self.solver.set_decomposition(self.world, self.rank)
        if precision == "fp32":
            self.solver.set_precision(PREC_FP32)
        # the context enqueues on a torch stream, so that the point-to-point calls made with
        # it current are ordered after one iteration and before the next
        self.stream = torch.cuda.Stream(device=self.device)
        self.solver.set_stream(self.stream.cuda_stream)
        self.solver.setup_physical_grid(image)
        self.params = params

    def close(self):
        self.solver.close()

    def _buffers(self):
        snd, rcv = [], []
        for side in (0, 1):
            sp, rp, sb, rb = self.solver.halo_buffers(side)
            snd.append(device_bytes(sp, sb, self.device))
            rcv.append(device_bytes(rp, rb, self.device))
        return snd, rcv

    def iterate(self, n=1):
        import torch
        for _ in range(n):
            with torch.cuda.stream(self.stream):
                snd, rcv = self._buffers()
                exchange(snd, rcv, self.rank, self.world, self.group)
            self.solver.iterate(1)

    def chk_converge(self):
        """(mass, k, error) of rank 0, on every rank."""
        import torch
        import torch.distributed as dist
        m, k, e = self.solver.chk_converge()
        if self.world == 1:
            return m, k, e
        with torch.cuda.stream(self.stream):
            t = torch.tensor([m, k, e], dtype=torch.float64, device=self.device)
            dist.broadcast(t, src=0, group=self.group)
            out = t.cpu().tolist()
        return tuple(out)

    def owned_macro(self):
        """(xl, xu, [Rho, Ux, Uy, Uz] over the owned planes, (Nz, Ny, xu - xl + 1))."""
        sl = self.solver.slab()
        mac = self.solver.get_macro()
        return sl["xl"], sl["xu"], [a[:, :, sl["xl"] - 1:sl["xu"]] for a in mac]


class LocalSlabs:
    """`nranks` x slabs of one box in one process, each a context on devices[r % len]
    (several on one GPU run one after another), the halos moved by device copies between
    iterations. For tests and single-process use; `SlabSolver` is the multi-GPU path."""

    def __init__(self, params, image, nranks, devices=(0,), precision="fp64", tiles=None, schedule=None):
        self.solvers = []
        for r in range(nranks):
            s = Solver(params, device=devices[r % len(devices)])
            s.set_decomposition(nranks, r)
            if tiles is not None:
                s.set_tiles(*tiles)
            if schedule is not None:
                s.set_schedule(schedule)
            if precision == "fp32":
                s.set_precision(PREC_FP32)
            s.setup_physical_grid(image)
            self.solvers.append(s)
        self.devices = [devices[r % len(devices)] for r in range(nranks)]

    def close(self):
        for s in self.solvers:
            s.close()

    def exchange(self):
        import torch
        n = len(self.solvers)
        if n == 1:
            return
        for s in self.solvers:
            s.synchronize()
        bufs = []
        for s, d in zip(self.solvers, self.devices):
            dev = torch.device("cuda", d)
            sides = [s.halo_buffers(side) for side in (0, 1)]
            bufs.append(([device_bytes(sp, sb, dev) for sp, _, sb, _ in sides],
                         [device_bytes(rp, rb, dev) for _, rp, _, rb in sides]))
        for r in range(n):
            west, east = neighbours(r, n)
            bufs[r][1][0].copy_(bufs[west][0][1])
            bufs[r][1][1].copy_(bufs[east][0][0])
        for d in set(self.devices):
            torch.cuda.synchronize(d)

    def iterate(self, n=1):
        for _ in range(n):
            self.exchange()
            for s in self.solvers:
                s.iterate(1)

    def chk_converge(self):
        return self.solvers[0].chk_converge()

    def set_precision(self, prec):
        for s in self.solvers:
            s.set_precision(prec)

    def macro(self):
        """Rho, Ux, Uy, Uz over the box (Nz, Ny, Nx), each plane from its owning rank."""
        parts = []
        for s in self.solvers:
            sl = s.slab()
            mac = s.get_macro()
            parts.append([a[:, :, sl["xl"] - 1:sl["xu"]] for a in mac])
        return [np.concatenate([p[q] for p in parts], axis=2) for q in range(4)]
