"""piks3d_b200 — B200 solver for PIKS3D's discrete-velocity source iteration.

Python bindings of libpiks3d_b200.so (the C ABI in include/piks3d_gpu.h). The compute
path is the CUDA library; there is no CPU fallback: importing works without a GPU (to
read parameters or build images), but creating a Solver needs the built library and a
CUDA device and raises otherwise.

The call sequence mirrors PIKS3D's main.F90:
    p, image_file = read_params("para.in")      # initParams
    s = Solver(p)                                # setupVelocityGrid
    s.setup_physical_grid(raw_bytes)             # setupPhysicalGrid + setupFlow
    s.iterate(10); s.chk_converge()              # iterate / chkConverge
    s.save_fields(".", p.saveFormat)             # saveFlowFieldVTI / VTK / Tecplot
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpiks3d_b200.so")

__all__ = ["Params", "Solver", "read_params", "default_params", "PiksError", "load_library",
           "KERNEL_NAMES"]


class PiksError(RuntimeError):
    """A piks_* call returned a non-zero status; .status holds it."""

    def __init__(self, status, message):
        super().__init__("piks status %d: %s" % (status, message))
        self.status = status


class Params(ctypes.Structure):
    """piks_params: the para.in namelist variables (parameters.F90:78-82)."""
    _fields_ = [
        ("Nx", ctypes.c_int32), ("Ny", ctypes.c_int32), ("Nz", ctypes.c_int32),
        ("wallExtOrder", ctypes.c_int32), ("fluidlayer", ctypes.c_int32),
        ("Ref_L", ctypes.c_double),
        ("Nc_fundamental", ctypes.c_int32), ("halfRange", ctypes.c_int32),
        ("mpi_xdim", ctypes.c_int32), ("mpi_ydim", ctypes.c_int32), ("mpi_zdim", ctypes.c_int32),
        ("block_repx", ctypes.c_int32), ("block_repy", ctypes.c_int32), ("block_repz", ctypes.c_int32),
        ("maxStep", ctypes.c_int32), ("chkConvergeStep", ctypes.c_int32), ("saveStep", ctypes.c_int32),
        ("eps", ctypes.c_double),
        ("saveLast", ctypes.c_int32), ("saveFormat", ctypes.c_int32),
        ("Kn", ctypes.c_double), ("pressDrop", ctypes.c_double), ("accom", ctypes.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_lib = None


def load_library(path=LIB_PATH):
    """Load libpiks3d_b200.so (built by piks3d_b200.build); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise OSError("libpiks3d_b200.so not built: run `python -m piks3d_b200.build` (%s)" % path)
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    c_void_p, i32, i64, dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    sig = {
        "piks_params_default": (i32, [P(Params)]),
        "piks_read_params": (i32, [ctypes.c_char_p, P(Params), ctypes.c_char_p, i32]),
        "piks_create": (i32, [P(Params), i32, P(c_void_p)]),
        "piks_setup_physical_grid": (i32, [c_void_p, ctypes.c_char_p, i64]),
        "piks_iterate": (i32, [c_void_p, i32]),
        "piks_chk_converge": (i32, [c_void_p, P(dbl), P(dbl), P(dbl)]),
        "piks_run": (i32, [c_void_p, ctypes.c_char_p, ctypes.c_char_p, i32, P(i32), P(dbl), P(dbl)]),
        "piks_get_macro": (i32, [c_void_p, P(dbl), P(dbl), P(dbl), P(dbl)]),
        "piks_save_fields": (i32, [c_void_p, ctypes.c_char_p, i32]),
        "piks_get_labels": (i32, [c_void_p, P(i32)]),
        "piks_get_info": (i32, [c_void_p, P(i64), i32]),
        "piks_get_f": (i32, [c_void_p, P(dbl), P(dbl)]),
        "piks_get_f_nodes": (i32, [c_void_p, P(i32), i32, P(dbl)]),
        "piks_geometry_array": (i32, [c_void_p, ctypes.c_char_p, c_void_p, i64, P(i64)]),
        "piks_set_stream": (i32, [c_void_p, c_void_p]),
        "piks_set_preprocessing": (i32, [c_void_p, i32]),
        "piks_setup_seconds": (i32, [c_void_p, P(dbl)]),
        "piks_set_decomposition": (i32, [c_void_p, i32, i32]),
        "piks_snapshot_slot": (i32, [c_void_p, i32, i32]),
        "piks_snapshot_gram": (i32, [c_void_p, i32, P(dbl)]),
        "piks_snapshot_combine": (i32, [c_void_p, i32, P(dbl)]),
        "piks_get_slab": (i32, [c_void_p, P(i32)]),
        "piks_halo_buffers": (i32, [c_void_p, i32, P(c_void_p), P(c_void_p), P(i64)]),
        "piks_kernel_times": (i32, [c_void_p, P(dbl), i32, i32]),
        "piks_kernel_names": (ctypes.c_char_p, []),
        "piks_enable_timing": (i32, [c_void_p, i32]),
        "piks_launches_per_iteration": (i32, [c_void_p, P(i64)]),
        "piks_set_precision": (i32, [c_void_p, i32]),
        "piks_set_tiles": (i32, [c_void_p, i32, i32, i32]),
        "piks_get_schedule": (i32, [c_void_p, P(i32), i32]),
        "piks_set_schedule": (i32, [c_void_p, i32]),
        "piks_autotune": (i32, [c_void_p, P(i32), i32, i32, P(i32), P(dbl)]),
        "piks_get_precision": (i32, [c_void_p, P(i32)]),
        "piks_run_refined": (i32, [c_void_p, ctypes.c_char_p, ctypes.c_char_p, i32, dbl, P(i32), P(i32), P(dbl),
                                   P(dbl)]),
        "piks_batch_create": (i32, [i32, P(c_void_p)]),
        "piks_batch_add": (i32, [c_void_p, c_void_p]),
        "piks_batch_remove": (i32, [c_void_p, c_void_p]),
        "piks_batch_size": (i32, [c_void_p, P(i32)]),
        "piks_batch_iterate": (i32, [c_void_p, i32]),
        "piks_batch_chk_converge": (i32, [c_void_p, P(dbl), P(dbl), P(dbl)]),
        "piks_batch_synchronize": (i32, [c_void_p]),
        "piks_batch_destroy": (i32, [c_void_p]),
        "piks_synchronize": (i32, [c_void_p]),
        "piks_selftest_wait_timeout": (i32, [c_void_p, P(dbl)]),
        "piks_destroy": (i32, [c_void_p]),
        "piks_last_error": (ctypes.c_char_p, []),
    }
    for name, (res, args) in sig.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status):
    if status != 0:
        raise PiksError(status, _lib.piks_last_error().decode(errors="replace"))


def default_params(**overrides):
    """piks_params with initParams' defaults (parameters.F90:91-98) and `overrides`."""
    lib = load_library()
    p = Params()
    _check(lib.piks_params_default(ctypes.byref(p)))
    for k, v in overrides.items():
        setattr(p, k, v)
    return p


def read_params(path):
    """Read para.in (initParams, parameters.F90:100-118) -> (Params, imageFileName)."""
    lib = load_library()
    p = Params()
    buf = ctypes.create_string_buffer(512)
    _check(lib.piks_read_params(os.fsencode(path), ctypes.byref(p), buf, 512))
    return p, buf.value.decode()


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


PREC_FP64, PREC_FP32 = 0, 1
SCHED_TILE_DATAFLOW, SCHED_TILE_DIAGONALS, SCHED_TILE_COLUMNS, SCHED_TILE_PIPELINED = 0, 1, 2, 3
PREP_HOST, PREP_DEVICE = 0, 1

KERNEL_NAMES = ("sweep", "commit", "capture", "walls", "inlet_outlet", "symmetry", "moments", "flux")


class Solver:
    """One solve on one GPU through the C ABI (a piks_ctx). device=-1 makes a host-only
    context: image preprocessing and the geometry getters work, iterate raises."""

    def __init__(self, params, device=0):
        self.lib = load_library()
        self.params = params
        self._ctx = ctypes.c_void_p()
        _check(self.lib.piks_create(ctypes.byref(params), int(device), ctypes.byref(self._ctx)))

    # -- life cycle -------------------------------------------------------------------
    def close(self):
        if self._ctx:
            self.lib.piks_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- main.F90 call sequence ---------------------------------------------------------
    def setup_physical_grid(self, raw):
        """setupPhysicalGrid + setupFlow from the raw uint8 image stream (x fastest)."""
        data = bytes(np.ascontiguousarray(raw, dtype=np.uint8).reshape(-1)) if not isinstance(raw, (bytes, bytearray)) else bytes(raw)
        _check(self.lib.piks_setup_physical_grid(self._ctx, data, len(data)))

    def iterate(self, nsteps=1):
        _check(self.lib.piks_iterate(self._ctx, int(nsteps)))

    def chk_converge(self):
        """-> (mass, permeability, error) as chkConverge computes them."""
        m, k, e = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        _check(self.lib.piks_chk_converge(self._ctx, ctypes.byref(m), ctypes.byref(k), ctypes.byref(e)))
        return m.value, k.value, e.value

    def run(self, results_path=None, out_dir=None, verbose=False):
        """main.F90's loop -> (steps, permeability, seconds)."""
        steps, perm, secs = ctypes.c_int32(), ctypes.c_double(), ctypes.c_double()
        _check(self.lib.piks_run(self._ctx, os.fsencode(results_path) if results_path else None,
                                 os.fsencode(out_dir) if out_dir else None, int(bool(verbose)),
                                 ctypes.byref(steps), ctypes.byref(perm), ctypes.byref(secs)))
        return steps.value, perm.value, secs.value

    def run_refined(self, switch_eps=1e-6, results_path=None, out_dir=None, verbose=False):
        """FP32 iterations until error <= switch_eps (or the FP32 error stops improving), then
        FP64 iterations until error <= eps -> (fp32_steps, steps, permeability, seconds)."""
        s32, steps, perm, secs = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double(), ctypes.c_double()
        _check(self.lib.piks_run_refined(self._ctx, os.fsencode(results_path) if results_path else None,
                                         os.fsencode(out_dir) if out_dir else None, int(bool(verbose)),
                                         float(switch_eps), ctypes.byref(s32), ctypes.byref(steps),
                                         ctypes.byref(perm), ctypes.byref(secs)))
        return s32.value, steps.value, perm.value, secs.value

    def set_precision(self, precision):
        """PREC_FP64 (reference arithmetic) or PREC_FP32 (FP32 f and sweep, FP64 moments,
        wall densities and flux); converts a live state on the device."""
        _check(self.lib.piks_set_precision(self._ctx, int(precision)))

    def set_preprocessing(self, where):
        """PREP_DEVICE (default with a device) or PREP_HOST: where setup_physical_grid classifies
        the voxels; both give identical geometry."""
        _check(self.lib.piks_set_preprocessing(self._ctx, int(where)))

    def setup_seconds(self):
        """Seconds of the last setup: (box and drill / thin, classification, rest of the
        geometry, the whole call)."""
        a = (ctypes.c_double * 4)()
        _check(self.lib.piks_setup_seconds(self._ctx, a))
        return tuple(a)

    def snapshot_slot(self, slot, nslots):
        """Copies the iteration state into snapshot slot `slot` of `nslots` (device memory)."""
        _check(self.lib.piks_snapshot_slot(self._ctx, int(slot), int(nslots)))

    def snapshot_gram(self, n):
        """(n-1) x (n-1) Gram matrix of the differences of slots 0 .. n-1 (FP64)."""
        g = np.zeros((n - 1) * (n - 1))
        _check(self.lib.piks_snapshot_gram(self._ctx, int(n), _dptr(g)))
        return g.reshape(n - 1, n - 1)

    def snapshot_combine(self, coef):
        """The state becomes sum_j coef[j] * slot_j."""
        c = np.ascontiguousarray(coef, dtype=np.float64)
        _check(self.lib.piks_snapshot_combine(self._ctx, len(c), _dptr(c)))

    def set_decomposition(self, nranks, rank):
        """Makes this context rank `rank` of `nranks` x slabs of the box (before
        setup_physical_grid, which then takes the whole image on every rank)."""
        _check(self.lib.piks_set_decomposition(self._ctx, int(nranks), int(rank)))

    def slab(self):
        """{'xl', 'xu', 'nranks', 'rank'}: the owned x planes (global, 1-based)."""
        a = (ctypes.c_int32 * 4)()
        _check(self.lib.piks_get_slab(self._ctx, a))
        return dict(zip(("xl", "xu", "nranks", "rank"), list(a)))

    def halo_buffers(self, side):
        """(send_ptr, recv_ptr, send_bytes, recv_bytes) of the exchange on `side` (0 west,
        1 east) that precedes the next iteration; device pointers (0 for one rank)."""
        snd, rcv = ctypes.c_void_p(), ctypes.c_void_p()
        b = (ctypes.c_int64 * 2)()
        _check(self.lib.piks_halo_buffers(self._ctx, int(side), ctypes.byref(snd), ctypes.byref(rcv), b))
        return snd.value or 0, rcv.value or 0, b[0], b[1]

    def set_tiles(self, tx, ty=None, tz=None):
        """Tile shape of the sweep schedule (0 = per-node hyperplanes); applies at the next
        setup_physical_grid."""
        ty = tx if ty is None else ty
        tz = tx if tz is None else tz
        _check(self.lib.piks_set_tiles(self._ctx, int(tx), int(ty), int(tz)))

    def set_schedule(self, schedule):
        """SCHED_TILE_DATAFLOW (one launch per sweep) or SCHED_TILE_DIAGONALS."""
        _check(self.lib.piks_set_schedule(self._ctx, int(schedule)))

    def autotune(self, candidates=None, sweeps=2):
        """Times each (TX, TY, TZ, schedule) candidate on this image right after setup, keeps
        the fastest and resets the state; -> (chosen, {candidate: ms per sweep})."""
        if candidates:
            flat = (ctypes.c_int32 * (4 * len(candidates)))(*[int(v) for c in candidates for v in c])
            n = len(candidates)
        else:
            flat, n = None, 5
        chosen = (ctypes.c_int32 * 4)()
        ms = (ctypes.c_double * max(n, 5))()
        _check(self.lib.piks_autotune(self._ctx, flat, len(candidates) if candidates else 0, int(sweeps), chosen, ms))
        return tuple(chosen), ms[:n]

    def schedule(self):
        """{'tiles': bool, 'TX', 'TY', 'TZ', 'max_slots', 'launch', 'jobs'} of the sweep schedule."""
        a = (ctypes.c_int32 * 7)()
        _check(self.lib.piks_get_schedule(self._ctx, a, 7))
        return {"tiles": bool(a[0]), "TX": a[1], "TY": a[2], "TZ": a[3], "max_slots": a[4], "launch": a[5],
                "jobs": a[6]}

    @property
    def precision(self):
        v = ctypes.c_int32()
        _check(self.lib.piks_get_precision(self._ctx, ctypes.byref(v)))
        return v.value

    def synchronize(self):
        _check(self.lib.piks_synchronize(self._ctx))

    def selftest_wait_timeout(self):
        """Runs one dataflow sweep in which a job waits on a flag nothing sets; returns the
        sweep's duration (s) once the wait has given up as designed (piks_selftest_wait_timeout).
        The state's values are not the solver's afterwards: set the image up again."""
        sec = ctypes.c_double()
        _check(self.lib.piks_selftest_wait_timeout(self._ctx, ctypes.byref(sec)))
        return sec.value

    # -- data out -----------------------------------------------------------------------
    def info(self):
        a = (ctypes.c_int64 * 11)()
        _check(self.lib.piks_get_info(self._ctx, a, 11))
        keys = ("Nx", "Ny", "Nz", "Nc8", "Nfluid", "nWall", "nCorner", "nNodes", "iStep", "nWallLevels",
                "device_bytes")
        return dict(zip(keys, list(a)))

    def get_macro(self):
        """Rho, Ux, Uy, Uz as (Nz, Ny, Nx) arrays (0 at non-fluid voxels)."""
        inf = self.info()
        shape = (inf["Nz"], inf["Ny"], inf["Nx"])
        out = [np.zeros(shape, dtype=np.float64) for _ in range(4)]
        _check(self.lib.piks_get_macro(self._ctx, *[_dptr(a) for a in out]))
        return tuple(out)

    def get_labels(self):
        inf = self.info()
        lab = np.zeros((inf["Nz"], inf["Ny"], inf["Nx"]), dtype=np.int32)
        _check(self.lib.piks_get_labels(self._ctx, lab.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return lab

    def get_f(self):
        """(f in the reference layout f(Ntotal, Nc8, 8) column-major, fw(nCorner, Nc8, 8))."""
        inf = self.info()
        ntot = (inf["Nx"] + 4) * (inf["Ny"] + 4) * (inf["Nz"] + 4)
        f = np.zeros(ntot * inf["Nc8"] * 8, dtype=np.float64)
        fw = np.zeros(max(1, inf["nCorner"]) * inf["Nc8"] * 8, dtype=np.float64)
        _check(self.lib.piks_get_f(self._ctx, _dptr(f), _dptr(fw)))
        return f, fw[: inf["nCorner"] * inf["Nc8"] * 8]

    def get_fw(self):
        """fw(nCorner, Nc8, 8) column-major, without the full-box f."""
        inf = self.info()
        fw = np.zeros(max(1, inf["nCorner"]) * inf["Nc8"] * 8, dtype=np.float64)
        _check(self.lib.piks_get_f(self._ctx, None, _dptr(fw)))
        return fw[: inf["nCorner"] * inf["Nc8"] * 8]

    def get_f_nodes(self, nodes):
        """f of the given compact nodes as (n, 8, Nc8) float64 (octant, then velocity)."""
        nd = np.ascontiguousarray(nodes, dtype=np.int32)
        out = np.zeros((len(nd), 8, self.info()["Nc8"]), dtype=np.float64)
        _check(self.lib.piks_get_f_nodes(self._ctx, nd.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(nd),
                                         _dptr(out)))
        return out

    _GEO_DTYPES = {"label": np.uint8, "sym_flag": np.uint8, "roles": np.uint16, "wall_e": np.float64,
                   "hyper_start": np.int64, "tile_row_begin": np.int64, "tile_task_begin": np.int64,
                   "tile_carry_begin": np.int64,
                   "tile_steps": np.uint16,
                   "cx": np.float64, "cy": np.float64, "cz": np.float64, "w": np.float64}

    def geometry_array(self, name):
        """Host-side preprocessed geometry array by name (see piks_geometry_array)."""
        n = ctypes.c_int64()
        _check(self.lib.piks_geometry_array(self._ctx, name.encode(), None, 0, ctypes.byref(n)))
        a = np.zeros(max(1, n.value), dtype=self._GEO_DTYPES.get(name, np.int32))
        _check(self.lib.piks_geometry_array(self._ctx, name.encode(), a.ctypes.data_as(ctypes.c_void_p),
                                            a.nbytes, ctypes.byref(n)))
        return a[: n.value]

    def save_fields(self, out_dir, fmt=1):
        _check(self.lib.piks_save_fields(self._ctx, os.fsencode(out_dir), int(fmt)))

    # -- instrumentation ----------------------------------------------------------------
    def set_stream(self, stream_handle):
        """Enqueue on an external cudaStream_t (an int handle, e.g. torch's stream.cuda_stream)."""
        _check(self.lib.piks_set_stream(self._ctx, ctypes.c_void_p(stream_handle) if stream_handle else None))

    def enable_timing(self, on=True):
        _check(self.lib.piks_enable_timing(self._ctx, int(bool(on))))

    def kernel_times(self, reset=True):
        """{kernel: (milliseconds, launch groups)} accumulated with CUDA events."""
        buf = (ctypes.c_double * (2 * len(KERNEL_NAMES)))()
        _check(self.lib.piks_kernel_times(self._ctx, buf, len(buf), int(bool(reset))))
        return {k: (buf[2 * i], int(buf[2 * i + 1])) for i, k in enumerate(KERNEL_NAMES)}

    def launches_per_iteration(self):
        n = ctypes.c_int64()
        _check(self.lib.piks_launches_per_iteration(self._ctx, ctypes.byref(n)))
        return n.value


class Batch:
    """Several solves iterated together on one GPU (piks_batch_*): one dataflow sweep launch
    per precision class over all members' tile jobs, then each member's boundary kernels,
    replayed from a captured CUDA graph while the membership is unchanged."""

    def __init__(self, device=0):
        self.lib = load_library()
        self._b = ctypes.c_void_p()
        self.members = []
        _check(self.lib.piks_batch_create(int(device), ctypes.byref(self._b)))

    def add(self, solver):
        _check(self.lib.piks_batch_add(self._b, solver._ctx))
        if solver not in self.members:
            self.members.append(solver)

    def remove(self, solver):
        _check(self.lib.piks_batch_remove(self._b, solver._ctx))
        self.members.remove(solver)

    def __len__(self):
        return len(self.members)

    def iterate(self, nsteps=1):
        _check(self.lib.piks_batch_iterate(self._b, int(nsteps)))

    def chk_converge(self):
        """-> (mass, permeability, error) arrays in membership order."""
        n = len(self.members)
        m, k, e = (np.zeros(max(1, n)) for _ in range(3))
        _check(self.lib.piks_batch_chk_converge(self._b, _dptr(m), _dptr(k), _dptr(e)))
        return m[:n], k[:n], e[:n]

    def synchronize(self):
        _check(self.lib.piks_batch_synchronize(self._b))

    def close(self):
        if self._b:
            self.lib.piks_batch_destroy(self._b)
            self._b = ctypes.c_void_p()
            self.members = []

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
