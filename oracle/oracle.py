"""TEST INFRASTRUCTURE — ctypes binding of the CPU oracle (oracle/liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg use this
module, as the checker or as the timed CPU baseline; the product never imports it.
See piks_oracle.h for what it restates and for its parity status (unpinned).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class OracleParams(ctypes.Structure):
    _fields_ = [
        ("Nx", ctypes.c_int32), ("Ny", ctypes.c_int32), ("Nz", ctypes.c_int32),
        ("wallExtOrder", ctypes.c_int32), ("fluidlayer", ctypes.c_int32), ("Ref_L", ctypes.c_double),
        ("Nc_fundamental", ctypes.c_int32), ("halfRange", ctypes.c_int32),
        ("block_repx", ctypes.c_int32), ("block_repy", ctypes.c_int32), ("block_repz", ctypes.c_int32),
        ("maxStep", ctypes.c_int32), ("chkConvergeStep", ctypes.c_int32), ("saveStep", ctypes.c_int32),
        ("eps", ctypes.c_double), ("saveLast", ctypes.c_int32), ("saveFormat", ctypes.c_int32),
        ("Kn", ctypes.c_double), ("pressDrop", ctypes.c_double), ("accom", ctypes.c_double),
    ]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        d, i32, i64 = ctypes.c_double, ctypes.c_int32, ctypes.c_int64
        lib.oracle_create.restype = ctypes.c_void_p
        lib.oracle_create.argtypes = [P(OracleParams), ctypes.c_char_p, i64, ctypes.c_int, ctypes.c_char_p, ctypes.c_int]
        lib.oracle_destroy.argtypes = [ctypes.c_void_p]
        lib.oracle_iterate.argtypes = [ctypes.c_void_p, i32]
        lib.oracle_chk_converge.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, P(d), P(d), P(d)]
        lib.oracle_run.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, P(i32), P(d), P(d)]
        lib.oracle_dims.argtypes = [ctypes.c_void_p, P(i64)]
        lib.oracle_scalars.argtypes = [ctypes.c_void_p, P(d)]
        lib.oracle_velocity.argtypes = [ctypes.c_void_p, P(d), P(d), P(d), P(d)]
        for name in ("oracle_get_image", "oracle_get_which_corner", "oracle_get_vecwall", "oracle_get_mapf"):
            getattr(lib, name).argtypes = [ctypes.c_void_p, P(i32)]
        for name in ("oracle_get_extcoef", "oracle_get_f", "oracle_get_fw"):
            getattr(lib, name).argtypes = [ctypes.c_void_p, P(d)]
        lib.oracle_set_f.argtypes = [ctypes.c_void_p, P(d)]
        lib.oracle_get_f_at.argtypes = [ctypes.c_void_p, P(i64), i32, P(d)]
        lib.oracle_get_macro.argtypes = [ctypes.c_void_p, P(d), P(d), P(d), P(d)]
        lib.oracle_get_dir.argtypes = [ctypes.c_void_p, ctypes.c_int, P(i32)]
        lib.oracle_get_coef.argtypes = [ctypes.c_void_p, ctypes.c_int, P(d)]
        lib.oracle_save.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int]
        lib.oracle_save.restype = ctypes.c_int
        lib.oracle_create_rank.restype = ctypes.c_void_p
        lib.oracle_create_rank.argtypes = [P(OracleParams), ctypes.c_char_p, i64, ctypes.c_int, i32, i32,
                                           ctypes.c_char_p, ctypes.c_int]
        lib.oracle_slab.argtypes = [ctypes.c_void_p, P(i32)]
        lib.oracle_halo_size.restype = i64
        lib.oracle_halo_size.argtypes = [ctypes.c_void_p]
        lib.oracle_halo_send.argtypes = [ctypes.c_void_p, P(d), P(d)]
        lib.oracle_halo_recv.argtypes = [ctypes.c_void_p, P(d), P(d)]
        lib.oracle_set_fw.argtypes = [ctypes.c_void_p, P(d)]
        lib.oracle_set_macro.argtypes = [ctypes.c_void_p, P(d), P(d), P(d), P(d)]
        lib.oracle_set_halo_send.argtypes = [ctypes.c_void_p, P(d), P(d)]
        _lib = lib
    return _lib


def _d(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _i(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


DIM_KEYS = ("Nx", "Ny", "Nz", "Nxtotal", "Nytotal", "Nztotal", "Ntotal", "Nc8", "nWall", "nCorner",
            "Nfluid", "iStep") + tuple("Nstencil%d" % o for o in range(1, 9))


class Oracle:
    """CPU restatement of PIKS3D for one rank (reference layout f(Ntotal, Nc8, 8) over the
    rank's ghosted box); `nranks` > 1 makes it rank `rank` of an x-only process grid."""

    def __init__(self, params, raw, nthreads=0, nranks=1, rank=0):
        lib = load()
        op = OracleParams()
        for name, _ in OracleParams._fields_:
            setattr(op, name, getattr(params, name) if not isinstance(params, dict) else params[name])
        data = bytes(np.ascontiguousarray(raw, dtype=np.uint8).reshape(-1)) if not isinstance(raw, (bytes, bytearray)) else bytes(raw)
        err = ctypes.create_string_buffer(256)
        self.h = lib.oracle_create_rank(ctypes.byref(op), data, len(data), int(nthreads), int(nranks), int(rank),
                                        err, 256)
        if not self.h:
            raise ValueError(err.value.decode())
        self.lib = lib

    def close(self):
        if self.h:
            self.lib.oracle_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def dims(self):
        a = np.zeros(20, dtype=np.int64)
        self.lib.oracle_dims(self.h, a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
        return dict(zip(DIM_KEYS, a.tolist()))

    def scalars(self):
        a = np.zeros(6)
        self.lib.oracle_scalars(self.h, _d(a))
        return dict(zip(("ds", "mu", "DiffFlux", "mass", "error", "permeability"), a.tolist()))

    def velocity(self):
        n = self.dims()["Nc8"]
        out = [np.zeros(n) for _ in range(4)]
        self.lib.oracle_velocity(self.h, *[_d(a) for a in out])
        return out

    def iterate(self, n=1):
        self.lib.oracle_iterate(self.h, int(n))

    def chk_converge(self, results_path=None, verbose=False):
        m, k, e = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
        self.lib.oracle_chk_converge(self.h, os.fsencode(results_path) if results_path else None, int(verbose),
                                     ctypes.byref(m), ctypes.byref(k), ctypes.byref(e))
        return m.value, k.value, e.value

    def run(self, results_path=None, verbose=False):
        s, k, t = ctypes.c_int32(), ctypes.c_double(), ctypes.c_double()
        self.lib.oracle_run(self.h, os.fsencode(results_path) if results_path else None, int(verbose),
                            ctypes.byref(s), ctypes.byref(k), ctypes.byref(t))
        return s.value, k.value, t.value

    def image(self):
        d = self.dims()
        a = np.zeros(d["Ntotal"], dtype=np.int32)
        self.lib.oracle_get_image(self.h, _i(a))
        return a.reshape(d["Nztotal"], d["Nytotal"], d["Nxtotal"])

    def labels(self):
        """Interior labels as (Nz, Ny, Nx)."""
        return self.image()[2:-2, 2:-2, 2:-2]

    def f(self):
        d = self.dims()
        a = np.zeros(d["Ntotal"] * d["Nc8"] * 8)
        self.lib.oracle_get_f(self.h, _d(a))
        return a

    def f_at(self, gidx):
        """f of the voxels at 0-based ghosted linear indices gidx, as (n, 8, Nc8)."""
        g = np.ascontiguousarray(gidx, dtype=np.int64)
        n8 = self.dims()["Nc8"]
        out = np.zeros((len(g), 8, n8))
        self.lib.oracle_get_f_at(self.h, g.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), len(g), _d(out))
        return out

    def set_f(self, a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        self.lib.oracle_set_f(self.h, _d(a))

    def fw(self):
        d = self.dims()
        a = np.zeros(max(1, d["nCorner"]) * d["Nc8"] * 8)
        self.lib.oracle_get_fw(self.h, _d(a))
        return a[: d["nCorner"] * d["Nc8"] * 8]

    def macro(self):
        """Rho, Ux, Uy, Uz over the ghosted box, shaped (Nztotal, Nytotal, Nxtotal)."""
        d = self.dims()
        out = [np.zeros(d["Ntotal"]) for _ in range(4)]
        self.lib.oracle_get_macro(self.h, *[_d(a) for a in out])
        return [a.reshape(d["Nztotal"], d["Nytotal"], d["Nxtotal"]) for a in out]

    def extcoef(self):
        n = self.dims()["nWall"]
        a = np.zeros(max(1, 2 * n))
        self.lib.oracle_get_extcoef(self.h, _d(a))
        return a[: 2 * n].reshape(2, n)

    def vecwall(self):
        n = self.dims()["nWall"]
        a = np.zeros(max(1, n), dtype=np.int32)
        self.lib.oracle_get_vecwall(self.h, _i(a))
        return a[:n]

    def save(self, out_dir, fmt):
        return self.lib.oracle_save(self.h, os.fsencode(out_dir), int(fmt))

    def slab(self):
        """{'xl', 'xu', 'xlg', 'nranks', 'rank'} (global 1-based x)."""
        a = np.zeros(5, dtype=np.int32)
        self.lib.oracle_slab(self.h, _i(a))
        return dict(zip(("xl", "xu", "xlg", "nranks", "rank"), a.tolist()))

    def halo_send(self):
        """(west, east): the x messages the last iteration packed (solver.F90:535-612)."""
        n = self.lib.oracle_halo_size(self.h)
        w, e = np.zeros(n), np.zeros(n)
        self.lib.oracle_halo_send(self.h, _d(w), _d(e))
        return w, e

    def state(self):
        """(f, fw, macro list, (west_snd, east_snd)): everything the next iteration reads."""
        return self.f(), self.fw().copy(), [m.copy() for m in self.macro()], self.halo_send()

    def set_state(self, st):
        f, fw, mac, (w, e) = st
        self.set_f(f)
        d = self.dims()
        fwb = np.zeros(max(1, d["nCorner"]) * d["Nc8"] * 8)
        fwb[:fw.size] = fw
        self.lib.oracle_set_fw(self.h, _d(fwb))
        m = [np.ascontiguousarray(a, dtype=np.float64).reshape(-1) for a in mac]
        self.lib.oracle_set_macro(self.h, *[_d(a) for a in m])
        w = np.ascontiguousarray(w, dtype=np.float64)
        e = np.ascontiguousarray(e, dtype=np.float64)
        self.lib.oracle_set_halo_send(self.h, _d(w), _d(e))

    def halo_recv(self, west, east):
        """Sets the messages received from the west / east neighbour for the next iteration."""
        w = np.ascontiguousarray(west, dtype=np.float64)
        e = np.ascontiguousarray(east, dtype=np.float64)
        self.lib.oracle_halo_recv(self.h, _d(w), _d(e))


class SlabOracle:
    """`nranks` oracle ranks along x in one process, iterated together with the x messages
    moved between them before every iteration as MPI moves them in solver.F90:146-170
    (rank r receives its west message from rank r-1's east buffer and its east message from
    rank r+1's west buffer, periodic in x)."""

    def __init__(self, params, raw, nranks, nthreads=0):
        self.ranks = [Oracle(params, raw, nthreads, nranks, r) for r in range(nranks)]

    def close(self):
        for o in self.ranks:
            o.close()

    def exchange(self):
        n = len(self.ranks)
        if n == 1:
            return
        sent = [o.halo_send() for o in self.ranks]
        for r, o in enumerate(self.ranks):
            o.halo_recv(sent[(r - 1) % n][1], sent[(r + 1) % n][0])

    def iterate(self, n=1):
        for _ in range(n):
            self.exchange()
            for o in self.ranks:
                o.iterate(1)

    def chk_converge(self):
        """The west-most rank's (mass, k, error) (output.F90:89-162)."""
        return self.ranks[0].chk_converge()

    def macro(self):
        """Rho, Ux, Uy, Uz over the whole box's interior, (Nz, Ny, Nx), from the owning ranks."""
        parts = []
        for o in self.ranks:
            sl = o.slab()
            a = o.macro()
            lo = sl["xl"] - sl["xlg"]
            parts.append([m[2:-2, 2:-2, lo:lo + sl["xu"] - sl["xl"] + 1] for m in a])
        return [np.concatenate([p[q] for p in parts], axis=2) for q in range(4)]

    def f_at_global(self, i, j, k):
        """f rows (n, 8, Nc8) at global 1-based voxels from their owning ranks."""
        i, j, k = (np.asarray(v, dtype=np.int64) for v in (i, j, k))
        d0 = self.ranks[0].dims()
        out = np.zeros((len(i), 8, d0["Nc8"]))
        for o in self.ranks:
            sl, d = o.slab(), o.dims()
            sel = (i >= sl["xl"]) & (i <= sl["xu"])
            if not sel.any():
                continue
            g = (i[sel] - sl["xlg"]) + (j[sel] + 1) * d["Nxtotal"] + (k[sel] + 1) * d["Nxtotal"] * d["Nytotal"]
            out[sel] = o.f_at(g)
        return out
