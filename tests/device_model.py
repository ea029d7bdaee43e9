"""CPU model of the device algorithm (test infrastructure).

Runs, in numpy over the velocity index, the same data flow as the CUDA kernels of
libpiks3d_b200 on the geometry the library's host preprocessing exports (compact node
list, static switch roles, post-sweep commits, lagged x ghost planes, wall programs and
their dependency levels, inlet/outlet, symmetry, moments, flux). The octant sweeps run in
raster order instead of the kernels' pencil wavefront; both respect the same upwind
dependencies. Comparing this model with the oracle checks the layout and the switch
resolution on the CPU; the GPU tests check the kernels themselves.
"""
import math
import os
import re

import numpy as np

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "piks3d_b200", "csrc")
SX = (1, -1, -1, 1, 1, -1, -1, 1)
SY = (1, 1, -1, -1, 1, 1, -1, -1)
SZ = (1, 1, 1, 1, -1, -1, -1, -1)
INCOMING = ((2, 3, 6, 7), (1, 4, 5, 8), (3, 4, 7, 8), (1, 2, 5, 6), (5, 6, 7, 8), (1, 2, 3, 4))
FACE = {20: 1, 21: 2, 22: 4, 23: 8, 24: 16, 25: 32}


def _face_mask(lab):
    m = {20: "E", 21: "W", 22: "N", 23: "S", 24: "F", 25: "B", 30: "EN", 31: "WN", 32: "ES", 33: "WS",
         40: "NF", 41: "NB", 42: "SF", 43: "SB", 50: "EF", 51: "EB", 52: "WF", 53: "WB",
         60: "ENF", 61: "WNF", 62: "WSF", 63: "ESF", 70: "ENB", 71: "WNB", 72: "WSB", 73: "ESB"}.get(int(lab), "")
    bits = {"E": 1, "W": 2, "N": 4, "S": 8, "F": 16, "B": 32}
    return sum(bits[c] for c in m)


FACE_MASK = np.array([_face_mask(i) for i in range(128)], dtype=np.int64)


def wall_programs():
    """Parse wall_table.inc rows -> {label: (faces, writes)} (0=F, 1=Z, 2=W stores)."""
    txt = open(os.path.join(CSRC, "wall_table.inc")).read()
    progs = {}
    store = {"ST_F": 0, "ST_Z": 1, "ST_W": 2}
    dirs = {"DIR_PX": 0, "DIR_MX": 1, "DIR_PY": 2, "DIR_MY": 3, "DIR_PZ": 4, "DIR_MZ": 5}
    for line in txt.splitlines():
        m = re.match(r"\s*/\*\s*(\w+)\s*\*/\s*\{(\d+), (\d+), \{(.*?)\}\}, (\d+), \{(.*)\}\},", line)
        if not m:
            continue
        lab = int(m.group(2))
        faces = [(dirs[a], store[b]) for a, b in re.findall(r"(DIR_\w+), (ST_\w)", m.group(4))]
        writes = [(store[a], int(b), int(c), store[d], int(e))
                  for a, b, c, d, e in re.findall(r"\{(ST_\w), (\d+), (\d+), (ST_\w), (\d+)\}", m.group(6))]
        progs[lab] = (faces, writes)
    return progs


class DeviceModel:
    def __init__(self, solver, params):
        g = solver.geometry_array
        inf = solver.info()
        self.Nx, self.Ny, self.Nz, self.Nc8 = inf["Nx"], inf["Ny"], inf["Nz"], inf["Nc8"]
        self.NF, self.nn, self.nCorner = inf["Nfluid"], inf["nNodes"], inf["nCorner"]
        self.GX, self.GY = self.Nx + 4, self.Ny + 4
        self.label = g("label").astype(np.int64)
        self.nodemap = g("nodemap").astype(np.int64)
        self.node_g = g("node_g").astype(np.int64)
        self.roles = g("roles").astype(np.int64).reshape(-1, 8)
        self.bcorner = g("bcorner")
        self.commit = g("commit").reshape(-1, 3)
        self.wall_node, self.wall_label = g("wall_node"), g("wall_label")
        self.wall_e, self.wall_corner = g("wall_e").reshape(-1, 2), g("wall_corner")
        self.wall_nb = g("wall_nb").reshape(-1, 6)
        self.wall_order, self.level_start = g("wall_order"), g("level_start")
        self.plane_x1, self.plane_xN = g("plane_x1"), g("plane_xN")
        self.sym_node, self.sym_flag = g("sym_node"), g("sym_flag")
        self.flux_list, self.flux_groups = g("flux_list"), g("flux_groups")
        self.cx, self.cy, self.cz, self.w = g("cx"), g("cy"), g("cz"), g("w")
        self.tasks = g("tasks").reshape(-1, 8)
        self.hyper_start = g("hyper_start")
        fl = params.fluidlayer
        self.ds = 1.0 / (self.Nx - 1 - 2 * fl)
        self.mu = math.sqrt((math.atan(1.0) * 4.0) / 2.0) / params.Kn
        self.p = params
        self.DiffFlux = self._diffflux()
        self.h = np.zeros((self.nn, 8, self.Nc8))
        self.fw = np.zeros((max(1, self.nCorner), 8, self.Nc8))
        self.mom = np.zeros((4, self.NF))
        rows = self.Ny * self.Nz
        self.gW = np.zeros((2, rows, 4, self.Nc8))
        self.gE = np.zeros((2, rows, 4, self.Nc8))
        self.iStep = 0
        self.progs = wall_programs()
        self.mass = 1.0
        # x halos of a slab (side 0 west, 1 east): node lists, send buffers by parity, receive
        sl = solver.slab()
        self.slab = sl
        self.nranks = sl["nranks"]
        self.hsend_nodes = [g("halo_send_w"), g("halo_send_e")]
        self.hrecv_nodes = [g("halo_recv_w"), g("halo_recv_e")]
        self.hs = [[np.zeros((len(self.hsend_nodes[sd]), 4, self.Nc8)) for _ in range(2)] for sd in range(2)]
        self.hr = [np.zeros((len(self.hrecv_nodes[sd]), 4, self.Nc8)) for sd in range(2)]
        self.wglob, self.eglob = sl["xl"] == 1, sl["xu"] == self.Nx

    def _diffflux(self):
        d = 0.0
        for l in range(self.Nc8):
            d = d + self.cz[l] * self.w[l]
        return d * 4

    def gidx(self, i, j, k):
        return (i + 1) + (j + 1) * self.GX + (k + 1) * self.GX * self.GY

    # --- sweep -------------------------------------------------------------------------
    def _upwind(self, gq, o, role):
        m = self.nodemap[gq]
        if 0 <= m < self.NF:
            return self.h[m, o]
        if m >= self.NF:
            b = m - self.NF
            src = (self.roles[b, o] >> (4 * role)) & 15 if role >= 0 else o
            if src < 8:
                return self.h[m, src]
            return self.fw[self.bcorner[b], o]
        return np.zeros(self.Nc8)

    def sweep(self, o):
        sx, sy, sz = SX[o], SY[o], SZ[o]
        Nx, Ny, Nz = self.Nx, self.Ny, self.Nz
        rng = lambda s, n: range(2, n + 1) if s > 0 else range(n - 1, 0, -1)
        c15, c20, c05, c10 = 1.5 / self.ds, 2.0 / self.ds, -0.5 / self.ds, 1.0 / self.ds
        sg = lambda s, v: v if s > 0 else -v
        SYs, SZs = sy * self.GX, sz * self.GX * self.GY
        cx, cy, cz, w, mu = self.cx, self.cy, self.cz, self.w, self.mu
        for k in rng(sz, Nz):
            for j in rng(sy, Ny):
                for i in rng(sx, Nx):
                    g = self.gidx(i, j, k)
                    m = self.nodemap[g]
                    if not (0 <= m < self.NF):
                        continue
                    u = i - 1 if sx > 0 else Nx - i
                    v = j - 1 if sy > 0 else Ny - j
                    ww = k - 1 if sz > 0 else Nz - k
                    fx = u == 1 or FACE_MASK[self.label[g - sx]] & (1 if sx > 0 else 2)
                    fy = v == 1 or FACE_MASK[self.label[g - SYs]] & (4 if sy > 0 else 8)
                    fz = ww == 1 or FACE_MASK[self.label[g - SZs]] & (16 if sz > 0 else 32)
                    x1 = self._upwind(g - sx, o, -1)
                    x2 = self._upwind(g - 2 * sx, o, -1)
                    y1 = self._upwind(g - SYs, o, 0)
                    y2 = self._upwind(g - 2 * SYs, o, 1)
                    z1 = self._upwind(g - SZs, o, 2)
                    z2 = self._upwind(g - 2 * SZs, o, 3)
                    fold = self.h[m, o]
                    ex = cx * self.mom[1, m]
                    ey = cy * self.mom[2, m]
                    ez = cz * self.mom[3, m]
                    if sx < 0: ex = -ex
                    if sy < 0: ey = -ey
                    if sz < 0: ez = -ez
                    feq = w * (self.mom[0, m] + ((ex + ey) + ez))
                    num = mu * (feq - 0.5 * fold)
                    for s, c, val, C in ((sx, cx, x1, c10 if fx else c20), (sx, cx, x2, 0.0 if fx else c05),
                                         (sy, cy, y1, c10 if fy else c20), (sy, cy, y2, 0.0 if fy else c05),
                                         (sz, cz, z1, c10 if fz else c20), (sz, cz, z2, 0.0 if fz else c05)):
                        t = (c * sg(s, C) if C != 0.0 else c * 0.0) * val
                        num = num + t if s > 0 else num - t
                    den = 0.5 * mu
                    for s, c, C in ((sx, cx, c10 if fx else c15), (sy, cy, c10 if fy else c15), (sz, cz, c10 if fz else c15)):
                        t = c * sg(s, C)
                        den = den + t if s > 0 else den - t
                    self.h[m, o] = num / den

    def _row(self, code):
        if code == -2:
            return None
        if code & (1 << 30):
            c = code & ~(1 << 30)
            return self.fw[c // 8, c % 8]
        return self.h[code // 8, code % 8]

    def sweep_tasks(self):
        """All eight octant sweeps from the library's task list, hyperplane by hyperplane."""
        c15, c10 = 1.5 / self.ds, 1.0 / self.ds
        P = {"x2": self.cx * (2.0 / self.ds), "x1": self.cx * c10, "xh": self.cx * (-0.5 / self.ds),
             "y2": self.cy * (2.0 / self.ds), "y1": self.cy * c10, "yh": self.cy * (-0.5 / self.ds),
             "z2": self.cz * (2.0 / self.ds), "z1": self.cz * c10, "zh": self.cz * (-0.5 / self.ds)}
        dens = {}
        for cls in range(8):
            d = 0.5 * self.mu + self.cx * (c10 if cls & 1 else c15)
            d = d + self.cy * (c10 if cls & 2 else c15)
            dens[cls] = d + self.cz * (c10 if cls & 4 else c15)
        for h in range(len(self.hyper_start) - 1):
            rows = self.tasks[self.hyper_start[h]:self.hyper_start[h + 1]]
            new = []
            for t in rows:
                m, fl = int(t[0]), int(t[1])
                o = fl & 7
                fx, fy, fz = bool(fl & 8), bool(fl & 16), bool(fl & 32)
                ex = (-self.cx if SX[o] < 0 else self.cx) * self.mom[1, m]
                ey = (-self.cy if SY[o] < 0 else self.cy) * self.mom[2, m]
                ez = (-self.cz if SZ[o] < 0 else self.cz) * self.mom[3, m]
                feq = self.w * (self.mom[0, m] + ((ex + ey) + ez))
                num = self.mu * (feq - 0.5 * self.h[m, o])
                num = num + (P["x1"] if fx else P["x2"]) * self._row(int(t[2]))
                if not fx:
                    num = num + P["xh"] * self._row(int(t[3]))
                num = num + (P["y1"] if fy else P["y2"]) * self._row(int(t[4]))
                if not fy:
                    num = num + P["yh"] * self._row(int(t[5]))
                num = num + (P["z1"] if fz else P["z2"]) * self._row(int(t[6]))
                if not fz:
                    num = num + P["zh"] * self._row(int(t[7]))
                cls = (1 if fx else 0) | (2 if fy else 0) | (4 if fz else 0)
                new.append((m, o, num / dens[cls]))
            for m, o, val in new:   # a hyperplane's tasks are independent
                self.h[m, o] = val

    def sweep_tiles(self, solver):
        """All eight octant sweeps from the library's tile jobs, diagonal by diagonal: every
        job of a diagonal first copies its rows (as the CTAs do at their start), then sweeps
        its local hyperplanes on the copies, then writes its own rows back."""
        g = solver.geometry_array
        rows, rbeg, rcnt = g("tile_rows"), g("tile_row_begin"), g("tile_row_count")
        tasks, tbeg = g("tile_tasks").reshape(-1, 4), g("tile_task_begin")
        steps, dbeg = g("tile_steps"), g("tile_diag_begin")
        stride = len(steps) // (len(rbeg) - 1)
        nst = int(solver.schedule()["TX"] + solver.schedule()["TY"] + solver.schedule()["TZ"] - 2)
        c15, c10 = 1.5 / self.ds, 1.0 / self.ds
        P = {"x2": self.cx * (2.0 / self.ds), "x1": self.cx * c10, "xh": self.cx * (-0.5 / self.ds),
             "y2": self.cy * (2.0 / self.ds), "y1": self.cy * c10, "yh": self.cy * (-0.5 / self.ds),
             "z2": self.cz * (2.0 / self.ds), "z1": self.cz * c10, "zh": self.cz * (-0.5 / self.ds)}
        dens = {}
        for cls in range(8):
            d = 0.5 * self.mu + self.cx * (c10 if cls & 1 else c15)
            d = d + self.cy * (c10 if cls & 2 else c15)
            dens[cls] = d + self.cz * (c10 if cls & 4 else c15)
        for d in range(len(dbeg) - 1):
            jobs = range(dbeg[d], dbeg[d + 1])
            smem = {}
            for j in jobs:
                S = [np.zeros(self.Nc8)]
                assert rbeg[j] % 4 == 0
                for r in rows[rbeg[j]:rbeg[j] + rcnt[j]]:
                    S.append(self._row(int(r)).copy())
                smem[j] = S
            for j in jobs:
                S = smem[j]
                o = int(rows[rbeg[j]]) & 7
                T = tasks[tbeg[j]:tbeg[j + 1]]
                st = steps[j * stride:(j + 1) * stride]
                for s_ in range(nst):
                    for t in range(st[s_], st[s_ + 1]):
                        rec = [int(v) & 0xFFFFFFFF for v in T[t]]
                        m = rec[0] & ((1 << 27) - 1)
                        fx, fy, fz = bool(rec[0] >> 27 & 1), bool(rec[0] >> 28 & 1), bool(rec[0] >> 29 & 1)
                        sl = [rec[1] & 0xFFFF, rec[1] >> 16, rec[2] & 0xFFFF, rec[2] >> 16, rec[3] & 0xFFFF, rec[3] >> 16]
                        ex = (-self.cx if SX[o] < 0 else self.cx) * self.mom[1, m]
                        ey = (-self.cy if SY[o] < 0 else self.cy) * self.mom[2, m]
                        ez = (-self.cz if SZ[o] < 0 else self.cz) * self.mom[3, m]
                        feq = self.w * (self.mom[0, m] + ((ex + ey) + ez))
                        num = self.mu * (feq - 0.5 * S[1 + t])
                        num = num + (P["x1"] if fx else P["x2"]) * S[sl[0]]
                        if not fx:
                            num = num + P["xh"] * S[sl[1]]
                        num = num + (P["y1"] if fy else P["y2"]) * S[sl[2]]
                        if not fy:
                            num = num + P["yh"] * S[sl[3]]
                        num = num + (P["z1"] if fz else P["z2"]) * S[sl[4]]
                        if not fz:
                            num = num + P["zh"] * S[sl[5]]
                        cls = (1 if fx else 0) | (2 if fy else 0) | (4 if fz else 0)
                        S[1 + t] = num / dens[cls]
            for j in jobs:
                S = smem[j]
                for q in range(tbeg[j + 1] - tbeg[j]):
                    code = int(rows[rbeg[j] + q])
                    self.h[code // 8, code % 8] = S[1 + q]

    def sweep_columns(self, solver, arena_rows=None):
        """All eight octant sweeps as the column-march kernel runs them: columns in their
        dependency order, each column's jobs in z order; a job's region holds a zero row,
        the rows carried from the previous tile of the column (a dense buffer of two z layers
        per column, written at the end of each job), its own rows (previous values), the
        static rows and the dependent rows (written by the upwind columns' jobs, which come
        earlier in the list). Checks every slot, cell and count against the bounds the kernel
        sizes its shared memory by, and, when arena_rows is given, replays the producer's
        region allocation in an arena of that many rows (the consumer releasing each job's
        region one job later than it could)."""
        g = solver.geometry_array
        rows, rbeg = g("tile_rows"), g("tile_row_begin")
        tasks, tbeg = g("tile_tasks").reshape(-1, 4), g("tile_task_begin")
        steps = g("tile_steps")
        hdr = g("tile_hdr").reshape(-1, 8)
        carry, cbeg = g("tile_carry"), g("tile_carry_begin")
        cjobs, cbegin, clist = g("tile_col_jobs"), g("tile_col_begin"), g("tile_col_list")
        info = g("tile_column_info")
        assert info[0] in (1, 2)
        ncells, max_region, max_carry, max_tasks = int(info[1]), int(info[2]), int(info[3]), int(info[4])
        njobs = len(rbeg) - 1
        stride = len(steps) // njobs
        sch = solver.schedule()
        nst = int(sch["TX"] + sch["TY"] + sch["TZ"] - 2)
        c15, c10 = 1.5 / self.ds, 1.0 / self.ds
        P = {"x2": self.cx * (2.0 / self.ds), "x1": self.cx * c10, "xh": self.cx * (-0.5 / self.ds),
             "y2": self.cy * (2.0 / self.ds), "y1": self.cy * c10, "yh": self.cy * (-0.5 / self.ds),
             "z2": self.cz * (2.0 / self.ds), "z1": self.cz * c10, "zh": self.cz * (-0.5 / self.ds)}
        dens = {}
        for cls in range(8):
            d = 0.5 * self.mu + self.cx * (c10 if cls & 1 else c15)
            d = d + self.cy * (c10 if cls & 2 else c15)
            dens[cls] = d + self.cz * (c10 if cls & 4 else c15)
        assert sorted(cjobs.tolist()) == list(range(njobs))
        done = np.zeros(njobs, dtype=bool)
        up = g("tile_up").reshape(-1, 4)
        live, tail = [], 0                       # arena replay: (base, n) of unreleased regions
        for col in clist:
            cbuf = [None] * ncells
            for q in range(cbegin[col], cbegin[col + 1]):
                j = int(cjobs[q])
                rb, tb, cb, nrows, ntask, dep0, ncin, ncout = (int(v) for v in hdr[j])
                assert rb == rbeg[j] and tb == tbeg[j] and cb == cbeg[j] and rb % 4 == 0 and cb % 4 == 0
                assert ntask == tbeg[j + 1] - tbeg[j] <= max_tasks and ncin + ncout <= max_carry
                n = 1 + ncin + nrows
                assert n <= max_region
                for u in up[j, :3]:
                    assert u < 0 or done[u], "dependent rows read before their job ran"
                if arena_rows is not None:
                    assert n <= arena_rows
                    while True:
                        if not live:
                            base = 0
                            break
                        head = live[0][0]
                        if tail > head:
                            if arena_rows - tail >= n:
                                base = tail
                                break
                            if head >= n:
                                base = 0
                                break
                        elif head - tail >= n:
                            base = tail
                            break
                        live.pop(0)
                    tail = base + n
                    for b0, n0 in live:
                        assert base + n <= b0 or b0 + n0 <= base, "regions overlap"
                    live.append((base, n))
                    if len(live) > 2:                # released one job after its successor ran
                        live.pop(0)
                S = [np.zeros(self.Nc8)]
                for e in range(ncin):
                    cell, slot = carry[cb + e] & 0xFFFF, carry[cb + e] >> 16
                    assert slot == 1 + e and 0 <= cell < ncells and cbuf[cell] is not None
                    S.append(cbuf[cell].copy())
                for r in rows[rb:rb + nrows]:
                    S.append(self._row(int(r)).copy())
                o = int(rows[rb]) & 7
                own0 = 1 + ncin
                T = tasks[tb:tb + ntask]
                st = steps[j * stride:(j + 1) * stride]
                for s_ in range(nst):
                    for t in range(st[s_], st[s_ + 1]):
                        rec = [int(v) & 0xFFFFFFFF for v in T[t]]
                        m = rec[0] & ((1 << 27) - 1)
                        fx, fy, fz = bool(rec[0] >> 27 & 1), bool(rec[0] >> 28 & 1), bool(rec[0] >> 29 & 1)
                        sl = [rec[1] & 0xFFFF, rec[1] >> 16, rec[2] & 0xFFFF, rec[2] >> 16, rec[3] & 0xFFFF, rec[3] >> 16]
                        assert all(0 <= v < n for v in sl)
                        ex = (-self.cx if SX[o] < 0 else self.cx) * self.mom[1, m]
                        ey = (-self.cy if SY[o] < 0 else self.cy) * self.mom[2, m]
                        ez = (-self.cz if SZ[o] < 0 else self.cz) * self.mom[3, m]
                        feq = self.w * (self.mom[0, m] + ((ex + ey) + ez))
                        num = self.mu * (feq - 0.5 * S[own0 + t])
                        num = num + (P["x1"] if fx else P["x2"]) * S[sl[0]]
                        if not fx:
                            num = num + P["xh"] * S[sl[1]]
                        num = num + (P["y1"] if fy else P["y2"]) * S[sl[2]]
                        if not fy:
                            num = num + P["yh"] * S[sl[3]]
                        num = num + (P["z1"] if fz else P["z2"]) * S[sl[4]]
                        if not fz:
                            num = num + P["zh"] * S[sl[5]]
                        cls = (1 if fx else 0) | (2 if fy else 0) | (4 if fz else 0)
                        S[own0 + t] = num / dens[cls]
                for t in range(ntask):
                    code = int(rows[rb + t])
                    self.h[code // 8, code % 8] = S[own0 + t]
                for e in range(ncout):
                    r, cell = carry[cb + ncin + e] & 0xFFFF, carry[cb + ncin + e] >> 16
                    assert 0 <= r < ntask and 0 <= cell < ncells
                    cbuf[cell] = S[own0 + r].copy()
                done[j] = True

    # --- the rest of one iteration -------------------------------------------------------
    def _far(self, code, o, gbuf):
        if code >= 0:
            return self.h[code, o]
        if code == -1:
            return np.zeros(self.Nc8)
        c = -code - 2
        plane = self.gE[gbuf] if c & 1 else self.gW[gbuf]
        return plane[c >> 1, o >> 1]

    def walls(self, gbuf):
        for L in range(len(self.level_start) - 1):
            for widx in range(self.level_start[L], self.level_start[L + 1]):
                q = self.wall_order[widx]
                node, lab, corner = self.wall_node[q], self.wall_label[q], self.wall_corner[q]
                e1, e2 = self.wall_e[q]
                faces, writes = self.progs[int(lab)]
                nb = self.wall_nb[q]
                zvals = {}
                tface = []
                for fi, (d, st) in enumerate(faces):
                    vals = []
                    for oo in INCOMING[d]:
                        v = e1 * self.h[nb[2 * fi], oo - 1] + e2 * self._far(nb[2 * fi + 1], oo - 1, gbuf)
                        if st == 0:
                            self.h[node, oo - 1] = v
                        elif st == 2:
                            self.fw[corner, oo - 1] = v
                        else:
                            zvals[oo - 1] = v
                        vals.append(v)
                    ca = self.cx if d < 2 else self.cy if d < 4 else self.cz
                    tface.append(ca * (((vals[0] + vals[1]) + vals[2]) + vals[3]))
                rho = []
                for t in tface:
                    r = 0.0
                    for l in range(self.Nc8):
                        r = r + t[l]
                    rho.append(r / self.DiffFlux)
                aw = self.p.accom * self.w
                one_m = 1.0 - self.p.accom
                for dst_st, dst_o, fi, src_st, src_o in writes:
                    src = self.h[node, src_o - 1] if src_st == 0 else self.fw[corner, src_o - 1] if src_st == 2 else zvals[src_o - 1]
                    v = aw * rho[fi] + one_m * src
                    if dst_st == 0:
                        self.h[node, dst_o - 1] = v
                    else:
                        self.fw[corner, dst_o - 1] = v

    def iterate(self, n=1, schedule="tasks", solver=None, arena_rows=None):
        for _ in range(n):
            it = self.iStep + 1
            cap, prev = it & 1, (it - 1) & 1
            if schedule == "tasks":
                self.sweep_tasks()
            elif schedule == "tiles":
                self.sweep_tiles(solver)
            elif schedule == "columns":
                self.sweep_columns(solver, arena_rows)
            else:
                for o in range(8):
                    self.sweep(o)
            for node, o, src in self.commit:
                self.h[node, o] = self.h[node, src] if src < 8 else self.fw[self.bcorner[node - self.NF], o]
            for r in range(self.Ny * self.Nz):
                nW, nE = self.plane_xN[r], self.plane_x1[r]
                for q, (oW, oE) in enumerate(((0, 1), (3, 2), (4, 5), (7, 6))):
                    self.gW[cap, r, q] = self.h[nW, oW] if nW >= 0 else 0.0
                    self.gE[cap, r, q] = self.h[nE, oE] if nE >= 0 else 0.0
            if self.nranks > 1:
                pos, neg = [0, 3, 4, 7], [1, 2, 5, 6]
                for sd in range(2):
                    # the west neighbour reads cx < 0 rows, the east one cx > 0 rows
                    self.hs[sd][cap] = self.h[self.hsend_nodes[sd]][:, pos if sd == 1 else neg]
                    nodes = self.hrecv_nodes[sd]
                    if len(nodes):
                        rows = self.h[nodes]
                        rows[:, pos if sd == 0 else neg] = self.hr[sd]
                        self.h[nodes] = rows
            self.walls(prev)
            wdp = self.w * self.p.pressDrop
            for r in range(self.Ny * self.Nz):
                n1, nN = self.plane_x1[r], self.plane_xN[r]
                for q, (oW, oE) in enumerate(((0, 1), (3, 2), (4, 5), (7, 6))):
                    if n1 >= 0:
                        self.h[n1, oW] = self.gW[prev, r, q] + wdp
                    if nN >= 0:
                        self.h[nN, oE] = self.gE[prev, r, q] - wdp
            for n, f in zip(self.sym_node, self.sym_flag):
                hp = self.h[n]
                if f & 1:
                    hp[1] = hp[2]; hp[0] = hp[3]; hp[5] = hp[6]; hp[4] = hp[7]
                if f & 2:
                    hp[2] = hp[1]; hp[3] = hp[0]; hp[6] = hp[5]; hp[7] = hp[4]
                if f & 4:
                    hp[0] = hp[4]; hp[1] = hp[5]; hp[2] = hp[6]; hp[3] = hp[7]
                if f & 8:
                    hp[4] = hp[0]; hp[5] = hp[1]; hp[6] = hp[2]; hp[7] = hp[3]
            for m in range(self.NF):
                f = self.h[m]
                r = ux = uy = uz = 0.0
                for l in range(self.Nc8):
                    f1, f2, f3, f4, f5, f6, f7, f8 = f[:, l]
                    r = r + f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8
                    ux = ux + self.cx[l] * (f1 - f2 - f3 + f4 + f5 - f6 - f7 + f8)
                    uy = uy + self.cy[l] * (f1 + f2 - f3 - f4 + f5 + f6 - f7 - f8)
                    uz = uz + self.cz[l] * (f1 + f2 + f3 + f4 - f5 - f6 - f7 - f8)
                self.mom[:, m] = (r, ux, uy, uz)
            self.iStep = it

    def mass_flux(self):
        part = []
        for gi in range(9):
            s = 0.0
            for e in range(self.flux_groups[gi], self.flux_groups[gi + 1]):
                n = self.flux_list[e]
                u = self.mom[1, n] if n >= 0 else 0.0
                t = u * self.ds * self.ds
                if 1 <= gi <= 4:
                    t = t * 0.5
                elif gi >= 5:
                    t = t * 0.25
                s = s + t if gi <= 4 else t
            part.append(s)
        m = part[0]
        for x in part[1:]:
            m = m + x
        inv = 1.0 / self.p.Ref_L
        return m * math.sqrt(1.0 / 2.0) / self.p.pressDrop / (inv * inv)

    def f_reference_layout(self):
        """h scattered into the reference layout f(Ntotal, Nc8, 8) (zeros elsewhere)."""
        ntot = self.GX * self.GY * (self.Nz + 4)
        f = np.zeros((8, self.Nc8, ntot))
        for n in range(self.nn):
            f[:, :, self.node_g[n]] = self.h[n]
        return f.reshape(-1)


    def halo(self, side):
        """(send, recv) arrays of the exchange before the next iteration on `side`, as
        piks_halo_buffers names them: the inlet / outlet planes at the box's edge, the slab
        halos elsewhere."""
        par = self.iStep & 1
        if (self.wglob if side == 0 else self.eglob):
            return (self.gE[par], self.gW[par]) if side == 0 else (self.gW[par], self.gE[par])
        return self.hs[side][par], self.hr[side]


def exchange(models):
    """Moves every rank's send arrays into its neighbours' receive arrays (periodic in x):
    rank r's west receive gets rank r-1's east send, its east receive rank r+1's west send."""
    n = len(models)
    if n == 1:
        return
    sends = [(m.halo(0)[0].copy(), m.halo(1)[0].copy()) for m in models]
    for r, m in enumerate(models):
        m.halo(0)[1][...] = sends[(r - 1) % n][1]
        m.halo(1)[1][...] = sends[(r + 1) % n][0]


def iterate_slabs(models, n=1):
    for _ in range(n):
        exchange(models)
        for m in models:
            m.iterate(1)
