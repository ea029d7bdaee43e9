"""Pins the oracle and the product to the reference's own sources and fixture.

reference_tables.json holds data parsed from PIKS3D's Fortran (tests/golden/make_golden.py):
the Gauss-Hermite tables, the 26 wall re-emission programs, the in-sweep switch rules and
the sha256 of the shipped tutorial image. The oracle's and the library's transcriptions
must reproduce them exactly; oracle_traces.json pins the oracle's chkConverge trajectory
on the shipped tutorial case and on the 32^3 sphere.
"""
import hashlib
import json
import math
import os
import re

import numpy as np
import pytest

import piks3d_b200 as pk
from piks3d_b200 import images
from conftest import ROOT, base_params
from oracle import Oracle

GOLD = os.path.join(ROOT, "tests", "golden")
TABLES = json.load(open(os.path.join(GOLD, "reference_tables.json")))
LABELS = dict(wallE=20, wallW=21, wallN=22, wallS=23, wallF=24, wallB=25, wallEN=30, wallWN=31, wallES=32,
              wallWS=33, wallNF=40, wallNB=41, wallSF=42, wallSB=43, wallEF=50, wallEB=51, wallWF=52, wallWB=53,
              wallENF=60, wallWNF=61, wallWSF=62, wallESF=63, wallENB=70, wallWNB=71, wallWSB=72, wallESB=73)
INCOMING = {"DIR_PX": (2, 3, 6, 7), "DIR_MX": (1, 4, 5, 8), "DIR_PY": (3, 4, 7, 8), "DIR_MY": (1, 2, 5, 6),
            "DIR_PZ": (5, 6, 7, 8), "DIR_MZ": (1, 2, 3, 4)}
OFFSET = {"DIR_PX": ("+1", "+2"), "DIR_MX": ("-1", "-2"), "DIR_PY": ("+Nxtotal", "+2*Nxtotal"),
          "DIR_MY": ("-Nxtotal", "-2*Nxtotal"), "DIR_PZ": ("+Nxytotal", "+2*Nxytotal"),
          "DIR_MZ": ("-Nxytotal", "-2*Nxytotal")}
AXIS = {"DIR_PX": "x", "DIR_MX": "x", "DIR_PY": "y", "DIR_MY": "y", "DIR_PZ": "z", "DIR_MZ": "z"}
STORE = {"ST_F": "F", "ST_Z": "Z", "ST_W": "W"}


def _ops_from_table(path):
    """wall_table.inc rows -> the reference's statement sequence for each label."""
    out = {}
    for line in open(path):
        m = re.match(r"\s*/\*\s*(\w+)\s*\*/\s*\{(\d+), (\d+), \{(.*?)\}\}, (\d+), \{(.*)\}\},", line)
        if not m:
            continue
        name = m.group(1)
        assert LABELS[name] == int(m.group(2))
        faces = re.findall(r"(DIR_\w+), (ST_\w)", m.group(4))
        writes = re.findall(r"\{(ST_\w), (\d+), (\d+), (ST_\w), (\d+)\}", m.group(6))
        ops = []
        for d, st in faces:
            for o in INCOMING[d]:
                ops.append(["EXT", STORE[st] + str(o), o, OFFSET[d][0], OFFSET[d][1]])
        rho = ["RhoWall", "RhoWall2", "RhoWall3"]
        for fi, (d, st) in enumerate(faces):
            ops.append(["RHO", rho[fi], AXIS[d], [STORE[st] + str(o) for o in INCOMING[d]]])
        for fi in range(len(faces)):
            ops.append(["DIV", rho[fi]])
        for ds, do, fi, ss, so in writes:
            ops.append(["WR", STORE[ds] + do, rho[int(fi)], STORE[ss] + so])
        out[name] = ops
    return out


@pytest.mark.parametrize("path", ["oracle/wall_table.inc", "piks3d_b200/csrc/wall_table.inc"])
def test_wall_programs_match_reference(path):
    ours = _ops_from_table(os.path.join(ROOT, path))
    ref = TABLES["wall_program"]
    assert set(ours) == set(ref)
    for name in ref:
        assert ours[name] == ref[name], name


def _switch_rows_product():
    rows = []
    for line in open(os.path.join(ROOT, "piks3d_b200", "csrc", "switch_table.inc")):
        m = re.match(r"\s*\{(\d), (\d), (\d+), (\d)\},", line)
        if m:
            rows.append(tuple(int(x) for x in m.groups()))
    return rows


def _switch_rows_oracle():
    src = open(os.path.join(ROOT, "oracle", "piks_oracle.cpp")).read()
    block = src[src.index("const OctSwitch kSwitch[8] = {"):]
    block = block[:block.index("};")]
    rows = []
    for o, line in enumerate(re.findall(r"\{3, \{(.*?)\}, 5, \{(.*?)\}\}", block)):
        for axis, part in enumerate(line):
            for lab, src_ in re.findall(r"(wall\w+), (\d)", part):
                s = int(src_)
                rows.append((o, axis, LABELS[lab], 8 if s == 0 else s - 1))
    return rows


def test_switch_rules_match_reference():
    ref = []
    for o in range(1, 9):
        for axis, off, name, src in TABLES["switch"][str(o)]:
            ref.append((o - 1, 0 if axis == "y" else 1, LABELS[name], 8 if src == "fw" else int(src) - 1))
    assert _switch_rows_product() == ref
    assert _switch_rows_oracle() == ref


def test_gauss_hermite_velocity_sets_match_reference():
    gh = TABLES["gauss_hermite"]
    for half, (xn, wn) in ((1, ("hxi", "hwi")), (0, ("xi", "wi"))):
        for n in (2, 4, 6, 8, 12, 16):
            xi = [float(v) * math.sqrt(2.0) for v in gh[xn + str(n)]]
            w1 = [float(v) for v in gh[wn + str(n)]]
            cx = np.array([xi[c] for a in range(n) for b in range(n) for c in range(n)])
            cy = np.array([xi[b] for a in range(n) for b in range(n) for c in range(n)])
            cz = np.array([xi[a] for a in range(n) for b in range(n) for c in range(n)])
            w = np.array([w1[c] * w1[b] * w1[a] for a in range(n) for b in range(n) for c in range(n)])
            p = base_params(6, Nc_fundamental=n, halfRange=half)
            o = Oracle(p, np.zeros(216, np.uint8).tobytes(), nthreads=1)
            s = pk.Solver(p, device=-1)
            for ref_arr, name, oa in zip((cx, cy, cz, w), ("cx", "cy", "cz", "w"), o.velocity()):
                assert np.array_equal(ref_arr, oa), (n, half, name)
                assert np.array_equal(ref_arr, s.geometry_array(name)), (n, half, name)


def test_tutorial_image_generator_matches_shipped_file():
    img = images.quarter_sphere(100, 0.75)
    assert hashlib.sha256(img.tobytes()).hexdigest() == TABLES["tutorial_sha256"]


TRACES = os.path.join(GOLD, "oracle_traces.json")


@pytest.mark.skipif(not os.path.exists(TRACES), reason="oracle_traces.json not generated")
def test_oracle_sphere32_trace():
    tr = json.load(open(TRACES))["sphere32_r12_nv64_kn1"]
    p = base_params(32, Nc_fundamental=2, Kn=1.0, eps=1e-8, maxStep=2000)
    o = Oracle(p, images.centred_sphere(32, 12.0).tobytes(), nthreads=os.cpu_count())
    for step, mass, perm, err in tr["checks"][:4]:
        o.iterate(p.chkConvergeStep)
        m, k, e = o.chk_converge()
        assert (repr(m), repr(k), repr(e)) == (mass, perm, err), step
