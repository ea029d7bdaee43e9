"""Generates the golden fixtures in this directory (run in a tree where the PIKS3D
reference is mounted; the fixtures are committed so the tests never read it).

  python tests/golden/make_golden.py --reference DIR tables   # parse the reference Fortran sources
  python tests/golden/make_golden.py --reference DIR traces   # run the oracle on the shipped tutorial case

DIR is the root of a PIKS3D source tree (src/, tutorials/); it can also be given in the
environment as PIKS3D_REFERENCE.

tables -> reference_tables.json:
  gauss_hermite : every xi*/wi*/hxi*/hwi* array of src/gaussHermite.F90 as decimal text
  wall_program  : the 26 `case` blocks of src/solver.F90 (iterate, wall boundary condition)
                  as ordered operation lists (extrapolations, density sums, writes)
  switch        : the in-sweep switch rules of the 8 octant sweeps of src/solver.F90
  tutorial_sha256 : sha256 of tutorials/cubicSpherePacking/singleSphere100^3.raw
traces -> oracle_traces.json: mass / permeability / error at every chkConverge of the
  tutorial case (its para.in, its image) and of the 32^3 centred-sphere case, computed
  by the oracle; they pin the oracle and the GPU path against later changes.
"""
import hashlib
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.environ.get("PIKS3D_REFERENCE")
ROOT = os.path.dirname(os.path.dirname(HERE))


def _joined_statements(path):
    out, buf = [], ""
    for ln in open(path).read().split("\n"):
        s = ln.split("!")[0].rstrip() if not ln.strip().startswith("!$") else ""
        if not s.strip():
            continue
        st = s.strip()
        if st.startswith("&"):
            st = st[1:].strip()
        buf = (buf + " " + st) if buf else st
        if buf.endswith("&"):
            buf = buf[:-1].rstrip()
            continue
        out.append(buf)
        buf = ""
    return out


def _ref(tok):
    tok = tok.replace(" ", "")
    m = re.fullmatch(r"f\(k([+-]?[0-9]*\*?N?x?y?total|[+-][12])?,l,(\d)\)", tok)
    if m:
        return ("F", int(m.group(2)), m.group(1) or "")
    m = re.fullmatch(r"fwZ\(l,(\d)\)", tok)
    if m:
        return ("Z", int(m.group(1)), "")
    m = re.fullmatch(r"fw\(j,l,(\d)\)", tok)
    if m:
        return ("W", int(m.group(1)), "")
    raise ValueError(tok)


def parse_wall_program(solver_path):
    cases, cur = {}, None
    for s in _joined_statements(solver_path):
        t = s.replace(" ", "")
        m = re.match(r"case\((wall\w+)\)", t, re.I)
        if m:
            cur = m.group(1)
            cases[cur] = []
            continue
        if t.lower().startswith("endselect"):
            cur = None
            continue
        if cur is None or t.startswith("do") or t.startswith("enddo"):
            continue
        m = re.fullmatch(r"(.+?)=extCoef\(i,1\)\*(.+?)\+extCoef\(i,2\)\*(.+)", t)
        if m:
            d, a, b = _ref(m.group(1)), _ref(m.group(2)), _ref(m.group(3))
            cases[cur].append(["EXT", d[0] + str(d[1]), a[1], a[2], b[2]])
            continue
        m = re.fullmatch(r"(RhoWall\d?)=\1\+c([xyz])\(l\)\*\((.+)\)", t)
        if m:
            terms = [_ref(x) for x in m.group(3).split("+")]
            cases[cur].append(["RHO", m.group(1), m.group(2), [x[0] + str(x[1]) for x in terms]])
            continue
        m = re.fullmatch(r"(RhoWall\d?)=\1/DiffFlux", t)
        if m:
            cases[cur].append(["DIV", m.group(1)])
            continue
        m = re.fullmatch(r"(.+?)=accom\*w\(l\)\*(RhoWall\d?)\+\(1\.d0-accom\)\*(.+)", t)
        if m:
            d, s2 = _ref(m.group(1)), _ref(m.group(3))
            cases[cur].append(["WR", d[0] + str(d[1]), m.group(2), s2[0] + str(s2[1])])
            continue
        raise ValueError((cur, t))
    return cases


def parse_switch(solver_path):
    lines = open(solver_path).read().split("\n")
    start = next(i for i, l in enumerate(lines) if "In the 1st group of direction" in l)
    end = next(i for i, l in enumerate(lines) if "MPI_WAITALL(4, MPI_REQ_X" in l)
    txt = "\n".join(l.split("!")[0] for l in lines[start:end])
    txt = re.sub(r"&\s*\n\s*", " ", txt).replace(" ", "")
    out, conds = {}, []
    for ln in txt.split("\n"):
        m = re.match(r"(?:else)?if\((.*)\)then$", ln)
        if m:
            conds = re.findall(r"image\(ii,jj([+-]\d)?,kk\)==(wall\w+)|image\(ii,jj,kk([+-]\d)\)==(wall\w+)", m.group(1))
            continue
        m = re.match(r"f\(k([+-]N\w+),l,(\d)\)=(.*)$", ln)
        if m and conds:
            ms = re.match(r"f\(k[+-]N\w+,l,(\d)\)", m.group(3))
            src = int(ms.group(1)) if ms else "fw"
            o = int(m.group(2))
            for c in conds:
                if c[1]:
                    out.setdefault(str(o), []).append(["y", c[0], c[1], src])
                else:
                    out.setdefault(str(o), []).append(["z", c[2], c[3], src])
            conds = []
    return out


def parse_gauss_hermite(path):
    src = open(path).read()
    arrs = {}
    for m in re.finditer(r"dimension\((\d+)\)\s*::\s*(\w+)\s*=\s*\(/&(.*?)/\)", src, re.S):
        vals = re.findall(r"([0-9.]+d[+-]\d+)", m.group(3))
        assert len(vals) == int(m.group(1))
        arrs[m.group(2)] = [v.replace("d", "e") for v in vals]
    return arrs


def tables():
    solver = os.path.join(REF, "src", "solver.F90")
    data = {
        "source": "PIKS3D src/gaussHermite.F90, src/solver.F90, tutorials/cubicSpherePacking",
        "gauss_hermite": parse_gauss_hermite(os.path.join(REF, "src", "gaussHermite.F90")),
        "wall_program": parse_wall_program(solver),
        "switch": parse_switch(solver),
        "tutorial_sha256": hashlib.sha256(open(os.path.join(
            REF, "tutorials", "cubicSpherePacking", "singleSphere100^3.raw"), "rb").read()).hexdigest(),
    }
    with open(os.path.join(HERE, "reference_tables.json"), "w") as fh:
        json.dump(data, fh, indent=1, sort_keys=True)
    print("wrote reference_tables.json: %d wall labels, %d octants" % (len(data["wall_program"]), len(data["switch"])))


def traces():
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import piks3d_b200 as pk
    from piks3d_b200 import images
    from oracle import Oracle

    out = {}
    para = os.path.join(REF, "tutorials", "cubicSpherePacking", "para.in")
    p, image_name = pk.read_params(para)
    raw = open(os.path.join(os.path.dirname(para), image_name), "rb").read()
    out["tutorial_cubicSpherePacking"] = _trace(Oracle(p, raw, nthreads=os.cpu_count()), p,
                                                "tutorials/cubicSpherePacking/para.in (mpi dims ignored: one rank)")
    p = pk.default_params(Nx=32, Ny=32, Nz=32, Nc_fundamental=2, Kn=1.0, pressDrop=1.0, eps=1e-8, maxStep=2000)
    out["sphere32_r12_nv64_kn1"] = _trace(Oracle(p, images.centred_sphere(32, 12.0).tobytes(), nthreads=os.cpu_count()),
                                          p, "32^3 box, centred sphere r=12, Nc_fundamental=2, Kn=1, eps=1e-8")
    with open(os.path.join(HERE, "oracle_traces.json"), "w") as fh:
        json.dump(out, fh, indent=1)
    print("wrote oracle_traces.json")


def _trace(o, p, what):
    rows = []
    step = 0
    err = 1.0
    while step < p.maxStep:
        o.iterate(p.chkConvergeStep)
        step += p.chkConvergeStep
        mass, perm, err = o.chk_converge()
        rows.append([step, repr(mass), repr(perm), repr(err)])
        if err <= p.eps:
            break
    return {"what": what, "params": {k: getattr(p, k) for k, _ in p._fields_}, "checks": rows}


if __name__ == "__main__":
    argv = sys.argv[1:]
    if "--reference" in argv:
        i = argv.index("--reference")
        REF = argv[i + 1]
        del argv[i:i + 2]
    if not REF or not os.path.isdir(REF):
        sys.exit("make_golden.py: give the PIKS3D source tree with --reference DIR or PIKS3D_REFERENCE")
    which = argv or ["tables"]
    if "tables" in which:
        tables()
    if "traces" in which:
        traces()
