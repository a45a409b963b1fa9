"""Extract the reference's CG and CR golden vectors into a small JSON fixture.

Reads FrontISTR's own end-to-end solver tests (tests/solver/CG/{SSOR,ILU0,DIAG,
ILU1,ILU2} and tests/solver/CR/{SSOR,ILU0,DIAG,ILU1,ILU2} .msh/.cnt/.res.0.1 in
the FrontISTR tree): one 99-node TET4 (type 341) cantilever, the same mesh in
every file, solved by CG (METHOD=CG) and by CR (METHOD=CR) with SSOR
(PRECOND=1), ILU(0) (10), DIAG (3), block ILU(1) (11) and block ILU(2) (12) to a
relative residual of 1e-8.  The fixture keeps the mesh in the reference's
internal node order (the order of the result file), the boundary conditions,
and the DISPLACEMENT field that fistr1 wrote for every (method, PRECOND):
"displacement" holds the CG results by PRECOND, "displacement_by_method" holds
{"CG": {PRECOND: field}, "CR": {PRECOND: field}}.

Run once in a container that has the reference tree (the path is required):
    python tests/golden/make_golden.py /path/to/FrontISTR
The output, tests/golden/tet4_cantilever_cg.json, is committed; nothing at
test time reads the reference tree.
"""
import argparse
import json
import os


def parse_msh(path):
    nodes, elems, groups = {}, [], {}
    section = None
    material = None
    lines = open(path).read().splitlines()
    i = 0
    while i < len(lines):
        line = lines[i].strip()
        i += 1
        if not line or line.startswith("!!") or line.startswith("#"):
            continue
        if line.startswith("!"):
            head = line.upper()
            if head.startswith("!NODE"):
                section = ("node", None)
            elif head.startswith("!ELEMENT"):
                etype = int(head.split("TYPE=")[1].split(",")[0])
                section = ("elem", etype)
            elif head.startswith("!NGROUP"):
                name = head.split("NGRP=")[1].split(",")[0].strip()
                section = ("ngrp", (name, "GENERATE" in head))
            elif head.startswith("!ITEM=1"):
                section = ("item1", None)
            else:
                section = ("skip", None)
            continue
        kind, arg = section
        vals = [v.strip() for v in line.split(",") if v.strip()]
        if kind == "node":
            nodes[int(vals[0])] = [float(v) for v in vals[1:4]]
        elif kind == "elem":
            elems.append((arg, [int(v) for v in vals[1:]]))
        elif kind == "ngrp":
            name, gen = arg
            ids = [int(v) for v in vals]
            if gen:
                a, b, s = ids
                ids = list(range(a, b + 1, s))
            groups.setdefault(name, []).extend(ids)
        elif kind == "item1" and material is None:
            material = [float(v) for v in vals[:2]]
    return nodes, elems, groups, material


def parse_cnt(path):
    bcs, loads, solver = [], [], None
    section = None
    for raw in open(path).read().splitlines():
        line = raw.strip()
        if not line or line.startswith("!!"):
            continue
        if line.startswith("!"):
            head = line.upper()
            section = head.split(",")[0]
            if section == "!SOLVER":
                solver = {kv.split("=")[0].strip(): kv.split("=")[1].strip()
                          for kv in head.split(",")[1:] if "=" in kv}
            continue
        vals = [v.strip() for v in line.split(",")]
        if section == "!BOUNDARY":
            bcs.append([vals[0], int(vals[1]), int(vals[2]), float(vals[3])])
        elif section == "!CLOAD":
            loads.append([vals[0], int(vals[1]), float(vals[2])])
    return bcs, loads, solver


def parse_res(path):
    tok = open(path).read().split()
    k = tok.index("*data")
    n_node, n_elem = int(tok[k + 1]), int(tok[k + 2])
    nnf = int(tok[k + 3])
    k += 5
    ncomp = [int(t) for t in tok[k:k + nnf]]
    k += nnf
    names = tok[k:k + nnf]
    k += nnf
    width = sum(ncomp)
    order, disp = [], []
    di = names.index("DISPLACEMENT")
    off = sum(ncomp[:di])
    for _ in range(n_node):
        nid = int(tok[k])
        vals = [float(t) for t in tok[k + 1:k + 1 + width]]
        k += 1 + width
        order.append(nid)
        disp.append(vals[off:off + 3])
    return order, disp, n_elem


def main(ref_root):
    base = os.path.join(ref_root, "tests", "solver", "CG")
    nodes, elems, groups, material = parse_msh(os.path.join(base, "SSOR.msh"))
    order, _, n_elem = parse_res(os.path.join(base, "SSOR.res.0.1"))
    assert n_elem == len(elems)
    index = {nid: i for i, nid in enumerate(order)}
    bcs, loads, _ = parse_cnt(os.path.join(base, "SSOR.cnt"))
    fixed = []
    for grp, d0, d1, val in bcs:
        for nid in groups[grp]:
            for d in range(d0, d1 + 1):
                fixed.append([index[nid], d, val])
    cloads = []
    for grp, d, val in loads:
        for nid in groups[grp]:
            cloads.append([index[nid], d, val])
    out = {
        "source": "FrontISTR tests/solver/CG (SSOR, ILU0, DIAG): .msh, .cnt, .res.0.1",
        "etype": 341,
        "node_ids": order,
        "coords": [nodes[nid] for nid in order],
        "elements": [[index[n] for n in conn] for (_, conn) in elems],
        "E": material[0],
        "nu": material[1],
        "fixed": fixed,
        "cload": cloads,
        "tol": 1.0e-8,
        "displacement": {},
    }
    mesh_text = open(os.path.join(base, "SSOR.msh")).read()
    out["displacement_by_method"] = {}
    out["source"] = ("FrontISTR tests/solver/CG and tests/solver/CR (SSOR, ILU0, DIAG, ILU1, ILU2): "
                     ".msh, .cnt, .res.0.1")
    for method in ("CG", "CR"):
        mdir = os.path.join(ref_root, "tests", "solver", method)
        by_pc = out["displacement_by_method"].setdefault(method, {})
        for name, precond in (("SSOR", 1), ("ILU0", 10), ("DIAG", 3), ("ILU1", 11), ("ILU2", 12)):
            assert open(os.path.join(mdir, name + ".msh")).read() == mesh_text  # one mesh throughout
            bc2, ld2, solver = parse_cnt(os.path.join(mdir, name + ".cnt"))
            assert (bc2, ld2) == (bcs, loads)
            assert solver["METHOD"] == method and int(solver["PRECOND"]) == precond
            o2, disp, _ = parse_res(os.path.join(mdir, name + ".res.0.1"))
            assert o2 == order
            by_pc[str(precond)] = disp
            if method == "CG" and precond in (1, 10, 3):
                out["displacement"][str(precond)] = disp
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tet4_cantilever_cg.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", dst, len(order), "nodes", len(elems), "elements")


if __name__ == "__main__":
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("reference_root", help="root of a FrontISTR source tree (the directory holding tests/)")
    main(ap.parse_args().reference_root)
