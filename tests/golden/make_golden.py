"""Extract the reference's own golden vectors and in-code test meshes into tests/golden/reference_golden.json.

Run once in a checkout that has the DGKernel sources: pass the project root as the first argument or in
DGK_REFERENCE_ROOT (`python tests/golden/make_golden.py <DGKernel root>`); the JSON it writes is committed, so the tests never read the reference at run time.  It reads the reference's
Go test files as text:

  * element/library/gonudg/jacobi_quadrature_test.go  TestJacobiGL table (alpha, beta, N, expected nodes)
  * element/library/gonudg/jacobip_test.go            P_0^(a,0) values and the P_{0,0,0} product
  * utils/mesh_test_helpers.go                        createCubeNodes / createCubeMesh / createTwoTetMesh
  * mesh/cube-partitioned.neu                         the 565-tet partitioned cube (-> cube_partitioned.json:
                                                      nodes, elements, groups and boundary sets as lists)
"""
from __future__ import annotations

import json
import math
import os
import re
import sys

ROOT = ""
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.json")
MESH_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cube_partitioned.json")


def _go_expr(expr: str) -> float:
    expr = expr.replace("math.Sqrt", "math.sqrt").replace("math.Pi", "math.pi")
    return float(eval(expr, {"math": math, "__builtins__": {}}))


def jacobi_gl_table(text: str):
    body = text[text.index("func TestJacobiGL("):text.index("func TestJacobiGQ(")]
    cases = []
    for m in re.finditer(r"\{\s*name:\s*\"([^\"]+)\",(.*?)\n\t\t\},", body, re.S):
        blk = m.group(2)
        alpha = float(re.search(r"alpha:\s*([-\d.]+)", blk).group(1))
        beta = float(re.search(r"beta:\s*([-\d.]+)", blk).group(1))
        n = int(re.search(r"\bN:\s*(\d+)", blk).group(1))
        exp = re.search(r"expected:\s*\[\]float64\{(.*?)\}", blk, re.S).group(1)
        vals = [float(v) for v in re.findall(r"[-+]?\d*\.?\d+(?:e[-+]?\d+)?", exp)]
        tol = float(re.search(r"tol:\s*([-\d.e]+)", blk).group(1))
        cases.append({"name": m.group(1), "alpha": alpha, "beta": beta, "N": n, "expected": vals, "tol": tol})
    return cases


def jacobi_p_values(text: str):
    vals = []
    for m in re.finditer(r"(\w+)\s*:=\s*JacobiP\(x,\s*([-\d.]+),\s*([-\d.]+),\s*(\d+)\)\s*\n\s*(\w+)\s*:=\s*([^\n]+)",
                         text):
        vals.append({"alpha": float(m.group(2)), "beta": float(m.group(3)), "N": int(m.group(4)),
                     "x": [-1.0, 0.0, 1.0], "value": _go_expr(m.group(6).split("//")[0].strip()), "tol": 1e-14})
    return vals


def meshes(text: str):
    nodes_blk = re.search(r"func createCubeNodes\(\) NodeSet \{(.*?)\n\}", text, re.S).group(1)
    coords = [[float(v) for v in row.split(",")] for row in re.findall(r"\{([-\d., ]+)\},\s*//", nodes_blk)]
    names = dict((k, int(v)) for k, v in re.findall(r"\"(\w+)\":\s*(\d+)", nodes_blk))
    cube_blk = re.search(r"func createCubeMesh\(\) CompleteMesh \{(.*?)\n\}", text, re.S).group(1)
    cube = [[names[n] for n in re.findall(r"\"(\w+)\"", row)] for row in re.findall(r"\{(\"[^}]*)\}", cube_blk)]
    two_blk = re.search(r"func createTwoTetMesh\(\) CompleteMesh \{(.*?)\n\}", text, re.S).group(1)
    node_part = two_blk[two_blk.index("Nodes: [][]float64{"):two_blk.index("NodeMap")]
    two_nodes = [[float(v) for v in row.split(",")] for row in re.findall(r"\{([-\d., ]+)\},", node_part)]
    two_names = dict((k, int(v)) for k, v in re.findall(r"\"(v\d)\":\s*(\d+)", two_blk))
    two = [[two_names[n] for n in re.findall(r"\"(v\d)\"", row)]
           for row in re.findall(r"\{(\"v\d\",[^}]*)\}", two_blk)]
    return {"cube_nodes": coords[:8], "cube_tets": [t for t in cube if len(t) == 4],
            "two_tet_nodes": two_nodes, "two_tet_tets": two}


def gambit_fixture(text: str):
    """The partitioned cube mesh as plain lists: nodes [id, x, y, z] and elements [id, n1..n4] in file order,
    element groups [tag, name, element ids], boundary sets [name, [[element id, face], ...]] (1-based ids)."""
    lines = text.split("\n")
    i = next(k for k, l in enumerate(lines) if "NUMNP" in l) + 1
    numnp, nelem, ngrps, nbsets = (int(x) for x in lines[i].split()[:4])
    nodes, elements, groups, bcs = [], [], [], []
    while i < len(lines):
        t = lines[i].strip()
        i += 1
        if "NODAL COORDINATES" in t:
            for _ in range(numnp):
                f = lines[i].split()
                i += 1
                nodes.append([int(f[0]), float(f[1]), float(f[2]), float(f[3])])
        elif "ELEMENTS/CELLS" in t:
            for _ in range(nelem):
                f = lines[i].split()
                i += 1
                elements.append([int(f[0])] + [int(x) for x in f[3:7]])
        elif "ELEMENT GROUP" in t:
            f = lines[i].split()
            tag, count = int(f[f.index("GROUP:") + 1]), int(f[f.index("ELEMENTS:") + 1])
            name = lines[i + 1].strip()
            i += 3
            els = []
            while len(els) < count:
                els += [int(x) for x in lines[i].split()]
                i += 1
            groups.append([tag, name, els])
        elif "BOUNDARY CONDITIONS" in t:
            for _ in range(nbsets):
                f = lines[i].split()
                i += 1
                ents = []
                for _ in range(int(f[2])):
                    e = lines[i].split()
                    i += 1
                    ents.append([int(e[0]), int(e[2])])
                bcs.append([f[0], ents])
    assert len(groups) == ngrps
    return {"source": "mesh/cube-partitioned.neu of DGKernel, extracted by tests/golden/make_golden.py",
            "nodes": nodes, "elements": elements, "groups": groups, "bcs": bcs}


def main():
    global ROOT
    ROOT = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("DGK_REFERENCE_ROOT", "")
    if not ROOT or not os.path.isdir(ROOT):
        sys.stderr.write("usage: make_golden.py <DGKernel root>  (or set DGK_REFERENCE_ROOT)\n")
        return 2
    g = os.path.join(ROOT, "element", "library", "gonudg")
    with open(os.path.join(g, "jacobi_quadrature_test.go")) as f:
        quad = f.read()
    with open(os.path.join(g, "jacobip_test.go")) as f:
        jp = f.read()
    with open(os.path.join(ROOT, "utils", "mesh_test_helpers.go")) as f:
        helpers = f.read()
    out = {
        "source": "DGKernel test files read as text by tests/golden/make_golden.py",
        "jacobi_gl": jacobi_gl_table(quad),
        "jacobi_p": jacobi_p_values(jp),
        "simplex3dp_000": math.sqrt(3.0) / 2.0,
        "meshes": meshes(helpers),
    }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1)
    with open(os.path.join(ROOT, "mesh", "cube-partitioned.neu")) as f:
        fx = gambit_fixture(f.read())
    with open(MESH_OUT, "w") as f:
        json.dump(fx, f, separators=(",", ":"))
    print(f"wrote {MESH_OUT}: {len(fx['nodes'])} nodes, {len(fx['elements'])} tets, {len(fx['groups'])} groups")
    print(f"wrote {OUT}: {len(out['jacobi_gl'])} JacobiGL cases, {len(out['jacobi_p'])} JacobiP values")


if __name__ == "__main__":
    sys.exit(main())
