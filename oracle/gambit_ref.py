"""Restatement of ReadGambitNeutral for tetrahedral meshes (test infrastructure only).

Follows mesh/readers/gambit_reader.go:13-338: the control header gives NUMNP NELEM NGRPS NBSETS; vertices keep
file order (node id -> position); elements keep file order with node ids mapped through that table; a group
named "p<N>" puts its elements in partition N, EToP existing only when NGRPS > 1 (-1 for unassigned elements);
boundary-condition entries of ITYPE 1 give (element, face - 1, set).  Used by the tests to check the library's
reader (dgk_read_gambit) and to build the oracle side of the partitioned-mesh parity tests.
"""
from __future__ import annotations

import numpy as np


def read(path_or_text: str, is_text: bool = False):
    text = path_or_text if is_text else open(path_or_text).read()
    lines = text.split("\n")
    i = 0
    numnp = nelem = ngrps = nbsets = 0
    while i < len(lines):
        t = lines[i].strip()
        i += 1
        if "NUMNP" in t and "NELEM" in t:
            v = lines[i].split()
            i += 1
            numnp, nelem, ngrps, nbsets = (int(x) for x in v[:4])
            break
    VX, VY, VZ = np.zeros(numnp), np.zeros(numnp), np.zeros(numnp)
    EToV = np.zeros((nelem, 4), dtype=np.int64)
    EToP = None
    node_ix, elem_ix = {}, {}
    groups, bfaces = [], []
    while i < len(lines):
        t = lines[i].strip()
        i += 1
        if t == "ENDOFSECTION":
            continue
        if "NODAL COORDINATES" in t:
            for k in range(numnp):
                f = lines[i].split()
                i += 1
                node_ix[int(f[0])] = k
                VX[k], VY[k], VZ[k] = float(f[1]), float(f[2]), float(f[3])
        elif "ELEMENTS/CELLS" in t:
            for k in range(nelem):
                f = lines[i].split()
                i += 1
                if int(f[1]) != 6 or int(f[2]) != 4:
                    raise ValueError("only 4-node tetrahedra")
                EToV[k] = [node_ix[int(x)] for x in f[3:7]]
                elem_ix[int(f[0])] = k
        elif "ELEMENT GROUP" in t:
            if ngrps > 1 and EToP is None:
                EToP = np.full(nelem, -1, dtype=np.int64)
            f = lines[i].split()
            i += 1
            gid = int(f[f.index("GROUP:") + 1])
            count = int(f[f.index("ELEMENTS:") + 1])
            name = lines[i].strip()
            i += 2  # name, flags
            part = int(name[1:]) if len(name) > 1 and name[0] == "p" and name[1:].lstrip("-").isdigit() else -1
            els, got = [], 0
            while got < count and i < len(lines):
                ln = lines[i].strip()
                i += 1
                if ln == "ENDOFSECTION":
                    break
                for w in ln.split():
                    if not w.lstrip("-").isdigit() or int(w) <= 0:
                        continue
                    e = elem_ix.get(int(w))
                    if e is not None:
                        els.append(e)
                        if part >= 0 and EToP is not None:
                            EToP[e] = part
                    got += 1
                    if got >= count:
                        break
            groups.append((gid, name, els))
        elif "BOUNDARY CONDITIONS" in t:
            for b in range(nbsets):
                f = lines[i].split()
                i += 1
                itype, nentry = int(f[1]), int(f[2])
                for _ in range(nentry):
                    e = lines[i].split()
                    i += 1
                    if itype == 1 and int(e[0]) in elem_ix:
                        bfaces.append((elem_ix[int(e[0])], int(e[2]) - 1, b))
    return {"VX": VX, "VY": VY, "VZ": VZ, "EToV": EToV, "EToP": EToP, "groups": groups,
            "bfaces": np.array(bfaces, dtype=np.int64).reshape(-1, 3)}


def write(path, nodes, elements, groups, bcs, title="mesh"):
    """Gambit neutral text from nodes [(id, x, y, z)], elements [(id, n1..n4)], groups [(tag, name, [elem ids])]
    and bcs [(name, [(elem id, face)])] (1-based ids, tetrahedra), in the layout the reader expects."""
    out = ["        CONTROL INFO 2.0.0", "** GAMBIT NEUTRAL FILE", title, "PROGRAM:  dgkernel_b200 tests",
           "", "     NUMNP     NELEM     NGRPS    NBSETS     NDFCD     NDFVL",
           f"{len(nodes):10d}{len(elements):10d}{len(groups):10d}{len(bcs):10d}         3         3", "ENDOFSECTION",
           "   NODAL COORDINATES 2.0.0"]
    out += [f"{nid:10d}{x:20.11e}{y:20.11e}{z:20.11e}" for nid, x, y, z in nodes]
    out += ["ENDOFSECTION", "      ELEMENTS/CELLS 2.0.0"]
    out += [f"{eid:8d} {6:2d} {4:2d} " + "".join(f"{v:8d}" for v in vs) for eid, *vs in elements]
    out += ["ENDOFSECTION"]
    for tag, name, els in groups:
        out += ["       ELEMENT GROUP 2.0.0",
                f"GROUP: {tag:10d} ELEMENTS: {len(els):10d} MATERIAL: {0:10d} NFLAGS: {1:10d}",
                f"{name:>32s}", "       0"]
        out += ["".join(f"{e:8d}" for e in els[k:k + 10]) for k in range(0, len(els), 10)]
        out += ["ENDOFSECTION"]
    if bcs:
        out += ["       BOUNDARY CONDITIONS 2.0.0"]
        for name, ents in bcs:
            out += [f"{name:>32s}{1:8d}{len(ents):8d}{0:8d}{51:8d}"]
            out += [f"{e:10d}{6:5d}{f:5d}" for e, f in ents]
        out += ["ENDOFSECTION"]
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")
