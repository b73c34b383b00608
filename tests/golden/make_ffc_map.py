"""Tabulate the reference's full-face-copy cell mapping
(GhostCellFullFaceCopy.set_up_cell_mapping, src/eilmer/bc/ghost_cell_effect/
full_face_copy.d): for every pair of faces (and, in 3-D, every orientation)
the partner cell that fills each of the two ghost layers behind face cells
(p, q), evaluated from the reference's own index expressions for a partner
of 5 x 7 x 3 cells, written as ffc_map.json next to this script.  Run where
the reference tree is available:

    python tests/golden/make_ffc_map.py <reference-root>

The source is read, not run: each case's assignments to i_src, j_src, k_src
and the index triples handed to ijk_0n_indices_to_cell_id are evaluated with
this block's face-cell indices bound to (p, q).
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
FACES = ["north", "east", "south", "west", "top", "bottom"]
# this block's loop variables on each face: (p, q)
LOOP = {"north": "ik", "south": "ik", "east": "jk", "west": "jk", "top": "ij", "bottom": "ij"}
EXT = {"ni": 5, "nj": 7, "nk": 3}


def evaluate(expr, env):
    e = (expr.replace("other_blk.nicell", str(EXT["ni"])).replace("other_blk.njcell", str(EXT["nj"]))
         .replace("other_blk.nkcell", str(EXT["nk"])))
    return eval(e, {"__builtins__": {}}, env)


def collect(lines, dim):
    """(this, other, orientation) -> (statements before the orientation
    switch, the orientation's statements, the cell-id argument triples)."""
    cases = {}
    this = other = None
    pre, ids = [], []
    per_r = {}

    def flush():
        if this and other:
            if dim == 3:
                for r, st in per_r.items():
                    cases[(this, other, r)] = (list(pre), st, list(ids))
            else:
                cases[(this, other, 0)] = (list(pre), [], list(ids))

    for line in lines:
        s = line.strip()
        m = re.match(r"case Face\.(\w+):", s)
        if m:
            name = m.group(1)
            indent = len(line) - len(line.lstrip())
            flush()
            pre, ids, per_r = [], [], {}
            if indent <= 12:
                this, other = name, None
            else:
                other = name
            continue
        if other is None:
            continue
        m = re.match(r"case (\d): (.*)", s)
        if m:
            per_r[int(m.group(1))] = re.findall(r"(\w)_src = ([^;]+);", m.group(2))
            continue
        if per_r and not re.search(r"_src|cell_id", s) and s and not s.startswith("}"):
            # the continuation of a 'case 3:' line
            pass
        if per_r and re.match(r"\w_src = ", s) and "cell_id" not in s:
            last = max(per_r)
            per_r[last] += re.findall(r"(\w)_src = ([^;]+);", s)
            continue
        m = re.findall(r"(\w)_src = ([^;]+);", s)
        if m and "cell_id" not in s:
            pre += m
            continue
        m = re.search(r"ijk_0n_indices_to_cell_id\(([^)]*)\)", s)
        if m and "nghost3" not in s:
            ids.append([a.strip() for a in m.group(1).split(",")])
    flush()
    return cases


def main(ref):
    path = os.path.join(ref, "src", "eilmer", "bc", "ghost_cell_effect", "full_face_copy.d")
    with open(path) as f:
        text = f.read().split("\n")
    start = next(n for n, l in enumerate(text) if "void set_up_cell_mapping_phase0()" in l)
    split = next(n for n in range(start, len(text)) if "Continue on with 3D work" in text[n])
    end = next(n for n in range(split, len(text)) if "end set_up_cell_mapping_phase0" in text[n]
               or re.match(r"\s*void set_up_cell_mapping_phase1", text[n]))
    rows = []
    for dim, lines in ((2, text[start:split]), (3, text[split:end])):
        cases = collect(lines, dim)
        for (this, other, r), (pre, st, ids) in sorted(cases.items()):
            if len(ids) != 2:
                raise ValueError(f"{dim}-D {this}/{other}/{r}: {len(ids)} cell ids")
            lp = LOOP[this]
            for p in range(3):
                for q in range(3 if dim == 3 else 1):
                    env = {lp[0]: p, lp[1]: q}
                    for a, e in pre + st:
                        env[a + "_src"] = evaluate(e, env)
                    env.setdefault("k_src", 0)
                    for g, triple in enumerate(ids):
                        cell = [evaluate(x, env) for x in triple]
                        if len(cell) == 2:
                            cell.append(0)
                        rows.append([dim, FACES.index(this), FACES.index(other), r, p, q, g] + cell)
    out = {"source": "src/eilmer/bc/ghost_cell_effect/full_face_copy.d (set_up_cell_mapping_phase0)",
           "partner_extents": [EXT["ni"], EXT["nj"], EXT["nk"]],
           "columns": ["dim", "face", "other_face", "orientation", "p", "q", "ghost_layer",
                       "i_src", "j_src", "k_src"],
           "rows": rows}
    with open(os.path.join(HERE, "ffc_map.json"), "w") as f:
        json.dump(out, f, separators=(",", ":"))
    print(len(rows), "rows")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.environ.get("E4_REFERENCE_ROOT", "/root/reference"))
