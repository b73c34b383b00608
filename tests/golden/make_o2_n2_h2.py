"""Extract the O2-N2-H2 thermally perfect mixture of the reference's
mixture-EOS unit test (src/gas/sample-data/O2-N2-H2.lua, used by
src/gas/thermo/therm_perf_gas_mix_eos.d:179-200): molar masses and the
9-coefficient CEA thermo curves, written as o2_n2_h2_thermo.json next to this
script.  Run where the reference tree is available:

    python tests/golden/make_o2_n2_h2.py <reference-root>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def table_body(text, start):
    depth = 0
    for i in range(start, len(text)):
        if text[i] == "{":
            depth += 1
        elif text[i] == "}":
            depth -= 1
            if depth == 0:
                return text[start + 1:i]
    raise ValueError("unbalanced braces")


def numbers(s):
    return [float(x) for x in re.findall(r"[-+]?\d+\.?\d*(?:[eE][-+]?\d+)?", s)]


def main(ref):
    path = os.path.join(ref, "src", "gas", "sample-data", "O2-N2-H2.lua")
    with open(path) as f:
        text = f.read()
    species = re.findall(r"'(\w+)'", re.search(r"species\s*=\s*\{([^}]*)\}", text).group(1))
    out = {"source": "src/gas/sample-data/O2-N2-H2.lua", "species": []}
    for sp in species:
        M = float(re.search(r"\b%s\.M\s*=\s*([-+0-9.eE]+)" % sp, text).group(1))
        i = text.index("%s.cea_thermo" % sp)
        body = table_body(text, text.index("{", i))
        nseg = int(re.search(r"nsegments\s*=\s*(\d+)", body).group(1))
        tb = numbers(table_body(body, body.index("{", body.index("T_break_points"))))
        bl = numbers(table_body(body, body.index("{", body.index("T_blend_ranges"))))
        segs = []
        for q in range(nseg):
            j = body.index("segment%d" % q)
            segs.append(numbers(table_body(body, body.index("{", j))))
        assert len(tb) == nseg + 1 and len(bl) == nseg - 1 and all(len(c) == 9 for c in segs)
        out["species"].append({"name": sp, "M": M, "T_break": tb, "T_blend": bl, "coeffs": segs})
    with open(os.path.join(HERE, "o2_n2_h2_thermo.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_o2_n2_h2.py <reference-root>")
    main(sys.argv[1])
