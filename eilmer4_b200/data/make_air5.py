"""Extract the 5-species air gas model used by the reacting workload.

Reads the thermally perfect gas-model deck that ships with the reference
(src/gas/sample-data/therm-perf-5-species-air.lua: species N2, O2, NO, N, O,
molar masses and the NASA Glenn/CEA 9-coefficient thermo curves) and the
1-T Gupta air mechanism (examples/kinetics/air-chemistry-1T/
GuptaEtAl-air-reactions.lua), keeping reactions r1, r2, r4, r5, r6, and
writes air5_gas_model.json next to this script.  Run once where the
reference is available:

    python eilmer4_b200/data/make_air5.py <reference-root>
"""
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def lua_table_body(text, start):
    """Text between the braces of the table opening at text[start] == '{'."""
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


def species_data(text, sp):
    m = re.search(r"db\.%s\.M\s*=\s*([-+0-9.eE]+)" % re.escape(sp), text)
    M = float(m.group(1))
    i = text.index("db.%s.thermoCoeffs" % sp)
    body = lua_table_body(text, text.index("{", i))
    nseg = int(re.search(r"nsegments\s*=\s*(\d+)", body).group(1))
    tb = numbers(lua_table_body(body, body.index("{", body.index("T_break_points"))))
    bl = numbers(lua_table_body(body, body.index("{", body.index("T_blend_ranges"))))
    segs = []
    for s in range(nseg):
        j = body.index("segment%d" % s)
        segs.append(numbers(lua_table_body(body, body.index("{", j))))
    return {"M": M, "nsegments": nseg, "T_break_points": tb, "T_blend_ranges": bl,
            "segments": segs}


def reactions(text, labels):
    out = []
    for m in re.finditer(r"Reaction\s*\{", text):
        body = lua_table_body(text, text.index("{", m.start()))
        lab = re.search(r"label\s*=\s*'(\w+)'", body).group(1)
        if lab not in labels:
            continue
        eq = re.search(r"'([^']*<=>[^']*)'", body).group(1)
        fr = re.search(r"fr\s*=\s*\{[^}]*A\s*=\s*([-+0-9.eE]+)\s*,\s*n\s*=\s*([-+0-9.eE]+)\s*,"
                       r"\s*C\s*=\s*([-+0-9.eE]+)", body)
        br = re.search(r"br\s*=\s*\{[^}]*A\s*=\s*([-+0-9.eE]+)\s*,\s*n\s*=\s*([-+0-9.eE]+)\s*,"
                       r"\s*C\s*=\s*([-+0-9.eE]+)", body)
        eff = {}
        em = re.search(r"efficiencies\s*=\s*\{([^}]*)\}", body)
        if em:
            for k, v in re.findall(r"(\w+)\s*=\s*([-+0-9.eE]+)", em.group(1)):
                eff[k] = float(v)
        out.append({"label": lab, "equation": eq,
                    "fr": [float(x) for x in fr.groups()], "br": [float(x) for x in br.groups()],
                    "efficiencies": eff})
    return out


def main(ref):
    gas = open(os.path.join(ref, "src/gas/sample-data/therm-perf-5-species-air.lua")).read()
    species = ["N2", "O2", "NO", "N", "O"]
    mech = open(os.path.join(ref, "examples/kinetics/air-chemistry-1T/"
                                  "GuptaEtAl-air-reactions.lua")).read()
    lim = re.search(r"tempLimits\s*=\s*\{\s*lower\s*=\s*([-+0-9.eE]+)\s*,\s*upper\s*=\s*"
                    r"([-+0-9.eE]+)", mech)
    data = {
        "source": "NASA Glenn (CEA) thermo curves and the 1-T Gupta et al. air mechanism as "
                  "carried by the Eilmer4 sample decks; reactions r1, r2, r4, r5, r6",
        "species": species,
        "thermo": {sp: species_data(gas, sp) for sp in species},
        "reactions": reactions(mech, {"r1", "r2", "r4", "r5", "r6"}),
        "temp_limits": [float(lim.group(1)), float(lim.group(2))],
    }
    with open(os.path.join(HERE, "air5_gas_model.json"), "w") as f:
        json.dump(data, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python eilmer4_b200/data/make_air5.py <reference-root>")
    main(sys.argv[1])
