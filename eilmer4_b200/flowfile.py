"""Flow files of structured blocks in the format Eilmer4 reads and writes.

``write_flow`` / ``read_flow`` restate ``SFluidBlock.write_solution`` and
``read_solution`` (src/eilmer/sfluidblock.d:1778-1956) for the variables this
path carries, so that the D host's restart and the ``e4shared --post``
post-processor can read the GPU's results, and GPU runs can start from the
reference's flow files.  Two formats, as ``flow_format``:

* ``gziptext``: a gzip stream of a header (``structured_grid_flow 1.0``,
  ``label:``, ``sim_time:``, ``variables:`` with the quoted names,
  ``dimensions:``, ``nicell:``, ``njcell:``, ``nkcell:``) and one line per
  cell, i fastest, each value ``%.18e`` after a space (the shock-detector
  flag S as ``%d``), as ``cell_data_as_string`` (fvcell.d:2374-2460) writes;
* ``rawbinary``: the same header and values as native ints and doubles
  (fvcell.d:2464-2560).

The variable list is ``GlobalConfig.build_flow_variable_list``
(globalconfig.d:791-836) without the optional MHD, quality, radiation,
multi-temperature and local-time-stepping entries, none of which this path
has: pos.x pos.y pos.z volume rho vel.x vel.y vel.z p a mu k mu_t k_t S tke
omega massf[i]-<species> [dt_chem when more than one species] u T.  On this
inviscid path mu, k, mu_t and k_t are 0, S is 0, and tke, omega are 0 and 1
(the values the reference writes without the k-omega model).

Cell centroids and volumes follow ``xyplane_quad_cell_properties``
(src/geom/elements/properties.d:177-215) in 2-D and ``hex_cell_properties``
(properties.d:568-648, six pyramids of four tetrahedra each) in 3-D.
"""
from __future__ import annotations

import gzip
import struct

import numpy as np

HEADER = "structured_grid_flow 1.0"


def variable_names(species):
    """Names of the flow-file variables for a gas with these species."""
    names = ["pos.x", "pos.y", "pos.z", "volume", "rho", "vel.x", "vel.y", "vel.z",
             "p", "a", "mu", "k", "mu_t", "k_t", "S", "tke", "omega"]
    for i, sp in enumerate(species):
        names.append("massf[%d]-%s" % (i, "-".join(str(sp).split())))
    if len(species) > 1:
        names.append("dt_chem")
    names += ["u", "T"]
    return names


def _corners(vtx, ni, nj, nk, dimensions):
    nk1 = nk + 1 if dimensions == 3 else 1
    v = np.asarray(vtx, dtype=np.float64).reshape(nk1, nj + 1, ni + 1, 3)
    if dimensions == 2:
        p0 = v[0, :-1, :-1]
        p1 = v[0, :-1, 1:]
        p2 = v[0, 1:, 1:]
        p3 = v[0, 1:, :-1]
        return [p.reshape(-1, 3) for p in (p0, p1, p2, p3)]
    p = []
    for dk, dj, di in ((0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 0),
                       (1, 0, 0), (1, 0, 1), (1, 1, 1), (1, 1, 0)):
        p.append(v[dk:dk + nk, dj:dj + nj, di:di + ni].reshape(-1, 3))
    return p


def _tet(p0, p1, p2, p3):
    c = 0.25 * (p0 + p1 + p2 + p3)
    d01 = p1 - p0
    d02 = p2 - p0
    cr = np.stack([d01[:, 1] * d02[:, 2] - d01[:, 2] * d02[:, 1],
                   d01[:, 2] * d02[:, 0] - d01[:, 0] * d02[:, 2],
                   d01[:, 0] * d02[:, 1] - d01[:, 1] * d02[:, 0]], axis=1)
    d03 = p3 - p0
    vol = (d03[:, 0] * cr[:, 0] + d03[:, 1] * cr[:, 1] + d03[:, 2] * cr[:, 2]) / 6.0
    return c, vol


def _pyramid(p0, p1, p2, p3, p4):
    pmB = 0.25 * (p0 + p1 + p2 + p3)
    vol = np.zeros(p0.shape[0])
    mom = np.zeros_like(p0)
    for a, b in ((p0, p1), (p1, p2), (p2, p3), (p3, p0)):
        c, v = _tet(a, b, pmB, p4)
        vol = vol + v
        mom = mom + c * v[:, None]
    nz = np.abs(vol) > 0.0
    cen = np.where(nz[:, None], mom / np.where(nz, vol, 1.0)[:, None], mom)
    return cen, vol


def cell_geometry(vtx, ni, nj, nk, dimensions):
    """Centroids (n, 3) and volumes (n,) of the interior cells, i fastest."""
    if dimensions == 2:
        p0, p1, p2, p3 = _corners(vtx, ni, nj, nk, 2)
        xA, yA = p1[:, 0], p1[:, 1]
        xB, yB = p2[:, 0], p2[:, 1]
        xC, yC = p3[:, 0], p3[:, 1]
        xD, yD = p0[:, 0], p0[:, 1]
        area = 0.5 * ((xB + xA) * (yB - yA) + (xC + xB) * (yC - yB) +
                      (xD + xC) * (yD - yC) + (xA + xD) * (yA - yD))
        x = 1.0 / (area * 6.0) * ((yB - yA) * (xA * xA + xA * xB + xB * xB) +
                                  (yC - yB) * (xB * xB + xB * xC + xC * xC) +
                                  (yD - yC) * (xC * xC + xC * xD + xD * xD) +
                                  (yA - yD) * (xD * xD + xD * xA + xA * xA))
        y = -1.0 / (area * 6.0) * ((xB - xA) * (yA * yA + yA * yB + yB * yB) +
                                   (xC - xB) * (yB * yB + yB * yC + yC * yC) +
                                   (xD - xC) * (yC * yC + yC * yD + yD * yD) +
                                   (xA - xD) * (yD * yD + yD * yA + yA * yA))
        return np.stack([x, y, np.zeros_like(x)], axis=1), area
    p = _corners(vtx, ni, nj, nk, 3)
    cen0 = 0.125 * (p[0] + p[1] + p[2] + p[3] + p[4] + p[5] + p[6] + p[7])
    vol = np.zeros(p[0].shape[0])
    mom = np.zeros_like(p[0])
    for q in ((6, 7, 3, 2), (5, 6, 2, 1), (4, 5, 1, 0), (7, 4, 0, 3), (7, 6, 5, 4), (0, 1, 2, 3)):
        c, v = _pyramid(p[q[0]], p[q[1]], p[q[2]], p[q[3]], cen0)
        vol = vol + v
        mom = mom + c * v[:, None]
    nz = np.abs(vol) > 0.0
    cen = np.where(nz[:, None], mom / np.where(nz, vol, 1.0)[:, None], mom)
    return cen, vol


def flow_columns(prim, pos, volume, nsp, dt_chem=None):
    """(nvar, n) values in flow-file order from the primitive SoA array
    (rho, vx, vy, vz, p, T, u, a, massf...)."""
    prim = np.asarray(prim, dtype=np.float64)
    n = prim.shape[1]
    z = np.zeros(n)
    cols = [pos[:, 0], pos[:, 1], pos[:, 2], volume, prim[0], prim[1], prim[2], prim[3],
            prim[4], prim[7], z, z, z, z, z, z, np.ones(n)]
    if nsp > 1:
        cols += [prim[8 + s] for s in range(nsp)]
        cols.append(np.asarray(dt_chem, dtype=np.float64) if dt_chem is not None else np.full(n, -1.0))
    else:
        cols.append(np.ones(n))
    cols += [prim[6], prim[5]]
    return np.stack(cols)


def write_flow(path, *, prim, pos, volume, dimensions, ni, nj, nk, species, sim_time,
               label="", dt_chem=None, fmt="gziptext"):
    """Write one block's flow file."""
    names = variable_names(species)
    data = flow_columns(prim, pos, volume, len(species), dt_chem)
    assert data.shape[0] == len(names)
    iS = names.index("S")
    if fmt == "rawbinary":
        with open(path, "wb") as f:
            f.write(HEADER.encode())
            f.write(struct.pack("=i", len(label)))
            if label:
                f.write(label.encode())
            f.write(struct.pack("=d", float(sim_time)))
            f.write(struct.pack("=i", len(names)))
            for nm in names:
                f.write(struct.pack("=i", len(nm)))
                f.write(nm.encode())
            f.write(struct.pack("=4i", dimensions, ni, nj, nk))
            f.write(np.ascontiguousarray(data.T).astype("<f8").tobytes())
        return
    head = [HEADER, "label: %s" % label, "sim_time: %.18e" % sim_time,
            "variables: %d" % len(names), "".join(' "%s"' % nm for nm in names),
            "dimensions: %d" % dimensions, "nicell: %d" % ni, "njcell: %d" % nj,
            "nkcell: %d" % nk]
    fmts = ["%.18e"] * len(names)
    fmts[iS] = "%d"
    line = " " + " ".join(fmts) + "\n"
    with gzip.open(path, "wt") as f:
        f.write("\n".join(head) + "\n")
        rows = data.T.tolist()
        for r in rows:
            r[iS] = int(r[iS])
            f.write(line % tuple(r))


def read_flow(path, fmt="gziptext"):
    """Read one block's flow file: a dict with label, sim_time, variables,
    dimensions, nicell, njcell, nkcell and data (nvar, n)."""
    if fmt == "rawbinary":
        with open(path, "rb") as f:
            buf = f.read()
        o = len(HEADER)
        if buf[:o].decode() != HEADER:
            raise ValueError("unexpected header in %s" % path)
        (nl,) = struct.unpack_from("=i", buf, o)
        o += 4
        label = buf[o:o + nl].decode()
        o += nl
        (sim_time,) = struct.unpack_from("=d", buf, o)
        o += 8
        (nv,) = struct.unpack_from("=i", buf, o)
        o += 4
        names = []
        for _ in range(nv):
            (ln,) = struct.unpack_from("=i", buf, o)
            o += 4
            names.append(buf[o:o + ln].decode())
            o += ln
        dims, ni, nj, nk = struct.unpack_from("=4i", buf, o)
        o += 16
        data = np.frombuffer(buf, dtype="<f8", count=nv * ni * nj * nk, offset=o)
        data = data.reshape(ni * nj * nk, nv).T.copy()
    else:
        with gzip.open(path, "rt") as f:
            lines = f.read().splitlines()
        if lines[0].strip() != HEADER:
            raise ValueError("unexpected header in %s" % path)
        label = lines[1].split(":", 1)[1].strip()
        sim_time = float(lines[2].split(":", 1)[1])
        nv = int(lines[3].split(":", 1)[1])
        names = [t.strip('"') for t in lines[4].split()]
        assert len(names) == nv
        dims = int(lines[5].split(":", 1)[1])
        ni = int(lines[6].split(":", 1)[1])
        nj = int(lines[7].split(":", 1)[1])
        nk = int(lines[8].split(":", 1)[1])
        data = np.array([[float(x) for x in ln.split()] for ln in lines[9:9 + ni * nj * nk]]).T
    return {"label": label, "sim_time": sim_time, "variables": names, "dimensions": dims,
            "nicell": ni, "njcell": nj, "nkcell": nk, "data": data}


def prim_from_flow(flow, nsp):
    """The primitive SoA array (rho, vx, vy, vz, p, T, u, a, massf...) and the
    per-cell dt_chem (None for one species) of a flow file read by read_flow."""
    names = flow["variables"]
    d = flow["data"]

    def col(nm):
        return d[names.index(nm)]

    rows = [col("rho"), col("vel.x"), col("vel.y"), col("vel.z"), col("p"), col("T"), col("u"),
            col("a")]
    massf = [n for n in names if n.startswith("massf[")]
    if nsp > 1:
        if len(massf) != nsp:
            raise ValueError("the flow file has %d species, the gas %d" % (len(massf), nsp))
        rows += [col(n) for n in massf]
    dt_chem = col("dt_chem") if (nsp > 1 and "dt_chem" in names) else None
    return np.ascontiguousarray(np.stack(rows)), dt_chem
