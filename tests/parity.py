"""Shared helpers of the GPU parity tests: run a workload on the CPU oracle
and on the CUDA library (through its C ABI) and compare the results with ==."""
import numpy as np

FLUX = {"ausmdv": 0, "hllc": 1, "hanel": 2, "adaptive_hanel_ausmdv": 3}


def run_oracle(oracle, wl, nsteps, max_time=1.0e300, **cfgkw):
    cfg = oracle.default_config(dimensions=wl.dimensions,
                                flux_calculator=FLUX[wl.flux_calculator], n_threads=0, **cfgkw)
    sim = oracle.OracleSim(cfg)
    for b in wl.blocks:
        h = sim.add_block(b.ni, b.nj, b.nk, b.vtx, b.bc, b.inflow)
        sim.set_flow(h, b.prim)
    rc = sim.run(nsteps, max_time)
    out = [sim.get_flow(h) for h in range(len(wl.blocks))]
    return rc, sim.step, sim.time, sim.dt_global, out


def run_gpu(wl, nsteps, max_time=1.0e300, precision="fp64", use_graphs=True, **cfgkw):
    from eilmer4_b200.simcore import Simulation
    cfgd = {}
    ctl = {}
    for k, v in cfgkw.items():
        if k in ("cfl_value", "cfl_count", "dt_init", "dt_max"):
            ctl[k] = v
        else:
            cfgd[k] = v
    with Simulation.from_workload(wl, precision=precision, control=ctl, use_graphs=use_graphs,
                                  **cfgd) as sim:
        info = sim.run(nsteps, max_time)
        out = [sim.download(h) for h in range(len(wl.blocks))]
        t, dt, st = sim.state()
    return info, st, t, dt, out


def assert_same(a, b, what):
    a = np.asarray(a)
    b = np.asarray(b)
    if not np.array_equal(a, b):
        bad = np.argwhere(a != b)
        q = tuple(bad[0])
        rel = np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300))
        raise AssertionError(f"{what}: {len(bad)} values differ; first at {q}: "
                             f"gpu={a[q]!r} oracle={b[q]!r}; max rel {rel:.3e}")


def compare(oracle, wl, nsteps, max_time=1.0e300, use_graphs=True, **kw):
    orc, ost, otime, odt, oout = run_oracle(oracle, wl, nsteps, max_time,
                                            **{k: v for k, v in kw.items() if k in
                                               ("cfl_value", "update_scheme",
                                                "interpolation_order", "cfl_count")})
    assert orc == 0
    gkw = {}
    if "update_scheme" in kw:
        gkw["gasdynamic_update_scheme"] = "euler" if kw["update_scheme"] == 0 else "pc"
    if "interpolation_order" in kw:
        gkw["interpolation_order"] = kw["interpolation_order"]
    if "cfl_value" in kw:
        gkw["cfl_value"] = kw["cfl_value"]
    info, gst, gtime, gdt, gout = run_gpu(wl, nsteps, max_time, use_graphs=use_graphs, **gkw)
    assert gst == ost, (gst, ost)
    assert gtime == otime and gdt == odt, (gtime, otime, gdt, odt)
    for b, ((gp, gc), (op, oc)) in enumerate(zip(gout, oout)):
        assert_same(gc, oc, f"block {b} conserved")
        assert_same(gp[:8], op[:8], f"block {b} primitive")
    return info
