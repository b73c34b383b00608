"""The reference's GPU chemistry kernel (alpha-QSS, new_qss in
src/eilmer/utils/alpha_qss_kernel_cuda_tmplt.cu) for the 5-species air
mechanism: the generated source terms against the mechanism's rates, the
NumPy restatement of the kernel against an independent integration, and on
the GPU the compiled kernel against its restatement and against this
library's point-implicit chemistry on the same cell states."""
import os
import time

import numpy as np
import pytest

from oracle import ref_qss as RQ


def mech_q_L(tc, kf, kb, c):
    """Production and loss rates of every species (eval_split_rates,
    reaction_mechanism.d:68-82), NumPy, per cell."""
    q = np.zeros_like(c)
    L = np.zeros_like(c)
    for r in range(tc.nreac):
        M = (tc.eff[r][:, None] * c).sum(axis=0) if tc.third_body[r] else 1.0
        wf = kf[r] * M * np.prod(c ** tc.nu_r[r][:, None], axis=0)
        wb = kb[r] * M * np.prod(c ** tc.nu_p[r][:, None], axis=0)
        for i in range(tc.nsp):
            nu = tc.nu_p[r][i] - tc.nu_r[r][i]
            if nu > 0:
                q[i] += nu * wf
                L[i] += nu * wb
            elif nu < 0:
                q[i] += -nu * wb
                L[i] += -nu * wf
    return q, L


def hot_cells(n, seed):
    from eilmer4_b200.thermochem import load_air5
    tc = load_air5()
    rng = np.random.default_rng(seed)
    T = 3000.0 + 5000.0 * rng.random(n)
    y = np.array([0.74, 0.2, 0.02, 0.01, 0.03])[:, None] + 0.01 * rng.random((5, n))
    y /= y.sum(axis=0)
    rho = 0.01 + 0.05 * rng.random(n)
    return tc, rho, T, y


def test_source_terms_are_the_mechanism_rates(oracle):
    tc, rho, T, y = hot_cells(64, 1)
    conc, kf, kb, h = oracle.gpuchem_prepare(tc, rho, T, y, np.full(64, -1.0))
    ydot = RQ.compile_terms(RQ.source_terms(tc))
    q, p, _ = ydot([conc[s] for s in range(5)], kf, kb, 5, 5)
    qm, Lm = mech_q_L(tc, kf, kb, conc)
    for s in range(5):
        assert np.allclose(q[s], qm[s], rtol=1e-13, atol=0.0), s
        assert np.allclose(p[s] * conc[s], Lm[s], rtol=1e-13, atol=1e-300), s
    # the step estimate is estimateStepSize's, within its clamps
    assert np.all((h >= 1e-15) & (h <= 1e-10))


def test_template_takes_the_source_terms():
    from __graft_entry__ import reference_root
    template = RQ.template_path(reference_root())
    if not os.path.exists(template):
        pytest.skip("reference tree not present")
    from eilmer4_b200.thermochem import load_air5
    with open(template) as f:
        text = f.read()
    assert text.count(RQ.MARK) == 1
    assert "__global__ void new_qss" in text and "kernel_launcher" in text
    terms = RQ.source_terms(load_air5())
    assert terms.count("q[idx+numcell*") == 5 and terms.count("p[idx+numcell*") == 5
    assert terms.count("MM[idx+numcell*") >= 3


def test_alpha_qss_restatement_follows_the_exact_solution(oracle):
    """The restated kernel integrates the constant-temperature rate equations
    over 10 us to within its own tolerance (e = 1e-3, relative to the change)
    of an implicit Radau solution."""
    scipy_integrate = pytest.importorskip("scipy.integrate")
    from eilmer4_b200.thermochem import load_air5
    tc = load_air5()
    y0 = np.array([0.767, 0.233, 0.0, 0.0, 0.0])
    T = np.array([4000.0, 6000.0])
    rho = np.array([0.05, 0.02])
    conc, kf, kb, h = oracle.gpuchem_prepare(tc, rho, T, np.repeat(y0[:, None], 2, axis=1),
                                             np.full(2, -1.0))
    dt = 1.0e-5
    Y, h_out, passes = RQ.new_qss_numpy(tc, kf, kb, conc, h, dt)
    assert passes.max() < 5000
    for c in range(2):
        def rhs(_t, cc):
            q, L = mech_q_L(tc, kf[:, c:c + 1], kb[:, c:c + 1], np.maximum(cc, 0.0)[:, None])
            return (q - L)[:, 0]
        sol = scipy_integrate.solve_ivp(rhs, (0.0, dt), conc[:, c], method="Radau", rtol=1e-10,
                                        atol=1e-14 * conc[:, c].sum())
        ye = sol.y[:, -1]
        change = np.abs(ye - conc[:, c]).max()
        assert change > 1e-3 * conc[:, c].sum()
        assert np.abs(Y[:, c] - ye).max() <= 1e-3 * change, (Y[:, c], ye)


# ---------------------------------------------------------------------------
# GPU: the compiled reference kernel
# ---------------------------------------------------------------------------
def _run_reference_kernel(tc, kf, kb, conc, h, dt):
    import torch
    L = RQ.load()
    n = conc.shape[1]
    dev = torch.device("cuda:0")
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=dev)
    z = lambda rows: torch.zeros(rows * n, dtype=torch.float64, device=dev)
    bufs = {"kf": t(kf), "kb": t(kb), "MM": z(tc.nreac), "Y": t(conc), "Yp": z(5), "Yc": z(5),
            "h": t(h), "alpha": z(5), "q": z(5), "p": z(5), "qp": z(5), "pp": z(5),
            "q_bar": z(5), "p_bar": z(5), "alpha_bar": z(5), "Ypo": z(5)}
    dbg = torch.zeros(1, dtype=torch.float64, device=dev)
    order = ["kf", "kb", "MM", "Y", "Yp", "Yc", "h", "alpha", "q", "p", "qp", "pp", "q_bar",
             "p_bar", "alpha_bar", "Ypo"]
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    L.kernel_launcher(*[bufs[k].data_ptr() for k in order], tc.nsp, tc.nreac, n, dt,
                      dbg.data_ptr(), 1, 1, n, 1)
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    Y = bufs["Y"].cpu().numpy().reshape(5, n)
    h_out = bufs["h"].cpu().numpy()
    return Y, h_out, ms


@pytest.mark.gpu
def test_reference_gpu_chemistry_against_its_restatement_and_ours(oracle, e4lib):
    """On the states of the high-enthalpy channel after 60 steps: the
    reference kernel, compiled for sm_100a, gives what its NumPy restatement
    gives (the sub-step loop bounded on the CPU first); this library's
    point-implicit update lands within the integrators' first-order error of
    it; and both are timed on the same cells."""
    if not os.path.exists(RQ.LIB):
        pytest.skip("reference kernel not built (oracle/_ref)")
    from eilmer4_b200 import _lib
    from eilmer4_b200 import workloads as W
    from eilmer4_b200.simcore import Simulation
    wl = W.reacting_channel_hot(ni=128, nj=64)
    tc = wl.thermochem
    n = wl.ncell
    with Simulation.from_workload(wl, reacting=True) as sim:
        sim.run(60)
        prim, _ = sim.download(0)
        dtc = np.zeros(n)
        sim.L.e4c_block_get_dt_chem(0, _lib.dptr(dtc))
        _, dt, _ = sim.state()
        sim.chemistry_counters(reset=True)
        sim.synchronize()
        t0 = time.perf_counter()
        sim.chemistry_step([0], dt)
        sim.synchronize()
        ours_ms = (time.perf_counter() - t0) * 1e3
        ours, _ = sim.download(0)
    rho, T, u, p, y = prim[0], prim[5], prim[6], prim[4], prim[8:13]
    conc, kf, kb, h = oracle.gpuchem_prepare(tc, rho, T, y, dtc)
    Yn, hn, passes = RQ.new_qss_numpy(tc, kf, kb, conc, h, dt, max_outer=20000)
    assert passes.max() < 20000
    Yg, hg, ref_ms = _run_reference_kernel(tc, kf, kb, conc, h, dt)
    assert np.all(np.isfinite(Yg))
    change = np.abs(Yn - conc).max(axis=0)
    tot = conc.sum(axis=0)
    # nvcc contracts to FMA by default, so a sub-step can be accepted or
    # rejected differently at its threshold: agreement to the kernel's own
    # tolerance, relative to each cell's change
    assert np.all(np.abs(Yg - Yn).max(axis=0) <= 1e-2 * change + 1e-12 * tot)
    rc, fin = oracle.gpuchem_finish(tc, Yg, hg, rho, T, u, p)
    assert rc == 0
    # ours against the reference kernel's mass fractions: both integrate the
    # same rates over dt; the point-implicit step is first order
    d_ref = fin["massf"] - y
    d_ours = ours[8:13] - y
    hot = np.abs(d_ref).max(axis=0) > 1e-4
    assert hot.sum() > 100
    err = np.abs(d_ours - d_ref).max(axis=0)
    rel = err[hot] / np.abs(d_ref).max(axis=0)[hot]
    assert np.median(rel) < 0.05 and rel.max() < 0.1, (np.median(rel), rel.max())
    print(f"\nreference new_qss kernel: {ref_ms:.3f} ms for {n} cells "
          f"({n / ref_ms * 1e3:.3e} cells/s; sub-steps per cell mean {passes.mean():.1f}, "
          f"max {passes.max()}); this library's chemistry step: {ours_ms:.3f} ms "
          f"({n / ours_ms * 1e3:.3e} cells/s)")
