"""The reference's own GPU chemistry kernel, built for sm_100a, and a NumPy
restatement of it.  Test and measurement infrastructure only.

Eilmer4's optional GPU chemistry (``version(gpu_chem)``, src/eilmer/
cuda_gpu_chem.d) integrates every cell's concentrations with the alpha-QSS
method in ``new_qss`` (src/eilmer/utils/alpha_qss_kernel_cuda_tmplt.cu:17-127),
one cell per one-thread CUDA block.  The template's ``ydot`` body (the
production and loss terms of the mechanism) is generated for each mechanism by
src/eilmer/utils/prep-cuda-gpu-chem-kernel.py, a Python 2 script that does not
run under Python 3.  ``source_terms`` restates what it writes -- the
compact-notation terms of Turns' textbook, as the script forms them (third-body
sums first, then q and p per species, reactions in order) -- for the
mechanism of a ``ThermoChem``.

``build`` substitutes those terms into the template where it lies in the
reference tree and compiles it as the script does (``nvcc --shared -fPIC``,
nvcc's default floating-point flags), for sm_100a, into ``oracle/_ref/``.
Nothing of the reference is copied into this repository: the generated
source and the library stay in ``oracle/_ref/``, which git ignores.

``new_qss_numpy`` restates the kernel, vectorised over cells with NumPy, to
check the compiled kernel and to bound its sub-step loop on the CPU before
the kernel runs on a GPU; ``kernel_launcher`` calls the compiled library.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libcudakernel.so")
SRC = os.path.join(OUT, "alpha_qss_kernel.cu")
# the kernel template, relative to the root of the reference tree (the
# caller names the root: the build step, or E4_REFERENCE_ROOT)
TEMPLATE_REL = os.path.join("src", "eilmer", "utils", "alpha_qss_kernel_cuda_tmplt.cu")


def template_path(reference_root: str) -> str:
    return os.path.join(reference_root, TEMPLATE_REL)
MARK = "// <insert-source-terms-here>"


def _num(x: float) -> str:
    return repr(float(x))


def _ys(counts, skip_one_of=None):
    """'*Y[idx+numcell*l]' once per unit of each positive coefficient; one
    unit of species skip_one_of is left out (the p*y form of the loss)."""
    out = []
    for l, c in enumerate(counts):
        c = int(c)
        if l == skip_one_of:
            c -= 1
        out.extend(["*Y[idx+numcell*%d]" % l] * max(c, 0))
    return "".join(out)


def source_terms(tc) -> str:
    """C statements of the ydot body for the mechanism of tc."""
    nsp, nr = tc.nsp, tc.nreac
    nu_r = np.asarray(tc.nu_r, dtype=int)
    nu_p = np.asarray(tc.nu_p, dtype=int)
    lines = []
    # third-body concentrations of the reactions that have a collider
    for r in range(nr):
        if not tc.third_body[r]:
            continue
        terms = ["Y[idx+numcell*%d]*%s" % (j, _num(tc.eff[r][j]))
                 for j in range(nsp) if float(tc.eff[r][j]) != 0.0]
        lines.append("MM[idx+numcell*%d]=%s;" % (r, "+".join(terms)))
    mm = lambda r: ("*MM[idx+numcell*%d]" % r) if tc.third_body[r] else ""
    # production terms q
    for j in range(nsp):
        terms = []
        for r in range(nr):
            v = nu_p[r, j] - nu_r[r, j]
            if v < 0:    # produced by the backward reaction
                terms.append("+kb[idx+numcell*%d]*%s%s%s" % (r, _num(-v), _ys(nu_p[r]), mm(r)))
            elif v > 0:  # produced by the forward reaction
                terms.append("+kf[idx+numcell*%d]*%s%s%s" % (r, _num(v), _ys(nu_r[r]), mm(r)))
        lines.append("q[idx+numcell*%d]=%s;" % (j, "".join(terms) if terms else "0.0"))
    # loss terms p (the loss rate divided by Y_j)
    for j in range(nsp):
        terms = []
        for r in range(nr):
            v = nu_p[r, j] - nu_r[r, j]
            if v < 0:    # lost in the forward reaction
                terms.append("+kf[idx+numcell*%d]*%s%s%s" % (r, _num(-v), _ys(nu_r[r], j), mm(r)))
            elif v > 0:  # lost in the backward reaction
                terms.append("+kb[idx+numcell*%d]*%s%s%s" % (r, _num(v), _ys(nu_p[r], j), mm(r)))
        lines.append("p[idx+numcell*%d]=%s;" % (j, "".join(terms) if terms else "0.0"))
    return "\n".join(lines) + "\n"


def build(tc, template: str, force: bool = False) -> str:
    """Generate and compile the reference kernel for tc's mechanism from the
    template file `template` (template_path of the reference tree)."""
    if os.path.exists(LIB) and not force:
        return LIB
    with open(template) as f:
        text = f.read()
    if MARK not in text:
        raise ValueError("the kernel template has no source-term marker")
    os.makedirs(OUT, exist_ok=True)
    with open(SRC, "w") as f:
        f.write(text.replace(MARK, source_terms(tc)))
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "--shared", "-o", LIB,
                    SRC, "--compiler-options", "-fPIC"], check=True)
    return LIB


def compile_terms(terms: str):
    """A Python function ydot(Y, kf, kb) -> (q, p, MM) evaluating the C
    statements in their own order (arrays indexed [species or reaction])."""
    body = re.sub(r"\[idx\+numcell\*(\d+)\]", r"[\1]", terms).replace(";", "")
    code = ["def ydot(Y, kf, kb, nsp, nr):",
            "    q = [None] * nsp", "    p = [None] * nsp", "    MM = [None] * nr"]
    code += ["    " + ln for ln in body.strip().splitlines()]
    code += ["    return q, p, MM"]
    ns = {}
    exec("\n".join(code), ns)
    return ns["ydot"]


def new_qss_numpy(tc, kf, kb, Y, h, dt_flow, max_outer: int = 1_000_000):
    """alpha_qss_kernel_cuda_tmplt.cu:17-127 for every cell at once.

    kf, kb (nreac, n), Y concentrations (nsp, n), h (n,).  Returns Y, h and
    the number of outer passes (sub-steps tried) per cell; raises if a cell
    needs more than max_outer passes."""
    nsp = tc.nsp
    ydot_f = compile_terms(source_terms(tc))

    def ydot(Yv, kfv, kbv):
        q, p, _ = ydot_f([Yv[s] for s in range(nsp)], kfv, kbv, nsp, tc.nreac)
        bc = lambda a: np.broadcast_to(np.asarray(a, dtype=np.float64), Yv[0].shape)
        return np.stack([bc(a) for a in q]), np.stack([bc(a) for a in p])

    def alpha_func(p, dt):
        rr = 1.0 / (p * dt + 1.0e-50)
        return ((180.0 * rr * rr * rr + 60.0 * rr * rr + 11.0 * rr + 1.0) /
                (360.0 * rr * rr * rr + 60.0 * rr * rr + 12.0 * rr + 1.0))

    Y = np.array(Y, dtype=np.float64)
    h = np.array(h, dtype=np.float64)
    n = Y.shape[1]
    kf = np.asarray(kf, dtype=np.float64)
    kb = np.asarray(kb, dtype=np.float64)
    e = 0.001
    epsilon = e / 2.0
    max_iterations = 10
    t = np.zeros(n)
    dt_chem = h.copy()
    dt_chem_temp = np.zeros(n)
    passes = np.zeros(n, dtype=np.int64)
    with np.errstate(all="ignore"):
        for _ in range(max_outer):
            act = np.nonzero(t < dt_flow)[0]
            if act.size == 0:
                return Y, h, passes
            passes[act] += 1
            Ya, kfa, kba, dt = Y[:, act], kf[:, act], kb[:, act], dt_chem[act]
            q, p = ydot(Ya, kfa, kba)
            alpha = alpha_func(p, dt)
            Yp = Ya + (dt * (q - p * Ya)) / (1.0 + alpha * dt * p)
            Ypo = Yp.copy()
            Yc = np.empty_like(Ya)
            flag = np.zeros(act.size, dtype=bool)
            live = np.ones(act.size, dtype=bool)    # step_fail == 1
            count = np.zeros(act.size, dtype=np.int64)
            while live.any():
                li = np.nonzero(live)[0]
                qp, pp = ydot(Yp[:, li], kfa[:, li], kba[:, li])
                p_bar = 0.5 * (pp + p[:, li])
                alpha_bar = alpha_func(p_bar, dt[li])
                q_bar = alpha_bar * qp + (1.0 - alpha_bar) * q[:, li]
                Ycl = Ya[:, li] + (dt[li] * (q_bar - p_bar * Ya[:, li])) / (1.0 + alpha_bar * dt[li] * p_bar)
                Yc[:, li] = Ycl
                cond = np.abs(Ycl - Ypo[:, li])
                fail = (cond >= e * (Ycl + 1.0e-10)).any(axis=0)
                count[li] += 1
                over = count[li] > max_iterations
                flag[li[over]] = True
                fail &= ~over
                Yp[:, li[fail]] = Ycl[:, fail]
                live[li] = fail
            ok = ~flag
            Y[:, act[ok]] = Yc[:, ok]
            t[act[ok]] += dt[ok]
            h[act[ok]] = dt_chem_temp[act[ok]]
            sigma = np.full(act.size, 1.0e-50)
            for s in range(nsp):
                cond = np.abs(Yc[s] - Ypo[s]) / (epsilon * Yc[s])
                sigma = np.where(cond > sigma, cond, sigma)
            x0 = sigma.copy()
            for _k in range(3):
                x0 = x0 - 0.5 * (x0 * x0 - sigma) / x0
            temp = np.where(sigma <= 0.0, dt, dt * ((1.0 / x0) + 0.005))
            ratio = temp / dt
            grow = np.where(ratio > 1.15, 1.15 * dt, temp)
            shrink = np.where(ratio > (1.0 / 3.0), (1.0 / 3.0) * dt,
                              np.where(ratio < 0.01, 0.01 * dt, temp))
            dtn = np.where(ok, grow, shrink)
            dt_chem_temp[act] = dtn
            dt_chem[act] = np.fmin(dt_flow - t[act], dtn)
    raise RuntimeError("new_qss restatement: a cell needs more than %d sub-steps" % max_outer)


def load(path: str = LIB):
    """ctypes handle of the compiled kernel library (kernel_launcher)."""
    L = ctypes.CDLL(path)
    vp, ci, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    L.kernel_launcher.argtypes = [vp] * 16 + [ci, ci, ci, ctypes.c_double, vp, sz, sz, sz, sz]
    L.kernel_launcher.restype = None
    return L
