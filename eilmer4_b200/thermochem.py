"""Thermally perfect 5-species air and its reaction mechanism, as plain arrays.

Plays the part of the reference's ``prep-gas`` / ``prep-chem`` steps for the
reacting workload: reads ``data/air5_gas_model.json`` (extracted from the
reference's sample decks by ``data/make_air5.py``), parses the reaction
equations into integer stoichiometric coefficients and converts the
Arrhenius pre-exponential factors from cm-mol-s to SI units the way
``src/kinetics/reaction.lua:20-36`` does (factor 1e-6^(nc-1), nc = sum of the
reactant coefficients of that direction, plus one for an anonymous collider).
The arrays fill the ``e4c_thermochem`` struct of the C ABI.
"""
from __future__ import annotations

import json
import os
import re
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "data", "air5_gas_model.json")
R_UNIVERSAL = 8.31451
MAXSP, MAXSEG, MAXR = 8, 4, 8


def _side(text, species):
    coeffs = {}
    third = False
    for term in [t.strip() for t in text.split("+")]:
        if term == "M":
            third = True
            continue
        m = re.match(r"^(\d*)\s*(\S+)$", term)
        n = int(m.group(1)) if m.group(1) else 1
        sp = m.group(2)
        coeffs[species.index(sp)] = coeffs.get(species.index(sp), 0) + n
    return coeffs, third


@dataclass
class ThermoChem:
    species: list
    M: np.ndarray
    nseg: np.ndarray
    T_break: np.ndarray       # (nsp, MAXSEG+1)
    T_blend: np.ndarray       # (nsp, MAXSEG)
    coeffs: np.ndarray        # (nsp, MAXSEG, 9)
    A_f: np.ndarray
    n_f: np.ndarray
    C_f: np.ndarray
    A_b: np.ndarray
    n_b: np.ndarray
    C_b: np.ndarray
    nu_r: np.ndarray          # (nreac, nsp) int
    nu_p: np.ndarray
    third_body: np.ndarray    # (nreac,) int
    eff: np.ndarray           # (nreac, nsp)
    T_lower: float
    T_upper: float

    @property
    def nsp(self):
        return len(self.species)

    @property
    def nreac(self):
        return len(self.A_f)

    @property
    def R(self):
        return R_UNIVERSAL / self.M

    def fill(self, st):
        """Fill a ctypes e4c_thermochem / e4o_thermochem structure."""
        st.nsp = self.nsp
        for i in range(self.nsp):
            st.M[i] = float(self.M[i])
            st.nseg[i] = int(self.nseg[i])
            for q in range(MAXSEG + 1):
                st.T_break[i][q] = float(self.T_break[i, q])
            for q in range(MAXSEG):
                st.T_blend[i][q] = float(self.T_blend[i, q])
                for c in range(9):
                    st.coeffs[i][q][c] = float(self.coeffs[i, q, c])
        st.nreac = self.nreac
        for r in range(self.nreac):
            st.A_f[r], st.n_f[r], st.C_f[r] = float(self.A_f[r]), float(self.n_f[r]), float(self.C_f[r])
            st.A_b[r], st.n_b[r], st.C_b[r] = float(self.A_b[r]), float(self.n_b[r]), float(self.C_b[r])
            st.third_body[r] = int(self.third_body[r])
            for i in range(self.nsp):
                st.nu_r[r][i] = int(self.nu_r[r, i])
                st.nu_p[r][i] = int(self.nu_p[r, i])
                st.eff[r][i] = float(self.eff[r, i])
        st.T_lower = float(self.T_lower)
        st.T_upper = float(self.T_upper)
        return st

    # -- thermodynamics for preparing initial states (host side, numpy) ----
    def _coeffs_at(self, isp, T):
        tb, bl, c = self.T_break[isp], self.T_blend[isp], self.coeffs[isp]
        ns = int(self.nseg[isp])
        if T < tb[1] - 0.5 * bl[0]:
            return c[0]
        if T > tb[ns - 1] + 0.5 * bl[ns - 2]:
            return c[ns - 1]
        for i in range(1, ns):
            lo, hi = tb[i] - 0.5 * bl[i - 1], tb[i] + 0.5 * bl[i - 1]
            if lo <= T <= hi:
                wB = (1.0 / bl[i - 1]) * (T - lo)
                return (1.0 - wB) * c[i - 1] + wB * c[i]
            if hi < T < tb[i + 1] - 0.5 * bl[i]:
                return c[i]
        raise ValueError("temperature outside the curves")

    def h(self, isp, T):
        a = self._coeffs_at(isp, T)
        h_on_RT = (-a[0] / (T * T) + a[1] / T * np.log(T) + a[2] + a[3] * T / 2.0
                   + a[4] * T * T / 3.0 + a[5] * T ** 3 / 4.0 + a[6] * T ** 4 / 5.0 + a[7] / T)
        return self.R[isp] * T * h_on_RT

    def Cp(self, isp, T):
        a = self._coeffs_at(isp, T)
        return self.R[isp] * (a[0] / (T * T) + a[1] / T + a[2] + a[3] * T + a[4] * T * T
                              + a[5] * T ** 3 + a[6] * T ** 4)

    def state_pT(self, p, T, massf):
        """rho, u, a of a mixture at (p, T) (update_thermo_from_pT + frozen sound speed)."""
        massf = np.asarray(massf, dtype=np.float64)
        R = self.R
        Rmix = float(np.dot(massf, R))
        rho = p / (Rmix * T)
        u = float(sum(massf[i] * (self.h(i, T) - R[i] * T) for i in range(self.nsp)))
        Cp = float(sum(massf[i] * self.Cp(i, T) for i in range(self.nsp)))
        Cv = float(sum(massf[i] * (self.Cp(i, T) - R[i]) for i in range(self.nsp)))
        a = np.sqrt(Cp / Cv * (Rmix * T))
        return rho, u, float(a)


def load_air5(path: str = DATA) -> ThermoChem:
    with open(path) as f:
        d = json.load(f)
    species = d["species"]
    nsp = len(species)
    M = np.array([d["thermo"][s]["M"] for s in species])
    nseg = np.array([d["thermo"][s]["nsegments"] for s in species], dtype=np.int32)
    T_break = np.zeros((nsp, MAXSEG + 1))
    T_blend = np.zeros((nsp, MAXSEG))
    coeffs = np.zeros((nsp, MAXSEG, 9))
    for i, s in enumerate(species):
        t = d["thermo"][s]
        T_break[i, :len(t["T_break_points"])] = t["T_break_points"]
        T_blend[i, :len(t["T_blend_ranges"])] = t["T_blend_ranges"]
        for q, seg in enumerate(t["segments"]):
            coeffs[i, q, :] = seg
    reacs = d["reactions"]
    nr = len(reacs)
    A_f, n_f, C_f = np.zeros(nr), np.zeros(nr), np.zeros(nr)
    A_b, n_b, C_b = np.zeros(nr), np.zeros(nr), np.zeros(nr)
    nu_r = np.zeros((nr, nsp), dtype=np.int32)
    nu_p = np.zeros((nr, nsp), dtype=np.int32)
    third = np.zeros(nr, dtype=np.int32)
    eff = np.zeros((nr, nsp))
    for r, rx in enumerate(reacs):
        lhs, rhs = [x.strip() for x in rx["equation"].split("<=>")]
        reac, tb1 = _side(lhs, species)
        prod, tb2 = _side(rhs, species)
        third[r] = int(tb1 or tb2)
        for i, n in reac.items():
            nu_r[r, i] = n
        for i, n in prod.items():
            nu_p[r, i] = n
        # reaction.lua:20-36: A in cm^3 mol^-1 s^-1 units -> SI
        nc_f = sum(reac.values()) + (1 if third[r] else 0)
        nc_b = sum(prod.values()) + (1 if third[r] else 0)
        A_f[r] = rx["fr"][0] * (1.0e-6 ** (nc_f - 1))
        A_b[r] = rx["br"][0] * (1.0e-6 ** (nc_b - 1))
        n_f[r], C_f[r] = rx["fr"][1], rx["fr"][2]
        n_b[r], C_b[r] = rx["br"][1], rx["br"][2]
        for i, s in enumerate(species):
            eff[r, i] = rx["efficiencies"].get(s, 1.0 if third[r] else 0.0)
    lo, hi = d["temp_limits"]
    return ThermoChem(species, M, nseg, T_break, T_blend, coeffs, A_f, n_f, C_f, A_b, n_b, C_b,
                      nu_r, nu_p, third, eff, lo, hi)
