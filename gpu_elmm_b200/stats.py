"""Horizontally averaged vertical profiles of a run, as the reference's
Profiles type computes them (src/vertical_profiles.f90): the mean velocity
u(k), v(k) over the staggered points of each level, the resolved variances
uu = <U^2> - u^2 (and vv, ww on the W levels), and the resolved TKE of a
pressure level, (uu(k) + vv(k) + (ww(k-1) + ww(k)) / 2) / 2
(src/vertical_profiles.f90:348-381).  Time averages weigh every sample
equally.  Host-side numpy on downloaded states; used to compare the mixed and
the FP64 path over long runs.
"""
from __future__ import annotations

import numpy as np

from .config import Grid
from .workloads import interior


class Profiles:
    def __init__(self, grid: Grid):
        self.g = grid
        self.n = 0
        g = grid
        self.u = np.zeros(g.Unz)
        self.v = np.zeros(g.Vnz)
        self.uu = np.zeros(g.Unz)
        self.vv = np.zeros(g.Vnz)
        self.ww = np.zeros(g.Prnz + 1)  # W levels 0..Prnz; W = 0 on wall levels
        self.theta = np.zeros(g.Prnz)

    def add(self, U, V, W, theta=None):
        """One sample: host arrays in the Fortran layout of workloads.py."""
        g = self.g
        Ui = interior(U, -2, (g.Unx, g.Uny, g.Unz))
        Vi = interior(V, -2, (g.Vnx, g.Vny, g.Vnz))
        Wi = interior(W, -2, (g.Wnx, g.Wny, g.Wnz))
        self.u += Ui.mean(axis=(1, 2))
        self.v += Vi.mean(axis=(1, 2))
        self.uu += (Ui * Ui).mean(axis=(1, 2))
        self.vv += (Vi * Vi).mean(axis=(1, 2))
        self.ww[1:1 + g.Wnz] += (Wi * Wi).mean(axis=(1, 2))
        if theta is not None:
            self.theta += interior(theta, -2, (g.Prnx, g.Prny, g.Prnz)).mean(axis=(1, 2))
        self.n += 1

    def result(self):
        n = max(self.n, 1)
        u, v = self.u / n, self.v / n
        uu, vv, ww = self.uu / n - u ** 2, self.vv / n - v ** 2, self.ww / n
        nz = self.g.Prnz
        tke = np.zeros(nz)
        m = min(len(uu), len(vv), nz)
        tke[:m] = (uu[:m] + vv[:m] + (ww[0:m] + ww[1:m + 1]) / 2) / 2
        return {"u": u, "v": v, "uu": uu, "vv": vv, "ww": ww, "tke": tke, "theta": self.theta / n}


def compare(a: dict, b: dict, keys=("u", "tke")) -> dict:
    """max |a - b| / max |b| per profile; theta compared as its deviation
    from the mean of b (the field sits near T_ref)."""
    out = {}
    for k in keys:
        if k == "theta":
            continue
        s = float(np.abs(b[k]).max())
        out[k] = float(np.abs(a[k] - b[k]).max()) / (s if s > 0 else 1.0)
    if "theta" in keys:
        ref = float(b["theta"].mean())
        s = float(np.abs(b["theta"] - ref).max())
        out["theta"] = float(np.abs(a["theta"] - b["theta"]).max()) / (s if s > 0 else 1.0)
    return out
