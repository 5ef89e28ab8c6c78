"""Helpers shared by the tests: golden fixtures and comparison metrics."""
from __future__ import annotations

import os

import numpy as np

from lps_b200.files import InputSet

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_inputs(name: str) -> InputSet:
    z = np.load(os.path.join(GOLDEN, f"{name}_inputs.npz"))
    sc = z["scal"]
    n_nodes = int(z["nodes"].shape[0])
    return InputSet(n_nodes=n_nodes, n_steps=int(z["n_steps"]), n_abc=int(z["n_abc"]),
                    max_cloud=int(z["max_cloud"]), E=sc[0], nu=sc[1], rho=sc[2], wf=sc[3], t0=sc[4],
                    t1=sc[5], dt=sc[6], delta=sc[7], dx=sc[8], dy=sc[9], s0=sc[10],
                    data2_extra=z["data2_extra"], nodes=z["nodes"], bctypes=z["bctypes"], u0=z["u0"],
                    v0=z["v0"], inf_nodes=z["inf_nodes"], clouds=z["clouds"], gu=z["gu"], gv=z["gv"],
                    gtheta=z["gtheta"])


def load_golden(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    return {k: z[k] for k in z.files}


def rel_l2(a, b) -> float:
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


# column maps of the reference logs (src/main.cpp:1108-1122)
ENERGY_COL = dict(t=0, E=1, Ek=2, Ep=3, Px=4, Py=5, max_u=6, theta_max=7, uB_rms=8, vB_rms=9)
VERIFY_COL = dict(t=0, E=1, dE_rel=2, Px=3, Py=4, theta_max=5, max_u=6, max_v=7, max_a=8)

# golden variant -> solver switches
VARIANT_OPTS = {
    "m1": dict(abcs_step=2, theta_method=1, kinematic_v=0),
    "m0": dict(abcs_step=2, theta_method=0, kinematic_v=0),
    "kin": dict(abcs_step=2, theta_method=1, kinematic_v=1),
    "off": dict(abcs_step=-1, theta_method=1, kinematic_v=0),
    "nu35": dict(abcs_step=2, theta_method=1, kinematic_v=0),
    "stock": dict(abcs_step=2, theta_method=1, kinematic_v=0),
}

GOLDEN_CASES = [("td", "m1"), ("td", "nu35"), ("r10", "m1"), ("r10", "m0"), ("r10", "kin"),
                ("r10", "off"), ("r10", "nu35"), ("r20", "m1"), ("r20", "m0")]


def inputs_for(case: str, variant: str) -> InputSet:
    s = load_inputs(case)
    if variant == "nu35":
        s.nu = 0.35
    return s


def compare_series(diag: dict, g: dict, tol_abs: float):
    """Max abs difference of each logged column (diag: name -> array)."""
    out = {}
    for name, c in ENERGY_COL.items():
        key = "theta_max" if name == "theta_max" else name
        if key in diag:
            out["energy." + name] = float(np.max(np.abs(diag[key] - g["energy"][:, c]), initial=0.0))
    for name, c in VERIFY_COL.items():
        if name in diag:
            out["verify." + name] = float(np.max(np.abs(diag[name] - g["verify"][:, c]), initial=0.0))
    return out
