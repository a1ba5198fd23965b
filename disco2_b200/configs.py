"""Named workloads as Disco2 parfiles.

Every workload is a parfile in the reference's own key/value format
(reader: src/Sim/sim_readpar.c:48-122, 52 keys), so the same text drives the
reference C oracle and this package.  Three keys the reference reader never
asks for carry the parameters of the new initial conditions (IC_HoR,
IC_Noise, IC_Seed); InitialDataType 7/8/9 select the Gresho vortex, the
viscous Keplerian ring and the circumbinary disk.

Grid choices follow the reference's own rules: annuli per sim_set_rz
(src/Sim/sim_set.c:73-143; RLogScale >> R_Max gives near-uniform spacing,
RLogScale << R_Min gives log spacing), cells per annulus per sim_set_N_p
(src/Sim/sim_set.c:10-33) with aspect 1, one ghost annulus on each side
(ng = 1), fixed radial boundaries.
"""
from __future__ import annotations

import math
import random

# Parfile key order of src/Sim/sim_readpar.c:55-106, then the initial-data keys.
_KEYS = [
    "Restart", "InitialDataType", "GravMassType", "MassRatio", "OrbShrinkTscale",
    "OrbShrinkT0", "BoundTypeR", "BoundTypeZ", "NoInnerBC", "NumR", "NumZ", "ng",
    "R_Min", "R_Max", "Z_Min", "Z_Max", "NP_CONST", "NPCAP", "aspect", "NUM_C", "NUM_N",
    "Time_Max", "Num_Checkpoints", "Num_Diag_Dump", "Num_Diag_Measure", "w_numeric_type",
    "RiemannSolver", "Adiabatic_Index", "Cooling", "Explicit_Viscosity", "ViscConst",
    "PoRho_r1", "CFL", "PLM", "Grav_2D", "G_EPS", "RhoSinkOn", "PHI_ORDER", "Rho_Floor",
    "Cs_Floor", "Cs_Cap", "Vel_Cap", "DAMP_TIME", "RDAMP_INNER", "RDAMP_OUTER",
    "RLogScale", "ZLogScale", "HiResSigma", "HiResR0a", "HiResR0b", "HiResFac",
    "w_analytic_type", "IC_HoR", "IC_Noise", "IC_Seed",
]

_BASE = {
    "Restart": 0, "GravMassType": 0, "MassRatio": 1.0,
    "OrbShrinkTscale": 1.0e19, "OrbShrinkT0": 0.0,
    "BoundTypeR": 0, "BoundTypeZ": 2, "NoInnerBC": 0,
    "NumZ": 1, "ng": 1, "Z_Min": -1.0, "Z_Max": 1.0,
    "NP_CONST": -1, "NPCAP": 100000, "aspect": 1.0, "NUM_C": 5, "NUM_N": 0,
    "Time_Max": 1.0e30, "Num_Checkpoints": 1, "Num_Diag_Dump": 1, "Num_Diag_Measure": 1,
    "w_numeric_type": 0, "RiemannSolver": 0, "Adiabatic_Index": 5.0 / 3.0, "Cooling": 0,
    "Explicit_Viscosity": -1.0, "ViscConst": 0, "PoRho_r1": 1.0, "CFL": 0.4, "PLM": 1.5,
    "Grav_2D": 1, "G_EPS": 0.0, "RhoSinkOn": 0, "PHI_ORDER": 2,
    "Rho_Floor": 1.0e-8, "Cs_Floor": 1.0e-6, "Cs_Cap": 10.0, "Vel_Cap": 10.0,
    "DAMP_TIME": -1.0, "RDAMP_INNER": 0.0, "RDAMP_OUTER": 1.0e30,
    "RLogScale": 1.0e-6, "ZLogScale": 1.0e9, "HiResSigma": 1.0e9, "HiResR0a": 1.0e9,
    "HiResR0b": 1.0e9, "HiResFac": 0.0, "w_analytic_type": 0,
    "IC_HoR": 0.05, "IC_Noise": 0.0, "IC_Seed": 0,
}


def gresho(num_r: int = 96, **over) -> dict:
    """Steady Gresho vortex on the rigidly rotating (C_RIGID) mesh, HLLC."""
    p = dict(_BASE)
    p.update({
        "InitialDataType": 7, "NumR": num_r, "R_Min": 0.1, "R_Max": 1.0,
        "RLogScale": 1.0e9, "w_numeric_type": 2, "w_analytic_type": 0,
        "RiemannSolver": 0, "PLM": 1.5, "CFL": 0.4,
        "Rho_Floor": 1.0e-5, "Cs_Floor": 1.0e-4, "Cs_Cap": 100.0, "Vel_Cap": 100.0,
        "IC_Noise": 1.0e-6, "IC_Seed": 0,
    })
    p.update(over)
    return p


def kepler_ring(num_r: int = 256, **over) -> dict:
    """Viscous Keplerian ring around a unit point mass, HLL, constant nu."""
    p = dict(_BASE)
    p.update({
        "InitialDataType": 8, "GravMassType": 1, "NumR": num_r, "R_Min": 0.5, "R_Max": 4.0,
        "RiemannSolver": 1, "Explicit_Viscosity": 1.0e-3, "ViscConst": 1,
        "w_analytic_type": 1, "w_numeric_type": 0,
        "IC_HoR": 0.05, "IC_Noise": 1.0e-3, "IC_Seed": 1,
    })
    p.update(over)
    return p


def circumbinary(num_r: int = 400, r_max: float = 20.0, q: float = 1.0, alpha: float = 0.1,
                 hor: float = 0.1, seed: int = 2, **over) -> dict:
    """Equal-mass circular binary in an alpha-viscous disk, HLLC, outer damping."""
    p = dict(_BASE)
    p.update({
        "InitialDataType": 9, "GravMassType": 2, "MassRatio": q, "NumR": num_r,
        "R_Min": 0.4, "R_Max": r_max, "RiemannSolver": 0,
        "Explicit_Viscosity": alpha, "ViscConst": 0, "G_EPS": 0.05, "PHI_ORDER": 2,
        "w_analytic_type": 1, "w_numeric_type": 0,
        "DAMP_TIME": 2.0 * math.pi, "RDAMP_INNER": 0.0, "RDAMP_OUTER": 0.8 * r_max,
        "IC_HoR": hor, "IC_Noise": 1.0e-4, "IC_Seed": seed,
    })
    p.update(over)
    return p


def circumbinary_sweep(n: int = 48, seed: int = 3) -> list[dict]:
    """Independent circumbinary disks with q log-uniform in [0.01, 1], alpha in
    [0.01, 0.1], h/r in [0.05, 0.1], N_r in [128, 512], R_out in [10, 30]."""
    rng = random.Random(seed)
    out = []
    for k in range(n):
        q = 10.0 ** rng.uniform(-2.0, 0.0)
        alpha = rng.uniform(0.01, 0.1)
        hor = rng.uniform(0.05, 0.1)
        num_r = rng.randint(128, 512)
        r_max = rng.uniform(10.0, 30.0)
        out.append(circumbinary(num_r=num_r, r_max=r_max, q=q, alpha=alpha, hor=hor,
                                seed=1000 * seed + k))
    return out


# The reference's own test problems (parfiles/code_tests/*.par) and the other
# initial-data families of src/Cell/initial_data/, as 2-D disks.

def shear_test(num_r: int = 128, **over) -> dict:
    """Viscous shear layer (SHEAR) on a uniform grid, the settings of
    parfiles/code_tests/shear.par: outflow radial boundary, cooling on."""
    p = dict(_BASE)
    p.update({
        "InitialDataType": 0, "GravMassType": 0, "MassRatio": 0.0, "NumR": num_r, "ng": 2,
        "R_Min": 1.0, "R_Max": 10.0, "BoundTypeR": 1, "NoInnerBC": 0, "w_numeric_type": 0,
        "RiemannSolver": 0, "Adiabatic_Index": 1.3333333333333, "Cooling": 1,
        "Explicit_Viscosity": 0.05, "ViscConst": 1, "RhoSinkOn": 0, "PoRho_r1": 1.0, "CFL": 0.1,
        "PLM": 1.0, "w_analytic_type": 0, "Grav_2D": 1, "G_EPS": 0.0, "PHI_ORDER": 2,
        "Rho_Floor": 1.0e-5, "Cs_Floor": 1.0e-4, "Cs_Cap": 100.0, "Vel_Cap": 100.0,
        "DAMP_TIME": -1.0, "RLogScale": 1.0e6, "ZLogScale": 1.0e6, "HiResSigma": 1.0e6,
        "HiResR0a": 1.0e6, "HiResR0b": 1.0e6, "HiResFac": 0.0,
    })
    p.update(over)
    return p


def sstest(num_r: int = 128, **over) -> dict:
    """Shakura-Sunyaev disk around a point mass (SSTEST), the settings of
    parfiles/code_tests/SStest.par: two cells per annulus, log grid, no inner
    boundary, outflow, cooling, sink and a damping zone."""
    p = dict(_BASE)
    p.update({
        "InitialDataType": 2, "GravMassType": 1, "MassRatio": 0.0, "NumR": num_r, "ng": 2,
        "R_Min": 0.05, "R_Max": 100.0, "NP_CONST": 2, "NPCAP": 2, "BoundTypeR": 1,
        "NoInnerBC": 1, "w_numeric_type": 0, "RiemannSolver": 0, "Cooling": 1,
        "Explicit_Viscosity": 0.1, "ViscConst": 0, "RhoSinkOn": 1, "PoRho_r1": 0.01, "CFL": 0.1,
        "PLM": 1.0, "w_analytic_type": 1, "Grav_2D": 1, "G_EPS": 0.0, "PHI_ORDER": 2,
        "Rho_Floor": 1.0e-6, "Cs_Floor": 1.0e-5, "Cs_Cap": 1.0, "Vel_Cap": 10.0,
        "DAMP_TIME": 0.001, "RDAMP_INNER": 0.0, "RDAMP_OUTER": 90.0, "RLogScale": 1.0,
        "ZLogScale": 1000.0, "HiResSigma": 1.0e4, "HiResR0a": 1.0e5, "HiResR0b": 1.0e5,
        "HiResFac": 0.0,
    })
    p.update(over)
    return p


def vortex_test(num_r: int = 64, **over) -> dict:
    """Isentropic vortex (VORTEX) on the rigidly rotating mesh, the settings of
    parfiles/code_tests/vortex.par without its passive scalar (NUM_N 0)."""
    p = dict(_BASE)
    p.update({
        "InitialDataType": 1, "GravMassType": 0, "MassRatio": 1.0, "NumR": num_r, "ng": 2,
        "R_Min": 0.015, "R_Max": 0.9, "BoundTypeR": 0, "NoInnerBC": 1, "w_numeric_type": 2,
        "RiemannSolver": 0, "Cooling": 0, "Explicit_Viscosity": -1.0, "ViscConst": 0,
        "RhoSinkOn": 0, "PoRho_r1": 1.0, "CFL": 0.5, "PLM": 1.0, "w_analytic_type": 0,
        "Rho_Floor": 1.0e-5, "Cs_Floor": 1.0e-4, "Cs_Cap": 100.0, "Vel_Cap": 100.0,
        "DAMP_TIME": -1.0e-5, "RLogScale": 1.0e5, "ZLogScale": 1.0e5, "HiResSigma": 1.0e5,
        "HiResR0a": 1.0e5, "HiResR0b": 1.0e5, "HiResFac": 0.0,
    })
    p.update(over)
    return p


def torus_2d(num_r: int = 80, **over) -> dict:
    """Constant-angular-momentum torus (TORUS) in the midplane: the settings of
    parfiles/torus.par with one z layer (the reference parfile is 3-D)."""
    p = dict(_BASE)
    p.update({
        "InitialDataType": 3, "GravMassType": 1, "MassRatio": 0.0, "NumR": num_r, "ng": 2,
        "R_Min": 0.2, "R_Max": 3.0, "NPCAP": 20, "BoundTypeR": 1, "NoInnerBC": 0,
        "w_numeric_type": 6, "RiemannSolver": 0, "Cooling": 0, "Explicit_Viscosity": -1.0,
        "PoRho_r1": 1.0, "CFL": 0.5, "PLM": 1.0, "w_analytic_type": 4, "Grav_2D": 0,
        "G_EPS": 0.1, "PHI_ORDER": 2, "Rho_Floor": 1.0e-7, "Cs_Floor": 1.0e-6, "Cs_Cap": 2.0,
        "Vel_Cap": 2.0, "DAMP_TIME": -1.0, "RLogScale": 1.0e4, "ZLogScale": 1.0e4,
        "HiResSigma": 1.0e4, "HiResR0a": 1.0e4, "HiResR0b": 1.0e4, "HiResFac": 0.0,
    })
    p.update(over)
    return p


def torus_3d(num_r: int = 80, num_z: int = 80, **over) -> dict:
    """The reference's own 3-D parfile (parfiles/torus.par): a torus about a
    point mass, 80 annuli x 80 layers, at most 20 cells per ring, two ghost
    annuli and layers, outflow in r, periodic in z, HLLC, no viscosity."""
    p = torus_2d(num_r=num_r, NumZ=num_z, ng=2, Z_Min=-1.0, Z_Max=1.0, NPCAP=20, BoundTypeZ=2,
                 BoundTypeR=1, Grav_2D=0)
    p.update(over)
    return p


def milos_macfadyen(num_r: int = 128, **over) -> dict:
    """Circumbinary disk of MacFadyen & Milosavljevic (MILOS_MACFADYEN): binary,
    Keplerian mesh, no inner boundary, outflow, an outer damping zone."""
    p = dict(_BASE)
    p.update({
        "InitialDataType": 4, "GravMassType": 2, "MassRatio": 1.0, "NumR": num_r, "ng": 2,
        "R_Min": 0.5, "R_Max": 20.0, "BoundTypeR": 1, "NoInnerBC": 1, "w_numeric_type": 3,
        "RiemannSolver": 0, "Adiabatic_Index": 1.001, "Explicit_Viscosity": 0.1, "ViscConst": 0,
        "PoRho_r1": 0.01, "CFL": 0.5, "PLM": 1.0, "w_analytic_type": 0, "G_EPS": 0.05,
        "PHI_ORDER": 4, "Rho_Floor": 1.0e-6, "Cs_Floor": 1.0e-5, "Cs_Cap": 1.0, "Vel_Cap": 10.0,
        "DAMP_TIME": 1.0, "RDAMP_INNER": 0.0, "RDAMP_OUTER": 16.0, "RLogScale": 5.0,
    })
    p.update(over)
    return p


def rad_dom(num_r: int = 128, **over) -> dict:
    """Radiation-dominated alpha disk (RAD_DOM) around a point mass, fixed
    radial boundaries."""
    p = dict(_BASE)
    p.update({
        "InitialDataType": 5, "GravMassType": 1, "MassRatio": 0.0, "NumR": num_r, "ng": 2,
        "R_Min": 1.0, "R_Max": 20.0, "BoundTypeR": 0, "w_numeric_type": 0, "RiemannSolver": 1,
        "Explicit_Viscosity": 0.1, "ViscConst": 0, "PoRho_r1": 0.01, "CFL": 0.4,
        "w_analytic_type": 1, "Rho_Floor": 1.0e-6, "Cs_Floor": 1.0e-5, "Cs_Cap": 10.0,
        "Vel_Cap": 10.0, "RLogScale": 1.0,
    })
    p.update(over)
    return p


def middle(num_r: int = 128, **over) -> dict:
    """Alpha disk with a central cavity (MIDDLE) around a point mass, outflow
    radial boundary and an outer damping zone."""
    p = dict(_BASE)
    p.update({
        "InitialDataType": 6, "GravMassType": 1, "MassRatio": 0.0, "NumR": num_r, "ng": 2,
        "R_Min": 0.5, "R_Max": 10.0, "BoundTypeR": 1, "NoInnerBC": 0, "w_numeric_type": 0,
        "RiemannSolver": 0, "Explicit_Viscosity": 0.1, "ViscConst": 0, "PoRho_r1": 0.01,
        "CFL": 0.4, "w_analytic_type": 1, "Rho_Floor": 1.0e-6, "Cs_Floor": 1.0e-5,
        "Cs_Cap": 1.0, "Vel_Cap": 10.0, "DAMP_TIME": 1.0, "RDAMP_INNER": 0.0, "RDAMP_OUTER": 8.0,
        "RLogScale": 1.0,
    })
    p.update(over)
    return p


WORKLOADS = {
    "gresho": gresho,
    "kepler_ring": kepler_ring,
    "circumbinary": circumbinary,
    "shear": shear_test,
    "sstest": sstest,
    "vortex": vortex_test,
    "torus": torus_2d,
    "torus3d": torus_3d,
    "milos_macfadyen": milos_macfadyen,
    "rad_dom": rad_dom,
    "middle": middle,
}


def _fmt(v) -> str:
    if isinstance(v, bool):
        return str(int(v))
    if isinstance(v, int):
        return str(v)
    return repr(float(v))


def parfile_text(p: dict) -> str:
    """Render a parameter dict as parfile text (one `key value` per line)."""
    lines = ["//Disco Parameter File//"]
    for k in _KEYS:
        lines.append(f"{k} {_fmt(p[k])}")
    for k, v in p.items():
        if k not in _KEYS:
            lines.append(f"{k} {_fmt(v)}")
    return "\n".join(lines) + "\n"


def write_parfile(p: dict, path) -> str:
    with open(path, "w") as f:
        f.write(parfile_text(p))
    return str(path)
