"""The reference's integrated quantities (CAMR::sum_integrated_quantities,
Source/Utils/SumIQ.cpp:6-60): volume-weighted sums over the valid cells of
density, the three momenta, rho e, the kinetic energy density, rho E and
temperature (AmrLevel::volWgtSum: value x cell volume), and their drift
between two states, a conservation check reported beside the timings."""
import numpy as np

# component order of the 3-D state (Source/Utils/IndexDefines.H:46-51)
URHO, UMX, UMY, UMZ, UEDEN, UEINT, UTEMP = 0, 1, 2, 3, 4, 5, 6


def integrated_quantities(state, dx):
    """{name: volume-weighted sum} of a state (NVAR, nz, ny, nx)."""
    vol = float(dx[0]) * float(dx[1]) * float(dx[2])
    s = np.asarray(state, dtype=np.float64)
    rho = s[URHO]
    kin = 0.5 * (s[UMX] ** 2 + s[UMY] ** 2 + s[UMZ] ** 2) / rho
    out = {"mass": rho.sum(), "xmom": s[UMX].sum(), "ymom": s[UMY].sum(),
           "zmom": s[UMZ].sum(), "rho_e": s[UEINT].sum(), "kineng": kin.sum(),
           "rho_E": s[UEDEN].sum(), "Temp": s[UTEMP].sum()}
    return {k: float(v) * vol for k, v in out.items()}


def drift(before, after):
    """Relative change of mass and total energy, and the change of each
    momentum relative to the largest momentum magnitude (momentum sums may
    be near zero)."""
    rel = {k: (after[k] - before[k]) / abs(before[k]) for k in ("mass", "rho_E")}
    scale = max(abs(before[k]) for k in ("xmom", "ymom", "zmom")) or 1.0
    mom = {k: (after[k] - before[k]) / scale for k in ("xmom", "ymom", "zmom")}
    return {"mass_rel": rel["mass"], "rho_E_rel": rel["rho_E"], "momentum_rel": mom}
