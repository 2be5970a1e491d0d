"""Taped FP64 CPU version of the MOL level step, for the adjoint tests.

A restatement of the reference's MOL path on a periodic uniform level
(CAMR_advance with do_mol = 1, Source/CAMR_advance.cpp:124-136, plus
post_timestep's clean_state) in torch float64 tensor operations, so that
torch.autograd records the tape of one or more steps and gives the
reference gradient the hand-written adjoint is checked against.  Branches
are written with torch.where in the reference's order, so the recorded
derivative takes the branch the forward value took, as the adjoint does.

Pieces (reference lines): clean_state = normalize_species + computeTemp
(Source/CAMR.cpp:866-908, :1141-1185, Utils/CAMR_reset_internal_e.H:94-119);
hydro_ctoprim (Hydro/Hydro_ctoprim.H:11-101); mol_slope_{x,y,z}
(MOL/MOL_hydro_K.H:11-255); mol_riemann edge states (MOL/MOL_riemann_K.H);
hydro_cmpflx + riemannus (Hydro_cmpflx.H:153-311, Hydro_riemann.H:8-173);
nodal divu, artificial viscosity, species flux normalisation, area scaling,
p div u and consup (Hydro_utils_K.H, hydro_artif_visc.H).
Test infrastructure only.
"""
import torch
import torch.nn.functional as F

URHO, UMX, UMY, UMZ, UEDEN, UEINT, UTEMP, UFS = 0, 1, 2, 3, 4, 5, 6, 7
NSP = 3
RU = 8.31446261815324e7
AIRMW = 26.93
NG = 4


class Par:
    def __init__(self, gamma=1.4, small=1e-8, small_dens=1e-7, small_pres=1e-200, smallu=1e-12,
                 small_num=1e-8, difmag=0.1, eta1=1.0, eta2=1e-4, small_temp=1e2):
        self.gamma, self.small, self.small_dens, self.small_pres = gamma, small, small_dens, small_pres
        self.smallu, self.small_num, self.difmag = smallu, small_num, difmag
        self.eta1, self.eta2, self.small_temp = eta1, eta2, small_temp


def hmax(a, b):
    """std::max(a, b): (a < b) ? b : a"""
    return torch.where(a < b, b, a)


def hmin(a, b):
    """std::min(a, b): (b < a) ? b : a"""
    return torch.where(b < a, b, a)


def const(x, like):
    return torch.full_like(like, x)


def clean(S, P):
    """normalize_species then reset_internal_energy + T (default flags)."""
    rho = S[URHO]
    ys = []
    for sp in range(NSP):
        a = S[UFS + sp]
        m = hmin(rho, a)
        ys.append(hmax(m, torch.zeros_like(m)))
    s = (ys[0] + ys[1]) + ys[2]
    pos = rho > 0.0
    s2 = torch.where(pos, s / rho, torch.ones_like(s))
    ys = [torch.where(pos, y / s2, y) for y in ys]
    rhoInv = 1.0 / rho
    Up, Vp, Wp = S[UMX] * rhoInv, S[UMY] * rhoInv, S[UMZ] * rhoInv
    ke = 0.5 * (Up * Up + Vp * Vp + Wp * Wp)
    eden, eint = S[UEDEN], S[UEINT]
    cvT = RU / (AIRMW * (P.gamma - 1.0)) * P.small_temp
    mf = [y * rhoInv for y in ys]
    e_small = ((mf[0] * cvT) + mf[1] * cvT) + mf[2] * cvT
    # UEDEN < 0
    eint_a = torch.where(eint < 0.0, rho * e_small, eint)
    eden_a = eint_a + rho * ke
    # UEDEN >= 0
    rho_eint = eden - rho * ke
    c1 = (rho_eint > 0.0) & (rho_eint / eden > P.eta2)
    c2 = (~c1) & (eint > 0.0)
    c3 = (~c1) & (~c2) & (eint <= 0.0)
    eint_b = torch.where(c1, rho_eint, torch.where(c3, rho * e_small, eint))
    eden_b = torch.where(c2, eint + rho * ke, eden)
    neg = eden < 0.0
    eint_n = torch.where(neg, eint_a, eint_b)
    eden_n = torch.where(neg, eden_a, eden_b)
    temp = (P.gamma - 1.0) * (eint_n * (1.0 / rho)) * AIRMW / RU
    return torch.stack([rho, S[UMX], S[UMY], S[UMZ], eden_n, eint_n, temp, ys[0], ys[1], ys[2]])


def expand(S, P):
    """expand_state on a periodic level: clean, then the periodic ghost cells."""
    C = clean(S, P)
    return F.pad(C.unsqueeze(0), (NG,) * 6, mode="circular").squeeze(0)


def ctoprim(U, P):
    rho = U[URHO]
    rhoinv = 1.0 / rho
    vx, vy, vz = U[UMX] * rhoinv, U[UMY] * rhoinv, U[UMZ] * rhoinv
    kin = 0.5 * rho * (vx * vx + vy * vy + vz * vz)
    e = torch.where((U[UEDEN] - kin) / U[UEDEN] > P.eta1, (U[UEDEN] - kin) * rhoinv,
                    U[UEINT] * rhoinv)
    p = (P.gamma - 1.0) * rho * e
    q = {"rho": rho, "u": [vx, vy, vz], "p": p, "re": e * rho,
         "y": [U[UFS + sp] * rhoinv for sp in range(NSP)]}
    q["c"] = torch.sqrt(P.gamma * p / rho)
    q["csml"] = hmax(const(P.small_num, p), P.small_num * q["c"])
    return q


AX = {0: 3, 1: 2, 2: 1}  # direction -> tensor axis of a (comp, k, j, i) state


def sh(x, d, o):
    """x shifted so that index c holds x[c + o] along direction d (periodic
    roll; only interior values are used)."""
    return torch.roll(x, shifts=-o, dims=AX[d] - 1)


def limiter(dl, dr):
    dcen = 0.5 * (dl + dr)
    dsgn = torch.copysign(torch.ones_like(dcen), dcen)
    slop = 2.0 * hmin(torch.abs(dl), torch.abs(dr))
    dlim = torch.where(dl * dr >= 0.0, slop, torch.zeros_like(slop))
    return dsgn * hmin(dlim, torch.abs(dcen))


def slopes(q, d, P):
    t1 = 1 if d == 0 else 0
    t2 = 1 if d == 2 else 2
    c = q["c"]
    rho, p, un = q["rho"], q["p"], q["u"][d]
    pm, pp = sh(p, d, -1), sh(p, d, 1)
    unm, unp = sh(un, d, -1), sh(un, d, 1)
    o = {}
    dl = 0.5 * (p - pm) / c - 0.5 * rho * (un - unm)
    dr = 0.5 * (pp - p) / c - 0.5 * rho * (unp - un)
    o["s0"] = limiter(dl, dr)
    cs2 = c * c
    dl = 0.5 * (p - pm) / c + 0.5 * rho * (un - unm)
    dr = 0.5 * (pp - p) / c + 0.5 * rho * (unp - un)
    o["s2"] = limiter(dl, dr)
    for name, t in (("s3", t1), ("s4", t2)):
        v = q["u"][t]
        o[name] = limiter(v - sh(v, d, -1), sh(v, d, 1) - v)
    re = q["re"]
    enth = (re + p) / hmax(rho, const(P.small_dens, rho))
    dl = (re - sh(re, d, -1)) - enth * (p - pm) / cs2
    dr = (sh(re, d, 1) - re) - enth * (pp - p) / cs2
    o["sre"] = limiter(dl, dr)
    o["sy"] = []
    for sp in range(NSP):
        y = q["y"][sp]
        ry = rho * y
        dl = ry - sh(rho, d, -1) * sh(y, d, -1) - y * (p - pm) / cs2
        dr = sh(rho, d, 1) * sh(y, d, 1) - ry - y * (pp - p) / cs2
        o["sy"].append(limiter(dl, dr))
    return o


def edge(q, s, d, sign, yfall, P):
    t1 = 1 if d == 0 else 0
    t2 = 1 if d == 2 else 2
    c = q["c"]
    rho = q["rho"]
    enth = (q["re"] + q["p"]) / hmax(rho, const(P.small_dens, rho))
    a = s["s0"] + s["s2"]
    p0 = q["p"] + 0.5 * a * c if sign > 0 else q["p"] - 0.5 * a * c
    e = {"p": hmax(p0, const(P.small_pres, p0))}
    if sign > 0:
        e["un"] = q["u"][d] + 0.5 * ((s["s2"] - s["s0"]) / rho)
        e["t1"] = q["u"][t1] + 0.5 * s["s3"]
        e["t2"] = q["u"][t2] + 0.5 * s["s4"]
    else:
        e["un"] = q["u"][d] - 0.5 * ((s["s2"] - s["s0"]) / rho)
        e["t1"] = q["u"][t1] - 0.5 * s["s3"]
        e["t2"] = q["u"][t2] - 0.5 * s["s4"]
    sd = []
    for sp in range(NSP):
        y = q["y"][sp]
        if sign > 0:
            sd.append(rho * y + 0.5 * (s["sy"][sp] + y * a / c))
        else:
            sd.append(rho * y - 0.5 * (s["sy"][sp] + y * a / c))
    tot = (sd[0] + sd[1]) + sd[2]
    fb = tot < P.small_dens
    e["y"] = [torch.where(fb, yfall[sp], sd[sp] / tot) for sp in range(NSP)]
    e["rho"] = hmax(tot, const(P.small_dens, tot))
    if sign > 0:
        e["re"] = q["re"] + 0.5 * (s["sre"] + enth * a / c)
    else:
        e["re"] = q["re"] - 0.5 * (s["sre"] + enth * a / c)
    return e


def riemann(l, r, cav, smallc, P):
    g = P.gamma
    sd, spr = P.small_dens, P.small_pres
    wsmall = smallc * sd
    rl = hmax(l["rho"], const(sd, cav))
    pl = hmax(l["p"], const(spr, cav))
    rr = hmax(r["rho"], const(sd, cav))
    pr = hmax(r["p"], const(spr, cav))
    ul, ur = l["un"], r["un"]
    wl = hmax(wsmall, torch.sqrt(torch.abs(g * pl * rl)))
    wr = hmax(wsmall, torch.sqrt(torch.abs(g * pr * rr)))
    pstar = ((wr * pl + wl * pr) + wl * wr * (ul - ur)) / (wl + wr)
    pstar = hmax(pstar, const(spr, cav))
    ustar = ((wl * ul + wr * ur) + (pl - pr)) / (wl + wr)
    mask = torch.abs(ustar) < P.smallu * 0.5 * (torch.abs(ul) + torch.abs(ur))
    ustar = torch.where(mask, torch.zeros_like(ustar), ustar)
    pos, negv = ustar > 0.0, ustar < 0.0

    def sel(a, b, avg):
        return torch.where(pos, a, torch.where(negv, b, avg))

    ro = sel(rl, rr, 0.5 * (rl + rr))
    uo = sel(ul, ur, 0.5 * (ul + ur))
    po = sel(pl, pr, 0.5 * (pl + pr))
    reo = sel(l["re"], r["re"], 0.5 * (l["re"] + r["re"]))
    gamco = g  # both sides carry the same gamma
    ro = hmax(ro, const(sd, ro))
    roinv = 1.0 / ro
    co = torch.sqrt(torch.abs(gamco * po * roinv))
    co = hmax(smallc, co)
    co2inv = 1.0 / (co * co)
    drho = (pstar - po) * co2inv
    rstar = hmax(const(sd, ro), ro + drho)
    entho = (reo + po) * roinv * co2inv
    estar = reo + (pstar - po) * entho
    cstar = torch.sqrt(torch.abs(gamco * pstar / rstar))
    cstar = hmax(cstar, smallc)
    sgnm = torch.where(ustar < 0.0, -torch.ones_like(ustar), torch.ones_like(ustar))
    spout = co - sgnm * uo
    spin = cstar - sgnm * ustar
    ushock = 0.5 * (spin + spout)
    shock = pstar - po > 0.0
    spin = torch.where(shock, ushock, spin)
    spout = torch.where(shock, ushock, spout)
    scr = torch.where(spout - spin == 0.0, P.small * cav, spout - spin)
    frac = (1.0 + (spout + spin) / scr) * 0.5
    frac = hmax(torch.zeros_like(frac), hmin(torch.ones_like(frac), frac))
    iv1 = torch.where(pos, l["t1"], r["t1"])
    iv2 = torch.where(pos, l["t2"], r["t2"])
    z = ustar == 0.0
    iv1 = torch.where(z, 0.5 * (l["t1"] + r["t1"]), iv1)
    iv2 = torch.where(z, 0.5 * (l["t2"] + r["t2"]), iv2)
    rho_gd = frac * rstar + (1.0 - frac) * ro
    iu = frac * ustar + (1.0 - frac) * uo
    gdp = frac * pstar + (1.0 - frac) * po
    re_gd = frac * estar + (1.0 - frac) * reo
    m = spout < 0.0
    rho_gd, iu = torch.where(m, ro, rho_gd), torch.where(m, uo, iu)
    gdp, re_gd = torch.where(m, po, gdp), torch.where(m, reo, re_gd)
    m = spin >= 0.0
    rho_gd, iu = torch.where(m, rstar, rho_gd), torch.where(m, ustar, iu)
    gdp, re_gd = torch.where(m, pstar, gdp), torch.where(m, estar, re_gd)
    gdp = hmax(gdp, const(spr, gdp))
    frho = rho_gd * iu
    out = {"rho": frho, "un": frho * iu + gdp, "ut1": frho * iv1, "ut2": frho * iv2,
           "eint": iu * re_gd, "qun": iu, "qp": gdp, "ustar": ustar}
    rhoetot = re_gd + 0.5 * rho_gd * (iu * iu + iv1 * iv1 + iv2 * iv2)
    out["eden"] = iu * (rhoetot + gdp)
    return out


def divu_nodes(q, dx):
    """Nodal div u at node (k, j, i) = low corner of cell (k, j, i)."""
    u, v, w = q["u"]

    def R(x, dk, dj, di):
        return torch.roll(x, shifts=(dk, dj, di), dims=(0, 1, 2))

    def corner(x, ax):
        # sum over the 4 cells at the node's high index along ax minus the 4 at low
        tot = None
        for dk in (0, 1):
            for dj in (0, 1):
                for di in (0, 1):
                    o = (dk, dj, di)
                    hi = o[ax] == 0
                    term = R(x, dk, dj, di)
                    term = term if hi else -term
                    tot = term if tot is None else tot + term
        return tot

    ux = 0.25 * corner(u, 2) / dx[0]
    vy = 0.25 * corner(v, 1) / dx[1]
    wz = 0.25 * corner(w, 0) / dx[2]
    return ux + vy + wz


def hydro(B, dx, P):
    """dSdt on the padded array's valid interior [NG:-NG]^3 (MOL, periodic)."""
    q = ctoprim(B, P)
    dv = divu_nodes(q, dx)
    vol = dx[0] * dx[1] * dx[2]
    areas = [dx[1] * dx[2], dx[0] * dx[2], dx[0] * dx[1]]
    flux, qf = [], []
    for d in range(3):
        s = slopes(q, d, P)
        sl = {k: (sh(v, d, -1) if k != "sy" else [sh(x, d, -1) for x in v]) for k, v in s.items()}
        ql = {"rho": sh(q["rho"], d, -1), "u": [sh(x, d, -1) for x in q["u"]],
              "p": sh(q["p"], d, -1), "re": sh(q["re"], d, -1),
              "y": [sh(x, d, -1) for x in q["y"]], "c": sh(q["c"], d, -1),
              "csml": sh(q["csml"], d, -1)}
        el = edge(ql, sl, d, +1, q["y"], P)
        er = edge(q, s, d, -1, q["y"], P)
        cav = 0.5 * (q["c"] + ql["c"])
        smallc = hmax(q["csml"], ql["csml"])
        o = riemann(el, er, cav, smallc, P)
        f = [None] * 10
        fu = 1 + d
        fv = 2 if d == 0 else 1
        fv2 = 2 if d == 2 else 3
        f[URHO], f[fu], f[fv], f[fv2] = o["rho"], o["un"], o["ut1"], o["ut2"]
        f[UEDEN], f[UEINT], f[UTEMP] = o["eden"], o["eint"], torch.zeros_like(o["rho"])
        for sp in range(NSP):
            f[UFS + sp] = torch.where(o["ustar"] > 0.0, o["rho"] * el["y"][sp],
                                      torch.where(o["ustar"] < 0.0, o["rho"] * er["y"][sp],
                                                  o["rho"] * 0.5 * (el["y"][sp] + er["y"][sp])))
        # artificial viscosity with the 4 nodes of the face
        t1 = 1 if d == 0 else 0
        t2 = 1 if d == 2 else 2
        dvs = dv + sh(dv, t1, 1) + sh(dv, t2, 1) + sh(sh(dv, t1, 1), t2, 1)
        div = P.difmag * hmin(torch.zeros_like(dvs), 0.25 * dvs)
        for n in range(10):
            if n == UTEMP:
                continue
            f[n] = f[n] + dx[d] * div * (B[n] - sh(B[n], d, -1))
        summ = (f[UFS] + f[UFS + 1]) + f[UFS + 2]
        fac = torch.where(summ != 0.0, f[URHO] / summ, torch.ones_like(summ))
        for n in range(UFS, UFS + NSP):
            f[n] = f[n] * fac
        f = [x * areas[d] for x in f]
        flux.append(f)
        qf.append((o["qp"], o["qun"]))
    vi = (slice(NG, -NG),) * 3
    ds = []
    for n in range(10):
        acc = None
        for d in range(3):
            term = flux[d][n] - sh(flux[d][n], d, 1)
            acc = term if acc is None else acc + term
        ds.append(0.0 + acc * (1.0 / vol))
    pdivu = None
    for d in range(3):
        qp, qu = qf[d]
        term = (sh(qp, d, 1) + qp) * (sh(qu, d, 1) * areas[d] - qu * areas[d])
        pdivu = term if pdivu is None else pdivu + term
    pdivu = 0.5 * pdivu / vol
    ds[UEINT] = ds[UEINT] - pdivu
    return torch.stack([x[vi] for x in ds])


def step(S, dt, dx, P, grav=True):
    """One MOL RK2 step + the end-of-step cleans (S on valid cells)."""
    vi = (slice(None),) + (slice(NG, -NG),) * 3
    S_old = clean(S, P)
    B = expand(S_old, P)
    k1 = hydro(B, dx, P)
    Sstar = B[vi] + dt * k1
    B2 = expand(Sstar, P)
    k2 = hydro(B2, dx, P)
    Snew = 0.5 * B2[vi] + 0.5 * S_old
    Snew = Snew + 0.5 * dt * k2
    Snew = clean(Snew, P)
    if grav:
        Snew = clean(Snew, P)
    return clean(Snew, P)
