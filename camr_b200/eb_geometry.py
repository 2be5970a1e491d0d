"""Embedded-boundary geometry of a rigid sphere on a uniform grid (host side).

Produces, on a cell region G = [lo, hi] (inclusive), the arrays the EB
hydro reads, in Array4 layout (components outermost, i fastest):

    flag   uint32 (nz, ny, nx): bits 0-1 the cell type (0 regular, 1 cut,
           3 covered), bit 2 + (di+1) + 3 (dj+1) + 9 (dk+1) set when the cell
           is connected to its neighbour (di, dj, dk) (the cell itself
           included)
    vfrac  (nz, ny, nx)        fluid volume fraction
    ap[d]  face area fractions on surroundingNodes(G, d)
    fc[d]  (2, ...) face-centroid offsets of the fluid part of each face in
           its two transverse directions (x before y before z), in cell
           widths from the face centre
    cent   (3, nz, ny, nx)     cell-centroid offsets

The fluid is outside the sphere (an obstacle).  Cut cells and faces are
integrated by sampling ns points per direction; cells with a volume fraction
under `small_vfrac` are made covered and their faces closed.  Connectivity:
face neighbours are connected when the shared face is open; edge and corner
neighbours when some path of unit steps through face-connected cells
reaches them.  The reference builds these with AMReX's EB2 from the same
implicit function (Exec/SodPlusSphere: sphere, fluid outside); AMReX is not
available here, so the moments are this module's own integration.
"""
import itertools

import numpy as np

REGULAR, CUT, COVERED = 0, 1, 3


def _bit(di, dj, dk):
    return 2 + (di + 1) + 3 * (dj + 1) + 9 * (dk + 1)


def sphere_geometry(lo, hi, dx, prob_lo=(0.0, 0.0, 0.0), center=(0.5, 0.5, 0.5), radius=0.15,
                    ns=16, small_vfrac=1e-4):
    lo = np.array(lo)
    hi = np.array(hi)
    # compute on G grown by one cell so that connectivity to the neighbours
    # outside G is known, then crop
    glo, ghi = lo - 1, hi + 1
    n = ghi - glo + 1
    c = np.array(center, dtype=np.float64)
    pl = np.array(prob_lo, dtype=np.float64)
    h = float(dx)
    sub = (np.arange(ns) + 0.5) / ns - 0.5  # sample offsets in cell widths

    idx = [np.arange(glo[d], ghi[d] + 1) for d in range(3)]
    cen = [pl[d] + (idx[d] + 0.5) * h for d in range(3)]
    X = cen[0][None, None, :]
    Y = cen[1][None, :, None]
    Z = cen[2][:, None, None]
    dist = np.sqrt((X - c[0]) ** 2 + (Y - c[1]) ** 2 + (Z - c[2]) ** 2)
    half_diag = np.sqrt(3.0) / 2.0 * h
    vfrac = np.where(dist - radius > half_diag, 1.0, 0.0)
    cent = np.zeros((3,) + vfrac.shape)
    cut = np.abs(dist - radius) <= half_diag
    ks, js, is_ = np.nonzero(cut)
    if len(ks):
        oz, oy, ox = np.meshgrid(sub, sub, sub, indexing="ij")
        off = np.stack([ox.ravel(), oy.ravel(), oz.ravel()])  # (3, ns^3)
        for a in range(0, len(ks), 4096):
            sl = slice(a, a + 4096)
            px = cen[0][is_[sl]][:, None] + off[0][None, :] * h
            py = cen[1][js[sl]][:, None] + off[1][None, :] * h
            pz = cen[2][ks[sl]][:, None] + off[2][None, :] * h
            fluid = (px - c[0]) ** 2 + (py - c[1]) ** 2 + (pz - c[2]) ** 2 >= radius ** 2
            cnt = fluid.sum(axis=1)
            vf = cnt / off.shape[1]
            vfrac[ks[sl], js[sl], is_[sl]] = vf
            with np.errstate(invalid="ignore", divide="ignore"):
                for d in range(3):
                    m = (fluid * off[d][None, :]).sum(axis=1) / np.maximum(cnt, 1)
                    cent[d, ks[sl], js[sl], is_[sl]] = np.where(cnt > 0, m, 0.0)
    covered = vfrac < small_vfrac
    vfrac = np.where(covered, 0.0, vfrac)
    cent[:, covered] = 0.0

    # faces
    ap, fc = [], []
    sub2a, sub2b = np.meshgrid(sub, sub, indexing="ij")
    for d in range(3):
        shape = list(vfrac.shape)
        shape[2 - d] += 1
        fidx = [idx[e] if e != d else np.arange(glo[d], ghi[d] + 2) for e in range(3)]
        fpos = [pl[e] + (fidx[e] + (0.0 if e == d else 0.5)) * h for e in range(3)]
        FX = fpos[0][None, None, :]
        FY = fpos[1][None, :, None]
        FZ = fpos[2][:, None, None]
        fd = np.sqrt((FX - c[0]) ** 2 + (FY - c[1]) ** 2 + (FZ - c[2]) ** 2)
        fd = np.broadcast_to(fd, shape)
        hd2 = np.sqrt(2.0) / 2.0 * h
        a_ = np.where(fd - radius > hd2, 1.0, 0.0)
        f_ = np.zeros((2,) + tuple(shape))
        t = [e for e in range(3) if e != d]
        fcut = np.abs(fd - radius) <= hd2
        ks, js, is_ = np.nonzero(fcut)
        if len(ks):
            o1 = sub2a.ravel()
            o2 = sub2b.ravel()
            for a in range(0, len(ks), 8192):
                sl = slice(a, a + 8192)
                p = [fpos[0][is_[sl]][:, None] * np.ones((1, len(o1))),
                     fpos[1][js[sl]][:, None] * np.ones((1, len(o1))),
                     fpos[2][ks[sl]][:, None] * np.ones((1, len(o1)))]
                p[t[0]] = p[t[0]] + o1[None, :] * h
                p[t[1]] = p[t[1]] + o2[None, :] * h
                fluid = (p[0] - c[0]) ** 2 + (p[1] - c[1]) ** 2 + (p[2] - c[2]) ** 2 >= radius ** 2
                cnt = fluid.sum(axis=1)
                a_[ks[sl], js[sl], is_[sl]] = cnt / len(o1)
                for q, o in enumerate((o1, o2)):
                    m = (fluid * o[None, :]).sum(axis=1) / np.maximum(cnt, 1)
                    f_[q, ks[sl], js[sl], is_[sl]] = np.where(cnt > 0, m, 0.0)
        # faces of covered cells are closed
        cov = covered
        lo_cov = np.zeros(shape, dtype=bool)
        hi_cov = np.zeros(shape, dtype=bool)
        ax = 2 - d
        sl_lo = [slice(None)] * 3
        sl_hi = [slice(None)] * 3
        sl_lo[ax] = slice(1, None)   # face f has cell f-1 on its low side
        sl_hi[ax] = slice(0, -1)     # and cell f on its high side
        lo_cov[tuple(sl_lo)] = cov
        hi_cov[tuple(sl_hi)] = cov
        closed = lo_cov | hi_cov
        a_ = np.where(closed, 0.0, a_)
        f_[:, closed] = 0.0
        ap.append(a_)
        fc.append(f_)

    # flags and connectivity
    regular = (vfrac == 1.0)
    for d in range(3):
        ax = 2 - d
        a_ = ap[d]
        s0 = [slice(None)] * 3
        s1 = [slice(None)] * 3
        s0[ax] = slice(0, -1)
        s1[ax] = slice(1, None)
        regular &= (a_[tuple(s0)] == 1.0) & (a_[tuple(s1)] == 1.0)
    typ = np.where(covered, COVERED, np.where(regular, REGULAR, CUT)).astype(np.uint32)

    def face_open(d, sign):
        """open[k,j,i]: the face between cell and its neighbour at sign in d."""
        ax = 2 - d
        a_ = ap[d]
        s = [slice(None)] * 3
        s[ax] = slice(1, None) if sign > 0 else slice(0, -1)
        return a_[tuple(s)] > 0.0

    def shifted(arr, off, fill):
        """arr at cell + off (di, dj, dk), `fill` outside."""
        out = np.full(arr.shape, fill, dtype=arr.dtype)
        src = []
        dst = []
        for ax, o in zip((2, 1, 0), off):
            nlen = arr.shape[ax]
            if o >= 0:
                src.append(slice(o, nlen))
                dst.append(slice(0, nlen - o))
            else:
                src.append(slice(0, nlen + o))
                dst.append(slice(-o, nlen))
        s_src = [None] * 3
        s_dst = [None] * 3
        for q, ax in enumerate((2, 1, 0)):
            s_src[ax] = src[q]
            s_dst[ax] = dst[q]
        out[tuple(s_dst)] = arr[tuple(s_src)]
        return out

    notcov = ~covered
    # step[d][sign]: cell -> neighbour in d at sign is face-connected
    step = {}
    for d in range(3):
        for sgn in (-1, 1):
            off = [0, 0, 0]
            off[d] = sgn
            step[(d, sgn)] = face_open(d, sgn) & notcov & shifted(notcov, off, False)
    flag = typ.copy()
    for di, dj, dk in itertools.product((-1, 0, 1), repeat=3):
        o = (di, dj, dk)
        if o == (0, 0, 0):
            conn = notcov
        else:
            moves = [(d, o[d]) for d in range(3) if o[d] != 0]
            conn = np.zeros(vfrac.shape, dtype=bool)
            for perm in itertools.permutations(moves):
                ok = notcov.copy()
                pos = [0, 0, 0]
                for d, sgn in perm:
                    ok &= shifted(step[(d, sgn)], pos, False)
                    pos[d] += sgn
                conn |= ok
        flag |= (conn.astype(np.uint32) << np.uint32(_bit(*o)))

    crop = (slice(1, -1),) * 3
    out = {"lo": tuple(int(v) for v in lo), "hi": tuple(int(v) for v in hi),
           "flag": np.ascontiguousarray(flag[crop]),
           "vfrac": np.ascontiguousarray(vfrac[crop]),
           "cent": np.ascontiguousarray(cent[(slice(None),) + crop])}
    out["ap"], out["fc"] = [], []
    for d in range(3):
        ax = 2 - d
        s = [slice(1, -1)] * 3
        s[ax] = slice(1, -1)  # faces lo..hi+1 of G: drop the outermost face on each side
        out["ap"].append(np.ascontiguousarray(ap[d][tuple(s)]))
        out["fc"].append(np.ascontiguousarray(fc[d][(slice(None),) + tuple(s)]))
    return out


def set_covered(state, geo, lo=(0, 0, 0)):
    """EB_set_covered(S, 0) (Source/CAMR.cpp:418-420): zero every component
    of the covered cells of state (NVAR, nz, ny, nx) whose first cell is
    `lo`; geo covers a region containing it."""
    n = state.shape[1:]
    off = [lo[d] - geo["lo"][d] for d in range(3)]
    flag = geo["flag"][off[2]:off[2] + n[0], off[1]:off[1] + n[1], off[0]:off[0] + n[2]]
    state[:, (flag & 3) == COVERED] = 0.0
    return state
