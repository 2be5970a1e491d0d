"""Initial data of the benchmark configurations (host side, numpy).

Each generator returns the conserved state on the valid cells of the domain
as a float64 array of shape (NVAR, nz, ny, nx) (component planes outermost,
i fastest: the Array4 layout), before CAMR::initData's epilogue
(enforce_consistent_e + computeTemp), which the level driver applies.

State layout (Source/Utils/IndexDefines.H:17-83): URHO 0, UMX 1, UMY 2, UMZ 3,
UEDEN 4, UEINT 5, UTEMP 6, UFS 7..9.
"""
import numpy as np

NVAR = 10
URHO, UMX, UMY, UMZ, UEDEN, UEINT, UTEMP, UFS = 0, 1, 2, 3, 4, 5, 6, 7


def cell_centres(n, prob_lo=(0.0, 0.0, 0.0), dx=None, lo=(0, 0, 0)):
    """x, y, z of cell centres as prob_lo + (i + 0.5)*dx (Exec/Sod/prob.H:24)."""
    out = []
    for d in range(3):
        i = np.arange(lo[d], lo[d] + n[d], dtype=np.float64)
        out.append(prob_lo[d] + (i + 0.5) * dx[d])
    return out


def sod(n, dx, prob_lo=(0.0, 0.0, 0.0), direction=0, gamma=1.4, p_l=1.0, p_r=0.1,
        rho_l=1.0, rho_r=0.125, u_l=0.0, u_r=0.0, x0=0.5):
    """Sod shock tube, CAMR_initdata of Exec/Sod/prob.H:15-107 (prob.type = direction)."""
    s = np.zeros((NVAR, n[2], n[1], n[0]))
    xs = cell_centres(n, prob_lo, dx)
    x = xs[direction]
    left = x < x0
    shape = [1, 1, 1]
    shape[2 - direction] = n[direction]
    left = left.reshape(shape)
    Pt = np.where(left, p_l, p_r)
    rhot = np.where(left, rho_l, rho_r)
    ut = np.where(left, u_l, u_r)
    full = (n[2], n[1], n[0])
    Pt, rhot, ut = (np.broadcast_to(a, full) for a in (Pt, rhot, ut))
    s[URHO] = rhot
    mom = [UMX, UMY, UMY][direction]  # prob.type 2 writes UMY, as the reference does
    s[mom] = rhot * ut
    et = Pt / (gamma - 1.0)
    s[UEINT] = et
    s[UEDEN] = et + 0.5 * rhot * ut * ut
    s[UTEMP] = 0.0
    s[UFS] = 1.0 * s[URHO]
    s[UFS + 1] = 0.0 * s[URHO]
    s[UFS + 2] = 0.0 * s[URHO]
    return s


def blobs(n, dx, prob_lo=(0.0, 0.0, 0.0), gamma=1.4, nblobs=16, seed=1, p_blob=10.0,
          r_min=0.03, r_max=0.08, amp=0.1, p0=1.0, lo=(0, 0, 0), vel=None,
          domain_len=None):
    """Smooth periodic density with seeded spherical overpressure blobs.

    rho = 1 + amp*sin(2 pi x) sin(2 pi y) sin(2 pi z), p = p0, zero velocity,
    p = p_blob inside each blob (periodic distance to the centre < radius).
    Blob draws from numpy's PCG64 generator seeded with `seed`: per blob the
    centre (x, y, z) then the radius.  `lo` offsets the cell indices (a box
    of a finer level, with `domain_len` the periodic domain's length); `vel`
    adds a uniform velocity (u, v, w).
    """
    x, y, z = cell_centres(n, prob_lo, dx, lo)
    X = x[None, None, :]
    Y = y[None, :, None]
    Z = z[:, None, None]
    rho = 1.0 + amp * np.sin(2 * np.pi * X) * np.sin(2 * np.pi * Y) * np.sin(2 * np.pi * Z)
    p = np.full((n[2], n[1], n[0]), p0)
    rng = np.random.default_rng(seed)
    L = list(domain_len) if domain_len is not None else [n[d] * dx[d] for d in range(3)]
    for _ in range(nblobs):
        c = rng.uniform(0.0, 1.0, size=3) * np.array(L) + np.array(prob_lo)
        r = rng.uniform(r_min, r_max)
        dxs = []
        for d, arr in enumerate((X, Y, Z)):
            dd = np.abs(arr - c[d])
            dd = np.minimum(dd, L[d] - dd)
            dxs.append(dd)
        inside = dxs[0] ** 2 + dxs[1] ** 2 + dxs[2] ** 2 < r * r
        p = np.where(inside, p_blob, p)
    s = np.zeros((NVAR, n[2], n[1], n[0]))
    s[URHO] = rho
    et = p / (gamma - 1.0)
    s[UEINT] = et
    s[UEDEN] = et
    if vel is not None:
        for d in range(3):
            s[UMX + d] = rho * vel[d]
        s[UEDEN] = et + 0.5 * rho * (vel[0] ** 2 + vel[1] ** 2 + vel[2] ** 2)
    s[UFS] = 1.0 * rho
    s[UFS + 1] = 0.0 * rho
    s[UFS + 2] = 0.0 * rho
    return s


def random_smooth(n, seed=0, amp=0.2, vel=0.3, gamma=1.4):
    """Seeded smooth random state with non-zero velocities and species mix.

    Used by parity tests: every field is a sum of a few random Fourier modes,
    so slopes, limiters and Riemann branches take many different paths.
    """
    rng = np.random.default_rng(seed)
    grids = np.meshgrid(*(np.arange(n[d]) / n[d] for d in (2, 1, 0)), indexing="ij")
    Z, Y, X = grids

    def field(a):
        f = np.zeros((n[2], n[1], n[0]))
        for _ in range(3):
            k = rng.integers(1, 4, size=3)
            ph = rng.uniform(0, 2 * np.pi, size=3)
            f += a * np.sin(2 * np.pi * k[0] * X + ph[0]) * np.sin(2 * np.pi * k[1] * Y + ph[1]) \
                * np.sin(2 * np.pi * k[2] * Z + ph[2])
        return f

    rho = 1.0 + field(amp) + 0.5 * amp * rng.uniform(-1, 1, size=(n[2], n[1], n[0]))
    p = 1.0 + field(2 * amp) + amp * rng.uniform(-1, 1, size=(n[2], n[1], n[0]))
    # a few sharp jumps so that flattening and the shock branches fire
    jump = rng.uniform(0, 1, size=(n[2], n[1], n[0])) < 0.05
    p = np.where(jump, p * 8.0, p)
    u = [field(vel) for _ in range(3)]
    y0 = 0.6 + field(0.1)
    y1 = 0.3 - 0.5 * field(0.1)
    y2 = 1.0 - y0 - y1
    s = np.zeros((NVAR, n[2], n[1], n[0]))
    s[URHO] = rho
    for d in range(3):
        s[UMX + d] = rho * u[d]
    ke = 0.5 * rho * (u[0] ** 2 + u[1] ** 2 + u[2] ** 2)
    s[UEINT] = p / (gamma - 1.0)
    s[UEDEN] = s[UEINT] + ke
    s[UFS] = rho * y0
    s[UFS + 1] = rho * y1
    s[UFS + 2] = rho * y2
    return s


def amr_box_list(nbox=350, fine_n=512, sizes=(16, 24, 32, 48, 64), seed=7, nblobs=16,
                 blob_seed=1, align=8, near_tries=400, far_tries=4000):
    """Synthetic fine-level box list of the two-level configuration.

    Each box's per-dimension sizes are drawn uniformly from `sizes`; the box
    is then placed without overlap on the fine index space (fine_n^3,
    refinement ratio 2 of the base level) at an `align`-aligned corner:
    first near one of the overpressure blobs of the base data (where the
    flow has its gradients), and if no free place turns up there, anywhere
    in the domain.  A drawn size is kept, never redrawn, so the list has the
    size distribution the configuration states (expected volume per box
    mean(sizes)^3, 350 x 36.8^3 = 17.4M cells).  Returns a list of (lo, hi)
    integer triples.  The reference builds its boxes with AMReX's clusterer,
    which is not available here; this list stands in for it with the same
    box-size statistics.
    """
    rng = np.random.default_rng(seed)
    brng = np.random.default_rng(blob_seed)
    centres = []
    for _ in range(nblobs):
        c = brng.uniform(0.0, 1.0, size=3)
        brng.uniform(0.03, 0.08)
        centres.append(c * fine_n)
    occ = np.zeros((fine_n // align,) * 3, dtype=bool)
    boxes = []

    def place(lo, sz):
        lo = np.clip(lo, 0, fine_n - sz)
        lo = (lo // align) * align
        a = lo // align
        b = (lo + sz + align - 1) // align
        if occ[a[0]:b[0], a[1]:b[1], a[2]:b[2]].any():
            return False
        occ[a[0]:b[0], a[1]:b[1], a[2]:b[2]] = True
        boxes.append((tuple(int(v) for v in lo), tuple(int(v) for v in lo + sz - 1)))
        return True

    for _ in range(nbox):
        sz = rng.choice(sizes, size=3)
        done = False
        for _t in range(near_tries):
            c = centres[rng.integers(len(centres))] + rng.normal(0.0, fine_n * 0.08, size=3)
            if place(np.floor((c - sz / 2) / align).astype(int) * align, sz):
                done = True
                break
        if not done:
            for _t in range(far_tries):
                if place(rng.integers(0, fine_n - sz + 1, size=3), sz):
                    break
    return boxes


def amr_initial(n0, boxes, vel=(0.4, -0.3, 0.2), **kw):
    """Two-level initial data of a periodic unit cube: the base level (n0
    cells per side) and the fine boxes (refinement ratio 2) sampled from the
    same `blobs` field at their own cell centres.  boxes: (lo, hi) fine
    index triples.  Returns (S0, S1) with S1 the boxes' states back to back,
    flattened."""
    dx0 = tuple(1.0 / v for v in n0)
    S0 = blobs(n0, dx0, vel=vel, **kw)
    dx1 = tuple(0.5 / v for v in n0)
    parts = []
    for lo, hi in boxes:
        nb = tuple(hi[d] - lo[d] + 1 for d in range(3))
        parts.append(blobs(nb, dx1, lo=tuple(lo), vel=vel, domain_len=(1.0, 1.0, 1.0),
                           **kw).ravel())
    S1 = np.concatenate(parts) if parts else np.zeros(0)
    return S0, S1


def grf_blast(n, seed=3, corr=0.1, amp=0.05, p_blast=20.0, r_blast=0.05, gamma=1.4):
    """Adjoint configuration initial data on the periodic unit cube:
    rho = 1 + amp * g with g a Gaussian random field (white noise from
    numpy's PCG64 seeded with `seed`, filtered in Fourier space by a Gaussian
    kernel exp(-|x|^2 / (2 corr^2)), normalised to zero mean and unit
    variance), p = 1, zero velocity, and a centred blast p = p_blast for
    r < r_blast.  Species (1, 0, 0).  Returns (state, r) with r the distance
    of each cell centre from the centre."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((n[2], n[1], n[0]))
    kz = np.fft.fftfreq(n[2]) * n[2]
    ky = np.fft.fftfreq(n[1]) * n[1]
    kx = np.fft.fftfreq(n[0]) * n[0]
    K2 = kz[:, None, None] ** 2 + ky[None, :, None] ** 2 + kx[None, None, :] ** 2
    g = np.real(np.fft.ifftn(np.fft.fftn(w) * np.exp(-2.0 * np.pi ** 2 * corr ** 2 * K2)))
    g = (g - g.mean()) / g.std()
    x, y, z = cell_centres(n, dx=tuple(1.0 / v for v in n))
    r = np.sqrt((x[None, None, :] - 0.5) ** 2 + (y[None, :, None] - 0.5) ** 2 +
                (z[:, None, None] - 0.5) ** 2)
    rho = 1.0 + amp * g
    p = np.where(r < r_blast, p_blast, 1.0)
    s = np.zeros((NVAR, n[2], n[1], n[0]))
    s[URHO] = rho
    s[UEINT] = p / (gamma - 1.0)
    s[UEDEN] = s[UEINT]
    s[UFS] = rho
    return s, r


def sod_sphere(n, dx, geo, p_l=1.0, p_r=0.1, rho_l=1.0, rho_r=0.125, x0=0.5):
    """Sod states (x < x0 left) with a rigid sphere: CAMR_initdata of
    Exec/SodPlusSphere/prob.H:12-47 on every cell, then EB_set_covered
    (covered cells zero).  geo: the sphere geometry over a region containing
    the domain [0, n-1]."""
    from .eb_geometry import set_covered
    s = sod(n, dx, p_l=p_l, p_r=p_r, rho_l=rho_l, rho_r=rho_r, x0=x0)
    return set_covered(s, geo)
