"""A level whose boxes are spread over processes (one process per GPU),
advanced through the library's per-box and fab-level calls, with the ghost
cells exchanged over torch.distributed (NCCL between GPUs, gloo on CPU).

This is the multi-GPU form of the reference's single-level step
(CAMR::CAMR_advance, Source/CAMR_advance.cpp:38-164), where AMReX would
distribute the boxes of a MultiFab over MPI ranks:

* partition: the boxes ordered along a Morton space-filling curve of their
  low corners and cut into contiguous runs of about equal cell count (the
  idea of AMReX's space-filling-curve distribution map);
* ghost cells: the FillPatch of expand_state (Source/CAMR.cpp:1243-1250) and
  the FillBoundary inside clean_state (:884-908) become a plan computed
  identically on every rank: for each ghost cell of each box, the valid cell
  it takes its value from (periodic image, or past a physical boundary the
  BC map's source cell, Source/Utils/CAMR_setup.cpp:19-21) and the sign of
  each component (reflect_odd).  Cells owned on the same rank are copied
  locally; the others travel in one message per pair of ranks, in the
  plan's order on both sides;
* the time step: each rank's CFL estimate over its own boxes (camr_est_dt),
  then an all-reduce(min), as ParallelDescriptor::ReduceRealMin does
  (Source/CAMR.cpp:543), then computeNewDt on every rank.

The hydro of each box is camr_hydro_umdrv; the Saxpys of CAMR_advance are
done elementwise with one rounding per operation, in the reference's order.
"""
import ctypes as C

import numpy as np

from . import native

NVAR = native.NVAR
NG = 4
RR = 2  # refinement ratio of a two-level hierarchy


def _box_coords(lo, hi):
    """(i, j, k) of every cell of [lo, hi], i fastest, as three arrays."""
    ax = [np.arange(lo[e], hi[e] + 1, dtype=np.int64) for e in range(3)]
    K, J, I = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    return [I.ravel(), J.ravel(), K.ravel()]


def _flat(ijk, dlo, n):
    """Flat index (i fastest) of in-domain cells of a domain at dlo of size n."""
    return (ijk[0] - dlo[0]) + n[0] * ((ijk[1] - dlo[1]) + n[1] * (ijk[2] - dlo[2]))


def _wrap_flat(ijk, dlo, n):
    """Flat index of the periodic images of any cells."""
    return _flat([(ijk[e] - dlo[e]) % n[e] + dlo[e] for e in range(3)], dlo, n)


def _hierarchy_maps(cboxes, fboxes, dlo, n):
    """The checks and maps the two-level pieces share.  The coarse boxes
    must lie in the domain, be disjoint and cover it; the fine boxes must be
    aligned to the refinement ratio (lo even, hi odd), lie in the fine
    domain and be disjoint.  Returns, over the flat coarse cells: the coarse
    box holding each, its flat place in that box, and the fine box covering
    it (-1 if none)."""
    ncell = int(np.prod(n))
    dhi = [dlo[d] + n[d] - 1 for d in range(3)]
    cbox_of = np.full(ncell, -1, dtype=np.int64)
    cloc = np.full(ncell, -1, dtype=np.int64)
    for c, (lo, hi) in enumerate(cboxes):
        if any(lo[d] < dlo[d] or hi[d] > dhi[d] or hi[d] < lo[d] for d in range(3)):
            raise ValueError(f"coarse box {c} lies outside the domain or is empty")
        cell = _flat(_box_coords(lo, hi), dlo, n)
        if (cbox_of[cell] >= 0).any():
            raise ValueError(f"coarse box {c} overlaps another")
        cbox_of[cell] = c
        cloc[cell] = np.arange(cell.size)
    if (cbox_of < 0).any():
        raise ValueError("the coarse boxes do not cover the domain")
    cmap = np.full(ncell, -1, dtype=np.int64)
    for b, (lo, hi) in enumerate(fboxes):
        if any(lo[d] % RR or (hi[d] + 1) % RR or hi[d] < lo[d] for d in range(3)):
            raise ValueError(f"fine box {b} is not aligned to the refinement ratio")
        clo = [lo[d] // RR for d in range(3)]
        chi = [hi[d] // RR for d in range(3)]
        if any(clo[d] < dlo[d] or chi[d] > dhi[d] for d in range(3)):
            raise ValueError(f"fine box {b} lies outside the domain")
        cells = _flat(_box_coords(clo, chi), dlo, n)
        if (cmap[cells] >= 0).any():
            raise ValueError(f"fine box {b} overlaps another")
        cmap[cells] = b
    return cbox_of, cloc, cmap


def morton_key(lo, bits=21):
    """Interleaved bits of three non-negative integers (x lowest)."""
    key = 0
    for b in range(bits):
        for d in range(3):
            key |= ((int(lo[d]) >> b) & 1) << (3 * b + d)
    return key


def sfc_partition(boxes, nranks, dom_lo=(0, 0, 0)):
    """Owner rank of each box: boxes in Morton order of their low corners,
    cut into nranks contiguous runs of about equal cell count."""
    cells = [int(np.prod([hi[d] - lo[d] + 1 for d in range(3)])) for lo, hi in boxes]
    order = sorted(range(len(boxes)),
                   key=lambda b: morton_key([boxes[b][0][d] - dom_lo[d] for d in range(3)]))
    total = float(sum(cells))
    owner = [0] * len(boxes)
    acc = 0.0
    for b in order:
        # the rank whose share of the total this box's midpoint falls in
        mid = acc + 0.5 * cells[b]
        owner[b] = min(nranks - 1, int(mid * nranks / total))
        acc += cells[b]
    return owner


def _bc_kinds(n, phys):
    """BC kind of component n in direction d for the BC word phys: 1 ext_dir,
    2 foextrap, 3 reflect_even, 4 reflect_odd (Source/Utils/CAMR_setup.cpp:19-21)."""
    scalar = [0, 1, 2, 3, 3, 3]
    norm = [0, 1, 2, 4, 4, 4]
    tang = [0, 1, 2, 3, 3, 4]
    return scalar, norm, tang


class GhostPlan:
    """For every ghost cell (within ng) of every box: the source cell, its
    owner box, the sign of each component, and whether a physical boundary
    was crossed.  Computed from the global box list alone, so every rank
    holds the same plan."""

    def __init__(self, geom, boxes, ng=NG):
        self.ng = ng
        dlo = np.array([geom.dom_lo[d] for d in range(3)])
        dhi = np.array([geom.dom_hi[d] for d in range(3)])
        n = dhi - dlo + 1
        per = [geom.is_periodic[d] for d in range(3)]
        bclo = [geom.bc_lo[d] for d in range(3)]
        bchi = [geom.bc_hi[d] for d in range(3)]
        owner = np.full((n[2], n[1], n[0]), -1, dtype=np.int32)
        for b, (lo, hi) in enumerate(boxes):
            owner[lo[2] - dlo[2]:hi[2] - dlo[2] + 1, lo[1] - dlo[1]:hi[1] - dlo[1] + 1,
                  lo[0] - dlo[0]:hi[0] - dlo[0] + 1] = b
        scalar, normv, tangv = _bc_kinds(0, 0)
        self.entries = []
        for b, (lo, hi) in enumerate(boxes):
            lo = np.array(lo)
            hi = np.array(hi)
            glo = lo - ng
            ghi = hi + ng
            gn = ghi - glo + 1
            z, y, x = np.meshgrid(np.arange(glo[2], ghi[2] + 1), np.arange(glo[1], ghi[1] + 1),
                                  np.arange(glo[0], ghi[0] + 1), indexing="ij")
            c = [x.ravel(), y.ravel(), z.ravel()]
            inside = np.ones(c[0].shape, dtype=bool)
            for d in range(3):
                inside &= (c[d] >= lo[d]) & (c[d] <= hi[d])
            ghost = np.nonzero(~inside)[0]
            c = [v[ghost] for v in c]
            src = [v.copy() for v in c]
            physical = np.zeros(ghost.shape, dtype=bool)
            neg = np.zeros((NVAR, ghost.size), dtype=bool)
            for d in range(3):
                low = c[d] < dlo[d]
                high = c[d] > dhi[d]
                if per[d]:
                    src[d] = dlo[d] + np.mod(c[d] - dlo[d], n[d])
                    continue
                physical |= low | high
                for side, sel, word in ((0, low, bclo[d]), (1, high, bchi[d])):
                    if not sel.any():
                        continue
                    kind = scalar[word]
                    if kind in (1, 2):
                        src[d][sel] = dlo[d] if side == 0 else dhi[d]
                    else:
                        src[d][sel] = (2 * dlo[d] - c[d][sel] - 1 if side == 0
                                       else 2 * dhi[d] - c[d][sel] + 1)
                    for comp in range(NVAR):
                        if 1 <= comp <= 3:
                            kk = normv[word] if comp - 1 == d else tangv[word]
                        else:
                            kk = scalar[word]
                        if kk == 4:
                            neg[comp, sel] ^= True
            own = owner[src[2] - dlo[2], src[1] - dlo[1], src[0] - dlo[0]]
            dst_flat = ((c[2] - glo[2]) * gn[1] + (c[1] - glo[1])) * gn[0] + (c[0] - glo[0])
            self.entries.append({"dst_flat": dst_flat, "src": src, "owner": own,
                                 "physical": physical, "neg": neg})
        self.boxes = boxes

    def src_flat(self, e, sel, src_ng):
        """Flat indices of the source cells e[sel] in their owners' tensors
        that cover each owner box grown by src_ng."""
        out = np.empty(int(sel.sum()), dtype=np.int64)
        own = e["owner"][sel]
        s = [v[sel] for v in e["src"]]
        for o in np.unique(own):
            m = own == o
            lo, hi = self.boxes[o]
            glo = [lo[d] - src_ng for d in range(3)]
            gn = [hi[d] - lo[d] + 1 + 2 * src_ng for d in range(3)]
            out[m] = ((s[2][m] - glo[2]) * gn[1] + (s[1][m] - glo[1])) * gn[0] + (s[0][m] - glo[0])
        return out


class Exchange:
    """The ghost-cell fills of a GhostPlan for this rank: local copies and one
    message per peer rank, over torch.distributed (pg None: one process)."""

    def __init__(self, plan, owner_rank, rank, nranks, device, pg=None):
        import torch
        self.plan = plan
        self.rank = rank
        self.nranks = nranks
        self.pg = pg
        self.owner_rank = np.asarray(owner_rank)
        self.device = device
        self.torch = torch
        self._cache = {}

    def _select(self, e, kind):
        if kind == "all":
            sel = e["owner"] >= 0
        elif kind == "interior":
            sel = (e["owner"] >= 0) & ~e["physical"]
        else:
            raise ValueError(kind)
        return sel

    def _groups(self, kind, src_ng):
        """Per (dst box on this rank, src box): index tensors for local
        copies; per peer: the cells to send (src box, index) and to receive
        (dst box, index, sign), in the plan's order."""
        key = (kind, src_ng)
        if key in self._cache:
            return self._cache[key]
        T = self.torch
        dev = self.device
        local, send, recv = [], {}, {}
        for b, e in enumerate(self.plan.entries):
            sel = self._select(e, kind)
            if not sel.any():
                continue
            own = e["owner"][sel]
            sflat = self.plan.src_flat(e, sel, src_ng)
            dflat = e["dst_flat"][sel]
            neg = e["neg"][:, sel]
            orank = self.owner_rank[own]
            brank = self.owner_rank[b]
            for o in np.unique(own):
                m = own == o
                r_src = self.owner_rank[o]
                if r_src == self.rank and brank == self.rank:
                    local.append((int(b), int(o), T.as_tensor(sflat[m], device=dev),
                                  T.as_tensor(dflat[m], device=dev),
                                  T.as_tensor(neg[:, m], device=dev)))
            if brank == self.rank:
                for r in np.unique(orank):
                    if r == self.rank:
                        continue
                    m = orank == r
                    recv.setdefault(int(r), []).append(
                        (int(b), T.as_tensor(dflat[m], device=dev),
                         T.as_tensor(neg[:, m], device=dev)))
            else:
                m = orank == self.rank
                if m.any():
                    # cells of this rank's boxes that box b (elsewhere) needs,
                    # in the plan's order
                    send.setdefault(int(brank), []).append(
                        (T.as_tensor(own[m].astype(np.int64), device=dev),
                         T.as_tensor(sflat[m], device=dev)))
        self._cache[key] = (local, send, recv)
        return self._cache[key]

    def fill(self, src, dst, kind="all", src_ng=0):
        """Ghost cells of the dst tensors (this rank's boxes, each covering
        its box grown by ng) from the valid cells of the src tensors (each
        covering its box grown by src_ng).  src / dst: dicts box -> tensor
        (NVAR, ...)."""
        T = self.torch
        local, send, recv = self._groups(kind, src_ng)
        for b, o, sidx, didx, neg in local:
            v = src[o].reshape(NVAR, -1)[:, sidx]
            dst[b].reshape(NVAR, -1)[:, didx] = T.where(neg, -v, v)
        if self.pg is None or self.nranks == 1:
            return
        dist = self.pg
        ops, bufs = [], {}
        for r, items in sorted(send.items()):
            parts = []
            for own, sidx in items:
                vals = T.empty((NVAR, sidx.numel()), dtype=T.float64, device=self.device)
                for o in T.unique(own).tolist():
                    m = own == o
                    vals[:, m] = src[o].reshape(NVAR, -1)[:, sidx[m]]
                parts.append(vals)
            buf = T.cat(parts, dim=1).contiguous()
            ops.append(dist.isend(buf, dst=r))
            bufs[("s", r)] = buf
        for r, items in sorted(recv.items()):
            cnt = sum(int(d.numel()) for _, d, _ in items)
            buf = T.empty((NVAR, cnt), dtype=T.float64, device=self.device)
            ops.append(dist.irecv(buf, src=r))
            bufs[("r", r)] = buf
        for op in ops:
            op.wait()
        for r, items in sorted(recv.items()):
            buf = bufs[("r", r)]
            at = 0
            for b, didx, neg in items:
                k = didx.numel()
                v = buf[:, at:at + k]
                dst[b].reshape(NVAR, -1)[:, didx] = T.where(neg, -v, v)
                at += k

    def zero_physical(self, dst):
        """Ghost cells past a physical boundary set to zero (the ghosts of
        sources_for_hydro that no FillBoundary reaches)."""
        for b, e in enumerate(self.plan.entries):
            if self.owner_rank[b] != self.rank:
                continue
            sel = e["physical"] | (e["owner"] < 0)
            if sel.any():
                idx = self.torch.as_tensor(e["dst_flat"][sel], device=self.device)
                dst[b].reshape(NVAR, -1)[:, idx] = 0.0


class DistributedLevel:
    """One level whose boxes are partitioned over the ranks of a process
    group; rank r advances its own boxes.  geom, params: as for
    hydro.Level; max_grid_size chops the domain into the level's boxes (the
    reference's BoxArray).  pg: torch.distributed (None: one process).  All
    ranks make the same calls in the same order."""

    def __init__(self, geom, params, max_grid_size, rank=0, nranks=1, pg=None, device=None):
        import torch

        from . import hydro
        self.torch = torch
        self.hydro = hydro
        self.lib = native.lib()
        self.geom = geom
        self.params = params
        self.rank, self.nranks, self.pg = rank, nranks, pg
        self.device = device or torch.device("cuda", torch.cuda.current_device())
        self.n = tuple(geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3))
        self.boxes = hydro.level_boxes(self.n, max_grid_size, tuple(geom.dom_lo))
        self.owner = sfc_partition(self.boxes, nranks, tuple(geom.dom_lo))
        self.mine = [b for b in range(len(self.boxes)) if self.owner[b] == rank]
        self.plan = GhostPlan(geom, self.boxes, NG)
        self.ex = Exchange(self.plan, self.owner, rank, nranks, self.device, pg)
        self.S = {}
        self.dt_prev = None
        self.steps = 0
        self.mol = params.do_mol != 0
        self.grav = params.add_grav_src != 0
        self.registers = []

    @classmethod
    def from_inputs(cls, table, rank=0, nranks=1, pg=None, device=None):
        """The level a CAMR inputs file describes (camr_b200.inputs: the
        `CAMR.` parameters, the base geometry and boundary words,
        amr.max_grid_size, which the file must give)."""
        from . import inputs
        geom, mgs = inputs.geometry(table)
        if mgs is None:
            raise ValueError("amr.max_grid_size is required for a box-distributed level")
        return cls(geom, inputs.hydro_params(table), mgs, rank, nranks, pg, device)

    def attach_flux_register(self, fr, role):
        """After every hydro call of this level, pass its boxes' face fluxes
        to the flux register fr: CrseAdd when this level is the register's
        coarse level (role "coarse": the register's coarse boxes are this
        level's boxes, in their order), FineAdd when it is the fine level
        (role "fine": the register's fine boxes are this level's boxes, in
        their order, as for a fine level that covers its domain), scaled as
        construct_hydro_source does
        (Source/Hydro/CAMR_construct_hydro_source.cpp:240-252).  A register
        built on other boxes is refused here (ValueError)."""
        if role not in ("coarse", "fine"):
            raise ValueError(role)
        theirs = getattr(fr, "cboxes" if role == "coarse" else "fboxes", None)
        if theirs is not None:
            norm = [(tuple(lo), tuple(hi)) for lo, hi in theirs]
            if norm != [(tuple(lo), tuple(hi)) for lo, hi in self.boxes]:
                raise ValueError(f"the register's {role} boxes are not this level's boxes")
        self.registers.append((fr, role))

    # ---- state in and out (the valid cells of this rank's boxes) ----
    def _shape(self, b, ng):
        lo, hi = self.boxes[b]
        return (NVAR,) + tuple(hi[d] - lo[d] + 1 + 2 * ng for d in (2, 1, 0))

    def set_state(self, state):
        """state: the whole level (NVAR, nz, ny, nx) (host array); each rank
        keeps its own boxes."""
        T = self.torch
        dlo = self.geom.dom_lo
        for b in self.mine:
            lo, hi = self.boxes[b]
            part = state[:, lo[2] - dlo[2]:hi[2] - dlo[2] + 1, lo[1] - dlo[1]:hi[1] - dlo[1] + 1,
                         lo[0] - dlo[0]:hi[0] - dlo[0] + 1]
            self.S[b] = T.from_numpy(np.ascontiguousarray(part)).to(self.device)
        self.steps = 0
        self.dt_prev = None

    def get_state(self):
        """The whole level on every rank (gathered from all ranks)."""
        T = self.torch
        dlo = self.geom.dom_lo
        out = np.zeros((NVAR, self.n[2], self.n[1], self.n[0]))
        for b in range(len(self.boxes)):
            lo, hi = self.boxes[b]
            if self.nranks > 1:
                t = (self.S[b] if b in self.S
                     else T.empty(self._shape(b, 0), dtype=T.float64, device=self.device))
                self.pg.broadcast(t, src=int(self.owner[b]))
            else:
                t = self.S[b]
            out[:, lo[2] - dlo[2]:hi[2] - dlo[2] + 1, lo[1] - dlo[1]:hi[1] - dlo[1] + 1,
                lo[0] - dlo[0]:hi[0] - dlo[0] + 1] = t.cpu().numpy()
        return out

    # ---- fab-level calls over this rank's boxes ----
    def _arr(self, tensors, ng):
        boxes = [self.boxes[b] for b in self.mine]
        return boxes, [tensors[b] for b in self.mine]

    def _clean(self, tensors, ng, parts):
        boxes, ts = self._arr(tensors, ng)
        arr = self.hydro.box_fabs(boxes, ts, ng)
        native.check(self.lib.camr_clean_state_parts(
            C.byref(self.geom), len(boxes), arr, int(ng), C.byref(self.params), int(parts),
            C.c_void_p(self.torch.cuda.current_stream().cuda_stream)), "camr_clean_state_parts")

    def clean_valid(self, tensors):
        """clean_state of valid-only tensors (Source/CAMR.cpp:1253-1262)."""
        self._clean(tensors, 0, native.CLEAN_VALID | native.CLEAN_VALID_TEMP)

    def expand(self, src):
        """expand_state: FillPatch of the valid tensors src into tensors
        grown by 4, then clean_state of those (Source/CAMR.cpp:1243-1262)."""
        T = self.torch
        B = {}
        for b in self.mine:
            t = T.full(self._shape(b, NG), float("nan"), dtype=T.float64, device=self.device)
            t[:, NG:-NG, NG:-NG, NG:-NG] = src[b]
            B[b] = t
        # FillPatch: every ghost from the raw valid data (the physical-BC
        # ghosts keep these values)
        self.ex.fill(src, B, "all", src_ng=0)
        self._clean(B, NG, native.CLEAN_VALID)
        # normalize_species' FillBoundary: interior and periodic ghosts from
        # the owners' cleaned valid cells
        self.ex.fill(B, B, "interior", src_ng=NG)
        self._clean(B, NG, native.CLEAN_GHOSTS_TEMP | native.CLEAN_VALID_TEMP)
        return B

    def est_dt(self):
        """estTimeStep over the level: each rank's boxes, then the minimum
        over the ranks (Source/CAMR.cpp:490-563)."""
        boxes, ts = self._arr(self.S, 0)
        v = C.c_double()
        native.check(self.lib.camr_est_dt(C.byref(self.geom), len(boxes),
                                          self.hydro.box_fabs(boxes, ts, 0),
                                          C.byref(self.params), C.byref(v),
                                          C.c_void_p(self.torch.cuda.current_stream().cuda_stream)),
                     "camr_est_dt")
        est = v.value
        if self.nranks > 1:
            t = self.torch.tensor([est], dtype=self.torch.float64, device=self.device)
            self.pg.all_reduce(t, op=self.pg.ReduceOp.MIN)
            est = float(t.item())
        return est

    def _hydro(self, B, src_h, dt):
        T = self.torch
        out, fluxes = {}, {}
        for b in self.mine:
            lo, hi = self.boxes[b]
            dsdt = T.zeros(self._shape(b, 0), dtype=T.float64, device=self.device)
            flx = []
            for d in range(3):
                sh = list(self._shape(b, 0))
                sh[3 - d] += 1
                flx.append(T.empty(sh, dtype=T.float64, device=self.device))
            uin_lo = [lo[d] - NG for d in range(3)]
            self.hydro.hydro_umdrv(list(lo), list(hi), self.geom, B[b], uin_lo, dsdt, flx,
                                   self.params, dt, src=src_h[b] if src_h else None)
            out[b] = dsdt
            fluxes[b] = flx
        dx = [self.geom.dx[d] for d in range(3)]
        for fr, role in self.registers:
            if role == "coarse":
                fr.crse_add(fluxes, FluxRegister.crse_scale(dx, dt, self.mol))
            else:
                fr.fine_add(fluxes, FluxRegister.fine_scale(dx, dt, self.mol))
        return out

    def _grav(self, rho, mz, g):
        """The gravity source of CAMR (Source/GravitySrc.cpp:36-121): zero
        but for z momentum (g x rho) and energy (g x rho w); the correction
        passes the state differences and g/2."""
        T = self.torch
        src = T.zeros((NVAR,) + tuple(rho.shape), dtype=T.float64, device=self.device)
        src[3] = g * rho
        src[4] = g * mz
        return src

    def advance(self, nsteps=1):
        """nsteps level steps (CAMR_advance + post_timestep's clean_state),
        dt from computeInitialDt / computeNewDt over all ranks."""
        p = self.params
        for _ in range(nsteps):
            est = self.est_dt()
            if p.fixed_dt > 0.0:
                dt = p.fixed_dt
            elif self.steps == 0:
                dt = p.initial_dt if p.initial_dt > 0.0 else p.init_shrink * est
            else:
                dt = min(est, p.change_max * self.dt_prev)
            self.step(dt)
            self.dt_prev = dt
            self.steps += 1

    def step(self, dt):
        T = self.torch
        p = self.params
        S_old = {b: self.S[b].clone() for b in self.mine}
        self.clean_valid(S_old)
        B = self.expand(S_old)
        S = {b: B[b][:, NG:-NG, NG:-NG, NG:-NG].contiguous() for b in self.mine}
        src_old = {}
        if self.grav:
            for b in self.mine:
                src_old[b] = self._grav(S_old[b][0], S_old[b][3], p.const_grav)
                S[b] = S[b] + dt * src_old[b]
        if self.mol:
            k1 = self._hydro(B, None, dt)
            for b in self.mine:
                S[b] = S[b] + dt * k1[b]
            B2 = self.expand(S)
            k2 = self._hydro(B2, None, dt)
            for b in self.mine:
                B2v = B2[b][:, NG:-NG, NG:-NG, NG:-NG]
                S[b] = 0.5 * B2v + 0.5 * S_old[b]
                S[b] = S[b] + (0.5 * dt) * k2[b]
        else:
            src_h = None
            if self.grav and p.const_grav != 0.0:
                # sources_for_hydro: 0 + 1.0 x the old source on valid cells,
                # FillBoundary to interior and periodic ghosts, 0 beyond a
                # physical boundary
                src_h = {}
                for b in self.mine:
                    t = T.zeros(self._shape(b, NG), dtype=T.float64, device=self.device)
                    t[:, NG:-NG, NG:-NG, NG:-NG] = 0.0 + 1.0 * src_old[b]
                    src_h[b] = t
                self.ex.fill(src_h, src_h, "interior", src_ng=NG)
                self.ex.zero_physical(src_h)
            k = self._hydro(B, src_h, dt)
            for b in self.mine:
                S[b] = S[b] + dt * k[b]
        S = {b: S[b].contiguous() for b in self.mine}
        self.clean_valid(S)
        if self.grav:
            for b in self.mine:
                # 0.5 g (S_new - S_old) in the reference's order
                src_new = self._grav(S[b][0] - S_old[b][0], S[b][3] - S_old[b][3],
                                     0.5 * p.const_grav)
                S[b] = (S[b] + dt * src_new).contiguous()
            self.clean_valid(S)
        # post_timestep's clean_state (Source/CAMR.cpp:679-718)
        self.clean_valid(S)
        self.S = S



class FluxRegister:
    """The two-level flux register (refinement ratio 2) of a hierarchy whose
    coarse boxes and fine boxes are both spread over the ranks: AMReX's
    YAFluxRegister as the reference drives it -- CrseAdd and FineAdd after
    every hydro call of the coarse and the fine level
    (Source/Hydro/CAMR_construct_hydro_source.cpp:211-250), then Reflux in
    post_timestep (Source/CAMR.cpp:686, 803-825).

    Semantics (those of the two-level driver on one GPU and of its oracle):

    * the coarse cells outside the fine region that share a face with a
      fine-covered cell are the register's boundary cells (periodic
      neighbours included; the domain must be periodic, as the two-level
      driver's is);
    * crse_add: at each boundary cell of a coarse box, for the faces in the
      order x-, x+, y-, y+, z-, z+ whose other side is fine-covered, d -=
      dtdx * flux on a low face and d += dtdx * flux on a high face;
    * fine_add: for each fine box, direction and side (low, high), every
      uncovered coarse cell just outside the box gets its 4 fine face fluxes
      (slower transverse index outer), scaled by dtdx, subtracted on the
      box's low side and added on its high side, into cfp;
    * reflux: every coarse cell S = S + (d + cfp).

    Across ranks the fine face values travel from each fine box's owner to
    the owners of the coarse cells they correct, one message per pair of
    ranks at reflux time, and each coarse owner adds them in the order the
    single-process register does (call, fine box, direction, side, sub-face
    per cell), so the result does not depend on the partition, bit for bit.

    cboxes / fboxes: [(lo, hi)] of the coarse level's boxes (coarse index
    space) and of the fine boxes (fine index space, lo even and hi odd in
    each direction, disjoint); cowner / fowner: their ranks.  Fluxes are
    tensors (NVAR, nk, nj, ni) on a box's faces in one direction (the
    extent in that direction one larger), as camr_hydro_umdrv writes them.
    pg: torch.distributed (None: one process).  Every rank makes the same
    calls in the same order (crse_add and fine_add with possibly empty
    dicts)."""

    def __init__(self, geom, cboxes, cowner, fboxes, fowner, rank=0, nranks=1, device=None,
                 pg=None):
        import torch
        self.torch = torch
        self.rank, self.nranks, self.pg = rank, nranks, pg
        self.device = device or torch.device("cpu")
        if not all(geom.is_periodic[d] for d in range(3)):
            raise ValueError("the flux register needs a periodic domain")
        dlo = np.array([geom.dom_lo[d] for d in range(3)])
        n = np.array([geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3)])
        self.dlo, self.n = dlo, n
        ncell = int(np.prod(n))
        self.cboxes = [(tuple(lo), tuple(hi)) for lo, hi in cboxes]
        self.fboxes = [(tuple(lo), tuple(hi)) for lo, hi in fboxes]
        self.cowner = np.asarray(cowner, dtype=np.int64)
        self.fowner = np.asarray(fowner, dtype=np.int64)

        # coarse cell (flat, i fastest) -> coarse box, and -> fine box or -1
        cbox_of, _, cmap = _hierarchy_maps(self.cboxes, self.fboxes, dlo, n)
        cov = (cmap >= 0).reshape(n[2], n[1], n[0])
        near = np.zeros_like(cov)
        for ax in range(3):
            near |= np.roll(cov, 1, axis=ax) | np.roll(cov, -1, axis=ax)
        bnd = (near & ~cov).ravel()
        self.cmap, self.cbox_of = cmap, cbox_of

        # this rank's register: its boundary cells, numbered in flat order
        mine_bnd = bnd & (self.cowner[cbox_of] == rank)
        reg_of = np.full(ncell, -1, dtype=np.int64)
        reg_of[mine_bnd] = np.arange(int(mine_bnd.sum()))
        self.nreg = int(mine_bnd.sum())
        self.reg_of = reg_of
        self.mine_c = [c for c in range(len(self.cboxes)) if self.cowner[c] == rank]
        self.mine_f = [b for b in range(len(self.fboxes)) if self.fowner[b] == rank]

        T = torch
        dev = self.device
        # CrseAdd of each coarse box of this rank: per (direction, side),
        # the register slots and the face indices
        self._crse = {}
        unit = np.eye(3, dtype=np.int64)
        for c in self.mine_c:
            lo, hi = self.cboxes[c]
            ijk = _box_coords(lo, hi)
            cell = _wrap_flat(ijk, dlo, n)
            sel = bnd[cell]
            ijk = [a[sel] for a in ijk]
            reg = reg_of[cell[sel]]
            items = []
            for d in range(3):
                ext = [hi[e] - lo[e] + 1 + (e == d) for e in range(3)]
                for side in (0, 1):
                    nb = [ijk[e] + (unit[d][e] if side else -unit[d][e]) for e in range(3)]
                    m = cmap[_wrap_flat(nb, dlo, n)] >= 0
                    if not m.any():
                        continue
                    f = [ijk[e][m] + (unit[d][e] if side else 0) - lo[e] for e in range(3)]
                    fflat = f[0] + ext[0] * (f[1] + ext[1] * f[2])
                    items.append((d, side, T.as_tensor(reg[m], device=dev),
                                  T.as_tensor(fflat, device=dev)))
            self._crse[c] = items

        # FineAdd contributions of all fine boxes in the single-process
        # order: fine box, direction, side, cell, sub-face (a2 outer)
        parts = {k: [] for k in ("b", "d", "flat", "cell", "neg")}
        for b, (flo, fhi) in enumerate(self.fboxes):
            clo = [flo[e] // RR for e in range(3)]
            chi = [fhi[e] // RR for e in range(3)]
            for d in range(3):
                t1 = 1 if d == 0 else 0
                t2 = 1 if d == 2 else 2
                ext = [fhi[e] - flo[e] + 1 + (e == d) for e in range(3)]
                for side in (0, 1):
                    alo, ahi = list(clo), list(chi)
                    alo[d] = ahi[d] = chi[d] + 1 if side else clo[d] - 1
                    fface = RR * (chi[d] + 1) if side else RR * clo[d]
                    ijk = _box_coords(alo, ahi)
                    cell = _wrap_flat(ijk, dlo, n)
                    keep = cmap[cell] < 0
                    ijk = [a[keep] for a in ijk]
                    cell = cell[keep]
                    sub = []
                    for a2 in range(RR):
                        for a1 in range(RR):
                            fi = [None] * 3
                            fi[d] = np.full(cell.shape, fface)
                            fi[t1] = RR * ijk[t1] + a1
                            fi[t2] = RR * ijk[t2] + a2
                            f = [fi[e] - flo[e] for e in range(3)]
                            sub.append(f[0] + ext[0] * (f[1] + ext[1] * f[2]))
                    k = cell.size
                    # per cell its sub-faces, a2 outer
                    parts["flat"].append(np.stack(sub, axis=1).ravel())
                    parts["cell"].append(np.repeat(cell, RR * RR))
                    parts["b"].append(np.full(k * RR * RR, b))
                    parts["d"].append(np.full(k * RR * RR, d))
                    parts["neg"].append(np.full(k * RR * RR, side == 0))
        cat = {k: (np.concatenate(v) if v else np.zeros(0, dtype=np.int64))
               for k, v in parts.items()}
        src_rank = self.fowner[cat["b"]] if cat["b"].size else cat["b"]
        dst_rank = self.cowner[cbox_of[cat["cell"]]] if cat["cell"].size else cat["cell"]

        # sender side: per destination rank, per (fine box, direction) of
        # this rank, the face indices and signs, in the global order
        self._send = {}
        for r in range(nranks):
            m = (src_rank == rank) & (dst_rank == r)
            if not m.any():
                continue
            segs = []
            bb, dd = cat["b"][m], cat["d"][m]
            key = bb * 3 + dd
            starts = np.flatnonzero(np.r_[True, key[1:] != key[:-1]])
            ends = np.r_[starts[1:], key.size]
            fl, ng = cat["flat"][m], cat["neg"][m]
            for s0, s1 in zip(starts, ends):
                segs.append((int(bb[s0]), int(dd[s0]), T.as_tensor(fl[s0:s1], device=dev),
                             T.as_tensor(ng[s0:s1], device=dev)))
            self._send[r] = (segs, int(m.sum()))

        # receiver side: the contributions to this rank's cells in the
        # global order, where each sender's part sits, and the rounds in
        # which no two contributions share a register slot
        m = dst_rank == rank
        tgt = reg_of[cat["cell"][m]]
        srcs = src_rank[m]
        self._recv_pos = {int(r): T.as_tensor(np.flatnonzero(srcs == r), device=dev)
                          for r in np.unique(srcs)}
        self._nrecv = int(m.sum())
        order = np.argsort(tgt, kind="stable")
        rnd = np.empty(tgt.size, dtype=np.int64)
        if tgt.size:
            st = tgt[order]
            first = np.r_[True, st[1:] != st[:-1]]
            start_of = np.maximum.accumulate(np.where(first, np.arange(st.size), 0))
            rnd[order] = np.arange(st.size) - start_of
        self._rounds = []
        for k in range(int(rnd.max()) + 1 if rnd.size else 0):
            sel = np.flatnonzero(rnd == k)
            self._rounds.append((T.as_tensor(sel, device=dev), T.as_tensor(tgt[sel], device=dev)))

        # reflux of each coarse box of this rank: its register slots
        self._apply = {}
        for c in self.mine_c:
            lo, hi = self.cboxes[c]
            cell = _wrap_flat(_box_coords(lo, hi), dlo, n)
            loc = np.flatnonzero(reg_of[cell] >= 0)
            self._apply[c] = (T.as_tensor(loc, device=dev), T.as_tensor(reg_of[cell[loc]], device=dev))
        self.reset()

    @staticmethod
    def crse_scale(dx, dt, mol):
        """CrseAdd's factor for one hydro call of the coarse level:
        fac_for_reflux * dt / vol, fac_for_reflux 0.5 for MOL (each of its
        two stages adds) and 1 for CTU (Source/Hydro/
        CAMR_construct_hydro_source.cpp:24, 240-247)."""
        return ((0.5 if mol else 1.0) * dt) / (dx[0] * dx[1] * dx[2])

    @staticmethod
    def fine_scale(dx_f, dt_f, mol):
        """FineAdd's factor for one hydro call of the fine level: the fine
        call's fac_for_reflux * dt / vol, over the ratio^3 fine cells of a
        coarse cell (YAFluxRegister's FineAdd, ratio 2)."""
        return ((0.5 if mol else 1.0) * dt_f) / ((dx_f[0] * dx_f[1] * dx_f[2]) * float(RR ** 3))

    # ---- the register ----
    def reset(self):
        """Zero the register (FluxRegister::reset at the start of each
        coarse step) and drop the fine calls kept since the last reset."""
        T = self.torch
        self.d = T.zeros((NVAR, self.nreg), dtype=T.float64, device=self.device)
        self.cfp = T.zeros((NVAR, self.nreg), dtype=T.float64, device=self.device)
        self._fine = []

    def crse_add(self, fluxes, dtdx):
        """CrseAdd of the coarse boxes of this rank: fluxes {box: [fx, fy,
        fz]} (face fluxes, area-weighted), scaled by dtdx."""
        for c in sorted(fluxes):
            if c not in self._crse:
                raise ValueError(f"coarse box {c} is not on rank {self.rank}")
            f = fluxes[c]
            for d, side, reg, fflat in self._crse[c]:
                v = dtdx * f[d].reshape(NVAR, -1)[:, fflat]
                if side:
                    self.d[:, reg] = self.d[:, reg] + v
                else:
                    self.d[:, reg] = self.d[:, reg] - v

    def fine_add(self, fluxes, dtdx):
        """FineAdd of one fine hydro call: fluxes {fine box: [fx, fy, fz]}
        for every fine box of this rank (an empty dict on a rank with none),
        scaled by dtdx.  The scaled values of each destination rank are kept
        until reflux."""
        T = self.torch
        if sorted(fluxes) != self.mine_f:
            raise ValueError("fine_add needs the fluxes of exactly this rank's fine boxes")
        out = {}
        for r, (segs, cnt) in self._send.items():
            vals = T.empty((NVAR, cnt), dtype=T.float64, device=self.device)
            at = 0
            for b, d, fflat, neg in segs:
                k = fflat.numel()
                v = dtdx * fluxes[b][d].reshape(NVAR, -1)[:, fflat]
                vals[:, at:at + k] = T.where(neg, -v, v)
                at += k
            out[r] = vals
        self._fine.append(out)

    def reflux(self, S, ng=0):
        """Reflux: the fine values travel to the coarse owners, the register
        adds them in the single-process order, then every valid cell of this
        rank's coarse boxes becomes S + (d + cfp).  S: {coarse box: tensor
        (NVAR, ...) covering the box grown by ng}, updated in place."""
        T = self.torch
        ncall = len(self._fine)
        if ncall == 0:
            self._apply_corrections(S, ng)
            return
        got = {}
        if self.rank in self._send:
            got[self.rank] = [call[self.rank] for call in self._fine]
        if self.pg is not None and self.nranks > 1:
            ops, bufs = [], {}
            for r in sorted(self._send):
                if r == self.rank:
                    continue
                buf = T.cat([call[r] for call in self._fine], dim=1).contiguous()
                bufs[("s", r)] = buf
                ops.append(self.pg.isend(buf, dst=r))
            for r, pos in sorted(self._recv_pos.items()):
                if r == self.rank:
                    continue
                buf = T.empty((NVAR, ncall * pos.numel()), dtype=T.float64, device=self.device)
                bufs[("r", r)] = buf
                ops.append(self.pg.irecv(buf, src=r))
            for op in ops:
                op.wait()
            for r, pos in self._recv_pos.items():
                if r != self.rank:
                    got[r] = list(bufs[("r", r)].split(pos.numel(), dim=1))
        for s in range(ncall):
            allv = T.empty((NVAR, self._nrecv), dtype=T.float64, device=self.device)
            for r, pos in self._recv_pos.items():
                allv[:, pos] = got[r][s]
            for sel, reg in self._rounds:
                self.cfp[:, reg] = self.cfp[:, reg] + allv[:, sel]
        self._apply_corrections(S, ng)

    def _apply_corrections(self, S, ng):
        T = self.torch
        for c in sorted(S):
            if c not in self._apply:
                raise ValueError(f"coarse box {c} is not on rank {self.rank}")
            lo, hi = self.cboxes[c]
            ext = [hi[e] - lo[e] + 1 for e in range(3)]
            loc, reg = self._apply[c]
            corr = T.zeros((NVAR, ext[0] * ext[1] * ext[2]), dtype=T.float64, device=self.device)
            corr[:, loc] = self.d[:, reg] + self.cfp[:, reg]
            t = S[c]
            v = t[:, ng:ng + ext[2], ng:ng + ext[1], ng:ng + ext[0]] if ng else t
            v.add_(corr.reshape(NVAR, ext[2], ext[1], ext[0]))


class AverageDown:
    """avgDown of a two-level hierarchy (refinement ratio 2) whose coarse
    and fine boxes are spread over the ranks (CAMR::avgDown,
    Source/CAMR.cpp:693, 1048-1064, amrex::average_down): every coarse cell
    that a fine box covers becomes 1/8 of the sum of its 8 children, summed
    from 0.0 with the x index fastest, then z.

    Each fine box's owner forms the averages of its box and sends them to
    the owners of the coarse cells, one message per pair of ranks, so the
    result does not depend on the partition, bit for bit.  Boxes and owners
    as for FluxRegister; every rank makes the same calls."""

    def __init__(self, geom, cboxes, cowner, fboxes, fowner, rank=0, nranks=1, device=None,
                 pg=None):
        import torch
        self.torch = torch
        self.rank, self.nranks, self.pg = rank, nranks, pg
        self.device = device or torch.device("cpu")
        dlo = np.array([geom.dom_lo[d] for d in range(3)])
        dhi = np.array([geom.dom_hi[d] for d in range(3)])
        n = dhi - dlo + 1
        self.cboxes = [(tuple(lo), tuple(hi)) for lo, hi in cboxes]
        self.fboxes = [(tuple(lo), tuple(hi)) for lo, hi in fboxes]
        cowner = np.asarray(cowner, dtype=np.int64)
        fowner = np.asarray(fowner, dtype=np.int64)
        cbox_of, cloc, _ = _hierarchy_maps(self.cboxes, self.fboxes, dlo, n)
        self.mine_f = [b for b in range(len(self.fboxes)) if fowner[b] == rank]
        T = torch
        dev = self.device

        def kji(c, places):
            # flat places inside coarse box c -> (k, j, i) offsets in it
            lo, hi = self.cboxes[c]
            nx, ny = hi[0] - lo[0] + 1, hi[1] - lo[1] + 1
            return tuple(T.as_tensor(a, device=dev)
                         for a in (places // (nx * ny), (places // nx) % ny, places % nx))

        # per fine box: its coarse cells' (coarse box, place) and owner
        self._send = {}   # dest rank -> [(fine box, positions in the box's averages)]
        self._recv = {}   # src rank -> [(coarse box, place) per entry, in message order]
        self._local = []  # (fine box, positions, coarse box, places) on this rank
        for b, (flo, fhi) in enumerate(self.fboxes):
            clo = [flo[d] // RR for d in range(3)]
            chi = [fhi[d] // RR for d in range(3)]
            cell = _flat(_box_coords(clo, chi), dlo, n)
            cb, pl = cbox_of[cell], cloc[cell]
            dest = cowner[cb]
            src = int(fowner[b])
            for r in np.unique(dest):
                r = int(r)
                pos = np.flatnonzero(dest == r)
                if src == rank and r == rank:
                    for c in np.unique(cb[pos]):
                        m = pos[cb[pos] == c]
                        self._local.append((b, T.as_tensor(m, device=dev), int(c),
                                            kji(int(c), pl[m])))
                elif src == rank:
                    self._send.setdefault(r, []).append((b, T.as_tensor(pos, device=dev)))
                elif r == rank:
                    self._recv.setdefault(src, []).append((cb[pos], pl[pos]))
        # the receiver's writes grouped by coarse box: (start, stop) of each
        # run within the concatenated message
        self._recv_groups = {}
        for s, items in self._recv.items():
            cbs = np.concatenate([x[0] for x in items])
            pls = np.concatenate([x[1] for x in items])
            groups = []
            for c in np.unique(cbs):
                m = np.flatnonzero(cbs == c)
                groups.append((int(c), T.as_tensor(m, device=dev), kji(int(c), pls[m])))
            self._recv_groups[s] = (groups, int(cbs.size))

    def _averages(self, t, ng):
        """(NVAR, cells of the coarsened box) from a fine box's tensor."""
        T = self.torch
        v = t[:, ng:t.shape[1] - ng, ng:t.shape[2] - ng, ng:t.shape[3] - ng] if ng else t
        c = T.zeros((NVAR, v.shape[1] // RR, v.shape[2] // RR, v.shape[3] // RR),
                    dtype=T.float64, device=self.device)
        for kr in range(RR):
            for jr in range(RR):
                for ir in range(RR):
                    c = c + v[:, kr::RR, jr::RR, ir::RR]
        return ((1.0 / float(RR ** 3)) * c).reshape(NVAR, -1)

    def __call__(self, S_fine, S_coarse, ng_f=0, ng_c=0):
        """S_fine: {fine box: tensor (NVAR, ...) covering the box grown by
        ng_f} for this rank's fine boxes; S_coarse: {coarse box: tensor
        covering it grown by ng_c} for this rank's coarse boxes, whose
        covered valid cells are overwritten."""
        T = self.torch
        if sorted(S_fine) != self.mine_f:
            raise ValueError("average-down needs exactly this rank's fine boxes")
        avg = {b: self._averages(S_fine[b], ng_f) for b in self.mine_f}

        def put(c, at, vals):
            t = S_coarse[c]
            v = t[:, ng_c:t.shape[1] - ng_c, ng_c:t.shape[2] - ng_c,
                  ng_c:t.shape[3] - ng_c] if ng_c else t
            v[:, at[0], at[1], at[2]] = vals

        for b, pos, c, places in self._local:
            put(c, places, avg[b][:, pos])
        if self.pg is None or self.nranks == 1:
            return
        ops, bufs = [], {}
        for r, items in sorted(self._send.items()):
            buf = T.cat([avg[b][:, pos] for b, pos in items], dim=1).contiguous()
            bufs[("s", r)] = buf
            ops.append(self.pg.isend(buf, dst=r))
        for s, (groups, cnt) in sorted(self._recv_groups.items()):
            buf = T.empty((NVAR, cnt), dtype=T.float64, device=self.device)
            bufs[("r", s)] = buf
            ops.append(self.pg.irecv(buf, src=s))
        for op in ops:
            op.wait()
        for s, (groups, _) in sorted(self._recv_groups.items()):
            buf = bufs[("r", s)]
            for c, sel, places in groups:
                put(c, places, buf[:, sel])



class TwoLevelFill:
    """The ghost cells of the fine boxes of a two-level hierarchy (ratio 2,
    periodic domain) whose coarse and fine boxes are spread over the ranks:
    the fill of FillPatchTwoLevels as the two-level driver does it
    (Source/CAMR.cpp:1243-1250, AMReX FillPatchTwoLevels with
    CellConservativeLinear):

    * a ghost cell that a fine box covers (through the periodic domain)
      takes that box's valid value;
    * every other ghost cell takes the conservative linear interpolation of
      the coarse data at time t: per direction an MC-limited slope of the
      coarse cell holding it, one factor alpha <= 1 for the three slopes so
      that no child leaves the min/max of the 27 coarse neighbours, and the
      child at -+1/4 of each slope; the coarse data at t is the new (old)
      state within 1e-3 (t1 - t0) of t1 (t0), else alpha old + beta new
      (StateData::getData).

    The coarse owners send the coarse cells each fine box's interpolation
    reads (combined in time), the fine owners the valid cells other fine
    boxes' ghosts copy, one message per pair of ranks; every value is formed
    with the same operations in the same order as on one process, so the
    result does not depend on the partition, bit for bit.  Boxes and owners
    as for FluxRegister; every rank makes the same calls."""

    def __init__(self, geom, cboxes, cowner, fboxes, fowner, rank=0, nranks=1, device=None,
                 pg=None, ng=NG):
        import torch
        self.torch = torch
        self.rank, self.nranks, self.pg, self.ng = rank, nranks, pg, ng
        self.device = device or torch.device("cpu")
        if not all(geom.is_periodic[d] for d in range(3)):
            raise ValueError("the two-level fill needs a periodic domain")
        T = torch
        dev = self.device
        dlo = np.array([geom.dom_lo[d] for d in range(3)])
        n = np.array([geom.dom_hi[d] - geom.dom_lo[d] + 1 for d in range(3)])
        fdlo, fn = RR * dlo, RR * n
        self.cboxes = [(tuple(lo), tuple(hi)) for lo, hi in cboxes]
        self.fboxes = [(tuple(lo), tuple(hi)) for lo, hi in fboxes]
        cowner = np.asarray(cowner, dtype=np.int64)
        fowner = np.asarray(fowner, dtype=np.int64)
        self.mine_c = [c for c in range(len(self.cboxes)) if cowner[c] == rank]
        self.mine_f = [b for b in range(len(self.fboxes)) if fowner[b] == rank]
        cbox_of, cloc, cmap = _hierarchy_maps(self.cboxes, self.fboxes, dlo, n)

        # per fine box: fine-fine sources and the interpolated cells
        coarse_items = {}   # (src rank, dst rank) -> [(fine box, coarse box, places, positions)]
        fine_items = {}     # (src rank, dst rank) -> [(dst box, src box, src idx, dst idx)]
        self._interp = {}   # fine box of this rank -> plan of its interpolated cells
        for b, (lo, hi) in enumerate(self.fboxes):
            glo = [lo[d] - ng for d in range(3)]
            ghi = [hi[d] + ng for d in range(3)]
            gext = [ghi[d] - glo[d] + 1 for d in range(3)]
            f = _box_coords(glo, ghi)
            gflat = np.arange(f[0].size)
            ghost = np.zeros(f[0].size, dtype=bool)
            for d in range(3):
                ghost |= (f[d] < lo[d]) | (f[d] > hi[d])
            f = [a[ghost] for a in f]
            gflat = gflat[ghost]
            w = [(f[d] - fdlo[d]) % fn[d] + fdlo[d] for d in range(3)]
            ob = cmap[_flat([w[d] // RR for d in range(3)], dlo, n)]
            rb = int(fowner[b])
            # fine-fine copies, grouped by source box
            for o in np.unique(ob[ob >= 0]):
                m = ob == o
                olo, ohi = self.fboxes[o]
                oext = [ohi[d] - olo[d] + 1 + 2 * ng for d in range(3)]
                sidx = ((w[0][m] - olo[0] + ng) + oext[0] * ((w[1][m] - olo[1] + ng)
                                                              + oext[1] * (w[2][m] - olo[2] + ng)))
                fine_items.setdefault((int(fowner[o]), rb), []).append(
                    (b, int(o), sidx, gflat[m]))
            # interpolated cells: the coarse cell holding each, its 27
            # neighbours (dk, dj, di from -1 to 1) and the child's offsets
            m = ob < 0
            fi = [a[m] for a in f]
            cc = [a // RR for a in fi]
            # every coarse cell those read lies in one index box around the
            # coarsened ghost region; a mask over it picks the ones read
            blo = [(lo[d] - ng) // RR - 1 for d in range(3)]
            bext = [(hi[d] + ng) // RR + 1 - blo[d] + 1 for d in range(3)]
            nbr = []
            for dk in (-1, 0, 1):
                for dj in (-1, 0, 1):
                    for di in (-1, 0, 1):
                        nbr.append((cc[0] + di - blo[0]) + bext[0] * (
                            (cc[1] + dj - blo[1]) + bext[1] * (cc[2] + dk - blo[2])))
            nbr = np.stack(nbr) if fi[0].size else np.zeros((27, 0), dtype=np.int64)
            need = np.zeros(bext[0] * bext[1] * bext[2], dtype=bool)
            need[nbr.ravel()] = True
            inv = (np.cumsum(need) - 1)[nbr]
            loc = np.flatnonzero(need)
            bc = [loc % bext[0] + blo[0], (loc // bext[0]) % bext[1] + blo[1],
                  loc // (bext[0] * bext[1]) + blo[2]]
            uniq = _wrap_flat(bc, dlo, n)
            off = [np.where(fi[d] - RR * cc[d] == 0, -0.25, 0.25) for d in range(3)]
            if rb == rank:
                self._interp[b] = (T.as_tensor(gflat[m], device=dev),
                                   T.as_tensor(inv, device=dev),
                                   [T.as_tensor(o, device=dev) for o in off], int(uniq.size))
            ucb = cbox_of[uniq]
            uown = cowner[ucb]
            for c in np.unique(ucb):
                sel = np.flatnonzero(ucb == c)
                coarse_items.setdefault((int(uown[sel[0]]), rb), []).append(
                    (b, int(c), cloc[uniq[sel]], sel))

        def tens(a):
            return T.as_tensor(np.asarray(a, dtype=np.int64), device=dev)

        # this rank's part of the plan: what it sends to and receives from
        # each rank (itself included), in one order on both sides
        self._send, self._recv = {}, {}
        for r in range(nranks):
            ci = coarse_items.get((rank, r), [])
            fi_ = fine_items.get((rank, r), [])
            if ci or fi_:
                self._send[r] = ([(c, tens(pl)) for _, c, pl, _ in ci],
                                 [(o, tens(si)) for _, o, si, _ in fi_],
                                 sum(len(pl) for _, _, pl, _ in ci) + sum(len(si) for _, _, si, _ in fi_))
            ci = coarse_items.get((r, rank), [])
            fi_ = fine_items.get((r, rank), [])
            if ci or fi_:
                self._recv[r] = ([(b, tens(pos)) for b, _, _, pos in ci],
                                 [(b, tens(di)) for b, _, _, di in fi_],
                                 sum(len(pos) for _, _, _, pos in ci) + sum(len(di) for _, _, _, di in fi_))

    @staticmethod
    def time_weights(t0, t1, t):
        """StateData::getData's choice: (0, new), (1, old) or (2, alpha, beta)."""
        teps = (t1 - t0) * 1.e-3
        if t1 - teps < t < t1 + teps:
            return (0, 0.0, 0.0)
        if t0 - teps < t < t0 + teps:
            return (1, 0.0, 0.0)
        return (2, (t1 - t) / (t1 - t0), (t - t0) / (t1 - t0))

    def __call__(self, fine, c_old, c_new, t0, t1, t):
        """fine: {fine box: contiguous tensor (NVAR, ...) covering the box
        grown by ng, valid cells set} for this rank's fine boxes, whose
        ghost cells are filled in place; c_old / c_new: {coarse box: tensor
        (NVAR, ...) of its valid cells} for this rank's coarse boxes at
        times t0 / t1."""
        T = self.torch
        if sorted(fine) != self.mine_f:
            raise ValueError("the fill needs exactly this rank's fine boxes")
        mode, wa, wb = self.time_weights(t0, t1, t)
        cache = {}

        def coarse_at(c):
            if c not in cache:
                o = c_old[c].reshape(NVAR, -1)
                nw = c_new[c].reshape(NVAR, -1)
                cache[c] = nw if mode == 0 else o if mode == 1 else wa * o + wb * nw
            return cache[c]

        def pack(r):
            citems, fitems, _ = self._send[r]
            parts = [coarse_at(c)[:, pl] for c, pl in citems]
            parts += [fine[o].view(NVAR, -1)[:, si] for o, si in fitems]
            return T.cat(parts, dim=1)

        got = {}
        if self.rank in self._send:
            got[self.rank] = pack(self.rank)
        if self.pg is not None and self.nranks > 1:
            ops, bufs = [], {}
            for r in sorted(self._send):
                if r == self.rank:
                    continue
                bufs[("s", r)] = pack(r).contiguous()
                ops.append(self.pg.isend(bufs[("s", r)], dst=r))
            for r, (_, _, cnt) in sorted(self._recv.items()):
                if r == self.rank:
                    continue
                bufs[("r", r)] = T.empty((NVAR, cnt), dtype=T.float64, device=self.device)
                ops.append(self.pg.irecv(bufs[("r", r)], src=r))
            for op in ops:
                op.wait()
            for r in self._recv:
                if r != self.rank:
                    got[r] = bufs[("r", r)]
        # the coarse cells each fine box reads, and the fine-fine copies
        compact = {b: T.empty((NVAR, self._interp[b][3]), dtype=T.float64, device=self.device)
                   for b in self.mine_f}
        for r, (citems, fitems, _) in self._recv.items():
            buf = got[r]
            at = 0
            for b, pos in citems:
                k = pos.numel()
                compact[b][:, pos] = buf[:, at:at + k]
                at += k
            for b, di in fitems:
                k = di.numel()
                fine[b].view(NVAR, -1)[:, di] = buf[:, at:at + k]
                at += k
        for b in self.mine_f:
            gidx, inv, off, _ = self._interp[b]
            if gidx.numel():
                fine[b].view(NVAR, -1)[:, gidx] = self._cons_interp(compact[b], inv, off)

    def _cons_interp(self, cv, inv, off):
        """CellConservativeLinear (ratio 2, limited), the operations of the
        single-process fill in its order; std::min / std::max are written
        as the selects they are."""
        T = self.torch
        at = [cv[:, inv[q]] for q in range(27)]     # (dk, dj, di) from -1 to 1
        uc = at[13]
        sl = []
        for step in (1, 3, 9):                      # x, y, z neighbours
            up, um = at[13 + step], at[13 - step]
            dc = 0.5 * (up - um)
            df = 2.0 * (up - uc)
            db = 2.0 * (uc - um)
            adf, adb = df.abs(), db.abs()
            sv = T.where(df * db >= 0.0, T.where(adb < adf, adb, adf), T.zeros_like(df))
            adc = dc.abs()
            sv = T.copysign(T.ones_like(dc), dc) * T.where(adc < sv, adc, sv)
            sl.append(sv)
        anyn = (sl[0] != 0.0) | (sl[1] != 0.0) | (sl[2] != 0.0)
        dumax = sl[0].abs() * 0.25 + sl[1].abs() * 0.25 + sl[2].abs() * 0.25
        umax, umin = uc, uc
        for q in range(27):
            v = at[q]
            umax = T.where(umax < v, v, umax)
            umin = T.where(v < umin, v, umin)
        alpha = T.ones_like(uc)
        alpha = T.where(anyn & (dumax * alpha > (umax - uc)), (umax - uc) / dumax, alpha)
        alpha = T.where(anyn & (dumax * alpha > (uc - umin)), (uc - umin) / dumax, alpha)
        return uc + off[0] * (sl[0] * alpha) + off[1] * (sl[1] * alpha) + off[2] * (sl[2] * alpha)
