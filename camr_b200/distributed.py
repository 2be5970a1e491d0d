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
        out = {}
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
