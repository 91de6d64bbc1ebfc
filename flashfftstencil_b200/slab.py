"""One grid over several ranks: slabs along the slowest axis with one ghost
exchange of width r*tau per fused pass.

The reference runs one grid on one GPU (``src/2D/2d_main.cu:120-190``); this
module spreads a grid that is too large or too slow for one B200 over ranks of
a ``torch.distributed`` group (NCCL over NVLink between GPUs, gloo on CPU).

Rank k owns rows [lo_k, hi_k) of the slowest axis (z in 3D, y in 2D, x in 1D;
with row-major storage a slab is one contiguous block of memory).  Its buffer
holds those rows plus ``g = r * tau`` ghost rows on every side that has a
neighbour (both sides when the boundary is periodic).  A solve of tau steps on
that extended slab is exact on every row at least g rows from its ends -- the
rank's own rows -- whatever the local solve does at the ends (it holds a fixed
ring or wraps around): the error made there travels r rows per step and stops
inside the ghost rows, which the next exchange overwrites.  So every pass is:

1. send the first and last g own rows to the neighbours, receive the ghosts
   (grouped point-to-point sends and receives);
2. solve the whole extended slab (one fused pass; its cut ends are "open
   faces", so no boundary work is spent there).

With ``overlap=True`` a pass instead solves the "core" rows [lo, hi) alone
(exact on [lo+g, hi-g)) while the exchange is in flight, then two edge strips
of 3g rows ([lo-g, lo+2g) and [hi-2g, hi+g)) into scratch whose middle g rows
are copied into place.  That hides the exchange but adds two small solves and
two copies per pass, which cost more than a ghost exchange over NVLink unless
the slab is tall; slabs thinner than 4g rows never split.  A side without a
neighbour (the ends of a fixed-boundary grid) is the grid's true face: every
local solve treats it as such, and no strip is needed there.
"""
from __future__ import annotations

from dataclasses import dataclass


def slab_bounds(n: int, world: int, rank: int) -> tuple[int, int]:
    """Rows [lo, hi) of rank `rank` when n rows are split as evenly as possible."""
    base, extra = divmod(n, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


@dataclass(frozen=True)
class PassGeom:
    tau: int
    g: int        # ghost rows per side that has a neighbour
    gl: int       # ghost rows above (0 without an upper neighbour)
    gh: int       # ghost rows below
    split: bool   # core + strips (overlaps the exchange) or one solve after it


class SlabPlan:
    """This rank's part of a T-step solve of one grid split into slabs.

    ``extents`` are the global (nx, ny, nz), x fastest, as for :class:`Plan`.
    ``stepper(extents, tau, open_faces)`` returns a function ``f(src, dst)`` that
    runs tau steps on a contiguous tensor of those extents, where ``open_faces``
    (the ``ffs_problem`` bit mask) marks the slab ends that are cuts through the
    grid rather than its boundary; the default builds an FP64
    :class:`~flashfftstencil_b200.Plan` on the current CUDA device (one fused
    pass, launched on the current stream), which then spends no boundary work
    on those ends.
    """

    def __init__(self, dim, shape, extents, T, weights=None, radius=None, boundary="periodic", rank=0, world=1,
                 tau=0, form="fp64", stepper=None, overlap=False):
        import flashfftstencil_b200 as ffs

        if boundary not in ("periodic", "fixed"):
            raise ValueError("boundary must be 'periodic' or 'fixed'")
        if not 0 <= rank < world:
            raise ValueError("rank out of range")
        self.dim, self.T, self.boundary = dim, int(T), boundary
        self.extents = tuple(int(e) for e in extents)[:dim]
        if len(self.extents) != dim:
            raise ValueError("need one extent per dimension")
        if shape is not None:
            si = ffs.shape_info(shape)
            radius = si.radius if radius is None else radius
            weights = si.weights if weights is None else weights
        if radius is None or weights is None:
            raise ValueError("give a named shape or both weights and radius")
        self.radius, self.weights, self.form = int(radius), weights, form
        self.rank, self.world = rank, world
        self.overlap = bool(overlap)
        self.n = self.extents[-1]                      # rows of the slowest axis
        self.lo, self.hi = slab_bounds(self.n, world, rank)
        self.rows = self.hi - self.lo
        periodic = boundary == "periodic"
        self.up = (rank - 1) % world if (periodic or rank > 0) else None
        self.down = (rank + 1) % world if (periodic or rank < world - 1) else None
        if world == 1:  # one slab is the whole grid: the local solve sees the true boundary
            self.up = self.down = None

        # pass structure of the global problem (same tile family, same fused step counts); a
        # step count modelled on the slab a rank solves (ffs_plan_info.model_ms) measured slower
        # at 8 ranks of a 4096^2 grid (tau 11: 0.237 ms per rank against 0.148 at the global 8),
        # because the model underrates the band kernel's cost at high tau
        if self.T == 0:
            self.passes = []
        else:
            info = ffs.describe(dim, None, extents, T, weights=weights, radius=self.radius, boundary=boundary,
                                form=form, tau=tau)
            taus = [info["tau"]] * (info["passes"] - 1) + [info["tau_last"]]
            self.passes = [self._geom(t) for t in taus]
        need = max((p.g for p in self.passes), default=0)
        if (self.up is not None or self.down is not None) and self.rows < need:
            raise ValueError(f"slab of {self.rows} rows is thinner than the ghost width {need} (r * tau); "
                             "use fewer ranks or a smaller tau")
        self.gmax = need if self.up is not None else 0, need if self.down is not None else 0
        self._stepper = stepper or self._plan_stepper
        self._steppers = {}

    # ---- geometry ---------------------------------------------------------------------
    def _geom(self, tau: int) -> PassGeom:
        g = self.radius * tau
        gl = g if self.up is not None else 0
        gh = g if self.down is not None else 0
        split = self.overlap and (gl or gh) and self.rows >= 4 * g
        return PassGeom(tau, g, gl, gh, bool(split))

    def bounds(self, rank: int | None = None) -> tuple[int, int]:
        return slab_bounds(self.n, self.world, self.rank if rank is None else rank)

    def local_shape(self, rows: int | None = None) -> tuple[int, ...]:
        rows = self.rows if rows is None else rows
        return (rows,) + tuple(reversed(self.extents[:-1]))

    def _ext(self, rows: int) -> tuple[int, ...]:
        return tuple(self.extents[:-1]) + (rows,)

    def _plan_stepper(self, ext, tau, open_faces):
        import torch

        import flashfftstencil_b200 as ffs
        plan = ffs.Plan(self.dim, None, ext, tau, weights=self.weights, radius=self.radius,
                        boundary=self.boundary, form=self.form, tau=tau, open_faces=open_faces)

        def run(src, dst):
            plan.execute(src.data_ptr(), dst.data_ptr(), torch.cuda.current_stream(src.device).cuda_stream)
        run.plan = plan
        return run

    def _step(self, rows: int, tau: int, low_open: bool, high_open: bool):
        """Solver of tau steps on `rows` rows whose low / high end is a cut (open) or the grid's face."""
        axis = self.dim - 1
        faces = (int(low_open) << (2 * axis)) | (int(high_open) << (2 * axis + 1))
        key = (rows, tau, faces)
        if key not in self._steppers:
            self._steppers[key] = self._stepper(self._ext(rows), tau, faces)
        return self._steppers[key]

    # ---- buffers ----------------------------------------------------------------------
    def allocate(self, like):
        """Two extended buffers and a strip scratch, on `like`'s device and dtype."""
        import torch
        gl, gh = self.gmax
        shape = self.local_shape(self.rows + gl + gh)
        g = max((p.g for p in self.passes), default=0)
        return (torch.empty(shape, dtype=like.dtype, device=like.device),
                torch.empty(shape, dtype=like.dtype, device=like.device),
                torch.empty(self.local_shape(max(3 * g, 1)), dtype=like.dtype, device=like.device))

    def load(self, bufs, x):
        """Copy this rank's rows into the first buffer's own-row window."""
        gl = self.gmax[0]
        bufs[0][gl:gl + self.rows].copy_(x)

    def own(self, buf):
        gl = self.gmax[0]
        return buf[gl:gl + self.rows]

    # ---- one pass ---------------------------------------------------------------------
    def send_views(self, E, p: PassGeom):
        """(rows for the upper neighbour, rows for the lower neighbour); None where absent."""
        gl = self.gmax[0]
        top = E[gl:gl + p.g] if self.up is not None else None
        bot = E[gl + self.rows - p.g:gl + self.rows] if self.down is not None else None
        return top, bot

    def recv_views(self, E, p: PassGeom):
        """(ghost rows above, ghost rows below); None where absent."""
        gl = self.gmax[0]
        above = E[gl - p.g:gl] if self.up is not None else None
        below = E[gl + self.rows:gl + self.rows + p.g] if self.down is not None else None
        return above, below

    def compute_core(self, E, O, p: PassGeom):
        """Rows that need no ghost (split passes only); run while the exchange is in flight."""
        if p.split:
            gl = self.gmax[0]
            self._step(self.rows, p.tau, p.gl > 0, p.gh > 0)(E[gl:gl + self.rows], O[gl:gl + self.rows])

    def compute_rest(self, E, O, S, p: PassGeom):
        """Everything the ghosts feed; call after the exchange has landed."""
        gl = self.gmax[0]
        if not p.split:
            a, b = gl - p.gl, gl + self.rows + p.gh
            self._step(b - a, p.tau, p.gl > 0, p.gh > 0)(E[a:b], O[a:b])
            return
        g = p.g
        strip = self._step(3 * g, p.tau, True, True)
        if p.gl:
            strip(E[gl - g:gl + 2 * g], S[:3 * g])
            O[gl:gl + g].copy_(S[g:2 * g])
        if p.gh:
            e = gl + self.rows
            strip(E[e - 2 * g:e + g], S[:3 * g])
            O[e - g:e].copy_(S[g:2 * g])

    # ---- distributed driver -----------------------------------------------------------
    def exchange(self, E, p: PassGeom, group=None):
        """Start the ghost exchange; returns the requests to wait on."""
        import torch.distributed as dist
        top, bot = self.send_views(E, p)
        above, below = self.recv_views(E, p)
        # the same order on every rank: NCCL pairs the k-th send to a peer with the peer's
        # k-th receive from this rank (tags are for gloo)
        ops = []
        if top is not None:
            ops.append(dist.P2POp(dist.isend, top, self.up, group, 0))
        if bot is not None:
            ops.append(dist.P2POp(dist.isend, bot, self.down, group, 1))
        if below is not None:
            ops.append(dist.P2POp(dist.irecv, below, self.down, group, 0))
        if above is not None:
            ops.append(dist.P2POp(dist.irecv, above, self.up, group, 1))
        return dist.batch_isend_irecv(ops) if ops else []

    def run(self, x, group=None, bufs=None):
        """T steps of this rank's slab `x` (shape `local_shape()`); every rank of
        `group` calls it together.  Returns the new own rows (a view into `bufs`)."""
        if tuple(x.shape) != self.local_shape():
            raise ValueError(f"slab shape {tuple(x.shape)} != {self.local_shape()}")
        bufs = bufs or self.allocate(x)
        self.load(bufs, x)
        E, O, S = bufs
        for p in self.passes:
            reqs = self.exchange(E, p, group)
            self.compute_core(E, O, p)
            for r in reqs:
                r.wait()
            self.compute_rest(E, O, S, p)
            E, O = O, E
        return self.own(E)


def run_local(plans, xs):
    """Emulates the ranks of one decomposition inside one process: ``plans[k]``
    is rank k's :class:`SlabPlan`, ``xs[k]`` its slab.  Ghosts are copied
    between the ranks' buffers directly, so nothing ever waits on another rank.
    Returns the ranks' new slabs."""
    bufs = [pl.allocate(x) for pl, x in zip(plans, xs)]
    for pl, b, x in zip(plans, bufs, xs):
        pl.load(b, x)
    cur = [0] * len(plans)
    for i in range(len(plans[0].passes)):
        for k, pl in enumerate(plans):
            p = pl.passes[i]
            above, below = pl.recv_views(bufs[k][cur[k]], p)
            if above is not None:
                up = plans[pl.up]
                above.copy_(up.send_views(bufs[pl.up][cur[pl.up]], up.passes[i])[1])
            if below is not None:
                dn = plans[pl.down]
                below.copy_(dn.send_views(bufs[pl.down][cur[pl.down]], dn.passes[i])[0])
        for k, pl in enumerate(plans):
            p = pl.passes[i]
            E, O, S = bufs[k][cur[k]], bufs[k][1 - cur[k]], bufs[k][2]
            pl.compute_core(E, O, p)
            pl.compute_rest(E, O, S, p)
            cur[k] = 1 - cur[k]
    return [pl.own(b[c]) for pl, b, c in zip(plans, bufs, cur)]
