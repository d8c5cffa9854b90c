"""Multi-GPU decomposition of the vlp4d path: one process per GPU.

The reference distributes one run of vlp4d_mpi over MPI ranks:
Distrib::createDecomposition cuts the 4D grid by recursive bisection
(miniapps/vlp4d_mpi/thrust/Communication.cpp:10-124), Distrib::exchangeHalo
packs, sends and unpacks the halo regions around every rank's block
(Communication.cpp:471-562, called from Timestep.hpp:39), and field_reduce
sums the rank-local densities with MPI_Allreduce (Field.cpp:31-40, called
from Timestep.hpp:59,88).  Here a run is cut along vy only:

* x, y and vx sweeps never leave a vy plane, so only the vy sweep needs
  planes of other ranks: `halo` planes on each side of the owned ones;
* vy is the slowest index of the layout_left array, so a rank's halo on
  each side is ONE contiguous block of the f buffer (halo*nvx*ny*nx
  elements) that NCCL receives in place, and the neighbour's edge planes
  are one contiguous block that NCCL sends from where they lie: there is no
  pack or unpack step;
* rho is the sum of the ranks' moments over their owned planes: an
  all-reduce of nx*ny doubles, after which every rank solves the same field
  and computes the same diagnostics.

`SlabRun` advances one rank's slab through the stage entry points of a
slab context (vlp4d_ctx_create_slab) and hands the two communication steps
to a communicator: `TorchComm` (torch.distributed, NCCL between GPUs, gloo
on CPU) for one process per rank, or `LocalComm`, which runs several ranks'
slabs in one process (its exchanges are copies between their buffers).

The batched ensemble shards with no communication at all: each rank runs
its share of the members (`partition_members`).
"""
from __future__ import annotations

import math
from typing import Iterator, List, Sequence, Tuple

# Communication requests a SlabRun step yields to its driver.
REDUCE_RHO = "reduce_rho"   # sum rho over the ranks, in place, before the field solve
HALO_START = "halo_start"   # start filling the halo planes of an f buffer from the neighbours
HALO_WAIT = "halo_wait"     # the halo planes of that buffer must be in place from here on


def partition_vy(nvy: int, world: int) -> List[Tuple[int, int]]:
    """Contiguous, balanced vy ranges: rank r owns planes [ivy0, ivy0 + n)
    with n = nvy // world or one more (the first nvy % world ranks)."""
    if world < 1 or nvy < world:
        raise ValueError(f"cannot cut {nvy} vy planes over {world} ranks")
    base, extra = divmod(nvy, world)
    out, start = [], 0
    for r in range(world):
        n = base + (1 if r < extra else 0)
        out.append((start, n))
        start += n
    return out


def halo_for_shift(max_shift_cells: float) -> int:
    """Halo planes that a vy shift of up to max_shift_cells cells
    (max |dt * Ey| / dvy) needs: floor(|d|) + 3, at least 3."""
    return int(math.floor(abs(max_shift_cells))) + 3


def neighbours(rank: int, world: int) -> Tuple[int, int]:
    """(left, right): the ranks owning the planes just below and just above
    this rank's (periodic in vy)."""
    return (rank - 1) % world, (rank + 1) % world


def halo_views(f, nloc: int, halo: int):
    """Views of an f buffer shaped (nloc + 2*halo, ...): (left halo, right
    halo, first `halo` owned planes, last `halo` owned planes).  Each is a
    contiguous block."""
    return f[:halo], f[halo + nloc:], f[halo:2 * halo], f[nloc:nloc + halo]


class TorchComm:
    """The two exchanges of a slab step over torch.distributed: NCCL
    between GPUs (one process per GPU), gloo between CPU processes.

    The rho all-reduce is issued first and waited for on the current stream
    (the field solve needs it); the halo send/recv pairs are issued next and
    waited for only before the vy sweep, so that their transfer overlaps
    the field solve, the diagnostic and the v-table build."""

    def __init__(self, group=None):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self._pending = []
        self.halo_bytes = 0  # bytes this rank received into halos so far

    def _global(self, r):
        return self.dist.get_global_rank(self.group, r) if self.group is not None else r

    def reduce_rho(self, rho):
        if self.world > 1:
            self.dist.all_reduce(rho, op=self.dist.ReduceOp.SUM, group=self.group)

    def halo_start(self, f, nloc, halo):
        lh, rh, first, last = halo_views(f, nloc, halo)
        self.halo_bytes += 2 * lh.numel() * lh.element_size()
        if self.world == 1:  # periodic in vy: this rank is its own neighbour
            lh.copy_(last)
            rh.copy_(first)
            return
        left, right = neighbours(self.rank, self.world)
        P2POp = self.dist.P2POp
        # Both sides issue: receive the left halo, receive the right halo,
        # send the last planes to the right neighbour, send the first planes
        # to the left one.  With two ranks both messages go to the same
        # peer and match in issue order: the first received block is the
        # peer's last planes (this rank's left halo), the second its first
        # planes.  Tags keep the pairing explicit where the backend uses them.
        ops = [P2POp(self.dist.irecv, lh, self._global(left), self.group, tag=1),
               P2POp(self.dist.irecv, rh, self._global(right), self.group, tag=2),
               P2POp(self.dist.isend, last, self._global(right), self.group, tag=1),
               P2POp(self.dist.isend, first, self._global(left), self.group, tag=2)]
        self._pending = self.dist.batch_isend_irecv(ops)

    def halo_wait(self, f):
        for w in self._pending:
            w.wait()
        self._pending = []

    def serve(self, requests: Iterator):
        """Runs one rank's step generator to the end, serving its requests."""
        for req in requests:
            kind = req[0]
            if kind == REDUCE_RHO:
                self.reduce_rho(req[1])
            elif kind == HALO_START:
                self.halo_start(*req[1:])
            elif kind == HALO_WAIT:
                self.halo_wait(req[1])
            else:
                raise ValueError(f"unknown request {kind}")


class LocalComm:
    """Several ranks' slabs in one process: the generators of all ranks
    advance in lockstep and every request is served across them (rho summed
    in rank order, halos copied between the ranks' buffers).  Used to run
    the decomposition on one GPU and in tests."""

    def serve(self, runs: Sequence["SlabRun"], gens: Sequence[Iterator]):
        world = len(gens)
        while True:
            reqs = []
            for g in gens:
                reqs.append(next(g, None))
            if all(r is None for r in reqs):
                return
            if any(r is None for r in reqs):
                raise RuntimeError("ranks' step sequences diverged")
            kind = reqs[0][0]
            if any(r[0] != kind for r in reqs):
                raise RuntimeError(f"ranks' requests diverged: {[r[0] for r in reqs]}")
            if kind == REDUCE_RHO:
                total = reqs[0][1].clone()
                for r in reqs[1:]:
                    total += r[1]
                for r in reqs:
                    r[1].copy_(total)
            elif kind == HALO_START:
                for rank, r in enumerate(reqs):
                    f, nloc, halo = r[1:]
                    left, right = neighbours(rank, world)
                    lh, rh, _, _ = halo_views(f, nloc, halo)
                    fl, nl, hl = reqs[left][1:]
                    fr, nr, hr = reqs[right][1:]
                    if halo > nl or halo > nr:
                        raise ValueError(f"halo of {halo} planes is wider than a neighbour's owned planes")
                    lh.copy_(fl[hl + nl - halo:hl + nl])  # the left neighbour's last owned planes
                    rh.copy_(fr[hr:hr + halo])            # the right neighbour's first owned planes
            elif kind != HALO_WAIT:
                raise ValueError(f"unknown request {kind}")


class SlabRun:
    """One rank's share of a vlp4d run cut into vy slabs.

    `ctx` is a slab context (Context(dom, dtype, slab=(ivy0, nloc, halo)))
    or an object with the same stage methods; `fa`, `fb` its two f buffers.
    The step methods are generators: they launch the stages of the time loop
    on the context and yield a request wherever the ranks must communicate
    (REDUCE_RHO, HALO_START, HALO_WAIT); the communicator serves them.  The
    stages and their order are those of vlp4d_steps (timestep.hpp:14-67 per
    step, the closing x/y half step of one step joined with the opening one
    of the next where the context supports it), with the two exchanges
    between them."""

    def __init__(self, ctx, dt: float, join_xy=None):
        self.ctx = ctx
        self.dt = float(dt)
        self.nloc = ctx.nvy_local
        self.halo = ctx.halo
        # As vlp4d_steps: join the x/y half steps of consecutive steps where
        # the library does (vlp4d_steps_joins_xy).
        if join_xy is None:
            join_xy = bool(getattr(ctx, "joins_xy", False))
        self.join_xy = join_xy
        self.fa = ctx.empty_f()
        self.fb = ctx.empty_f()
        self.state = self.fa  # the buffer holding the current state

    # -- the field of the current state
    def _field(self, it):
        yield (REDUCE_RHO, self.ctx.rho)
        self.ctx.field_poisson()
        self.ctx.diags_compute(it)

    def start(self, it: int = 0):
        """Moment of the current state, summed over the ranks, field solve and
        diagnostic `it` (vlp4d.cpp:58-61)."""
        self.ctx.field_rho(self.state)
        yield from self._field(it)

    def steps(self, iter0: int, nsteps: int):
        """nsteps Strang steps from self.state, diagnostics iter0 ..; the final
        state ends in self.state."""
        ctx, dt = self.ctx, self.dt
        cur = self.state
        oth = self.fb if cur is self.fa else self.fa
        ctx.advect_xy_moment(cur, oth, 0.5 * dt)  # timestep.hpp:17-28 of the first step
        cur, oth = oth, cur
        for k in range(nsteps):
            yield (REDUCE_RHO, ctx.rho)
            yield (HALO_START, cur, self.nloc, self.halo)
            ctx.field_poisson()  # timestep.hpp:30-38
            ctx.diags_compute(iter0 + k)
            yield (HALO_WAIT, cur)
            ctx.advect_vxvy(cur, oth, dt)  # timestep.hpp:40-48, reads cur's halos
            cur, oth = oth, cur
            if k + 1 == nsteps:
                break
            # timestep.hpp:50-58 of step k and :17-28 of step k+1.
            if not self._xyxy(cur, oth):
                ctx.advect_xy(cur, oth, 0.5 * dt)
                cur, oth = oth, cur
                ctx.advect_xy_moment(cur, oth, 0.5 * dt)
            cur, oth = oth, cur
        ctx.advect_xy(cur, oth, 0.5 * dt)  # timestep.hpp:50-58 of the last step
        self.state = oth

    def _xyxy(self, cur, oth) -> bool:
        if not self.join_xy:
            return False
        try:
            self.ctx.advect_xyxy(cur, oth, 0.5 * self.dt)
            return True
        except Exception as e:  # the one-pass kernel does not fit: two x/y passes
            if getattr(e, "code", None) != 3:  # VLP4D_ERR_UNSUPPORTED
                raise
            self.join_xy = False
            return False


def run_distributed(run: SlabRun, comm: TorchComm, nsteps: int, iter0: int = 1, start: bool = True):
    """Initial field (diagnostic iter0 - 1) when `start`, then nsteps steps of
    this rank, serving the exchanges with `comm`."""
    if start:
        comm.serve(run.start(iter0 - 1))
    comm.serve(run.steps(iter0, nsteps))


def run_local(runs: Sequence[SlabRun], nsteps: int, iter0: int = 1, start: bool = True):
    """All ranks' slabs in this process, in lockstep (LocalComm)."""
    comm = LocalComm()
    if start:
        comm.serve(runs, [r.start(iter0 - 1) for r in runs])
    comm.serve(runs, [r.steps(iter0, nsteps) for r in runs])


def partition_members(members: Sequence, world: int, cost=None) -> List[List[int]]:
    """Member indices of each rank for an ensemble split over `world` ranks
    with no communication: members are dealt, largest first, to the rank with
    the least work so far (cost(member), default its cell count), ties to
    the lower rank.  Deterministic, so every rank computes the same split."""
    if world < 1:
        raise ValueError("world must be at least 1")
    if cost is None:
        def cost(m):
            n = m.n if hasattr(m, "n") else m
            return n[0] * n[1] * n[2] * n[3]
    order = sorted(range(len(members)), key=lambda i: (-cost(members[i]), i))
    load = [0] * world
    parts: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += cost(members[i])
    return [sorted(p) for p in parts]
