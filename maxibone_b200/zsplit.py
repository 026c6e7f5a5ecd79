"""One volume split into z-slabs over several GPUs, one process per GPU.

The reference's only multi-device code cuts a host volume into blocks and
exchanges their halos through host memory on every repetition
(src/lib/cpp/gpu/diffusion.cc:952-953,1013-1073).  Here each rank keeps its
z-slab of the field on its own GPU for the whole run:

* rank i owns the core planes [z0_i, z1_i) and holds them with H = k x radius
  halo planes on each side that is not the volume's edge;
* the repetitions run in rounds of k: a round is one library call over the
  extended slab (maxi_diffusion_device_ex) that starts from the slab's field,
  narrows its plane window by `radius` per repetition on cut sides, and writes
  the FP32 field of the planes it still holds exactly -- the core after k
  repetitions, since a plane's value after k repetitions depends only on planes
  within k x radius of it;
* between rounds every rank sends the H core planes next to each neighbour and
  receives the neighbour's into its halo: one grouped send/receive per
  neighbour (torch.distributed P2P: NCCL over NVLink on GPUs, gloo on CPU
  tensors), H x ny x nx x 4 bytes per side and round.

k x radius is never thicker than the thinnest slab, so halos only ever come
from direct neighbours; within that, split_plan picks k from an estimate of
the planes computed and the per-round field passes.  FP32 results equal the single-volume form bit for bit (the core's
planes see the same inputs in the same order); the 16-bit forms restart each
round from the FP32 field (rounded to the storage type).

The compute step is a callable, so that the bookkeeping runs unchanged on CPU
ranks in the tests (with a CPU restatement of the step) and on GPUs with
:func:`library_step`.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _lib


def _device_bitpack(mask: torch.Tensor, stream) -> torch.Tensor:
    """The diffusion's mask (set where > 0) as bit-packed words."""
    from .device import bitpack
    with torch.cuda.stream(stream):
        binary = (mask > 0).to(torch.uint8)
    return bitpack(binary, stream=stream)


@dataclass(frozen=True)
class SplitPlan:
    """Slab bounds of every rank and the rounds' repetition count."""

    nz: int
    radius: int
    reps: int
    bounds: tuple  # ((z0, z1), ...) per rank
    k: int         # repetitions per round

    @property
    def halo(self) -> int:
        return min(self.nz, self.k * self.radius)

    def extended(self, rank: int) -> tuple:
        """Planes [e0, e1) the rank holds: its core plus the halos of its cut sides."""
        z0, z1 = self.bounds[rank]
        return (max(0, z0 - self.halo) if z0 > 0 else 0, min(self.nz, z1 + self.halo) if z1 < self.nz else self.nz)

    @property
    def rounds(self) -> int:
        return max(1, -(-self.reps // self.k))


def split_plan(nz: int, world: int, radius: int, reps: int, k: int | None = None,
               round_cost: float = 0.75) -> SplitPlan:
    """Balanced contiguous z-slabs for `world` ranks and the repetitions per
    round.  Raises ValueError when a slab would be thinner than `radius` (the
    halo of one repetition would have to come from beyond a neighbour).

    k (when not given): a round of k repetitions computes on average
    S + (k + 1) r planes per repetition on a slab of S planes with two cut
    sides (its windows shrink by r per repetition), and exchanges k r planes
    per side -- the same bytes per repetition for every k -- so small rounds
    compute less, while each round also starts from and writes back the FP32
    field over its S + 2 k r planes: `round_cost` is that work per plane
    relative to one repetition's (0.75 follows the FP32 form's slab rounds run
    one after another on one B200, 1024^3, radius 32: for 2 slabs 1.45 / 1.49 /
    1.50 times the single volume's work at k = 2 / 3 / 4, for 4 slabs 1.94 /
    1.78 at k = 1 / 2, for 8 slabs 2.26 / 2.17 at k = 1 / 2).  k minimises
    (S + (k + 1) r) + round_cost (S + 2 k r) / k."""
    if world < 1 or nz < world:
        raise ValueError(f"cannot split {nz} planes over {world} ranks")
    base, extra = divmod(nz, world)
    bounds, z = [], 0
    for i in range(world):
        t = base + (1 if i < extra else 0)
        bounds.append((z, z + t))
        z += t
    thin = min(z1 - z0 for z0, z1 in bounds)
    if world > 1 and radius > thin:
        raise ValueError(f"slabs of {thin} planes are thinner than the kernel radius {radius}: use fewer ranks")
    k_max = max(1, reps) if world == 1 else max(1, min(max(1, reps), thin // max(1, radius)))
    if k is None:
        if world == 1:
            k = k_max
        else:
            def cost(kk):
                return base + (kk + 1) * radius + round_cost * (base + 2 * kk * radius) / kk
            k = min(range(1, k_max + 1), key=cost)
    k = max(1, min(k, k_max))
    return SplitPlan(nz=nz, radius=radius, reps=reps, bounds=tuple(bounds), k=k)


def library_step(field: str = "f32", flags: int = 0, stream=None):
    """The compute step on this process's GPU: one round of `reps` repetitions
    over an extended slab through maxi_diffusion_device_ex.

    step(mask, kernel, reps, init_field, field_out, output, shrink_lo, shrink_hi)
    with CUDA tensors: mask uint8 [ez, ny, nx]; init_field float32 [ez, ny, nx]
    or None (start from the mask); field_out float32 [ez, ny, nx] or None;
    output uint16 [ez, ny, nx] or None.  With shrinking, the last repetition
    writes only the planes it still computes (the core and up to `radius`
    planes around it).  The step keeps one device workspace per slab shape and
    the slab's mask packed to bits (it is the same every round), so the rounds
    allocate and pack nothing."""
    lib = _lib.lib()
    workspaces, packed = {}, {}

    def step(mask, kernel, reps, init_field, field_out, output, shrink_lo, shrink_hi):
        nz, ny, nx = mask.shape
        k = np.ascontiguousarray(kernel, dtype=np.float32)
        st = stream if stream is not None else torch.cuda.current_stream(mask.device)
        key = (tuple(mask.shape), mask.device)
        if key not in workspaces:
            n_ws = int(lib.maxi_diffusion_workspace_size(nz, ny, nx, _lib.FIELD_TYPES[field]))
            workspaces[key] = torch.empty(n_ws, dtype=torch.uint8, device=mask.device)
        ws = workspaces[key]
        pkey = (mask.data_ptr(), tuple(mask.shape))
        if pkey not in packed:  # one entry per slab; the mask is kept alive with its packed words
            packed[pkey] = (mask, _device_bitpack(mask, st))
        bits = packed[pkey][1]
        _lib.check(lib.maxi_diffusion_device_ex(
            bits.data_ptr(), _lib.MASK_FORMATS["bitpacked"], nz, ny, nx, k.ctypes.data, k.shape[0], int(reps),
            output.data_ptr() if output is not None else None,
            field_out.data_ptr() if field_out is not None else None,
            _lib.FIELD_TYPES[field], flags, ws.data_ptr(), ws.numel(), st.cuda_stream,
            init_field.data_ptr() if init_field is not None else None, int(shrink_lo), int(shrink_hi)))

    return step


class SlabRun:
    """One rank's slab: its extended mask, its field between rounds and the
    round it runs next."""

    def __init__(self, mask_ext: torch.Tensor, kernel, plan: SplitPlan, rank: int, step, want_output: bool):
        self.plan, self.rank, self.step, self.kernel = plan, rank, step, kernel
        self.e0, self.e1 = plan.extended(rank)
        self.z0, self.z1 = plan.bounds[rank]
        ez = self.e1 - self.e0
        if mask_ext.shape[0] != ez:
            raise ValueError(f"rank {rank} needs mask planes [{self.e0}, {self.e1}), got {mask_ext.shape[0]} planes")
        self.mask = mask_ext
        shape = (ez,) + tuple(mask_ext.shape[1:])
        dev = mask_ext.device
        self.field = torch.empty(shape, dtype=torch.float32, device=dev)  # the slab's field between rounds
        self.next = torch.empty(shape, dtype=torch.float32, device=dev)
        self.u16 = torch.empty(shape, dtype=torch.uint16, device=dev) if want_output else None
        self.done = 0

    @property
    def core(self) -> slice:
        return slice(self.z0 - self.e0, self.z1 - self.e0)

    def run_round(self, rnd: int) -> None:
        """Round `rnd`: k repetitions (fewer in the last round) from the slab's
        field (the mask in round 0); afterwards the core holds the volume's values."""
        plan, r = self.plan, self.plan.radius
        kr = min(plan.k, plan.reps - self.done) if plan.reps > 0 else 0
        last = rnd == plan.rounds - 1
        self.step(self.mask, self.kernel, kr, self.field if rnd > 0 else None, self.next,
                  self.u16 if last else None, r if self.e0 > 0 else 0, r if self.e1 < plan.nz else 0)
        self.done += kr
        self.field[self.core].copy_(self.next[self.core])

    def send_planes(self):
        """(to the lower neighbour, to the upper neighbour): the H core planes next
        to each neighbour (None where the core meets the volume's edge).  A
        neighbour exists wherever the core does not reach the edge, even when
        the halo does (then the halo holds the neighbour's whole core)."""
        h, c = self.plan.halo, self.core
        lo = self.field[c.start:c.start + h] if self.z0 > 0 else None
        hi = self.field[c.stop - h:c.stop] if self.z1 < self.plan.nz else None
        return lo, hi

    def receive_planes(self, lo, hi) -> None:
        """Writes the neighbours' planes into the halos (H planes each: a slab is
        at least H planes thick, so a halo never reaches past a neighbour)."""
        h = self.plan.halo
        if lo is not None:
            self.field[:h].copy_(lo)
        if hi is not None:
            self.field[self.field.shape[0] - h:].copy_(hi)

    def results(self, output=None, field_out=None) -> None:
        if output is not None:
            output.copy_(self.u16[self.core])
        if field_out is not None:
            field_out.copy_(self.field[self.core])


def _exchange(slab: SlabRun, world: int, group=None) -> None:
    """The halo exchange between rounds: one grouped send / receive per
    neighbour (batch_isend_irecv: NCCL over NVLink for CUDA tensors, gloo on CPU)."""
    import torch.distributed as dist

    rank = slab.rank
    lo, hi = slab.send_planes()
    ops, got_lo, got_hi = [], None, None
    if lo is not None:
        got_lo = torch.empty_like(lo)
        ops += [dist.P2POp(dist.isend, lo.contiguous(), rank - 1, group=group),
                dist.P2POp(dist.irecv, got_lo, rank - 1, group=group)]
    if hi is not None:
        got_hi = torch.empty_like(hi)
        ops += [dist.P2POp(dist.isend, hi.contiguous(), rank + 1, group=group),
                dist.P2POp(dist.irecv, got_hi, rank + 1, group=group)]
    if ops:
        for req in dist.batch_isend_irecv(ops):
            req.wait()
    slab.receive_planes(got_lo, got_hi)


def diffuse_split(mask_ext: torch.Tensor, kernel, plan: SplitPlan, rank: int, world: int, step,
                  output: torch.Tensor | None = None, field_out: torch.Tensor | None = None, group=None) -> None:
    """Runs the plan's repetitions on this rank's slab.

    mask_ext: uint8 [e1 - e0, ny, nx] tensor of the planes plan.extended(rank);
    output / field_out: uint16 / float32 tensors of the rank's core planes
    [z0, z1) (either may be None).  Every rank of the group calls this with the
    same plan (the exchanges pair up rank by rank)."""
    slab = SlabRun(mask_ext, kernel, plan, rank, step, output is not None)
    for rnd in range(plan.rounds):
        slab.run_round(rnd)
        if rnd < plan.rounds - 1:
            _exchange(slab, world, group)
    slab.results(output, field_out)


def diffuse_slabs_in_process(mask: torch.Tensor, kernel, plan: SplitPlan, step, output=None, field_out=None) -> None:
    """The same split run by one process over all slabs in turn, the exchanges
    done by copies: the split's bookkeeping and the library's slab rounds on a
    single device (no kernel of one slab waits for another's).  mask: the whole
    uint8 volume; output / field_out: whole-volume tensors or None."""
    world = len(plan.bounds)
    slabs = []
    for rank in range(world):
        e0, e1 = plan.extended(rank)
        slabs.append(SlabRun(mask[e0:e1].contiguous(), kernel, plan, rank, step, output is not None))
    for rnd in range(plan.rounds):
        for s in slabs:
            s.run_round(rnd)
        if rnd < plan.rounds - 1:
            sends = [s.send_planes() for s in slabs]
            for i, s in enumerate(slabs):
                s.receive_planes(sends[i - 1][1] if i > 0 else None, sends[i + 1][0] if i < world - 1 else None)
    for rank, s in enumerate(slabs):
        z0, z1 = plan.bounds[rank]
        s.results(output[z0:z1] if output is not None else None, field_out[z0:z1] if field_out is not None else None)


def assign_volumes(shapes, radii, reps, world: int) -> list:
    """Independent volumes of a batch spread over `world` ranks (no collective:
    each rank runs a batch plan of its own volumes).  Greedy longest-first
    packing by estimated work: voxels x repetitions x the tensor-core passes' K
    per output, (128 + 2r) / 128, so heavy volumes are placed first, each on the
    least loaded rank.  Returns one list of volume indices per rank."""
    cost = [float(np.prod(s)) * max(1, int(n)) * (1.0 + 2.0 * r / 128.0) for s, r, n in zip(shapes, radii, reps)]
    loads = [0.0] * world
    out = [[] for _ in range(world)]
    for i in sorted(range(len(cost)), key=lambda i: (-cost[i], i)):
        k = min(range(world), key=lambda w: (loads[w], w))
        out[k].append(i)
        loads[k] += cost[i]
    return [sorted(v) for v in out]
