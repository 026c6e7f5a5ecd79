"""The z-slab split of one volume over several ranks (maxibone_b200.zsplit) on
CPU: two and three `gloo` ranks (127.0.0.1), each running the split's rounds on
its extended slab with a CPU restatement of the library's slab step, and
exchanging halos with its neighbours between rounds.  The assembled FP32 field
must equal the single-volume oracle bit for bit: the halo bookkeeping, slab
bounds and shrinking windows are exact or they are not."""
import datetime
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from maxibone_b200.zsplit import split_plan


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def oracle_step(mask, kernel, reps, init_field, field_out, output, shrink_lo, shrink_hi):
    """The slab step on CPU tensors: `reps` repetitions over the whole extended
    slab with a zero boundary at its ends (no window shrinking: the planes near
    a cut side are wrong afterwards, the core is exact either way)."""
    import oracle

    m = mask.numpy()
    if init_field is None:
        f = oracle.diffusion_in_memory(m, kernel, reps)[1] if reps > 0 else (m > 0).astype(np.float32)
    else:
        f = oracle.diffusion_from_field(init_field.numpy(), m, kernel, reps)
    field_out.copy_(torch.from_numpy(f))
    if output is not None:
        q = np.clip(np.floor(f * np.float32(65535.0)), 0, 65535).astype(np.uint16)
        output.copy_(torch.from_numpy(q.view(np.int16)).view(torch.uint16))


def _case():
    from maxibone_b200.kernels import gauss_kernel
    from maxibone_b200.synthetic import spheres_mask
    mask = spheres_mask((37, 12, 20), 6, (2, 5), seed=3)
    return mask, gauss_kernel(1.0).astype(np.float32)  # radius 4


def _rank(rank, world, port, reps, k, queue):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch.distributed as dist

    from maxibone_b200.zsplit import diffuse_split
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    mask, kernel = _case()
    plan = split_plan(mask.shape[0], world, kernel.shape[0] // 2, reps, k)
    e0, e1 = plan.extended(rank)
    z0, z1 = plan.bounds[rank]
    field = torch.empty((z1 - z0,) + mask.shape[1:], dtype=torch.float32)
    out = torch.empty((z1 - z0,) + mask.shape[1:], dtype=torch.uint16)
    diffuse_split(torch.from_numpy(np.ascontiguousarray(mask[e0:e1])), kernel, plan, rank, world, oracle_step,
                  output=out, field_out=field)
    dist.barrier()
    dist.destroy_process_group()
    queue.put((rank, z0, field.numpy(), out.view(torch.int16).numpy().view(np.uint16), plan.rounds))


@pytest.mark.parametrize("world,reps,k", [(2, 9, None), (3, 4, None)])
def test_split_equals_single_volume_bit_for_bit(world, reps, k):
    import oracle

    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, reps, k, queue)) for r in range(world)]
    for p in procs:
        p.start()
    got = [queue.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mask, kernel = _case()
    want_u16, want = oracle.diffusion_in_memory(mask, kernel, reps)
    field = np.empty_like(want)
    u16 = np.empty_like(want_u16)
    rounds = set()
    for rank, z0, f, o, nr in got:
        field[z0:z0 + f.shape[0]] = f
        u16[z0:z0 + o.shape[0]] = o
        rounds.add(nr)
    assert max(rounds) > 1  # the case exercises exchanges
    np.testing.assert_array_equal(field, want)
    np.testing.assert_array_equal(u16, want_u16)


def test_split_plan_bounds_and_rounds():
    p = split_plan(1024, 8, 32, 100, k=4)
    assert p.bounds[0] == (0, 128) and p.bounds[-1] == (896, 1024)
    assert p.k == 4 and p.halo == 128 and p.rounds == 25
    assert p.extended(0) == (0, 256) and p.extended(3) == (256, 640) and p.extended(7) == (768, 1024)
    # the chosen round length: thin slabs exchange every repetition, thick ones
    # less often (fewer round starts), never beyond the slab thickness
    assert split_plan(1024, 8, 32, 100).k == 2
    assert split_plan(1024, 4, 32, 100).k == 2
    assert split_plan(1024, 2, 32, 100, round_cost=4.0).k > 4
    assert split_plan(1024, 2, 32, 100, k=40).k == 16
    q = split_plan(37, 3, 4, 7, 2)
    assert [b[1] - b[0] for b in q.bounds] == [13, 12, 12] and q.k == 2 and q.rounds == 4
    assert split_plan(100, 1, 32, 100).k == 100  # one rank: a single round, no exchange
    with pytest.raises(ValueError):
        split_plan(60, 4, 32, 10)  # 15-plane slabs are thinner than radius 32


@pytest.mark.parametrize("world,reps,k", [(2, 9, None), (3, 7, 2), (2, 5, 1), (3, 4, None), (4, 6, 1), (2, 1, None),
                                          (3, 0, None)])
def test_split_rounds_in_one_process_equal_single_volume(world, reps, k):
    # The same bookkeeping with the exchanges done by copies in one process
    # (the form the single-GPU test runs with the library's step).
    import oracle
    from maxibone_b200.zsplit import diffuse_slabs_in_process

    mask, kernel = _case()
    plan = split_plan(mask.shape[0], world, kernel.shape[0] // 2, reps, k)
    out = torch.empty(mask.shape, dtype=torch.uint16)
    field = torch.empty(mask.shape, dtype=torch.float32)
    diffuse_slabs_in_process(torch.from_numpy(mask), kernel, plan, oracle_step, output=out, field_out=field)
    want_u16, want = oracle.diffusion_in_memory(mask, kernel, reps)
    np.testing.assert_array_equal(field.numpy(), want)
    np.testing.assert_array_equal(out.view(torch.int16).numpy().view(np.uint16), want_u16)


def test_assign_volumes_balances_the_batch():
    from maxibone_b200.synthetic import batch_shapes
    from maxibone_b200.zsplit import assign_volumes
    specs = batch_shapes(64, seed=0)
    shapes = [s for s, _, _ in specs]
    radii = [int(round(4 * sig)) for _, sig, _ in specs]
    for world in (1, 2, 4, 8):
        parts = assign_volumes(shapes, radii, [50] * 64, world)
        assert sorted(i for p in parts for i in p) == list(range(64))
        work = [sum(np.prod(shapes[i]) * (1 + 2 * radii[i] / 128) for i in p) for p in parts]
        # greedy longest-first: within the largest single volume of the mean
        biggest = max(np.prod(s) * (1 + 2 * r / 128) for s, r in zip(shapes, radii))
        assert max(work) - min(work) <= biggest
