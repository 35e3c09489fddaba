"""Right-hand-side sharding across ranks (one process per GPU).

Source positions (and with them their 12 spin-colour columns and their
Pi_mu_nu) are independent on a replicated gauge field, so they are dealt
round-robin to ranks; each rank solves and contracts its own sources and the
only communication is the final gather of the results (and, for timing, the
maximum of the ranks' step times).  Works with any torch.distributed backend:
NCCL over NVLink for CUDA tensors, gloo on the host.
"""
import torch
import torch.distributed as dist


def world_rank(group=None):
    if not dist.is_available() or not dist.is_initialized():
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def my_items(items, world, rank):
    """Round-robin share of `items` for `rank` (the same on every rank)."""
    return list(items)[rank::world]


def run_sharded(items, compute, group=None):
    """compute(item) -> picklable result on this rank's share; returns the
    results of all ranks as {item: result} on every rank."""
    world, rank = world_rank(group)
    mine = {it: compute(it) for it in my_items(items, world, rank)}
    if world == 1:
        return mine
    gathered = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    out = {}
    for part in gathered:
        out.update(part)
    return {it: out[it] for it in items}


def gather_tensors(local, n_items, group=None):
    """All-gather of per-item tensors of one shape and dtype produced with
    my_items(range(n_items)): returns a tensor [n_items, *shape] in item
    order on every rank.  Ranks with fewer items pad with zeros, so every
    rank contributes the same number of rows to the collective."""
    world, rank = world_rank(group)
    if world == 1:
        return torch.stack(local)
    per = (n_items + world - 1) // world
    shape, dtype, device = local[0].shape, local[0].dtype, local[0].device
    buf = torch.zeros((per,) + tuple(shape), dtype=dtype, device=device)
    for k, t in enumerate(local):
        buf[k] = t
    out = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(out, buf, group=group)
    rows = []
    for it in range(n_items):
        rows.append(out[it % world][it // world])
    return torch.stack(rows)


def broadcast_field(field, n, device=None, group=None, src=0):
    """Rank `src` holds `field` (n doubles, numpy or None elsewhere); every
    rank returns it as a numpy array after one broadcast (over NVLink with
    NCCL when `device` is a CUDA device).  The gauge field is generated once
    and sent, instead of being generated on every rank."""
    import numpy as np
    world, rank = world_rank(group)
    if world == 1:
        return np.ascontiguousarray(field, np.float64)
    if rank == src:
        t = torch.from_numpy(np.ascontiguousarray(field, np.float64)).to(device or "cpu")
    else:
        t = torch.empty(n, dtype=torch.float64, device=device or "cpu")
    dist.broadcast(t, src, group=group)
    return t.cpu().numpy()


def pi_sharded(sources, compute, group=None):
    """Pi_mu_nu for every source position, computed by the rank that owns it
    (round-robin) and gathered: compute(source) -> (conn tensor of 32*V
    doubles, contact tensor of 8 doubles) on this rank's device; returns
    (conn [n_sources, 32*V], contact [n_sources, 8]) on every rank."""
    world, rank = world_rank(group)
    if len(sources) < world:  # the same decision on every rank, before any collective
        raise ValueError(f"{len(sources)} source positions for {world} ranks")
    mine = my_items(range(len(sources)), world, rank)
    conns, contacts = [], []
    for i in mine:
        c, ct = compute(sources[i])
        conns.append(c)
        contacts.append(ct)
    return gather_tensors(conns, len(sources), group), gather_tensors(contacts, len(sources), group)


def max_over_ranks(value, device=None, group=None):
    """Maximum of a float over ranks (step times are reported this way)."""
    world, _ = world_rank(group)
    if world == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())
