"""Sharded insert of one input over N ranks (one process per GPU).

The single-GPU insert (tile_kernel insert, replacing the reference's
insert_sequence_kmers_kernel, include/cusbf/detail/kernels.cuh:214-242) ORs
every super-k-mer run's four word masks into its shard.  OR is commutative,
so the work splits over ranks with one exchange step:

1. **Emit.** Rank r takes the windows [r*N/W, (r+1)*N/W) of the input (its
   byte slice overlaps the next by k-1 bytes, so every window is processed
   exactly once) and emits one record (shard, 4 x uint64 masks) per
   super-k-mer run instead of ORing it into a filter.
2. **Route.** Shards are split into W contiguous ranges by their high bits;
   rank r owns range r.  Each rank orders its records by owner and exchanges
   them with one all-to-all (counts first, then records).
3. **Apply.** Each rank ORs the records it received into its own shard range.
4. **Gather (optional).** An all-gather of the shard ranges gives every rank
   the whole filter, bit-identical to one GPU inserting the whole input, so
   queries run on replicas with no exchange.

Per rank this moves about 40 B x R x (W-1)/W^2 bytes of records (R = runs of
the whole input) instead of a partial filter.  Record emission and the OR are
the library's kernels (sbf_emit_runs_async, sbf_apply_runs_async); the
orchestration here uses torch.distributed for the exchange (NCCL on GPUs, gloo
for CPU tests), with TMA multicast nowhere on this path.
"""
from __future__ import annotations

import numpy as np

RECORD_WORDS = 5  # int64 words per routed record: shard, then the four masks


def window_range(n_windows: int, world: int, rank: int) -> tuple[int, int]:
    """Windows [w0, w1) of `n_windows` that rank `rank` of `world` emits."""
    per = -(-n_windows // world) if n_windows else 0
    w0 = min(rank * per, n_windows)
    return w0, min(w0 + per, n_windows)


def byte_slice(n_bytes: int, k: int, world: int, rank: int) -> tuple[int, int]:
    """Input bytes [b0, b1) holding exactly the windows of `window_range`
    (one byte per symbol): the slice overlaps the next rank's by k-1 bytes."""
    n_windows = max(0, n_bytes - k + 1)
    w0, w1 = window_range(n_windows, world, rank)
    if w1 <= w0:
        return 0, 0
    return w0, w1 + k - 1


def shards_per_owner(num_shards: int, world: int) -> int:
    """Shards in each owner's contiguous range (the last range may be short)."""
    return -(-num_shards // world)


def owner_of(shards, num_shards: int, world: int):
    """Owner rank of each shard id (torch tensor or numpy array)."""
    return shards // shards_per_owner(num_shards, world)


def pack_records(shards, masks, torch):
    """(R,) shard ids and (R, 4) uint64 masks -> (R, 5) int64 records."""
    rec = torch.empty((shards.shape[0], RECORD_WORDS), dtype=torch.int64, device=shards.device)
    rec[:, 0] = shards.to(torch.int64)
    rec[:, 1:] = masks.view(torch.int64)
    return rec


def route_records(records, num_shards: int, group, torch, dist):
    """Sends every record to the owner of its shard with one all-to-all and
    returns the records this rank owns ((n, 5) int64 on the same device)."""
    world = dist.get_world_size(group)
    owner = owner_of(records[:, 0], num_shards, world)
    order = torch.argsort(owner, stable=True)
    records = records.index_select(0, order)
    send_counts = torch.bincount(owner, minlength=world).to(torch.int64)
    recv_counts = torch.empty_like(send_counts)
    dist.all_to_all_single(recv_counts, send_counts, group=group)
    sc = [int(x) * RECORD_WORDS for x in send_counts.tolist()]
    rc = [int(x) * RECORD_WORDS for x in recv_counts.tolist()]
    out = torch.empty(sum(rc), dtype=torch.int64, device=records.device)
    dist.all_to_all_single(out, records.reshape(-1).contiguous(), output_split_sizes=rc,
                           input_split_sizes=sc, group=group)
    return out.view(-1, RECORD_WORDS)


def gather_shards(words, num_shards: int, group, torch, dist) -> None:
    """All-gathers every owner's shard range into `words` ((num_shards * 4,)
    int64 view of the whole filter) so that each rank holds the full filter."""
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    per = shards_per_owner(num_shards, world)
    padded = per * world
    if padded == num_shards and dist.get_backend(group) == "nccl":
        mine = words[rank * per * 4:(rank + 1) * per * 4]
        dist.all_gather_into_tensor(words, mine, group=group)
        return
    buf = torch.zeros(padded * 4, dtype=torch.int64, device=words.device)
    lo, hi = rank * per, min((rank + 1) * per, num_shards)
    buf[lo * 4:hi * 4] = words[lo * 4:hi * 4]
    parts = list(buf.view(world, per * 4).unbind(0))
    gathered = [torch.empty_like(p) for p in parts]
    dist.all_gather(gathered, parts[rank].contiguous(), group=group)
    words.copy_(torch.cat(gathered)[:num_shards * 4])


def sharded_insert(filt, d_seq, group=None, gather: bool = True, stream=None,
                   timings: dict | None = None) -> int:
    """Inserts device bytes `d_seq` into `filt` on every rank of `group`
    (each rank passes the same input and a filter of the same size on its own
    GPU): rank r emits the runs of its windows, the records are routed to the
    owners of their shards and ORed there, and with `gather` every rank ends
    with the whole filter.  Returns the valid k-mers this rank emitted.  With
    `timings`, the device milliseconds of the emit, route, apply and gather
    phases are added to it under those keys."""
    import torch
    import torch.distributed as dist

    from . import Filter  # noqa: F401  (the library is loaded by the package)

    ev = []

    def mark():
        if timings is not None:
            e = torch.cuda.Event(enable_timing=True)
            e.record()
            ev.append(e)

    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    k = filt.config.k
    b0, b1 = byte_slice(d_seq.numel(), k, world, rank)
    num_shards = filt.num_shards()
    mark()
    shards, masks, valid = filt.emit_runs(d_seq[b0:b1], stream=stream)
    mark()
    per = shards_per_owner(num_shards, world)
    if world == 1:
        mine_sh, mine_m = shards, masks  # every shard is this rank's
    else:
        mine = route_records(pack_records(shards, masks, torch), num_shards, group, torch, dist)
        mine_sh, mine_m = mine[:, 0].to(torch.int32).contiguous(), mine[:, 1:].contiguous()
    mark()
    # The records come from torch ops on the current stream; the OR runs on
    # `stream`, and the gather reads the words on the current stream again.
    torch.cuda.current_stream().synchronize()
    filt.apply_runs(mine_sh, mine_m, rank * per, min((rank + 1) * per, num_shards),
                    stream=stream)
    filt.synchronize(stream)
    mark()
    if gather and world > 1:
        gather_shards(filt.words().view(torch.int64), num_shards, group, torch, dist)
    mark()
    if timings is not None:
        torch.cuda.synchronize()
        for name, x, y in zip(("emit", "route", "apply", "gather"), ev, ev[1:]):
            timings[name] = timings.get(name, 0.0) + x.elapsed_time(y)
    return valid


def apply_records_host(words: np.ndarray, records: np.ndarray, shard_lo: int,
                       shard_hi: int) -> None:
    """ORs (n, 5) int64 records whose shards lie in [shard_lo, shard_hi) into
    `words` ((num_shards * 4,) uint64) on the host (the CPU form of
    sbf_apply_runs_async, for ranks without a GPU)."""
    sh = records[:, 0].astype(np.int64)
    if sh.size and (sh.min() < shard_lo or sh.max() >= shard_hi):
        raise ValueError("record outside this rank's shard range")
    w = words.reshape(-1, 4)
    np.bitwise_or.at(w, sh, records[:, 1:].view(np.uint64))
