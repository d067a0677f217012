"""Seeded synthetic DNA workloads with the shapes of the benchmark configs.

No public genome is used: the plain-method, genome-scale and ragged workloads
are stood in for by seeded generators with their sizes and value
distributions (GC content, tandem repeats, N runs, diverged interspersed
repeat families, reads with substitution errors, log-normal lengths).

All generators are deterministic functions of their seed (numpy PCG64 on the
CPU).  ``reads_device`` samples reads on a CUDA device with a seeded torch
generator, for the 10^7-10^8 read sets of the large workloads.
"""
from __future__ import annotations

import numpy as np

SEPARATOR = ord("N")
_BASES = np.frombuffer(b"ACGT", dtype=np.uint8)


def _base_lut(gc: float) -> np.ndarray:
    """256-entry byte -> base table with P(C)=P(G)=gc/2, P(A)=P(T)=(1-gc)/2."""
    c = int(round(256 * gc / 2))
    a = int(round(256 * (1 - gc) / 2))
    t = 256 - 2 * c - a
    lut = np.empty(256, dtype=np.uint8)
    lut[:a] = ord("A")
    lut[a:a + c] = ord("C")
    lut[a + c:a + 2 * c] = ord("G")
    lut[a + 2 * c:] = ord("T")
    assert t >= 0
    return lut


def uniform_dna(n: int, seed: int, gc: float = 0.5, rng=None) -> np.ndarray:
    """n i.i.d. bases (uint8 ASCII) with the given GC fraction."""
    rng = rng if rng is not None else np.random.default_rng(seed)
    lut = _base_lut(gc)
    out = np.empty(n, dtype=np.uint8)
    step = 1 << 26
    for i in range(0, n, step):
        m = min(step, n - i)
        out[i:i + m] = lut[rng.integers(0, 256, size=m, dtype=np.uint8)]
    return out


def _mutate(seq: np.ndarray, rate: float, rng) -> np.ndarray:
    """Substitutes each base with a different base with probability `rate`."""
    if rate <= 0 or seq.size == 0:
        return seq
    n_sub = rng.binomial(seq.size, rate)
    if n_sub == 0:
        return seq
    pos = rng.choice(seq.size, size=n_sub, replace=False) if n_sub < seq.size // 4 else \
        np.flatnonzero(rng.random(seq.size) < rate)
    out = seq.copy()
    cur = out[pos]
    code = (cur >> 1) & 3  # A0 C1 T2 G3
    new = (code + rng.integers(1, 4, size=pos.size)) & 3
    out[pos] = np.frombuffer(b"ACTG", dtype=np.uint8)[new]
    return out


def record_lengths(total_bp: int, n_records: int, lo: int, hi: int, seed: int) -> list[int]:
    """n lengths drawn uniformly in [lo, hi], rescaled to sum to total_bp."""
    rng = np.random.default_rng(seed)
    raw = rng.uniform(lo, hi, size=n_records)
    raw = raw / raw.sum() * total_bp
    lens = np.floor(raw).astype(np.int64)
    lens[-1] += total_bp - lens.sum()
    return [int(x) for x in lens]


def _repeat_units(seed: int, n_units: int, unit_len: tuple[int, int], gc: float) -> list[np.ndarray]:
    rng = np.random.default_rng([seed, 0xFA11])
    return [uniform_dna(int(rng.integers(unit_len[0], unit_len[1] + 1)), seed=0, gc=gc, rng=rng)
            for _ in range(n_units)]


def genome_record(index: int, length: int, seed: int, gc: float = 0.41,
                  tandem_frac: float = 0.0, n_run_frac: float = 0.0,
                  interspersed_frac: float = 0.0, n_units: int = 2000,
                  unit_len: tuple[int, int] = (300, 6000),
                  divergence: tuple[float, float] = (0.05, 0.20)) -> np.ndarray:
    """Record `index` of a genome-like workload (seeded by (seed, index)).

    * background: i.i.d. bases at GC fraction `gc`;
    * interspersed repeats: copies of `n_units` repeat units shared by all
      records (seeded by `seed`, lengths uniform in `unit_len`), each copy
      substituted at a divergence drawn from `divergence`, placed until
      `interspersed_frac` of the record is covered;
    * tandem repeats: regions of 100-2000 bp filled with a period-2..200 unit;
    * N runs of 10-1000 bp covering `n_run_frac` of the record.
    """
    rng = np.random.default_rng([seed, index])
    rec = uniform_dna(length, seed=0, gc=gc, rng=rng)

    def place(n_bases_target: int, make_piece):
        covered = 0
        while covered < n_bases_target:
            piece = make_piece()
            if piece.size >= length:
                break
            p = int(rng.integers(0, length - piece.size))
            rec[p:p + piece.size] = piece
            covered += piece.size

    if interspersed_frac > 0:
        units = _repeat_units(seed, n_units, unit_len, gc)
        place(int(interspersed_frac * length),
              lambda: _mutate(units[int(rng.integers(0, n_units))],
                              float(rng.uniform(*divergence)), rng))
    if tandem_frac > 0:
        def tandem():
            period = int(rng.integers(2, 201))
            unit = uniform_dna(period, seed=0, gc=gc, rng=rng)
            return np.resize(unit, int(rng.integers(100, 2001)))
        place(int(tandem_frac * length), tandem)
    if n_run_frac > 0:
        place(int(n_run_frac * length),
              lambda: np.full(int(rng.integers(10, 1001)), SEPARATOR, dtype=np.uint8))
    return rec


def _record_job(args):
    return genome_record(*args[0], **args[1])


def genome_records(total_bp: int, n_records: int, seed: int, gc: float = 0.41,
                   lengths: list[int] | None = None, processes: int = 1,
                   **features) -> list[np.ndarray]:
    """Genome-like records (see genome_record); `processes` > 1 builds them in
    a spawn-context process pool (start it before any CUDA call)."""
    if lengths is None:
        lengths = [total_bp // n_records] * n_records
        lengths[-1] += total_bp - sum(lengths)
    jobs = [((i, L, seed, gc), features) for i, L in enumerate(lengths)]
    if processes > 1 and len(jobs) > 1:
        import multiprocessing as mp

        with mp.get_context("spawn").Pool(min(processes, len(jobs))) as pool:
            return pool.map(_record_job, jobs)
    return [_record_job(j) for j in jobs]


def join_records(records: list[np.ndarray]) -> tuple[np.ndarray, np.ndarray]:
    """Concatenates records with one 'N' separator between consecutive
    records (include/cusbf/normalized_record_batch.hpp:113-121, DNA) and
    returns (bytes, ranges[n, 2] of (offset, length))."""
    n = len(records)
    total = sum(r.size for r in records) + max(n - 1, 0)
    out = np.empty(total, dtype=np.uint8)
    ranges = np.zeros((n, 2), dtype=np.uint64)
    pos = 0
    for i, r in enumerate(records):
        if i:
            out[pos] = SEPARATOR
            pos += 1
        out[pos:pos + r.size] = r
        ranges[i] = (pos, r.size)
        pos += r.size
    return out, ranges


def reads_host(records: list[np.ndarray], n_reads: int, length: int, seed: int,
               sub_rate: float = 0.01, positive_frac: float = 0.5, gc: float = 0.5) -> np.ndarray:
    """(n_reads, length) uint8 reads: a `positive_frac` share sampled from the
    records with substitutions at `sub_rate`, the rest i.i.d. random."""
    rng = np.random.default_rng(seed)
    out = uniform_dna(n_reads * length, seed=0, gc=gc, rng=rng).reshape(n_reads, length)
    n_pos = int(round(n_reads * positive_frac))
    lens = np.array([r.size for r in records], dtype=np.int64)
    w = np.clip(lens - length, 0, None).astype(np.float64)
    rec = rng.choice(len(records), size=n_pos, p=w / w.sum())
    for i in range(n_pos):
        r = records[rec[i]]
        p = int(rng.integers(0, r.size - length + 1))
        out[i] = _mutate(r[p:p + length], sub_rate, rng)
    return out


def lognormal_lengths(n: int, median: float, sigma: float, lo: int, hi: int, seed: int) -> np.ndarray:
    """n integer lengths, log-normal with the given median, clipped to [lo, hi]."""
    rng = np.random.default_rng(seed)
    x = rng.lognormal(mean=np.log(median), sigma=sigma, size=n)
    return np.clip(np.round(x), lo, hi).astype(np.int64)


def reads_device(source, n_reads: int, length: int, seed: int, sub_rate: float = 0.01,
                 positive_frac: float = 0.5, device: str = "cuda"):
    """(n_reads, length) uint8 CUDA tensor of reads: the first
    `positive_frac` share sampled from `source` (a 1-D uint8 CUDA tensor of
    joined records) with substitutions at `sub_rate`, the rest uniform random.
    Deterministic for a given seed, torch version and device type."""
    import torch

    g = torch.Generator(device=device)
    g.manual_seed(seed)
    lut = torch.tensor(list(b"ACGT"), dtype=torch.uint8, device=device)
    sub = torch.tensor(list(b"ACTG"), dtype=torch.uint8, device=device)
    out = torch.empty((n_reads, length), dtype=torch.uint8, device=device)
    n_pos = int(round(n_reads * positive_frac))
    step = 1 << 20
    span = source.numel() - length
    offs = torch.arange(length, device=device, dtype=torch.int64)
    for i in range(0, n_reads, step):
        m = min(step, n_reads - i)
        blk = out[i:i + m]
        blk.copy_(lut[torch.randint(0, 4, (m, length), device=device, generator=g,
                                    dtype=torch.int32).long()])
        p_hi = min(i + m, n_pos)
        if p_hi > i:
            k = p_hi - i
            starts = torch.randint(0, span, (k,), device=device, generator=g, dtype=torch.int64)
            src = source[(starts[:, None] + offs[None, :])]
            mask = torch.rand((k, length), device=device, generator=g) < sub_rate
            shift = torch.randint(1, 4, (k, length), device=device, generator=g, dtype=torch.int32)
            code = ((src >> 1) & 3).to(torch.int32)
            mutated = sub[((code + shift) & 3).long()]
            blk[:k] = torch.where(mask, mutated, src)
    return out


def ragged_reads_device(source, rec_off: np.ndarray, rec_len: np.ndarray, lengths: np.ndarray,
                        seed: int, positive_frac: float, sub_rate: float, gc: float,
                        device: str = "cuda", chunk_bytes: int = 1 << 26):
    """Reads of the given lengths, back to back in one uint8 CUDA tensor, and
    their (offset, bytes) ranges.  A `positive_frac` share (chosen at random)
    is copied from `source` (records at rec_off/rec_len, picked with
    probability proportional to length) with substitutions at `sub_rate`;
    the rest are i.i.d. bases at the given GC fraction."""
    import torch

    rng = np.random.default_rng(seed)
    n = lengths.size
    lengths = lengths.astype(np.int64)
    offsets = np.zeros(n, np.int64)
    if n > 1:
        offsets[1:] = np.cumsum(lengths)[:-1]
    total = int(lengths.sum())
    positive = rng.random(n) < positive_frac
    rec = rng.choice(rec_len.size, size=n, p=rec_len / rec_len.sum())
    room = np.maximum(rec_len[rec] - lengths, 0)
    starts = rec_off[rec] + np.floor(rng.random(n) * (room + 1)).astype(np.int64)
    starts = np.minimum(starts, source.numel() - lengths)
    g = torch.Generator(device=device)
    g.manual_seed(seed)
    lut = torch.from_numpy(_base_lut(gc)).to(device)
    sub = torch.tensor(list(b"ACTG"), dtype=torch.uint8, device=device)
    out = torch.empty(total, dtype=torch.uint8, device=device)
    d_len = torch.from_numpy(lengths).to(device)
    d_off = torch.from_numpy(offsets).to(device)
    d_start = torch.from_numpy(starts).to(device)
    d_pos = torch.from_numpy(positive).to(device)
    ends = offsets + lengths
    i = 0
    while i < n:
        j = int(np.searchsorted(ends, offsets[i] + chunk_bytes, side="right"))
        j = max(j, i + 1)
        b0, b1 = int(offsets[i]), int(ends[j - 1])
        nb = b1 - b0
        rid = torch.repeat_interleave(torch.arange(i, j, device=device), d_len[i:j])
        rel = torch.arange(b0, b1, device=device, dtype=torch.int64) - d_off[rid]
        src = source[d_start[rid] + rel]
        code = ((src >> 1) & 3).to(torch.int32)
        shift = torch.randint(1, 4, (nb,), device=device, generator=g, dtype=torch.int32)
        mutated = torch.where(torch.rand(nb, device=device, generator=g) < sub_rate,
                              sub[((code + shift) & 3).long()], src)
        rand = lut[torch.randint(0, 256, (nb,), device=device, generator=g,
                                 dtype=torch.int32).long()]
        out[b0:b1] = torch.where(d_pos[rid], mutated, rand)
        i = j
    return out, np.stack([offsets, lengths], axis=1).astype(np.uint64)
