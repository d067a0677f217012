"""Benchmark of the Super Bloom engine: k-mers/s insert + query at k=31.

    python bench.py [--gpus N] [--steps K] [--warmup W]
                    [--config c3|c2|c1|c4|c5|fastx|sharded|configs|fpr]
                    [--impl ours|reference] [--scale S]

Workload (default `c3`, the configuration the metric is quoted on): a seeded
synthetic genome of 3.1 Gbp in 24 records of 46-248 Mbp at GC 41%, ~50%
covered by diverged copies (5-20%) of 2000 repeat units of 300 bp-6 kbp and
5% by tandem repeats, inserted into a filter of 21.4 bits per k-mer (2^36
bits, 8 GiB); then 100M reads of 150 bp, half sampled from the genome with 1%
substitutions and half uniform random, are queried.  k=31, s=28, m=16, 4
hashes.  No public dataset is used; the inputs are seeded stand-ins with the
configuration's shapes.

One step = clear the filter, insert every genome record (one launch over the
records joined with separator bases), query every read (one launch over the
reads joined with separators; one result byte per window).  Inputs stay
resident in HBM; they are far larger than the 126 MB L2, so no flush is
needed between steps.  `value` = valid k-mers inserted + queried per second
of device time (CUDA events on the launching stream), summed over ranks
(weak scaling: every rank holds its own filter and workload, seeded by
rank), over the max time across ranks.

`e2e` times the same step through the public host API with pinned host
buffers: sbf_insert_sequence (host genome) + sbf_contains_sequence (host
reads -> host result bytes), so every host<->device copy is inside it.

`--impl reference` times the reference cuSBF path's own arithmetic on the
host cores (oracle/_ref, built from the reference headers; the C oracle
port when that is absent) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "k-mers/s insert+query (3.1 Gbp, k=31); ragged-batch & served p50/p99 vs plain"
K, S, M, H = 31, 28, 16, 4


# ---------------------------------------------------------------------------
# Workloads
# ---------------------------------------------------------------------------

def workload_spec(name: str, scale: float) -> dict:
    if name == "c3":
        return dict(name="plain-large", genome_bp=int(3.1e9 * scale), n_records=24,
                    rec_lo=int(46e6 * scale), rec_hi=int(248e6 * scale), gc=0.41,
                    features=dict(interspersed_frac=0.5, tandem_frac=0.05),
                    bits_per_kmer=21.4, n_reads=int(100e6 * scale), read_len=150,
                    positive_frac=0.5, sub_rate=0.01)
    if name == "c2":
        return dict(name="plain-genome-small", genome_bp=int(100e6 * scale), n_records=6,
                    rec_lo=int(13e6 * scale), rec_hi=int(21e6 * scale), gc=0.36,
                    features=dict(tandem_frac=0.03, n_run_frac=0.001),
                    bits_per_kmer=21.4, n_reads=int(20e6 * scale), read_len=150,
                    positive_frac=0.5, sub_rate=0.01,
                    l2="filter 256 MiB (about 2x L2); query input 3 GB, larger than L2 "
                       "(no flush)")
    if name == "c1":
        return dict(name="plain-small", genome_bp=int(2e6 * scale), n_records=1,
                    rec_lo=int(2e6 * scale), rec_hi=int(2e6 * scale), gc=0.5, features={},
                    bits_per_kmer=85.7, n_reads=0, read_len=150, positive_frac=0.5,
                    sub_rate=0.0, fresh_query_bp=int(2e6 * scale),
                    l2="L2-resident by design: 32 MiB filter and 2-4 MB inputs stay in L2 "
                       "between steps (no flush); its roofline is the L2 bandwidth")
    raise SystemExit(f"unknown config {name}")


def build_host_genome(spec: dict, seed: int):
    from workloads.synthetic import (genome_records, join_records, record_lengths,
                                      uniform_dna)

    if spec["n_records"] == 1 and not spec["features"]:
        recs = [uniform_dna(spec["genome_bp"], seed=seed, gc=spec["gc"])]
    else:
        lens = record_lengths(spec["genome_bp"], spec["n_records"], spec["rec_lo"],
                              spec["rec_hi"], seed=seed)
        recs = genome_records(spec["genome_bp"], spec["n_records"], seed=seed, gc=spec["gc"],
                              lengths=lens, processes=min(len(lens), os.cpu_count() or 1),
                              **spec["features"])
    joined, ranges = join_records(recs)
    valid = int(sum(max(0, r.size - K + 1) for r in recs))
    return joined, ranges, valid


def max_over_ranks(values: list[float], dist=None, device="cpu") -> list[float]:
    """Element-wise maximum of per-rank timings over all ranks (the slowest
    rank sets the step time); the values themselves for one process."""
    if dist is None:
        return [float(v) for v in values]
    import torch

    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t.tolist()]


def whole_job_rate(world: int, units_per_rank: float, ms_per_step: float) -> float:
    """Weak scaling: every rank processes `units_per_rank` per step, and the
    step takes the slowest rank's time."""
    return world * units_per_rank / (ms_per_step / 1e3)


def random_sector_rate(words_tensor, torch, n_reads: int = 1 << 26, reps: int = 3) -> float:
    """Random 32-byte sectors per second that this GPU's memory system
    serves: torch.take of one 8-byte word from each of `n_reads` uniformly
    random 32-byte sectors of the filter words (one sector access each),
    best of `reps`, CUDA events.  The denominator for kernels whose traffic
    is one random sector per super-k-mer run."""
    flat = words_tensor.view(torch.int64)
    g = torch.Generator(device=flat.device).manual_seed(7)
    idx = torch.randint(0, flat.numel() // 4, (n_reads,), device=flat.device, generator=g) * 4
    best = None
    for _ in range(reps + 1):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record()
        out = torch.take(flat, idx)
        b.record()
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        best = ms if best is None else min(best, ms)
        del out
    return n_reads / (best / 1e3)


def l2_copy_bandwidth(torch, dev, nbytes: int = 24 << 20, reps: int = 200) -> float:
    """Bytes/s (read + write) of a device copy whose source and destination
    (2 x 24 MiB) stay in L2: `reps` copies replayed as one CUDA graph, best
    of 5 replays, CUDA events.  The denominator for L2-resident filters."""
    a = torch.ones(nbytes, dtype=torch.uint8, device=dev)
    b = torch.empty_like(a)
    side = torch.cuda.Stream(dev)
    side.wait_stream(torch.cuda.current_stream(dev))
    with torch.cuda.stream(side):
        for _ in range(3):
            b.copy_(a)
    torch.cuda.current_stream(dev).wait_stream(side)
    torch.cuda.synchronize(dev)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(reps):
            b.copy_(a)
    g.replay()
    torch.cuda.synchronize(dev)
    best = None
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g.replay()
        e1.record()
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    del g
    return 2 * nbytes * reps / (best / 1e3)


def valid_windows(seq: np.ndarray) -> int:
    """Windows of `seq` whose K bases are all A/C/G/T (any case)."""
    up = seq & 0xDF
    ok = (up == ord("A")) | (up == ord("C")) | (up == ord("G")) | (up == ord("T"))
    if seq.size < K:
        return 0
    c = np.concatenate([[0], np.cumsum(~ok, dtype=np.int64)])
    return int(np.count_nonzero(c[K:] - c[:-K] == 0))


def sample_runs(seq: np.ndarray, n_shards: int) -> tuple[int, int]:
    """Super-k-mer runs and valid windows of `seq` (the R and N of the
    algorithmic-bytes model), counted by the oracle."""
    from oracle.oracle import Oracle

    return Oracle(K, S, M, H).count_runs(seq, n_shards)


# ---------------------------------------------------------------------------
# Clock sampling
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines: list[str] = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.thread.join(timeout=5)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# Reference arm: the reference's arithmetic on the host cores
# ---------------------------------------------------------------------------

CPU_SAMPLE_BP = 32_000_000
CPU_SAMPLE_READS = 80_000
CPU_BASELINE_STEPS = 20


def cpu_sample(spec: dict, joined: np.ndarray, seed: int) -> tuple[np.ndarray, np.ndarray]:
    """The bounded sample of a plain workload that both CPU legs time (the
    main arm's cpu_baseline and --impl reference): the first CPU_SAMPLE_BP
    bytes of the joined genome, and CPU_SAMPLE_READS reads of the workload's
    length drawn from that prefix (same positive share and substitution
    rate), joined with separators.  Without reads (the small plain workload)
    the query is the workload's own: genome + separator + fresh sequence."""
    from workloads.synthetic import SEPARATOR, reads_host, uniform_dna

    ins = joined[:min(joined.size, CPU_SAMPLE_BP)]
    if spec["n_reads"] > 0:
        rl = spec["read_len"]
        rd = reads_host([ins], CPU_SAMPLE_READS, rl, seed=seed + 7, sub_rate=spec["sub_rate"],
                        positive_frac=spec["positive_frac"])
        q = np.full((CPU_SAMPLE_READS, rl + 1), SEPARATOR, dtype=np.uint8)
        q[:, :-1] = rd
        return ins, q.reshape(-1)[:-1]
    fresh = uniform_dna(spec["fresh_query_bp"], seed=1337, gc=spec["gc"])
    return ins, np.concatenate([joined, np.frombuffer(b"N", np.uint8), fresh])


def query_counts(spec: dict, joined: np.ndarray) -> tuple[int, int]:
    """(valid k-mers, windows) of the workload's query input, computed on the
    host: reads of one length joined by one separator, or (small plain
    workload) genome + separator + fresh sequence."""
    if spec["n_reads"] > 0:
        rl = spec["read_len"]
        n_bytes = spec["n_reads"] * (rl + 1) - 1
        return spec["n_reads"] * max(0, rl - K + 1), max(0, n_bytes - K + 1)
    from workloads.synthetic import uniform_dna

    fresh = uniform_dna(spec["fresh_query_bp"], seed=1337, gc=spec["gc"])
    q = np.concatenate([joined, np.frombuffer(b"N", np.uint8), fresh])
    return valid_windows(q), max(0, q.size - K + 1)


def plain_config(spec: dict, world: int, filter_bits: int, n_ins_valid: int, n_q_valid: int,
                 n_q_windows: int) -> dict:
    """The `config` object of a plain workload's JSON line (both arms)."""
    if spec["n_reads"] > 0:
        query = f"{spec['n_reads']:,} x {spec['read_len']} bp reads queried"
    else:
        query = (f"the same {spec['genome_bp'] / 1e6:.3g} Mbp + a fresh "
                 f"{spec['fresh_query_bp'] / 1e6:.3g} Mbp queried")
    return {
        "workload": f"{spec['name']}: {spec['genome_bp'] / 1e9:.3g} Gbp in "
                    f"{spec['n_records']} records inserted, {query}",
        "k": K, "s": S, "m": M, "hashes": H, "filter_bits": int(filter_bits),
        "bits_per_kmer_requested": spec["bits_per_kmer"],
        "insert_kmers": int(n_ins_valid), "query_kmers": int(n_q_valid),
        "query_windows": int(n_q_windows), "parallelism": f"replicas x{world} (weak)",
        "l2": spec.get("l2", "inputs larger than L2 (no flush needed)"),
        "step": "clear (untimed memset inside the step) + insert launch + query launch",
    }


def cpu_reference_run(ins: np.ndarray, qry: np.ndarray, n_shards: int, steps: int,
                      warmup: int, threads: int) -> dict:
    """Times the reference's own arithmetic (oracle/_ref, else the C port)
    inserting `ins` into an empty filter of `n_shards` shards and querying
    `qry` against it, `steps` times after `warmup`, on `threads` host
    threads."""
    from oracle import oracle as o

    if o.RefCpu.available():
        impl, kind = o.RefCpu(K, S, M, H, threads=threads), "reference"
        desc = ("oracle/_ref: the reference cuSBF host-callable arithmetic (encode, "
                "extractPackedSubwindow, minimizer_hash64, hash64, sectorizedBitAddress) "
                "driven window by window, std::thread over all host cores")
    else:
        impl, kind = o.Oracle(K, S, M, H, threads=threads), "port"
        desc = "oracle/sbf_oracle.c: C restatement of the reference semantics, pthreads"
    n_ins = valid_windows(ins)
    n_q = valid_windows(qry)
    words = np.zeros(n_shards * 4, dtype=np.uint64)
    times = []
    for i in range(warmup + steps):
        words[:] = 0
        t0 = time.perf_counter()
        impl.insert(words, ins)
        impl.contains(words, qry)
        dt = time.perf_counter() - t0
        if i >= warmup:
            times.append(dt)
    per = float(np.mean(times))
    return dict(value=(n_ins + n_q) / per, unit="k-mers/s", cores=threads, kind=kind,
                sample=f"{ins.size / 1e6:.1f} Mbp of the genome inserted + "
                       f"{qry.size / 1e6:.1f} MB of joined reads queried "
                       f"({n_ins + n_q:,} valid k-mers) per step, filter {n_shards * 32 >> 20} MiB; "
                       + desc,
                ms_per_step=per * 1e3, kmers_per_step=n_ins + n_q, steps=len(times))


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---------------------------------------------------------------------------
# Ragged batches (config c4)
# ---------------------------------------------------------------------------

RAGGED_METRIC = ("k-mers/s insert+query, ragged batch (200k log-normal records ~2 Gbp into a "
                 "4 GiB filter + 50M log-normal reads, k=31) vs plain per-record launches")


def ragged_spec(scale: float) -> dict:
    return dict(name="ragged", n_records=max(int(200_000 * scale), 10), rec_median=5000,
                rec_sigma=1.18, rec_lo=100, rec_hi=1_000_000, gc=0.45,
                filter_bits=max(int((1 << 35) * scale), 1 << 20),
                n_reads=max(int(50_000_000 * scale), 1000), read_median=150, read_sigma=1.0,
                read_lo=50, read_hi=20_000, positive_frac=0.6, sub_rate=0.005)


def _ev(torch):
    return torch.cuda.Event(enable_timing=True)


def run_ragged(args, world: int, rank: int, local_rank: int) -> None:
    """One step = clear, one ragged insert launch over every record in place,
    one ragged query launch over every read in place (device-resident
    inputs).  Compared with plain per-record launches (insert_sequence_async
    / contains_sequence_async per record, the reference's only per-record
    form) on a sample, and end to end with the reference's single-launch
    record batch (host normalisation + one launch)."""
    from workloads.synthetic import lognormal_lengths, ragged_reads_device, uniform_dna

    spec = ragged_spec(args.scale)
    seed = args.seed + 1000 * rank
    rec_len = lognormal_lengths(spec["n_records"], spec["rec_median"], spec["rec_sigma"],
                                spec["rec_lo"], spec["rec_hi"], seed=seed)
    rec_off = np.zeros_like(rec_len)
    rec_off[1:] = np.cumsum(rec_len)[:-1]
    genome = uniform_dna(int(rec_len.sum()), seed=seed + 1, gc=spec["gc"])
    g_ranges = np.stack([rec_off, rec_len], axis=1).astype(np.uint64)
    read_len = lognormal_lengths(spec["n_reads"], spec["read_median"], spec["read_sigma"],
                                 spec["read_lo"], spec["read_hi"], seed=seed + 2)

    import torch

    import cusbf_b200 as sbf

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)
    f = sbf.Filter(spec["filter_bits"], k=K, s=S, m=M, hashes=H)
    d_genome = torch.from_numpy(genome).to(dev)
    d_granges = torch.from_numpy(g_ranges.view(np.int64)).to(dev)
    d_reads, r_ranges = ragged_reads_device(d_genome, rec_off, rec_len, read_len, seed + 3,
                                            spec["positive_frac"], spec["sub_rate"], spec["gc"],
                                            device=str(dev))
    d_rranges = torch.from_numpy(r_ranges.view(np.int64)).to(dev)
    n_out = f.kmer_count(d_reads.numel())
    d_out = torch.empty(max(n_out, 1), dtype=torch.uint8, device=dev)
    ins_counts = torch.zeros(2, dtype=torch.int64, device=dev)
    q_counts = torch.zeros(2, dtype=torch.int64, device=dev)
    torch.cuda.synchronize(dev)

    def step(ev):
        f.clear(stream)
        ins_counts.zero_()
        q_counts.zero_()
        ev[0].record(stream)
        f.ragged_insert_async(d_genome, d_granges, ins_counts, stream)
        ev[1].record(stream)
        f.ragged_contains_async(d_reads, d_rranges, d_out, q_counts, stream)
        ev[2].record(stream)

    for _ in range(args.warmup):
        step([_ev(torch) for _ in range(3)])
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    evs = [[_ev(torch) for _ in range(3)] for _ in range(args.steps)]
    t0, t1 = _ev(torch), _ev(torch)
    t0.record(stream)
    for i in range(args.steps):
        step(evs[i])
    t1.record(stream)
    torch.cuda.synchronize(dev)
    clock_info = clocks.stop()
    total_ms = t0.elapsed_time(t1)
    ins_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
    q_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))
    ins_valid, q_valid, q_pos = int(ins_counts[0]), int(q_counts[0]), int(q_counts[1])
    total_ms, ins_ms, q_ms = max_over_ranks([total_ms, ins_ms, q_ms], dist, dev)
    ms_per_step = total_ms / args.steps
    kmers_step = ins_valid + q_valid
    value = whole_job_rate(world, kmers_step, ms_per_step)
    ragged_hits = d_out.clone()

    # Plain per-record launches on a sample: the first records / reads up to
    # ~16 MB each, one launch per record, same filter state.
    plain = None
    if not args.no_baselines:
        n_rs = int(np.searchsorted(np.cumsum(rec_len), 16_000_000)) + 1
        n_qs = int(np.searchsorted(np.cumsum(read_len), 16_000_000)) + 1
        n_rs, n_qs = min(n_rs, rec_len.size), min(n_qs, read_len.size)
        pf = sbf.Filter(spec["filter_bits"], k=K, s=S, m=M, hashes=H)
        a, b = _ev(torch), _ev(torch)
        torch.cuda.synchronize(dev)
        a.record(stream)
        for i in range(n_rs):
            o, n = int(rec_off[i]), int(rec_len[i])
            pf.insert_sequence_async(d_genome[o:o + n], stream)
        b.record(stream)
        torch.cuda.synchronize(dev)
        p_ins_ms = a.elapsed_time(b)
        p_ins_k = int(np.maximum(rec_len[:n_rs] - K + 1, 0).sum())
        # Query the sample against the full filter, compare with the ragged hits.
        chk = torch.zeros_like(d_out[: int(r_ranges[n_qs - 1, 0] + r_ranges[n_qs - 1, 1])])
        a.record(stream)
        for i in range(n_qs):
            o, n = int(r_ranges[i, 0]), int(r_ranges[i, 1])
            if n >= K:
                f.contains_sequence_async(d_reads[o:o + n], chk[o:o + n - K + 1], stream)
        b.record(stream)
        torch.cuda.synchronize(dev)
        p_q_ms = a.elapsed_time(b)
        p_q_k = int(np.maximum(read_len[:n_qs] - K + 1, 0).sum())
        same = True
        for i in range(n_qs):
            o, n = int(r_ranges[i, 0]), int(r_ranges[i, 1])
            if n >= K and not torch.equal(chk[o:o + n - K + 1], ragged_hits[o:o + n - K + 1]):
                same = False
                break
        plain = {"insert_kmers_per_s": p_ins_k / (p_ins_ms / 1e3),
                 "query_kmers_per_s": p_q_k / (p_q_ms / 1e3),
                 "kmers_per_s": (p_ins_k + p_q_k) / ((p_ins_ms + p_q_ms) / 1e3),
                 "us_per_launch": 1e3 * (p_ins_ms + p_q_ms) / (n_rs + n_qs),
                 "sample": f"{n_rs} records ({int(rec_len[:n_rs].sum()) / 1e6:.1f} Mbp) + "
                           f"{n_qs} reads ({int(read_len[:n_qs].sum()) / 1e6:.1f} MB), one "
                           "insert_sequence_async / contains_sequence_async per record from Python",
                 "query_hits_identical_to_ragged": same}
        pf.close()

    # End to end through the host API: pinned inputs and outputs.
    e2e = e2e_tuned = e2e_bits = rb = None
    if not args.no_e2e:
        h_genome = torch.from_numpy(genome).pin_memory().numpy()
        h_reads_t = torch.empty(d_reads.numel(), dtype=torch.uint8).pin_memory()
        h_reads_t.copy_(d_reads)
        h_reads = h_reads_t.numpy()
        h_out = torch.empty(max(n_out, 1), dtype=torch.uint8).pin_memory().numpy()

        def e2e_run(tuning):
            f.clear(stream)
            torch.cuda.synchronize(dev)
            w0 = time.perf_counter()
            ri = f.ragged_insert(h_genome, g_ranges, tuning=tuning, stream=stream)
            w1 = time.perf_counter()
            _, rq = f.ragged_query(h_reads, r_ranges, out=h_out, tuning=tuning, stream=stream)
            w2 = time.perf_counter()
            assert ri.inserted_kmers == ins_valid and rq.positive_kmers == q_pos
            return (w1 - w0) * 1e3, (w2 - w1) * 1e3

        def e2e_obj(res, tuning):
            ims = float(np.median([r[0] for r in res]))
            qms = float(np.median([r[1] for r in res]))
            expand = sbf.host_expand_threads()
            return {"value": world * kmers_step / ((ims + qms) / 1e3), "unit": "k-mers/s",
                    "h2d_bytes_per_step": int(genome.size + h_reads.size + 32 * (
                        g_ranges.shape[0] + r_ranges.shape[0])),
                    "d2h_bytes_per_step": int(4 * ((n_out + 31) // 32) if expand else n_out),
                    "host_result_bytes": int(n_out), "host_expand_threads": expand,
                    "ms_per_step": ims + qms,
                    "insert_ms": ims, "query_ms": qms, "tuning": tuning,
                    "api": "sbf_ragged_insert + sbf_ragged_query (host buffers, pinned)"}

        e2e_run(None)
        e2e = e2e_obj([e2e_run(None) for _ in range(max(1, args.e2e_steps))], "default")
        ti = f.ragged_autotune(h_genome, g_ranges, query=False, stream=stream)
        tq = f.ragged_autotune(h_reads, r_ranges, query=True, stream=stream)
        res = []
        for _ in range(max(1, args.e2e_steps)):
            f.clear(stream)
            torch.cuda.synchronize(dev)
            w0 = time.perf_counter()
            f.ragged_insert(h_genome, g_ranges, tuning=ti, stream=stream)
            w1 = time.perf_counter()
            f.ragged_query(h_reads, r_ranges, out=h_out, tuning=tq, stream=stream)
            w2 = time.perf_counter()
            res.append(((w1 - w0) * 1e3, (w2 - w1) * 1e3))
        e2e_tuned = e2e_obj(res, {"insert": ti.as_dict(), "query": tq.as_dict()})
        # The same step with bit-packed query results (an eighth of the download).
        h_bits = torch.empty(max((n_out + 31) // 32, 1), dtype=torch.int32).pin_memory().numpy()
        res = []
        for _ in range(max(1, args.e2e_steps) + 1):
            f.clear(stream)
            torch.cuda.synchronize(dev)
            w0 = time.perf_counter()
            f.ragged_insert(h_genome, g_ranges, tuning=ti, stream=stream)
            w1 = time.perf_counter()
            _, rqb = f.ragged_query_bits(h_reads, r_ranges, out=h_bits.view(np.uint32), tuning=tq,
                                         stream=stream)
            w2 = time.perf_counter()
            assert rqb.positive_kmers == q_pos
            res.append(((w1 - w0) * 1e3, (w2 - w1) * 1e3))
        e2e_bits = e2e_obj(res[1:], {"insert": ti.as_dict(), "query": tq.as_dict()})
        e2e_bits["d2h_bytes_per_step"] = int(4 * ((n_out + 31) // 32))
        e2e_bits["host_result_bytes"] = e2e_bits["d2h_bytes_per_step"]
        e2e_bits.pop("host_expand_threads", None)
        e2e_bits["api"] = ("sbf_ragged_insert + sbf_ragged_query_bits (host buffers, pinned; "
                           "one result bit per window)")
        # The reference's single-launch record batch (host normalisation with
        # separators, one plain launch), insert and aggregate query.
        if not args.no_baselines:
            # One untimed call first, so staging buffers are allocated.
            f.insert_record_batch(h_genome, g_ranges, stream=stream)
            f.query_record_batch(h_reads, r_ranges, stream=stream)
            f.clear(stream)
            torch.cuda.synchronize(dev)
            w0 = time.perf_counter()
            f.insert_record_batch(h_genome, g_ranges, stream=stream)
            w1 = time.perf_counter()
            qr = f.query_record_batch(h_reads, r_ranges, stream=stream)
            w2 = time.perf_counter()
            assert qr.positive_kmers == q_pos
            rb = {"value": kmers_step / (w2 - w0), "unit": "k-mers/s",
                  "insert_ms": (w1 - w0) * 1e3, "query_ms": (w2 - w1) * 1e3,
                  "api": "sbf_insert_record_batch + sbf_query_record_batch (normalised copy, "
                         "one plain launch each, per-record counts only)"}

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return
    q_sample = d_reads[: min(d_reads.numel(), 3_000_000)].cpu().numpy()
    runs_q, valid_q = sample_runs(q_sample, f.num_shards())
    r_per_q = runs_q / max(valid_q, 1)
    q_bytes = d_reads.numel() + n_out + 32 * r_per_q * q_valid
    peaks = {}
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peaks = json.load(open(peaks_path))
    peak = float(peaks.get("hbm_gbs", 6650.0))
    q_ach = q_bytes / (q_ms / 1e3) / 1e9
    line = {
        "metric": RAGGED_METRIC, "value": value, "unit": "k-mers/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded log-normal records and reads with the configuration's shapes)",
        "config": {"workload": f"ragged: {spec['n_records']:,} records ({genome.size / 1e9:.2f} "
                               f"Gbp, log-normal median 5 kbp) inserted, {spec['n_reads']:,} "
                               f"reads ({d_reads.numel() / 1e9:.2f} GB, log-normal median 150 bp) "
                               "queried, records in place",
                   "k": K, "s": S, "m": M, "hashes": H, "filter_bits": f.filter_bits(),
                   "insert_kmers": ins_valid, "query_kmers": q_valid,
                   "parallelism": f"replicas x{world} (weak)",
                   "l2": "inputs larger than L2 (no flush needed)",
                   "step": "clear + one ragged insert launch + one ragged query launch"},
        "insert": {"ms": ins_ms, "kmers_per_s": ins_valid / (ins_ms / 1e3)},
        "query": {"ms": q_ms, "kmers_per_s": q_valid / (q_ms / 1e3), "positives": q_pos},
        "roofline": {"bound": "hbm", "kernel": "query (tile_kernel<31,28,16,4> ragged query)",
                     "achieved": round(q_ach, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(q_ach / peak, 4),
                     "peak_source": "measured" if "hbm_gbs" in peaks else "fallback",
                     "traffic": None, "algorithmic_bytes": int(q_bytes),
                     "model": f"L + N + 32R (R/N={r_per_q:.4f} counted by the oracle on 3 MB)"},
        "plain_per_record": plain,
        "speedup_vs_plain": (value / plain["kmers_per_s"]) if plain else None,
        "record_batch_e2e": rb,
        "e2e": e2e,
        "e2e_tuned": e2e_tuned,
        "e2e_bits": e2e_bits,
        "gpu_launches": 4 * args.steps,
        "clocks": clock_info,
    }
    print(json.dumps(line), flush=True)
    f.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# Serving (config c5)
# ---------------------------------------------------------------------------

SERVED_METRIC = ("served k-mers/s and p50/p99/p999 latency, Poisson 20k req/s (log-uniform "
                 "1-100k x 150 bp reads, 5% inserts of 1-10 Mbp) on the resident 100 Mbp filter")


SHARDED_METRIC = ("k-mers/s of one 3.1 Gbp genome inserted over N GPUs by the sharded insert "
                  "(emit runs, all-to-all to shard owners, OR, all-gather to replicas)")


def run_sharded(args, world: int, rank: int, local_rank: int) -> None:
    """Strong scaling of the insert: every rank holds the same genome; each
    step clears the filter and runs cusbf_b200.sharded.sharded_insert (each
    rank emits the runs of 1/N of the windows, records go to the owners of
    their shards, owners OR them in, an all-gather restores the whole filter
    on every rank).  The step time and the per-phase times are the max over
    ranks.  After timing, rank 0's filter is compared word for word with a
    single-GPU insert, which is also timed."""
    import datetime

    import torch
    import torch.distributed as dist

    import cusbf_b200 as sbf
    from cusbf_b200 import sharded

    spec = workload_spec("c3", args.scale)
    joined, _, n_ins_valid = build_host_genome(spec, seed=args.seed)
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ.setdefault("MASTER_PORT", "29517")
    dist.init_process_group("nccl", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120), device_id=dev)
    bits = int(round(spec["bits_per_kmer"] * n_ins_valid))
    f = sbf.Filter(bits, k=K, s=S, m=M, hashes=H)
    d_genome = torch.from_numpy(joined).to(dev)
    times, phases = [], {}
    for i in range(args.warmup + args.steps):
        f.clear()
        torch.cuda.synchronize(dev)
        dist.barrier()
        a, b = _ev(torch), _ev(torch)
        a.record()
        sharded.sharded_insert(f, d_genome, timings=phases if i >= args.warmup else None)
        b.record()
        torch.cuda.synchronize(dev)
        if i >= args.warmup:
            times.append(a.elapsed_time(b))
    names = ("emit", "route", "apply", "gather")
    got = max_over_ranks([float(np.mean(times))] + [phases.get(n, 0.0) / args.steps
                                                     for n in names], dist, dev)
    ms, phase_ms = got[0], dict(zip(names, got[1:]))
    same = single_ms = None
    if rank == 0:
        g = sbf.Filter(bits, k=K, s=S, m=M, hashes=H)
        st = []
        for i in range(1 + args.steps):
            g.clear()
            a, b = _ev(torch), _ev(torch)
            a.record()
            g.insert_sequence_async(d_genome)
            b.record()
            torch.cuda.synchronize(dev)
            if i:
                st.append(a.elapsed_time(b))
        single_ms = float(np.mean(st))
        same = bool(torch.equal(f.words(), g.words()))
        g.close()
    dist.barrier()
    if rank == 0:
        print(json.dumps({
            "metric": SHARDED_METRIC, "value": n_ins_valid / (ms / 1e3), "unit": "k-mers/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "u8",
            "data": "synthetic (seeded stand-in with the configuration's shapes; no public genome)",
            "config": {"workload": f"{spec['name']}: {spec['genome_bp'] / 1e9:.3g} Gbp in "
                                   f"{spec['n_records']} records, one insert over all ranks",
                       "filter_bits": f.filter_bits(), "insert_kmers": n_ins_valid,
                       "parallelism": f"sharded insert x{world} (strong)"},
            "phase_ms": phase_ms, "single_gpu_insert_ms": single_ms,
            "identical_to_single_gpu_insert": same}), flush=True)
    f.close()
    dist.destroy_process_group()


FASTX_METRIC = ("GB/s of FASTA insert and FASTQ query from files, parsed on the GPU, each block "
                "replayed as one CUDA graph vs stream launches vs the host parser")


def run_fastx_files(args) -> None:
    """FASTA insert (100 Mbp genome, 80-column lines) and FASTQ query (4M x
    150 bp reads, half sampled from the genome with 1% substitutions) through
    insert_fastx_file / query_fastx_file, with the GPU parser replaying each
    block as one CUDA graph, with stream launches, and with the host parser.
    Reports and filter words must agree across the three."""
    import tempfile

    import torch

    import cusbf_b200 as sbf
    from workloads.synthetic import reads_device, uniform_dna

    n_reads = max(int(4_000_000 * args.scale), 1000)
    genome = uniform_dna(max(int(100_000_000 * args.scale), 10_000), seed=args.seed, gc=0.41)
    dev = torch.device("cuda", 0)
    d_genome = torch.from_numpy(genome).to(dev)
    reads = reads_device(d_genome, n_reads, 150, seed=args.seed + 7, sub_rate=0.01,
                         positive_frac=0.5, device=str(dev)).cpu().numpy()
    del d_genome
    rec = np.empty((n_reads, 307), np.uint8)  # "@r\n" seq "\n+\n" qual "\n"
    rec[:, 0:3] = np.frombuffer(b"@r\n", np.uint8)
    rec[:, 3:153] = reads
    rec[:, 153:156] = np.frombuffer(b"\n+\n", np.uint8)
    rec[:, 156:306] = ord("I")
    rec[:, 306] = ord("\n")
    width = 80
    n_lines = -(-genome.size // width)
    fa = np.full(n_lines * (width + 1), ord("\n"), np.uint8)
    body = fa[:n_lines * (width + 1)].reshape(n_lines, width + 1)
    pad = np.zeros(n_lines * width, np.uint8)
    pad[:genome.size] = genome
    body[:, :width] = pad.reshape(n_lines, width)
    tail = n_lines * width - genome.size
    fa_bytes = b">genome\n" + (fa.tobytes()[:-(tail + 1)] + b"\n" if tail else fa.tobytes())
    results = {}
    with tempfile.TemporaryDirectory() as tmp:
        fq_path, fa_path = os.path.join(tmp, "reads.fq"), os.path.join(tmp, "genome.fa")
        rec.tofile(fq_path)
        with open(fa_path, "wb") as fh:
            fh.write(fa_bytes)
        fq_bytes, fa_size = os.path.getsize(fq_path), os.path.getsize(fa_path)
        bits = 1 << 31
        for mode in ("graph", "stream", "host"):
            os.environ["SBF_FASTX_PARSER"] = "host" if mode == "host" else "device"
            os.environ["SBF_FASTX_GRAPH"] = "1" if mode == "graph" else "0"
            f = sbf.Filter(bits, k=K, s=S, m=M, hashes=H)
            ins_t, q_t = [], []
            for rep_i in range(1 + max(args.steps, 1)):
                f.clear()
                torch.cuda.synchronize(dev)
                t0 = time.perf_counter()
                irep = f.insert_fastx_file(fa_path)
                t1 = time.perf_counter()
                qrep = f.query_fastx_file(fq_path)
                t2 = time.perf_counter()
                if rep_i:
                    ins_t.append(t1 - t0)
                    q_t.append(t2 - t1)
            words = f.words_host()
            f.close()
            results[mode] = {"insert_gb_per_s": fa_size / min(ins_t) / 1e9,
                             "query_gb_per_s": fq_bytes / min(q_t) / 1e9,
                             "insert_kmers_per_s": irep.inserted_kmers / min(ins_t),
                             "query_kmers_per_s": qrep.queried_kmers / min(q_t),
                             "insert_report": irep.as_dict(), "query_report": qrep.as_dict(),
                             "_words": words}
        os.environ.pop("SBF_FASTX_PARSER", None)
        os.environ.pop("SBF_FASTX_GRAPH", None)
    same = all(results[m]["insert_report"] == results["graph"]["insert_report"] and
               results[m]["query_report"] == results["graph"]["query_report"] and
               np.array_equal(results[m]["_words"], results["graph"]["_words"])
               for m in ("stream", "host"))
    for m in results:
        results[m].pop("_words")
    g = results["graph"]
    line = {"metric": FASTX_METRIC, "value": g["query_gb_per_s"], "unit": "GB/s",
            "n_gpus": 1, "steps": max(args.steps, 1), "warmup": 1, "higher_is_better": True,
            "dtype": "u8", "data": "synthetic (seeded genome and reads written to files)",
            "config": {"workload": f"FASTA insert of {genome.size / 1e6:.0f} Mbp "
                                   f"({fa_size / 1e6:.0f} MB, {width}-column lines), FASTQ query "
                                   f"of {n_reads:,} x 150 bp reads ({fq_bytes / 1e9:.2f} GB)",
                       "filter_bits": bits, "block_bytes": "256 MiB (SBF_FASTQ_BLOCK_BYTES)",
                       "timing": "host wall clock around each file call, best of the steps"},
            "graph": g, "stream": results["stream"], "host_parser": results["host"],
            "graph_vs_stream_query": g["query_gb_per_s"] / results["stream"]["query_gb_per_s"],
            "identical_across_paths": bool(same)}
    print(json.dumps(line), flush=True)


CONFIGS_METRIC = ("windows/s of insert and query for other filter configurations (1 GiB "
                  "device-resident inputs, 2^34-bit filter)")
# (name, configuration id of the reference build in oracle/_ref, engine
# configuration, input letters)
OTHER_CONFIGS = (
    ("k31_s28_m21_h4", 7, dict(k=31, s=28, m=21, hashes=4), b"ACGT"),
    ("k25_s22_m13_h4", 8, dict(k=25, s=22, m=13, hashes=4), b"ACGT"),
    ("k21_s19_m11_h4", 6, dict(k=21, s=19, m=11, hashes=4), b"ACGT"),
    ("k31_s28_m16_h8", 4, dict(k=31, s=28, m=16, hashes=8), b"ACGT"),
    ("k31_s28_m16_h16", 5, dict(k=31, s=28, m=16, hashes=16), b"ACGT"),
    ("protein_k12_s10_m6_h4", 9, dict(k=12, s=10, m=6, hashes=4, alphabet=2),
     b"ACDEFGHIKLMNPQRSTVWY"),
)


def other_config_inputs(torch, dev, letters: bytes, n: int, seed: int):
    """Insert input: n uniform letters; query input: the insert input's first
    half followed by n - n/2 fresh letters (about half the windows present)."""
    g = torch.Generator(device=dev).manual_seed(seed)
    lut = torch.tensor(list(letters), dtype=torch.uint8, device=dev)
    ins = lut[torch.randint(0, len(letters), (n,), device=dev, generator=g, dtype=torch.int32)]
    qry = ins.clone()
    h = n // 2
    qry[h:] = lut[torch.randint(0, len(letters), (n - h,), device=dev, generator=g,
                                dtype=torch.int32)]
    return ins, qry


def run_other_configs(args) -> None:
    """Insert and query of 1 GiB device inputs for each of OTHER_CONFIGS,
    timed with CUDA events on the launching stream (inputs are 8x L2, so no
    flush is needed).  The main arm runs the engine; --impl reference runs the
    unmodified reference GPU path (oracle/_ref) on the same seeded inputs."""
    import torch

    reference = args.impl == "reference"
    if reference:
        from oracle.oracle import RefGpu

        if not RefGpu.available():
            print(json.dumps({"impl": "reference", "metric": CONFIGS_METRIC,
                              "unavailable": "oracle/_ref/libsbf_refgpu.so was not built"}))
            return
    else:
        import cusbf_b200 as sbf
    dev = torch.device("cuda", 0)
    n = max(int((1 << 30) * args.scale), 1 << 20)
    bits = max(int((1 << 34) * args.scale), 1 << 24)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    steps, warmup = max(args.steps, 1), max(args.warmup, 3)
    clocks = ClockSampler(0)
    clocks.start()
    results = {}
    total_windows, total_ms = 0, 0.0
    for name, cfg_id, cfg, letters in OTHER_CONFIGS:
        ins, qry = other_config_inputs(torch, dev, letters, n, args.seed + cfg_id)
        n_out = n - cfg["k"] + 1
        out = torch.empty(n_out, dtype=torch.uint8, device=dev)
        if reference:
            filt = RefGpu(bits, cfg_id)
            clear = lambda: filt.clear(sp)  # noqa: E731
            insert = lambda: filt.insert_async(ins.data_ptr(), n, sp)  # noqa: E731
            query = lambda: filt.contains_async(qry.data_ptr(), n, out.data_ptr(),  # noqa: E731
                                                n_out, sp)
        else:
            filt = sbf.Filter(bits, **cfg)
            clear = lambda: filt.clear(stream)  # noqa: E731
            insert = lambda: filt.insert_sequence_async(ins, stream)  # noqa: E731
            query = lambda: filt.contains_sequence_async(qry, out, stream)  # noqa: E731
        ins_ms, q_ms = [], []
        for i in range(warmup + steps):
            clear()
            a, b, c = _ev(torch), _ev(torch), _ev(torch)
            a.record(stream)
            insert()
            b.record(stream)
            query()
            c.record(stream)
            torch.cuda.synchronize(dev)
            if i >= warmup:
                ins_ms.append(a.elapsed_time(b))
                q_ms.append(b.elapsed_time(c))
        i_ms, qm = float(np.mean(ins_ms)), float(np.mean(q_ms))
        results[name] = {"insert_windows_per_s": n_out / (i_ms / 1e3), "insert_ms": i_ms,
                         "query_windows_per_s": n_out / (qm / 1e3), "query_ms": qm,
                         "positive_windows": int(torch.count_nonzero(out))}
        if not reference:
            results[name]["kernel_path"] = ("compiled in", "compiled at run time",
                                            "generic")[filt.kernel_path()]
        total_windows += 2 * n_out
        total_ms += i_ms + qm
        filt.close()
        del ins, qry, out
        torch.cuda.empty_cache()
    clock_info = clocks.stop()
    line = {"metric": CONFIGS_METRIC, "value": total_windows / (total_ms / 1e3),
            "unit": "windows/s", "n_gpus": 1, "steps": steps, "warmup": warmup,
            "ms_per_step": total_ms, "higher_is_better": True, "dtype": "u8",
            "data": "synthetic (seeded uniform letters generated on the device)",
            "config": {"workload": f"{n} letters inserted and {n} queried per configuration",
                       "filter_bits": bits, "l2": "inputs are 8x L2; no flush"},
            "configs": results, "clocks": clock_info}
    if reference:
        line["impl"] = "reference"
        line["path"] = ("reference cuSBF filter<Config<...>> insert_sequence_async + "
                        "contains_sequence_async, device-resident inputs, CUDA events")
    print(json.dumps(line), flush=True)


FPR_METRIC = ("false-positive rate of uniform random 31-mers against the 100 Mbp genome of the "
              "small plain workload, s = 28 / 30 / 31 at 21.4 / 85.7 / 342.6 bits per k-mer")
# (s, configuration id of the reference build in oracle/_ref)
FPR_S = ((28, 0), (30, 10), (31, 11))
# Filter sizes: the workload's 21.4 bits per k-mer, and 4x and 16x that.
FPR_SIZE_FACTORS = (1, 4, 16)
# The reference's published table (README.md:59-63, a real genome), percent.
FPR_PUBLISHED = {28: (0.848, 0.091, 0.0095), 30: (0.951, 0.107, 0.0114),
                 31: (1.593, 0.210, 0.0264)}


def run_fpr(args) -> None:
    """False-positive rates in the form of the reference's sweep
    (benchmarks/fpr_fastx_sweep.cu): the genome of the small plain workload
    inserted into filters of 1x, 4x and 16x its 21.4 bits per k-mer, then 1e9
    uniform random 31-mers queried (records of 2^28 windows generated on the
    device from one seed, the same for every filter); FPR = positive windows /
    queried windows.  The main arm runs the engine, --impl reference the
    unmodified reference GPU path on the same inputs."""
    import torch

    reference = args.impl == "reference"
    if reference:
        from oracle.oracle import RefGpu

        if not RefGpu.available():
            print(json.dumps({"impl": "reference", "metric": FPR_METRIC,
                              "unavailable": "oracle/_ref/libsbf_refgpu.so was not built"}))
            return
    else:
        import cusbf_b200 as sbf
    spec = workload_spec("c2", args.scale)
    joined, _, n_ins_valid = build_host_genome(spec, seed=args.seed)
    dev = torch.device("cuda", 0)
    d_genome = torch.from_numpy(joined).to(dev)
    del joined
    base_bits = int(round(spec["bits_per_kmer"] * n_ins_valid))
    n_query = max(int(1e9 * args.scale), 1 << 20)
    chunk = 1 << 28
    lut = torch.tensor(list(b"ACGT"), dtype=torch.uint8, device=dev)
    out = torch.empty(min(chunk, n_query), dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    rows = []
    t0 = time.perf_counter()
    for s, ref_id in FPR_S:
        for i, factor in enumerate(FPR_SIZE_FACTORS):
            requested = base_bits * factor
            if reference:
                filt = RefGpu(requested, ref_id)
                filt.insert_async(d_genome.data_ptr(), d_genome.numel(), stream.cuda_stream)
                filter_bits = filt.num_shards() * 256
            else:
                filt = sbf.Filter(requested, k=31, s=s, m=16, hashes=4)
                filt.insert_sequence_async(d_genome, stream)
                filter_bits = filt.filter_bits()
            gen = torch.Generator(device=dev).manual_seed(1337)
            positives = 0
            for off in range(0, n_query, chunk):
                w = min(chunk, n_query - off)
                q = lut[torch.randint(0, 4, (w + 30,), device=dev, generator=gen,
                                      dtype=torch.int32)]
                if reference:
                    filt.contains_async(q.data_ptr(), q.numel(), out.data_ptr(), w,
                                        stream.cuda_stream)
                else:
                    filt.contains_sequence_async(q, out[:w], stream)
                positives += int(torch.count_nonzero(out[:w]))
                del q
            filt.close()
            rows.append({"s": s, "requested_bits": requested, "filter_bits": filter_bits,
                         "bits_per_kmer": filter_bits / n_ins_valid, "positives": positives,
                         "queried": n_query, "fpr_pct": 100.0 * positives / n_query,
                         "published_pct": FPR_PUBLISHED[s][i]})
    torch.cuda.synchronize(dev)
    line = {"metric": FPR_METRIC, "value": rows[0]["fpr_pct"], "unit": "%",
            "higher_is_better": False, "n_gpus": 1,
            "data": "synthetic (seeded genome with repeats and N runs; uniform random queries "
                    "generated on the device); the published table is on a real genome",
            "config": {"workload": f"{n_ins_valid:,} k-mers inserted, {n_query:,} random "
                                   f"31-mers queried per filter", "k": 31, "m": 16, "hashes": 4},
            "fpr": rows, "seconds": time.perf_counter() - t0}
    if reference:
        line["impl"] = "reference"
    print(json.dumps(line), flush=True)


def summarize_fpr(d: dict) -> dict:
    if "fpr" not in d:
        return d
    return {"metric": d["metric"], "workload": d["config"]["workload"],
            "fpr_pct": {f"s{r['s']}@{r['bits_per_kmer']:.1f}": round(r["fpr_pct"], 4)
                        for r in d["fpr"]},
            "published_pct": {f"s{r['s']}@{r['bits_per_kmer']:.1f}": r["published_pct"]
                              for r in d["fpr"]},
            "positives": [r["positives"] for r in d["fpr"]]}


def summarize_configs(d: dict) -> dict:
    if "configs" not in d:
        return d
    return {"metric": d["metric"], "workload": d["config"]["workload"],
            "filter_bits": d["config"]["filter_bits"],
            "g_windows_per_s": {name: [round(r["insert_windows_per_s"] / 1e9, 2),
                                       round(r["query_windows_per_s"] / 1e9, 2)]
                                for name, r in d["configs"].items()},
            "kernel_path": {name: r.get("kernel_path") for name, r in d["configs"].items()},
            "positive_windows": {name: r["positive_windows"] for name, r in d["configs"].items()},
            "clocks": d.get("clocks")}


def _poisson_schedule(seed: int, rate: float, duration: float, pool_reads: int,
                      ins_pool: int, scale: float):
    """Arrival offsets (s), insert flags, reads per query, first read, insert
    bytes and insert offsets of the requests."""
    rng = np.random.default_rng(seed)
    n = int(rate * duration * 1.2) + 16
    t = np.cumsum(rng.exponential(1.0 / rate, size=n))
    t = t[t < duration]
    n = t.size
    is_ins = rng.random(n) < 0.05
    n_reads = np.floor(np.exp(rng.uniform(0.0, np.log(100_001 * scale), size=n))).astype(np.int64)
    n_reads = np.clip(n_reads, 1, pool_reads)
    first = (rng.random(n) * (pool_reads - n_reads + 1)).astype(np.int64)
    ins_bytes = np.clip((rng.uniform(1e6, 10e6, size=n) * scale).astype(np.int64), 1000, ins_pool)
    ins_off = (rng.random(n) * (ins_pool - ins_bytes + 1)).astype(np.int64)
    return t, is_ins, n_reads, first, ins_bytes, ins_off


def run_served(args, world: int, rank: int, local_rank: int) -> None:
    """Open-loop load: requests arrive on a seeded Poisson schedule and are
    submitted at their arrival times; latency is completion minus scheduled
    arrival.  The same schedule is replayed against one-request-per-launch
    serving, and the per-read launch cost of the plain per-record path is
    measured.  Query requests are slices of a pinned pool of reads (half
    sampled from the genome with 1% substitutions, half random); insert
    requests are slices of a pinned pool of uniform sequence."""
    import torch

    import cusbf_b200 as sbf
    from workloads.synthetic import reads_device, uniform_dna

    scale = args.scale
    spec = workload_spec("c2", 1.0)
    joined, _, n_valid = build_host_genome(spec, seed=args.seed + 1000 * rank)
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    bits = int(round(spec["bits_per_kmer"] * n_valid))
    rate = (args.rate or 20_000.0) * min(scale, 1.0)
    duration = args.duration
    pool_reads = int(26_000_000 * min(1.0, max(scale, 0.02)))
    read_len = 150
    d_genome = torch.from_numpy(joined).to(dev)
    reads = reads_device(d_genome, pool_reads, read_len, seed=args.seed + 11, sub_rate=0.01,
                         positive_frac=0.5, device=str(dev))
    perm = torch.randperm(pool_reads, device=dev,
                          generator=torch.Generator(device=dev).manual_seed(args.seed + 12))
    reads = reads[perm].reshape(-1)
    pool = torch.empty(reads.numel(), dtype=torch.uint8).pin_memory()
    pool.copy_(reads)
    del reads, perm
    pool_np = pool.numpy()
    rng_t = torch.empty((pool_reads, 2), dtype=torch.int64).pin_memory()
    rng_np = rng_t.numpy().view(np.uint64)
    rng_np[:, 0] = np.arange(pool_reads, dtype=np.uint64) * read_len
    rng_np[:, 1] = read_len
    ins_pool_bytes = int(1 << 30) if scale >= 1 else int(max((1 << 30) * scale, 1 << 24))
    ins_pool = torch.from_numpy(uniform_dna(ins_pool_bytes, seed=args.seed + 13)).pin_memory()
    ins_np = ins_pool.numpy()
    t_arr, is_ins, n_reads, first, ins_bytes, ins_off = _poisson_schedule(
        args.seed + 14, rate, duration, pool_reads, ins_pool_bytes, min(scale, 1.0))
    n_req = t_arr.size
    out_ring_bytes = int(min(8 << 30, max(pool_np.size * 2, 1 << 26)))
    out_ring = torch.empty(out_ring_bytes, dtype=torch.uint8).pin_memory()
    out_np = out_ring.numpy()
    check_idx = set(range(0, n_req, max(1, n_req // 64)))
    op_q = 3 if args.server_counts else 2 if args.server_bits else 1
    # Dense wire format: request bodies are 2-bit packed words (packed once,
    # as a client would store them); ranges count symbols.
    dense_flag = 0x10 if args.server_dense else 0
    q_body, i_body = pool_np, ins_np
    if dense_flag:
        def packed_pinned(host_u8):
            d = torch.from_numpy(host_u8).to(dev)
            d_w = torch.empty(sbf.Filter.dense_packed_word_count(d.numel()), dtype=torch.int64,
                              device=dev)
            sbf.pack_dense_sequence_device(d, d.numel(), d_w)
            h = torch.empty(d_w.numel(), dtype=torch.int64).pin_memory()
            torch.cuda.synchronize(dev)
            h.copy_(d_w)
            return h
        q_words, i_words = packed_pinned(pool_np), packed_pinned(ins_np)
        q_body, i_body = q_words.numpy(), i_words.numpy()

    def result_len(nr):
        """Result bytes of a query of nr reads: hit bytes, bit words, or
        (valid, positive) uint64 pairs per read."""
        w = nr * read_len - K + 1
        return 16 * nr if op_q == 3 else 4 * ((w + 31) // 32) if op_q == 2 else w

    check_out = {i: np.zeros(max(result_len(int(n_reads[i])), 1), np.uint8)
                 for i in check_idx if not is_ins[i]}
    ins_range_t = torch.empty((n_req, 2), dtype=torch.int64).pin_memory()
    ins_range = ins_range_t.numpy().view(np.uint64)
    ins_range[:, 0] = ins_off.astype(np.uint64)
    ins_range[:, 1] = ins_bytes.astype(np.uint64)

    def run_stream(srv):
        """Submits the schedule at its arrival times."""
        ring_pos = 0
        ring_live = []  # (ticket, start, end) of output regions in use, oldest first
        lags = []
        t0 = sbf.Server.now() + 0.05
        for i in range(n_req):
            arrival = t0 + float(t_arr[i])
            while sbf.Server.now() < arrival:
                pass
            if is_ins[i]:
                srv.submit_raw(dense_flag, i_body.ctypes.data, ins_range.ctypes.data + 16 * i, 1,
                               None, 0,
                               arrival)
            else:
                nr = int(n_reads[i])
                w = result_len(nr)
                if i in check_out:
                    optr = check_out[i].ctypes.data
                else:
                    if ring_pos + w > out_ring_bytes:
                        ring_pos = 0
                    lo, hi = ring_pos, ring_pos + w
                    while ring_live and ring_live[0][1] < hi and ring_live[0][2] > lo:
                        srv.wait(ring_live.pop(0)[0])
                    optr = out_np.ctypes.data + lo
                    ring_pos = hi
                t = srv.submit_raw(op_q | dense_flag, q_body.ctypes.data,
                                   rng_np.ctypes.data + 16 * int(first[i]), nr, optr, w, arrival)
                if i not in check_out:
                    ring_live.append((t, lo, hi))
                    while len(ring_live) > 4096:
                        srv.wait(ring_live.pop(0)[0])
            lags.append(sbf.Server.now() - arrival)
        srv.drain()
        return {"submit_lag_p50_ms": float(np.median(lags)) * 1e3,
                "submit_lag_p99_ms": float(np.quantile(lags, 0.99)) * 1e3}

    def serve(**cfg):
        f = sbf.Filter(bits, k=K, s=S, m=M, hashes=H)
        f.insert_sequence(joined)
        srv = sbf.Server(f, staging_bytes=16 << 30, **cfg)
        lag = run_stream(srv)
        st = srv.stats()
        srv.close()
        words_sum = int(np.bitwise_xor.reduce(f.words_host()))
        f.close()
        kmers = st["query_windows"] + st["insert_windows"]
        return {"kmers_per_s": kmers / st["wall_s"] if st["wall_s"] else None,
                "config": cfg, "requests": st["requests"],
                "requests_per_s": st["requests"] / st["wall_s"] if st["wall_s"] else None,
                "batches": st["batches"], "mean_batch_requests": st["mean_batch_requests"],
                "latency_ms": {"p50": st["p50_s"] * 1e3, "p99": st["p99_s"] * 1e3,
                               "p999": st["p999_s"] * 1e3, "max": st["max_s"] * 1e3,
                               "mean": st["mean_s"] * 1e3},
                "wall_s": st["wall_s"], "worker_busy_s": st["worker_busy_s"],
                "admission_wait_s": st["admission_wait_s"], "slot_wait_s": st["slot_wait_s"],
                **lag}, words_sum, {i: o.copy() for i, o in check_out.items()}

    clocks = ClockSampler(local_rank)
    clocks.start()
    served, served_words, served_checks = serve(max_inflight=args.server_inflight,
                                                max_batch_bytes=args.server_batch_mb << 20,
                                                use_graph=args.server_graph)
    clock_info = clocks.stop()
    serial = identical = None
    if not args.no_serial:
        serial, serial_words, serial_checks = serve(max_batch_requests=1, max_inflight=1)
        identical = bool(served_words == serial_words and all(
            np.array_equal(served_checks[i], serial_checks[i]) for i in served_checks))

    # Plain per-record launches: one contains_sequence_async per read.
    f = sbf.Filter(bits, k=K, s=S, m=M, hashes=H)
    f.insert_sequence(joined)
    d_pool = torch.from_numpy(pool_np[: 4000 * read_len].copy()).to(dev)
    d_o = torch.empty(4000 * read_len, dtype=torch.uint8, device=dev)
    stream = torch.cuda.current_stream(dev)
    a, b = _ev(torch), _ev(torch)
    torch.cuda.synchronize(dev)
    a.record(stream)
    for r in range(4000):
        f.contains_sequence_async(d_pool[r * read_len:(r + 1) * read_len],
                                  d_o[r * read_len:(r + 1) * read_len - K + 1], stream)
    b.record(stream)
    torch.cuda.synchronize(dev)
    per_read_ms = a.elapsed_time(b) / 4000
    mean_reads = float(np.mean(n_reads[~is_ins]))
    plain = {"us_per_read_launch": per_read_ms * 1e3,
             "kmers_per_s": (read_len - K + 1) / (per_read_ms / 1e3),
             "service_ms_per_mean_request": per_read_ms * mean_reads,
             "sustainable_requests_per_s": 1e3 / (per_read_ms * mean_reads),
             "note": "device-resident reads, one launch per read from Python; the offered "
                     f"{rate:.0f} req/s is far beyond it"}
    f.close()
    offered = float(np.sum(np.where(is_ins, ins_bytes, n_reads * read_len)))
    line = {
        "metric": SERVED_METRIC, "value": served["kmers_per_s"], "unit": "k-mers/s",
        "n_gpus": world, "steps": 1, "warmup": 0, "ms_per_step": served["wall_s"] * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded Poisson request stream over seeded reads and sequences)",
        "config": {"workload": f"served: {n_req:,} requests over {duration:.1f} s at "
                               f"{rate:.0f} req/s, filter of the 100 Mbp genome resident",
                   "query_results": {1: "one byte per window", 2: "bit-packed (op 2)",
                                     3: "per-read (valid, positive) counts (op 3)"}[op_q],
                   "host_expand_threads": (sbf.host_expand_threads() if op_q == 1 else 0),
                   "request_bodies": ("2-bit dense-packed words (op | 0x10; N packs as G)"
                                      if dense_flag else "ASCII bytes"),
                   "k": K, "s": S, "m": M, "hashes": H, "filter_bits": bits,
                   "staging_budget_bytes": 16 << 30, "offered_bytes": int(offered),
                   "offered_gb_per_s": offered / duration / 1e9,
                   "wire_gb_per_s": offered / duration / 1e9 / (4 if dense_flag else 1),
                   "read_pool": f"{pool_reads:,} reads of 150 bp (half sampled with 1% "
                                "substitutions, half random); requests are pool slices",
                   "l2": "inputs larger than L2 (no flush needed)"},
        "served": served,
        "one_request_per_launch": serial,
        "plain_per_record": plain,
        "identical_to_one_at_a_time": identical,
        "checked_requests": len(served_checks),
        "gpu_launches": 2 * served["batches"],
        "clocks": clock_info,
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# Main
# ---------------------------------------------------------------------------

def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default="c3",
                    choices=["c1", "c2", "c3", "c4", "c5", "fastx", "sharded", "configs",
                             "fpr"])
    ap.add_argument("--duration", type=float, default=2.0, help="c5: seconds of arrivals")
    ap.add_argument("--server-inflight", type=int, default=0, help="c5: batches in flight")
    ap.add_argument("--server-batch-mb", type=int, default=0, help="c5: batch cap in MiB")
    ap.add_argument("--server-graph", type=int, default=0, help="c5: graph replay")
    ap.add_argument("--no-serial", action="store_true", help="c5: skip the one-per-launch run")
    ap.add_argument("--server-bits", action="store_true",
                    help="c5: queries ask for bit-packed results")
    ap.add_argument("--server-counts", action="store_true",
                    help="c5: queries ask for per-read (valid, positive) counts only")
    ap.add_argument("--server-dense", action="store_true",
                    help="c5: request bodies are 2-bit dense-packed words")
    ap.add_argument("--rate", type=float, default=0.0, help="c5: offered req/s (default 20k)")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="reference arm: skip timing the reference GPU path")
    ap.add_argument("--no-forms", action="store_true",
                    help="c3: skip the ragged-batch and served child runs")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0,
                    help="size multiplier for small profiling runs (1.0 = the named config)")
    ap.add_argument("--seed", type=int, default=42)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-baselines", action="store_true",
                    help="c4: skip the per-record and record-batch comparisons")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours" and args.scale == 1.0:
        print("note: at least 3 warm-up steps are used for reported numbers", file=sys.stderr)

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.config == "c4":
        if args.impl == "reference":
            print(json.dumps({"impl": "reference", "metric": RAGGED_METRIC,
                              "unavailable": "the ragged form has no reference counterpart; "
                                             "its baselines (plain per-record launches, record "
                                             "batch) are inside the c4 line"}))
            return
        run_ragged(args, world, rank, local_rank)
        return
    if args.config == "sharded":
        if args.impl == "reference":
            if rank == 0:
                print(json.dumps({"impl": "reference", "metric": SHARDED_METRIC,
                                  "unavailable": "the reference has no multi-GPU insert"}))
            return
        run_sharded(args, world, rank, local_rank)
        return
    if args.config == "fastx":
        if args.impl == "reference" or rank != 0:
            if rank == 0:
                print(json.dumps({"impl": "reference", "metric": FASTX_METRIC,
                                  "unavailable": "the reference parses FASTA/FASTQ on the host; "
                                                 "its parser is the host-parser leg of this line"}))
            return
        run_fastx_files(args)
        return
    if args.config == "configs":
        if rank == 0:
            run_other_configs(args)
        return
    if args.config == "fpr":
        if rank == 0:
            run_fpr(args)
        return
    if args.config == "c5":
        if args.impl == "reference" or rank != 0:
            if rank == 0:
                print(json.dumps({"impl": "reference", "metric": SERVED_METRIC,
                                  "unavailable": "the served form has no reference counterpart; "
                                                 "its baselines are inside the c5 line"}))
            return
        run_served(args, world, rank, local_rank)
        return
    spec = workload_spec(args.config, args.scale)

    # Host data is generated before any CUDA call (the generator may fork a
    # spawn pool).
    if args.impl == "reference":
        if rank == 0:
            run_reference_arm(args, spec, world)
        return
    joined, ranges, n_ins_valid = build_host_genome(spec, seed=args.seed + 1000 * rank)

    import torch

    import cusbf_b200 as sbf

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream(dev)

    n_kmers_genome = max(0, joined.size - K + 1)
    requested_bits = int(round(spec["bits_per_kmer"] * n_ins_valid))
    f = sbf.Filter(requested_bits, k=K, s=S, m=M, hashes=H)
    n_shards = f.num_shards()

    d_genome = torch.from_numpy(joined).to(dev)
    from workloads.synthetic import SEPARATOR, reads_device, uniform_dna

    if spec["n_reads"] > 0:
        reads = reads_device(d_genome, spec["n_reads"], spec["read_len"],
                             seed=args.seed + 7 + 1000 * rank, sub_rate=spec["sub_rate"],
                             positive_frac=spec["positive_frac"], device=str(dev))
        rl = spec["read_len"]
        d_query = torch.full((spec["n_reads"], rl + 1), SEPARATOR, dtype=torch.uint8, device=dev)
        d_query[:, :rl] = reads
        d_query = d_query.reshape(-1)[:-1].contiguous()
        del reads
        n_q_valid = spec["n_reads"] * (rl - K + 1)
    else:
        fresh = uniform_dna(spec["fresh_query_bp"], seed=1337, gc=spec["gc"])
        q_host = np.concatenate([joined, np.frombuffer(b"N", np.uint8), fresh])
        d_query = torch.from_numpy(q_host).to(dev)
        n_q_valid = valid_windows(q_host)
    n_q_windows = f.kmer_count(d_query.numel())
    d_out = torch.empty(max(n_q_windows, 1), dtype=torch.uint8, device=dev)
    torch.cuda.synchronize(dev)

    def step(ev):
        f.clear(stream)  # synchronous, outside the insert/query events
        ev[0].record(stream)
        f.insert_sequence_async(d_genome, stream)
        ev[1].record(stream)
        f.contains_sequence_async(d_query, d_out, stream)
        ev[2].record(stream)

    for _ in range(args.warmup):
        step([torch.cuda.Event(enable_timing=True) for _ in range(3)])
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()

    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    t_start.record(stream)
    for i in range(args.steps):
        step(evs[i])
    t_end.record(stream)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clock_info = clocks.stop()
    total_ms = t_start.elapsed_time(t_end)
    ins_ms = float(np.mean([e[0].elapsed_time(e[1]) for e in evs]))
    q_ms = float(np.mean([e[1].elapsed_time(e[2]) for e in evs]))
    kmers_step = n_ins_valid + n_q_valid

    # Max over ranks of the timed region; sum of the work.
    total_ms, ins_ms, q_ms = max_over_ranks([total_ms, ins_ms, q_ms], dist, dev)
    ms_per_step = total_ms / args.steps
    value = whole_job_rate(world, kmers_step, ms_per_step)

    # Positive windows of the device-resident query: the end-to-end forms
    # below must return the same count (bit-exact parity with the reference
    # at this size is a GPU test, not part of the timed arm).
    positives = int(d_out.sum(dtype=torch.int64).item())

    # End-to-end through the host API with pinned buffers.
    e2e = e2e_bits = e2e_dense = None
    if not args.no_e2e:
        h_genome = torch.from_numpy(joined).pin_memory()
        h_query = torch.empty(d_query.numel(), dtype=torch.uint8).pin_memory()
        h_query.copy_(d_query)
        h_out = torch.empty(max(n_q_windows, 1), dtype=torch.uint8).pin_memory()
        gnp, qnp, onp = h_genome.numpy(), h_query.numpy(), h_out.numpy()

        def e2e_step():
            f.clear(stream)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            w0 = time.perf_counter()
            a.record(stream)
            f.insert_sequence(gnp, stream)
            sbf._check(sbf._lib.sbf_contains_sequence(f.handle, qnp.ctypes.data, qnp.size,
                                                       onp.ctypes.data, n_q_windows,
                                                       stream.cuda_stream))
            b.record(stream)
            torch.cuda.synchronize(dev)
            return a.elapsed_time(b), (time.perf_counter() - w0) * 1e3

        e2e_step()
        if dist:
            dist.barrier()
        res = [e2e_step() for _ in range(max(1, args.e2e_steps))]
        e_ms = float(np.mean([r[0] for r in res]))
        e_wall = float(np.mean([r[1] for r in res]))
        e_ms, e_wall = max_over_ranks([e_ms, e_wall], dist, dev)
        assert int(h_out[:n_q_windows].sum(dtype=torch.int64)) == positives, \
            "host-API query disagrees with the device-resident query"
        expand = sbf.host_expand_threads()
        e2e = {"value": world * kmers_step / (max(e_ms, e_wall) / 1e3), "unit": "k-mers/s",
               "h2d_bytes_per_step": int(joined.size + qnp.size),
               "d2h_bytes_per_step": int(4 * ((n_q_windows + 31) // 32) if expand
                                         else n_q_windows),
               "host_result_bytes": int(n_q_windows), "host_expand_threads": expand,
               "ms_per_step": max(e_ms, e_wall), "steps": len(res),
               "api": "sbf_insert_sequence + sbf_contains_sequence (host buffers, pinned; one "
                      "result byte per window in host memory, downloaded as bits and expanded "
                      "by host threads when host_expand_threads > 0)"}
        # The same step with bit-packed results (one bit per window).
        n_words = (n_q_windows + 31) // 32
        h_bits = torch.empty(max(n_words, 1), dtype=torch.int32).pin_memory()
        bnp = h_bits.numpy()

        def e2e_bits_step():
            f.clear(stream)
            torch.cuda.synchronize(dev)
            w0 = time.perf_counter()
            f.insert_sequence(gnp, stream)
            sbf._check(sbf._lib.sbf_contains_sequence_bits(f.handle, qnp.ctypes.data, qnp.size,
                                                            bnp.ctypes.data, n_words,
                                                            stream.cuda_stream))
            return (time.perf_counter() - w0) * 1e3

        e2e_bits_step()
        b_ms = float(np.mean([e2e_bits_step() for _ in range(max(1, args.e2e_steps))]))
        (b_ms,) = max_over_ranks([b_ms], dist, dev)
        got_pos = int(np.unpackbits(bnp.view(np.uint8), bitorder="little")[:n_q_windows].sum())
        assert got_pos == positives, "bit-packed query disagrees with the byte query"
        e2e_bits = {"value": world * kmers_step / (b_ms / 1e3), "unit": "k-mers/s",
                    "h2d_bytes_per_step": int(joined.size + qnp.size),
                    "d2h_bytes_per_step": int(4 * n_words), "ms_per_step": b_ms,
                    "api": "sbf_insert_sequence + sbf_contains_sequence_bits (host buffers, "
                           "pinned; one result bit per window)"}

        # The same step with 2-bit dense-packed input (the reference's dense
        # wire format, packed by the client before the step) and bit-packed
        # results: a quarter byte in and an eighth of a byte out per window.
        n_gs, n_qs = d_genome.numel(), d_query.numel()
        d_gw = torch.empty(sbf.Filter.dense_packed_word_count(n_gs), dtype=torch.int64, device=dev)
        d_qw = torch.empty(sbf.Filter.dense_packed_word_count(n_qs), dtype=torch.int64, device=dev)
        sbf.pack_dense_sequence_device(d_genome, n_gs, d_gw, stream)
        sbf.pack_dense_sequence_device(d_query, n_qs, d_qw, stream)
        h_gw = torch.empty(d_gw.numel(), dtype=torch.int64).pin_memory()
        h_qw = torch.empty(d_qw.numel(), dtype=torch.int64).pin_memory()
        torch.cuda.synchronize(dev)
        h_gw.copy_(d_gw)
        h_qw.copy_(d_qw)
        del d_gw, d_qw
        gw_np, qw_np = h_gw.numpy().view(np.uint64), h_qw.numpy().view(np.uint64)
        n_dense_windows = (n_gs - K + 1) + (n_qs - K + 1)

        def e2e_dense_step():
            f.clear(stream)
            torch.cuda.synchronize(dev)
            w0 = time.perf_counter()
            f.insert_dense_packed(gw_np, n_gs, stream)
            sbf._check(sbf._lib.sbf_contains_dense_packed_bits(
                f.handle, qw_np.ctypes.data, qw_np.size, n_qs, bnp.ctypes.data, n_words,
                stream.cuda_stream))
            return (time.perf_counter() - w0) * 1e3

        e2e_dense_step()
        d_ms = float(np.mean([e2e_dense_step() for _ in range(max(1, args.e2e_steps))]))
        (d_ms,) = max_over_ranks([d_ms], dist, dev)
        e2e_dense = {"value": world * n_dense_windows / (d_ms / 1e3), "unit": "k-mers/s",
                     "h2d_bytes_per_step": int(gw_np.nbytes + qw_np.nbytes),
                     "d2h_bytes_per_step": int(4 * n_words), "ms_per_step": d_ms,
                     "windows_per_step": int(n_dense_windows),
                     "api": "sbf_insert_dense_packed + sbf_contains_dense_packed_bits (host "
                            "buffers, pinned; 2-bit input, one result bit per window)",
                     "note": "dense packing stores N as a base (the reference's "
                             "pack_dense_sequence does the same), so every window is valid and "
                             "hit counts differ from the byte path on windows with N"}
        del h_bits, bnp, h_gw, h_qw, gw_np, qw_np

    if rank != 0:
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    # Roofline of the dominant kernel (query) and of insert: algorithmic bytes
    # from runs counted by the oracle on samples of this workload.
    q_sample = d_query[: min(d_query.numel(), 3_000_000)].cpu().numpy()
    runs_q, valid_q = sample_runs(q_sample, n_shards)
    r_per_q = runs_q / max(valid_q, 1)
    g_sample = joined[: min(joined.size, 6_000_000)]
    runs_i, valid_i = sample_runs(g_sample, n_shards)
    r_per_i = runs_i / max(valid_i, 1)
    q_bytes = d_query.numel() + n_q_windows + 32 * r_per_q * n_q_valid
    i_bytes = joined.size + 64 * r_per_i * n_ins_valid
    peaks = {}
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peaks = json.load(open(peaks_path))
    peak = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    traffic = i_traffic = None
    tr_path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if os.path.exists(tr_path):
        # DRAM bytes per unit from one ncu capture of this workload, scaled
        # to this run's units.
        tr = json.load(open(tr_path))
        if "query_bytes_per_window" in tr:
            traffic = int(tr["query_bytes_per_window"] * n_q_windows)
        if "insert_bytes_per_kmer" in tr:
            i_traffic = int(tr["insert_bytes_per_kmer"] * n_ins_valid)
    q_achieved = q_bytes / (q_ms / 1e3) / 1e9
    i_achieved = i_bytes / (ins_ms / 1e3) / 1e9
    sector_rate = random_sector_rate(f.words(), torch)
    sector = {"random_32B_sectors_per_s": sector_rate,
              "calibration": "torch.take of one 8-byte word from each of 2^26 random 32-byte "
                             "sectors of the filter words, best of 3",
              "query_runs_per_s": r_per_q * n_q_valid / (q_ms / 1e3),
              "insert_runs_per_s": r_per_i * n_ins_valid / (ins_ms / 1e3)}
    sector["query_frac"] = round(sector["query_runs_per_s"] / sector_rate, 4)
    sector["insert_frac"] = round(sector["insert_runs_per_s"] / sector_rate, 4)
    roofline = {"bound": "hbm", "kernel": "query (tile_kernel<31,28,16,4> query, bytes)",
                "achieved": round(q_achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(q_achieved / peak, 4), "peak_source": peak_src,
                "traffic": traffic,
                "algorithmic_bytes": int(q_bytes),
                "model": "L + N + 32R (input bytes + one output byte per window + one 32-byte "
                         f"sector per super-k-mer run; R/N={r_per_q:.4f} counted by the oracle "
                         "on a 3 MB sample)",
                "insert": {"achieved": round(i_achieved, 1), "frac": round(i_achieved / peak, 4),
                           "algorithmic_bytes": int(i_bytes), "traffic": i_traffic,
                           "model": f"L + 64R (R/N={r_per_i:.4f} counted on a 6 Mbp sample)"}}
    roofline_other = None
    if args.config != "c3" or args.scale != 1.0:
        # The committed DRAM bytes per window come from the 3.1 Gbp capture.
        roofline["traffic"] = None
        roofline["insert"]["traffic"] = None
    if args.config in ("c1", "c2"):
        # L2-resident (c1) or L2-straddling (c2) filters: the same algorithmic
        # bytes against the L2 copy bandwidth measured live.
        l2_peak = l2_copy_bandwidth(torch, dev) / 1e9
        l2_roof = dict(roofline, bound="l2", peak=round(l2_peak, 1),
                       frac=round(q_achieved / l2_peak, 4),
                       peak_source="measured live: L2-resident device copy (2 x 24 MiB, 200 "
                                   "copies in one CUDA graph, read + write bytes)",
                       insert=dict(roofline["insert"], frac=round(i_achieved / l2_peak, 4)))
        if args.config == "c1":
            roofline, roofline_other = l2_roof, ("roofline_hbm", roofline)
        else:
            roofline_other = ("roofline_l2", l2_roof)

    cpu = None
    if not args.no_cpu_baseline:
        c_ins, c_qry = cpu_sample(spec, joined, args.seed)
        cpu = cpu_reference_run(c_ins, c_qry, n_shards, steps=CPU_BASELINE_STEPS, warmup=1,
                                threads=host_cores())
        cpu = {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample", "steps")}

    line = {
        "metric": METRIC, "value": value, "unit": "k-mers/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded stand-in with the configuration's shapes; no public genome)",
        "config": plain_config(spec, world, f.filter_bits(), n_ins_valid, n_q_valid,
                               n_q_windows),
        "insert": {"ms": ins_ms, "kmers_per_s": n_ins_valid / (ins_ms / 1e3)},
        "query": {"ms": q_ms, "kmers_per_s": n_q_valid / (q_ms / 1e3),
                  "positives": positives},
        "roofline": roofline,
        **(dict([roofline_other]) if roofline_other else {}),
        "sector_roofline": sector,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "e2e_bits": e2e_bits,
        "e2e_dense": e2e_dense,
        "gpu_launches": 2 * args.steps,
        "clocks": clock_info,
    }
    f.close()
    if world == 1 and args.config == "c3" and args.scale == 1.0 and not args.no_forms:
        # The ragged-batch and served forms of the metric, each measured in a
        # child process on this GPU once this workload's buffers are freed.
        del d_genome, d_query, d_out
        if not args.no_e2e:
            del h_genome, h_query, h_out, gnp, qnp, onp
        torch.cuda.synchronize(dev)
        torch.cuda.empty_cache()
        line["ragged_batch"] = run_form(["--config", "c4", "--steps", "5", "--warmup", "3"],
                                        summarize_ragged)
        line["served"] = run_form(["--config", "c5", "--duration", "2.0"], summarize_served)
        line["served_bits"] = run_form(["--config", "c5", "--duration", "2.0", "--server-bits",
                                        "--no-serial"], summarize_served)
        line["served_counts"] = run_form(["--config", "c5", "--duration", "2.0",
                                          "--server-counts", "--no-serial"], summarize_served)
        line["served_dense_bits"] = run_form(["--config", "c5", "--duration", "2.0",
                                              "--server-dense", "--server-bits", "--no-serial"],
                                             summarize_served)
        line["fastx_files"] = run_form(["--config", "fastx", "--steps", "2"], summarize_fastx)
        line["c1"] = run_form(["--config", "c1", "--steps", "20", "--warmup", "5"],
                              summarize_plain)
        line["c2"] = run_form(["--config", "c2", "--steps", "10", "--warmup", "3"],
                              summarize_plain)
        line["other_configs"] = run_form(["--config", "configs", "--steps", "5", "--warmup", "3"],
                                         summarize_configs)
        line["fpr"] = run_form(["--config", "fpr"], summarize_fpr)
        # Last, so that it stays in the tail of the line: the headline figures
        # of every configuration in a few hundred bytes.
        line["summary"] = compact_summary(line)
    print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_form(extra: list[str], summarize) -> dict:
    """Runs bench.py with `extra` arguments in a child process and returns the
    summary of its JSON line (or the failure)."""
    cmd = [sys.executable, os.path.join(ROOT, "bench.py"), *extra]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=900)
    except subprocess.TimeoutExpired:
        return {"error": "timed out", "command": " ".join(extra)}
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    if r.returncode != 0 or not lines:
        return {"error": f"exit {r.returncode}: {r.stderr.strip()[-300:]}",
                "command": " ".join(extra)}
    out = summarize(json.loads(lines[-1]))
    out["command"] = "python bench.py " + " ".join(extra)
    return out


def summarize_ragged(d: dict) -> dict:
    pl = d.get("plain_per_record") or {}
    e2e, tuned, rb = d.get("e2e") or {}, d.get("e2e_tuned") or {}, d.get("record_batch_e2e") or {}
    return {"metric": d["metric"], "workload": d["config"]["workload"],
            "kmers_per_s": d["value"], "insert_kmers_per_s": d["insert"]["kmers_per_s"],
            "query_kmers_per_s": d["query"]["kmers_per_s"],
            "roofline_frac": d["roofline"]["frac"],
            "plain_per_record_kmers_per_s": pl.get("kmers_per_s"),
            "speedup_vs_plain_per_record": d.get("speedup_vs_plain"),
            "plain_hits_identical": pl.get("query_hits_identical_to_ragged"),
            "e2e_kmers_per_s": e2e.get("value"), "e2e_tuned_kmers_per_s": tuned.get("value"),
            "e2e_bits_kmers_per_s": (d.get("e2e_bits") or {}).get("value"),
            "record_batch_e2e_kmers_per_s": rb.get("value")}


def summarize_plain(d: dict) -> dict:
    """Summary of a plain-configuration line (c1, c2) for the default run."""
    out = {"metric": d["metric"], "workload": d["config"]["workload"],
           "filter_bits": d["config"]["filter_bits"], "l2": d["config"]["l2"],
           "kmers_per_s": d["value"], "insert_kmers_per_s": d["insert"]["kmers_per_s"],
           "query_kmers_per_s": d["query"]["kmers_per_s"], "ms_per_step": d["ms_per_step"],
           "steps": d["steps"], "warmup": d["warmup"],
           "e2e_kmers_per_s": (d.get("e2e") or {}).get("value"),
           "cpu_baseline": d.get("cpu_baseline")}
    for key in ("roofline", "roofline_l2", "roofline_hbm"):
        r = d.get(key)
        if r:
            out[key] = {"bound": r["bound"], "achieved": r["achieved"], "peak": r["peak"],
                        "unit": r["unit"], "frac": r["frac"], "insert_frac": r["insert"]["frac"],
                        "peak_source": r["peak_source"]}
    return out


def summarize_fastx(d: dict) -> dict:
    keep = ("insert_gb_per_s", "query_gb_per_s", "insert_kmers_per_s", "query_kmers_per_s")
    return {"metric": d["metric"], "workload": d["config"]["workload"],
            "graph": {k: d["graph"][k] for k in keep},
            "stream": {k: d["stream"][k] for k in keep},
            "host_parser": {k: d["host_parser"][k] for k in keep},
            "identical_across_paths": d["identical_across_paths"]}


def compact_summary(line: dict) -> dict:
    """Headline numbers of the default run, G k-mers/s unless named."""
    def g(x):
        return None if x is None else round(x / 1e9, 2)

    out = {"c3": {"gkmers": g(line["value"]), "ins": g(line["insert"]["kmers_per_s"]),
                  "qry": g(line["query"]["kmers_per_s"]), "e2e": g((line.get("e2e") or {}).get("value")),
                  "frac_hbm": line["roofline"]["frac"],
                  "sector_frac_q": line["sector_roofline"]["query_frac"]}}
    for c in ("c1", "c2"):
        d = line.get(c) or {}
        if "kmers_per_s" in d:
            out[c] = {"gkmers": g(d["kmers_per_s"]), "ins": g(d["insert_kmers_per_s"]),
                      "qry": g(d["query_kmers_per_s"]), "e2e": g(d.get("e2e_kmers_per_s")),
                      "frac": (d.get("roofline") or {}).get("frac"),
                      "bound": (d.get("roofline") or {}).get("bound")}
            if "roofline_l2" in d:
                out[c]["frac_l2"] = d["roofline_l2"]["frac"]
    rb = line.get("ragged_batch") or {}
    if "kmers_per_s" in rb:
        out["c4"] = {"gkmers": g(rb["kmers_per_s"]), "e2e": g(rb.get("e2e_kmers_per_s")),
                     "e2e_tuned": g(rb.get("e2e_tuned_kmers_per_s")),
                     "plain_per_record": g(rb.get("plain_per_record_kmers_per_s")),
                     "speedup_vs_plain": rb.get("speedup_vs_plain_per_record"),
                     "identical": rb.get("plain_hits_identical")}
    fp = line.get("fpr") or {}
    if "fpr_pct" in fp:
        out["fpr_pct"] = fp["fpr_pct"]
    oc = line.get("other_configs") or {}
    if "g_windows_per_s" in oc:
        out["other_configs_gwin_s"] = oc["g_windows_per_s"]
    fx = line.get("fastx_files") or {}
    if "graph" in fx:
        out["fastx_gb_s"] = {m: [round(fx[m]["insert_gb_per_s"], 2), round(fx[m]["query_gb_per_s"], 2)]
                             for m in ("graph", "stream", "host_parser")}
    for key in ("served", "served_bits", "served_counts", "served_dense_bits"):
        sv = line.get(key) or {}
        if "latency_ms" in sv:
            lat = sv["latency_ms"]
            out[key] = {"req_s": round(sv["requests_per_s"]), "p50_ms": round(lat["p50"], 2),
                        "p99_ms": round(lat["p99"], 2), "p999_ms": round(lat["p999"], 2)}
    return out


def summarize_served(d: dict) -> dict:
    sv, one, pl = d["served"], d.get("one_request_per_launch") or {}, d["plain_per_record"]
    return {"metric": d["metric"], "workload": d["config"]["workload"],
            "query_results": d["config"]["query_results"],
            "request_bodies": d["config"].get("request_bodies"),
            "offered_gb_per_s": d["config"]["offered_gb_per_s"],
            "kmers_per_s": sv["kmers_per_s"], "requests_per_s": sv["requests_per_s"],
            "latency_ms": sv["latency_ms"], "mean_batch_requests": sv["mean_batch_requests"],
            "one_request_per_launch": {"requests_per_s": one.get("requests_per_s"),
                                       "latency_ms": one.get("latency_ms")},
            "plain_per_record_sustainable_requests_per_s": pl["sustainable_requests_per_s"],
            "identical_to_one_at_a_time": d.get("identical_to_one_at_a_time")}


def run_reference_arm(args, spec, world) -> None:
    """The reference's own CPU implementation of the path (rank 0 only), on
    the bounded sample that the main arm's cpu_baseline also times
    (cpu_sample), with the full workload's filter size and the main arm's
    `config`.  Nothing here loads the engine's library."""
    from oracle.oracle import num_shards

    joined, _, n_ins_valid = build_host_genome(spec, seed=args.seed)
    requested = int(round(spec["bits_per_kmer"] * n_ins_valid))
    shards = num_shards(requested)
    n_q_valid, n_q_windows = query_counts(spec, joined)
    c_ins, c_qry = cpu_sample(spec, joined, args.seed)
    res = cpu_reference_run(c_ins, c_qry, shards, steps=args.steps, warmup=args.warmup,
                            threads=host_cores())
    line = {
        "metric": METRIC, "value": res["value"], "unit": "k-mers/s", "impl": "reference",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": res["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded stand-in with the configuration's shapes; no public genome)",
        "config": plain_config(spec, world, shards * 256, n_ins_valid, n_q_valid, n_q_windows),
        "cpu_baseline": {"value": res["value"], "unit": "k-mers/s", "cores": res["cores"],
                         "kind": res["kind"], "sample": res["sample"]},
        "e2e": {"value": res["value"], "unit": "k-mers/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if not args.no_reference_gpu:
        line["reference_gpu"] = reference_gpu_run(args, spec, joined, n_ins_valid)
        if world == 1 and args.config == "c3" and args.scale == 1.0 and not args.no_forms:
            line["reference_gpu_other_configs"] = run_form(
                ["--config", "configs", "--impl", "reference", "--steps", "5", "--warmup", "3"],
                summarize_configs)
            line["reference_gpu_fpr"] = run_form(["--config", "fpr", "--impl", "reference"],
                                                 summarize_fpr)
    print(json.dumps(line), flush=True)


def reference_gpu_run(args, spec, joined: np.ndarray, n_ins_valid: int) -> dict:
    """The unmodified reference cuSBF GPU path (oracle/_ref, compiled from the
    reference headers) on this workload at full size, device-resident inputs,
    timed like the main arm: insert_sequence_async over the genome joined with
    separators, contains_sequence_async over the reads joined with separators."""
    from oracle.oracle import RefGpu

    if not RefGpu.available():
        return {"unavailable": "oracle/_ref/libsbf_refgpu.so was not built"}
    import torch

    from workloads.synthetic import SEPARATOR, reads_device, uniform_dna

    dev = torch.device("cuda", 0)
    d_genome = torch.from_numpy(joined).to(dev)
    if spec["n_reads"] > 0:
        rl = spec["read_len"]
        reads = reads_device(d_genome, spec["n_reads"], rl, seed=args.seed + 7,
                             sub_rate=spec["sub_rate"], positive_frac=spec["positive_frac"],
                             device=str(dev))
        d_query = torch.full((spec["n_reads"], rl + 1), SEPARATOR, dtype=torch.uint8, device=dev)
        d_query[:, :rl] = reads
        d_query = d_query.reshape(-1)[:-1].contiguous()
        del reads
        n_q_valid = spec["n_reads"] * (rl - K + 1)
    else:
        fresh = uniform_dna(spec["fresh_query_bp"], seed=1337, gc=spec["gc"])
        q_host = np.concatenate([joined, np.frombuffer(b"N", np.uint8), fresh])
        d_query = torch.from_numpy(q_host).to(dev)
        n_q_valid = valid_windows(q_host)
    n_out = max(d_query.numel() - K + 1, 1)
    d_out = torch.empty(n_out, dtype=torch.uint8, device=dev)
    ref = RefGpu(int(round(spec["bits_per_kmer"] * n_ins_valid)))
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    ins, qry = [], []
    for i in range(3 + max(args.steps, 1)):
        ref.clear(sp)
        a, b, c = _ev(torch), _ev(torch), _ev(torch)
        a.record(stream)
        assert ref.lib.sbf_refgpu_insert_async(ref.h, d_genome.data_ptr(), d_genome.numel(),
                                               sp) == 0
        b.record(stream)
        assert ref.lib.sbf_refgpu_contains_async(ref.h, d_query.data_ptr(), d_query.numel(),
                                                 d_out.data_ptr(), n_out, sp) == 0
        c.record(stream)
        torch.cuda.synchronize(dev)
        if i >= 3:
            ins.append(a.elapsed_time(b))
            qry.append(b.elapsed_time(c))
    ref.close()
    ins_ms, q_ms = float(np.mean(ins)), float(np.mean(qry))
    return {"kmers_per_s": (n_ins_valid + n_q_valid) / ((ins_ms + q_ms) / 1e3),
            "insert_kmers_per_s": n_ins_valid / (ins_ms / 1e3), "insert_ms": ins_ms,
            "query_kmers_per_s": n_q_valid / (q_ms / 1e3), "query_ms": q_ms,
            "steps": len(ins), "warmup": 3,
            "path": "reference cuSBF filter<Config<31,28,16,4>> insert_sequence_async + "
                    "contains_sequence_async, device-resident inputs, CUDA events"}


if __name__ == "__main__":
    main()
