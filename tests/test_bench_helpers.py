"""bench.py helpers shared by the main arm and the reference arm: the CPU
sample both arms time is one deterministic function of the workload, and the
host-side query counts equal a direct count over the query bytes the main arm
builds on the device."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def test_cpu_sample_is_deterministic_and_bounded():
    import bench

    spec = bench.workload_spec("c3", 0.01)
    joined, _, _ = bench.build_host_genome(spec, seed=42)
    a_ins, a_q = bench.cpu_sample(spec, joined, 42)
    b_ins, b_q = bench.cpu_sample(spec, joined, 42)
    assert np.array_equal(a_ins, b_ins) and np.array_equal(a_q, b_q)
    assert a_ins.size == min(joined.size, bench.CPU_SAMPLE_BP)
    assert a_q.size == bench.CPU_SAMPLE_READS * (spec["read_len"] + 1) - 1
    # Reads are joined by one separator each.
    rl = spec["read_len"]
    assert (a_q[rl::rl + 1] == ord("N")).all()


def test_query_counts_match_the_query_layout():
    import bench

    spec = bench.workload_spec("c3", 0.001)
    n_q_valid, n_q_windows = bench.query_counts(spec, np.zeros(0, np.uint8))
    rl, n = spec["read_len"], spec["n_reads"]
    q = np.full((n, rl + 1), ord("N"), np.uint8)
    q[:, :rl] = ord("A")
    q = q.reshape(-1)[:-1]
    assert n_q_windows == q.size - bench.K + 1
    assert n_q_valid == bench.valid_windows(q)


def test_plain_config_is_the_same_for_both_arms():
    import bench

    spec = bench.workload_spec("c3", 1.0)
    a = bench.plain_config(spec, 1, 1 << 36, 3099999280, 12000000000, 15099999969)
    b = bench.plain_config(spec, 1, 1 << 36, 3099999280, 12000000000, 15099999969)
    assert a == b
    assert a["workload"].startswith("plain-large: 3.1 Gbp in 24 records")
    assert a["filter_bits"] == 1 << 36


def test_other_config_inputs_share_the_insert_half():
    """Both arms of `--config configs` build their inputs with this function:
    the query repeats the insert input's first half, the rest is fresh, and
    only the configuration's letters occur."""
    import torch

    import bench

    for name, cfg_id, cfg, letters in bench.OTHER_CONFIGS:
        a_ins, a_q = bench.other_config_inputs(torch, torch.device("cpu"), letters, 10_001, 5)
        b_ins, b_q = bench.other_config_inputs(torch, torch.device("cpu"), letters, 10_001, 5)
        assert torch.equal(a_ins, b_ins) and torch.equal(a_q, b_q)
        assert torch.equal(a_q[:5000], a_ins[:5000])
        assert not torch.equal(a_q[5000:], a_ins[5000:])
        assert set(a_ins.unique().tolist()) | set(a_q.unique().tolist()) <= set(letters)
        assert cfg["k"] <= 31 and cfg_id in range(10), name


def test_fpr_form_tables():
    """The FPR form sweeps s = 28, 30, 31 at three filter sizes, each beside
    the reference's published rate for that cell, and its summary keeps one
    entry per cell."""
    import bench

    assert [s for s, _ in bench.FPR_S] == [28, 30, 31]
    for s, _ in bench.FPR_S:
        assert len(bench.FPR_PUBLISHED[s]) == len(bench.FPR_SIZE_FACTORS)
    rows = [{"s": s, "bits_per_kmer": 21.47 * f, "fpr_pct": 0.5, "published_pct": p,
             "positives": 5} for s, _ in bench.FPR_S
            for f, p in zip(bench.FPR_SIZE_FACTORS, bench.FPR_PUBLISHED[s])]
    d = {"metric": bench.FPR_METRIC, "config": {"workload": "w"}, "fpr": rows}
    out = bench.summarize_fpr(d)
    assert len(out["fpr_pct"]) == len(out["published_pct"]) == 9
    assert bench.summarize_fpr({"unavailable": "x"}) == {"unavailable": "x"}


def test_reference_forms_report_unavailable_without_the_build(monkeypatch, capsys):
    """Without oracle/_ref/libsbf_refgpu.so the reference arm's configuration
    and false-positive forms print one `unavailable` line and touch no GPU."""
    import argparse
    import json

    import bench
    from oracle import oracle

    monkeypatch.setattr(oracle.RefGpu, "available", staticmethod(lambda: False))
    args = argparse.Namespace(impl="reference", scale=1.0, seed=42, steps=1, warmup=3)
    for run, metric in ((bench.run_other_configs, bench.CONFIGS_METRIC),
                        (bench.run_fpr, bench.FPR_METRIC)):
        run(args)
        line = json.loads(capsys.readouterr().out.strip().splitlines()[-1])
        assert line["impl"] == "reference" and line["metric"] == metric
        assert "unavailable" in line
