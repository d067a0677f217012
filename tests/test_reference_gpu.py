"""Bit-identity with the reference cuSBF GPU path itself: the unmodified
filter<Config> insert_sequence_async / contains_sequence_async, compiled from
the reference headers into oracle/_ref/libsbf_refgpu.so, run on the same
device input with the same requested filter size.  The shard word arrays and
every query byte must be equal (compared on the device)."""
import numpy as np
import pytest

from conftest import random_dna

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refgpu(oracle_mod):
    if not oracle_mod.RefGpu.available():
        pytest.skip("oracle/_ref/libsbf_refgpu.so is not built (needs the reference sources)")
    return oracle_mod.RefGpu


def _ref_words(torch, ref, n_words):
    from cuda.bindings import runtime as rt

    out = torch.empty(n_words, dtype=torch.int64, device="cuda")
    (err,) = rt.cudaMemcpy(out.data_ptr(), ref.words_ptr(), n_words * 8,
                           rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
    assert int(err) == 0
    return out


def _compare(sbf, torch, refgpu, cfg_id, cfg, bits, d_ins, d_qry):
    f = sbf.Filter(bits, **cfg)
    ref = refgpu(bits, cfg_id)
    assert ref.num_shards() == f.num_shards()
    f.insert_sequence_async(d_ins)
    ref.insert_async(d_ins.data_ptr(), d_ins.numel())
    n_out = max(f.kmer_count(d_qry.numel()), 1)
    ours = torch.full((n_out,), 7, dtype=torch.uint8, device="cuda")
    theirs = torch.full((n_out,), 9, dtype=torch.uint8, device="cuda")
    f.contains_sequence_async(d_qry, ours)
    ref.contains_async(d_qry.data_ptr(), d_qry.numel(), theirs.data_ptr(), n_out)
    torch.cuda.synchronize()
    p, n = f.words_ptr()
    mine = torch.empty(n, dtype=torch.int64, device="cuda")
    from cuda.bindings import runtime as rt

    (err,) = rt.cudaMemcpy(mine.data_ptr(), p, n * 8, rt.cudaMemcpyKind.cudaMemcpyDeviceToDevice)
    assert int(err) == 0
    assert torch.equal(mine, _ref_words(torch, ref, n)), "shard words differ from the reference"
    if d_qry.numel() >= cfg["k"]:
        assert torch.equal(ours, theirs), "query bytes differ from the reference"
    assert int(mine.count_nonzero()) > 0 or d_ins.numel() < cfg["k"]
    ref.close()
    f.close()


def test_plain_small_workload(sbf, cuda, refgpu):
    """2 Mbp uniform record at 85.7 bits per k-mer; query it plus a fresh 2 Mbp."""
    torch = cuda
    from workloads.synthetic import uniform_dna

    ins = uniform_dna(2_000_000, seed=42)
    qry = np.concatenate([ins, np.frombuffer(b"N", np.uint8), uniform_dna(2_000_000, seed=1337)])
    bits = int(round(85.7 * (ins.size - 30)))
    _compare(sbf, torch, refgpu, 0, dict(k=31, s=28, m=16, hashes=4), bits,
             torch.from_numpy(ins).cuda(), torch.from_numpy(qry).cuda())


def test_genome_like_with_repeats_and_n_runs(sbf, cuda, refgpu):
    """Records with tandem repeats, interspersed repeat copies and N runs,
    joined with separators; reads with substitutions joined with separators."""
    torch = cuda
    from workloads.synthetic import SEPARATOR, genome_records, join_records, reads_device

    recs = genome_records(24_000_000, 4, seed=5, gc=0.38, tandem_frac=0.03, n_run_frac=0.001,
                          interspersed_frac=0.3, processes=1)
    joined, _ = join_records(recs)
    d_g = torch.from_numpy(joined).cuda()
    reads = reads_device(d_g, 300_000, 150, seed=6, sub_rate=0.01, positive_frac=0.5)
    q = torch.full((300_000, 151), SEPARATOR, dtype=torch.uint8, device="cuda")
    q[:, :150] = reads
    bits = int(round(21.4 * joined.size))
    _compare(sbf, torch, refgpu, 0, dict(k=31, s=28, m=16, hashes=4), bits, d_g,
             q.reshape(-1)[:-1].contiguous())


def test_large_single_launch(sbf, cuda, refgpu):
    """600 Mbp in one launch (beyond 2^29 windows), 2^33-bit filter."""
    torch = cuda
    g = torch.Generator(device="cuda").manual_seed(11)
    lut = torch.tensor(list(b"ACGT"), dtype=torch.uint8, device="cuda")
    d = lut[torch.randint(0, 4, (600_000_000,), device="cuda", generator=g, dtype=torch.int32)]
    q = d.clone()
    q[300_000_000:] = lut[torch.randint(0, 4, (300_000_000,), device="cuda", generator=g,
                                        dtype=torch.int32)]
    _compare(sbf, torch, refgpu, 0, dict(k=31, s=28, m=16, hashes=4), 1 << 33, d, q)


@pytest.mark.parametrize("cfg_id,cfg", [(4, dict(k=31, s=28, m=16, hashes=8)),
                                        (5, dict(k=31, s=28, m=16, hashes=16)),
                                        (6, dict(k=21, s=19, m=11, hashes=4)),
                                        (1, dict(k=5, s=4, m=3, hashes=4)),
                                        (7, dict(k=31, s=28, m=21, hashes=4)),
                                        (8, dict(k=25, s=22, m=13, hashes=4)),
                                        (9, dict(k=12, s=10, m=6, hashes=4, alphabet=2)),
                                        (10, dict(k=31, s=30, m=16, hashes=4)),
                                        (11, dict(k=31, s=31, m=16, hashes=4))])
def test_other_configs(sbf, cuda, refgpu, cfg_id, cfg):
    """Specialised (4, 5, 6, 1, 7, 10, 11) and generic (8, and the protein
    alphabet 9) engine kernels against the reference GPU path for that
    configuration."""
    torch = cuda
    rng = np.random.default_rng(cfg_id)
    if cfg.get("alphabet") == 2:
        a = np.frombuffer(b"ACDEFGHIKLMNPQRSTVWYacdefghiklmnpqrstvwy*X-", np.uint8)
        ins = a[rng.integers(0, a.size, 3_000_000)]
        qry = np.concatenate([ins[:1_000_000], a[rng.integers(0, a.size, 1_000_000)]])
    else:
        ins = random_dna(rng, 3_000_000, b"ACGTACGTACGTACGTACGTN")
        qry = np.concatenate([ins[:1_000_000], random_dna(rng, 1_000_000)])
    _compare(sbf, torch, refgpu, cfg_id, cfg, 1 << 24, torch.from_numpy(ins).cuda(),
             torch.from_numpy(qry).cuda())
