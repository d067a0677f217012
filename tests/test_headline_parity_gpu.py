"""Bit-identity with the reference cuSBF GPU path at the benchmark's full sizes.

The workloads are built by the same functions and seeds as bench.py:
  * plain-large: 3.1 Gbp in 24 records (2^36-bit filter, 2^28 shards)
    inserted, 100M x 150 bp reads joined by separators queried
    (1.51e10 windows, beyond 2^32, so every 64-bit index path of the tile
    kernels runs);
  * plain-genome-small: 100 Mbp in 6 records with tandem repeats and N runs
    (2^31-bit filter), 20M x 150 bp reads.
The engine and the unmodified reference filter<Config<31,28,16,4>>
(oracle/_ref/libsbf_refgpu.so) run on the same device buffers; every shard
word and every query byte is compared on the device.  The engine's
bit-packed query output is also checked against the reference's bytes."""
import os
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

SEED = 42  # bench.py's default --seed


@pytest.fixture(scope="module")
def refgpu(oracle_mod):
    if not oracle_mod.RefGpu.available():
        pytest.skip("oracle/_ref/libsbf_refgpu.so is not built (needs the reference sources)")
    return oracle_mod.RefGpu


def _device_view(torch, ptr: int, n_words: int):
    """A uint64 CUDA tensor over `n_words` words at device address `ptr`."""

    class _View:
        __cuda_array_interface__ = {"shape": (n_words,), "typestr": "<u8", "data": (ptr, False),
                                    "version": 3, "strides": None}

    return torch.as_tensor(_View(), device="cuda")


def _workload(torch, name):
    import bench
    from workloads.synthetic import SEPARATOR, reads_device

    spec = bench.workload_spec(name, 1.0)
    joined, _, n_ins_valid = bench.build_host_genome(spec, seed=SEED)
    d_genome = torch.from_numpy(joined).cuda()
    del joined
    rl = spec["read_len"]
    reads = reads_device(d_genome, spec["n_reads"], rl, seed=SEED + 7, sub_rate=spec["sub_rate"],
                         positive_frac=spec["positive_frac"], device="cuda")
    d_query = torch.full((spec["n_reads"], rl + 1), SEPARATOR, dtype=torch.uint8, device="cuda")
    d_query[:, :rl] = reads
    del reads
    d_query = d_query.reshape(-1)[:-1]
    bits = int(round(spec["bits_per_kmer"] * n_ins_valid))
    return d_genome, d_query, bits


def _bits_match_bytes(torch, bits, hits, n_windows):
    """Bit i % 32 of word i / 32 of `bits` equals byte i of `hits`, in chunks."""
    shifts = torch.arange(32, device="cuda", dtype=torch.int64)
    chunk = 1 << 28
    for c0 in range(0, n_windows, chunk):
        c1 = min(c0 + chunk, n_windows)
        h = hits[c0:c1]
        pad = (-h.numel()) % 32
        if pad:
            h = torch.cat([h, torch.zeros(pad, dtype=torch.uint8, device="cuda")])
        packed = (h.view(-1, 32).to(torch.int64) << shifts).sum(1)
        words = bits[c0 // 32:c0 // 32 + packed.numel()].to(torch.int64) & 0xFFFFFFFF
        if not torch.equal(packed, words):
            return False
    return True


@pytest.mark.parametrize("name", ["c2", "c3"])
def test_full_size_equals_reference(sbf, cuda, refgpu, name):
    torch = cuda
    d_genome, d_query, bits = _workload(torch, name)
    f = sbf.Filter(bits, k=31, s=28, m=16, hashes=4)
    ref = refgpu(bits, 0)
    assert ref.num_shards() == f.num_shards()
    if name == "c3":
        assert f.filter_bits() == 1 << 36
    f.insert_sequence_async(d_genome)
    ref.insert_async(d_genome.data_ptr(), d_genome.numel())
    torch.cuda.synchronize()
    p, n = f.words_ptr()
    mine = _device_view(torch, p, n)
    theirs = _device_view(torch, ref.words_ptr(), n)
    assert torch.equal(mine, theirs), "shard words differ from the reference"
    del d_genome

    n_out = f.kmer_count(d_query.numel())
    if name == "c3":
        assert n_out > 1 << 32
    ours = torch.full((n_out,), 7, dtype=torch.uint8, device="cuda")
    f.contains_sequence_async(d_query, ours)
    torch.cuda.synchronize()
    ref_out = torch.full((n_out,), 9, dtype=torch.uint8, device="cuda")
    ref.contains_async(d_query.data_ptr(), d_query.numel(), ref_out.data_ptr(), n_out)
    torch.cuda.synchronize()
    assert torch.equal(ours, ref_out), "query bytes differ from the reference"
    # Counted in slices: a reduction over the whole byte array would
    # materialise it as int64 (8x its size).
    positives = sum(int(torch.count_nonzero(ours[i:i + (1 << 28)]))
                    for i in range(0, n_out, 1 << 28))
    assert 0 < positives < n_out
    del ours

    out_bits = torch.zeros((n_out + 31) // 32, dtype=torch.int32, device="cuda")
    f.contains_sequence_bits_async(d_query, out_bits)
    torch.cuda.synchronize()
    assert _bits_match_bytes(torch, out_bits, ref_out, n_out), \
        "bit-packed query differs from the reference's bytes"
    ref.close()
    f.close()
