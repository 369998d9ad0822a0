"""The reference arm of bench.py (`--impl reference`) runs the CPU restatement
of the reference's TBPM time step on the host cores.  On a small grid its one
JSON line must carry the benchmark contract: the same metric and unit as the
GPU arm, impl = "reference", a cpu_baseline describing the run, and an e2e
object with no host/device copies.  The algorithmic byte model of the GPU arm
is checked against a term-by-term count of the flush schedule.
"""

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_reference_arm_prints_the_contract_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "3", "--nx", "32", "--ny", "32"],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    d = json.loads(out.stdout.strip().splitlines()[-1])
    assert d["impl"] == "reference"
    assert d["metric"] == "orbital-steps/s (TBPM DOS time step, FP64)"
    assert d["unit"] == "orbital-steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["warmup"] >= 3 and d["steps"] == 1
    cb = d["cpu_baseline"]
    assert cb["kind"] in ("port", "reference") and cb["cores"] >= 1 and cb["value"] == d["value"]
    e2e = d["e2e"]
    assert e2e["value"] == d["value"] and e2e["unit"] == d["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


@pytest.mark.parametrize("n_bes", [20, 16, 7])
def test_algorithmic_bytes_follow_the_flush_schedule(n_bes):
    """Terms k = 1..n_bes-1: CSR + gathered p_{k-1}; k = 1 writes p_1; later terms
    read p_{k-2} and write p_k (not the last term); a flush at k = 2, after three
    pending terms, and at the last term reads and writes the accumulator (only
    writes it at k = 2); the last term also reads the correlation reference."""
    n, nnz, ld, rb = 1000, 3000, 16, 8
    sv = 2 * rb
    vec = n * ld * sv
    mat = (n + 1) * 4 + nnz * (4 + sv)
    want = 0
    last = 1
    for k in range(1, n_bes):
        b = mat + vec + vec  # CSR, gather, and p_1 (k = 1) or p_{k-2}
        if k >= 2 and k < n_bes - 1:
            b += vec  # write p_k
        if k >= 2 and (k == 2 or k - last == 3 or k == n_bes - 1):
            b += vec if k == 2 else 2 * vec
            last = k
        if k == n_bes - 1:
            b += vec
        want += b
    assert bench.algorithmic_bytes_per_step(n, nnz, ld, n_bes, rb) == want


@pytest.mark.parametrize("n_bes", [4, 5, 7, 20, 21])
@pytest.mark.parametrize("with_ref", [True, False])
def test_paired_bytes_drop_the_second_terms_l2_reads(n_bes, with_ref):
    """Paired terms (k, k+1) for k = 1, 3, ...: the second term of each pair
    reads the CSR, p_k and its own p_{k-1} rows from L2, so each pair saves
    the CSR and two vector passes; a last term with the correlation and two
    flush terms in a row stay single."""
    n, nnz, ld, rb = 1000, 3000, 16, 8
    sv = 2 * rb
    vec = n * ld * sv
    mat = (n + 1) * 4 + nnz * (4 + sv)
    flush, last = set(), -1
    for k in range(2, n_bes):
        if k == 2 or k - last == 3 or k == n_bes - 1:
            flush.add(k)
            last = k
    pairs, k = 0, 1
    while k < n_bes:
        if k + 1 < n_bes and not (with_ref and k + 1 == n_bes - 1) and \
                not (k in flush and k + 1 in flush):
            pairs += 1
            k += 2
        else:
            k += 1
    single = bench.algorithmic_bytes_per_step(n, nnz, ld, n_bes, rb, with_ref=with_ref)
    paired = bench.algorithmic_bytes_per_step(n, nnz, ld, n_bes, rb, paired=True,
                                              with_ref=with_ref)
    assert paired == pytest.approx(single - pairs * (mat + 2 * vec), rel=1e-15)
    if n_bes == 20 and with_ref:
        assert pairs == 9
