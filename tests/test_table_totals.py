"""Per-sample totals of a borrowed table (Table::compute_totals, the
reference's biom_inmem sample sums in observation order,
src/biom_inmem.cpp:513-526).  Large tables are summed by observation ranges
on several threads when every entry is an integer (partial sums of integers
below 2^52 are exact in any order); the totals must equal the
observation-order sums bit for bit whatever the thread count, for integer
counts and, through the sequential fallback, for fractional values.  A host
program built from the table source checks this on the CPU."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "unifrac-binaries_b200", "csrc")

PROBE = r"""
#include <cstdio>
#include <cstring>
#include <vector>
#include "ssu_table.hpp"
int main(int argc, char **argv) {
    std::FILE *f = std::fopen(argv[1], "rb");
    uint32_t n_obs = 0, n_samples = 0;
    uint64_t nnz = 0;
    if (std::fread(&n_obs, 4, 1, f) != 1 || std::fread(&n_samples, 4, 1, f) != 1 || std::fread(&nnz, 8, 1, f) != 1)
        return 2;
    std::vector<uint32_t> indptr(n_obs + 1), indices(nnz);
    std::vector<double> data(nnz);
    if (std::fread(indptr.data(), 4, n_obs + 1, f) != n_obs + 1 || std::fread(indices.data(), 4, nnz, f) != nnz ||
        std::fread(data.data(), 8, nnz, f) != nnz)
        return 3;
    std::fclose(f);
    std::vector<const char *> ids(n_obs > n_samples ? n_obs : n_samples, "x");
    ssu::Table t = ssu::Table::borrow(n_obs, n_samples, indptr.data(), indices.data(), data.data(), ids.data(),
                                      ids.data());
    std::FILE *o = std::fopen(argv[2], "wb");
    std::fwrite(t.totals.data(), 8, t.totals.size(), o);
    const uint8_t flags[2] = {static_cast<uint8_t>(t.nonneg), static_cast<uint8_t>(t.malformed)};
    std::fwrite(flags, 1, 2, o);
    std::fclose(o);
    return 0;
}
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    d = tmp_path_factory.mktemp("totals")
    src = d / "probe.cpp"
    src.write_text(PROBE)
    exe = d / "probe"
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", CSRC, str(src), os.path.join(CSRC, "ssu_table.cpp"), "-o",
                    str(exe), "-lpthread"], check=True)
    return exe, d


def _run(probe, indptr, indices, data, n_samples, threads):
    exe, d = probe
    inp, out = d / "in.bin", d / f"out{threads}.bin"
    with open(inp, "wb") as f:
        np.array([len(indptr) - 1, n_samples], np.uint32).tofile(f)
        np.array([len(indices)], np.uint64).tofile(f)
        np.asarray(indptr, np.uint32).tofile(f)
        np.asarray(indices, np.uint32).tofile(f)
        np.asarray(data, np.float64).tofile(f)
    env = dict(os.environ, OMP_NUM_THREADS=str(threads))
    subprocess.run([str(exe), str(inp), str(out)], check=True, env=env)
    raw = np.fromfile(out, np.uint8)
    totals = raw[: 8 * n_samples].view(np.float64)
    return totals, bool(raw[-2]), bool(raw[-1])


def _table(rng, n_obs, n_samples, per_obs, values):
    counts = rng.integers(per_obs // 2, per_obs * 3 // 2, size=n_obs)
    indptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    indices = np.concatenate([np.sort(rng.choice(n_samples, c, replace=False)) for c in counts]).astype(np.uint32)
    return indptr, indices, values(int(indptr[-1]))


def _observation_order(indptr, indices, data, n_samples):
    t = np.zeros(n_samples)
    for i in range(len(indptr) - 1):  # the reference's order, one observation after another
        np.add.at(t, indices[indptr[i]:indptr[i + 1]], data[indptr[i]:indptr[i + 1]])
    return t


@pytest.mark.parametrize("kind", ["counts", "fractions", "negative_counts"])
def test_threaded_totals_equal_observation_order_bit_for_bit(probe, kind):
    rng = np.random.default_rng({"counts": 1, "fractions": 2, "negative_counts": 3}[kind])
    n_obs, n_samples = 6000, 3000
    if kind == "counts":
        values = lambda m: rng.integers(1, 1000, m).astype(np.float64)
    elif kind == "fractions":
        values = lambda m: rng.lognormal(0.0, 2.0, m)
    else:
        values = lambda m: rng.integers(-50, 1000, m).astype(np.float64)
    indptr, indices, data = _table(rng, n_obs, n_samples, 400, values)
    assert indptr[-1] >= (1 << 21)  # large enough for the threaded pass
    ref = _observation_order(indptr, indices, data, n_samples)
    for threads in (1, 3, 8):
        totals, nonneg, malformed = _run(probe, indptr, indices, data, n_samples, threads)
        np.testing.assert_array_equal(totals, ref)
        assert nonneg == (kind != "negative_counts") and not malformed


def test_threaded_totals_flag_a_sample_position_out_of_range(probe):
    rng = np.random.default_rng(4)
    indptr, indices, data = _table(rng, 6000, 3000, 400, lambda m: np.ones(m))
    indices = indices.copy()
    indices[len(indices) // 2] = 3000  # one position past the samples
    totals, _, malformed = _run(probe, indptr, indices, data, 3000, 8)
    assert malformed
