"""BIOM-HDF5 table files (src/biom.cpp:18-255) and the file-based entry
points' checks that run before any device work.

The fixtures are the reference's own data files, copied byte for byte by
tests/golden/make_golden.py into tests/golden/fixtures/: the crawford table
and tree with the outputs ci/crawford_test.sh compares against
(unweighted_fp64, its variance-adjusted form, Faith PD), the absquant table
with its weighted-normalized matrices with and without sample-count
normalisation, and the 6 x 5 table of the reference's unit tests.

Here the reader's tables go through the oracle (CPU): reader and oracle
together reproduce the reference's expected outputs."""
import ctypes
import os

import numpy as np
import pytest

import ssu_synth
from conftest import ROOT, rel_err

FIX = os.path.join(ROOT, "tests", "golden", "fixtures")


def fixture(name):
    return os.path.join(FIX, name)


def read_dm(path):
    """A tab/space separated square matrix with a header row of ids."""
    lines = [ln for ln in open(path).read().splitlines() if ln.strip()]
    ids = lines[0].split()
    rows = [ln.split() for ln in lines[1:]]
    assert [r[0] for r in rows] == ids
    return ids, np.array([[float(x) for x in r[1:]] for r in rows])


def read_faith(path):
    rows = [ln.split() for ln in open(path).read().splitlines() if ln.strip()]
    return [r[0] for r in rows], np.array([float(r[1]) for r in rows])


def crawford():
    tree = ssu_synth.parse_newick(open(fixture("crawford.tre")).read())
    return tree, fixture("crawford.biom"), fixture("crawford.tre")


def test_reader_returns_the_reference_unit_test_table(ssu, test_table):
    t = ssu.read_biom(fixture("test.biom"))
    assert t.obs_ids == test_table.obs_ids and t.sample_ids == test_table.sample_ids
    np.testing.assert_array_equal(t.indptr, test_table.indptr)
    np.testing.assert_array_equal(t.indices, test_table.indices)
    np.testing.assert_array_equal(t.data, test_table.data)


def test_reader_on_the_crawford_and_absquant_tables(ssu):
    t = ssu.read_biom(fixture("crawford.biom"))
    assert (t.n_obs, t.n_samples, t.nnz) == (365, 9, 557)
    ids, _ = read_dm(fixture("test.ssu.exp"))
    assert t.sample_ids == ids
    assert t.indptr[0] == 0 and t.indptr[-1] == t.nnz and np.all(np.diff(t.indptr.astype(np.int64)) >= 0)
    assert np.all(t.data > 0) and np.all(t.data == np.round(t.data))
    a = ssu.read_biom(fixture("absquant.biom"))
    assert a.sample_ids == ["SampleA", "SampleB", "SampleC"] and a.n_obs == 7
    np.testing.assert_array_equal(a.dense().sum(axis=0), [10, 18, 14])


@pytest.mark.parametrize("vaw,expected", [(False, "test.ssu.exp"), (True, "test.ssu_vaw.exp")])
def test_reader_and_oracle_reproduce_the_crawford_expected_matrices(ssu, oracle_mod, vaw, expected):
    tree, biom, _ = crawford()
    table = ssu.read_biom(biom)
    got = oracle_mod.oracle_one_off(tree, table, "unweighted_fp64", variance_adjust=vaw)["matrix"]
    ids, want = read_dm(fixture(expected))
    assert table.sample_ids == ids
    r, z = rel_err(got, want)
    assert r <= 1e-12 and z <= 1e-15, (r, z)


def test_reader_and_oracle_reproduce_the_crawford_faith_pd(ssu, oracle_mod):
    tree, biom, _ = crawford()
    table = ssu.read_biom(biom)
    got = oracle_mod.oracle_faith_pd(tree, table)
    ids, want = read_faith(fixture("test.faith.exp"))
    assert table.sample_ids == ids
    np.testing.assert_allclose(np.asarray(got["values"]), want, rtol=1e-12)


# src/testdata/validation_tests.sh:135-146: --normalize-sample-counts false is
# compared with test.absquant.wn.dm (absolute quantities), true with
# test.absquant_not.wn.dm
@pytest.mark.parametrize("normalize,expected", [(False, "test.absquant.wn.dm"), (True, "test.absquant_not.wn.dm")])
def test_reader_and_oracle_reproduce_the_absquant_matrices(ssu, oracle_mod, normalize, expected):
    tree = ssu_synth.parse_newick(open(fixture("absquant.tree")).read())
    table = ssu.read_biom(fixture("absquant.biom"))
    got = oracle_mod.oracle_one_off(tree, table, "weighted_normalized_fp64", normalize=normalize)["matrix"]
    ids, want = read_dm(fixture(expected))
    assert table.sample_ids == ids
    # the expected files carry six decimals
    np.testing.assert_allclose(got, want, atol=1.01e-6)


def test_file_entry_point_statuses_before_device_work(ssu, tmp_path):
    """CHECK_FILE order (table first), unreadable table files, trees that do
    not hold the table's ids, and partial_v3's early method check
    (src/api.cpp:527-536, 605-616, 718-729)."""
    missing = str(tmp_path / "nope.biom")
    tre = fixture("crawford.tre")
    biom = fixture("crawford.biom")
    truncated = tmp_path / "t.biom"
    truncated.write_bytes(open(biom, "rb").read()[:4096])
    notbiom = tmp_path / "n.biom"
    notbiom.write_text("not an hdf5 file\n")
    other = tmp_path / "other.tre"
    other.write_text("(a:1,b:2)r;")
    for entry in ("one_off_matrix_v3", "one_off_matrix_fp32_v2", "one_off_matrix"):
        for b, t, want in [(missing, tre, 2), (biom, missing, 1), (missing, missing, 2), (str(truncated), tre, 2),
                           (str(notbiom), tre, 2), (biom, str(other), 5)]:
            with pytest.raises(ssu.SSUError) as e:
                ssu.file_matrix(entry, b, t, "unweighted_fp64")
            assert e.value.status == want, (entry, b, t)
    with pytest.raises(ssu.SSUError) as e:
        ssu.file_partial(biom, tre, "bogus", 0, 2)
    assert e.value.status == 4
    with pytest.raises(ssu.SSUError) as e:
        ssu.file_faith_pd(str(notbiom), tre)
    assert e.value.status == 2
    opaque = ssu.OpaqueTree(path=str(other))
    with pytest.raises(ssu.SSUError) as e:
        ssu.file_matrix("one_off_matrix_v3t", biom, opaque, "unweighted_fp64")
    assert e.value.status == 5
    L = ssu.lib()
    res = ctypes.POINTER(ssu.SupportBiom)()
    assert L.ssu_b200_read_biom(missing.encode(), ctypes.byref(res)) == 2       # open_error
    assert L.ssu_b200_read_biom(str(notbiom).encode(), ctypes.byref(res)) == 3  # read_error
    assert not res
