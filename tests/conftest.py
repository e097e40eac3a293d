import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "unifrac-binaries_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)

import ssu_synth  # noqa: E402

GOLDEN = os.path.join(ROOT, "tests", "golden", "reference_golden.json")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libssu_b200.so")


@pytest.fixture(scope="session")
def golden():
    with open(GOLDEN) as f:
        return json.load(f)


@pytest.fixture(scope="session")
def test_table(golden):
    """The reference's 6-sample x 5-feature test table (test/capi_inmem_test.c:21-27)."""
    c = golden["table_csr"]
    return ssu_synth.Table(list(c["obs_ids"]), list(c["sample_ids"]), np.array(c["indptr"], np.uint32),
                           np.array(c["indices"], np.uint32), np.array(c["data"], np.float64))


@pytest.fixture(scope="session")
def test_tree(golden):
    return ssu_synth.parse_newick(golden["trees"]["test.tre"])


def stripes_from_golden(entry, prefix=""):
    arrays = entry["arrays"]
    out = []
    i = 1
    while f"{prefix}stride{i}" in arrays:
        out.append(arrays[f"{prefix}stride{i}"][0])
        i += 1
    return np.array(out)


def matrix_from_stripes(stripes, n):
    m = np.zeros((n, n))
    for s in range(stripes.shape[0]):
        for k in range(n):
            l = (k + s + 1) % n
            m[k, l] = m[l, k] = stripes[s, k]
    return m


def rel_err(a, b):
    """max |a-b| / |b| over entries where b != 0, and max |a-b| where b == 0."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    assert not (np.isnan(a) ^ np.isnan(b)).any(), "NaN pattern differs"
    d = np.abs(a - b)
    d[both_nan] = 0
    nz = (b != 0) & ~both_nan
    r = d[nz] / np.abs(b[nz]) if nz.any() else np.zeros(1)
    z = d[~nz] if (~nz).any() else np.zeros(1)
    return float(r.max()), float(z.max())


@pytest.fixture(scope="session")
def oracle_mod():
    import oracle_py
    if not os.path.exists(oracle_py.ORACLE_SO):
        pytest.fail("oracle/liboracle.so is not built; run `make -C oracle oracle` (or __graft_entry__.build())")
    return oracle_py


def have_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def ssu():
    import ssu_b200
    return ssu_b200
