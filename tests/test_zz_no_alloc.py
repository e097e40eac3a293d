"""ssu_b200_weighted_pairs_noalloc: the weighted pair stage for callers that
cannot allocate device memory (code inside a framework that owns every
device buffer through its own arena, or under a fixed memory budget).

The test builds the proportion embedding on the host, hands the entry point
device buffers it allocated itself (through torch, as such a caller's arena
would), and checks the result against the full-matrix entry point
one_off_matrix_inmem_v3 at the fp64 parity tolerance, over consecutive calls
that reuse the library's shared scratch array.  Collected last so that a run
stopping at the first failure has run every other test first."""
import ctypes

import numpy as np
import pytest

import ssu_synth
from conftest import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12


def host_embedding(ssu, tree, table):
    """Proportions of every non-root node of the sheared, collapsed tree,
    rows in postorder, and their branch lengths."""
    s, lengths, names = ssu.shear_collapse(tree, table.obs_ids, collapse=True)
    n = len(s)
    match = [0] * n
    stack = []
    for i in range(n):
        if s[i]:
            stack.append(i)
        else:
            o = stack.pop()
            match[o], match[i] = i, o
    dense = table.dense()
    totals = dense.sum(axis=0)
    row_of_obs = {name: i for i, name in enumerate(table.obs_ids)}
    post = [match[i] for i in range(n) if not s[i]][:-1]  # the root closes last
    vec = {}
    rows, lens = [], []
    for o in post:
        if not s[o + 1]:  # a tip
            v = dense[row_of_obs[names[o]]] / totals
        else:
            v = np.zeros(table.n_samples)
            c = o + 1
            while c < n and s[c]:
                v = v + vec[c]
                c = match[c] + 1
        vec[o] = v
        rows.append(v)
        lens.append(lengths[o])
    return np.array(rows), np.array(lens)


def call_noalloc(ssu, torch, U, lens, n, normalized):
    L = ssu.lib()
    f = L.ssu_b200_weighted_pairs_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    ld = ((n + 127) // 128) * 128
    padded = np.zeros((U.shape[0], ld))
    padded[:, :n] = U
    d_u = torch.from_numpy(padded).cuda()
    d_len = torch.from_numpy(np.ascontiguousarray(lens)).cuda()
    d_out = torch.full((n, n), float("nan"), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    st = f(d_u.data_ptr(), d_len.data_ptr(), U.shape[0], n, ld, 1 if normalized else 0, d_out.data_ptr(), None)
    torch.cuda.synchronize()
    return st, d_out.cpu().numpy()


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("needs a CUDA device")
    return torch


def test_noalloc_matches_full_matrix_entry_point_on_consecutive_calls(ssu, torch_cuda):
    cases = []
    # 129 samples: the last diagonal block holds one sample and has no tile
    for seed, n_samples, n_tips in [(71, 150, 400), (72, 300, 250), (73, 129, 300)]:
        tree = ssu_synth.random_binary_tree(n_tips, 0.1, seed)
        table = ssu_synth.geometric_table(tree.tip_names()[: n_tips - 20], n_samples, 0.08, 12.0, seed + 1)
        cases.append((tree, table))
    calls = [(0, True), (0, True), (1, False), (2, True), (0, True), (1, True), (2, False)]
    for idx, normalized in calls:
        tree, table = cases[idx]
        U, lens = host_embedding(ssu, tree, table)
        method = "weighted_normalized_fp64" if normalized else "weighted_unnormalized_fp64"
        expected, _ = ssu.one_off_matrix(tree, table, method)
        st, got = call_noalloc(ssu, torch_cuda, U, lens, table.n_samples, normalized)
        assert st == 0
        r, z = rel_err(got, expected)
        assert r <= TOL and z <= TOL * 0.1, (idx, normalized, r, z)


def test_noalloc_rejects_sizes_beyond_its_limit(ssu, torch_cuda):
    L = ssu.lib()
    f = L.ssu_b200_weighted_pairs_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_int,
                  ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    dummy = torch_cuda.zeros(16, dtype=torch_cuda.float64, device="cuda")
    p = dummy.data_ptr()
    assert f(p, p, 1, 100001, 100096, 1, p, None) == 6   # beyond the sample limit
    assert f(p, p, 1, 200, 100, 1, p, None) == 6         # ld smaller than n_samples
    assert f(p, p, 1, 0, 128, 1, p, None) == 3           # no samples
    assert f(p + 8, p, 1, 100, 128, 1, p, None) == 6     # embedding not 16-byte aligned
    assert f(p, p + 4, 1, 100, 128, 1, p, None) == 6     # lengths not 8-byte aligned
    assert f(p, p, 1, 100, 128, 1, p + 4, None) == 6     # output not 8-byte aligned


def test_noalloc_call_captured_in_a_graph_replays_correctly(ssu, torch_cuda):
    """After a first call on the device, a call made while its stream is
    being captured becomes part of the graph: it reads no host memory at
    replay time (the tile list and table descriptor are written on the
    device), so replaying the graph recomputes the same matrix."""
    torch = torch_cuda
    tree = ssu_synth.random_binary_tree(300, 0.1, 81)
    table = ssu_synth.geometric_table(tree.tip_names()[:280], 140, 0.08, 12.0, 82)
    U, lens = host_embedding(ssu, tree, table)
    n = table.n_samples
    st, first = call_noalloc(ssu, torch, U, lens, n, True)  # the first call sets the device up
    assert st == 0
    L = ssu.lib()
    f = L.ssu_b200_weighted_pairs_noalloc
    ld = ((n + 127) // 128) * 128
    padded = np.zeros((U.shape[0], ld))
    padded[:, :n] = U
    d_u = torch.from_numpy(padded).cuda()
    d_len = torch.from_numpy(np.ascontiguousarray(lens)).cuda()
    d_out = torch.zeros((n, n), dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    status = []
    with torch.cuda.graph(graph, stream=stream):
        status.append(f(d_u.data_ptr(), d_len.data_ptr(), U.shape[0], n, ld, 1, d_out.data_ptr(),
                        ctypes.c_void_p(stream.cuda_stream)))
    assert status == [0]
    d_out.fill_(float("nan"))
    graph.replay()
    torch.cuda.synchronize()
    got = d_out.cpu().numpy()
    r, z = rel_err(got, first)
    assert r == 0.0 and z == 0.0, (r, z)
    del graph
