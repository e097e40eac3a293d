"""Partial result files and their merge (src/api.hpp:816-991), on the CPU.

Mirrors the reference's own checks in src/test_api.cpp:145-626 (the six-
sample partials of fill_test_pm: write / read / read a header then stripes
on demand, merge in and out of order into fp64 and fp32 matrices, the error
statuses of the merge), and pins the file format: files this library writes
are read back with the system's LZ4 library (liblz4.so.1, the codec the
reference links), and files written with that library's compressor are read
by this library's own LZ4 decoder."""
import ctypes as C
import os
import struct

import numpy as np
import pytest

import ssu_b200

MAGIC = 0x088ABA02
IDS = ["A", "B", "Cx", "D", "E", "F"]
# src/test_api.cpp:37-65, cases 0, 1, 2
CASES = {
    0: (0, 3, [[1, 2, 3, 4, 5, 6], [7, 8, 9, 10, 11, 12], [13, 14, 15, 16, 17, 18]]),
    1: (0, 2, [[1, 2, 3, 4, 5, 6], [7, 8, 9, 10, 11, 12]]),
    2: (2, 3, [[16, 17, 18, 16, 17, 18]]),
}
# src/test_api.cpp:113-142
THREE_REP = np.array([[0, 1, 7, 16, 11, 6], [1, 0, 2, 8, 17, 12], [7, 2, 0, 3, 9, 18], [16, 8, 3, 0, 4, 10],
                      [11, 17, 9, 4, 0, 5], [6, 12, 18, 10, 5, 0]], dtype=np.float64)


class PartialDyn(C.Structure):
    _fields_ = [("n_samples", C.c_uint32), ("sample_ids", C.POINTER(C.c_char_p)),
                ("offsets", C.POINTER(C.c_uint64)), ("stripes", C.POINTER(C.POINTER(C.c_double))),
                ("stripe_start", C.c_uint32), ("stripe_stop", C.c_uint32), ("stripe_total", C.c_uint32),
                ("is_upper_triangle", C.c_bool), ("filename", C.c_char_p)]


@pytest.fixture(scope="module")
def L():
    lib = ssu_b200.lib()
    P, PP = C.POINTER, C.POINTER
    lib.write_partial.argtypes = [C.c_char_p, P(ssu_b200.PartialMat)]
    lib.read_partial.argtypes = [C.c_char_p, PP(P(ssu_b200.PartialMat))]
    lib.read_partial_header.argtypes = [C.c_char_p, PP(P(PartialDyn))]
    lib.read_partial_one_stripe.argtypes = [P(PartialDyn), C.c_uint32]
    lib.validate_partial.argtypes = [P(P(PartialDyn)), C.c_int]
    lib.destroy_partial_dyn_mat.argtypes = [PP(P(PartialDyn))]
    lib.destroy_partial_dyn_mat.restype = None
    for name, res in [("merge_partial_to_matrix", ssu_b200.MatFull64),
                      ("merge_partial_to_matrix_fp32", ssu_b200.MatFull32)]:
        getattr(lib, name).argtypes = [P(P(PartialDyn)), C.c_int, PP(P(res))]
    for name, res in [("merge_partial_to_mmap_matrix", ssu_b200.MatFull64),
                      ("merge_partial_to_mmap_matrix_fp32", ssu_b200.MatFull32)]:
        getattr(lib, name).argtypes = [P(P(PartialDyn)), C.c_int, C.c_char_p, PP(P(res))]
    return lib


class Holder:
    """Keeps the ctypes buffers of a hand-built partial alive."""


def make_pm(case, ids=IDS):
    start, stop, stripes = CASES[case]
    h = Holder()
    h.ids = (C.c_char_p * len(ids))(*[s.encode() for s in ids])
    h.rows = [(C.c_double * len(ids))(*row) for row in stripes]
    h.ptrs = (C.POINTER(C.c_double) * len(stripes))(*[C.cast(r, C.POINTER(C.c_double)) for r in h.rows])
    h.pm = ssu_b200.PartialMat(len(ids), h.ids, h.ptrs, start, stop, 3, True)
    return h


def make_pdm(case):
    """A partial_dyn_mat_t with its stripes in memory, allocated with the C
    allocator (the merge releases them), as make_test_pdm."""
    libc = C.CDLL(None)
    libc.malloc.restype = C.c_void_p
    libc.malloc.argtypes = [C.c_size_t]
    libc.strdup.restype = C.c_void_p
    libc.strdup.argtypes = [C.c_char_p]
    start, stop, stripes = CASES[case]
    ids = C.cast(libc.malloc(8 * 6), C.POINTER(C.c_char_p))
    id_addrs = C.cast(ids, C.POINTER(C.c_void_p))
    for i, s in enumerate(IDS):
        id_addrs[i] = libc.strdup(s.encode())
    rows = C.cast(libc.malloc(8 * len(stripes)), C.POINTER(C.POINTER(C.c_double)))
    for i, row in enumerate(stripes):
        r = C.cast(libc.malloc(8 * 6), C.POINTER(C.c_double))
        for k, v in enumerate(row):
            r[k] = v
        rows[i] = r
    offs = C.cast(libc.malloc(8 * len(stripes)), C.POINTER(C.c_uint64))
    for i in range(len(stripes)):
        offs[i] = 0
    pdm = C.cast(libc.malloc(C.sizeof(PartialDyn)), C.POINTER(PartialDyn))
    pdm.contents.n_samples = 6
    pdm.contents.sample_ids = ids
    pdm.contents.offsets = offs
    pdm.contents.stripes = rows
    pdm.contents.stripe_start, pdm.contents.stripe_stop, pdm.contents.stripe_total = start, stop, 3
    pdm.contents.is_upper_triangle = True
    pdm.contents.filename = C.cast(libc.strdup(b"dummy"), C.c_char_p)
    return pdm


def merged(L, pms, fp32=False, mmap_dir=None):
    arr = (C.POINTER(PartialDyn) * len(pms))(*pms)
    res = C.POINTER(ssu_b200.MatFull32 if fp32 else ssu_b200.MatFull64)()
    if mmap_dir is None:
        st = (L.merge_partial_to_matrix_fp32 if fp32 else L.merge_partial_to_matrix)(arr, len(pms), C.byref(res))
    else:
        fn = L.merge_partial_to_mmap_matrix_fp32 if fp32 else L.merge_partial_to_mmap_matrix
        st = fn(arr, len(pms), mmap_dir.encode(), C.byref(res))
    if st != 0:
        return st, None, None
    n = res.contents.n_samples
    m = np.ctypeslib.as_array(res.contents.matrix, shape=(n, n)).copy()
    ids = [res.contents.sample_ids[i].decode() for i in range(n)]
    (L.destroy_mat_full_fp32 if fp32 else L.destroy_mat_full_fp64)(C.byref(res))
    return 0, m, ids


def test_write_then_read_partial(L, tmp_path):
    """src/test_api.cpp:145-245"""
    f = str(tmp_path / "ssu_io.dat")
    h = make_pm(0)
    assert L.write_partial(f.encode(), C.byref(h.pm)) == 1  # write_okay
    obs = C.POINTER(ssu_b200.PartialMat)()
    assert L.read_partial(f.encode(), C.byref(obs)) == 0
    o = obs.contents
    assert (o.n_samples, o.stripe_start, o.stripe_stop, o.stripe_total, o.is_upper_triangle) == (6, 0, 3, 3, True)
    assert [o.sample_ids[i].decode() for i in range(6)] == IDS
    for s, row in enumerate(CASES[0][2]):
        assert [o.stripes[s][k] for k in range(6)] == row
    L.destroy_partial_mat(C.byref(obs))
    dyn = C.POINTER(PartialDyn)()
    assert L.read_partial_header(f.encode(), C.byref(dyn)) == 0
    d = dyn.contents
    assert (d.n_samples, d.stripe_start, d.stripe_stop, d.stripe_total) == (6, 0, 3, 3)
    assert not d.stripes[0] and not d.stripes[1] and not d.stripes[2]
    for s in (1, 0, 2):  # out of order, as the reference test
        assert L.read_partial_one_stripe(dyn, s) == 0
        assert [d.stripes[s][k] for k in range(6)] == CASES[0][2][s]
    assert L.read_partial_one_stripe(dyn, 3) == 5  # bad_header: past the last stripe
    L.destroy_partial_dyn_mat(C.byref(dyn))


@pytest.mark.parametrize("fp32", [False, True])
def test_merge_in_memory_partials_in_and_out_of_order(L, fp32):
    """src/test_api.cpp:343-399: the merged matrix, and the partials' stripes
    released by the merge."""
    for order in ((1, 2), (2, 1)):
        pms = [make_pdm(c) for c in order]
        st, m, ids = merged(L, pms, fp32=fp32)
        assert st == 0 and ids == IDS
        np.testing.assert_array_equal(m, THREE_REP)
        for p in pms:
            for s in range(p.contents.stripe_stop - p.contents.stripe_start):
                assert not p.contents.stripes[s]
        for p in pms:
            L.destroy_partial_dyn_mat(C.byref(p))


def test_merge_error_statuses(L):
    """src/test_api.cpp:401-458"""
    pm1, pm2, pm3 = make_pdm(1), make_pdm(2), make_pdm(0)
    pm1.contents.stripe_start, pm1.contents.stripe_stop, pm1.contents.stripe_total = 0, 3, 9
    pm2.contents.stripe_start, pm2.contents.stripe_stop, pm2.contents.stripe_total = 3, 5, 9
    pm3.contents.stripe_start, pm3.contents.stripe_stop, pm3.contents.stripe_total = 6, 9, 9
    pms = [pm2, pm3, pm1]
    arr = (C.POINTER(PartialDyn) * 3)(*pms)
    assert merged(L, pms)[0] == 1                                   # incomplete_stripe_set
    assert L.validate_partial(arr, 3) == 1
    pm2.contents.stripe_start, pm2.contents.stripe_stop = 2, 6
    assert merged(L, pms)[0] == 5                                   # stripes_overlap
    pm2.contents.stripe_start = 3
    id2 = C.cast(pm2.contents.sample_ids, C.POINTER(C.c_void_p))[2]  # the C string itself
    C.memmove(id2, b"X", 1)
    assert merged(L, pms)[0] == 2                                   # sample_id_consistency
    C.memmove(id2, b"C", 1)
    pm3.contents.n_samples = 2
    assert merged(L, pms)[0] == 4                                   # partials_mismatch
    pm3.contents.n_samples = 6
    pm3.contents.stripe_total = 12
    assert merged(L, pms)[0] == 4                                   # partials_mismatch
    pm3.contents.stripe_total = 9
    pm3.contents.is_upper_triangle = False
    assert L.validate_partial(arr, 3) == 3                          # square_mismatch
    assert L.validate_partial(arr, 0) == 1                          # no partials


@pytest.mark.parametrize("fp32", [False, True])
def test_merge_partials_read_from_files(L, tmp_path, fp32):
    """src/test_api.cpp:465-626: partials written, their headers read, the
    stripes read on demand by the merge (mmap-backed result too)."""
    dyns = []
    for i, case in enumerate((2, 1)):
        f = str(tmp_path / f"p{i}.partial")
        h = make_pm(case)
        assert L.write_partial(f.encode(), C.byref(h.pm)) == 1
        d = C.POINTER(PartialDyn)()
        assert L.read_partial_header(f.encode(), C.byref(d)) == 0
        dyns.append(d)
    for mmap_dir in (None, str(tmp_path)):
        st, m, ids = merged(L, dyns, fp32=fp32, mmap_dir=mmap_dir)
        assert st == 0 and ids == IDS
        np.testing.assert_array_equal(m, THREE_REP)
    for d in dyns:
        L.destroy_partial_dyn_mat(C.byref(d))


def test_read_statuses_on_malformed_files(L, tmp_path):
    obs = C.POINTER(ssu_b200.PartialMat)()
    assert L.read_partial(str(tmp_path / "none").encode(), C.byref(obs)) == 2         # open_error
    bad = tmp_path / "bad"
    bad.write_bytes(struct.pack("<8I", 0x12345678, 6, 3, 0, 3, 1, 14, 14))
    assert L.read_partial(str(bad).encode(), C.byref(obs)) == 4                       # magic_incompatible
    bad.write_bytes(struct.pack("<8I", MAGIC, 6, 3, 0, 6, 1, 14, 14))                 # stripe_total >= n
    assert L.read_partial(str(bad).encode(), C.byref(obs)) == 5                       # bad_header
    good = tmp_path / "good"
    h = make_pm(0)
    assert L.write_partial(str(good).encode(), C.byref(h.pm)) == 1
    data = good.read_bytes()
    for cut in (40, len(data) - 30, len(data) - 2):
        (tmp_path / "cut").write_bytes(data[:cut])
        assert L.read_partial(str(tmp_path / "cut").encode(), C.byref(obs)) == 4      # magic_incompatible
    assert not obs


def system_lz4():
    for name in ("liblz4.so.1", "liblz4.so"):
        try:
            lib = C.CDLL(name)
        except OSError:
            continue
        lib.LZ4_decompress_safe.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int]
        lib.LZ4_compress_default.argtypes = [C.c_char_p, C.c_char_p, C.c_int, C.c_int]
        lib.LZ4_compressBound.argtypes = [C.c_int]
        return lib
    pytest.skip("no system LZ4 library to cross-check the format with")


def parse_with(lz4, data):
    w = struct.unpack_from("<8I", data, 0)
    assert w[0] == MAGIC
    n, ns, start, total, upper, id_len, id_cmp = w[1:]
    out = C.create_string_buffer(id_len)
    assert lz4.LZ4_decompress_safe(data[32:32 + id_cmp], out, id_cmp, id_len) == id_len
    ids = out.raw.split(b"\0")[:n]
    pos = 32 + id_cmp
    stripes = []
    for _ in range(ns):
        (c,) = struct.unpack_from("<I", data, pos)
        buf = C.create_string_buffer(8 * n)
        assert lz4.LZ4_decompress_safe(data[pos + 4:pos + 4 + c], buf, c, 8 * n) == 8 * n
        stripes.append(np.frombuffer(buf.raw, dtype=np.float64).copy())
        pos += 4 + c
    assert struct.unpack_from("<I", data, pos)[0] == MAGIC and pos + 4 == len(data)
    return [i.decode() for i in ids], start, total, np.array(stripes)


def test_files_written_here_decode_with_the_system_lz4(L, tmp_path):
    lz4 = system_lz4()
    rng = np.random.default_rng(5)
    n = 1000
    ids = [f"sample.{i}.{'x' * (i % 7)}" for i in range(n)]
    for kind in ("random", "repetitive", "zeros"):
        if kind == "random":
            stripes = rng.random((7, n))
        elif kind == "repetitive":
            stripes = np.tile(np.round(rng.random(10), 3), (7, n // 10))
        else:
            stripes = np.zeros((7, n))
        h = Holder()
        h.ids = (C.c_char_p * n)(*[s.encode() for s in ids])
        h.rows = [np.ascontiguousarray(r) for r in stripes]
        h.ptrs = (C.POINTER(C.c_double) * 7)(*[r.ctypes.data_as(C.POINTER(C.c_double)) for r in h.rows])
        h.pm = ssu_b200.PartialMat(n, h.ids, h.ptrs, 10, 17, 500, True)
        f = tmp_path / f"{kind}.partial"
        assert L.write_partial(str(f).encode(), C.byref(h.pm)) == 1
        got_ids, start, total, got = parse_with(lz4, f.read_bytes())
        assert got_ids == ids and (start, total) == (10, 500)
        np.testing.assert_array_equal(got, stripes)
        if kind != "random":
            assert os.path.getsize(f) < 8 * n * 7 / 4  # the blocks really are compressed


def test_files_compressed_by_the_system_lz4_are_read_here(L, tmp_path):
    lz4 = system_lz4()
    rng = np.random.default_rng(6)
    n = 513
    ids = [f"s{i}" for i in range(n)]
    stripes = np.vstack([rng.random(n), np.tile([0.25, 0.5, 0.5], n // 3 + 1)[:n], np.zeros(n)])

    def block(raw):
        cap = lz4.LZ4_compressBound(len(raw))
        out = C.create_string_buffer(cap)
        c = lz4.LZ4_compress_default(raw, out, len(raw), cap)
        assert c > 0
        return out.raw[:c]

    id_raw = b"".join(s.encode() + b"\0" for s in ids)
    idc = block(id_raw)
    data = struct.pack("<8I", MAGIC, n, 3, 4, 257, 1, len(id_raw), len(idc)) + idc
    for r in stripes:
        b = block(r.astype(np.float64).tobytes())
        data += struct.pack("<I", len(b)) + b
    data += struct.pack("<I", MAGIC)
    f = tmp_path / "sys.partial"
    f.write_bytes(data)
    obs = C.POINTER(ssu_b200.PartialMat)()
    assert L.read_partial(str(f).encode(), C.byref(obs)) == 0
    o = obs.contents
    assert (o.n_samples, o.stripe_start, o.stripe_stop, o.stripe_total) == (n, 4, 7, 257)
    assert [o.sample_ids[i].decode() for i in range(n)] == ids
    for s in range(3):
        np.testing.assert_array_equal(np.ctypeslib.as_array(o.stripes[s], shape=(n,)), stripes[s])
    L.destroy_partial_mat(C.byref(obs))
