"""ctypes binding of libssu_b200.so (include/unifrac_b200.h).

Mirrors the reference's C API for Python callers and tests: tables and trees
are passed as `support_biom_t` / `support_bptree_t` built from the
`ssu_synth.Table` / `ssu_synth.BPTree` containers (or any object with the
same attributes), results come back as numpy arrays after the library's
destroy_*() has been called.  The library must be built (`make` in this
directory, or `__graft_entry__.build()`); loading fails loudly otherwise.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import weakref

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libssu_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "unifrac_b200.h")

STATUS = ["okay", "tree_missing", "table_missing", "table_empty", "unknown_method",
          "table_and_tree_do_not_overlap", "output_error", "invalid_method", "grouping_missing"]
IO_STATUS = ["read_okay", "write_okay", "open_error", "read_error", "magic_incompatible", "bad_header",
             "unexpected_end", "write_error"]
MERGE_STATUS = ["merge_okay", "incomplete_stripe_set", "sample_id_consistency", "square_mismatch",
                "partials_mismatch", "stripes_overlap"]

_strpp = C.POINTER(C.c_char_p)


class SupportBiom(C.Structure):
    _fields_ = [("obs_ids", _strpp), ("sample_ids", _strpp), ("indices", C.POINTER(C.c_uint32)),
                ("indptr", C.POINTER(C.c_uint32)), ("data", C.POINTER(C.c_double)), ("n_obs", C.c_int),
                ("n_samples", C.c_int), ("nnz", C.c_int)]


class SupportBPTree(C.Structure):
    _fields_ = [("structure", C.POINTER(C.c_bool)), ("lengths", C.POINTER(C.c_double)), ("names", _strpp),
                ("n_parens", C.c_int)]


class MatFull64(C.Structure):
    _fields_ = [("n_samples", C.c_uint32), ("flags", C.c_uint32), ("matrix", C.POINTER(C.c_double)),
                ("sample_ids", _strpp)]


class MatFull32(C.Structure):
    _fields_ = [("n_samples", C.c_uint32), ("flags", C.c_uint32), ("matrix", C.POINTER(C.c_float)),
                ("sample_ids", _strpp)]


class Mat(C.Structure):
    _fields_ = [("n_samples", C.c_uint), ("cf_size", C.c_uint), ("is_upper_triangle", C.c_bool),
                ("condensed_form", C.POINTER(C.c_double)), ("sample_ids", _strpp)]


class RVec(C.Structure):
    _fields_ = [("n_samples", C.c_uint), ("values", C.POINTER(C.c_double)), ("sample_ids", _strpp)]


class PartialDynMat(C.Structure):
    _fields_ = [("n_samples", C.c_uint32), ("sample_ids", _strpp), ("offsets", C.POINTER(C.c_uint64)),
                ("stripes", C.POINTER(C.POINTER(C.c_double))), ("stripe_start", C.c_uint32),
                ("stripe_stop", C.c_uint32), ("stripe_total", C.c_uint32), ("is_upper_triangle", C.c_bool),
                ("filename", C.c_char_p)]


class PartialMat(C.Structure):
    _fields_ = [("n_samples", C.c_uint32), ("sample_ids", _strpp), ("stripes", C.POINTER(C.POINTER(C.c_double))),
                ("stripe_start", C.c_uint32), ("stripe_stop", C.c_uint32), ("stripe_total", C.c_uint32),
                ("is_upper_triangle", C.c_bool)]


class SSUError(RuntimeError):
    def __init__(self, status, where=""):
        self.status = status
        name = STATUS[status] if 0 <= status < len(STATUS) else str(status)
        super().__init__(f"{where}: {name}" if where else name)


def declared_functions(header=HEADER):
    """Names of every function the public header declares."""
    text = open(header).read()
    return sorted(set(re.findall(r"SSU_EXTERN[^;(]*?\b(\w+)\s*\(", text, flags=re.S)))


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is not built; run `make` in {HERE}")
        L = C.CDLL(LIB_PATH)
        P, PP = C.POINTER, C.POINTER
        common = [P(SupportBiom), P(SupportBPTree), C.c_char_p, C.c_bool, C.c_double, C.c_bool, C.c_bool, C.c_uint]
        L.one_off_matrix_inmem_v3.argtypes = common + [C.c_uint, C.c_bool, C.c_char_p, PP(P(MatFull64))]
        L.one_off_matrix_inmem_fp32_v3.argtypes = common + [C.c_uint, C.c_bool, C.c_char_p, PP(P(MatFull32))]
        L.ssu_b200_one_off_inmem_v3.argtypes = common + [PP(P(Mat))]
        L.ssu_b200_partial_inmem_v3.argtypes = common + [C.c_uint, C.c_uint, PP(P(PartialMat))]
        L.ssu_b200_faith_pd_inmem.argtypes = [P(SupportBiom), P(SupportBPTree), PP(P(RVec))]
        L.one_dense_pair_v3.argtypes = [C.c_uint, _strpp, P(C.c_double), P(C.c_double), P(SupportBPTree), C.c_char_p,
                                        C.c_bool, C.c_double, C.c_bool, C.c_bool, P(C.c_double)]
        L.one_dense_pair_v3t.argtypes = [C.c_uint, _strpp, P(C.c_double), P(C.c_double), C.c_void_p, C.c_char_p,
                                         C.c_bool, C.c_double, C.c_bool, C.c_bool, P(C.c_double)]
        L.load_bptree_opaque.argtypes = [C.c_char_p, P(C.c_void_p)]
        L.load_bptree_opaque.restype = None
        L.read_bptree_opaque.argtypes = [C.c_char_p, P(C.c_void_p)]
        L.convert_bptree_opaque.argtypes = [P(SupportBPTree), P(C.c_void_p)]
        L.convert_bptree_opaque.restype = None
        L.destroy_bptree_opaque.argtypes = [P(C.c_void_p)]
        L.destroy_bptree_opaque.restype = None
        L.get_bptree_opaque_els.argtypes = [C.c_void_p]
        L.ssu_b200_tree_arrays.argtypes = [C.c_void_p, C.c_int, P(C.c_bool), P(C.c_double), _strpp, P(C.c_int)]
        L.ssu_b200_shear_collapse.argtypes = [P(SupportBPTree), _strpp, C.c_int, C.c_int, P(C.c_bool),
                                              P(C.c_double), _strpp, P(C.c_int)]
        for name, typ in [("destroy_mat_full_fp64", MatFull64), ("destroy_mat_full_fp32", MatFull32),
                          ("destroy_mat", Mat), ("destroy_results_vec", RVec), ("destroy_partial_mat", PartialMat)]:
            f = getattr(L, name)
            f.argtypes = [PP(P(typ))]
            f.restype = None
        for name in ["one_off_v3", "one_off_matrix_v3", "faith_pd_one_off", "partial_v3"]:
            getattr(L, name).restype = C.c_int
        L.faith_pd_one_off.argtypes = [C.c_char_p, C.c_char_p, PP(P(RVec))]
        L.ssu_set_random_seed.argtypes = [C.c_uint]
        L.ssu_set_random_seed.restype = None
        L.write_partial.argtypes = [C.c_char_p, P(PartialMat)]
        L.read_partial_header.argtypes = [C.c_char_p, PP(P(PartialDynMat))]
        L.destroy_partial_dyn_mat.argtypes = [PP(P(PartialDynMat))]
        L.destroy_partial_dyn_mat.restype = None
        L.validate_partial.argtypes = [P(P(PartialDynMat)), C.c_int]
        L.merge_partial_to_mmap_matrix.argtypes = [P(P(PartialDynMat)), C.c_int, C.c_char_p, PP(P(MatFull64))]
        L.merge_partial_to_mmap_matrix_fp32.argtypes = [P(P(PartialDynMat)), C.c_int, C.c_char_p,
                                                        PP(P(MatFull32))]
        L.ssu_b200_read_biom.argtypes = [C.c_char_p, PP(P(SupportBiom))]
        L.ssu_b200_rarefy_batch.argtypes = [P(SupportBiom), C.c_uint, C.c_uint, C.c_bool, P(P(SupportBiom))]
        L.ssu_b200_destroy_biom.argtypes = [PP(P(SupportBiom))]
        L.ssu_b200_destroy_biom.restype = None
        fcommon = [C.c_char_p, C.c_void_p, C.c_char_p, C.c_bool, C.c_double, C.c_bool]
        for name, res in [("one_off_matrix_v3", MatFull64), ("one_off_matrix_v3t", MatFull64),
                          ("one_off_matrix_fp32_v3", MatFull32), ("one_off_matrix_fp32_v3t", MatFull32)]:
            getattr(L, name).argtypes = fcommon + [C.c_bool, C.c_uint, C.c_uint, C.c_bool, C.c_char_p,
                                                   PP(P(res))]
        for name, res in [("one_off_matrix_v2", MatFull64), ("one_off_matrix_v2t", MatFull64),
                          ("one_off_matrix_fp32_v2", MatFull32), ("one_off_matrix_fp32_v2t", MatFull32)]:
            getattr(L, name).argtypes = fcommon + [C.c_uint, C.c_uint, C.c_bool, C.c_char_p, PP(P(res))]
        L.one_off_matrix.argtypes = fcommon + [C.c_uint, C.c_char_p, PP(P(MatFull64))]
        L.one_off_matrix_fp32.argtypes = fcommon + [C.c_uint, C.c_char_p, PP(P(MatFull32))]
        L.one_off_v3.argtypes = fcommon + [C.c_bool, C.c_uint, PP(P(Mat))]
        L.one_off_wtree_v3.argtypes = fcommon + [C.c_bool, C.c_uint, PP(P(Mat))]
        L.partial_v3.argtypes = fcommon + [C.c_bool, C.c_uint, C.c_uint, C.c_uint, PP(P(PartialMat))]
        L.ssu_b200_plan_create.argtypes = common[:-1] + [P(C.c_void_p)]
        L.ssu_b200_plan_execute.argtypes = [C.c_void_p, C.c_void_p]
        L.ssu_b200_plan_device_result.argtypes = [C.c_void_p]
        L.ssu_b200_plan_device_result.restype = C.c_void_p
        L.ssu_b200_plan_copy_result.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        L.ssu_b200_plan_work_units.argtypes = [C.c_void_p]
        L.ssu_b200_plan_work_units.restype = C.c_uint64
        L.ssu_b200_plan_n_samples.argtypes = [C.c_void_p]
        L.ssu_b200_plan_n_samples.restype = C.c_uint32
        L.ssu_b200_plan_n_embedded.argtypes = [C.c_void_p]
        L.ssu_b200_plan_n_embedded.restype = C.c_uint64
        L.ssu_b200_plan_launches.argtypes = [C.c_void_p]
        L.ssu_b200_plan_launches.restype = C.c_uint32
        L.ssu_b200_plan_tensor_flops.argtypes = [C.c_void_p]
        L.ssu_b200_plan_tensor_flops.restype = C.c_uint64
        L.ssu_b200_plan_set_timing.argtypes = [C.c_void_p, C.c_int]
        L.ssu_b200_plan_set_timing.restype = None
        L.ssu_b200_plan_stage_ms.argtypes = [C.c_void_p, P(C.c_float), P(C.c_float), P(C.c_float)]
        L.ssu_b200_plan_destroy.argtypes = [P(C.c_void_p)]
        L.ssu_b200_plan_destroy.restype = None
        L.ssu_b200_plan_pair_kernel.argtypes = [C.c_void_p]
        L.ssu_b200_plan_pair_kernel.restype = C.c_char_p
        L.ssu_b200_version.restype = C.c_char_p
        batch_common = [P(P(SupportBiom)), C.c_uint, P(SupportBPTree), C.c_char_p, C.c_bool, C.c_double, C.c_bool,
                        C.c_bool]
        L.ssu_b200_one_off_batch_inmem_v3.argtypes = batch_common + [P(P(MatFull64))]
        L.ssu_b200_one_off_batch_inmem_fp32_v3.argtypes = batch_common + [P(P(MatFull32))]
        sub_common = [P(SupportBiom), P(SupportBPTree), C.c_char_p, C.c_bool, C.c_double, C.c_bool, C.c_bool,
                      C.c_uint, C.c_uint, C.c_bool]
        L.ssu_b200_subsample_batch_inmem_v3.argtypes = sub_common + [P(P(MatFull64))]
        L.ssu_b200_subsample_batch_inmem_fp32_v3.argtypes = sub_common + [P(P(MatFull32))]
        L.ssu_b200_batch_plan_create.argtypes = batch_common + [C.c_uint64, C.c_int, P(C.c_void_p)]
        for name, res in [("ssu_b200_plan_n_tables", C.c_uint32), ("ssu_b200_plan_n_groups", C.c_uint32)]:
            getattr(L, name).argtypes = [C.c_void_p]
            getattr(L, name).restype = res
        for name, res in [("ssu_b200_plan_table_samples", C.c_uint32), ("ssu_b200_plan_table_offset", C.c_uint64),
                          ("ssu_b200_plan_table_embedded", C.c_uint64)]:
            getattr(L, name).argtypes = [C.c_void_p, C.c_uint32]
            getattr(L, name).restype = res
        L.ssu_b200_plan_set_graph.argtypes = [C.c_void_p, C.c_int]
        L.ssu_b200_plan_set_graph.restype = None
        L.ssu_b200_plan_tuning.argtypes = [C.c_void_p]
        L.ssu_b200_plan_tuning.restype = C.c_char_p
        for name, real, out in (("pcoa", C.c_double, C.c_double), ("pcoa_fp32", C.c_float, C.c_float),
                                ("pcoa_mixed", C.c_double, C.c_float)):
            getattr(L, name).argtypes = [P(real), C.c_uint32, C.c_uint32, PP(P(out)), PP(P(out)), PP(P(out))]
            getattr(L, name).restype = None
        for name, real in (("find_eigens_fast", C.c_double), ("find_eigens_fast_fp32", C.c_float)):
            getattr(L, name).argtypes = [C.c_uint32, C.c_uint32, P(real), PP(P(real)), PP(P(real))]
            getattr(L, name).restype = None
        L.compute_permanova_fp64.argtypes = [C.c_char_p, C.c_uint, _strpp, P(MatFull64), C.c_uint,
                                             P(C.c_double), P(C.c_double)]
        L.compute_permanova_fp32.argtypes = [C.c_char_p, C.c_uint, _strpp, P(MatFull32), C.c_uint,
                                             P(C.c_float), P(C.c_float)]
        L.ssu_b200_read_grouping.argtypes = [C.c_char_p, C.c_char_p, C.c_uint32, _strpp, P(C.c_uint32),
                                             P(C.c_uint32)]
        L.ssu_b200_permanova_fp64.argtypes = [P(C.c_double), C.c_uint32, P(C.c_uint32), C.c_uint,
                                              P(C.c_double), P(C.c_double)]
        L.ssu_b200_permanova_fp32.argtypes = [P(C.c_float), C.c_uint32, P(C.c_uint32), C.c_uint,
                                              P(C.c_float), P(C.c_float)]
        L.ssu_b200_read_h5_doubles.argtypes = [C.c_char_p, C.c_char_p, PP(P(C.c_double)), P(C.c_uint32),
                                               P(C.c_uint64)]
        L.ssu_b200_read_h5_strings.argtypes = [C.c_char_p, C.c_char_p, P(_strpp), P(C.c_uint64)]
        L.ssu_b200_free_h5_strings.argtypes = [_strpp, C.c_uint64]
        L.ssu_b200_free_h5_strings.restype = None
        _lib = L
    return _lib


# ------------------------------------------------------------ marshalling

class _StrArray:
    """char** over one NUL-separated buffer (built without a per-string
    ctypes conversion); keeps its buffers alive."""

    def __init__(self, strings):
        n = len(strings)
        blob = ("\0".join(strings) + "\0").encode()
        self.buf = C.create_string_buffer(blob, len(blob))
        nul = np.flatnonzero(np.frombuffer(blob, dtype=np.uint8) == 0)
        off = np.zeros(max(n, 1), dtype=np.uint64)
        if n > 1:
            off[1:n] = nul[: n - 1] + 1
        self.ptrs = off + np.uint64(C.addressof(self.buf))
        self.arr = (C.c_char_p * max(n, 1)).from_buffer(self.ptrs)


def _strarr(strings):
    holder = _StrArray(strings)
    arr = holder.arr
    arr._holder = holder  # the array keeps its buffers alive
    return arr


class TableInputs:
    """support_biom_t view of a table; keeps the backing arrays alive."""

    def __init__(self, table):
        self.indptr = np.ascontiguousarray(table.indptr, dtype=np.uint32)
        self.indices = np.ascontiguousarray(table.indices, dtype=np.uint32)
        self.data = np.ascontiguousarray(table.data, dtype=np.float64)
        self.obs = _strarr(table.obs_ids)
        self.samples = _strarr(table.sample_ids)
        self.biom = SupportBiom(self.obs, self.samples, self.indices.ctypes.data_as(C.POINTER(C.c_uint32)),
                                self.indptr.ctypes.data_as(C.POINTER(C.c_uint32)),
                                self.data.ctypes.data_as(C.POINTER(C.c_double)), len(table.obs_ids),
                                len(table.sample_ids), int(self.indptr[-1]) if len(self.indptr) else 0)
        self.arrays = (self.indptr, self.indices, self.data)


class TreeInputs:
    """support_bptree_t view of a tree; keeps the backing arrays alive."""

    def __init__(self, tree):
        self.structure = np.ascontiguousarray(tree.structure, dtype=np.bool_)
        self.lengths = np.ascontiguousarray(tree.lengths, dtype=np.float64)
        self.names = _strarr(tree.names)
        self.tree = SupportBPTree(self.structure.ctypes.data_as(C.POINTER(C.c_bool)),
                                  self.lengths.ctypes.data_as(C.POINTER(C.c_double)), self.names,
                                  len(tree.names))
        self.arrays = (self.structure, self.lengths)


_MARSHALLED = {}


def _marshalled(obj, make, arrays, names):
    """The C view of a table or tree, reused while the object, its arrays and
    its name lists are the same objects (name lists are not expected to be
    edited in place between calls)."""
    key = tuple(id(a) for a in arrays) + tuple((id(n), len(n)) for n in names)
    hit = _MARSHALLED.get(id(obj))
    if hit is not None and hit[0]() is obj and hit[1] == key:
        return hit[2]
    view = make(obj)
    # only views that share the caller's arrays (no dtype or layout copy)
    shared = all(np.ascontiguousarray(a, dtype=b.dtype) is a for a, b in zip(arrays, view.arrays))
    if shared:
        try:
            ref = weakref.ref(obj, lambda _, i=id(obj): _MARSHALLED.pop(i, None))
            _MARSHALLED[id(obj)] = (ref, key, view)
        except TypeError:
            pass
    return view


class Inputs:
    """support_biom_t + support_bptree_t views of a (tree, table) pair; keeps
    the backing numpy arrays alive while the call runs."""

    def __init__(self, tree, table):
        self._table = _marshalled(table, TableInputs, (table.indptr, table.indices, table.data),
                                  (table.obs_ids, table.sample_ids))
        self._tree = _marshalled(tree, TreeInputs, (tree.structure, tree.lengths), (tree.names,))
        self.biom = self._table.biom
        self.tree = self._tree.tree


class BatchInputs:
    """support_biom_t* array over several tables plus one tree."""

    def __init__(self, tree, tables):
        self._tables = [TableInputs(t) for t in tables]
        self._tree = TreeInputs(tree)
        self.tree = self._tree.tree
        self.n = len(tables)
        self.array = (C.POINTER(SupportBiom) * max(self.n, 1))(*[C.pointer(t.biom) for t in self._tables])


def _ids(ptr, n):
    return [ptr[i].decode() for i in range(n)]


def is_fp64(method):
    return method.endswith("_fp64")


# ------------------------------------------------------------ entry points

def _owned_view(res, destroy, ctype, n):
    """numpy view of a C result matrix; the C result is destroyed when the
    last array referring to it is gone (the ctypes buffer is the base)."""
    buf = (ctype * (n * n)).from_address(C.addressof(res.contents.matrix.contents)) if n else (ctype * 1)()
    holder = res

    def release(h=holder):
        destroy(C.byref(h))

    weakref.finalize(buf, release)
    dt = np.float64 if ctype is C.c_double else np.float32
    return np.frombuffer(buf, dtype=dt, count=n * n).reshape(n, n)


def one_off_matrix(tree, table, method, variance_adjust=False, alpha=1.0, bypass_tips=False, normalize=True,
                   subsample_depth=0, with_replacement=False, mmap_dir=None, copy=True):
    """Full n x n matrix through one_off_matrix_inmem_v3 (fp64 methods) or
    one_off_matrix_inmem_fp32_v3 (fp32 methods).  Returns (matrix, ids).
    copy=False returns a zero-copy view of the library's result, released
    when no array refers to it any more."""
    L = lib()
    x = Inputs(tree, table)
    md = mmap_dir.encode() if mmap_dir else None
    if is_fp64(method):
        res = C.POINTER(MatFull64)()
        st = L.one_off_matrix_inmem_v3(C.byref(x.biom), C.byref(x.tree), method.encode(), variance_adjust, alpha,
                                       bypass_tips, normalize, 1, subsample_depth, with_replacement, md,
                                       C.byref(res))
        if st != 0:
            raise SSUError(st, "one_off_matrix_inmem_v3")
        n = res.contents.n_samples
        ids = _ids(res.contents.sample_ids, n)
        if not copy:
            return _owned_view(res, L.destroy_mat_full_fp64, C.c_double, n), ids
        out = np.ctypeslib.as_array(res.contents.matrix, shape=(n, n)).copy()
        L.destroy_mat_full_fp64(C.byref(res))
    else:
        res = C.POINTER(MatFull32)()
        st = L.one_off_matrix_inmem_fp32_v3(C.byref(x.biom), C.byref(x.tree), method.encode(), variance_adjust,
                                            alpha, bypass_tips, normalize, 1, subsample_depth, with_replacement, md,
                                            C.byref(res))
        if st != 0:
            raise SSUError(st, "one_off_matrix_inmem_fp32_v3")
        n = res.contents.n_samples
        ids = _ids(res.contents.sample_ids, n)
        if not copy:
            return _owned_view(res, L.destroy_mat_full_fp32, C.c_float, n), ids
        out = np.ctypeslib.as_array(res.contents.matrix, shape=(n, n)).copy()
        L.destroy_mat_full_fp32(C.byref(res))
    return out, ids


def _take_results(res, n_tables, destroy, ctype, copy):
    out = []
    for t in range(n_tables):
        r = res[t]
        n = r.contents.n_samples
        ids = _ids(r.contents.sample_ids, n)
        if copy:
            m = np.ctypeslib.as_array(r.contents.matrix, shape=(n, n)).copy() if n else np.zeros((0, 0))
            destroy(C.byref(r))
        else:
            m = _owned_view(r, destroy, ctype, n)
        out.append((m, ids))
    return out


def one_off_batch(tree, tables, method, variance_adjust=False, alpha=1.0, bypass_tips=False, normalize=True,
                  copy=True):
    """Full matrices of several tables sharing `tree`, as one batch
    (ssu_b200_one_off_batch_inmem_v3 / _fp32_v3).  Returns [(matrix, ids)]."""
    L = lib()
    x = BatchInputs(tree, tables)
    fp64 = is_fp64(method)
    typ = MatFull64 if fp64 else MatFull32
    res = (C.POINTER(typ) * max(len(tables), 1))()
    fn = L.ssu_b200_one_off_batch_inmem_v3 if fp64 else L.ssu_b200_one_off_batch_inmem_fp32_v3
    st = fn(x.array, len(tables), C.byref(x.tree), method.encode(), variance_adjust, alpha, bypass_tips, normalize,
            res)
    if st != 0:
        raise SSUError(st, fn.__name__)
    return _take_results(res, len(tables), L.destroy_mat_full_fp64 if fp64 else L.destroy_mat_full_fp32,
                         C.c_double if fp64 else C.c_float, copy)


def subsample_batch(tree, table, method, n_subsamples, depth, with_replacement=False, variance_adjust=False,
                    alpha=1.0, bypass_tips=False, normalize=True, copy=True):
    """Rarefied replicates of `table` as one batch
    (ssu_b200_subsample_batch_inmem_v3 / _fp32_v3).  Returns [(matrix, ids)]."""
    L = lib()
    x = Inputs(tree, table)
    fp64 = is_fp64(method)
    typ = MatFull64 if fp64 else MatFull32
    res = (C.POINTER(typ) * max(n_subsamples, 1))()
    fn = L.ssu_b200_subsample_batch_inmem_v3 if fp64 else L.ssu_b200_subsample_batch_inmem_fp32_v3
    st = fn(C.byref(x.biom), C.byref(x.tree), method.encode(), variance_adjust, alpha, bypass_tips, normalize,
            n_subsamples, depth, with_replacement, res)
    if st != 0:
        raise SSUError(st, fn.__name__)
    return _take_results(res, n_subsamples, L.destroy_mat_full_fp64 if fp64 else L.destroy_mat_full_fp32,
                         C.c_double if fp64 else C.c_float, copy)


def status_of_matrix_call(tree, table, method, fp32_entry=False, **kw):
    """Status code of a full-matrix call (no exception), for error-path tests."""
    L = lib()
    x = Inputs(tree, table)
    if fp32_entry:
        res = C.POINTER(MatFull32)()
        st = L.one_off_matrix_inmem_fp32_v3(C.byref(x.biom), C.byref(x.tree), method.encode(), False, 1.0, False,
                                            True, 1, 0, False, None, C.byref(res))
        if st == 0:
            L.destroy_mat_full_fp32(C.byref(res))
    else:
        res = C.POINTER(MatFull64)()
        st = L.one_off_matrix_inmem_v3(C.byref(x.biom), C.byref(x.tree), method.encode(), False, 1.0, False, True,
                                       1, 0, False, None, C.byref(res))
        if st == 0:
            L.destroy_mat_full_fp64(C.byref(res))
    return st


def one_off(tree, table, method, variance_adjust=False, alpha=1.0, bypass_tips=False, normalize=True):
    """Condensed form (mat_t) through ssu_b200_one_off_inmem_v3."""
    L = lib()
    x = Inputs(tree, table)
    res = C.POINTER(Mat)()
    st = L.ssu_b200_one_off_inmem_v3(C.byref(x.biom), C.byref(x.tree), method.encode(), variance_adjust, alpha,
                                     bypass_tips, normalize, 1, C.byref(res))
    if st != 0:
        raise SSUError(st, "ssu_b200_one_off_inmem_v3")
    m = res.contents
    cf = np.ctypeslib.as_array(m.condensed_form, shape=(m.cf_size,)).copy() if m.cf_size else np.zeros(0)
    ids = _ids(m.sample_ids, m.n_samples)
    upper = bool(m.is_upper_triangle)
    L.destroy_mat(C.byref(res))
    return cf, ids, upper


def partial(tree, table, method, stripe_start, stripe_stop, variance_adjust=False, alpha=1.0, bypass_tips=False,
            normalize=True):
    """Stripes [start, stop) (partial_mat_t) through ssu_b200_partial_inmem_v3."""
    L = lib()
    x = Inputs(tree, table)
    res = C.POINTER(PartialMat)()
    st = L.ssu_b200_partial_inmem_v3(C.byref(x.biom), C.byref(x.tree), method.encode(), variance_adjust, alpha,
                                     bypass_tips, normalize, 1, stripe_start, stripe_stop, C.byref(res))
    if st != 0:
        raise SSUError(st, "ssu_b200_partial_inmem_v3")
    p = res.contents
    rows = p.stripe_stop - p.stripe_start
    stripes = np.zeros((rows, p.n_samples))
    for s in range(rows):
        stripes[s] = np.ctypeslib.as_array(p.stripes[s], shape=(p.n_samples,))
    meta = {"start": p.stripe_start, "stop": p.stripe_stop, "total": p.stripe_total,
            "upper": bool(p.is_upper_triangle), "ids": _ids(p.sample_ids, p.n_samples)}
    L.destroy_partial_mat(C.byref(res))
    return stripes, meta


def partial_to_file(tree, table, method, stripe_start, stripe_stop, path, variance_adjust=False, alpha=1.0,
                    bypass_tips=False, normalize=True):
    """Stripes [start, stop) through ssu_b200_partial_inmem_v3, written to
    `path` with write_partial (the reference's partial file format)."""
    L = lib()
    x = Inputs(tree, table)
    res = C.POINTER(PartialMat)()
    st = L.ssu_b200_partial_inmem_v3(C.byref(x.biom), C.byref(x.tree), method.encode(), variance_adjust, alpha,
                                     bypass_tips, normalize, 1, stripe_start, stripe_stop, C.byref(res))
    if st != 0:
        raise SSUError(st, "ssu_b200_partial_inmem_v3")
    io = L.write_partial(str(path).encode(), res)
    L.destroy_partial_mat(C.byref(res))
    if io != 1:
        raise RuntimeError(f"write_partial: {IO_STATUS[io]}")


def merge_partial_files(paths, fp32=False, mmap_dir=None):
    """Headers of the partial files read (read_partial_header), checked and
    merged (merge_partial_to_mmap_matrix[_fp32]); the stripes are read on
    demand by the merge.  Returns (matrix, ids)."""
    L = lib()
    mats = []
    try:
        for p in paths:
            d = C.POINTER(PartialDynMat)()
            io = L.read_partial_header(str(p).encode(), C.byref(d))
            if io != 0:
                raise RuntimeError(f"read_partial_header({p}): {IO_STATUS[io]}")
            mats.append(d)
        arr = (C.POINTER(PartialDynMat) * len(mats))(*mats)
        res = C.POINTER(MatFull32 if fp32 else MatFull64)()
        fn = L.merge_partial_to_mmap_matrix_fp32 if fp32 else L.merge_partial_to_mmap_matrix
        st = fn(arr, len(mats), mmap_dir.encode() if mmap_dir else None, C.byref(res))
        if st != 0:
            raise RuntimeError(f"merge of partial files: {MERGE_STATUS[st]}")
        n = res.contents.n_samples
        out = np.ctypeslib.as_array(res.contents.matrix, shape=(n, n)).copy()
        ids = _ids(res.contents.sample_ids, n)
        (L.destroy_mat_full_fp32 if fp32 else L.destroy_mat_full_fp64)(C.byref(res))
        return out, ids
    finally:
        for d in mats:
            L.destroy_partial_dyn_mat(C.byref(d))


def faith_pd(tree, table):
    L = lib()
    x = Inputs(tree, table)
    res = C.POINTER(RVec)()
    st = L.ssu_b200_faith_pd_inmem(C.byref(x.biom), C.byref(x.tree), C.byref(res))
    if st != 0:
        raise SSUError(st, "ssu_b200_faith_pd_inmem")
    r = res.contents
    vals = np.ctypeslib.as_array(r.values, shape=(r.n_samples,)).copy()
    ids = _ids(r.sample_ids, r.n_samples)
    L.destroy_results_vec(C.byref(res))
    return vals, ids


def dense_pair(tree, obs_ids, s1, s2, method, variance_adjust=False, alpha=1.0, bypass_tips=False, normalize=True):
    L = lib()
    x = Inputs(tree, _EmptyTable())
    ids = _strarr(obs_ids)
    a = np.ascontiguousarray(s1, dtype=np.float64)
    b = np.ascontiguousarray(s2, dtype=np.float64)
    out = C.c_double(0.0)
    st = L.one_dense_pair_v3(len(obs_ids), ids, a.ctypes.data_as(C.POINTER(C.c_double)),
                             b.ctypes.data_as(C.POINTER(C.c_double)), C.byref(x.tree), method.encode(),
                             variance_adjust, alpha, bypass_tips, normalize, C.byref(out))
    if st != 0:
        raise SSUError(st, "one_dense_pair_v3")
    return out.value


class _EmptyTable:
    obs_ids, sample_ids = [], []
    indptr = np.zeros(1, np.uint32)
    indices = np.zeros(0, np.uint32)
    data = np.zeros(0)


class OpaqueTree:
    """opaque_bptree_t from a newick string (load_bptree_opaque) or file."""

    def __init__(self, newick=None, path=None):
        self.ptr = C.c_void_p()
        if path is not None:
            st = lib().read_bptree_opaque(path.encode(), C.byref(self.ptr))
            if st != 0:
                raise RuntimeError(f"read_bptree_opaque: {IO_STATUS[st]}")
        else:
            lib().load_bptree_opaque(newick.encode(), C.byref(self.ptr))

    def arrays(self):
        n = C.c_int(0)
        lib().ssu_b200_tree_arrays(self.ptr, 0, None, None, None, C.byref(n))
        cap = n.value
        s = np.zeros(cap, dtype=np.bool_)
        ln = np.zeros(cap, dtype=np.float64)
        nm = (C.c_char_p * max(cap, 1))()
        rc = lib().ssu_b200_tree_arrays(self.ptr, cap, s.ctypes.data_as(C.POINTER(C.c_bool)),
                                        ln.ctypes.data_as(C.POINTER(C.c_double)), nm, C.byref(n))
        assert rc == 0
        return s, ln, [nm[i].decode() for i in range(cap)]

    def n_tips(self):
        return lib().get_bptree_opaque_els(self.ptr)

    def close(self):
        if self.ptr:
            lib().destroy_bptree_opaque(C.byref(self.ptr))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def read_biom(path):
    """A BIOM-HDF5 table file as a synthetic-module Table (ssu_b200_read_biom)."""
    L = lib()
    res = C.POINTER(SupportBiom)()
    st = L.ssu_b200_read_biom(str(path).encode(), C.byref(res))
    if st != 0:
        raise RuntimeError(f"ssu_b200_read_biom: {IO_STATUS[st]}")
    t = _table_of(res.contents)
    L.ssu_b200_destroy_biom(C.byref(res))
    return t


def _table_of(b):
    import ssu_synth
    nnz = b.nnz
    return ssu_synth.Table(_ids(b.obs_ids, b.n_obs), _ids(b.sample_ids, b.n_samples),
                           np.ctypeslib.as_array(b.indptr, shape=(b.n_obs + 1,)).copy(),
                           np.ctypeslib.as_array(b.indices, shape=(max(nnz, 1),))[:nnz].copy(),
                           np.ctypeslib.as_array(b.data, shape=(max(nnz, 1),))[:nnz].copy())


def rarefy_batch(table, n_subsamples, depth, with_replacement=False):
    """n_subsamples replicates of `table` rarefied to `depth` on the GPU
    (ssu_b200_rarefy_batch), as synthetic-module Tables."""
    L = lib()
    x = TableInputs(table)
    res = (C.POINTER(SupportBiom) * n_subsamples)()
    st = L.ssu_b200_rarefy_batch(C.byref(x.biom), n_subsamples, depth, with_replacement, res)
    if st != 0:
        raise SSUError(st, "ssu_b200_rarefy_batch")
    out = []
    for r in range(n_subsamples):
        out.append(_table_of(res[r].contents))
        p = C.POINTER(SupportBiom)(res[r].contents)
        L.ssu_b200_destroy_biom(C.byref(p))
    return out


def file_matrix(entry, biom_path, tree, method, variance_adjust=False, alpha=1.0, bypass_tips=False,
                normalize=True, subsample_depth=0, with_replacement=False, mmap_dir=None):
    """One of the file-based one_off_matrix* calls by name.  `tree` is a
    newick file path for the plain forms and an OpaqueTree for the *t forms.
    Returns (matrix, ids); raises SSUError with the status otherwise."""
    L = lib()
    f = getattr(L, entry)
    fp32 = "fp32" in entry
    res = C.POINTER(MatFull32 if fp32 else MatFull64)()
    tree_arg = tree.ptr if isinstance(tree, OpaqueTree) else str(tree).encode()
    md = mmap_dir.encode() if mmap_dir else None
    head = [str(biom_path).encode(), tree_arg, method.encode(), variance_adjust, alpha, bypass_tips]
    if entry.endswith("_v3") or entry.endswith("_v3t"):
        args = head + [normalize, 1, subsample_depth, with_replacement, md]
    elif entry.endswith("_v2") or entry.endswith("_v2t"):
        args = head + [1, subsample_depth, with_replacement, md]
    else:
        args = head + [1, md]
    st = f(*args, C.byref(res))
    if st != 0:
        raise SSUError(st, entry)
    n = res.contents.n_samples
    ids = _ids(res.contents.sample_ids, n)
    out = np.ctypeslib.as_array(res.contents.matrix, shape=(n, n)).copy()
    (L.destroy_mat_full_fp32 if fp32 else L.destroy_mat_full_fp64)(C.byref(res))
    return out, ids


def file_one_off(biom_path, tree_path, method, variance_adjust=False, alpha=1.0, bypass_tips=False,
                 normalize=True):
    """one_off_v3: the condensed matrix.  Returns (condensed, ids)."""
    L = lib()
    res = C.POINTER(Mat)()
    st = L.one_off_v3(str(biom_path).encode(), str(tree_path).encode(), method.encode(), variance_adjust, alpha,
                      bypass_tips, normalize, 1, C.byref(res))
    if st != 0:
        raise SSUError(st, "one_off_v3")
    m = res.contents
    cf = np.ctypeslib.as_array(m.condensed_form, shape=(max(m.cf_size, 1),))[:m.cf_size].copy()
    ids = _ids(m.sample_ids, m.n_samples)
    L.destroy_mat(C.byref(res))
    return cf, ids


def file_partial(biom_path, tree_path, method, stripe_start, stripe_stop, variance_adjust=False, alpha=1.0,
                 bypass_tips=False, normalize=True):
    """partial_v3: stripes [start, stop) as a (stop - start, n) array, ids."""
    L = lib()
    res = C.POINTER(PartialMat)()
    st = L.partial_v3(str(biom_path).encode(), str(tree_path).encode(), method.encode(), variance_adjust, alpha,
                      bypass_tips, normalize, 1, stripe_start, stripe_stop, C.byref(res))
    if st != 0:
        raise SSUError(st, "partial_v3")
    p = res.contents
    n = p.n_samples
    out = np.array([np.ctypeslib.as_array(p.stripes[s], shape=(n,)).copy()
                    for s in range(p.stripe_stop - p.stripe_start)])
    ids = _ids(p.sample_ids, n)
    L.destroy_partial_mat(C.byref(res))
    return out, ids


def file_faith_pd(biom_path, tree_path):
    """faith_pd_one_off: (values, ids)."""
    L = lib()
    res = C.POINTER(RVec)()
    st = L.faith_pd_one_off(str(biom_path).encode(), str(tree_path).encode(), C.byref(res))
    if st != 0:
        raise SSUError(st, "faith_pd_one_off")
    r = res.contents
    vals = np.ctypeslib.as_array(r.values, shape=(r.n_samples,)).copy()
    ids = _ids(r.sample_ids, r.n_samples)
    L.destroy_results_vec(C.byref(res))
    return vals, ids


def shear_collapse(tree, names=None, collapse=True):
    """Host-side shear(names) [+ collapse()] of the library (no device work);
    names=None keeps every tip."""
    x = Inputs(tree, _EmptyTable())
    n = len(tree.names)
    s = np.zeros(n, dtype=np.bool_)
    ln = np.zeros(n, dtype=np.float64)
    nm = (C.c_char_p * max(n, 1))()
    keep = _strarr(names) if names is not None else None
    out_n = C.c_int(0)
    rc = lib().ssu_b200_shear_collapse(C.byref(x.tree), keep, len(names) if names is not None else 0,
                                       1 if collapse else 0, s.ctypes.data_as(C.POINTER(C.c_bool)),
                                       ln.ctypes.data_as(C.POINTER(C.c_double)), nm, C.byref(out_n))
    assert rc == 0
    m = out_n.value
    return s[:m].copy(), ln[:m].copy(), [nm[i].decode() for i in range(m)]


class Plan:
    """Device-resident plan: inputs uploaded once, execute() recomputes the
    full matrix in HBM."""

    def __init__(self, tree, table, method, variance_adjust=False, alpha=1.0, bypass_tips=False, normalize=True):
        L = lib()
        self._x = Inputs(tree, table)
        self.ptr = C.c_void_p()
        st = L.ssu_b200_plan_create(C.byref(self._x.biom), C.byref(self._x.tree), method.encode(), variance_adjust,
                                    alpha, bypass_tips, normalize, C.byref(self.ptr))
        if st != 0:
            raise SSUError(st, "ssu_b200_plan_create")
        self.method = method
        self.n = L.ssu_b200_plan_n_samples(self.ptr)

    def execute(self, stream=None):
        st = lib().ssu_b200_plan_execute(self.ptr, C.c_void_p(stream) if stream else None)
        if st != 0:
            raise SSUError(st, "ssu_b200_plan_execute")

    def result(self, stream=None):
        dt = np.float64 if is_fp64(self.method) else np.float32
        out = np.empty((self.n, self.n), dtype=dt)
        st = lib().ssu_b200_plan_copy_result(self.ptr, out.ctypes.data_as(C.c_void_p),
                                             C.c_void_p(stream) if stream else None)
        if st != 0:
            raise SSUError(st, "ssu_b200_plan_copy_result")
        return out

    def device_result(self):
        return lib().ssu_b200_plan_device_result(self.ptr)

    def work_units(self):
        return int(lib().ssu_b200_plan_work_units(self.ptr))

    def n_embedded(self):
        return int(lib().ssu_b200_plan_n_embedded(self.ptr))

    def launches(self):
        return int(lib().ssu_b200_plan_launches(self.ptr))

    def tensor_flops(self):
        return int(lib().ssu_b200_plan_tensor_flops(self.ptr))

    def pair_kernel(self):
        return lib().ssu_b200_plan_pair_kernel(self.ptr).decode()

    def tuning(self):
        return lib().ssu_b200_plan_tuning(self.ptr).decode()

    def set_graph(self, on=True):
        lib().ssu_b200_plan_set_graph(self.ptr, 1 if on else 0)

    def set_timing(self, on=True):
        lib().ssu_b200_plan_set_timing(self.ptr, 1 if on else 0)

    def stage_ms(self):
        e, p, f = C.c_float(), C.c_float(), C.c_float()
        if lib().ssu_b200_plan_stage_ms(self.ptr, C.byref(e), C.byref(p), C.byref(f)) != 0:
            raise RuntimeError("stage timing unavailable")
        return e.value, p.value, f.value

    def close(self):
        if self.ptr:
            lib().ssu_b200_plan_destroy(C.byref(self.ptr))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchPlan(Plan):
    """Device-resident batch plan over several tables sharing one tree."""

    def __init__(self, tree, tables, method, variance_adjust=False, alpha=1.0, bypass_tips=False, normalize=True,
                 group_bytes=0, autotune=-1):
        L = lib()
        self._x = BatchInputs(tree, tables)
        self.ptr = C.c_void_p()
        st = L.ssu_b200_batch_plan_create(self._x.array, len(tables), C.byref(self._x.tree), method.encode(),
                                          variance_adjust, alpha, bypass_tips, normalize, group_bytes, autotune,
                                          C.byref(self.ptr))
        if st != 0:
            raise SSUError(st, "ssu_b200_batch_plan_create")
        self.method = method
        self.n = L.ssu_b200_plan_n_samples(self.ptr)
        self.n_tables = L.ssu_b200_plan_n_tables(self.ptr)
        self.sizes = [L.ssu_b200_plan_table_samples(self.ptr, t) for t in range(self.n_tables)]
        self.offsets = [int(L.ssu_b200_plan_table_offset(self.ptr, t)) for t in range(self.n_tables)]

    def n_groups(self):
        return int(lib().ssu_b200_plan_n_groups(self.ptr))

    def table_embedded(self, t):
        return int(lib().ssu_b200_plan_table_embedded(self.ptr, t))

    def result_of(self, t):
        """Table t's n x n result alone, copied from the plan's device buffer
        (after execute; synchronous)."""
        dt = np.float64 if is_fp64(self.method) else np.float32
        n = self.sizes[t]
        out = np.empty((n, n), dtype=dt)
        rt = C.CDLL("libcudart.so.12")
        rt.cudaMemcpy.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_int]
        if rt.cudaDeviceSynchronize() != 0:  # the plan's work runs on its own stream
            raise SSUError(6, "cudaDeviceSynchronize")
        src = self.device_result() + self.offsets[t] * out.itemsize
        if n and rt.cudaMemcpy(out.ctypes.data_as(C.c_void_p), C.c_void_p(src), out.nbytes, 2) != 0:
            raise SSUError(6, "cudaMemcpy of one table's result")
        return out

    def results(self, stream=None):
        dt = np.float64 if is_fp64(self.method) else np.float32
        total = sum(n * n for n in self.sizes)
        flat = np.empty(max(total, 1), dtype=dt)
        st = lib().ssu_b200_plan_copy_result(self.ptr, flat.ctypes.data_as(C.c_void_p),
                                             C.c_void_p(stream) if stream else None)
        if st != 0:
            raise SSUError(st, "ssu_b200_plan_copy_result")
        return [flat[o:o + n * n].reshape(n, n) for o, n in zip(self.offsets, self.sizes)]


# ------------------------------------------------- statistics on the matrix

_libc = C.CDLL(None)
_libc.free.argtypes = [C.c_void_p]
_libc.free.restype = None


def _take(ptr, shape, dtype):
    """Copy of a malloc'ed array returned by the library, which is then freed."""
    if not ptr:
        raise SSUError(6, "statistics call failed (see stderr)")
    n = int(np.prod(shape))
    out = np.ctypeslib.as_array(ptr, shape=(max(n, 1),))[:n].astype(dtype, copy=True).reshape(shape)
    _libc.free(C.cast(ptr, C.c_void_p))
    return out


def pcoa(mat, n_dims, entry="pcoa"):
    """pcoa / pcoa_fp32 / pcoa_mixed on an n x n matrix: (eigenvalues[n_dims],
    samples[n, n_dims], proportion_explained[n_dims])."""
    L = lib()
    real, out = {"pcoa": (C.c_double, C.c_double), "pcoa_fp32": (C.c_float, C.c_float),
                 "pcoa_mixed": (C.c_double, C.c_float)}[entry]
    dt = np.float64 if real is C.c_double else np.float32
    m = np.ascontiguousarray(mat, dtype=dt)
    n = m.shape[0]
    ev, sm, pr = C.POINTER(out)(), C.POINTER(out)(), C.POINTER(out)()
    getattr(L, entry)(m.ctypes.data_as(C.POINTER(real)), n, n_dims, C.byref(ev), C.byref(sm), C.byref(pr))
    odt = np.float64 if out is C.c_double else np.float32
    if not (ev and sm and pr):
        raise SSUError(6, entry)
    return _take(ev, (n_dims,), odt), _take(sm, (n, n_dims), odt), _take(pr, (n_dims,), odt)


def pcoa_device(dptr, n, n_dims):
    """pcoa on an n x n fp64 matrix in device memory (address dptr), read in place."""
    L = lib()
    ev, sm, pr = C.POINTER(C.c_double)(), C.POINTER(C.c_double)(), C.POINTER(C.c_double)()
    L.pcoa(C.cast(C.c_void_p(dptr), C.POINTER(C.c_double)), n, n_dims, C.byref(ev), C.byref(sm), C.byref(pr))
    if not (ev and sm and pr):
        raise SSUError(6, "pcoa")
    return (_take(ev, (n_dims,), np.float64), _take(sm, (n, n_dims), np.float64),
            _take(pr, (n_dims,), np.float64))


def find_eigens_fast(centered, n_dims, fp32=False):
    """find_eigens_fast(_fp32): (eigenvalues[n_dims], eigenvectors[n, n_dims])."""
    L = lib()
    real = C.c_float if fp32 else C.c_double
    dt = np.float32 if fp32 else np.float64
    m = np.ascontiguousarray(centered, dtype=dt)
    n = m.shape[0]
    ev, vec = C.POINTER(real)(), C.POINTER(real)()
    getattr(L, "find_eigens_fast_fp32" if fp32 else "find_eigens_fast")(
        n, n_dims, m.ctypes.data_as(C.POINTER(real)), C.byref(ev), C.byref(vec))
    if not (ev and vec):
        raise SSUError(6, "find_eigens_fast")
    return _take(ev, (n_dims,), dt), _take(vec, (n, n_dims), dt)


def permanova(mat, grouping, perms, fp32=False):
    """ssu_b200_permanova_fp64/_fp32: (pseudo-F, p-value)."""
    L = lib()
    real = C.c_float if fp32 else C.c_double
    m = np.ascontiguousarray(mat, dtype=np.float32 if fp32 else np.float64)
    g = np.ascontiguousarray(grouping, dtype=np.uint32)
    f, p = real(), real()
    st = getattr(L, "ssu_b200_permanova_fp32" if fp32 else "ssu_b200_permanova_fp64")(
        m.ctypes.data_as(C.POINTER(real)), m.shape[0], g.ctypes.data_as(C.POINTER(C.c_uint32)), perms,
        C.byref(f), C.byref(p))
    if st != 0:
        raise SSUError(st, "ssu_b200_permanova")
    return f.value, p.value


def compute_permanova(path, columns, mat, ids, perms, fp32=False):
    """compute_permanova_fp64/_fp32 over a full matrix with sample ids:
    (status, fstats, pvalues)."""
    L = lib()
    real = C.c_float if fp32 else C.c_double
    m = np.ascontiguousarray(mat, dtype=np.float32 if fp32 else np.float64)
    res = (MatFull32 if fp32 else MatFull64)()
    res.n_samples = m.shape[0]
    res.flags = 0
    res.matrix = m.ctypes.data_as(C.POINTER(real))
    id_arr = _strarr(ids)
    res.sample_ids = C.cast(id_arr, _strpp)
    cols = _strarr(columns)
    fs = (real * max(len(columns), 1))()
    ps = (real * max(len(columns), 1))()
    f = L.compute_permanova_fp32 if fp32 else L.compute_permanova_fp64
    st = f(str(path).encode() if path is not None else None, len(columns), C.cast(cols, _strpp), C.byref(res),
           perms, fs, ps)
    return st, list(fs)[:len(columns)], list(ps)[:len(columns)]


def read_grouping(path, column, ids):
    """ssu_b200_read_grouping: (status, grouping array, n_groups)."""
    L = lib()
    g = np.zeros(max(len(ids), 1), dtype=np.uint32)
    ng = C.c_uint32()
    id_arr = _strarr(ids)
    st = L.ssu_b200_read_grouping(str(path).encode(), column.encode(), len(ids), C.cast(id_arr, _strpp),
                                  g.ctypes.data_as(C.POINTER(C.c_uint32)), C.byref(ng))
    return st, g[:len(ids)], ng.value


def read_h5(path, dataset, strings=False):
    """A numeric dataset (as a float64 array of its shape) or, with strings,
    a string dataset (as a list) of an HDF5 file, through the library's reader."""
    L = lib()
    if not strings:
        vals = C.POINTER(C.c_double)()
        rank = C.c_uint32()
        dims = (C.c_uint64 * 8)()
        st = L.ssu_b200_read_h5_doubles(str(path).encode(), dataset.encode(), C.byref(vals), C.byref(rank), dims)
        if st != 0:
            raise RuntimeError(f"{path}:{dataset}: {IO_STATUS[st]}")
        return _take(vals, tuple(int(dims[i]) for i in range(rank.value)), np.float64)
    strs = _strpp()
    n = C.c_uint64()
    st = L.ssu_b200_read_h5_strings(str(path).encode(), dataset.encode(), C.byref(strs), C.byref(n))
    if st != 0:
        raise RuntimeError(f"{path}:{dataset}: {IO_STATUS[st]}")
    out = _ids(strs, n.value)
    L.ssu_b200_free_h5_strings(strs, n.value)
    return out
