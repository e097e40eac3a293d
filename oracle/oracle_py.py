"""Test infrastructure only: ctypes bindings to the oracle.

Two oracles live under this directory:

* `liboracle.so` - the C restatement of the reference algorithm
  (oracle/unifrac_oracle.c), always built by `make -C oracle oracle`;
* `_ref/libssu_ref.so` - the reference's own CPU hot path compiled from its
  sources (oracle/Makefile, target `ref`), present when it could be built.

Only tests/, `__graft_entry__.smoke()` and bench.py's CPU-baseline leg import
this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libssu_ref.so")

_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)
_f64p = C.POINTER(C.c_double)
_boolp = C.POINTER(C.c_bool)
_strpp = C.POINTER(C.c_char_p)


def _strarr(strings):
    arr = (C.c_char_p * len(strings))()
    arr[:] = [s.encode() for s in strings]
    return arr


def _ptr(a, t):
    return a.ctypes.data_as(t)


class _Marshalled:
    """Keeps ctypes views of a (tree, table) pair alive for one call."""

    def __init__(self, tree, table):
        self.indptr = np.ascontiguousarray(table.indptr, dtype=np.uint32)
        self.indices = np.ascontiguousarray(table.indices, dtype=np.uint32)
        self.data = np.ascontiguousarray(table.data, dtype=np.float64)
        self.obs = _strarr(table.obs_ids)
        self.samples = _strarr(table.sample_ids)
        self.structure = np.ascontiguousarray(tree.structure, dtype=np.bool_)
        self.lengths = np.ascontiguousarray(tree.lengths, dtype=np.float64)
        self.names = _strarr(tree.names)
        self.n_obs = table.n_obs
        self.n_samples = table.n_samples
        self.n_parens = tree.n_parens

    def table_args(self):
        return (_ptr(self.indptr, _u32p), _ptr(self.indices, _u32p), _ptr(self.data, _f64p),
                self.n_obs, self.n_samples, self.obs, self.samples)

    def tree_args(self):
        return (_ptr(self.structure, _boolp), _ptr(self.lengths, _f64p), self.names, self.n_parens)


_TABLE_TREE_ARGS = [_u32p, _u32p, _f64p, C.c_int, C.c_int, _strpp, _strpp, _boolp, _f64p, _strpp, C.c_int]


class OracleError(RuntimeError):
    pass


def ref_available() -> bool:
    return os.path.exists(REF_SO)


_ref_lib = None
_oracle_lib = None


def _load_ref():
    global _ref_lib
    if _ref_lib is None:
        lib = C.CDLL(REF_SO)
        lib.ssu_ref_one_off.restype = C.c_int
        lib.ssu_ref_one_off.argtypes = _TABLE_TREE_ARGS + [
            C.c_char_p, C.c_bool, C.c_double, C.c_bool, C.c_bool, C.c_uint, C.c_uint, C.c_uint,
            _f64p, _f64p, _f64p, _u64p, _f64p]
        lib.ssu_ref_faith_pd.restype = C.c_int
        lib.ssu_ref_faith_pd.argtypes = _TABLE_TREE_ARGS + [_f64p, _u32p, _u32p, _f64p]
        _ref_lib = lib
    return _ref_lib


def _load_oracle():
    global _oracle_lib
    if _oracle_lib is None:
        lib = C.CDLL(ORACLE_SO)
        lib.oracle_one_off.restype = C.c_int
        lib.oracle_one_off.argtypes = _TABLE_TREE_ARGS + [
            C.c_char_p, C.c_bool, C.c_double, C.c_bool, C.c_bool, C.c_uint, C.c_uint,
            _f64p, _f64p, _u64p]
        lib.oracle_faith_pd.restype = C.c_int
        lib.oracle_faith_pd.argtypes = _TABLE_TREE_ARGS + [_f64p, _u32p, _u32p]
        _oracle_lib = lib
    return _oracle_lib


def _n_stripes(n):
    return (n + 1) // 2


def ref_one_off(tree, table, method, variance_adjust=False, alpha=1.0, bypass_tips=False,
                normalize=True, n_substeps=1, stripe_start=0, stripe_stop=0, want_matrix=True,
                with_timing=False):
    """Run the reference's compiled CPU path.  Returns a dict with `stripes`
    (stop-start, n), `matrix` (n, n) when the full range was asked for,
    `condensed`, `n_embedded` and, when asked, `seconds` = (stripes, matrix)."""
    lib = _load_ref()
    m = _Marshalled(tree, table)
    n = table.n_samples
    stop = stripe_stop if stripe_stop else _n_stripes(n)
    stripes = np.zeros((stop - stripe_start, n), dtype=np.float64)
    full = want_matrix and stripe_start == 0 and stop == _n_stripes(n)
    matrix = np.zeros((n, n), dtype=np.float64) if full else None
    cond = np.zeros(n * (n - 1) // 2, dtype=np.float64) if full else None
    n_emb = C.c_uint64(0)
    secs = np.zeros(2, dtype=np.float64)
    rc = lib.ssu_ref_one_off(*m.table_args(), *m.tree_args(), method.encode(), variance_adjust, alpha,
                             bypass_tips, normalize, n_substeps, stripe_start, stripe_stop,
                             _ptr(stripes, _f64p), _ptr(matrix, _f64p) if full else None,
                             _ptr(cond, _f64p) if full else None, C.byref(n_emb), _ptr(secs, _f64p))
    if rc != 0:
        raise OracleError(f"reference one_off status {rc}")
    out = {"stripes": stripes, "matrix": matrix, "condensed": cond, "n_embedded": int(n_emb.value)}
    if with_timing:
        out["seconds"] = (float(secs[0]), float(secs[1]))
    return out


def ref_faith_pd(tree, table, with_timing=False):
    lib = _load_ref()
    m = _Marshalled(tree, table)
    n = table.n_samples
    vals = np.zeros(n, dtype=np.float64)
    kept = np.zeros(n, dtype=np.uint32)
    n_kept = C.c_uint32(0)
    secs = np.zeros(1, dtype=np.float64)
    rc = lib.ssu_ref_faith_pd(*m.table_args(), *m.tree_args(), _ptr(vals, _f64p), _ptr(kept, _u32p),
                              C.byref(n_kept), _ptr(secs, _f64p))
    if rc != 0:
        raise OracleError(f"reference faith_pd status {rc}")
    k = int(n_kept.value)
    out = {"values": vals[:k].copy(), "kept": kept[:k].copy()}
    if with_timing:
        out["seconds"] = float(secs[0])
    return out


def oracle_one_off(tree, table, method, variance_adjust=False, alpha=1.0, bypass_tips=False,
                   normalize=True, stripe_start=0, stripe_stop=0):
    """Run the C restatement.  Returns `stripes` (stop-start, n), `matrix`
    (n, n) for the full stripe range, and `n_embedded`."""
    lib = _load_oracle()
    m = _Marshalled(tree, table)
    n = table.n_samples
    stop = stripe_stop if stripe_stop else _n_stripes(n)
    stripes = np.zeros((stop - stripe_start, n), dtype=np.float64)
    full = stripe_start == 0 and stop == _n_stripes(n)
    matrix = np.zeros((n, n), dtype=np.float64) if full else None
    n_emb = C.c_uint64(0)
    rc = lib.oracle_one_off(*m.table_args(), *m.tree_args(), method.encode(), variance_adjust, alpha,
                            bypass_tips, normalize, stripe_start, stripe_stop, _ptr(stripes, _f64p),
                            _ptr(matrix, _f64p) if full else None, C.byref(n_emb))
    if rc != 0:
        raise OracleError(f"oracle one_off status {rc}")
    return {"stripes": stripes, "matrix": matrix, "n_embedded": int(n_emb.value)}


def oracle_faith_pd(tree, table):
    lib = _load_oracle()
    m = _Marshalled(tree, table)
    n = table.n_samples
    vals = np.zeros(n, dtype=np.float64)
    kept = np.zeros(n, dtype=np.uint32)
    n_kept = C.c_uint32(0)
    rc = lib.oracle_faith_pd(*m.table_args(), *m.tree_args(), _ptr(vals, _f64p), _ptr(kept, _u32p),
                             C.byref(n_kept))
    if rc != 0:
        raise OracleError(f"oracle faith_pd status {rc}")
    k = int(n_kept.value)
    return {"values": vals[:k].copy(), "kept": kept[:k].copy()}
