"""Host-side checks of libssu_b200.so that need no GPU: it loads, exports
every function include/unifrac_b200.h declares, parses newick and shears /
collapses trees as the reference (src/test_su.cpp goldens), and returns the
reference's status codes for inputs rejected before any device work."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import ssu_synth


@pytest.fixture(scope="module")
def L(ssu):
    return ssu.lib()


def test_library_exports_every_declared_function(ssu, L):
    declared = ssu.declared_functions()
    assert len(declared) >= 45
    out = subprocess.run(["nm", "-D", "--defined-only", ssu.LIB_PATH], capture_output=True, text=True, check=True)
    exported = {line.split()[-1] for line in out.stdout.splitlines() if line.strip()}
    missing = [f for f in declared if f not in exported]
    assert not missing, missing
    for f in declared:
        assert hasattr(L, f)


def test_reference_api_names_present(ssu):
    # the drop-in subset of src/api.hpp named by the boundary contract
    must = ["one_off", "one_off_v3", "one_off_wtree", "one_off_wtree_v3", "one_off_matrix_inmem_v3",
            "one_off_matrix_inmem_fp32_v3", "one_off_matrix_inmem_v2", "one_off_matrix_inmem_fp32_v2",
            "one_off_inmem", "one_off_inmem_fp32", "one_off_matrix_v3", "one_off_matrix_fp32_v3",
            "one_dense_pair_v3", "one_dense_pair_v3t", "one_dense_pair_v2", "one_dense_pair_v2t",
            "faith_pd_one_off", "partial", "partial_v3", "read_bptree_opaque", "load_bptree_opaque",
            "convert_bptree_opaque", "destroy_bptree_opaque", "get_bptree_opaque_els", "destroy_mat",
            "destroy_mat_full_fp64", "destroy_mat_full_fp32", "destroy_partial_mat", "destroy_partial_dyn_mat",
            "destroy_results_vec", "ssu_set_random_seed"]
    declared = set(ssu.declared_functions())
    assert not [m for m in must if m not in declared]


def test_struct_layouts_match_c_header(tmp_path):
    """The ctypes mirror has the header's layout (field offsets and sizes
    measured by a C compiler against include/unifrac_b200.h)."""
    import ssu_b200 as s
    structs = {"support_biom_t": s.SupportBiom, "support_bptree_t": s.SupportBPTree,
               "mat_full_fp64_t": s.MatFull64, "mat_full_fp32_t": s.MatFull32, "mat_t": s.Mat,
               "r_vec": s.RVec, "partial_mat_t": s.PartialMat}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "unifrac_b200.h"', 'int main(void){']
    for cname, py in structs.items():
        lines.append(f'printf("{cname} %zu\\n", sizeof({cname}));')
        for fname, _ in py._fields_:
            lines.append(f'printf("{cname}.{fname} %zu\\n", offsetof({cname}, {fname}));')
    lines.append("return 0;}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-I", inc, str(src), "-o", str(exe)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.splitlines())
    for cname, py in structs.items():
        assert int(got[cname]) == ctypes.sizeof(py), cname
        for fname, _ in py._fields_:
            assert int(got[f"{cname}.{fname}"]) == getattr(py, fname).offset, (cname, fname)


NEWICK_CASES = [
    ("test_bptree_constructor_edgecases", [f"structure_arr{i}" for i in range(1, 6)]),
    ("test_bptree_constructor_single_descendent", ["structure_arr"]),
    ("test_bptree_constructor_complex", ["structure_arr"]),
    ("test_bptree_constructor_semicolon", ["structure_arr"]),
]


@pytest.mark.parametrize("func,arrays", NEWICK_CASES)
def test_newick_structure_goldens(ssu, golden, func, arrays):
    entry = golden["test_su"][func]
    for newick, arr in zip(entry["newick"], arrays):
        t = ssu.OpaqueTree(newick=newick)
        s, ln, names = t.arrays()
        assert s.astype(int).tolist() == [int(v) for v in entry["arrays"][arr][0]], newick
        if "length_arr" in entry["arrays"] and len(arrays) == 1:
            np.testing.assert_allclose(ln, np.float32(entry["arrays"]["length_arr"][0]).astype(np.float64))
        t.close()


@pytest.mark.parametrize("func", ["test_bptree_constructor_quoted_comma", "test_bptree_constructor_quoted_parens"])
def test_newick_quoted_names(ssu, golden, func):
    entry = golden["test_su"][func]
    t = ssu.OpaqueTree(newick=entry["newick"][0])
    _, _, names = t.arrays()
    assert names == entry["vectors"]["exp_names"]


def test_newick_lengths_read_in_single_precision(ssu):
    t = ssu.OpaqueTree(newick="(a:0.1,b:0.3)r;")
    _, ln, names = t.arrays()
    assert names[1] == "a" and ln[1] == float(np.float32(0.1)) and ln[1] != 0.1
    assert t.n_tips() == 2


def _tree_arrays(newick):
    return ssu_synth.parse_newick(newick)


@pytest.mark.parametrize("func,collapse", [("test_bptree_shear_simple", False), ("test_bptree_shear_deep", False),
                                           ("test_bptree_collapse_simple", True)])
def test_shear_and_collapse_goldens(ssu, golden, func, collapse):
    entry = golden["test_su"][func]
    tree = _tree_arrays(entry["newick"][0])
    names = entry["to_keep"][0] if entry["to_keep"] else None
    s, ln, nm = ssu.shear_collapse(tree, names, collapse=collapse)
    v = entry["vectors"]
    assert s.tolist() == v["exp_structure"]
    np.testing.assert_allclose(ln, v["exp_lengths"])
    assert nm == v["exp_names"]


def test_collapse_edge_against_root(ssu, golden):
    tree = _tree_arrays("((a),b)r;")
    exp = _tree_arrays("(a,b)r;")
    s, ln, nm = ssu.shear_collapse(tree, None, collapse=True)
    assert s.tolist() == exp.structure.tolist()
    assert nm == exp.names


def test_shear_collapse_matches_oracle_embedding_count(ssu, oracle_mod):
    tree = ssu_synth.random_binary_tree(300, 0.1, 3)
    keep = tree.tip_names()[::3]
    s, _, _ = ssu.shear_collapse(tree, keep, collapse=True)
    table = ssu_synth.geometric_table(keep, 10, 0.3, 5.0, 9)
    r = oracle_mod.oracle_one_off(tree, table, "unweighted_fp64")
    assert r["n_embedded"] == len(s) // 2 - 1


def test_pre_device_status_codes(ssu, test_tree, test_table):
    # method strings and precision entry points (src/api.cpp:775-829)
    assert ssu.status_of_matrix_call(test_tree, test_table, "bogus") == 4            # unknown_method
    assert ssu.status_of_matrix_call(test_tree, test_table, "unweighted") == 7       # invalid_method
    assert ssu.status_of_matrix_call(test_tree, test_table, "unweighted_fp64", fp32_entry=True) == 7
    other = ssu_synth.parse_newick("(a:1,b:2)r;")
    assert ssu.status_of_matrix_call(other, test_table, "unweighted_fp64") == 5     # no overlap
    empty = ssu_synth.Table([], ["S1"], np.zeros(1, np.uint32), np.zeros(0, np.uint32), np.zeros(0))
    assert ssu.status_of_matrix_call(test_tree, empty, "unweighted_fp64") == 3      # table_empty


def test_file_entry_points_statuses(ssu, L, tmp_path):
    missing = str(tmp_path / "nope.biom")
    tre = tmp_path / "t.tre"
    tre.write_text("(GG_OTU_1:1,GG_OTU_2:1);")
    biom = tmp_path / "t.biom"
    biom.write_bytes(b"\x89HDF\r\n\x1a\n")
    for b, t, want in [(missing, str(tre), 2), (str(biom), missing, 1), (str(biom), str(tre), 2)]:
        with pytest.raises(ssu.SSUError) as e:   # an HDF5 signature alone is not a readable table
            ssu.file_faith_pd(b, t)
        assert e.value.status == want
    t = ssu.OpaqueTree(path=str(tre))
    assert t.n_tips() == 2


def test_header_is_plain_c(tmp_path):
    src = tmp_path / "t.c"
    inc = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")
    src.write_text('#include "unifrac_b200.h"\nint main(void){ mat_t *m = 0; destroy_mat(&m); return 0; }\n')
    exe = tmp_path / "t"
    cc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
    import ssu_b200
    libdir = os.path.dirname(ssu_b200.LIB_PATH)
    subprocess.run([cc, "-std=c99", "-Wall", "-Werror", "-I", inc, str(src), "-o", str(exe), "-L", libdir,
                    "-lssu_b200", f"-Wl,-rpath,{libdir}"], check=True)
    assert subprocess.run([str(exe)]).returncode == 0


def test_malformed_csr_is_rejected_before_device_work(ssu, test_tree, test_table):
    """A borrowed CSR whose offsets or sample positions are out of range would
    be read and scattered out of bounds; it is reported as table_missing
    (the reference has no check and reads out of bounds)."""
    t = test_table

    def with_arrays(indptr, indices):
        return ssu_synth.Table(t.obs_ids, t.sample_ids, indptr, indices, t.data)

    bad_index = t.indices.copy()
    bad_index[len(bad_index) // 2] = t.n_samples
    assert ssu.status_of_matrix_call(test_tree, with_arrays(t.indptr, bad_index), "unweighted_fp64") == 2
    shifted = t.indptr.copy()
    shifted[0] = 1
    assert ssu.status_of_matrix_call(test_tree, with_arrays(shifted, t.indices), "unweighted_fp64") == 2
    decreasing = t.indptr.copy()
    decreasing[2] = decreasing[1] - 1 if decreasing[1] > 0 else decreasing[3] + 1
    assert ssu.status_of_matrix_call(test_tree, with_arrays(decreasing, t.indices), "weighted_normalized_fp64") == 2
    # the well-formed table passes this check (without a GPU it stops later,
    # at the device)
    assert ssu.status_of_matrix_call(test_tree, t, "unweighted_fp64") != 2


def test_unbalanced_tree_is_rejected_before_device_work(ssu, test_tree, test_table):
    """Parentheses that do not pair up are reported as tree_missing."""
    t = test_tree
    open_end = np.array(t.structure, dtype=bool).copy()
    open_end[-1] = True  # the root never closes
    tree = ssu_synth.BPTree(open_end, t.lengths, t.names)
    assert ssu.status_of_matrix_call(tree, test_table, "unweighted_fp64") == 1
    odd = ssu_synth.BPTree(np.array(t.structure, dtype=bool)[:-1], t.lengths[:-1], t.names[:-1])
    assert ssu.status_of_matrix_call(odd, test_table, "weighted_normalized_fp64") == 1
