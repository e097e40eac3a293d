"""Regenerate tests/golden/reference_golden.json from the reference's own tests.

Reads the reference checkout as text only (nothing is compiled or run):

* src/test_su.cpp   - per test function, every `double|uint32_t NAME[] = {...}`
                      array, every `std::vector<...> NAME = {...}` literal,
                      every newick string given to su::BPTree and every
                      `to_keep = {...}` set;
* test/capi_inmem_test.c - the inline CSR copy of test.biom (obs ids, sample
                      ids, indices, indptr, data);
* src/test*.tre     - the newick trees the API tests load.

It also copies, byte for byte, the data files the reference's own checks run
on into tests/golden/fixtures/ (the BIOM-HDF5 tables, their trees and the
expected outputs the reference compares against):

* ci/crawford.biom, ci/crawford.tre and the outputs ci/crawford_test.sh
  compares with: ci/test.ssu.exp (unweighted_fp64), ci/test.ssu_vaw.exp
  (unweighted_fp64, variance adjusted), ci/test.faith.exp (Faith PD);
* src/testdata/absquant.biom, absquant.tree and the weighted-normalized
  matrices without and with sample-count normalisation
  (test.absquant.wn.dm, test.absquant_not.wn.dm);
* src/test.biom, the 6 x 5 table of the reference's unit tests;
* src/test_ska_pcoa_big.dat (57 x 57 matrix with its PCoA, test_pcoa_big),
  src/testdata/test500.tsv (sample metadata) and two of the reference's
  HDF5 outputs on its 500-sample table (distance matrix, sample order and
  4-axis PCoA): test500.unweighted_fp32.f.h5 and
  test500.weighted_unnormalized_fp32.h5.

From src/test_ska.cpp (the statistics tests) it keeps, per test function,
every numeric array and every `exp_*` scalar; from
src/testdata/validation_tests.sh every PERMANOVA check
(compare_unifrac_stats.py arguments with the method and grouping column of
the ssu run before it) and every PCoA check (compare_unifrac_pcoa.py: file,
axes compared, relative precision).

Usage: python tests/golden/make_golden.py [/path/to/reference]
(default: $UNIFRAC_REFERENCE_PATH, else BASELINE.json's reference_path)
"""
import json
import os
import re
import sys

def _default_reference():
    """UNIFRAC_REFERENCE_PATH, else BASELINE.json's reference_path."""
    if os.environ.get("UNIFRAC_REFERENCE_PATH"):
        return os.environ["UNIFRAC_REFERENCE_PATH"]
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "..", "..", "BASELINE.json")) as f:
        return json.load(f)["reference_path"]


REF = sys.argv[1] if len(sys.argv) > 1 else _default_reference()
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_golden.json")


def _numbers(body):
    """Parse a C initialiser list of numbers; None if it holds anything else."""
    body = re.sub(r"//[^\n]*", "", body)
    vals = []
    try:
        for tok in body.replace("\n", " ").split(","):
            tok = tok.strip()
            if not tok:
                continue
            if "/" in tok:  # e.g. 1.0/3
                a, b = tok.split("/")
                vals.append(float(a) / float(b))
            else:
                vals.append(float(tok))
    except ValueError:
        return None
    return vals


def _split_functions(text):
    funcs = {}
    for m in re.finditer(r"^void (test_\w+)\(\)\s*\{", text, flags=re.M):
        start = m.end()
        depth = 1
        i = start
        while depth and i < len(text):
            if text[i] == "{":
                depth += 1
            elif text[i] == "}":
                depth -= 1
            i += 1
        funcs[m.group(1)] = text[start:i]
    return funcs


def parse_test_su(path):
    text = open(path).read()
    out = {}
    for name, body in _split_functions(text).items():
        entry = {"arrays": {}, "vectors": {}, "newick": [], "to_keep": []}
        for m in re.finditer(r"(?:const\s+)?(double|uint32_t)\s+(\w+)\s*\[\d*\]\s*=\s*\{([^}]*)\}", body):
            vals = _numbers(m.group(3))
            if vals is not None:
                entry["arrays"].setdefault(m.group(2), []).append(vals)
        for m in re.finditer(r"bool\s+(\w+)\s*\[\d*\]\s*=\s*\{([^}]*)\}", body):
            toks = [t.strip() for t in m.group(2).split(",") if t.strip()]
            if all(t in ("0", "1", "true", "false") for t in toks):
                entry["arrays"].setdefault(m.group(1), []).append([1.0 if t in ("1", "true") else 0.0 for t in toks])
        for m in re.finditer(r"std::vector<(bool|double|std::string)>\s+(\w+)\s*=\s*\{([^}]*)\}", body):
            kind, vname, content = m.groups()
            if kind == "bool":
                vals = [t.strip() == "true" for t in content.split(",") if t.strip()]
            elif kind == "double":
                vals = _numbers(content)
            else:
                vals = re.findall(r'"([^"]*)"', content)
            entry["vectors"][vname] = vals
        entry["newick"] = re.findall(r'su::BPTree\s+\w+\("([^"]*)"\)', body)
        for m in re.finditer(r"to_keep\s*=\s*\{([^}]*)\}", body):
            entry["to_keep"].append(re.findall(r'"([^"]*)"', m.group(1)))
        if any(entry.values()):
            out[name] = entry
    return out


def parse_test_ska(path):
    text = open(path).read()
    out = {}
    for name, body in _split_functions(text).items():
        entry = {"arrays": {}, "scalars": {}}
        for m in re.finditer(r"(?:const\s+)?(double|float|uint32_t)\s+(\w+)\s*\[\d*\]\s*=\s*\{([^}]*)\}", body):
            vals = _numbers(m.group(3))
            if vals is not None:
                entry["arrays"].setdefault(m.group(2), []).append(vals)
        for m in re.finditer(r"(?:const\s+)?(?:float|double)\s+(exp_\w+)\s*=\s*([-+0-9.eE]+)\s*;", body):
            entry["scalars"][m.group(1)] = float(m.group(2))
        if entry["arrays"] or entry["scalars"]:
            out[name] = entry
    return out


def parse_validation(path):
    """PERMANOVA and PCoA checks of validation_tests.sh."""
    stats, pcoa = [], []
    method = column = perms = None
    for line in open(path):
        m = re.search(r"\bssu\s.*?-m\s+(\S+)", line)
        if m:
            method = m.group(1)
            c = re.search(r"\s-c\s+(\S+)", line)
            column = c.group(1) if c else None
            q = re.search(r"--permanova\s+(\d+)", line)
            perms = int(q.group(1)) if q else None
            continue
        m = re.search(r"compare_unifrac_stats\.py\s+\S+\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)\s+(\S+)", line)
        if m:
            g, n, v, pv, pr_v, pr_p = m.groups()
            stats.append({"method": method, "column": column, "permanova_flag": perms, "n_groups": int(g),
                          "n_perms": int(n), "value": float(v), "pvalue": float(pv), "prec_value": float(pr_v),
                          "prec_pvalue": float(pr_p)})
            continue
        m = re.search(r"compare_unifrac_pcoa\.py\s+(\S+)\s+\S+\s+(\d+)\s+(\S+)", line)
        if m:
            pcoa.append({"method": method, "expected": m.group(1), "axes": int(m.group(2)),
                         "precision": float(m.group(3))})
    return {"permanova": stats, "pcoa": pcoa}


def parse_capi_inmem(path):
    text = open(path).read()

    def strings(var):
        m = re.search(var + r"\[\]\s*=\s*\{([^}]*)\}", text)
        return re.findall(r'"([^"]*)"', m.group(1))

    def nums(var):
        m = re.search(var + r"\[\]\s*=\s*\{([^}]*)\}", text)
        return _numbers(m.group(1))

    return {
        "obs_ids": strings("obs_ids"),
        "sample_ids": strings("samp_ids"),
        "indices": [int(v) for v in nums("indices")],
        "indptr": [int(v) for v in nums("indptr")],
        "data": nums("data"),
    }


def main():
    golden = {
        "source": "biocore/unifrac-binaries tests, read as text by tests/golden/make_golden.py",
        "test_su": parse_test_su(os.path.join(REF, "src", "test_su.cpp")),
        "table_csr": parse_capi_inmem(os.path.join(REF, "test", "capi_inmem_test.c")),
        "trees": {},
        "test_ska": parse_test_ska(os.path.join(REF, "src", "test_ska.cpp")),
        "validation": parse_validation(os.path.join(REF, "src", "testdata", "validation_tests.sh")),
    }
    for fn in sorted(os.listdir(os.path.join(REF, "src"))):
        if fn.endswith(".tre"):
            golden["trees"][fn] = open(os.path.join(REF, "src", fn)).read().strip()
    with open(OUT, "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)
    print("wrote", OUT)
    fixtures = os.path.join(os.path.dirname(OUT), "fixtures")
    os.makedirs(fixtures, exist_ok=True)
    for rel in FIXTURES:
        src = os.path.join(REF, rel)
        dst = os.path.join(fixtures, os.path.basename(rel))
        with open(src, "rb") as a, open(dst, "wb") as b:
            b.write(a.read())
        print("copied", rel)


FIXTURES = ["ci/crawford.biom", "ci/crawford.tre", "ci/test.ssu.exp", "ci/test.ssu_vaw.exp", "ci/test.faith.exp",
            "src/testdata/absquant.biom", "src/testdata/absquant.tree", "src/testdata/test.absquant.wn.dm",
            "src/testdata/test.absquant_not.wn.dm", "src/test.biom", "src/test_ska_pcoa_big.dat",
            "src/testdata/test500.tsv", "src/testdata/test500.unweighted_fp32.f.h5",
            "src/testdata/test500.weighted_unnormalized_fp32.h5"]


if __name__ == "__main__":
    main()
