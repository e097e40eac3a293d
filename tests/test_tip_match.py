"""Tip matching (BPTree::match_tips, the name check of the reference's
VALIDATE_TREE_TABLE, src/api.cpp:94-100): each tip of the tree takes the
table row of the observation with its name.  Trees of 65,536 parentheses or
more are matched on several host threads; the tags, the count of distinct
rows matched and the all-tips flag must be the same whatever the thread
count, with tips missing from the table, table names missing from the tree
and a name repeated in the table (the last row wins).  A host program built
from the tree source checks this on the CPU."""
import os
import subprocess

import numpy as np
import pytest

import ssu_synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "unifrac-binaries_b200", "csrc")

PROBE = r"""
#include <cstdio>
#include <fstream>
#include <memory>
#include <string>
#include <vector>
#include "ssu_names.hpp"
#include "ssu_tree.hpp"
static std::vector<std::string> lines(const char *p) {
    std::ifstream f(p);
    std::vector<std::string> v;
    std::string s;
    while (std::getline(f, s)) v.push_back(s);
    return v;
}
int main(int argc, char **argv) {
    std::vector<std::string> open_s = lines(argv[1]), names = lines(argv[2]), obs = lines(argv[3]);
    const size_t n = open_s.size();
    std::unique_ptr<bool[]> open(new bool[n]);
    std::vector<double> len(n, 1.0);
    std::vector<const char *> np(n);
    names.resize(n);
    for (size_t i = 0; i < n; i++) {
        open[i] = open_s[i] == "1";
        np[i] = names[i].c_str();
    }
    ssu::BPTree t = ssu::BPTree::from_arrays(open.get(), len.data(), np.data(), static_cast<int>(n), false);
    ssu::NameMap m(obs.size());
    for (size_t i = 0; i < obs.size(); i++) m.set(obs[i], static_cast<uint32_t>(i));
    const ssu::TipMatch tm = t.match_tips(m, static_cast<uint32_t>(obs.size()));
    std::FILE *o = std::fopen(argv[4], "w");
    std::fprintf(o, "%u %d\n", tm.rows_matched, tm.all_tips ? 1 : 0);
    for (int32_t x : tm.tags) std::fprintf(o, "%d\n", x);
    std::fclose(o);
    return 0;
}
"""


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    d = tmp_path_factory.mktemp("tipmatch")
    src = d / "probe.cpp"
    src.write_text(PROBE)
    exe = d / "probe"
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-O2", "-std=c++17", "-I", CSRC, str(src), os.path.join(CSRC, "ssu_tree.cpp"), "-o",
                    str(exe), "-lpthread"], check=True)
    return exe, d


def _match(probe, tree, obs, threads):
    exe, d = probe
    (d / "open.txt").write_text("\n".join("1" if b else "0" for b in tree.structure))
    (d / "names.txt").write_text("\n".join(tree.names))
    (d / "obs.txt").write_text("\n".join(obs))
    out = d / f"tags{threads}.txt"
    subprocess.run([str(exe), str(d / "open.txt"), str(d / "names.txt"), str(d / "obs.txt"), str(out)], check=True,
                   env=dict(os.environ, OMP_NUM_THREADS=str(threads)))
    head, *tags = out.read_text().split("\n")
    matched, all_tips = (int(x) for x in head.split())
    return matched, bool(all_tips), np.array([int(x) for x in tags if x])


@pytest.mark.parametrize("case", ["all_tips", "some_missing"])
def test_threaded_tip_matching_equals_one_thread(probe, case):
    tree = ssu_synth.random_binary_tree(40000, 0.05, 17)  # 159,998 parentheses: the threaded path
    tips = tree.tip_names()
    rng = np.random.default_rng(5)
    if case == "all_tips":
        obs = list(tips) + [tips[123]]  # a repeated name: the last row wins
    else:
        keep = rng.random(len(tips)) < 0.7
        obs = [t for t, k in zip(tips, keep) if k] + ["not_in_tree_%d" % i for i in range(50)]
    obs = [obs[i] for i in rng.permutation(len(obs))]
    ref = _match(probe, tree, obs, 1)
    for threads in (2, 4, 7):
        got = _match(probe, tree, obs, threads)
        assert got[0] == ref[0] and got[1] == ref[1]
        np.testing.assert_array_equal(got[2], ref[2])
    row_of = {}
    for i, o in enumerate(obs):
        row_of[o] = i
    n_tips_in_table = sum(t in row_of for t in tips)
    assert ref[0] == len({row_of[t] for t in tips if t in row_of})
    assert ref[1] == (n_tips_in_table == len(tips))
