// Host-side phylogeny handling for the B200 UniFrac engine: balanced-
// parentheses trees, newick parsing, shear/collapse and the flattened
// postorder that the device embedding consumes.
#pragma once

#include <cstdint>
#include <deque>
#include <memory>
#include <string>
#include <string_view>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include "ssu_names.hpp"

namespace ssu {

using NameSet = std::unordered_set<std::string_view>;
using NameIndex = std::unordered_map<std::string_view, uint32_t>;

struct BPTree;

// The tips of a tree matched against a table's observation names, computed
// once per call and shared by validation and the shear: tags[i] = table row of
// the tip opening at i (-1 for unmatched tips and internal nodes).
struct TipMatch {
    std::vector<int32_t> tags;
    uint32_t rows_matched = 0;  // distinct table rows some tip carries
    bool all_tips = false;      // every tip matched: the shear keeps the whole tree
    const uint8_t *tree_id = nullptr;  // the tree it was computed for
    uint32_t tree_size = 0;
};

// A rooted tree in balanced-parentheses form.  open[i] is true for '(' and
// the length and name of a node live at its opening index, as the
// reference's BPTree (src/tree.hpp:21-153).  match[i] pairs every
// parenthesis with its partner.  Names are views: into `storage` when the
// tree owns them, else into the caller's arrays for the duration of a call.
struct BPTree {
    std::vector<uint8_t> open;
    std::vector<double> length;
    std::vector<std::string_view> name;
    std::vector<uint32_t> match;
    std::shared_ptr<std::deque<std::string>> storage;
    // optional per-parenthesis tag carried through shear/collapse: the table
    // row of each kept tip (-1 elsewhere)
    std::vector<int32_t> tag;
    // parentheses that do not pair up (odd count, a close without an open, or
    // opens left at the end): validation rejects the tree before device work
    bool malformed = false;

    uint32_t size() const { return static_cast<uint32_t>(open.size()); }
    bool leaf(uint32_t i) const { return open[i] && i + 1 < open.size() && !open[i + 1]; }
    void pair_parentheses();

    // src/tree.cpp:72-99.  With copy_names the tree owns its names;
    // otherwise it views the caller's strings.
    static BPTree from_arrays(const bool *structure, const double *lengths, const char *const *names, int n,
                              bool copy_names);
    // Newick text -> tree, following the reference parser's rules
    // (src/tree.cpp:315-455): quotes group a label and are dropped, newlines
    // are skipped, a label's last ':' splits name and length, and lengths are
    // read in single precision (std::stof, src/tree.cpp:446,449).
    static bool from_newick(const std::string &text, BPTree &out);

    // Keep the tips named in `keep` and all their ancestors (src/tree.cpp:145-163).
    BPTree shear(const NameSet &keep) const;
    // The same shear for the observation names of a table (`obs` maps a name
    // to its row): kept tips are tagged with their row.  *n_rows_matched, when
    // given, receives how many distinct rows some tip carries.
    BPTree shear_to(const NameMap &obs, uint32_t n_obs, uint32_t *n_rows_matched) const;
    // Tips against a table's names (obs: name -> row).
    TipMatch match_tips(const NameMap &obs, uint32_t n_obs) const;
    // shear_to with the tips already matched; `m` must not be all_tips.
    BPTree shear_matched(const TipMatch &m) const;
    // Remove non-root nodes with a single child, adding their length to the
    // child, in preorder (src/tree.cpp:165-191).  `tags` (default: the
    // tree's own) are carried to the result.
    BPTree collapse(const std::vector<int32_t> *tags = nullptr) const;
    // Whether collapse() would change the tree.
    bool has_single_child() const;
    // The parentheses flagged in `keep`, with `lengths` (and `tags`, or this
    // tree's own tags) carried along.
    BPTree masked(const std::vector<uint8_t> &keep, const std::vector<double> &lengths,
                  const std::vector<int32_t> *tags = nullptr) const;

    NameSet tip_names() const;
    uint32_t n_tips() const;
};

// The sheared tree flattened for the device.  Non-root nodes are numbered by
// rows: the embedded nodes (postorder, minus tips when bypass_tips) take rows
// [0, n_embedded), bypassed tips follow.  Children of a row are listed left
// to right, the order the reference sums them in (src/unifrac_internal.cpp:249-257).
struct FlatTree {
    uint32_t n_nodes = 0;      // non-root nodes
    uint32_t n_embedded = 0;   // rows that enter the pair sums
    std::vector<double> length;        // per row
    std::vector<int32_t> leaf_obs;     // per row: table row of a tip, -1 for internal nodes
    std::vector<uint32_t> child_ptr;   // per row, CSR into child_rows
    std::vector<uint32_t> child_rows;
    std::vector<uint32_t> leaf_rows;   // rows of tips
    std::vector<uint32_t> level_ptr;   // internal rows grouped by height (1, 2, ...)
    std::vector<uint32_t> level_rows;
    std::vector<uint32_t> postorder_row;  // postorder index -> row
};

FlatTree flatten(const BPTree &tree, const NameIndex &obs_index, bool bypass_tips);
// Flatten a tree whose tips carry table rows in `tag` (from shear_to), or in
// `tags` when given.  `single_child`, when given, reports whether some
// non-root node has a single child (the tree is then not collapsed: the
// caller collapses and flattens again).
FlatTree flatten(const BPTree &tree, bool bypass_tips, const std::vector<int32_t> *tags = nullptr,
                 bool *single_child = nullptr);

// Embedded node count of the tree sheared to the observations o with
// obs_row[o] >= 0 and then collapsed, computed on a flattened tree of a
// superset of those observations: kept tips (unless bypassed) plus the
// non-root internal nodes with at least two kept children.  With `active`,
// also which embedded rows of `tree` carry length into that table's sums:
// rows above at least one kept tip, or at least two with bypassed tips
// (a chain above a single tip merges into the tip).
uint32_t table_embedded(const FlatTree &tree, const std::vector<int32_t> &obs_row, bool bypass_tips,
                        std::vector<uint8_t> *active);

}  // namespace ssu
