// Host-side phylogeny handling: BP trees, newick, shear, collapse, flatten.
#include "ssu_tree.hpp"

#include "ssu_host.hpp"

#include <algorithm>
#include <cstdlib>

namespace ssu {

void BPTree::pair_parentheses() {
    match.assign(open.size(), 0);
    std::vector<uint32_t> stack(open.size() + 1);
    size_t top = 0;
    malformed = open.size() % 2 != 0;
    for (uint32_t i = 0; i < open.size(); i++) {
        if (open[i]) {
            stack[top++] = i;
        } else if (top > 0) {
            const uint32_t o = stack[--top];
            match[o] = i;
            match[i] = o;
        } else {
            malformed = true;
        }
    }
    if (top != 0) malformed = true;
}

BPTree BPTree::from_arrays(const bool *structure, const double *lengths, const char *const *names, int n,
                           bool copy_names) {
    BPTree t;
    const uint32_t m = n > 0 ? static_cast<uint32_t>(n) : 0;
    t.open.resize(m);
    t.length.resize(m);
    t.name.resize(m);
    if (copy_names) t.storage = std::make_shared<std::deque<std::string>>();
    for (uint32_t i = 0; i < m; i++) {
        t.open[i] = structure[i] ? 1 : 0;
        t.length[i] = lengths[i];
        const char *nm = names[i] ? names[i] : "";
        if (copy_names) {
            t.storage->emplace_back(nm);
            t.name[i] = t.storage->back();
        } else {
            t.name[i] = nm;
        }
    }
    t.pair_parentheses();
    return t;
}

namespace {

// Rooted tree as child lists, the intermediate form of the newick parser.
struct ChildTree {
    std::vector<std::vector<uint32_t>> children;
    std::vector<double> length;
    std::vector<std::string> name;
    uint32_t add() {
        children.emplace_back();
        length.push_back(0.0);
        name.emplace_back();
        return static_cast<uint32_t>(children.size() - 1);
    }
};

BPTree serialise(const ChildTree &ct, uint32_t root) {
    BPTree t;
    t.storage = std::make_shared<std::deque<std::string>>(ct.name.begin(), ct.name.end());
    const std::deque<std::string> &names = *t.storage;
    const size_t n = 2 * ct.children.size();
    t.open.reserve(n);
    t.length.reserve(n);
    t.name.reserve(n);
    // explicit stack: (node, next child index)
    std::vector<std::pair<uint32_t, uint32_t>> stack;
    stack.emplace_back(root, 0);
    t.open.push_back(1);
    t.length.push_back(ct.length[root]);
    t.name.push_back(names[root]);
    while (!stack.empty()) {
        auto &top = stack.back();
        const auto &kids = ct.children[top.first];
        if (top.second < kids.size()) {
            uint32_t c = kids[top.second++];
            t.open.push_back(1);
            t.length.push_back(ct.length[c]);
            t.name.push_back(names[c]);
            stack.emplace_back(c, 0);
        } else {
            t.open.push_back(0);
            t.length.push_back(0.0);
            t.name.emplace_back("");  // a NUL-terminated empty name
            stack.pop_back();
        }
    }
    t.pair_parentheses();
    return t;
}

void apply_label(ChildTree &ct, uint32_t node, const std::string &label) {
    if (label.empty()) return;
    const size_t colon = label.find_last_of(':');
    if (colon == std::string::npos) {
        ct.name[node] = label;
        ct.length[node] = 0.0;
        return;
    }
    ct.name[node] = label.substr(0, colon);
    // single precision, as std::stof in the reference parser
    ct.length[node] = static_cast<double>(std::strtof(label.c_str() + colon + 1, nullptr));
}

}  // namespace

bool BPTree::from_newick(const std::string &text, BPTree &out) {
    size_t end = text.size();
    while (end > 0 && (text[end - 1] == ' ' || text[end - 1] == '\t' || text[end - 1] == '\n' ||
                       text[end - 1] == '\r'))
        end--;
    ChildTree ct;
    const uint32_t root = ct.add();
    std::vector<uint32_t> stack;
    uint32_t cur = root;
    std::string label;
    bool in_quote = false;
    for (size_t i = 0; i < end; i++) {
        const char c = text[i];
        if (c == '\n') continue;
        if (c == '\'') {
            in_quote = !in_quote;
            continue;
        }
        if (in_quote) {
            label.push_back(c);
            continue;
        }
        if (c == '(') {
            apply_label(ct, cur, label);
            label.clear();
            stack.push_back(cur);
            cur = ct.add();
            ct.children[stack.back()].push_back(cur);
        } else if (c == ',') {
            apply_label(ct, cur, label);
            label.clear();
            if (stack.empty()) return false;
            cur = ct.add();
            ct.children[stack.back()].push_back(cur);
        } else if (c == ')') {
            apply_label(ct, cur, label);
            label.clear();
            if (stack.empty()) return false;
            cur = stack.back();
            stack.pop_back();
        } else if (c == ';') {
            break;
        } else {
            label.push_back(c);
        }
    }
    apply_label(ct, cur, label);
    if (!stack.empty()) return false;
    out = serialise(ct, root);
    return true;
}

BPTree BPTree::masked(const std::vector<uint8_t> &keep, const std::vector<double> &lengths,
                      const std::vector<int32_t> *tags) const {
    BPTree r;
    r.storage = storage;
    size_t m = 0;
    for (uint8_t k : keep) m += k;
    r.open.reserve(m);
    r.length.reserve(m);
    r.name.reserve(m);
    const std::vector<int32_t> &tg = tags ? *tags : tag;
    const bool tagged = !tg.empty();
    r.open.resize(m);
    r.length.resize(m);
    r.name.resize(m);
    if (tagged) r.tag.resize(m);
    size_t j = 0;
    for (uint32_t i = 0; i < size(); i++) {
        if (!keep[i]) continue;
        r.open[j] = open[i];
        r.length[j] = lengths[i];
        r.name[j] = name[i];
        if (tagged) r.tag[j] = tg[i];
        j++;
    }
    r.pair_parentheses();
    return r;
}

TipMatch BPTree::match_tips(const NameMap &obs, uint32_t n_obs) const {
    TipMatch m;
    const uint32_t n = size();
    m.tags.assign(n, -1);
    m.tree_id = open.data();
    m.tree_size = n;
    // the lookups (read-only on the map, disjoint tags) on up to four host
    // threads for large trees, then the distinct rows counted in one pass
    const unsigned threads = n >= (1u << 16) ? host_threads(4) : 1u;
    const uint32_t span = (n + threads - 1) / threads;
    std::vector<uint8_t> missing(threads, 0);
    parallel_for(threads, threads, [&](unsigned p) {
        const uint32_t lo = p * span, hi = std::min(n ? n - 1 : 0, lo + span);
        bool miss = false;
        for (uint32_t i = lo; i < hi; i++) {
            if (!leaf(i)) continue;
            const int64_t row = obs.find(name[i]);
            if (row < 0)
                miss = true;
            else
                m.tags[i] = static_cast<int32_t>(row);
        }
        missing[p] = miss ? 1 : 0;
    });
    std::vector<uint8_t> seen(n_obs, 0);
    for (uint32_t i = 0; i + 1 < n; i++) {
        const int32_t row = m.tags[i];
        if (row >= 0 && !seen[row]) {
            seen[row] = 1;
            m.rows_matched++;
        }
    }
    m.all_tips = std::find(missing.begin(), missing.end(), 1) == missing.end();
    return m;
}

BPTree BPTree::shear_matched(const TipMatch &m) const {
    const uint32_t n = size();
    std::vector<uint8_t> mask(n, 0);
    std::vector<uint32_t> parent(n, UINT32_MAX);
    std::vector<uint32_t> stack;
    stack.reserve(64);
    for (uint32_t i = 0; i < n; i++) {
        if (open[i]) {
            parent[i] = stack.empty() ? UINT32_MAX : stack.back();
            stack.push_back(i);
        } else if (!stack.empty()) {
            stack.pop_back();
        }
    }
    for (uint32_t i = 0; i + 1 < n; i++) {
        if (m.tags[i] < 0) continue;
        mask[i] = mask[i + 1] = 1;
        for (uint32_t p = parent[i]; p != UINT32_MAX && !mask[p]; p = parent[p]) mask[p] = mask[match[p]] = 1;
    }
    return masked(mask, length, &m.tags);
}

bool BPTree::has_single_child() const {
    const uint32_t n = size();
    for (uint32_t cur = 1; cur < n; cur++) {
        if (!open[cur] || leaf(cur)) continue;
        if (cur + 1 == match[match[cur] - 1]) return true;  // first child is also the last
    }
    return false;
}

BPTree BPTree::shear_to(const NameMap &obs, uint32_t n_obs, uint32_t *n_rows_matched) const {
    const uint32_t n = size();
    std::vector<uint8_t> mask(n, 0);
    std::vector<uint32_t> parent(n, UINT32_MAX);
    std::vector<uint32_t> stack;
    for (uint32_t i = 0; i < n; i++) {
        if (open[i]) {
            parent[i] = stack.empty() ? UINT32_MAX : stack.back();
            stack.push_back(i);
        } else if (!stack.empty()) {
            stack.pop_back();
        }
    }
    std::vector<int32_t> tags(n, -1);
    std::vector<uint8_t> seen(n_obs, 0);
    uint32_t matched = 0;
    for (uint32_t i = 0; i + 1 < n; i++) {
        if (!leaf(i)) continue;
        const int64_t row = obs.find(name[i]);
        if (row < 0) continue;
        tags[i] = static_cast<int32_t>(row);
        if (!seen[row]) {
            seen[row] = 1;
            matched++;
        }
        mask[i] = mask[i + 1] = 1;
        for (uint32_t p = parent[i]; p != UINT32_MAX && !mask[p]; p = parent[p]) mask[p] = mask[match[p]] = 1;
    }
    if (n_rows_matched) *n_rows_matched = matched;
    return masked(mask, length, &tags);
}

BPTree BPTree::shear(const NameSet &keep) const {
    const uint32_t n = size();
    std::vector<uint8_t> mask(n, 0);
    std::vector<uint32_t> parent(n, UINT32_MAX);
    std::vector<uint32_t> stack;
    for (uint32_t i = 0; i < n; i++) {
        if (open[i]) {
            parent[i] = stack.empty() ? UINT32_MAX : stack.back();
            stack.push_back(i);
        } else if (!stack.empty()) {
            stack.pop_back();
        }
    }
    for (uint32_t i = 0; i + 1 < n; i++) {
        if (!leaf(i) || keep.count(name[i]) == 0) continue;
        mask[i] = mask[i + 1] = 1;
        for (uint32_t p = parent[i]; p != UINT32_MAX && !mask[p]; p = parent[p]) mask[p] = mask[match[p]] = 1;
    }
    return masked(mask, length);
}

BPTree BPTree::collapse(const std::vector<int32_t> *tags) const {
    const uint32_t n = size();
    std::vector<uint8_t> mask(n, 0);
    std::vector<double> len(length);
    for (uint32_t cur = 0; cur < n; cur++) {  // opening parentheses in index order = preorder
        if (!open[cur]) continue;
        if (leaf(cur) || cur == 0) {
            mask[cur] = mask[match[cur]] = 1;
            continue;
        }
        const uint32_t first = cur + 1;
        const uint32_t last = match[match[cur] - 1];
        if (first == last)
            len[first] = len[first] + len[cur];
        else
            mask[cur] = mask[match[cur]] = 1;
    }
    return masked(mask, len, tags);
}

NameSet BPTree::tip_names() const {
    NameSet out;
    out.reserve(size() / 2 + 1);
    for (uint32_t i = 0; i + 1 < size(); i++)
        if (leaf(i)) out.insert(name[i]);
    return out;
}

uint32_t BPTree::n_tips() const {
    uint32_t c = 0;
    for (uint32_t i = 0; i + 1 < size(); i++) c += leaf(i);
    return c;
}

namespace {

template <class ObsOf>
FlatTree flatten_impl(const BPTree &t, bool bypass_tips, ObsOf obs_of, bool *single_child) {
    FlatTree f;
    const uint32_t n = t.size();
    const uint32_t total = n / 2;
    f.n_nodes = total > 0 ? total - 1 : 0;
    const uint32_t N = f.n_nodes;
    if (single_child) *single_child = false;
    // Rows: the k-th closing parenthesis closes the k-th postorder node and
    // the root closes last, without a row (src/unifrac_cmp.cpp:97-100).
    // Embedded nodes take rows in postorder; with bypassed tips the tips
    // follow them, in postorder too.
    uint32_t n_leaves = 0;
    if (bypass_tips)
        for (uint32_t i = 0; i + 1 < n; i++) n_leaves += (t.open[i] && !t.open[i + 1]) ? 1u : 0u;
    f.n_embedded = bypass_tips ? N - std::min(N, n_leaves) : N;
    f.length.resize(N);
    f.leaf_obs.assign(N, -1);
    f.postorder_row.resize(N);
    f.child_ptr.assign(N + 1, 0);
    f.child_rows.reserve(N);
    f.leaf_rows.reserve(bypass_tips ? n_leaves : N / 2 + 1);
    std::vector<uint32_t> height(N, 0);

    // One walk over the parentheses: an open node keeps its opening index,
    // the tallest child seen + 1 and where its children start on `pend`,
    // the stack of rows whose parent has not closed yet (left to right).
    struct Open {
        uint32_t o, h, first;
    };
    std::vector<Open> stack;
    stack.reserve(64);
    std::vector<uint32_t> pend;
    pend.reserve(64);
    uint32_t k = 0, emb = 0, tip = 0, max_height = 0;
    for (uint32_t i = 0; i < n; i++) {
        if (t.open[i]) {
            stack.push_back({i, 0, static_cast<uint32_t>(pend.size())});
            continue;
        }
        if (stack.empty()) continue;
        const Open e = stack.back();
        stack.pop_back();
        if (stack.empty() || k >= N) break;  // the root
        const bool leaf = e.o + 1 == i;
        const uint32_t row = (bypass_tips && leaf) ? f.n_embedded + tip++ : emb++;
        f.postorder_row[k++] = row;
        f.length[row] = t.length[e.o];
        uint32_t h = 0;
        if (leaf) {
            f.leaf_rows.push_back(row);
            f.leaf_obs[row] = obs_of(e.o);
        } else {
            // internal rows are numbered in closing order, so their child
            // lists are appended in row order
            const uint32_t nk = static_cast<uint32_t>(pend.size()) - e.first;
            if (nk == 1 && single_child) *single_child = true;
            f.child_ptr[row] = static_cast<uint32_t>(f.child_rows.size());
            f.child_rows.insert(f.child_rows.end(), pend.begin() + e.first, pend.end());
            f.child_ptr[row + 1] = static_cast<uint32_t>(f.child_rows.size());
            h = e.h;
            height[row] = h;
            max_height = std::max(max_height, h);
        }
        pend.resize(e.first);
        pend.push_back(row);
        stack.back().h = std::max(stack.back().h, h + 1);
    }
    // rows without children (tips) point at the end of their predecessor's list
    for (uint32_t row = 0; row < N; row++)
        if (f.child_ptr[row + 1] < f.child_ptr[row]) f.child_ptr[row + 1] = f.child_ptr[row];
    // internal rows bucketed by height 1..max_height, rows ascending
    f.level_ptr.assign(max_height + 1, 0);
    for (uint32_t row = 0; row < N; row++)
        if (height[row] > 0) f.level_ptr[height[row]]++;
    for (uint32_t h = 1; h <= max_height; h++) f.level_ptr[h] += f.level_ptr[h - 1];
    f.level_rows.assign(f.level_ptr[max_height], 0);
    std::vector<uint32_t> fill(f.level_ptr.begin(), f.level_ptr.end());
    for (uint32_t row = 0; row < N; row++)
        if (height[row] > 0) f.level_rows[fill[height[row] - 1]++] = row;
    return f;
}

}  // namespace

FlatTree flatten(const BPTree &t, const NameIndex &obs_index, bool bypass_tips) {
    return flatten_impl(
        t, bypass_tips,
        [&](uint32_t o) -> int32_t {
            auto it = obs_index.find(t.name[o]);
            return it != obs_index.end() ? static_cast<int32_t>(it->second) : -1;
        },
        nullptr);
}

FlatTree flatten(const BPTree &t, bool bypass_tips, const std::vector<int32_t> *tags, bool *single_child) {
    const std::vector<int32_t> &tg = tags ? *tags : t.tag;
    return flatten_impl(t, bypass_tips, [&](uint32_t o) -> int32_t { return tg.empty() ? -1 : tg[o]; }, single_child);
}

uint32_t table_embedded(const FlatTree &f, const std::vector<int32_t> &obs_row, bool bypass_tips,
                        std::vector<uint8_t> *active) {
    std::vector<uint32_t> tips(f.n_nodes, 0);  // kept tips below each row
    uint32_t count = 0;
    if (active) active->assign(f.n_embedded, 0);
    for (uint32_t k = 0; k < f.n_nodes; k++) {
        const uint32_t row = f.postorder_row[k];
        if (f.child_ptr[row] == f.child_ptr[row + 1]) {
            const int32_t o = f.leaf_obs[row];
            const bool kept = o >= 0 && static_cast<size_t>(o) < obs_row.size() && obs_row[o] >= 0;
            tips[row] = kept ? 1 : 0;
            if (kept && !bypass_tips) count++;
            if (active && row < f.n_embedded) (*active)[row] = kept ? 1 : 0;
            continue;
        }
        uint32_t below = 0, kids = 0;
        for (uint32_t q = f.child_ptr[row]; q < f.child_ptr[row + 1]; q++) {
            const uint32_t c = f.child_rows[q];
            below += tips[c];
            kids += tips[c] > 0;
        }
        tips[row] = below;
        if (kids >= 2) count++;
        if (active && row < f.n_embedded) (*active)[row] = below >= (bypass_tips ? 2u : 1u);
    }
    return count;
}

}  // namespace ssu
