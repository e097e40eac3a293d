#include "ssu_grouping.hpp"

#include <fstream>
#include <iterator>
#include <string_view>
#include <unordered_map>

namespace ssu {
namespace {

std::vector<std::string_view> split_tabs(std::string_view line) {
    std::vector<std::string_view> out;
    size_t p = 0;
    while (true) {
        const size_t t = line.find('\t', p);
        if (t == std::string_view::npos) {
            out.push_back(line.substr(p));
            return out;
        }
        out.push_back(line.substr(p, t - p));
        p = t + 1;
    }
}

}  // namespace

bool read_grouping_tsv(const std::string &path, const std::string &column, uint32_t n, const char *const *ids,
                       std::vector<uint32_t> &grouping, uint32_t &n_groups, std::string &err) {
    std::ifstream in(path, std::ios::binary);
    if (!in) {
        err = "cannot open grouping file " + path;
        return false;
    }
    const std::string text((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    const std::string_view all(text);
    std::unordered_map<std::string_view, uint32_t> index;
    for (uint32_t i = 0; i < n; i++) index.emplace(ids[i], i);

    size_t pos = 0;
    auto next_line = [&](std::string_view &line) {
        if (pos >= all.size()) return false;
        const size_t e = all.find('\n', pos);
        line = all.substr(pos, (e == std::string_view::npos ? all.size() : e) - pos);
        pos = e == std::string_view::npos ? all.size() : e + 1;
        return true;
    };
    std::string_view line;
    if (!next_line(line)) {
        err = "grouping file " + path + " is empty";
        return false;
    }
    const std::vector<std::string_view> header = split_tabs(line);
    size_t col = 0;
    for (size_t i = 1; i < header.size() && !col; i++)
        if (header[i] == column) col = i;
    if (!col) {
        err = "column " + column + " not found in " + path;
        return false;
    }
    const uint32_t unset = ~0u;
    grouping.assign(n, unset);
    std::unordered_map<std::string_view, uint32_t> groups;
    while (next_line(line)) {
        const std::vector<std::string_view> row = split_tabs(line);
        auto it = index.find(row[0]);
        if (it == index.end()) continue;
        if (row.size() <= col) {
            err = "sample " + std::string(row[0]) + " has no " + column + " field";
            return false;
        }
        auto g = groups.emplace(row[col], static_cast<uint32_t>(groups.size())).first;
        grouping[it->second] = g->second;
    }
    for (uint32_t i = 0; i < n; i++)
        if (grouping[i] == unset) {
            err = std::string("sample ") + ids[i] + " not found in " + path;
            return false;
        }
    n_groups = static_cast<uint32_t>(groups.size());
    return true;
}

}  // namespace ssu
