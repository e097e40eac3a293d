// Grouping column of a sample-metadata TSV file, the input of PERMANOVA.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace ssu {

// The reference's indexed_tsv::read_grouping (src/tsv.cpp:118-180): the
// first line is the header, its first field the index column; `column` is
// looked up among the other header fields.  Every later line whose first
// field is one of `ids` gives that sample the group of its `column` field;
// groups are numbered 0, 1, ... in the order their values first appear
// (lines of other samples are skipped, a later line of the same sample
// overrides an earlier one).  Fields are tab-separated, lines end at '\n'.
// Fails (false, `err` set) when the file cannot be read, the column is not in
// the header, a matched line has no such field, or a sample has no line -
// the reference does not check the first sample; this checks all of them.
bool read_grouping_tsv(const std::string &path, const std::string &column, uint32_t n, const char *const *ids,
                       std::vector<uint32_t> &grouping, uint32_t &n_groups, std::string &err);

}  // namespace ssu
