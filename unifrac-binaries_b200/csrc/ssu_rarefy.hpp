// Rarefied replicates of one table drawn on the device (ssu_rarefy.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "ssu_table.hpp"

namespace ssu {

// `n_reps` replicates of `table` (totals computed): samples with a total
// below `depth` dropped, each kept sample reduced to `depth` counts drawn
// without or with replacement, observations left without counts dropped.
// Replicate r's draws depend only on seed + r and the sample, not on how many
// replicates are drawn together (replicate r of seed s equals replicate 0 of
// seed s + r).  The tables own their arrays; their id views
// point into `table`'s ids.  Returns 0, or output_error (6) with `err` set.
int rarefy_on_device(const Table &table, uint32_t depth, bool with_replacement, uint64_t seed, uint32_t n_reps,
                     std::vector<Table> &out, std::string &err);

}  // namespace ssu
