// Weighted (normalized / unnormalized) pair-kernel instances
// (src/unifrac_task_impl.hpp:333-433, 743-846).
#include "ssu_pairs.cuh"

namespace ssu {

template <typename T>
std::vector<PairKernel<T>> weighted_candidates(bool normalized) {
    constexpr int KC = sizeof(T) == 8 ? 16 : 32;
    if (normalized)
        return {values_kernel<T, dev::OpWeighted<T, true>, 128, 128, 8, 8, KC>("pair_values<weighted_normalized>",
                                                                               "128x128/8x8"),
                values_kernel<T, dev::OpWeighted<T, true>, 128, 64, 8, 4, KC>("pair_values<weighted_normalized>",
                                                                              "128x64/8x4"),
                values_kernel<T, dev::OpWeighted<T, true>, 64, 64, 4, 4, KC>("pair_values<weighted_normalized>",
                                                                             "64x64/4x4")};
    return {values_kernel<T, dev::OpWeighted<T, false>, 128, 128, 8, 8, KC>("pair_values<weighted_unnormalized>",
                                                                            "128x128/8x8"),
            values_kernel<T, dev::OpWeighted<T, false>, 128, 64, 8, 4, KC>("pair_values<weighted_unnormalized>",
                                                                           "128x64/8x4"),
            values_kernel<T, dev::OpWeighted<T, false>, 64, 64, 4, 4, KC>("pair_values<weighted_unnormalized>",
                                                                          "64x64/4x4")};
}

template std::vector<PairKernel<double>> weighted_candidates<double>(bool);
template std::vector<PairKernel<float>> weighted_candidates<float>(bool);

}  // namespace ssu
