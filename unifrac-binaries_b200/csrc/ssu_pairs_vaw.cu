// Variance-adjusted pair-kernel instances (src/unifrac_task_impl.hpp:435-502,
// 848-922, 1042-1119, 1755-1932).
#include "ssu_pairs.cuh"

namespace ssu {

namespace {
template <typename T, class Op>
std::vector<PairKernel<T>> family(const char *name) {
    return {values_kernel<T, Op, 128, 64, 8, 4, 16>(name, "128x64/8x4"),
            values_kernel<T, Op, 64, 64, 4, 4, 16>(name, "64x64/4x4")};
}
}  // namespace

template <typename T>
std::vector<PairKernel<T>> vaw_candidates(Method method, int ak) {
    switch (method) {
    case Method::unweighted: return family<T, dev::OpVawUnweighted<T, true>>("pair_values<vaw_unweighted>");
    case Method::unweighted_unnormalized:
        return family<T, dev::OpVawUnweighted<T, false>>("pair_values<vaw_unweighted_unnormalized>");
    case Method::weighted_normalized:
        return family<T, dev::OpVawWeighted<T, true>>("pair_values<vaw_weighted_normalized>");
    case Method::weighted_unnormalized:
        return family<T, dev::OpVawWeighted<T, false>>("pair_values<vaw_weighted_unnormalized>");
    case Method::generalized:
        switch (ak) {
        case 1: return family<T, dev::OpVawGeneralized<T, 1>>("pair_values<vaw_generalized>");
        case 2: return family<T, dev::OpVawGeneralized<T, 2>>("pair_values<vaw_generalized>");
        case 3: return family<T, dev::OpVawGeneralized<T, 3>>("pair_values<vaw_generalized>");
        default: return family<T, dev::OpVawGeneralized<T, 0>>("pair_values<vaw_generalized>");
        }
    }
    return {};
}

template std::vector<PairKernel<double>> vaw_candidates<double>(Method, int);
template std::vector<PairKernel<float>> vaw_candidates<float>(Method, int);

}  // namespace ssu
