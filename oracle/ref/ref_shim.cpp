/*
 * Test infrastructure only (the oracle), never linked into the product.
 *
 * The reference's build turns every `static inline ... _T(` template of
 * src/unifrac_task_impl.hpp and src/unifrac_accapi_impl.hpp into concrete
 * `su_cpu::` functions with a Python code generator
 * (src/generate_unifrac_task_noclass.py, src/generate_unifrac_accapi.py,
 * src/ssu_generate_helper.py:128-241).  This file is a hand-written
 * stand-in for those two generated files: it defines the same `su_cpu::`
 * symbols declared in src/unifrac_task_noclass.hpp:33-206 and
 * src/unifrac_accapi.hpp:29-58 by forwarding to the reference templates, for
 * the CPU backend only (no OpenACC / OpenMP-offload).
 */
#include "unifrac_task_noclass.hpp"
#include "unifrac_task_impl.hpp"
#include "unifrac_accapi_impl.hpp"

namespace su_cpu {

bool acc_found_gpu() { return acc_found_gpu_T(); }
bool acc_need_alt() { return acc_need_alt_T(); }
void acc_wait() { acc_wait_T(); }

template <class T> void acc_create_buf(T *buf, uint64_t s, uint64_t e) { acc_create_buf_T(buf, s, e); }
template <class T> void acc_copyin_buf(T *buf, uint64_t s, uint64_t e) { acc_copyin_buf_T(buf, s, e); }
template <class T> void acc_update_device(T *buf, uint64_t s, uint64_t e) { acc_update_device_T(buf, s, e); }
template <class T> void acc_copyout_buf(T *buf, uint64_t s, uint64_t e) { acc_copyout_buf_T(buf, s, e); }
template <class T> void acc_destroy_buf(T *buf, uint64_t s, uint64_t e) { acc_destroy_buf_T(buf, s, e); }

#define SSU_ORACLE_ACC(T)                                         \
    template void acc_create_buf<T>(T *, uint64_t, uint64_t);     \
    template void acc_copyin_buf<T>(T *, uint64_t, uint64_t);     \
    template void acc_update_device<T>(T *, uint64_t, uint64_t);  \
    template void acc_copyout_buf<T>(T *, uint64_t, uint64_t);    \
    template void acc_destroy_buf<T>(T *, uint64_t, uint64_t);
SSU_ORACLE_ACC(float)
SSU_ORACLE_ACC(double)
SSU_ORACLE_ACC(uint64_t)
SSU_ORACLE_ACC(uint32_t)
SSU_ORACLE_ACC(bool)
#undef SSU_ORACLE_ACC

template <class TFloat>
void compute_stripes_totals(TFloat *const __restrict__ a, const TFloat *const __restrict__ b, const uint64_t n) {
    compute_stripes_totals_T(a, b, n);
}

template <class TFloat>
void run_UnnormalizedWeightedTask(const uint64_t es, const unsigned int fe, const uint64_t s0, const uint64_t s1,
                                  const uint64_t n, const uint64_t nr, const TFloat *const __restrict__ len,
                                  const TFloat *const __restrict__ emb, TFloat *const __restrict__ dm,
                                  bool *const __restrict__ z, TFloat *const __restrict__ sums) {
    run_UnnormalizedWeightedTask_T(es, fe, s0, s1, n, nr, len, emb, dm, z, sums);
}

template <class TFloat>
void run_NormalizedWeightedTask(const uint64_t es, const unsigned int fe, const uint64_t s0, const uint64_t s1,
                                const uint64_t n, const uint64_t nr, const TFloat *const __restrict__ len,
                                const TFloat *const __restrict__ emb, TFloat *const __restrict__ dm,
                                TFloat *const __restrict__ dmt, bool *const __restrict__ z,
                                TFloat *const __restrict__ sums) {
    run_NormalizedWeightedTask_T(es, fe, s0, s1, n, nr, len, emb, dm, dmt, z, sums);
}

template <class TFloat>
void run_UnweightedTask(const uint64_t es, const unsigned int fe, const uint64_t s0, const uint64_t s1,
                        const uint64_t n, const uint64_t nr, const TFloat *const __restrict__ len,
                        const uint64_t *const __restrict__ emb, TFloat *const __restrict__ dm,
                        TFloat *const __restrict__ dmt, TFloat *const __restrict__ sums,
                        bool *const __restrict__ z, uint32_t *const __restrict__ idxs,
                        TFloat *const __restrict__ ss) {
    run_UnweightedTask_T(es, fe, s0, s1, n, nr, len, emb, dm, dmt, sums, z, idxs, ss);
}

template <class TFloat>
void run_UnnormalizedUnweightedTask(const uint64_t es, const unsigned int fe, const uint64_t s0, const uint64_t s1,
                                    const uint64_t n, const uint64_t nr, const TFloat *const __restrict__ len,
                                    const uint64_t *const __restrict__ emb, TFloat *const __restrict__ dm,
                                    TFloat *const __restrict__ sums, bool *const __restrict__ z,
                                    uint32_t *const __restrict__ idxs, TFloat *const __restrict__ ss) {
    run_UnnormalizedUnweightedTask_T(es, fe, s0, s1, n, nr, len, emb, dm, sums, z, idxs, ss);
}

template <class TFloat>
void run_GeneralizedTask(const uint64_t es, const unsigned int fe, const uint64_t s0, const uint64_t s1,
                         const uint64_t n, const uint64_t nr, const TFloat *const __restrict__ len,
                         const TFloat *const __restrict__ emb, TFloat *const __restrict__ dm,
                         TFloat *const __restrict__ dmt, const TFloat alpha) {
    run_GeneralizedTask_T(es, fe, s0, s1, n, nr, len, emb, dm, dmt, alpha);
}

template <class TFloat>
void run_VawUnnormalizedWeightedTask(const unsigned int fe, const uint64_t s0, const uint64_t s1, const uint64_t n,
                                     const uint64_t nr, const TFloat *const __restrict__ len,
                                     const TFloat *const __restrict__ emb, const TFloat *const __restrict__ cnt,
                                     const TFloat *const __restrict__ tot, TFloat *const __restrict__ dm) {
    run_VawUnnormalizedWeightedTask_T(fe, s0, s1, n, nr, len, emb, cnt, tot, dm);
}

template <class TFloat>
void run_VawNormalizedWeightedTask(const unsigned int fe, const uint64_t s0, const uint64_t s1, const uint64_t n,
                                   const uint64_t nr, const TFloat *const __restrict__ len,
                                   const TFloat *const __restrict__ emb, const TFloat *const __restrict__ cnt,
                                   const TFloat *const __restrict__ tot, TFloat *const __restrict__ dm,
                                   TFloat *const __restrict__ dmt) {
    run_VawNormalizedWeightedTask_T(fe, s0, s1, n, nr, len, emb, cnt, tot, dm, dmt);
}

template <class TFloat>
void run_VawUnweightedTask(const unsigned int fe, const uint64_t s0, const uint64_t s1, const uint64_t n,
                           const uint64_t nr, const TFloat *const __restrict__ len,
                           const uint32_t *const __restrict__ emb, const TFloat *const __restrict__ cnt,
                           const TFloat *const __restrict__ tot, TFloat *const __restrict__ dm,
                           TFloat *const __restrict__ dmt) {
    run_VawUnweightedTask_T(fe, s0, s1, n, nr, len, emb, cnt, tot, dm, dmt);
}

template <class TFloat>
void run_VawUnnormalizedUnweightedTask(const unsigned int fe, const uint64_t s0, const uint64_t s1, const uint64_t n,
                                       const uint64_t nr, const TFloat *const __restrict__ len,
                                       const uint32_t *const __restrict__ emb, const TFloat *const __restrict__ cnt,
                                       const TFloat *const __restrict__ tot, TFloat *const __restrict__ dm) {
    run_VawUnnormalizedUnweightedTask_T(fe, s0, s1, n, nr, len, emb, cnt, tot, dm);
}

template <class TFloat>
void run_VawGeneralizedTask(const unsigned int fe, const uint64_t s0, const uint64_t s1, const uint64_t n,
                            const uint64_t nr, const TFloat *const __restrict__ len,
                            const TFloat *const __restrict__ emb, const TFloat *const __restrict__ cnt,
                            const TFloat *const __restrict__ tot, TFloat *const __restrict__ dm,
                            TFloat *const __restrict__ dmt, const TFloat alpha) {
    run_VawGeneralizedTask_T(fe, s0, s1, n, nr, len, emb, cnt, tot, dm, dmt, alpha);
}

#define SSU_ORACLE_TASKS(T)                                                                                         \
    template void compute_stripes_totals<T>(T *const, const T *const, const uint64_t);                              \
    template void run_UnnormalizedWeightedTask<T>(const uint64_t, const unsigned int, const uint64_t,               \
                                                  const uint64_t, const uint64_t, const uint64_t, const T *const,    \
                                                  const T *const, T *const, bool *const, T *const);                  \
    template void run_NormalizedWeightedTask<T>(const uint64_t, const unsigned int, const uint64_t, const uint64_t, \
                                                const uint64_t, const uint64_t, const T *const, const T *const,      \
                                                T *const, T *const, bool *const, T *const);                          \
    template void run_UnweightedTask<T>(const uint64_t, const unsigned int, const uint64_t, const uint64_t,         \
                                        const uint64_t, const uint64_t, const T *const, const uint64_t *const,       \
                                        T *const, T *const, T *const, bool *const, uint32_t *const, T *const);       \
    template void run_UnnormalizedUnweightedTask<T>(const uint64_t, const unsigned int, const uint64_t,             \
                                                    const uint64_t, const uint64_t, const uint64_t, const T *const,  \
                                                    const uint64_t *const, T *const, T *const, bool *const,          \
                                                    uint32_t *const, T *const);                                      \
    template void run_GeneralizedTask<T>(const uint64_t, const unsigned int, const uint64_t, const uint64_t,        \
                                         const uint64_t, const uint64_t, const T *const, const T *const, T *const,   \
                                         T *const, const T);                                                         \
    template void run_VawUnnormalizedWeightedTask<T>(const unsigned int, const uint64_t, const uint64_t,            \
                                                     const uint64_t, const uint64_t, const T *const, const T *const, \
                                                     const T *const, const T *const, T *const);                      \
    template void run_VawNormalizedWeightedTask<T>(const unsigned int, const uint64_t, const uint64_t,              \
                                                   const uint64_t, const uint64_t, const T *const, const T *const,   \
                                                   const T *const, const T *const, T *const, T *const);              \
    template void run_VawUnweightedTask<T>(const unsigned int, const uint64_t, const uint64_t, const uint64_t,      \
                                           const uint64_t, const T *const, const uint32_t *const, const T *const,    \
                                           const T *const, T *const, T *const);                                      \
    template void run_VawUnnormalizedUnweightedTask<T>(const unsigned int, const uint64_t, const uint64_t,          \
                                                       const uint64_t, const uint64_t, const T *const,               \
                                                       const uint32_t *const, const T *const, const T *const,        \
                                                       T *const);                                                    \
    template void run_VawGeneralizedTask<T>(const unsigned int, const uint64_t, const uint64_t, const uint64_t,     \
                                            const uint64_t, const T *const, const T *const, const T *const,          \
                                            const T *const, T *const, T *const, const T);
SSU_ORACLE_TASKS(float)
SSU_ORACLE_TASKS(double)
#undef SSU_ORACLE_TASKS

}  // namespace su_cpu
