// Rarefied replicates of one table drawn on the device.
//
// The reference subsamples on the host, one OpenMP task per observation over
// a transposed copy of the table (src/biom_subsampled.cpp:155-353): samples
// whose total is below the depth are dropped, every kept sample is reduced
// to `depth` counts drawn without replacement (std::sample over the expanded
// count units, counts truncated to integers) or with replacement
// (std::discrete_distribution over the counts as weights), and observations
// left without counts are dropped.  Its random stream depends on libstdc++
// and the thread count, so it cannot be reproduced; this kernel draws the
// same distributions from a counter-based generator, so each (replicate,
// sample) draw is independent of launch shape and reproducible for a seed.
//
// One thread per (replicate, kept sample):
//  * without replacement: selection sampling over the sample's count units
//    in observation order - each unit is taken with probability
//    needed / remaining (Knuth, TAOCP vol. 2, 3.4.2, Algorithm S), which
//    gives every subset of `depth` units the same probability; a sample with
//    fewer integer units than `depth` keeps them all, as std::sample does;
//  * with replacement: `depth` uniform draws on [0, total) mapped to an
//    observation by binary search over the sample's prefix sums of weights.
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel
// random numbers: as easy as 1, 2, 3", SC'11), key = seed + replicate,
// counter = (sample, block index), so replicate r of seed s is replicate 0
// of seed s + r.
#include <algorithm>
#include <cstring>
#include <system_error>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "ssu_rarefy.hpp"

namespace ssu {
namespace {

struct Philox {
    uint32_t k0, k1;
    __device__ __forceinline__ uint4 operator()(uint4 c) const {
        uint32_t a = k0, b = k1;
#pragma unroll
        for (int r = 0; r < 10; r++) {
            const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
            const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
            c = make_uint4(hi1 ^ c.y ^ a, lo1, hi0 ^ c.w ^ b, lo0);
            a += 0x9E3779B9u;
            b += 0xBB67AE85u;
        }
        return c;
    }
};

// 32-bit random words of one (sample, replicate) stream, four per Philox call.
struct Stream {
    Philox ph;
    uint4 ctr;
    uint4 buf;
    int left = 0;
    __device__ __forceinline__ uint32_t next() {
        if (left == 0) {
            buf = ph(ctr);
            ctr.z++;
            if (ctr.z == 0) ctr.w++;
            left = 4;
        }
        const uint32_t v = left == 4 ? buf.x : left == 3 ? buf.y : left == 2 ? buf.z : buf.w;
        left--;
        return v;
    }
    // uniform double on [0, 1) with 53 random bits
    __device__ __forceinline__ double uniform() {
        const uint64_t hi = next() >> 5, lo = next() >> 6;
        return static_cast<double>((hi << 26) | lo) * (1.0 / 9007199254740992.0);
    }
};

// col_ptr[jj]..col_ptr[jj+1]: kept sample jj's entries, in observation order;
// col_pos: each entry's position in the (kept-sample) observation-major CSR;
// col_val: its count (weight); col_cum: inclusive prefix sums of the weights.
struct RarefyArgs {
    const uint32_t *col_ptr;
    const uint32_t *col_pos;
    const double *col_val;
    const double *col_cum;
    uint32_t n_kept;
    uint32_t rep0;    // first replicate of this launch
    uint32_t n_reps;  // replicates in this launch
    uint32_t depth;
    uint64_t seed;
    uint64_t nnz;     // entries per replicate (the output's row length)
    int with_replacement;
    uint32_t *out;    // [n_reps][nnz] counts
};

__global__ void rarefy_kernel(const RarefyArgs a) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<uint64_t>(a.n_reps) * a.n_kept) return;
    const uint32_t r = static_cast<uint32_t>(t / a.n_kept), jj = static_cast<uint32_t>(t % a.n_kept);
    const uint32_t rep = a.rep0 + r;
    // replicate r of seed s draws from key s + r: the same stream as
    // replicate 0 of seed s + r
    const uint64_t key = a.seed + rep;
    Stream rs;
    rs.ph = Philox{static_cast<uint32_t>(key), static_cast<uint32_t>(key >> 32)};
    rs.ctr = make_uint4(jj, 0u, 0u, 0u);
    uint32_t *out = a.out + static_cast<uint64_t>(r) * a.nnz;
    const uint32_t e0 = a.col_ptr[jj], e1 = a.col_ptr[jj + 1];
    if (!a.with_replacement) {
        uint64_t remaining = 0;
        for (uint32_t e = e0; e < e1; e++) remaining += static_cast<uint64_t>(a.col_val[e]);
        uint64_t needed = a.depth;
        for (uint32_t e = e0; e < e1; e++) {
            const uint64_t c = static_cast<uint64_t>(a.col_val[e]);
            uint32_t x = 0;
            if (needed >= remaining) {
                x = static_cast<uint32_t>(c);  // every unit left is taken
                needed -= c;
            } else if (needed > 0) {
                for (uint64_t u = 0; u < c && needed > 0; u++) {
                    // take this unit with probability needed / (remaining - u)
                    const uint64_t left = remaining - u;
                    const bool take = left < (uint64_t(1) << 32)
                                          ? static_cast<uint64_t>(rs.next()) * left < (needed << 32)
                                          : rs.uniform() * static_cast<double>(left) < static_cast<double>(needed);
                    if (take) {
                        x++;
                        needed--;
                    }
                }
            }
            remaining -= c;
            out[a.col_pos[e]] = x;
        }
    } else {
        for (uint32_t e = e0; e < e1; e++) out[a.col_pos[e]] = 0;
        const double total = e1 > e0 ? a.col_cum[e1 - 1] : 0.0;
        if (!(total > 0.0)) return;
        for (uint32_t d = 0; d < a.depth; d++) {
            const double u = rs.uniform() * total;
            // first entry whose inclusive prefix sum exceeds u
            uint32_t lo = e0, hi = e1 - 1;
            while (lo < hi) {
                const uint32_t mid = (lo + hi) / 2;
                if (a.col_cum[mid] > u)
                    hi = mid;
                else
                    lo = mid + 1;
            }
            out[a.col_pos[lo]]++;
        }
    }
}

#define RF_CK(call)                                            \
    do {                                                       \
        const cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) {                               \
            err = std::string(#call) + ": " + cudaGetErrorString(e_); \
            return 6;                                          \
        }                                                      \
    } while (0)

}  // namespace

int rarefy_on_device(const Table &table, uint32_t depth, bool with_replacement, uint64_t seed, uint32_t n_reps,
                     std::vector<Table> &out, std::string &err) {
    out.clear();
    out.resize(n_reps);
    // kept samples and the kept-sample observation-major CSR (positions)
    std::vector<uint32_t> keep, new_idx(table.n_samples, UINT32_MAX);
    for (uint32_t j = 0; j < table.n_samples; j++)
        if (table.totals[j] >= depth) {
            new_idx[j] = static_cast<uint32_t>(keep.size());
            keep.push_back(j);
        }
    const uint32_t n_kept = static_cast<uint32_t>(keep.size());
    std::vector<uint32_t> row_ptr(table.n_obs + 1, 0), row_col;
    std::vector<double> row_val;
    for (uint32_t i = 0; i < table.n_obs; i++) {
        for (uint32_t q = table.indptr[i]; q < table.indptr[i + 1]; q++)
            if (new_idx[table.indices[q]] != UINT32_MAX) {
                row_col.push_back(new_idx[table.indices[q]]);
                row_val.push_back(table.data[q]);
            }
        row_ptr[i + 1] = static_cast<uint32_t>(row_col.size());
    }
    const uint64_t nnz = row_col.size();
    if (n_kept == 0 || nnz == 0) {
        for (Table &t : out) t.adopt();
        return 0;
    }
    // sample-major view: per kept sample its entries in observation order
    std::vector<uint32_t> col_ptr(n_kept + 1, 0), col_pos(nnz);
    std::vector<double> col_val(nnz), col_cum(nnz);
    for (uint64_t q = 0; q < nnz; q++) col_ptr[row_col[q] + 1]++;
    for (uint32_t jj = 0; jj < n_kept; jj++) col_ptr[jj + 1] += col_ptr[jj];
    {
        std::vector<uint32_t> fill(col_ptr.begin(), col_ptr.end() - 1);
        for (uint32_t i = 0; i < table.n_obs; i++)
            for (uint32_t q = row_ptr[i]; q < row_ptr[i + 1]; q++) {
                const uint32_t e = fill[row_col[q]]++;
                col_pos[e] = q;
                col_val[e] = row_val[q] > 0.0 ? row_val[q] : 0.0;
            }
        for (uint32_t jj = 0; jj < n_kept; jj++) {
            double s = 0.0;
            for (uint32_t e = col_ptr[jj]; e < col_ptr[jj + 1]; e++) col_cum[e] = (s += col_val[e]);
        }
    }
    cudaStream_t st = nullptr;
    RF_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct Guard {
        cudaStream_t s;
        std::vector<void *> p;
        ~Guard() {
            for (void *q : p) cudaFreeAsync(q, s);
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    } g{st, {}};
    auto dalloc = [&](void **p, size_t bytes) {
        const cudaError_t e = cudaMallocAsync(p, std::max<size_t>(bytes, 16), st);
        if (e == cudaSuccess) g.p.push_back(*p);
        return e;
    };
    uint32_t *d_ptr = nullptr, *d_pos = nullptr, *d_out = nullptr;
    double *d_val = nullptr, *d_cum = nullptr;
    RF_CK(dalloc(reinterpret_cast<void **>(&d_ptr), sizeof(uint32_t) * col_ptr.size()));
    RF_CK(dalloc(reinterpret_cast<void **>(&d_pos), sizeof(uint32_t) * nnz));
    RF_CK(dalloc(reinterpret_cast<void **>(&d_val), sizeof(double) * nnz));
    RF_CK(dalloc(reinterpret_cast<void **>(&d_cum), sizeof(double) * nnz));
    RF_CK(cudaMemcpyAsync(d_ptr, col_ptr.data(), sizeof(uint32_t) * col_ptr.size(), cudaMemcpyHostToDevice, st));
    RF_CK(cudaMemcpyAsync(d_pos, col_pos.data(), sizeof(uint32_t) * nnz, cudaMemcpyHostToDevice, st));
    RF_CK(cudaMemcpyAsync(d_val, col_val.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
    RF_CK(cudaMemcpyAsync(d_cum, col_cum.data(), sizeof(double) * nnz, cudaMemcpyHostToDevice, st));
    // replicates in launches whose counts fit 1 GiB of device memory
    const uint32_t per_launch = static_cast<uint32_t>(
        std::max<uint64_t>(1, std::min<uint64_t>(n_reps, (uint64_t(1) << 30) / (sizeof(uint32_t) * nnz))));
    RF_CK(dalloc(reinterpret_cast<void **>(&d_out), sizeof(uint32_t) * nnz * per_launch));
    std::vector<uint32_t> counts(static_cast<size_t>(nnz) * per_launch);
    for (uint32_t r0 = 0; r0 < n_reps; r0 += per_launch) {
        const uint32_t nr = std::min(per_launch, n_reps - r0);
        RarefyArgs a{d_ptr, d_pos, d_val, d_cum, n_kept, r0, nr, depth, seed, nnz, with_replacement ? 1 : 0, d_out};
        const uint64_t threads = static_cast<uint64_t>(nr) * n_kept;
        rarefy_kernel<<<static_cast<uint32_t>((threads + 127) / 128), 128, 0, st>>>(a);
        RF_CK(cudaGetLastError());
        RF_CK(cudaMemcpyAsync(counts.data(), d_out, sizeof(uint32_t) * nnz * nr, cudaMemcpyDeviceToHost, st));
        RF_CK(cudaStreamSynchronize(st));
        // observation-major tables, observations without counts dropped
        auto build = [&](uint32_t rr) {
            const uint32_t *c = counts.data() + static_cast<uint64_t>(rr) * nnz;
            Table &t = out[r0 + rr];
            t.n_samples = n_kept;
            t.sample_ids.reserve(n_kept);
            for (uint32_t jj = 0; jj < n_kept; jj++) t.sample_ids.push_back(table.sample_ids[keep[jj]]);
            t.own_indptr.assign(1, 0);
            for (uint32_t i = 0; i < table.n_obs; i++) {
                const size_t before = t.own_indices.size();
                for (uint32_t q = row_ptr[i]; q < row_ptr[i + 1]; q++)
                    if (c[q]) {
                        t.own_indices.push_back(row_col[q]);
                        t.own_data.push_back(static_cast<double>(c[q]));
                    }
                if (t.own_indices.size() > before) {
                    t.obs_ids.push_back(table.obs_ids[i]);
                    t.own_indptr.push_back(static_cast<uint32_t>(t.own_indices.size()));
                }
            }
            t.n_obs = static_cast<uint32_t>(t.obs_ids.size());
            t.adopt();
            t.compute_totals();
        };
        const unsigned hw = std::max(1u, std::min<unsigned>(nr, std::min(16u, std::thread::hardware_concurrency())));
        std::vector<std::thread> pool;
        try {
            for (unsigned w = 1; w < hw; w++)
                pool.emplace_back([&, w] {
                    for (uint32_t rr = w; rr < nr; rr += hw) build(rr);
                });
        } catch (const std::system_error &) {
        }
        for (uint32_t rr = 0; rr < nr; rr += hw) build(rr);
        for (std::thread &th : pool) th.join();
        // a thread that could not be started leaves its replicates: build them here
        for (unsigned w = static_cast<unsigned>(pool.size()) + 1; w < hw; w++)
            for (uint32_t rr = w; rr < nr; rr += hw) build(rr);
    }
    return 0;
}

}  // namespace ssu
