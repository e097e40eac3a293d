// Weighted UniFrac over a sparse embedding (sm_100a).
//
// Most embedded nodes are zero for most samples: with 1% of the features
// present per sample, a node is non-zero for ~5% of the samples on average.
// For a node with u = a in sample k and b in sample l,
//     |a - b| = a + b - 2 min(a, b),
// and min(a, b) = 0 unless both are non-zero.  So over a set S of "sparse"
// nodes
//     sum_S L |a - b| = Ws_k + Ws_l - 2 sum_{S, a>0, b>0} L min(a, b),
// Ws_j = sum_S L u(j) being one number per sample.  Nodes are split per call:
//   dense rows  (non-zero in more than an eighth of the columns): summed as
//               L |a - b| in registers, exactly as the dense pair kernel;
//   sparse rows (the rest, all-zero rows dropped): only the pairs where both
//               samples are non-zero are touched, -2 L min(a, b) accumulated
//               in an fp64 tile in shared memory.  fp64 plans: each warp owns
//               8 tile rows and walks every row, in order, one lane per element
//               (bit-reproducible).  fp32 plans: each row is handled by one
//               warp, which gathers only the present values and adds the
//               products with shared-memory atomics (13% faster on rarefied
//               replicate tables; the order of these additions, so the last bits of the
//               fp64 sums, can vary between runs).
// d = D + (M + Ws_k + Ws_l) subtracts; where d < tau (Ws_k + Ws_l) the
// rounding of that subtraction could reach 1e-13 relative, so the tile is
// flagged and recomputed exactly (all nodes, |a - b| form) by the dense pair
// kernel afterwards.
//
// Presence masks, word-major: bit i of masks[w * E + e] is U[e][64 w + i] > 0,
// so the masks of consecutive rows for one 64-column word are contiguous; the
// embedding kernels write them (and the per-row counts) as they fill U.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ssu_kernels.cuh"

namespace ssu {
namespace dev {

// Rows in order into dense (count > threshold) and sparse (0 < count <=
// threshold) lists, and each row's class (0 all zero, 1 sparse, 2 dense);
// one CTA of 1024 threads.  n_out = {dense, sparse}.
static __global__ void __launch_bounds__(1024) classify_rows_kernel(const uint32_t *__restrict__ counts, uint32_t E,
                                                                    uint32_t threshold, uint32_t *__restrict__ dense,
                                                                    uint32_t *__restrict__ sparse,
                                                                    uint8_t *__restrict__ row_class,
                                                                    uint32_t *__restrict__ n_out) {
    __shared__ uint32_t warp_base[32][2];
    __shared__ uint32_t run[2];
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (threadIdx.x < 2) run[threadIdx.x] = 0;
    __syncthreads();
    for (uint32_t c0 = 0; c0 < E; c0 += blockDim.x) {
        const uint32_t e = c0 + threadIdx.x;
        const uint32_t cnt = e < E ? counts[e] : 0;
        const bool is_dense = cnt > threshold;
        const bool is_sparse = cnt > 0 && !is_dense;
        if (e < E) row_class[e] = is_dense ? 2 : (is_sparse ? 1 : 0);
        const uint32_t bd = __ballot_sync(0xffffffffu, is_dense);
        const uint32_t bs = __ballot_sync(0xffffffffu, is_sparse);
        if (lane == 0) {
            warp_base[warp][0] = __popc(bd);
            warp_base[warp][1] = __popc(bs);
        }
        __syncthreads();
        if (threadIdx.x < 2) {
            uint32_t r = run[threadIdx.x];
            for (uint32_t w = 0; w < nw; w++) {
                const uint32_t t = warp_base[w][threadIdx.x];
                warp_base[w][threadIdx.x] = r;
                r += t;
            }
            run[threadIdx.x] = r;
        }
        __syncthreads();
        const uint32_t below = (1u << lane) - 1u;
        if (is_dense) dense[warp_base[warp][0] + __popc(bd & below)] = e;
        if (is_sparse) sparse[warp_base[warp][1] + __popc(bs & below)] = e;
        __syncthreads();
    }
    if (threadIdx.x < 2) n_out[threadIdx.x] = run[threadIdx.x];
}

// Ws[j] = sum over the sparse rows (in order, in fixed chunks) of L u[j],
// in fp64; partial sums per chunk, then reduce_partials_kernel<double>.
// (weighted unnormalized: no W is needed, so only the sparse rows are read)
template <typename T>
__global__ void sparse_sums_partial_kernel(const T *__restrict__ U, const T *__restrict__ len,
                                           const uint32_t *__restrict__ rows, const uint32_t *__restrict__ n_rows,
                                           uint64_t ld, uint32_t chunk, double *__restrict__ partial) {
    const uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= ld) return;
    const uint32_t n = n_rows[1];
    const uint32_t i0 = blockIdx.y * chunk;
    const uint32_t i1 = min(n, i0 + chunk);
    double s = 0.0;
    for (uint32_t i = i0; i < i1; i++) {
        const uint32_t e = rows[i];
        s = fma(static_cast<double>(U[static_cast<uint64_t>(e) * ld + j]), static_cast<double>(len[e]), s);
    }
    partial[static_cast<uint64_t>(blockIdx.y) * ld + j] = s;
}

// One pass over the embedding for both one-sided sums of the hybrid, per
// column j and chunk of `chunk` rows (weighted normalized): W[j] = sum of
// L u[j] over every row, in T as the dense kernels'
// weighted_sums_partial_kernel, and Ws[j] = the same over the sparse rows
// (row_class 1), in fp64; partial sums per chunk, then reduce_partials_kernel.
template <typename T>
__global__ void hybrid_sums_partial_kernel(const T *__restrict__ U, const T *__restrict__ len,
                                           const uint8_t *__restrict__ row_class, uint32_t E, uint64_t ld,
                                           uint32_t chunk, T *__restrict__ w_part, double *__restrict__ ws_part) {
    const uint64_t j = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= ld) return;
    const uint32_t e0 = blockIdx.y * chunk;
    const uint32_t e1 = min(E, e0 + chunk);
    T s = T(0);
    double ss = 0.0;
    for (uint32_t e = e0; e < e1; e++) {
        const T u = U[static_cast<uint64_t>(e) * ld + j];
        const T L = len[e];
        s = fma(u, L, s);
        if (row_class[e] == 1) ss = fma(static_cast<double>(u), static_cast<double>(L), ss);
    }
    w_part[static_cast<uint64_t>(blockIdx.y) * ld + j] = s;
    ws_part[static_cast<uint64_t>(blockIdx.y) * ld + j] = ss;
}

template <typename T>
struct HybridArgs {
    const uint4 *tiles;  // 128 x 128 tiles: x, y blocks of 128 columns, z table
    uint32_t n_tiles, n_splits;
    const TableDesc *tables;
    const T *U;
    const T *len;        // per embedded row
    const unsigned long long *masks;  // word-major, E rows per word
    const uint8_t *row_class;         // 0 zero, 1 sparse, 2 dense
    uint32_t E;          // embedded rows
    uint64_t ld;
    const uint32_t *dense_rows;
    const uint32_t *n_rows;  // {dense, sparse}
    const T *W;          // full one-sided sums (normalized)
    const double *Ws;    // one-sided sums over the sparse rows
    double tau;
    int *tile_flags;     // tiles that need the exact recomputation
    double *partial;     // per (split, tile) 128 x 128 fp64 raw sums; nullptr: no splits
    OutSpec out;
    // pair-scatter form: the sparse rows' sums S = sum L min(a, b) per pair
    // k < l of a table, 64-bit fixed point at td.out_off + k n + l (nullptr:
    // the tile kernel walks the sparse rows itself)
    const unsigned long long *Sq;
    double sq_unit;      // value of one fixed-point unit (2^-s)
};

constexpr int HB = 128;      // tile edge
constexpr int HKC = 8;       // rows per pipeline stage (warps 0..7 load one each)
constexpr int HSTAGES = 5;   // stages in the ring
constexpr int HTHREADS = 512;
constexpr int HWARPS = HTHREADS / 32;
constexpr int HROWS = HB / HWARPS;  // tile rows owned by a warp in the sparse phase
constexpr int HSLOTS = 4;           // active rows gathered together per warp

template <typename T>
constexpr size_t hybrid_smem() {
    return sizeof(double) * HB * HB + HSTAGES * (sizeof(T) * HKC * 2 * HB + sizeof(T) * HKC) + 64;
}

// Epilogue of one element: value from the raw sum x = D - 2 M.
template <typename T, bool NORM>
__device__ __forceinline__ void hybrid_emit(const HybridArgs<T> &a, const TableDesc &td, OutSpec o, uint32_t ti,
                                            uint32_t kc, uint32_t lc, double x) {
    const uint32_t k = kc - td.base, l = lc - td.base;
    if (!(k < l && l < td.n)) return;
    if (a.Sq)
        x -= 2.0 * static_cast<double>(static_cast<long long>(a.Sq[td.out_off + static_cast<uint64_t>(k) * td.n + l])) *
             a.sq_unit;
    const double ws = a.Ws[kc] + a.Ws[lc];
    const double d = x + ws;
    if (d < a.tau * ws) atomicOr(a.tile_flags + ti, 1);
    const T v = NORM ? static_cast<T>(d) / (a.W[kc] + a.W[lc]) : static_cast<T>(d);
    emit_pair<T>(o, td.n, k, l, v);
}

// ATOMIC: the sparse rows' updates go one warp per row with shared-memory
// atomics (default for fp32 plans); otherwise the owner-per-element walk
// (bit-reproducible; always for fp64 plans).
template <typename T, bool NORM, bool ATOMIC = (sizeof(T) == 4)>
__global__ void __launch_bounds__(HTHREADS, 1) pair_hybrid_kernel(const HybridArgs<T> a) {
    constexpr int TX = 16;         // dense phase: 16 (l) x 32 (k) threads, 4 x 8 pairs each
    constexpr int TM = 4, TN = 8;
    constexpr int VEC = 16 / sizeof(T);
    constexpr int CPR = 2 * HB / VEC;  // 16-byte pieces per staged row (k block then l block)
    constexpr int PPT = CPR / 32;      // pieces per thread: warp w loads row w of a chunk
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *Mt = reinterpret_cast<double *>(smem_raw);                                      // [128][128]
    T *Vs = reinterpret_cast<T *>(Mt + HB * HB);                                            // [S][HKC][256]
    T *Ls = Vs + HSTAGES * HKC * 2 * HB;                                                    // [S][HKC]

    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int lane = tid & 31, warp = tid >> 5;
    const uint32_t n_dense = a.n_rows[0];
    const uint32_t n_work = a.n_tiles * a.n_splits;
    for (uint32_t w = blockIdx.x; w < n_work; w += gridDim.x) {
        const uint32_t split = w / a.n_tiles, ti = w - split * a.n_tiles;
        const uint4 tile = a.tiles[ti];
        const uint32_t k0 = tile.x * HB, l0 = tile.y * HB;
        const uint32_t dr = (n_dense + a.n_splits - 1) / a.n_splits;
        const uint32_t d_begin = min(n_dense, split * dr), d_end = min(n_dense, d_begin + dr);

        // Data of row `warp` of a chunk, issued by that warp: both value
        // blocks (PPT 16-byte pieces per lane) and the length.  `e` is the row
        // id, `ok` whether it exists.
        auto load_row = [&](int st, uint32_t e, bool ok) {
            if (warp >= HKC) return;
            T *dst = Vs + (st * HKC + warp) * 2 * HB;
            const T *src = a.U + static_cast<uint64_t>(e) * a.ld;
#pragma unroll
            for (int m = 0; m < PPT; m++) {
                const int q = lane + 32 * m;
                const uint32_t col = q < CPR / 2 ? k0 + q * VEC : l0 + (q - CPR / 2) * VEC;
                cp_async16(dst + q * VEC, src + col, ok ? 16 : 0);
            }
            if (lane == 4) cp_async_small<sizeof(T)>(Ls + st * HKC + warp, a.len + e, ok ? (int)sizeof(T) : 0);
        };
        // Ring of HSTAGES chunks over rows [begin, end) of `rows`: chunk c is
        // issued HSTAGES - 1 iterations before it is consumed; each warp keeps
        // the row ids of its next two chunks in registers.
        auto stream_rows = [&](const uint32_t *rows, uint32_t begin, uint32_t end, auto consume) {
            const uint32_t n_chunks = end > begin ? (end - begin + HKC - 1) / HKC : 0;
            if (n_chunks == 0) return;
            auto id_of = [&](uint32_t chunk) -> uint32_t {
                const uint32_t i = begin + chunk * HKC + warp;
                return (warp < HKC && chunk < n_chunks && i < end) ? rows[i] : 0u;
            };
            auto ok_of = [&](uint32_t chunk) {
                return warp < HKC && chunk < n_chunks && begin + chunk * HKC + warp < end;
            };
            for (uint32_t c = 0; c + 1 < HSTAGES; c++) {
                if (c < n_chunks) load_row(static_cast<int>(c), id_of(c), ok_of(c));
                cp_async_commit();
            }
            uint32_t id1 = id_of(HSTAGES - 1), id2 = id_of(HSTAGES);
            for (uint32_t ch = 0; ch < n_chunks; ch++) {
                const uint32_t nxt = ch + HSTAGES - 1;
                if (nxt < n_chunks) load_row(static_cast<int>(nxt % HSTAGES), id1, ok_of(nxt));
                cp_async_commit();
                id1 = id2;
                id2 = id_of(ch + HSTAGES + 1);
                cp_async_wait<HSTAGES - 1>();
                __syncthreads();
                consume(static_cast<int>(ch % HSTAGES));
                __syncthreads();
            }
            cp_async_wait<0>();
        };

        // ---- dense rows: L |a - b| in registers, 4 x 8 pairs per thread
        double acc[TM][TN];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++) acc[i][j] = 0.0;
        stream_rows(a.dense_rows, d_begin, d_end, [&](int st) {
            const T *vs = Vs + st * HKC * 2 * HB;
            if constexpr (sizeof(T) == 4) {
                // single precision: each stage's 8 rows summed in fp32 (the
                // reference fp32 build's own arithmetic), then folded into the
                // fp64 totals, so no fp32 sum runs over more than 8 terms
                float part[TM][TN];
#pragma unroll
                for (int i = 0; i < TM; i++)
#pragma unroll
                    for (int j = 0; j < TN; j++) part[i][j] = 0.0f;
#pragma unroll 2
                for (int c = 0; c < HKC; c++) {
                    T av[TM], bv[TN];
                    load_half<T, TM / 2>(av, vs + c * 2 * HB + ty * (TM / 2));
                    load_half<T, TM / 2>(av + TM / 2, vs + c * 2 * HB + HB / 2 + ty * (TM / 2));
                    load_half<T, TN / 2>(bv, vs + c * 2 * HB + HB + tx * (TN / 2));
                    load_half<T, TN / 2>(bv + TN / 2, vs + c * 2 * HB + HB + HB / 2 + tx * (TN / 2));
                    const float L = static_cast<float>(Ls[st * HKC + c]);
#pragma unroll
                    for (int i = 0; i < TM; i++)
#pragma unroll
                        for (int j = 0; j < TN; j++) part[i][j] = fmaf(fabsf(av[i] - bv[j]), L, part[i][j]);
                }
#pragma unroll
                for (int i = 0; i < TM; i++)
#pragma unroll
                    for (int j = 0; j < TN; j++) acc[i][j] += static_cast<double>(part[i][j]);
            } else {
#pragma unroll 2
                for (int c = 0; c < HKC; c++) {
                    T av[TM], bv[TN];
                    load_half<T, TM / 2>(av, vs + c * 2 * HB + ty * (TM / 2));
                    load_half<T, TM / 2>(av + TM / 2, vs + c * 2 * HB + HB / 2 + ty * (TM / 2));
                    load_half<T, TN / 2>(bv, vs + c * 2 * HB + HB + tx * (TN / 2));
                    load_half<T, TN / 2>(bv + TN / 2, vs + c * 2 * HB + HB + HB / 2 + tx * (TN / 2));
                    const double L = static_cast<double>(Ls[st * HKC + c]);
#pragma unroll
                    for (int i = 0; i < TM; i++)
#pragma unroll
                        for (int j = 0; j < TN; j++)
                            acc[i][j] =
                                fma(fabs(static_cast<double>(av[i]) - static_cast<double>(bv[j])), L, acc[i][j]);
                }
            }
        });
        // the dense sums seed the shared tile
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++)
                Mt[tile_row<HB, TM>(ty, i) * HB + tile_row<HB, TN>(tx, j)] = acc[i][j];
        __syncthreads();

        if (a.Sq) {
            // ---- sparse rows: already scattered into Sq (sparse_pairs_kernel)
        } else if constexpr (ATOMIC) {
            // ---- sparse rows, fp32 plans: -2 L min(a, b) where both are non-zero.  Warp w
            // takes batches w, w + 16, ... of 32 consecutive rows (lane i: row i's
            // class, its k-block and l-block mask words and length, fetched two
            // batches ahead), so each row is handled once per tile.  For a row
            // with nk present k columns and nl present l columns, lanes gather
            // the present values (one lane per present column, HSLOTS rows at a
            // time so the loads overlap) and the nk x nl products are added into
            // the shared tile with shared-memory atomics (k by k, lanes over l).
            {
                const uint32_t er = (a.E + a.n_splits - 1) / a.n_splits;
                const uint32_t r_begin = min(a.E, split * er), r_end = min(a.E, r_begin + er);
                const uint32_t n_batches = r_end > r_begin ? (r_end - r_begin + 31) / 32 : 0;
                const uint64_t kwd = k0 / 64, lwd = l0 / 64;
                const unsigned long long *k0_base = a.masks + kwd * a.E;
                const unsigned long long *k1_base = a.masks + (kwd + 1) * a.E;
                const unsigned long long *l0_base = a.masks + lwd * a.E;
                const unsigned long long *l1_base = a.masks + (lwd + 1) * a.E;
                struct Fetch {
                    unsigned long long k0, k1, l0, l1;
                    double L;
                    bool ok;
                };
                auto fetch = [&](uint32_t batch) {
                    Fetch f{0ull, 0ull, 0ull, 0ull, 0.0, false};
                    const uint32_t e = r_begin + batch * 32 + lane;
                    if (batch < n_batches && e < r_end && a.row_class[e] == 1) {
                        f.k0 = k0_base[e];
                        f.k1 = k1_base[e];
                        f.l0 = l0_base[e];
                        f.l1 = l1_base[e];
                        f.L = static_cast<double>(a.len[e]);
                        f.ok = true;
                    }
                    return f;
                };
                // the col-th set bit (0-based) of the 128-bit word pair (w0, w1)
                auto nth_bit = [](unsigned long long w0, unsigned long long w1, int col) -> int {
                    const int c0 = __popcll(w0);
                    const unsigned long long w = col < c0 ? w0 : w1;
                    int r = col < c0 ? col : col - c0;
                    const uint32_t lo = static_cast<uint32_t>(w), hi = static_cast<uint32_t>(w >> 32);
                    const int pl = __popc(lo);
                    const int bit = r < pl ? static_cast<int>(__fns(lo, 0, r + 1))
                                           : 32 + static_cast<int>(__fns(hi, 0, r - pl + 1));
                    return (col < c0 ? 0 : 64) + bit;
                };
                uint32_t b = warp;
                Fetch cur = fetch(b), nxt = fetch(b + HWARPS);
                for (; b < n_batches; b += HWARPS) {
                    const Fetch after = fetch(b + 2 * HWARPS);
                    const uint32_t e_cur = r_begin + b * 32 + lane;
                    const int nk_l = __popcll(cur.k0) + __popcll(cur.k1);
                    const int nl_l = __popcll(cur.l0) + __popcll(cur.l1);
                    uint32_t active = __ballot_sync(0xffffffffu, cur.ok && nk_l > 0 && nl_l > 0);
                    // rows with more than 32 present k or l columns take the
                    // chunked path one at a time
                    uint32_t wide = __ballot_sync(0xffffffffu, cur.ok && nk_l > 0 && nl_l > 0 &&
                                                                  (nk_l > 32 || nl_l > 32));
                    uint32_t narrow = active & ~wide;
                    while (narrow) {
                        int src[HSLOTS];
                        int cnt = 0;
    #pragma unroll
                        for (int j = 0; j < HSLOTS; j++) {
                            src[j] = narrow ? __ffs(narrow) - 1 : 0;
                            cnt += narrow ? 1 : 0;
                            narrow &= narrow ? narrow - 1 : 0u;
                        }
                        double va[HSLOTS], vb[HSLOTS];
                        int kid[HSLOTS], lid[HSLOTS], nk[HSLOTS], nl[HSLOTS];
    #pragma unroll
                        for (int j = 0; j < HSLOTS; j++) {
                            const int c = src[j];
                            const uint32_t e = __shfl_sync(0xffffffffu, e_cur, c);
                            const unsigned long long w0 = __shfl_sync(0xffffffffu, cur.k0, c);
                            const unsigned long long w1 = __shfl_sync(0xffffffffu, cur.k1, c);
                            const unsigned long long v0 = __shfl_sync(0xffffffffu, cur.l0, c);
                            const unsigned long long v1 = __shfl_sync(0xffffffffu, cur.l1, c);
                            nk[j] = j < cnt ? __popcll(w0) + __popcll(w1) : 0;
                            nl[j] = j < cnt ? __popcll(v0) + __popcll(v1) : 0;
                            const T *row = a.U + static_cast<uint64_t>(e) * a.ld;
                            kid[j] = lane < nk[j] ? nth_bit(w0, w1, lane) : 0;
                            lid[j] = lane < nl[j] ? nth_bit(v0, v1, lane) : 0;
                            va[j] = lane < nk[j] ? static_cast<double>(row[k0 + kid[j]]) : 0.0;
                            vb[j] = lane < nl[j] ? static_cast<double>(row[l0 + lid[j]]) : 0.0;
                        }
    #pragma unroll
                        for (int j = 0; j < HSLOTS; j++) {
                            if (j < cnt) {
                                const double L2 = -2.0 * __shfl_sync(0xffffffffu, cur.L, src[j]);
                                for (int kk = 0; kk < nk[j]; kk++) {
                                    const double av = __shfl_sync(0xffffffffu, va[j], kk);
                                    const int kr = __shfl_sync(0xffffffffu, kid[j], kk);
                                    if (lane < nl[j]) atomicAdd(Mt + kr * HB + lid[j], L2 * fmin(av, vb[j]));
                                }
                            }
                        }
                    }
                    while (wide) {
                        const int c = __ffs(wide) - 1;
                        wide &= wide - 1;
                        const uint32_t e = __shfl_sync(0xffffffffu, e_cur, c);
                        const unsigned long long w0 = __shfl_sync(0xffffffffu, cur.k0, c);
                        const unsigned long long w1 = __shfl_sync(0xffffffffu, cur.k1, c);
                        const unsigned long long v0 = __shfl_sync(0xffffffffu, cur.l0, c);
                        const unsigned long long v1 = __shfl_sync(0xffffffffu, cur.l1, c);
                        const double L2 = -2.0 * __shfl_sync(0xffffffffu, cur.L, c);
                        const int nkw = __popcll(w0) + __popcll(w1), nlw = __popcll(v0) + __popcll(v1);
                        const T *row = a.U + static_cast<uint64_t>(e) * a.ld;
                        for (int kc = 0; kc < nkw; kc += 32) {
                            const int kq = kc + lane;
                            const int kr_l = kq < nkw ? nth_bit(w0, w1, kq) : 0;
                            const double a_l = kq < nkw ? static_cast<double>(row[k0 + kr_l]) : 0.0;
                            for (int lc = 0; lc < nlw; lc += 32) {
                                const int lq = lc + lane;
                                const int lr = lq < nlw ? nth_bit(v0, v1, lq) : 0;
                                const double b_l = lq < nlw ? static_cast<double>(row[l0 + lr]) : 0.0;
                                const int kn = min(32, nkw - kc);
                                for (int kk = 0; kk < kn; kk++) {
                                    const double av = __shfl_sync(0xffffffffu, a_l, kk);
                                    const int kr = __shfl_sync(0xffffffffu, kr_l, kk);
                                    if (lq < nlw) atomicAdd(Mt + kr * HB + lr, L2 * fmin(av, b_l));
                                }
                            }
                        }
                    }
                    cur = nxt;
                    nxt = after;
                }
            }
        } else {
            // ---- sparse rows: -2 L min(a, b) where both are non-zero.  Each warp
            // walks the embedded rows on its own (no block barrier) in batches of
            // 32 consecutive rows, owning tile rows HROWS warp .. HROWS warp +
            // HROWS - 1.  Lane i holds row i's class, mask words (its rows' word
            // and the two words of the l block, coalesced over the batch) and
            // length, fetched two batches ahead.  One ballot finds the sparse rows
            // with a non-zero in both the warp's rows and the l block; their values
            // are gathered HSLOTS rows at a time (lane r < HROWS: row value r,
            // lane j: columns j + 32 m) and the updates of row r take its value
            // from lane r by shuffle.
            {
                const uint64_t kwd = k0 / 64 + (warp * HROWS) / 64, lwd = l0 / 64;
                const int kshift = (warp * HROWS) % 64;
                constexpr uint32_t kmask = (1u << HROWS) - 1u;
                double *Mw = Mt + HROWS * warp * HB;
                const uint32_t er = (a.E + a.n_splits - 1) / a.n_splits;
                const uint32_t r_begin = min(a.E, split * er), r_end = min(a.E, r_begin + er);
                const uint32_t n_batches = r_end > r_begin ? (r_end - r_begin + 31) / 32 : 0;
                const unsigned long long *mk_base = a.masks + kwd * a.E;
                const unsigned long long *m0_base = a.masks + lwd * a.E;
                const unsigned long long *m1_base = a.masks + (lwd + 1) * a.E;
                struct Fetch {
                    unsigned long long km, m0, m1;
                    double L;
                    bool ok;
                };
                auto fetch = [&](uint32_t batch) {
                    Fetch f{0ull, 0ull, 0ull, 0.0, false};
                    const uint32_t e = r_begin + batch * 32 + lane;
                    if (batch < n_batches && e < r_end && a.row_class[e] == 1) {
                        f.km = mk_base[e];
                        f.m0 = m0_base[e];
                        f.m1 = m1_base[e];
                        f.L = static_cast<double>(a.len[e]);
                        f.ok = true;
                    }
                    return f;
                };
                Fetch cur = fetch(0), nxt = fetch(1);
                for (uint32_t b = 0; b < n_batches; b++) {
                    const Fetch after = fetch(b + 2);
                    const uint32_t e_cur = r_begin + b * 32 + lane;
                    const uint32_t mk_l = static_cast<uint32_t>(cur.km >> kshift) & kmask;
                    uint32_t active = __ballot_sync(0xffffffffu, cur.ok && mk_l != 0 && (cur.m0 | cur.m1) != 0ull);
                    while (active) {
                        int slot_lane[HSLOTS];
                        int cnt = 0;
    #pragma unroll
                        for (int j = 0; j < HSLOTS; j++) {
                            slot_lane[j] = active ? __ffs(active) - 1 : 0;
                            cnt += active ? 1 : 0;
                            active &= active ? active - 1 : 0u;
                        }
                        double va[HSLOTS], vb[HSLOTS][4];
    #pragma unroll
                        for (int j = 0; j < HSLOTS; j++) {
                            const int c = slot_lane[j];
                            const uint32_t e = __shfl_sync(0xffffffffu, e_cur, c);
                            const uint32_t mk = __shfl_sync(0xffffffffu, mk_l, c);
                            const unsigned long long m0 = __shfl_sync(0xffffffffu, cur.m0, c);
                            const unsigned long long m1 = __shfl_sync(0xffffffffu, cur.m1, c);
                            const T *row = a.U + static_cast<uint64_t>(e) * a.ld;
                            const bool live = j < cnt;
                            va[j] = (live && lane < HROWS && ((mk >> lane) & 1u))
                                        ? static_cast<double>(row[k0 + HROWS * warp + lane]) : 0.0;
    #pragma unroll
                            for (int m = 0; m < 4; m++) {
                                const unsigned long long wv = m < 2 ? m0 : m1;
                                const bool on = live && ((wv >> (32 * (m & 1) + lane)) & 1ull);
                                vb[j][m] = on ? static_cast<double>(row[l0 + 32 * m + lane]) : -1.0;
                            }
                        }
    #pragma unroll
                        for (int j = 0; j < HSLOTS; j++) {
                            if (j < cnt) {
                                const int c = slot_lane[j];
                                uint32_t mk = __shfl_sync(0xffffffffu, mk_l, c);
                                const double L2 = -2.0 * __shfl_sync(0xffffffffu, cur.L, c);
                                while (mk) {
                                    const int r = __ffs(mk) - 1;
                                    mk &= mk - 1;
                                    const double av = __shfl_sync(0xffffffffu, va[j], r);
    #pragma unroll
                                    for (int m = 0; m < 4; m++) {
                                        if (vb[j][m] >= 0.0) {
                                            double *p = Mw + r * HB + 32 * m + lane;
                                            *p = fma(L2, fmin(av, vb[j][m]), *p);
                                        }
                                    }
                                }
                            }
                        }
                    }
                    cur = nxt;
                    nxt = after;
                }
            }
        }
        __syncthreads();

        // ---- epilogue: raw sums to the split buffer, or finished values
        if (a.partial) {
            double *dst = a.partial + (static_cast<uint64_t>(split) * a.n_tiles + ti) * HB * HB;
            for (int e = tid; e < HB * HB; e += HTHREADS) dst[e] = Mt[e];
        } else {
            const TableDesc td = a.tables[tile.z];
            OutSpec o = a.out;
            if (o.mode == 0) o.ptr = static_cast<T *>(o.ptr) + td.out_off;
            for (int e = tid; e < HB * HB; e += HTHREADS)
                hybrid_emit<T, NORM>(a, td, o, ti, k0 + e / HB, l0 + e % HB, Mt[e]);
        }
        __syncthreads();  // the shared tile is reused by the next work item
    }
}

// Split partials of each tile summed in split order, then the epilogue.
// ---- pair-scatter form of the sparse rows
//
// For each (sparse row e, table t) of a group, one warp lists the table's
// samples where the row is non-zero (from the presence masks, in column
// order, up to SC_CAP at a time in shared memory with their values) and adds
// L min(a, b) of every pair k < l of the list to S[k][l] with a 64-bit
// integer atomic: the term in fixed point, round(L min(a, b) 2^s), with 2^s
// chosen on the host so that no pair's sum can reach 2^62.  Integer addition
// is associative, so the sums (and the results) do not depend on the order
// of the atomics.  Each (row, table) is visited once, against once per tile
// of the table in the tile walk; the work is the row's pair count.
constexpr int SC_WARPS = 8;
constexpr int SC_CAP = 256;

template <typename T>
struct ScatterArgs {
    const uint32_t *sparse_rows;
    const uint32_t *n_rows;  // {dense, sparse}
    const unsigned long long *masks;
    uint32_t E;
    const TableDesc *tables;
    uint32_t t0, n_tables;  // the group's tables
    const T *U;
    const T *len;
    uint64_t ld;
    unsigned long long *Sq;
    double scale;  // 2^s
    unsigned long long *next;  // task counter, zero at launch
    uint32_t band_rows;        // rows k of the sums per band
    uint32_t n_bands;          // bands per table (each table of the launch)
};

template <typename T>
__global__ void __launch_bounds__(SC_WARPS * 32) sparse_pairs_kernel(const ScatterArgs<T> a) {
    __shared__ uint32_t col_s[SC_WARPS][2][SC_CAP];
    __shared__ double val_s[SC_WARPS][2][SC_CAP];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint32_t n_sparse = a.n_rows[1];
    const uint64_t per_table = static_cast<uint64_t>(n_sparse) * a.n_bands;
    const uint64_t tasks = per_table * a.n_tables;
    for (;;) {
        // tasks (table, band, sparse row) in that order, taken from a counter:
        // the warps in flight hold a window of consecutive tasks, so they
        // share one band of one table's sums in L2 (a fixed grid stride lets
        // warps with heavy rows fall behind until the tasks in flight span
        // many bands)
        unsigned long long task = 0;
        if (lane == 0) task = atomicAdd(a.next, 1ull);
        task = __shfl_sync(0xffffffffu, task, 0);
        if (task >= tasks) break;
        const uint32_t e = a.sparse_rows[task % n_sparse];
        const TableDesc td = a.tables[a.t0 + static_cast<uint32_t>(task / per_table)];
        const uint32_t band = static_cast<uint32_t>((task % per_table) / n_sparse);
        const uint32_t klo = band * a.band_rows, khi = min(td.n, klo + a.band_rows);
        const uint64_t w0 = td.base / 64;  // tables start on 128-column boundaries
        const uint32_t nw = (td.n + 63) / 64;
        const unsigned long long *mrow = a.masks + w0 * a.E + e;
        // P present columns, Plo of them before the band, Phi before its end:
        // the band's k are the list ranks [Plo, Phi)
        uint32_t P = 0, Plo = 0, Phi = 0;
        auto below = [](unsigned long long m, uint32_t c0, uint32_t lim) -> uint32_t {
            return c0 + 64 <= lim ? __popcll(m) : c0 >= lim ? 0u : __popcll(m & ((1ull << (lim - c0)) - 1ull));
        };
        for (uint32_t w = lane; w < nw; w += 32) {
            const unsigned long long m = mrow[static_cast<uint64_t>(w) * a.E];
            P += __popcll(m);
            Plo += below(m, w * 64, klo);
            Phi += below(m, w * 64, khi);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            P += __shfl_xor_sync(0xffffffffu, P, o);
            Plo += __shfl_xor_sync(0xffffffffu, Plo, o);
            Phi += __shfl_xor_sync(0xffffffffu, Phi, o);
        }
        if (Phi <= Plo || Plo + 1 >= P) continue;  // no k in the band, or no l after it
        const double L = static_cast<double>(a.len[e]) * a.scale;
        const T *row = a.U + static_cast<uint64_t>(e) * a.ld + td.base;
        unsigned long long *S = a.Sq + td.out_off;
        // list b <- the present columns of rank [r0, r0 + SC_CAP), with values
        auto collect = [&](int b, uint32_t r0) {
            uint32_t base = 0;
            for (uint32_t w = lane; w - lane < nw && base < r0 + SC_CAP; w += 32) {
                const unsigned long long m = w < nw ? mrow[static_cast<uint64_t>(w) * a.E] : 0ull;
                const uint32_t c = __popcll(m);
                uint32_t incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const uint32_t y = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += y;
                }
                uint32_t rank = base + incl - c;  // rank of this word's first set bit
                unsigned long long mm = m;
                while (mm) {
                    const int bit = __ffsll(mm) - 1;
                    mm &= mm - 1;
                    if (rank >= r0 && rank < r0 + SC_CAP) {
                        const uint32_t col = w * 64 + bit;
                        col_s[warp][b][rank - r0] = col;
                        val_s[warp][b][rank - r0] = static_cast<double>(row[col]);
                    }
                    rank++;
                }
                base += __shfl_sync(0xffffffffu, incl, 31);
            }
            __syncwarp();
        };
        for (uint32_t i0 = Plo; i0 < Phi; i0 += SC_CAP) {
            const uint32_t ni = min(static_cast<uint32_t>(SC_CAP), Phi - i0);
            collect(0, i0);
            for (uint32_t j0 = i0; j0 < P; j0 += SC_CAP) {
                const bool same = j0 == i0;
                const uint32_t nj = min(static_cast<uint32_t>(SC_CAP), P - j0);
                if (!same) collect(1, j0);
                const int bl = same ? 0 : 1;
                for (uint32_t i = 0; i < ni; i++) {
                    const uint32_t k = col_s[warp][0][i];
                    const double av = val_s[warp][0][i];
                    unsigned long long *Sk = S + static_cast<uint64_t>(k) * td.n;
                    for (uint32_t j = (same ? i + 1 : 0) + lane; j < nj; j += 32) {
                        const double t = L * fmin(av, val_s[warp][bl][j]);
                        atomicAdd(Sk + col_s[warp][bl][j], static_cast<unsigned long long>(__double2ll_rn(t)));
                    }
                }
                __syncwarp();
            }
        }
    }
}

template <typename T, bool NORM>
__global__ void __launch_bounds__(HTHREADS) hybrid_finalize_kernel(const HybridArgs<T> a) {
    const uint32_t ti = blockIdx.x;
    const uint4 tile = a.tiles[ti];
    const TableDesc td = a.tables[tile.z];
    OutSpec o = a.out;
    if (o.mode == 0) o.ptr = static_cast<T *>(o.ptr) + td.out_off;
    for (int e = threadIdx.x; e < HB * HB; e += HTHREADS) {
        double x = 0.0;
        for (uint32_t s = 0; s < a.n_splits; s++) x += a.partial[(static_cast<uint64_t>(s) * a.n_tiles + ti) * HB * HB + e];
        hybrid_emit<T, NORM>(a, td, o, ti, tile.x * HB + e / HB, tile.y * HB + e % HB, x);
    }
}

}  // namespace dev
}  // namespace ssu
