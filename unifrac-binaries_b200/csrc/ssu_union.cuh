// Generalized and variance-adjusted UniFrac over a sparse embedding (sm_100a).
//
// A node adds nothing to a pair where neither sample has it: the VAW weight
// mi (m - mi) is 0 there (mi = counts of both samples), and so is the
// generalized u + v.  Per node, only the pairs with the row sample present
// (row pass: all 64 columns of the tile) or only the column sample present
// (column pass: the rows without it) are evaluated, each with the method's
// own term - no rearrangement, so the result matches the dense form up to
// the order of the summation (no cancellation, nothing to recompute).  Rows
// non-zero in more than ld / div columns run the dense loop in registers
// first.
//
// Tile: 128 (k) x 64 (l) pairs, 512 threads.  Sparse rows stream through a
// cp.async ring 16 at a time (one row per warp).  Row pass: warp w owns tile
// rows 8w .. 8w + 7 (fp64 numerator / denominator tiles in shared memory,
// lanes over columns).  Column pass: warp w owns columns 4w .. 4w + 3 over
// all 128 rows (registers, lanes over rows).  Every element has one owner
// per pass, so the sums are deterministic.  Uses the presence masks and row
// classes of ssu_sparse.cuh.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "ssu_kernels.cuh"

namespace ssu {
namespace dev {

template <typename T>
struct UnionArgs {
    const uint4 *tiles;  // 128 x 64 tiles: x block of 128 columns, y block of 64, z table
    uint32_t n_tiles, n_splits;
    const TableDesc *tables;
    const T *U, *C;      // proportions, raw counts (variance adjusted)
    const T *tot;        // per-column totals (variance adjusted)
    const T *len;        // per embedded row
    const unsigned long long *masks;  // word-major presence masks, E rows per word
    const uint8_t *row_class;         // 0 zero, 1 sparse, 2 dense
    uint32_t E;
    uint64_t ld;
    const uint32_t *dense_rows, *sparse_rows;
    const uint32_t *n_rows;  // {dense, sparse}
    double alpha;
    double *partial;     // per (split, tile) 2 x 128 x 64 fp64; nullptr: no splits
    OutSpec out;
};

constexpr int UK = 128, UL = 64;             // tile: k rows x l columns
constexpr int UKC = 8;                       // rows per dense pipeline stage
constexpr int USTAGES = 3;
constexpr int UTHREADS = 512;
constexpr int UWARPS = UTHREADS / 32;
constexpr int UROWS = UK / UWARPS;           // 8 tile rows per warp (row pass)
constexpr int UCOLS = UL / UWARPS;           // 4 tile columns per warp (column pass)
constexpr int USK = UWARPS;                  // sparse rows per stage, one per warp

template <bool CNT>
__host__ __device__ constexpr int union_sparse_stages() {
    return CNT ? 2 : 3;
}

// staged sparse row: k block, l block, 16 bytes of padding (bank spread)
template <typename T>
__host__ __device__ constexpr int union_row_pitch() {
    return UK + UL + 16 / static_cast<int>(sizeof(T));
}

template <typename T, bool CNT>
__host__ __device__ constexpr size_t union_stage_bytes() {
    constexpr size_t dense = USTAGES * (sizeof(T) * UKC * (UK + UL) * (CNT ? 2 : 1) + sizeof(T) * UKC);
    constexpr size_t sparse = union_sparse_stages<CNT>() *
                              (sizeof(T) * USK * union_row_pitch<T>() * (CNT ? 2 : 1) + sizeof(T) * USK);
    return ((dense > sparse ? dense : sparse) + 15) / 16 * 16;
}

template <typename T, bool CNT>
__host__ __device__ constexpr size_t union_smem() {
    return 2 * sizeof(double) * UK * UL + union_stage_bytes<T, CNT>() + (CNT ? sizeof(double) * (UK + UL) : 0);
}

template <typename T, class Op>
__device__ __forceinline__ void union_emit(const TableDesc &td, OutSpec o, uint32_t kc, uint32_t lc, double num,
                                           double den) {
    const uint32_t k = kc - td.base, l = lc - td.base;
    if (!(k < l && l < td.n)) return;
    const double acc[2] = {num, den};
    emit_pair<T>(o, td.n, k, l, static_cast<T>(Op::value(acc, 0.0, 0.0)));
}

// Op: the method's operator in double precision (its term and value).
template <typename T, class Op>
__global__ void __launch_bounds__(UTHREADS, 1) pair_union_kernel(const UnionArgs<T> a) {
    constexpr bool CNT = Op::COUNTS;
    constexpr int TX = UL / 4, TM = 4, TN = 4;  // dense phase: 16 (l) x 32 (k) threads, 4 x 4 pairs
    constexpr int VEC = 16 / sizeof(T);
    constexpr int ROW = UK + UL;                // dense staged values per row: k block then l block
    constexpr int CPR = ROW / VEC;              // 16-byte pieces per staged row
    constexpr int PITCH = union_row_pitch<T>();
    constexpr int SST = union_sparse_stages<CNT>();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *Mn = reinterpret_cast<double *>(smem_raw);  // [128][64] numerator
    double *Md = Mn + UK * UL;                          // [128][64] denominator
    unsigned char *stage = reinterpret_cast<unsigned char *>(Md + UK * UL);
    double *Ts = reinterpret_cast<double *>(stage + union_stage_bytes<T, CNT>());  // [192] column totals
    // dense phase staging
    T *Vs = reinterpret_cast<T *>(stage);               // [S][UKC][ROW] values
    T *Cs = Vs + USTAGES * UKC * ROW;                   // [S][UKC][ROW] counts (variance adjusted)
    T *Ls = Cs + (CNT ? USTAGES * UKC * ROW : 0);       // [S][UKC]
    // sparse phase staging (same bytes)
    T *Sv = reinterpret_cast<T *>(stage);               // [SST][USK][PITCH] values
    T *Sc = Sv + SST * USK * PITCH;                     // [SST][USK][PITCH] counts
    T *Sl = Sc + (CNT ? SST * USK * PITCH : 0);         // [SST][USK]

    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int lane = tid & 31, warp = tid >> 5;
    const uint32_t n_dense = a.n_rows[0], n_sparse = a.n_rows[1];
    const uint32_t n_work = a.n_tiles * a.n_splits;
    for (uint32_t w = blockIdx.x; w < n_work; w += gridDim.x) {
        const uint32_t split = w / a.n_tiles, ti = w - split * a.n_tiles;
        const uint4 tile = a.tiles[ti];
        const uint32_t k0 = tile.x * UK, l0 = tile.y * UL;
        const uint32_t dr = (n_dense + a.n_splits - 1) / a.n_splits;
        const uint32_t d_begin = min(n_dense, split * dr), d_end = min(n_dense, d_begin + dr);
        if (CNT)
            for (int c = tid; c < UK + UL; c += UTHREADS)
                Ts[c] = static_cast<double>(a.tot[c < UK ? k0 + c : l0 + (c - UK)]);
        __syncthreads();

        // ---- dense rows, 4 x 4 pairs per thread in registers
        double acc[TM][TN][2];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
        double tkd[TM], tld[TN];
#pragma unroll
        for (int i = 0; i < TM; i++) tkd[i] = CNT ? Ts[tile_row<UK, TM>(ty, i)] : 0.0;
#pragma unroll
        for (int j = 0; j < TN; j++) tld[j] = CNT ? Ts[UK + tile_row<UL, TN>(tx, j)] : 0.0;
        {
            // warp r < UKC stages row r of a chunk
            auto load_row = [&](int st, uint32_t e, bool ok) {
                T *dv = Vs + (st * UKC + warp) * ROW;
                T *dc = Cs + (st * UKC + warp) * ROW;
                const uint64_t base = static_cast<uint64_t>(e) * a.ld;
                for (int q = lane; q < CPR; q += 32) {
                    const uint32_t col = q < UK / VEC ? k0 + q * VEC : l0 + (q - UK / VEC) * VEC;
                    cp_async16(dv + q * VEC, a.U + base + col, ok ? 16 : 0);
                    if (CNT) cp_async16(dc + q * VEC, a.C + base + col, ok ? 16 : 0);
                }
                if (lane == 0) cp_async_small<sizeof(T)>(Ls + st * UKC + warp, a.len + e, ok ? (int)sizeof(T) : 0);
            };
            const uint32_t n_chunks = d_end > d_begin ? (d_end - d_begin + UKC - 1) / UKC : 0;
            auto ok_of = [&](uint32_t chunk) {
                return warp < UKC && chunk < n_chunks && d_begin + chunk * UKC + warp < d_end;
            };
            auto id_of = [&](uint32_t chunk) -> uint32_t { return ok_of(chunk) ? a.dense_rows[d_begin + chunk * UKC + warp] : 0u; };
            if (n_chunks > 0) {
                for (uint32_t c = 0; c + 1 < USTAGES; c++) {
                    if (c < n_chunks && warp < UKC) load_row(static_cast<int>(c), id_of(c), ok_of(c));
                    cp_async_commit();
                }
                uint32_t id1 = id_of(USTAGES - 1), id2 = id_of(USTAGES);
                for (uint32_t ch = 0; ch < n_chunks; ch++) {
                    const uint32_t nxt = ch + USTAGES - 1;
                    if (nxt < n_chunks && warp < UKC) load_row(static_cast<int>(nxt % USTAGES), id1, ok_of(nxt));
                    cp_async_commit();
                    id1 = id2;
                    id2 = id_of(ch + USTAGES + 1);
                    cp_async_wait<USTAGES - 1>();
                    __syncthreads();
                    const int st = static_cast<int>(ch % USTAGES);
                    const T *vs = Vs + st * UKC * ROW;
                    const T *cs = Cs + st * UKC * ROW;
                    for (int c = 0; c < UKC; c++) {
                        T av[TM], bv[TN], ac[TM], bc[TN];
                        load_half<T, TM / 2>(av, vs + c * ROW + ty * (TM / 2));
                        load_half<T, TM / 2>(av + TM / 2, vs + c * ROW + UK / 2 + ty * (TM / 2));
                        load_half<T, TN / 2>(bv, vs + c * ROW + UK + tx * (TN / 2));
                        load_half<T, TN / 2>(bv + TN / 2, vs + c * ROW + UK + UL / 2 + tx * (TN / 2));
                        if (CNT) {
                            load_half<T, TM / 2>(ac, cs + c * ROW + ty * (TM / 2));
                            load_half<T, TM / 2>(ac + TM / 2, cs + c * ROW + UK / 2 + ty * (TM / 2));
                            load_half<T, TN / 2>(bc, cs + c * ROW + UK + tx * (TN / 2));
                            load_half<T, TN / 2>(bc + TN / 2, cs + c * ROW + UK + UL / 2 + tx * (TN / 2));
                        }
                        const double L = static_cast<double>(Ls[st * UKC + c]);
#pragma unroll
                        for (int i = 0; i < TM; i++)
#pragma unroll
                            for (int j = 0; j < TN; j++)
                                Op::term(acc[i][j], static_cast<double>(av[i]), static_cast<double>(bv[j]),
                                         CNT ? static_cast<double>(ac[i]) : 0.0,
                                         CNT ? static_cast<double>(bc[j]) : 0.0, tkd[i] + tld[j], L, a.alpha);
                    }
                    __syncthreads();
                }
                cp_async_wait<0>();
            }
        }
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++) {
                const int at = tile_row<UK, TM>(ty, i) * UL + tile_row<UL, TN>(tx, j);
                Mn[at] = acc[i][j][0];
                Md[at] = acc[i][j][1];
            }
        __syncthreads();

        // ---- sparse rows, 16 per stage
        {
            const int r0 = UROWS * warp, c0 = UCOLS * warp;
            const uint32_t sr = (n_sparse + a.n_splits - 1) / a.n_splits;
            const uint32_t s_begin = min(n_sparse, split * sr), s_end = min(n_sparse, s_begin + sr);
            const uint32_t n_chunks = s_end > s_begin ? (s_end - s_begin + USK - 1) / USK : 0;
            // warp w stages row w of a chunk
            auto load = [&](uint32_t chunk) {
                const int st = static_cast<int>(chunk % SST);
                const uint32_t i = s_begin + chunk * USK + warp;
                const bool ok = i < s_end;
                const uint32_t e = ok ? a.sparse_rows[i] : 0u;
                const uint64_t base = static_cast<uint64_t>(e) * a.ld;
                T *dv = Sv + (st * USK + warp) * PITCH;
                T *dc = Sc + (st * USK + warp) * PITCH;
                for (int q = lane; q < CPR; q += 32) {
                    const uint32_t col = q < UK / VEC ? k0 + q * VEC : l0 + (q - UK / VEC) * VEC;
                    cp_async16(dv + q * VEC, a.U + base + col, ok ? 16 : 0);
                    if (CNT) cp_async16(dc + q * VEC, a.C + base + col, ok ? 16 : 0);
                }
                if (lane == 0) cp_async_small<sizeof(T)>(Sl + st * USK + warp, a.len + e, ok ? (int)sizeof(T) : 0);
            };
            // column pass accumulators: rows lane + 32 j of columns c0 + cc
            double bacc[UCOLS][4][2];
#pragma unroll
            for (int cc = 0; cc < UCOLS; cc++)
#pragma unroll
                for (int j = 0; j < 4; j++) bacc[cc][j][0] = bacc[cc][j][1] = 0.0;
            const double tl0 = CNT ? Ts[UK + lane] : 0.0, tl1 = CNT ? Ts[UK + lane + 32] : 0.0;
            for (uint32_t c = 0; c + 1 < SST; c++) {
                if (c < n_chunks) load(c);
                cp_async_commit();
            }
            for (uint32_t ch = 0; ch < n_chunks; ch++) {
                if (ch + SST - 1 < n_chunks) load(ch + SST - 1);
                cp_async_commit();
                cp_async_wait<SST - 1>();
                __syncthreads();
                const int st = static_cast<int>(ch % SST);
                const T *vs = Sv + st * USK * PITCH;
                const T *cs = Sc + st * USK * PITCH;
                const T *ls = Sl + st * USK;
                const int hn = lane & 15, hq = lane >> 4;

                // row pass: rows r0 + rr present; bit n of word rr: staged row n
                uint32_t rmask[UROWS / 2];
#pragma unroll
                for (int q = 0; q < UROWS / 2; q++)
                    rmask[q] = __ballot_sync(0xffffffffu, vs[hn * PITCH + r0 + 2 * q + hq] > T(0));
#pragma unroll
                for (int rr = 0; rr < UROWS; rr++) {
                    uint32_t nm = (rmask[rr / 2] >> (16 * (rr % 2))) & 0xffffu;
                    if (!nm) continue;
                    const int r = r0 + rr;
                    double t0[2] = {Mn[r * UL + lane], Md[r * UL + lane]};
                    double t1[2] = {Mn[r * UL + lane + 32], Md[r * UL + lane + 32]};
                    const double tk = CNT ? Ts[r] : 0.0;
                    while (nm) {
                        const int n = __ffs(nm) - 1;
                        nm &= nm - 1;
                        const T *v = vs + n * PITCH;
                        const T *cv = cs + n * PITCH;
                        const double L = static_cast<double>(ls[n]);
                        const double av = static_cast<double>(v[r]);
                        const double ca = CNT ? static_cast<double>(cv[r]) : 0.0;
                        Op::term(t0, av, static_cast<double>(v[UK + lane]), ca,
                                 CNT ? static_cast<double>(cv[UK + lane]) : 0.0, tk + tl0, L, a.alpha);
                        Op::term(t1, av, static_cast<double>(v[UK + lane + 32]), ca,
                                 CNT ? static_cast<double>(cv[UK + lane + 32]) : 0.0, tk + tl1, L, a.alpha);
                    }
                    Mn[r * UL + lane] = t0[0];
                    Md[r * UL + lane] = t0[1];
                    Mn[r * UL + lane + 32] = t1[0];
                    Md[r * UL + lane + 32] = t1[1];
                }

                // column pass: columns c0 + cc present, rows without the node
                uint32_t cmask[UCOLS / 2];
#pragma unroll
                for (int q = 0; q < UCOLS / 2; q++)
                    cmask[q] = __ballot_sync(0xffffffffu, vs[hn * PITCH + UK + c0 + 2 * q + hq] > T(0));
#pragma unroll
                for (int cc = 0; cc < UCOLS; cc++) {
                    uint32_t nm = (cmask[cc / 2] >> (16 * (cc % 2))) & 0xffffu;
                    const double tl = CNT ? Ts[UK + c0 + cc] : 0.0;
                    while (nm) {
                        const int n = __ffs(nm) - 1;
                        nm &= nm - 1;
                        const T *v = vs + n * PITCH;
                        const double L = static_cast<double>(ls[n]);
                        const double bv = static_cast<double>(v[UK + c0 + cc]);
                        const double cb = CNT ? static_cast<double>(cs[n * PITCH + UK + c0 + cc]) : 0.0;
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            const int r = lane + 32 * j;
                            if (v[r] == T(0))
                                Op::term(bacc[cc][j], 0.0, bv, 0.0, cb, (CNT ? Ts[r] : 0.0) + tl, L, a.alpha);
                        }
                    }
                }
                __syncthreads();
            }
            cp_async_wait<0>();
            // the row pass is complete (barrier above): add the column pass
#pragma unroll
            for (int cc = 0; cc < UCOLS; cc++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int at = (lane + 32 * j) * UL + c0 + cc;
                    Mn[at] += bacc[cc][j][0];
                    Md[at] += bacc[cc][j][1];
                }
        }
        __syncthreads();

        if (a.partial) {
            double *dst = a.partial + (static_cast<uint64_t>(split) * a.n_tiles + ti) * 2 * UK * UL;
            for (int e = tid; e < 2 * UK * UL; e += UTHREADS) dst[e] = Mn[e];
        } else {
            const TableDesc td = a.tables[tile.z];
            OutSpec o = a.out;
            if (o.mode == 0) o.ptr = static_cast<T *>(o.ptr) + td.out_off;
            for (int e = tid; e < UK * UL; e += UTHREADS)
                union_emit<T, Op>(td, o, k0 + e / UL, l0 + e % UL, Mn[e], Md[e]);
        }
        __syncthreads();  // the shared tiles are reused by the next work item
    }
}

// Split partials of each tile summed in split order, then the epilogue.
template <typename T, class Op>
__global__ void __launch_bounds__(UTHREADS) union_finalize_kernel(const UnionArgs<T> a) {
    const uint32_t ti = blockIdx.x;
    const uint4 tile = a.tiles[ti];
    const TableDesc td = a.tables[tile.z];
    OutSpec o = a.out;
    if (o.mode == 0) o.ptr = static_cast<T *>(o.ptr) + td.out_off;
    for (int e = threadIdx.x; e < UK * UL; e += UTHREADS) {
        double num = 0.0, den = 0.0;
        for (uint32_t s = 0; s < a.n_splits; s++) {
            const double *src = a.partial + (static_cast<uint64_t>(s) * a.n_tiles + ti) * 2 * UK * UL;
            num += src[e];
            den += src[UK * UL + e];
        }
        union_emit<T, Op>(td, o, tile.x * UK + e / UL, tile.y * UL + e % UL, num, den);
    }
}

// Method dispatch (ssu_union.cu): shared-memory limit of the method's
// instance, and the launch of its kernel (+ the split finalize).
template <typename T>
cudaError_t union_configure(const MethodSpec &spec, size_t *smem);
template <typename T>
cudaError_t union_launch(const MethodSpec &spec, const UnionArgs<T> &a, uint32_t ctas, cudaStream_t s);

}  // namespace dev
}  // namespace ssu
