// Generalized and variance-adjusted UniFrac over a sparse embedding (sm_100a).
//
// A node adds nothing to a pair where neither sample has it: the VAW weight
// mi (m - mi) is 0 there (mi = counts of both samples), and so is the
// generalized u + v.  Per node, only the pairs with the row sample present
// (row pass: all 64 columns of the tile) or the column sample present (column
// pass: the rows without it) are evaluated, each with the method's own term -
// no rearrangement, so the result matches the dense form up to the order of
// the summation (no cancellation, nothing to recompute).  Rows non-zero in
// more than ld / div columns run the dense loop in registers first.
//
// Tile: 128 (k) x 64 (l) pairs, 512 threads; fp64 numerator and denominator
// tiles in shared memory; warp w owns tile rows 8w .. 8w + 7 and updates them
// in row order, one lane per element (deterministic).  Uses the presence masks
// and row classes of ssu_sparse.cuh.
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
    const uint32_t *dense_rows;
    const uint32_t *n_rows;  // {dense, sparse}
    double alpha;
    double *partial;     // per (split, tile) 2 x 128 x 64 fp64; nullptr: no splits
    OutSpec out;
};

constexpr int UK = 128, UL = 64;             // tile: k rows x l columns
constexpr int UKC = 8;                       // rows per dense pipeline stage
constexpr int USTAGES = 3;
constexpr int UTHREADS = 512;
constexpr int UROWS = UK / (UTHREADS / 32);  // 8 tile rows per warp
constexpr int USLOTS = 4;                    // active rows gathered together per warp

template <typename T, bool CNT>
constexpr size_t union_smem() {
    return 2 * sizeof(double) * UK * UL + USTAGES * (sizeof(T) * UKC * (UK + UL) * (CNT ? 2 : 1) + sizeof(T) * UKC) +
           64;
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
    constexpr int ROW = UK + UL;                // staged values per row: k block then l block
    constexpr int CPR = ROW / VEC;              // 16-byte pieces per staged row
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *Mn = reinterpret_cast<double *>(smem_raw);  // [128][64] numerator
    double *Md = Mn + UK * UL;                          // [128][64] denominator
    T *Vs = reinterpret_cast<T *>(Md + UK * UL);        // [S][UKC][ROW] values
    T *Cs = Vs + USTAGES * UKC * ROW;                   // [S][UKC][ROW] counts (variance adjusted)
    T *Ls = Cs + (CNT ? USTAGES * UKC * ROW : 0);       // [S][UKC]

    const int tid = threadIdx.x, tx = tid % TX, ty = tid / TX;
    const int lane = tid & 31, warp = tid >> 5;
    const uint32_t n_dense = a.n_rows[0];
    const uint32_t n_work = a.n_tiles * a.n_splits;
    for (uint32_t w = blockIdx.x; w < n_work; w += gridDim.x) {
        const uint32_t split = w / a.n_tiles, ti = w - split * a.n_tiles;
        const uint4 tile = a.tiles[ti];
        const uint32_t k0 = tile.x * UK, l0 = tile.y * UL;
        const uint32_t dr = (n_dense + a.n_splits - 1) / a.n_splits;
        const uint32_t d_begin = min(n_dense, split * dr), d_end = min(n_dense, d_begin + dr);

        // ---- dense rows, 4 x 4 pairs per thread in registers
        double acc[TM][TN][2];
#pragma unroll
        for (int i = 0; i < TM; i++)
#pragma unroll
            for (int j = 0; j < TN; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
        double tkd[TM], tld[TN];
#pragma unroll
        for (int i = 0; i < TM; i++) tkd[i] = CNT ? static_cast<double>(a.tot[k0 + tile_row<UK, TM>(ty, i)]) : 0.0;
#pragma unroll
        for (int j = 0; j < TN; j++) tld[j] = CNT ? static_cast<double>(a.tot[l0 + tile_row<UL, TN>(tx, j)]) : 0.0;
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

        // ---- sparse rows, walked in order by each warp on its own in batches
        // of 32; lane i holds row i's class, mask words (the warp's rows, the
        // l block) and length, fetched two batches ahead
        {
            const int r0 = UROWS * warp;
            const uint64_t kwd = k0 / 64 + r0 / 64, lwd = l0 / 64;
            const int kshift = r0 % 64;
            constexpr uint32_t kmask = (1u << UROWS) - 1u;
            double *Wn = Mn + r0 * UL, *Wd = Md + r0 * UL;
            const double tl0 = CNT ? static_cast<double>(a.tot[l0 + lane]) : 0.0;
            const double tl1 = CNT ? static_cast<double>(a.tot[l0 + lane + 32]) : 0.0;
            const double tk_lane = (CNT && lane < UROWS) ? static_cast<double>(a.tot[k0 + r0 + lane]) : 0.0;
            const uint32_t er = (a.E + a.n_splits - 1) / a.n_splits;
            const uint32_t e_begin = min(a.E, split * er), e_end = min(a.E, e_begin + er);
            const uint32_t n_batches = e_end > e_begin ? (e_end - e_begin + 31) / 32 : 0;
            const unsigned long long *mk_base = a.masks + kwd * a.E;
            const unsigned long long *ml_base = a.masks + lwd * a.E;
            struct Fetch {
                unsigned long long km, ml;
                double L;
                bool ok;
            };
            auto fetch = [&](uint32_t batch) {
                Fetch f{0ull, 0ull, 0.0, false};
                const uint32_t e = e_begin + batch * 32 + lane;
                if (batch < n_batches && e < e_end && a.row_class[e] == 1) {
                    f.km = mk_base[e];
                    f.ml = ml_base[e];
                    f.L = static_cast<double>(a.len[e]);
                    f.ok = true;
                }
                return f;
            };
            Fetch cur = fetch(0), nxt = fetch(1);
            for (uint32_t b = 0; b < n_batches; b++) {
                const Fetch after = fetch(b + 2);
                const uint32_t e_cur = e_begin + b * 32 + lane;
                const uint32_t mk_l = static_cast<uint32_t>(cur.km >> kshift) & kmask;
                uint32_t active = __ballot_sync(0xffffffffu, cur.ok && (mk_l != 0 || cur.ml != 0ull));
                while (active) {
                    int slot_lane[USLOTS];
                    int cnt = 0;
#pragma unroll
                    for (int j = 0; j < USLOTS; j++) {
                        slot_lane[j] = active ? __ffs(active) - 1 : 0;
                        cnt += active ? 1 : 0;
                        active &= active ? active - 1 : 0u;
                    }
                    // gather: lanes r < 8 the row values present, every lane its
                    // two columns when present
                    double va[USLOTS], vca[USLOTS], vb[USLOTS][2], vcb[USLOTS][2];
#pragma unroll
                    for (int j = 0; j < USLOTS; j++) {
                        const int c = slot_lane[j];
                        const uint32_t e = __shfl_sync(0xffffffffu, e_cur, c);
                        const uint32_t mk = __shfl_sync(0xffffffffu, mk_l, c);
                        const unsigned long long ml = __shfl_sync(0xffffffffu, cur.ml, c);
                        const uint64_t base = static_cast<uint64_t>(e) * a.ld;
                        const bool live = j < cnt;
                        const bool ron = live && lane < UROWS && ((mk >> lane) & 1u);
                        va[j] = ron ? static_cast<double>(a.U[base + k0 + r0 + lane]) : 0.0;
                        vca[j] = (CNT && ron) ? static_cast<double>(a.C[base + k0 + r0 + lane]) : 0.0;
#pragma unroll
                        for (int m = 0; m < 2; m++) {
                            const bool con = live && ((ml >> (lane + 32 * m)) & 1ull);
                            vb[j][m] = con ? static_cast<double>(a.U[base + l0 + lane + 32 * m]) : 0.0;
                            vcb[j][m] = (CNT && con) ? static_cast<double>(a.C[base + l0 + lane + 32 * m]) : 0.0;
                        }
                    }
#pragma unroll
                    for (int j = 0; j < USLOTS; j++) {
                        if (j < cnt) {  // uniform
                            const int c = slot_lane[j];
                            const uint32_t mk = __shfl_sync(0xffffffffu, mk_l, c);
                            const unsigned long long ml = __shfl_sync(0xffffffffu, cur.ml, c);
                            const double L = __shfl_sync(0xffffffffu, cur.L, c);
                            // row pass: the warp's rows present x every column
                            uint32_t rows = mk;
                            while (rows) {
                                const int r = __ffs(rows) - 1;
                                rows &= rows - 1;
                                const double av = __shfl_sync(0xffffffffu, va[j], r);
                                const double cav = __shfl_sync(0xffffffffu, vca[j], r);
                                const double tk = __shfl_sync(0xffffffffu, tk_lane, r);
#pragma unroll
                                for (int m = 0; m < 2; m++) {
                                    const int at = r * UL + lane + 32 * m;
                                    double t[2] = {Wn[at], Wd[at]};
                                    Op::term(t, av, vb[j][m], cav, vcb[j][m], tk + (m ? tl1 : tl0), L, a.alpha);
                                    Wn[at] = t[0];
                                    Wd[at] = t[1];
                                }
                            }
                            // column pass: columns present x the warp's rows
                            // absent, 4 columns x 8 rows per round
                            const uint32_t absent = ~mk & kmask;
                            const uint32_t lo = static_cast<uint32_t>(ml), hi = static_cast<uint32_t>(ml >> 32);
                            const int plo = __popc(lo), ncol = absent ? plo + __popc(hi) : 0;
                            for (int ib = 0; ib < ncol; ib += 32 / UROWS) {
                                const int i = ib + lane / UROWS, r = lane % UROWS;
                                int col = 0;
                                if (i < ncol)
                                    col = i < plo ? static_cast<int>(__fns(lo, 0, i + 1))
                                                  : 32 + static_cast<int>(__fns(hi, 0, i - plo + 1));
                                const int src = col & 31;
                                const double b0 = __shfl_sync(0xffffffffu, vb[j][0], src);
                                const double b1 = __shfl_sync(0xffffffffu, vb[j][1], src);
                                const double c0 = __shfl_sync(0xffffffffu, vcb[j][0], src);
                                const double c1 = __shfl_sync(0xffffffffu, vcb[j][1], src);
                                const double t0 = __shfl_sync(0xffffffffu, tl0, src);
                                const double t1 = __shfl_sync(0xffffffffu, tl1, src);
                                const double tk = __shfl_sync(0xffffffffu, tk_lane, r);
                                if (i < ncol && ((absent >> r) & 1u)) {
                                    const bool up = col >= 32;
                                    const int at = r * UL + col;
                                    double t[2] = {Wn[at], Wd[at]};
                                    Op::term(t, 0.0, up ? b1 : b0, 0.0, up ? c1 : c0, tk + (up ? t1 : t0), L,
                                             a.alpha);
                                    Wn[at] = t[0];
                                    Wd[at] = t[1];
                                }
                            }
                            // the next row's passes give an element to another lane
                            __syncwarp();
                        }
                    }
                }
                cur = nxt;
                nxt = after;
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
