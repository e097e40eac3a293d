// PCoA and PERMANOVA of a distance matrix on the device (interfaces and the
// methods in ssu_stats.hpp).  The n x n matrix is read from HBM once per
// multiply (PCoA) or once per batch of 32 permutations (PERMANOVA); the
// centred matrix and the permuted groupings are never materialised as n x n.
// The small dense problems (Gram matrices and the Rayleigh-Ritz matrix, at
// most 64 x 64) are solved on the host by cyclic Jacobi rotations.
#include "ssu_stats.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <numeric>
#include <random>
#include <vector>

#include <cuda_runtime.h>

namespace ssu {
namespace {

constexpr int kRows = 16;   // rows (one warp each) per PERMANOVA block
constexpr int kLmax = 32;   // basis columns per multiply pass
constexpr int kPb = 32;     // permutations per PERMANOVA pass
constexpr int kOversample = 10;
constexpr int kMinSteps = 4;   // multiplies by the matrix, at least
constexpr int kMaxSteps = 60;  // and at most

#define ST_CK(call)                                                   \
    do {                                                              \
        const cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) {                                      \
            err = std::string(#call) + ": " + cudaGetErrorString(e_); \
            return 6;                                                 \
        }                                                             \
    } while (0)

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// e(d): the entry of the matrix whose eigenpairs are sought, -d^2 / 2 for
// PCoA (before centring), d itself for an already centred matrix.
template <bool kSquare>
__device__ __forceinline__ double entry(double d) {
    return kSquare ? -0.5 * d * d : d;
}

// msum[i] = sum_j e(d_ij) / n (row means), diag[i] = e(d_ii); one warp per row.
template <typename TIn, bool kSquare>
__global__ void row_means_kernel(const TIn *__restrict__ D, uint32_t n, double *__restrict__ mean,
                                 double *__restrict__ diag) {
    const uint32_t i = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    if (i >= n) return;
    const TIn *row = D + static_cast<uint64_t>(i) * n;
    double s = 0.0;
    for (uint32_t j = lane; j < n; j += 32) s += entry<kSquare>(static_cast<double>(row[j]));
    s = warp_sum(s);
    if (lane == 0) {
        mean[i] = s / n;
        diag[i] = entry<kSquare>(static_cast<double>(row[i]));
    }
}

// Yt[c0 + c][i] = sum_j e(d_ij) Qt[c0 + c][j] for c < lc (<= 32); basis
// columns stored column-major ([column][row]).  A register-blocked tile
// product: a CTA of 128 threads owns 64 rows i x 32 columns c, each thread
// 4 x 4 of them; per step it stages e(d) of 64 rows x 32 j (transposed, so
// a thread reads its 4 rows of one j at once) and 32 j x 32 columns of Q in
// shared memory (the next step's tiles are loaded into registers while this
// one is multiplied), and every pair of staged loads feeds 16 FMAs.
constexpr int MI = 64, MC = 32, MJ = 32;  // rows, columns, j per step

template <typename TIn, bool kSquare>
__global__ void __launch_bounds__(128) multiply_kernel(const TIn *__restrict__ D, uint32_t n,
                                                       const double *__restrict__ Qt, uint32_t c0, uint32_t lc,
                                                       double *__restrict__ Yt) {
    __shared__ __align__(16) double ds[MJ][MI + 2];  // e(d) transposed: [j][i]
    __shared__ __align__(16) double qs[MJ][MC + 2];  // [j][c]
    const int tid = threadIdx.x;
    const int ti = tid % 16, tc = tid / 16;  // 16 x 8 threads, 4 x 4 each
    const uint32_t i0 = blockIdx.x * MI;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
    // staging assignment: D tile 64 x 32 (16 per thread: row r = tid / 2,
    // j = 16 (tid % 2) .. + 15), Q tile 32 x 32 (8 per thread: column
    // cq = tid / 4, j = 8 (tid % 4) .. + 7)
    const int dr = tid / 2, dj = 16 * (tid % 2);
    const int qc = tid / 4, qj = 8 * (tid % 4);
    const uint32_t drow = i0 + dr;
    const TIn *dsrc = D + static_cast<uint64_t>(drow < n ? drow : 0) * n;
    const bool qok = static_cast<uint32_t>(qc) < lc;
    const double *qsrc = Qt + static_cast<uint64_t>(c0 + (qok ? qc : 0)) * n;
    double dv[16], qv[8];
    auto load = [&](uint32_t j0) {
#pragma unroll
        for (int t = 0; t < 16; t++) {
            const uint32_t j = j0 + dj + t;
            dv[t] = (drow < n && j < n) ? entry<kSquare>(static_cast<double>(dsrc[j])) : 0.0;
        }
#pragma unroll
        for (int t = 0; t < 8; t++) {
            const uint32_t j = j0 + qj + t;
            qv[t] = (qok && j < n) ? qsrc[j] : 0.0;
        }
    };
    load(0);
    for (uint32_t j0 = 0; j0 < n; j0 += MJ) {
        __syncthreads();
#pragma unroll
        for (int t = 0; t < 16; t++) ds[dj + t][dr] = dv[t];
#pragma unroll
        for (int t = 0; t < 8; t++) qs[qj + t][qc] = qv[t];
        __syncthreads();
        if (j0 + MJ < n) load(j0 + MJ);
#pragma unroll 8
        for (int j = 0; j < MJ; j++) {
            double av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; a++) av[a] = ds[j][4 * ti + a];
#pragma unroll
            for (int b = 0; b < 4; b++) bv[b] = qs[j][4 * tc + b];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int b = 0; b < 4; b++) acc[a][b] = fma(av[a], bv[b], acc[a][b]);
        }
    }
#pragma unroll
    for (int b = 0; b < 4; b++) {
        const uint32_t c = 4 * tc + b;
        if (c >= lc) continue;
#pragma unroll
        for (int a = 0; a < 4; a++) {
            const uint32_t i = i0 + 4 * ti + a;
            if (i < n) Yt[static_cast<uint64_t>(c0 + c) * n + i] = acc[a][b];
        }
    }
}

// Gower centring applied to a product: (F Q)_ic = (E Q)_ic - m_i s_c - t_c + g s_c
// with m the row means of E, s_c = sum_j Q_jc, t_c = sum_j m_j Q_jc, g = mean(m).
__global__ void center_fixup_kernel(double *__restrict__ Yt, uint32_t n, uint32_t l, const double *__restrict__ m,
                                    const double *__restrict__ st, double g) {  // st: [s; t]
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<uint64_t>(n) * l) return;
    const uint32_t c = static_cast<uint32_t>(t / n), i = static_cast<uint32_t>(t % n);
    Yt[t] += -m[i] * st[c] - st[l + c] + g * st[c];
}

// G[a][b] = sum_i At[a][i] Bt[b][i]; one block per entry, fixed reduction order.
__global__ void dot_kernel(const double *__restrict__ At, const double *__restrict__ Bt, uint32_t n, uint32_t lb,
                           double *__restrict__ G) {
    __shared__ double red[256];
    const uint32_t a = blockIdx.x / lb, b = blockIdx.x % lb;
    const double *x = At + static_cast<uint64_t>(a) * n, *y = Bt + static_cast<uint64_t>(b) * n;
    double s = 0.0;
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x) s = fma(x[i], y[i], s);
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (static_cast<int>(threadIdx.x) < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) G[blockIdx.x] = red[0];
}

// Out[k][i] = sum_c Yt[c][i] T[c][k] (T is l x r, row-major).
__global__ void combine_kernel(const double *__restrict__ Yt, uint32_t n, uint32_t l, const double *__restrict__ T,
                               uint32_t r, double *__restrict__ Out) {
    const uint64_t t = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<uint64_t>(n) * r) return;
    const uint32_t k = static_cast<uint32_t>(t / n), i = static_cast<uint32_t>(t % n);
    double s = 0.0;
    for (uint32_t c = 0; c < l; c++) s = fma(Yt[static_cast<uint64_t>(c) * n + i], T[c * r + k], s);
    Out[t] = s;
}

// Per row i (one warp) and permutation p of a pass, sum over j > i of d^2
// where the two samples share a group, scaled by 1 / (that group's size);
// partial[block][p] sums the block's rows.  Pass 0 also sums all d^2, j > i.
template <typename TIn>
__global__ void __launch_bounds__(kRows * 32) permanova_kernel(const TIn *__restrict__ D, uint32_t n,
                                                                 const uint16_t *__restrict__ lab, uint32_t stride,
                                                                 uint32_t p0, const double *__restrict__ inv_size,
                                                                 double *__restrict__ partial,
                                                                 double *__restrict__ total_partial) {
    __shared__ double wsum[kRows][kPb + 1];
    const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    const uint32_t i = blockIdx.x * kRows + warp;
    double acc[kPb];
#pragma unroll
    for (int p = 0; p < kPb; p++) acc[p] = 0.0;
    double all = 0.0;
    uint16_t li[kPb] = {};
    if (i < n) {
        const uint16_t *ri = lab + static_cast<uint64_t>(i) * stride + p0;
#pragma unroll
        for (int p = 0; p < kPb; p++) li[p] = ri[p];
        const TIn *row = D + static_cast<uint64_t>(i) * n;
        for (uint32_t j = i + 1 + lane; j < n; j += 32) {
            const double d = static_cast<double>(row[j]);
            const double d2 = d * d;
            all += d2;
            const uint4 *rj = reinterpret_cast<const uint4 *>(lab + static_cast<uint64_t>(j) * stride + p0);
#pragma unroll
            for (int q = 0; q < kPb / 8; q++) {
                const uint4 w = rj[q];
                const uint32_t v[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
                for (int h = 0; h < 8; h++) {
                    const uint16_t lj = static_cast<uint16_t>(v[h / 2] >> (16 * (h % 2)));
                    acc[q * 8 + h] += lj == li[q * 8 + h] ? d2 : 0.0;
                }
            }
        }
    }
#pragma unroll
    for (int p = 0; p < kPb; p++) {
        const double s = warp_sum(acc[p]);
        if (lane == 0) wsum[warp][p] = i < n ? s * inv_size[li[p]] : 0.0;
    }
    all = warp_sum(all);
    if (lane == 0) wsum[warp][kPb] = i < n ? all : 0.0;
    __syncthreads();
    // fixed summation order: equal groupings give equal statistics
    if (threadIdx.x <= kPb) {
        double s = 0.0;
        for (int w = 0; w < kRows; w++) s += wsum[w][threadIdx.x];
        if (threadIdx.x < kPb)
            partial[static_cast<uint64_t>(blockIdx.x) * kPb + threadIdx.x] = s;
        else if (total_partial)
            total_partial[blockIdx.x] = s;
    }
}

// s_w[c] = sum over blocks (in order) of the per-block sums of grouping c,
// from partial[(c / 32) * blocks + b][c % 32].
__global__ void column_sums_kernel(const double *__restrict__ partial, uint32_t blocks, uint32_t cols,
                                   double *__restrict__ s_w) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    const double *p = partial + static_cast<size_t>(c / kPb) * blocks * kPb + c % kPb;
    double s = 0.0;
    for (uint32_t b = 0; b < blocks; b++) s += p[static_cast<size_t>(b) * kPb];
    s_w[c] = s;
}

// Cyclic Jacobi eigen-decomposition of a symmetric m x m matrix (row-major):
// eigenvalues w (descending) and eigenvectors as the columns of V.
void jacobi_eigen(std::vector<double> a, uint32_t m, std::vector<double> &w, std::vector<double> &V) {
    V.assign(static_cast<size_t>(m) * m, 0.0);
    for (uint32_t i = 0; i < m; i++) V[i * m + i] = 1.0;
    for (int sweep = 0; sweep < 100; sweep++) {
        double off = 0.0, diag = 0.0;
        for (uint32_t p = 0; p < m; p++)
            for (uint32_t q = 0; q < m; q++) (p == q ? diag : off) += a[p * m + q] * a[p * m + q];
        if (off <= 1e-30 * std::max(diag, std::numeric_limits<double>::min())) break;
        for (uint32_t p = 0; p + 1 < m; p++)
            for (uint32_t q = p + 1; q < m; q++) {
                const double apq = a[p * m + q];
                if (std::fabs(apq) < 1e-300) continue;
                const double theta = (a[q * m + q] - a[p * m + p]) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (uint32_t k = 0; k < m; k++) {  // columns p, q
                    const double akp = a[k * m + p], akq = a[k * m + q];
                    a[k * m + p] = c * akp - s * akq;
                    a[k * m + q] = s * akp + c * akq;
                }
                for (uint32_t k = 0; k < m; k++) {  // rows p, q
                    const double apk = a[p * m + k], aqk = a[q * m + k];
                    a[p * m + k] = c * apk - s * aqk;
                    a[q * m + k] = s * apk + c * aqk;
                }
                for (uint32_t k = 0; k < m; k++) {
                    const double vkp = V[k * m + p], vkq = V[k * m + q];
                    V[k * m + p] = c * vkp - s * vkq;
                    V[k * m + q] = s * vkp + c * vkq;
                }
            }
    }
    std::vector<uint32_t> order(m);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return a[x * m + x] > a[y * m + y]; });
    w.resize(m);
    std::vector<double> Vs(static_cast<size_t>(m) * m);
    for (uint32_t k = 0; k < m; k++) {
        w[k] = a[order[k] * m + order[k]];
        for (uint32_t i = 0; i < m; i++) Vs[i * m + k] = V[i * m + order[k]];
    }
    V.swap(Vs);
}

struct Dev {
    std::vector<void *> ptrs;
    cudaStream_t s = nullptr;
    ~Dev() {
        for (void *p : ptrs) cudaFreeAsync(p, s);
        if (s) {
            cudaStreamSynchronize(s);
            cudaStreamDestroy(s);
        }
    }
    template <typename P>
    cudaError_t alloc(P **p, size_t bytes) {
        void *q = nullptr;
        const cudaError_t e = cudaMallocAsync(&q, std::max<size_t>(bytes, 16), s);
        if (e == cudaSuccess) ptrs.push_back(q);
        *p = static_cast<P *>(q);
        return e;
    }
};

// True when `p` is device or managed memory (used in place, no copy).
bool on_device(const void *p) {
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// The n x n matrix on the device: `mat` itself when it is device memory, else
// a copy.
template <typename TIn>
int stage_matrix(Dev &dv, const TIn *mat, uint32_t n, const TIn *&dD, std::string &err) {
    if (on_device(mat)) {
        dD = mat;
        return 0;
    }
    TIn *p = nullptr;
    const size_t bytes = sizeof(TIn) * static_cast<size_t>(n) * n;
    ST_CK(dv.alloc(&p, bytes));
    ST_CK(cudaMemcpyAsync(p, mat, bytes, cudaMemcpyHostToDevice, dv.s));
    dD = p;
    return 0;
}

void launch_combine(Dev &dv, const double *Yt, uint32_t n, uint32_t l, const double *T, uint32_t r, double *Out) {
    const uint64_t total = static_cast<uint64_t>(n) * r;
    combine_kernel<<<static_cast<uint32_t>((total + 255) / 256), 256, 0, dv.s>>>(Yt, n, l, T, r, Out);
}

// Orthonormal basis of the columns of Yt (device, n x l, column-major) by
// scaled SVQB (Stathopoulos and Wu 2002): S = diag(G)^(-1/2), S G S = W w W',
// Q = Y S W_r w_r^(-1/2) over the eigenvalues above 1e-14 of the largest, so
// dependent and negligible columns drop out.  Sets r to the rank kept.
int svqb(Dev &dv, const double *Yt, uint32_t n, uint32_t l, double *Qt, double *dG, double *dT, uint32_t &r,
         std::string &err) {
    r = 0;
    if (l == 0) return 0;
    dot_kernel<<<l * l, 256, 0, dv.s>>>(Yt, Yt, n, l, dG);
    std::vector<double> G(static_cast<size_t>(l) * l);
    ST_CK(cudaMemcpyAsync(G.data(), dG, sizeof(double) * G.size(), cudaMemcpyDeviceToHost, dv.s));
    ST_CK(cudaStreamSynchronize(dv.s));
    // columns below 1e-14 of the longest are rounding noise (A Q with q in
    // A's null space): scaled to zero, they drop out with the dependent ones
    double top = 0.0;
    for (uint32_t c = 0; c < l; c++) top = std::max(top, G[c * l + c]);
    std::vector<double> sc(l);
    for (uint32_t c = 0; c < l; c++) sc[c] = G[c * l + c] > 1e-28 * top ? 1.0 / std::sqrt(G[c * l + c]) : 0.0;
    for (uint32_t a = 0; a < l; a++)
        for (uint32_t b = a; b < l; b++)
            G[a * l + b] = G[b * l + a] = 0.5 * (G[a * l + b] + G[b * l + a]) * sc[a] * sc[b];
    std::vector<double> w, W;
    jacobi_eigen(G, l, w, W);
    std::vector<uint32_t> keep;
    for (uint32_t k = 0; k < l; k++)
        if (w[k] > 1e-14 * w[0] && w[k] > 0.0) keep.push_back(k);
    r = static_cast<uint32_t>(keep.size());
    if (r == 0) return 0;
    std::vector<double> T(static_cast<size_t>(l) * r);
    for (uint32_t c = 0; c < l; c++)
        for (uint32_t k = 0; k < r; k++) T[c * r + k] = sc[c] * W[c * l + keep[k]] / std::sqrt(w[keep[k]]);
    ST_CK(cudaMemcpyAsync(dT, T.data(), sizeof(double) * T.size(), cudaMemcpyHostToDevice, dv.s));
    launch_combine(dv, Yt, n, l, dT, r, Qt);
    ST_CK(cudaGetLastError());
    return 0;
}

// The k = min(dims, rank) largest eigenpairs of the symmetric matrix A, where
// A = F (Gower-centred -D^2 / 2) when kSquare, else A = D: theta[k]
// descending, U[c * n + i] entry i of unit eigenvector c with its
// largest-magnitude entry positive, trace = trace(A).
template <typename TIn, bool kSquare>
int subspace_eigen(const TIn *mat, uint32_t n, uint32_t dims, std::vector<double> &theta, std::vector<double> &U,
                   double &trace, std::string &err) {
    theta.clear();
    U.clear();
    trace = 0.0;
    Dev dv;
    ST_CK(cudaStreamCreateWithFlags(&dv.s, cudaStreamNonBlocking));
    const TIn *dD = nullptr;
    if (stage_matrix(dv, mat, n, dD, err)) return 6;
    const uint32_t l0 = std::min<uint32_t>(dims + kOversample, n);
    double *dmean = nullptr, *ddiag = nullptr, *dm1 = nullptr, *dst = nullptr, *dY = nullptr, *dQ = nullptr,
           *dG = nullptr, *dT = nullptr;
    ST_CK(dv.alloc(&dmean, sizeof(double) * n));
    ST_CK(dv.alloc(&ddiag, sizeof(double) * n));
    ST_CK(dv.alloc(&dm1, sizeof(double) * 2 * n));
    ST_CK(dv.alloc(&dst, sizeof(double) * 2 * l0));
    ST_CK(dv.alloc(&dY, sizeof(double) * n * l0));
    ST_CK(dv.alloc(&dQ, sizeof(double) * n * l0));
    ST_CK(dv.alloc(&dG, sizeof(double) * l0 * l0));
    ST_CK(dv.alloc(&dT, sizeof(double) * l0 * l0));
    row_means_kernel<TIn, kSquare><<<(n + 7) / 8, 256, 0, dv.s>>>(dD, n, dmean, ddiag);
    std::vector<double> m1(2 * static_cast<size_t>(n), 1.0), diag(n);
    ST_CK(cudaMemcpyAsync(m1.data() + n, dmean, sizeof(double) * n, cudaMemcpyDeviceToHost, dv.s));
    ST_CK(cudaMemcpyAsync(diag.data(), ddiag, sizeof(double) * n, cudaMemcpyDeviceToHost, dv.s));
    ST_CK(cudaStreamSynchronize(dv.s));
    double g = 0.0;
    for (uint32_t i = 0; i < n; i++) {
        g += m1[n + i];
        trace += diag[i];
    }
    g /= n;
    if (kSquare) trace -= static_cast<double>(n) * g;  // sum_i (e_ii - 2 m_i + g)
    ST_CK(cudaMemcpyAsync(dm1, m1.data(), sizeof(double) * m1.size(), cudaMemcpyHostToDevice, dv.s));

    // Yt = A Q for the r columns of Qt (multiply passes of <= 32 columns)
    auto apply = [&](const double *Qt, uint32_t r) -> int {
        for (uint32_t c0 = 0; c0 < r; c0 += kLmax)
            multiply_kernel<TIn, kSquare><<<(n + MI - 1) / MI, 128, 0, dv.s>>>(dD, n, Qt, c0,
                                                                              std::min<uint32_t>(kLmax, r - c0), dY);
        if (kSquare) {
            // s_c = sum_j Q_jc and t_c = sum_j m_j Q_jc in one pass ([ones; m] . Q)
            dot_kernel<<<2 * r, 256, 0, dv.s>>>(dm1, Qt, n, r, dst);
            const uint64_t total = static_cast<uint64_t>(n) * r;
            center_fixup_kernel<<<static_cast<uint32_t>((total + 255) / 256), 256, 0, dv.s>>>(dY, n, r, dm1 + n,
                                                                                              dst, g);
        }
        ST_CK(cudaGetLastError());
        return 0;
    };

    // random start (fixed seed: the same input gives the same result)
    std::mt19937_64 gen(0x5EEDu);
    std::normal_distribution<double> normal;
    std::vector<double> omega(static_cast<size_t>(n) * l0);
    for (double &x : omega) x = normal(gen);
    ST_CK(cudaMemcpyAsync(dY, omega.data(), sizeof(double) * omega.size(), cudaMemcpyHostToDevice, dv.s));
    uint32_t r = 0;
    if (svqb(dv, dY, n, l0, dQ, dG, dT, r, err)) return 6;
    // Subspace iteration: Y = A Q, Rayleigh-Ritz on B = Q'Y, stop once the
    // wanted Ritz values move by at most 1e-12 of the largest (their error
    // is the square of the vectors'), else Q = orth(Y) and again.
    std::vector<double> V, prev, B;
    for (int it = 0; r > 0; it++) {
        if (apply(dQ, r)) return 6;
        dot_kernel<<<r * r, 256, 0, dv.s>>>(dQ, dY, n, r, dG);
        B.assign(static_cast<size_t>(r) * r, 0.0);
        ST_CK(cudaMemcpyAsync(B.data(), dG, sizeof(double) * B.size(), cudaMemcpyDeviceToHost, dv.s));
        ST_CK(cudaStreamSynchronize(dv.s));
        for (uint32_t a = 0; a < r; a++)  // symmetrise rounding
            for (uint32_t b = a + 1; b < r; b++) B[a * r + b] = B[b * r + a] = 0.5 * (B[a * r + b] + B[b * r + a]);
        jacobi_eigen(B, r, theta, V);
        const uint32_t kk = std::min(dims, r);
        bool done = it + 1 >= kMaxSteps;
        if (it + 1 >= kMinSteps && prev.size() == kk) {
            double move = 0.0, scale = 0.0;
            for (uint32_t c = 0; c < kk; c++) {
                move = std::max(move, std::fabs(theta[c] - prev[c]));
                scale = std::max(scale, std::fabs(theta[c]));
            }
            done = done || move <= 1e-12 * scale;
        }
        if (done) break;
        prev.assign(theta.begin(), theta.begin() + kk);
        uint32_t r1 = 0;
        if (svqb(dv, dY, n, r, dQ, dG, dT, r1, err)) return 6;
        ST_CK(cudaMemcpyAsync(dY, dQ, sizeof(double) * n * r1, cudaMemcpyDeviceToDevice, dv.s));
        if (svqb(dv, dY, n, r1, dQ, dG, dT, r, err)) return 6;  // second pass: orthogonal to rounding
    }
    if (r == 0) return 0;
    const uint32_t k = std::min(dims, r);
    theta.resize(k);
    std::vector<double> T(static_cast<size_t>(r) * k);
    for (uint32_t c = 0; c < r; c++)
        for (uint32_t q = 0; q < k; q++) T[c * k + q] = V[c * r + q];
    ST_CK(cudaMemcpyAsync(dT, T.data(), sizeof(double) * T.size(), cudaMemcpyHostToDevice, dv.s));
    launch_combine(dv, dQ, n, r, dT, k, dY);
    ST_CK(cudaGetLastError());
    U.resize(static_cast<size_t>(n) * k);
    ST_CK(cudaMemcpyAsync(U.data(), dY, sizeof(double) * U.size(), cudaMemcpyDeviceToHost, dv.s));
    ST_CK(cudaStreamSynchronize(dv.s));
    for (uint32_t c = 0; c < k; c++) {
        double *u = U.data() + static_cast<size_t>(c) * n;
        uint32_t big = 0;
        for (uint32_t i = 1; i < n; i++)
            if (std::fabs(u[i]) > std::fabs(u[big])) big = i;
        if (u[big] < 0)
            for (uint32_t i = 0; i < n; i++) u[i] = -u[i];
    }
    return 0;
}

}  // namespace

template <typename TIn>
int pcoa_device(const TIn *mat, uint32_t n, uint32_t dims, double *eigenvalues, double *samples, double *proportion,
                std::string &err) {
    std::fill(eigenvalues, eigenvalues + dims, 0.0);
    std::fill(proportion, proportion + dims, 0.0);
    std::fill(samples, samples + static_cast<size_t>(n) * dims, 0.0);
    if (n < 2 || dims == 0) return 0;
    std::vector<double> theta, U;
    double trace = 0.0;
    if (subspace_eigen<TIn, true>(mat, n, dims, theta, U, trace, err)) return 6;
    for (uint32_t c = 0; c < theta.size(); c++) {
        const double scale = std::sqrt(std::max(theta[c], 0.0));
        eigenvalues[c] = theta[c];
        proportion[c] = trace > 0 ? theta[c] / trace : 0.0;
        for (uint32_t i = 0; i < n; i++) samples[static_cast<size_t>(i) * dims + c] = U[static_cast<size_t>(c) * n + i] * scale;
    }
    return 0;
}

template <typename TIn>
int eigens_device(const TIn *mat, uint32_t n, uint32_t dims, double *eigenvalues, double *vectors, std::string &err) {
    std::fill(eigenvalues, eigenvalues + dims, 0.0);
    std::fill(vectors, vectors + static_cast<size_t>(n) * dims, 0.0);
    if (n == 0 || dims == 0) return 0;
    std::vector<double> theta, U;
    double trace = 0.0;
    if (subspace_eigen<TIn, false>(mat, n, dims, theta, U, trace, err)) return 6;
    for (uint32_t c = 0; c < theta.size(); c++) {
        eigenvalues[c] = theta[c];
        for (uint32_t i = 0; i < n; i++) vectors[static_cast<size_t>(i) * dims + c] = U[static_cast<size_t>(c) * n + i];
    }
    return 0;
}

template <typename TIn>
int permanova_device(const TIn *mat, uint32_t n, const uint32_t *grouping, uint32_t n_groups, uint32_t perms,
                     uint64_t seed, double &fstat, double &pvalue, std::string &err) {
    const double nan = std::numeric_limits<double>::quiet_NaN();
    fstat = pvalue = nan;
    if (n_groups > 65535) {
        err = "more than 65535 groups";
        return 6;
    }
    if (n_groups < 2 || n_groups >= n) return 0;
    std::vector<double> size(n_groups, 0.0);
    for (uint32_t i = 0; i < n; i++) {
        if (grouping[i] >= n_groups) {
            err = "grouping label out of range";
            return 6;
        }
        size[grouping[i]] += 1.0;
    }
    std::vector<double> inv(n_groups);
    for (uint32_t g = 0; g < n_groups; g++) inv[g] = size[g] > 0 ? 1.0 / size[g] : 0.0;
    // grouping 0 is the observed one, 1..perms permuted (Fisher-Yates, one
    // stream from `seed`), evaluated in chunks of columns so that the labels
    // on the device stay within about 256 MiB whatever the permutation count;
    // the host draws chunk c + 1 while the device evaluates chunk c.
    const uint32_t total = (perms + 1 + kPb - 1) / kPb * kPb;
    uint64_t budget = uint64_t(256) << 20;  // UNIFRAC_B200_PERMANOVA_LABEL_BYTES
    if (const char *v = std::getenv("UNIFRAC_B200_PERMANOVA_LABEL_BYTES"))
        budget = std::max<uint64_t>(1, std::strtoull(v, nullptr, 10));
    const uint64_t fit = budget / (2ull * n) / kPb * kPb;
    const uint32_t chunk = static_cast<uint32_t>(std::min<uint64_t>(total, std::max<uint64_t>(kPb, fit)));
    Dev dv;
    ST_CK(cudaStreamCreateWithFlags(&dv.s, cudaStreamNonBlocking));
    const uint32_t blocks = (n + kRows - 1) / kRows;
    const TIn *dD = nullptr;
    if (stage_matrix(dv, mat, n, dD, err)) return 6;
    uint16_t *dl = nullptr;
    double *dinv = nullptr, *dpart = nullptr, *dtot = nullptr, *dsw = nullptr;
    ST_CK(dv.alloc(&dl, sizeof(uint16_t) * n * chunk));
    ST_CK(dv.alloc(&dinv, sizeof(double) * n_groups));
    ST_CK(dv.alloc(&dpart, sizeof(double) * blocks * chunk));
    ST_CK(dv.alloc(&dtot, sizeof(double) * blocks));
    ST_CK(dv.alloc(&dsw, sizeof(double) * chunk));
    ST_CK(cudaMemcpyAsync(dinv, inv.data(), sizeof(double) * n_groups, cudaMemcpyHostToDevice, dv.s));
    std::vector<uint16_t> lab(static_cast<size_t>(n) * chunk, 0);
    std::vector<uint32_t> cur(grouping, grouping + n);
    std::mt19937_64 gen(seed);
    std::vector<double> s_w(total, 0.0);
    uint32_t next_p = 0;  // next grouping to draw
    auto draw = [&](uint32_t cn) {  // the next cn groupings, row stride cn
        for (uint32_t c = 0; c < cn; c++, next_p++) {
            if (next_p > 0 && next_p <= perms)
                for (uint32_t i = n - 1; i > 0; i--) {
                    std::uniform_int_distribution<uint32_t> pick(0, i);
                    std::swap(cur[i], cur[pick(gen)]);
                }
            // columns past `perms` (padding to whole passes) repeat the last grouping; never read
            for (uint32_t i = 0; i < n; i++) lab[static_cast<size_t>(i) * cn + c] = static_cast<uint16_t>(cur[i]);
        }
    };
    uint32_t c0 = 0, cn = std::min(chunk, total);
    draw(cn);
    while (cn > 0) {
        ST_CK(cudaMemcpyAsync(dl, lab.data(), sizeof(uint16_t) * n * cn, cudaMemcpyHostToDevice, dv.s));
        for (uint32_t p0 = 0; p0 < cn; p0 += kPb)
            permanova_kernel<TIn><<<blocks, kRows * 32, 0, dv.s>>>(dD, n, dl, cn, p0, dinv,
                                                                   dpart + static_cast<size_t>(p0 / kPb) * blocks * kPb,
                                                                   c0 == 0 && p0 == 0 ? dtot : nullptr);
        column_sums_kernel<<<(cn + 255) / 256, 256, 0, dv.s>>>(dpart, blocks, cn, dsw);
        ST_CK(cudaGetLastError());
        const uint32_t c1 = c0 + cn, cn1 = std::min(chunk, total - c1);
        if (cn1 > 0) draw(cn1);  // overlaps the device's chunk
        ST_CK(cudaMemcpyAsync(s_w.data() + c0, dsw, sizeof(double) * cn, cudaMemcpyDeviceToHost, dv.s));
        ST_CK(cudaStreamSynchronize(dv.s));
        c0 = c1;
        cn = cn1;
    }
    std::vector<double> tot(blocks);
    ST_CK(cudaMemcpyAsync(tot.data(), dtot, sizeof(double) * blocks, cudaMemcpyDeviceToHost, dv.s));
    ST_CK(cudaStreamSynchronize(dv.s));
    double s_t = 0.0;
    for (uint32_t b = 0; b < blocks; b++) s_t += tot[b];
    s_t /= n;
    auto f_of = [&](uint32_t p) { return ((s_t - s_w[p]) / (n_groups - 1)) / (s_w[p] / (n - n_groups)); };
    fstat = f_of(0);
    if (perms > 0) {
        uint32_t ge = 0;
        for (uint32_t p = 1; p <= perms; p++) ge += f_of(p) >= fstat ? 1u : 0u;
        pvalue = (ge + 1.0) / (perms + 1.0);
    }
    return 0;
}

template int pcoa_device<double>(const double *, uint32_t, uint32_t, double *, double *, double *, std::string &);
template int pcoa_device<float>(const float *, uint32_t, uint32_t, double *, double *, double *, std::string &);
template int eigens_device<double>(const double *, uint32_t, uint32_t, double *, double *, std::string &);
template int eigens_device<float>(const float *, uint32_t, uint32_t, double *, double *, std::string &);
template int permanova_device<double>(const double *, uint32_t, const uint32_t *, uint32_t, uint32_t, uint64_t,
                                      double &, double &, std::string &);
template int permanova_device<float>(const float *, uint32_t, const uint32_t *, uint32_t, uint32_t, uint64_t,
                                     double &, double &, std::string &);

}  // namespace ssu
