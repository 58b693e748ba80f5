// LDMD / LDJ for large N (NPAD = 64*m <= 1024; N above 200 by default, any N
// when this family is selected for an N range): the matrices of
// a batch live in global memory (L2 / HBM) as lower 8x8 tiles in the DMMA
// accumulator layout of warp_dmma.cuh (tile t = I(I+1)/2 + J, lane l holds
// (8I + l/4, 8J + 2(l%4) + s)).  Included by propagator.cu after
// kernels_cta.cuh.
//
// Inversion is the symmetric Gauss-Jordan sweep of warp_dmma.cuh with 64
// pivots a round (one tile row/column block P of 8 tiles), in three batched
// kernels per round over all matrices of the batch:
//   factor  one CTA per matrix: unpivoted LDL^T of D = A_PP (lower triangle
//           only), Lam = L^{-1} (in the panel's fragment order) and
//           1/delta_k, negative pivots counted (SYMINV's KOUNT, syminv.f:27-49);
//   panel   every 8-row block: Lam by one bulk copy, c = A[i, P] Lam^T on DMMA, written as the
//           update operands X = -c/delta, B = c (rows of P: X = Lam^T/delta,
//           B = -Lam^T) in A-fragment order;
//   update  every lower tile: tiles of row/column block P zeroed, then
//           A_IJ += X_I B_J^T on DMMA (64 k-steps of m8n8k4), X and B staged
//           in shared memory by bulk (TMA) copies; split into the next
//           round's diagonal block, the rest of its block row and column,
//           and everything else (the look-ahead).
// which leaves A_ij - sum_k c_k(i) c_k(j)/delta_k outside P, A_iP D^{-1} in
// the columns of P and -D^{-1} in A_PP, the scalar sweep's values.  All reads
// take the lower triangle, so rounding left in the upper halves of diagonal
// tiles never feeds back.
//
// The step's elementwise parts (HAMMAT W, the reference-potential solutions,
// the Y updates of mdprop.f / ldprop.f) are separate batched kernels; a
// device-side step counter lets one step's launch sequence repeat unchanged.
#pragma once
#include "kernels_cta.cuh"

namespace mgpu {
namespace big {

using wf::tix;

constexpr int NB = 64;      // pivots per round
constexpr int KB = NB / 8;  // tile columns per round
constexpr int MC = NB / 4;  // m8n8k4 k-steps per round
// Factor CTA sizes: a whole SM's registers (1024 threads at 64) where the
// update beside it is small (NT <= FACT_BIG_MAX_NT), half of them above.
constexpr int FACT_THREADS = 512;
constexpr int FACT_THREADS_BIG = 1024;
constexpr int FACT_BIG_MAX_NT = 32;
constexpr int PANEL_WARPS = 8;
#ifndef MGPU_UPD_WARPS
#define MGPU_UPD_WARPS 4
#endif
#ifndef MGPU_UPD_ROWS
#define MGPU_UPD_ROWS 4
#endif
constexpr int UPD_WARPS = MGPU_UPD_WARPS;     // warps of an update CTA
constexpr int UPD_ROWS = MGPU_UPD_ROWS;       // tile rows of C per CTA (8: a whole 64x64 block)
constexpr int UPD_SPLIT = 8 / UPD_ROWS;       // CTAs per 64x64 block
constexpr int UPD_RPW = UPD_ROWS / UPD_WARPS; // tile rows per warp
static_assert(UPD_WARPS * UPD_RPW == UPD_ROWS && UPD_SPLIT * UPD_ROWS == 8, "update CTA shape");
#ifndef MGPU_UPD_UNROLL
#define MGPU_UPD_UNROLL 2
#endif
constexpr int UPD_UNROLL = MGPU_UPD_UNROLL;  // k-steps of the update loop unrolled
constexpr int EW_THREADS = 256;
constexpr int kBigMaxNT = 128;  // NPAD <= 1024

// One matrix of an inversion batch.
struct MatDesc {
    double *a;   // lower tiles, NT(NT+1)/2 * 64 doubles
    int *cnt;    // negative-pivot counter, incremented by sign * count
    int *stat;   // failure status (atomicMax)
    int *kfail;  // step of the first failure (atomicMin)
    int n;       // channels; rows >= n are padding (zero, unit pivot)
    int sign;    // +1 or -1
    int nstep;   // the matrix takes part while the step counter is <= nstep
    int kfix;    // > 0: report this step on failure instead of the counter
};

// Per-matrix scratch of one round.
struct Panels {
    double *lam;  // [M][64*64] Lam row-major
    double *rd;   // [M][64] 1/delta
    double *xf;   // [M][NT][MC][32] X in A-fragment order
    double *bf;   // [M][NT][MC][32] B in A-fragment order
};

__device__ __forceinline__ size_t sym_index(int i, int j)
{
    const int R = i > j ? i : j, C = i > j ? j : i;
    return (size_t)tix(R >> 3, C >> 3) * 64 + ((R & 7) * 4 + ((C & 7) >> 1)) * 2 + (C & 1);
}

// tile t -> (I, J), I >= J.  8t + 1 is exact in single precision (t < 2^21,
// NT <= 128 gives t < 8256); the loops correct the rounded root by one either way.
__device__ __forceinline__ void tile_ij(int t, int &I, int &J)
{
    int i = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
    while (i * (i + 1) / 2 > t) --i;
    while ((i + 1) * (i + 2) / 2 <= t) ++i;
    I = i;
    J = t - i * (i + 1) / 2;
}

// element x of a tiled matrix -> (row, column)
__device__ __forceinline__ void elem_ij(size_t x, int &i, int &j)
{
    int I, J;
    tile_ij((int)(x >> 6), I, J);
    const int l = (int)(x >> 1) & 31, s = (int)x & 1;
    i = 8 * I + (l >> 2);
    j = 8 * J + 2 * (l & 3) + s;
}

__device__ __forceinline__ void report_failure(const MatDesc &md, int flags, int k)
{
    const int code = (flags & 1) ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
    atomicMax(md.stat, code);
    atomicMin(md.kfail, md.kfix > 0 ? md.kfix : k);
}

// ---------------------------------------------------------------------------
// factor: LDL^T of the 64x64 pivot block, Lam = L^{-1}, 1/delta
// Sixteen sub-blocks of four pivots (the 4-pivot step of warp_dmma.cuh).  For
// sub-block p: rows below form c = Lam4 D[i, p..p+3]; the trailing lower part
// of D and the rows of Lam below take the rank-4 updates
//     D_ij -= sum_m c_m(i) c_m(j)/delta_m ,  Lam_i -= sum_m (c_m(i)/delta_m) Lam_p+m
// (elimination applied to I).  Look-ahead: warp 0 owns no trailing element;
// while the other warps update, it updates the next 4x4 diagonal block first
// and factors it (ldl_block4), so the chain of pivot reciprocals overlaps the
// rank-4 updates.
// ---------------------------------------------------------------------------
constexpr size_t kFactSmem = 2 * (size_t)NB * (NB + 1) * sizeof(double);  // D and Lam, padded rows
// element ownership in a factor CTA of T threads (warp 0 factors the sub-blocks)
template <int T>
struct FactShape {
    static_assert(T >= 5 * NB && T % 32 == 0, "factor CTA: 4 NB rows of c(i) and every Lam column at once");
    static constexpr int own = T - 32;                                   // threads owning elements
    static constexpr int d = (NB * (NB + 1) / 2 + own - 1) / own;        // D elements per thread
    static constexpr int l = (NB * (NB - 1) / 2 + own - 1) / own;        // Lam elements per thread
};

__device__ __forceinline__ void tri_rc(int e, int &i, int &j)  // e -> (i, j), j <= i
{
    int r = (int)((sqrtf(8.0f * e + 1.0f) - 1.0f) * 0.5f);
    while (r * (r + 1) / 2 > e) --r;
    while ((r + 1) * (r + 2) / 2 <= e) ++r;
    i = r;
    j = e - r * (r + 1) / 2;
}

template <int T>
__global__ void __launch_bounds__(T)
big_factor_kernel(const MatDesc *__restrict__ mds, Panels pn, int round, const int *__restrict__ kstep)
{
    constexpr int kFactOwn = FactShape<T>::own, kFactD = FactShape<T>::d, kFactL = FactShape<T>::l;
    extern __shared__ __align__(16) double fsm[];
    double (*D)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(fsm);
    double (*L)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(fsm + NB * (NB + 1));
    __shared__ __align__(16) double s_c[NB][4];  // c(i) of the current sub-block
    __shared__ __align__(16) double s_t[NB][4];  // c(i) / delta
    __shared__ double s_f[16];                   // ldl_block4 operands of the current sub-block
    __shared__ double s_r[NB];
    __shared__ int s_cnt, s_flags;
    const MatDesc md = mds[blockIdx.x];
    const int k = *kstep;
    if (k > md.nstep) return;
    const int p0 = NB * round, K0 = KB * round;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) s_cnt = s_flags = 0;
    for (int x = tid; x < NB * NB; x += T) {
        const int i = x >> 6, j = x & 63;
        double v = 0.0;
        if (j <= i) v = md.a[(size_t)tix(K0 + (i >> 3), K0 + (j >> 3)) * 64 + ((i & 7) * 4 + ((j & 7) >> 1)) * 2 + (j & 1)];
        D[i][j] = v;
        L[i][j] = (i == j) ? 1.0 : 0.0;
    }
    // owned elements (packed (i << 8) | j, -1 when none): D lower triangle, Lam strictly lower
    int od[kFactD], ol[kFactL];
#pragma unroll
    for (int u = 0; u < kFactD; ++u) {
        const int e = (tid - 32) + u * kFactOwn;
        int i = 0, j = 0;
        const bool ok = warp > 0 && e < NB * (NB + 1) / 2;
        if (ok) tri_rc(e, i, j);
        od[u] = ok ? ((i << 8) | j) : -1;
    }
#pragma unroll
    for (int u = 0; u < kFactL; ++u) {
        const int e = (tid - 32) + u * kFactOwn;
        int i = 0, c = 0;
        const bool ok = warp > 0 && e < NB * (NB - 1) / 2;
        if (ok) tri_rc(e, i, c);
        ol[u] = ok ? (((i + 1) << 8) | c) : -1;
    }
    __syncthreads();
    // warp 0 factors one 4x4 diagonal sub-block (rows q..q+3 of D final)
    auto sub_factor = [&](int q) {
        double f[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j <= i; ++j) f[i][j] = D[q + i][q + j];
        int cnt = 0, flags = 0;
        wf::ldl_block4(f, md.n - p0 - q, cnt, flags);
        if (lane == 0) {
            s_cnt += cnt;
            s_flags |= flags;
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) s_f[i * 4 + j] = f[i][j];
        }
    };
    if (warp == 0) sub_factor(0);
    for (int sb = 0; sb < NB / 4; ++sb) {
        const int p = 4 * sb;
        __syncthreads();
        double f[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j) f[i][j] = s_f[i * 4 + j];
        if (tid < 4) s_r[p + tid] = (tid == 0) ? f[0][0] : (tid == 1) ? f[1][1] : (tid == 2) ? f[2][2] : f[3][3];
        // c(i) = Lam4 D[i, p..p+3] for rows below; Lam rows of the sub-block = Lam4 Lam_sub
        if (tid < 4 * NB) {
            const int i = tid >> 2, m = tid & 3;
            if (i >= p + 4) {
                double lq[3], rq;
                wf::lane_operands(f, m, lq, rq);  // row m of Lam4 below the diagonal, 1/delta_m
                const double c = fma(lq[0], D[i][p], fma(lq[1], D[i][p + 1], fma(lq[2], D[i][p + 2], D[i][p + m])));
                s_c[i][m] = c;
                s_t[i][m] = c * rq;
            }
        } else {
            // one column per thread, in place from the last row up (row m reads the old rows above it)
            const int c = tid - 4 * NB;
            if (c < p + 4) {
#pragma unroll
                for (int m = 3; m >= 1; --m) {
                    double v = L[p + m][c];
#pragma unroll
                    for (int mm = 0; mm < 3; ++mm)
                        if (mm < m) v = fma(f[m][mm], L[p + mm][c], v);
                    L[p + m][c] = v;
                }
            }
        }
        __syncthreads();
        const int q = p + 4;  // next sub-block
        if (warp == 0) {
            if (q < NB) {
                if (lane < 10) {
                    int ii, jj;
                    tri_rc(lane, ii, jj);
                    const int i = q + ii, j = q + jj;
                    double v = D[i][j];
#pragma unroll
                    for (int m = 0; m < 4; ++m) v = fma(-s_t[i][m], s_c[j][m], v);
                    D[i][j] = v;
                }
                __syncwarp();
                sub_factor(q);
            }
        } else {
#pragma unroll
            for (int u = 0; u < kFactD; ++u) {
                const int i = od[u] >> 8, j = od[u] & 255;
                if (od[u] >= 0 && j >= q && !(i < q + 4)) {  // the next diagonal block is warp 0's
                    const double2 t01 = *reinterpret_cast<const double2 *>(&s_t[i][0]);
                    const double2 t23 = *reinterpret_cast<const double2 *>(&s_t[i][2]);
                    const double2 c01 = *reinterpret_cast<const double2 *>(&s_c[j][0]);
                    const double2 c23 = *reinterpret_cast<const double2 *>(&s_c[j][2]);
                    double v = D[i][j];
                    v = fma(-t01.x, c01.x, v);
                    v = fma(-t01.y, c01.y, v);
                    v = fma(-t23.x, c23.x, v);
                    v = fma(-t23.y, c23.y, v);
                    D[i][j] = v;
                }
            }
#pragma unroll
            for (int u = 0; u < kFactL; ++u) {
                const int i = ol[u] >> 8, c = ol[u] & 255;
                if (ol[u] >= 0 && i >= q && c < q) {
                    const double2 t01 = *reinterpret_cast<const double2 *>(&s_t[i][0]);
                    const double2 t23 = *reinterpret_cast<const double2 *>(&s_t[i][2]);
                    double v = L[i][c];
                    v = fma(-t01.x, L[p][c], v);
                    v = fma(-t01.y, L[p + 1][c], v);
                    v = fma(-t23.x, L[p + 2][c], v);
                    v = fma(-t23.y, L[p + 3][c], v);
                    L[i][c] = v;
                }
            }
        }
    }
    __syncthreads();
    // Lam in the panel's B-fragment order: (row 8kt + ln/4, column 4mc + ln%4) at (kt MC + mc) 32 + ln
    double *lam = pn.lam + (size_t)blockIdx.x * NB * NB;
    for (int x = tid; x < NB * NB; x += T) {
        const int ln = x & 31, mc = (x >> 5) % MC, kt = x / (32 * MC);
        lam[x] = L[8 * kt + (ln >> 2)][4 * mc + (ln & 3)];
    }
    if (tid < NB) pn.rd[(size_t)blockIdx.x * NB + tid] = s_r[tid];
    if (tid == 0) {
        if (s_cnt) atomicAdd(md.cnt, md.sign * s_cnt);
        if (s_flags) report_failure(md, s_flags, k);
    }
}

// ---------------------------------------------------------------------------
// panel: operand rows X, B of every 8-row block (one warp each)
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32 * PANEL_WARPS)
big_panel_kernel(const MatDesc *__restrict__ mds, Panels pn, int nt, int round, const int *__restrict__ kstep)
{
    // B fragments of Lam^T, as the factor wrote them: (k-row q, column r) of output tile kt, k-step mc
    __shared__ __align__(128) double lamB[KB][MC][32];
    __shared__ double s_r[NB];
    __shared__ __align__(8) uint64_t bar;
    const int m = blockIdx.y;
    const MatDesc md = mds[m];
    if (*kstep > md.nstep) return;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) bulk_load(&lamB[0][0][0], pn.lam + (size_t)m * NB * NB, NB * NB * sizeof(double), &bar);
    if (threadIdx.x < NB) s_r[threadIdx.x] = pn.rd[(size_t)m * NB + threadIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, r = lane >> 2, q = lane & 3;
    const int I = blockIdx.x * PANEL_WARPS + warp;
    const int p0 = NB * round, K0 = KB * round;
    const bool inP = I >= K0 && I < K0 + KB;
    const int i = 8 * I + r;
    double v[MC];  // A[i, p0 + 4mc + q] (A fragments), in flight while Lam lands
#pragma unroll
    for (int mc = 0; mc < MC; ++mc) v[mc] = (I < nt && !inP) ? md.a[sym_index(i, p0 + 4 * mc + q)] : 0.0;
    const bool landed = mbar_wait_bounded(&bar, 0);
    if (!__syncthreads_and(landed)) {  // every thread leaves here together
        if (threadIdx.x == 0) atomicMax(md.stat, MGPU_ERR_TIMEOUT);
        mbar_wait_bounded(&bar, 0);  // let the copy land before the CTA's shared memory goes
        return;
    }
    if (I >= nt) return;
    double *xf = pn.xf + ((size_t)m * nt + I) * MC * 32;
    double *bf = pn.bf + ((size_t)m * nt + I) * MC * 32;
    if (inP) {
        // rows of P: X(p0+a, k) = Lam[k][a] / delta_k, B(p0+a, k) = -Lam[k][a]
        const int a = 8 * (I - K0) + r;
        for (int mc = 0; mc < MC; ++mc) {
            const int kk = 4 * mc + q;
            const double la = lamB[kk >> 3][a >> 2][((kk & 7) << 2) | (a & 3)];
            xf[mc * 32 + lane] = la * s_r[kk];
            bf[mc * 32 + lane] = -la;
        }
        return;
    }
    double acc[KB][2];
#pragma unroll
    for (int kt = 0; kt < KB; ++kt) acc[kt][0] = acc[kt][1] = 0.0;
    // Lam is unit lower triangular: output columns 8kt..8kt+7 need k-steps mc <= 2kt+1 only
#pragma unroll
    for (int mc = 0; mc < MC; ++mc)
#pragma unroll
        for (int kt = 0; kt < KB; ++kt)
            if (mc <= 2 * kt + 1) wf::dmma(acc[kt][0], acc[kt][1], v[mc], lamB[kt][mc][lane]);
    // acc[kt][s] = c(8I + r, 8kt + 2q + s) -> A-fragment slot (k-step 2kt + q/2, lane r*4 + 2(q&1) + s)
#pragma unroll
    for (int kt = 0; kt < KB; ++kt) {
        const int col = 8 * kt + 2 * q;
        const int o = (2 * kt + (q >> 1)) * 32 + r * 4 + 2 * (q & 1);
        *reinterpret_cast<double2 *>(bf + o) = make_double2(acc[kt][0], acc[kt][1]);
        *reinterpret_cast<double2 *>(xf + o) = make_double2(acc[kt][0] * -s_r[col], acc[kt][1] * -s_r[col + 1]);
    }
}

// ---------------------------------------------------------------------------
// update: A_IJ = [IJ outside P] A_IJ + X_I B_J^T over a block of 8x8 tiles
// ---------------------------------------------------------------------------
constexpr uint32_t kUpdHalfBytes = KB * MC * 32 * sizeof(double);  // 32 KB: 8 tile rows of X (or B)
constexpr uint32_t kUpdXBytes = kUpdHalfBytes / UPD_SPLIT;         // X rows of one CTA
constexpr size_t kUpdSmem = (size_t)kUpdHalfBytes + kUpdXBytes;

// Which 64x64 blocks of tiles a launch updates: all of them; only block row and
// column `cblk` without the diagonal block (grid.x = UPD_SPLIT * (NT/8 - 1));
// all but block row and column `cblk`; only the diagonal block (cblk, cblk)
// (grid.x = UPD_SPLIT) -- the look-ahead split.  UPD_SPLIT consecutive CTAs
// share one block, UPD_ROWS tile rows each.
enum { UPD_ALL = 0, UPD_ONLY = 1, UPD_EXCEPT = 2, UPD_DIAG = 3 };

__global__ void __launch_bounds__(32 * UPD_WARPS)
big_update_kernel(const MatDesc *__restrict__ mds, Panels pn, int nt, int round, const int *__restrict__ kstep,
                  int mode, int cblk)
{
    extern __shared__ __align__(128) double usm[];
    __shared__ __align__(8) uint64_t bar;
    const int m = blockIdx.y;
    const MatDesc md = mds[m];
    if (*kstep > md.nstep) return;
    int BI, BJ;
    const int blk = (int)blockIdx.x / UPD_SPLIT, part = (int)blockIdx.x % UPD_SPLIT;
    if (mode == UPD_DIAG) {
        BI = BJ = cblk;
    } else if (mode == UPD_ONLY) {
        const int x = blk < cblk ? blk : blk + 1;  // block row cblk left of the diagonal, column cblk below it
        BI = x < cblk ? cblk : x;
        BJ = x < cblk ? x : cblk;
    } else {
        tile_ij(blk, BI, BJ);
        if (mode == UPD_EXCEPT && (BI == cblk || BJ == cblk)) return;  // whole CTA
    }
    double *Xs = usm, *Bs = usm + kUpdXBytes / sizeof(double);
    if (threadIdx.x == 0) {
        mbar_init(&bar, 2);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        bulk_load(Xs, pn.xf + ((size_t)m * nt + 8 * BI + UPD_ROWS * part) * MC * 32, kUpdXBytes, &bar);
        bulk_load(Bs, pn.bf + ((size_t)m * nt + 8 * BJ) * MC * 32, kUpdHalfBytes, &bar);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool inP = (BI == round) || (BJ == round);  // whole tiles of row/column block P
    const int I0 = 8 * BI + UPD_ROWS * part + UPD_RPW * warp;
    double acc[UPD_RPW][KB][2];
#pragma unroll
    for (int ii = 0; ii < UPD_RPW; ++ii)
#pragma unroll
        for (int jt = 0; jt < KB; ++jt) {
            const int I = I0 + ii, J = 8 * BJ + jt;
            double2 c = make_double2(0.0, 0.0);
            if (I >= J && !inP) c = *reinterpret_cast<const double2 *>(md.a + (size_t)tix(I, J) * 64 + lane * 2);
            acc[ii][jt][0] = c.x;
            acc[ii][jt][1] = c.y;
        }
    if (!mbar_wait_bounded(&bar, 0)) {
        if (threadIdx.x == 0) atomicMax(md.stat, MGPU_ERR_TIMEOUT);
        mbar_wait_bounded(&bar, 0);  // let the copies land before the CTA's shared memory goes
        return;
    }
    const double *xa = Xs + (UPD_RPW * warp) * MC * 32 + lane;
#pragma unroll UPD_UNROLL
    for (int mc = 0; mc < MC; ++mc) {
        double a[UPD_RPW];
#pragma unroll
        for (int ii = 0; ii < UPD_RPW; ++ii) a[ii] = xa[ii * MC * 32 + mc * 32];
#pragma unroll
        for (int jt = 0; jt < KB; ++jt) {
            const double b = Bs[(jt * MC + mc) * 32 + lane];
            const int J = 8 * BJ + jt;
#pragma unroll
            for (int ii = 0; ii < UPD_RPW; ++ii)
                if (I0 + ii >= J) wf::dmma(acc[ii][jt][0], acc[ii][jt][1], a[ii], b);
        }
    }
#pragma unroll
    for (int ii = 0; ii < UPD_RPW; ++ii)
#pragma unroll
        for (int jt = 0; jt < KB; ++jt) {
            const int I = I0 + ii, J = 8 * BJ + jt;
            if (I >= J)
                *reinterpret_cast<double2 *>(md.a + (size_t)tix(I, J) * 64 + lane * 2) =
                    make_double2(acc[ii][jt][0], acc[ii][jt][1]);
        }
}

// ---------------------------------------------------------------------------
// elementwise parts of a step (one job per blockIdx.y)
// ---------------------------------------------------------------------------
struct StepArgs {
    const SysDev *sys;
    const JobDev *jobs;
    const MatDesc *md;    // per job: its (Z) matrix, counters and status
    double *tiles2;       // LDJ: U matrices, [M][TD]
    double *vec;          // LDMD: [M][3][NPAD] y14, y14' = y14 - D1 W_ii, y23
    const int *kstep;
    int npad;
    size_t td;            // doubles of one tiled matrix
};

__device__ __forceinline__ const double *ptab_row(const SysDev &S, int ir) { return S.ptab + (size_t)ir * S.nham; }

// MDPROP start: Y tiles = H Y0 + D1 W(RSTART) (mdprop.f:89-93); counters reset
__global__ void __launch_bounds__(EW_THREADS) big_ldmd_init_kernel(StepArgs a, const double *__restrict__ y)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];
    const MatDesc md = a.md[m];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *md.cnt = 0;
        *md.stat = S.prep[1];  // a failed preparation fails every job of the system
        *md.kfail = S.prep[1] ? S.prep[2] : INT_MAX;
    }
    const double h = S.dr / 2.0, d1 = h * h / 3.0;
    const double *yj = y + job.yoff;
    const int n = S.n;
    for (size_t x = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; x < a.td; x += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        elem_ij(x, i, j);
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        const double y0 = (i < n && j < n) ? yj[(size_t)lo * n + hi] : 0.0;
        md.a[x] = h * y0 + d1 * cta::w_elem(S, ptab_row(S, 0), (int)x, i, j, 0, job.ered, true);
    }
}

// reference-potential solutions of step k and Y += y14' on the diagonal (mdprop.f:143-164)
__global__ void __launch_bounds__(EW_THREADS) big_ldmd_pre_kernel(StepArgs a)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];
    const MatDesc md = a.md[m];
    const int k = *a.kstep;
    if (k > md.nstep) return;
    const int i = blockIdx.x * EW_THREADS + threadIdx.x;
    if (i >= a.npad) return;
    double *v = a.vec + (size_t)m * 3 * a.npad;
    double y14 = 0.0, y14b = 0.0, y23 = 0.0;
    if (i < S.n) {
        const double h = S.dr / 2.0, d1 = h * h / 3.0;
        const int ir = 2 * k - 1;
        const size_t e = (size_t)tix(i >> 3, i >> 3) * 64 + ((i & 7) * 4 + ((i & 7) >> 1)) * 2 + (i & 1);
        const double wref = cta::w_elem(S, ptab_row(S, ir), (int)e, i, i, ir, job.ered, true);
        ref_solutions(wref, 0.5 * h, y14, y23);
        y14b = y14 - d1 * wref;
        md.a[e] += y14b;
    }
    v[i] = y14;
    v[a.npad + i] = y14b;
    v[2 * a.npad + i] = y23;
}

// W(R) of the element pair (i, j), (i, j + 1) at tiled offsets 2p, 2p + 1:
// HAMMAT + SUMLAM (hammat.f:85-113, sumlam.f:74-86) with the arithmetic of
// cta::w_elem, both elements from one 16-byte load per term.
__device__ __forceinline__ double2 w_pair(const SysDev &S, const double *__restrict__ P, size_t p, int i, int j, int ir,
                                          double ered)
{
    const size_t tdp = (size_t)S.ntiles * 32;  // pairs per coupling term
    double w0 = 0.0, w1 = 0.0;
    const double2 *vl = reinterpret_cast<const double2 *>(S.vlt) + p;
    if (S.ivlfl <= 0) {
        for (int l = 0; l < S.nham; ++l) {
            const double2 v = __ldg(vl + l * tdp);
            const double pl = __ldg(P + l);
            w0 = fma(v.x, pl, w0);
            w1 = fma(v.y, pl, w1);
        }
    } else {
        const int2 *iv = reinterpret_cast<const int2 *>(S.ivt) + p;
        for (int l = 0; l < S.nham; ++l) {
            const double2 v = __ldg(vl + l * tdp);
            const int2 ix = __ldg(iv + l * tdp);
            if (v.x != 0.0) w0 = fma(v.x, __ldg(P + ix.x), w0);
            if (v.y != 0.0) w1 = fma(v.y, __ldg(P + ix.y), w1);
        }
    }
    const int d = (i == j) ? 0 : (i == j + 1) ? 1 : -1;  // which element is on the diagonal
    if (d >= 0 && i < S.n) {
        double w = d ? w1 : w0;
        const double R = __ldg(S.rtab + ir);
        const double rsq = fmin(1.0 / (R * R), 1.0e16);
        if (S.nrsq == 0) w += rsq * S.cent[i];
        if (S.nconst == 0) w += S.eint[i];
        if (S.conlen > 0.0) {
            const double c2 = S.conlen * S.conlen;
            w += R * R / (c2 * c2);
        }
        w -= ered;
        if (d) w1 = w; else w0 = w;
    }
    return make_double2(w0, w1);
}

// pair p of a tiled matrix -> row i and first column j (the pair is (i, j), (i, j + 1))
__device__ __forceinline__ void pair_ij(size_t p, int &i, int &j)
{
    int I, J;
    tile_ij((int)(p >> 5), I, J);
    const int l = (int)p & 31;
    i = 8 * I + (l >> 2);
    j = 8 * J + 2 * (l & 3);
}

// Y = 2HQ(C_k) + 2 Y14 - Y23 Y^-1 Y23  (tiles hold -Y^-1; mdprop.f:156,181-185)
__global__ void __launch_bounds__(EW_THREADS) big_ldmd_mid_kernel(StepArgs a)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];  // by value: the stores below cannot alias it
    const MatDesc md = a.md[m];
    const int k = *a.kstep;
    if (k > md.nstep) return;
    const double *v = a.vec + (size_t)m * 3 * a.npad;
    const double2 *qk = reinterpret_cast<const double2 *>(S.q + (size_t)(k - 1) * a.td);
    double2 *y = reinterpret_cast<double2 *>(md.a);
    for (size_t p = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; p < a.td / 2; p += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        pair_ij(p, i, j);
        const double2 q = __ldg(qk + p), yp = y[p];
        const double v23i = v[2 * a.npad + i];
        double w0 = q.x + v23i * yp.x * v[2 * a.npad + j];
        double w1 = q.y + v23i * yp.y * v[2 * a.npad + j + 1];
        if (i == j) w0 += 2.0 * v[i];
        if (i == j + 1) w1 += 2.0 * v[i];
        y[p] = make_double2(w0, w1);
    }
}

// Y = D2 W(B) - Y23 Y^-1 Y23 + Y14' (D1 at the last step; mdprop.f:196-230)
__global__ void __launch_bounds__(EW_THREADS) big_ldmd_post_kernel(StepArgs a)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];  // by value: the stores below cannot alias it
    const MatDesc md = a.md[m];
    const int k = *a.kstep;
    if (k > md.nstep) return;
    const double h = S.dr / 2.0, d1 = h * h / 3.0, d2 = 2.0 * d1;
    const double dd = (k == S.nstep) ? d1 : d2;
    const double *v = a.vec + (size_t)m * 3 * a.npad;
    const double *P = ptab_row(S, 2 * k);
    double2 *y = reinterpret_cast<double2 *>(md.a);
    for (size_t p = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; p < a.td / 2; p += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        pair_ij(p, i, j);
        const double2 w = w_pair(S, P, p, i, j, 2 * k, job.ered), yp = y[p];
        const double v23i = v[2 * a.npad + i];
        double r0 = dd * w.x + v23i * yp.x * v[2 * a.npad + j];
        double r1 = dd * w.y + v23i * yp.y * v[2 * a.npad + j + 1];
        if (i == j) r0 += v[a.npad + i];
        if (i == j + 1) r1 += v[a.npad + i];
        y[p] = make_double2(r0, r1);
    }
}

// LDPROP start: Z = H Y0 + D1 W(RSTART) + I (ldprop.f:30-44)
__global__ void __launch_bounds__(EW_THREADS) big_ldj_init_kernel(StepArgs a, const double *__restrict__ y)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];
    const MatDesc md = a.md[m];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *md.cnt = 0;
        *md.stat = 0;
        *md.kfail = INT_MAX;
    }
    const double h = S.dr / 2.0, d1 = h * h / 3.0;
    const double *yj = y + job.yoff;
    const int n = S.n;
    for (size_t x = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; x < a.td; x += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        elem_ij(x, i, j);
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        const double y0 = (i < n && j < n) ? yj[(size_t)lo * n + hi] : 0.0;
        md.a[x] = h * y0 + d1 * cta::w_elem(S, ptab_row(S, 0), (int)x, i, j, 0, job.ered, true) +
                  ((i == j && i < n) ? 1.0 : 0.0);
    }
}

// U(C) = I/8 + D4 W(C) (ldprop.f:60-76)
__global__ void __launch_bounds__(EW_THREADS) big_ldj_pre_kernel(StepArgs a)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];
    const MatDesc md = a.md[m];
    const int k = *a.kstep;
    if (k > md.nstep) return;
    const double h = S.dr / 2.0, d4 = -h * h / 48.0;
    double2 *u = reinterpret_cast<double2 *>(a.tiles2 + (size_t)m * a.td);
    const double *P = ptab_row(S, 2 * k - 1);
    for (size_t p = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; p < a.td / 2; p += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        pair_ij(p, i, j);
        const double2 w = w_pair(S, P, p, i, j, 2 * k - 1, job.ered);
        u[p] = make_double2(d4 * w.x + ((i == j && i < S.n) ? 0.125 : 0.0),
                            d4 * w.y + ((i == j + 1 && i < S.n) ? 0.125 : 0.0));
    }
}

// Z = -U^-1 ... : Z <- (-U^{-1}) + (-Z^{-1}) - 6I in the sweep's signs (ldprop.f:92-97)
__global__ void __launch_bounds__(EW_THREADS) big_ldj_mid_kernel(StepArgs a)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];
    const MatDesc md = a.md[m];
    if (*a.kstep > md.nstep) return;
    const double2 *u = reinterpret_cast<const double2 *>(a.tiles2 + (size_t)m * a.td);
    double2 *z = reinterpret_cast<double2 *>(md.a);
    for (size_t p = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; p < a.td / 2; p += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        pair_ij(p, i, j);
        const double2 up = u[p], zp = z[p];
        z[p] = make_double2(-up.x + zp.x - ((i == j && i < S.n) ? 6.0 : 0.0),
                            -up.y + zp.y - ((i == j + 1 && i < S.n) ? 6.0 : 0.0));
    }
}

// Z = D2 W(B) + 2I + Z (D1 at the last step; ldprop.f:103-126)
__global__ void __launch_bounds__(EW_THREADS) big_ldj_post_kernel(StepArgs a)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];
    const MatDesc md = a.md[m];
    const int k = *a.kstep;
    if (k > md.nstep) return;
    const double h = S.dr / 2.0, d1 = h * h / 3.0, d2 = 2.0 * d1;
    const double dd = (k == S.nstep) ? d1 : d2;
    const double *P = ptab_row(S, 2 * k);
    double2 *z = reinterpret_cast<double2 *>(md.a);
    for (size_t p = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; p < a.td / 2; p += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        pair_ij(p, i, j);
        const double2 w = w_pair(S, P, p, i, j, 2 * k, job.ered), zp = z[p];
        z[p] = make_double2(dd * w.x + ((i == j && i < S.n) ? 2.0 : 0.0) + zp.x,
                            dd * w.y + ((i == j + 1 && i < S.n) ? 2.0 : 0.0) + zp.y);
    }
}

// MGPROP start: the tiles hold Y0 (mgprop.f:63), the counters cleared.
__global__ void __launch_bounds__(EW_THREADS) big_ldmg_init_kernel(StepArgs a, const double *__restrict__ y)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];
    const MatDesc md = a.md[m];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *md.cnt = 0;
        *md.stat = 0;
        *md.kfail = INT_MAX;
    }
    const double *yj = y + job.yoff;
    const int n = S.n;
    for (size_t x = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; x < a.td; x += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        elem_ij(x, i, j);
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        md.a[x] = (i < n && j < n) ? yj[(size_t)lo * n + hi] : 0.0;
    }
}

// MGPROP stage k of sector kstep (mgprop.f:94-104): X = Y + b_k h W(R) at
// radius row (kstep-1)*stride + k, then for a_k != 0 the matrix to invert,
// I + a_k h X (a_k = 0: Y = X); h is the matrix's own sector width.
__global__ void __launch_bounds__(EW_THREADS) big_ldmg_stage_kernel(StepArgs a, int stride, int k, double bk, double ak)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];
    const MatDesc md = a.md[m];
    const int ks = *a.kstep;
    if (ks > md.nstep) return;
    const double bh = bk * S.dr, ah = ak * S.dr;
    const int ir = (ks - 1) * stride + k;
    const double *P = ptab_row(S, ir);
    double2 *yv = reinterpret_cast<double2 *>(md.a);
    for (size_t p = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; p < a.td / 2; p += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        pair_ij(p, i, j);
        const double2 w = w_pair(S, P, p, i, j, ir, job.ered), yp = yv[p];
        double x0 = fma(bh, w.x, yp.x), x1 = fma(bh, w.y, yp.y);
        if (ah != 0.0) {
            x0 = ah * x0 + ((i == j && i < S.n) ? 1.0 : 0.0);
            x1 = ah * x1 + ((i == j + 1 && i < S.n) ? 1.0 : 0.0);
        }
        yv[p] = make_double2(x0, x1);
    }
}

// After the inversion (the tiles hold -(I + a_k h X)^-1): Y = [I - inverse]/(a_k h)
__global__ void __launch_bounds__(EW_THREADS) big_ldmg_after_kernel(StepArgs a, double ak)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];
    const MatDesc md = a.md[m];
    if (*a.kstep > md.nstep) return;
    const double d1 = 1.0 / (ak * S.dr);
    double2 *yv = reinterpret_cast<double2 *>(md.a);
    for (size_t p = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; p < a.td / 2; p += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        pair_ij(p, i, j);
        const double2 yp = yv[p];
        yv[p] = make_double2((yp.x + ((i == j && i < S.n) ? 1.0 : 0.0)) * d1,
                             (yp.y + ((i == j + 1 && i < S.n) ? 1.0 : 0.0)) * d1);
    }
}

// Results: Y = tiles/H (MDPROP, mdprop.f:269-275), Z/H - I/H (LDPROP,
// ldprop.f:140-147) or the tiles as they are (MGPROP) into the caller's
// column-major Y, both triangles; NODES (MDPROP: minus the U(C) count
// NSAVE), status and failing step.  mode: 0 MDPROP, 1 LDPROP, 2 MGPROP.
__global__ void __launch_bounds__(EW_THREADS)
big_finish_kernel(StepArgs a, int mode, double *__restrict__ y, int *__restrict__ nodes_out, int *__restrict__ status_out,
                  int *__restrict__ kfail_out)
{
    const int m = blockIdx.y;
    const JobDev job = a.jobs[m];
    const SysDev S = a.sys[job.sys];
    const MatDesc md = a.md[m];
    const int st = *md.stat;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        status_out[job.out] = st;
        kfail_out[job.out] = st ? *md.kfail : 0;
        nodes_out[job.out] = st ? 0 : (*md.cnt - (mode == 0 ? S.prep[0] : 0));
    }
    if (st) return;
    const bool ldj = mode == 1;
    const double hi = mode == 2 ? 1.0 : 2.0 / S.dr;
    const int n = S.n;
    double *yj = y + job.yoff;
    for (size_t x = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; x < a.td; x += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        elem_ij(x, i, j);
        if (i < n && j <= i) {
            const double v = hi * md.a[x] - ((ldj && i == j) ? hi : 0.0);
            yj[(size_t)j * n + i] = v;
            yj[(size_t)i * n + j] = v;
        }
    }
}

__global__ void big_step_advance_kernel(int *kstep, int value)
{
    if (value >= 0) *kstep = value;
    else ++*kstep;
}

// ---------------------------------------------------------------------------
// MDPROP preparation: U(C_k) = I/8 - (H^2/48) W_off(C_k) for a range of steps
// of one system, inverted in place as a batch, then 2HQ(C_k) = U^{-1} - 8I
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(EW_THREADS) big_prep_build_kernel(const SysDev *__restrict__ sys, int s, int k0, size_t td)
{
    const SysDev S = sys[s];
    const int k = k0 + blockIdx.y;
    if (k > S.nstep) return;
    const double h = S.dr / 2.0, d4 = -h * h / 48.0;
    double *u = S.q + (size_t)(k - 1) * td;
    const double *P = ptab_row(S, 2 * k - 1);
    for (size_t x = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; x < td; x += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        elem_ij(x, i, j);
        u[x] = (i == j) ? (i < S.n ? 0.125 : 0.0) : d4 * cta::w_elem(S, P, (int)x, i, j, 2 * k - 1, 0.0, false);
    }
}

__global__ void __launch_bounds__(EW_THREADS) big_prep_finish_kernel(const SysDev *__restrict__ sys, int s, int k0, size_t td)
{
    const SysDev S = sys[s];
    const int k = k0 + blockIdx.y;
    if (k > S.nstep) return;
    double *u = S.q + (size_t)(k - 1) * td;
    for (size_t x = (size_t)blockIdx.x * EW_THREADS + threadIdx.x; x < td; x += (size_t)gridDim.x * EW_THREADS) {
        int i, j;
        elem_ij(x, i, j);
        // tiles = -U^{-1};  2HQ(C) = U^{-1} - 8I
        u[x] = (i >= S.n || j >= S.n) ? 0.0 : (i == j ? -u[x] - 8.0 : -u[x]);
    }
}

}  // namespace big
}  // namespace mgpu
