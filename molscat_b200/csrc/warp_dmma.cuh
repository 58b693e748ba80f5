// One warp per symmetric matrix, held in FP64 tensor-core (DMMA) fragments.
//
// The matrix (padded to NPAD = 8*NT) is cut into 8x8 tiles; the lower
// triangle of tiles, t = I*(I+1)/2 + J (I >= J), lives in registers in the
// accumulator layout of mma.sync.m8n8k4.f64: lane l holds elements
// (row 8I + (l>>2), col 8J + 2(l&3) + s), s = 0,1.  Diagonal tiles hold both
// triangles.  Padding rows/columns are zero.
//
// Inversion is the symmetric Gauss-Jordan sweep done four pivots at a time
// (block sweep).  For the pivot block P = {p0..p0+3} with D = A_PP = L Delta L^T
// (unpivoted, the scalar sweep's own pivots delta_k) and Lam = L^{-1}:
//     c_k(i) = sum_m Lam[k][m] A_{i,p0+m}          (i not in P)
//     A_ij  -= sum_k c_k(i) c_k(j) / delta_k        (i, j not in P)
//     A_iP   = A_iP D^{-1} ,  A_PP = -D^{-1}
// which after all blocks leaves -A^{-1}.  The trailing update is the scalar
// sweep's own sum of rank-one terms, so the block sweep keeps its rounding
// behaviour; forming D^{-1} first and updating with A_iP D^{-1} A_Pj instead
// loses accuracy when a pivot is small next to its neighbours.  As in
// tiles.cuh the owners zero row/column block P and the operands carry the
// pivot block, so every lower tile gets the same update
//     A_IJ += X_I B_J          (one m8n8k4 DMMA per lower tile)
// with X(i,k) = -c_k(i)/delta_k, B(j,k) = c_k(j) for rows outside P and
// X(p0+a,k) = Lam[k][a]/delta_k, B(p0+b,k) = -Lam[k][b] for rows of P, which
// writes A_iP D^{-1} into the columns of P and -D^{-1} into A_PP.  The panel
// A_{:,P} goes through a small per-warp shared-memory buffer.  Every read of
// a diagonal tile takes the lower triangle, so the stored matrix is symmetric
// for the algorithm whatever rounding left in the upper triangle.
//
// The pivots delta_k are those of the unpivoted LDL^T SYMINV forms
// (syminv.f:27-49); their negative count is SYMINV's KOUNT (and DSYNEG's
// inertia by Sylvester's law); a zero pivot is the reference's IFAIL = N+1.
#pragma once
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdint.h>

#include "tiles.cuh"  // pivot_reciprocal, pivot_flags

namespace mgpu {
namespace wf {

template <int NT>
struct G {
    static constexpr int NTL = NT * (NT + 1) / 2;  // lower tiles
    static constexpr int NPAD = 8 * NT;
    static constexpr int PAN = NPAD * 4;           // panel doubles per warp
    static constexpr int WSM = PAN + 16;           // panel + pivot-block buffer
};

__host__ __device__ constexpr int tix(int I, int J) { return I * (I + 1) / 2 + J; }

// Not volatile: the result registers carry every dependency, and leaving
// the compiler free to schedule DMMAs between other work helps it overlap
// them with the look-ahead factorisation.
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Unpivoted LDL^T of the symmetric 4x4 pivot block D, read from the lower
// triangle of d (the upper triangle is ignored), pivot by pivot as the scalar
// sweep meets them.  On return d holds the block's operands:
//     d[k][k] = 1/delta_k ,  d[i][k] = Lam[i][k] (i > k) ,  d[k][i] = 0
// with Lam = L^{-1} (unit lower).  Negative pivots of the first `nreal` rows
// are added to cnt; the rest are padding, zero off the diagonal, and taken as
// exact unit pivots (not counted, never singular).
__device__ __forceinline__ void ldl_block4(double d[4][4], int nreal, int &cnt, int &flags)
{
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i][i] = (i >= nreal) ? 1.0 : d[i][i];
    double l[4][4], rd[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double dk = d[k][k];
        flags |= pivot_flags(dk);
        cnt += (dk < 0.0);
        const double rk = pivot_reciprocal(dk);
        rd[k] = rk;
#pragma unroll
        for (int i = k + 1; i < 4; ++i) l[i][k] = d[i][k] * rk;
#pragma unroll
        for (int i = k + 1; i < 4; ++i)
#pragma unroll
            for (int j = k + 1; j <= i; ++j) d[i][j] = fma(-l[i][k], d[j][k], d[i][j]);
    }
    // Lam = L^{-1} by forward substitution
    double lam[4][4];
#pragma unroll
    for (int i = 1; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < i; ++j) {
            double s = -l[i][j];
#pragma unroll
            for (int m = j + 1; m < i; ++m) s = fma(-l[i][m], lam[m][j], s);
            lam[i][j] = s;
        }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) d[i][j] = (i == j) ? rd[i] : (i > j ? lam[i][j] : 0.0);
}

// Gather the 4x4 pivot block rows/cols 4H..4H+3 of diagonal tile (K, K)
// into every lane with shuffles, lower triangle only: element (i, j), i >= j,
// sits in lane (4H+i)*4 + 2H + (j>>1), slot j&1.  Ten shuffles.
template <int NT, int K, int H>
__device__ __forceinline__ void gather_block(const double (&a)[G<NT>::NTL][2], int lane, double (&f)[4][4])
{
    (void)lane;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) {
            const int src = (4 * H + i) * 4 + 2 * H + (j >> 1);
            f[i][j] = __shfl_sync(0xffffffffu, a[tix(K, K)][j & 1], src);
        }
}

// This lane's share of the block operands (ldl_block4 layout in f): row q of
// Lam below the diagonal (lq[m], m < q; zero for m >= q) and 1/delta_q.
__device__ __forceinline__ void lane_operands(const double (&f)[4][4], int q, double (&lq)[3], double &rq)
{
    lq[0] = (q == 1) ? f[1][0] : (q == 2) ? f[2][0] : (q == 3) ? f[3][0] : 0.0;
    lq[1] = (q == 2) ? f[2][1] : (q == 3) ? f[3][1] : 0.0;
    lq[2] = (q == 3) ? f[3][2] : 0.0;
    rq = (q == 1) ? f[1][1] : (q == 2) ? f[2][2] : (q == 3) ? f[3][3] : f[0][0];
}

// Lam[q][a] from this lane's row of Lam
__device__ __forceinline__ double lam_qa(const double (&lq)[3], int q, int a)
{
    const double x = (a == 0) ? lq[0] : (a == 1) ? lq[1] : (a == 2) ? lq[2] : 0.0;
    return (a == q) ? 1.0 : x;
}

// One block of four pivots, tile column K, half H (p0 = 8K + 4H).  f holds
// the block's operands (ldl_block4) on entry and the next block's on exit
// (computed right after the next block's diagonal tile is updated, so its
// latency overlaps the rest of this block's DMMAs).
template <int NT, int K, int H>
__device__ __forceinline__ void sweep_round(double (&a)[G<NT>::NTL][2], double *pan, int n,
                                            int lane, double (&f)[4][4], int &cnt, int &flags)
{
    const int r = lane >> 2, q = lane & 3;
    constexpr int K2 = H ? K + 1 : K;  // next block
    constexpr int H2 = H ? 0 : 1;
    constexpr int p2 = 8 * K2 + 4 * H2;  // first pivot of the next block
    // publish the panel A[i, P] (row i -> pan[4i .. 4i+3]) from the lower
    // triangle: tiles below the diagonal in tile column K directly, tiles left
    // of it in tile row K transposed; in diagonal tile K the rows of the other
    // half come from whichever side of it lies in the lower triangle (rows of
    // P themselves are not needed)
    __syncwarp();
    if ((q >> 1) == H) {
#pragma unroll
        for (int I = (H ? K + 1 : K); I < NT; ++I) {
            pan[(8 * I + r) * 4 + 2 * q - 4 * H] = a[tix(I, K)][0];
            pan[(8 * I + r) * 4 + 2 * q - 4 * H + 1] = a[tix(I, K)][1];
        }
    }
    if ((r >> 2) == H) {
#pragma unroll
        for (int J = 0; J < K; ++J) {
            pan[(8 * J + 2 * q) * 4 + (r & 3)] = a[tix(K, J)][0];
            pan[(8 * J + 2 * q + 1) * 4 + (r & 3)] = a[tix(K, J)][1];
        }
        if (H == 1 && q < 2) {
            pan[(8 * K + 2 * q) * 4 + (r & 3)] = a[tix(K, K)][0];
            pan[(8 * K + 2 * q + 1) * 4 + (r & 3)] = a[tix(K, K)][1];
        }
    }
    __syncwarp();
    double lq[3], rq;
    lane_operands(f, q, lq, rq);
    const double nrq = -rq;
    // zero row/column block P
#pragma unroll
    for (int I = K; I < NT; ++I) {
        a[tix(I, K)][0] = ((q >> 1) == H) ? 0.0 : a[tix(I, K)][0];
        a[tix(I, K)][1] = ((q >> 1) == H) ? 0.0 : a[tix(I, K)][1];
    }
#pragma unroll
    for (int J = 0; J <= K; ++J) {
        a[tix(K, J)][0] = ((r >> 2) == H) ? 0.0 : a[tix(K, J)][0];
        a[tix(K, J)][1] = ((r >> 2) == H) ? 0.0 : a[tix(K, J)][1];
    }
    // operands: X_I (A fragment: row r, col q), B_J (B fragment: row q, col r)
    double X[NT], B[NT];
#pragma unroll
    for (int I = 0; I < NT; ++I) {
        const double2 *row = reinterpret_cast<const double2 *>(pan + (8 * I + r) * 4);
        const double2 x01 = row[0];
        const double x2 = row[1].x;
        const double vq = pan[(8 * I + r) * 4 + q];
        const double c = fma(lq[0], x01.x, fma(lq[1], x01.y, fma(lq[2], x2, vq)));
        X[I] = c * nrq;
        B[I] = c;
    }
    if ((r >> 2) == H) {
        // rows of P: X = Lam[q][a] / delta_q , B = -Lam[q][a]  (a = r & 3)
        const double la = lam_qa(lq, q, r & 3);
        X[K] = la * rq;
        B[K] = -la;
    }
    // The next block's diagonal tile first; its operands are formed while the
    // other DMMAs run.  Then the rest of the next panel's tile column and row,
    // so the next round can publish early; the remaining tiles last.
    if (K2 < NT) {
        constexpr int KG = K2 < NT ? K2 : 0;
        dmma(a[tix(KG, KG)][0], a[tix(KG, KG)][1], X[KG], B[KG]);
        gather_block<NT, KG, H2>(a, lane, f);
        ldl_block4(f, n - p2, cnt, flags);  // n - p2 <= 0: all padding, counts nothing
#pragma unroll
        for (int I = KG + 1; I < NT; ++I) dmma(a[tix(I, KG)][0], a[tix(I, KG)][1], X[I], B[KG]);
#pragma unroll
        for (int J = 0; J < KG; ++J) dmma(a[tix(KG, J)][0], a[tix(KG, J)][1], X[KG], B[J]);
    }
#pragma unroll
    for (int I = 0; I < NT; ++I)
#pragma unroll
        for (int J = 0; J <= I; ++J)
            if (I != K2 && J != K2) dmma(a[tix(I, J)][0], a[tix(I, J)][1], X[I], B[J]);
}

template <int NT, int R>
struct Rounds {
    static __device__ __forceinline__ void run(double (&a)[G<NT>::NTL][2], double *pan, int n, int lane,
                                               double (&f)[4][4], int &cnt, int &flags)
    {
        constexpr int K = R / 2, H = R % 2;
        if (8 * K + 4 * H < n) sweep_round<NT, K, H>(a, pan, n, lane, f, cnt, flags);
        Rounds<NT, R + 1>::run(a, pan, n, lane, f, cnt, flags);
    }
};
template <int NT>
struct Rounds<NT, 2 * NT> {
    static __device__ __forceinline__ void run(double (&)[G<NT>::NTL][2], double *, int, int, double (&)[4][4],
                                               int &, int &)
    {
    }
};

// -A^{-1} in place; returns the negative-pivot count, `bad` as in tiles.cuh.
// pan: G<NT>::PAN + 16 doubles of shared memory owned by this warp.
template <int NT>
__device__ __forceinline__ int warp_sweep_invert(double (&a)[G<NT>::NTL][2], double *pan, int n, int lane, int &bad)
{
    int cnt = 0, flags = 0;
    double f[4][4];
    gather_block<NT, 0, 0>(a, lane, f);
    ldl_block4(f, n, cnt, flags);
    Rounds<NT, 0>::run(a, pan, n, lane, f, cnt, flags);
    bad = flags_to_status(flags);
    return cnt;
}

// ---- element bookkeeping ----------------------------------------------------
// Row and column (global) of element s of tile (I, J) held by `lane`.
__device__ __forceinline__ int frow(int I, int lane) { return 8 * I + (lane >> 2); }
__device__ __forceinline__ int fcol(int J, int lane, int s) { return 8 * J + 2 * (lane & 3) + s; }

}  // namespace wf
}  // namespace mgpu
