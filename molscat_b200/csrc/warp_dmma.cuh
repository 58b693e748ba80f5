// One warp per symmetric matrix, held in FP64 tensor-core (DMMA) fragments.
//
// The matrix (padded to NPAD = 8*NT) is cut into 8x8 tiles; the lower
// triangle of tiles, t = I*(I+1)/2 + J (I >= J), lives in registers in the
// accumulator layout of mma.sync.m8n8k4.f64: lane l holds elements
// (row 8I + (l>>2), col 8J + 2(l&3) + s), s = 0,1.  Diagonal tiles hold both
// triangles.  Padding rows/columns are zero.
//
// Inversion is the symmetric Gauss-Jordan sweep done four pivots at a time
// (block sweep).  For the pivot block P = {p0..p0+3} with D = A_PP and
// F = -D^{-1}:
//     A_ij += (A_iP F) A_Pj          i,j not in P
//     A_iP  = -(A_iP F) ,  A_Pj = -(F A_Pj) ,  A_PP = F
// which after all blocks leaves -A^{-1} (the same result as the scalar sweep
// in tiles.cuh).  As there, the owners zero row/column block P and the
// operands carry the pivot block, so every tile gets the same update
//     A_IJ += X_I B_J          (one m8n8k4 DMMA per lower tile)
// with X_I = A_{I,P} F (rows of P replaced by -F) and B_J = A_{P,J}
// (columns of P replaced by -I).  The panel A_{:,P} goes through a small
// per-warp shared-memory buffer.
//
// F comes from D by 2x2 blocks (two reciprocals per block of four pivots).
// The pivots of that block LDL^T are those of the unpivoted LDL^T SYMINV
// forms (syminv.f:27-49): d1 = a00, d2 = det(A)/a00 for the leading 2x2 A,
// d3, d4 likewise for the Schur complement S = C - B A^{-1} B^T.  Their
// negative count is SYMINV's KOUNT (and DSYNEG's inertia by Sylvester's
// law); a zero a00 or det is the reference's IFAIL = N+1.
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

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// -D^{-1} of a symmetric 4x4 block by 2x2 blocks, counting negative pivots
// of the first `nreal` rows (the rest are padding and are treated as 1).
__device__ __forceinline__ void neg_inverse4(double d[4][4], int nreal, int &cnt, int &flags)
{
    // padding rows/columns of the matrix are zero off the diagonal; a padding
    // pivot is taken as exactly 1 (not counted, never singular)
#pragma unroll
    for (int i = 0; i < 4; ++i) d[i][i] = (i >= nreal) ? 1.0 : d[i][i];
    // leading 2x2 block A
    const double a00 = d[0][0], a01 = d[1][0], a11 = d[1][1];
    const double detA = fma(a00, a11, -a01 * a01);
    const double rA = pivot_reciprocal(detA);
    const double i00 = a11 * rA, i01 = -a01 * rA, i11 = a00 * rA;  // A^{-1}
    // W = B A^{-1}, B = rows 2,3 x cols 0,1
    const double b00 = d[2][0], b01 = d[2][1], b10 = d[3][0], b11 = d[3][1];
    const double w00 = fma(b00, i00, b01 * i01), w01 = fma(b00, i01, b01 * i11);
    const double w10 = fma(b10, i00, b11 * i01), w11 = fma(b10, i01, b11 * i11);
    // Schur complement S = C - W B^T
    const double s00 = d[2][2] - fma(w00, b00, w01 * b01);
    const double s01 = d[3][2] - fma(w10, b00, w11 * b01);
    const double s11 = d[3][3] - fma(w10, b10, w11 * b11);
    const double detS = fma(s00, s11, -s01 * s01);
    const double rS = pivot_reciprocal(detS);
    const double j00 = s11 * rS, j01 = -s01 * rS, j11 = s00 * rS;  // S^{-1}
    // pivots d1 = a00, d2 = detA/a00, d3 = s00, d4 = detS/s00 (padding rows are
    // exact unit pivots: positive, finite, so counting all four is exact)
    flags |= pivot_flags(a00) | pivot_flags(detA) | pivot_flags(s00) | pivot_flags(detS);
    cnt += (a00 < 0.0) + ((detA < 0.0) != (a00 < 0.0)) + (s00 < 0.0) + ((detS < 0.0) != (s00 < 0.0));
    // E21 = -S^{-1} W ; E11 = A^{-1} - W^T E21 ; E22 = S^{-1}
    const double e20 = -fma(j00, w00, j01 * w10), e21 = -fma(j00, w01, j01 * w11);
    const double e30 = -fma(j01, w00, j11 * w10), e31 = -fma(j01, w01, j11 * w11);
    const double e00 = i00 - fma(w00, e20, w10 * e30);
    const double e01 = i01 - fma(w00, e21, w10 * e31);
    const double e11 = i11 - fma(w01, e21, w11 * e31);
    // store F = -E (symmetric)
    d[0][0] = -e00; d[0][1] = d[1][0] = -e01; d[1][1] = -e11;
    d[2][0] = d[0][2] = -e20; d[2][1] = d[1][2] = -e21;
    d[3][0] = d[0][3] = -e30; d[3][1] = d[1][3] = -e31;
    d[2][2] = -j00; d[3][2] = d[2][3] = -j01; d[3][3] = -j11;
}

__device__ __forceinline__ double sel4(const double (&v)[4], int i)
{
    double x = v[0];
    x = (i == 1) ? v[1] : x;
    x = (i == 2) ? v[2] : x;
    x = (i == 3) ? v[3] : x;
    return x;
}

// Gather the 4x4 pivot block rows/cols 4H..4H+3 of diagonal tile (K, K)
// into every lane with shuffles: element (i, j) sits in lane
// (4H+i)*4 + 2H + (j>>1), slot j&1.  Symmetric, so ten shuffles.
template <int NT, int K, int H>
__device__ __forceinline__ void gather_block(const double (&a)[G<NT>::NTL][2], int lane, double (&f)[4][4])
{
    (void)lane;
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = i; j < 4; ++j) {
            const int src = (4 * H + i) * 4 + 2 * H + (j >> 1);
            const double v = __shfl_sync(0xffffffffu, a[tix(K, K)][j & 1], src);
            f[i][j] = v;
            f[j][i] = v;
        }
}

// One block of four pivots, tile column K, half H (p0 = 8K + 4H).  f holds
// F = -D^{-1} of this block on entry and the next block's on exit (computed
// right after the next block's diagonal tile is updated, so its latency
// overlaps the rest of this block's DMMAs).
template <int NT, int K, int H>
__device__ __forceinline__ void sweep_round(double (&a)[G<NT>::NTL][2], double *__restrict__ pan, int n,
                                            int lane, double (&f)[4][4], int &cnt, int &flags)
{
    const int r = lane >> 2, q = lane & 3;
    constexpr int K2 = H ? K + 1 : K;  // next block
    constexpr int H2 = H ? 0 : 1;
    constexpr int p2 = 8 * K2 + 4 * H2;  // first pivot of the next block
    // publish the panel A[:, P] (row i -> pan[4i .. 4i+3])
    __syncwarp();
    if ((q >> 1) == H) {
#pragma unroll
        for (int I = K; I < NT; ++I) {
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
    }
    __syncwarp();
    double fq[4];  // column q of F
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        double x = f[m][0];
        x = (q == 1) ? f[m][1] : x;
        x = (q == 2) ? f[m][2] : x;
        x = (q == 3) ? f[m][3] : x;
        fq[m] = x;
    }
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
        const double2 x01 = row[0], x23 = row[1];
        X[I] = fma(x01.x, fq[0], fma(x01.y, fq[1], fma(x23.x, fq[2], x23.y * fq[3])));
        B[I] = pan[(8 * I + r) * 4 + q];
    }
    if ((r >> 2) == H) {
        // rows of P: X = -F ; columns of P: B = -I
        X[K] = -sel4(fq, r & 3);
        B[K] = (q == (r & 3)) ? -1.0 : 0.0;
    }
    // The next block's diagonal tile first; its F is computed while the other
    // DMMAs run.  Then the rest of the next panel's tile column and row, so
    // the next round can publish early; the remaining tiles last.
    if (K2 < NT) {
        constexpr int KG = K2 < NT ? K2 : 0;
        dmma(a[tix(KG, KG)][0], a[tix(KG, KG)][1], X[KG], B[KG]);
        gather_block<NT, KG, H2>(a, lane, f);
        neg_inverse4(f, n - p2, cnt, flags);  // n - p2 <= 0: all padding, counts nothing
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
    neg_inverse4(f, n, cnt, flags);
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
