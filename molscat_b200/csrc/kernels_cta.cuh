// LDMD / LDJ kernels for 40 < N <= 200: one CTA (4-16 warps) per matrix.
// Included by propagator.cu after kernels_frag.cuh.
//
// The lower 8x8 tiles of the matrix live in shared memory in the DMMA
// accumulator layout of warp_dmma.cuh ([t][lane][s], 512 bytes a tile), so
// VL and the 2HQ(C) table use exactly the same layout as the one-warp
// kernels.  The block sweep is the same four-pivots-per-round algorithm
// (warp_dmma.cuh states it):
//   1. thread i gathers row i of the panel A[i, P] from the lower triangle
//      and forms its operand rows c(i) = Lam A[i, P] (B) and
//      -c(i)/delta (X); rows of P carry -Lam^T and Lam^T/delta;   barrier
//   2. every warp loads the accumulators of its tiles (round robin), zeroes
//      the entries of row/column block P, issues A_IJ += X_I B_J (DMMA) and
//      stores the tile back.  The warp that owns the next pivot block's
//      diagonal tile does that tile first and factors the next block from it
//      (look-ahead), counting its pivots;                     barrier
// Elementwise parts of the step run over all tile elements with all threads.
#pragma once
#include "kernels_frag.cuh"

namespace mgpu {
namespace cta {

using wf::tix;

template <int NT, int W>
struct CG {
    static constexpr int NTL = NT * (NT + 1) / 2;
    static constexpr int NPAD = 8 * NT;
    static constexpr int NTHR = 32 * W;
    static constexpr int TD = NTL * 64;  // doubles of one tiled matrix
};

// Shared-memory carve-up (doubles) of one CTA: nmat tiled matrices, panel,
// X rows, F for two rounds, y14 / y14' / y23.
template <int NT, int W>
struct CSmem {
    static constexpr int PAN = CG<NT, W>::NPAD * 4;
    // the second panel / operand pair of the register-resident sweep, after the rest
    __host__ __device__ static constexpr size_t extra(int nmat)
    {
        return (size_t)nmat * CG<NT, W>::TD + 2 * PAN + 32 + 3 * CG<NT, W>::NPAD;
    }
    // + 32 doubles of slack: a padding tile's operand reads run up to 31 past the last buffer
    __host__ __device__ static constexpr size_t bytes(int nmat) { return (extra(nmat) + 2 * PAN + 32) * 8; }
};

struct TileRC {
    unsigned char I, J;
};

// element x of a tiled matrix -> (row, column)
__device__ __forceinline__ void elem_rc(const TileRC *__restrict__ tab, int x, int &i, int &j)
{
    const int t = x >> 6, l = (x >> 1) & 31, s = x & 1;
    i = 8 * tab[t].I + (l >> 2);
    j = 8 * tab[t].J + 2 * (l & 3) + s;
}

// Element (i, j) of the symmetric matrix, read from the lower triangle.
__device__ __forceinline__ double sym_elem(const double *tiles, int i, int j)
{
    const int R = i > j ? i : j, C = i > j ? j : i;
    return tiles[tix(R >> 3, C >> 3) * 64 + ((R & 7) * 4 + ((C & 7) >> 1)) * 2 + (C & 1)];
}

// The 4x4 block rows/cols p..p+3 (lower triangle) of the tiled matrix.
__device__ __forceinline__ void load_block4(const double *tiles, int p, double (&f)[4][4])
{
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j <= i; ++j) f[i][j] = sym_elem(tiles, p + i, p + j);
}

// -A^{-1} in place for the CTA's tiled matrix `tiles` (shared memory).
// Returns the negative-pivot count; `bad` as in tiles.cuh.
// The buffers are shared memory written and read by different threads across
// barriers, so none of the pointers is declared __restrict__ (that would let
// the compiler keep a thread's own earlier value in a register).
template <int NT, int W>
__device__ int cta_sweep_invert(double *tiles, double *pan, double *xs, double *fbuf, volatile int *cnt_flags, int n,
                                int &bad)
{
    using C = CG<NT, W>;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int r = lane >> 2, q = lane & 3;
    // operands of the first block, by warp 0
    if (warp == 0) {
        double f[4][4];
        load_block4(tiles, 0, f);
        int c = 0, fl = 0;
        wf::ldl_block4(f, n, c, fl);
        if (lane == 0) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) fbuf[i * 4 + j] = f[i][j];
            cnt_flags[0] = c;
            cnt_flags[1] = fl;
        }
    }
    __syncthreads();
    const int nround = (n + 3) >> 2;
    for (int rd = 0; rd < nround; ++rd) {
        const int p0 = 4 * rd, K = p0 >> 3, H = (p0 >> 2) & 1;
        const int p2 = p0 + 4, K2 = p2 >> 3;
        const double *F = fbuf + (rd & 1) * 16;
        // 1. operand rows: B = c = Lam A[i, P], X = -c / delta (rows of P:
        //    B = -Lam[.][a], X = Lam[.][a] / delta, a = i - p0)
        for (int i = tid; i < C::NPAD; i += C::NTHR) {
            double c[4], x[4];
            if (i >= p0 && i < p0 + 4) {
                const int a = i - p0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const double la = (k == a) ? 1.0 : (k > a ? F[k * 4 + a] : 0.0);
                    c[k] = -la;
                    x[k] = la * F[k * 5];
                }
            } else {
                double v[4];
#pragma unroll
                for (int m = 0; m < 4; ++m) v[m] = sym_elem(tiles, i, p0 + m);
                c[0] = v[0];
                c[1] = fma(F[4], v[0], v[1]);
                c[2] = fma(F[8], v[0], fma(F[9], v[1], v[2]));
                c[3] = fma(F[12], v[0], fma(F[13], v[1], fma(F[14], v[2], v[3])));
#pragma unroll
                for (int k = 0; k < 4; ++k) x[k] = c[k] * -F[k * 5];
            }
            *reinterpret_cast<double2 *>(pan + i * 4) = make_double2(c[0], c[1]);
            *reinterpret_cast<double2 *>(pan + i * 4 + 2) = make_double2(c[2], c[3]);
            *reinterpret_cast<double2 *>(xs + i * 4) = make_double2(x[0], x[1]);
            *reinterpret_cast<double2 *>(xs + i * 4 + 2) = make_double2(x[2], x[3]);
        }
        __syncthreads();
        // 2. trailing update, next pivot block's diagonal tile first
        const int tnext = (K2 < NT) ? tix(K2, K2) : -1;
        const int owner = tnext >= 0 ? tnext % W : -1;
        for (int pass = 0; pass < 2; ++pass) {
            for (int t = warp; t < C::NTL; t += W) {
                if ((pass == 0) != (t == tnext)) continue;
                int I = 0;
                while ((I + 1) * (I + 2) / 2 <= t) ++I;
                const int J = t - I * (I + 1) / 2;
                double2 cv = *reinterpret_cast<const double2 *>(tiles + t * 64 + lane * 2);
                if ((J == K && (q >> 1) == H) || (I == K && (r >> 2) == H)) cv.x = cv.y = 0.0;
                wf::dmma(cv.x, cv.y, xs[(8 * I + r) * 4 + q], pan[(8 * J + r) * 4 + q]);
                *reinterpret_cast<double2 *>(tiles + t * 64 + lane * 2) = cv;
            }
            if (pass == 0 && warp == owner && p2 < n) {
                // look-ahead: operands of the next block from the tile just written
                __syncwarp();
                double f[4][4];
                load_block4(tiles, p2, f);
                int c = 0, fl = 0;
                wf::ldl_block4(f, n - p2, c, fl);
                if (lane == 0) {
                    double *Fn = fbuf + ((rd + 1) & 1) * 16;
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) Fn[i * 4 + j] = f[i][j];
                    cnt_flags[0] += c;
                    cnt_flags[1] |= fl;
                }
            }
        }
        __syncthreads();
    }
    const int cnt = cnt_flags[0];
    bad = flags_to_status(cnt_flags[1]);
    __syncthreads();  // everyone has read the counters before they are reused
    return cnt;
}

// 1: the register-resident sweep alternates two panel / operand buffers and
// drops the round's closing barrier; 0: one buffer, three barriers a round.
#ifndef MGPU_CTA_DB
#define MGPU_CTA_DB 1
#endif

// The same sweep with the tiles held in registers for the whole inversion:
// warp w owns tiles [w*TPW, (w+1)*TPW) (TPW = ceil(NTL/W), row-major order so
// a warp's tiles share rows), loaded from shared memory at the start and
// stored back at the end.  A round then moves only the panel and the
// operands through shared memory instead of every tile:
//   0. the owners of tile column K (at and below the diagonal) and of tile
//      row K (left of it) publish A[i, P] into `pan` as the one-warp sweep
//      does;                                                      barrier
//   1. thread i turns its panel row into the operand rows c(i) (B, in place)
//      and -c(i)/delta (X), rows of P as in cta_sweep_invert;       barrier
//   2. every warp zeroes row/column block P in its tiles and issues the DMMAs,
//      the next pivot block's diagonal tile first; its owner gathers that
//      block with shuffles and factors it (look-ahead);            barrier
// Per tile the operands, the DMMA and its order are those of
// cta_sweep_invert, so the result is the same bit for bit.
template <int NT, int W>
__device__ int cta_sweep_invert_reg(double *tiles, double *pan0, double *xs0, double *fbuf, volatile int *cnt_flags,
                                    int n, const TileRC *tab, double *pan1, int &bad)
{
    using C = CG<NT, W>;
    constexpr int TPW = (C::NTL + W - 1) / W;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int r = lane >> 2, q = lane & 3;
    const int t0 = warp * TPW;
    double acc[TPW][2];
#pragma unroll
    for (int u = 0; u < TPW; ++u) {
        const int t = t0 + u;
        double2 v = make_double2(0.0, 0.0);
        if (t < C::NTL) v = *reinterpret_cast<const double2 *>(tiles + t * 64 + lane * 2);
        acc[u][0] = v.x;
        acc[u][1] = v.y;
    }
    // operands of the first block, by warp 0 (shared memory holds the matrix)
    if (warp == 0) {
        double f[4][4];
        load_block4(tiles, 0, f);
        int c = 0, fl = 0;
        wf::ldl_block4(f, n, c, fl);
        if (lane == 0) {
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) fbuf[i * 4 + j] = f[i][j];
            cnt_flags[0] = c;
            cnt_flags[1] = fl;
        }
    }
    __syncthreads();
    const int nround = (n + 3) >> 2;
    for (int rd = 0; rd < nround; ++rd) {
        const int p0 = 4 * rd, K = p0 >> 3, H = (p0 >> 2) & 1;
        const int p2 = p0 + 4, K2 = p2 >> 3, H2 = (p2 >> 2) & 1;
        const double *F = fbuf + (rd & 1) * 16;
#if MGPU_CTA_DB
        // alternate panel / operand buffers: a round's publication cannot
        // overwrite what a slower warp still reads in the previous round's
        // DMMAs, so the round needs no closing barrier
        double *pan = (rd & 1) ? pan1 : pan0;
        double *xs = (rd & 1) ? pan1 + CSmem<NT, W>::PAN : xs0;
#else
        double *pan = pan0;
        double *xs = xs0;
#endif
        // 0. publish A[i, P] from the lower triangle (row i -> pan[4i .. 4i+3]),
        //    then zero row / column block P in the tiles that hold it (tile
        //    row and tile column K, the only ones with entries there)
#pragma unroll
        for (int u = 0; u < TPW; ++u) {
            const TileRC ij = tab[t0 + u];
            const int I = ij.I, J = ij.J;
            if (I != K && J != K) continue;
            if (J == K && (q >> 1) == H && (I > K || H == 0)) {
                pan[(8 * I + r) * 4 + 2 * q - 4 * H] = acc[u][0];
                pan[(8 * I + r) * 4 + 2 * q - 4 * H + 1] = acc[u][1];
            }
            if (I == K && (r >> 2) == H && (J < K || (H == 1 && q < 2))) {
                pan[(8 * J + 2 * q) * 4 + (r & 3)] = acc[u][0];
                pan[(8 * J + 2 * q + 1) * 4 + (r & 3)] = acc[u][1];
            }
            if ((J == K && (q >> 1) == H) || (I == K && (r >> 2) == H)) acc[u][0] = acc[u][1] = 0.0;
        }
        __syncthreads();
        // 1. operand rows, in place in pan (B = c) and in xs (X)
        for (int i = tid; i < C::NPAD; i += C::NTHR) {
            double c[4], x[4];
            if (i >= p0 && i < p0 + 4) {
                const int a = i - p0;
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const double la = (k == a) ? 1.0 : (k > a ? F[k * 4 + a] : 0.0);
                    c[k] = -la;
                    x[k] = la * F[k * 5];
                }
            } else {
                const double2 v01 = *reinterpret_cast<const double2 *>(pan + i * 4);
                const double2 v23 = *reinterpret_cast<const double2 *>(pan + i * 4 + 2);
                c[0] = v01.x;
                c[1] = fma(F[4], v01.x, v01.y);
                c[2] = fma(F[8], v01.x, fma(F[9], v01.y, v23.x));
                c[3] = fma(F[12], v01.x, fma(F[13], v01.y, fma(F[14], v23.x, v23.y)));
#pragma unroll
                for (int k = 0; k < 4; ++k) x[k] = c[k] * -F[k * 5];
            }
            *reinterpret_cast<double2 *>(pan + i * 4) = make_double2(c[0], c[1]);
            *reinterpret_cast<double2 *>(pan + i * 4 + 2) = make_double2(c[2], c[3]);
            *reinterpret_cast<double2 *>(xs + i * 4) = make_double2(x[0], x[1]);
            *reinterpret_cast<double2 *>(xs + i * 4 + 2) = make_double2(x[2], x[3]);
        }
        __syncthreads();
        // 2. trailing update, the next pivot block's diagonal tile first
        const int tnext = (K2 < NT) ? tix(K2, K2) : -1;
        const int unext = tnext - t0;  // in [0, TPW) for the warp that owns it
        const bool own_next = unext >= 0 && unext < TPW;
        const double *xr = xs + r * 4 + q;   // X_I = xr[32 I], B_J = br[32 J]
        const double *br = pan + r * 4 + q;
        // (tab has W*TPW entries; those past NTL name a tile beyond the matrix
        // whose operand reads stay inside shared memory and whose result is
        // never stored, so the loops need no bound test)
#pragma unroll
        for (int pass = 0; pass < 2; ++pass) {
#pragma unroll
            for (int u = 0; u < TPW; ++u) {
                if ((pass == 0) != (u == unext)) continue;
                const TileRC ij = tab[t0 + u];
                wf::dmma(acc[u][0], acc[u][1], xr[32 * ij.I], br[32 * ij.J]);
            }
            // the look-ahead after this warp's other DMMAs are issued, so they
            // run while it factors
            if (pass == 1 && own_next && p2 < n) {
                // look-ahead: the next block's 4x4 from the tile just updated, by shuffles
                double v0 = 0.0, v1 = 0.0;
#pragma unroll
                for (int u = 0; u < TPW; ++u)
                    if (t0 + u == tnext) {
                        v0 = acc[u][0];
                        v1 = acc[u][1];
                    }
                double f[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j <= i; ++j) {
                        const int src = (4 * H2 + i) * 4 + 2 * H2 + (j >> 1);
                        const double a0 = __shfl_sync(0xffffffffu, v0, src);
                        const double a1 = __shfl_sync(0xffffffffu, v1, src);
                        f[i][j] = (j & 1) ? a1 : a0;
                    }
                int c = 0, fl = 0;
                wf::ldl_block4(f, n - p2, c, fl);
                if (lane == 0) {
                    double *Fn = fbuf + ((rd + 1) & 1) * 16;
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < 4; ++j) Fn[i * 4 + j] = f[i][j];
                    cnt_flags[0] += c;
                    cnt_flags[1] |= fl;
                }
            }
        }
#if !MGPU_CTA_DB
        __syncthreads();
#endif
    }
#if MGPU_CTA_DB
    __syncthreads();  // the last round's look-ahead counters are in
#endif
#pragma unroll
    for (int u = 0; u < TPW; ++u) {
        const int t = t0 + u;
        if (t < C::NTL) *reinterpret_cast<double2 *>(tiles + t * 64 + lane * 2) = make_double2(acc[u][0], acc[u][1]);
    }
    const int cnt = cnt_flags[0];
    bad = flags_to_status(cnt_flags[1]);
    __syncthreads();  // every tile is back and the counters are read before they are reused
    return cnt;
}

// The sweep the kernels use: tiles in registers from NT = MGPU_CTA_REG_NT up
// (N > 80: 1.1x at N = 96, 1.3x at 106, 2.1x at 150 and 200 on B200, double
// buffered), in shared memory below it (where more CTAs per SM make up for
// it: 0.76x at N = 48, equal at 72 with the tiles in registers).  Both give
// the same result bit for bit.
#ifndef MGPU_CTA_REG_NT
#define MGPU_CTA_REG_NT 12
#endif
template <int NT, int W>
__device__ __forceinline__ int cta_invert(double *tiles, double *pan, double *xs, double *fbuf, volatile int *cnt_flags,
                                          int n, const TileRC *tab, double *extra, int &bad)
{
    if constexpr (NT >= MGPU_CTA_REG_NT) {
        return cta_sweep_invert_reg<NT, W>(tiles, pan, xs, fbuf, cnt_flags, n, tab, extra, bad);
    } else {
        (void)tab;
        (void)extra;
        return cta_sweep_invert<NT, W>(tiles, pan, xs, fbuf, cnt_flags, n, bad);
    }
}

// W(R) for element x (HAMMAT + SUMLAM), optionally with the diagonal terms.
__device__ __forceinline__ double w_elem(const SysDev &S, const double *__restrict__ P, int x, int i, int j, int ir,
                                         double ered, bool diag_terms)
{
    const size_t td = (size_t)S.ntiles * 64;
    double w = 0.0;
    if (S.ivlfl <= 0) {
        for (int l = 0; l < S.nham; ++l) w = fma(__ldg(S.vlt + l * td + x), __ldg(P + l), w);
    } else {
        for (int l = 0; l < S.nham; ++l) {
            const double v = __ldg(S.vlt + l * td + x);
            if (v != 0.0) w = fma(v, __ldg(P + __ldg(S.ivt + l * td + x)), w);
        }
    }
    if (diag_terms && i == j && i < S.n) {
        const double R = __ldg(S.rtab + ir);
        const double rsq = fmin(1.0 / (R * R), 1.0e16);
        if (S.nrsq == 0) w += rsq * S.cent[i];
        if (S.nconst == 0) w += S.eint[i];
        if (S.conlen > 0.0) {
            const double c2 = S.conlen * S.conlen;
            w += R * R / (c2 * c2);
        }
        w -= ered;
    }
    return w;
}

// Tile t -> (I, J); entries from NTL up to the padded count tabn<NT, W>()
// name (NT, NT), a tile beyond the matrix (see cta_sweep_invert_reg).
template <int NT, int W>
__host__ __device__ constexpr int tabn() { return W * ((CG<NT, W>::NTL + W - 1) / W); }

template <int NT, int W>
__device__ __forceinline__ void build_table(TileRC *tab)
{
    for (int t = threadIdx.x; t < tabn<NT, W>(); t += CG<NT, W>::NTHR) {
        if (t >= CG<NT, W>::NTL) {
            tab[t].I = tab[t].J = (unsigned char)NT;
            continue;
        }
        int I = 0;
        while ((I + 1) * (I + 2) / 2 <= t) ++I;
        tab[t].I = (unsigned char)I;
        tab[t].J = (unsigned char)(t - I * (I + 1) / 2);
    }
}

// ---------------------------------------------------------------------------
// MDPROP energy-independent half: one CTA per (step, system).
// ---------------------------------------------------------------------------
template <int NT, int W>
__global__ void __launch_bounds__(32 * W)
ldmd_prep_cta_kernel(const SysDev *__restrict__ systems, const int *__restrict__ sys_list)
{
    using C = CG<NT, W>;
    extern __shared__ __align__(16) double sm[];
    __shared__ TileRC tab[tabn<NT, W>()];
    __shared__ int cf[2];
    __shared__ SysDev s_sys;
    if (threadIdx.x == 0) s_sys = systems[sys_list[blockIdx.y]];
    build_table<NT, W>(tab);
    __syncthreads();
    const SysDev &S = s_sys;
    const int k = blockIdx.x + 1;
    if (k > S.nstep) return;  // whole CTA
    double *tiles = sm;
    double *pan = tiles + C::TD;
    double *xs = pan + CSmem<NT, W>::PAN;
    double *fbuf = xs + CSmem<NT, W>::PAN;
    const double h = S.dr / 2.0;
    const double d1 = h * h / 3.0;
    const double d4 = -d1 / 16.0;
    const double *P = S.ptab + (size_t)(2 * k - 1) * S.nham;
    for (int x = threadIdx.x; x < C::TD; x += C::NTHR) {
        int i, j;
        elem_rc(tab, x, i, j);
        const double w = w_elem(S, P, x, i, j, 2 * k - 1, 0.0, false);
        tiles[x] = (i == j) ? (i < S.n ? 0.125 : 0.0) : d4 * w;
    }
    __syncthreads();
    int bad = SWEEP_OK;
    const int cnt = cta_invert<NT, W>(tiles, pan, xs, fbuf, cf, S.n, tab, sm + CSmem<NT, W>::extra(1), bad);
    if (bad != SWEEP_OK) {
        if (threadIdx.x == 0) {
            atomicMax(&S.prep[1], bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE);
            atomicMin(&S.prep[2], k);
        }
        return;
    }
    if (threadIdx.x == 0 && cnt) atomicAdd(&S.prep[0], cnt);
    double *qk = S.q + (size_t)(k - 1) * C::TD;
    for (int x = threadIdx.x; x < C::TD; x += C::NTHR) {
        int i, j;
        elem_rc(tab, x, i, j);
        // tiles = -U^{-1};  2HQ(C) = U^{-1} - 8I
        qk[x] = (i >= S.n || j >= S.n) ? 0.0 : (i == j ? -tiles[x] - 8.0 : -tiles[x]);
    }
}

// ---------------------------------------------------------------------------
// MDPROP step loop, one CTA per job.
// ---------------------------------------------------------------------------
template <int NT, int W>
__global__ void __launch_bounds__(32 * W)
ldmd_prop_cta_kernel(const SysDev *__restrict__ systems, const JobDev *__restrict__ jobs, double *__restrict__ y,
                     int *__restrict__ nodes_out, int *__restrict__ status_out, int *__restrict__ kfail_out)
{
    using C = CG<NT, W>;
    extern __shared__ __align__(16) double sm[];
    __shared__ TileRC tab[tabn<NT, W>()];
    __shared__ int cf[2];
    __shared__ int s_stop;
    __shared__ SysDev s_sys;
    const JobDev job = jobs[blockIdx.x];
    if (threadIdx.x == 0) s_sys = systems[job.sys];
    build_table<NT, W>(tab);
    __syncthreads();
    const SysDev &S = s_sys;
    const int tid = threadIdx.x;
    double *tiles = sm;
    double *pan = tiles + C::TD;
    double *xs = pan + CSmem<NT, W>::PAN;
    double *fbuf = xs + CSmem<NT, W>::PAN;
    double *s_y14 = fbuf + 32;
    double *s_y14b = s_y14 + C::NPAD;
    double *s_y23 = s_y14b + C::NPAD;
    const int n = S.n;
    const int nstep = S.nstep;
    const double ered = job.ered;
    if (S.prep[1] != 0) {
        if (tid == 0) {
            status_out[job.out] = S.prep[1];
            kfail_out[job.out] = S.prep[2];
            nodes_out[job.out] = 0;
        }
        return;
    }
    const double h = S.dr / 2.0;
    const double d1 = h * h / 3.0;
    const double d2 = 2.0 * d1;
    const double half = 0.5 * h;
    double *yj = y + job.yoff;
    for (int i = tid; i < C::NPAD; i += C::NTHR) s_y14[i] = s_y14b[i] = s_y23[i] = 0.0;
    {
        const double *P = S.ptab;
        for (int x = tid; x < C::TD; x += C::NTHR) {
            int i, j;
            elem_rc(tab, x, i, j);
            const int lo = i < j ? i : j, hi = i < j ? j : i;
            const double y0 = (i < n && j < n) ? yj[(size_t)lo * n + hi] : 0.0;
            tiles[x] = h * y0 + d1 * w_elem(S, P, x, i, j, 0, ered, true);  // mdprop.f:89-93
        }
    }
    __syncthreads();
    int nodes = 0, status = MGPU_OK, kfail = 0;
    const unsigned long long t0 = global_ns();
    for (int k = 1; k <= nstep; ++k) {
        if (stop_poll_step(k)) {  // host cancel / time limit: thread 0's reading for the CTA
            if (tid == 0) s_stop = stop_requested(S.ctl, t0);
            __syncthreads();  // the next write comes kStopPoll steps (and their barriers) later
            const int stop = s_stop;
            if (stop != MGPU_OK) {
                status = stop;
                kfail = k;
                break;
            }
        }
        // reference-potential solutions (mdprop.f:143-164)
        for (int i = tid; i < n; i += C::NTHR) {
            const double wref = wf::w_diag_frag<NT>(S, i, 2 * k - 1, ered);
            double y14, y23;
            ref_solutions(wref, half, y14, y23);
            s_y14[i] = y14;
            s_y14b[i] = y14 - d1 * wref;
            s_y23[i] = y23;
        }
        __syncthreads();
        for (int x = tid; x < C::TD; x += C::NTHR) {
            int i, j;
            elem_rc(tab, x, i, j);
            if (i == j) tiles[x] += s_y14b[i];
        }
        __syncthreads();
        int bad = SWEEP_OK;
        nodes += cta_invert<NT, W>(tiles, pan, xs, fbuf, cf, n, tab, sm + CSmem<NT, W>::extra(1), bad);
        if (bad != SWEEP_OK) {
            status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        const double *qk = S.q + (size_t)(k - 1) * C::TD;
        for (int x = tid; x < C::TD; x += C::NTHR) {
            int i, j;
            elem_rc(tab, x, i, j);
            // Y = 2HQ(C) + 2 Y14 - Y23 Y^-1 Y23  (tiles hold -Y^-1), mdprop.f:156,181-185
            double v = __ldg(qk + x) + s_y23[i] * tiles[x] * s_y23[j];
            if (i == j) v += 2.0 * s_y14[i];
            tiles[x] = v;
        }
        __syncthreads();
        nodes += cta_invert<NT, W>(tiles, pan, xs, fbuf, cf, n, tab, sm + CSmem<NT, W>::extra(1), bad);
        if (bad != SWEEP_OK) {
            status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        const double dd = (k == nstep) ? d1 : d2;
        const double *P = S.ptab + (size_t)(2 * k) * S.nham;
        for (int x = tid; x < C::TD; x += C::NTHR) {
            int i, j;
            elem_rc(tab, x, i, j);
            // Y = D2 W(B) - Y23 Y^-1 Y23 + Y14'  (mdprop.f:196-230)
            double v = dd * w_elem(S, P, x, i, j, 2 * k, ered, true) + s_y23[i] * tiles[x] * s_y23[j];
            if (i == j) v += s_y14b[i];
            tiles[x] = v;
        }
        __syncthreads();
    }
    if (status == MGPU_OK) {
        const double hi = 1.0 / h;
        for (int x = tid; x < C::TD; x += C::NTHR) {
            int i, j;
            elem_rc(tab, x, i, j);
            if (i < n && j <= i) {
                const double v = hi * tiles[x];
                yj[(size_t)j * n + i] = v;
                yj[(size_t)i * n + j] = v;
            }
        }
    }
    if (tid == 0) {
        status_out[job.out] = status;
        kfail_out[job.out] = kfail;
        nodes_out[job.out] = status == MGPU_OK ? nodes - S.prep[0] : 0;
    }
}

// ---------------------------------------------------------------------------
// LDPROP step loop, one CTA per job (two tiled matrices in shared memory).
// ---------------------------------------------------------------------------
template <int NT, int W>
__global__ void __launch_bounds__(32 * W)
ldj_prop_cta_kernel(const SysDev *__restrict__ systems, const JobDev *__restrict__ jobs, double *__restrict__ y,
                    int *__restrict__ nodes_out, int *__restrict__ status_out, int *__restrict__ kfail_out)
{
    using C = CG<NT, W>;
    extern __shared__ __align__(16) double sm[];
    __shared__ TileRC tab[tabn<NT, W>()];
    __shared__ int cf[2];
    __shared__ int s_stop;
    __shared__ SysDev s_sys;
    const JobDev job = jobs[blockIdx.x];
    if (threadIdx.x == 0) s_sys = systems[job.sys];
    build_table<NT, W>(tab);
    __syncthreads();
    const SysDev &S = s_sys;
    const int tid = threadIdx.x;
    double *zt = sm;
    double *ut = zt + C::TD;
    double *pan = ut + C::TD;
    double *xs = pan + CSmem<NT, W>::PAN;
    double *fbuf = xs + CSmem<NT, W>::PAN;
    const int n = S.n;
    const double ered = job.ered;
    const double h = S.dr / 2.0;
    const double d1 = h * h / 3.0;
    const double d2 = 2.0 * d1;
    const double d4 = -d1 / 16.0;
    double *yj = y + job.yoff;
    for (int x = tid; x < C::TD; x += C::NTHR) {
        int i, j;
        elem_rc(tab, x, i, j);
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        const double y0 = (i < n && j < n) ? yj[(size_t)lo * n + hi] : 0.0;
        zt[x] = h * y0 + d1 * w_elem(S, S.ptab, x, i, j, 0, ered, true) + ((i == j && i < n) ? 1.0 : 0.0);
    }
    __syncthreads();
    int nodes = 0, status = MGPU_OK, kfail = 0;
    const unsigned long long t0 = global_ns();
    for (int k = 1; k <= S.nstep; ++k) {
        if (stop_poll_step(k)) {
            if (tid == 0) s_stop = stop_requested(S.ctl, t0);
            __syncthreads();  // the next write comes kStopPoll steps (and their barriers) later
            const int stop = s_stop;
            if (stop != MGPU_OK) {
                status = stop;
                kfail = k;
                break;
            }
        }
        const double *P = S.ptab + (size_t)(2 * k - 1) * S.nham;
        for (int x = tid; x < C::TD; x += C::NTHR) {
            int i, j;
            elem_rc(tab, x, i, j);
            ut[x] = d4 * w_elem(S, P, x, i, j, 2 * k - 1, ered, true) + ((i == j && i < n) ? 0.125 : 0.0);
        }
        __syncthreads();
        int bad = SWEEP_OK, bad2 = SWEEP_OK;
        const int ncu = cta_invert<NT, W>(ut, pan, xs, fbuf, cf, n, tab, sm + CSmem<NT, W>::extra(2), bad);   // ldprop.f:78
        const int ncz = cta_invert<NT, W>(zt, pan, xs, fbuf, cf, n, tab, sm + CSmem<NT, W>::extra(2), bad2);  // ldprop.f:83
        if (bad != SWEEP_OK || bad2 != SWEEP_OK) {
            status = (bad == SWEEP_ZERO || bad2 == SWEEP_ZERO) ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        nodes += ncz;
        for (int x = tid; x < C::TD; x += C::NTHR) {
            int i, j;
            elem_rc(tab, x, i, j);
            zt[x] = -ut[x] + zt[x] - ((i == j && i < n) ? 6.0 : 0.0);  // ldprop.f:92-97
        }
        __syncthreads();
        const int ncz2 = cta_invert<NT, W>(zt, pan, xs, fbuf, cf, n, tab, sm + CSmem<NT, W>::extra(2), bad);  // ldprop.f:99
        if (bad != SWEEP_OK) {
            status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        nodes += ncz2 - ncu;
        const double dd = (k == S.nstep) ? d1 : d2;
        const double *PB = S.ptab + (size_t)(2 * k) * S.nham;
        for (int x = tid; x < C::TD; x += C::NTHR) {
            int i, j;
            elem_rc(tab, x, i, j);
            zt[x] = dd * w_elem(S, PB, x, i, j, 2 * k, ered, true) + ((i == j && i < n) ? 2.0 : 0.0) + zt[x];
        }
        __syncthreads();
    }
    if (status == MGPU_OK) {
        const double hi = 1.0 / h;
        for (int x = tid; x < C::TD; x += C::NTHR) {
            int i, j;
            elem_rc(tab, x, i, j);
            if (i < n && j <= i) {
                const double v = hi * zt[x] - ((i == j) ? hi : 0.0);
                yj[(size_t)j * n + i] = v;
                yj[(size_t)i * n + j] = v;
            }
        }
    }
    if (tid == 0) {
        status_out[job.out] = status;
        kfail_out[job.out] = kfail;
        nodes_out[job.out] = status == MGPU_OK ? nodes : 0;
    }
}

// ---------------------------------------------------------------------------
// MGPROP step loop on one CTA per job (40 < N <= 200): the one-warp
// kernel's stages (kernels_frag.cuh, ldmg_prop_frag_kernel) with Y as tiles
// in shared memory and the CTA sweep for the inversions.
// ---------------------------------------------------------------------------
template <int NT, int W>
__global__ void __launch_bounds__(32 * W)
ldmg_prop_cta_kernel(const SysDev *__restrict__ systems, const JobDev *__restrict__ jobs, int method,
                     double *__restrict__ y, int *__restrict__ nodes_out, int *__restrict__ status_out,
                     int *__restrict__ kfail_out)
{
    using C = CG<NT, W>;
    extern __shared__ __align__(16) double sm[];
    __shared__ TileRC tab[tabn<NT, W>()];
    __shared__ int cf[2];
    __shared__ int s_stop;
    __shared__ SysDev s_sys;
    const JobDev job = jobs[blockIdx.x];
    if (threadIdx.x == 0) s_sys = systems[job.sys];
    build_table<NT, W>(tab);
    __syncthreads();
    const SysDev &S = s_sys;
    const wf::MGCoef &M = wf::c_mg[method];
    const int tid = threadIdx.x;
    double *yt = sm;
    double *pan = yt + C::TD;
    double *xs = pan + CSmem<NT, W>::PAN;
    double *fbuf = xs + CSmem<NT, W>::PAN;
    const int n = S.n;
    const double ered = job.ered;
    const double h = S.dr;
    double *yj = y + job.yoff;
    for (int x = tid; x < C::TD; x += C::NTHR) {
        int i, j;
        elem_rc(tab, x, i, j);
        const int lo = i < j ? i : j, hi = i < j ? j : i;
        yt[x] = (i < n && j < n) ? yj[(size_t)lo * n + hi] : 0.0;
    }
    __syncthreads();
    int nodes = 0, status = MGPU_OK, kfail = 0;
    const unsigned long long t0 = global_ns();
    for (int sec = 0; sec < S.nstep && status == MGPU_OK; ++sec) {
        if (stop_poll_step(sec + 1)) {
            if (tid == 0) s_stop = stop_requested(S.ctl, t0);
            __syncthreads();  // the next write comes kStopPoll sectors (and their barriers) later
            const int stop = s_stop;
            if (stop != MGPU_OK) {
                status = stop;
                kfail = sec + 1;
                break;
            }
        }
        for (int k = 0; k < M.m; ++k) {
            const int ir = sec * M.stride + k;
            const double *P = S.ptab + (size_t)ir * S.nham;
            const double bh = M.b[k] * h, ak = M.a[k], ah = ak * h;
            for (int x = tid; x < C::TD; x += C::NTHR) {
                int i, j;
                elem_rc(tab, x, i, j);
                const double xv = fma(bh, w_elem(S, P, x, i, j, ir, ered, true), yt[x]);  // X = Y + b_k h W
                yt[x] = ak == 0.0 ? xv : ah * xv + ((i == j && i < n) ? 1.0 : 0.0);      // I + a_k h X
            }
            __syncthreads();
            if (ak == 0.0) continue;
            int bad = SWEEP_OK;
            const int cnt = cta_invert<NT, W>(yt, pan, xs, fbuf, cf, n, tab, sm + CSmem<NT, W>::extra(1), bad);
            if (bad != SWEEP_OK) {
                status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
                kfail = sec + 1;
                break;
            }
            nodes += ak >= 0.0 ? cnt : -cnt;
            const double d1 = 1.0 / ah;
            for (int x = tid; x < C::TD; x += C::NTHR) {
                int i, j;
                elem_rc(tab, x, i, j);
                yt[x] = (yt[x] + ((i == j && i < n) ? 1.0 : 0.0)) * d1;  // [I - inverse]/(a_k h)
            }
            __syncthreads();
        }
    }
    if (status == MGPU_OK) {
        for (int x = tid; x < C::TD; x += C::NTHR) {
            int i, j;
            elem_rc(tab, x, i, j);
            if (i < n && j <= i) {
                yj[(size_t)j * n + i] = yt[x];
                yj[(size_t)i * n + j] = yt[x];
            }
        }
    }
    if (tid == 0) {
        status_out[job.out] = status;
        kfail_out[job.out] = kfail;
        nodes_out[job.out] = status == MGPU_OK ? nodes : 0;
    }
}

}  // namespace cta
}  // namespace mgpu
