// Register-tiled symmetric matrices for the log-derivative step kernels.
//
// One CTA owns one N x N symmetric matrix (padded to NPAD = T*NT).  The lower
// triangle is cut into T x T tiles, tile t = I*(I+1)/2 + J (I >= J), and
// thread t keeps its tile in registers.  Diagonal tiles hold both triangles
// (kept symmetric by every update).  Padding rows/columns are exactly zero and
// stay zero, so they never contribute.
//
// Inversion is the symmetric Gauss-Jordan "sweep": for k = 0..n-1 with pivot
// d = a_kk, p = 1/d,
//     a_ij -= a_ik a_kj p   (i,j != k),   a_ik = a_ki = a_ik p,   a_kk = -p
// which leaves -A^{-1}.  The pivots d are the D of the unpivoted LDL^T that
// SYMINV forms (syminv.f:27-49), so the number of negative pivots is SYMINV's
// KOUNT and, by Sylvester's law of inertia, the DSYNEG count of SYMINL
// (dsyneg.f) for the N > 30 matrices the reference factors with DSYTRF.
// A pivot that is exactly zero is the reference's IFAIL = N+1 (syminv.f:95).
// The work is N^3/2 FMA per inversion (only the lower triangle), the same N^3
// flops the reference's SYMINV spends.
//
// Every thread runs the same rank-1 FMA update: the owners of row/column k
// zero those entries when they publish column k, and the broadcast vectors
// carry x_k = -1 and y_k = -p, so  a_ij - x_i y_j  yields v_i p on column k,
// v_j p on row k and -p on the pivot without a divergent special case.  The
// pivot index only enters through uniform switches (same k in every thread).
#pragma once
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdint.h>

namespace mgpu {

template <int T, int NT>
struct Geom {
    static constexpr int NPAD = T * NT;
    static constexpr int NTILES = NT * (NT + 1) / 2;
    static constexpr int NTHR = ((NTILES + 31) / 32) * 32;
    static constexpr int TT = T * T;
    static constexpr int VS = NPAD + 2;  // published column + reciprocal pivot (+pad, 16-B multiple)
    // resident CTAs per SM the register budget is sized for (<= 128 registers a thread)
    static constexpr int MINB = (65536 / (NTHR * 128)) < 1 ? 1 : (65536 / (NTHR * 128)) > 16 ? 16 : (65536 / (NTHR * 128));
};

__device__ __forceinline__ void tile_of(int t, int &I, int &J)
{
    int i = 0;
    while ((i + 1) * (i + 2) / 2 <= t) ++i;
    I = i;
    J = t - i * (i + 1) / 2;
}

// Reciprocal of a pivot: hardware seed (rcp.approx.ftz.f64, about 2^-23
// relative error) refined by one step of the third-order iteration
//     e = 1 - d r,   r <- r + r (e + e^2)
// (Newton-Raphson with the quadratic correction term; the error goes from e
// to about e^3, see e.g. J.-M. Muller et al., Handbook of Floating-Point
// Arithmetic, ch. 5).  Magnitudes outside [2^-1000, 2^1000] are brought in
// range by an exact power-of-two scaling, so the code has no branch.  Within
// one ulp of the correctly rounded 1/d (checked against 1.0/x on the GPU).
__device__ __forceinline__ double pivot_reciprocal(double d)
{
    const double ad = fabs(d);
    const double sc = ad > 0x1p+1000 ? 0x1p-512 : (ad < 0x1p-1000 ? 0x1p+512 : 1.0);
    const double ds = d * sc;
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(ds));
    const double e = fma(-ds, r, 1.0);
    const double t = fma(e, e, e);
    return fma(r, t, r) * sc;
}

// Publish column k (and 1/a_kk) into dst and zero this thread's entries of
// row and column k.  Column k's lower part lives in tile column K, its upper
// part (equal by symmetry) in tile row K.  Branch-free: predicated stores and
// selects, so threads that own nothing of row/column k run the same code.
template <int T, int NPAD, int KK>
__device__ __forceinline__ void publish_clear_kk(double (&a)[T][T], double *dst, int K, int I, int J,
                                                 bool act = true)
{
    const bool colown = act && (J == K);            // publishes a[.][KK]: column k, rows of tile row I
    const bool rowown = act && (I == K) && (J != K);  // publishes a[KK][.]: row k = column k by symmetry
    const bool diag = act && (I == K) && (J == K);
    const double dv = diag ? a[KK][KK] : 1.0;
    const double pinv = pivot_reciprocal(dv);
#pragma unroll
    for (int r = 0; r < T; ++r)
        if (colown) dst[I * T + r] = a[r][KK];
#pragma unroll
    for (int c = 0; c < T; ++c)
        if (rowown) dst[J * T + c] = a[KK][c];
    if (diag) dst[NPAD] = pinv;
#pragma unroll
    for (int r = 0; r < T; ++r) a[r][KK] = (J == K) ? 0.0 : a[r][KK];
#pragma unroll
    for (int c = 0; c < T; ++c) a[KK][c] = (I == K) ? 0.0 : a[KK][c];
}

template <int T, int NPAD>
__device__ __forceinline__ void publish_clear(double (&a)[T][T], double *dst, int k, int I, int J)
{
    const int K = k / T;
    switch (k - K * T) {
    case 0: publish_clear_kk<T, NPAD, 0>(a, dst, K, I, J); break;
    case 1: if (T > 1) publish_clear_kk<T, NPAD, (T > 1 ? 1 : 0)>(a, dst, K, I, J); break;
    case 2: if (T > 2) publish_clear_kk<T, NPAD, (T > 2 ? 2 : 0)>(a, dst, K, I, J); break;
    case 3: if (T > 3) publish_clear_kk<T, NPAD, (T > 3 ? 3 : 0)>(a, dst, K, I, J); break;
    default: break;
    }
}

enum { SWEEP_OK = 0, SWEEP_ZERO = 1, SWEEP_NONFINITE = 2 };

// Pivot flags: a zero pivot is the reference's inversion failure, anything
// non-finite is reported separately.  Accumulated, checked once per inversion.
__device__ __forceinline__ int pivot_flags(double d)
{
    return (d == 0.0 ? 1 : 0) | (fabs(d) <= DBL_MAX ? 0 : 2);
}

__device__ __forceinline__ int flags_to_status(int f)
{
    return (f & 1) ? SWEEP_ZERO : (f & 2) ? SWEEP_NONFINITE : SWEEP_OK;
}

// One pivot of the sweep, pivot k = K*T + KK with KK a compile-time constant
// (register indices are static; no switch, no branch on data).
template <int T, int NT, int KK>
__device__ __forceinline__ void sweep_pivot(double (&a)[T][T], double *vb, int k, int K, int n, int I,
                                            int J, bool act, int &cnt, int &flags)
{
    constexpr int NPAD = Geom<T, NT>::NPAD;
    constexpr int VS = Geom<T, NT>::VS;
    constexpr int KN = (KK + 1) % T;  // in-tile index of pivot k+1
    const double *v = vb + (k & 1) * VS;
    const double d = v[k];
    flags |= pivot_flags(d);
    cnt += (d < 0.0) ? 1 : 0;
    // inactive threads (tile 0 with zeros) compute harmlessly; they never store
    const double p = v[NPAD];
    double x[T], y[T];
#pragma unroll
    for (int r = 0; r < T; ++r) x[r] = v[I * T + r];
#pragma unroll
    for (int c = 0; c < T; ++c) y[c] = v[J * T + c] * p;
    x[KK] = (I == K) ? -1.0 : x[KK];
    y[KK] = (J == K) ? -p : y[KK];
    // the entry that becomes pivot k+1 first, so its reciprocal starts early
    {
        constexpr int KR = (KN == 0) ? 0 : KN;
        a[KR][KR] = fma(-x[KR], y[KR], a[KR][KR]);
    }
#pragma unroll
    for (int r = 0; r < T; ++r)
#pragma unroll
        for (int c = 0; c < T; ++c)
            if (!(r == ((KN == 0) ? 0 : KN) && c == r)) a[r][c] = fma(-x[r], y[c], a[r][c]);
    if (k + 1 < n) publish_clear_kk<T, NPAD, KN>(a, vb + ((k + 1) & 1) * VS, KN == 0 ? K + 1 : K, I, J, act);
    __syncthreads();
}

// In-place -A^{-1} of the CTA's tiled matrix.  vb: 2*VS doubles of shared
// memory (double-buffered pivot column + reciprocal, one barrier per pivot).
// Returns the number of negative pivots; `bad` gets SWEEP_ZERO /
// SWEEP_NONFINITE if a pivot failed (identical in every thread).  After a
// failed pivot the remaining arithmetic runs on inf/NaN and is discarded.
template <int T, int NT>
__device__ __forceinline__ int sweep_invert(double (&a)[T][T], double *vb, int n, int I, int J,
                                            bool act, int &bad)
{
    static_assert(T >= 1 && T <= 4, "tile edge 1..4");
    constexpr int NPAD = Geom<T, NT>::NPAD;
    publish_clear_kk<T, NPAD, 0>(a, vb, 0, I, J, act);
    __syncthreads();
    int cnt = 0, flags = 0;
    for (int K = 0; K * T < n; ++K) {
        const int k0 = K * T;
        sweep_pivot<T, NT, 0>(a, vb, k0, K, n, I, J, act, cnt, flags);
        if (T > 1 && k0 + 1 < n) sweep_pivot<T, NT, (T > 1 ? 1 : 0)>(a, vb, k0 + 1, K, n, I, J, act, cnt, flags);
        if (T > 2 && k0 + 2 < n) sweep_pivot<T, NT, (T > 2 ? 2 : 0)>(a, vb, k0 + 2, K, n, I, J, act, cnt, flags);
        if (T > 3 && k0 + 3 < n) sweep_pivot<T, NT, (T > 3 ? 3 : 0)>(a, vb, k0 + 3, K, n, I, J, act, cnt, flags);
    }
    bad = flags_to_status(flags);
    return cnt;
}

// Two independent matrices inverted together (one barrier per pivot serves
// both).  Returns a's negative pivots; b's go to cnt_b.
template <int T, int NT, int KK>
__device__ __forceinline__ void sweep_pivot2(double (&a)[T][T], double (&b)[T][T], double *va,
                                             double *vbb, int k, int K, int n, int I, int J, bool act,
                                             int &ca, int &cb, int &flags)
{
    constexpr int NPAD = Geom<T, NT>::NPAD;
    constexpr int VS = Geom<T, NT>::VS;
    constexpr int KN = (KK + 1) % T;
    const double *v = va + (k & 1) * VS;
    const double *u = vbb + (k & 1) * VS;
    const double d = v[k], e = u[k];
    flags |= pivot_flags(d) | pivot_flags(e);
    ca += (d < 0.0) ? 1 : 0;
    cb += (e < 0.0) ? 1 : 0;
    const double p = v[NPAD], pe = u[NPAD];
    double x[T], y[T], xu[T], yu[T];
#pragma unroll
    for (int r = 0; r < T; ++r) { x[r] = v[I * T + r]; xu[r] = u[I * T + r]; }
#pragma unroll
    for (int c = 0; c < T; ++c) { y[c] = v[J * T + c] * p; yu[c] = u[J * T + c] * pe; }
    x[KK] = (I == K) ? -1.0 : x[KK];
    xu[KK] = (I == K) ? -1.0 : xu[KK];
    y[KK] = (J == K) ? -p : y[KK];
    yu[KK] = (J == K) ? -pe : yu[KK];
#pragma unroll
    for (int r = 0; r < T; ++r)
#pragma unroll
        for (int c = 0; c < T; ++c) {
            a[r][c] = fma(-x[r], y[c], a[r][c]);
            b[r][c] = fma(-xu[r], yu[c], b[r][c]);
        }
    if (k + 1 < n) {
        publish_clear_kk<T, NPAD, KN>(a, va + ((k + 1) & 1) * VS, KN == 0 ? K + 1 : K, I, J, act);
        publish_clear_kk<T, NPAD, KN>(b, vbb + ((k + 1) & 1) * VS, KN == 0 ? K + 1 : K, I, J, act);
    }
    __syncthreads();
}

template <int T, int NT>
__device__ __forceinline__ int sweep_invert2(double (&a)[T][T], double (&b)[T][T], double *va,
                                             double *vbb, int n, int I, int J, bool act, int &cnt_b,
                                             int &bad)
{
    constexpr int NPAD = Geom<T, NT>::NPAD;
    publish_clear_kk<T, NPAD, 0>(a, va, 0, I, J, act);
    publish_clear_kk<T, NPAD, 0>(b, vbb, 0, I, J, act);
    __syncthreads();
    int ca = 0, cb = 0, flags = 0;
    for (int K = 0; K * T < n; ++K) {
        const int k0 = K * T;
        sweep_pivot2<T, NT, 0>(a, b, va, vbb, k0, K, n, I, J, act, ca, cb, flags);
        if (T > 1 && k0 + 1 < n) sweep_pivot2<T, NT, (T > 1 ? 1 : 0)>(a, b, va, vbb, k0 + 1, K, n, I, J, act, ca, cb, flags);
        if (T > 2 && k0 + 2 < n) sweep_pivot2<T, NT, (T > 2 ? 2 : 0)>(a, b, va, vbb, k0 + 2, K, n, I, J, act, ca, cb, flags);
        if (T > 3 && k0 + 3 < n) sweep_pivot2<T, NT, (T > 3 ? 3 : 0)>(a, b, va, vbb, k0 + 3, K, n, I, J, act, ca, cb, flags);
    }
    bad = flags_to_status(flags);
    cnt_b = cb;
    return ca;
}

// --------------------------------------------------------------------------
// TMA bulk copies global -> shared, completion on an mbarrier.
// --------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t *bar)
{
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void fence_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// One thread: announce `bytes` and start the copy (bytes and both addresses
// must be multiples of 16).
__device__ __forceinline__ void bulk_load(void *dst_smem, const void *src_gmem, uint32_t bytes, uint64_t *bar)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst_smem)),
        "l"(src_gmem), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for phase `parity` of an mbarrier.  Returns false if the copy
// did not land within the limit (the caller reports a timeout status).
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit = kWaitLimit)
{
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_test(bar, parity)) return true;
    return false;
}

// Iteration limit of the one-warp kernels' per-step wait for the next
// 2HQ(C) copy (kWaitLimit unless a test lowers it through
// mgpu_set_step_wait_limit; the waits that drain copies before an early
// exit always use kWaitLimit).
__device__ uint32_t g_step_wait_limit = kWaitLimit;

// A stop the host asks for, polled by the step kernels every kStopPoll steps
// (k = 1, 1 + kStopPoll, ...): ctl points at the plan's control words in
// device memory (volatile reads: L2, where the host's copies land; reading
// them from mapped host memory cost every warp a PCIe round trip and the
// batched workload 24 %), ctl[0] != 0 cancels, ctl[1] > 0 is each step kernel's
// time budget in nanoseconds on the device's global timer, counted from that
// kernel's start.  The kernel then records the status and the step and
// leaves its loop as it does after a failed inversion.
#ifndef MGPU_STOP_POLL
#define MGPU_STOP_POLL 128
#endif
constexpr int kStopPoll = MGPU_STOP_POLL;

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ bool stop_poll_step(int k) { return ((k - 1) % kStopPoll) == 0; }

__device__ __forceinline__ int stop_requested(const volatile long long *ctl, unsigned long long t0)
{
    if (!ctl) return MGPU_OK;
    if (ctl[0] != 0) return MGPU_ERR_CANCELLED;
    const long long budget = ctl[1];
    if (budget > 0 && (long long)(global_ns() - t0) > budget) return MGPU_ERR_DEADLINE;
    return MGPU_OK;
}

}  // namespace mgpu
