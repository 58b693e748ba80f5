// libmolscat_gpu: B200 (sm_100a) FP64 log-derivative propagators behind the
// MDPROP / LDPROP boundary.  C ABI in include/molscat_gpu.h.
//
// Kernels (one CTA per matrix, the matrix register-tiled, see tiles.cuh):
//   ldmd_prep_kernel  energy-independent part of MDPROP: for every step k the
//                     inverse 2HQ(C_k) = [I/8 - (H^2/48) W_off(C_k)]^-1 - 8I and
//                     its negative-pivot count (mdprop.f:113-139).  One CTA
//                     per (system, step): all steps run in parallel.
//   ldmd_prop_kernel  the sequential MDPROP step loop for one (system, ERED)
//                     job: reference-potential tan/tanh terms, two symmetric
//                     inversions, W(B) assembly (mdprop.f:143-230), final
//                     Y/H (mdprop.f:269-275), NODES (mdprop.f:170,193,279).
//   ldj_prop_kernel   the LDPROP step loop (ldprop.f:46-147): U and Z are
//                     inverted together (one barrier per pivot for both).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <map>
#include <mutex>
#include <new>
#include <string>
#include <tuple>
#include <vector>

#include "molscat_gpu.h"
#include "tiles.cuh"

namespace mgpu {

constexpr int kT = 4;  // tile edge of every compiled bucket
constexpr size_t kSmemBudget = 96 * 1024;  // dynamic shared memory per CTA we allow

struct SysDev {
    int n, nham, ivlfl, nconst, nrsq, nstep, ntiles, kind;  // kind: 0 = 4x4 register tiles, 1 = 8x8 DMMA fragments
    double conlen, dr;
    const double *vlt;  // [nham][T*T][ntiles] tile layout, zero padding
    const int *ivt;     // same shape, 0-based P index (ivlfl > 0 only)
    const double *eint; // [npad]
    const double *cent; // [npad]
    const double *rtab; // [2*nstep+1]
    const double *ptab; // [2*nstep+1][nham]
    double *q;          // LDMD: [nstep][T*T][ntiles] 2HQ(C_k)
    double *wt;         // LDMD one-warp kernels or null: [nstep+1][ntiles][64] coupling sum
                        // sum_l VL_l P_l(R) at R_0, R_2, .., R_2nstep (fragment layout)
    double *wd;         // LDMD one-warp kernels or null: [nstep][npad] its diagonal at R_1, R_3, ..
    int *prep;          // LDMD: [0] negative pivots of all U inversions (NSAVE), [1] status, [2] kfail
    const volatile long long *ctl;  // plan's stop controls (device memory) or null: stop_requested
};

struct JobDev {
    int sys;
    int out;          // index of the job in the caller's order
    double ered;
    long long yoff;   // first double of this job's Y
};

// W(R) restricted to one tile (HAMMAT + SUMLAM, hammat.f:85-113, sumlam.f).
// vl points at the [nham][T*T][ntiles] tile array, in shared or global memory.
// diag_terms=false gives the coupling sum only (what MDPROP's U uses).
template <int T>
__device__ __forceinline__ void w_tile(const SysDev &S, const double *__restrict__ vl, int t, int I, int J, int ir,
                                       double ered, bool diag_terms, double (&w)[T][T])
{
    constexpr int TT = T * T;
    const int nt = S.ntiles;
    const double *P = S.ptab + (size_t)ir * S.nham;
#pragma unroll
    for (int r = 0; r < T; ++r)
#pragma unroll
        for (int c = 0; c < T; ++c) w[r][c] = 0.0;
    if (S.ivlfl <= 0) {
        for (int l = 0; l < S.nham; ++l) {
            const double pl = __ldg(P + l);
            const double *v = vl + (size_t)l * TT * nt + t;
#pragma unroll
            for (int r = 0; r < T; ++r)
#pragma unroll
                for (int c = 0; c < T; ++c) w[r][c] = fma(v[(size_t)(r * T + c) * nt], pl, w[r][c]);
        }
    } else {
        for (int l = 0; l < S.nham; ++l) {
            const double *v = vl + (size_t)l * TT * nt + t;
            const int *iv = S.ivt + (size_t)l * TT * nt + t;
#pragma unroll
            for (int r = 0; r < T; ++r)
#pragma unroll
                for (int c = 0; c < T; ++c) {
                    const double x = v[(size_t)(r * T + c) * nt];
                    if (x != 0.0) w[r][c] = fma(x, __ldg(P + __ldg(iv + (size_t)(r * T + c) * nt)), w[r][c]);
                }
        }
    }
    if (diag_terms && I == J) {
        const double R = __ldg(S.rtab + ir);
        double rsq = 1.0 / (R * R);
        rsq = fmin(rsq, 1.0e16);
        double conf = 0.0;
        if (S.conlen > 0.0) {
            const double c2 = S.conlen * S.conlen;
            conf = R * R / (c2 * c2);
        }
#pragma unroll
        for (int r = 0; r < T; ++r) {
            const int i = I * T + r;
            if (i < S.n) {
                double x = w[r][r];
                if (S.nrsq == 0) x += rsq * S.cent[i];
                if (S.nconst == 0) x += S.eint[i];
                if (S.conlen > 0.0) x += conf;
                w[r][r] = x - ered;
            }
        }
    }
}

// W(R)_ii for one channel (the DIAG array HAMMAT returns).
template <int T>
__device__ __forceinline__ double w_diag(const SysDev &S, const double *__restrict__ vl, int i, int ir, double ered)
{
    constexpr int TT = T * T;
    const int nt = S.ntiles;
    const int I = i / T, r = i - I * T;
    const int t = I * (I + 1) / 2 + I;
    const size_t e = (size_t)(r * T + r) * nt + t;
    const double *P = S.ptab + (size_t)ir * S.nham;
    double x = 0.0;
    for (int l = 0; l < S.nham; ++l) {
        const double v = vl[(size_t)l * TT * nt + e];
        if (S.ivlfl <= 0) x = fma(v, __ldg(P + l), x);
        else if (v != 0.0) x = fma(v, __ldg(P + __ldg(S.ivt + (size_t)l * TT * nt + e)), x);
    }
    const double R = __ldg(S.rtab + ir);
    double rsq = fmin(1.0 / (R * R), 1.0e16);
    if (S.nrsq == 0) x += rsq * S.cent[i];
    if (S.nconst == 0) x += S.eint[i];
    if (S.conlen > 0.0) {
        const double c2 = S.conlen * S.conlen;
        x += R * R / (c2 * c2);
    }
    return x - ered;
}

// The sector reference-potential solutions of MDPROP (mdprop.f:143-164).
__device__ __noinline__ void ref_solutions(double wref, double half, double &y14, double &y23)
{
    const double arg = half * sqrt(fabs(wref));
    if (wref < 0.0) {
        const double tn = tan(arg);
        y14 = arg / tn - arg * tn;
        y23 = arg / tn + arg * tn;
    } else {
        const double th = tanh(arg);
        y14 = arg / th + arg * th;
        y23 = arg / th - arg * th;
    }
}

template <int T>
__device__ __forceinline__ void load_lower(const double *__restrict__ y, int n, int I, int J,
                                           double (&a)[T][T])
{
#pragma unroll
    for (int r = 0; r < T; ++r)
#pragma unroll
        for (int c = 0; c < T; ++c) {
            const int i = I * T + r, j = J * T + c;
            const int lo = i < j ? i : j, hi = i < j ? j : i;
            a[r][c] = (i < n && j < n) ? y[(size_t)lo * n + hi] : 0.0;
        }
}

template <int T>
__device__ __forceinline__ void store_full(double *__restrict__ y, int n, int I, int J, double scale,
                                          const double (&a)[T][T])
{
#pragma unroll
    for (int r = 0; r < T; ++r)
#pragma unroll
        for (int c = 0; c < T; ++c) {
            const int i = I * T + r, j = J * T + c;
            if (i < n && j <= i) {
                const double x = scale * a[r][c];
                y[(size_t)j * n + i] = x;
                y[(size_t)i * n + j] = x;
            }
        }
}

// Copy the system's VL tiles into shared memory (once per CTA).
__device__ __forceinline__ void stage_vl(const SysDev &S, double *__restrict__ dst, int tt, int nthr)
{
    const int cnt = S.nham * tt * S.ntiles;
    for (int i = threadIdx.x; i < cnt; i += nthr) dst[i] = __ldg(S.vlt + i);
}

// ---------------------------------------------------------------------------
// MDPROP, energy-independent half: 2HQ(C_k) for every step of every system.
// grid = (max nstep in bucket, systems in bucket)
// ---------------------------------------------------------------------------
template <int T, int NT>
__global__ void __launch_bounds__(Geom<T, NT>::NTHR, Geom<T, NT>::MINB)
ldmd_prep_kernel(const SysDev *__restrict__ systems, const int *__restrict__ sys_list)
{
    using G = Geom<T, NT>;
    __shared__ __align__(16) double vb[2 * G::VS];
    __shared__ SysDev s_sys;
    if (threadIdx.x == 0) s_sys = systems[sys_list[blockIdx.y]];
    __syncthreads();
    const SysDev &S = s_sys;
    const int k = blockIdx.x + 1;
    if (k > S.nstep) return;
    const int tid = threadIdx.x;
    const bool act = tid < G::NTILES;
    int I = 0, J = 0;
    tile_of(act ? tid : 0, I, J);
    const double h = S.dr / 2.0;
    const double d1 = h * h / 3.0;
    const double d4 = -d1 / 16.0;
    double a[T][T];
    if (act) {
        w_tile<T>(S, S.vlt, tid, I, J, 2 * k - 1, 0.0, false, a);
#pragma unroll
        for (int r = 0; r < T; ++r)
#pragma unroll
            for (int c = 0; c < T; ++c) {
                const int i = I * T + r, j = J * T + c;
                a[r][c] = (i == j) ? (i < S.n ? 0.125 : 0.0) : d4 * a[r][c];
            }
    } else {
#pragma unroll
        for (int r = 0; r < T; ++r)
#pragma unroll
            for (int c = 0; c < T; ++c) a[r][c] = 0.0;
    }
    int bad = SWEEP_OK;
    const int cnt = sweep_invert<T, NT>(a, vb, S.n, I, J, act, bad);
    if (bad != SWEEP_OK) {
        if (tid == 0) {
            atomicMax(&S.prep[1], bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE);
            atomicMin(&S.prep[2], k);
        }
        return;
    }
    if (tid == 0 && cnt) atomicAdd(&S.prep[0], cnt);
    if (act) {
        double *q = S.q + (size_t)(k - 1) * G::TT * S.ntiles + tid;
#pragma unroll
        for (int r = 0; r < T; ++r)
#pragma unroll
            for (int c = 0; c < T; ++c) {
                const int i = I * T + r, j = J * T + c;
                // a = -U^{-1};  2HQ(C) = U^{-1} - 8I
                const double x = (i == j && i < S.n) ? (-a[r][c] - 8.0) : -a[r][c];
                q[(size_t)(r * T + c) * S.ntiles] = x;
            }
    }
}

// ---------------------------------------------------------------------------
// MDPROP step loop, one CTA per job.  Dynamic shared memory: two 2HQ(C)
// tile buffers filled by TMA bulk copies one step ahead, then (vl_smem) the
// system's VL tiles.
// ---------------------------------------------------------------------------
template <int T, int NT>
__global__ void __launch_bounds__(Geom<T, NT>::NTHR, Geom<T, NT>::MINB)
ldmd_prop_kernel(const SysDev *__restrict__ systems, const JobDev *__restrict__ jobs,
                 double *__restrict__ y, int *__restrict__ nodes_out, int *__restrict__ status_out,
                 int *__restrict__ kfail_out, int vl_smem)
{
    using G = Geom<T, NT>;
    constexpr int NPAD = G::NPAD;
    extern __shared__ __align__(16) double dsm[];
    __shared__ __align__(16) double vb[2 * G::VS];
    __shared__ double s_y14[2][NPAD], s_y14b[2][NPAD], s_y23[2][NPAD];
    __shared__ __align__(8) uint64_t qbar[2];
    __shared__ int s_stop;
    __shared__ SysDev s_sys;
    const JobDev job = jobs[blockIdx.x];
    if (threadIdx.x == 0) s_sys = systems[job.sys];
    __syncthreads();
    const SysDev &S = s_sys;
    const int tid = threadIdx.x;
    const bool act = tid < G::NTILES;
    int I = 0, J = 0;
    tile_of(act ? tid : 0, I, J);
    const int n = S.n;
    const int nt = S.ntiles;
    const double ered = job.ered;
    const size_t qdoubles = (size_t)G::TT * nt;
    const uint32_t qbytes = (uint32_t)(qdoubles * sizeof(double));
    double *qbuf0 = dsm;
    double *vls = vl_smem ? dsm + 2 * qdoubles : nullptr;
    const double *vl = vl_smem ? vls : S.vlt;

    const int prep_status = S.prep[1];
    if (prep_status != 0) {
        if (tid == 0) {
            status_out[job.out] = prep_status;
            kfail_out[job.out] = S.prep[2];
            nodes_out[job.out] = 0;
        }
        return;
    }
    if (tid == 0) {
        mbar_init(&qbar[0], 1);
        mbar_init(&qbar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < NPAD; i += G::NTHR) {
        s_y14[0][i] = s_y14[1][i] = 0.0;
        s_y14b[0][i] = s_y14b[1][i] = 0.0;
        s_y23[0][i] = s_y23[1][i] = 0.0;
    }
    if (vl_smem) stage_vl(S, vls, G::TT, G::NTHR);
    __syncthreads();
    if (tid == 0) bulk_load(qbuf0 + qdoubles, S.q, qbytes, &qbar[1]);  // 2HQ(C_1) -> buffer 1

    const double h = S.dr / 2.0;
    const double d1 = h * h / 3.0;
    const double d2 = 2.0 * d1;
    const double half = 0.5 * h;
    double *yj = y + job.yoff;

    double a[T][T];
    if (act) {
        double w[T][T];
        load_lower<T>(yj, n, I, J, a);
        w_tile<T>(S, vl, tid, I, J, 0, ered, true, w);
#pragma unroll
        for (int r = 0; r < T; ++r)
#pragma unroll
            for (int c = 0; c < T; ++c) a[r][c] = h * a[r][c] + d1 * w[r][c];  // mdprop.f:89-93
    } else {
#pragma unroll
        for (int r = 0; r < T; ++r)
#pragma unroll
            for (int c = 0; c < T; ++c) a[r][c] = 0.0;
    }

    int nodes = 0;
    int status = MGPU_OK, kfail = 0;
    int issued = 1;    // last step whose 2HQ(C) copy has been started
    int consumed = 0;  // last step whose copy has been waited for
    const unsigned long long t0 = global_ns();
    for (int k = 1; k <= S.nstep; ++k) {
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
        const int sb = k & 1;
        if (tid == 0 && k + 1 <= S.nstep) {
            // buffer (k+1)&1 was last read in step k-1; every thread has passed
            // that step's barriers, so the async proxy may overwrite it now
            fence_async_shared();
            bulk_load(qbuf0 + ((k + 1) & 1) * qdoubles, S.q + (size_t)k * qdoubles, qbytes, &qbar[(k + 1) & 1]);
            issued = k + 1;
        }
        // reference-potential solutions in the sector (mdprop.f:143-164)
        for (int i = tid; i < n; i += G::NTHR) {
            const double wref = w_diag<T>(S, vl, i, 2 * k - 1, ered);
            double y14, y23;
            ref_solutions(wref, half, y14, y23);
            s_y14[sb][i] = y14;
            s_y14b[sb][i] = y14 - d1 * wref;
            s_y23[sb][i] = y23;
        }
        __syncthreads();
        if (act && I == J) {
#pragma unroll
            for (int r = 0; r < T; ++r) a[r][r] += s_y14b[sb][I * T + r];
        }
        int bad = SWEEP_OK;
        nodes += sweep_invert<T, NT>(a, vb, n, I, J, act, bad);
        if (bad != SWEEP_OK) {
            status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        // 2HQ(C_k) has landed in buffer k&1?  (bounded wait, uniform verdict)
        const bool landed = mbar_wait_bounded(&qbar[sb], ((k - 1) >> 1) & 1);
        if (__syncthreads_or(!landed)) {
            status = MGPU_ERR_TIMEOUT;
            kfail = k;
            break;
        }
        consumed = k;
        const double *qs = qbuf0 + sb * qdoubles + tid;
        double y23r[T], y23c[T];
#pragma unroll
        for (int r = 0; r < T; ++r) y23r[r] = s_y23[sb][I * T + r];
#pragma unroll
        for (int c = 0; c < T; ++c) y23c[c] = s_y23[sb][J * T + c];
        if (act) {
            // Y = 2HQ(C) + 2 Y14 - Y23 Y^-1 Y23   (a holds -Y^-1), mdprop.f:156,181-185
#pragma unroll
            for (int r = 0; r < T; ++r)
#pragma unroll
                for (int c = 0; c < T; ++c) a[r][c] = qs[(size_t)(r * T + c) * nt] + y23r[r] * a[r][c] * y23c[c];
            if (I == J) {
#pragma unroll
                for (int r = 0; r < T; ++r) a[r][r] += 2.0 * s_y14[sb][I * T + r];
            }
        }
        nodes += sweep_invert<T, NT>(a, vb, n, I, J, act, bad);
        if (bad != SWEEP_OK) {
            status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        if (act) {
            // Y = D2 W(B) - Y23 Y^-1 Y23 + Y14'   (mdprop.f:196-230)
            const double dd = (k == S.nstep) ? d1 : d2;
            double w[T][T];
            w_tile<T>(S, vl, tid, I, J, 2 * k, ered, true, w);
#pragma unroll
            for (int r = 0; r < T; ++r)
#pragma unroll
                for (int c = 0; c < T; ++c) a[r][c] = dd * w[r][c] + y23r[r] * a[r][c] * y23c[c];
            if (I == J) {
#pragma unroll
                for (int r = 0; r < T; ++r) a[r][r] += s_y14b[sb][I * T + r];
            }
        }
    }
    if (status != MGPU_OK && tid == 0) {
        // an early exit can leave up to two copies in flight: let them land
        // (bounded) before this CTA's shared memory can be reused
        for (int s2 = consumed + 1; s2 <= issued; ++s2) mbar_wait_bounded(&qbar[s2 & 1], ((s2 - 1) >> 1) & 1);
    }
    if (status == MGPU_OK && act) store_full<T>(yj, n, I, J, 1.0 / h, a);
    if (tid == 0) {
        status_out[job.out] = status;
        kfail_out[job.out] = kfail;
        nodes_out[job.out] = status == MGPU_OK ? nodes - S.prep[0] : 0;
    }
}

// ---------------------------------------------------------------------------
// LDPROP step loop, one CTA per job (ldprop.f:46-147).  U(C) and Z are
// inverted together; they are independent.
// ---------------------------------------------------------------------------
template <int T, int NT>
__global__ void __launch_bounds__(Geom<T, NT>::NTHR, Geom<T, NT>::MINB)
ldj_prop_kernel(const SysDev *__restrict__ systems, const JobDev *__restrict__ jobs,
                double *__restrict__ y, int *__restrict__ nodes_out, int *__restrict__ status_out,
                int *__restrict__ kfail_out, int vl_smem)
{
    using G = Geom<T, NT>;
    extern __shared__ __align__(16) double dsm[];
    __shared__ __align__(16) double vz[2 * G::VS];
    __shared__ __align__(16) double vu[2 * G::VS];
    __shared__ int s_stop;
    __shared__ SysDev s_sys;
    const JobDev job = jobs[blockIdx.x];
    if (threadIdx.x == 0) s_sys = systems[job.sys];
    __syncthreads();
    const SysDev &S = s_sys;
    const int tid = threadIdx.x;
    const bool act = tid < G::NTILES;
    int I = 0, J = 0;
    tile_of(act ? tid : 0, I, J);
    const int n = S.n;
    const double ered = job.ered;
    const double h = S.dr / 2.0;
    const double d1 = h * h / 3.0;
    const double d2 = 2.0 * d1;
    const double d4 = -d1 / 16.0;
    double *yj = y + job.yoff;
    if (vl_smem) stage_vl(S, dsm, G::TT, G::NTHR);
    __syncthreads();
    const double *vl = vl_smem ? dsm : S.vlt;

    double z[T][T], u[T][T];
#pragma unroll
    for (int r = 0; r < T; ++r)
#pragma unroll
        for (int c = 0; c < T; ++c) { z[r][c] = 0.0; u[r][c] = 0.0; }
    if (act) {
        load_lower<T>(yj, n, I, J, z);
        w_tile<T>(S, vl, tid, I, J, 0, ered, true, u);
#pragma unroll
        for (int r = 0; r < T; ++r)
#pragma unroll
            for (int c = 0; c < T; ++c) {
                const int i = I * T + r, j = J * T + c;
                z[r][c] = h * z[r][c] + d1 * u[r][c] + ((i == j && i < n) ? 1.0 : 0.0);  // ldprop.f:46-51
            }
    }
    int nodes = 0, status = MGPU_OK, kfail = 0;
    const unsigned long long t0 = global_ns();
    for (int k = 1; k <= S.nstep; ++k) {
        if (stop_poll_step(k)) {
            if (tid == 0) s_stop = stop_requested(S.ctl, t0);
            __syncthreads();
            const int stop = s_stop;
            if (stop != MGPU_OK) {
                status = stop;
                kfail = k;
                break;
            }
        }
        if (act) {
            w_tile<T>(S, vl, tid, I, J, 2 * k - 1, ered, true, u);
#pragma unroll
            for (int r = 0; r < T; ++r)
#pragma unroll
                for (int c = 0; c < T; ++c) {
                    const int i = I * T + r, j = J * T + c;
                    u[r][c] = d4 * u[r][c] + ((i == j && i < n) ? 0.125 : 0.0);  // ldprop.f:67-72
                }
        }
        int bad = SWEEP_OK, ncz = 0;
        const int ncu = sweep_invert2<T, NT>(u, z, vu, vz, n, I, J, act, ncz, bad);  // ldprop.f:78,83
        if (bad != SWEEP_OK) {
            status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        nodes += ncz;
        if (act) {
            // Z = U^-1 - Z^-1 - 6I with u = -U^-1, z = -Z^-1 (ldprop.f:92-97)
#pragma unroll
            for (int r = 0; r < T; ++r)
#pragma unroll
                for (int c = 0; c < T; ++c) {
                    const int i = I * T + r, j = J * T + c;
                    z[r][c] = -u[r][c] + z[r][c] - ((i == j && i < n) ? 6.0 : 0.0);
                }
        }
        const int ncz2 = sweep_invert<T, NT>(z, vz, n, I, J, act, bad);  // ldprop.f:99
        if (bad != SWEEP_OK) {
            status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        nodes += ncz2 - ncu;
        if (act) {
            const double dd = (k == S.nstep) ? d1 : d2;
            w_tile<T>(S, vl, tid, I, J, 2 * k, ered, true, u);
#pragma unroll
            for (int r = 0; r < T; ++r)
#pragma unroll
                for (int c = 0; c < T; ++c) {
                    const int i = I * T + r, j = J * T + c;
                    // Z = D2 W(B) + 2I - Z^-1 (ldprop.f:114-131)
                    z[r][c] = dd * u[r][c] + ((i == j && i < n) ? 2.0 : 0.0) + z[r][c];
                }
        }
    }
    if (status == MGPU_OK && act) {
        // Y = Z/H - I/H (ldprop.f:140-147)
        const double hi = 1.0 / h;
#pragma unroll
        for (int r = 0; r < T; ++r)
#pragma unroll
            for (int c = 0; c < T; ++c) {
                const int i = I * T + r, j = J * T + c;
                z[r][c] = hi * z[r][c] - ((i == j) ? hi : 0.0);
            }
        store_full<T>(yj, n, I, J, 1.0, z);
    }
    if (tid == 0) {
        status_out[job.out] = status;
        kfail_out[job.out] = kfail;
        nodes_out[job.out] = status == MGPU_OK ? nodes : 0;
    }
}

}  // namespace mgpu
#include "kernels_frag.cuh"
#include "kernels_cta.cuh"
#include "kernels_big.cuh"
#include "kernels_smatrix.cuh"
#include "kernels_match.cuh"
namespace mgpu {

__global__ void prep_reset_kernel(int *prep, int nsys)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < nsys) {
        prep[3 * s] = 0;
        prep[3 * s + 1] = 0;
        prep[3 * s + 2] = 0x7fffffff;
    }
}

// FP64 FMA pipe probe: 8 independent dependent-chains per thread.
__global__ void __launch_bounds__(256) fp64_fma_probe_kernel(double *out, int iters)
{
    double x[8];
    const double s = 1.0 + 1e-9 * threadIdx.x;
#pragma unroll
    for (int i = 0; i < 8; ++i) x[i] = 0.5 + 0.01 * i + 1e-7 * blockIdx.x;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int i = 0; i < 8; ++i) x[i] = fma(x[i], s, -0.25);
    }
    double acc = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) acc += x[i];
    if (acc == 12345.678) out[0] = acc;  // practically never true; keeps the chains live
}

// pivot_reciprocal on a vector, for the test that holds it to 1.0/x
__global__ void __launch_bounds__(256) pivot_reciprocal_probe_kernel(const double *x, double *r, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) r[i] = pivot_reciprocal(x[i]);
}

// ---------------------------------------------------------------------------
// bucket dispatch
// ---------------------------------------------------------------------------
#define MGPU_BUCKETS(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(12) X(14) X(16)
#define MGPU_FRAG_BUCKETS(X) X(1) X(2) X(3) X(4) X(5)
// (NT, warps) of the one-CTA-per-matrix buckets, N = 8*NT up to 200
#ifndef MGPU_CTA_BUCKETS
#define MGPU_CTA_BUCKETS(X) X(6, 4) X(7, 4) X(8, 4) X(10, 8) X(12, 8) X(14, 8) X(16, 8) X(20, 16) X(25, 16)
#endif

// NT of the large-N buckets (matrices in global memory, 64 pivots a round):
// N up to 1024 in steps of 64
#define MGPU_BIG_BUCKETS(X) X(8) X(16) X(24) X(32) X(40) X(48) X(56) X(64) X(72) X(80) X(88) X(96) X(104) X(112) X(120) X(128)

// KIND_FRAG8: one warp per matrix; KIND_CTA8: one CTA per matrix (same 8x8
// fragment data layout); KIND_BIG: batched kernels over matrices held in
// global memory (same layout); KIND_TILE4: 4x4 register tiles.
enum { KIND_TILE4 = 0, KIND_FRAG8 = 1, KIND_CTA8 = 2, KIND_BIG = 3 };

struct Bucket {
    int kind;
    int nt;
    int warps;  // KIND_CTA8
};

// 8x8-fragment buckets first (one warp for N <= 40, one CTA up to 200), then
// the 4x4 register tiles (N <= 64).
static const Bucket kBuckets[] = {
#define X(nt) {KIND_FRAG8, nt, 1},
    MGPU_FRAG_BUCKETS(X)
#undef X
#define X(nt, w) {KIND_CTA8, nt, w},
    MGPU_CTA_BUCKETS(X)
#undef X
#define X(nt) {KIND_BIG, nt, 0},
    MGPU_BIG_BUCKETS(X)
#undef X
#define X(nt) {KIND_TILE4, nt, 0},
    MGPU_BUCKETS(X)
#undef X
};
static const int kNumBuckets = sizeof(kBuckets) / sizeof(kBuckets[0]);

static bool frag_layout(int b) { return kBuckets[b].kind != KIND_TILE4; }
static int bucket_edge(int b) { return frag_layout(b) ? 8 : kT; }
static int bucket_npad(int b) { return bucket_edge(b) * kBuckets[b].nt; }
static int ntiles_of(int b) { return kBuckets[b].nt * (kBuckets[b].nt + 1) / 2; }
static size_t tile_elems(int b) { return (size_t)bucket_edge(b) * bucket_edge(b); }  // doubles per tile
static size_t matrix_elems(int b) { return tile_elems(b) * ntiles_of(b); }         // doubles per tiled matrix

// LDJ keeps two tiled matrices in shared memory: CTA buckets up to N = 128.
static bool is_ldmg(int iprop) { return iprop == MGPU_PROP_LDMG4 || iprop == MGPU_PROP_LDMG5; }

// LDMG runs on the fragment-layout families: one warp, one CTA, batched large N.
static bool bucket_allows(int b, int iprop)
{
    if (is_ldmg(iprop)) return kBuckets[b].kind != KIND_TILE4;
    return !(iprop == MGPU_PROP_LDJ && kBuckets[b].kind == KIND_CTA8 && kBuckets[b].nt > 16);
}

// Smallest bucket that holds N: the fragment kernels first, then the 4x4
// register tiles; g_prefer_tile4 puts the 4x4 tiles first where they fit.
static int g_prefer_tile4 = 0;

// Per-N family choices (from the autotuner): 0 = the default order (one
// warp, one CTA, batched large-N), 1 = 4x4 register tiles, 2 = batched
// large-N kernels.  Consulted before the default order; a family that has no
// bucket for N falls back to it.
struct FamilyRange {
    int iprop, lo, hi, family;  // iprop 0: both propagators
};
static std::vector<FamilyRange> g_family_ranges;
static std::mutex g_family_mu;

static int bucket_of_kind(int n, int iprop, int kind)
{
    for (int b = 0; b < kNumBuckets; ++b)
        if (kBuckets[b].kind == kind && bucket_npad(b) >= n && bucket_allows(b, iprop)) return b;
    return -1;
}

static int bucket_for(int n, int iprop = MGPU_PROP_LDMD, bool tuned = true)
{
    if (tuned && !is_ldmg(iprop)) {
        std::lock_guard<std::mutex> lk(g_family_mu);
        for (const auto &r : g_family_ranges)
            if ((r.iprop == 0 || r.iprop == iprop) && n >= r.lo && n <= r.hi && r.family != 0) {
                const int b = bucket_of_kind(n, iprop, r.family == 1 ? KIND_TILE4 : KIND_BIG);
                if (b >= 0) return b;
            }
    }
    for (int pass = 0; pass < 2; ++pass) {
        const bool tile4 = (pass == 0) == (g_prefer_tile4 != 0);
        for (int b = 0; b < kNumBuckets; ++b)
            if ((kBuckets[b].kind == KIND_TILE4) == tile4 && bucket_npad(b) >= n && bucket_allows(b, iprop))
                return b;
    }
    return -1;
}

// Raise a kernel's dynamic shared-memory limit, once per (device, kernel)
// and size: setting attributes again on every launch is not free, and a
// launch path that runs beside other work should not touch a kernel that is
// executing.
template <class K>
static cudaError_t set_smem(K kernel, size_t bytes)
{
    if (bytes == 0) return cudaSuccess;
    static std::mutex mu;
    static std::vector<std::pair<std::pair<int, const void *>, size_t>> done;
    int dev = 0;
    cudaGetDevice(&dev);
    const void *key = (const void *)kernel;
    std::lock_guard<std::mutex> lk(mu);
    for (auto &d : done)
        if (d.first.first == dev && d.first.second == key && d.second >= bytes) return cudaSuccess;
    // the 48 KB default covers static plus dynamic shared memory
    cudaFuncAttributes fa{};
    cudaError_t e = cudaFuncGetAttributes(&fa, (const void *)kernel);
    if (e != cudaSuccess) return e;
    if (bytes + fa.sharedSizeBytes > 48 * 1024) {
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
        // resident CTAs are limited by registers, not by the L1/shared split
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
        if (e != cudaSuccess) return e;
    }
    done.push_back({{dev, key}, bytes});
    return cudaSuccess;
}

// grid.x counts steps, grid.y systems
static cudaError_t launch_prep(int b, int max_nstep, int nsys, cudaStream_t st, const SysDev *sys, const int *list)
{
    const int nt = kBuckets[b].nt;
    if (kBuckets[b].kind == KIND_BIG) return cudaErrorInvalidValue;
    if (kBuckets[b].kind == KIND_CTA8) {
        dim3 grid(max_nstep, nsys);
        cudaError_t e = cudaSuccess;
        switch (nt) {
#define X(t, w)                                                                                   \
    case t: {                                                                                     \
        const size_t sm = cta::CSmem<t, w>::bytes(1);                                             \
        if ((e = set_smem(cta::ldmd_prep_cta_kernel<t, w>, sm))) return e;                        \
        cta::ldmd_prep_cta_kernel<t, w><<<grid, 32 * w, sm, st>>>(sys, list);                    \
        break;                                                                                    \
    }
            MGPU_CTA_BUCKETS(X)
#undef X
        default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    if (kBuckets[b].kind == KIND_FRAG8) {
        dim3 grid((max_nstep + wf::kWPB - 1) / wf::kWPB, nsys);
        switch (nt) {
#define X(t)                                                                          \
    case t: wf::ldmd_prep_frag_kernel<t><<<grid, 32 * wf::kWPB, 0, st>>>(sys, list); \
        break;
            MGPU_FRAG_BUCKETS(X)
#undef X
        default: return cudaErrorInvalidValue;
        }
    } else {
        dim3 grid(max_nstep, nsys);
        switch (nt) {
#define X(t)                                                                                 \
    case t: ldmd_prep_kernel<kT, t><<<grid, Geom<kT, t>::NTHR, 0, st>>>(sys, list); \
        break;
            MGPU_BUCKETS(X)
#undef X
        default: return cudaErrorInvalidValue;
        }
    }
    return cudaGetLastError();
}

// Dynamic shared memory a propagation launch of bucket b needs (vl_smem: the
// 4x4-tile kernels stage VL when it fits).
static size_t prop_smem(int iprop, int b, int nham, int *vl_smem)
{
    if (kBuckets[b].kind == KIND_BIG) {
        *vl_smem = 0;
        return 0;
    }
    if (kBuckets[b].kind == KIND_CTA8) {
        *vl_smem = 0;
        switch (kBuckets[b].nt) {
#define X(t, w) case t: return cta::CSmem<t, w>::bytes(iprop == MGPU_PROP_LDJ ? 2 : 1);
            MGPU_CTA_BUCKETS(X)
#undef X
        }
        return 0;
    }
    if (kBuckets[b].kind == KIND_FRAG8) {
        *vl_smem = 0;
        size_t per = 0;
        switch (kBuckets[b].nt) {
#define X(t) case t: per = wf::WarpSmem<t>::BYTES; break;
            MGPU_FRAG_BUCKETS(X)
#undef X
        }
        return iprop == MGPU_PROP_LDMD ? per * wf::kWPB : 0;
    }
    const size_t tile_bytes = matrix_elems(b) * sizeof(double);
    const size_t base = iprop == MGPU_PROP_LDMD ? 2 * tile_bytes : 0;
    const size_t vlb = (size_t)nham * tile_bytes;
    *vl_smem = (base + vlb <= kSmemBudget) ? 1 : 0;
    return base + (*vl_smem ? vlb : 0);
}

static cudaError_t launch_prop(int iprop, int b, int njobs, size_t smem, int vl_smem, cudaStream_t st,
                               const SysDev *sys, const JobDev *jobs, double *y, int *nodes, int *status, int *kfail)
{
    cudaError_t e = cudaSuccess;
    const int nt = kBuckets[b].nt;
    if (kBuckets[b].kind == KIND_CTA8) {
        switch (nt) {
#define X(t, w)                                                                                              \
    case t:                                                                                                  \
        if (iprop == MGPU_PROP_LDMD) {                                                                       \
            if ((e = set_smem(cta::ldmd_prop_cta_kernel<t, w>, smem))) return e;                             \
            cta::ldmd_prop_cta_kernel<t, w><<<njobs, 32 * w, smem, st>>>(sys, jobs, y, nodes, status, kfail); \
        } else if (is_ldmg(iprop)) {                                                                         \
            if ((e = set_smem(cta::ldmg_prop_cta_kernel<t, w>, smem))) return e;                             \
            cta::ldmg_prop_cta_kernel<t, w><<<njobs, 32 * w, smem, st>>>(                                    \
                sys, jobs, iprop == MGPU_PROP_LDMG5 ? 1 : 0, y, nodes, status, kfail);                       \
        } else {                                                                                             \
            if ((e = set_smem(cta::ldj_prop_cta_kernel<t, w>, smem))) return e;                              \
            cta::ldj_prop_cta_kernel<t, w><<<njobs, 32 * w, smem, st>>>(sys, jobs, y, nodes, status, kfail);  \
        }                                                                                                    \
        break;
            MGPU_CTA_BUCKETS(X)
#undef X
        default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    if (kBuckets[b].kind == KIND_FRAG8) {
        const int blocks = (njobs + wf::kWPB - 1) / wf::kWPB;
        switch (nt) {
#define X(t)                                                                                                  \
    case t:                                                                                                   \
        if (iprop == MGPU_PROP_LDMD) {                                                                        \
            if ((e = set_smem(wf::ldmd_prop_frag_kernel<t>, smem))) return e;                                 \
            wf::ldmd_prop_frag_kernel<t><<<blocks, 32 * wf::kWPB, smem, st>>>(sys, jobs, njobs, y, nodes,     \
                                                                              status, kfail);                 \
        } else if (is_ldmg(iprop)) {                                                                          \
            wf::ldmg_prop_frag_kernel<t><<<blocks, 32 * wf::kWPB, 0, st>>>(                                   \
                sys, jobs, njobs, iprop == MGPU_PROP_LDMG5 ? 1 : 0, y, nodes, status, kfail);                 \
        } else {                                                                                              \
            wf::ldj_prop_frag_kernel<t><<<blocks, 32 * wf::kWPB, 0, st>>>(sys, jobs, njobs, y, nodes, status, \
                                                                          kfail);                             \
        }                                                                                                     \
        break;
            MGPU_FRAG_BUCKETS(X)
#undef X
        default: return cudaErrorInvalidValue;
        }
        return cudaGetLastError();
    }
    switch (nt) {
#define X(t)                                                                                                \
    case t:                                                                                                 \
        if (iprop == MGPU_PROP_LDMD) {                                                                      \
            if ((e = set_smem(ldmd_prop_kernel<kT, t>, smem))) return e;                                    \
            ldmd_prop_kernel<kT, t><<<njobs, Geom<kT, t>::NTHR, smem, st>>>(sys, jobs, y, nodes, status,    \
                                                                           kfail, vl_smem);                 \
        } else {                                                                                            \
            if ((e = set_smem(ldj_prop_kernel<kT, t>, smem))) return e;                                     \
            ldj_prop_kernel<kT, t><<<njobs, Geom<kT, t>::NTHR, smem, st>>>(sys, jobs, y, nodes, status,     \
                                                                          kfail, vl_smem);                  \
        }                                                                                                   \
        break;
        MGPU_BUCKETS(X)
#undef X
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// Element (i, j) of tile t, position e, for either layout.
static void tile_element(int b, int t, int e, int *i, int *j)
{
    int I = 0;
    while ((I + 1) * (I + 2) / 2 <= t) ++I;
    const int J = t - I * (I + 1) / 2;
    if (frag_layout(b)) {
        const int lane = e >> 1, s = e & 1;
        *i = 8 * I + (lane >> 2);
        *j = 8 * J + 2 * (lane & 3) + s;
    } else {
        *i = kT * I + e / kT;
        *j = kT * J + e % kT;
    }
}

// Offset of (term l, tile t, position e) in the system's VL/IV/2HQ(C) arrays.
static size_t tile_offset(int b, int l, int t, int e)
{
    const int nt = ntiles_of(b);
    if (frag_layout(b)) return ((size_t)l * nt + t) * 64 + e;
    return ((size_t)l * tile_elems(b) + e) * nt + t;
}

}  // namespace mgpu

// ===========================================================================
// host side
// ===========================================================================
using namespace mgpu;

static thread_local std::string g_last_error;

static int set_err(int code, const char *what, cudaError_t e = cudaSuccess)
{
    char buf[512];
    if (e != cudaSuccess)
        snprintf(buf, sizeof buf, "%s: %s", what, cudaGetErrorString(e));
    else
        snprintf(buf, sizeof buf, "%s", what);
    g_last_error = buf;
    return code;
}

// Device state of one large-N bucket of a run: per-job tiled matrices, one
// round's scratch (X/B twice for the look-ahead), descriptors, step counter.
struct BigBucket {
    int b = 0, nt = 0, npad = 0, max_nstep = 0;
    size_t td = 0;                        // doubles of one tiled matrix
    int M = 0;                            // jobs
    const JobDev *d_jobs = nullptr;       // this bucket's jobs
    big::MatDesc *d_md = nullptr;         // per job: Y (MDPROP) or Z (LDPROP)
    big::MatDesc *d_mduz = nullptr;       // LDPROP: [U of every job, Z of every job]; MGPROP: Y counted with sign -1
    double *tiles = nullptr, *tiles2 = nullptr, *vec = nullptr;
    int *ctr = nullptr;                   // [3][M]: pivot count, status, failing step
    big::Panels pn[2]{};                  // shared Lam / 1/delta, X and B twice
    int pcap = 0;                         // matrices one round's scratch holds
    int *kstep = nullptr, *kzero = nullptr;
    cudaGraphExec_t step_graph = nullptr; // one step of the loop, captured once, replayed NSTEP times
    std::vector<int> prep_sys;            // MDPROP: systems whose U(C) this bucket prepares ...
    std::vector<big::MatDesc *> prep_md;  // ... and the descriptors of their steps
};

// Device allocation and host -> device upload, injected so that plans
// (synchronous) and server batches (stream-ordered) share the set-up code.
using AllocFn = std::function<cudaError_t(void **, size_t)>;
using UploadFn = std::function<cudaError_t(void *, const void *, size_t)>;

template <class X>
static cudaError_t alloc_n(const AllocFn &al, X **p, size_t n)
{
    void *q = nullptr;
    cudaError_t e = al(&q, std::max<size_t>(n, 1) * sizeof(X));
    *p = (X *)q;
    return e;
}

template <class X>
static cudaError_t put_n(const AllocFn &al, const UploadFn &up, X **p, const X *src, size_t n)
{
    cudaError_t e = alloc_n(al, p, n);
    if (e == cudaSuccess && n) e = up(*p, src, n * sizeof(X));
    return e;
}

// The look-ahead streams and events of a large-N bucket.
struct BigAux {
    cudaStream_t side;  // high priority: factor and panel (and, above NT = 32, the diagonal-block update)
    cudaEvent_t evf, evj;
};

struct mgpu_plan {
    int iprop = 0;
    int nsys = 0, njobs = 0;
    std::vector<int> sys_n, sys_bucket, sys_nstep, sys_nham;
    std::vector<int> sys_owner;    // the system whose tables (and U(C) preparation) this one uses; itself if none
    int nshared = 0;               // systems using another's tables
    std::vector<size_t> yoff;      // per job, caller order
    size_t yelems = 0;
    double flops = 0.0;       // 3N^3 + 2 NHAM N(N+1) per job step (the reference's count)
    double flops_prop = 0.0;  // what the propagation kernels do: (2|3)N^3 + 2 NHAM N(N+1) per job step
    double flops_prep = 0.0;  // LDMD preparation: N^3 + NHAM N(N+1) per system step
    // device memory
    std::vector<void *> allocs;
    SysDev *d_sys = nullptr;
    JobDev *d_jobs = nullptr;
    int *d_syslists = nullptr;
    int *d_prep = nullptr;
    // per bucket ranges (jobs sorted by bucket, systems listed by bucket)
    std::vector<int> bucket_ids, job_begin, job_count, sys_begin, sys_count, max_nstep, vl_smem;
    std::vector<size_t> smem;
    std::vector<BigBucket> big;            // large-N buckets (KIND_BIG)
    // Y -> S on the device (every system N <= 1024): channel order NB per system, NOPEN and S offsets per job;
    // jobs with N <= 64 in shared memory (d_sjobs), the others with their matrices in a global scratch
    bool s_ok = false;
    std::vector<int> nopen;
    std::vector<size_t> soff;
    size_t selems = 0;
    size_t s_smem = 0, s_smem_g = 0;
    int ns_small = 0, ns_large = 0;
    size_t sscr_elems = 0;
    double *d_sscr = nullptr;
    smx::SJob *d_sjobs = nullptr, *d_sjobs_g = nullptr;
    int *d_nb = nullptr, *d_nb_off = nullptr;
    double *d_sr = nullptr, *d_si = nullptr;
    size_t s_cap = 0;
    // per-system inputs of Y -> S: thresholds and L(L+1) (host copies for the
    // channel order, device pointers for the kernels), the matching radius,
    // and YTRANS's asymptotic basis where the caller set one
    std::vector<std::vector<double>> s_eint;
    std::vector<const double *> s_deint, s_dcent, s_devec;
    std::vector<double> s_rmatch;
    std::vector<int> job_sys;
    std::vector<double> job_ered;
    int n_evec = 0;                        // systems with an asymptotic basis
    double *d_yz = nullptr, *d_yt = nullptr;  // the transform's product and result (yelems each)
    int sn_max = 0;
    // Streams of the large-N buckets: each bucket's step loop runs on its own
    // stream (never the legacy stream: graph capture) with a high-priority
    // look-ahead stream beside it, so buckets of different N overlap on the GPU.
    struct BigStreams {
        cudaStream_t st = nullptr, side = nullptr;
        cudaEvent_t evf = nullptr, evj = nullptr, done = nullptr;
        BigAux aux() const { return BigAux{side, evf, evj}; }
    };
    std::vector<BigStreams> bstreams;
    cudaStream_t own = nullptr;            // run_host's copies and launches
    cudaEvent_t ev_in = nullptr;
    // stop controls the step kernels poll: [0] cancel, [1] time budget (ns).
    // They live in device memory (a poll is an L2 read, not a PCIe round
    // trip from every warp); the host writes them from a pinned mirror on a
    // stream of their own, which the copy engine serves while kernels run.
    long long *ctl = nullptr;            // pinned host mirror
    long long *d_ctl = nullptr;
    cudaStream_t ctl_stream = nullptr;
    std::mutex ctl_mu;
    // host staging for run_host
    double *d_y = nullptr;
    std::vector<int> job_n;           // N of each job, caller order
    long long *d_job_yoff = nullptr;  // caller-order Y offsets and N, for the matching kernel
    int *d_job_n = nullptr;
    int *d_mpairs = nullptr, *d_mcounts = nullptr;
    int m_cap = 0;
    int *d_nodes = nullptr, *d_status = nullptr, *d_kfail = nullptr;
    size_t y_cap = 0;
    int out_cap = 0;

    ~mgpu_plan()
    {
        if (own) cudaStreamSynchronize(own);
        for (auto &q : bstreams)
            if (q.st) cudaStreamSynchronize(q.st);
        for (auto &g : big)
            if (g.step_graph) cudaGraphExecDestroy(g.step_graph);
        for (auto &q : bstreams) {
            if (q.evf) cudaEventDestroy(q.evf);
            if (q.evj) cudaEventDestroy(q.evj);
            if (q.done) cudaEventDestroy(q.done);
            if (q.side) cudaStreamDestroy(q.side);
            if (q.st) cudaStreamDestroy(q.st);
        }
        if (ev_in) cudaEventDestroy(ev_in);
        if (own) cudaStreamDestroy(own);
        for (void *p : allocs) cudaFree(p);
        if (d_y) cudaFree(d_y);
        if (d_sscr) cudaFree(d_sscr);
        if (d_mpairs) cudaFree(d_mpairs);
        if (d_mcounts) cudaFree(d_mcounts);
        if (d_nodes) cudaFree(d_nodes);
        if (d_status) cudaFree(d_status);
        if (d_kfail) cudaFree(d_kfail);
        if (d_sr) cudaFree(d_sr);
        if (d_si) cudaFree(d_si);
        if (d_yz) cudaFree(d_yz);
        if (d_yt) cudaFree(d_yt);
        if (ctl) cudaFreeHost((void *)ctl);  // d_ctl is one of `allocs`
        if (ctl_stream) cudaStreamDestroy(ctl_stream);
    }
    void dfree(void *q)
    {
        if (!q) return;
        for (auto it = allocs.begin(); it != allocs.end(); ++it)
            if (*it == q) {
                allocs.erase(it);
                break;
            }
        cudaFree(q);
    }
    template <class X>
    cudaError_t dalloc(X **p, size_t count)
    {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(X));
        if (e == cudaSuccess) allocs.push_back(q);
        *p = (X *)q;
        return e;
    }
};

template <class X>
static cudaError_t upload(mgpu_plan *p, X **dst, const X *src, size_t count)
{
    cudaError_t e = p->dalloc(dst, count);
    if (e != cudaSuccess) return e;
    if (count) e = cudaMemcpy(*dst, src, count * sizeof(X), cudaMemcpyHostToDevice);
    return e;
}

// -A^{-1} in place for M matrices of a large-N bucket, 64 pivots a round
// (factor, panel and update kernels); the X/B operands alternate between two
// buffers.  Look-ahead: once the next round's diagonal block is updated, its
// factor runs on the high-priority `side` stream; once the rest of the next
// panel's tile row and column is updated, the next round's panel follows it
// there, while `st` updates the remaining tiles.  Above NT = 32 (N > 256) the
// diagonal-block update itself runs on `side`, beside the block row and
// column on `st` (+1.2-1.7 % at N = 512 and 1024, 3 % slower at N = 256;
// bit-identical: the three update launches of a round touch disjoint tiles).
// Each wait on `evf` takes the record made just before it.
static cudaError_t big_invert(const big::MatDesc *md, int M, int nt, const big::Panels (&pn)[2], const int *kstep,
                              cudaStream_t st, const BigAux &ax)
{
    const int rounds = nt / big::KB;
    const int nbk = nt / 8;
    const dim3 gp((nt + big::PANEL_WARPS - 1) / big::PANEL_WARPS, M), gall(big::UPD_SPLIT * nbk * (nbk + 1) / 2, M),
        gcol(big::UPD_SPLIT * (nbk - 1), M), gdiag(big::UPD_SPLIT, M);
    const int ut = 32 * big::UPD_WARPS, pt = 32 * big::PANEL_WARPS;
    cudaStream_t side = ax.side;
    const bool diag_side = nt > big::FACT_BIG_MAX_NT;
    cudaError_t e;
    auto factor = [&](const big::Panels &p, int R, cudaStream_t s) {
        if (nt <= big::FACT_BIG_MAX_NT)
            big::big_factor_kernel<big::FACT_THREADS_BIG><<<M, big::FACT_THREADS_BIG, big::kFactSmem, s>>>(md, p, R, kstep);
        else
            big::big_factor_kernel<big::FACT_THREADS><<<M, big::FACT_THREADS, big::kFactSmem, s>>>(md, p, R, kstep);
    };
    factor(pn[0], 0, st);
    big::big_panel_kernel<<<gp, pt, 0, st>>>(md, pn[0], nt, 0, kstep);
    for (int R = 0; R < rounds; ++R) {
        const big::Panels &cur = pn[R & 1], &nxt = pn[(R + 1) & 1];
        if (R + 1 < rounds) {
            if (diag_side) {
                if ((e = cudaEventRecord(ax.evf, st)) || (e = cudaStreamWaitEvent(side, ax.evf, 0))) return e;
                big::big_update_kernel<<<gdiag, ut, big::kUpdSmem, side>>>(md, cur, nt, R, kstep, big::UPD_DIAG, R + 1);
                factor(nxt, R + 1, side);
                big::big_update_kernel<<<gcol, ut, big::kUpdSmem, st>>>(md, cur, nt, R, kstep, big::UPD_ONLY, R + 1);
                if ((e = cudaEventRecord(ax.evf, st)) || (e = cudaStreamWaitEvent(side, ax.evf, 0))) return e;
                big::big_panel_kernel<<<gp, pt, 0, side>>>(md, nxt, nt, R + 1, kstep);
                if ((e = cudaEventRecord(ax.evj, side))) return e;
                big::big_update_kernel<<<gall, ut, big::kUpdSmem, st>>>(md, cur, nt, R, kstep, big::UPD_EXCEPT, R + 1);
                if ((e = cudaStreamWaitEvent(st, ax.evj, 0))) return e;
            } else {
                big::big_update_kernel<<<gdiag, ut, big::kUpdSmem, st>>>(md, cur, nt, R, kstep, big::UPD_DIAG, R + 1);
                if ((e = cudaEventRecord(ax.evf, st)) || (e = cudaStreamWaitEvent(side, ax.evf, 0))) return e;
                factor(nxt, R + 1, side);
                big::big_update_kernel<<<gcol, ut, big::kUpdSmem, st>>>(md, cur, nt, R, kstep, big::UPD_ONLY, R + 1);
                if ((e = cudaEventRecord(ax.evf, st)) || (e = cudaStreamWaitEvent(side, ax.evf, 0))) return e;
                big::big_panel_kernel<<<gp, pt, 0, side>>>(md, nxt, nt, R + 1, kstep);
                if ((e = cudaEventRecord(ax.evj, side))) return e;
                big::big_update_kernel<<<gall, ut, big::kUpdSmem, st>>>(md, cur, nt, R, kstep, big::UPD_EXCEPT, R + 1);
                if ((e = cudaStreamWaitEvent(st, ax.evj, 0))) return e;
            }
        } else {
            big::big_update_kernel<<<gall, ut, big::kUpdSmem, st>>>(md, cur, nt, R, kstep, big::UPD_ALL, -1);
        }
    }
    return cudaGetLastError();
}

static unsigned big_ew_blocks(size_t td) { return (unsigned)std::min<size_t>((td + big::EW_THREADS - 1) / big::EW_THREADS, 256); }

// One system in bucket b's tile layout on the device: VL/IV tiled (sumlam.f
// pair order), EINT/CENT padded, radial tables, MDPROP 2HQ(C) storage.
static int build_sysdev(const mgpu_coupling &c, const mgpu_grid &g, int iprop, int b, SysDev &d, const AllocFn &al,
                        const UploadFn &up)
{
    const int npad = bucket_npad(b);
    const int nt = ntiles_of(b);
    const size_t TT = tile_elems(b);
    const size_t tsz = (size_t)std::max(c.nham, 1) * TT * nt;
    std::vector<double> vlt(tsz, 0.0);
    std::vector<int> ivt(c.ivlfl > 0 ? tsz : 1, 0);
    for (int t = 0; t < nt; ++t)
        for (int ee = 0; ee < (int)TT; ++ee) {
            int i = 0, j = 0;
            tile_element(b, t, ee, &i, &j);
            if (i >= c.n || j >= c.n) continue;
            const int lo = std::min(i, j), hi = std::max(i, j);
            // pair (row lo, column hi) of the packed upper triangle (sumlam.f:33-36,74-86)
            const size_t pair = (size_t)hi * (hi + 1) / 2 + lo;
            for (int l = 0; l < c.nham; ++l) {
                const size_t src = pair * c.nvlblk + l;
                const size_t dst = tile_offset(b, l, t, ee);
                vlt[dst] = c.vl[src];
                if (c.ivlfl > 0) {
                    const int ix = c.iv[src] - 1;
                    if (ix < 0 || ix >= c.nham) return set_err(MGPU_ERR_ARG, "IV index outside 1..NHAM");
                    ivt[dst] = ix;
                }
            }
        }
    std::vector<double> eint(npad, 0.0), cent(npad, 0.0);
    std::copy(c.eint, c.eint + c.n, eint.begin());
    std::copy(c.cent, c.cent + c.n, cent.begin());
    memset(&d, 0, sizeof d);
    d.n = c.n;
    d.nham = c.nham;
    d.ivlfl = c.ivlfl;
    d.nconst = c.nconst;
    d.nrsq = c.nrsq;
    d.nstep = g.nstep;
    d.ntiles = nt;
    d.kind = frag_layout(b) ? 1 : 0;
    d.conlen = c.conlen;
    d.dr = g.dr;
    // rows of the radial tables: MDPROP/LDPROP's half steps, MGPROP's stages
    const size_t nr = is_ldmg(iprop) ? (size_t)(iprop == MGPU_PROP_LDMG5 ? 6 * (size_t)g.nstep : 4 * (size_t)g.nstep + 1)
                                     : 2 * (size_t)g.nstep + 1;
    double *dv = nullptr, *de = nullptr, *dc = nullptr, *drt = nullptr, *dpt = nullptr, *dq = nullptr;
    int *di = nullptr;
    std::vector<double> pt(std::max<size_t>(nr * c.nham, 1), 0.0);
    if (c.nham > 0) std::copy(g.ptab, g.ptab + nr * c.nham, pt.begin());
    cudaError_t e;
    if ((e = put_n(al, up, &dv, vlt.data(), vlt.size())) || (e = put_n(al, up, &di, ivt.data(), ivt.size())) ||
        (e = put_n(al, up, &de, eint.data(), eint.size())) || (e = put_n(al, up, &dc, cent.data(), cent.size())) ||
        (e = put_n(al, up, &drt, g.rtab, nr)) || (e = put_n(al, up, &dpt, pt.data(), pt.size())))
        return set_err(MGPU_ERR_NOMEM, "uploading a system", e);
    if (iprop == MGPU_PROP_LDMD && (e = alloc_n(al, &dq, (size_t)g.nstep * TT * nt)))
        return set_err(MGPU_ERR_NOMEM, "allocating the 2HQ(C) table", e);
    double *dwt = nullptr, *dwd = nullptr;
    if (iprop == MGPU_PROP_LDMD && kBuckets[b].kind == KIND_FRAG8 &&
        ((e = alloc_n(al, &dwt, ((size_t)g.nstep + 1) * TT * nt)) || (e = alloc_n(al, &dwd, (size_t)g.nstep * npad))))
        return set_err(MGPU_ERR_NOMEM, "allocating the coupling-sum tables", e);
    d.vlt = dv;
    d.ivt = di;
    d.eint = de;
    d.cent = dc;
    d.rtab = drt;
    d.ptab = dpt;
    d.q = dq;
    d.wt = dwt;
    d.wd = dwd;
    d.ctl = nullptr;
    return MGPU_OK;
}

// Two systems share device tables when they differ at most in EINT and CENT:
// the same VL, IV, P and R arrays (by address) and the same sizes and flags.
// EINT and CENT enter W only on its diagonal, and MDPROP's U(C) uses only the
// off-diagonal coupling (mdprop.f:104-130), so such systems also share the
// 2HQ(C) tables and their preparation.  A field sweep in a basis where the
// field term is diagonal (the uncoupled alkali-pair basis, whose Zeeman term
// becomes a per-field EINT) is the case this serves: one preparation for
// every field.
static bool shares_tables(const mgpu_coupling &a, const mgpu_grid &ga, const mgpu_coupling &b, const mgpu_grid &gb)
{
    return a.n == b.n && a.nham == b.nham && a.nvlblk == b.nvlblk && a.ivlfl == b.ivlfl && a.nconst == b.nconst &&
           a.nrsq == b.nrsq && a.conlen == b.conlen && a.vl == b.vl && (a.ivlfl <= 0 || a.iv == b.iv) &&
           ga.nstep == gb.nstep && ga.dr == gb.dr && ga.rtab == gb.rtab && ga.ptab == gb.ptab;
}

constexpr int kPrepChunk = 128;  // U(C) steps inverted per preparation batch

// Device state of one large-N bucket: M jobs (host copies `jobs`, device
// `d_jobs`), and for MDPROP the U(C) descriptors of the systems `prep_sys`.
// hs / sys_n / sys_nstep are indexed by the system ids the jobs carry;
// d_prep points at the [3] counters of system 0.
static int setup_big(BigBucket &g, int iprop, int b, const JobDev *jobs, const JobDev *d_jobs, int M, int max_nstep,
                     const std::vector<int> &prep_sys, const std::vector<SysDev> &hs, const std::vector<int> &sys_n,
                     const std::vector<int> &sys_nstep, int *d_prep, const AllocFn &al, const UploadFn &up)
{
    cudaError_t e;
    const bool ldj = iprop == MGPU_PROP_LDJ;
    g.b = b;
    g.nt = kBuckets[b].nt;
    g.npad = bucket_npad(b);
    g.td = matrix_elems(b);
    g.M = M;
    g.d_jobs = d_jobs;
    g.max_nstep = max_nstep;
    if (M > 65535) return set_err(MGPU_ERR_UNSUPPORTED, "more than 65535 large-N propagations in one bucket");
    int maxsteps = 0;
    for (int sidx : prep_sys) maxsteps = std::max(maxsteps, sys_nstep[sidx]);
    g.pcap = std::max({(ldj ? 2 : 1) * M, std::min(maxsteps, kPrepChunk), 1});
    const size_t fr = (size_t)g.nt * big::MC * 32;  // doubles of one operand panel
    int zero = 0;
    if ((e = alloc_n(al, &g.pn[0].lam, (size_t)g.pcap * big::NB * big::NB)) ||
        (e = alloc_n(al, &g.pn[0].rd, (size_t)g.pcap * big::NB)) || (e = alloc_n(al, &g.pn[0].xf, (size_t)g.pcap * fr)) ||
        (e = alloc_n(al, &g.pn[0].bf, (size_t)g.pcap * fr)) || (e = alloc_n(al, &g.pn[1].xf, (size_t)g.pcap * fr)) ||
        (e = alloc_n(al, &g.pn[1].bf, (size_t)g.pcap * fr)) || (e = put_n(al, up, &g.kstep, &zero, 1)) ||
        (e = put_n(al, up, &g.kzero, &zero, 1)) ||
        (M && ((e = alloc_n(al, &g.tiles, (size_t)M * g.td)) || (e = alloc_n(al, &g.ctr, (size_t)3 * M)) ||
               (ldj && (e = alloc_n(al, &g.tiles2, (size_t)M * g.td))) ||
               (iprop == MGPU_PROP_LDMD && (e = alloc_n(al, &g.vec, (size_t)M * 3 * g.npad))))))
        return set_err(MGPU_ERR_NOMEM, "allocating large-N matrices", e);
    g.pn[1].lam = g.pn[0].lam;
    g.pn[1].rd = g.pn[0].rd;
    if (M) {
        std::vector<big::MatDesc> md(M), uz;
        for (int j = 0; j < M; ++j) {
            big::MatDesc &d = md[j];
            d.a = g.tiles + (size_t)j * g.td;
            d.cnt = g.ctr + j;
            d.stat = g.ctr + M + j;
            d.kfail = g.ctr + 2 * M + j;
            d.n = sys_n[jobs[j].sys];
            d.sign = 1;
            d.nstep = sys_nstep[jobs[j].sys];
            d.kfix = 0;
        }
        if (ldj) {
            uz = md;
            for (int j = 0; j < M; ++j) {
                uz[j].a = g.tiles2 + (size_t)j * g.td;
                uz[j].sign = -1;
            }
            uz.insert(uz.end(), md.begin(), md.end());
        } else if (is_ldmg(iprop)) {
            uz = md;  // the same matrices counted with sign -1: MGPROP's stages with a_k < 0
            for (int j = 0; j < M; ++j) uz[j].sign = -1;
        }
        if ((e = put_n(al, up, &g.d_md, md.data(), md.size())) ||
            (!uz.empty() && (e = put_n(al, up, &g.d_mduz, uz.data(), uz.size()))))
            return set_err(MGPU_ERR_NOMEM, "uploading large-N descriptors", e);
    }
    if (!ldj)
        for (int sidx : prep_sys) {
            const int ns = sys_nstep[sidx];
            std::vector<big::MatDesc> md(ns);
            for (int k = 1; k <= ns; ++k) {
                big::MatDesc &d = md[k - 1];
                d.a = hs[sidx].q + (size_t)(k - 1) * g.td;
                d.cnt = d_prep + 3 * sidx;
                d.stat = d_prep + 3 * sidx + 1;
                d.kfail = d_prep + 3 * sidx + 2;
                d.n = sys_n[sidx];
                d.sign = 1;
                d.nstep = 0x7fffffff;
                d.kfix = k;
            }
            big::MatDesc *dm = nullptr;
            if ((e = put_n(al, up, &dm, md.data(), md.size())))
                return set_err(MGPU_ERR_NOMEM, "uploading preparation descriptors", e);
            g.prep_sys.push_back(sidx);
            g.prep_md.push_back(dm);
        }
    return MGPU_OK;
}

// MDPROP preparation of a large-N bucket's systems: U(C_k) for every step,
// inverted in batches of steps, turned into 2HQ(C_k).
static cudaError_t run_big_prep(const BigBucket &g, const SysDev *d_sys, const std::vector<int> &sys_nstep,
                                cudaStream_t st, const BigAux &ax)
{
    cudaError_t e;
    for (size_t i = 0; i < g.prep_sys.size(); ++i) {
        const int s = g.prep_sys[i], ns = sys_nstep[s];
        for (int k0 = 1; k0 <= ns; k0 += g.pcap) {
            const int c = std::min(g.pcap, ns - k0 + 1);
            const dim3 grid(big_ew_blocks(g.td), c);
            big::big_prep_build_kernel<<<grid, big::EW_THREADS, 0, st>>>(d_sys, s, k0, g.td);
            if ((e = big_invert(g.prep_md[i] + (k0 - 1), c, g.nt, g.pn, g.kzero, st, ax))) return e;
            big::big_prep_finish_kernel<<<grid, big::EW_THREADS, 0, st>>>(d_sys, s, k0, g.td);
            if ((e = cudaGetLastError())) return e;
        }
    }
    return cudaSuccess;
}

// The step loop of a large-N bucket: start, NSTEP x (elementwise, inversions),
// results into y / nodes / status / kfail (indexed by JobDev::yoff / ::out).
// `st` must not be the legacy default stream: one step (its ~5 x NT/8 x 2
// launches, look-ahead fork/join included) is captured into a CUDA graph on
// first use and replayed NSTEP times; the device-side step counter makes
// every replay the next step.  The graph stays in g.step_graph for reuse.
static cudaError_t run_big_prop(BigBucket &g, int iprop, const SysDev *d_sys, double *y, int *nodes, int *status,
                                int *kfail, cudaStream_t st, const BigAux &ax)
{
    if (g.M == 0) return cudaSuccess;
    cudaError_t e = cudaSuccess;
    const bool ldj = iprop == MGPU_PROP_LDJ;
    big::StepArgs a{d_sys, g.d_jobs, g.d_md, g.tiles2, g.vec, g.kstep, g.npad, g.td};
    const dim3 ew(big_ew_blocks(g.td), g.M), ev((g.npad + big::EW_THREADS - 1) / big::EW_THREADS, g.M);
    auto one_step = [&]() -> cudaError_t {
        cudaError_t x;
        if (is_ldmg(iprop)) {
            // one sector: the stages of mgprop.f:75-131 with the coefficients of the method
            const wf::MGCoef &mc = wf::kMGCoef[iprop == MGPU_PROP_LDMG5 ? 1 : 0];
            for (int k = 0; k < mc.m; ++k) {
                big::big_ldmg_stage_kernel<<<ew, big::EW_THREADS, 0, st>>>(a, mc.stride, k, mc.b[k], mc.a[k]);
                if (mc.a[k] == 0.0) continue;
                if ((x = big_invert(mc.a[k] >= 0.0 ? g.d_md : g.d_mduz, g.M, g.nt, g.pn, g.kstep, st, ax)))
                    return x;
                big::big_ldmg_after_kernel<<<ew, big::EW_THREADS, 0, st>>>(a, mc.a[k]);
            }
        } else if (ldj) {
            big::big_ldj_pre_kernel<<<ew, big::EW_THREADS, 0, st>>>(a);
            if ((x = big_invert(g.d_mduz, 2 * g.M, g.nt, g.pn, g.kstep, st, ax))) return x;  // U and Z
            big::big_ldj_mid_kernel<<<ew, big::EW_THREADS, 0, st>>>(a);
            if ((x = big_invert(g.d_md, g.M, g.nt, g.pn, g.kstep, st, ax))) return x;
            big::big_ldj_post_kernel<<<ew, big::EW_THREADS, 0, st>>>(a);
        } else {
            big::big_ldmd_pre_kernel<<<ev, big::EW_THREADS, 0, st>>>(a);
            if ((x = big_invert(g.d_md, g.M, g.nt, g.pn, g.kstep, st, ax))) return x;
            big::big_ldmd_mid_kernel<<<ew, big::EW_THREADS, 0, st>>>(a);
            if ((x = big_invert(g.d_md, g.M, g.nt, g.pn, g.kstep, st, ax))) return x;
            big::big_ldmd_post_kernel<<<ew, big::EW_THREADS, 0, st>>>(a);
        }
        big::big_step_advance_kernel<<<1, 1, 0, st>>>(g.kstep, -1);
        return cudaGetLastError();
    };
    if (!g.step_graph) {
        cudaGraph_t graph = nullptr;
        if ((e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal))) return e;
        const cudaError_t e1 = one_step();
        const cudaError_t e2 = cudaStreamEndCapture(st, &graph);
        if (e1 || e2) {
            if (graph) cudaGraphDestroy(graph);
            return e1 ? e1 : e2;
        }
        e = cudaGraphInstantiate(&g.step_graph, graph, 0);
        cudaGraphDestroy(graph);
        if (e) {
            g.step_graph = nullptr;
            return e;
        }
    }
    big::big_step_advance_kernel<<<1, 1, 0, st>>>(g.kstep, 1);
    if (is_ldmg(iprop)) big::big_ldmg_init_kernel<<<ew, big::EW_THREADS, 0, st>>>(a, y);
    else if (ldj) big::big_ldj_init_kernel<<<ew, big::EW_THREADS, 0, st>>>(a, y);
    else big::big_ldmd_init_kernel<<<ew, big::EW_THREADS, 0, st>>>(a, y);
    for (int k = 1; k <= g.max_nstep; ++k)
        if ((e = cudaGraphLaunch(g.step_graph, st))) return e;
    big::big_finish_kernel<<<ew, big::EW_THREADS, 0, st>>>(a, is_ldmg(iprop) ? 2 : (ldj ? 1 : 0), y, nodes, status,
                                                            kfail);
    return cudaGetLastError();
}

// the kernels' attributes (dynamic shared memory above 48 KB), once per device
static cudaError_t big_kernel_attributes()
{
    cudaError_t e;
    if ((e = set_smem(big::big_update_kernel, big::kUpdSmem)) || (e = set_smem(big::big_factor_kernel<big::FACT_THREADS>, big::kFactSmem)) ||
        (e = set_smem(big::big_factor_kernel<big::FACT_THREADS_BIG>, big::kFactSmem)))
        return e;
    return cudaSuccess;
}

static int check_coupling(const mgpu_coupling *c, const mgpu_grid *g, int iprop)
{
    if (!c || !g) return set_err(MGPU_ERR_ARG, "null system or grid");
    if (c->n < 1) return set_err(MGPU_ERR_ARG, "N must be >= 1");
    if (c->nham < 0 || c->nvlblk < c->nham) return set_err(MGPU_ERR_ARG, "need 0 <= NHAM <= NVLBLK");
    if (c->nham > 0 && !c->vl) return set_err(MGPU_ERR_ARG, "VL is null");
    if (c->ivlfl > 0 && !c->iv) return set_err(MGPU_ERR_ARG, "IVLFL>0 but IV is null");
    if (!c->eint || !c->cent) return set_err(MGPU_ERR_ARG, "EINT/CENT null");
    if (g->nstep < 1) return set_err(MGPU_ERR_ARG, "NSTEP must be >= 1");
    if (!g->rtab || (c->nham > 0 && !g->ptab)) return set_err(MGPU_ERR_ARG, "radial tables null");
    if (!(g->dr != 0.0) || !std::isfinite(g->dr)) return set_err(MGPU_ERR_ARG, "DR must be finite and non-zero");
    if (bucket_for(c->n, iprop) < 0)
        return set_err(MGPU_ERR_UNSUPPORTED, "N above 1024 (largest compiled bucket)");
    return MGPU_OK;
}

extern "C" {

int mgpu_ldmg_radii(int iprop, double rstart, double dr, int nstep, double *rtab)
{
    if (!is_ldmg(iprop) || nstep < 1) return -1;
    const wf::MGCoef &m = wf::kMGCoef[iprop == MGPU_PROP_LDMG5 ? 1 : 0];
    int cnt = 0;
    for (int s = 0; s < nstep; ++s) {
        double r = rstart + s * dr;  // mgprop.f:76
        for (int k = 0; k < m.m; ++k) {
            const bool reused = (k == 0 && s > 0 && m.stride < m.m);  // the previous sector's last W
            if (!reused) {
                if (rtab) rtab[cnt] = r;
                ++cnt;
            }
            r = r + m.a[k] * dr;  // mgprop.f:129
        }
    }
    return cnt;
}

int mgpu_max_n(void)
{
    int m = 0;
    for (int b = 0; b < kNumBuckets; ++b) m = std::max(m, bucket_npad(b));
    return m;
}

int mgpu_set_kernel_family(int family)
{
    const int old = g_prefer_tile4;
    g_prefer_tile4 = family == 1 ? 1 : 0;
    return old;
}

int mgpu_set_family_for_n(int iprop, int n_lo, int n_hi, int family)
{
    std::lock_guard<std::mutex> lk(g_family_mu);
    if (iprop != 0 && iprop != MGPU_PROP_LDMD && iprop != MGPU_PROP_LDJ)
        return set_err(MGPU_ERR_ARG, "IPROP must be 0 (both), 5 or 6");
    if (family < 0) {
        g_family_ranges.erase(std::remove_if(g_family_ranges.begin(), g_family_ranges.end(),
                                             [iprop](const FamilyRange &r) { return iprop == 0 || r.iprop == iprop; }),
                              g_family_ranges.end());
        return MGPU_OK;
    }
    if (family > 2 || n_lo < 1 || n_hi < n_lo) return set_err(MGPU_ERR_ARG, "family 0..2 and 1 <= n_lo <= n_hi");
    g_family_ranges.insert(g_family_ranges.begin(), FamilyRange{iprop, n_lo, n_hi, family});  // latest wins
    return MGPU_OK;
}

int mgpu_probe_fp64_fma(double *out_dev, int iters, void *stream, double *flops_out)
{
    if (!out_dev || iters < 1) return set_err(MGPU_ERR_ARG, "probe arguments");
    int dev = 0, sms = 0, perSM = 0;
    cudaError_t e;
    if ((e = cudaGetDevice(&dev)) || (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)))
        return set_err(MGPU_ERR_CUDA, "probe device query", e);
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fp64_fma_probe_kernel, 256, 0)))
        return set_err(MGPU_ERR_CUDA, "probe occupancy", e);
    const int blocks = sms * std::max(perSM, 1);
    fp64_fma_probe_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(out_dev, iters);
    if ((e = cudaGetLastError())) return set_err(MGPU_ERR_CUDA, "probe launch", e);
    if (flops_out) *flops_out = 2.0 * 8.0 * 16.0 * (double)iters * 256.0 * (double)blocks;
    return MGPU_OK;
}

// Write the stop controls to the device: from the pinned mirror, on the
// controls' own stream (served by the copy engine beside running kernels),
// waited for before returning.
static int push_ctl(mgpu_plan *plan)
{
    cudaError_t e;
    if ((e = cudaMemcpyAsync(plan->d_ctl, plan->ctl, 2 * sizeof(long long), cudaMemcpyHostToDevice,
                             plan->ctl_stream)) ||
        (e = cudaStreamSynchronize(plan->ctl_stream)))
        return set_err(MGPU_ERR_CUDA, "writing the stop controls", e);
    return MGPU_OK;
}

int mgpu_plan_cancel(mgpu_plan *plan, int on)
{
    if (!plan || !plan->ctl) return set_err(MGPU_ERR_ARG, "null plan");
    std::lock_guard<std::mutex> lk(plan->ctl_mu);
    plan->ctl[0] = on ? 1 : 0;
    return push_ctl(plan);
}

int mgpu_plan_set_time_limit(mgpu_plan *plan, double seconds)
{
    if (!plan || !plan->ctl) return set_err(MGPU_ERR_ARG, "null plan");
    if (!(seconds >= 0.0) || !std::isfinite(seconds)) return set_err(MGPU_ERR_ARG, "time limit must be >= 0");
    const double ns = seconds * 1.0e9;
    std::lock_guard<std::mutex> lk(plan->ctl_mu);
    plan->ctl[1] = (seconds == 0.0) ? 0 : (ns < 1.0 ? 1 : (ns > 9.0e18 ? (long long)9e18 : (long long)ns));
    return push_ctl(plan);
}

int mgpu_set_step_wait_limit(int limit)
{
    const uint32_t v = limit < 0 ? kWaitLimit : (uint32_t)limit;
    cudaError_t e = cudaMemcpyToSymbol(g_step_wait_limit, &v, sizeof v);
    if (e != cudaSuccess) return set_err(MGPU_ERR_CUDA, "setting the step wait limit", e);
    return MGPU_OK;
}

int mgpu_probe_pivot_reciprocal(const double *x_dev, double *r_dev, int n, void *stream)
{
    if (!x_dev || !r_dev || n < 0) return set_err(MGPU_ERR_ARG, "probe arguments");
    if (n == 0) return MGPU_OK;
    pivot_reciprocal_probe_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(x_dev, r_dev, n);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_err(MGPU_ERR_CUDA, "probe launch", e);
    return MGPU_OK;
}

const char *mgpu_last_error(void) { return g_last_error.c_str(); }

const char *mgpu_status_string(int s)
{
    switch (s) {
    case MGPU_OK: return "ok";
    case MGPU_ERR_INVERSION: return "matrix inversion error (zero pivot)";
    case MGPU_ERR_NONFINITE: return "non-finite pivot";
    case MGPU_ERR_ARG: return "invalid argument";
    case MGPU_ERR_CUDA: return "CUDA error";
    case MGPU_ERR_UNSUPPORTED: return "unsupported size";
    case MGPU_ERR_NOMEM: return "device allocation failed";
    case MGPU_ERR_TIMEOUT: return "bounded wait for an asynchronous copy expired";
    case MGPU_ERR_CANCELLED: return "cancelled by the host";
    case MGPU_ERR_DEADLINE: return "time limit of a step kernel exceeded";
    default: return "unknown status";
    }
}

void mgpu_plan_destroy(mgpu_plan *plan) { delete plan; }

size_t mgpu_plan_y_elems(const mgpu_plan *p) { return p ? p->yelems : 0; }

size_t mgpu_plan_y_offset(const mgpu_plan *p, int job)
{
    return (p && job >= 0 && job < p->njobs) ? p->yoff[job] : 0;
}

double mgpu_plan_flops(const mgpu_plan *p) { return p ? p->flops : 0.0; }

int mgpu_plan_shared_systems(const mgpu_plan *p) { return p ? p->nshared : 0; }

double mgpu_plan_flops_phase(const mgpu_plan *p, int phases)
{
    if (!p) return 0.0;
    return ((phases & 1) ? p->flops_prep : 0.0) + ((phases & 2) ? p->flops_prop : 0.0);
}

int mgpu_plan_launches(const mgpu_plan *p)
{
    if (!p) return 0;
    int l = (p->iprop == MGPU_PROP_LDMD) ? 1 : 0;  // prep_reset_kernel
    for (size_t b = 0; b < p->bucket_ids.size(); ++b) {
        if (kBuckets[p->bucket_ids[b]].kind == KIND_BIG) continue;
        if (p->iprop == MGPU_PROP_LDMD && p->sys_count[b] > 0) l += (p->sys_count[b] + 65534) / 65535;
        if (p->job_count[b] > 0) ++l;
    }
    for (const auto &g : p->big) {
        // first factor and panel; then a round: three update launches, factor, panel; one update in the last round
        const int per_inv = 5 * (g.nt / big::KB) - 2;
        if (p->iprop == MGPU_PROP_LDMD)
            for (size_t i = 0; i < g.prep_sys.size(); ++i) {
                const int ns = p->sys_nstep[g.prep_sys[i]];
                const int chunks = (ns + g.pcap - 1) / g.pcap;
                l += chunks * (2 + per_inv);
            }
        if (g.M > 0) {
            int per_step = 4 + 2 * per_inv;  // MDPROP: three elementwise kernels, two inversions, the counter
            if (p->iprop == MGPU_PROP_LDJ) {
                per_step = 4 + 2 * per_inv;
            } else if (is_ldmg(p->iprop)) {
                const wf::MGCoef &mc = wf::kMGCoef[p->iprop == MGPU_PROP_LDMG5 ? 1 : 0];
                per_step = 1;
                for (int k = 0; k < mc.m; ++k) per_step += 1 + (mc.a[k] != 0.0 ? 1 + per_inv : 0);
            }
            l += 3 + g.max_nstep * per_step;
        }
    }
    return l;
}

// The S-matrix descriptors from the plan's per-system S inputs: channel
// order (CHNSRT, chnsrt.f:16-30: by threshold, equal thresholds within
// 1e-11 keep their order), open channels and S offsets per job; jobs with
// N <= 64 in shared memory, the others with their matrices in a scratch.
static int build_s(mgpu_plan *p)
{
    const int nsys = p->nsys, njobs = p->njobs;
    std::vector<int> nb_all, nb_off(nsys);
    for (int s = 0; s < nsys; ++s) {
        const std::vector<double> &ei = p->s_eint[s];
        const int n = (int)ei.size();
        nb_off[s] = (int)nb_all.size();
        std::vector<int> nb(n);
        for (int i = 0; i < n; ++i) nb[i] = i;
        for (int i = 0; i + 1 < n; ++i)
            for (int j = i + 1; j < n; ++j) {
                const double a = ei[nb[i]], bb = ei[nb[j]];
                if (a <= bb || std::fabs(a - bb) < 1.0e-11) continue;
                std::swap(nb[i], nb[j]);
            }
        nb_all.insert(nb_all.end(), nb.begin(), nb.end());
    }
    std::vector<smx::SJob> sj, sjg;
    p->nopen.assign(njobs, 0);
    p->soff.assign(njobs, 0);
    p->s_smem = p->s_smem_g = 0;
    size_t so = 0, scr = 0;
    for (int j = 0; j < njobs; ++j) {
        const int sy = p->job_sys[j];
        const std::vector<double> &ei = p->s_eint[sy];
        const int n = (int)ei.size();
        int no = 0;
        for (int i = 0; i < n; ++i) no += (p->job_ered[j] - ei[i] > 0.0) ? 1 : 0;
        p->nopen[j] = no;
        p->soff[j] = so;
        so += (size_t)no * no;
        smx::SJob q;
        q.sys = sy;
        q.nopen = no;
        q.out = j;
        q.pad = 0;
        q.ered = p->job_ered[j];
        q.yoff = (long long)p->yoff[j];
        q.soff = (long long)p->soff[j];
        q.scr = 0;
        q.eint = p->s_deint[sy];
        q.cent = p->s_dcent[sy];
        q.evec = p->s_devec[sy];
        q.rmatch = p->s_rmatch[sy];
        if (n <= smx::kMaxNShared) {
            p->s_smem = std::max(p->s_smem, smx::smem_bytes(n, no));
            sj.push_back(q);
        } else {
            if (no > 0) {
                q.scr = (long long)scr;
                scr += smx::mat_doubles(n, no);
            }
            p->s_smem_g = std::max(p->s_smem_g, smx::chan_smem_bytes(n));
            sjg.push_back(q);
        }
    }
    p->selems = so;
    if (scr != p->sscr_elems && p->d_sscr) {
        cudaFree(p->d_sscr);
        p->d_sscr = nullptr;
    }
    p->sscr_elems = scr;
    p->ns_small = (int)sj.size();
    p->ns_large = (int)sjg.size();
    p->dfree(p->d_sjobs);
    p->dfree(p->d_sjobs_g);
    p->dfree(p->d_nb);
    p->dfree(p->d_nb_off);
    p->d_sjobs = p->d_sjobs_g = nullptr;
    p->d_nb = p->d_nb_off = nullptr;
    cudaError_t e;
    if (njobs > 0 && ((!sj.empty() && (e = upload(p, &p->d_sjobs, sj.data(), sj.size()))) ||
                      (!sjg.empty() && (e = upload(p, &p->d_sjobs_g, sjg.data(), sjg.size()))) ||
                      (e = upload(p, &p->d_nb, nb_all.data(), nb_all.size())) ||
                      (e = upload(p, &p->d_nb_off, nb_off.data(), nb_off.size()))))
        return set_err(MGPU_ERR_NOMEM, "uploading S-matrix descriptors", e);
    return MGPU_OK;
}

int mgpu_plan_create(mgpu_plan **out, int iprop, int nsys, const mgpu_coupling *systems,
                     const mgpu_grid *grids, int njobs, const int *job_sys, const double *job_ered)
{
    if (!out) return set_err(MGPU_ERR_ARG, "null plan pointer");
    *out = nullptr;
    if (iprop != MGPU_PROP_LDMD && iprop != MGPU_PROP_LDJ && !is_ldmg(iprop))
        return set_err(MGPU_ERR_ARG, "IPROP must be 5, 6, 84 or 85");
    if (nsys < 1 || njobs < 0 || !systems || !grids || (njobs > 0 && (!job_sys || !job_ered)))
        return set_err(MGPU_ERR_ARG, "bad system/job arrays");
    for (int s = 0; s < nsys; ++s) {
        int rc = check_coupling(&systems[s], &grids[s], iprop);
        if (rc) return rc;
    }
    for (int j = 0; j < njobs; ++j)
        if (job_sys[j] < 0 || job_sys[j] >= nsys || !std::isfinite(job_ered[j]))
            return set_err(MGPU_ERR_ARG, "job references a bad system or ERED");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_err(MGPU_ERR_CUDA, "no CUDA device", e);

    mgpu_plan *p = new (std::nothrow) mgpu_plan();
    if (!p) return set_err(MGPU_ERR_NOMEM, "host allocation failed");
    p->iprop = iprop;
    p->nsys = nsys;
    p->njobs = njobs;

    const AllocFn sync_alloc = [p](void **q, size_t bytes) {
        cudaError_t e = cudaMalloc(q, bytes);
        if (e == cudaSuccess) p->allocs.push_back(*q);
        return e;
    };
    const UploadFn sync_upload = [](void *dst, const void *src, size_t bytes) {
        return cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice);
    };
    std::vector<SysDev> hs(nsys);
    // owners by table identity (pointer and scalar key)
    std::map<std::tuple<const double *, const int *, const double *, const double *, int, int, int>, std::vector<int>>
        owners_by_key;
    for (int s = 0; s < nsys; ++s) {
        const int b = bucket_for(systems[s].n, iprop);
        p->sys_n.push_back(systems[s].n);
        p->sys_bucket.push_back(b);
        p->sys_nstep.push_back(grids[s].nstep);
        p->sys_nham.push_back(systems[s].nham);
        int owner = s;
        {
            // IV is part of the key only where SUMLAM reads it (IVLFL > 0)
            const int *ivkey = systems[s].ivlfl > 0 ? systems[s].iv : nullptr;
            auto &cand = owners_by_key[std::make_tuple(systems[s].vl, ivkey, grids[s].ptab, grids[s].rtab,
                                                       systems[s].n, grids[s].nstep, b)];
            for (int r : cand)
                if (shares_tables(systems[r], grids[r], systems[s], grids[s])) {
                    owner = r;
                    break;
                }
            if (owner == s) cand.push_back(s);
        }
        p->sys_owner.push_back(owner);
        int rc;
        if (owner == s) {
            rc = build_sysdev(systems[s], grids[s], iprop, b, hs[s], sync_alloc, sync_upload);
        } else {
            // the owner's tables; this system's own EINT and CENT
            hs[s] = hs[owner];
            const int npad = bucket_npad(b);
            std::vector<double> eint(npad, 0.0), cent(npad, 0.0);
            std::copy(systems[s].eint, systems[s].eint + systems[s].n, eint.begin());
            std::copy(systems[s].cent, systems[s].cent + systems[s].n, cent.begin());
            double *de = nullptr, *dc = nullptr;
            cudaError_t e2;
            rc = MGPU_OK;
            if ((e2 = put_n(sync_alloc, sync_upload, &de, eint.data(), eint.size())) ||
                (e2 = put_n(sync_alloc, sync_upload, &dc, cent.data(), cent.size())))
                rc = set_err(MGPU_ERR_NOMEM, "uploading a system", e2);
            hs[s].eint = de;
            hs[s].cent = dc;
            ++p->nshared;
        }
        if (rc) {
            delete p;
            return rc;
        }
    }
    if (iprop == MGPU_PROP_LDMD)
        for (int s = 0; s < nsys; ++s) {
            if (p->sys_owner[s] != s) continue;
            const double n = systems[s].n, nh = systems[s].nham;
            p->flops_prep += (n * n * n + nh * n * (n + 1.0)) * grids[s].nstep;
        }
    if ((e = p->dalloc(&p->d_prep, (size_t)3 * nsys))) {
        delete p;
        return set_err(MGPU_ERR_NOMEM, "allocating prep counters", e);
    }
    for (int s = 0; s < nsys; ++s) hs[s].prep = p->d_prep + 3 * p->sys_owner[s];
    {
        void *h = nullptr;
        if ((e = cudaHostAlloc(&h, 2 * sizeof(long long), cudaHostAllocDefault))) {
            delete p;
            return set_err(MGPU_ERR_NOMEM, "allocating the stop controls", e);
        }
        p->ctl = static_cast<long long *>(h);
        p->ctl[0] = 0;
        p->ctl[1] = 0;
        if ((e = cudaStreamCreateWithFlags(&p->ctl_stream, cudaStreamNonBlocking)) ||
            (e = p->dalloc(&p->d_ctl, 2)) ||
            (e = cudaMemcpy(p->d_ctl, p->ctl, 2 * sizeof(long long), cudaMemcpyHostToDevice))) {
            delete p;
            return set_err(MGPU_ERR_NOMEM, "allocating the stop controls", e);
        }
    }
    for (int s = 0; s < nsys; ++s) hs[s].ctl = p->d_ctl;
    if ((e = upload(p, &p->d_sys, hs.data(), hs.size()))) {
        delete p;
        return set_err(MGPU_ERR_NOMEM, "uploading system descriptors", e);
    }

    // jobs: caller-order Y offsets; device order sorted by bucket then system
    p->yoff.resize(njobs);
    size_t off = 0;
    for (int j = 0; j < njobs; ++j) {
        p->yoff[j] = off;
        const double n = systems[job_sys[j]].n;
        off += (size_t)n * (size_t)n;
        const double nh = systems[job_sys[j]].nham;
        const double ns = grids[job_sys[j]].nstep;
        if (is_ldmg(iprop)) {
            // per sector: an inversion for every stage with a_k != 0, a W for every stage
            const wf::MGCoef &m = wf::kMGCoef[iprop == MGPU_PROP_LDMG5 ? 1 : 0];
            int ninv = 0;
            for (int k = 0; k < m.m; ++k) ninv += m.a[k] != 0.0 ? 1 : 0;
            const double f = (ninv * n * n * n + m.m * nh * n * (n + 1.0)) * ns;
            p->flops += f;
            p->flops_prop += f;
        } else {
            p->flops += (3.0 * n * n * n + 2.0 * nh * n * (n + 1.0)) * ns;
            p->flops_prop += ((iprop == MGPU_PROP_LDMD ? 2.0 : 3.0) * n * n * n + 2.0 * nh * n * (n + 1.0)) * ns;
        }
    }
    p->yelems = off;
    std::vector<int> order(njobs);
    for (int j = 0; j < njobs; ++j) order[j] = j;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        const int ba = p->sys_bucket[job_sys[a]], bb = p->sys_bucket[job_sys[b]];
        if (ba != bb) return ba > bb;  // largest matrices first
        return job_sys[a] < job_sys[b];
    });
    std::vector<JobDev> hj(njobs);
    for (int k = 0; k < njobs; ++k) {
        const int j = order[k];
        hj[k].sys = job_sys[j];
        hj[k].out = j;
        hj[k].ered = job_ered[j];
        hj[k].yoff = (long long)p->yoff[j];
    }
    std::vector<int> syslist;
    for (int b = kNumBuckets - 1; b >= 0; --b) {
        int jb = -1, jc = 0;
        for (int k = 0; k < njobs; ++k)
            if (p->sys_bucket[hj[k].sys] == b) {
                if (jb < 0) jb = k;
                ++jc;
            }
        int sb = (int)syslist.size(), sc = 0, mx = 0, nhmax = 0;
        for (int s = 0; s < nsys; ++s)
            if (p->sys_bucket[s] == b && p->sys_owner[s] == s) {  // prepared once per owner
                syslist.push_back(s);
                ++sc;
                mx = std::max(mx, p->sys_nstep[s]);
                nhmax = std::max(nhmax, p->sys_nham[s]);
            }
        if (jc == 0 && sc == 0) continue;
        p->bucket_ids.push_back(b);
        p->job_begin.push_back(jb < 0 ? 0 : jb);
        p->job_count.push_back(jc);
        p->sys_begin.push_back(sb);
        p->sys_count.push_back(sc);
        p->max_nstep.push_back(mx);
        int use_vl = 0;
        const size_t smem = prop_smem(iprop, b, nhmax, &use_vl);
        p->vl_smem.push_back(use_vl);
        p->smem.push_back(smem);
    }
    std::vector<long long> jyoff(njobs);
    std::vector<int> jn(njobs);
    for (int j = 0; j < njobs; ++j) {
        jyoff[j] = (long long)p->yoff[j];
        jn[j] = systems[job_sys[j]].n;
    }
    p->job_n = jn;
    if ((e = upload(p, &p->d_jobs, hj.data(), hj.size())) ||
        (e = upload(p, &p->d_syslists, syslist.data(), syslist.size())) ||
        (njobs > 0 && ((e = upload(p, &p->d_job_yoff, jyoff.data(), jyoff.size())) ||
                       (e = upload(p, &p->d_job_n, jn.data(), jn.size()))))) {
        delete p;
        return set_err(MGPU_ERR_NOMEM, "uploading jobs", e);
    }
    // large-N buckets: per-job tiled matrices and one round's scratch in device memory
    for (size_t slot = 0; slot < p->bucket_ids.size(); ++slot) {
        const int b = p->bucket_ids[slot];
        if (kBuckets[b].kind != KIND_BIG) continue;
        {
            int lo = 0, hi = 0;
            p->bstreams.emplace_back();
            mgpu_plan::BigStreams &q = p->bstreams.back();
            if ((e = cudaDeviceGetStreamPriorityRange(&lo, &hi)) ||
                (e = cudaStreamCreateWithPriority(&q.side, cudaStreamNonBlocking, hi)) ||
                (e = cudaStreamCreateWithFlags(&q.st, cudaStreamNonBlocking)) ||
                (e = cudaEventCreateWithFlags(&q.evf, cudaEventDisableTiming)) ||
                (e = cudaEventCreateWithFlags(&q.evj, cudaEventDisableTiming)) ||
                (e = cudaEventCreateWithFlags(&q.done, cudaEventDisableTiming)) ||
                (!p->ev_in && (e = cudaEventCreateWithFlags(&p->ev_in, cudaEventDisableTiming))) ||
                (e = big_kernel_attributes())) {
                delete p;
                return set_err(MGPU_ERR_CUDA, "large-N set-up", e);
            }
        }
        std::vector<int> prep;
        if (iprop == MGPU_PROP_LDMD)
            for (int i = 0; i < p->sys_count[slot]; ++i) prep.push_back(syslist[p->sys_begin[slot] + i]);
        BigBucket g;
        const int rc = setup_big(g, iprop, b, hj.data() + p->job_begin[slot], p->d_jobs + p->job_begin[slot],
                                 p->job_count[slot], p->max_nstep[slot], prep, hs, p->sys_n, p->sys_nstep, p->d_prep,
                                 sync_alloc, sync_upload);
        if (rc) {
            delete p;
            return rc;
        }
        p->big.push_back(std::move(g));
    }
    // inputs of Y -> S: the couplings' EINT and CENT, the grids' last radius
    p->s_ok = true;
    p->s_eint.resize(nsys);
    p->s_deint.resize(nsys);
    p->s_dcent.resize(nsys);
    p->s_devec.assign(nsys, nullptr);
    p->s_rmatch.resize(nsys);
    for (int s = 0; s < nsys; ++s) {
        p->s_ok = p->s_ok && systems[s].n <= smx::kMaxN;
        p->s_eint[s].assign(systems[s].eint, systems[s].eint + systems[s].n);
        p->s_deint[s] = hs[s].eint;
        p->s_dcent[s] = hs[s].cent;
        p->s_rmatch[s] = is_ldmg(iprop) ? grids[s].rtab[0] + grids[s].nstep * grids[s].dr
                                        : grids[s].rtab[2 * (size_t)grids[s].nstep];
        p->sn_max = std::max(p->sn_max, systems[s].n);
    }
    p->job_sys.assign(job_sys, job_sys + njobs);
    p->job_ered.assign(job_ered, job_ered + njobs);
    int rc0;
    if (p->s_ok && (rc0 = build_s(p))) {
        delete p;
        return rc0;
    }
    *out = p;
    return MGPU_OK;
}

int mgpu_plan_run_device(mgpu_plan *p, double *y_dev, int *nodes_dev, int *status_dev, int *kfail_dev,
                         void *stream)
{
    return mgpu_plan_run_device_phases(p, y_dev, nodes_dev, status_dev, kfail_dev, stream, 3);
}

int mgpu_plan_run_device_phases(mgpu_plan *p, double *y_dev, int *nodes_dev, int *status_dev, int *kfail_dev,
                                void *stream, int phases)
{
    if (!p) return set_err(MGPU_ERR_ARG, "null plan");
    if (p->njobs > 0 && (!y_dev || !nodes_dev || !status_dev || !kfail_dev))
        return set_err(MGPU_ERR_ARG, "null device buffer");
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    if (p->iprop == MGPU_PROP_LDMD && (phases & 1)) {
        // reset NSAVE / status / kfail of every system
        prep_reset_kernel<<<(p->nsys + 127) / 128, 128, 0, st>>>(p->d_prep, p->nsys);
        if ((e = cudaGetLastError())) return set_err(MGPU_ERR_CUDA, "launching prep_reset_kernel", e);
        for (size_t b = 0; b < p->bucket_ids.size(); ++b) {
            if (p->sys_count[b] == 0 || kBuckets[p->bucket_ids[b]].kind == KIND_BIG) continue;
            for (int s0 = 0; s0 < p->sys_count[b]; s0 += 65535) {
                if ((e = launch_prep(p->bucket_ids[b], p->max_nstep[b], std::min(65535, p->sys_count[b] - s0), st,
                                     p->d_sys, p->d_syslists + p->sys_begin[b] + s0)))
                    return set_err(MGPU_ERR_CUDA, "launching ldmd_prep_kernel", e);
            }
        }
    }
    if (!p->big.empty()) {
        // every large-N bucket on its own stream pair, ordered after the caller's stream
        if ((e = cudaEventRecord(p->ev_in, st))) return set_err(MGPU_ERR_CUDA, "ordering the large-N work", e);
        for (size_t i = 0; i < p->big.size(); ++i) {
            BigBucket &g = p->big[i];
            const mgpu_plan::BigStreams &q = p->bstreams[i];
            if ((e = cudaStreamWaitEvent(q.st, p->ev_in, 0))) return set_err(MGPU_ERR_CUDA, "ordering the large-N work", e);
            if (p->iprop == MGPU_PROP_LDMD && (phases & 1) &&
                (e = run_big_prep(g, p->d_sys, p->sys_nstep, q.st, q.aux())))
                return set_err(MGPU_ERR_CUDA, "large-N preparation", e);
            if ((phases & 2) && (e = run_big_prop(g, p->iprop, p->d_sys, y_dev, nodes_dev, status_dev, kfail_dev,
                                                  q.st, q.aux())))
                return set_err(MGPU_ERR_CUDA, "large-N propagation", e);
            if ((e = cudaEventRecord(q.done, q.st))) return set_err(MGPU_ERR_CUDA, "ordering the large-N work", e);
        }
    }
    // the small-N buckets on the caller's stream, beside the large-N streams
    for (size_t b = 0; b < p->bucket_ids.size() && (phases & 2); ++b) {
        if (p->job_count[b] == 0 || kBuckets[p->bucket_ids[b]].kind == KIND_BIG) continue;
        if ((e = launch_prop(p->iprop, p->bucket_ids[b], p->job_count[b], p->smem[b], p->vl_smem[b], st, p->d_sys,
                             p->d_jobs + p->job_begin[b], y_dev, nodes_dev, status_dev, kfail_dev)))
            return set_err(MGPU_ERR_CUDA, "launching the propagation kernel", e);
    }
    // the caller's stream waits for every large-N bucket
    for (size_t i = 0; i < p->big.size(); ++i)
        if ((e = cudaStreamWaitEvent(st, p->bstreams[i].done, 0)))
            return set_err(MGPU_ERR_CUDA, "ordering the large-N work", e);
    return MGPU_OK;
}

int mgpu_plan_run_host(mgpu_plan *p, double *y, int *nodes, int *status, int *kfail)
{
    if (!p) return set_err(MGPU_ERR_ARG, "null plan");
    if (p->njobs == 0) return MGPU_OK;
    if (!y || !nodes || !status || !kfail) return set_err(MGPU_ERR_ARG, "null host buffer");
    cudaError_t e;
    // everything on the plan's own stream, waited for alone (no device-wide
    // synchronisation: other threads may be capturing graphs meanwhile)
    if (!p->own && (e = cudaStreamCreateWithFlags(&p->own, cudaStreamNonBlocking)))
        return set_err(MGPU_ERR_CUDA, "plan stream", e);
    if (p->y_cap < p->yelems) {
        if (p->d_y) cudaFree(p->d_y);
        p->d_y = nullptr;
        if ((e = cudaMalloc(&p->d_y, p->yelems * sizeof(double)))) return set_err(MGPU_ERR_NOMEM, "Y buffer", e);
        p->y_cap = p->yelems;
    }
    if (p->out_cap < p->njobs) {
        if (p->d_nodes) cudaFree(p->d_nodes);
        if (p->d_status) cudaFree(p->d_status);
        if (p->d_kfail) cudaFree(p->d_kfail);
        p->d_nodes = p->d_status = p->d_kfail = nullptr;
        if ((e = cudaMalloc(&p->d_nodes, p->njobs * sizeof(int))) ||
            (e = cudaMalloc(&p->d_status, p->njobs * sizeof(int))) ||
            (e = cudaMalloc(&p->d_kfail, p->njobs * sizeof(int))))
            return set_err(MGPU_ERR_NOMEM, "output buffers", e);
        p->out_cap = p->njobs;
    }
    if ((e = cudaMemcpyAsync(p->d_y, y, p->yelems * sizeof(double), cudaMemcpyHostToDevice, p->own)))
        return set_err(MGPU_ERR_CUDA, "copying Y to the device", e);
    int rc = mgpu_plan_run_device(p, p->d_y, p->d_nodes, p->d_status, p->d_kfail, p->own);
    if (rc) return rc;
    if ((e = cudaMemcpyAsync(y, p->d_y, p->yelems * sizeof(double), cudaMemcpyDeviceToHost, p->own)) ||
        (e = cudaMemcpyAsync(nodes, p->d_nodes, p->njobs * sizeof(int), cudaMemcpyDeviceToHost, p->own)) ||
        (e = cudaMemcpyAsync(status, p->d_status, p->njobs * sizeof(int), cudaMemcpyDeviceToHost, p->own)) ||
        (e = cudaMemcpyAsync(kfail, p->d_kfail, p->njobs * sizeof(int), cudaMemcpyDeviceToHost, p->own)))
        return set_err(MGPU_ERR_CUDA, "copying results to the host", e);
    if ((e = cudaStreamSynchronize(p->own))) return set_err(MGPU_ERR_CUDA, "propagation", e);
    return MGPU_OK;
}

int mgpu_plan_match_counts_device(mgpu_plan *p, const double *y_dev, int npairs, const int *pairs_dev,
                                  int *counts_dev, void *stream)
{
    if (!p) return set_err(MGPU_ERR_ARG, "null plan");
    if (npairs < 0) return set_err(MGPU_ERR_ARG, "negative pair count");
    if (npairs == 0) return MGPU_OK;
    if (!y_dev || !pairs_dev || !counts_dev) return set_err(MGPU_ERR_ARG, "null device buffer");
    int nmax = 0;
    for (int n : p->sys_n) nmax = std::max(nmax, n);
    if (nmax > match::kMatchMaxN) return set_err(MGPU_ERR_UNSUPPORTED, "device matching counts need N <= 240");
    const size_t smem = match::packed(nmax, 0) * sizeof(double);
    cudaError_t e;
    if ((e = set_smem(match::match_count_kernel, smem))) return set_err(MGPU_ERR_CUDA, "matching kernel set-up", e);
    for (int b0 = 0; b0 < npairs; b0 += 65535) {
        const int nb = std::min(65535, npairs - b0);
        match::match_count_kernel<<<nb, match::kThreads, smem, (cudaStream_t)stream>>>(
            y_dev, p->d_job_yoff, p->d_job_n, pairs_dev + 2 * (size_t)b0, counts_dev + b0);
        if ((e = cudaGetLastError())) return set_err(MGPU_ERR_CUDA, "launching the matching kernel", e);
    }
    return MGPU_OK;
}

int mgpu_plan_match_counts(mgpu_plan *p, int npairs, const int *pairs, int *counts)
{
    if (!p) return set_err(MGPU_ERR_ARG, "null plan");
    if (npairs < 0 || (npairs > 0 && (!pairs || !counts))) return set_err(MGPU_ERR_ARG, "bad pair arrays");
    if (npairs == 0) return MGPU_OK;
    for (int k = 0; k < 2 * npairs; ++k)
        if (pairs[k] < 0 || pairs[k] >= p->njobs) return set_err(MGPU_ERR_ARG, "pair references a bad job");
    for (int k = 0; k < npairs; ++k)
        if (p->job_n[pairs[2 * k]] != p->job_n[pairs[2 * k + 1]])
            return set_err(MGPU_ERR_ARG, "paired jobs differ in N");
    if (!p->d_y || p->y_cap < p->yelems) return set_err(MGPU_ERR_ARG, "no Y on the device: run the plan first");
    cudaError_t e;
    if (p->m_cap < npairs) {
        if (p->d_mpairs) cudaFree(p->d_mpairs);
        if (p->d_mcounts) cudaFree(p->d_mcounts);
        p->d_mpairs = p->d_mcounts = nullptr;
        if ((e = cudaMalloc(&p->d_mpairs, 2 * (size_t)npairs * sizeof(int))) ||
            (e = cudaMalloc(&p->d_mcounts, (size_t)npairs * sizeof(int))))
            return set_err(MGPU_ERR_NOMEM, "matching buffers", e);
        p->m_cap = npairs;
    }
    if (!p->own && (e = cudaStreamCreateWithFlags(&p->own, cudaStreamNonBlocking)))
        return set_err(MGPU_ERR_CUDA, "plan stream", e);
    if ((e = cudaMemcpyAsync(p->d_mpairs, pairs, 2 * (size_t)npairs * sizeof(int), cudaMemcpyHostToDevice, p->own)))
        return set_err(MGPU_ERR_CUDA, "copying pairs", e);
    const int rc = mgpu_plan_match_counts_device(p, p->d_y, npairs, p->d_mpairs, p->d_mcounts, p->own);
    if (rc) return rc;
    if ((e = cudaMemcpyAsync(counts, p->d_mcounts, (size_t)npairs * sizeof(int), cudaMemcpyDeviceToHost, p->own)) ||
        (e = cudaStreamSynchronize(p->own)))
        return set_err(MGPU_ERR_CUDA, "matching counts", e);
    return MGPU_OK;
}

size_t mgpu_plan_s_elems(const mgpu_plan *p) { return p ? p->selems : 0; }

size_t mgpu_plan_s_offset(const mgpu_plan *p, int job)
{
    return (p && job >= 0 && job < p->njobs) ? p->soff[job] : 0;
}

int mgpu_plan_nopen(const mgpu_plan *p, int job) { return (p && job >= 0 && job < p->njobs) ? p->nopen[job] : -1; }

int mgpu_plan_smatrix_device(mgpu_plan *p, const double *y_dev, double *sr_dev, double *si_dev, int *status_dev,
                             void *stream)
{
    if (!p) return set_err(MGPU_ERR_ARG, "null plan");
    if (!p->s_ok) return set_err(MGPU_ERR_UNSUPPORTED, "device S matrices need N <= 1024 in every system");
    if (p->njobs == 0 || p->selems == 0) return MGPU_OK;
    if (!y_dev || !sr_dev || !si_dev || !status_dev) return set_err(MGPU_ERR_ARG, "null device buffer");
    cudaError_t e;
    cudaStream_t st = (cudaStream_t)stream;
    if (p->n_evec > 0) {
        // YTRANS: Y in the asymptotic basis first, into the plan's own buffer
        if (!p->d_yt && ((e = cudaMalloc(&p->d_yt, std::max<size_t>(p->yelems, 1) * sizeof(double))) ||
                         (e = cudaMalloc(&p->d_yz, std::max<size_t>(p->yelems, 1) * sizeof(double)))))
            return set_err(MGPU_ERR_NOMEM, "asymptotic-basis transform buffers", e);
        const int tx = (p->sn_max + smx::kTT - 1) / smx::kTT;
        for (int pass = 1; pass <= 2; ++pass)
            for (int list = 0; list < 2; ++list) {
                const int cnt = list ? p->ns_large : p->ns_small;
                const smx::SJob *jl = list ? p->d_sjobs_g : p->d_sjobs;
                for (int j0 = 0; j0 < cnt; j0 += 65535) {
                    smx::ytrans_kernel<<<dim3(tx * tx, std::min(65535, cnt - j0)), 256, 0, st>>>(
                        p->d_sys, jl + j0, pass, y_dev, p->d_yz, p->d_yt);
                    if ((e = cudaGetLastError())) return set_err(MGPU_ERR_CUDA, "launching the YTRANS kernel", e);
                }
            }
        y_dev = p->d_yt;
    }
    for (int j0 = 0; j0 < p->ns_small; j0 += 65535) {
        if ((e = set_smem(smx::smatrix_kernel, p->s_smem))) return set_err(MGPU_ERR_CUDA, "S-matrix kernel set-up", e);
        smx::smatrix_kernel<<<std::min(65535, p->ns_small - j0), smx::kThreads, p->s_smem, st>>>(
            p->d_sys, p->d_sjobs + j0, p->d_nb, p->d_nb_off, y_dev, sr_dev, si_dev, status_dev);
        if ((e = cudaGetLastError())) return set_err(MGPU_ERR_CUDA, "launching the S-matrix kernel", e);
    }
    if (p->ns_large > 0) {
        if (!p->d_sscr && p->sscr_elems > 0 && (e = cudaMalloc(&p->d_sscr, p->sscr_elems * sizeof(double))))
            return set_err(MGPU_ERR_NOMEM, "S-matrix scratch", e);
        if ((e = set_smem(smx::smatrix_kernel_g, p->s_smem_g)))
            return set_err(MGPU_ERR_CUDA, "S-matrix kernel set-up", e);
        for (int j0 = 0; j0 < p->ns_large; j0 += 65535) {
            smx::smatrix_kernel_g<<<std::min(65535, p->ns_large - j0), smx::kThreads, p->s_smem_g, st>>>(
                p->d_sys, p->d_sjobs_g + j0, p->d_nb, p->d_nb_off, y_dev, sr_dev, si_dev, status_dev, p->d_sscr);
            if ((e = cudaGetLastError())) return set_err(MGPU_ERR_CUDA, "launching the S-matrix kernel", e);
        }
    }
    return MGPU_OK;
}

int mgpu_plan_set_asymptote(mgpu_plan *p, int sys, const double *eint, const double *cent, const double *evec,
                            double rmatch)
{
    if (!p) return set_err(MGPU_ERR_ARG, "null plan");
    if (sys < 0 || sys >= p->nsys) return set_err(MGPU_ERR_ARG, "system index out of range");
    if (!p->s_ok) return set_err(MGPU_ERR_UNSUPPORTED, "device S matrices need N <= 1024 in every system");
    if (!eint || !cent) return set_err(MGPU_ERR_ARG, "EINT/CENT null");
    const int n = p->sys_n[sys];
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(eint[i]) || !(cent[i] > -1.0e-10)) return set_err(MGPU_ERR_ARG, "bad EINT or CENT");
    if (!(rmatch > 0.0) || !std::isfinite(rmatch)) return set_err(MGPU_ERR_ARG, "RMATCH must be positive");
    cudaError_t e;
    double *de = nullptr, *dc = nullptr, *dv = nullptr;
    if ((e = upload(p, &de, eint, n)) || (e = upload(p, &dc, cent, n)) ||
        (evec && (e = upload(p, &dv, evec, (size_t)n * n))))
        return set_err(MGPU_ERR_NOMEM, "uploading an asymptotic basis", e);
    // the previous setting's arrays, unless they are the coupling's own
    if (p->s_devec[sys]) {
        p->dfree(const_cast<double *>(p->s_deint[sys]));
        p->dfree(const_cast<double *>(p->s_dcent[sys]));
        p->dfree(const_cast<double *>(p->s_devec[sys]));
        --p->n_evec;
    }
    p->s_eint[sys].assign(eint, eint + n);
    p->s_deint[sys] = de;
    p->s_dcent[sys] = dc;
    p->s_devec[sys] = dv;
    p->s_rmatch[sys] = rmatch;
    if (dv) ++p->n_evec;
    return build_s(p);
}

int mgpu_plan_smatrix_host(mgpu_plan *p, const double *y, double *sr, double *si, int *status)
{
    if (!p) return set_err(MGPU_ERR_ARG, "null plan");
    if (!p->s_ok) return set_err(MGPU_ERR_UNSUPPORTED, "device S matrices need N <= 1024 in every system");
    if (p->njobs == 0) return MGPU_OK;
    if (!y || !status || (p->selems && (!sr || !si))) return set_err(MGPU_ERR_ARG, "null host buffer");
    cudaError_t e;
    if (!p->own && (e = cudaStreamCreateWithFlags(&p->own, cudaStreamNonBlocking)))
        return set_err(MGPU_ERR_CUDA, "plan stream", e);
    if (p->y_cap < p->yelems) {
        if (p->d_y) cudaFree(p->d_y);
        p->d_y = nullptr;
        if ((e = cudaMalloc(&p->d_y, p->yelems * sizeof(double)))) return set_err(MGPU_ERR_NOMEM, "Y buffer", e);
        p->y_cap = p->yelems;
    }
    if (!p->d_status && (e = cudaMalloc(&p->d_status, (size_t)p->njobs * sizeof(int))))
        return set_err(MGPU_ERR_NOMEM, "status buffer", e);
    if (p->selems && p->s_cap < p->selems) {
        if (p->d_sr) cudaFree(p->d_sr);
        if (p->d_si) cudaFree(p->d_si);
        p->d_sr = p->d_si = nullptr;
        if ((e = cudaMalloc(&p->d_sr, p->selems * sizeof(double))) ||
            (e = cudaMalloc(&p->d_si, p->selems * sizeof(double))))
            return set_err(MGPU_ERR_NOMEM, "S buffers", e);
        p->s_cap = p->selems;
    }
    if ((e = cudaMemcpyAsync(p->d_y, y, p->yelems * sizeof(double), cudaMemcpyHostToDevice, p->own)) ||
        (e = cudaMemcpyAsync(p->d_status, status, (size_t)p->njobs * sizeof(int), cudaMemcpyHostToDevice, p->own)))
        return set_err(MGPU_ERR_CUDA, "copying Y in", e);
    int rc = mgpu_plan_smatrix_device(p, p->d_y, p->d_sr, p->d_si, p->d_status, p->own);
    if (rc) return rc;
    if ((p->selems && ((e = cudaMemcpyAsync(sr, p->d_sr, p->selems * sizeof(double), cudaMemcpyDeviceToHost, p->own)) ||
                       (e = cudaMemcpyAsync(si, p->d_si, p->selems * sizeof(double), cudaMemcpyDeviceToHost, p->own)))) ||
        (e = cudaMemcpyAsync(status, p->d_status, (size_t)p->njobs * sizeof(int), cudaMemcpyDeviceToHost, p->own)) ||
        (e = cudaStreamSynchronize(p->own)))
        return set_err(MGPU_ERR_CUDA, "copying S out", e);
    return MGPU_OK;
}

int mgpu_plan_run_host_smatrix(mgpu_plan *p, const double *y, double *sr, double *si, int *nodes, int *status,
                               int *kfail)
{
    if (!p) return set_err(MGPU_ERR_ARG, "null plan");
    if (!p->s_ok) return set_err(MGPU_ERR_UNSUPPORTED, "device S matrices need N <= 1024 in every system");
    if (p->njobs == 0) return MGPU_OK;
    if (!y || !nodes || !status || !kfail || (p->selems && (!sr || !si))) return set_err(MGPU_ERR_ARG, "null host buffer");
    cudaError_t e;
    if (!p->own && (e = cudaStreamCreateWithFlags(&p->own, cudaStreamNonBlocking)))
        return set_err(MGPU_ERR_CUDA, "plan stream", e);
    if (p->y_cap < p->yelems) {
        if (p->d_y) cudaFree(p->d_y);
        p->d_y = nullptr;
        if ((e = cudaMalloc(&p->d_y, p->yelems * sizeof(double)))) return set_err(MGPU_ERR_NOMEM, "Y buffer", e);
        p->y_cap = p->yelems;
    }
    if (p->out_cap < p->njobs) {
        if (p->d_nodes) cudaFree(p->d_nodes);
        if (p->d_status) cudaFree(p->d_status);
        if (p->d_kfail) cudaFree(p->d_kfail);
        p->d_nodes = p->d_status = p->d_kfail = nullptr;
        if ((e = cudaMalloc(&p->d_nodes, p->njobs * sizeof(int))) ||
            (e = cudaMalloc(&p->d_status, p->njobs * sizeof(int))) ||
            (e = cudaMalloc(&p->d_kfail, p->njobs * sizeof(int))))
            return set_err(MGPU_ERR_NOMEM, "output buffers", e);
        p->out_cap = p->njobs;
    }
    if (p->s_cap < p->selems) {
        if (p->d_sr) cudaFree(p->d_sr);
        if (p->d_si) cudaFree(p->d_si);
        p->d_sr = p->d_si = nullptr;
        if ((e = cudaMalloc(&p->d_sr, p->selems * sizeof(double))) || (e = cudaMalloc(&p->d_si, p->selems * sizeof(double))))
            return set_err(MGPU_ERR_NOMEM, "S buffers", e);
        p->s_cap = p->selems;
    }
    if ((e = cudaMemcpyAsync(p->d_y, y, p->yelems * sizeof(double), cudaMemcpyHostToDevice, p->own)))
        return set_err(MGPU_ERR_CUDA, "copying Y to the device", e);
    int rc = mgpu_plan_run_device(p, p->d_y, p->d_nodes, p->d_status, p->d_kfail, p->own);
    if (!rc) rc = mgpu_plan_smatrix_device(p, p->d_y, p->d_sr, p->d_si, p->d_status, p->own);
    if (rc) return rc;
    if ((p->selems && ((e = cudaMemcpyAsync(sr, p->d_sr, p->selems * sizeof(double), cudaMemcpyDeviceToHost, p->own)) ||
                       (e = cudaMemcpyAsync(si, p->d_si, p->selems * sizeof(double), cudaMemcpyDeviceToHost, p->own)))) ||
        (e = cudaMemcpyAsync(nodes, p->d_nodes, p->njobs * sizeof(int), cudaMemcpyDeviceToHost, p->own)) ||
        (e = cudaMemcpyAsync(status, p->d_status, p->njobs * sizeof(int), cudaMemcpyDeviceToHost, p->own)) ||
        (e = cudaMemcpyAsync(kfail, p->d_kfail, p->njobs * sizeof(int), cudaMemcpyDeviceToHost, p->own)))
        return set_err(MGPU_ERR_CUDA, "copying results to the host", e);
    if ((e = cudaStreamSynchronize(p->own))) return set_err(MGPU_ERR_CUDA, "propagation", e);
    return MGPU_OK;
}

static int single(int iprop, const mgpu_coupling *c, const mgpu_grid *g, double ered, double *y, int *nodes,
                  int *kfail)
{
    if (!y || !nodes || !kfail) return set_err(MGPU_ERR_ARG, "null output pointer");
    mgpu_plan *p = nullptr;
    int sys = 0;
    int rc = mgpu_plan_create(&p, iprop, 1, c, g, 1, &sys, &ered);
    if (rc) return rc;
    int status = 0;
    rc = mgpu_plan_run_host(p, y, nodes, &status, kfail);
    mgpu_plan_destroy(p);
    if (rc) return rc;
    return status;
}

int mgpu_mdprop(const mgpu_coupling *c, const mgpu_grid *g, double ered, double *y, int *nodes, int *kfail)
{
    return single(MGPU_PROP_LDMD, c, g, ered, y, nodes, kfail);
}

int mgpu_ldprop(const mgpu_coupling *c, const mgpu_grid *g, double ered, double *z, int *nodes, int *kfail)
{
    return single(MGPU_PROP_LDJ, c, g, ered, z, nodes, kfail);
}

int mgpu_mgprop(int imgsel, const mgpu_coupling *c, const mgpu_grid *g, double ered, double *y, int *nodes,
                int *kfail)
{
    if (imgsel != 4 && imgsel != 5) return set_err(MGPU_ERR_ARG, "IMGSEL must be 4 (CS4) or 5 (MA5)");
    return single(imgsel == 4 ? MGPU_PROP_LDMG4 : MGPU_PROP_LDMG5, c, g, ered, y, nodes, kfail);
}

// Fortran calling convention: every argument by reference, no structures.
static void single_f(int iprop, const int *n, const int *nham, const int *nvlblk, const int *ivlfl,
                     const int *nconst, const int *nrsq, const double *conlen, double *y, const double *vl,
                     const int *iv, const double *eint, const double *cent, const int *nstep, const double *dr,
                     const double *rtab, const double *ptab, const double *ered, int *nodes, int *kfail,
                     int *istat)
{
    if (!istat) return;
    if (!n || !nham || !nvlblk || !ivlfl || !nconst || !nrsq || !conlen || !nstep || !dr || !ered || !nodes ||
        !kfail) {
        *istat = set_err(MGPU_ERR_ARG, "null argument");
        return;
    }
    mgpu_coupling c;
    c.n = *n;
    c.nham = *nham;
    c.nvlblk = *nvlblk;
    c.ivlfl = *ivlfl;
    c.nconst = *nconst;
    c.nrsq = *nrsq;
    c.conlen = *conlen;
    c.vl = vl;
    c.iv = iv;
    c.eint = eint;
    c.cent = cent;
    mgpu_grid g;
    g.nstep = *nstep;
    g.dr = *dr;
    g.rtab = rtab;
    g.ptab = ptab;
    *nodes = 0;
    *kfail = 0;
    *istat = single(iprop, &c, &g, *ered, y, nodes, kfail);
}

void mgpu_mdprop_f(const int *n, const int *nham, const int *nvlblk, const int *ivlfl, const int *nconst,
                   const int *nrsq, const double *conlen, double *y, const double *vl, const int *iv,
                   const double *eint, const double *cent, const int *nstep, const double *dr, const double *rtab,
                   const double *ptab, const double *ered, int *nodes, int *kfail, int *istat)
{
    single_f(MGPU_PROP_LDMD, n, nham, nvlblk, ivlfl, nconst, nrsq, conlen, y, vl, iv, eint, cent, nstep, dr, rtab,
             ptab, ered, nodes, kfail, istat);
}

void mgpu_ldprop_f(const int *n, const int *nham, const int *nvlblk, const int *ivlfl, const int *nconst,
                   const int *nrsq, const double *conlen, double *z, const double *vl, const int *iv,
                   const double *eint, const double *cent, const int *nstep, const double *dr, const double *rtab,
                   const double *ptab, const double *ered, int *nodes, int *kfail, int *istat)
{
    single_f(MGPU_PROP_LDJ, n, nham, nvlblk, ivlfl, nconst, nrsq, conlen, z, vl, iv, eint, cent, nstep, dr, rtab,
             ptab, ered, nodes, kfail, istat);
}

void mgpu_mgprop_f(const int *imgsel, const int *n, const int *nham, const int *nvlblk, const int *ivlfl,
                   const int *nconst, const int *nrsq, const double *conlen, double *y, const double *vl,
                   const int *iv, const double *eint, const double *cent, const int *nstep, const double *dr,
                   const double *rtab, const double *ptab, const double *ered, int *nodes, int *kfail, int *istat)
{
    if (!istat) return;
    if (!imgsel || (*imgsel != 4 && *imgsel != 5)) {
        *istat = set_err(MGPU_ERR_ARG, "IMGSEL must be 4 (CS4) or 5 (MA5)");
        return;
    }
    single_f(*imgsel == 4 ? MGPU_PROP_LDMG4 : MGPU_PROP_LDMG5, n, nham, nvlblk, ivlfl, nconst, nrsq, conlen, y, vl,
             iv, eint, cent, nstep, dr, rtab, ptab, ered, nodes, kfail, istat);
}

}  // extern "C"

// ===========================================================================
// Allocation-free LDMD entry point (mgpu_mdprop_noalloc).
//
// Some callers cannot allocate device memory: a host program whose device
// memory all comes from its own pool or framework allocator, or one that
// must not call cudaMalloc/cudaFree inside a time-critical loop because
// those calls can synchronise the whole device.  For them this entry point
// uses no memory beyond the caller's own input/output buffers and one
// file-scope scratch array of fixed size, reserved on every GPU that loads
// this library until the process exits.  The kernels are the same ones the
// plan API launches.
// ===========================================================================
namespace mgpu {

constexpr size_t kNoAllocScratchBytes = (size_t)64 << 20;  // 64 MiB per device
constexpr int kNoAllocMaxJobs = 4096;
constexpr int kNoAllocMaxDevices = 64;

// Holds, for one call at a time: the system descriptor, the job list, the
// NSAVE/status counters, padded EINT/CENT, VL (and IV) in tile layout, and
// the 2HQ(C) table of every step.
static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchBytes / sizeof(double)];

static double *g_noalloc_addr[kNoAllocMaxDevices];  // device address of the array, per device
static std::mutex g_noalloc_mu;

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Builds everything the LDMD kernels read from the scratch: descriptor, jobs
// (ERED from the caller's device array), zeroed counters, padded EINT/CENT,
// and VL/IV converted to the tile layout.  Every element the kernels read is
// written, so nothing from an earlier call survives into this one.
__global__ void noalloc_setup_kernel(SysDev proto, SysDev *sys_out, JobDev *jobs, int njobs, const double *ered,
                                     int *syslist, const double *vl, const int *iv, int nvlblk, const double *eint,
                                     const double *cent, double *eint_p, double *cent_p, double *vlt, int *ivt,
                                     int npad, int edge)
{
    const int TT = edge * edge;
    const int nt = proto.ntiles;
    const size_t nvlt = (size_t)proto.nham * TT * nt;
    const size_t total = nvlt > (size_t)njobs ? nvlt : (size_t)njobs;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t x = (size_t)blockIdx.x * blockDim.x + threadIdx.x; x < total || x < (size_t)npad; x += stride) {
        if (x == 0) {
            *sys_out = proto;
            syslist[0] = 0;
            proto.prep[0] = 0;
            proto.prep[1] = 0;
            proto.prep[2] = 0x7fffffff;
        }
        if (x < (size_t)njobs) {
            JobDev j;
            j.sys = 0;
            j.out = (int)x;
            j.ered = ered[x];
            j.yoff = (long long)x * proto.n * proto.n;
            jobs[x] = j;
        }
        if (x < (size_t)npad) {
            eint_p[x] = x < (size_t)proto.n ? eint[x] : 0.0;
            cent_p[x] = x < (size_t)proto.n ? cent[x] : 0.0;
        }
        if (x < nvlt) {
            // x enumerates the destination array in its own layout
            int l, t, e;
            if (proto.kind == 1) {  // [term][tile][lane][s]
                e = (int)(x % TT);
                t = (int)((x / TT) % nt);
                l = (int)(x / ((size_t)TT * nt));
            } else {  // [term][element][tile]
                t = (int)(x % nt);
                e = (int)((x / nt) % TT);
                l = (int)(x / ((size_t)nt * TT));
            }
            int I = 0;
            while ((I + 1) * (I + 2) / 2 <= t) ++I;
            const int J = t - I * (I + 1) / 2;
            int i, j;
            if (proto.kind == 1) {
                const int lane = e >> 1, s2 = e & 1;
                i = 8 * I + (lane >> 2);
                j = 8 * J + 2 * (lane & 3) + s2;
            } else {
                i = I * edge + e / edge;
                j = J * edge + e % edge;
            }
            double v = 0.0;
            int ix = 0;
            if (i < proto.n && j < proto.n) {
                const int lo = i < j ? i : j, hi = i < j ? j : i;
                const size_t src = ((size_t)hi * (hi + 1) / 2 + lo) * nvlblk + l;
                v = vl[src];
                if (proto.ivlfl > 0) {
                    ix = iv[src] - 1;
                    if (ix < 0 || ix >= proto.nham) {  // bad index: make the prep pass report it
                        ix = 0;
                        v = __longlong_as_double(0x7ff8000000000000LL);
                    }
                }
            }
            vlt[x] = v;
            if (proto.ivlfl > 0) ivt[x] = ix;
        }
    }
}

}  // namespace mgpu

extern "C" int mgpu_mdprop_noalloc(const mgpu_coupling *c, const mgpu_grid *g, int njobs, const double *ered_dev,
                                   double *y_dev, int *nodes_dev, int *status_dev, int *kfail_dev, void *stream)
{
    using namespace mgpu;
    if (!c || !g) return set_err(MGPU_ERR_ARG, "null system or grid");
    if (c->n < 1 || c->nham < 0 || c->nvlblk < c->nham || g->nstep < 1 || !(g->dr != 0.0) || !std::isfinite(g->dr))
        return set_err(MGPU_ERR_ARG, "bad N/NHAM/NVLBLK/NSTEP/DR");
    if (njobs < 1 || njobs > kNoAllocMaxJobs) return set_err(MGPU_ERR_UNSUPPORTED, "njobs must be 1..4096");
    if ((c->nham > 0 && (!c->vl || !g->ptab)) || (c->ivlfl > 0 && !c->iv) || !c->eint || !c->cent || !g->rtab ||
        !ered_dev || !y_dev || !nodes_dev || !status_dev || !kfail_dev)
        return set_err(MGPU_ERR_ARG, "null device pointer");
    const int b = bucket_for(c->n, MGPU_PROP_LDMD, false);  // the default order, whatever the tuning
    // the one-warp and one-CTA kernels only (N <= 200): the large-N kernels need per-job device matrices
    if (b < 0 || kBuckets[b].kind == KIND_BIG)
        return set_err(MGPU_ERR_UNSUPPORTED, "N above 200 (largest size of the allocation-free entry point)");
    const int nt = ntiles_of(b);
    const int npad = bucket_npad(b);
    const size_t tile = matrix_elems(b);  // doubles per tiled matrix

    // scratch layout
    size_t off = 0;
    const size_t o_sys = off;
    off = align256(off + sizeof(SysDev));
    const size_t o_jobs = off;
    off = align256(off + sizeof(JobDev) * (size_t)njobs);
    const size_t o_prep = off;
    off = align256(off + 4 * sizeof(int));
    const size_t o_eint = off;
    off = align256(off + sizeof(double) * npad);
    const size_t o_cent = off;
    off = align256(off + sizeof(double) * npad);
    const size_t o_vlt = off;
    off = align256(off + sizeof(double) * tile * (size_t)std::max(c->nham, 1));
    const size_t o_ivt = off;
    if (c->ivlfl > 0) off = align256(off + sizeof(int) * tile * (size_t)c->nham);
    const size_t o_q = off;
    off = align256(off + sizeof(double) * tile * (size_t)g->nstep);
    if (off > kNoAllocScratchBytes) {
        char buf[160];
        snprintf(buf, sizeof buf, "mgpu_mdprop_noalloc needs %zu bytes of scratch; the fixed limit is %zu (64 MiB)",
                 off, kNoAllocScratchBytes);
        return set_err(MGPU_ERR_UNSUPPORTED, buf);
    }

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_err(MGPU_ERR_CUDA, "no CUDA device", e);
    if (dev < 0 || dev >= kNoAllocMaxDevices) return set_err(MGPU_ERR_UNSUPPORTED, "device ordinal above 63");
    char *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {
            // once per device, with that device current: the array's device address
            double *ptr = nullptr;
            e = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
            if (e != cudaSuccess) return set_err(MGPU_ERR_CUDA, "cudaGetSymbolAddress(scratch)", e);
            g_noalloc_addr[dev] = ptr;
        }
        base = reinterpret_cast<char *>(g_noalloc_addr[dev]);
    }

    SysDev proto;
    memset(&proto, 0, sizeof proto);
    proto.n = c->n;
    proto.nham = c->nham;
    proto.ivlfl = c->ivlfl;
    proto.nconst = c->nconst;
    proto.nrsq = c->nrsq;
    proto.nstep = g->nstep;
    proto.ntiles = nt;
    proto.kind = frag_layout(b) ? 1 : 0;
    proto.conlen = c->conlen;
    proto.dr = g->dr;
    proto.vlt = reinterpret_cast<double *>(base + o_vlt);
    proto.ivt = reinterpret_cast<int *>(base + o_ivt);
    proto.eint = reinterpret_cast<double *>(base + o_eint);
    proto.cent = reinterpret_cast<double *>(base + o_cent);
    proto.rtab = g->rtab;
    proto.ptab = g->ptab;
    proto.q = reinterpret_cast<double *>(base + o_q);
    proto.prep = reinterpret_cast<int *>(base + o_prep);
    SysDev *d_sys = reinterpret_cast<SysDev *>(base + o_sys);
    JobDev *d_jobs = reinterpret_cast<JobDev *>(base + o_jobs);
    int *d_list = proto.prep + 3;

    cudaStream_t st = (cudaStream_t)stream;
    const size_t work = std::max(std::max(tile * (size_t)std::max(c->nham, 1), (size_t)njobs), (size_t)npad);
    const int blocks = (int)std::min<size_t>((work + 255) / 256, 4096);
    noalloc_setup_kernel<<<blocks, 256, 0, st>>>(proto, d_sys, d_jobs, njobs, ered_dev, d_list, c->vl, c->iv,
                                                 c->nvlblk, c->eint, c->cent, const_cast<double *>(proto.eint),
                                                 const_cast<double *>(proto.cent), const_cast<double *>(proto.vlt),
                                                 const_cast<int *>(proto.ivt), npad, bucket_edge(b));
    if ((e = cudaGetLastError())) return set_err(MGPU_ERR_CUDA, "launching noalloc_setup_kernel", e);
    if ((e = launch_prep(b, g->nstep, 1, st, d_sys, d_list)))
        return set_err(MGPU_ERR_CUDA, "launching ldmd_prep_kernel", e);
    int use_vl = 0;
    const size_t smem = prop_smem(MGPU_PROP_LDMD, b, c->nham, &use_vl);
    if ((e = launch_prop(MGPU_PROP_LDMD, b, njobs, smem, use_vl, st, d_sys, d_jobs, y_dev, nodes_dev, status_dev,
                         kfail_dev)))
        return set_err(MGPU_ERR_CUDA, "launching ldmd_prop_kernel", e);
    return MGPU_OK;
}
#include "kernels_ldma.cuh"

// ---- MAPROP for the energies of one system (tables from the host) --------
struct mgpu_ldma {
    mgpu::ldma::Tables t{};
    std::vector<void *> allocs;
    cudaStream_t own = nullptr;
    ~mgpu_ldma()
    {
        if (own) cudaStreamSynchronize(own);
        for (void *p : allocs) cudaFree(p);
        if (own) cudaStreamDestroy(own);
    }
};

extern "C" int mgpu_ldma_create(mgpu_ldma **out, int n, int nstep, double dr, int inward, const double *eival,
                                const double *q, const double *corr, const double *tfin, const double *qfin)
{
    if (!out) return set_err(MGPU_ERR_ARG, "null handle pointer");
    *out = nullptr;
    if (n < 1 || n > mgpu::ldma::kMaxN) return set_err(MGPU_ERR_UNSUPPORTED, "LDMA runs for 1 <= N <= 100");
    if (nstep < 1 || !(dr != 0.0) || !std::isfinite(dr)) return set_err(MGPU_ERR_ARG, "bad NSTEP or DR");
    if (!eival || !q || !corr || !tfin || !qfin) return set_err(MGPU_ERR_ARG, "null table");
    mgpu_ldma *h = new (std::nothrow) mgpu_ldma();
    if (!h) return set_err(MGPU_ERR_NOMEM, "host allocation failed");
    const size_t nn = (size_t)n * n;
    const AllocFn al = [h](void **p, size_t nb) {
        cudaError_t e = cudaMalloc(p, nb);
        if (e == cudaSuccess) h->allocs.push_back(*p);
        return e;
    };
    const UploadFn up = [](void *dst, const void *src, size_t nb) {
        return cudaMemcpy(dst, src, nb, cudaMemcpyHostToDevice);
    };
    double *de = nullptr, *dq = nullptr, *dc = nullptr, *dt = nullptr, *dqf = nullptr;
    cudaError_t e;
    if ((e = put_n(al, up, &de, eival, (size_t)nstep * n)) || (e = put_n(al, up, &dq, q, (size_t)nstep * nn)) ||
        (e = put_n(al, up, &dc, corr, (size_t)nstep * nn)) || (e = put_n(al, up, &dt, tfin, nn)) ||
        (e = put_n(al, up, &dqf, qfin, nn)) || (e = cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking))) {
        delete h;
        return set_err(MGPU_ERR_NOMEM, "uploading the LDMA tables", e);
    }
    h->t = mgpu::ldma::Tables{n, nstep, inward ? 1 : 0, dr, de, dq, dc, dt, dqf};
    *out = h;
    return MGPU_OK;
}

extern "C" int mgpu_ldma_run_host(mgpu_ldma *h, int njobs, const double *ered, double *y, int *nodes, int *status)
{
    if (!h) return set_err(MGPU_ERR_ARG, "null handle");
    if (njobs < 0 || njobs > 65535) return set_err(MGPU_ERR_ARG, "0 <= jobs <= 65535");
    if (njobs == 0) return MGPU_OK;
    if (!ered || !y || !nodes || !status) return set_err(MGPU_ERR_ARG, "null host buffer");
    for (int j = 0; j < njobs; ++j)
        if (!std::isfinite(ered[j])) return set_err(MGPU_ERR_ARG, "ERED not finite");
    const size_t nn = (size_t)h->t.n * h->t.n;
    double *de = nullptr, *dy = nullptr;
    int *dn = nullptr, *ds = nullptr;
    cudaError_t e;
    cudaStream_t st = h->own;
    if ((e = cudaMallocAsync((void **)&de, njobs * sizeof(double), st)) ||
        (e = cudaMallocAsync((void **)&dy, njobs * nn * sizeof(double), st)) ||
        (e = cudaMallocAsync((void **)&dn, njobs * sizeof(int), st)) ||
        (e = cudaMallocAsync((void **)&ds, njobs * sizeof(int), st)))
        return set_err(MGPU_ERR_NOMEM, "LDMA buffers", e);
    int rc = MGPU_OK;
    if ((e = cudaMemcpyAsync(de, ered, njobs * sizeof(double), cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(dy, y, njobs * nn * sizeof(double), cudaMemcpyHostToDevice, st)))
        rc = set_err(MGPU_ERR_CUDA, "copying LDMA inputs", e);
    if (!rc) {
        const size_t sm = mgpu::ldma::smem_bytes(h->t.n);
        if ((e = set_smem(mgpu::ldma::ldma_kernel, sm))) {
            rc = set_err(MGPU_ERR_CUDA, "ldma_kernel set-up", e);
        } else {
            mgpu::ldma::ldma_kernel<<<njobs, mgpu::ldma::kThreads, sm, st>>>(h->t, de, dy, dn, ds);
            if ((e = cudaGetLastError())) rc = set_err(MGPU_ERR_CUDA, "launching ldma_kernel", e);
        }
    }
    if (!rc && ((e = cudaMemcpyAsync(y, dy, njobs * nn * sizeof(double), cudaMemcpyDeviceToHost, st)) ||
                (e = cudaMemcpyAsync(nodes, dn, njobs * sizeof(int), cudaMemcpyDeviceToHost, st)) ||
                (e = cudaMemcpyAsync(status, ds, njobs * sizeof(int), cudaMemcpyDeviceToHost, st))))
        rc = set_err(MGPU_ERR_CUDA, "copying LDMA results", e);
    cudaFreeAsync(de, st);
    cudaFreeAsync(dy, st);
    cudaFreeAsync(dn, st);
    cudaFreeAsync(ds, st);
    if ((e = cudaStreamSynchronize(st)) && !rc) rc = set_err(MGPU_ERR_CUDA, "LDMA run", e);
    return rc;
}

extern "C" void mgpu_ldma_destroy(mgpu_ldma *h) { delete h; }

// ---- AIRY's sweep for the energies of one system (sector tables from the host)
struct mgpu_airy {
    mgpu::ldma::AiryTables t{};
    std::vector<void *> allocs;
    cudaStream_t own = nullptr;
    ~mgpu_airy()
    {
        if (own) cudaStreamSynchronize(own);
        for (void *p : allocs) cudaFree(p);
        if (own) cudaStreamDestroy(own);
    }
};

extern "C" int mgpu_airy_create(mgpu_airy **out, int n, int nsect, int inward, const double *tmat, const double *vfin)
{
    if (!out) return set_err(MGPU_ERR_ARG, "null handle pointer");
    *out = nullptr;
    if (n < 1 || n > mgpu::ldma::kMaxN) return set_err(MGPU_ERR_UNSUPPORTED, "AIRY's sweep runs for 1 <= N <= 100");
    if (nsect < 1 || !tmat || !vfin) return set_err(MGPU_ERR_ARG, "bad sector tables");
    mgpu_airy *h = new (std::nothrow) mgpu_airy();
    if (!h) return set_err(MGPU_ERR_NOMEM, "host allocation failed");
    const size_t nn = (size_t)n * n;
    const AllocFn al = [h](void **p, size_t nb) {
        cudaError_t e = cudaMalloc(p, nb);
        if (e == cudaSuccess) h->allocs.push_back(*p);
        return e;
    };
    const UploadFn up = [](void *dst, const void *src, size_t nb) {
        return cudaMemcpy(dst, src, nb, cudaMemcpyHostToDevice);
    };
    double *dt = nullptr, *dv = nullptr;
    cudaError_t e;
    if ((e = put_n(al, up, &dt, tmat, (size_t)nsect * nn)) || (e = put_n(al, up, &dv, vfin, nn)) ||
        (e = cudaStreamCreateWithFlags(&h->own, cudaStreamNonBlocking))) {
        delete h;
        return set_err(MGPU_ERR_NOMEM, "uploading the AIRY tables", e);
    }
    h->t = mgpu::ldma::AiryTables{n, nsect, inward ? 1 : 0, dt, dv};
    *out = h;
    return MGPU_OK;
}

extern "C" int mgpu_airy_run_host(mgpu_airy *h, int njobs, const double *y124, double *z, int *nodes, int *status)
{
    if (!h) return set_err(MGPU_ERR_ARG, "null handle");
    if (njobs < 0 || njobs > 65535) return set_err(MGPU_ERR_ARG, "0 <= jobs <= 65535");
    if (njobs == 0) return MGPU_OK;
    if (!y124 || !z || !nodes || !status) return set_err(MGPU_ERR_ARG, "null host buffer");
    const size_t nn = (size_t)h->t.n * h->t.n, ny = (size_t)h->t.nsect * h->t.n * 3;
    double *dy = nullptr, *dz = nullptr;
    int *dn = nullptr, *ds = nullptr;
    cudaError_t e;
    cudaStream_t st = h->own;
    if ((e = cudaMallocAsync((void **)&dy, njobs * ny * sizeof(double), st)) ||
        (e = cudaMallocAsync((void **)&dz, njobs * nn * sizeof(double), st)) ||
        (e = cudaMallocAsync((void **)&dn, njobs * sizeof(int), st)) ||
        (e = cudaMallocAsync((void **)&ds, njobs * sizeof(int), st)))
        return set_err(MGPU_ERR_NOMEM, "AIRY buffers", e);
    int rc = MGPU_OK;
    if ((e = cudaMemcpyAsync(dy, y124, njobs * ny * sizeof(double), cudaMemcpyHostToDevice, st)) ||
        (e = cudaMemcpyAsync(dz, z, njobs * nn * sizeof(double), cudaMemcpyHostToDevice, st)))
        rc = set_err(MGPU_ERR_CUDA, "copying AIRY inputs", e);
    if (!rc) {
        const size_t sm = mgpu::ldma::smem_bytes(h->t.n);
        if ((e = set_smem(mgpu::ldma::airy_kernel, sm))) {
            rc = set_err(MGPU_ERR_CUDA, "airy_kernel set-up", e);
        } else {
            mgpu::ldma::airy_kernel<<<njobs, mgpu::ldma::kThreads, sm, st>>>(h->t, dy, dz, dn, ds);
            if ((e = cudaGetLastError())) rc = set_err(MGPU_ERR_CUDA, "launching airy_kernel", e);
        }
    }
    if (!rc && ((e = cudaMemcpyAsync(z, dz, njobs * nn * sizeof(double), cudaMemcpyDeviceToHost, st)) ||
                (e = cudaMemcpyAsync(nodes, dn, njobs * sizeof(int), cudaMemcpyDeviceToHost, st)) ||
                (e = cudaMemcpyAsync(status, ds, njobs * sizeof(int), cudaMemcpyDeviceToHost, st))))
        rc = set_err(MGPU_ERR_CUDA, "copying AIRY results", e);
    cudaFreeAsync(dy, st);
    cudaFreeAsync(dz, st);
    cudaFreeAsync(dn, st);
    cudaFreeAsync(ds, st);
    if ((e = cudaStreamSynchronize(st)) && !rc) rc = set_err(MGPU_ERR_CUDA, "AIRY run", e);
    return rc;
}

extern "C" void mgpu_airy_destroy(mgpu_airy *h) { delete h; }

#include "server.cuh"
