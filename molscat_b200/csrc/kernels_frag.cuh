// LDMD / LDJ kernels on DMMA fragments: one warp per matrix (N <= 40).
// Included by propagator.cu after SysDev, JobDev, ref_solutions.
//
// Fragment layout (see warp_dmma.cuh): for every lower 8x8 tile t and lane l,
// the two doubles of element (8I + (l>>2), 8J + 2(l&3) + s) are stored at
// [t][l][s], so one warp reads or writes a tile as 512 contiguous bytes.
// VL is stored [term][t][l][s]; the 2HQ(C) table [step][t][l][s].
#pragma once
#include "warp_dmma.cuh"

namespace mgpu {
namespace wf {

constexpr int kWPB = 4;  // warps (matrices) per CTA

// per-warp shared memory (doubles): panel, y14, y14', y23, the 2HQ(C) tile
template <int NT>
struct WarpSmem {
    static constexpr int PAN = G<NT>::WSM;
    static constexpr int VEC = G<NT>::NPAD;
    static constexpr int QD = G<NT>::NTL * 64;
    static constexpr int DOUBLES = PAN + 3 * VEC + QD;
    static constexpr size_t BYTES = (size_t)DOUBLES * 8;
};

// The coupling sum sum_l VL_l P_l(R_ir) on this lane's fragment (SUMLAM,
// sumlam.f:29-36,74-86): the part of W(R) that does not depend on the
// energy or on EINT/CENT.
template <int NT>
__device__ __forceinline__ void w_sum_frag(const SysDev &S, int lane, int ir, double (&w)[G<NT>::NTL][2])
{
    constexpr int NTL = G<NT>::NTL;
    const double *P = S.ptab + (size_t)ir * S.nham;
#pragma unroll
    for (int t = 0; t < NTL; ++t) w[t][0] = w[t][1] = 0.0;
    for (int l = 0; l < S.nham; ++l) {
        const double *v = S.vlt + (size_t)l * NTL * 64 + lane * 2;
        if (S.ivlfl <= 0) {
            const double pl = __ldg(P + l);
#pragma unroll
            for (int t = 0; t < NTL; ++t) {
                const double2 x = __ldg(reinterpret_cast<const double2 *>(v + t * 64));
                w[t][0] = fma(x.x, pl, w[t][0]);
                w[t][1] = fma(x.y, pl, w[t][1]);
            }
        } else {
            const int *iv = S.ivt + (size_t)l * NTL * 64 + lane * 2;
#pragma unroll
            for (int t = 0; t < NTL; ++t)
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const double x = __ldg(v + t * 64 + s);
                    if (x != 0.0) w[t][s] = fma(x, __ldg(P + __ldg(iv + t * 64 + s)), w[t][s]);
                }
        }
    }
}

// The diagonal terms of W(R_ir) (HAMMAT, hammat.f:85-113): CENT/R^2 (the
// 1e16 clamp), EINT, the confinement term, then -ERED.  x is the coupling
// sum of channel i's diagonal element.
__device__ __forceinline__ double w_diag_terms(const SysDev &S, int i, double x, double rsq, double conf, double ered)
{
    if (S.nrsq == 0) x += rsq * S.cent[i];
    if (S.nconst == 0) x += S.eint[i];
    if (S.conlen > 0.0) x += conf;
    return x - ered;
}

__device__ __forceinline__ void w_radial(const SysDev &S, int ir, double &rsq, double &conf)
{
    const double R = __ldg(S.rtab + ir);
    rsq = fmin(1.0 / (R * R), 1.0e16);
    conf = 0.0;
    if (S.conlen > 0.0) {
        const double c2 = S.conlen * S.conlen;
        conf = R * R / (c2 * c2);
    }
}

template <int NT>
__device__ __forceinline__ void w_diag_frag_terms(const SysDev &S, int lane, int ir, double ered,
                                                  double (&w)[G<NT>::NTL][2])
{
    double rsq, conf;
    w_radial(S, ir, rsq, conf);
    const int r = lane >> 2, q = lane & 3;
#pragma unroll
    for (int I = 0; I < NT; ++I)
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const int i = 8 * I + r;
            if (r == 2 * q + s && i < S.n) w[tix(I, I)][s] = w_diag_terms(S, i, w[tix(I, I)][s], rsq, conf, ered);
        }
}

// W(R) on this lane's fragment (HAMMAT + SUMLAM, hammat.f:85-113).
template <int NT>
__device__ __forceinline__ void w_frag(const SysDev &S, int lane, int ir, double ered, bool diag_terms,
                                       double (&w)[G<NT>::NTL][2])
{
    w_sum_frag<NT>(S, lane, ir, w);
    if (diag_terms) w_diag_frag_terms<NT>(S, lane, ir, ered, w);
}

// W(R_2m) for the step loop: the coupling sum from the system's table when
// it has one (the preparation wrote it), else from VL; then the diagonal.
template <int NT>
__device__ __forceinline__ void w_step_frag(const SysDev &S, int lane, int m, double ered, double (&w)[G<NT>::NTL][2])
{
    constexpr int NTL = G<NT>::NTL;
    if (S.wt != nullptr) {
        const double *src = S.wt + (size_t)m * NTL * 64 + lane * 2;
#pragma unroll
        for (int t = 0; t < NTL; ++t) {
            const double2 x = __ldg(reinterpret_cast<const double2 *>(src + t * 64));
            w[t][0] = x.x;
            w[t][1] = x.y;
        }
    } else {
        w_sum_frag<NT>(S, lane, 2 * m, w);
    }
    w_diag_frag_terms<NT>(S, lane, 2 * m, ered, w);
}

// The coupling sum of W(R_ir)_ii for channel i.
template <int NT>
__device__ __forceinline__ double w_diag_sum_frag(const SysDev &S, int i, int ir)
{
    constexpr int NTL = G<NT>::NTL;
    const int I = i >> 3, r = i & 7;
    const int lane = r * 4 + (r >> 1), s = r & 1;  // lane holding (r, r) of tile (I, I)
    const size_t e = (size_t)tix(I, I) * 64 + lane * 2 + s;
    const double *P = S.ptab + (size_t)ir * S.nham;
    double x = 0.0;
    for (int l = 0; l < S.nham; ++l) {
        const double v = __ldg(S.vlt + (size_t)l * NTL * 64 + e);
        if (S.ivlfl <= 0) x = fma(v, __ldg(P + l), x);
        else if (v != 0.0) x = fma(v, __ldg(P + __ldg(S.ivt + (size_t)l * NTL * 64 + e)), x);
    }
    return x;
}

// W(R)_ii (the DIAG array of HAMMAT) for channel i.
template <int NT>
__device__ __forceinline__ double w_diag_frag(const SysDev &S, int i, int ir, double ered)
{
    double rsq, conf;
    w_radial(S, ir, rsq, conf);
    return w_diag_terms(S, i, w_diag_sum_frag<NT>(S, i, ir), rsq, conf, ered);
}

// W(R_2k-1)_ii for the step loop, the coupling sum from the system's table
// when it has one.
template <int NT>
__device__ __forceinline__ double w_mid_diag_frag(const SysDev &S, int i, int k, double ered)
{
    double rsq, conf;
    w_radial(S, 2 * k - 1, rsq, conf);
    const double x = S.wd != nullptr ? __ldg(S.wd + (size_t)(k - 1) * G<NT>::NPAD + i)
                                     : w_diag_sum_frag<NT>(S, i, 2 * k - 1);
    return w_diag_terms(S, i, x, rsq, conf, ered);
}

template <int NT>
__device__ __forceinline__ void load_lower_frag(const double *__restrict__ y, int n, int lane,
                                                double (&a)[G<NT>::NTL][2])
{
#pragma unroll
    for (int I = 0; I < NT; ++I)
#pragma unroll
        for (int J = 0; J <= I; ++J)
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const int i = frow(I, lane), j = fcol(J, lane, s);
                const int lo = i < j ? i : j, hi = i < j ? j : i;
                a[tix(I, J)][s] = (i < n && j < n) ? y[(size_t)lo * n + hi] : 0.0;
            }
}

template <int NT>
__device__ __forceinline__ void store_full_frag(double *__restrict__ y, int n, int lane, double scale,
                                                const double (&a)[G<NT>::NTL][2])
{
#pragma unroll
    for (int I = 0; I < NT; ++I)
#pragma unroll
        for (int J = 0; J <= I; ++J)
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const int i = frow(I, lane), j = fcol(J, lane, s);
                if (i < n && j <= i) {
                    const double x = scale * a[tix(I, J)][s];
                    y[(size_t)j * n + i] = x;
                    y[(size_t)i * n + j] = x;
                }
            }
}

// ---------------------------------------------------------------------------
// MDPROP energy-independent half on fragments: grid (ceil(NSTEP/kWPB), systems).
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(32 * kWPB)
ldmd_prep_frag_kernel(const SysDev *__restrict__ systems, const int *__restrict__ sys_list)
{
    constexpr int NTL = G<NT>::NTL;
    __shared__ __align__(16) double pans[kWPB][G<NT>::WSM];
    __shared__ SysDev s_sys;
    if (threadIdx.x == 0) s_sys = systems[sys_list[blockIdx.y]];
    __syncthreads();
    const SysDev &S = s_sys;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k = blockIdx.x * kWPB + warp + 1;
    if (k > S.nstep) return;  // whole warp
    const double h = S.dr / 2.0;
    const double d1 = h * h / 3.0;
    const double d4 = -d1 / 16.0;
    double a[NTL][2];
    if (S.wt != nullptr) {
        // the step loop's coupling sums: W at R_2k (and R_0 for the first
        // step) and the diagonal at R_2k-1, the same arithmetic as there
        for (int m = (k == 1 ? 0 : k); m <= k; ++m) {
            w_sum_frag<NT>(S, lane, 2 * m, a);
            double *dst = S.wt + (size_t)m * NTL * 64 + lane * 2;
#pragma unroll
            for (int t = 0; t < NTL; ++t)
                *reinterpret_cast<double2 *>(dst + t * 64) = make_double2(a[t][0], a[t][1]);
        }
    }
    w_sum_frag<NT>(S, lane, 2 * k - 1, a);
    if (S.wd != nullptr) {
        const int r = lane >> 2, q = lane & 3;
#pragma unroll
        for (int I = 0; I < NT; ++I)
#pragma unroll
            for (int s = 0; s < 2; ++s)
                if (r == 2 * q + s) S.wd[(size_t)(k - 1) * G<NT>::NPAD + 8 * I + r] = a[tix(I, I)][s];
    }
#pragma unroll
    for (int I = 0; I < NT; ++I)
#pragma unroll
        for (int J = 0; J <= I; ++J)
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const int i = frow(I, lane), j = fcol(J, lane, s);
                a[tix(I, J)][s] = (i == j) ? (i < S.n ? 0.125 : 0.0) : d4 * a[tix(I, J)][s];
            }
    int bad = SWEEP_OK;
    const int cnt = warp_sweep_invert<NT>(a, pans[warp], S.n, lane, bad);
    if (bad != SWEEP_OK) {
        if (lane == 0) {
            atomicMax(&S.prep[1], bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE);
            atomicMin(&S.prep[2], k);
        }
        return;
    }
    if (lane == 0 && cnt) atomicAdd(&S.prep[0], cnt);
    double *q = S.q + (size_t)(k - 1) * NTL * 64 + lane * 2;
#pragma unroll
    for (int I = 0; I < NT; ++I)
#pragma unroll
        for (int J = 0; J <= I; ++J) {
            double2 v;
            const int i = frow(I, lane);
            // a = -U^{-1};  2HQ(C) = U^{-1} - 8I
            const int j0 = fcol(J, lane, 0), j1 = fcol(J, lane, 1);
            v.x = (i >= S.n || j0 >= S.n) ? 0.0 : (i == j0 ? -a[tix(I, J)][0] - 8.0 : -a[tix(I, J)][0]);
            v.y = (i >= S.n || j1 >= S.n) ? 0.0 : (i == j1 ? -a[tix(I, J)][1] - 8.0 : -a[tix(I, J)][1]);
            *reinterpret_cast<double2 *>(q + tix(I, J) * 64) = v;
        }
}

// Resident CTAs per SM the register budget is set for: NT = 5 (N 33-40) is
// capped at 168 registers, three CTAs (12 warps) per SM hiding more of the
// per-round latency than its few spills cost (+7 % at N = 36); the smaller NT
// keep the occupancy their natural register counts give (an unconstrained
// bound lets the compiler spend registers and lose a CTA per SM).
constexpr int frag_min_blocks(int nt) { return nt <= 1 ? 5 : (nt <= 3 ? 4 : 3); }
// ---------------------------------------------------------------------------
// MDPROP step loop, one warp per job.
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(32 * kWPB, frag_min_blocks(NT))
ldmd_prop_frag_kernel(const SysDev *__restrict__ systems, const JobDev *__restrict__ jobs, int njobs,
                      double *__restrict__ y, int *__restrict__ nodes_out, int *__restrict__ status_out,
                      int *__restrict__ kfail_out)
{
    constexpr int NTL = G<NT>::NTL;
    constexpr int NPAD = G<NT>::NPAD;
    using W = WarpSmem<NT>;
    extern __shared__ __align__(16) double dsm[];
    __shared__ __align__(8) uint64_t qbar[kWPB];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int jix = blockIdx.x * kWPB + warp;
    if (jix >= njobs) return;  // whole warp; the kernel has no CTA-wide barrier
    const JobDev job = jobs[jix];
    const SysDev &S = systems[job.sys];
    double *pan = dsm + (size_t)warp * W::DOUBLES;
    double *s_y14 = pan + W::PAN;
    double *s_y14b = s_y14 + W::VEC;
    double *s_y23 = s_y14b + W::VEC;
    double *qbuf = s_y23 + W::VEC;
    const int n = S.n;
    const int nstep = S.nstep;
    const double ered = job.ered;
    const uint32_t qbytes = (uint32_t)(NTL * 64 * sizeof(double));
    uint64_t *bar = &qbar[warp];

    if (S.prep[1] != 0) {
        if (lane == 0) {
            status_out[job.out] = S.prep[1];
            kfail_out[job.out] = S.prep[2];
            nodes_out[job.out] = 0;
        }
        return;
    }
    for (int i = lane; i < NPAD; i += 32) s_y14[i] = s_y14b[i] = s_y23[i] = 0.0;
    if (lane == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (lane == 0) bulk_load(qbuf, S.q, qbytes, bar);  // 2HQ(C_1); copy m completes phase m&1

    const double h = S.dr / 2.0;
    const double d1 = h * h / 3.0;
    const double d2 = 2.0 * d1;
    const double half = 0.5 * h;
    double *yj = y + job.yoff;

    double a[NTL][2];
    {
        double w[NTL][2];
        load_lower_frag<NT>(yj, n, lane, a);
        w_step_frag<NT>(S, lane, 0, ered, w);
#pragma unroll
        for (int t = 0; t < NTL; ++t)
#pragma unroll
            for (int s = 0; s < 2; ++s) a[t][s] = h * a[t][s] + d1 * w[t][s];  // mdprop.f:89-93
    }
    const int r = lane >> 2, q = lane & 3;
    int nodes = 0, status = MGPU_OK, kfail = 0;
    int issued = 1, consumed = 0;
    const unsigned long long t0 = global_ns();
    const uint32_t wait_limit = g_step_wait_limit;
    for (int k = 1; k <= nstep; ++k) {
        if (stop_poll_step(k)) {  // host cancel / time limit, lane 0's reading for the warp
            int stop = lane == 0 ? stop_requested(S.ctl, t0) : MGPU_OK;
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (stop != MGPU_OK) {
                status = stop;
                kfail = k;
                break;
            }
        }
        // reference-potential solutions in the sector (mdprop.f:143-164)
        __syncwarp();
        for (int i = lane; i < n; i += 32) {
            const double wref = w_mid_diag_frag<NT>(S, i, k, ered);
            double y14, y23;
            ref_solutions(wref, half, y14, y23);
            s_y14[i] = y14;
            s_y14b[i] = y14 - d1 * wref;
            s_y23[i] = y23;
        }
        __syncwarp();
#pragma unroll
        for (int I = 0; I < NT; ++I)
#pragma unroll
            for (int s = 0; s < 2; ++s)
                if (r == 2 * q + s) a[tix(I, I)][s] += s_y14b[8 * I + r];
        int bad = SWEEP_OK;
        nodes += warp_sweep_invert<NT>(a, pan, n, lane, bad);
        if (bad != SWEEP_OK) {
            status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        const bool landed = mbar_wait_bounded(bar, (k - 1) & 1, wait_limit);
        if (__any_sync(0xffffffffu, !landed)) {
            status = MGPU_ERR_TIMEOUT;
            kfail = k;
            break;
        }
        consumed = k;
        double yr[NT], yc[NT][2];
#pragma unroll
        for (int I = 0; I < NT; ++I) {
            yr[I] = s_y23[8 * I + r];
            yc[I][0] = s_y23[8 * I + 2 * q];
            yc[I][1] = s_y23[8 * I + 2 * q + 1];
        }
        {
            const double *qs = qbuf + lane * 2;
            // Y = 2HQ(C) + 2 Y14 - Y23 Y^-1 Y23   (a holds -Y^-1), mdprop.f:156,181-185
#pragma unroll
            for (int I = 0; I < NT; ++I)
#pragma unroll
                for (int J = 0; J <= I; ++J) {
                    const double2 qq = *reinterpret_cast<const double2 *>(qs + tix(I, J) * 64);
                    a[tix(I, J)][0] = qq.x + yr[I] * a[tix(I, J)][0] * yc[J][0];
                    a[tix(I, J)][1] = qq.y + yr[I] * a[tix(I, J)][1] * yc[J][1];
                }
#pragma unroll
            for (int I = 0; I < NT; ++I)
#pragma unroll
                for (int s = 0; s < 2; ++s)
                    if (r == 2 * q + s) a[tix(I, I)][s] += 2.0 * s_y14[8 * I + r];
        }
        // every lane has read 2HQ(C_k): the async proxy may refill the buffer
        __syncwarp();
        if (lane == 0 && k + 1 <= nstep) {
            fence_async_shared();
            bulk_load(qbuf, S.q + (size_t)k * NTL * 64, qbytes, bar);
            issued = k + 1;
        }
        nodes += warp_sweep_invert<NT>(a, pan, n, lane, bad);
        if (bad != SWEEP_OK) {
            status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        {
            const double dd = (k == nstep) ? d1 : d2;
            double w[NTL][2];
            w_step_frag<NT>(S, lane, k, ered, w);
#pragma unroll
            for (int I = 0; I < NT; ++I)
#pragma unroll
                for (int J = 0; J <= I; ++J)
#pragma unroll
                    for (int s = 0; s < 2; ++s)
                        a[tix(I, J)][s] = dd * w[tix(I, J)][s] + yr[I] * a[tix(I, J)][s] * yc[J][s];
#pragma unroll
            for (int I = 0; I < NT; ++I)
#pragma unroll
                for (int s = 0; s < 2; ++s)
                    if (r == 2 * q + s) a[tix(I, I)][s] += s_y14b[8 * I + r];
        }
    }
    if (status != MGPU_OK && lane == 0 && issued > consumed) {
        // an early exit can leave one copy in flight: let it land (bounded)
        // before this warp's shared memory can be reused
        mbar_wait_bounded(bar, (issued - 1) & 1);
    }
    __syncwarp();
    if (status == MGPU_OK) store_full_frag<NT>(yj, n, lane, 1.0 / h, a);
    if (lane == 0) {
        status_out[job.out] = status;
        kfail_out[job.out] = kfail;
        nodes_out[job.out] = status == MGPU_OK ? nodes - S.prep[0] : 0;
    }
}

// ---------------------------------------------------------------------------
// LDPROP step loop, one warp per job (ldprop.f:46-147).
// ---------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(32 * kWPB)
ldj_prop_frag_kernel(const SysDev *__restrict__ systems, const JobDev *__restrict__ jobs, int njobs,
                     double *__restrict__ y, int *__restrict__ nodes_out, int *__restrict__ status_out,
                     int *__restrict__ kfail_out)
{
    constexpr int NTL = G<NT>::NTL;
    __shared__ __align__(16) double pans[kWPB][G<NT>::WSM];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int jix = blockIdx.x * kWPB + warp;
    if (jix >= njobs) return;
    const JobDev job = jobs[jix];
    const SysDev &S = systems[job.sys];
    double *pan = pans[warp];
    const int n = S.n;
    const double ered = job.ered;
    const double h = S.dr / 2.0;
    const double d1 = h * h / 3.0;
    const double d2 = 2.0 * d1;
    const double d4 = -d1 / 16.0;
    double *yj = y + job.yoff;
    const int r = lane >> 2, q = lane & 3;

    double z[NTL][2], u[NTL][2];
    load_lower_frag<NT>(yj, n, lane, z);
    w_frag<NT>(S, lane, 0, ered, true, u);
#pragma unroll
    for (int I = 0; I < NT; ++I)
#pragma unroll
        for (int J = 0; J <= I; ++J)
#pragma unroll
            for (int s = 0; s < 2; ++s) {
                const bool dg = (I == J) && (r == 2 * q + s) && (8 * I + r < n);
                z[tix(I, J)][s] = h * z[tix(I, J)][s] + d1 * u[tix(I, J)][s] + (dg ? 1.0 : 0.0);  // ldprop.f:46-51
            }
    int nodes = 0, status = MGPU_OK, kfail = 0;
    const unsigned long long t0 = global_ns();
    for (int k = 1; k <= S.nstep; ++k) {
        if (stop_poll_step(k)) {
            int stop = lane == 0 ? stop_requested(S.ctl, t0) : MGPU_OK;
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (stop != MGPU_OK) {
                status = stop;
                kfail = k;
                break;
            }
        }
        w_frag<NT>(S, lane, 2 * k - 1, ered, true, u);
#pragma unroll
        for (int I = 0; I < NT; ++I)
#pragma unroll
            for (int J = 0; J <= I; ++J)
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const bool dg = (I == J) && (r == 2 * q + s) && (8 * I + r < n);
                    u[tix(I, J)][s] = d4 * u[tix(I, J)][s] + (dg ? 0.125 : 0.0);  // ldprop.f:67-72
                }
        int bad = SWEEP_OK;
        const int ncu = warp_sweep_invert<NT>(u, pan, n, lane, bad);  // ldprop.f:78
        int bad2 = SWEEP_OK;
        const int ncz = warp_sweep_invert<NT>(z, pan, n, lane, bad2);  // ldprop.f:83
        if (bad != SWEEP_OK || bad2 != SWEEP_OK) {
            status = (bad == SWEEP_ZERO || bad2 == SWEEP_ZERO) ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        nodes += ncz;
#pragma unroll
        for (int I = 0; I < NT; ++I)
#pragma unroll
            for (int J = 0; J <= I; ++J)
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const bool dg = (I == J) && (r == 2 * q + s) && (8 * I + r < n);
                    // Z = U^-1 - Z^-1 - 6I with u = -U^-1, z = -Z^-1 (ldprop.f:92-97)
                    z[tix(I, J)][s] = -u[tix(I, J)][s] + z[tix(I, J)][s] - (dg ? 6.0 : 0.0);
                }
        const int ncz2 = warp_sweep_invert<NT>(z, pan, n, lane, bad);  // ldprop.f:99
        if (bad != SWEEP_OK) {
            status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
            kfail = k;
            break;
        }
        nodes += ncz2 - ncu;
        const double dd = (k == S.nstep) ? d1 : d2;
        w_frag<NT>(S, lane, 2 * k, ered, true, u);
#pragma unroll
        for (int I = 0; I < NT; ++I)
#pragma unroll
            for (int J = 0; J <= I; ++J)
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const bool dg = (I == J) && (r == 2 * q + s) && (8 * I + r < n);
                    // Z = D2 W(B) + 2I - Z^-1 (ldprop.f:114-131)
                    z[tix(I, J)][s] = dd * u[tix(I, J)][s] + (dg ? 2.0 : 0.0) + z[tix(I, J)][s];
                }
    }
    if (status == MGPU_OK) {
        // Y = Z/H - I/H (ldprop.f:140-147)
        const double hi = 1.0 / h;
#pragma unroll
        for (int I = 0; I < NT; ++I)
#pragma unroll
            for (int J = 0; J <= I; ++J)
#pragma unroll
                for (int s = 0; s < 2; ++s) {
                    const bool dg = (I == J) && (r == 2 * q + s);
                    z[tix(I, J)][s] = hi * z[tix(I, J)][s] - (dg ? hi : 0.0);
                }
        store_full_frag<NT>(yj, n, lane, 1.0, z);
    }
    if (lane == 0) {
        status_out[job.out] = status;
        kfail_out[job.out] = kfail;
        nodes_out[job.out] = status == MGPU_OK ? nodes : 0;
    }
}

// ---------------------------------------------------------------------------
// MGPROP step loop (the symplectic log-derivative propagator of Manolopoulos
// and Gray, mgprop.f:63-134), one warp per job.  Per sector, stage k forms
// X = Y + b_k h W(R) and, where a_k != 0, Y = [I - (I + a_k h X)^-1]/(a_k h)
// (the negative pivots of I + a_k h X added to NODES, subtracted where
// a_k < 0); R advances by a_k h.  W of stage k of sector s is row
// s*stride + k of the radial tables (stride = stages, or stages - 1 when
// a_M = 0 and the last stage's W serves as the next sector's first).
// ---------------------------------------------------------------------------
struct MGCoef {
    int m, stride;
    double a[6], b[6];
};
// Table I of D. E. Manolopoulos and S. K. Gray, J. Chem. Phys. 102, 9214
// (1995): [0] CS4 (IMGSEL = 4), [1] McLachlan and Atela's MA5 (IMGSEL = 5).
// The host lays out the radial tables from the same numbers.
#define MGPU_MG_COEFS { \
        {5, 4, \
         {0.20517766154229, 0.40302128160421, -0.12092087633891, 0.51272193319241, 0.0, 0.0}, \
         {0.061758858135626, 0.33897802655364, 0.61479130717558, -0.14054801465937, 0.12501982279453, 0.0}}, \
        {6, 6, \
         {0.33983962583911, -0.088601336903027, 0.58585647682596, -0.60303935653649, 0.32358079655470, \
          0.44236379421975}, \
         {0.11939002928757, 0.69892737038248, -0.17131235827160, 0.40126950225135, 0.010705081848236, \
          -0.058979625498031}}, \
    }
constexpr MGCoef kMGCoef[2] = MGPU_MG_COEFS;
// the device copy, initialised from the same literal list
__constant__ MGCoef c_mg[2] = MGPU_MG_COEFS;
#undef MGPU_MG_COEFS

template <int NT>
__global__ void __launch_bounds__(32 * kWPB)
ldmg_prop_frag_kernel(const SysDev *__restrict__ systems, const JobDev *__restrict__ jobs, int njobs, int method,
                      double *__restrict__ y, int *__restrict__ nodes_out, int *__restrict__ status_out,
                      int *__restrict__ kfail_out)
{
    constexpr int NTL = G<NT>::NTL;
    __shared__ __align__(16) double pans[kWPB][G<NT>::WSM];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int jix = blockIdx.x * kWPB + warp;
    if (jix >= njobs) return;
    const JobDev job = jobs[jix];
    const SysDev &S = systems[job.sys];
    const MGCoef &C = c_mg[method];
    double *pan = pans[warp];
    const int n = S.n;
    const double ered = job.ered;
    const double h = S.dr;
    double *yj = y + job.yoff;
    const int r = lane >> 2, q = lane & 3;

    double a[NTL][2], w[NTL][2];
    load_lower_frag<NT>(yj, n, lane, a);
    int nodes = 0, status = MGPU_OK, kfail = 0;
    const unsigned long long t0 = global_ns();
    for (int sec = 0; sec < S.nstep; ++sec) {
        if (stop_poll_step(sec + 1)) {
            int stop = lane == 0 ? stop_requested(S.ctl, t0) : MGPU_OK;
            stop = __shfl_sync(0xffffffffu, stop, 0);
            if (stop != MGPU_OK) {
                status = stop;
                kfail = sec + 1;
                break;
            }
        }
#pragma unroll 1
        for (int k = 0; k < C.m; ++k) {
            w_frag<NT>(S, lane, sec * C.stride + k, ered, true, w);
            const double bh = C.b[k] * h;
#pragma unroll
            for (int t = 0; t < NTL; ++t)
#pragma unroll
                for (int s = 0; s < 2; ++s) a[t][s] = fma(bh, w[t][s], a[t][s]);  // X = Y + b_k h W
            const double ak = C.a[k];
            if (ak == 0.0) continue;  // Y = X
            const double ah = ak * h;
#pragma unroll
            for (int I = 0; I < NT; ++I)
#pragma unroll
                for (int J = 0; J <= I; ++J)
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        const bool dg = (I == J) && (r == 2 * q + s) && (8 * I + r < n);
                        a[tix(I, J)][s] = ah * a[tix(I, J)][s] + (dg ? 1.0 : 0.0);  // I + a_k h X
                    }
            int bad = SWEEP_OK;
            const int cnt = warp_sweep_invert<NT>(a, pan, n, lane, bad);  // a = -(I + a_k h X)^-1
            if (bad != SWEEP_OK) {
                status = bad == SWEEP_ZERO ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
                kfail = sec + 1;
                break;
            }
            nodes += ak >= 0.0 ? cnt : -cnt;
            const double d1 = 1.0 / ah;
#pragma unroll
            for (int I = 0; I < NT; ++I)
#pragma unroll
                for (int J = 0; J <= I; ++J)
#pragma unroll
                    for (int s = 0; s < 2; ++s) {
                        const bool dg = (I == J) && (r == 2 * q + s) && (8 * I + r < n);
                        a[tix(I, J)][s] = (a[tix(I, J)][s] + (dg ? 1.0 : 0.0)) * d1;  // [I - inverse]/(a_k h)
                    }
        }
        if (status != MGPU_OK) break;
    }
    if (status == MGPU_OK) store_full_frag<NT>(yj, n, lane, 1.0, a);
    if (lane == 0) {
        status_out[job.out] = status;
        kfail_out[job.out] = kfail;
        nodes_out[job.out] = status == MGPU_OK ? nodes : 0;
    }
}

}  // namespace wf
}  // namespace mgpu
