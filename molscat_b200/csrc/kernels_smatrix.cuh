// Y -> K -> S on the device (YTOK/YTOKG/KSYM ytok.f:21-47, ytokg.f:71-126;
// KTOS ktos.f:149-169), one CTA per propagation: N <= 64 with the matrices in
// shared memory, N <= 1024 with them in a global-memory scratch per job (L2
// resident for the CTAs in flight).  Included by propagator.cu.
//
// For channel i with wavevector w_i = sign(E - EINT_i) sqrt|E - EINT_i| and
// L from CENT_i = L(L+1), at the matching radius R (the grid's last radius
// unless the caller set another, with YTRANS's thresholds where it set an
// asymptotic basis):
//   open   (E > EINT):  sj = x j_L(x)/sqrt(w), sjp = (x j_L)'(x) sqrt(w),
//                       sn = x y_L(x)/sqrt(w), snp = (x y_L)'(x) sqrt(w),  x = w R
//   closed:             sn = 1, snp = |w| d/dx ln[x k_L(x)],  x = |w| R
// In channel order NB (CHNSRT: open channels first, by threshold), with
// KM = Y diag(sn) - diag(snp) and T = Y[:, open] diag(sj) - diag(sjp), the
// K matrix is the open block of KM^{-1} T, symmetrised, and
//   S = (I + iK)(I - iK)^{-1}:  SR = 2(I + K^2)^{-1} - I,  SI = 2(I + K^2)^{-1} K.
// The spherical Bessel functions come from their standard three-term
// recurrences (y_L upward; j_L upward while L < x, otherwise Miller's downward
// recurrence normalised by j_0 or j_1; k_L upward in its scaled form).
#pragma once

namespace mgpu {
namespace smx {

constexpr int kMaxNShared = 64;  // matrices in shared memory up to here
constexpr int kMaxN = 1024;       // global-memory scratch above
constexpr int kThreads = 128;
// the matrices: [KM | T] with padded rows, then K (doubles)
__host__ __device__ constexpr size_t mat_doubles(int n, int no) { return (size_t)n * (n + no + 1) + (size_t)no * no; }
__host__ __device__ constexpr size_t smem_bytes(int n, int no) { return mat_doubles(n, no) * 8; }
// the global-scratch kernel's shared memory: per channel sj, sjp, sn, snp, s_f and the order
__host__ __device__ constexpr size_t chan_smem_bytes(int n) { return (size_t)n * (5 * 8 + 4); }

struct SJob {
    int sys;         // system index
    int nopen;       // open channels
    int out;         // index in the caller's order (status, Y offset)
    int pad;
    double ered;
    long long yoff;  // first double of the job's Y
    long long soff;  // first double of the job's SR / SI
    long long scr;   // first double of the job's matrices in the scratch (N > 64)
    const double *eint;  // [n] thresholds: the coupling's EINT, or YTRANS's asymptotic ones
    const double *cent;  // [n] L(L+1)
    const double *evec;  // [n*n] column-major asymptotic basis, or null (Y already in it)
    double rmatch;       // R of the matching: the grid's last radius unless set
};

// x j_L, (x j_L)', x y_L, (x y_L)'
__device__ void riccati(int l, double x, double &uj, double &ujp, double &un, double &unp)
{
    double s, c;
    sincos(x, &s, &c);
    // y: upward from y_{-1} = sin x / x, y_0 = -cos x / x
    double yprev = s / x, ycur = -c / x;
    for (int m = 0; m < l; ++m) {
        const double t = (2 * m + 1) / x * ycur - yprev;
        yprev = ycur;
        ycur = t;
    }
    double jl, jlm1;
    if (l < x) {
        double jprev = c / x, jcur = s / x;  // j_{-1}, j_0
        for (int m = 0; m < l; ++m) {
            const double t = (2 * m + 1) / x * jcur - jprev;
            jprev = jcur;
            jcur = t;
        }
        jl = jcur;
        jlm1 = jprev;
    } else {
        const int L = (int)fmax((double)l, x) + 40;
        double fp1 = 0.0, f = 1e-280, f1 = 0.0;
        jl = jlm1 = 0.0;
        for (int m = L; m > 0; --m) {
            const double fm1 = (2 * m + 1) / x * f - fp1;
            if (m == l) {
                jl = f;
                jlm1 = fm1;
            }
            if (m == 1) f1 = f;
            fp1 = f;
            f = fm1;
            if (fabs(f) > 1e250) {
                fp1 *= 1e-250;
                f *= 1e-250;
                jl *= 1e-250;
                jlm1 *= 1e-250;
                f1 *= 1e-250;
            }
        }
        const double j0 = s / x, j1 = s / (x * x) - c / x;
        const double scale = fabs(j0) > fabs(j1) ? j0 / f : j1 / f1;
        jl *= scale;
        jlm1 *= scale;
        if (l == 0) jlm1 = c / x;
    }
    uj = x * jl;
    un = x * ycur;
    ujp = x * jlm1 - l * jl;
    unp = x * yprev - l * ycur;
}

// d/dx ln[x k_L(x)] from the scaled recurrence k_{-1} = k_0, k_{m+1} = k_{m-1} + (2m+1)/x k_m
__device__ double klogd(int l, double x)
{
    double kprev = 1.0 / x, kcur = 1.0 / x;
    for (int m = 0; m < l; ++m) {
        const double t = kprev + (2 * m + 1) / x * kcur;
        kprev = kcur;
        kcur = t;
    }
    return -kprev / kcur - l / x;
}

// Gauss-Jordan on the first `nr` rows of A (row stride lda): columns [0, nr)
// are reduced to I, columns [nr, ncol) become A^{-1} B.  Partial pivoting when
// `pivot`.  Returns false (all threads) on a zero pivot.
__device__ bool gauss_jordan(double *A, int lda, int nr, int ncol, bool pivot, int *s_p, double *s_f)
{
    const int tid = threadIdx.x;
    for (int k = 0; k < nr; ++k) {
        if (pivot && tid < 32) {
            double best = -1.0;
            int bi = k;
            for (int i = k + tid; i < nr; i += 32) {
                const double v = fabs(A[i * lda + k]);
                if (v > best) {
                    best = v;
                    bi = i;
                }
            }
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_down_sync(0xffffffffu, best, o);
                const int oi = __shfl_down_sync(0xffffffffu, bi, o);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            if (tid == 0) *s_p = bi;
        }
        __syncthreads();
        const int p = pivot ? *s_p : k;
        if (p != k)
            for (int j = tid; j < ncol; j += kThreads) {
                const double t = A[k * lda + j];
                A[k * lda + j] = A[p * lda + j];
                A[p * lda + j] = t;
            }
        __syncthreads();
        const double piv = A[k * lda + k];
        if (piv == 0.0 || !isfinite(piv)) return false;
        const double rp = 1.0 / piv;
        for (int j = k + 1 + tid; j < ncol; j += kThreads) A[k * lda + j] *= rp;
        for (int i = tid; i < nr; i += kThreads) s_f[i] = A[i * lda + k];
        __syncthreads();
        if (tid == 0) A[k * lda + k] = 1.0;
        const int w = ncol - k - 1;
        for (int e = tid; e < nr * w; e += kThreads) {
            const int i = e / w, j = k + 1 + e % w;
            if (i != k) A[i * lda + j] = fma(-s_f[i], A[k * lda + j], A[i * lda + j]);
        }
        for (int i = tid; i < nr; i += kThreads)
            if (i != k) A[i * lda + k] = 0.0;
        __syncthreads();
    }
    return true;
}

// One job: channel functions, [KM | T], Gauss-Jordan, K, then S.  A and K
// point at shared or global memory; the channel arrays at shared memory.
__device__ void smatrix_job(const SysDev &S, const SJob &job, const int *__restrict__ nb_all,
                            const int *__restrict__ nb_off, const double *__restrict__ y, double *__restrict__ sr,
                            double *__restrict__ si, int *__restrict__ status, double *A, double *K, double *sj,
                            double *sjp, double *sn, double *snp, double *s_f, int *s_nb, int *s_p)
{
    const int n = S.n, no = job.nopen, tid = threadIdx.x;
    const int lda = n + no + 1;
    const double R = job.rmatch;
    for (int c = tid; c < n; c += kThreads) {
        s_nb[c] = nb_all[nb_off[job.sys] + c];
        const double dif = job.ered - job.eint[c];
        const double w = copysign(sqrt(fabs(dif)), dif);
        const int ell = (int)lrint(sqrt(job.cent[c] + 0.25) - 0.5);
        if (dif > 0.0) {
            double uj, ujp, un, unp;
            riccati(ell, w * R, uj, ujp, un, unp);
            const double rd = sqrt(w);
            sj[c] = uj / rd;
            sjp[c] = ujp * rd;
            sn[c] = un / rd;
            snp[c] = unp * rd;
        } else {
            const double aw = fabs(w);
            sj[c] = sjp[c] = 0.0;
            sn[c] = 1.0;
            snp[c] = klogd(ell, aw * R) * aw;
        }
    }
    __syncthreads();
    const double *yj = y + job.yoff;
    for (int e = tid; e < n * (n + no); e += kThreads) {
        const int i = e / (n + no), j = e % (n + no);
        const int a = s_nb[i];
        if (j < n) {
            const int b = s_nb[j];
            A[i * lda + j] = yj[a + (size_t)b * n] * sn[b] - (i == j ? snp[a] : 0.0);
        } else {
            const int b = s_nb[j - n];
            A[i * lda + j] = yj[a + (size_t)b * n] * sj[b] - (i == j - n ? sjp[a] : 0.0);
        }
    }
    __syncthreads();
    bool ok = gauss_jordan(A, lda, n, n + no, true, s_p, s_f);
    // K = symmetrised open block of KM^{-1} T
    if (ok) {
        for (int e = tid; e < no * no; e += kThreads) {
            const int i = e / no, j = e % no;
            K[i * no + j] = 0.5 * (A[i * lda + n + j] + A[j * lda + n + i]);
        }
        __syncthreads();
        // [0.5 K K + 0.5 I | I] in the first `no` rows of A, then Gauss-Jordan (I + K^2 is positive definite)
        for (int e = tid; e < no * 2 * no; e += kThreads) {
            const int i = e / (2 * no), j = e % (2 * no);
            double v;
            if (j < no) {
                v = 0.0;
                for (int m = 0; m < no; ++m) v = fma(K[i * no + m], K[m * no + j], v);
                v = 0.5 * v + (i == j ? 0.5 : 0.0);
            } else {
                v = (i == j - no) ? 1.0 : 0.0;
            }
            A[i * lda + j] = v;
        }
        __syncthreads();
        ok = gauss_jordan(A, lda, no, 2 * no, false, s_p, s_f);
    }
    if (!ok) {
        if (tid == 0) status[job.out] = MGPU_ERR_INVERSION;
        return;
    }
    // SR = SRINV - I, SI = SRINV K (column-major, channel order NB)
    double *srj = sr + job.soff, *sij = si + job.soff;
    for (int e = tid; e < no * no; e += kThreads) {
        const int i = e % no, j = e / no;
        const double inv = A[i * lda + no + j];
        double v = 0.0;
        for (int m = 0; m < no; ++m) v = fma(A[i * lda + no + m], K[m * no + j], v);
        srj[e] = inv - (i == j ? 1.0 : 0.0);
        sij[e] = v;
    }
}

// N <= 64: everything in shared memory
__global__ void __launch_bounds__(kThreads)
smatrix_kernel(const SysDev *__restrict__ systems, const SJob *__restrict__ jobs, const int *__restrict__ nb_all,
               const int *__restrict__ nb_off, const double *__restrict__ y, double *__restrict__ sr,
               double *__restrict__ si, int *__restrict__ status)
{
    extern __shared__ __align__(16) double smx_sm[];
    __shared__ double sj[kMaxNShared], sjp[kMaxNShared], sn[kMaxNShared], snp[kMaxNShared], s_f[kMaxNShared];
    __shared__ int s_nb[kMaxNShared], s_p;
    const SJob job = jobs[blockIdx.x];
    const SysDev &S = systems[job.sys];
    if (status[job.out] != MGPU_OK || job.nopen == 0) return;  // the propagation failed, or no open channel: no S
    double *A = smx_sm;                                          // n x (n + no): [KM | T]
    double *K = smx_sm + (size_t)S.n * (S.n + job.nopen + 1);    // no x no
    smatrix_job(S, job, nb_all, nb_off, y, sr, si, status, A, K, sj, sjp, sn, snp, s_f, s_nb, &s_p);
}

// N <= 1024: the matrices in the global scratch at job.scr, the channel
// arrays in shared memory (chan_smem_bytes)
__global__ void __launch_bounds__(kThreads)
smatrix_kernel_g(const SysDev *__restrict__ systems, const SJob *__restrict__ jobs, const int *__restrict__ nb_all,
                 const int *__restrict__ nb_off, const double *__restrict__ y, double *__restrict__ sr,
                 double *__restrict__ si, int *__restrict__ status, double *__restrict__ scratch)
{
    extern __shared__ __align__(16) double smx_sm[];
    __shared__ int s_p;
    const SJob job = jobs[blockIdx.x];
    const SysDev &S = systems[job.sys];
    if (status[job.out] != MGPU_OK || job.nopen == 0) return;
    const int n = S.n;
    double *sj = smx_sm, *sjp = sj + n, *sn = sjp + n, *snp = sn + n, *s_f = snp + n;
    int *s_nb = reinterpret_cast<int *>(s_f + n);
    double *A = scratch + job.scr;
    double *K = A + (size_t)n * (n + job.nopen + 1);
    smatrix_job(S, job, nb_all, nb_off, y, sr, si, status, A, K, sj, sjp, sn, snp, s_f, s_nb, &s_p);
}

// YTRANS's transform (TRNSFM, ytrans.f90:410-413) Y' = EVEC^T Y EVEC for
// the jobs whose system has an asymptotic basis, as two products of 32x32
// output tiles (pass 1: Z = Y EVEC; pass 2: Y' = EVEC^T Z); a job without
// one is copied by pass 2.  grid (ceil(nmax/32)^2, jobs); 256 threads, each
// four outputs of the tile's column.
constexpr int kTT = 32;
__global__ void __launch_bounds__(256)
ytrans_kernel(const SysDev *__restrict__ systems, const SJob *__restrict__ jobs, int pass,
              const double *__restrict__ y, double *__restrict__ z, double *__restrict__ yt)
{
    __shared__ double As[kTT][kTT + 1], Bs[kTT][kTT + 1];
    const SJob job = jobs[blockIdx.y];
    const int n = systems[job.sys].n;
    const int tilesx = (n + kTT - 1) / kTT;
    const int ti = (int)blockIdx.x % tilesx, tj = (int)blockIdx.x / tilesx;
    if (tj >= tilesx) return;  // the grid covers the largest n
    const int i0 = ti * kTT, j0 = tj * kTT, t = threadIdx.x;
    const int tc = t & 31, tr = t >> 5;
    const double *T = job.evec;
    const double *A = pass == 1 ? y + job.yoff : T;   // pass 1: Y;  pass 2: EVEC (read transposed)
    const double *B = pass == 1 ? T : z + job.yoff;    // pass 1: EVEC; pass 2: Z
    double *C = (pass == 1 ? z : yt) + job.yoff;
    if (T == nullptr) {
        if (pass == 1) return;
        for (int e = t; e < kTT * kTT; e += 256) {
            const int r = e & 31, c = e >> 5;
            if (i0 + r < n && j0 + c < n) C[(i0 + r) + (size_t)(j0 + c) * n] = y[job.yoff + (i0 + r) + (size_t)(j0 + c) * n];
        }
        return;
    }
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int k0 = 0; k0 < n; k0 += kTT) {
        for (int e = t; e < kTT * kTT; e += 256) {
            const int f = e & 31, g = e >> 5;
            if (pass == 1) {  // As[r][k] = Y(i0 + r, k0 + k), r fastest
                As[f][g] = (i0 + f < n && k0 + g < n) ? A[(i0 + f) + (size_t)(k0 + g) * n] : 0.0;
            } else {          // As[r][k] = EVEC(k0 + k, i0 + r), k fastest
                As[g][f] = (i0 + g < n && k0 + f < n) ? A[(k0 + f) + (size_t)(i0 + g) * n] : 0.0;
            }
            Bs[f][g] = (k0 + f < n && j0 + g < n) ? B[(k0 + f) + (size_t)(j0 + g) * n] : 0.0;  // Bs[k][c]
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < kTT; ++k) {
            const double b = Bs[k][tc];
#pragma unroll
            for (int u = 0; u < 4; ++u) acc[u] = fma(As[tr + 8 * u][k], b, acc[u]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int r = tr + 8 * u;
        if (i0 + r < n && j0 + tc < n) C[(i0 + r) + (size_t)(j0 + tc) * n] = acc[u];
    }
}

}  // namespace smx
}  // namespace mgpu
