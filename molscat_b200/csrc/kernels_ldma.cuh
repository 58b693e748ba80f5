// MAPROP (maprop.f:33-290), the quasi-adiabatic log-derivative propagator,
// for the energies of one system: one CTA per energy, Y dense in shared
// memory (N <= 100).  Everything that does not depend on the energy -- the
// adiabatic bases at the sector midpoints and their eigenvalues, the basis
// changes Q_k = T_{k-1}^T U_k and the first-order corrections in the old
// basis -- comes from tables the host builds once per system (what the
// reference keeps on its ISCRU file after the first energy).  Per sector:
//   Y += C_k;  Y = Q_k^T Y Q_k;  Y_ii += y1_i;  Y = -y2 Y^-1 y2 + diag(y1)
// with the half-angle propagators of EIVAL - ERED (y3 = y2, y4 = y1), NODES
// from the inversion's negative pivots unless a channel is deeper than
// 24/DR^2; at the end Y = T Y T^T + Q_end.
// Included by propagator.cu.
#pragma once

namespace mgpu {
namespace ldma {

constexpr int kMaxN = 100;  // two n x n matrices in shared memory: 160 KB at 100
constexpr int kThreads = 256;
inline size_t smem_bytes(int n) { return 2 * (size_t)n * n * sizeof(double); }

struct Tables {
    int n, nstep, inward;
    double dr;
    const double *eival;  // [nstep][n]
    const double *q;      // [nstep][n*n] column-major
    const double *corr;   // [nstep][n*n]
    const double *tfin;   // [n*n]
    const double *qfin;   // [n*n]
};

// C = A B for dense n x n matrices, column-major with ld n: A in shared
// memory, B in global memory (read-only for the kernel's lifetime).
__device__ __forceinline__ void gemm(const double *A, const double *__restrict__ B, double *C, int n)
{
    for (int e = threadIdx.x; e < n * n; e += kThreads) {
        const int i = e % n, j = e / n;
        double v = 0.0;
        for (int m = 0; m < n; ++m) v = fma(A[i + m * n], __ldg(B + m + (size_t)j * n), v);
        C[e] = v;
    }
}

__global__ void __launch_bounds__(kThreads)
ldma_kernel(Tables T, const double *__restrict__ ered, double *__restrict__ y, int *__restrict__ nodes_out,
            int *__restrict__ status_out)
{
    extern __shared__ __align__(16) double ldma_sm[];  // A and Z: n*n doubles each
    __shared__ double y1[kMaxN], y2[kMaxN], s_r;
    __shared__ int s_neg, s_bad, s_check;
    const int n = T.n, nn = n * n, tid = threadIdx.x;
    double *A = ldma_sm, *Z = ldma_sm + nn;
    const int job = blockIdx.x;
    const double e = ered[job];
    double *yj = y + (size_t)job * nn;
    for (int x = tid; x < nn; x += kThreads) A[x] = yj[x];
    int nodes = 0, status = MGPU_OK;
    const double wmax = 24.0 / (T.dr * T.dr);
    if (tid == 0) s_bad = 0;
    __syncthreads();
    for (int k = 0; k < T.nstep; ++k) {
        const double *C = T.corr + (size_t)k * nn, *Q = T.q + (size_t)k * nn;
        for (int x = tid; x < nn; x += kThreads) A[x] += __ldg(C + x);  // the correction in the old basis
        __syncthreads();
        gemm(A, Q, Z, n);  // Y Q
        __syncthreads();
        // Q^T (Y Q): Q from global, transposed
        for (int x = tid; x < nn; x += kThreads) {
            const int i = x % n, j = x / n;
            double v = 0.0;
            for (int m = 0; m < n; ++m) v = fma(__ldg(Q + m + (size_t)i * n), Z[m + j * n], v);
            A[x] = v;
        }
        if (tid == 0) {
            s_neg = 0;
            s_check = 0;
        }
        __syncthreads();
        for (int i = tid; i < n; i += kThreads) {
            const double wref = __ldg(T.eival + (size_t)k * n + i) - e;
            const double flam = 0.5 * sqrt(fabs(wref));
            if (wref < 0.0) {
                const double tn = tan(flam * T.dr);
                y1[i] = flam / tn - flam * tn;
                y2[i] = flam / tn + flam * tn;
            } else {
                if (wref > wmax) atomicAdd(&s_check, 1);
                const double th = tanh(flam * T.dr);
                y1[i] = flam / th + flam * th;
                y2[i] = flam / th - flam * th;
            }
        }
        __syncthreads();
        // Y + diag(y1): the lower triangle, mirrored, then an unpivoted
        // Gauss-Jordan inverse (SYMINV's pivots; their negative count)
        for (int x = tid; x < nn; x += kThreads) {
            const int i = x % n, j = x / n;
            Z[x] = (i >= j ? A[x] : A[j + i * n]) + (i == j ? y1[i] : 0.0);
        }
        __syncthreads();
        for (int p = 0; p < n; ++p) {
            if (tid == 0) {
                const double d = Z[p + p * n];
                if (d < 0.0) ++s_neg;
                if (d == 0.0 || !isfinite(d)) s_bad = d == 0.0 ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
                s_r = 1.0 / d;
            }
            __syncthreads();
            const double r = s_r;
            // rows i != p: A_ij -= A_ip A_pj / A_pp (j != p); column p: -A_ip / A_pp; row p: A_pj / A_pp
            for (int x = tid; x < nn; x += kThreads) {
                const int i = x % n, j = x / n;
                if (i != p && j != p) A[x] = Z[x] - Z[i + p * n] * Z[p + j * n] * r;
            }
            __syncthreads();
            for (int x = tid; x < nn; x += kThreads) {
                const int i = x % n, j = x / n;
                if (i == p && j == p) Z[x] = r;
                else if (j == p) Z[x] = -Z[x] * r;
                else if (i == p) Z[x] = Z[x] * r;
                else Z[x] = A[x];
            }
            __syncthreads();
        }
        if (s_bad) {
            status = s_bad;
            break;
        }
        // Z holds (Y + y1)^-1, taken from its lower triangle as SYMINV
        // leaves it: Y = -y2 Z y2 + diag(y1)
        for (int x = tid; x < nn; x += kThreads) {
            const int i = x % n, j = x / n;
            const double zl = i >= j ? Z[x] : Z[j + i * n];
            A[x] = -y2[i] * zl * y2[j] + (i == j ? y1[i] : 0.0);
        }
        const int cnt = T.inward ? n - s_neg : s_neg;
        if (s_check == 0) nodes += cnt;
        __syncthreads();
    }
    if (status == MGPU_OK) {
        // back to the primitive basis: Y = T Y T^T + Q_end (maprop.f:281-287)
        const double *Tf = T.tfin;
        for (int x = tid; x < nn; x += kThreads) {  // Z = Y T^T
            const int i = x % n, j = x / n;
            double v = 0.0;
            for (int m = 0; m < n; ++m) v = fma(A[i + m * n], __ldg(Tf + j + (size_t)m * n), v);
            Z[x] = v;
        }
        __syncthreads();
        for (int x = tid; x < nn; x += kThreads) {  // T Z + Q_end
            const int i = x % n, j = x / n;
            double v = 0.0;
            for (int m = 0; m < n; ++m) v = fma(__ldg(Tf + i + (size_t)m * n), Z[m + j * n], v);
            yj[x] = v + __ldg(T.qfin + x);
        }
    }
    if (tid == 0) {
        status_out[job] = status;
        nodes_out[job] = status == MGPU_OK ? nodes : 0;
    }
}

// AIRY's sweep (aiprop.f:160-250) for the energies of one system: per
// sector Z = T_k^T Z T_k (symmetrised), (Z + Y1)^-1 by the same unpivoted
// Gauss-Jordan with its negative-pivot count (NODES += count outwards,
// N - count inwards), Z = -Y2 (Z + Y1)^-1 Y2 + Y4; at the end V Z V^T.  The
// sector functions (Y1, Y2, Y4) of every job, sector and channel come from
// the host: y124[job][sector][channel][3].
struct AiryTables {
    int n, nsect, inward;
    const double *tmat;  // [nsect][n*n] column-major
    const double *vfin;  // [n*n]
};

__global__ void __launch_bounds__(kThreads)
airy_kernel(AiryTables T, const double *__restrict__ y124, double *__restrict__ z, int *__restrict__ nodes_out,
            int *__restrict__ status_out)
{
    extern __shared__ __align__(16) double airy_sm[];  // A and Z: n*n doubles each
    __shared__ double s_r;
    __shared__ int s_neg, s_bad;
    const int n = T.n, nn = n * n, tid = threadIdx.x;
    double *A = airy_sm, *Z = airy_sm + nn;
    const int job = blockIdx.x;
    const double *yj = y124 + (size_t)job * T.nsect * n * 3;
    double *zj = z + (size_t)job * nn;
    for (int x = tid; x < nn; x += kThreads) A[x] = zj[x];
    if (tid == 0) s_bad = 0;
    int nodes = 0, status = MGPU_OK;
    __syncthreads();
    for (int k = 0; k < T.nsect; ++k) {
        const double *Q = T.tmat + (size_t)k * nn, *yk = yj + (size_t)k * n * 3;
        gemm(A, Q, Z, n);  // Z T
        __syncthreads();
        for (int x = tid; x < nn; x += kThreads) {  // T^T (Z T)
            const int i = x % n, j = x / n;
            double v = 0.0;
            for (int m = 0; m < n; ++m) v = fma(__ldg(Q + m + (size_t)i * n), Z[m + j * n], v);
            A[x] = v;
        }
        if (tid == 0) s_neg = 0;
        __syncthreads();
        // symmetrised, plus Y1 on the diagonal
        for (int x = tid; x < nn; x += kThreads) {
            const int i = x % n, j = x / n;
            Z[x] = 0.5 * (A[x] + A[j + i * n]) + (i == j ? __ldg(yk + 3 * i) : 0.0);
        }
        __syncthreads();
        for (int p = 0; p < n; ++p) {
            if (tid == 0) {
                const double d = Z[p + p * n];
                if (d < 0.0) ++s_neg;
                if (d == 0.0 || !isfinite(d)) s_bad = d == 0.0 ? MGPU_ERR_INVERSION : MGPU_ERR_NONFINITE;
                s_r = 1.0 / d;
            }
            __syncthreads();
            const double r = s_r;
            for (int x = tid; x < nn; x += kThreads) {
                const int i = x % n, j = x / n;
                if (i != p && j != p) A[x] = Z[x] - Z[i + p * n] * Z[p + j * n] * r;
            }
            __syncthreads();
            for (int x = tid; x < nn; x += kThreads) {
                const int i = x % n, j = x / n;
                if (i == p && j == p) Z[x] = r;
                else if (j == p) Z[x] = -Z[x] * r;
                else if (i == p) Z[x] = Z[x] * r;
                else Z[x] = A[x];
            }
            __syncthreads();
        }
        if (s_bad) {
            status = s_bad;
            break;
        }
        for (int x = tid; x < nn; x += kThreads) {
            const int i = x % n, j = x / n;
            const double zl = i >= j ? Z[x] : Z[j + i * n];
            A[x] = -__ldg(yk + 3 * i + 1) * zl * __ldg(yk + 3 * j + 1) + (i == j ? __ldg(yk + 3 * i + 2) : 0.0);
        }
        nodes += T.inward ? n - s_neg : s_neg;
        __syncthreads();
    }
    if (status == MGPU_OK) {
        const double *V = T.vfin;
        for (int x = tid; x < nn; x += kThreads) {  // Z = A V^T
            const int i = x % n, j = x / n;
            double v = 0.0;
            for (int m = 0; m < n; ++m) v = fma(A[i + m * n], __ldg(V + j + (size_t)m * n), v);
            Z[x] = v;
        }
        __syncthreads();
        for (int x = tid; x < nn; x += kThreads) {  // V Z
            const int i = x % n, j = x / n;
            double v = 0.0;
            for (int m = 0; m < n; ++m) v = fma(__ldg(V + i + (size_t)m * n), Z[m + j * n], v);
            A[x] = v;
        }
        __syncthreads();
        for (int x = tid; x < nn; x += kThreads) zj[x] = 0.5 * (A[x] + A[(x / n) + (x % n) * n]);
    }
    if (tid == 0) {
        status_out[job] = status;
        nodes_out[job] = status == MGPU_OK ? nodes : 0;
    }
}

}  // namespace ldma
}  // namespace mgpu
