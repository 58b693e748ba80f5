// The BOUND/FIELD matching count on the device: the number of non-positive
// eigenvalues of Y_out - Y_in at RMATCH (bdctrl.f:221-257 counts them from
// DIAGVL's eigenvalues) obtained as the inertia of an unpivoted LDL^T of the
// difference: by Sylvester's law the negative pivots are the negative
// eigenvalues, and a pivot that is exactly zero or not finite (where the
// count would need the eigenvalues) is reported as -1 for the host to count.
// One CTA per pair; the lower triangle is packed in shared memory
// (N(N+1)/2 doubles, N <= kMatchMaxN).
#pragma once
#include <cuda_runtime.h>
#include <math.h>

namespace mgpu {
namespace match {

constexpr int kThreads = 256;
constexpr int kMatchMaxN = 240;  // 240*241/2 doubles = 226 KB of shared memory

__host__ __device__ constexpr size_t packed(int i, int j) { return (size_t)i * (i + 1) / 2 + j; }  // i >= j

// pairs[2k], pairs[2k+1]: the caller-order jobs whose Y are subtracted;
// yoff / jn: each job's first Y double and N.
__global__ void __launch_bounds__(kThreads) match_count_kernel(const double *__restrict__ y,
                                                               const long long *__restrict__ yoff,
                                                               const int *__restrict__ jn,
                                                               const int *__restrict__ pairs, int *__restrict__ counts)
{
    extern __shared__ __align__(16) double a[];
    __shared__ int s_cnt, s_bad;
    const int pr = blockIdx.x;
    const int ja = pairs[2 * pr], jb = pairs[2 * pr + 1];
    const int n = jn[ja];
    const double *ya = y + yoff[ja];
    const double *yb = y + yoff[jb];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    if (tid == 0) {
        s_cnt = 0;
        s_bad = (jn[jb] != n) ? 1 : 0;
    }
    // lower triangle of Y_a - Y_b (column-major, element (i, j) at i + j n)
    for (int i = warp; i < n; i += nw)
        for (int j = lane; j <= i; j += 32) a[packed(i, j)] = ya[i + (size_t)j * n] - yb[i + (size_t)j * n];
    __syncthreads();
    for (int k = 0; k < n && !s_bad; ++k) {
        const double d = a[packed(k, k)];
        const bool ok = isfinite(d) && d != 0.0;
        if (tid == 0) {
            if (!ok) s_bad = 1;
            else if (d < 0.0) ++s_cnt;
        }
        if (!ok) break;  // every thread read the same d
        const double rd = 1.0 / d;
        // trailing update A(i, j) -= A(i, k) A(j, k) / d for k < j <= i, a warp per row
        for (int i = k + 1 + warp; i < n; i += nw) {
            const double lik = a[packed(i, k)] * rd;
            double *row = a + packed(i, 0);
            for (int j = k + 1 + lane; j <= i; j += 32) row[j] = fma(-lik, a[packed(j, k)], row[j]);
        }
        __syncthreads();
    }
    __syncthreads();
    if (tid == 0) counts[pr] = s_bad ? -1 : s_cnt;
}

}  // namespace match
}  // namespace mgpu
