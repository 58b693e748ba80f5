/*
 * CPU ORACLE -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain-C restatement of the MOLSCAT log-derivative propagator hot path.
 * It exists to check the CUDA implementation (tests, the smoke check and the
 * timed CPU baseline of bench.py).  Nothing in the product links it.
 *
 * Every routine cites the Fortran it restates (paths relative to the
 * reference project root, source_code/...).  Indexing is 0-based here; a
 * Fortran element A(I,J) of an array dimensioned A(IA,*) is a[(J-1)*IA+(I-1)].
 *
 * Parity of this restatement is pinned end to end against the reference's
 * own example outputs (S matrices printed to 14 digits) by the Python driver
 * oracle/oracle.py and tests/test_oracle_golden.py.
 *
 * LAPACK (DSYTRF / DSYTRI, used by SYMINL for N > 30) is not part of the
 * reference; the oracle calls the LP64 OpenBLAS that ships inside the scipy
 * wheel.  Its entry points are handed in at run time by oracle_set_lapack().
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef void (*dsytrf_fn)(const char *uplo, const int *n, double *a,
                          const int *lda, int *ipiv, double *work,
                          const int *lwork, int *info, size_t uplo_len);
typedef void (*dsytri_fn)(const char *uplo, const int *n, double *a,
                          const int *lda, const int *ipiv, double *work,
                          int *info, size_t uplo_len);

static dsytrf_fn g_dsytrf = 0;
static dsytri_fn g_dsytri = 0;

void oracle_set_lapack(void *dsytrf, void *dsytri)
{
    g_dsytrf = (dsytrf_fn)dsytrf;
    g_dsytri = (dsytri_fn)dsytri;
}

#define A_(i, j) a[(size_t)(j) * (size_t)ia + (size_t)(i)]

/* ------------------------------------------------------------------------
 * DSYNEG, lower branch (source_code/dsyneg.f:47-74).
 * Number of negative eigenvalues of the Bunch-Kaufman block diagonal D
 * left by DSYTRF('L').  kpvt holds Fortran (1-based, signed) pivots.
 * ---------------------------------------------------------------------- */
static int dsyneg_lower(const double *a, int ia, const int *kpvt, int n)
{
    int inert = 0;
    double t = 0.0;
    for (int k = n - 1; k >= 0; --k) {
        double d = A_(k, k);
        if (kpvt[k] <= 0) {
            /* 2x2 block: det = (d/t * c - t) * t, two passes (dsyneg.f:63-70) */
            if (t != 0.0) {
                d = t;
                t = 0.0;
            } else {
                t = fabs(A_(k, k - 1));
                d = (d / t) * A_(k - 1, k - 1) - t;
            }
        }
        if (d < 0.0) inert++;
    }
    return inert;
}

/* ------------------------------------------------------------------------
 * SYMINL (source_code/syminl-alloc.f:1-43): DSYTRF('L') + DSYNEG + DSYTRI('L').
 * Returns the inertia in *inert; non-zero return = LAPACK INFO failure
 * (the reference STOPs there, syminl-alloc.f:23-27,37-41).
 * ---------------------------------------------------------------------- */
static int syminl(double *a, int ia, int n, int *inert)
{
    int info = 0, lwork = -1;
    double wq = 0.0;
    if (!g_dsytrf || !g_dsytri) return -1000;
    int *ipiv = (int *)malloc(sizeof(int) * (size_t)n);
    /* workspace query: DSYTRF reports N*NB with NB = ILAENV(1,'DSYTRF',..) */
    g_dsytrf("L", &n, a, &ia, ipiv, &wq, &lwork, &info, 1);
    lwork = (int)wq;
    if (lwork < n) lwork = n;
    double *work = (double *)malloc(sizeof(double) * (size_t)lwork);
    g_dsytrf("L", &n, a, &ia, ipiv, work, &lwork, &info, 1);
    if (info != 0) {
        free(work);
        free(ipiv);
        return info;
    }
    *inert = dsyneg_lower(a, ia, ipiv, n);
    g_dsytri("L", &n, a, &ia, ipiv, work, &info, 1);
    free(work);
    free(ipiv);
    return info;
}

/* ------------------------------------------------------------------------
 * SYMINV (source_code/syminv.f:1-97).  In-place inverse of a symmetric
 * matrix; returns KOUNT (negative pivots) or N+1 when a pivot is exactly 0.
 * N > 30 goes to SYMINL (syminv.f:11-14); LAPACK failure maps to N+1 too.
 * ---------------------------------------------------------------------- */
int oracle_syminv(double *a, int ia, int n)
{
    if (n > 30) {
        int inert = 0;
        int info = syminl(a, ia, n, &inert);
        return info == 0 ? inert : n + 1;
    }
    int kount = 0;
    double x = A_(0, 0);
    if (x < 0.0) kount++;
    if (x == 0.0) return n + 1;
    A_(0, 0) = 1.0 / x;
    if (n == 1) return kount;
    /* form L (syminv.f:27-49) */
    for (int i = 1; i < n; ++i) {
        for (int j = 1; j < i; ++j) {
            x = A_(i, j);
            for (int k = 0; k < j; ++k) x = x - A_(i, k) * A_(j, k);
            A_(i, j) = x;
        }
        x = A_(i, i);
        for (int k = 0; k < i; ++k) {
            double y = A_(i, k);
            double z = y * A_(k, k);
            A_(i, k) = z;
            x = x - y * z;
        }
        if (x < 0.0) kount++;
        if (x == 0.0) return n + 1;
        A_(i, i) = 1.0 / x;
    }
    /* invert L (syminv.f:50-64) */
    for (int i = 0; i < n - 1; ++i) {
        int i1 = i + 1;
        A_(i1, i) = -A_(i1, i);
        for (int j = i1; j < n - 1; ++j) {
            int j1 = j + 1;
            x = -A_(j1, i);
            for (int k = i1; k <= j; ++k) x = x - A_(j1, k) * A_(k, i);
            A_(j1, i) = x;
        }
    }
    /* form the inverse (syminv.f:65-85) */
    for (int i = 0; i < n - 1; ++i) {
        int i1 = i + 1;
        x = A_(i, i);
        for (int k = i1; k < n; ++k) {
            double y = A_(k, i);
            double z = y * A_(k, k);
            A_(k, i) = z;
            x = x + y * z;
        }
        A_(i, i) = x;
        for (int j = i1; j < n - 1; ++j) {
            int j1 = j + 1;
            x = A_(j, i);
            for (int k = j1; k < n; ++k) x = x + A_(k, j) * A_(k, i);
            A_(j, i) = x;
        }
    }
    /* copy into the upper triangle (syminv.f:86-92) */
    for (int i = 1; i < n; ++i)
        for (int j = 0; j < i; ++j) A_(j, i) = A_(i, j);
    return kount;
}

#undef A_

/* ------------------------------------------------------------------------
 * The R-dependent inputs of HAMMAT.  POTENL/SCAPOT/PERTRB/VCONST/EP2RU/RSQ
 * (source_code/hammat.f:37-83) are user code evaluated on the host; the
 * boundary receives, for every radius the propagator visits, the finished
 * P vector (length NHAM) and the radius itself.
 * ---------------------------------------------------------------------- */
typedef struct {
    int n, nham, nvlblk, ivlfl, nconst, nrsq;
    double conlen;
    const double *vl;
    const int *iv;
    const double *eint, *cent;
} oracle_sys;

/* HAMMAT after the P evaluation (hammat.f:85-113) with SUMLAM
 * (sumlam.f:29-36 for IVLFL=0, sumlam.f:74-86 for IVLFL>0) and DSYFIL('L').
 * W is the full N x N column-major matrix; DIAG gets W(I,I). */
static void hammat(const oracle_sys *s, double r, const double *p, double ered,
                   double *w, double *diag)
{
    const int n = s->n, nham = s->nham, nvlblk = s->nvlblk;
    double rsq = 1.0 / (r * r);
    if (rsq > 1.0e16) rsq = 1.0e16; /* hammat.f:31-33 */
    if (s->ivlfl <= 0) {
        /* DGEMV('T',NHAM,J,...) per column J: W(K,J)=sum_i VL(I+i+(K-1)NVLBLK)P(i) */
        size_t i0 = 0;
        for (int j = 0; j < n; ++j) {
            for (int k = 0; k <= j; ++k) {
                double acc = 0.0;
                const double *v = s->vl + i0 + (size_t)k * nvlblk;
                for (int t = 0; t < nham; ++t) acc += v[t] * p[t];
                w[(size_t)j * n + k] = acc;
            }
            i0 += (size_t)(j + 1) * nvlblk;
        }
        for (int j = 0; j < n - 1; ++j) /* DSYFIL('L') dsyfil.f:13-16 */
            for (int i = j + 1; i < n; ++i) w[(size_t)j * n + i] = w[(size_t)i * n + j];
    } else {
        size_t i2 = 0;
        for (int j = 0; j < n; ++j) {
            for (int k = 0; k <= j; ++k) {
                size_t i1 = i2;
                i2 += (size_t)nvlblk;
                double ww = 0.0;
                for (size_t i = i1; i < i1 + (size_t)nham; ++i)
                    if (s->vl[i] != 0.0) ww = ww + s->vl[i] * p[s->iv[i] - 1];
                w[(size_t)k * n + j] = ww;
                w[(size_t)j * n + k] = ww;
            }
        }
    }
    if (s->nrsq == 0)
        for (int i = 0; i < n; ++i) w[(size_t)i * n + i] += rsq * s->cent[i];
    if (s->nconst == 0)
        for (int i = 0; i < n; ++i) w[(size_t)i * n + i] += s->eint[i];
    if (s->conlen > 0.0) {
        double c2 = s->conlen * s->conlen;
        double rc = r * r / (c2 * c2);
        for (int i = 0; i < n; ++i) w[(size_t)i * n + i] += rc;
    }
    for (int i = 0; i < n; ++i) {
        w[(size_t)i * n + i] -= ered;
        if (diag) diag[i] = w[(size_t)i * n + i];
    }
}

void oracle_hammat(int n, int nham, int nvlblk, int ivlfl, int nconst, int nrsq,
                   double conlen, const double *vl, const int *iv,
                   const double *eint, const double *cent, double r,
                   const double *p, double ered, double *w)
{
    oracle_sys s = {n, nham, nvlblk, ivlfl, nconst, nrsq, conlen, vl, iv, eint, cent};
    hammat(&s, r, p, ered, w, 0);
}

/* Status codes shared with the CUDA library's header. */
#define ORC_OK 0
#define ORC_INVERSION 1

/* ------------------------------------------------------------------------
 * MDPROP (source_code/mdprop.f:1-289), WAVE=.FALSE., no ISCRU scratch file.
 * rtab[k], ptab[k*nham..] for k=0..2*nstep are the radii R = RSTART + k*H
 * in the order the reference visits them and the matching P vectors.
 * y (N x N, column-major) holds the initial log-derivative on entry (lower
 * triangle read, mdprop.f:89-93) and Y(RSTOP) on exit (full, :269-275).
 * Returns 0 or ORC_INVERSION with *kfail = KSTEP (1-based).
 * ---------------------------------------------------------------------- */
int oracle_mdprop(int n, int nham, int nvlblk, int ivlfl, int nconst, int nrsq,
                  double conlen, const double *vl, const int *iv,
                  const double *eint, const double *cent, const double *rtab,
                  const double *ptab, int nstep, double dr, double ered,
                  double *y, int *nodes, int *kfail)
{
    oracle_sys s = {n, nham, nvlblk, ivlfl, nconst, nrsq, conlen, vl, iv, eint, cent};
    const size_t nn = (size_t)n * n;
    double h = dr / 2.0;
    double d1 = h * h / 3.0;
    double d2 = 2.0 * d1;
    double d4 = -d1 / 16.0;
    double half = 0.5 * h;
    int nsave = 0, kount;
    double *u = (double *)malloc(sizeof(double) * nn);
    double *diag = (double *)malloc(sizeof(double) * n);
    double *y14 = (double *)malloc(sizeof(double) * n);
    double *y23 = (double *)malloc(sizeof(double) * n);
    int status = ORC_OK;
    *nodes = 0;
    *kfail = 0;
#define U_(i, j) u[(size_t)(j) * n + (i)]
#define Y_(i, j) y[(size_t)(j) * n + (i)]
    int ir = 0;
    hammat(&s, rtab[ir], ptab + (size_t)ir * nham, ered, u, diag);
    for (int j = 0; j < n; ++j)
        for (int i = j; i < n; ++i) Y_(i, j) = h * Y_(i, j) + d1 * U_(i, j);
    for (int kstep = 1; kstep <= nstep; ++kstep) {
        /* 2HQ(C) = [I/8 - (H^2/48) W(C)]^-1 - 8I  (mdprop.f:113-137) */
        ++ir;
        hammat(&s, rtab[ir], ptab + (size_t)ir * nham, ered, u, diag);
        for (int j = 0; j < n; ++j)
            for (int i = j; i < n; ++i) U_(i, j) = d4 * U_(i, j);
        for (int i = 0; i < n; ++i) U_(i, i) = 0.125;
        kount = oracle_syminv(u, n, n);
        if (kount > n) { status = ORC_INVERSION; *kfail = kstep; goto done; }
        nsave += kount;
        for (int i = 0; i < n; ++i) U_(i, i) = U_(i, i) - 8.0;
        /* reference-potential solutions (mdprop.f:143-164) */
        for (int i = 0; i < n; ++i) {
            double wref = diag[i];
            double arg = half * sqrt(fabs(wref));
            if (wref < 0.0) {
                double tn = tan(arg);
                y14[i] = arg / tn - arg * tn;
                y23[i] = arg / tn + arg * tn;
            } else {
                double th = tanh(arg);
                y14[i] = arg / th + arg * th;
                y23[i] = arg / th - arg * th;
            }
            U_(i, i) = U_(i, i) + 2.0 * y14[i];
            y14[i] = y14[i] - d1 * diag[i];
            Y_(i, i) = Y_(i, i) + y14[i];
        }
        kount = oracle_syminv(y, n, n);
        if (kount > n) { status = ORC_INVERSION; *kfail = kstep; goto done; }
        *nodes += kount;
        for (int j = 0; j < n; ++j)
            for (int i = j; i < n; ++i) Y_(i, j) = U_(i, j) - y23[i] * Y_(i, j) * y23[j];
        kount = oracle_syminv(y, n, n);
        if (kount > n) { status = ORC_INVERSION; *kfail = kstep; goto done; }
        *nodes += kount;
        if (kstep == nstep) d2 = d1; /* mdprop.f:196 */
        ++ir;
        hammat(&s, rtab[ir], ptab + (size_t)ir * nham, ered, u, diag);
        for (int j = 0; j < n; ++j)
            for (int i = j; i < n; ++i) U_(i, j) = d2 * U_(i, j);
        for (int j = 0; j < n; ++j)
            for (int i = j; i < n; ++i) {
                double wav = y23[i] * Y_(i, j) * y23[j];
                Y_(i, j) = U_(i, j) - wav;
            }
        for (int i = 0; i < n; ++i) Y_(i, i) = Y_(i, i) + y14[i];
    }
    {
        double hi = 1.0 / h; /* mdprop.f:269-275 */
        for (int j = 0; j < n; ++j)
            for (int i = j; i < n; ++i) {
                Y_(i, j) = hi * Y_(i, j);
                Y_(j, i) = Y_(i, j);
            }
    }
    *nodes -= nsave;
done:
#undef U_
#undef Y_
    free(u);
    free(diag);
    free(y14);
    free(y23);
    return status;
}

/* ------------------------------------------------------------------------
 * LDPROP (source_code/ldprop.f:1-154), no ISCRU scratch file.
 * Same table convention as oracle_mdprop.
 * ---------------------------------------------------------------------- */
int oracle_ldprop(int n, int nham, int nvlblk, int ivlfl, int nconst, int nrsq,
                  double conlen, const double *vl, const int *iv,
                  const double *eint, const double *cent, const double *rtab,
                  const double *ptab, int nstep, double dr, double ered,
                  double *z, int *nodes, int *kfail)
{
    oracle_sys s = {n, nham, nvlblk, ivlfl, nconst, nrsq, conlen, vl, iv, eint, cent};
    const size_t nn = (size_t)n * n;
    double h = dr / 2.0;
    double d1 = h * h / 3.0;
    double d2 = 2.0 * d1;
    double d4 = -d1 / 16.0;
    double *u = (double *)malloc(sizeof(double) * nn);
    int status = ORC_OK, ncu, ncz;
    *nodes = 0;
    *kfail = 0;
#define U_(i, j) u[(size_t)(j) * n + (i)]
#define Z_(i, j) z[(size_t)(j) * n + (i)]
    int ir = 0;
    hammat(&s, rtab[ir], ptab + (size_t)ir * nham, ered, u, 0);
    for (int j = 0; j < n; ++j) {
        for (int i = j; i < n; ++i) Z_(i, j) = h * Z_(i, j) + d1 * U_(i, j);
        Z_(j, j) = 1.0 + Z_(j, j);
    }
    for (int istep = 1; istep <= nstep; ++istep) {
        ++ir;
        hammat(&s, rtab[ir], ptab + (size_t)ir * nham, ered, u, 0);
        for (int j = 0; j < n; ++j) {
            for (int i = j; i < n; ++i) U_(i, j) = d4 * U_(i, j);
            U_(j, j) = 0.125 + U_(j, j);
        }
        ncu = oracle_syminv(u, n, n); /* ldprop.f:78 */
        if (ncu > n) { status = ORC_INVERSION; *kfail = istep; goto done; }
        ncz = oracle_syminv(z, n, n); /* ldprop.f:83 */
        if (ncz > n) { status = ORC_INVERSION; *kfail = istep; goto done; }
        *nodes += ncz;
        for (int j = 0; j < n; ++j) {
            for (int i = j; i < n; ++i) Z_(i, j) = U_(i, j) - Z_(i, j);
            Z_(j, j) = Z_(j, j) - 6.0;
        }
        ncz = oracle_syminv(z, n, n); /* ldprop.f:99 */
        if (ncz > n) { status = ORC_INVERSION; *kfail = istep; goto done; }
        *nodes += ncz - ncu;
        if (istep == nstep) d2 = d1; /* ldprop.f:106 */
        ++ir;
        hammat(&s, rtab[ir], ptab + (size_t)ir * nham, ered, u, 0);
        for (int j = 0; j < n; ++j) {
            for (int i = j; i < n; ++i) U_(i, j) = d2 * U_(i, j);
            U_(j, j) = U_(j, j) + 2.0;
        }
        for (int j = 0; j < n; ++j)
            for (int i = j; i < n; ++i) Z_(i, j) = U_(i, j) - Z_(i, j);
    }
    {
        double hi = 1.0 / h; /* ldprop.f:140-147 */
        for (int j = 0; j < n; ++j) {
            for (int i = j; i < n; ++i) {
                Z_(i, j) = hi * Z_(i, j);
                Z_(j, i) = Z_(i, j);
            }
            Z_(j, j) = Z_(j, j) - hi;
        }
    }
done:
#undef U_
#undef Z_
    free(u);
    return status;
}
