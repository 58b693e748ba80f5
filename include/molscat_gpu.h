/*
 * molscat_gpu.h -- C ABI of the B200 (sm_100a, FP64) log-derivative
 * propagator library libmolscat_gpu.so.
 *
 * It replaces the MOLSCAT / BOUND / FIELD hot path
 *
 *   SUBROUTINE MDPROP(N,MXLAM,NHAM,Y,VL,IV,EINT,CENT,RSTART,RSTOP,NSTEP,DR,
 *                     NODES,IREC,WAVE,ERED,EP2RU,CM2RU,RSCALE,IPRINT)
 *                                     (source_code/mdprop.f:1-4)
 *   SUBROUTINE LDPROP(N,MXLAM,NHAM,Z,VL,IV,EINT,CENT,RSTART,RSTOP,NSTEP,DR,
 *                     NODES,ERED,EP2RU,CM2RU,RSCALE,IPRINT)
 *                                     (source_code/ldprop.f:1-4)
 *
 * and the HAMMAT/SUMLAM/SYMINV work they do per step.  Argument meaning is
 * unchanged: N channels, Y the N x N column-major log-derivative matrix
 * (lower triangle read on entry, full symmetric matrix on exit), VL/IV the
 * coupling array in the reference layout VL(NVLBLK, N(N+1)/2) packed
 * upper-triangle-by-columns, EINT/CENT the thresholds and L(L+1), ERED the
 * reduced total energy, DR the step (negative for inward propagation) and
 * NODES the negative-pivot count.  Everything is in the reference's reduced
 * units (1/RUNIT^2 energies).
 *
 * The only thing that moves across the boundary differently is the
 * potential: POTENL/SCAPOT/PERTRB/VCONST/EP2RU scaling (hammat.f:37-83) is
 * user code, so the caller evaluates the P vector that SUMLAM multiplies
 * into VL at every radius the propagator visits (R_k = RSTART + k*DR/2,
 * k = 0..2*NSTEP, accumulated as R=R+H like mdprop.f:117,203) and passes
 * the table.  CENT/R^2, EINT, confinement and -ERED are added on the device
 * exactly as hammat.f:85-113 does.
 *
 * All pointers are plain host pointers unless the name says _dev.  No
 * CUDA or torch types appear in the signatures.  Return value: MGPU_OK or
 * one of the MGPU_ERR_* codes; the reference STOPs where these are returned.
 */
#ifndef MOLSCAT_GPU_H
#define MOLSCAT_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes (per call and per propagation) */
#define MGPU_OK 0
#define MGPU_ERR_INVERSION 1   /* exactly singular pivot: mdprop.f:282-283, ldprop.f:151-153 */
#define MGPU_ERR_NONFINITE 2   /* NaN/Inf pivot met during an inversion */
#define MGPU_ERR_ARG 3         /* invalid argument (sizes, null pointers) */
#define MGPU_ERR_CUDA 4        /* CUDA runtime failure (no device, launch error) */
#define MGPU_ERR_UNSUPPORTED 5 /* N above the largest compiled bucket */
#define MGPU_ERR_NOMEM 6       /* device allocation failed */
#define MGPU_ERR_TIMEOUT 7     /* a bounded in-kernel wait (TMA copy) expired */
#define MGPU_ERR_CANCELLED 8   /* the host cancelled the plan (mgpu_plan_cancel) */
#define MGPU_ERR_DEADLINE 9    /* a step kernel ran past the plan's time limit (mgpu_plan_set_time_limit) */

/* propagator ids (IPROP values of scctrl.f:170-196) */
#define MGPU_PROP_LDJ 5  /* Johnson log-derivative, LDPROP */
#define MGPU_PROP_LDMD 6 /* Manolopoulos diabatic modified log-derivative, MDPROP */
/* MGPROP (mgprop.f:1-134): the symplectic log-derivative propagator of
 * Manolopoulos and Gray, the reference's IPROP = 8 with IMGSEL = 4 (CS4,
 * five stages, four inversions a sector) or 5 (MA5, six stages and
 * inversions).  N <= 1024 (the one-warp, one-CTA and large-N families).  Its grid's
 * NSTEP is the number of sectors of width DR, and RTAB/PTAB list the radii
 * where the stages evaluate W, in order (mgpu_ldmg_radii): 4*NSTEP + 1 rows
 * for CS4, 6*NSTEP for MA5. */
#define MGPU_PROP_LDMG4 84
#define MGPU_PROP_LDMG5 85

/* One coupled-channel system: a (JTOT, symmetry block[, field]) basis.
 * Mirrors the arguments and hidden inputs SUMLAM/HAMMAT read
 * (hammat.f:1-5, sumlam.f:4,22-23). */
typedef struct mgpu_coupling {
    int n;              /* N */
    int nham;           /* NHAM: terms summed into W */
    int nvlblk;         /* NVLBLK (module potential): stride of VL per pair, >= nham */
    int ivlfl;          /* IVLFL (COMMON /VLFLAG/): 0 -> P index = term, >0 -> IV */
    int nconst;         /* NCONST: >0 means EINT is not added (hammat.f:95) */
    int nrsq;           /* NRSQ: >0 means CENT/R^2 is not added (hammat.f:89) */
    double conlen;      /* CONLEN: harmonic confinement if > 0 (hammat.f:103-108) */
    const double *vl;   /* VL(NVLBLK, N(N+1)/2) */
    const int *iv;      /* IV, same shape as VL, 1-based P indices (ivlfl > 0) */
    const double *eint; /* EINT(N) */
    const double *cent; /* CENT(N) */
} mgpu_coupling;

/* The radial grid of one propagation segment and its potential table. */
typedef struct mgpu_grid {
    int nstep;          /* NSTEP */
    double dr;          /* DR (H = DR/2) */
    const double *rtab; /* [2*NSTEP+1] radii R_k in visiting order */
    const double *ptab; /* [2*NSTEP+1][NHAM] P vectors at R_k */
} mgpu_grid;

/* ---- drop-in single propagations (host buffers) ------------------------
 * mgpu_mdprop replaces MDPROP with WAVE=.FALSE. and no ISCRU scratch file
 * (mdprop.f:1-289); mgpu_ldprop replaces LDPROP (ldprop.f:1-154).
 * y: in = initial log-derivative (lower triangle), out = Y(RSTOP).
 * *nodes: NODES.  *kfail: 1-based step of a failed inversion, else 0. */
int mgpu_mdprop(const mgpu_coupling *c, const mgpu_grid *g, double ered,
                double *y, int *nodes, int *kfail);
int mgpu_ldprop(const mgpu_coupling *c, const mgpu_grid *g, double ered,
                double *z, int *nodes, int *kfail);
/* mgpu_mgprop replaces MGPROP (mgprop.f:1-134) with IMGSEL = 4 (CS4) or 5
 * (MA5): g's tables are the stage radii of mgpu_ldmg_radii; y in and out
 * as MGPROP's Y.  N <= 1024. */
int mgpu_mgprop(int imgsel, const mgpu_coupling *c, const mgpu_grid *g, double ered,
                double *y, int *nodes, int *kfail);

/* The same two calls in the Fortran calling convention, every argument by
 * reference and no structures, for an ISO_C_BINDING interface block with
 * plain arrays (molscat_b200/fortran/mdprop_gpu.f, the replacement for
 * source_code/mdprop.f and ldprop.f, binds these).  The arguments are the
 * fields of mgpu_coupling / mgpu_grid, then Y (in/out), ERED, NODES, the
 * failing step and *istat = MGPU_OK or the status mgpu_mdprop returns. */
void mgpu_mdprop_f(const int *n, const int *nham, const int *nvlblk, const int *ivlfl, const int *nconst,
                   const int *nrsq, const double *conlen, double *y, const double *vl, const int *iv,
                   const double *eint, const double *cent, const int *nstep, const double *dr, const double *rtab,
                   const double *ptab, const double *ered, int *nodes, int *kfail, int *istat);
void mgpu_ldprop_f(const int *n, const int *nham, const int *nvlblk, const int *ivlfl, const int *nconst,
                   const int *nrsq, const double *conlen, double *z, const double *vl, const int *iv,
                   const double *eint, const double *cent, const int *nstep, const double *dr, const double *rtab,
                   const double *ptab, const double *ered, int *nodes, int *kfail, int *istat);
/* MGPROP in the same convention, IMGSEL first. */
void mgpu_mgprop_f(const int *imgsel, const int *n, const int *nham, const int *nvlblk, const int *ivlfl,
                   const int *nconst, const int *nrsq, const double *conlen, double *y, const double *vl,
                   const int *iv, const double *eint, const double *cent, const int *nstep, const double *dr,
                   const double *rtab, const double *ptab, const double *ered, int *nodes, int *kfail, int *istat);

/* ---- batched propagation plans -----------------------------------------
 * A plan holds many systems and many jobs (one job = one propagation of a
 * system at one ERED) resident on the device.  For LDMD the energy
 * independent 2HQ(C) inverses of every step (mdprop.f:113-139; the
 * reference reuses them across energies through its ISCRU file,
 * mdprop.f:106-110) are computed once per system and shared by all of its
 * jobs.  Y buffers hold, job after job in job order, the N*N column-major
 * matrix of each job (offsets from mgpu_plan_y_offset). */
typedef struct mgpu_plan mgpu_plan;

int mgpu_plan_create(mgpu_plan **plan, int iprop, int nsys,
                     const mgpu_coupling *systems, const mgpu_grid *grids,
                     int njobs, const int *job_sys, const double *job_ered);
void mgpu_plan_destroy(mgpu_plan *plan);
size_t mgpu_plan_y_elems(const mgpu_plan *plan);          /* doubles in a Y buffer */
size_t mgpu_plan_y_offset(const mgpu_plan *plan, int job); /* first double of job */
double mgpu_plan_flops(const mgpu_plan *plan);            /* counted FP64 work (3N^3+2NHAM N(N+1) per step) */
/* Systems of the plan that use another system's device tables: those that
 * differ from an earlier system only in EINT and CENT, with the
 * same VL, IV, P and R arrays by address.  They also share its MDPROP U(C)
 * tables and preparation (U uses only the off-diagonal coupling). */
int mgpu_plan_shared_systems(const mgpu_plan *plan);

/* BOUND/FIELD matching counts (bdctrl.f:221-257): for each pair k of jobs
 * (pairs[2k], pairs[2k+1], the same N <= 240) the number of negative
 * eigenvalues of Y_a - Y_b, from the inertia of an unpivoted LDL^T of the
 * difference on the device (Sylvester's law); -1 where a pivot is exactly
 * zero or not finite, for the caller to count from the eigenvalues.  The
 * _device form reads Y from y_dev laid out as the plan's Y buffer, with pairs
 * and counts in device memory, on `stream`; mgpu_plan_match_counts reads the
 * Y of the plan's last mgpu_plan_run_host from device memory (host pairs and
 * counts, synchronous). */
int mgpu_plan_match_counts_device(mgpu_plan *plan, const double *y_dev, int npairs, const int *pairs_dev,
                                  int *counts_dev, void *stream);
int mgpu_plan_match_counts(mgpu_plan *plan, int npairs, const int *pairs, int *counts);

/* Host buffers: copies Y in, runs every job, copies Y, NODES and status out. */
int mgpu_plan_run_host(mgpu_plan *plan, double *y, int *nodes, int *status, int *kfail);

/* Device buffers (y_dev in/out, nodes_dev/status_dev/kfail_dev out) on the
 * given cudaStream_t passed as void* (NULL = legacy default stream).
 * Asynchronous: returns after the launches are queued.  Each large-N bucket
 * runs on a stream pair of the plan's own, forked from and joined back into
 * `stream`, so buckets of different N overlap; the stream must therefore not
 * be capturing a graph. */
int mgpu_plan_run_device(mgpu_plan *plan, double *y_dev, int *nodes_dev,
                         int *status_dev, int *kfail_dev, void *stream);

/* As mgpu_plan_run_device, restricted to some phases: bit 0 = the
 * energy-independent LDMD preparation (2HQ(C) inverses), bit 1 = the
 * propagation itself.  phases = 3 is a full run.  Lets a caller time the
 * propagation kernel alone. */
int mgpu_plan_run_device_phases(mgpu_plan *plan, double *y_dev, int *nodes_dev,
                                int *status_dev, int *kfail_dev, void *stream,
                                int phases);

/* ---- MAPROP (LDMA) ----------------------------------------------------------
 * The quasi-adiabatic log-derivative propagator (maprop.f:1-290, IPROP = 7)
 * for many energies of one system, N <= 100.  Its energy-independent half --
 * per sector k the eigenvalues EIVAL of W at the midpoint (with ERED = 0),
 * the basis change Q_k = T_{k-1}^T U_k and the first-order correction C_k
 * in the old basis, then the last basis T and end correction Q_end -- is
 * built on the host once per system (what the reference keeps on its ISCRU
 * file after the first energy; molscat_b200.ldma builds them).  Tables:
 * eival[nstep][n], q[nstep][n*n], corr[nstep][n*n], tfin[n*n], qfin[n*n],
 * matrices column-major.  inward != 0 for DR < 0 (a sector adds N - count).
 * mgpu_ldma_run_host: y[njobs][n*n] in (the initial Y in the primitive
 * basis) and out (Y at the end), nodes and status per job. */
typedef struct mgpu_ldma mgpu_ldma;
int mgpu_ldma_create(mgpu_ldma **out, int n, int nstep, double dr, int inward, const double *eival,
                     const double *q, const double *corr, const double *tfin, const double *qfin);
int mgpu_ldma_run_host(mgpu_ldma *h, int njobs, const double *ered, double *y, int *nodes, int *status);
void mgpu_ldma_destroy(mgpu_ldma *h);

/* ---- AIRY (the long-range propagator's sweep) ------------------------------
 * aiprop.f:160-250 for many energies of one system, N <= 100: per sector k
 * Z = T_k^T Z T_k, Z = Y4 - Y2 (Z + Y1)^-1 Y2 with NODES from the
 * inversion's negative pivots (N - count for inward = 1), at the end
 * V Z V^T.  The sector geometry (tmat[nsect][n*n]: previous local basis ->
 * this one, the first from the primitive basis; vfin[n*n]: the last local
 * basis) and, per energy, the diagonal sector functions
 * y124[njobs][nsect][n][3] = (Y1, Y2, Y4) come from the host
 * (molscat_b200.airy: the reference's first-energy geometry, Airy functions
 * of the linear reference potential).  z[njobs][n*n]: Z at RSTART in the
 * primitive basis in, at RSTOP out. */
typedef struct mgpu_airy mgpu_airy;
int mgpu_airy_create(mgpu_airy **out, int n, int nsect, int inward, const double *tmat, const double *vfin);
int mgpu_airy_run_host(mgpu_airy *h, int njobs, const double *y124, double *z, int *nodes, int *status);
void mgpu_airy_destroy(mgpu_airy *h);

/* ---- Y -> K -> S on the device ---------------------------------------------
 * YTOK/YTOKG/KSYM (ytok.f:21-47, ytokg.f:71-126) and KTOS (ktos.f:149-169)
 * for every job after its propagation, at R = the grid's last radius: the
 * Riccati-Bessel (open) and modified spherical Bessel (closed) boundary
 * functions, K from Y by a pivoted linear solve, S = (I + iK)(I - iK)^{-1}.
 * Channels in CHNSRT order (chnsrt.f:16-30: by threshold; the NOPEN open
 * channels first).  S buffers hold, job after job, the NOPEN x NOPEN
 * column-major real (SR) and imaginary (SI) parts.  Up to N = 64 a job's
 * matrices live in shared memory; up to N = 1024 (every system of the plan,
 * else MGPU_ERR_UNSUPPORTED) in a device scratch of N(N+NOPEN+1)+NOPEN^2
 * doubles per job, allocated by the plan on first use.  A job whose propagation
 * failed keeps its status and gets no S; a singular K system sets status to
 * MGPU_ERR_INVERSION. */
size_t mgpu_plan_s_elems(const mgpu_plan *plan);          /* doubles in an SR (or SI) buffer */
size_t mgpu_plan_s_offset(const mgpu_plan *plan, int job); /* first double of job's S */
int mgpu_plan_nopen(const mgpu_plan *plan, int job);       /* open channels of job */
/* device buffers: y_dev after a run, status_dev as the run left it */
int mgpu_plan_smatrix_device(mgpu_plan *plan, const double *y_dev, double *sr_dev, double *si_dev,
                             int *status_dev, void *stream);
/* host buffers: initial Y in, S matrices and NODES / status / failing step out */
int mgpu_plan_run_host_smatrix(mgpu_plan *plan, const double *y, double *sr, double *si, int *nodes,
                               int *status, int *kfail);

/* YTRANS (ytrans.f90:1-485) before YTOK: system `sys`'s Y -> S inputs from
 * now on are the asymptotic basis EVEC (n x n column-major; its columns the
 * asymptotic channels, the eigenvectors of the asymptotic Hamiltonian block
 * by block, as YTRANS leaves them in EVEC) or NULL (Y already in that
 * basis), the thresholds EINT[n] and L(L+1) values CENT[n] of those
 * channels (YTRANS's EINT and CENT on exit), and the matching radius RMATCH
 * (the reference's RMAX when a long-range segment follows the plan's grid).
 * The device transforms Y' = EVEC^T Y EVEC (TRNSFM, ytrans.f90:410-413)
 * into a buffer of the plan's own and runs YTOK/KTOS on Y'; CHNSRT order,
 * NOPEN and the S offsets follow the new thresholds (mgpu_plan_nopen,
 * mgpu_plan_s_offset and mgpu_plan_s_elems change accordingly).  The
 * propagation is not affected: it keeps the coupling's EINT and CENT.  The
 * asymptotic Hamiltonian and its diagonalisation stay on the host (they do
 * not depend on the energy: once per system). */
int mgpu_plan_set_asymptote(mgpu_plan *plan, int sys, const double *eint, const double *cent,
                            const double *evec, double rmatch);
/* Y -> K -> S alone, from host matrices (the jobs' Y at their matching
 * radius, in the plan's Y layout): status[njobs] in (the propagations'
 * statuses; a job with a non-zero status gets no S) and out (as
 * mgpu_plan_smatrix_device leaves it).  For a long-range segment that ran
 * elsewhere between the plan's propagation and the matching. */
int mgpu_plan_smatrix_host(mgpu_plan *plan, const double *y, double *sr, double *si, int *status);

/* Stopping a plan's runs from the host.  The step kernels of the one-warp,
 * one-CTA and 4x4-tile families (N <= 200; LDPROP <= 128) poll the plan's
 * controls every 128 steps (steps 1, 129, 257, ...) and a job that sees a
 * stop leaves its step loop with the status and the step recorded, as after
 * a failed inversion; the large-N kernels run their steps to the end.
 * mgpu_plan_cancel(plan, 1): runs in progress and later runs stop with
 *   MGPU_ERR_CANCELLED (callable from any host thread while a run is in
 *   flight: the controls live in device memory and are written by a copy
 *   on a stream of their own, which the copy engine serves beside running
 *   kernels; the call returns once the copy has landed); (plan, 0) clears it.
 * mgpu_plan_set_time_limit(plan, s): a step kernel that has run longer than s
 *   seconds (the device's global timer, from that kernel's start) stops its
 *   jobs with MGPU_ERR_DEADLINE; 0 removes the limit. */
int mgpu_plan_cancel(mgpu_plan *plan, int on);
int mgpu_plan_set_time_limit(mgpu_plan *plan, double seconds);

/* For tests of the timeout path: the iteration limit of the one-warp step
 * kernels' wait for each step's 2HQ(C) copy (limit >= 0; 0 gives up at
 * once, so every job reports MGPU_ERR_TIMEOUT at step 1; -1 restores the
 * default).  The waits that let copies in flight land before an early exit
 * keep the full limit.  Process-wide, current device. */
int mgpu_set_step_wait_limit(int limit);

/* The number of kernel launches one run of the plan makes. */
int mgpu_plan_launches(const mgpu_plan *plan);
/* FP64 work the propagation phase alone does, and the LDMD preparation alone
 * (counted like mgpu_plan_flops: N^3 per inversion, 2 NHAM N(N+1) per W). */
double mgpu_plan_flops_phase(const mgpu_plan *plan, int phases);

/* FP64 FMA throughput probe: `iters` dependent-chain DFMA rounds in every
 * thread of a full-occupancy grid; *flops_out gets the flops executed.
 * Launch is asynchronous on `stream`; out_dev (>= 1 double) receives a
 * checksum so the work cannot be optimised away. */
int mgpu_probe_fp64_fma(double *out_dev, int iters, void *stream, double *flops_out);

/* The pivot reciprocal every inversion uses (a third-order Newton refinement
 * of the hardware seed, exact power-of-two scaling), applied to n doubles:
 * r_dev[i] = 1/x_dev[i] within one ulp for normal results.  Device buffers;
 * asynchronous on `stream`.  For tests of that claim. */
int mgpu_probe_pivot_reciprocal(const double *x_dev, double *r_dev, int n, void *stream);

/* ---- allocation-free variant ---------------------------------------------
 * mgpu_mdprop_noalloc: MDPROP for njobs energies of one system that makes no
 * device allocation at all.  It has no counterpart in the reference.
 *
 * It exists for callers that cannot allocate device memory, for instance a
 * program whose device memory all comes from its own pool or a framework
 * allocator, or one that must not call cudaMalloc/cudaFree inside a
 * latency-critical loop because those calls can synchronise the device.
 *
 * Every pointer inside *c and *g and every array argument is a DEVICE pointer
 * owned by the caller: y_dev holds njobs consecutive N*N column-major
 * matrices (initial Y in, Y(RSTOP) out), ered_dev the njobs reduced
 * energies, and nodes_dev/status_dev/kfail_dev get one value per job, with
 * the meanings of mgpu_mdprop.  The work is queued on `stream` (a
 * cudaStream_t passed as void*, NULL = legacy default stream) and the call
 * returns without waiting.
 *
 * Instead of allocating, the library uses one fixed 64 MiB scratch array,
 * reserved on every GPU that loads the library until the process exits.  A
 * request that needs more, more than 4096 jobs or N above 200 (the large-N
 * kernels need per-job device matrices) is rejected with
 * MGPU_ERR_UNSUPPORTED.  Most of a request's scratch is the per-step 2HQ(C)
 * table: 512*NSTEP*NT*(NT+1)/2 bytes, NT = the 8x8 tile count of N's kernel
 * bucket (ceil(N/8) for N <= 64; 10, 12, 14, 16, 20 or 25 above, the
 * smallest that holds ceil(N/8)); the VL tiles, 512*NHAM*NT*(NT+1)/2 bytes
 * (half again with IVLFL > 0), and a few KB of descriptors come on top.  So
 * N = 36 fits about 8,600 steps and N = 200 about 400.
 *
 * All calls share that array and it keeps the last call's contents (each
 * call rewrites what it reads and zeroes its counters), so calls that overlap
 * on the GPU -- on different streams or from different host threads -- race
 * with each other: serialise them.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and keeps it for the life of
 * the process; make that first call before any stream capture, and make no
 * call after a cudaDeviceReset on that device (the address may be stale).
 *
 * An IV entry outside 1..NHAM (IVLFL > 0) is not checked on the host, since
 * IV lives in device memory here: it turns the coupling into NaN, so every
 * job reports MGPU_ERR_NONFINITE with step 1 (mgpu_plan_create rejects the
 * same input with MGPU_ERR_ARG). */
int mgpu_mdprop_noalloc(const mgpu_coupling *c, const mgpu_grid *g, int njobs,
                        const double *ered_dev, double *y_dev, int *nodes_dev,
                        int *status_dev, int *kfail_dev, void *stream);

/* ---- request server (continuous batching) --------------------------------
 * No counterpart in the reference: its drivers call MDPROP/LDPROP once per
 * (JTOT, parity block, energy) in sequence (mol.driver.f:1181-1855,
 * scctrl.f:173,185).  The server keeps registered systems on the device
 * (VL/IV tiles, EINT/CENT, radial tables and, for MDPROP, the energy-
 * independent 2HQ(C) table, computed once per system) and runs single
 * propagations submitted at any time.  A scheduler thread forms batches of
 * pending requests of one N-bucket (oldest request first), launches each
 * batch on its own stream as soon as a stream slot and enough of the HBM
 * budget are free, and retires batches as they finish, so requests that
 * arrive while others run are admitted without waiting for them and their
 * work overlaps on the device.  A request's result does not depend on the
 * batch it runs in.
 *
 * mgpu_server_create: iprop MGPU_PROP_LDMD or MGPU_PROP_LDJ; hbm_budget_bytes caps
 *   the device memory of batches in flight (registered systems come on top);
 *   `streams` concurrent batches, at most max_batch requests each, at most
 *   max_systems registered systems.
 * mgpu_server_add_system: uploads one system (same arguments as mgpu_mdprop)
 *   and returns its id; blocks until its preparation is done.
 * mgpu_submit: queues one propagation; Y0 (N*N, column-major, host) is
 *   copied, the host outputs y_out (N*N), nodes, status, kfail must stay
 *   valid until the request completes.  *ticket identifies the request.
 * mgpu_poll: 1 when the request is complete, 0 while queued or running.
 * mgpu_wait: blocks until complete; returns MGPU_OK or the error that kept the
 *   request from running (MGPU_ERR_NOMEM when it alone exceeds the budget);
 *   the propagation's own status (zero pivot, ...) is in *status.
 * mgpu_request_times: t3 = {submitted, launched, completed}, seconds on the
 *   host's steady clock.
 * mgpu_release: forgets a completed request.
 * mgpu_server_in_flight: batches on the device, queued requests, bytes in use.
 * mgpu_server_destroy: waits for the work in flight, frees everything. */
typedef struct mgpu_server mgpu_server;
int mgpu_server_create(mgpu_server **server, int iprop, size_t hbm_budget_bytes, int streams, int max_batch,
                       int max_systems);
void mgpu_server_destroy(mgpu_server *server);
int mgpu_server_add_system(mgpu_server *server, const mgpu_coupling *c, const mgpu_grid *g, int *sys_id);
int mgpu_submit(mgpu_server *server, int sys_id, double ered, const double *y0, double *y_out, int *nodes,
                int *status, int *kfail, long long *ticket);
int mgpu_poll(mgpu_server *server, long long ticket);
int mgpu_wait(mgpu_server *server, long long ticket);
int mgpu_request_times(mgpu_server *server, long long ticket, double *t3);
int mgpu_release(mgpu_server *server, long long ticket);
int mgpu_server_in_flight(mgpu_server *server, int *batches, int *queued, size_t *bytes);

/* Kernel family for the sizes two families cover (N <= 64): 0 = FP64
 * tensor-core (DMMA) 8x8 fragments, one warp (N <= 40) or one CTA per
 * matrix (the default); 1 = 4x4 register tiles with the scalar sweep.
 * Affects plans created afterwards; returns the previous setting. */
int mgpu_set_kernel_family(int family);

/* Kernel family for plans and servers created afterwards, for propagator
 * iprop (0 = both) and n_lo <= N <= n_hi -- the autotuner's per-bucket choice
 * (molscat_b200/autotune.py): 0 = the default order (one warp for N <= 40,
 * one CTA up to 200, batched large-N above), 1 = 4x4 register tiles
 * (N <= 64), 2 = the batched large-N kernels (any N).  The latest call
 * covering N wins; a family without a bucket for N falls back to the default.
 * family < 0 clears the choices of iprop (0: all). */
int mgpu_set_family_for_n(int iprop, int n_lo, int n_hi, int family);

/* ---- diagnostics --------------------------------------------------------- */
const char *mgpu_status_string(int status);
const char *mgpu_last_error(void);   /* text of the last CUDA/argument error */
int mgpu_max_n(void);                /* largest N the propagators accept (1024) */
/* The radii MGPROP visits for IPROP = MGPU_PROP_LDMG4 / LDMG5 from RSTART in
 * NSTEP sectors of DR: sector s starts at RSTART + s*DR and stage k moves R
 * by a_k*DR (mgprop.f:75-134).  Writes them to rtab (if not NULL) and
 * returns how many there are (-1 for another IPROP or NSTEP < 1). */
int mgpu_ldmg_radii(int iprop, double rstart, double dr, int nstep, double *rtab);

#ifdef __cplusplus
}
#endif
#endif /* MOLSCAT_GPU_H */
