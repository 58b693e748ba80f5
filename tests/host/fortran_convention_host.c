/*
 * A test host that calls libmolscat_gpu the way a Fortran caller does:
 * the replacement MDPROP/LDPROP in molscat_b200/fortran/mdprop_gpu.f binds
 * mgpu_mdprop_f / mgpu_ldprop_f / mgpu_mgprop_f through a BIND(C) interface block without
 * VALUE attributes, so every scalar arrives as the address of a variable
 * and every array as the address of its first element, column-major.
 *
 *     fortran_convention_host <input file> <output file>
 *
 * Input (native binary): int32 iprop, n, nham, nvlblk, ivlfl, nconst, nrsq,
 * nstep; float64 conlen, dr, ered; then float64 vl[nvlblk*n(n+1)/2],
 * int32 iv[same], float64 eint[n], cent[n], rtab[2*nstep+1],
 * ptab[(2*nstep+1)*nham], y[n*n].
 * Output: int32 istat, nodes, kfail; float64 y[n*n].
 */
#include <stdio.h>
#include <stdlib.h>

#include "molscat_gpu.h"

static void *take(FILE *f, size_t bytes)
{
    void *p = malloc(bytes ? bytes : 1);
    if (!p || (bytes && fread(p, 1, bytes, f) != bytes)) {
        fprintf(stderr, "short input\n");
        exit(2);
    }
    return p;
}

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s input output\n", argv[0]);
        return 2;
    }
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 2;
    int hdr[8];
    double hd[3];
    if (fread(hdr, sizeof(int), 8, f) != 8 || fread(hd, sizeof(double), 3, f) != 3) return 2;
    /* Fortran-style locals: the call passes their addresses */
    int iprop = hdr[0], n = hdr[1], nham = hdr[2], nvlblk = hdr[3], ivlfl = hdr[4], nconst = hdr[5],
        nrsq = hdr[6], nstep = hdr[7];
    double conlen = hd[0], dr = hd[1], ered = hd[2];
    const size_t npair = n > 0 ? (size_t)n * (n + 1) / 2 : 0, nn = n > 0 ? (size_t)n * n : 0;
    const int ldmg = iprop == MGPU_PROP_LDMG4 || iprop == MGPU_PROP_LDMG5;
    const size_t nr = nstep < 1 ? 0 : ldmg ? (size_t)mgpu_ldmg_radii(iprop, 0.0, 1.0, nstep, NULL) : 2 * (size_t)nstep + 1;
    double *vl = take(f, sizeof(double) * nvlblk * npair);
    int *iv = take(f, sizeof(int) * nvlblk * npair);
    double *eint = take(f, sizeof(double) * (n > 0 ? n : 0));
    double *cent = take(f, sizeof(double) * (n > 0 ? n : 0));
    double *rtab = take(f, sizeof(double) * nr);
    double *ptab = take(f, sizeof(double) * nr * nham);
    double *y = take(f, sizeof(double) * nn);
    fclose(f);

    int nodes = -1, kfail = -1, istat = -1;
    int imgsel = iprop == MGPU_PROP_LDMG5 ? 5 : 4;
    if (iprop == MGPU_PROP_LDMD)
        mgpu_mdprop_f(&n, &nham, &nvlblk, &ivlfl, &nconst, &nrsq, &conlen, y, vl, iv, eint, cent, &nstep, &dr, rtab,
                      ptab, &ered, &nodes, &kfail, &istat);
    else if (ldmg)
        mgpu_mgprop_f(&imgsel, &n, &nham, &nvlblk, &ivlfl, &nconst, &nrsq, &conlen, y, vl, iv, eint, cent, &nstep,
                      &dr, rtab, ptab, &ered, &nodes, &kfail, &istat);
    else
        mgpu_ldprop_f(&n, &nham, &nvlblk, &ivlfl, &nconst, &nrsq, &conlen, y, vl, iv, eint, cent, &nstep, &dr, rtab,
                      ptab, &ered, &nodes, &kfail, &istat);

    FILE *o = fopen(argv[2], "wb");
    if (!o) return 2;
    int out[3] = {istat, nodes, kfail};
    fwrite(out, sizeof(int), 3, o);
    fwrite(y, sizeof(double), nn, o);
    fclose(o);
    free(vl);
    free(iv);
    free(eint);
    free(cent);
    free(rtab);
    free(ptab);
    free(y);
    return 0;
}
