/* A C caller of libfold3dpmm: a whole 512^3 solve of the reference's
 * workload from host buffers, and the reference's own output file
 * (tests/test_abi.py compiles and links it). */
#include <stdio.h>
#include <stdlib.h>

#include "fold3dpmm.h"

int main(void)
{
    fold3d_ctx *ctx;
    if (fold3d_create(&ctx, 0) != FOLD3D_OK) {
        fprintf(stderr, "%s\n", fold3d_last_error());
        return 1;
    }
    fold3d_grid g = {512, 512, 512, 10.0 / 511, 10.0 / 511, 10.0 / 511};
    fold3d_medium m = {1.1, -0.35, 0.4, 0.7};
    double *T = malloc(sizeof(double) * 514 * 514 * 514);
    fold3d_init_implicit(T, &g, &m);
    fold3d_opts o;
    fold3d_default_opts(&o);
    o.max_sweeps = 8;
    o.fixed = 1;
    fold3d_report r;
    int rc = fold3d_solve_host(ctx, &g, &m, T, T, &o, NULL, &r);
    if (rc != FOLD3D_OK) fprintf(stderr, "%s\n", fold3d_last_error());
    else printf("%d sweeps in %.1f ms\n", r.sweeps, r.elapsed_ms);
    fold3d_write_text("an_iso_1_openacc.txt", T, &g);
    free(T);
    fold3d_destroy(ctx);
    return rc != FOLD3D_OK;
}
