/* One source's traveltime gradient through the elliptical solver and its
 * adjoint (tests/test_abi.py compiles it). */
#include <cuda_runtime.h>

#include "fold3dpmm.h"

/* One source's traveltime gradient on a 256^3 grid.  M: the six metric
 * arrays (xx xy xz yy yz zz; device, float, field layout); T_dev: the
 * initial field (the source), solved in place; dLdT_dev: dL/dT, e.g. the
 * residuals at the receivers and 0 elsewhere; dLdM_dev: 6 x 258^3 doubles. */
int gradient(fold3d_ctx *ctx, float *const M[6], double *T_dev, const double *dLdT_dev, double *lambda_dev,
             double *dLdM_dev, void *stream)
{
    fold3d_ellip m = {M[0], M[1], M[2], M[3], M[4], M[5]};
    fold3d_grid g = {256, 256, 256, 10.0, 10.0, 10.0};
    unsigned char *W;  /* the winner record: one byte per cell */
    if (cudaMalloc((void **)&W, (size_t)258 * 258 * 258) != cudaSuccess) return FOLD3D_ERR_NOMEM;
    fold3d_opts o;
    fold3d_default_opts(&o);
    o.tol = 1e-10;
    fold3d_report r;
    int rc = fold3d_solve_ellip_record(ctx, &g, &m, T_dev, W, &o, stream, &r);   /* forward */
    if (rc == FOLD3D_OK)                                                         /* adjoint */
        rc = fold3d_adjoint_ellip(ctx, &g, &m, T_dev, W, dLdT_dev, lambda_dev, dLdM_dev, 1000, 1e-12, stream, &r);
    cudaFree(W);
    return rc;
}
