/* A reference-side caller of every host helper the reference's Fold3dPMM.h
 * declares (InitFoldFromPoint, ImpSurfF, InitNode, updateVoxel, x, y, z,
 * ImplicitInitialiser), on an 8^3 grid (pitch 10).  Built with
 * -DREF_HEADER it includes the reference's own header; otherwise this
 * library's.  tests/test_oracle.py links it once against libfold3dpmm.so
 * alone and once against the reference's host build, runs both and compares
 * the printed bits. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef REF_HEADER
#include "Fold3dPMM.h"
#else
#include "fold3dpmm.h"
#endif

#define N 8
#define P (N + 2)

static unsigned long long fnv(const double *a, size_t n)
{
    unsigned long long h = 1469598103934665603ull;
    const unsigned char *b = (const unsigned char *)a;
    for (size_t q = 0; q < n * sizeof(double); ++q) h = (h ^ b[q]) * 1099511628211ull;
    return h;
}

static void bits(const char *name, double v)
{
    unsigned long long u;
    memcpy(&u, &v, sizeof u);
    printf("%s %016llx\n", name, u);
}

int main(void)
{
    const double h = 10.0 / (N - 1.0);
    double *T = malloc(sizeof(double) * P * P * P);
    if (!T) return 1;
    ImplicitInitialiser(T, N, N, N, h, h, h);
    printf("init %016llx\n", fnv(T, P * P * P));
    /* point sources seeded by hand, as a caller of the helpers would */
    for (int q = 0; q < P * P * P; ++q) T[q] = (q % 3) ? 1e16 : -1e16;
    InitNode(0.3 * h, -0.2 * h, 0.1 * h, 4, 5, 3, T);
    InitNode(-0.7 * h, 0.45 * h, -0.25 * h, 6, 2, 7, T);
    updateVoxel(T, 3, 4, 5, x(3, h) - 0.37 * h, y(4, h) + 0.21 * h, z(5, h) - 0.5 * h, h, h, h);
    updateVoxel(T, 5, 5, 2, 0.61 * h, 0.13 * h, 0.88 * h, h, 1.5 * h, 0.75 * h);
    printf("seeded %016llx\n", fnv(T, P * P * P));
    bits("x", x(7, h));
    bits("y", y(0, 0.3));
    bits("z", z(9, 1.7));
    bits("exact", InitFoldFromPoint(1.1, -0.35, 0.4, 0.7, 0.3, -1.2, 2.5));
    bits("surface", ImpSurfF(1.3, 4.2, 7.7));
    free(T);
    return 0;
}
