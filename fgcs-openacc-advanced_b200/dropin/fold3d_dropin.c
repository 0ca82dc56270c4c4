/*
 * fold3d_dropin.c -- strong definitions of the reference's six sweep
 * functions that forward to libfold3dpmm.
 *
 * The reference's single-GPU program defines its sweeps in the same
 * translation unit as its main (Stencil-OpenACC/AN_ISO_1_OpenACC.c:180-1092).
 * To run that program unchanged on this library, compile its translation
 * unit to an object, weaken its six sweep symbols, and link this file in:
 *
 *   gcc -O2 -fPIC -fno-inline -c AN_ISO_1_OpenACC.c -o an_iso_1.o
 *   objcopy --weaken-symbol=function_x_down ... --weaken-symbol=function_k_down an_iso_1.o
 *   gcc an_iso_1.o fold3d_dropin.c -I<repo>/include -L<pkg> -lfold3dpmm -lm -o an_iso_1_gpu
 *
 * The program's own acc_malloc / acc_memcpy_* calls and ImplicitInitialiser
 * then also resolve to the library (which exports them), as long as no other
 * OpenACC runtime is linked ahead of it.
 */
#include "fold3dpmm.h"

#define FOLD3D_FORWARD(name, dir)                                                             \
    void name(double *T, int p, double dzz, double dxx, double dyy, double dxy, double dxz,   \
              double dyz, double F, double ay, double ax, double az)                          \
    {                                                                                         \
        fold3d_compat_plane(dir, T, p, dzz, dxx, dyy, dxy, dxz, dyz, F, ay, ax, az);          \
    }

FOLD3D_FORWARD(function_x_down, FOLD3D_X_DOWN)
FOLD3D_FORWARD(function_x_up, FOLD3D_X_UP)
FOLD3D_FORWARD(function_y_up, FOLD3D_Y_UP)
FOLD3D_FORWARD(function_y_down, FOLD3D_Y_DOWN)
FOLD3D_FORWARD(function_k_up, FOLD3D_K_UP)
FOLD3D_FORWARD(function_k_down, FOLD3D_K_DOWN)
