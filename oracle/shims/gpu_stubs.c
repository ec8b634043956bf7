/* oracle/shims/gpu_stubs.c -- link stubs for the reference's extern "C" GPU entry points, so
 * that its host functions (CPML, Ricker, smoothing, coefficients...) can be loaded and
 * called on a machine without a GPU.  The tests never call these; each aborts if reached. */
#include <stdio.h>
#include <stdlib.h>
static void swd_stub_abort(const char *n) { fprintf(stderr, "GPU stub %s called\n", n); abort(); }
void getdevice(int *n) { *n = 0; }
void fdtd_2d_GPU_forward(void) { swd_stub_abort("fdtd_2d_GPU_forward"); }
void fdtd_2d_GPU_backward(void) { swd_stub_abort("fdtd_2d_GPU_backward"); }
void variables_malloc(void) { swd_stub_abort("variables_malloc"); }
void variables_free(void) { swd_stub_abort("variables_free"); }
void hilbert_transform1d(void) { swd_stub_abort("hilbert_transform1d"); }
