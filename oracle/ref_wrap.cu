/* ref_wrap.cu -- builds the reference coder (PabloEnfedaque/CUDA_BPC-PaCo,
 * source/BPC_PaCo.cu + source/common.cu, compiled from where they lie, never
 * copied) into a shared library with a C entry point for tests and timing.
 *
 * TEST INFRASTRUCTURE ONLY: the secondary oracle and the timing bar for
 * "the reference kernel rebuilt for the B200".  Built by oracle/Makefile into
 * oracle/_ref/ (git-ignored).
 *
 * ref_launch() calls the reference's own Kernel_launcher (BPC_PaCo.cu:1232)
 * on caller-provided device buffers, so the caller controls allocation (the
 * LUT buffer is zero-padded past the loader's array, which keeps the
 * reference's reads at bitplanes >= 15 inside the allocation) and can time the
 * kernel alone with events.  Mode (CPASS_3, DWT_LEVELS) is fixed at compile
 * time as in the reference.
 */
#include "BPC_PaCo.cu"

extern "C" int ref_launch(int direction, int *d_in, int *d_out, int X, int Y, int *d_lut, void *stream) {
    (void)stream; /* the reference launches on the default stream */
    Kernel_launcher(direction, X, Y, d_in, d_out, d_lut);
    return (int)cudaGetLastError();
}

extern "C" int ref_mode(int *passes, int *levels) {
    *passes = CPASS_3 ? 3 : 2;
    *levels = DWT_LEVELS;
    return 0;
}
