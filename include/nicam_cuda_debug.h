/* Test and debugging hooks of libnicamcuda.so, kept out of the drop-in
 * surface of nicam_cuda.h: none of them has a counterpart in the reference's
 * step interface.  They serve the parity tests (reading a named work field,
 * stopping a step after a phase, checking the division the kernels use) and
 * follow the same conventions: int status, nc_last_error() for the text. */
#ifndef NICAM_CUDA_DEBUG_H
#define NICAM_CUDA_DEBUG_H

#include "nicam_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Debugging aid: run only the first nphases phases of one large step
 * (phase boundaries sit after each halo exchange / kernel group, in the order
 * of Dyn.dynamics_step), without graph capture, then synchronize. */
int nc_run_phases(nc_handle* h, int32_t nphases);

/* Copy a named device work field to host in the reference layout
 * (regional (i,j,k,l), pole (g,k,l)).  Names are those registered by
 * nc_create: the state ("RHOG", "RHOGVX", .., "RHOGQ.<n>") and the work
 * fields of the step (e.g. "rho", "pre", "eth", "gT0.<n>", "Mc").  Returns
 * NC_ERR_ARG for an unknown name.  Debugging and parity tests only. */
int nc_get_field(nc_handle* h, const char* name, double* host_reg, double* host_pl);

/* Self-check of the divisions the kernels use in place of a general division
 * (the reference divides with numpy's IEEE division, e.g.
 * kernels/horizontalizevec.py:51-54, kernels/oprtdiffusion.py, kernels/diag.py,
 * mod_src_tracer.py): a quotient formed from RN(1/b) and a tail with three
 * fused multiply-adds and a multiply.  With y NULL every x[i] is divided by the
 * constant b (reciprocal pair set on the host, as for rscale and 3); otherwise
 * x[i] is divided by y[i] with the pair formed on the device from the
 * correctly rounded reciprocal (as for the density that the diagnostics and
 * the tracer Courant numbers divide by).  Copies the n host doubles in, writes q, copies it
 * back (synchronous).  For finite operands with a normal-range quotient the
 * bits equal the IEEE quotient; the tests compare them.  0 <= n <= 2^28; with
 * y NULL, b finite and nonzero; else NC_ERR_ARG. */
int nc_divide_known(const double* x, const double* y, double* q, int64_t n, double b);

#ifdef __cplusplus
}
#endif

#endif /* NICAM_CUDA_DEBUG_H */
