/* isg_refapi.h - the reference's own call surface, backed by libisg.so.
 *
 * libisg_ref.so defines exactly the routines that the reference's driver
 * (mom.cpp) and measurement setup (setup_born.cpp) call, with the same names,
 * signatures and semantics, so those files link against it unchanged in place
 * of setup_mlfma.cpp, gpu.cu, bicgs_gpu.cu, matvec_gpu.cu and kernels.cu.
 *
 * As in the reference, state lives in globals that the caller defines
 * (mom.cpp:4-69): res, box, level, k0, numunk, numrx, toli, iti, pos, unkmap,
 * and the counters bicgst, innert, outert, matvecin, matvecout.  Vectors are
 * host arrays of std::complex<double> in the reference's tree order; each call
 * copies them to the GPU as complex64 and back, as the reference's bicgs does
 * (bicgs_gpu.cu:129-131, 222).  One process drives one GPU (the reference's
 * MPI_COMM_MLFMA collapses to a single rank).  Failures print a message and
 * exit, as gpuAssert would (kernels.h:6-14).
 */
#ifndef ISG_REFAPI_H
#define ISG_REFAPI_H

#include <complex>

/* setup_mlfma.cpp:50 - builds the MLFMA tables for the grid the globals
 * describe and allocates pos[numunk] and unkmap[numunk] (setup_mlfma.cpp:105,
 * 122, 156-185). */
void setup_mlfma();
/* gpu.cu:69 - uploads the tables and allocates the device workspaces. */
void setup_gpu();
/* bicgs_gpu.cu:89 - nothing left to allocate; kept for the call sequence. */
void setup_bicgs();
/* bicgs_gpu.cu:116 - BiCGSTAB on (I - G diag(o)) x = b (or its adjoint) from
 * the caller's x, to relative residual toli within iti iterations. */
void bicgs(std::complex<double> *x, std::complex<double> *o, std::complex<double> *b, bool ishermitian);
/* bicgs_gpu.cu:61 - r = x - G(o x), or r = x - conj(o G(conj x)). */
void matvec(std::complex<double> *x, std::complex<double> *o, std::complex<double> *r, bool ishermitian);
/* matvec_gpu.cu:65, 80 - r = G x and r = conj(G conj(x)). */
void mlfma(std::complex<double> *x, std::complex<double> *r);
void mlfmah(std::complex<double> *x, std::complex<double> *r);
/* matvec_gpu.cu:266, 369 - far-field receiver samples of x (rx[numrx]) and the
 * back-projection of rx onto x[numunk]. */
void aggregate(std::complex<double> *x, std::complex<double> *rx);
void aggregateh(std::complex<double> *x, std::complex<double> *rx);

#endif
