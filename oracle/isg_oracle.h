/* Restated FP64 oracle of the reference's MLFMA forward/adjoint solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the CPU
 * baseline leg of bench.py load this library, and only as the checker.  It is
 * pinned against the reference's own CPU path (oracle/_ref, built by
 * oracle/Makefile from the reference sources) by tests/test_oracle_pin.py and
 * against the committed fixtures under tests/golden/.
 *
 * Complex arrays are C99 double complex (interleaved re, im) in the
 * reference's tree order: leaf-major, box*box pixels per leaf, row-major
 * inside the leaf (setup_mlfma.cpp:124-175).
 */
#ifndef ISG_ORACLE_H
#define ISG_ORACLE_H

#include <complex.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_ctx orc_ctx;

/* setup_mlfma.cpp:50-640 and setup_interp (:642-695). */
orc_ctx *orc_create(int level, double k0, double res, int box, int beta, int ninter, int numrx);
void orc_destroy(orc_ctx *c);

int orc_numunk(const orc_ctx *c);
int orc_numsamp(const orc_ctx *c, int lvl);
const void *orc_table(const orc_ctx *c, const char *name, int lvl);

/* integrate.cpp:15-41: one dense MoM entry (i/4) res^2 H0(k0|t-b|) with the
 * analytic self term. */
double complex orc_integrate(const orc_ctx *c, double complex post, double complex posb);

/* r = G x through the MLFMA (solve.cpp:25-248) and its conjugate form
 * (solve.cpp:8-24). */
void orc_mlfma(orc_ctx *c, const double complex *x, double complex *r);
void orc_mlfmah(orc_ctx *c, const double complex *x, double complex *r);

/* r = G x with every entry from orc_integrate; O(U^2), small grids only. */
void orc_dense_matvec(const orc_ctx *c, const double complex *x, double complex *r);

/* bicgs.cpp:62-87: y = x - G(g x), or y = x - conj(g G(conj x)) when hermitian. */
void orc_matvec(orc_ctx *c, const double complex *x, const double complex *g, double complex *y, int hermitian);

/* bicgs.cpp:88-179 BiCGSTAB from the caller's x; returns the iteration count
 * and writes the final recursive relative residual to *err. */
int orc_bicgs(orc_ctx *c, double complex *x, const double complex *g, const double complex *b, int hermitian,
              double tol, int maxit, double *err);

/* solve.cpp:249-355 receiver projection (numrx far-field samples) and
 * solve.cpp:356-456 its back-projection onto the pixels. */
void orc_aggregate(orc_ctx *c, const double complex *x, double complex *rx);
void orc_aggregateh(orc_ctx *c, double complex *x, const double complex *rx);

/* The reference's inversion driver: synthetic measurements of chi_true
 * (setup_born.cpp:139-168), then the gradient (mom.cpp:247-271) and
 * `iterations` Polak-Ribiere steps (mom.cpp:277-399) from chi = 0.  inc holds
 * ntx incident fields, chi and chi_true are contrasts (eps_r - 1), all in tree
 * order.  hist receives 5 numbers per record (write_error, setup_born.cpp:
 * 239-240: misfit, object error, regularisation cost, gradient norm, object
 * norm), iterations + 1 records; alpha and beta one per iteration. */
int orc_dbim(orc_ctx *c, int ntx, const double complex *inc, const double complex *chi_true, int iterations,
             double regular, double tol, int maxit, double complex *chi, double *hist, double *alpha,
             double complex *beta);

/* Near-field receivers (setup_born.cpp:52-60): go[m][n] = integrate(rx_m, pos_n)
 * for numrx points at the given radius; radius 0 removes them.  orc_receive /
 * orc_receiveh apply go / conj(go)^T (the far-field aggregate / aggregateh when
 * none are set), and orc_dbim uses them in place of aggregate / aggregateh. */
void orc_set_nearfield(orc_ctx *c, double radius);
void orc_receive(orc_ctx *c, const double complex *x, double complex *rx);
void orc_receiveh(orc_ctx *c, double complex *x, const double complex *rx);

/* Seeded inputs (isg_inputs.c): the library's random-ellipse contrast
 * chi = eps_r - 1 in raster order, and plane waves exp(i k0 d.r) of
 * transmitters first..first+count-1 of ntx, written in tree order through
 * unkmap (raster order when unkmap is NULL); bit-identical to
 * isg_make_phantom (kind 0) and isg_make_plane_waves. */
void orc_in_ellipses(int side, double res, int count, double axis_min, double axis_max, double eps_min,
                     double eps_max, double tand_max, uint64_t seed, double complex *chi);
void orc_in_plane_waves(int side, double res, double k0, int ntx, int first, int count, const int *unkmap,
                        double complex *inc);

#ifdef __cplusplus
}
#endif
#endif
