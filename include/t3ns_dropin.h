/*
 * t3ns_dropin.h — the reference entry points exported by libt3ns_dropin.so.
 *
 * These are exactly the declarations of the reference's own headers, so the
 * reference's unchanged sweep driver links against libt3ns_dropin.so in place
 * of the reference objects Heff.o, davidson.o, wrapper_solvers.o,
 * rOperators_pUpdate.o and rOperators_bUpdate.o, and ahead of the LAPACK
 * library for the decomposition's factorisations.  The
 * structs are the reference's (include/Heff.h, include/rOperators.h,
 * include/siteTensor.h); the library is compiled against those headers
 * because the driver allocates struct Heffdata itself.  All arithmetic runs
 * in the engine (t3ns_b200.h) on the GPU.
 */
#ifndef T3NS_DROPIN_H
#define T3NS_DROPIN_H

#ifdef __cplusplus
extern "C" {
#endif

struct Heffdata;
struct rOperators;
struct siteTensor;
struct symsecs;

/* Replaces init_Heffdata, reference include/Heff.h:166-167, src/Heff.c:1167-1221:
 * fills the driver-visible fields of *data (isdmrg, operators, symsecs,
 * instruction set, nr_qnB) and builds the device plan of the step's matvec. */
void init_Heffdata(struct Heffdata *data, const struct rOperators *Operators,
                   const struct siteTensor *siteObject);

/* Replaces matvecT3NS, reference include/Heff.h:177, src/Heff.c:1049-1062:
 * result = Heff vec on host buffers. */
void matvecT3NS(const double *vec, double *result, void *vdata);

/* Replaces make_diagonal, reference include/Heff.h:185, src/Heff.c:1268-1312:
 * returns malloc'd memory that the driver frees. */
double *make_diagonal(const struct Heffdata *data);

/* Replaces destroy_Heffdata, reference include/Heff.h:192, src/Heff.c:1242-1266. */
void destroy_Heffdata(struct Heffdata *data);

/* Replaces davidson_diagonal_preconditioner, reference include/davidson.h:36-39,
 * src/davidson.c:223-257. */
void davidson_diagonal_preconditioner(const double *result, const double theta, const int size,
                                      const double *diagonal, double *vec_t);

/* Replaces davidson, reference include/davidson.h:56-60, src/davidson.c:259-328.
 * With matvec == matvecT3NS the whole solve is device resident; any other
 * matvec callback is called on host buffers once per iteration. */
int davidson(double *result, double *energy, int size, int max_vecs, int keep_deflate,
             double davidson_tol, int max_its, const double *diagonal,
             void (*matvec)(const double *, double *, void *), void *vdat);

/* Replaces sparse_eigensolve, reference include/wrapper_solvers.h:56-60,
 * src/wrapper_solvers.c:107-128 ("D" = Davidson; any other name falls back to
 * Davidson with the reference's message). */
int sparse_eigensolve(double *result, double *energy, int size, int max_vecs,
                      int keep_deflate, double tol, int max_its, const double *diagonal,
                      void (*matvec)(const double *, double *, void *), void *vdat,
                      const char solver[]);

/* Replaces update_rOperators_physical, reference include/rOperators.h:276-278,
 * src/rOperators_pUpdate.c:364-387: *rops is destroyed and replaced by the
 * set renormalised through the physical site tensor tens. */
void update_rOperators_physical(struct rOperators *rops, const struct siteTensor *tens,
                                const struct symsecs *internalss);

/* Replaces rOperators_append_phys, reference include/rOperators.h:265-266,
 * src/rOperators_pUpdate.c:665-673: *newrops receives oldrops with the site
 * operators of the next physical site appended. */
void rOperators_append_phys(struct rOperators *newrops, const struct rOperators *oldrops);

/* Replaces sum_unique_rOperators, reference include/rOperators.h:159-160,
 * src/rOperators_init.c:228-265: the new set summed from the unique
 * operators `ur` with the instruction set, zero blocks removed (the sums on
 * the GPU).  The drop-in's own updates sum on the device without this call. */
struct instructionset;
struct rOperators sum_unique_rOperators(const struct rOperators *ur, const struct instructionset *set);

/* Replaces update_rOperators_branching, reference include/rOperators.h:289-291,
 * src/rOperators_bUpdate.c:229-248: *newops receives the set on the free bond
 * of the branching tensor tens, built from Operator[0] and Operator[1]. */
void update_rOperators_branching(struct rOperators *newops, const struct rOperators *Operator,
                                 const struct siteTensor *tens);

/* Replace the LAPACKE entry points through which the reference's site-tensor
 * decomposition factorises each symmetry sector (src/siteTensor_decompose.c:
 * LAPACKE_dgesdd at :1060 and :565, LAPACKE_dgeqrf at :285, LAPACKE_dorgqr at
 * :295; LAPACKE's own declarations, column-major layout only).  Link
 * libt3ns_dropin.so ahead of the BLAS/LAPACK library.  Return LAPACK's info
 * codes (0, -i for a bad argument, 1 when the SVD did not converge). */
int LAPACKE_dgesdd(int layout, char jobz, int m, int n, double *a, int lda, double *s, double *u,
                   int ldu, double *vt, int ldvt);
int LAPACKE_dgeqrf(int layout, int m, int n, double *a, int lda, double *tau);
int LAPACKE_dorgqr(int layout, int m, int n, int k, double *a, int lda, const double *tau);

/* Test hook (no counterpart in the reference): writes the compiled schedule
 * of *data to `path` in the step-file layout without using the GPU. */
int t3ns_dropin_schedule_write(const struct Heffdata *data, const char *path);

/* Test hooks (no counterpart in the reference): the compiled schedules of a
 * physical and of a branching update, written to `path` without the GPU. */
int t3ns_dropin_pupdate_write(const struct rOperators *rops, const struct siteTensor *tens,
                              const struct symsecs *internalss, const char *path);
int t3ns_dropin_bupdate_write(const struct rOperators *Operator, const struct siteTensor *tens,
                              const char *path);

#ifdef __cplusplus
}
#endif

#endif /* T3NS_DROPIN_H */
