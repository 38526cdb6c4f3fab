/*
 * t3ns_b200.h — C ABI of the B200 effective-Hamiltonian engine.
 *
 * Plain pointers and sizes only.  Two layers sit behind this header:
 *
 *  1. The engine (this header): a matvec plan built from the flattened
 *     schedule of one optimisation step, device-resident operator blocks,
 *     hand-written sm_100a kernels, and a device-resident Davidson solver.
 *  2. The drop-in (t3ns_dropin.h): the reference's own entry points
 *     (init_Heffdata, matvecT3NS, make_diagonal, destroy_Heffdata,
 *     davidson, sparse_eigensolve, ...) implemented on top of layer 1, so
 *     the unchanged reference sweep driver links against this library.
 *
 * Every call returns 0 on success and a negative T3NS_E* code on failure;
 * t3ns_last_error() gives the message of the last failure on this thread.
 * No call falls back to a CPU implementation.
 */
#ifndef T3NS_B200_H
#define T3NS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define T3NS_OK 0
#define T3NS_E_ARG -1      /* invalid argument / inconsistent schedule       */
#define T3NS_E_CUDA -2     /* a CUDA runtime call failed                     */
#define T3NS_E_NOMEM -3    /* device or host allocation failed               */
#define T3NS_E_LIMIT -4    /* a size beyond what the kernels support         */
#define T3NS_E_DEVICE -5   /* the kernel reported an error status            */
#define T3NS_E_EIG -6      /* the subspace eigensolver did not converge      */

/* Matvec arithmetic.  FP64 computes every product and sum in double.
 * The split modes run the block contractions on the tensor cores as three
 * products of {hi, lo} operand pairs with FP32 accumulation; results stay
 * double in HBM.  3xTF32: TF32 pairs (about 2^-22 relative per product, every
 * kernel configuration).  BF16x3: BF16 pairs, half the operand bytes (about
 * 2^-16 relative per product, configurations 0-2). */
#define T3NS_PREC_FP64 0
#define T3NS_PREC_3XTF32 1
#define T3NS_PREC_BF16X3 2

/* One renormalised-operator set (reference struct rOperators,
 * include/rOperators.h:91-123), flattened.  Operator k has op_nblocks[k]
 * symmetry blocks whose element offsets are op_beginblock[k][0..nblocks]
 * (exactly the reference's sparseblocks.beginblock) into op_tel[k]. */
typedef struct {
        int nrops;
        const int *op_nblocks;              /* [nrops]                        */
        const int *const *op_beginblock;    /* [nrops] -> [op_nblocks[k] + 1] */
        const double *const *op_tel;        /* [nrops] -> host elements       */
} t3ns_ropset;

/* The matvec schedule of one optimisation step.  It carries the same
 * information as the reference's replay schedule (struct secondrun,
 * include/Heff.h:36-51): for every new (output) block, the old blocks it
 * couples to, and per (new, old) pair the MPO combinations with their
 * operator symmetry blocks and symmetry prefactor; the merge instruction set
 * (include/instructions.h:39-66) then supplies, per MPO combination, the
 * operator triples and instruction prefactors. */
typedef struct {
        int isdmrg;                  /* 1: two operators (DMRG-type step)      */
        int map[3];                  /* memory axis j <- operator map[j]       */
        int nblocks;                 /* symmetry blocks of the site tensor     */
        const int64_t *block_off;    /* [nblocks + 1] element offsets          */
        const int *dims;             /* [nblocks * 3] leg dim per operator     */
        const int *pair_ptr;         /* [nblocks + 1] CSR over new blocks      */
        const int *pair_old;         /* [npairs] old block of each pair        */
        const int *pair_order;       /* [npairs] contraction order (0..5)      */
        const int64_t *combo_ptr;    /* [npairs + 1] CSR over pairs            */
        const int *combo_mpo;        /* [ncombos] index into MPOc_beg          */
        const int *combo_sbops;      /* [ncombos * 3] operator symmetry blocks */
        const double *combo_pref;    /* [ncombos] symmetry prefactor           */
        int nr_instr;
        const int *instr;            /* [nr_instr * 3] operator indices        */
        const double *instr_pref;    /* [nr_instr]                             */
        int nrMPOc;
        const int *MPOc_beg;         /* [nrMPOc + 1]                           */
        t3ns_ropset ops[3];          /* ops[2] unused when isdmrg              */
} t3ns_heff_desc;

typedef struct t3ns_heff t3ns_heff;

/* Statistics of a plan (host-side figures, computed once at creation). */
typedef struct {
        int64_t size;            /* elements of the site tensor (vector length) */
        int64_t nblocks;
        int64_t npairs;          /* (new, old) block pairs                      */
        int64_t ntasks;          /* (pair, instruction) terms with all operator */
                                 /* blocks present                              */
        double flops_ref;        /* algorithmic FLOPs per matvec, reference     */
                                 /* contraction order (see DESIGN)              */
        double flops_exec;       /* FLOPs the kernels execute per matvec        */
        double bytes_alg;        /* algorithmic bytes: Psi in/out + distinct    */
                                 /* operator blocks, each once                  */
        int64_t op_elems;        /* operator elements resident on the device    */
        int64_t scratch_bytes;   /* device scratch held by the plan             */
} t3ns_heff_stats;

/* Replaces the schedule build of init_Heffdata + exec_firstrun
 * (reference src/Heff.c:1167-1221, 1002-1047): uploads the operator blocks
 * and the flattened task list to device memory on the current device. */
int t3ns_heff_create(const t3ns_heff_desc *desc, int precision, t3ns_heff **out);

/* y = Heff x with x, y device pointers of t3ns_heff_stats.size doubles,
 * launched on `stream` (a cudaStream_t, NULL = legacy default stream).
 * Replaces exec_secondrun (reference src/Heff.c:945-1000). */
int t3ns_heff_matvec_device(t3ns_heff *h, const double *x, double *y, void *stream);

/* The same product dispatched block by block: one launch of the matvec
 * kernel per output block, over that block's work units (FP64; the grouped
 * single launch above is the engine's path).  For measuring what one
 * persistent grouped launch saves over per-block dispatch, the way the
 * reference's loop over new blocks in exec_secondrun (src/Heff.c:945-1000)
 * would map to the GPU. */
int t3ns_heff_matvec_device_per_block(t3ns_heff *h, const double *x, double *y, void *stream);

/* Same with host buffers: x is copied to the device, y back to the host.
 * Synchronises and returns T3NS_E_DEVICE if the kernel reported an error. */
int t3ns_heff_matvec_host(t3ns_heff *h, const double *x, double *y);

/* Error status of the matvecs enqueued so far on `stream`: waits for the
 * stream, returns T3NS_E_DEVICE (and clears the status) if a matvec kernel
 * reported an error, else T3NS_OK.  t3ns_heff_matvec_device is asynchronous
 * and does not wait; callers of the device entry point check here (the
 * device Davidson checks after every iteration by itself). */
int t3ns_heff_check_status(t3ns_heff *h, void *stream);

/* Diagonal of Heff into a device (or host) buffer of size doubles.
 * Replaces make_diagonal (reference src/Heff.c:1268-1312). */
int t3ns_heff_diagonal_device(t3ns_heff *h, double *diag, void *stream);
int t3ns_heff_diagonal_host(t3ns_heff *h, double *diag);

/* Kernel configurations of the matvec: 0 = one 512-thread CTA per SM with
 * large shared-memory output tiles, 1 = two 256-thread CTAs per SM with small
 * tiles, 2 = one 768-thread CTA per SM (more warps, fewer registers a thread)
 * with mid-size tiles; 3 and 4 = the contraction-ordered kernel (every stage
 * contracts the fastest axis of its input, operators transposed on the
 * device) with 768 and 512 threads, FP64 and 3xTF32; 5, 6, 7 = the shapes of
 * 0, 1, 2 with buffers sized for BF16x3 (twice the elements in the same
 * shared memory), BF16x3 only.  Each has its own tiling of the plan (built on
 * first use).  Selecting a configuration that does not run the plan's
 * precision is an error (T3NS_E_ARG); switching the precision falls back to
 * configuration 0 when the active one does not run the new precision. */
#define T3NS_NUM_CONFIGS 8
int t3ns_heff_set_config(t3ns_heff *h, int config);
int t3ns_heff_get_config(const t3ns_heff *h);

/* Autotuner: times `reps` matvecs of every configuration on the plan's own
 * stream and buffers (after one untimed run each) and makes the fastest the
 * active one.  The choice is remembered for the plan's size bucket (powers of
 * two of the vector length, of the largest block and of the FLOP count), and
 * t3ns_heff_create starts every later plan of a known bucket on it; with
 * force == 0 a plan whose bucket is known is not re-timed.  ms_out, if not
 * NULL, receives the median time per configuration (0 when not timed). */
int t3ns_heff_autotune(t3ns_heff *h, int reps, int force, double *ms_out);

/* Switch the arithmetic of subsequent matvecs (T3NS_PREC_*). */
int t3ns_heff_set_precision(t3ns_heff *h, int precision);

int t3ns_heff_get_stats(const t3ns_heff *h, t3ns_heff_stats *st);

/* Launches of engine kernels issued by the last matvec call on this plan. */
int t3ns_heff_last_launches(const t3ns_heff *h);

void t3ns_heff_destroy(t3ns_heff *h);

/* Outcome of one Davidson solve. */
typedef struct {
        int iterations;          /* Davidson iterations (= matvecs issued)    */
        int max_vecs;            /* subspace size actually used                */
        double d_energy;         /* last energy change                         */
        double residual;         /* final residual norm                        */
        double seconds;          /* wall time of the solve                     */
        int fp64_iterations;     /* of those, iterations with an FP64 matvec   */
} t3ns_davidson_info;

/* Davidson for the lowest eigenpair, device resident (reference
 * src/davidson.c:259-328: same subspace bound, deflation, Olsen-corrected
 * diagonal preconditioner with cutoff 1e-12, and stopping rule).  With the
 * plan in T3NS_PREC_3XTF32 the solve runs its iterations on the
 * split-precision matvec until the residual reaches tol or, once below
 * 1e-4 * max(1, |energy|), stops improving; then it continues from that
 * vector with FP64 matvecs (defect correction) until the FP64 residual
 * reaches tol, so energy and residual are FP64 quantities.  `result`
 * holds the initial guess and receives the normalised eigenvector; `energy`
 * receives the Ritz value.  Returns 0 when converged, 1 when max_its was
 * reached, T3NS_E* on failure.  `info` may be NULL. */
int t3ns_davidson_host(t3ns_heff *h, double *result, double *energy,
                       int max_vecs, int keep_deflate, double tol, int max_its,
                       const double *diagonal, t3ns_davidson_info *info);

/* Same with device-resident guess/result and diagonal, on `stream`. */
int t3ns_davidson_device(t3ns_heff *h, double *result, double *energy,
                         int max_vecs, int keep_deflate, double tol, int max_its,
                         const double *diagonal, t3ns_davidson_info *info,
                         void *stream);

/* Davidson with a caller-supplied host matvec (any operator): the subspace
 * algebra runs on the device, each new basis vector is handed to
 * `matvec(in, out, ctx)` in host memory.  Same algorithm and return codes as
 * t3ns_davidson_host. */
int t3ns_davidson_callback(int64_t size, void (*matvec)(const double *, double *, void *),
                           void *ctx, double *result, double *energy, int max_vecs,
                           int keep_deflate, double tol, int max_its,
                           const double *diagonal, t3ns_davidson_info *info);

/* The diagonal preconditioner with Olsen correction on host buffers
 * (reference davidson_diagonal_preconditioner, src/davidson.c:223-257). */
int t3ns_precondition_host(int64_t size, const double *result, double theta,
                           const double *diagonal, double *vec_t);

/* Update of a physical renormalised-operator set through its site tensor
 * (reference update_rOperators_physical, src/rOperators_pUpdate.c:364-387,
 * pUpdate_block :323-362), flattened.  Every entry couples one updated
 * operator block (a "unit" groups the entries with the same updated block)
 * to one original block through the site-tensor block T and its adjoint
 * block Ta:
 *   left  (is_left):  U_i += pref * Ta^T O_i T   (O_i: M0 x M1, T: M1 x N1,
 *                                                 Ta: M0 x N0, U_i: N0 x N1)
 *   right:            U_i += pref * Ta O_i T^T   (T: N1 x M1, Ta: N0 x M0)
 * for every operator i of the entry's MPO sector whose two blocks are
 * present (op pair list).  Offsets index the site-tensor elements, the
 * concatenation of the original operators' elements, and the concatenation
 * of the updated operators' elements. */
typedef struct {
        int is_left;
        int nunits;
        const int *unit_ptr;        /* [nunits + 1] CSR into entries          */
        int nentries;
        const int *dims;            /* [nentries * 4]: M0, M1, N0, N1         */
        const int64_t *t_off;       /* [nentries] T block                     */
        const int64_t *ta_off;      /* [nentries] adjoint block               */
        const double *pref;         /* [nentries] symmetry prefactor          */
        const int *op_ptr;          /* [nentries + 1] CSR into op pairs       */
        const int64_t *old_off;     /* [npairs] original operator block       */
        const int64_t *new_off;     /* [npairs] updated operator block        */
        int64_t t_elems, old_elems, new_elems;
} t3ns_pupdate_desc;

/* Runs a physical update on host buffers: new_tel (new_elems doubles) is
 * overwritten with the updated operators' elements. */
int t3ns_pupdate_host(const t3ns_pupdate_desc *d, const double *t_tel, const double *old_tel,
                      double *new_tel);

/* Scaled block copies: dst[dst_off[e] + j] = scale[e] * src[src_off[e] + j]
 * for j < len[e]; every other element of dst is zero.  This is the
 * arithmetic of appending a site operator to a renormalised-operator set
 * (reference rOperators_append_phys / pAppend_block,
 * src/rOperators_pUpdate.c:537-640, 665-673). */
typedef struct {
        int nentries;
        const int64_t *dst_off;
        const int64_t *src_off;
        const int *len;
        const double *scale;
        int64_t src_elems, dst_elems;
} t3ns_scalecopy_desc;

int t3ns_scalecopy_host(const t3ns_scalecopy_desc *d, const double *src, double *dst);

/* Update through a branching tensor (reference update_rOperators_branching,
 * src/rOperators_bUpdate.c:229-248, update_selected_blocks :1043-1072),
 * flattened.  An entry couples one block of each input operator set
 * (O1 on memory axis ax[0] of the site tensor, O2 on axis ax[1]), the
 * site-tensor block T (ket indices, dims kd[3]) and the block Ta at the bra
 * indices (dims bd[3]); for each op triple of the entry
 *   New(b_g, k_g) += pref * sum Ta(b) O1(b_a, k_a) O2(b_b, k_b) T(k)
 * summing over the bra and ket indices of axes ax[0], ax[1] (g = ax[2]).
 * Operator blocks are (bra x ket) column-major.  Units group the entries of
 * one new block and run concurrently, so the new blocks a unit writes must
 * not be written by any other unit; new_tel is overwritten (zero + sums). */
typedef struct {
        int ax[3];
        int nunits;
        const int *unit_ptr;        /* [nunits + 1] CSR into entries           */
        int nentries;
        const int *dims;            /* [nentries * 6]: kd[0..2], bd[0..2]      */
        const int64_t *t_off;       /* [nentries] T block (ket indices)        */
        const int64_t *ta_off;      /* [nentries] T block at the bra indices   */
        const double *pref;         /* [nentries]                              */
        const int *op_ptr;          /* [nentries + 1] CSR into op triples      */
        const int64_t *o1_off, *o2_off, *new_off;   /* [ntriples]              */
        int64_t t_elems, o1_elems, o2_elems, new_elems;
} t3ns_bupdate_desc;

int t3ns_bupdate_host(const t3ns_bupdate_desc *d, const double *t_tel, const double *o1_tel,
                      const double *o2_tel, double *new_tel);

/* Sum of unique renormalised operators into a new set, then removal of the
 * blocks whose elements are all below 1e-20 in magnitude (reference
 * sum_unique_rOperators, src/rOperators_init.c:228-265, with
 * kick_zero_blocks, src/sparseblocks.c:73-107).  New operator k gets, for
 * each instruction writing it (in instruction order), pref times the unique
 * operator at element offset instr_src; its block layout before removal is
 * begin[begin_ptr[k] .. begin_ptr[k+1]) (starting at 0, the last entry its
 * size) and its elements sit at new_base[k] in the unsummed layout
 * (new_base[k+1] - new_base[k] = its size). */
typedef struct {
        int nnew;
        const int64_t *begin_ptr;   /* [nnew + 1] into begin                  */
        const int *begin;           /* block begin offsets before removal     */
        const int64_t *new_base;    /* [nnew + 1]                             */
        const int *instr_ptr;       /* [nnew + 1] CSR into the instructions   */
        const int64_t *instr_src;   /* [ninstr] unique operator element base  */
        const double *instr_pref;   /* [ninstr]                               */
        int64_t unique_elems;       /* size of unique_tel (standalone call)   */
} t3ns_sumunique_desc;

/* Outputs of the sums: new_tel (new_base[nnew] doubles at most) receives the
 * kept blocks of every new operator back to back, operator k from
 * out_base[k] (out_base has nnew + 1 entries); new_begin (shaped like
 * begin) the block begin offsets after removal.  Host arrays. */
int t3ns_sum_unique_host(const t3ns_sumunique_desc *s, const double *unique_tel, double *new_tel,
                         int *new_begin, int64_t *out_base);

/* The site-operator append (t3ns_scalecopy_host) and the branching update
 * (t3ns_bupdate_host) followed by the sum on the device: the unique
 * operators never leave the GPU, only the summed set is downloaded
 * (reference rOperators_append_phys, src/rOperators_pUpdate.c:665-673, and
 * update_rOperators_branching, src/rOperators_bUpdate.c:229-248, which end
 * in sum_unique_rOperators). */
int t3ns_scalecopy_sum_host(const t3ns_scalecopy_desc *d, const t3ns_sumunique_desc *s,
                            const double *src, double *new_tel, int *new_begin, int64_t *out_base);
int t3ns_bupdate_sum_host(const t3ns_bupdate_desc *d, const t3ns_sumunique_desc *s,
                          const double *t_tel, const double *o1_tel, const double *o2_tel,
                          double *new_tel, int *new_begin, int64_t *out_base);

/* Dense FP64 factorisations of one symmetry sector of the site-tensor
 * decomposition, on host column-major arrays, with LAPACK's argument
 * meaning.  They replace the reference's LAPACKE_dgesdd ('S' and 'N'),
 * LAPACKE_dgeqrf and LAPACKE_dorgqr calls (src/siteTensor_decompose.c:1060,
 * :565, :285, :295).  Safe to call from several host threads at once (each
 * thread has its own stream).  t3ns_gesdd_host returns T3NS_E_EIG when the
 * Jacobi sweeps do not converge; singular values come out descending, and
 * singular vectors are unique up to sign (and rotation within a degenerate
 * singular value), as LAPACK's are. */
int t3ns_gesdd_host(char jobz, int m, int n, const double *a, int lda, double *s, double *u,
                    int ldu, double *vt, int ldvt);
int t3ns_geqrf_host(int m, int n, double *a, int lda, double *tau);
int t3ns_orgqr_host(int m, int n, int k, double *a, int lda, const double *tau);

/* Request loop for independent ground-state solves (no counterpart in the
 * reference, whose driver runs one solve per process).  A request is one
 * Davidson solve of an effective Hamiltonian, with the arguments of
 * t3ns_davidson_host.  Requests are admitted in arrival order against a
 * fixed device-memory budget (the first queued request that fits what the
 * running ones leave free); up to max_inflight run at once, each on its own
 * stream, so their work overlaps on the GPU.  A request whose estimated
 * footprint exceeds the whole budget is rejected by submit (T3NS_E_LIMIT).
 * The descriptor, guess/result and diagonal must stay valid until the
 * request has been waited for; the result is written into guess_and_result. */
typedef struct t3ns_server t3ns_server;
typedef struct {
        int64_t id;
        int status;              /* the solve's return code (0, 1 or T3NS_E_*) */
        double energy;
        t3ns_davidson_info info;
        int64_t bytes;           /* admitted footprint (estimate)             */
        double queue_seconds;    /* submit -> admission                       */
        double run_seconds;      /* admission -> result                       */
        double latency_seconds;  /* submit -> result                          */
} t3ns_request_result;

int t3ns_server_create(int64_t budget_bytes, int max_inflight, t3ns_server **out);
int t3ns_server_submit(t3ns_server *s, const t3ns_heff_desc *desc, int precision,
                       double *guess_and_result, const double *diagonal, double tol, int max_its,
                       int max_vecs, int keep, int64_t *id_out);
/* Blocks until request `id` has finished; returns its status. */
int t3ns_server_wait(t3ns_server *s, int64_t id, t3ns_request_result *out);
/* Device bytes admitted now, the peak so far, and requests waiting. */
int t3ns_server_stats(t3ns_server *s, int64_t *in_use, int64_t *peak, int *queued);
/* Finishes queued and running requests, then frees the server. */
void t3ns_server_destroy(t3ns_server *s);
/* The footprint estimate admission uses (host only, no GPU needed). */
int64_t t3ns_server_estimate_bytes(const t3ns_heff_desc *desc, int precision, int max_vecs);

/* Largest vector t3ns_precondition_device_noalloc accepts (elements). */
#define T3NS_NOALLOC_MAX_SIZE 16777216LL

/* Allocation-free diagonal preconditioner (no counterpart in the reference;
 * same arithmetic as t3ns_precondition_host).  For callers that cannot
 * allocate device memory when they need it -- a memory pool or arena that
 * owns the whole GPU, code that must not trigger the implicit device
 * synchronisation of cudaMalloc/cudaFree, drivers that forbid allocation
 * after start-up.  `result`, `diagonal` and `vec_t` are device buffers of
 * `size` doubles supplied by the caller; vec_t is updated in place on
 * `stream` (a cudaStream_t).  The reduction scratch is a fixed array inside
 * the library (about 1 MiB, held by every GPU that loads the library until
 * exit), so size must not exceed T3NS_NOALLOC_MAX_SIZE (T3NS_E_LIMIT
 * otherwise).  It calls no allocator.  The first call on a device looks up
 * the scratch address and should come before any stream capture.  All calls
 * share the scratch: calls that overlap on the GPU race and must be
 * serialised by the caller. */
int t3ns_precondition_device_noalloc(int64_t size, const double *result, double theta,
                                     const double *diagonal, double *vec_t, void *stream);

/* Diagnostic: builds the host-side plan of `desc` (no GPU needed) and writes
 * its work units, pair sequences and flattened terms to `path` (step-file
 * record layout), for host-side checks of the tiling and ordering. */
int t3ns_heff_plan_dump(const t3ns_heff_desc *desc, const char *path);
/* The same for kernel configuration `config` (0 .. T3NS_NUM_CONFIGS-1);
 * t3ns_heff_plan_dump writes configuration 0. */
int t3ns_heff_plan_dump_config(const t3ns_heff_desc *desc, int config, const char *path);

const char *t3ns_last_error(void);

/* Library build identification (git-independent). */
const char *t3ns_version(void);

#ifdef __cplusplus
}
#endif

#endif /* T3NS_B200_H */
