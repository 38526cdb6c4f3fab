/* t3ns_run: command-line driver for the reference T3NS sweep, used by the
 * tests as (a) the CPU oracle, when linked against the whole reference
 * library, and (b) the unchanged host driver of the drop-in, when linked
 * against the reference minus Heff/davidson/wrapper_solvers plus the product
 * library.  Test infrastructure only.
 *
 * It follows the reference's own test driver (tests/test1.c.in:31-54):
 * set bookie.sgs/target_state, make_network, readinteraction,
 * preparebookkeeper, init_calculation, execute_optScheme.
 *
 * Capture mode (oracle build only, --capture DIR): this executable defines
 * sparse_eigensolve, which interposes the reference's own
 * (src/wrapper_solvers.c:107-128) for the call in optimize_siteTensor
 * (src/optimize_network.c:217-221).  For every selected step it writes the
 * complete Heffdata inputs (site tensor structure, symsecs, the three
 * rOperators, the merge instruction set), the reference's replay schedule
 * (struct secondrun, include/Heff.h:36-51, filled by exec_firstrun,
 * src/Heff.c:1002-1047), the reference diagonal (make_diagonal) and
 * reference matvec outputs for seeded vectors, then the Davidson result of
 * the reference on the step, into DIR/step_NNN.t3c.
 */
#define _GNU_SOURCE
#include <dlfcn.h>
#include <pthread.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include "Heff.h"
#include "bookkeeper.h"
#include "davidson.h"
#include "hamiltonian.h"
#include "instructions.h"
#include "macros.h"
#include "network.h"
#include "optScheme.h"
#include "optimize_network.h"
#include "options.h"
#include "symmetries.h"

/* ------------------------------------------------------------------ */
/* capture file: "T3NSCAP1", then records {char name[48]; int32 dtype;
 * int32 pad; int64 count; payload}. dtype: 1=int32 2=int64 3=float64.   */

static FILE *cap_fp;

static void cap_put_f(FILE *f, const char *name, int dtype, int64_t count, const void *data)
{
        char nm[48] = {0};
        strncpy(nm, name, sizeof nm - 1);
        int32_t hdr[2] = {dtype, 0};
        fwrite(nm, 1, sizeof nm, f);
        fwrite(hdr, sizeof hdr, 1, f);
        fwrite(&count, sizeof count, 1, f);
        const size_t el = dtype == 1 ? 4 : 8;
        if (count > 0) fwrite(data, el, (size_t) count, f);
}

static void cap_put(const char *name, int dtype, int64_t count, const void *data)
{
        cap_put_f(cap_fp, name, dtype, count, data);
}

static void cap_i32(const char *name, int64_t n, const int *d) { cap_put(name, 1, n, d); }
static void cap_i64(const char *name, int64_t n, const int64_t *d) { cap_put(name, 2, n, d); }
static void cap_f64(const char *name, int64_t n, const double *d) { cap_put(name, 3, n, d); }
static void cap_int(const char *name, int v) { cap_i32(name, 1, &v); }
static void cap_dbl(const char *name, double v) { cap_f64(name, 1, &v); }

/* ------------------------------------------------------------------ */
/* options                                                              */

static const char *opt_capture_dir;
static long opt_capture_max = 2000000;   /* largest Psi captured        */
static long opt_capture_min = 0;         /* smallest Psi captured       */
static int opt_capture_limit = 1000000;  /* number of captures          */
static int opt_capture_stop;             /* exit after the last capture */
static int opt_capture_nvec = 2;         /* seeded matvec pairs         */
static int opt_capture_noeig;            /* skip Davidson in capture    */
static const char *opt_schedule_lib;     /* drop-in whose schedule to dump */
static const char *opt_capture_pupdate;  /* dir for physical-update captures */
static const char *opt_capture_dense;    /* dir for dense LAPACK call captures */
static int opt_dense_limit = 400;
static int opt_pupdate_limit = 4;
static int opt_pupdate_count;
static int opt_step_counter;
static int opt_captured;

static uint64_t splitmix(uint64_t *s)
{
        uint64_t z = (*s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
}

/* normalised vector with N(0,1) entries (Box-Muller on splitmix64) */
static void seeded_vector(double *v, int n, uint64_t seed)
{
        uint64_t s = seed;
        double nrm = 0;
        for (int i = 0; i < n; i += 2) {
                double u1 = ((splitmix(&s) >> 11) + 0.5) * 0x1.0p-53;
                double u2 = ((splitmix(&s) >> 11) + 0.5) * 0x1.0p-53;
                double r = sqrt(-2 * log(u1));
                v[i] = r * cos(2 * M_PI * u2);
                if (i + 1 < n) v[i + 1] = r * sin(2 * M_PI * u2);
        }
        for (int i = 0; i < n; ++i) nrm += v[i] * v[i];
        nrm = 1 / sqrt(nrm);
        for (int i = 0; i < n; ++i) v[i] *= nrm;
}

static void dump_symsecs(const char *pre, const struct symsecs *ss)
{
        char nm[64];
        snprintf(nm, sizeof nm, "%s.nrSecs", pre);
        cap_int(nm, ss->nrSecs);
        snprintf(nm, sizeof nm, "%s.irreps", pre);
        cap_i32(nm, (int64_t) ss->nrSecs * MAX_SYMMETRIES, (const int *) ss->irreps);
        snprintf(nm, sizeof nm, "%s.dims", pre);
        if (ss->dims) cap_i32(nm, ss->nrSecs, ss->dims);
}

static int opt_structure_only;          /* dump operator lengths, not values */

static void dump_rops(int i, const struct rOperators *op)
{
        char nm[64];
#define NM(x) (snprintf(nm, sizeof nm, "ops%d." x, i), nm)
        cap_int(NM("bond"), op->bond);
        cap_int(NM("is_left"), op->is_left);
        cap_int(NM("P_operator"), op->P_operator);
        cap_int(NM("nrhss"), op->nrhss);
        cap_int(NM("nrops"), op->nrops);
        if (op->nrops == 0) return;
        cap_i32(NM("begin_blocks_of_hss"), op->nrhss + 1, op->begin_blocks_of_hss);
        const int nqn = op->P_operator ? 3 : 1;
        cap_i64(NM("qnumbers"), (int64_t) op->begin_blocks_of_hss[op->nrhss] * nqn,
                (const int64_t *) op->qnumbers);
        cap_i32(NM("hss_of_ops"), op->nrops, op->hss_of_ops);
        /* per operator: beginblock (nblocks of its hss + 1) and tel, concatenated */
        int64_t nbb = 0, ntel = 0;
        for (int k = 0; k < op->nrops; ++k) {
                const int nb = rOperators_give_nr_blocks_for_hss(op, op->hss_of_ops[k]);
                nbb += nb + 1;
                ntel += op->operators[k].beginblock[nb];
        }
        int *bb = malloc(sizeof *bb * (size_t) nbb);
        double *tel = malloc(sizeof *tel * (size_t) (ntel ? ntel : 1));
        int64_t pb = 0, pt = 0;
        for (int k = 0; k < op->nrops; ++k) {
                const int nb = rOperators_give_nr_blocks_for_hss(op, op->hss_of_ops[k]);
                memcpy(bb + pb, op->operators[k].beginblock, sizeof *bb * (size_t) (nb + 1));
                const int sz = op->operators[k].beginblock[nb];
                if (sz) memcpy(tel + pt, op->operators[k].tel, sizeof *tel * (size_t) sz);
                pb += nb + 1;
                pt += sz;
        }
        cap_i32(NM("beginblock"), nbb, bb);
        if (opt_structure_only) {
                const int64_t len = ntel;
                cap_i64(NM("tel_len"), 1, &len);
        } else {
                cap_f64(NM("tel"), ntel, tel);
        }
        free(bb);
        free(tel);
#undef NM
}

static double now_s(void)
{
        struct timeval t;
        gettimeofday(&t, NULL);
        return t.tv_sec + 1e-6 * t.tv_usec;
}

typedef int (*eig_fn)(double *, double *, int, int, int, double, int,
                      const double *, void (*)(const double *, double *, void *),
                      void *, const char *);

static int capture_step(struct Heffdata *hd, double *guess, int size,
                        const double *diagonal, int max_vecs, int keep, double tol,
                        int max_its, eig_fn real_eig,
                        void (*matvec)(const double *, double *, void *),
                        double *energy_out)
{
        int ret = 0;
        *energy_out = 0;
        char path[4096];
        snprintf(path, sizeof path, "%s/step_%03d.t3c", opt_capture_dir, opt_step_counter);
        cap_fp = fopen(path, "wb");
        if (!cap_fp) { perror(path); exit(EXIT_FAILURE); }
        fwrite("T3NSCAP1", 1, 8, cap_fp);

        const struct siteTensor *st = &hd->siteObject;
        cap_int("step", opt_step_counter);
        cap_int("isdmrg", hd->isdmrg);
        cap_int("nrsites", st->nrsites);
        cap_i32("sites", st->nrsites, st->sites);
        cap_int("posB", hd->posB);
        cap_i32("rOperators_on_site", 3, hd->rOperators_on_site);
        cap_int("nrblocks", st->nrblocks);
        cap_i64("qnumbers", (int64_t) st->nrblocks * st->nrsites, (const int64_t *) st->qnumbers);
        cap_i32("beginblock", st->nrblocks + 1, st->blocks.beginblock);
        cap_int("nrSyms", bookie.nrSyms);
        cap_i32("sgs", bookie.nrSyms, (const int *) bookie.sgs);
        cap_int("MAX_SYMMETRIES", MAX_SYMMETRIES);
        char nm[64];
        for (int i = 0; i < st->nrsites; ++i)
                for (int j = 0; j < 3; ++j) {
                        snprintf(nm, sizeof nm, "symarr%d%d", i, j);
                        dump_symsecs(nm, &hd->symarr[i][j]);
                }
        dump_symsecs("MPOsymsec", &hd->MPOsymsec);
        for (int i = 0; i < (hd->isdmrg ? 2 : 3); ++i) dump_rops(i, &hd->Operators[i]);

        const struct instructionset *is = &hd->iset;
        cap_int("iset.nr_instr", is->nr_instr);
        cap_int("iset.step", is->step);
        {
                int *ins = malloc(sizeof *ins * 3 * (size_t) (is->nr_instr + 1));
                double *pr = malloc(sizeof *pr * (size_t) (is->nr_instr + 1));
                for (int k = 0; k < is->nr_instr; ++k) {
                        for (int c = 0; c < 3; ++c) ins[3 * k + c] = is->instr[k].instr[c];
                        pr[k] = is->instr[k].pref;
                }
                cap_i32("iset.instr", 3L * is->nr_instr, ins);
                cap_f64("iset.pref", is->nr_instr, pr);
                free(ins);
                free(pr);
        }
        cap_int("iset.nrMPOc", is->nrMPOc);
        cap_i32("iset.MPOc", is->nrMPOc, is->MPOc);
        cap_i32("iset.MPOc_beg", is->nrMPOc + 1, is->MPOc_beg);

        /* reference diagonal */
        cap_f64("diag", size, diagonal);

        /* reference matvecs: first run builds the replay schedule */
        double *x = malloc(sizeof *x * (size_t) size);
        double *y = malloc(sizeof *y * (size_t) size);
        double t_first = 0, t_second = 1e300;
        for (int v = 0; v < opt_capture_nvec; ++v) {
                seeded_vector(x, size, 1000003ull * (uint64_t) opt_step_counter + (uint64_t) v);
                double t0 = now_s();
                matvec(x, y, hd);
                double t1 = now_s();
                if (v == 0) t_first = t1 - t0;
                else if (t1 - t0 < t_second) t_second = t1 - t0;
                snprintf(nm, sizeof nm, "x%d", v);
                cap_f64(nm, size, x);
                snprintf(nm, sizeof nm, "y%d", v);
                cap_f64(nm, size, y);
        }
        cap_dbl("ref_matvec_first_s", t_first);
        cap_dbl("ref_matvec_second_s", t_second);

        /* replay schedule (struct secondrun) */
        const struct secondrun *sr = &hd->sr;
        const int n = st->nrblocks;
        int64_t npair = 0, ncombo = 0;
        for (int i = 0; i < n; ++i) {
                npair += sr->nr_oldsb[i];
                for (int j = 0; j < sr->nr_oldsb[i]; ++j) ncombo += sr->ntom[i][j].nmbr;
        }
        int *dims = malloc(sizeof *dims * 3 * (size_t) n);
        int *pair_ptr = malloc(sizeof *pair_ptr * (size_t) (n + 1));
        int *pair_old = malloc(sizeof *pair_old * (size_t) (npair + 1));
        int *pair_order = malloc(sizeof *pair_order * (size_t) (npair + 1));
        int64_t *combo_ptr = malloc(sizeof *combo_ptr * (size_t) (npair + 1));
        int *combo_sbops = malloc(sizeof *combo_sbops * 3 * (size_t) (ncombo + 1));
        int *combo_mpo = malloc(sizeof *combo_mpo * (size_t) (ncombo + 1));
        double *combo_pref = malloc(sizeof *combo_pref * (size_t) (ncombo + 1));
        int64_t p = 0, c = 0;
        for (int i = 0; i < n; ++i) {
                for (int k = 0; k < 3; ++k) dims[3 * i + k] = sr->dimsofsb[i][k];
                pair_ptr[i] = (int) p;
                for (int j = 0; j < sr->nr_oldsb[i]; ++j, ++p) {
                        const struct newtooldmatvec *t = &sr->ntom[i][j];
                        pair_old[p] = t->oldsb;
                        pair_order[p] = t->bestorder;
                        combo_ptr[p] = c;
                        for (int k = 0; k < t->nmbr; ++k, ++c) {
                                for (int q = 0; q < 3; ++q)
                                        combo_sbops[3 * c + q] = t->sbops[k][q];
                                combo_mpo[c] = t->MPO[k];
                                combo_pref[c] = t->prefactor[k];
                        }
                }
        }
        pair_ptr[n] = (int) p;
        combo_ptr[p] = c;
        cap_i32("sr.dims", 3L * n, dims);
        cap_i32("sr.pair_ptr", n + 1, pair_ptr);
        cap_i32("sr.pair_old", npair, pair_old);
        cap_i32("sr.pair_order", npair, pair_order);
        cap_i64("sr.combo_ptr", npair + 1, combo_ptr);
        cap_i32("sr.combo_sbops", 3 * ncombo, combo_sbops);
        cap_i32("sr.combo_mpo", ncombo, combo_mpo);
        cap_f64("sr.combo_pref", ncombo, combo_pref);
        cap_i32("sr.worksize", 2, sr->worksize);
        free(dims); free(pair_ptr); free(pair_old); free(pair_order);
        free(combo_ptr); free(combo_sbops); free(combo_mpo); free(combo_pref);

        /* the reference Davidson on this step, from the driver's guess */
        if (!opt_capture_noeig) {
                cap_f64("eig.guess", size, guess);
                double energy = 0;
                double t0 = now_s();
                ret = real_eig(guess, &energy, size, max_vecs, keep, tol, max_its,
                                   diagonal, matvec, hd, "D");
                double t1 = now_s();
                cap_int("eig.ret", ret);
                cap_dbl("eig.energy", energy);
                cap_dbl("eig.tol", tol);
                cap_int("eig.max_its", max_its);
                cap_int("eig.max_vecs", max_vecs);
                cap_int("eig.keep", keep);
                cap_dbl("eig.seconds", t1 - t0);
                cap_f64("eig.result", size, guess);
                *energy_out = energy;
        }
        free(x);
        free(y);
        fclose(cap_fp);
        cap_fp = NULL;
        if (opt_schedule_lib) {
                /* the product's schedule compiler on the same Heffdata, loaded
                 * privately so it does not replace the reference symbols */
                static int (*wr)(const struct Heffdata *, const char *);
                if (!wr) {
                        void *h = dlopen(opt_schedule_lib, RTLD_NOW | RTLD_LOCAL);
                        if (!h) { fprintf(stderr, "%s\n", dlerror()); exit(EXIT_FAILURE); }
                        wr = (int (*)(const struct Heffdata *, const char *))
                                dlsym(h, "t3ns_dropin_schedule_write");
                        if (!wr) { fprintf(stderr, "no t3ns_dropin_schedule_write\n"); exit(EXIT_FAILURE); }
                }
                char sp[4096];
                snprintf(sp, sizeof sp, "%s/step_%03d.sched", opt_capture_dir, opt_step_counter);
                if (wr(hd, sp) != 0) { fprintf(stderr, "schedule write failed\n"); exit(EXIT_FAILURE); }
        }
        ++opt_captured;
        fprintf(stdout, "CAPTURED %s size %d blocks %d\n", path, size, st->nrblocks);
        fflush(stdout);
        return ret;
}

/* --capture-structure DIR (either build): for every selected step, the step's
 * structure only -- site tensor blocks, symsecs, the operator sets' block
 * structure with their element counts (ops{i}.tel_len) instead of values,
 * the merge instruction set -- to DIR/step_NNN.t3c, and the schedule the
 * product's compiler builds for it (bit-identical to the reference's replay
 * schedule, which the drop-in tests check pair by pair) to
 * DIR/step_NNN.sched; the Davidson solve is skipped (the step keeps the
 * driver's guess).  The benchmark workloads are made from these pairs
 * (oracle/captures.py): in the drop-in build the initial operators and the
 * updates run on the GPU, which makes large bond dimensions reachable. */
static const char *opt_capture_structure;

static void capture_structure(const struct Heffdata *hd, int size)
{
        char path[4096];
        snprintf(path, sizeof path, "%s/step_%03d.t3c", opt_capture_structure, opt_step_counter);
        cap_fp = fopen(path, "wb");
        if (!cap_fp) { perror(path); exit(EXIT_FAILURE); }
        fwrite("T3NSCAP1", 1, 8, cap_fp);
        const struct siteTensor *st = &hd->siteObject;
        cap_int("step", opt_step_counter);
        cap_int("isdmrg", hd->isdmrg);
        cap_int("nrsites", st->nrsites);
        cap_i32("sites", st->nrsites, st->sites);
        cap_int("posB", hd->posB);
        cap_i32("rOperators_on_site", 3, hd->rOperators_on_site);
        cap_int("nrblocks", st->nrblocks);
        cap_i64("qnumbers", (int64_t) st->nrblocks * st->nrsites, (const int64_t *) st->qnumbers);
        cap_i32("beginblock", st->nrblocks + 1, st->blocks.beginblock);
        cap_int("nrSyms", bookie.nrSyms);
        cap_i32("sgs", bookie.nrSyms, (const int *) bookie.sgs);
        cap_int("MAX_SYMMETRIES", MAX_SYMMETRIES);
        char nm[64];
        for (int i = 0; i < st->nrsites; ++i)
                for (int j = 0; j < 3; ++j) {
                        snprintf(nm, sizeof nm, "symarr%d%d", i, j);
                        dump_symsecs(nm, &hd->symarr[i][j]);
                }
        dump_symsecs("MPOsymsec", &hd->MPOsymsec);
        opt_structure_only = 1;
        for (int i = 0; i < (hd->isdmrg ? 2 : 3); ++i) dump_rops(i, &hd->Operators[i]);
        opt_structure_only = 0;
        const struct instructionset *is = &hd->iset;
        cap_int("iset.nr_instr", is->nr_instr);
        cap_int("iset.step", is->step);
        int *ins = malloc(sizeof *ins * 3 * (size_t) (is->nr_instr + 1));
        double *pr = malloc(sizeof *pr * (size_t) (is->nr_instr + 1));
        for (int k = 0; k < is->nr_instr; ++k) {
                for (int c = 0; c < 3; ++c) ins[3 * k + c] = is->instr[k].instr[c];
                pr[k] = is->instr[k].pref;
        }
        cap_i32("iset.instr", 3L * is->nr_instr, ins);
        cap_f64("iset.pref", is->nr_instr, pr);
        free(ins);
        free(pr);
        cap_int("iset.nrMPOc", is->nrMPOc);
        cap_i32("iset.MPOc", is->nrMPOc, is->MPOc);
        cap_i32("iset.MPOc_beg", is->nrMPOc + 1, is->MPOc_beg);
        fclose(cap_fp);
        cap_fp = NULL;

        static int (*wr)(const struct Heffdata *, const char *);
        if (!wr) {
                /* the drop-in build links the compiler; the oracle build loads
                 * it privately from --schedule-lib (RTLD_DEFAULT is a null
                 * handle, so the two cases are told apart by the option) */
                if (opt_schedule_lib) {
                        void *h = dlopen(opt_schedule_lib, RTLD_NOW | RTLD_LOCAL);
                        if (h) wr = (int (*)(const struct Heffdata *, const char *))
                                        dlsym(h, "t3ns_dropin_schedule_write");
                } else {
                        wr = (int (*)(const struct Heffdata *, const char *))
                                dlsym(RTLD_DEFAULT, "t3ns_dropin_schedule_write");
                }
                if (!wr) { fprintf(stderr, "no t3ns_dropin_schedule_write\n"); exit(EXIT_FAILURE); }
        }
        char sp[4096];
        snprintf(sp, sizeof sp, "%s/step_%03d.sched", opt_capture_structure, opt_step_counter);
        if (wr(hd, sp) != 0) { fprintf(stderr, "schedule write failed\n"); exit(EXIT_FAILURE); }
        ++opt_captured;
        fprintf(stdout, "CAPTURED_STRUCTURE %s size %d blocks %d\n", path, size, st->nrblocks);
        fflush(stdout);
}

#ifdef T3NS_RUN_DROPIN
/* In the drop-in build only the structure capture interposes the drop-in's
 * sparse_eigensolve. */
int sparse_eigensolve(double *result, double *energy, int size, int max_vecs,
                      int keep_deflate, double tol, int max_its,
                      const double *diagonal,
                      void (*matvec)(const double *, double *, void *),
                      void *vdat, const char solver[])
{
        static eig_fn real_eig;
        if (!real_eig) real_eig = (eig_fn) dlsym(RTLD_NEXT, "sparse_eigensolve");
        if (!real_eig) { fprintf(stderr, "sparse_eigensolve not found\n"); exit(EXIT_FAILURE); }
        int ret = 0;
        if (opt_capture_structure) {
                if (opt_captured < opt_capture_limit && size <= opt_capture_max &&
                    size >= opt_capture_min) {
                        capture_structure((const struct Heffdata *) vdat, size);
                        if (opt_capture_stop && opt_captured >= opt_capture_limit) {
                                printf("CAPTURE_DONE\n");
                                fflush(stdout);
                                _exit(0);
                        }
                }
                *energy = 0;
        } else {
                ret = real_eig(result, energy, size, max_vecs, keep_deflate, tol, max_its,
                               diagonal, matvec, vdat, solver);
        }
        ++opt_step_counter;
        return ret;
}
#endif

#ifndef T3NS_RUN_DROPIN
static void dump_siteTensor(const char *pre, const struct siteTensor *t)
{
        char nm[64];
        snprintf(nm, sizeof nm, "%s.nrsites", pre);
        cap_int(nm, t->nrsites);
        snprintf(nm, sizeof nm, "%s.sites", pre);
        cap_i32(nm, t->nrsites, t->sites);
        snprintf(nm, sizeof nm, "%s.nrblocks", pre);
        cap_int(nm, t->nrblocks);
        snprintf(nm, sizeof nm, "%s.qnumbers", pre);
        cap_i64(nm, (int64_t) t->nrblocks * t->nrsites, (const int64_t *) t->qnumbers);
        snprintf(nm, sizeof nm, "%s.beginblock", pre);
        cap_i32(nm, t->nrblocks + 1, t->blocks.beginblock);
        snprintf(nm, sizeof nm, "%s.tel", pre);
        cap_f64(nm, t->blocks.beginblock[t->nrblocks], t->blocks.tel);
}

/* Captures the reference's physical update: its inputs, the product's
 * compiled schedule for them (loaded privately from --schedule-lib), and the
 * reference's output.  Interposes the reference's update_rOperators_physical
 * (src/rOperators_pUpdate.c:364-387). */
typedef void (*pupd_fn)(struct rOperators *, const struct siteTensor *, const struct symsecs *);
void update_rOperators_physical(struct rOperators *rops, const struct siteTensor *tens,
                                const struct symsecs *internalss)
{
        static pupd_fn real;
        if (!real) real = (pupd_fn) dlsym(RTLD_NEXT, "update_rOperators_physical");
        const int want = opt_capture_pupdate && opt_pupdate_count < opt_pupdate_limit;
        char path[4096];
        if (want) {
                snprintf(path, sizeof path, "%s/pupdate_%03d.t3c", opt_capture_pupdate, opt_pupdate_count);
                cap_fp = fopen(path, "wb");
                if (!cap_fp) { perror(path); exit(EXIT_FAILURE); }
                fwrite("T3NSCAP1", 1, 8, cap_fp);
                dump_rops(0, rops);
                dump_siteTensor("T", tens);
                if (opt_schedule_lib) {
                        void *h = dlopen(opt_schedule_lib, RTLD_NOW | RTLD_LOCAL);
                        int (*wr)(const struct rOperators *, const struct siteTensor *,
                                  const struct symsecs *, const char *) =
                                h ? dlsym(h, "t3ns_dropin_pupdate_write") : NULL;
                        if (!wr) { fprintf(stderr, "no t3ns_dropin_pupdate_write\n"); exit(EXIT_FAILURE); }
                        char sp[4096];
                        snprintf(sp, sizeof sp, "%s/pupdate_%03d.sched", opt_capture_pupdate,
                                 opt_pupdate_count);
                        if (wr(rops, tens, internalss, sp) != 0) exit(EXIT_FAILURE);
                }
        }
        real(rops, tens, internalss);
        if (want) {
                dump_rops(1, rops);
                fclose(cap_fp);
                cap_fp = NULL;
                ++opt_pupdate_count;
        }
}

/* --check-dropin LIB: every rOperators_append_phys call of the sweep also
 * runs the drop-in's (LIB loaded privately, so its symbols do not replace
 * the reference's) on the same input, and the two new sets are compared:
 * "CHECK_APPEND <call> <diff>" with diff the largest element difference
 * relative to the largest reference element, or -1 when the block
 * structures differ (operator count, sectors, surviving blocks). */
static const char *opt_check_dropin;
static int opt_check_count;

static double compare_rops(const struct rOperators *a, const struct rOperators *b)
{
        if (a->nrops != b->nrops || a->nrhss != b->nrhss || a->bond != b->bond ||
            a->is_left != b->is_left || a->P_operator != b->P_operator)
                return -1;
        double scale = 0, worst = 0;
        for (int i = 0; i < a->nrops; ++i) {
                if (a->hss_of_ops[i] != b->hss_of_ops[i]) return -1;
                const int nb = nblocks_in_operator(a, i);
                for (int q = 0; q <= nb; ++q)
                        if (a->operators[i].beginblock[q] != b->operators[i].beginblock[q]) return -1;
                for (int j = 0; j < a->operators[i].beginblock[nb]; ++j) {
                        const double x = a->operators[i].tel[j], y = b->operators[i].tel[j];
                        if (fabs(x) > scale) scale = fabs(x);
                        if (fabs(x - y) > worst) worst = fabs(x - y);
                }
        }
        return scale > 0 ? worst / scale : worst;
}

typedef void (*append_fn)(struct rOperators *, const struct rOperators *);
void rOperators_append_phys(struct rOperators *newrops, const struct rOperators *oldrops)
{
        static append_fn real, mine;
        if (!real) real = (append_fn) dlsym(RTLD_NEXT, "rOperators_append_phys");
        real(newrops, oldrops);
        if (!opt_check_dropin) return;
        if (!mine) {
                void *h = dlopen(opt_check_dropin, RTLD_NOW | RTLD_LOCAL);
                if (!h) { fprintf(stderr, "%s\n", dlerror()); exit(EXIT_FAILURE); }
                mine = (append_fn) dlsym(h, "rOperators_append_phys");
                if (!mine) { fprintf(stderr, "no rOperators_append_phys in %s\n", opt_check_dropin); exit(EXIT_FAILURE); }
        }
        struct rOperators other;
        mine(&other, oldrops);
        printf("CHECK_APPEND %d %.3e\n", opt_check_count++, compare_rops(newrops, &other));
        destroy_rOperators(&other);
}

/* Captures the reference's branching update the same way: both input sets
 * (ops0, ops1), the branching tensor, the product's compiled schedule and the
 * reference's output (ops2).  Interposes update_rOperators_branching
 * (src/rOperators_bUpdate.c:229-248). */
typedef void (*bupd_fn)(struct rOperators *, const struct rOperators *, const struct siteTensor *);
static int opt_bupdate_count;
void update_rOperators_branching(struct rOperators *newops, const struct rOperators *Operator,
                                 const struct siteTensor *tens)
{
        static bupd_fn real;
        if (!real) real = (bupd_fn) dlsym(RTLD_NEXT, "update_rOperators_branching");
        const int want = opt_capture_pupdate && opt_bupdate_count < opt_pupdate_limit;
        if (want) {
                char path[4096];
                snprintf(path, sizeof path, "%s/bupdate_%03d.t3c", opt_capture_pupdate, opt_bupdate_count);
                cap_fp = fopen(path, "wb");
                if (!cap_fp) { perror(path); exit(EXIT_FAILURE); }
                fwrite("T3NSCAP1", 1, 8, cap_fp);
                dump_rops(0, &Operator[0]);
                dump_rops(1, &Operator[1]);
                dump_siteTensor("T", tens);
                if (opt_schedule_lib) {
                        void *h = dlopen(opt_schedule_lib, RTLD_NOW | RTLD_LOCAL);
                        int (*wr)(const struct rOperators *, const struct siteTensor *, const char *) =
                                h ? dlsym(h, "t3ns_dropin_bupdate_write") : NULL;
                        if (!wr) { fprintf(stderr, "no t3ns_dropin_bupdate_write\n"); exit(EXIT_FAILURE); }
                        char sp[4096];
                        snprintf(sp, sizeof sp, "%s/bupdate_%03d.sched", opt_capture_pupdate,
                                 opt_bupdate_count);
                        if (wr(Operator, tens, sp) != 0) exit(EXIT_FAILURE);
                }
        }
        real(newops, Operator, tens);
        if (want) {
                dump_rops(2, newops);
                fclose(cap_fp);
                cap_fp = NULL;
                ++opt_bupdate_count;
        }
}

/* Captures the dense factorisations of the site-tensor decomposition: every
 * LAPACKE_dgesdd / dgeqrf / dorgqr call the reference makes
 * (src/siteTensor_decompose.c:285, :295, :1060, :565) is logged with its
 * sizes to dense_sizes.txt, and up to --capture-dense-limit calls of each
 * kind are written with their inputs and the reference LAPACK's outputs.  The calls
 * come from OpenMP threads, so the bookkeeping is under a mutex and every
 * capture has its own file. */
static pthread_mutex_t dense_mu = PTHREAD_MUTEX_INITIALIZER;
static int dense_count[3];   /* per kind: gesdd, geqrf, orgqr */

static FILE *dense_open(const char *kind, int m, int n, int k)
{
        if (!opt_capture_dense) return NULL;
        char path[4096];
        const int kid = kind[2] == 's' ? 0 : kind[2] == 'q' ? 1 : 2;
        pthread_mutex_lock(&dense_mu);
        const int idx = dense_count[kid]++;
        snprintf(path, sizeof path, "%s/dense_sizes.txt", opt_capture_dense);
        FILE *log = fopen(path, "a");
        if (log) {
                fprintf(log, "%s %d %d %d\n", kind, m, n, k);
                fclose(log);
        }
        pthread_mutex_unlock(&dense_mu);
        if (idx >= opt_dense_limit) return NULL;
        snprintf(path, sizeof path, "%s/%s_%05d.t3c", opt_capture_dense, kind, idx);
        FILE *f = fopen(path, "wb");
        if (f) fwrite("T3NSCAP1", 1, 8, f);
        return f;
}

/* column-major m x n with leading dimension ld, compacted */
static double *dense_copy(const double *a, int m, int n, int ld)
{
        double *c = malloc(sizeof *c * (size_t) (m > 0 && n > 0 ? m * n : 1));
        for (int j = 0; j < n; ++j)
                for (int i = 0; i < m; ++i) c[i + (size_t) j * m] = a[i + (size_t) j * ld];
        return c;
}

static void dense_put_mat(FILE *f, const char *nm, const double *a, int m, int n, int ld)
{
        double *c = dense_copy(a, m, n, ld);
        cap_put_f(f, nm, 3, (int64_t) m * n, c);
        free(c);
}

static void dense_put_int(FILE *f, const char *nm, int v) { cap_put_f(f, nm, 1, 1, &v); }

typedef int (*gesdd_fn)(int, char, int, int, double *, int, double *, double *, int, double *, int);
int LAPACKE_dgesdd(int layout, char jobz, int m, int n, double *a, int lda, double *s,
                   double *u, int ldu, double *vt, int ldvt)
{
        static gesdd_fn real;
        if (!real) real = (gesdd_fn) dlsym(RTLD_NEXT, "LAPACKE_dgesdd");
        const int mn = m < n ? m : n;
        FILE *f = dense_open("gesdd", m, n, jobz);
        if (f) {
                dense_put_int(f, "gesdd.m", m);
                dense_put_int(f, "gesdd.n", n);
                dense_put_int(f, "gesdd.jobz", jobz);
                dense_put_mat(f, "gesdd.a", a, m, n, lda);
        }
        const int info = real(layout, jobz, m, n, a, lda, s, u, ldu, vt, ldvt);
        if (f) {
                dense_put_int(f, "gesdd.info", info);
                cap_put_f(f, "gesdd.s", 3, mn, s);
                if (jobz == 'S') {
                        dense_put_mat(f, "gesdd.u", u, m, mn, ldu);
                        dense_put_mat(f, "gesdd.vt", vt, mn, n, ldvt);
                }
                fclose(f);
        }
        return info;
}

typedef int (*geqrf_fn)(int, int, int, double *, int, double *);
int LAPACKE_dgeqrf(int layout, int m, int n, double *a, int lda, double *tau)
{
        static geqrf_fn real;
        if (!real) real = (geqrf_fn) dlsym(RTLD_NEXT, "LAPACKE_dgeqrf");
        FILE *f = dense_open("geqrf", m, n, 0);
        if (f) {
                dense_put_int(f, "geqrf.m", m);
                dense_put_int(f, "geqrf.n", n);
                dense_put_mat(f, "geqrf.a", a, m, n, lda);
        }
        const int info = real(layout, m, n, a, lda, tau);
        if (f) {
                dense_put_int(f, "geqrf.info", info);
                dense_put_mat(f, "geqrf.qr", a, m, n, lda);
                cap_put_f(f, "geqrf.tau", 3, m < n ? m : n, tau);
                fclose(f);
        }
        return info;
}

typedef int (*orgqr_fn)(int, int, int, int, double *, int, const double *);
int LAPACKE_dorgqr(int layout, int m, int n, int k, double *a, int lda, const double *tau)
{
        static orgqr_fn real;
        if (!real) real = (orgqr_fn) dlsym(RTLD_NEXT, "LAPACKE_dorgqr");
        FILE *f = dense_open("orgqr", m, n, k);
        if (f) {
                dense_put_int(f, "orgqr.m", m);
                dense_put_int(f, "orgqr.n", n);
                dense_put_int(f, "orgqr.k", k);
                dense_put_mat(f, "orgqr.a", a, m, n, lda);
                cap_put_f(f, "orgqr.tau", 3, k, tau);
        }
        const int info = real(layout, m, n, k, a, lda, tau);
        if (f) {
                dense_put_int(f, "orgqr.info", info);
                dense_put_mat(f, "orgqr.q", a, m, n, lda);
                fclose(f);
        }
        return info;
}

int sparse_eigensolve(double *result, double *energy, int size, int max_vecs,
                      int keep_deflate, double tol, int max_its,
                      const double *diagonal,
                      void (*matvec)(const double *, double *, void *),
                      void *vdat, const char solver[])
{
        static eig_fn real_eig;
        if (!real_eig) real_eig = (eig_fn) dlsym(RTLD_NEXT, "sparse_eigensolve");
        if (!real_eig) { fprintf(stderr, "sparse_eigensolve not found\n"); exit(EXIT_FAILURE); }

        const int want = opt_capture_dir && opt_captured < opt_capture_limit &&
                size <= opt_capture_max && size >= opt_capture_min;
        int ret = 0;
        if (opt_capture_structure) {
                if (opt_captured < opt_capture_limit && size <= opt_capture_max &&
                    size >= opt_capture_min) {
                        /* one matvec builds the replay schedule that
                         * destroy_Heffdata frees */
                        double *tmp = malloc(sizeof *tmp * (size_t) size);
                        matvec(result, tmp, vdat);
                        free(tmp);
                        capture_structure((const struct Heffdata *) vdat, size);
                        if (opt_capture_stop && opt_captured >= opt_capture_limit) {
                                printf("CAPTURE_DONE\n");
                                fflush(stdout);
                                _exit(0);
                        }
                } else {
                        double *tmp = malloc(sizeof *tmp * (size_t) size);
                        matvec(result, tmp, vdat);
                        free(tmp);
                }
                *energy = 0;
        } else if (want) {
                /* runs the reference Davidson in place on result */
                ret = capture_step((struct Heffdata *) vdat, result, size, diagonal,
                                   max_vecs, keep_deflate, tol, max_its, real_eig,
                                   matvec, energy);
                if (opt_capture_stop && opt_captured >= opt_capture_limit) {
                        printf("CAPTURE_DONE\n");
                        fflush(stdout);
                        _exit(0);
                }
        } else if (opt_capture_dir && opt_capture_noeig) {
                /* one matvec builds the replay schedule that destroy_Heffdata
                 * frees (src/Heff.c:1223-1240 expects it to exist) */
                double *tmp = malloc(sizeof *tmp * (size_t) size);
                matvec(result, tmp, vdat);
                free(tmp);
                *energy = 0;
        } else {
                ret = real_eig(result, energy, size, max_vecs, keep_deflate, tol,
                               max_its, diagonal, matvec, vdat, solver);
        }
        ++opt_step_counter;
        return ret;
}
#endif

/* ------------------------------------------------------------------ */

static void usage(void)
{
        fprintf(stderr,
                "usage: t3ns_run --net FILE --inter STR --symm Z2,U1,SU2[,..] --ts a,b,c[,..]\n"
                "       [--regime minD,maxD,truncerr,sitesize,rtl,its,sweeps,econv,noise]...\n"
                "       [--init c|r] [--capture DIR] [--capture-max N] [--capture-min N]\n"
                "       [--capture-limit N] [--capture-stop] [--capture-nvec N] [--capture-noeig]\n");
        exit(2);
}

/* --precond-file IN OUT: one call of davidson_diagonal_preconditioner (the
 * reference's in t3ns_run_ref, the drop-in's in t3ns_run_dropin) on the
 * arrays of IN ({int64 n; double theta; double result[n], diagonal[n],
 * vec_t[n]}); the resulting vec_t is written to OUT. */
static int precond_file(const char *in, const char *out)
{
        FILE *f = fopen(in, "rb");
        if (!f) return 2;
        int64_t n = 0;
        double theta = 0;
        if (fread(&n, sizeof n, 1, f) != 1 || fread(&theta, sizeof theta, 1, f) != 1 || n <= 0 ||
            n > INT32_MAX) { fclose(f); return 2; }
        double *a = malloc(sizeof *a * 3 * (size_t) n);
        if (!a || fread(a, sizeof *a, 3 * (size_t) n, f) != 3 * (size_t) n) { fclose(f); return 2; }
        fclose(f);
        davidson_diagonal_preconditioner(a, theta, (int) n, a + n, a + 2 * n);
        f = fopen(out, "wb");
        if (!f) return 2;
        fwrite(a + 2 * n, sizeof *a, (size_t) n, f);
        fclose(f);
        free(a);
        return 0;
}

int main(int argc, char **argv)
{
        if (argc == 4 && !strcmp(argv[1], "--precond-file")) return precond_file(argv[2], argv[3]);
        const char *net = NULL, *inter = NULL, *symm = "Z2,U1,SU2", *ts = NULL;
        char init = 'c';
        struct regime regs[16];
        int nreg = 0;

        setvbuf(stdout, NULL, _IOLBF, 0);
        for (int i = 1; i < argc; ++i) {
                const char *a = argv[i];
                const char *v = i + 1 < argc ? argv[i + 1] : NULL;
                if (!strcmp(a, "--net") && v) { net = v; ++i; }
                else if (!strcmp(a, "--inter") && v) { inter = v; ++i; }
                else if (!strcmp(a, "--symm") && v) { symm = v; ++i; }
                else if (!strcmp(a, "--ts") && v) { ts = v; ++i; }
                else if (!strcmp(a, "--init") && v) { init = v[0]; ++i; }
                else if (!strcmp(a, "--capture") && v) { opt_capture_dir = v; ++i; }
                else if (!strcmp(a, "--capture-structure") && v) { opt_capture_structure = v; ++i; }
                else if (!strcmp(a, "--capture-max") && v) { opt_capture_max = atol(v); ++i; }
                else if (!strcmp(a, "--capture-min") && v) { opt_capture_min = atol(v); ++i; }
                else if (!strcmp(a, "--capture-limit") && v) { opt_capture_limit = atoi(v); ++i; }
                else if (!strcmp(a, "--capture-nvec") && v) { opt_capture_nvec = atoi(v); ++i; }
                else if (!strcmp(a, "--capture-stop")) { opt_capture_stop = 1; }
                else if (!strcmp(a, "--capture-noeig")) { opt_capture_noeig = 1; }
                else if (!strcmp(a, "--schedule-lib") && v) { opt_schedule_lib = v; ++i; }
#ifndef T3NS_RUN_DROPIN
                else if (!strcmp(a, "--check-dropin") && v) { opt_check_dropin = v; ++i; }
#endif
                else if (!strcmp(a, "--capture-pupdate") && v) { opt_capture_pupdate = v; ++i; }
                else if (!strcmp(a, "--capture-pupdate-limit") && v) { opt_pupdate_limit = atoi(v); ++i; }
                else if (!strcmp(a, "--capture-dense") && v) { opt_capture_dense = v; ++i; }
                else if (!strcmp(a, "--capture-dense-limit") && v) { opt_dense_limit = atoi(v); ++i; }
                else if (!strcmp(a, "--regime") && v) {
                        struct regime *r = &regs[nreg++];
                        memset(r, 0, sizeof *r);
                        if (sscanf(v, "%d,%d,%lf,%d,%lf,%d,%d,%lf,%lf",
                                   &r->svd_sel.minD, &r->svd_sel.maxD,
                                   &r->svd_sel.truncerr, &r->sitesize,
                                   &r->davidson_rtl, &r->davidson_max_its,
                                   &r->max_sweeps, &r->energy_conv, &r->noise) != 9)
                                usage();
                        r->svd_sel.truncType = 'E';
                        ++i;
                } else usage();
        }
        if (!net || !inter || !ts || nreg == 0) usage();

        char buf[256];
        strncpy(buf, symm, sizeof buf - 1);
        buf[sizeof buf - 1] = 0;
        bookie.nrSyms = 0;
        for (char *tok = strtok(buf, ","); tok; tok = strtok(NULL, ",")) {
                if (!which_symmgroup(tok, &bookie.sgs[bookie.nrSyms])) {
                        fprintf(stderr, "unknown symmetry %s\n", tok);
                        return 2;
                }
                ++bookie.nrSyms;
        }
        strncpy(buf, ts, sizeof buf - 1);
        int nts = 0;
        for (char *tok = strtok(buf, ","); tok; tok = strtok(NULL, ","))
                bookie.target_state[nts++] = atoi(tok);
        if (nts != bookie.nrSyms) { fprintf(stderr, "target state arity\n"); return 2; }

        make_network(net);
        readinteraction((char *) inter);
        preparebookkeeper(NULL, regs[0].svd_sel.minD, 1, DEFAULT_MINSTATES, NULL);

        struct siteTensor *T3NS = NULL;
        struct rOperators *rops = NULL;
        double t0 = now_s();
        init_calculation(&T3NS, &rops, init);
        double t1 = now_s();
        struct optScheme scheme = {nreg, regs};
        double energy = execute_optScheme(T3NS, rops, &scheme, NULL);
        double t2 = now_s();
        printf("INIT_SECONDS %.6f\n", t1 - t0);
        printf("SWEEP_SECONDS %.6f\n", t2 - t1);
        printf("FINAL_ENERGY %.15f\n", energy);
        return 0;
}
