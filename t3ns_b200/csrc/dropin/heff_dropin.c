/* Reference-ABI drop-in for the effective-Hamiltonian matvec and Davidson.
 *
 * Exports exactly the reference entry points of include/Heff.h:166-192,
 * include/davidson.h:36-60 and include/wrapper_solvers.h:56-60, with the
 * reference's struct layouts (this file is compiled against the reference
 * headers), so the unchanged sweep driver (optimize_siteTensor,
 * src/optimize_network.c:188-226) links against it in place of Heff.o,
 * davidson.o and wrapper_solvers.o.  All arithmetic runs in the engine
 * (libt3ns_b200.so, include/t3ns_b200.h); there is no CPU code path for it.
 *
 * The schedule compiler below produces the reference's replay schedule
 * (what exec_firstrun, src/Heff.c:1002-1047, records in struct secondrun):
 * for every new block, the old blocks it couples to, and per pair the MPO
 * combinations with their operator symmetry blocks and symmetry prefactor.
 * The symmetry bookkeeping is the reference's own: qnB compatibility from
 * the operator block tables (src/Heff.c:118-360), MPO combinations that
 * couple to a singlet (MPO_couples_to_singlet), positions in the merge
 * instruction set (adaptMPOcombos, :1110-1136), prefactors from
 * prefactor_add_P_operator / prefactor_combine_MPOs (calc_prefactor,
 * :507-524) and operator blocks by binary search (find_operator_sb,
 * :757-796) -- all by calling the reference's exported routines, so the
 * integers and prefactors are bit-identical.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "Heff.h"
#include "bookkeeper.h"
#include "davidson.h"
#include "hamiltonian.h"
#include "instructions.h"
#include "macros.h"
#include "network.h"
#include "rOperators.h"
#include "sort.h"
#include "symmetries.h"
#include "symsecs.h"
#include "wrapper_solvers.h"

#include "t3ns_b200.h"

/* ------------------------------------------------------------------ */
/* side table: Heffdata* -> engine plan (the struct layout is the driver's) */

struct plan_entry {
        const struct Heffdata *key;
        t3ns_heff *plan;
        struct plan_entry *next;
};
static struct plan_entry *plans;
static pthread_mutex_t plans_lock = PTHREAD_MUTEX_INITIALIZER;

static void plan_put(const struct Heffdata *k, t3ns_heff *p)
{
        struct plan_entry *e = malloc(sizeof *e);
        if (!e) { fprintf(stderr, "t3ns drop-in: out of memory\n"); exit(EXIT_FAILURE); }
        e->key = k;
        e->plan = p;
        pthread_mutex_lock(&plans_lock);
        e->next = plans;
        plans = e;
        pthread_mutex_unlock(&plans_lock);
}

static t3ns_heff *plan_get(const struct Heffdata *k)
{
        t3ns_heff *p = NULL;
        pthread_mutex_lock(&plans_lock);
        for (struct plan_entry *e = plans; e; e = e->next)
                if (e->key == k) { p = e->plan; break; }
        pthread_mutex_unlock(&plans_lock);
        return p;
}

static t3ns_heff *plan_take(const struct Heffdata *k)
{
        t3ns_heff *p = NULL;
        pthread_mutex_lock(&plans_lock);
        for (struct plan_entry **e = &plans; *e; e = &(*e)->next)
                if ((*e)->key == k) {
                        struct plan_entry *d = *e;
                        p = d->plan;
                        *e = d->next;
                        free(d);
                        break;
                }
        pthread_mutex_unlock(&plans_lock);
        return p;
}

static void die(const char *what)
{
        fprintf(stderr, "t3ns drop-in: %s: %s\n", what, t3ns_last_error());
        exit(EXIT_FAILURE);
}

static void *xmalloc(size_t n)
{
        void *p = malloc(n ? n : 1);
        if (!p) { fprintf(stderr, "t3ns drop-in: out of memory\n"); exit(EXIT_FAILURE); }
        return p;
}

/* growable arrays */
struct ivec { int *a; int64_t n, cap; };
struct lvec { int64_t *a; int64_t n, cap; };
struct dvec { double *a; int64_t n, cap; };
#define VPUSH(v, x) do { if ((v).n == (v).cap) { (v).cap = (v).cap ? 2 * (v).cap : 64; \
        (v).a = realloc((v).a, sizeof *(v).a * (size_t) (v).cap); \
        if (!(v).a) { fprintf(stderr, "t3ns drop-in: out of memory\n"); exit(EXIT_FAILURE); } } \
        (v).a[(v).n++] = (x); } while (0)

/* ------------------------------------------------------------------ */
/* per-block index data (the reference's struct indexdata, src/Heff.c:486-505) */

struct blockidx {
        int id[STEPSPECS_MSITES][3];      /* symsec index per site and bond */
        QN_TYPE qn[STEPSPECS_MSITES];     /* site quantum number            */
        int dim[3];                       /* leg dim per operator           */
};

static void block_indices(const struct Heffdata *d, int sb, struct blockidx *b)
{
        const int ns = d->siteObject.nrsites;
        for (int i = 0; i < ns; ++i) {
                b->qn[i] = d->siteObject.qnumbers[ns * sb + i];
                indexize(b->id[i], b->qn[i], d->symarr[i]);
        }
        /* leg dims as fill_indexes (src/Heff.c:695-739) */
        for (int i = 0; i < (d->isdmrg ? 2 : 3); ++i) {
                const int site = d->rOperators_on_site[i];
                if (!d->Operators[i].P_operator) {
                        const int loose = d->isdmrg ? 2 * (i == 1) : i;
                        b->dim[i] = d->symarr[site][loose].dims[b->id[site][loose]];
                } else {
                        const int loose = 2 * !d->Operators[i].is_left;
                        b->dim[i] = d->symarr[site][loose].dims[b->id[site][loose]] *
                                    d->symarr[site][1].dims[b->id[site][1]];
                }
        }
        if (d->isdmrg) b->dim[2] = 1;
}

/* contraction order with the fewest operations, as make_cinfo
 * (src/Heff.c:629-666): first minimum among the orders */
static int best_order(const int *dnew, const int *dold, int isdmrg)
{
        static const int order[6][3] = {{0,1,2},{1,0,2},{0,2,1},{1,2,0},{2,0,1},{2,1,0}};
        int best = 0;
        long long nbest = 0;
        for (int i = 0; i < (isdmrg ? 2 : 6); ++i) {
                long long cur = 0;
                long long w[3] = {dold[0], dold[1], dold[2]};
                for (int j = 0; j < (isdmrg ? 2 : 3); ++j) {
                        cur += w[0] * w[1] * w[2] * dnew[order[i][j]];
                        w[order[i][j]] = dnew[order[i][j]];
                }
                if (i == 0 || nbest > cur) { best = i; nbest = cur; }
        }
        return best;
}

/* ------------------------------------------------------------------ */
/* qnB compatibility and MPO combinations                               */

/* For operator set i: lists of MPO sectors per (bra, ket) index pair of the
 * inner bond (reference makeqnumbersarr_from_operator, src/Heff.c:118-178). */
struct hsslist { int *ptr; int *hss; int dim; };

static void make_hsslist(const struct rOperators *op, int dim, struct hsslist *L)
{
        const int cpl = rOperators_give_nr_of_couplings(op);
        const int nblk = op->begin_blocks_of_hss[op->nrhss];
        int *cnt = calloc((size_t) dim * dim + 1, sizeof *cnt);
        QN_TYPE prev = -1;
        int hss = 0;
        for (int pass = 0; pass < 2; ++pass) {
                prev = -1;
                hss = 0;
                if (pass == 1) {
                        L->ptr = xmalloc(sizeof *L->ptr * ((size_t) dim * dim + 1));
                        L->ptr[0] = 0;
                        for (int k = 0; k < dim * dim; ++k) L->ptr[k + 1] = L->ptr[k] + cnt[k];
                        L->hss = xmalloc(sizeof *L->hss * (size_t) (L->ptr[dim * dim] + 1));
                        memset(cnt, 0, sizeof *cnt * (size_t) dim * dim);
                }
                for (int b = 0; b < nblk; ++b) {
                        const QN_TYPE qn = op->qnumbers[cpl * b + cpl - 1];
                        while (b >= op->begin_blocks_of_hss[hss + 1]) ++hss;
                        if (qn == prev) continue;
                        prev = qn;
                        const int bra = (int) (qn % dim);
                        const int ket = (int) ((qn / dim) % dim);
                        const int k = bra + dim * ket;
                        if (pass == 1) L->hss[L->ptr[k] + cnt[k]] = hss;
                        ++cnt[k];
                }
        }
        L->dim = dim;
        free(cnt);
}

static void free_hsslist(struct hsslist *L)
{
        free(L->ptr);
        free(L->hss);
}

static int cmp_qn(const void *a, const void *b)
{
        const QN_TYPE x = *(const QN_TYPE *) a, y = *(const QN_TYPE *) b;
        return x < y ? -1 : x > y;
}

/* The MPO-combination positions (into iset.MPOc) coupling old qnB to new
 * qnB, in the reference's enumeration order.  Returns the count. */
static int mpo_combos_T3NS(const struct Heffdata *d, const struct hsslist L[3],
                           const int nidx[3], const int oidx[3], int *out, int cap)
{
        const int hdim = d->MPOsymsec.nrSecs;
        const struct hsslist *a = &L[0], *b = &L[1], *c = &L[2];
        const int ka = nidx[0] + a->dim * oidx[0];
        const int kb = nidx[1] + b->dim * oidx[1];
        const int kc = nidx[2] + c->dim * oidx[2];
        int n = 0;
        for (int i = a->ptr[ka]; i < a->ptr[ka + 1]; ++i)
                for (int j = b->ptr[kb]; j < b->ptr[kb + 1]; ++j)
                        for (int k = c->ptr[kc]; k < c->ptr[kc + 1]; ++k) {
                                int MPOs[3] = {a->hss[i], b->hss[j], hermitian_symsec(c->hss[k])};
                                if (!MPO_couples_to_singlet(3, MPOs)) continue;
                                const int code = a->hss[i] + b->hss[j] * hdim + c->hss[k] * hdim * hdim;
                                const int pos = linSearch(&code, d->iset.MPOc, d->iset.nrMPOc,
                                                          SORT_INT, sizeof(int));
                                if (pos != -1 && n < cap) out[n++] = pos;
                        }
        return n;
}

/* ------------------------------------------------------------------ */
/* schedule compiler                                                    */

struct schedule {
        struct ivec dims;        /* 3 per block, per operator */
        struct ivec pair_ptr, pair_old, pair_order;
        struct lvec combo_ptr;
        struct ivec combo_mpo, combo_sbops;
        struct dvec combo_pref;
};

/* operator symmetry block of operator set i for the (new, old) pair and MPO
 * sector idMPO (find_operator_sb, src/Heff.c:757-796); -1 if absent */
static int operator_block(const struct Heffdata *d, int i, const struct blockidx *bn,
                          const struct blockidx *bo, int idMPO)
{
        const struct rOperators *op = &d->Operators[i];
        const int site = d->rOperators_on_site[i];
        const int inner = op->P_operator ? 2 * op->is_left
                                         : (d->isdmrg ? 2 * !op->is_left : i);
        const int dinner = d->symarr[site][inner].nrSecs;
        const QN_TYPE qninner = bn->id[site][inner] + (QN_TYPE) bo->id[site][inner] * dinner +
                                (QN_TYPE) idMPO * dinner * dinner;
        const QN_TYPE *qna = rOperators_give_qnumbers_for_hss(op, idMPO);
        const int nb = rOperators_give_nr_blocks_for_hss(op, idMPO);
        if (!op->P_operator)
                return binSearch(&qninner, qna, nb, SORT_QN_TYPE, sizeof qninner);
        const QN_TYPE qn[3] = {bn->qn[site], bo->qn[site], qninner};
        return binSearch(qn, qna, nb, SORT_QN_TYPE3, sizeof qn);
}

static void compile_pair(const struct Heffdata *d, const struct blockidx *bn,
                         const struct blockidx *bo, int old_sb, const int *mpos, int nmpo,
                         struct schedule *S)
{
        const int nops = d->isdmrg ? 2 : 3;
        int *irreps[STEPSPECS_MSITES][2][3];
        for (int s = 0; s < d->siteObject.nrsites; ++s)
                for (int j = 0; j < 3; ++j) {
                        irreps[s][0][j] = d->symarr[s][j].irreps[bn->id[s][j]];
                        irreps[s][1][j] = d->symarr[s][j].irreps[bo->id[s][j]];
                }
        const int64_t start = S->combo_mpo.n;
        for (int c = 0; c < nmpo; ++c) {
                const int MPO = mpos[c];
                const int i0 = d->iset.MPOc_beg[MPO], i1 = d->iset.MPOc_beg[MPO + 1];
                if (i1 == i0) continue;
                /* MPO sectors of the combination, from its first instruction
                 * (fill_MPO_indexes, src/Heff.c:741-755) */
                int idMPO[3] = {0, 0, 0};
                int *irrMPO[3] = {NULL, NULL, NULL};
                for (int i = 0; i < nops; ++i) {
                        idMPO[i] = d->Operators[i].hss_of_ops[d->iset.instr[i0].instr[i]];
                        irrMPO[i] = d->MPOsymsec.irreps[idMPO[i]];
                }
                /* calc_prefactor (src/Heff.c:507-524) */
                double pref = 1;
                for (int i = 0; i < nops; ++i) {
                        if (!d->Operators[i].P_operator) continue;
                        pref *= prefactor_add_P_operator(irreps[d->rOperators_on_site[i]],
                                                         d->Operators[i].is_left,
                                                         bookie.sgs, bookie.nrSyms);
                }
                pref *= prefactor_combine_MPOs(irreps[d->posB], irrMPO, bookie.sgs,
                                               bookie.nrSyms, d->isdmrg,
                                               2 * !d->Operators[1].P_operator);
                if (COMPARE_ELEMENT_TO_ZERO(pref)) continue;
                int sb[3] = {0, 0, 0};
                int ok = 1;
                for (int i = 0; i < nops; ++i) {
                        sb[i] = operator_block(d, i, bn, bo, idMPO[i]);
                        if (sb[i] == -1) ok = 0;
                }
                if (!ok) continue;
                VPUSH(S->combo_mpo, MPO);
                for (int i = 0; i < 3; ++i) VPUSH(S->combo_sbops, sb[i]);
                VPUSH(S->combo_pref, pref);
        }
        if (S->combo_mpo.n > start) {
                VPUSH(S->pair_old, old_sb);
                VPUSH(S->pair_order, best_order(bn->dim, bo->dim, d->isdmrg));
                VPUSH(S->combo_ptr, start);
        }
}

static void compile_schedule(const struct Heffdata *d, struct schedule *S)
{
        const int nb = d->siteObject.nrblocks;
        const int ns = d->siteObject.nrsites;
        struct blockidx *bi = xmalloc(sizeof *bi * (size_t) nb);
        QN_TYPE *qnB = xmalloc(sizeof *qnB * (size_t) nb);
        for (int b = 0; b < nb; ++b) {
                block_indices(d, b, &bi[b]);
                for (int k = 0; k < 3; ++k) VPUSH(S->dims, bi[b].dim[k]);
                qnB[b] = d->siteObject.qnumbers[ns * b + d->posB];
        }
        /* unique qnB values (sorted) and the blocks carrying each */
        QN_TYPE *uq = xmalloc(sizeof *uq * (size_t) nb);
        memcpy(uq, qnB, sizeof *uq * (size_t) nb);
        qsort(uq, (size_t) nb, sizeof *uq, cmp_qn);
        int nq = 0;
        for (int b = 0; b < nb; ++b)
                if (nq == 0 || uq[nq - 1] != uq[b]) uq[nq++] = uq[b];
        int *qid = xmalloc(sizeof *qid * (size_t) nb);
        int *qptr = calloc((size_t) nq + 1, sizeof *qptr);
        int *qblk = xmalloc(sizeof *qblk * (size_t) nb);
        for (int b = 0; b < nb; ++b) {
                const QN_TYPE *f = bsearch(&qnB[b], uq, (size_t) nq, sizeof *uq, cmp_qn);
                qid[b] = (int) (f - uq);
                ++qptr[qid[b] + 1];
        }
        for (int q = 0; q < nq; ++q) qptr[q + 1] += qptr[q];
        {
                int *fill = calloc((size_t) nq, sizeof *fill);
                for (int b = 0; b < nb; ++b) qblk[qptr[qid[b]] + fill[qid[b]]++] = b;
                free(fill);
        }

        /* MPO combinations per (new qnB, old qnB) */
        const int cap = d->MPOsymsec.nrSecs * d->MPOsymsec.nrSecs * d->MPOsymsec.nrSecs + 8;
        int *combos = xmalloc(sizeof *combos * (size_t) cap);
        int **pc = calloc((size_t) nq * nq, sizeof *pc);   /* [new * nq + old] */
        int *pn = calloc((size_t) nq * nq, sizeof *pn);
        if (!d->isdmrg) {
                int dims[3];
                struct hsslist L[3];
                for (int i = 0; i < 3; ++i) {
                        dims[i] = d->symarr[d->posB][i].nrSecs;
                        make_hsslist(&d->Operators[i], dims[i], &L[i]);
                }
                for (int qn = 0; qn < nq; ++qn) {
                        int ni[3];
                        QN_TYPE t = uq[qn];
                        ni[0] = (int) (t % dims[0]); t /= dims[0];
                        ni[1] = (int) (t % dims[1]); ni[2] = (int) (t / dims[1]);
                        for (int qo = 0; qo < nq; ++qo) {
                                int oi[3];
                                QN_TYPE u = uq[qo];
                                oi[0] = (int) (u % dims[0]); u /= dims[0];
                                oi[1] = (int) (u % dims[1]); oi[2] = (int) (u / dims[1]);
                                const int n = mpo_combos_T3NS(d, L, ni, oi, combos, cap);
                                if (n) {
                                        pc[qn * nq + qo] = xmalloc(sizeof(int) * (size_t) n);
                                        memcpy(pc[qn * nq + qo], combos, sizeof(int) * (size_t) n);
                                        pn[qn * nq + qo] = n;
                                }
                        }
                }
                for (int i = 0; i < 3; ++i) free_hsslist(&L[i]);
        } else {
                /* DMRG: the P-operator's own blocks give the couplings
                 * (make_qnB_arrDMRG, src/Heff.c:362-442) */
                const int opid = d->Operators[1].P_operator;
                const struct rOperators *op = &d->Operators[opid];
                const int N = op->begin_blocks_of_hss[op->nrhss];
                const int hdim = d->MPOsymsec.nrSecs;
                int hss = 0;
                for (int j = 0; j < N; ++j) {
                        while (op->begin_blocks_of_hss[hss + 1] <= j) ++hss;
                        const QN_TYPE *fn = bsearch(&op->qnumbers[3 * j], uq, (size_t) nq, sizeof *uq, cmp_qn);
                        const QN_TYPE *fo = bsearch(&op->qnumbers[3 * j + 1], uq, (size_t) nq, sizeof *uq, cmp_qn);
                        if (!fn || !fo) continue;
                        const int k = (int) (fn - uq) * nq + (int) (fo - uq);
                        const int c1 = opid == 1 ? hermitian_symsec(hss) : hss;
                        const int c2 = opid != 1 ? hermitian_symsec(hss) : hss;
                        const int code = c1 + c2 * hdim;
                        const int pos = linSearch(&code, d->iset.MPOc, d->iset.nrMPOc, SORT_INT, sizeof(int));
                        if (pos == -1) continue;
                        pc[k] = realloc(pc[k], sizeof(int) * (size_t) (pn[k] + 1));
                        pc[k][pn[k]++] = pos;
                }
        }

        /* pairs and combinations, new block by new block */
        for (int b = 0; b < nb; ++b) {
                VPUSH(S->pair_ptr, (int) S->pair_old.n);
                const int qn = qid[b];
                for (int qo = 0; qo < nq; ++qo) {
                        const int k = qn * nq + qo;
                        if (!pn[k]) continue;
                        for (int j = qptr[qo]; j < qptr[qo + 1]; ++j)
                                compile_pair(d, &bi[b], &bi[qblk[j]], qblk[j], pc[k], pn[k], S);
                }
        }
        VPUSH(S->pair_ptr, (int) S->pair_old.n);
        VPUSH(S->combo_ptr, S->combo_mpo.n);

        for (int k = 0; k < nq * nq; ++k) free(pc[k]);
        free(pc); free(pn); free(combos); free(qid); free(qptr); free(qblk); free(uq);
        free(qnB); free(bi);
}

/* ------------------------------------------------------------------ */

static int nr_unique_qnB(const struct siteTensor *st, int posB)
{
        QN_TYPE *q = xmalloc(sizeof *q * (size_t) st->nrblocks);
        for (int b = 0; b < st->nrblocks; ++b) q[b] = st->qnumbers[st->nrsites * b + posB];
        qsort(q, (size_t) st->nrblocks, sizeof *q, cmp_qn);
        int n = 0;
        for (int b = 0; b < st->nrblocks; ++b)
                if (n == 0 || q[n - 1] != q[b]) q[n++] = q[b];
        free(q);
        return n;
}

/* Writes the compiled schedule of `data` to `path` in the step-file record
 * layout ("my.*" records), without touching the GPU.  Used by the tests to
 * compare the schedule compiler with the reference's replay schedule. */
static void put_rec(FILE *f, const char *name, int dtype, int64_t n, const void *a)
{
        char nm[48] = {0};
        strncpy(nm, name, sizeof nm - 1);
        int32_t hdr[2] = {dtype, 0};
        fwrite(nm, 1, sizeof nm, f);
        fwrite(hdr, sizeof hdr, 1, f);
        fwrite(&n, sizeof n, 1, f);
        if (n) fwrite(a, dtype == 1 ? 4 : 8, (size_t) n, f);
}

int t3ns_dropin_schedule_write(const struct Heffdata *data, const char *path)
{
        struct schedule S;
        memset(&S, 0, sizeof S);
        compile_schedule(data, &S);
        FILE *f = fopen(path, "wb");
        if (!f) return -1;
        fwrite("T3NSCAP1", 1, 8, f);
        const int nq = data->nr_qnB;
        put_rec(f, "my.nr_qnB", 1, 1, &nq);
        put_rec(f, "my.dims", 1, S.dims.n, S.dims.a);
        put_rec(f, "my.pair_ptr", 1, S.pair_ptr.n, S.pair_ptr.a);
        put_rec(f, "my.pair_old", 1, S.pair_old.n, S.pair_old.a);
        put_rec(f, "my.pair_order", 1, S.pair_order.n, S.pair_order.a);
        put_rec(f, "my.combo_ptr", 2, S.combo_ptr.n, S.combo_ptr.a);
        put_rec(f, "my.combo_mpo", 1, S.combo_mpo.n, S.combo_mpo.a);
        put_rec(f, "my.combo_sbops", 1, S.combo_sbops.n, S.combo_sbops.a);
        put_rec(f, "my.combo_pref", 3, S.combo_pref.n, S.combo_pref.a);
        fclose(f);
        free(S.dims.a); free(S.pair_ptr.a); free(S.pair_old.a); free(S.pair_order.a);
        free(S.combo_ptr.a); free(S.combo_mpo.a); free(S.combo_sbops.a); free(S.combo_pref.a);
        return 0;
}

static int precision_from_env(void)
{
        const char *p = getenv("T3NS_B200_PRECISION");
        if (!p || !strcmp(p, "fp64")) return T3NS_PREC_FP64;
        if (!strcmp(p, "3xtf32")) return T3NS_PREC_3XTF32;
        if (!strcmp(p, "bf16x3")) return T3NS_PREC_BF16X3;
        fprintf(stderr, "t3ns drop-in: T3NS_B200_PRECISION=%s is not one of fp64, 3xtf32, bf16x3\n", p);
        exit(EXIT_FAILURE);
}

void init_Heffdata(struct Heffdata *data, const struct rOperators *Operators,
                   const struct siteTensor *siteObject)
{
        memset(data, 0, sizeof *data);
        data->isdmrg = (siteObject->nrsites == 1 && is_psite(siteObject->sites[0])) ||
                       (siteObject->nrsites == 2 && is_psite(siteObject->sites[0]) &&
                        is_psite(siteObject->sites[1]));
        data->siteObject = *siteObject;
        data->Operators[0] = Operators[0];
        data->Operators[1] = Operators[1];
        data->Operators[2] = data->isdmrg ? null_rOperators() : Operators[2];
        for (int i = 0; i < siteObject->nrsites; ++i) {
                int bonds[3];
                get_bonds_of_site(siteObject->sites[i], bonds);
                get_symsecs_arr(3, data->symarr[i], bonds);
        }
        get_symsecs(&data->MPOsymsec, -1);
        for (int i = 0; i < (data->isdmrg ? 2 : 3); ++i) {
                const int site = rOperators_site_to_attach(&Operators[i]);
                for (int j = 0; j < siteObject->nrsites; ++j)
                        if (siteObject->sites[j] == site) { data->rOperators_on_site[i] = j; break; }
        }
        for (int i = 0; i < siteObject->nrsites; ++i)
                if (!is_psite(siteObject->sites[i])) data->posB = i;
        if (data->isdmrg) data->posB = siteObject->nrsites - 1;
        int *hss_ops[3] = {Operators[0].hss_of_ops, Operators[1].hss_of_ops,
                           data->isdmrg ? NULL : Operators[2].hss_of_ops};
        data->iset = fetch_merge(Operators[0].bond, data->isdmrg, hss_ops);
        data->nr_qnB = nr_unique_qnB(siteObject, data->posB);

        struct schedule S;
        memset(&S, 0, sizeof S);
        compile_schedule(data, &S);

        /* engine descriptor */
        const int nb = siteObject->nrblocks;
        t3ns_heff_desc desc;
        memset(&desc, 0, sizeof desc);
        desc.isdmrg = data->isdmrg;
        /* memory axis j carries operator map[j] (make_map, src/Heff.c:668-682) */
        const int swap = data->rOperators_on_site[1] != data->posB &&
                         data->rOperators_on_site[0] == data->posB;
        desc.map[0] = swap ? 1 : 0;
        desc.map[1] = swap ? 0 : 1;
        desc.map[2] = 2;
        desc.nblocks = nb;
        int64_t *boff = xmalloc(sizeof *boff * (size_t) (nb + 1));
        for (int b = 0; b <= nb; ++b) boff[b] = siteObject->blocks.beginblock[b];
        desc.block_off = boff;
        desc.dims = S.dims.a;
        desc.pair_ptr = S.pair_ptr.a;
        desc.pair_old = S.pair_old.a;
        desc.pair_order = S.pair_order.a;
        desc.combo_ptr = S.combo_ptr.a;
        desc.combo_mpo = S.combo_mpo.a;
        desc.combo_sbops = S.combo_sbops.a;
        desc.combo_pref = S.combo_pref.a;
        desc.nr_instr = data->iset.nr_instr;
        int *ins = xmalloc(sizeof *ins * 3 * (size_t) (data->iset.nr_instr + 1));
        double *ipr = xmalloc(sizeof *ipr * (size_t) (data->iset.nr_instr + 1));
        for (int k = 0; k < data->iset.nr_instr; ++k) {
                for (int c = 0; c < 3; ++c) ins[3 * k + c] = data->iset.instr[k].instr[c];
                ipr[k] = data->iset.instr[k].pref;
        }
        desc.instr = ins;
        desc.instr_pref = ipr;
        desc.nrMPOc = data->iset.nrMPOc;
        desc.MPOc_beg = data->iset.MPOc_beg;
        void *keep[3][3];
        for (int i = 0; i < (data->isdmrg ? 2 : 3); ++i) {
                const struct rOperators *op = &data->Operators[i];
                int *nbl = xmalloc(sizeof *nbl * (size_t) (op->nrops + 1));
                const int **bbs = xmalloc(sizeof *bbs * (size_t) (op->nrops + 1));
                const double **tels = xmalloc(sizeof *tels * (size_t) (op->nrops + 1));
                for (int k = 0; k < op->nrops; ++k) {
                        nbl[k] = rOperators_give_nr_blocks_for_hss(op, op->hss_of_ops[k]);
                        bbs[k] = op->operators[k].beginblock;
                        tels[k] = op->operators[k].tel;
                }
                desc.ops[i].nrops = op->nrops;
                desc.ops[i].op_nblocks = nbl;
                desc.ops[i].op_beginblock = (const int *const *) bbs;
                desc.ops[i].op_tel = (const double *const *) tels;
                keep[i][0] = nbl;
                keep[i][1] = bbs;
                keep[i][2] = tels;
        }
        t3ns_heff *plan = NULL;
        if (t3ns_heff_create(&desc, precision_from_env(), &plan) != T3NS_OK)
                die("init_Heffdata");
        /* the first step of each size bucket times the kernel configurations */
        const char *tune = getenv("T3NS_B200_AUTOTUNE");
        if ((!tune || strcmp(tune, "0")) && t3ns_heff_autotune(plan, 1, 0, NULL) != T3NS_OK)
                die("init_Heffdata (autotune)");
        plan_put(data, plan);

        for (int i = 0; i < (data->isdmrg ? 2 : 3); ++i)
                for (int j = 0; j < 3; ++j) free(keep[i][j]);
        free(ins); free(ipr); free(boff);
        free(S.dims.a); free(S.pair_ptr.a); free(S.pair_old.a); free(S.pair_order.a);
        free(S.combo_ptr.a); free(S.combo_mpo.a); free(S.combo_sbops.a); free(S.combo_pref.a);
}

void matvecT3NS(const double *vec, double *result, void *vdata)
{
        t3ns_heff *plan = plan_get(vdata);
        if (!plan) { fprintf(stderr, "t3ns drop-in: matvecT3NS on an unknown Heffdata\n"); exit(EXIT_FAILURE); }
        if (t3ns_heff_matvec_host(plan, vec, result) != T3NS_OK) die("matvecT3NS");
}

EL_TYPE *make_diagonal(const struct Heffdata *data)
{
        t3ns_heff *plan = plan_get(data);
        if (!plan) { fprintf(stderr, "t3ns drop-in: make_diagonal on an unknown Heffdata\n"); exit(EXIT_FAILURE); }
        const int size = siteTensor_get_size(&data->siteObject);
        double *diag = xmalloc(sizeof *diag * (size_t) size);
        if (t3ns_heff_diagonal_host(plan, diag) != T3NS_OK) die("make_diagonal");
        return diag;
}

void destroy_Heffdata(struct Heffdata *data)
{
        t3ns_heff_destroy(plan_take(data));
}

/* ------------------------------------------------------------------ */
/* Davidson (include/davidson.h, include/wrapper_solvers.h)             */

void davidson_diagonal_preconditioner(const double *result, const double theta, const int size,
                                      const double *diagonal, double *vec_t)
{
        if (t3ns_precondition_host(size, result, theta, diagonal, vec_t) != T3NS_OK)
                die("davidson_diagonal_preconditioner");
}

int davidson(double *result, double *energy, int size, int max_vecs, int keep_deflate,
             double davidson_tol, int max_its, const double *diagonal,
             void (*matvec)(const double *, double *, void *), void *vdat)
{
        t3ns_davidson_info info;
        memset(&info, 0, sizeof info);
        int rc;
        t3ns_heff *plan = matvec == matvecT3NS ? plan_get(vdat) : NULL;
        if (plan)
                rc = t3ns_davidson_host(plan, result, energy, max_vecs, keep_deflate,
                                        davidson_tol, max_its, diagonal, &info);
        else
                rc = t3ns_davidson_callback(size, matvec, vdat, result, energy, max_vecs,
                                            keep_deflate, davidson_tol, max_its, diagonal, &info);
        if (rc == T3NS_E_EIG) {
                fprintf(stderr, "Error @davidson: %s\n", t3ns_last_error());
                return -1;
        }
        if (rc < 0) die("davidson");
        printf("   * Davidson: (iter: %d), (d_eig: %.1e), (trunc: %.1e), (time: %.3g sec), "
               "(fp64 iter: %d)\n",
               info.iterations, info.d_energy, info.residual, info.seconds, info.fp64_iterations);
        if (info.residual > davidson_tol) printf("     - Davidson stopped before converging.\n");
        return rc;
}

int sparse_eigensolve(double *result, double *energy, int size, int max_vecs, int keep_deflate,
                      double tol, int max_its, const double *diagonal,
                      void (*matvec)(const double *, double *, void *), void *vdat,
                      const char solver[])
{
        if (strcmp(solver, "D") != 0)
                fprintf(stderr, "Error @%s: Undefined solver %s.\n"
                        "Will continue with the default davidson solver.\n", __func__, solver);
        return davidson(result, energy, size, max_vecs, keep_deflate, tol, max_its, diagonal,
                        matvec, vdat);
}
