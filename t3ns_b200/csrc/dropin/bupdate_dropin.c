/* Reference-ABI drop-in for the branching renormalised-operator update.
 *
 * Exports update_rOperators_branching (reference include/rOperators.h:289-291,
 * src/rOperators_bUpdate.c:229-248) with the reference's signature and
 * ownership rules: the two input sets are left untouched and *newops receives
 * a freshly allocated set.  The contractions run in the engine
 * (t3ns_bupdate_host); the unique operators are combined by the reference's
 * own sum_unique_rOperators.
 *
 * The three bonds of the branching site are alpha, beta, gamma (site order).
 * Operator[0] lives on one of them (axis a), Operator[1] on another (axis b),
 * the new operator on the remaining one (axis g, the "update case").  A new
 * block (bra g, ket g, MPO g) receives, for every MPO split (h1, h2) of its
 * sector (tprods_ham), every block of Operator[0] in h1 and Operator[1] in
 * h2 whose ket indices meet a site-tensor block and whose bra indices meet
 * the adjoint block:
 *
 *     New(bg, kg) += pref * sum Ta(b_a, b_b, bg) O1(b_a, k_a) O2(b_b, k_b) T(k_a, k_b, kg)
 *
 * pref = prefactor_bUpdate of the nine irreps (update_selected_blocks,
 * :1043-1072), for every unique instruction of fetch_bUpdate whose MPO combo
 * is (h1, h2, hg) and whose three blocks are present (get_tels_operators,
 * :1074-1097).
 *
 * The schedule compiler restates the enumeration of update_unique_ops_T3NS
 * (:596-630) and update_newblock_w_MPO_set (:731-768): the same loop order
 * (new block, MPO split, block of the first operator, site-tensor block,
 * block of the second operator), so the per-block accumulation order matches
 * the reference's.  The engine applies the two operators to the ket block and
 * contracts with the bra block; the reference picks the cheapest of six
 * orders (how_to_update, :1000-1015), which changes rounding only.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bookkeeper.h"
#include "hamiltonian.h"
#include "instructions.h"
#include "macros.h"
#include "network.h"
#include "rOperators.h"
#include "siteTensor.h"
#include "sort.h"
#include "sparseblocks.h"
#include "symmetries.h"
#include "symsecs.h"

#include "t3ns_b200.h"
#include "dropin_sum.h"

enum { BU_BRA = 0, BU_KET = 1, BU_MPO = 2 };

struct bu_key { QN_TYPE key; int idx; };

static int bu_key_cmp(const void *x, const void *y)
{
        const struct bu_key *a = x, *b = y;
        if (a->key != b->key) return a->key < b->key ? -1 : 1;
        return a->idx < b->idx ? -1 : a->idx > b->idx;
}

/* first position in sorted keys[0..n) with key >= k */
static int bu_lower(const struct bu_key *keys, int n, QN_TYPE k)
{
        int lo = 0, hi = n;
        while (lo < hi) {
                const int mid = (lo + hi) / 2;
                if (keys[mid].key < k) lo = mid + 1;
                else hi = mid;
        }
        return lo;
}

static int bu_lower_qn(const QN_TYPE *qn, int n, QN_TYPE k)
{
        int lo = 0, hi = n;
        while (lo < hi) {
                const int mid = (lo + hi) / 2;
                if (qn[mid] < k) lo = mid + 1;
                else hi = mid;
        }
        return lo;
}

struct bu_sched {
        struct rOperators uo;                /* unique new operators, zero-filled */
        struct instructionset set;           /* the reference's cached fetch_bUpdate set */
        int ax[3];
        struct dv_vec unit_ptr, dims, t_off, ta_off, pref, op_ptr, o1_off, o2_off, new_off;
        int64_t *base1, *base2, *ubase;
};

static void bu_compile(const struct rOperators Operator[2], const struct siteTensor *T,
                       struct bu_sched *S)
{
        memset(S, 0, sizeof *S);
        S->unit_ptr.el = S->dims.el = S->op_ptr.el = sizeof(int);
        S->t_off.el = S->ta_off.el = S->o1_off.el = S->o2_off.el = S->new_off.el = sizeof(int64_t);
        S->pref.el = sizeof(double);

        /* the update case (prepare_update_branching, :309-330) */
        const int site = T->sites[0];
        int bonds[3];
        get_bonds_of_site(site, bonds);
        int uc = 0;
        while (uc < 3 && (bonds[uc] == Operator[0].bond || bonds[uc] == Operator[1].bond)) ++uc;
        if (uc == 3) {
                fprintf(stderr, "t3ns drop-in: update_rOperators_branching: no free bond\n");
                exit(EXIT_FAILURE);
        }
        const int id_ops[3] = {uc == 0 ? 1 : 0, uc == 2 ? 1 : 2, uc};
        S->ax[0] = id_ops[0];
        S->ax[1] = id_ops[1];
        S->ax[2] = uc;
        S->set = fetch_bUpdate(bonds[uc], Operator[1].is_left);
        dropin_init_unique(&S->uo, bonds[uc], Operator[1].is_left, false, &S->set);
        const struct rOperators *uo = &S->uo;

        /* symsecs of bra, ket and MPO on the three bonds (initialize_indexhelper, :529-565) */
        struct symsecs ss[3][3];
        int md[3][3];
        for (int i = 0; i < 3; ++i) {
                const int b3[3] = {get_braT3NSbond(bonds[i]), get_ketT3NSbond(bonds[i]),
                                   get_hamiltonianbond(bonds[i])};
                get_symsecs_arr(3, ss[i], b3);
                for (int j = 0; j < 3; ++j) md[i][j] = ss[i][j].nrSecs;
        }

        /* site-tensor blocks keyed by the two ket indices known before the
         * block is picked (make_qntens, :332-395) */
        const int looptype = uc == 0;
        const QN_TYPE tdiv = looptype ? (QN_TYPE) md[0][BU_KET] * md[1][BU_KET] : md[0][BU_KET];
        struct bu_key *tkeys = safe_malloc(T->nrblocks + 1, struct bu_key);
        for (int i = 0; i < T->nrblocks; ++i) {
                tkeys[i].key = looptype ? T->qnumbers[i] % tdiv : T->qnumbers[i] / tdiv;
                tkeys[i].idx = i;
        }
        qsort(tkeys, T->nrblocks, sizeof *tkeys, bu_key_cmp);

        /* unique instructions keyed by their MPO combo (init_instrhelper, :467-527) */
        const QN_TYPE dimhss = get_nr_hamsymsec();
        struct bu_key *ikeys = safe_malloc(uo->nrops + 1, struct bu_key);
        int *uinstr = safe_malloc(uo->nrops + 1, int);
        {
                int ci = -1, u = 0;
                while (get_next_unique_instr(&ci, &S->set)) {
                        const int *in = S->set.instr[ci].instr;
                        ikeys[u].key = Operator[0].hss_of_ops[in[0]] +
                                Operator[1].hss_of_ops[in[1]] * dimhss +
                                S->set.hss_of_new[in[2]] * dimhss * dimhss;
                        ikeys[u].idx = u;
                        uinstr[u] = ci;
                        ++u;
                }
                qsort(ikeys, uo->nrops, sizeof *ikeys, bu_key_cmp);
        }

        S->base1 = dropin_op_bases(&Operator[0]);
        S->base2 = dropin_op_bases(&Operator[1]);
        S->ubase = dropin_op_bases(uo);

        const int first = looptype ? 0 : 1, second = !first;
        const int fb = id_ops[first], sbnd = id_ops[second];
        const int N = uo->begin_blocks_of_hss[uo->nrhss];
        for (int nsb = 0; nsb < N; ++nsb) {
                int id[3][3];
                {
                        QN_TYPE q = uo->qnumbers[nsb];
                        id[uc][BU_BRA] = (int) (q % md[uc][BU_BRA]);
                        q /= md[uc][BU_BRA];
                        id[uc][BU_KET] = (int) (q % md[uc][BU_KET]);
                        id[uc][BU_MPO] = (int) (q / md[uc][BU_KET]);
                }
                const int hn = id[uc][BU_MPO];
                const int sbn = nsb - uo->begin_blocks_of_hss[hn];
                const int entries_before = (int) S->pref.n;
                int nprods, *prods;
                tprods_ham(&nprods, &prods, hn, site);
                for (int p = 0; p < nprods; ++p) {
                        const int h[2] = {prods[2 * p], prods[2 * p + 1]};
                        const struct rOperators *F = &Operator[first], *Sd = &Operator[second];
                        const int nbf = rOperators_give_nr_blocks_for_hss(F, h[first]);
                        const QN_TYPE *qf = rOperators_give_qnumbers_for_hss(F, h[first]);
                        const int nbs = rOperators_give_nr_blocks_for_hss(Sd, h[second]);
                        const QN_TYPE *qs = rOperators_give_qnumbers_for_hss(Sd, h[second]);
                        const QN_TYPE sdiv = md[sbnd][BU_BRA];
                        for (int sbf = 0; sbf < nbf; ++sbf) {
                                QN_TYPE q = qf[sbf];
                                id[fb][BU_BRA] = (int) (q % md[fb][BU_BRA]);
                                q /= md[fb][BU_BRA];
                                id[fb][BU_KET] = (int) (q % md[fb][BU_KET]);
                                id[fb][BU_MPO] = (int) (q / md[fb][BU_KET]);
                                id[sbnd][BU_MPO] = h[second];
                                const QN_TYPE tk = looptype
                                        ? id[0][BU_KET] + (QN_TYPE) id[1][BU_KET] * md[0][BU_KET]
                                        : id[1][BU_KET] + (QN_TYPE) id[2][BU_KET] * md[1][BU_KET];
                                for (int ti = bu_lower(tkeys, T->nrblocks, tk);
                                     ti < T->nrblocks && tkeys[ti].key == tk; ++ti) {
                                        const int tb = tkeys[ti].idx;
                                        id[sbnd][BU_KET] = (int) (looptype ? T->qnumbers[tb] / tdiv
                                                                           : T->qnumbers[tb] % tdiv);
                                        /* blocks of the second operator with this ket and MPO */
                                        const QN_TYPE quot = id[sbnd][BU_KET] +
                                                (QN_TYPE) id[sbnd][BU_MPO] * md[sbnd][BU_KET];
                                        for (int k = bu_lower_qn(qs, nbs, quot * sdiv);
                                             k < nbs && qs[k] / sdiv == quot; ++k) {
                                                id[sbnd][BU_BRA] = (int) (qs[k] % sdiv);
                                                const int sb[2] = {first == 0 ? sbf : k, first == 0 ? k : sbf};
                                                /* the adjoint block (find_block_adj, :770-790) */
                                                QN_TYPE aq = 0;
                                                for (int i = 2; i >= 0; --i)
                                                        aq = aq * md[i][BU_BRA] + id[i][BU_BRA];
                                                const int ab = binSearch(&aq, T->qnumbers, T->nrblocks,
                                                                         SORT_QN_TYPE, sizeof aq);
                                                if (ab == -1) continue;
                                                int dm[6];
                                                int64_t prod = 1;
                                                for (int i = 0; i < 3; ++i) {
                                                        dm[i] = ss[i][BU_KET].dims[id[i][BU_KET]];
                                                        dm[3 + i] = ss[i][BU_BRA].dims[id[i][BU_BRA]];
                                                        prod *= (int64_t) dm[i] * dm[3 + i];
                                                }
                                                if (!prod) continue;
                                                int *irr[3][3];
                                                for (int i = 0; i < 3; ++i)
                                                        for (int j = 0; j < 3; ++j)
                                                                irr[i][j] = ss[i][j].irreps[id[i][j]];
                                                const double pf = prefactor_bUpdate(irr, uc, bookie.sgs,
                                                                                    bookie.nrSyms);
                                                /* matching unique instructions (find_matching_instr) */
                                                const QN_TYPE mk = id[id_ops[0]][BU_MPO] +
                                                        id[id_ops[1]][BU_MPO] * dimhss + hn * dimhss * dimhss;
                                                const int first_tr = (int) S->o1_off.n;
                                                for (int r = bu_lower(ikeys, uo->nrops, mk);
                                                     r < uo->nrops && ikeys[r].key == mk; ++r) {
                                                        const int u = ikeys[r].idx;
                                                        const int *in = S->set.instr[uinstr[u]].instr;
                                                        const struct sparseblocks *b1 = &Operator[0].operators[in[0]];
                                                        const struct sparseblocks *b2 = &Operator[1].operators[in[1]];
                                                        const struct sparseblocks *bn = &uo->operators[u];
                                                        if (!get_size_block(b1, sb[0]) || !get_size_block(b2, sb[1]) ||
                                                            !get_size_block(bn, sbn))
                                                                continue;
                                                        const int64_t o1 = S->base1[in[0]] + b1->beginblock[sb[0]];
                                                        const int64_t o2 = S->base2[in[1]] + b2->beginblock[sb[1]];
                                                        const int64_t on = S->ubase[u] + bn->beginblock[sbn];
                                                        dv_push(&S->o1_off, &o1);
                                                        dv_push(&S->o2_off, &o2);
                                                        dv_push(&S->new_off, &on);
                                                }
                                                if ((int) S->o1_off.n == first_tr) continue;
                                                for (int i = 0; i < 6; ++i) dv_push(&S->dims, &dm[i]);
                                                const int64_t to = T->blocks.beginblock[tb];
                                                const int64_t tao = T->blocks.beginblock[ab];
                                                dv_push(&S->t_off, &to);
                                                dv_push(&S->ta_off, &tao);
                                                dv_push(&S->pref, &pf);
                                                dv_push(&S->op_ptr, &first_tr);
                                        }
                                }
                        }
                }
                safe_free(prods);
                if ((int) S->pref.n > entries_before) dv_push(&S->unit_ptr, &entries_before);
        }
        const int ne = (int) S->pref.n, nt = (int) S->o1_off.n;
        dv_push(&S->unit_ptr, &ne);
        dv_push(&S->op_ptr, &nt);
        safe_free(tkeys);
        safe_free(ikeys);
        safe_free(uinstr);
}

static void bu_free(struct bu_sched *S)
{
        struct dv_vec *v[] = {&S->unit_ptr, &S->dims, &S->t_off, &S->ta_off, &S->pref,
                              &S->op_ptr, &S->o1_off, &S->o2_off, &S->new_off};
        for (size_t i = 0; i < sizeof v / sizeof v[0]; ++i) free(v[i]->a);
        safe_free(S->base1);
        safe_free(S->base2);
        safe_free(S->ubase);
}

static void bu_desc(const struct bu_sched *S, const struct rOperators Operator[2],
                    const struct siteTensor *T, t3ns_bupdate_desc *d)
{
        memset(d, 0, sizeof *d);
        for (int i = 0; i < 3; ++i) d->ax[i] = S->ax[i];
        d->nunits = (int) S->unit_ptr.n - 1;
        d->unit_ptr = S->unit_ptr.a;
        d->nentries = (int) S->pref.n;
        d->dims = S->dims.a;
        d->t_off = S->t_off.a;
        d->ta_off = S->ta_off.a;
        d->pref = S->pref.a;
        d->op_ptr = S->op_ptr.a;
        d->o1_off = S->o1_off.a;
        d->o2_off = S->o2_off.a;
        d->new_off = S->new_off.a;
        d->t_elems = T->blocks.beginblock[T->nrblocks];
        d->o1_elems = S->base1[Operator[0].nrops];
        d->o2_elems = S->base2[Operator[1].nrops];
        d->new_elems = S->ubase[S->uo.nrops];
}

void update_rOperators_branching(struct rOperators *newops, const struct rOperators *Operator,
                                 const struct siteTensor *tens)
{
        struct bu_sched S;
        bu_compile(Operator, tens, &S);
        t3ns_bupdate_desc d;
        bu_desc(&S, Operator, tens, &d);
        double *o1 = dropin_gather(&Operator[0], S.base1);
        double *o2 = dropin_gather(&Operator[1], S.base2);
        /* the unique operators stay on the device and are summed there
         * (sum_unique_rOperators, src/rOperators_init.c:228-265) */
        struct dropin_sum su;
        dropin_sum_build(&su, &S.uo, &S.set, S.ubase, newops);
        if (t3ns_bupdate_sum_host(&d, &su.d, tens->blocks.tel, o1, o2, su.new_tel, su.new_begin,
                                  su.out_base) != T3NS_OK) {
                fprintf(stderr, "t3ns drop-in: update_rOperators_branching: %s\n", t3ns_last_error());
                exit(EXIT_FAILURE);
        }
        dropin_sum_finish(&su, newops);
        destroy_rOperators(&S.uo);
        safe_free(o1);
        safe_free(o2);
        bu_free(&S);
}

/* Test hook: the compiled schedule of a branching update, written without
 * the GPU ("bu.*" records in the step-file layout), with the instruction set
 * and the unique operators' block layout needed to sum them. */
int t3ns_dropin_bupdate_write(const struct rOperators *Operator, const struct siteTensor *tens,
                              const char *path)
{
        struct bu_sched S;
        bu_compile(Operator, tens, &S);
        FILE *f = fopen(path, "wb");
        if (!f) {
                destroy_rOperators(&S.uo);
                bu_free(&S);
                return -1;
        }
        fwrite("T3NSCAP1", 1, 8, f);
        dropin_rec(f, "bu.ax", 1, 3, S.ax);
        dropin_rec(f, "bu.unit_ptr", 1, S.unit_ptr.n, S.unit_ptr.a);
        dropin_rec(f, "bu.dims", 1, S.dims.n, S.dims.a);
        dropin_rec(f, "bu.t_off", 2, S.t_off.n, S.t_off.a);
        dropin_rec(f, "bu.ta_off", 2, S.ta_off.n, S.ta_off.a);
        dropin_rec(f, "bu.pref", 3, S.pref.n, S.pref.a);
        dropin_rec(f, "bu.op_ptr", 1, S.op_ptr.n, S.op_ptr.a);
        dropin_rec(f, "bu.o1_off", 2, S.o1_off.n, S.o1_off.a);
        dropin_rec(f, "bu.o2_off", 2, S.o2_off.n, S.o2_off.a);
        dropin_rec(f, "bu.new_off", 2, S.new_off.n, S.new_off.a);
        dropin_rec(f, "bu.unique_base", 2, (int64_t) S.uo.nrops + 1, S.ubase);
        dropin_rec(f, "bu.unique_hss", 1, S.uo.nrops, S.uo.hss_of_ops);
        struct dv_vec bb = {0, 0, 0, sizeof(int)};
        for (int i = 0; i < S.uo.nrops; ++i) {
                const int nb = nblocks_in_operator(&S.uo, i);
                for (int b = 0; b <= nb; ++b) dv_push(&bb, &S.uo.operators[i].beginblock[b]);
        }
        dropin_rec(f, "bu.unique_beginblock", 1, bb.n, bb.a);
        free(bb.a);
        /* instructions with the unique operator each one reads (the
         * grouping of get_next_unique_instr / sum_unique_rOperators) */
        struct dv_vec ins = {0, 0, 0, sizeof(int)}, ipf = {0, 0, 0, sizeof(double)};
        struct dv_vec iun = {0, 0, 0, sizeof(int)}, hsn = {0, 0, 0, sizeof(int)};
        int u = -1, nnew = 0;
        for (int i = 0; i < S.set.nr_instr; ++i) {
                const int *in = S.set.instr[i].instr, *pin = S.set.instr[i ? i - 1 : 0].instr;
                if (i == 0 || in[0] != pin[0] || in[1] != pin[1] ||
                    S.set.hss_of_new[in[2]] != S.set.hss_of_new[pin[2]])
                        ++u;
                for (int j = 0; j < 3; ++j) dv_push(&ins, &in[j]);
                dv_push(&ipf, &S.set.instr[i].pref);
                dv_push(&iun, &u);
                if (in[2] + 1 > nnew) nnew = in[2] + 1;
        }
        for (int k = 0; k < nnew; ++k) dv_push(&hsn, &S.set.hss_of_new[k]);
        dropin_rec(f, "bu.instr", 1, ins.n, ins.a);
        dropin_rec(f, "bu.instr_pref", 3, ipf.n, ipf.a);
        dropin_rec(f, "bu.instr_unique", 1, iun.n, iun.a);
        dropin_rec(f, "bu.hss_of_new", 1, hsn.n, hsn.a);
        free(ins.a);
        free(ipf.a);
        free(iun.a);
        free(hsn.a);
        fclose(f);
        destroy_rOperators(&S.uo);
        bu_free(&S);
        return 0;
}
