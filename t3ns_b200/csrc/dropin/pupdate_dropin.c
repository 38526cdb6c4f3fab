/* Reference-ABI drop-in for the physical renormalised-operator update.
 *
 * Exports update_rOperators_physical (reference include/rOperators.h:276-278,
 * src/rOperators_pUpdate.c:364-387) with the reference's signature and
 * ownership rules: the input set is destroyed and replaced by the updated
 * one, whose arrays are host malloc memory the driver later frees.  The
 * arithmetic runs in the engine (t3ns_pupdate_host).
 *
 * The schedule compiler restates the reference's bookkeeping with the
 * reference's exported routines (indexize, translate_indices, qntypize,
 * binSearch, prefactor_adjoint, prefactor_pUpdate, init_rOperators,
 * kick_zero_blocks):
 *   - symsecs of the update (make_update_data, :127-158);
 *   - for each updated block, the range of original blocks that map onto it
 *     (make_usb_to_osb, :100-125);
 *   - per (updated, original) block pair: the site-tensor block, its
 *     adjoint, the dims M0, M1, N0, N1 and the symmetry prefactor
 *     (select_site_blocks, :210-271);
 *   - per pair, every operator of the block's MPO sector whose original and
 *     updated blocks are both present (pUpdate_block, :323-362).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "bookkeeper.h"
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

struct pu_sched {
        struct rOperators ur;        /* updated operators (structure + calloc'd tel) */
        struct dv_vec unit_ptr, dims, t_off, ta_off, pref, op_ptr, old_off, new_off;
        int64_t *old_base, *new_base;
        int64_t old_elems, new_elems;
};

/* the updated set's structure, as init_updated_rOperators (:65-83) */
static struct rOperators pu_init_updated(const struct rOperators *rops)
{
        struct rOperators urops;
        int **tmpbb;
        init_rOperators(&urops, &tmpbb, rops->bond, rops->is_left, false);
        urops.nrops = rops->nrops;
        urops.hss_of_ops = safe_malloc(urops.nrops, *urops.hss_of_ops);
        urops.operators = safe_malloc(urops.nrops, *urops.operators);
        for (int i = 0; i < rops->nrops; ++i) {
                const int chss = rops->hss_of_ops[i];
                const int nrbl = rOperators_give_nr_blocks_for_hss(&urops, chss);
                urops.hss_of_ops[i] = chss;
                init_sparseblocks(&urops.operators[i], tmpbb[chss], nrbl, 'c');
        }
        for (int i = 0; i < urops.nrhss; ++i) safe_free(tmpbb[i]);
        safe_free(tmpbb);
        return urops;
}

static void pu_compile(const struct rOperators *rops, const struct siteTensor *T,
                       const struct symsecs *iss, struct pu_sched *S)
{
        memset(S, 0, sizeof *S);
        S->unit_ptr.el = sizeof(int);
        S->dims.el = sizeof(int);
        S->t_off.el = sizeof(int64_t);
        S->ta_off.el = sizeof(int64_t);
        S->pref.el = sizeof(double);
        S->op_ptr.el = sizeof(int);
        S->old_off.el = sizeof(int64_t);
        S->new_off.el = sizeof(int64_t);
        S->ur = pu_init_updated(rops);
        const struct rOperators *ur = &S->ur;
        const int il = rops->is_left == 1;

        /* symsecs (make_update_data) */
        struct symsecs Tss[3], uss[3], oss[3][3];
        int bonds[3];
        get_bonds_of_site(T->sites[0], bonds);
        get_symsecs_arr(3, Tss, bonds);
        uss[0] = Tss[il ? 2 : 0];
        uss[1] = Tss[il ? 2 : 0];
        get_symsecs(&uss[2], get_hamiltonianbond(rops->bond));
        get_symsecs_arr(3, oss[0], bonds);
        get_symsecs_arr(3, oss[1], bonds);
        oss[0][il ? 2 : 0] = *iss;
        oss[1][il ? 2 : 0] = *iss;
        oss[2][0] = *iss;
        oss[2][1] = *iss;
        get_symsecs(&oss[2][2], get_hamiltonianbond(rops->bond));

        /* element bases of every operator in the concatenations */
        S->old_base = safe_malloc(rops->nrops + 1, int64_t);
        S->new_base = safe_malloc(rops->nrops + 1, int64_t);
        S->old_base[0] = S->new_base[0] = 0;
        for (int i = 0; i < rops->nrops; ++i) {
                const int nbo = rOperators_give_nr_blocks_for_hss(rops, rops->hss_of_ops[i]);
                const int nbn = rOperators_give_nr_blocks_for_hss(ur, ur->hss_of_ops[i]);
                S->old_base[i + 1] = S->old_base[i] + rops->operators[i].beginblock[nbo];
                S->new_base[i + 1] = S->new_base[i] + ur->operators[i].beginblock[nbn];
        }
        S->old_elems = S->old_base[rops->nrops];
        S->new_elems = S->new_base[rops->nrops];

        const int N = ur->begin_blocks_of_hss[ur->nrhss];
        const int NN = rops->begin_blocks_of_hss[rops->nrhss];
        int osb = 0, newhss = 0;
        for (int usb = 0; usb < N; ++usb) {
                while (usb >= ur->begin_blocks_of_hss[newhss + 1]) ++newhss;
                /* original blocks [osb_begin, osb_end) for this updated block */
                int id[3], nid[3];
                indexize(id, ur->qnumbers[usb], uss);
                translate_indices(id, uss, nid, oss[2], 2);
                nid[2] = id[2];
                const QN_TYPE qn = qntypize(nid, oss[2]);
                const int osb_begin = osb;
                while (osb < NN && !(qn < rops->qnumbers[3 * osb + 2])) ++osb;
                const int osb_end = osb;

                const int entries_before = (int) S->pref.n;
                for (int ob = osb_begin; ob < osb_end; ++ob) {
                        const int usb2 = usb - ur->begin_blocks_of_hss[newhss];
                        const int osb2 = ob - rops->begin_blocks_of_hss[newhss];
                        /* select_site_blocks */
                        const QN_TYPE *cqn = &rops->qnumbers[3 * ob];
                        int ids[3][3], Tids[2][3];
                        for (int k = 0; k < 3; ++k) indexize(ids[k], cqn[k], oss[k]);
                        translate_indices(ids[1], oss[0], Tids[0], Tss, 3);
                        if (Tids[0][0] < 0 || Tids[0][1] < 0 || Tids[0][2] < 0) continue;
                        translate_indices(ids[0], oss[1], Tids[1], Tss, 3);
                        if (Tids[1][0] < 0 || Tids[1][1] < 0 || Tids[1][2] < 0) continue;
                        const QN_TYPE Tqn = qntypize(Tids[0], Tss);
                        const QN_TYPE Thqn = qntypize(Tids[1], Tss);
                        const int Tsb = binSearch(&Tqn, T->qnumbers, T->nrblocks, SORT_QN_TYPE, sizeof Tqn);
                        const int Thsb = binSearch(&Thqn, T->qnumbers, T->nrblocks, SORT_QN_TYPE, sizeof Thqn);
                        if (Tsb == -1 || Thsb == -1) continue;
                        if (!get_size_block(&T->blocks, Tsb) || !get_size_block(&T->blocks, Thsb)) continue;
                        const int N0 = Tss[2 * il].dims[Tids[1][2 * il]];
                        const int N1 = Tss[2 * il].dims[Tids[0][2 * il]];
                        const int M0 = Tss[2 * !il].dims[Tids[1][2 * !il]] * Tss[1].dims[Tids[1][1]];
                        const int M1 = Tss[2 * !il].dims[Tids[0][2 * !il]] * Tss[1].dims[Tids[0][1]];
                        const int *irr[3][3];
                        for (int i = 0; i < 3; ++i)
                                for (int j = 0; j < 3; ++j) irr[i][j] = oss[i][j].irreps[ids[i][j]];
                        double pref = prefactor_adjoint(irr[0], (char) (il ? '3' : '1'),
                                                        bookie.sgs, bookie.nrSyms);
                        pref *= prefactor_pUpdate(irr, il, bookie.sgs, bookie.nrSyms);

                        /* operators of the sector with both blocks present */
                        const int first_pair = (int) S->old_off.n;
                        for (int i = 0; i < rops->nrops; ++i) {
                                if (rops->hss_of_ops[i] != newhss) continue;
                                const struct sparseblocks *ob_ = &rops->operators[i];
                                const struct sparseblocks *nb_ = &ur->operators[i];
                                if (!get_size_block(ob_, osb2) || !get_size_block(nb_, usb2)) continue;
                                const int64_t oo = S->old_base[i] + ob_->beginblock[osb2];
                                const int64_t no = S->new_base[i] + nb_->beginblock[usb2];
                                dv_push(&S->old_off, &oo);
                                dv_push(&S->new_off, &no);
                        }
                        if ((int) S->old_off.n == first_pair) continue;
                        const int dm[4] = {M0, M1, N0, N1};
                        for (int k = 0; k < 4; ++k) dv_push(&S->dims, &dm[k]);
                        const int64_t to = T->blocks.beginblock[Tsb], tao = T->blocks.beginblock[Thsb];
                        dv_push(&S->t_off, &to);
                        dv_push(&S->ta_off, &tao);
                        dv_push(&S->pref, &pref);
                        dv_push(&S->op_ptr, &first_pair);
                }
                if ((int) S->pref.n > entries_before) dv_push(&S->unit_ptr, &entries_before);
        }
        const int ne = (int) S->pref.n, np = (int) S->old_off.n;
        dv_push(&S->unit_ptr, &ne);
        dv_push(&S->op_ptr, &np);
}

static void pu_free(struct pu_sched *S)
{
        free(S->unit_ptr.a); free(S->dims.a); free(S->t_off.a); free(S->ta_off.a);
        free(S->pref.a); free(S->op_ptr.a); free(S->old_off.a); free(S->new_off.a);
        safe_free(S->old_base);
        safe_free(S->new_base);
}

static void pu_desc(const struct pu_sched *S, const struct rOperators *rops,
                    const struct siteTensor *T, t3ns_pupdate_desc *d)
{
        memset(d, 0, sizeof *d);
        d->is_left = rops->is_left == 1;
        d->nunits = (int) S->unit_ptr.n - 1;
        d->unit_ptr = S->unit_ptr.a;
        d->nentries = (int) S->pref.n;
        d->dims = S->dims.a;
        d->t_off = S->t_off.a;
        d->ta_off = S->ta_off.a;
        d->pref = S->pref.a;
        d->op_ptr = S->op_ptr.a;
        d->old_off = S->old_off.a;
        d->new_off = S->new_off.a;
        d->t_elems = T->blocks.beginblock[T->nrblocks];
        d->old_elems = S->old_elems;
        d->new_elems = S->new_elems;
}

void update_rOperators_physical(struct rOperators *rops, const struct siteTensor *tens,
                                const struct symsecs *internalss)
{
        struct pu_sched S;
        pu_compile(rops, tens, internalss, &S);
        t3ns_pupdate_desc d;
        pu_desc(&S, rops, tens, &d);

        double *old_tel = dropin_gather(rops, S.old_base);
        double *new_tel = safe_malloc(S.new_elems + 1, double);
        if (t3ns_pupdate_host(&d, tens->blocks.tel, old_tel, new_tel) != T3NS_OK) {
                fprintf(stderr, "t3ns drop-in: update_rOperators_physical: %s\n", t3ns_last_error());
                exit(EXIT_FAILURE);
        }
        struct rOperators *ur = &S.ur;
        dropin_scatter(ur, S.new_base, new_tel);
        safe_free(old_tel);
        safe_free(new_tel);
        /* the reference's cleanup_update (:181-190): the original set is
         * destroyed, all-zero blocks of the updated set are dropped */
        destroy_rOperators(rops);
        for (int i = 0; i < ur->nrops; ++i)
                kick_zero_blocks(&ur->operators[i], nblocks_in_operator(ur, i));
        *rops = *ur;
        pu_free(&S);
}

/* Test hook: the compiled schedule of a physical update, written without the
 * GPU (records "pu.*" in the step-file layout). */
int t3ns_dropin_pupdate_write(const struct rOperators *rops, const struct siteTensor *tens,
                              const struct symsecs *internalss, const char *path)
{
        struct pu_sched S;
        pu_compile(rops, tens, internalss, &S);
        FILE *f = fopen(path, "wb");
        if (!f) return -1;
        fwrite("T3NSCAP1", 1, 8, f);
        dropin_rec(f, "pu.unit_ptr", 1, S.unit_ptr.n, S.unit_ptr.a);
        dropin_rec(f, "pu.dims", 1, S.dims.n, S.dims.a);
        dropin_rec(f, "pu.t_off", 2, S.t_off.n, S.t_off.a);
        dropin_rec(f, "pu.ta_off", 2, S.ta_off.n, S.ta_off.a);
        dropin_rec(f, "pu.pref", 3, S.pref.n, S.pref.a);
        dropin_rec(f, "pu.op_ptr", 1, S.op_ptr.n, S.op_ptr.a);
        dropin_rec(f, "pu.old_off", 2, S.old_off.n, S.old_off.a);
        dropin_rec(f, "pu.new_off", 2, S.new_off.n, S.new_off.a);
        dropin_rec(f, "pu.new_base", 2, (int64_t) rops->nrops + 1, S.new_base);
        /* the updated set's block layout before zero-block removal */
        {
                struct dv_vec bb = {0, 0, 0, sizeof(int)};
                for (int i = 0; i < S.ur.nrops; ++i) {
                        const int nbn = nblocks_in_operator(&S.ur, i);
                        for (int b = 0; b <= nbn; ++b) dv_push(&bb, &S.ur.operators[i].beginblock[b]);
                }
                dropin_rec(f, "pu.new_beginblock", 1, bb.n, bb.a);
                free(bb.a);
        }
        const int il = rops->is_left == 1;
        dropin_rec(f, "pu.is_left", 1, 1, &il);
        fclose(f);
        destroy_rOperators(&S.ur);
        pu_free(&S);
        return 0;
}

/* ------------------------------------------------------------------ */
/* Appending a site operator: rOperators_append_phys (reference
 * include/rOperators.h:265-266, src/rOperators_pUpdate.c:665-673).
 *
 * The unique appended operators (init_unique_rOperators, :393-423) are built
 * from the instruction set of fetch_pUpdate; each of their blocks is the
 * original block scaled by prefactor_pAppend * el_siteop (pAppend_block,
 * :537-640); the GPU does the scaled copies, and the reference's own
 * sum_unique_rOperators (src/rOperators_init.c:228-265) combines them.   */

#include "instructions.h"
#include "hamiltonian.h"

struct pa_ops { int po, so, hss[3]; };

void rOperators_append_phys(struct rOperators *newrops, const struct rOperators *oldrops)
{
        const struct rOperators *or = oldrops;
        struct instructionset set = fetch_pUpdate(or->bond, or->is_left);
        const int site = netw.bonds[or->bond][or->is_left];
        int bonds[3];
        get_bonds_of_site(site, bonds);
        struct rOperators ur;
        dropin_init_unique(&ur, bonds[2 * or->is_left], or->is_left, true, &set);

        /* the unique instructions with their MPO sectors (compress_instructions) */
        struct pa_ops *ci = safe_malloc(set.nr_instr + 1, struct pa_ops);
        int nci = 0, cinstr = -1;
        while (get_next_unique_instr(&cinstr, &set)) {
                const int po = set.instr[cinstr].instr[0];
                const int so = set.instr[cinstr].instr[1];
                const int no = set.instr[cinstr].instr[2];
                ci[nci].po = po;
                ci[nci].so = so;
                ci[nci].hss[0] = or->hss_of_ops[po];
                ci[nci].hss[1] = symsec_siteop(so, site);
                ci[nci].hss[2] = set.hss_of_new[no];
                ++nci;
        }

        /* symsecs (init_append_data, :486-529) */
        struct symsecs uss[3][3], MPOss[3], oss[3];
        get_symsecs_arr(3, uss[0], bonds);
        get_symsecs_arr(3, uss[1], bonds);
        int b2[3] = {get_hamiltonianbond(bonds[0]), get_hamiltonianbond(bonds[1]),
                     get_hamiltonianbond(bonds[2])};
        get_symsecs_arr(3, MPOss, b2);
        b2[0] = get_braT3NSbond(ur.bond);
        b2[1] = get_ketT3NSbond(ur.bond);
        b2[2] = get_hamiltonianbond(ur.bond);
        get_symsecs_arr(3, uss[2], b2);
        const int pbond = 2 * !or->is_left;
        b2[0] = get_braT3NSbond(or->bond);
        b2[1] = get_ketT3NSbond(or->bond);
        b2[2] = get_hamiltonianbond(or->bond);
        get_symsecs_arr(3, oss, b2);

        int64_t *obase = dropin_op_bases(or);
        int64_t *ubase = dropin_op_bases(&ur);

        struct dv_vec dst = {0, 0, 0, sizeof(int64_t)}, src = {0, 0, 0, sizeof(int64_t)};
        struct dv_vec len = {0, 0, 0, sizeof(int)}, scl = {0, 0, 0, sizeof(double)};
        const int N = ur.begin_blocks_of_hss[ur.nrhss];
        for (int usb = 0; usb < N; ++usb) {
                const QN_TYPE *uqn = &ur.qnumbers[usb * 3];
                int ids[3][3];
                indexize(ids[0], uqn[0], uss[0]);
                indexize(ids[1], uqn[1], uss[1]);
                indexize(ids[2], uqn[2], uss[2]);
                const int hssn = ids[2][2];
                ids[2][pbond == 0 ? 2 : 0] = hssn;
                const int ublock = usb - ur.begin_blocks_of_hss[hssn];
                int *prods, nr_prods;
                tprods_ham(&nr_prods, &prods, hssn, site);
                for (int p = 0; p < nr_prods; ++p) {
                        const int hsss = prods[2 * p], hsso = prods[2 * p + 1];
                        ids[2][pbond] = hsso;
                        ids[2][1] = hsss;
                        const int id_old[3] = {ids[0][pbond], ids[1][pbond], ids[2][pbond]};
                        const QN_TYPE oqn = qntypize(id_old, oss);
                        const int *irr[3][3];
                        for (int i = 0; i < 2; ++i)
                                for (int j = 0; j < 3; ++j) irr[i][j] = uss[i][j].irreps[ids[i][j]];
                        for (int j = 0; j < 3; ++j) irr[2][j] = MPOss[j].irreps[ids[2][j]];
                        const double pref = prefactor_pAppend(irr, ur.is_left, bookie.sgs, bookie.nrSyms);
                        const QN_TYPE *oqn_arr = rOperators_give_qnumbers_for_hss(or, hsso);
                        const int nbl = rOperators_give_nr_blocks_for_hss(or, hsso);
                        const int oblock = binSearch(&oqn, oqn_arr, nbl, SORT_QN_TYPE, sizeof oqn);
                        if (oblock == -1 || COMPARE_ELEMENT_TO_ZERO(pref)) continue;
                        for (int i = 0; i < nci; ++i) {
                                if (!(ci[i].hss[0] == hsso && ci[i].hss[1] == hsss && ci[i].hss[2] == hssn))
                                        continue;
                                const struct sparseblocks *ob = &or->operators[ci[i].po];
                                const int n = get_size_block(ob, oblock);
                                if (!n) continue;
                                const double site_el = pref * el_siteop(ci[i].so, ids[0][1], ids[1][1]);
                                const int64_t d0 = ubase[i] + ur.operators[i].beginblock[ublock];
                                const int64_t s0 = obase[ci[i].po] + ob->beginblock[oblock];
                                dv_push(&dst, &d0);
                                dv_push(&src, &s0);
                                dv_push(&len, &n);
                                dv_push(&scl, &site_el);
                        }
                }
                safe_free(prods);
        }

        double *src_tel = dropin_gather(or, obase);
        t3ns_scalecopy_desc d = {(int) scl.n, dst.a, src.a, len.a, scl.a, obase[or->nrops],
                                 ubase[ur.nrops]};
        /* the scaled copies (the unique operators) are summed on the device
         * (sum_unique_rOperators, src/rOperators_init.c:228-265) */
        struct dropin_sum su;
        dropin_sum_build(&su, &ur, &set, ubase, newrops);
        if (t3ns_scalecopy_sum_host(&d, &su.d, src_tel, su.new_tel, su.new_begin, su.out_base) !=
            T3NS_OK) {
                fprintf(stderr, "t3ns drop-in: rOperators_append_phys: %s\n", t3ns_last_error());
                exit(EXIT_FAILURE);
        }
        dropin_sum_finish(&su, newrops);
        destroy_rOperators(&ur);   /* `set` is the reference's cached set: not ours to free */
        safe_free(src_tel);
        safe_free(obase);
        safe_free(ubase);
        safe_free(ci);
        free(dst.a); free(src.a); free(len.a); free(scl.a);
}
