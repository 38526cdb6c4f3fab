/* Drop-in sum of unique renormalised operators on the GPU.
 *
 * Replaces sum_unique_rOperators (reference include/rOperators.h:159-160,
 * src/rOperators_init.c:228-265): the new set has one operator per distinct
 * instr[2] of the instruction set, with the MPO sector set->hss_of_new[k]
 * and the block layout of the unique operators of that sector
 * (init_sum_unique, :191-226); each instruction adds pref times its unique
 * operator (the unique operator advances whenever instr[0], instr[1] or the
 * new operator's sector changes, as the reference walks them), and blocks
 * that come out zero are removed (kick_zero_blocks,
 * src/sparseblocks.c:73-107).  The sums and the zero test run on the device
 * (t3ns_sum_unique_host); the branching update and the site-operator append
 * hand their unique operators over on the device (t3ns_bupdate_sum_host,
 * t3ns_scalecopy_sum_host), so only the summed set comes back. */
#include "dropin_sum.h"

/* The new set's metadata: the unique set's bond, sectors and quantum
 * numbers (deep copies), one operator per new index with its sector. */
static void su_metadata(const struct rOperators *ur, const struct instructionset *set,
                        struct rOperators *res)
{
        *res = *ur;
        res->begin_blocks_of_hss = safe_malloc(ur->nrhss + 1, int);
        for (int i = 0; i < ur->nrhss + 1; ++i) res->begin_blocks_of_hss[i] = ur->begin_blocks_of_hss[i];
        const int nq = ur->begin_blocks_of_hss[ur->nrhss] * rOperators_give_nr_of_couplings(ur);
        res->qnumbers = safe_malloc(nq, QN_TYPE);
        for (int i = 0; i < nq; ++i) res->qnumbers[i] = ur->qnumbers[i];
        res->nrops = 0;
        for (int i = 0; i < set->nr_instr; ++i)
                if (set->instr[i].instr[2] + 1 > res->nrops) res->nrops = set->instr[i].instr[2] + 1;
        res->hss_of_ops = safe_malloc(res->nrops, int);
        res->operators = safe_malloc(res->nrops, struct sparseblocks);
        for (int k = 0; k < res->nrops; ++k) res->hss_of_ops[k] = set->hss_of_new[k];
}

void dropin_sum_build(struct dropin_sum *S, const struct rOperators *ur,
                      const struct instructionset *set, const int64_t *ubase,
                      struct rOperators *res)
{
        su_metadata(ur, set, res);
        const int nnew = res->nrops;
        S->begin_ptr = safe_malloc(nnew + 1, int64_t);
        S->new_base = safe_malloc(nnew + 1, int64_t);
        S->instr_ptr = safe_malloc(nnew + 1, int);
        S->instr_src = safe_malloc(set->nr_instr + 1, int64_t);
        S->instr_pref = safe_malloc(set->nr_instr + 1, double);
        /* block layout of each new operator: that of the first unique operator
         * of its sector */
        int64_t nbeg = 0, nel = 0;
        int *proto = safe_malloc(nnew + 1, int);
        for (int k = 0; k < nnew; ++k) {
                int j = 0;
                while (j < ur->nrops && ur->hss_of_ops[j] != res->hss_of_ops[k]) ++j;
                if (j == ur->nrops) {
                        fprintf(stderr, "t3ns drop-in: sum_unique_rOperators: no unique operator "
                                        "of sector %d\n", res->hss_of_ops[k]);
                        exit(EXIT_FAILURE);
                }
                proto[k] = j;
                const int nb = rOperators_give_nr_blocks_for_hss(res, res->hss_of_ops[k]);
                S->begin_ptr[k] = nbeg;
                S->new_base[k] = nel;
                nbeg += nb + 1;
                nel += ur->operators[j].beginblock[nb];
        }
        S->begin_ptr[nnew] = nbeg;
        S->new_base[nnew] = nel;
        S->begin = safe_malloc(nbeg + 1, int);
        S->new_begin = safe_malloc(nbeg + 1, int);
        for (int k = 0; k < nnew; ++k) {
                const int nb = (int) (S->begin_ptr[k + 1] - S->begin_ptr[k] - 1);
                for (int b = 0; b <= nb; ++b)
                        S->begin[S->begin_ptr[k] + b] = ur->operators[proto[k]].beginblock[b];
        }
        safe_free(proto);
        /* instructions in order, each with its unique operator, grouped by the
         * new operator they write (a stable grouping keeps the order) */
        int *uid = safe_malloc(set->nr_instr + 1, int);
        int u = 0;
        for (int i = 0; i < set->nr_instr; ++i) {
                const int *in = set->instr[i].instr;
                if (i > 0) {
                        const int *pin = set->instr[i - 1].instr;
                        if (in[0] != pin[0] || in[1] != pin[1] ||
                            set->hss_of_new[in[2]] != set->hss_of_new[pin[2]])
                                ++u;
                }
                uid[i] = u;
        }
        if (set->nr_instr > 0 && u + 1 != ur->nrops) {
                fprintf(stderr, "t3ns drop-in: sum_unique_rOperators: %d unique operators for "
                                "%d unique instructions\n", ur->nrops, u + 1);
                exit(EXIT_FAILURE);
        }
        for (int k = 0; k <= nnew; ++k) S->instr_ptr[k] = 0;
        for (int i = 0; i < set->nr_instr; ++i) ++S->instr_ptr[set->instr[i].instr[2] + 1];
        for (int k = 0; k < nnew; ++k) S->instr_ptr[k + 1] += S->instr_ptr[k];
        int *fill = safe_malloc(nnew + 1, int);
        for (int k = 0; k < nnew; ++k) fill[k] = S->instr_ptr[k];
        for (int i = 0; i < set->nr_instr; ++i) {
                const int k = set->instr[i].instr[2];
                S->instr_src[fill[k]] = ubase[uid[i]];
                S->instr_pref[fill[k]] = set->instr[i].pref;
                ++fill[k];
        }
        safe_free(fill);
        safe_free(uid);
        S->out_base = safe_malloc(nnew + 1, int64_t);
        S->new_tel = safe_malloc(nel + 1, double);
        memset(&S->d, 0, sizeof S->d);
        S->d.nnew = nnew;
        S->d.begin_ptr = S->begin_ptr;
        S->d.begin = S->begin;
        S->d.new_base = S->new_base;
        S->d.instr_ptr = S->instr_ptr;
        S->d.instr_src = S->instr_src;
        S->d.instr_pref = S->instr_pref;
        S->d.unique_elems = ubase[ur->nrops];
}

void dropin_sum_finish(struct dropin_sum *S, struct rOperators *res)
{
        for (int k = 0; k < res->nrops; ++k) {
                struct sparseblocks *op = &res->operators[k];
                const int nb = (int) (S->begin_ptr[k + 1] - S->begin_ptr[k] - 1);
                op->beginblock = safe_malloc(nb + 1, int);
                for (int b = 0; b <= nb; ++b) op->beginblock[b] = S->new_begin[S->begin_ptr[k] + b];
                const int64_t n = S->out_base[k + 1] - S->out_base[k];
                op->tel = safe_malloc(n > 0 ? n : 1, double);
                if (n > 0) memcpy(op->tel, S->new_tel + S->out_base[k], sizeof(double) * (size_t) n);
        }
        safe_free(S->begin_ptr);
        safe_free(S->begin);
        safe_free(S->new_begin);
        safe_free(S->new_base);
        safe_free(S->instr_ptr);
        safe_free(S->instr_src);
        safe_free(S->instr_pref);
        safe_free(S->out_base);
        safe_free(S->new_tel);
}

struct rOperators sum_unique_rOperators(const struct rOperators *ur, const struct instructionset *set)
{
        struct rOperators res;
        int64_t *ubase = dropin_op_bases(ur);
        struct dropin_sum S;
        dropin_sum_build(&S, ur, set, ubase, &res);
        double *utel = dropin_gather(ur, ubase);
        if (t3ns_sum_unique_host(&S.d, utel, S.new_tel, S.new_begin, S.out_base) != T3NS_OK) {
                fprintf(stderr, "t3ns drop-in: sum_unique_rOperators: %s\n", t3ns_last_error());
                exit(EXIT_FAILURE);
        }
        dropin_sum_finish(&S, &res);
        safe_free(utel);
        safe_free(ubase);
        return res;
}
