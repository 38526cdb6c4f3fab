/* Helpers shared by the renormalised-operator drop-ins: a growable array for
 * the compiled schedules, and the unique-operator set an instruction set
 * builds before its operators are summed. */
#pragma once
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "instructions.h"
#include "macros.h"
#include "rOperators.h"
#include "sparseblocks.h"

struct dv_vec { void *a; int64_t n, cap; size_t el; };

static inline void dv_push(struct dv_vec *v, const void *x)
{
        if (v->n == v->cap) {
                v->cap = v->cap ? 2 * v->cap : 256;
                v->a = realloc(v->a, v->el * (size_t) v->cap);
                if (!v->a) { fprintf(stderr, "t3ns drop-in: out of memory\n"); exit(EXIT_FAILURE); }
        }
        memcpy((char *) v->a + v->el * (size_t) v->n++, x, v->el);
}

/* One operator per unique instruction of `set`, in the order
 * get_next_unique_instr visits them, each with the MPO sector of the
 * instruction's new operator and zero-filled blocks (the reference's
 * init_uniqueOperators, src/rOperators_bUpdate.c:251-290, and
 * init_unique_rOperators, src/rOperators_pUpdate.c:393-423). */
static inline void dropin_init_unique(struct rOperators *ur, int bond, int is_left,
                                      bool P_operator, const struct instructionset *set)
{
        int **tmpbb;
        init_rOperators(ur, &tmpbb, bond, is_left, P_operator);
        int cinstr = -1;
        ur->nrops = 0;
        while (get_next_unique_instr(&cinstr, set)) ++ur->nrops;
        ur->hss_of_ops = safe_malloc(ur->nrops, *ur->hss_of_ops);
        int count = 0;
        cinstr = -1;
        while (get_next_unique_instr(&cinstr, set))
                ur->hss_of_ops[count++] = set->hss_of_new[set->instr[cinstr].instr[2]];
        ur->operators = safe_malloc(ur->nrops, *ur->operators);
        for (int i = 0; i < ur->nrops; ++i) {
                const int chss = ur->hss_of_ops[i];
                init_sparseblocks(&ur->operators[i], tmpbb[chss],
                                  rOperators_give_nr_blocks_for_hss(ur, chss), 'c');
        }
        for (int i = 0; i < ur->nrhss; ++i) safe_free(tmpbb[i]);
        safe_free(tmpbb);
}

/* Element offsets of every operator of `r` in the concatenation of their
 * element arrays ([nrops + 1], malloc'd). */
static inline int64_t *dropin_op_bases(const struct rOperators *r)
{
        int64_t *b = safe_malloc(r->nrops + 1, int64_t);
        b[0] = 0;
        for (int i = 0; i < r->nrops; ++i)
                b[i + 1] = b[i] + r->operators[i].beginblock[nblocks_in_operator(r, i)];
        return b;
}

/* Concatenated copy of the operators' elements (malloc'd, at least one
 * element so an empty set still has a valid pointer). */
static inline double *dropin_gather(const struct rOperators *r, const int64_t *base)
{
        double *t = safe_malloc(base[r->nrops] + 1, double);
        for (int i = 0; i < r->nrops; ++i)
                if (base[i + 1] > base[i])
                        memcpy(t + base[i], r->operators[i].tel,
                               sizeof(double) * (size_t) (base[i + 1] - base[i]));
        return t;
}

static inline void dropin_scatter(struct rOperators *r, const int64_t *base, const double *t)
{
        for (int i = 0; i < r->nrops; ++i)
                if (base[i + 1] > base[i])
                        memcpy(r->operators[i].tel, t + base[i],
                               sizeof(double) * (size_t) (base[i + 1] - base[i]));
}

/* Schedule-record writer in the step-file layout ("T3NSCAP1", then records of
 * a 48-byte name, an int32 type (1 int32, 2 int64, 3 double), an int32 pad,
 * an int64 count and the payload). */
static inline void dropin_rec(FILE *f, const char *name, int type, int64_t count, const void *a)
{
        char nm[48] = {0};
        strncpy(nm, name, sizeof nm - 1);
        int32_t hdr[2] = {type, 0};
        fwrite(nm, 1, sizeof nm, f);
        fwrite(hdr, sizeof hdr, 1, f);
        fwrite(&count, sizeof count, 1, f);
        if (count) fwrite(a, type == 1 ? 4 : 8, (size_t) count, f);
}
