/* The device sum of unique operators shared by the operator drop-ins
 * (sum_dropin.c): the descriptor arrays of t3ns_sum_unique_host built from a
 * unique set and its instruction set, and the new set filled from the
 * engine's output. */
#pragma once
#include "dropin_util.h"
#include "t3ns_b200.h"

struct dropin_sum {
        t3ns_sumunique_desc d;
        int64_t *begin_ptr, *new_base, *instr_src, *out_base;
        int *begin, *new_begin, *instr_ptr;
        double *instr_pref, *new_tel;
};

/* Builds the descriptor for summing `ur` (unique operators at element
 * offsets ubase of their concatenation) with `set`, and the new set's
 * metadata in *res (its operators are filled by dropin_sum_finish). */
void dropin_sum_build(struct dropin_sum *S, const struct rOperators *ur,
                      const struct instructionset *set, const int64_t *ubase,
                      struct rOperators *res);

/* Moves the engine's output (S->new_tel, new_begin, out_base) into the
 * operators of *res and frees the descriptor arrays. */
void dropin_sum_finish(struct dropin_sum *S, struct rOperators *res);
