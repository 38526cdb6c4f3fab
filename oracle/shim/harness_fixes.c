/* Harness-side workarounds linked into the reference oracle / driver builds.
 * Test infrastructure: never part of the product library.
 *
 * 1. glibc realloc(p, 0) frees p and returns NULL; several reference routines
 *    (src/Heff.c:1031-1038, src/Heff.c:354-356) treat that NULL as an
 *    out-of-memory failure and exit.  The link maps size 0 to size 1
 *    (-Wl,--wrap=realloc).
 * 2. src/instructions.c:204 calls NN_H_fetch_merge(instr, bond) although the
 *    second parameter is isdmrg (src/instructions_nn_hubbard.c:262), so every
 *    Hubbard T3NS merge at bond != 0 gets the two-operator DMRG list.  The
 *    build renames the reference's fetch_merge and its NN_H_fetch_merge
 *    reference inside instructions.o (objcopy --redefine-sym) so that the
 *    public fetch_merge below records isdmrg and the Hubbard call receives it.
 */
#include <stddef.h>

struct instructionset;

void *__real_realloc(void *p, size_t n);
void *__wrap_realloc(void *p, size_t n) { return __real_realloc(p, n ? n : 1); }

/* The layout of struct instructionset is only needed by value here; it is
 * returned as an opaque blob of the right size by the renamed original. */
#include "instructions.h"

struct instructionset t3ns_fix_fetch_merge_orig(const int bond, int isdmrg, int **hss_ops);
void NN_H_fetch_merge(struct instructionset *instr, int isdmrg);

static __thread int t3ns_fix_isdmrg;

struct instructionset fetch_merge(const int bond, int isdmrg, int **hss_ops)
{
        t3ns_fix_isdmrg = isdmrg;
        return t3ns_fix_fetch_merge_orig(bond, isdmrg, hss_ops);
}

void t3ns_fix_NN_H_fetch_merge(struct instructionset *instr, int bond_unused)
{
        (void) bond_unused;
        NN_H_fetch_merge(instr, t3ns_fix_isdmrg);
}
