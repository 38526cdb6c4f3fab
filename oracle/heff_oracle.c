/* CPU restatement of the reference effective-Hamiltonian matvec and diagonal.
 *
 * TEST INFRASTRUCTURE (the oracle).  Only the tests, smoke() and bench.py's
 * cpu_baseline leg may load it, as a checker.  The product library never
 * links or calls it.
 *
 * It consumes the same flattened schedule as the engine (t3ns_heff_desc,
 * include/t3ns_b200.h) and follows the reference step by step:
 *   - matvecT3NS / exec_secondrun (reference src/Heff.c:945-1000): result is
 *     zeroed, then every new block accumulates over its (old block, MPO
 *     combo) entries;
 *   - execute_heffcontr (src/Heff.c:916-943): for every instruction of the
 *     combo whose three operator blocks are all non-empty
 *     (find_operator_tel, src/Heff.c:798-813), the three operators are
 *     applied one after the other in the pair's order, the last one scaled by
 *     instr.pref * prefactor and accumulated into the new block
 *     (do_contract, src/sparseblocks.c:133-158, alpha/beta as called);
 *   - the stage shapes follow prepare_cinfo_T3NS / prepare_cinfo_DMRG
 *     (src/Heff.c:526-627): operator blocks are (new x old) column-major and
 *     memory axis j of a block carries operator map[j];
 *   - make_diagonal / diag_old_to_new_sb (src/Heff.c:1064-1108, 1268-1312).
 * Plain loops in double precision, no BLAS.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "t3ns_b200.h"

static const int orders3[6][3] = {{0, 1, 2}, {1, 0, 2}, {0, 2, 1},
                                  {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
static const int orders2[2][2] = {{0, 1}, {1, 0}};

/* out = op (r x d[ax]) applied on axis ax of in (d0,d1,d2), column-major */
static void apply_axis(int ax, const int d[3], int r, const double *op,
                       const double *in, double *out, double alpha, int accumulate)
{
        int od[3] = {d[0], d[1], d[2]};
        od[ax] = r;
        const int64_t osz = (int64_t) od[0] * od[1] * od[2];
        double *tmp = malloc(sizeof *tmp * (size_t) (osz ? osz : 1));
        for (int c = 0; c < od[2]; ++c)
                for (int b = 0; b < od[1]; ++b)
                        for (int a = 0; a < od[0]; ++a) {
                                int idx[3] = {a, b, c};
                                const int row = idx[ax];
                                double s = 0;
                                for (int k = 0; k < d[ax]; ++k) {
                                        idx[ax] = k;
                                        s += op[row + (int64_t) k * r] *
                                             in[idx[0] + (int64_t) d[0] * (idx[1] + (int64_t) d[1] * idx[2])];
                                }
                                tmp[a + (int64_t) od[0] * (b + (int64_t) od[1] * c)] = alpha * s;
                        }
        for (int64_t e = 0; e < osz; ++e) out[e] = accumulate ? out[e] + tmp[e] : tmp[e];
        free(tmp);
}

static const double *op_block(const t3ns_ropset *rs, int op, int sb, int *sz)
{
        const int *bb = rs->op_beginblock[op];
        *sz = bb[sb + 1] - bb[sb];
        return rs->op_tel[op] + bb[sb];
}

/* Accumulates new block nb of the matvec into y (zeroed by the caller). */
static void matvec_block(const t3ns_heff_desc *d, const double *x, double *y, int nb)
{
        const int nops = d->isdmrg ? 2 : 3;
        int map[3] = {0, 1, 2}, inv[3] = {0, 1, 2};
        if (!d->isdmrg)
                for (int j = 0; j < 3; ++j) { map[j] = d->map[j]; inv[map[j]] = j; }
        {
                int dn[3];
                for (int j = 0; j < 3; ++j) dn[j] = d->dims[3 * nb + map[j]];
                if (d->isdmrg) dn[2] = 1;
                for (int p = d->pair_ptr[nb]; p < d->pair_ptr[nb + 1]; ++p) {
                        const int ob = d->pair_old[p];
                        int dold[3];
                        for (int j = 0; j < 3; ++j) dold[j] = d->dims[3 * ob + map[j]];
                        if (d->isdmrg) dold[2] = 1;
                        const int *o = d->isdmrg ? orders2[d->pair_order[p]]
                                                 : orders3[d->pair_order[p]];
                        for (int64_t c = d->combo_ptr[p]; c < d->combo_ptr[p + 1]; ++c) {
                                const int m = d->combo_mpo[c];
                                for (int k = d->MPOc_beg[m]; k < d->MPOc_beg[m + 1]; ++k) {
                                        const double *opb[3] = {0, 0, 0};
                                        int ok = 1;
                                        for (int i = 0; i < nops; ++i) {
                                                int sz;
                                                opb[i] = op_block(&d->ops[i], d->instr[3 * k + i],
                                                                  d->combo_sbops[3 * c + i], &sz);
                                                if (sz == 0) { ok = 0; break; }
                                        }
                                        if (!ok) continue;
                                        const double pref = d->instr_pref[k] * d->combo_pref[c];
                                        int w[3] = {dold[0], dold[1], dold[2]};
                                        const double *in = x + d->block_off[ob];
                                        double *bufs[2] = {0, 0};
                                        for (int s = 0; s < nops; ++s) {
                                                const int opi = o[s];
                                                const int ax = d->isdmrg ? opi : inv[opi];
                                                const int last = s == nops - 1;
                                                int od[3] = {w[0], w[1], w[2]};
                                                od[ax] = dn[ax];
                                                double *out;
                                                if (last) {
                                                        out = y + d->block_off[nb];
                                                } else {
                                                        const int64_t osz = (int64_t) od[0] * od[1] * od[2];
                                                        bufs[s] = malloc(sizeof(double) * (size_t) (osz ? osz : 1));
                                                        out = bufs[s];
                                                }
                                                apply_axis(ax, w, dn[ax], opb[opi], in, out,
                                                           last ? pref : 1.0, last);
                                                w[ax] = dn[ax];
                                                in = out;
                                        }
                                        free(bufs[0]);
                                        free(bufs[1]);
                                }
                        }
                }
        }
}

int t3ns_oracle_matvec(const t3ns_heff_desc *d, const double *x, double *y)
{
        memset(y, 0, sizeof *y * (size_t) d->block_off[d->nblocks]);
        for (int nb = 0; nb < d->nblocks; ++nb) matvec_block(d, x, y, nb);
        return 0;
}

/* The matvec restricted to the new blocks blocks[0..n): those blocks of y are
 * computed exactly as t3ns_oracle_matvec computes them, every other element
 * of y is left untouched.  Lets the tests check large steps on a sample of
 * blocks in bounded CPU time. */
int t3ns_oracle_matvec_blocks(const t3ns_heff_desc *d, const double *x, double *y,
                              const int *blocks, int n)
{
        for (int i = 0; i < n; ++i) {
                const int nb = blocks[i];
                if (nb < 0 || nb >= d->nblocks) return -1;
                const int64_t b0 = d->block_off[nb], b1 = d->block_off[nb + 1];
                memset(y + b0, 0, sizeof *y * (size_t) (b1 - b0));
                matvec_block(d, x, y, nb);
        }
        return 0;
}

int t3ns_oracle_diagonal(const t3ns_heff_desc *d, double *diag)
{
        const int nops = d->isdmrg ? 2 : 3;
        int map[3] = {0, 1, 2};
        if (!d->isdmrg)
                for (int j = 0; j < 3; ++j) map[j] = d->map[j];
        memset(diag, 0, sizeof *diag * (size_t) d->block_off[d->nblocks]);
        for (int nb = 0; nb < d->nblocks; ++nb) {
                int dn[3];
                for (int j = 0; j < 3; ++j) dn[j] = d->dims[3 * nb + map[j]];
                if (d->isdmrg) dn[2] = 1;
                for (int p = d->pair_ptr[nb]; p < d->pair_ptr[nb + 1]; ++p) {
                        if (d->pair_old[p] != nb) continue;
                        for (int64_t c = d->combo_ptr[p]; c < d->combo_ptr[p + 1]; ++c) {
                                const int m = d->combo_mpo[c];
                                for (int k = d->MPOc_beg[m]; k < d->MPOc_beg[m + 1]; ++k) {
                                        const double *opb[3] = {0, 0, 0};
                                        int ok = 1;
                                        for (int i = 0; i < nops; ++i) {
                                                int sz;
                                                opb[i] = op_block(&d->ops[i], d->instr[3 * k + i],
                                                                  d->combo_sbops[3 * c + i], &sz);
                                                if (sz == 0) { ok = 0; break; }
                                        }
                                        if (!ok) continue;
                                        const double pref = d->instr_pref[k] * d->combo_pref[c];
                                        /* memory axis j carries operator map[j] */
                                        const double *X = opb[map[0]], *Y = opb[map[1]];
                                        const double *Z = d->isdmrg ? NULL : opb[map[2]];
                                        double *t = diag + d->block_off[nb];
                                        for (int cc = 0; cc < dn[2]; ++cc) {
                                                const double ek = pref * (Z ? Z[cc + (int64_t) cc * dn[2]] : 1.0);
                                                for (int b = 0; b < dn[1]; ++b) {
                                                        const double ekn = ek * Y[b + (int64_t) b * dn[1]];
                                                        for (int a = 0; a < dn[0]; ++a, ++t)
                                                                *t += ekn * X[a + (int64_t) a * dn[0]];
                                                }
                                        }
                                }
                        }
                }
        }
        return 0;
}
