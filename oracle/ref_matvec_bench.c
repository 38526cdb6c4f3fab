/* ref_matvec_bench: times the reference's own matvec on a captured step.
 *
 * TEST / BASELINE INFRASTRUCTURE: used only by bench.py's reference arm and
 * cpu_baseline leg.  It loads a step file (t3ns_b200/stepfile.py layout),
 * rebuilds the parts of the reference's struct Heffdata that the replay path
 * reads (siteObject block table, the three rOperators, the merge instruction
 * set and the replay schedule struct secondrun, include/Heff.h:36-155), and
 * calls the reference's matvecT3NS (src/Heff.c:1049-1062), which runs
 * exec_secondrun (src/Heff.c:945-1000) with OpenMP over new blocks and
 * OpenBLAS dgemm, exactly as inside the reference Davidson.
 *
 *   ref_matvec_bench STEPFILE [CALLS] [STRIDE]
 * prints one JSON line: seconds per matvec (median of CALLS), the algorithmic
 * FLOPs of the step, and the relative difference to the captured output.
 * With STRIDE > 1 only every STRIDE-th new block keeps its schedule (a
 * bounded sample of the step: the FLOPs reported are those of the kept
 * blocks, and the output comparison is skipped).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>

#include "Heff.h"

struct rec { char name[48]; int dtype; int64_t count; void *data; };
static struct rec *recs;
static int nrecs;

static void load(const char *path)
{
        FILE *f = fopen(path, "rb");
        if (!f) { perror(path); exit(2); }
        char magic[8];
        if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "T3NSCAP1", 8)) { fprintf(stderr, "bad file\n"); exit(2); }
        for (;;) {
                struct rec r;
                int32_t hdr[2];
                if (fread(r.name, 1, 48, f) != 48) break;
                if (fread(hdr, 4, 2, f) != 2 || fread(&r.count, 8, 1, f) != 1) exit(2);
                r.dtype = hdr[0];
                const size_t el = r.dtype == 1 ? 4 : 8;
                r.data = malloc(el * (size_t) (r.count ? r.count : 1));
                if (r.count && fread(r.data, el, (size_t) r.count, f) != (size_t) r.count) exit(2);
                recs = realloc(recs, sizeof *recs * (size_t) (nrecs + 1));
                recs[nrecs++] = r;
        }
        fclose(f);
}

static void *find(const char *name)
{
        for (int i = 0; i < nrecs; ++i)
                if (!strcmp(recs[i].name, name)) return recs[i].data;
        return NULL;
}

static void *get(const char *name)
{
        for (int i = 0; i < nrecs; ++i)
                if (!strcmp(recs[i].name, name)) return recs[i].data;
        fprintf(stderr, "missing record %s\n", name);
        exit(2);
}

static int geti(const char *name) { return *(int *) get(name); }

static double now(void)
{
        struct timeval t;
        gettimeofday(&t, NULL);
        return t.tv_sec + 1e-6 * t.tv_usec;
}

static int cmpd(const void *a, const void *b)
{
        double x = *(const double *) a, y = *(const double *) b;
        return x < y ? -1 : x > y;
}

int main(int argc, char **argv)
{
        if (argc < 2) { fprintf(stderr, "usage: %s STEPFILE [CALLS]\n", argv[0]); return 2; }
        load(argv[1]);
        const int calls = argc > 2 ? atoi(argv[2]) : 3;
        const int stride = argc > 3 ? atoi(argv[3]) : 1;
        struct Heffdata hd;
        memset(&hd, 0, sizeof hd);
        hd.isdmrg = geti("isdmrg");
        const int nops = hd.isdmrg ? 2 : 3;
        hd.posB = geti("posB");
        memcpy(hd.rOperators_on_site, get("rOperators_on_site"), 3 * sizeof(int));
        hd.siteObject.nrsites = geti("nrsites");
        const int nb = geti("nrblocks");
        hd.siteObject.nrblocks = nb;
        hd.siteObject.blocks.beginblock = get("beginblock");
        char nm[64];
        for (int i = 0; i < nops; ++i) {
                struct rOperators *op = &hd.Operators[i];
                snprintf(nm, sizeof nm, "ops%d.nrops", i);
                op->nrops = geti(nm);
                snprintf(nm, sizeof nm, "ops%d.P_operator", i);
                op->P_operator = geti(nm);
                if (!op->nrops) continue;
                snprintf(nm, sizeof nm, "ops%d.hss_of_ops", i);
                int *hss = get(nm);
                snprintf(nm, sizeof nm, "ops%d.begin_blocks_of_hss", i);
                int *bbh = get(nm);
                snprintf(nm, sizeof nm, "ops%d.beginblock", i);
                int *bb = get(nm);
                snprintf(nm, sizeof nm, "ops%d.tel", i);
                double *tel = find(nm);
                if (!tel) {
                        /* structure-only step file: any values do for timing */
                        snprintf(nm, sizeof nm, "ops%d.tel_len", i);
                        const int64_t n = *(int64_t *) get(nm);
                        tel = malloc(sizeof *tel * (size_t) (n ? n : 1));
                        uint64_t st = 2024u + (uint64_t) i;
                        for (int64_t e = 0; e < n; ++e) {
                                st = st * 6364136223846793005ull + 1442695040888963407ull;
                                tel[e] = ((double) (st >> 11) * 0x1.0p-53 - 0.5) * 0.2;
                        }
                }
                op->operators = calloc((size_t) op->nrops, sizeof *op->operators);
                int64_t pb = 0, pt = 0;
                for (int k = 0; k < op->nrops; ++k) {
                        const int n = bbh[hss[k] + 1] - bbh[hss[k]];
                        op->operators[k].beginblock = bb + pb;
                        op->operators[k].tel = tel + pt;
                        pt += bb[pb + n];
                        pb += n + 1;
                }
        }
        const int nri = geti("iset.nr_instr");
        int *ins = get("iset.instr");
        double *ipr = get("iset.pref");
        hd.iset.nr_instr = nri;
        hd.iset.instr = calloc((size_t) (nri ? nri : 1), sizeof *hd.iset.instr);
        for (int k = 0; k < nri; ++k) {
                for (int c = 0; c < 3; ++c) hd.iset.instr[k].instr[c] = ins[3 * k + c];
                hd.iset.instr[k].pref = ipr[k];
        }
        hd.iset.nrMPOc = geti("iset.nrMPOc");
        hd.iset.MPOc_beg = get("iset.MPOc_beg");
        hd.iset.MPOc = get("iset.MPOc");

        /* replay schedule */
        int *dims = get("sr.dims"), *pptr = get("sr.pair_ptr"), *pold = get("sr.pair_old");
        int *pord = get("sr.pair_order"), *csb = get("sr.combo_sbops"), *cmpo = get("sr.combo_mpo");
        int64_t *cptr = get("sr.combo_ptr");
        double *cpref = get("sr.combo_pref");
        memcpy(hd.sr.worksize, get("sr.worksize"), 2 * sizeof(int));
        hd.sr.dimsofsb = malloc(sizeof *hd.sr.dimsofsb * (size_t) nb);
        hd.sr.nr_oldsb = malloc(sizeof *hd.sr.nr_oldsb * (size_t) nb);
        hd.sr.ntom = malloc(sizeof *hd.sr.ntom * (size_t) nb);
        hd.sr.shufid = malloc(sizeof *hd.sr.shufid * (size_t) nb);
        static const int ord3[6][3] = {{0,1,2},{1,0,2},{0,2,1},{1,2,0},{2,0,1},{2,1,0}};
        static const int ord2[2][2] = {{0,1},{1,0}};
        double flops = 0, flops_full = 0;
        for (int i = 0; i < nb; ++i) {
                for (int k = 0; k < 3; ++k) hd.sr.dimsofsb[i][k] = dims[3 * i + k];
                const int sampled = i % stride == 0;
                const int npr = pptr[i + 1] - pptr[i];
                hd.sr.nr_oldsb[i] = sampled ? npr : 0;
                hd.sr.ntom[i] = malloc(sizeof **hd.sr.ntom * (size_t) (npr + 1));
                /* every block's pairs are counted (flops_full); only the
                 * sampled blocks keep them in the replay schedule */
                for (int j = 0; j < npr; ++j) {
                        const int p = pptr[i] + j;
                        struct newtooldmatvec *t = &hd.sr.ntom[i][j];
                        t->oldsb = pold[p];
                        t->bestorder = pord[p];
                        t->nmbr = (int) (cptr[p + 1] - cptr[p]);
                        t->sbops = (int (*)[3]) (csb + 3 * cptr[p]);
                        t->prefactor = cpref + cptr[p];
                        t->MPO = cmpo + cptr[p];
                        /* algorithmic FLOPs: reference order, present instructions */
                        const int *o = hd.isdmrg ? ord2[pord[p]] : ord3[pord[p]];
                        int w[3] = {dims[3 * t->oldsb], dims[3 * t->oldsb + 1],
                                    hd.isdmrg ? 1 : dims[3 * t->oldsb + 2]};
                        const int dn[3] = {dims[3 * i], dims[3 * i + 1], hd.isdmrg ? 1 : dims[3 * i + 2]};
                        double fl = 0;
                        for (int s = 0; s < nops; ++s) {
                                fl += (double) w[0] * w[1] * w[2] * dn[o[s]];
                                w[o[s]] = dn[o[s]];
                        }
                        for (int c = 0; c < t->nmbr; ++c) {
                                const int m = t->MPO[c];
                                for (int k = hd.iset.MPOc_beg[m]; k < hd.iset.MPOc_beg[m + 1]; ++k) {
                                        int ok = 1;
                                        for (int q = 0; q < nops && ok; ++q) {
                                                const int *b = hd.Operators[q].operators[hd.iset.instr[k].instr[q]].beginblock;
                                                const int sb = t->sbops[c][q];
                                                ok = b[sb] != b[sb + 1];
                                        }
                                        if (ok) {
                                                flops_full += 2 * fl;
                                                if (sampled) flops += 2 * fl;
                                        }
                                }
                        }
                }
        }
        srand(0);
        for (int i = 0; i < nb; ++i) hd.sr.shufid[i] = i;
        for (int i = nb - 1; i > 0; --i) {
                const int j = rand() % (i + 1);
                const int tmp = hd.sr.shufid[j];
                hd.sr.shufid[j] = hd.sr.shufid[i];
                hd.sr.shufid[i] = tmp;
        }

        const int size = hd.siteObject.blocks.beginblock[nb];
        double *x = find("x1"), *yref = find("y1");
        double *y = malloc(sizeof *y * (size_t) size);
        if (!x) {
                x = malloc(sizeof *x * (size_t) size);
                for (int i = 0; i < size; ++i) x[i] = 1.0 / sqrt((double) size);
        }
        double *ts = malloc(sizeof *ts * (size_t) (calls > 0 ? calls : 1));
        for (int c = 0; c < calls; ++c) {
                const double t0 = now();
                matvecT3NS(x, y, &hd);
                ts[c] = now() - t0;
        }
        double dn2 = 0, rn2 = 0;
        for (int i = 0; i < size && stride == 1 && yref; ++i) {
                dn2 += (y[i] - yref[i]) * (y[i] - yref[i]);
                rn2 += yref[i] * yref[i];
        }
        qsort(ts, (size_t) calls, sizeof *ts, cmpd);
        printf("{\"seconds_per_matvec\": %.6e, \"calls\": %d, \"flops\": %.6e, "
               "\"flops_full\": %.6e, \"sampled_blocks\": %d, \"blocks\": %d, "
               "\"rel_diff_vs_capture\": %.3e, \"size\": %d, \"stride\": %d}\n",
               ts[calls / 2], calls, flops, flops_full, (nb + stride - 1) / stride, nb,
               sqrt(dn2 / (rn2 > 0 ? rn2 : 1)), size, stride);
        return 0;
}
