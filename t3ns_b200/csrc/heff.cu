// Effective-Hamiltonian matvec engine: plan construction and FP64 kernels.
//
// The matvec (reference src/Heff.c:945-1000, execute_heffcontr :916-943)
// computes, for every new (output) block n of the site tensor,
//
//   Psi'[n] = sum_{old o} sum_{MPO combo c} sum_{instr i in c}
//             pref_i * pref_c * (X_i (x) Y_i (x) Z_i) Psi[o]
//
// where X_i, Y_i, Z_i are the operator blocks acting on the three memory
// axes of the block (memory axis j carries operator map[j]; reference
// make_map, src/Heff.c:668-682) and each block is stored column-major with
// the leg of axis 0 fastest.  The reference applies the three operators one
// at a time with cblas_dgemm (do_contract, src/sparseblocks.c:133-158) in the
// order chosen per (new, old) pair by make_cinfo (src/Heff.c:629-666).
//
// Here the host flattens the schedule into one task per (pair, instruction)
// whose three operator blocks are all present (find_operator_tel,
// src/Heff.c:798-813), groups the tasks by output block, and one persistent
// kernel walks them: each CTA owns whole output blocks (no atomics, as the
// reference owns a new block per OpenMP thread) and runs the three
// contractions of a task through shared-memory tiles, with the two
// intermediates in a per-CTA scratch slice that stays resident in L2.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "common.h"
#include "heff_internal.h"

namespace t3ns {

// ---------------------------------------------------------------------------
// CTA-wide FP64 GEMM on 64x64 output tiles, 256 threads, k-chunks of 16.
//   C_l = alpha * A_l * op(B_l) + beta * C_l,  l < L, all column-major,
//   op(B) = B (TB = false) or B^T (TB = true).
// beta == 0 never reads C.  Every access is bounds-checked against M, N, K.
template <bool TB>
__device__ void cta_gemm(int M, int N, int K, int L,
                         const double *__restrict__ A, int lda, int64_t sA,
                         const double *__restrict__ B, int ldb, int64_t sB,
                         double *C, int ldc, int64_t sC,
                         double alpha, double beta, double (*As)[65], double (*Bs)[65])
{
        const int tid = threadIdx.x;
        const int tx = tid & 15, ty = tid >> 4;
        const int tilesM = (M + 63) >> 6, tilesN = (N + 63) >> 6;
        for (int l = 0; l < L; ++l) {
                const double *Al = A + l * sA;
                const double *Bl = B + l * sB;
                double *Cl = C + l * sC;
                for (int tile = 0; tile < tilesM * tilesN; ++tile) {
                        const int m0 = (tile % tilesM) << 6;
                        const int n0 = (tile / tilesM) << 6;
                        double acc[4][4];
#pragma unroll
                        for (int i = 0; i < 4; ++i)
#pragma unroll
                                for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
                        for (int k0 = 0; k0 < K; k0 += 16) {
#pragma unroll
                                for (int r = 0; r < 4; ++r) {
                                        const int e = tid + 256 * r;
                                        const int m = e & 63, k = e >> 6;
                                        const int gm = m0 + m, gk = k0 + k;
                                        As[k][m] = (gm < M && gk < K)
                                                ? Al[gm + (int64_t) gk * lda] : 0.0;
                                }
#pragma unroll
                                for (int r = 0; r < 4; ++r) {
                                        const int e = tid + 256 * r;
                                        int n, k;
                                        if (TB) { n = e & 63; k = e >> 6; }
                                        else { k = e & 15; n = e >> 4; }
                                        const int gn = n0 + n, gk = k0 + k;
                                        double v = 0.0;
                                        if (gn < N && gk < K)
                                                v = TB ? Bl[gn + (int64_t) gk * ldb]
                                                       : Bl[gk + (int64_t) gn * ldb];
                                        Bs[k][n] = v;
                                }
                                __syncthreads();
#pragma unroll
                                for (int k = 0; k < 16; ++k) {
                                        double a[4], b[4];
#pragma unroll
                                        for (int i = 0; i < 4; ++i) a[i] = As[k][tx + 16 * i];
#pragma unroll
                                        for (int j = 0; j < 4; ++j) b[j] = Bs[k][ty + 16 * j];
#pragma unroll
                                        for (int i = 0; i < 4; ++i)
#pragma unroll
                                                for (int j = 0; j < 4; ++j)
                                                        acc[i][j] = fma(a[i], b[j], acc[i][j]);
                                }
                                __syncthreads();
                        }
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                                const int m = m0 + tx + 16 * i;
                                if (m >= M) continue;
#pragma unroll
                                for (int j = 0; j < 4; ++j) {
                                        const int n = n0 + ty + 16 * j;
                                        if (n >= N) continue;
                                        double *c = Cl + m + (int64_t) n * ldc;
                                        const double v = alpha * acc[i][j];
                                        *c = beta == 0.0 ? v : fma(beta, *c, v);
                                }
                        }
                }
        }
}

// Applies the (r x s) operator block `op` on memory axis `ax` of the tensor
// `in` with dims d[3] (d[ax] == s), writing `out` with d[ax] replaced by r.
__device__ void apply_axis(int ax, const int *d, int r, const double *op,
                           const double *in, double *out, double alpha, double beta,
                           double (*As)[65], double (*Bs)[65])
{
        if (ax == 0) {
                // out(r, d1 d2) = op(r x d0) * in(d0 x d1 d2)
                cta_gemm<false>(r, d[1] * d[2], d[0], 1, op, r, 0, in, d[0], 0,
                                out, r, 0, alpha, beta, As, Bs);
        } else if (ax == 1) {
                // out_l(d0 x r) = in_l(d0 x d1) * op^T, l < d2
                cta_gemm<true>(d[0], r, d[1], d[2], in, d[0], (int64_t) d[0] * d[1],
                               op, r, 0, out, d[0], (int64_t) d[0] * r,
                               alpha, beta, As, Bs);
        } else {
                // out(d0 d1 x r) = in(d0 d1 x d2) * op^T
                cta_gemm<true>(d[0] * d[1], r, d[2], 1, in, d[0] * d[1], 0,
                               op, r, 0, out, d[0] * d[1], 0, alpha, beta, As, Bs);
        }
}

__global__ void __launch_bounds__(256)
heff_fp64_kernel(const double *__restrict__ x, double *__restrict__ y,
                 const double *__restrict__ ops, const int64_t *__restrict__ blk_off,
                 const int4 *__restrict__ edims, const int *__restrict__ work_order,
                 int n_active, const int *__restrict__ task_ptr,
                 const HeffTask *__restrict__ tasks, double *scratch,
                 int64_t scratch_w1, int64_t scratch_w2, int *err)
{
        __shared__ double As[16][65];
        __shared__ double Bs[16][65];
        double *W1 = scratch + (int64_t) blockIdx.x * (scratch_w1 + scratch_w2);
        double *W2 = W1 + scratch_w1;

        for (int idx = blockIdx.x; idx < n_active; idx += gridDim.x) {
                const int nb = work_order[idx];
                const int4 en = edims[nb];
                const int dn[3] = {en.x, en.y, en.z};
                double *yn = y + blk_off[nb];
                for (int t = task_ptr[nb]; t < task_ptr[nb + 1]; ++t) {
                        const HeffTask tk = tasks[t];
                        const int4 eo = edims[tk.old];
                        int w[3] = {eo.x, eo.y, eo.z};
                        const double *in = x + blk_off[tk.old];
                        const int nst = (tk.axes >> 6) & 3;
                        for (int s = 0; s < nst; ++s) {
                                const int ax = (tk.axes >> (2 * s)) & 3;
                                const bool last = s == nst - 1;
                                double *out = last ? yn : (s == 0 ? W1 : W2);
                                const int64_t outsz = (int64_t) w[0] * w[1] * w[2] / w[ax] * dn[ax];
                                if (!last && outsz > (s == 0 ? scratch_w1 : scratch_w2)) {
                                        if (threadIdx.x == 0) atomicExch(err, 1);
                                        return;
                                }
                                apply_axis(ax, w, dn[ax], ops + tk.op_off[ax], in, out,
                                           last ? tk.pref : 1.0, last ? 1.0 : 0.0, As, Bs);
                                __syncthreads();
                                w[ax] = dn[ax];
                                in = out;
                        }
                }
        }
}

// Diagonal: diag[n](a,b,c) = sum over tasks of the (n, n) pair of
// pref * X[a,a] * Y[b,b] * Z[c,c]  (reference diag_old_to_new_sb,
// src/Heff.c:1064-1108).
__global__ void heff_diag_kernel(double *__restrict__ diag, const double *__restrict__ ops,
                                 const int64_t *__restrict__ blk_off,
                                 const int4 *__restrict__ edims, int nblocks,
                                 const int *__restrict__ task_ptr,
                                 const HeffTask *__restrict__ tasks)
{
        for (int nb = blockIdx.x; nb < nblocks; nb += gridDim.x) {
                const int4 e = edims[nb];
                const int64_t sz = (int64_t) e.x * e.y * e.z;
                double *d = diag + blk_off[nb];
                for (int64_t el = threadIdx.x; el < sz; el += blockDim.x) {
                        const int a = (int) (el % e.x);
                        const int b = (int) ((el / e.x) % e.y);
                        const int c = (int) (el / ((int64_t) e.x * e.y));
                        double acc = 0.0;
                        for (int t = task_ptr[nb]; t < task_ptr[nb + 1]; ++t) {
                                const HeffTask &tk = tasks[t];
                                if (tk.old != nb) continue;
                                const int nst = (tk.axes >> 6) & 3;
                                double v = tk.pref * ops[tk.op_off[0] + a + (int64_t) a * e.x];
                                v *= ops[tk.op_off[1] + b + (int64_t) b * e.y];
                                if (nst == 3) v *= ops[tk.op_off[2] + c + (int64_t) c * e.z];
                                acc += v;
                        }
                        d[el] = acc;
                }
        }
}

// ---------------------------------------------------------------------------
// Plan construction.

static const int kOrders3[6][3] = {{0, 1, 2}, {1, 0, 2}, {0, 2, 1},
                                   {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
static const int kOrders2[2][2] = {{0, 1}, {1, 0}};

int build_plan(const t3ns_heff_desc *d, HostPlan &hp)
{
        if (!d || d->nblocks < 0) return set_error(T3NS_E_ARG, "null descriptor");
        const int nops = d->isdmrg ? 2 : 3;
        hp.isdmrg = d->isdmrg;
        hp.nblocks = d->nblocks;
        for (int j = 0; j < 3; ++j) hp.map[j] = d->isdmrg ? j : d->map[j];
        int inv_map[3] = {-1, -1, -1};
        for (int j = 0; j < 3; ++j) {
                if (hp.map[j] < 0 || hp.map[j] > 2 || inv_map[hp.map[j]] != -1)
                        return set_error(T3NS_E_ARG, "map is not a permutation");
                inv_map[hp.map[j]] = j;
        }

        // memory-axis dims per block and block offsets
        hp.block_off.assign(d->block_off, d->block_off + d->nblocks + 1);
        hp.edims.resize(d->nblocks);
        for (int b = 0; b < d->nblocks; ++b) {
                int e[3];
                for (int j = 0; j < 3; ++j) e[j] = d->dims[3 * b + hp.map[j]];
                if (d->isdmrg) e[2] = 1;
                for (int j = 0; j < 3; ++j)
                        if (e[j] < 0) return set_error(T3NS_E_ARG, "negative block dim");
                if ((int64_t) e[0] * e[1] * e[2] != d->block_off[b + 1] - d->block_off[b])
                        return set_error(T3NS_E_ARG, "block size != product of dims at block " +
                                                          std::to_string(b));
                hp.edims[b] = make_int4(e[0], e[1], e[2], 0);
        }
        hp.size = d->block_off[d->nblocks];

        // operator base offsets
        hp.op_base.assign(nops, {});
        int64_t tot = 0;
        for (int i = 0; i < nops; ++i) {
                const t3ns_ropset &rs = d->ops[i];
                hp.op_base[i].resize(rs.nrops);
                for (int k = 0; k < rs.nrops; ++k) {
                        hp.op_base[i][k] = tot;
                        tot += rs.op_beginblock[k][rs.op_nblocks[k]];
                }
        }
        hp.op_elems = tot;

        // tasks
        hp.task_ptr.assign(d->nblocks + 1, 0);
        hp.tasks.clear();
        std::vector<double> work(d->nblocks, 0.0);
        std::vector<char> seen_block;
        double flops = 0;
        int64_t npairs = 0, max_w1 = 0, max_w2 = 0;
        for (int nb = 0; nb < d->nblocks; ++nb) {
                hp.task_ptr[nb] = (int) hp.tasks.size();
                const int dn[3] = {d->dims[3 * nb], d->dims[3 * nb + 1],
                                   d->isdmrg ? 1 : d->dims[3 * nb + 2]};
                for (int p = d->pair_ptr[nb]; p < d->pair_ptr[nb + 1]; ++p) {
                        ++npairs;
                        const int ob = d->pair_old[p];
                        if (ob < 0 || ob >= d->nblocks)
                                return set_error(T3NS_E_ARG, "old block out of range");
                        const int dold[3] = {d->dims[3 * ob], d->dims[3 * ob + 1],
                                             d->isdmrg ? 1 : d->dims[3 * ob + 2]};
                        const int ord = d->pair_order[p];
                        if (ord < 0 || ord >= (d->isdmrg ? 2 : 6))
                                return set_error(T3NS_E_ARG, "order out of range");
                        const int *o = d->isdmrg ? kOrders2[ord] : kOrders3[ord];
                        // reference FLOP count of one instruction for this pair
                        double fl = 0;
                        int wd[3] = {dold[0], dold[1], dold[2]};
                        int64_t w1 = 0, w2 = 0;
                        for (int s = 0; s < nops; ++s) {
                                fl += (double) wd[0] * wd[1] * wd[2] * dn[o[s]];
                                wd[o[s]] = dn[o[s]];
                                const int64_t sz = (int64_t) wd[0] * wd[1] * wd[2];
                                if (s == 0) w1 = sz;
                                if (s == 1 && nops == 3) w2 = sz;
                        }
                        int axes = 0;
                        for (int s = 0; s < nops; ++s) axes |= inv_map[o[s]] << (2 * s);
                        if (d->isdmrg) { axes = 0; for (int s = 0; s < 2; ++s) axes |= o[s] << (2 * s); }
                        axes |= nops << 6;

                        for (int64_t c = d->combo_ptr[p]; c < d->combo_ptr[p + 1]; ++c) {
                                const int m = d->combo_mpo[c];
                                if (m < 0 || m >= d->nrMPOc)
                                        return set_error(T3NS_E_ARG, "MPO combo out of range");
                                for (int k = d->MPOc_beg[m]; k < d->MPOc_beg[m + 1]; ++k) {
                                        HeffTask t;
                                        t.op_off[0] = t.op_off[1] = t.op_off[2] = 0;
                                        bool present = true;
                                        for (int i = 0; i < nops && present; ++i) {
                                                const t3ns_ropset &rs = d->ops[i];
                                                const int opk = d->instr[3 * k + i];
                                                const int sb = d->combo_sbops[3 * c + i];
                                                if (opk < 0 || opk >= rs.nrops)
                                                        return set_error(T3NS_E_ARG, "operator index out of range");
                                                if (sb < 0 || sb >= rs.op_nblocks[opk])
                                                        return set_error(T3NS_E_ARG, "operator block out of range");
                                                const int *bb = rs.op_beginblock[opk];
                                                if (bb[sb] == bb[sb + 1]) { present = false; break; }
                                                if ((int64_t) (bb[sb + 1] - bb[sb]) !=
                                                    (int64_t) dn[i] * dold[i])
                                                        return set_error(T3NS_E_ARG,
                                                                "operator block size mismatch");
                                                const int ax = d->isdmrg ? i : inv_map[i];
                                                t.op_off[ax] = hp.op_base[i][opk] + bb[sb];
                                        }
                                        if (!present) continue;
                                        t.pref = d->instr_pref[k] * d->combo_pref[c];
                                        t.old = ob;
                                        t.axes = axes;
                                        hp.tasks.push_back(t);
                                        flops += 2.0 * fl;
                                        work[nb] += 2.0 * fl + 64.0;
                                        max_w1 = std::max(max_w1, w1);
                                        max_w2 = std::max(max_w2, w2);
                                }
                        }
                }
        }
        hp.task_ptr[d->nblocks] = (int) hp.tasks.size();
        if (hp.tasks.size() > (size_t) INT32_MAX)
                return set_error(T3NS_E_LIMIT, "more than 2^31 tasks");
        hp.npairs = npairs;
        hp.flops_ref = flops;
        hp.flops_exec = flops;
        hp.max_w1 = max_w1;
        hp.max_w2 = max_w2;

        // algorithmic bytes: vectors in/out + each referenced operator block once
        {
                std::vector<int64_t> offs;
                offs.reserve(hp.tasks.size() * 3);
                double opbytes = 0;
                std::vector<std::pair<int64_t, int64_t>> blocks;
                for (int nb = 0; nb < d->nblocks; ++nb)
                        for (int t = hp.task_ptr[nb]; t < hp.task_ptr[nb + 1]; ++t) {
                                const HeffTask &tk = hp.tasks[t];
                                const int4 eo = hp.edims[tk.old], en = hp.edims[nb];
                                const int o3[3] = {eo.x, eo.y, eo.z}, n3[3] = {en.x, en.y, en.z};
                                for (int j = 0; j < nops; ++j)
                                        blocks.push_back({tk.op_off[j], (int64_t) o3[j] * n3[j]});
                        }
                std::sort(blocks.begin(), blocks.end());
                blocks.erase(std::unique(blocks.begin(), blocks.end()), blocks.end());
                for (auto &b : blocks) opbytes += 8.0 * b.second;
                hp.bytes_alg = 16.0 * hp.size + opbytes;
        }

        // active output blocks, heaviest first (longest-processing-time order)
        hp.work_order.clear();
        for (int nb = 0; nb < d->nblocks; ++nb)
                if (hp.task_ptr[nb + 1] > hp.task_ptr[nb]) hp.work_order.push_back(nb);
        std::stable_sort(hp.work_order.begin(), hp.work_order.end(),
                         [&](int a, int b) { return work[a] > work[b]; });
        return T3NS_OK;
}

int launch_heff_fp64(const DevicePlan &dp, const double *x, double *y, cudaStream_t s,
                     int *launches)
{
        T3NS_CUDA_TRY(cudaMemsetAsync(y, 0, sizeof(double) * dp.size, s));
        if (dp.n_active > 0) {
                heff_fp64_kernel<<<dp.grid, 256, 0, s>>>(
                        x, y, dp.ops, dp.blk_off, dp.edims, dp.work_order, dp.n_active,
                        dp.task_ptr, dp.tasks, dp.scratch, dp.scratch_w1, dp.scratch_w2,
                        dp.err);
                T3NS_CUDA_TRY(cudaGetLastError());
                if (launches) *launches = 1;
        } else if (launches) {
                *launches = 0;
        }
        return T3NS_OK;
}

int launch_heff_diag(const DevicePlan &dp, double *diag, cudaStream_t s)
{
        if (dp.nblocks == 0) return T3NS_OK;
        const int grid = std::min(dp.nblocks, 148 * 8);
        heff_diag_kernel<<<grid, 128, 0, s>>>(diag, dp.ops, dp.blk_off, dp.edims, dp.nblocks,
                                               dp.task_ptr, dp.tasks);
        T3NS_CUDA_TRY(cudaGetLastError());
        return T3NS_OK;
}

}  // namespace t3ns
