// Renormalised-operator updates on the GPU.
//
// Append of a site operator (reference rOperators_append_phys,
// src/rOperators_pUpdate.c:665-673): scaled copies of whole blocks, one CTA
// per block.
//
// Branching update (reference update_rOperators_branching,
// src/rOperators_bUpdate.c:229-248): per (new block, O1 block, O2 block,
// site-tensor block, bra block) entry and instruction, O1 and O2 are applied
// to the site-tensor block on their axes and the result is contracted with
// the bra block over both (update_selected_blocks, :1043-1072); a CTA owns a
// new block, intermediates in a per-CTA scratch slice.
//
// Physical update (reference update_rOperators_physical,
// src/rOperators_pUpdate.c:364-387): for every updated block and every
// original block that maps onto it (pUpdate_block, :323-362), all operators
// of the block's MPO sector are sandwiched between the site-tensor block and
// its adjoint with two GEMMs (get_upd_aide, :273-321).  One persistent
// kernel; a CTA owns an updated block (a unit) and accumulates its entries in
// order, so no two CTAs write the same output and the sum order is the
// reference's (original blocks in ascending order).  The first product goes
// to a per-CTA scratch slice, the second accumulates into the output; both
// run on the FP64 tensor pipe (cta_dgemm).
#include <algorithm>
#include <numeric>
#include <cstring>
#include <string>
#include <vector>

#include "common.h"
#include "dmma_gemm.cuh"
#include "thread_work.h"

namespace t3ns {
namespace {

constexpr int kUpdThreads = 256;

__global__ void __launch_bounds__(kUpdThreads)
pupdate_kernel(int is_left, int nunits, const int *__restrict__ unit_ptr,
               const int4 *__restrict__ dims, const int64_t *__restrict__ t_off,
               const int64_t *__restrict__ ta_off, const double *__restrict__ pref,
               const int *__restrict__ op_ptr, const int64_t *__restrict__ old_off,
               const int64_t *__restrict__ new_off, const double *__restrict__ T,
               const double *__restrict__ OLD, double *NEW, double *scratch,
               int64_t slot, int *counter)
{
        __shared__ int unit;
        double *W = scratch + (int64_t) blockIdx.x * slot;
        for (;;) {
                if (threadIdx.x == 0) unit = atomicAdd(counter, 1);
                __syncthreads();
                const int u = unit;
                __syncthreads();
                if (u >= nunits) break;
                for (int e = unit_ptr[u]; e < unit_ptr[u + 1]; ++e) {
                        const int4 dm = dims[e];
                        const int M0 = dm.x, M1 = dm.y, N0 = dm.z, N1 = dm.w;
                        const double *Tb = T + t_off[e];
                        const double *Ta = T + ta_off[e];
                        const double pf = pref[e];
                        for (int p = op_ptr[e]; p < op_ptr[e + 1]; ++p) {
                                const double *O = OLD + old_off[p];
                                double *U = NEW + new_off[p];
                                // W (M0 x N1) = O * op(T);  U += pref * op(Ta) * W
                                if (is_left) {
                                        cta_dgemm<false, false>(M0, N1, M1, 1.0, O, M0, Tb, M1, 0.0, W, M0);
                                        __syncthreads();
                                        cta_dgemm<true, false>(N0, N1, M0, pf, Ta, M0, W, M0, 1.0, U, N0);
                                } else {
                                        cta_dgemm<false, true>(M0, N1, M1, 1.0, O, M0, Tb, N1, 0.0, W, M0);
                                        __syncthreads();
                                        cta_dgemm<false, false>(N0, N1, M0, pf, Ta, N0, W, M0, 1.0, U, N0);
                                }
                                __syncthreads();
                        }
                }
        }
}

__global__ void scalecopy_kernel(int n, const int64_t *__restrict__ dst_off,
                                 const int64_t *__restrict__ src_off, const int *__restrict__ len,
                                 const double *__restrict__ scale, const double *__restrict__ src,
                                 double *__restrict__ dst)
{
        for (int e = blockIdx.x; e < n; e += gridDim.x) {
                const double s = scale[e];
                const double *a = src + src_off[e];
                double *b = dst + dst_off[e];
                for (int j = threadIdx.x; j < len[e]; j += blockDim.x) b[j] = s * a[j];
        }
}

// out = op (r x s, column-major) applied on axis ax of in (dims w, w[ax] = s)
__device__ void apply_axis_dmma(int ax, const int *w, int r, const double *op, const double *in,
                                double *out)
{
        if (ax == 0) {
                cta_dgemm<false, false>(r, w[1] * w[2], w[0], 1.0, op, r, in, w[0], 0.0, out, r);
        } else if (ax == 1) {
                // slices along axis 2 are independent outputs (no barrier needed)
                for (int c = 0; c < w[2]; ++c)
                        cta_dgemm<false, true>(w[0], r, w[1], 1.0, in + (int64_t) c * w[0] * w[1], w[0],
                                               op, r, 0.0, out + (int64_t) c * w[0] * r, w[0]);
        } else {
                cta_dgemm<false, true>(w[0] * w[1], r, w[2], 1.0, in, (int64_t) w[0] * w[1], op, r,
                                       0.0, out, (int64_t) w[0] * w[1]);
        }
}

// Branching update: for every entry of a unit (one new block) and every op
// triple of the entry, W1 = O1 on axis a of T, W2 = O2 on axis b of W1,
// New += pref * contraction of Ta and W2 over axes a and b.
__global__ void __launch_bounds__(kUpdThreads)
bupdate_kernel(int3 ax, int nunits, const int *__restrict__ unit_ptr,
               const int *__restrict__ dims, const int64_t *__restrict__ t_off,
               const int64_t *__restrict__ ta_off, const double *__restrict__ pref,
               const int *__restrict__ op_ptr, const int64_t *__restrict__ o1_off,
               const int64_t *__restrict__ o2_off, const int64_t *__restrict__ new_off,
               const double *__restrict__ T, const double *__restrict__ O1,
               const double *__restrict__ O2, double *NEW, double *scratch, int64_t w1cap,
               int64_t w2cap, int *counter)
{
        __shared__ int unit;
        double *W1 = scratch + (int64_t) blockIdx.x * (w1cap + w2cap);
        double *W2 = W1 + w1cap;
        const int a = ax.x, b = ax.y, g = ax.z;
        for (;;) {
                if (threadIdx.x == 0) unit = atomicAdd(counter, 1);
                __syncthreads();
                const int u = unit;
                __syncthreads();
                if (u >= nunits) break;
                for (int e = unit_ptr[u]; e < unit_ptr[u + 1]; ++e) {
                        const int kd[3] = {dims[6 * e], dims[6 * e + 1], dims[6 * e + 2]};
                        const int bd[3] = {dims[6 * e + 3], dims[6 * e + 4], dims[6 * e + 5]};
                        const double *Tk = T + t_off[e];
                        const double *Tb = T + ta_off[e];
                        const double pf = pref[e];
                        // cheaper of the two orders (the results differ by rounding only)
                        const bool a_first = (int64_t) kd[b] * bd[a] * (kd[a] + bd[b]) <=
                                             (int64_t) kd[a] * bd[b] * (kd[b] + bd[a]);
                        const int x1 = a_first ? a : b, x2 = a_first ? b : a;
                        int v1[3] = {kd[0], kd[1], kd[2]};
                        v1[x1] = bd[x1];
                        // the host orders an entry's triples by their first-applied
                        // operator: a first stage equal to the previous one is reused
                        // (W1 is written by the first stage only)
                        const double *prev = nullptr;
                        for (int p = op_ptr[e]; p < op_ptr[e + 1]; ++p) {
                                const double *P1 = a_first ? O1 + o1_off[p] : O2 + o2_off[p];
                                const double *P2 = a_first ? O2 + o2_off[p] : O1 + o1_off[p];
                                if (P1 != prev) {
                                        apply_axis_dmma(x1, kd, bd[x1], P1, Tk, W1);
                                        __syncthreads();
                                        prev = P1;
                                }
                                apply_axis_dmma(x2, v1, bd[x2], P2, W1, W2);
                                __syncthreads();
                                double *Nw = NEW + new_off[p];
                                // New (bd[g] x kd[g]) += pf * sum over axes a, b of Tb * W2
                                if (g == 2) {
                                        const int R = bd[0] * bd[1];
                                        cta_dgemm<true, false>(bd[2], kd[2], R, pf, Tb, R, W2, R, 1.0, Nw, bd[2]);
                                } else if (g == 0) {
                                        const int R = bd[1] * bd[2];
                                        cta_dgemm<false, true>(bd[0], kd[0], R, pf, Tb, bd[0], W2, kd[0], 1.0,
                                                               Nw, bd[0]);
                                } else {
                                        // the same warp owns the same output tile in every slice
                                        for (int c = 0; c < bd[2]; ++c)
                                                cta_dgemm<true, false>(bd[1], kd[1], bd[0], pf,
                                                                       Tb + (int64_t) c * bd[0] * bd[1], bd[0],
                                                                       W2 + (int64_t) c * bd[0] * kd[1], bd[0],
                                                                       1.0, Nw, bd[1]);
                                }
                                __syncthreads();
                        }
                }
        }
}

// Sum of unique operators (reference sum_unique_rOperators,
// src/rOperators_init.c:228-265): new operator k, element j =
// sum over the instructions writing k, in instruction order, of
// pref * unique[src + j] (fused multiply-adds from zero).  One CTA per new
// operator (grid-stride), threads over its elements.
__global__ void sum_unique_kernel(int nnew, const int64_t *__restrict__ new_base,
                                  const int *__restrict__ instr_ptr,
                                  const int64_t *__restrict__ instr_src,
                                  const double *__restrict__ instr_pref,
                                  const double *__restrict__ U, double *__restrict__ NEW)
{
        for (int k = blockIdx.x; k < nnew; k += gridDim.x) {
                const int64_t b = new_base[k], n = new_base[k + 1] - b;
                const int i0 = instr_ptr[k], i1 = instr_ptr[k + 1];
                for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
                        double acc = 0.0;
                        for (int i = i0; i < i1; ++i) acc = fma(instr_pref[i], U[instr_src[i] + j], acc);
                        NEW[b + j] = acc;
                }
        }
}

// Zero-block test of kick_zero_blocks (src/sparseblocks.c:73-107): a block
// is kept when one of its elements has magnitude 1e-20 or more
// (COMPARE_ELEMENT_TO_ZERO, include/macros.h:24).  Block q of the flattened
// list spans NEW[off[q], off[q] + len[q]); one warp per block.
__global__ void nonzero_blocks_kernel(int64_t nblocks, const int64_t *__restrict__ off,
                                      const int *__restrict__ len, const double *__restrict__ NEW,
                                      int *__restrict__ keep)
{
        const int lane = threadIdx.x & 31;
        const int64_t w0 = ((int64_t) blockIdx.x * blockDim.x + threadIdx.x) >> 5;
        const int64_t nw = ((int64_t) gridDim.x * blockDim.x) >> 5;
        for (int64_t q = w0; q < nblocks; q += nw) {
                const double *p = NEW + off[q];
                bool nz = false;
                for (int j = lane; j < len[q] && !nz; j += 32) nz = fabs(p[j]) >= 1e-20;
                nz = __any_sync(0xffffffffu, nz);
                if (lane == 0) keep[q] = nz ? 1 : 0;
        }
}

// Gathers the kept blocks: entry e copies len[e] elements from src_off[e]
// to dst_off[e] (one CTA per entry, grid-stride).
__global__ void gather_blocks_kernel(int64_t n, const int64_t *__restrict__ src_off,
                                     const int64_t *__restrict__ dst_off, const int *__restrict__ len,
                                     const double *__restrict__ SRC, double *__restrict__ DST)
{
        for (int64_t e = blockIdx.x; e < n; e += gridDim.x)
                for (int j = threadIdx.x; j < len[e]; j += blockDim.x) DST[dst_off[e] + j] = SRC[src_off[e] + j];
}

// The arrays of one call laid out in the thread's workspace: inputs first
// (staged in the pinned buffer at their device offsets and uploaded with one
// copy), then the zero-initialised outputs, then the scratch.
struct CallLayout {
        Carve c;
        struct Input {
                size_t off;
                const void *src;
                size_t bytes;
        };
        std::vector<Input> inputs;
        template <class T>
        size_t input(const T *src, size_t n)
        {
                const size_t o = c.take<T>(n);
                inputs.push_back({o, src, src ? sizeof(T) * n : 0});
                return o;
        }
};

// Stages and uploads the inputs (all placed before `in_end`) and zeroes
// [zero0, zero1) on the device; `host_extra` more pinned bytes are reserved
// for the download.
int stage_call(ThreadWork &tw, const CallLayout &L, size_t in_end, size_t zero0, size_t zero1,
               size_t host_extra)
{
        T3NS_TRY(tw.reserve(L.c.off, std::max(in_end, host_extra)));
        for (const auto &x : L.inputs)
                if (x.bytes) std::memcpy(tw.host + x.off, x.src, x.bytes);
        T3NS_CUDA_TRY(cudaMemcpyAsync(tw.dev, tw.host, in_end, cudaMemcpyHostToDevice, tw.st));
        if (zero1 > zero0) T3NS_CUDA_TRY(cudaMemsetAsync(tw.dev + zero0, 0, zero1 - zero0, tw.st));
        return T3NS_OK;
}

// Downloads `bytes` from device offset `off` into dst (through the pinned
// buffer) and waits for the call's stream.
int finish_call(ThreadWork &tw, size_t off, void *dst, size_t bytes)
{
        if (bytes)
                T3NS_CUDA_TRY(cudaMemcpyAsync(tw.host, tw.dev + off, bytes, cudaMemcpyDeviceToHost,
                                              tw.st));
        T3NS_CUDA_TRY(cudaStreamSynchronize(tw.st));
        if (bytes) std::memcpy(dst, tw.host, bytes);
        return T3NS_OK;
}

template <class T>
T *at(const ThreadWork &tw, size_t off)
{
        return reinterpret_cast<T *>(tw.dev + off);
}

// Checks a sum-of-unique-operators descriptor against the unique buffer it
// reads; returns the number of blocks of the new set.
int check_sum_desc(const t3ns_sumunique_desc *s, int64_t unique_elems, int64_t *nblocks_out)
{
        if (!s || s->nnew < 0) return set_error(T3NS_E_ARG, "sum_unique: bad descriptor");
        int64_t nbl = 0;
        for (int k = 0; k < s->nnew; ++k) {
                const int64_t b0 = s->begin_ptr[k], b1 = s->begin_ptr[k + 1];
                if (b1 <= b0) return set_error(T3NS_E_ARG, "sum_unique: empty begin array");
                const int *bb = s->begin + b0;
                if (bb[0] != 0) return set_error(T3NS_E_ARG, "sum_unique: begin array must start at 0");
                for (int64_t q = 1; q < b1 - b0; ++q)
                        if (bb[q] < bb[q - 1]) return set_error(T3NS_E_ARG, "sum_unique: begin array decreases");
                if (s->new_base[k + 1] - s->new_base[k] != bb[b1 - b0 - 1])
                        return set_error(T3NS_E_ARG, "sum_unique: operator size != its last begin offset");
                const int n = bb[b1 - b0 - 1];
                for (int i = s->instr_ptr[k]; i < s->instr_ptr[k + 1]; ++i)
                        if (s->instr_src[i] < 0 || s->instr_src[i] + n > unique_elems)
                                return set_error(T3NS_E_ARG, "sum_unique: unique operator out of range");
                nbl += b1 - b0 - 1;
        }
        *nblocks_out = nbl;
        return T3NS_OK;
}

// Layout of the arrays of the sum on the device, after the call's own.
struct SumLayout {
        size_t nbase, iptr, isrc, ipref, bptr, bbeg;   // inputs
        size_t sum, qoff, qlen, keep, goff_src, goff_dst, glen, out;   // work and output
};

// Adds the sum's inputs to the call's layout (before its in_end) ...
void sum_inputs(CallLayout &L, SumLayout &S, const t3ns_sumunique_desc *s)
{
        const int ninstr = s->nnew ? s->instr_ptr[s->nnew] : 0;
        S.nbase = L.input(s->new_base, s->nnew + 1);
        S.iptr = L.input(s->instr_ptr, s->nnew + 1);
        S.isrc = L.input(s->instr_src, ninstr);
        S.ipref = L.input(s->instr_pref, ninstr);
        S.bptr = L.input(s->begin_ptr, s->nnew + 1);
        S.bbeg = L.input(s->begin, s->nnew ? s->begin_ptr[s->nnew] : 0);
}

// ... and its work arrays after the call's outputs.
void sum_work(CallLayout &L, SumLayout &S, const t3ns_sumunique_desc *s, int64_t nbl)
{
        const int64_t nsum = s->new_base[s->nnew];
        S.sum = L.c.take<double>(nsum);
        S.qoff = L.c.take<int64_t>(nbl);
        S.qlen = L.c.take<int>(nbl);
        S.keep = L.c.take<int>(nbl);
        S.goff_src = L.c.take<int64_t>(nbl);
        S.goff_dst = L.c.take<int64_t>(nbl);
        S.glen = L.c.take<int>(nbl);
        S.out = L.c.take<double>(nsum);
}

// Runs the sum of the unique operators at d_unique (device) into the work
// arrays, removes the zero blocks and downloads the kept blocks of every new
// operator back to back (operator k from out_base[k]) with their begin
// offsets after removal (new_begin, shaped like s->begin).  The block list
// and the gather list go through the pinned buffer at host offset hoff.
int sum_run(ThreadWork &tw, const SumLayout &S, const t3ns_sumunique_desc *s, int64_t nbl,
            const double *d_unique, double *new_tel, int *new_begin, int64_t *out_base)
{
        cudaStream_t st = tw.st;
        const int nnew = s->nnew;
        if (nnew == 0) {
                if (out_base) out_base[0] = 0;
                return T3NS_OK;
        }
        // flattened block list: offset and length of every block before removal
        std::vector<int64_t> qoff((size_t) nbl);
        std::vector<int> qlen((size_t) nbl);
        {
                int64_t q = 0;
                for (int k = 0; k < nnew; ++k) {
                        const int *bb = s->begin + s->begin_ptr[k];
                        const int nb = (int) (s->begin_ptr[k + 1] - s->begin_ptr[k] - 1);
                        for (int b = 0; b < nb; ++b, ++q) {
                                qoff[q] = s->new_base[k] + bb[b];
                                qlen[q] = bb[b + 1] - bb[b];
                        }
                }
        }
        int *hkeep = reinterpret_cast<int *>(tw.host);
        T3NS_CUDA_TRY(cudaMemcpyAsync(tw.dev + S.qoff, qoff.data(), sizeof(int64_t) * nbl,
                                      cudaMemcpyHostToDevice, st));
        T3NS_CUDA_TRY(cudaMemcpyAsync(tw.dev + S.qlen, qlen.data(), sizeof(int) * nbl,
                                      cudaMemcpyHostToDevice, st));
        sum_unique_kernel<<<std::min(nnew, 148 * 8), 256, 0, st>>>(
                nnew, at<int64_t>(tw, S.nbase), at<int>(tw, S.iptr), at<int64_t>(tw, S.isrc),
                at<double>(tw, S.ipref), d_unique, at<double>(tw, S.sum));
        T3NS_CUDA_TRY(cudaGetLastError());
        if (nbl > 0) {
                const int grid = (int) std::min<int64_t>((nbl + 7) / 8, 148 * 16);
                nonzero_blocks_kernel<<<grid, 256, 0, st>>>(nbl, at<int64_t>(tw, S.qoff), at<int>(tw, S.qlen),
                                                           at<double>(tw, S.sum), at<int>(tw, S.keep));
                T3NS_CUDA_TRY(cudaGetLastError());
                T3NS_CUDA_TRY(cudaMemcpyAsync(hkeep, tw.dev + S.keep, sizeof(int) * nbl,
                                              cudaMemcpyDeviceToHost, st));
        }
        T3NS_CUDA_TRY(cudaStreamSynchronize(st));
        // begin offsets after removal and the gather list of the kept blocks
        std::vector<int64_t> gsrc, gdst;
        std::vector<int> glen;
        int64_t q = 0, tot = 0;
        for (int k = 0; k < nnew; ++k) {
                const int *bb = s->begin + s->begin_ptr[k];
                int *nbb = new_begin + s->begin_ptr[k];
                const int nb = (int) (s->begin_ptr[k + 1] - s->begin_ptr[k] - 1);
                out_base[k] = tot;
                nbb[0] = 0;
                for (int b = 0; b < nb; ++b, ++q) {
                        const int len = hkeep[q] ? bb[b + 1] - bb[b] : 0;
                        if (len > 0) {
                                gsrc.push_back(qoff[q]);
                                gdst.push_back(tot + nbb[b]);
                                glen.push_back(len);
                        }
                        nbb[b + 1] = nbb[b] + len;
                }
                tot += nbb[nb];
        }
        out_base[nnew] = tot;
        const int64_t ng = (int64_t) glen.size();
        if (ng > 0) {
                T3NS_CUDA_TRY(cudaMemcpyAsync(tw.dev + S.goff_src, gsrc.data(), sizeof(int64_t) * ng,
                                              cudaMemcpyHostToDevice, st));
                T3NS_CUDA_TRY(cudaMemcpyAsync(tw.dev + S.goff_dst, gdst.data(), sizeof(int64_t) * ng,
                                              cudaMemcpyHostToDevice, st));
                T3NS_CUDA_TRY(cudaMemcpyAsync(tw.dev + S.glen, glen.data(), sizeof(int) * ng,
                                              cudaMemcpyHostToDevice, st));
                gather_blocks_kernel<<<(int) std::min<int64_t>(ng, 148 * 16), 256, 0, st>>>(
                        ng, at<int64_t>(tw, S.goff_src), at<int64_t>(tw, S.goff_dst), at<int>(tw, S.glen),
                        at<double>(tw, S.sum), at<double>(tw, S.out));
                T3NS_CUDA_TRY(cudaGetLastError());
                T3NS_CUDA_TRY(cudaMemcpyAsync(new_tel, tw.dev + S.out, sizeof(double) * tot,
                                              cudaMemcpyDeviceToHost, st));
        }
        // the host vectors above are read by the copies: finish before they go
        T3NS_CUDA_TRY(cudaStreamSynchronize(st));
        return T3NS_OK;
}

}  // namespace

int pupdate_run(const t3ns_pupdate_desc *d, const double *t_tel, const double *old_tel,
                double *new_tel)
{
        if (!d || !new_tel || d->nunits < 0 || d->nentries < 0)
                return set_error(T3NS_E_ARG, "pupdate: bad descriptor");
        const int npairs = d->nentries ? d->op_ptr[d->nentries] : 0;
        // validate every block against its buffer, and size the scratch
        int64_t slot = 1;
        for (int e = 0; e < d->nentries; ++e) {
                const int M0 = d->dims[4 * e], M1 = d->dims[4 * e + 1];
                const int N0 = d->dims[4 * e + 2], N1 = d->dims[4 * e + 3];
                if (M0 < 0 || M1 < 0 || N0 < 0 || N1 < 0)
                        return set_error(T3NS_E_ARG, "pupdate: negative dims");
                const int64_t tsz = (int64_t) M1 * N1, tasz = (int64_t) M0 * N0;
                if (d->t_off[e] < 0 || d->t_off[e] + tsz > d->t_elems || d->ta_off[e] < 0 ||
                    d->ta_off[e] + tasz > d->t_elems)
                        return set_error(T3NS_E_ARG, "pupdate: site-tensor block out of range");
                for (int p = d->op_ptr[e]; p < d->op_ptr[e + 1]; ++p)
                        if (d->old_off[p] < 0 || d->old_off[p] + (int64_t) M0 * M1 > d->old_elems ||
                            d->new_off[p] < 0 || d->new_off[p] + (int64_t) N0 * N1 > d->new_elems)
                                return set_error(T3NS_E_ARG, "pupdate: operator block out of range");
                slot = std::max<int64_t>(slot, (int64_t) M0 * N1);
        }
        for (int u = 0; u < d->nunits; ++u)
                if (d->unit_ptr[u] > d->unit_ptr[u + 1] || d->unit_ptr[u + 1] > d->nentries)
                        return set_error(T3NS_E_ARG, "pupdate: unit list out of range");
        int dev = 0, sms = 148;
        T3NS_CUDA_TRY(cudaGetDevice(&dev));
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int grid = std::max(1, std::min(d->nunits, 4 * sms));
        CallLayout L;
        const size_t o_unit = L.input(d->unit_ptr, d->nunits + 1);
        const size_t o_op = L.input(d->op_ptr, d->nentries + 1);
        // dims: four ints per entry, the layout of int4
        const size_t o_dims = L.input(reinterpret_cast<const int4 *>(d->dims), d->nentries);
        const size_t o_t = L.input(d->t_off, d->nentries);
        const size_t o_ta = L.input(d->ta_off, d->nentries);
        const size_t o_pref = L.input(d->pref, d->nentries);
        const size_t o_old_off = L.input(d->old_off, npairs);
        const size_t o_new_off = L.input(d->new_off, npairs);
        const size_t o_T = L.input(t_tel, d->t_elems);
        const size_t o_OLD = L.input(old_tel, d->old_elems);
        const size_t in_end = L.c.off;
        const size_t o_NEW = L.c.take<double>(d->new_elems);
        const size_t o_counter = L.c.take<int>(1);
        const size_t zero_end = L.c.off;
        const size_t o_scratch = L.c.take<double>((size_t) grid * slot);
        const size_t new_bytes = sizeof(double) * d->new_elems;
        ThreadWork &tw = thread_work();
        T3NS_TRY(stage_call(tw, L, in_end, o_NEW, zero_end, new_bytes));
        if (d->nunits > 0) {
                pupdate_kernel<<<grid, kUpdThreads, 0, tw.st>>>(
                        d->is_left, d->nunits, at<int>(tw, o_unit), at<int4>(tw, o_dims),
                        at<int64_t>(tw, o_t), at<int64_t>(tw, o_ta), at<double>(tw, o_pref),
                        at<int>(tw, o_op), at<int64_t>(tw, o_old_off), at<int64_t>(tw, o_new_off),
                        at<double>(tw, o_T), at<double>(tw, o_OLD), at<double>(tw, o_NEW),
                        at<double>(tw, o_scratch), slot, at<int>(tw, o_counter));
                T3NS_CUDA_TRY(cudaGetLastError());
        }
        return finish_call(tw, o_NEW, new_tel, new_bytes);
}

// With sum (not null) the copies are unique operators that are summed into
// the new set on the device (sum_run): dst, new_begin and out_base then
// receive its kept blocks.
int scalecopy_run(const t3ns_scalecopy_desc *d, const double *src, double *dst,
                  const t3ns_sumunique_desc *sum = nullptr, int *new_begin = nullptr,
                  int64_t *out_base = nullptr)
{
        if (!d || !dst || d->nentries < 0) return set_error(T3NS_E_ARG, "scalecopy: bad descriptor");
        int64_t nbl = 0;
        if (sum) {
                T3NS_TRY(check_sum_desc(sum, d->dst_elems, &nbl));
                if (!new_begin || !out_base) return set_error(T3NS_E_ARG, "scalecopy: null output");
        }
        for (int e = 0; e < d->nentries; ++e)
                if (d->len[e] < 0 || d->src_off[e] < 0 || d->src_off[e] + d->len[e] > d->src_elems ||
                    d->dst_off[e] < 0 || d->dst_off[e] + d->len[e] > d->dst_elems)
                        return set_error(T3NS_E_ARG, "scalecopy: block out of range");
        CallLayout L;
        const size_t o_dst_off = L.input(d->dst_off, d->nentries);
        const size_t o_src_off = L.input(d->src_off, d->nentries);
        const size_t o_len = L.input(d->len, d->nentries);
        const size_t o_scale = L.input(d->scale, d->nentries);
        const size_t o_S = L.input(src, d->src_elems);
        SumLayout S{};
        if (sum) sum_inputs(L, S, sum);
        const size_t in_end = L.c.off;
        const size_t o_D = L.c.take<double>(d->dst_elems);
        const size_t zero_end = L.c.off;
        if (sum) sum_work(L, S, sum, nbl);
        const size_t dst_bytes = sizeof(double) * d->dst_elems;
        ThreadWork &tw = thread_work();
        T3NS_TRY(stage_call(tw, L, in_end, o_D, zero_end,
                            std::max(dst_bytes, sizeof(int) * (size_t) nbl)));
        if (d->nentries > 0) {
                scalecopy_kernel<<<std::min(d->nentries, 148 * 16), 256, 0, tw.st>>>(
                        d->nentries, at<int64_t>(tw, o_dst_off), at<int64_t>(tw, o_src_off),
                        at<int>(tw, o_len), at<double>(tw, o_scale), at<double>(tw, o_S),
                        at<double>(tw, o_D));
                T3NS_CUDA_TRY(cudaGetLastError());
        }
        if (sum) return sum_run(tw, S, sum, nbl, at<double>(tw, o_D), dst, new_begin, out_base);
        return finish_call(tw, o_D, dst, dst_bytes);
}

int sum_unique_run(const t3ns_sumunique_desc *sum, const double *unique_tel, double *new_tel,
                   int *new_begin, int64_t *out_base)
{
        if (!sum || !new_tel || !new_begin || !out_base || sum->unique_elems < 0)
                return set_error(T3NS_E_ARG, "sum_unique: bad arguments");
        int64_t nbl = 0;
        T3NS_TRY(check_sum_desc(sum, sum->unique_elems, &nbl));
        CallLayout L;
        const size_t o_U = L.input(unique_tel, sum->unique_elems);
        SumLayout S{};
        sum_inputs(L, S, sum);
        const size_t in_end = L.c.off;
        sum_work(L, S, sum, nbl);
        ThreadWork &tw = thread_work();
        T3NS_TRY(stage_call(tw, L, in_end, 0, 0, sizeof(int) * (size_t) nbl));
        return sum_run(tw, S, sum, nbl, at<double>(tw, o_U), new_tel, new_begin, out_base);
}

int bupdate_run(const t3ns_bupdate_desc *d, const double *t_tel, const double *o1_tel,
                const double *o2_tel, double *new_tel, const t3ns_sumunique_desc *sum = nullptr,
                int *new_begin = nullptr, int64_t *out_base = nullptr)
{
        if (!d || !new_tel || d->nunits < 0 || d->nentries < 0)
                return set_error(T3NS_E_ARG, "bupdate: bad descriptor");
        int64_t nbl = 0;
        if (sum) {
                T3NS_TRY(check_sum_desc(sum, d->new_elems, &nbl));
                if (!new_begin || !out_base) return set_error(T3NS_E_ARG, "bupdate: null output");
        }
        const int a = d->ax[0], b = d->ax[1], g = d->ax[2];
        if (a < 0 || a > 2 || b < 0 || b > 2 || g < 0 || g > 2 || a == b || a == g || b == g)
                return set_error(T3NS_E_ARG, "bupdate: axes are not a permutation");
        const int ntr = d->nentries ? d->op_ptr[d->nentries] : 0;
        int64_t w1cap = 1, w2cap = 1;
        for (int e = 0; e < d->nentries; ++e) {
                const int *kd = d->dims + 6 * e, *bd = kd + 3;
                for (int j = 0; j < 6; ++j)
                        if (kd[j] < 0) return set_error(T3NS_E_ARG, "bupdate: negative dims");
                int64_t tk = (int64_t) kd[0] * kd[1] * kd[2], tb = (int64_t) bd[0] * bd[1] * bd[2];
                if (d->t_off[e] < 0 || d->t_off[e] + tk > d->t_elems || d->ta_off[e] < 0 ||
                    d->ta_off[e] + tb > d->t_elems)
                        return set_error(T3NS_E_ARG, "bupdate: site-tensor block out of range");
                // either order of the two operator applications may be taken
                auto one_applied = [&](int x) {
                        int64_t v = bd[x];
                        for (int i = 0; i < 3; ++i)
                                if (i != x) v *= kd[i];
                        return v;
                };
                w1cap = std::max(w1cap, std::max(one_applied(a), one_applied(b)));
                w2cap = std::max(w2cap, (int64_t) bd[a] * bd[b] * kd[g]);
                for (int p = d->op_ptr[e]; p < d->op_ptr[e + 1]; ++p)
                        if (d->o1_off[p] < 0 || d->o1_off[p] + (int64_t) bd[a] * kd[a] > d->o1_elems ||
                            d->o2_off[p] < 0 || d->o2_off[p] + (int64_t) bd[b] * kd[b] > d->o2_elems ||
                            d->new_off[p] < 0 || d->new_off[p] + (int64_t) bd[g] * kd[g] > d->new_elems)
                                return set_error(T3NS_E_ARG, "bupdate: operator block out of range");
        }
        for (int u = 0; u < d->nunits; ++u)
                if (d->unit_ptr[u] > d->unit_ptr[u + 1] || d->unit_ptr[u + 1] > d->nentries)
                        return set_error(T3NS_E_ARG, "bupdate: unit list out of range");
        w1cap = (w1cap + 31) / 32 * 32;
        w2cap = (w2cap + 31) / 32 * 32;
        int dev = 0, sms = 148;
        T3NS_CUDA_TRY(cudaGetDevice(&dev));
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int grid = std::max(1, std::min(d->nunits, 4 * sms));
        CallLayout L;
        const size_t o_unit = L.input(d->unit_ptr, d->nunits + 1);
        const size_t o_op = L.input(d->op_ptr, d->nentries + 1);
        const size_t o_dims = L.input(d->dims, (size_t) 6 * d->nentries);
        const size_t o_t = L.input(d->t_off, d->nentries);
        const size_t o_ta = L.input(d->ta_off, d->nentries);
        const size_t o_pref = L.input(d->pref, d->nentries);
        // each entry's triples ordered by the operator the kernel applies
        // first (the same order choice as the kernel's), so equal first
        // stages run once; the triples of an entry write their own new
        // blocks, so only the summation order into a shared block changes
        std::vector<int64_t> s_o1(ntr), s_o2(ntr), s_new(ntr);
        {
                std::vector<int> idx;
                for (int e = 0; e < d->nentries; ++e) {
                        const int *kd = d->dims + 6 * e, *bd = kd + 3;
                        const bool a_first = (int64_t) kd[b] * bd[a] * (kd[a] + bd[b]) <=
                                             (int64_t) kd[a] * bd[b] * (kd[b] + bd[a]);
                        const int p0 = d->op_ptr[e], p1 = d->op_ptr[e + 1];
                        idx.resize(p1 - p0);
                        std::iota(idx.begin(), idx.end(), p0);
                        const int64_t *key = a_first ? d->o1_off : d->o2_off;
                        std::stable_sort(idx.begin(), idx.end(),
                                         [key](int x, int y) { return key[x] < key[y]; });
                        for (int q = p0; q < p1; ++q) {
                                s_o1[q] = d->o1_off[idx[q - p0]];
                                s_o2[q] = d->o2_off[idx[q - p0]];
                                s_new[q] = d->new_off[idx[q - p0]];
                        }
                }
        }
        const size_t o_o1_off = L.input(s_o1.data(), ntr);
        const size_t o_o2_off = L.input(s_o2.data(), ntr);
        const size_t o_new_off = L.input(s_new.data(), ntr);
        const size_t o_T = L.input(t_tel, d->t_elems);
        const size_t o_O1 = L.input(o1_tel, d->o1_elems);
        const size_t o_O2 = L.input(o2_tel, d->o2_elems);
        SumLayout S{};
        if (sum) sum_inputs(L, S, sum);
        const size_t in_end = L.c.off;
        const size_t o_NEW = L.c.take<double>(d->new_elems);
        const size_t o_counter = L.c.take<int>(1);
        const size_t zero_end = L.c.off;
        const size_t o_scratch = L.c.take<double>((size_t) grid * (w1cap + w2cap));
        if (sum) sum_work(L, S, sum, nbl);
        const size_t new_bytes = sizeof(double) * d->new_elems;
        ThreadWork &tw = thread_work();
        T3NS_TRY(stage_call(tw, L, in_end, o_NEW, zero_end,
                            std::max(new_bytes, sizeof(int) * (size_t) nbl)));
        if (d->nunits > 0) {
                bupdate_kernel<<<grid, kUpdThreads, 0, tw.st>>>(
                        make_int3(a, b, g), d->nunits, at<int>(tw, o_unit), at<int>(tw, o_dims),
                        at<int64_t>(tw, o_t), at<int64_t>(tw, o_ta), at<double>(tw, o_pref),
                        at<int>(tw, o_op), at<int64_t>(tw, o_o1_off), at<int64_t>(tw, o_o2_off),
                        at<int64_t>(tw, o_new_off), at<double>(tw, o_T), at<double>(tw, o_O1),
                        at<double>(tw, o_O2), at<double>(tw, o_NEW), at<double>(tw, o_scratch), w1cap,
                        w2cap, at<int>(tw, o_counter));
                T3NS_CUDA_TRY(cudaGetLastError());
        }
        if (sum) return sum_run(tw, S, sum, nbl, at<double>(tw, o_NEW), new_tel, new_begin, out_base);
        return finish_call(tw, o_NEW, new_tel, new_bytes);
}

}  // namespace t3ns

extern "C" int t3ns_bupdate_host(const t3ns_bupdate_desc *d, const double *t_tel,
                                 const double *o1_tel, const double *o2_tel, double *new_tel)
{
        return t3ns::bupdate_run(d, t_tel, o1_tel, o2_tel, new_tel);
}

extern "C" int t3ns_scalecopy_host(const t3ns_scalecopy_desc *d, const double *src, double *dst)
{
        return t3ns::scalecopy_run(d, src, dst);
}

extern "C" int t3ns_sum_unique_host(const t3ns_sumunique_desc *s, const double *unique_tel,
                                    double *new_tel, int *new_begin, int64_t *out_base)
{
        return t3ns::sum_unique_run(s, unique_tel, new_tel, new_begin, out_base);
}

extern "C" int t3ns_scalecopy_sum_host(const t3ns_scalecopy_desc *d, const t3ns_sumunique_desc *s,
                                       const double *src, double *new_tel, int *new_begin,
                                       int64_t *out_base)
{
        if (!s) return t3ns::set_error(T3NS_E_ARG, "scalecopy_sum: null sum descriptor");
        return t3ns::scalecopy_run(d, src, new_tel, s, new_begin, out_base);
}

extern "C" int t3ns_bupdate_sum_host(const t3ns_bupdate_desc *d, const t3ns_sumunique_desc *s,
                                     const double *t_tel, const double *o1_tel, const double *o2_tel,
                                     double *new_tel, int *new_begin, int64_t *out_base)
{
        if (!s) return t3ns::set_error(T3NS_E_ARG, "bupdate_sum: null sum descriptor");
        return t3ns::bupdate_run(d, t_tel, o1_tel, o2_tel, new_tel, s, new_begin, out_base);
}

extern "C" int t3ns_pupdate_host(const t3ns_pupdate_desc *d, const double *t_tel,
                                 const double *old_tel, double *new_tel)
{
        return t3ns::pupdate_run(d, t_tel, old_tel, new_tel);
}
