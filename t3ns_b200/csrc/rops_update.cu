// Renormalised-operator updates on the GPU.
//
// Append of a site operator (reference rOperators_append_phys,
// src/rOperators_pUpdate.c:665-673): scaled copies of whole blocks, one CTA
// per block.
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
#include <string>
#include <vector>

#include "common.h"
#include "dmma_gemm.cuh"

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

template <class T>
int upload(std::vector<void *> &allocs, T **p, const T *src, size_t n)
{
        *p = nullptr;
        cudaError_t e = cudaMalloc((void **) p, sizeof(T) * std::max<size_t>(n, 1));
        if (e != cudaSuccess) {
                cudaGetLastError();
                return set_error(T3NS_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
        }
        allocs.push_back(*p);
        if (src && n) T3NS_CUDA_TRY(cudaMemcpy(*p, src, sizeof(T) * n, cudaMemcpyHostToDevice));
        return T3NS_OK;
}

struct Allocs {
        std::vector<void *> v;
        ~Allocs() { for (void *p : v) cudaFree(p); }
};

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
        Allocs a;
        int *unit_ptr, *op_ptr, *counter;
        int4 *dims;
        int64_t *t_off, *ta_off, *old_off, *new_off;
        double *pref, *T, *OLD, *NEW, *scratch;
        std::vector<int4> dv(d->nentries);
        for (int e = 0; e < d->nentries; ++e)
                dv[e] = make_int4(d->dims[4 * e], d->dims[4 * e + 1], d->dims[4 * e + 2], d->dims[4 * e + 3]);
        T3NS_TRY(upload(a.v, &unit_ptr, d->unit_ptr, d->nunits + 1));
        T3NS_TRY(upload(a.v, &op_ptr, d->op_ptr, d->nentries + 1));
        T3NS_TRY(upload(a.v, &dims, dv.data(), dv.size()));
        T3NS_TRY(upload(a.v, &t_off, d->t_off, d->nentries));
        T3NS_TRY(upload(a.v, &ta_off, d->ta_off, d->nentries));
        T3NS_TRY(upload(a.v, &pref, d->pref, d->nentries));
        T3NS_TRY(upload(a.v, &old_off, d->old_off, npairs));
        T3NS_TRY(upload(a.v, &new_off, d->new_off, npairs));
        T3NS_TRY(upload(a.v, &T, t_tel, d->t_elems));
        T3NS_TRY(upload(a.v, &OLD, old_tel, d->old_elems));
        T3NS_TRY(upload<double>(a.v, &NEW, nullptr, d->new_elems));
        T3NS_TRY(upload<int>(a.v, &counter, nullptr, 1));
        int dev = 0, sms = 148;
        T3NS_CUDA_TRY(cudaGetDevice(&dev));
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        const int grid = std::max(1, std::min(d->nunits, 4 * sms));
        T3NS_TRY(upload<double>(a.v, &scratch, nullptr, (size_t) grid * slot));
        T3NS_CUDA_TRY(cudaMemset(NEW, 0, sizeof(double) * std::max<int64_t>(d->new_elems, 1)));
        T3NS_CUDA_TRY(cudaMemset(counter, 0, sizeof(int)));
        if (d->nunits > 0) {
                pupdate_kernel<<<grid, kUpdThreads>>>(d->is_left, d->nunits, unit_ptr, dims, t_off,
                                                      ta_off, pref, op_ptr, old_off, new_off, T, OLD,
                                                      NEW, scratch, slot, counter);
                T3NS_CUDA_TRY(cudaGetLastError());
        }
        if (d->new_elems)
                T3NS_CUDA_TRY(cudaMemcpy(new_tel, NEW, sizeof(double) * d->new_elems,
                                         cudaMemcpyDeviceToHost));
        return T3NS_OK;
}

int scalecopy_run(const t3ns_scalecopy_desc *d, const double *src, double *dst)
{
        if (!d || !dst || d->nentries < 0) return set_error(T3NS_E_ARG, "scalecopy: bad descriptor");
        for (int e = 0; e < d->nentries; ++e)
                if (d->len[e] < 0 || d->src_off[e] < 0 || d->src_off[e] + d->len[e] > d->src_elems ||
                    d->dst_off[e] < 0 || d->dst_off[e] + d->len[e] > d->dst_elems)
                        return set_error(T3NS_E_ARG, "scalecopy: block out of range");
        Allocs a;
        int64_t *dst_off, *src_off;
        int *len;
        double *scale, *S, *D;
        T3NS_TRY(upload(a.v, &dst_off, d->dst_off, d->nentries));
        T3NS_TRY(upload(a.v, &src_off, d->src_off, d->nentries));
        T3NS_TRY(upload(a.v, &len, d->len, d->nentries));
        T3NS_TRY(upload(a.v, &scale, d->scale, d->nentries));
        T3NS_TRY(upload(a.v, &S, src, d->src_elems));
        T3NS_TRY(upload<double>(a.v, &D, nullptr, d->dst_elems));
        T3NS_CUDA_TRY(cudaMemset(D, 0, sizeof(double) * std::max<int64_t>(d->dst_elems, 1)));
        if (d->nentries > 0) {
                scalecopy_kernel<<<std::min(d->nentries, 148 * 16), 256>>>(
                        d->nentries, dst_off, src_off, len, scale, S, D);
                T3NS_CUDA_TRY(cudaGetLastError());
        }
        if (d->dst_elems)
                T3NS_CUDA_TRY(cudaMemcpy(dst, D, sizeof(double) * d->dst_elems, cudaMemcpyDeviceToHost));
        return T3NS_OK;
}

}  // namespace t3ns

extern "C" int t3ns_scalecopy_host(const t3ns_scalecopy_desc *d, const double *src, double *dst)
{
        return t3ns::scalecopy_run(d, src, dst);
}

extern "C" int t3ns_pupdate_host(const t3ns_pupdate_desc *d, const double *t_tel,
                                 const double *old_tel, double *new_tel)
{
        return t3ns::pupdate_run(d, t_tel, old_tel, new_tel);
}
