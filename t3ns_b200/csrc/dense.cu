// Dense FP64 factorisations of the site-tensor decomposition: the thin SVD
// and the Householder QR that the reference's siteTensor_decompose.c asks
// LAPACK for (LAPACKE_dgesdd at src/siteTensor_decompose.c:1060 and :565,
// LAPACKE_dgeqrf at :285, LAPACKE_dorgqr at :295), one symmetry sector per
// call.  Each call runs as one CTA on the caller thread's own stream, so the
// reference's OpenMP loop over sectors keeps several sectors in flight, and
// costs one upload, one launch, one download and one synchronisation through
// the thread's workspace (thread_work.h).
//
// SVD: one-sided (Hestenes) Jacobi on the columns of the tall orientation W
// of A (A or A^T), parallel round-robin ordering, rotations accumulated into
// V; sigma_j = |w_j|, u_j = w_j / sigma_j, sorted descending.  Columns of U
// whose singular value is zero are completed to an orthonormal set from unit
// vectors (two Gram-Schmidt passes), as a thin LAPACK SVD returns them.
//
// QR: Householder reflectors with LAPACK's conventions (dlarfg: beta =
// -sign(alpha) |(alpha, x)|, tau = (beta - alpha) / beta, v = x / (alpha -
// beta), tau = 0 when x = 0; dgeqr2 / dorg2r column order), so R, the
// reflectors and Q agree with LAPACK's unblocked path up to rounding.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.h"
#include "thread_work.h"

namespace t3ns {
namespace {

constexpr int kDenseThreads = 512;
constexpr int kDenseWarps = kDenseThreads / 32;
constexpr int kMaxSweeps = 60;
// W and V are staged in shared memory when they fit in this many doubles
constexpr int kSvdSmemDoubles = 24576;
// a singular value at or below this is treated as exactly zero
constexpr double kZeroSigma = 1e-300;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
}

// Sum over the CTA, the same fixed order on every thread.  All threads call.
__device__ double block_sum(double v, double *red)
{
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        v = warp_sum(v);
        __syncthreads();
        if (lane == 0) red[warp] = v;
        __syncthreads();
        double t = 0.0;
        for (int i = 0; i < kDenseWarps; ++i) t += red[i];
        return t;
}

struct SvdOut {
        double *sig;     // [nn] sorted descending
        double *uw;      // [mm x nn] left vectors of the tall orientation, sorted
        double *vs;      // [nn x nn] right vectors of the tall orientation, sorted
        double *aux;     // [nn] unsorted norms
        int *rank;       // [nn]
};

__global__ void __launch_bounds__(kDenseThreads)
svd_jacobi_kernel(int m, int n, const double *__restrict__ A, double *W, double *V, int vectors,
                  SvdOut out, int *status)
{
        extern __shared__ double smem[];
        __shared__ double red[kDenseWarps];
        __shared__ int rotated, nonzero;
        __shared__ double cand_val[kDenseWarps];
        __shared__ int cand_idx[kDenseWarps];
        const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
        const bool trans = m < n;
        const int mm = trans ? n : m, nn = trans ? m : n;
        if (!W) {
                W = smem;
                V = smem + (size_t) mm * nn;
        }
        for (int64_t idx = tid; idx < (int64_t) mm * nn; idx += kDenseThreads) {
                const int i = (int) (idx % mm), j = (int) (idx / mm);
                W[idx] = trans ? A[j + (int64_t) i * m] : A[idx];
        }
        if (vectors)
                for (int64_t idx = tid; idx < (int64_t) nn * nn; idx += kDenseThreads)
                        V[idx] = (idx % nn == idx / nn) ? 1.0 : 0.0;
        __syncthreads();

        const int n2 = nn + (nn & 1);
        const double tol = 4.0 * DBL_EPSILON * sqrt((double) mm);
        int sweep = 0;
        for (; sweep < kMaxSweeps && n2 > 1; ++sweep) {
                if (tid == 0) rotated = 0;
                __syncthreads();
                for (int r = 0; r < n2 - 1; ++r) {
                        for (int k = warp; k < n2 / 2; k += kDenseWarps) {
                                // circle method: position 0 fixed, the others rotate
                                const int p = k == 0 ? 0 : ((k + r - 1) % (n2 - 1)) + 1;
                                const int q = ((n2 - 2 - k + r) % (n2 - 1)) + 1;
                                if (p >= nn || q >= nn) continue;
                                double *wp = W + (int64_t) p * mm, *wq = W + (int64_t) q * mm;
                                double a = 0.0, b = 0.0, g = 0.0;
                                for (int i = lane; i < mm; i += 32) {
                                        const double x = wp[i], y = wq[i];
                                        a = fma(x, x, a);
                                        b = fma(y, y, b);
                                        g = fma(x, y, g);
                                }
                                a = warp_sum(a);
                                b = warp_sum(b);
                                g = warp_sum(g);
                                const double den = sqrt(a) * sqrt(b);
                                if (!(den > 0.0) || !(fabs(g) > tol * den)) continue;
                                const double zeta = (b - a) / (2.0 * g);
                                const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(fma(zeta, zeta, 1.0)));
                                const double c = 1.0 / sqrt(fma(t, t, 1.0)), s = c * t;
                                for (int i = lane; i < mm; i += 32) {
                                        const double x = wp[i], y = wq[i];
                                        wp[i] = c * x - s * y;
                                        wq[i] = s * x + c * y;
                                }
                                if (vectors) {
                                        double *vp = V + (int64_t) p * nn, *vq = V + (int64_t) q * nn;
                                        for (int i = lane; i < nn; i += 32) {
                                                const double x = vp[i], y = vq[i];
                                                vp[i] = c * x - s * y;
                                                vq[i] = s * x + c * y;
                                        }
                                }
                                if (lane == 0) rotated = 1;
                        }
                        __syncthreads();
                }
                const int any = rotated;
                __syncthreads();
                if (!any) break;
        }
        if (tid == 0) *status = sweep == kMaxSweeps ? 1 : 0;

        // norms, ranks (descending, ties by index), sorted outputs
        for (int j = warp; j < nn; j += kDenseWarps) {
                const double *wj = W + (int64_t) j * mm;
                double a = 0.0;
                for (int i = lane; i < mm; i += 32) a = fma(wj[i], wj[i], a);
                a = warp_sum(a);
                if (lane == 0) out.aux[j] = sqrt(a);
        }
        __syncthreads();
        for (int j = tid; j < nn; j += kDenseThreads) {
                const double sj = out.aux[j];
                int rk = 0;
                for (int k = 0; k < nn; ++k) {
                        const double sk = out.aux[k];
                        rk += (sk > sj) || (sk == sj && k < j);
                }
                out.rank[j] = rk;
                out.sig[rk] = sj;
        }
        if (tid == 0) nonzero = 0;
        __syncthreads();
        if (!vectors) return;
        for (int j = warp; j < nn; j += kDenseWarps) {
                const int rk = out.rank[j];
                const double sj = out.aux[j];
                const double inv = sj > kZeroSigma ? 1.0 / sj : 0.0;
                const double *wj = W + (int64_t) j * mm;
                double *uo = out.uw + (int64_t) rk * mm;
                for (int i = lane; i < mm; i += 32) uo[i] = wj[i] * inv;
                const double *vj = V + (int64_t) j * nn;
                double *vo = out.vs + (int64_t) rk * nn;
                for (int i = lane; i < nn; i += 32) vo[i] = vj[i];
                if (lane == 0 && sj > kZeroSigma) atomicAdd(&nonzero, 1);
        }
        __syncthreads();

        // complete the columns of zero singular values (sorted last)
        const int nz = nonzero;
        for (int r = nz; r < nn; ++r) {
                // the unit vector with the largest component outside span(u_0..u_{r-1})
                double best = -1.0;
                int besti = 0;
                for (int i = tid; i < mm; i += kDenseThreads) {
                        double p = 0.0;
                        for (int c = 0; c < r; ++c) {
                                const double x = out.uw[i + (int64_t) c * mm];
                                p = fma(x, x, p);
                        }
                        const double rem = 1.0 - p;
                        if (rem > best) {
                                best = rem;
                                besti = i;
                        }
                }
#pragma unroll
                for (int o = 16; o; o >>= 1) {
                        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                        const int oi = __shfl_xor_sync(0xffffffffu, besti, o);
                        if (ob > best || (ob == best && oi < besti)) {
                                best = ob;
                                besti = oi;
                        }
                }
                if (lane == 0) {
                        cand_val[warp] = best;
                        cand_idx[warp] = besti;
                }
                __syncthreads();
                int e = cand_idx[0];
                double ev = cand_val[0];
                for (int w = 1; w < kDenseWarps; ++w)
                        if (cand_val[w] > ev || (cand_val[w] == ev && cand_idx[w] < e)) {
                                ev = cand_val[w];
                                e = cand_idx[w];
                        }
                double *ur = out.uw + (int64_t) r * mm;
                for (int i = tid; i < mm; i += kDenseThreads) ur[i] = i == e ? 1.0 : 0.0;
                __syncthreads();
                // two classical Gram-Schmidt passes against u_0 .. u_{r-1}
                for (int pass = 0; pass < 2; ++pass) {
                        for (int c = 0; c < r; ++c) {
                                const double *uc = out.uw + (int64_t) c * mm;
                                double d = 0.0;
                                for (int i = tid; i < mm; i += kDenseThreads) d = fma(uc[i], ur[i], d);
                                d = block_sum(d, red);
                                for (int i = tid; i < mm; i += kDenseThreads) ur[i] = fma(-d, uc[i], ur[i]);
                                __syncthreads();
                        }
                }
                double nr = 0.0;
                for (int i = tid; i < mm; i += kDenseThreads) nr = fma(ur[i], ur[i], nr);
                nr = block_sum(nr, red);
                const double inv = nr > 0.0 ? 1.0 / sqrt(nr) : 0.0;
                for (int i = tid; i < mm; i += kDenseThreads) ur[i] *= inv;
                __syncthreads();
        }
}

// dgeqr2: Householder QR of the m x n column-major A (ld m) in place, tau[k].
__global__ void __launch_bounds__(kDenseThreads)
geqr2_kernel(int m, int n, double *A, double *tau)
{
        __shared__ double red[kDenseWarps];
        __shared__ double sh_tau;
        const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
        const int k = min(m, n);
        for (int j = 0; j < k; ++j) {
                double *aj = A + (int64_t) j * m;
                double x2 = 0.0;
                for (int i = j + 1 + tid; i < m; i += kDenseThreads) x2 = fma(aj[i], aj[i], x2);
                x2 = block_sum(x2, red);
                const double alpha = aj[j];
                double t = 0.0, beta = alpha;
                if (x2 > 0.0) {
                        beta = -copysign(hypot(alpha, sqrt(x2)), alpha);
                        t = (beta - alpha) / beta;
                        const double scale = 1.0 / (alpha - beta);
                        for (int i = j + 1 + tid; i < m; i += kDenseThreads) aj[i] *= scale;
                }
                __syncthreads();
                if (tid == 0) {
                        aj[j] = beta;
                        tau[j] = t;
                        sh_tau = t;
                }
                __syncthreads();
                const double tj = sh_tau;
                if (tj != 0.0) {
                        // H = I - tau v v^T with v = (1, aj[j+1:]) on the trailing columns
                        for (int c = j + 1 + warp; c < n; c += kDenseWarps) {
                                double *ac = A + (int64_t) c * m;
                                double w = lane == 0 ? ac[j] : 0.0;
                                for (int i = j + 1 + lane; i < m; i += 32) w = fma(aj[i], ac[i], w);
                                w = warp_sum(w) * tj;
                                if (lane == 0) ac[j] -= w;
                                for (int i = j + 1 + lane; i < m; i += 32) ac[i] = fma(-w, aj[i], ac[i]);
                        }
                }
                __syncthreads();
        }
}

// dorg2r: the first n columns of H_0 ... H_{k-1} in place of the reflectors.
__global__ void __launch_bounds__(kDenseThreads)
org2r_kernel(int m, int n, int k, double *A, const double *__restrict__ tau)
{
        const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
        for (int j = k; j < n; ++j)
                for (int i = tid; i < m; i += kDenseThreads) A[i + (int64_t) j * m] = i == j ? 1.0 : 0.0;
        __syncthreads();
        for (int i = k - 1; i >= 0; --i) {
                double *ai = A + (int64_t) i * m;
                const double ti = tau[i];
                if (i < n - 1) {
                        // apply H_i to A(i:m, i+1:n); v = (1, ai[i+1:])
                        for (int c = i + 1 + warp; c < n; c += kDenseWarps) {
                                double *ac = A + (int64_t) c * m;
                                double w = lane == 0 ? ac[i] : 0.0;
                                for (int r = i + 1 + lane; r < m; r += 32) w = fma(ai[r], ac[r], w);
                                w = warp_sum(w) * ti;
                                if (lane == 0) ac[i] -= w;
                                for (int r = i + 1 + lane; r < m; r += 32) ac[r] = fma(-w, ai[r], ac[r]);
                        }
                }
                __syncthreads();
                for (int r = i + 1 + tid; r < m; r += kDenseThreads) ai[r] *= -ti;
                for (int r = tid; r < i; r += kDenseThreads) ai[r] = 0.0;
                if (tid == 0) ai[i] = 1.0 - ti;
                __syncthreads();
        }
}

// column-major m x n with leading dimension ld <-> compact
void pack(const double *a, int m, int n, int64_t ld, double *c)
{
        for (int j = 0; j < n; ++j) std::memcpy(c + (int64_t) j * m, a + j * ld, sizeof(double) * m);
}

void unpack(const double *c, int m, int n, double *a, int64_t ld)
{
        for (int j = 0; j < n; ++j) std::memcpy(a + j * ld, c + (int64_t) j * m, sizeof(double) * m);
}

}  // namespace

int gesdd_run(char jobz, int m, int n, const double *a, int lda, double *s, double *u, int ldu,
              double *vt, int ldvt)
{
        if (m < 0 || n < 0 || lda < std::max(1, m) || !(jobz == 'S' || jobz == 'N'))
                return set_error(T3NS_E_ARG, "gesdd: bad arguments");
        const int k = std::min(m, n);
        if (jobz == 'S' && (ldu < std::max(1, m) || ldvt < std::max(1, k)))
                return set_error(T3NS_E_ARG, "gesdd: bad leading dimensions");
        if (k == 0) return T3NS_OK;
        const bool trans = m < n;
        const int mm = trans ? n : m, nn = k;
        const int vectors = jobz == 'S';
        // device: A, then the outputs the host reads back (sigma, status and,
        // with vectors, UW and VS) as one contiguous range, then the rest
        const size_t need = (size_t) mm * nn + (vectors ? (size_t) nn * nn : 0);
        const bool in_smem = need <= (size_t) kSvdSmemDoubles;
        Carve dc;
        const size_t oA = dc.take<double>((size_t) m * n);
        const size_t oSig = dc.take<double>(nn);
        const size_t oStatus = dc.take<int>(1);
        const size_t oUw = dc.take<double>(vectors ? (size_t) mm * nn : 1);
        const size_t oVs = dc.take<double>(vectors ? (size_t) nn * nn : 1);
        const size_t oEnd = dc.off;
        const size_t oAux = dc.take<double>(nn);
        const size_t oRank = dc.take<int>(nn);
        const size_t oW = in_smem ? 0 : dc.take<double>((size_t) mm * nn);
        const size_t oV = in_smem ? 0 : dc.take<double>(vectors ? (size_t) nn * nn : 1);
        // host: packed A, then the copy of the output range
        Carve hc;
        const size_t hA = hc.take<double>((size_t) m * n);
        const size_t hOut = hc.take<char>(oEnd - oSig);
        ThreadWork &tw = thread_work();
        T3NS_TRY(tw.reserve(dc.off, hc.off));
        cudaStream_t st = tw.st;
        char *D = tw.dev, *H = tw.host;
        SvdOut o;
        o.sig = reinterpret_cast<double *>(D + oSig);
        o.uw = reinterpret_cast<double *>(D + oUw);
        o.vs = reinterpret_cast<double *>(D + oVs);
        o.aux = reinterpret_cast<double *>(D + oAux);
        o.rank = reinterpret_cast<int *>(D + oRank);
        int *status = reinterpret_cast<int *>(D + oStatus);
        double *dA = reinterpret_cast<double *>(D + oA);
        double *W = in_smem ? nullptr : reinterpret_cast<double *>(D + oW);
        double *V = in_smem ? nullptr : reinterpret_cast<double *>(D + oV);
        const size_t smem = in_smem ? need * sizeof(double) : 0;
        pack(a, m, n, lda, reinterpret_cast<double *>(H + hA));
        T3NS_CUDA_TRY(cudaMemcpyAsync(dA, H + hA, sizeof(double) * (size_t) m * n,
                                      cudaMemcpyHostToDevice, st));
        if (smem > 48 * 1024 && !tw.svd_smem_set) {
                T3NS_CUDA_TRY(cudaFuncSetAttribute(svd_jacobi_kernel,
                                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   kSvdSmemDoubles * (int) sizeof(double)));
                tw.svd_smem_set = true;
        }
        svd_jacobi_kernel<<<1, kDenseThreads, smem, st>>>(m, n, dA, W, V, vectors, o, status);
        T3NS_CUDA_TRY(cudaGetLastError());
        T3NS_CUDA_TRY(cudaMemcpyAsync(H + hOut, D + oSig, oEnd - oSig, cudaMemcpyDeviceToHost, st));
        T3NS_CUDA_TRY(cudaStreamSynchronize(st));
        const char *ho = H + hOut;
        const int hstatus = *reinterpret_cast<const int *>(ho + (oStatus - oSig));
        std::memcpy(s, ho, sizeof(double) * nn);
        const double *uw = reinterpret_cast<const double *>(ho + (oUw - oSig));
        const double *vs = reinterpret_cast<const double *>(ho + (oVs - oSig));
        if (hstatus) return set_error(T3NS_E_EIG, "gesdd: Jacobi sweeps did not converge");
        if (!vectors) return T3NS_OK;
        if (!trans) {
                // A = UW S VS^T: U = UW (m x k), VT = VS^T (k x n)
                unpack(uw, m, k, u, ldu);
                for (int j = 0; j < n; ++j)
                        for (int r = 0; r < k; ++r) vt[r + (int64_t) j * ldvt] = vs[j + (int64_t) r * nn];
        } else {
                // A^T = UW S VS^T: U = VS (m x k), VT = UW^T (k x n)
                unpack(vs, m, k, u, ldu);
                for (int j = 0; j < n; ++j)
                        for (int r = 0; r < k; ++r) vt[r + (int64_t) j * ldvt] = uw[j + (int64_t) r * mm];
        }
        return T3NS_OK;
}

int geqrf_run(int m, int n, double *a, int lda, double *tau)
{
        if (m < 0 || n < 0 || lda < std::max(1, m)) return set_error(T3NS_E_ARG, "geqrf: bad arguments");
        const int k = std::min(m, n);
        if (k == 0) return T3NS_OK;
        // device and host alike: A, then tau (read back together)
        const size_t na = (size_t) m * n;
        const size_t bytes = sizeof(double) * (na + k);
        ThreadWork &tw = thread_work();
        T3NS_TRY(tw.reserve(bytes, bytes));
        cudaStream_t st = tw.st;
        double *dA = reinterpret_cast<double *>(tw.dev), *hA = reinterpret_cast<double *>(tw.host);
        pack(a, m, n, lda, hA);
        T3NS_CUDA_TRY(cudaMemcpyAsync(dA, hA, sizeof(double) * na, cudaMemcpyHostToDevice, st));
        geqr2_kernel<<<1, kDenseThreads, 0, st>>>(m, n, dA, dA + na);
        T3NS_CUDA_TRY(cudaGetLastError());
        T3NS_CUDA_TRY(cudaMemcpyAsync(hA, dA, bytes, cudaMemcpyDeviceToHost, st));
        T3NS_CUDA_TRY(cudaStreamSynchronize(st));
        unpack(hA, m, n, a, lda);
        std::memcpy(tau, hA + na, sizeof(double) * k);
        return T3NS_OK;
}

int orgqr_run(int m, int n, int k, double *a, int lda, const double *tau)
{
        if (m < 0 || n < 0 || n > m || k < 0 || k > n || lda < std::max(1, m))
                return set_error(T3NS_E_ARG, "orgqr: bad arguments");
        if (n == 0) return T3NS_OK;
        // device and host alike: A, then tau (uploaded together)
        const size_t na = (size_t) m * n;
        const size_t bytes = sizeof(double) * (na + std::max(k, 1));
        ThreadWork &tw = thread_work();
        T3NS_TRY(tw.reserve(bytes, bytes));
        cudaStream_t st = tw.st;
        double *dA = reinterpret_cast<double *>(tw.dev), *hA = reinterpret_cast<double *>(tw.host);
        pack(a, m, n, lda, hA);
        if (k) std::memcpy(hA + na, tau, sizeof(double) * k);
        T3NS_CUDA_TRY(cudaMemcpyAsync(dA, hA, sizeof(double) * (na + k), cudaMemcpyHostToDevice, st));
        org2r_kernel<<<1, kDenseThreads, 0, st>>>(m, n, k, dA, dA + na);
        T3NS_CUDA_TRY(cudaGetLastError());
        T3NS_CUDA_TRY(cudaMemcpyAsync(hA, dA, sizeof(double) * na, cudaMemcpyDeviceToHost, st));
        T3NS_CUDA_TRY(cudaStreamSynchronize(st));
        unpack(hA, m, n, a, lda);
        return T3NS_OK;
}

}  // namespace t3ns

extern "C" int t3ns_gesdd_host(char jobz, int m, int n, const double *a, int lda, double *s,
                               double *u, int ldu, double *vt, int ldvt)
{
        return t3ns::gesdd_run(jobz, m, n, a, lda, s, u, ldu, vt, ldvt);
}

extern "C" int t3ns_geqrf_host(int m, int n, double *a, int lda, double *tau)
{
        return t3ns::geqrf_run(m, n, a, lda, tau);
}

extern "C" int t3ns_orgqr_host(int m, int n, int k, double *a, int lda, const double *tau)
{
        return t3ns::orgqr_run(m, n, k, a, lda, tau);
}
