// Device-resident Davidson solver for the lowest eigenpair of Heff.
//
// Algorithm, constants and stopping rule follow the reference
// (src/davidson.c:259-328):
//   - new search vector: orthogonalise t against the basis V, normalise
//     (new_search_vector, :117-130).  The reference uses modified
//     Gram-Schmidt with one dot/axpy pass per basis vector; here t is
//     orthogonalised with two block classical Gram-Schmidt passes (CGS2),
//     which is at least as stable and reads V twice instead of 2m times;
//   - one matvec into VA, new column of the projected matrix S = V^T VA
//     (expand_submatrix, :132-145);
//   - Rayleigh-Ritz on the m x m matrix S (do_eigsolve, :147-162; dsyev in
//     the reference) with an in-project cyclic Jacobi eigensolver in FP64;
//   - deflation to keep_deflate Ritz vectors when m reaches max_vecs
//     (deflate, :164-185);
//   - Ritz vector, residual and its norm (calculate_residue, :187-202);
//   - diagonal preconditioner with Olsen correction and cutoff 1e-12
//     (davidson_diagonal_preconditioner, :223-257).
// Every reduction is deterministic: per-block partial sums are reduced in a
// fixed order.  The host reads 4 doubles per iteration to decide whether to
// stop.
#include <chrono>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <cmath>
#include <functional>
#include <string>
#include <vector>

#include "common.h"
#include "heff_internal.h"

namespace t3ns {

static constexpr int kRedBlocks = 296;   // 2 x 148 SMs
static constexpr int kRedThreads = 256;
static constexpr int kChunk = 8;         // basis columns per register pass
static constexpr double kDiagCutoff = 1e-12;
static constexpr int kMaxVecs = 32;      // largest Davidson subspace
// see davidson_core's `stall`: the residual level below which a split-precision
// solve may level off, relative to max(1, |energy|): 3xTF32 matvecs are
// accurate to ~2e-6 relative, BF16x3 to ~1e-5 (more on small steps)
static constexpr double kStallLevel = 1e-4;
static constexpr double kStallLevelBf16 = 1e-2;

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        return v;
}

// Block-reduces `nv` per-thread values; thread 0 returns the sums in out[].
template <int NV>
__device__ void block_sums(double (&v)[NV], double *out)
{
        __shared__ double sh[NV][kRedThreads / 32];
        const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
        for (int k = 0; k < NV; ++k) {
                const double s = warp_sum(v[k]);
                if (lane == 0) sh[k][wid] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
#pragma unroll
                for (int k = 0; k < NV; ++k) {
                        double s = 0;
                        for (int w = 0; w < kRedThreads / 32; ++w) s += sh[k][w];
                        out[k] = s;
                }
        }
        __syncthreads();
}

// Counts and columns that depend on the current basis size m are read on
// the device (dm; nullptr means m = 0), so one captured graph serves every
// iteration: ncols = m + nadd, and a vector argument flagged "at m" is
// column m of its matrix (leading dimension ld).
__device__ __forceinline__ int dev_m(const int *dm) { return dm ? *dm : 0; }

// partials[b * ncols + j] = sum over the rows of block b of V[i, j] * t[i],
// ncols = m + nadd, t = tb (or column m of tb when t_at_m)
__global__ void __launch_bounds__(kRedThreads)
dots_kernel(const double *__restrict__ V, int64_t ld, const int *dm, int nadd,
            const double *__restrict__ tb, int t_at_m, int64_t n, double *__restrict__ partials)
{
        const int ncols = dev_m(dm) + nadd;
        const double *__restrict__ t = tb + (t_at_m ? (int64_t) dev_m(dm) * ld : 0);
        for (int j0 = 0; j0 < ncols; j0 += kChunk) {
                double acc[kChunk];
#pragma unroll
                for (int k = 0; k < kChunk; ++k) acc[k] = 0;
                const int nc = min(kChunk, ncols - j0);
                for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
                     i += (int64_t) gridDim.x * blockDim.x) {
                        const double ti = t[i];
#pragma unroll
                        for (int k = 0; k < kChunk; ++k)
                                if (k < nc) acc[k] = fma(V[i + (j0 + k) * ld], ti, acc[k]);
                }
                double s[kChunk];
                block_sums<kChunk>(acc, s);
                if (threadIdx.x == 0)
                        for (int k = 0; k < nc; ++k) partials[blockIdx.x * ncols + j0 + k] = s[k];
        }
}

// out[j * out_stride] = scale * sum_b partials[b * ncols + j]   (fixed order),
// ncols = m + nadd; out = ob (or ob + m * out_col when out_col != 0)
__global__ void reduce_partials_kernel(const double *__restrict__ partials, int nblk,
                                       const int *dm, int nadd, double *__restrict__ ob,
                                       int64_t out_col, int out_stride, double scale)
{
        const int ncols = dev_m(dm) + nadd;
        double *__restrict__ out = ob + (int64_t) dev_m(dm) * out_col;
        for (int j = threadIdx.x; j < ncols; j += blockDim.x) {
                double s = 0;
                for (int b = 0; b < nblk; ++b) s += partials[b * ncols + j];
                out[j * out_stride] = scale * s;
        }
}

// t[i] -= sum_j V[i, j] coef[j]; partials[b] = block sum of t[i]^2 afterwards
__global__ void __launch_bounds__(kRedThreads)
gs_update_kernel(const double *__restrict__ V, int64_t ld, const int *dm,
                 const double *__restrict__ coef, double *__restrict__ t, int64_t n,
                 double *__restrict__ partials)
{
        const int ncols = dev_m(dm);
        __shared__ double c[64];
        for (int j = threadIdx.x; j < ncols; j += blockDim.x) c[j] = coef[j];
        __syncthreads();
        double acc[1] = {0};
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x) {
                double s = 0;
                for (int j = 0; j < ncols; ++j) s = fma(V[i + j * ld], c[j], s);
                const double v = t[i] - s;
                t[i] = v;
                acc[0] = fma(v, v, acc[0]);
        }
        double out[1];
        block_sums<1>(acc, out);
        if (threadIdx.x == 0) partials[blockIdx.x] = out[0];
}

// partials[b] = block sum of t[i]^2
__global__ void __launch_bounds__(kRedThreads)
norm2_kernel(const double *__restrict__ t, int64_t n, double *__restrict__ partials)
{
        double acc[1] = {0};
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x)
                acc[0] = fma(t[i], t[i], acc[0]);
        double out[1];
        block_sums<1>(acc, out);
        if (threadIdx.x == 0) partials[blockIdx.x] = out[0];
}

// column m of V and out2 (if not null) = t / ||t||, with ||t||^2 = sum of
// the nblk partials (each block reduces them itself, in the same order)
__global__ void __launch_bounds__(kRedThreads)
normalize_kernel(const double *__restrict__ t, double *__restrict__ V, int64_t ld,
                 const int *dm, double *__restrict__ out2, int64_t n,
                 const double *__restrict__ partials, int nblk)
{
        double *__restrict__ out = V + (int64_t) dev_m(dm) * ld;
        __shared__ double inv;
        if (threadIdx.x == 0) {
                double s = 0;
                for (int b = 0; b < nblk; ++b) s += partials[b];
                inv = 1.0 / sqrt(s);
        }
        __syncthreads();
        const double a = inv;
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x) {
                const double v = t[i] * a;
                out[i] = v;
                if (out2) out2[i] = v;
        }
}

// column m of VA = y
__global__ void __launch_bounds__(kRedThreads)
store_column_kernel(const double *__restrict__ y, double *__restrict__ VA, int64_t ld,
                    const int *dm, int64_t n)
{
        double *__restrict__ out = VA + (int64_t) dev_m(dm) * ld;
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x)
                out[i] = y[i];
}

// m <- m + add, or m <- set when set >= 0
__global__ void set_m_kernel(int *dm, int add, int set)
{
        *dm = set >= 0 ? set : *dm + add;
}

// result = V y, t = VA y - theta result; partials[b*3 + {0,1,2}] =
// {sum t^2, sum uK t, sum uK result} with uK = result / (diag - theta)
// (cutoff kDiagCutoff), i.e. calculate_residue and the reductions of the
// preconditioner fused in one pass.
__global__ void __launch_bounds__(kRedThreads)
ritz_kernel(const double *__restrict__ V, const double *__restrict__ VA, int64_t ld, const int *dm,
            const double *__restrict__ y, const double *__restrict__ theta_p,
            const double *__restrict__ diag, double *__restrict__ result,
            double *__restrict__ t, int64_t n, double *__restrict__ partials)
{
        const int m = dev_m(dm);
        __shared__ double c[64];
        for (int j = threadIdx.x; j < m; j += blockDim.x) c[j] = y[j];
        __syncthreads();
        const double theta = *theta_p;
        double acc[3] = {0, 0, 0};
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x) {
                double r = 0, a = 0;
                for (int j = 0; j < m; ++j) {
                        r = fma(V[i + j * ld], c[j], r);
                        a = fma(VA[i + j * ld], c[j], a);
                }
                const double tt = a - theta * r;
                result[i] = r;
                t[i] = tt;
                const double diff = diag[i] - theta;
                const double uK = fabs(diff) > kDiagCutoff ? r / diff
                                                           : (diff < 0 ? -1 : 1) * r / kDiagCutoff;
                acc[0] = fma(tt, tt, acc[0]);
                acc[1] = fma(uK, tt, acc[1]);
                acc[2] = fma(uK, r, acc[2]);
        }
        double out[3];
        block_sums<3>(acc, out);
        if (threadIdx.x == 0)
                for (int k = 0; k < 3; ++k) partials[blockIdx.x * 3 + k] = out[k];
}

// partials[b*3 + {1,2}] = {sum uK t, sum uK result} (the preconditioner's
// reductions alone, for the standalone entry point)
__global__ void __launch_bounds__(kRedThreads)
precond_sums_kernel(const double *__restrict__ result, const double *__restrict__ t,
                    const double *__restrict__ diag, const double *__restrict__ theta_p,
                    int64_t n, double *__restrict__ partials)
{
        const double theta = *theta_p;
        double acc[3] = {0, 0, 0};
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x) {
                const double r = result[i];
                const double diff = diag[i] - theta;
                const double uK = fabs(diff) > kDiagCutoff ? r / diff
                                                           : (diff < 0 ? -1 : 1) * r / kDiagCutoff;
                acc[1] = fma(uK, t[i], acc[1]);
                acc[2] = fma(uK, r, acc[2]);
        }
        double out[3];
        block_sums<3>(acc, out);
        if (threadIdx.x == 0)
                for (int k = 0; k < 3; ++k) partials[blockIdx.x * 3 + k] = out[k];
}

// t = -(t + alpha result) / (diag - theta) with alpha = -uKr / uKu
__global__ void __launch_bounds__(kRedThreads)
precond_kernel(const double *__restrict__ result, double *__restrict__ t,
               const double *__restrict__ diag, const double *__restrict__ scal,
               const double *__restrict__ theta_p, int64_t n)
{
        const double theta = *theta_p;
        const double alpha = -scal[1] / scal[2];
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x) {
                const double v = fma(alpha, result[i], t[i]);
                const double diff = diag[i] - theta;
                t[i] = fabs(diff) > kDiagCutoff ? -v / diff : -(diff < 0 ? -1 : 1) * v / kDiagCutoff;
        }
}

// V[:, k] = V Y[:, k] for k < keep, row by row (in place is safe per row)
__global__ void __launch_bounds__(kRedThreads)
deflate_kernel(double *__restrict__ V, int64_t ld, int mcols, const double *__restrict__ Y,
               int ldy, int keep, int64_t n)
{
        __shared__ double y[64 * 4];
        for (int e = threadIdx.x; e < mcols * keep; e += blockDim.x)
                y[e] = Y[(e % mcols) + (e / mcols) * ldy];
        __syncthreads();
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x) {
                double o[4] = {0, 0, 0, 0};
                for (int j = 0; j < mcols; ++j) {
                        const double v = V[i + j * ld];
                        for (int k = 0; k < keep; ++k) o[k] = fma(v, y[j + k * mcols], o[k]);
                }
                for (int k = 0; k < keep; ++k) V[i + k * ld] = o[k];
        }
}

// Symmetric eigenproblem of the m x m projected matrix (upper triangle of S,
// leading dimension ld): eigenvalues ascending into w, eigenvectors into the
// columns of Z (leading dimension ld).  Parallel cyclic Jacobi with
// round-robin pairing (Golub & Van Loan, Alg. 8.4.3 / 8.4.4); one CTA.
// status: 0 converged, 1 no convergence within the sweep limit.
__global__ void jacobi_eig_kernel(const double *__restrict__ S, int ld, const int *dm,
                                  double *__restrict__ Z, double *__restrict__ w,
                                  int *__restrict__ status)
{
        const int m = dev_m(dm);
        __shared__ double A[kMaxVecs][kMaxVecs + 1];
        __shared__ double Q[kMaxVecs][kMaxVecs + 1];
        __shared__ double cs[kMaxVecs / 2][2];
        __shared__ int pp[kMaxVecs / 2], qq[kMaxVecs / 2];
        __shared__ int order[kMaxVecs];
        __shared__ double off_s, frob_s;
        const int tid = threadIdx.x, nt = blockDim.x;
        const int M = m + (m & 1);   // even number of players
        for (int e = tid; e < kMaxVecs * kMaxVecs; e += nt) {
                const int i = e % kMaxVecs, j = e / kMaxVecs;
                double v = 0;
                if (i < m && j < m) v = i <= j ? S[i + j * ld] : S[j + i * ld];
                A[i][j] = v;
                Q[i][j] = (i == j) ? 1.0 : 0.0;
        }
        __syncthreads();
        int sweep = 0;
        const int max_sweeps = 60;
        for (; sweep < max_sweeps; ++sweep) {
                if (tid == 0) {
                        double off = 0, fr = 0;
                        for (int i = 0; i < m; ++i)
                                for (int j = 0; j < m; ++j) {
                                        const double a2 = A[i][j] * A[i][j];
                                        fr += a2;
                                        if (i != j) off += a2;
                                }
                        off_s = off;
                        frob_s = fr;
                }
                __syncthreads();
                // rounding keeps the off-diagonal norm near eps * m * ||A||;
                // 1e-14 relative is below what the Ritz values can resolve
                if (off_s <= 1e-28 * frob_s || off_s == 0.0) break;
                for (int r = 0; r < M - 1; ++r) {
                        // round-robin pairing: player 0 fixed, others rotate
                        if (tid < M / 2) {
                                const int k = tid;
                                int a = k == 0 ? 0 : 1 + ((k - 1 + r) % (M - 1));
                                int b = 1 + ((M - 2 - k + r) % (M - 1));
                                int p = min(a, b), q = max(a, b);
                                pp[k] = p;
                                qq[k] = q;
                                double c = 1, s = 0;
                                if (q < m && p != q) {
                                        const double apq = A[p][q];
                                        if (apq != 0.0) {
                                                const double tau = (A[q][q] - A[p][p]) / (2 * apq);
                                                const double tt = (tau >= 0 ? 1.0 : -1.0) /
                                                                  (fabs(tau) + sqrt(1 + tau * tau));
                                                c = 1 / sqrt(1 + tt * tt);
                                                s = tt * c;
                                        }
                                }
                                cs[k][0] = c;
                                cs[k][1] = s;
                        }
                        __syncthreads();
                        // A <- A J, Q <- Q J   (column update)
                        for (int e = tid; e < (M / 2) * m; e += nt) {
                                const int k = e / m, i = e % m;
                                const int p = pp[k], q = qq[k];
                                if (q >= m || p == q) continue;
                                const double c = cs[k][0], s = cs[k][1];
                                const double aip = A[i][p], aiq = A[i][q];
                                A[i][p] = c * aip - s * aiq;
                                A[i][q] = s * aip + c * aiq;
                                const double qip = Q[i][p], qiq = Q[i][q];
                                Q[i][p] = c * qip - s * qiq;
                                Q[i][q] = s * qip + c * qiq;
                        }
                        __syncthreads();
                        // A <- J^T A   (row update)
                        for (int e = tid; e < (M / 2) * m; e += nt) {
                                const int k = e / m, j = e % m;
                                const int p = pp[k], q = qq[k];
                                if (q >= m || p == q) continue;
                                const double c = cs[k][0], s = cs[k][1];
                                const double apj = A[p][j], aqj = A[q][j];
                                A[p][j] = c * apj - s * aqj;
                                A[q][j] = s * apj + c * aqj;
                        }
                        __syncthreads();
                }
        }
        if (tid == 0) {
                for (int i = 0; i < m; ++i) order[i] = i;
                for (int i = 0; i < m; ++i) {       // selection sort, ascending
                        int best = i;
                        for (int j = i + 1; j < m; ++j)
                                if (A[order[j]][order[j]] < A[order[best]][order[best]]) best = j;
                        const int tmp = order[i];
                        order[i] = order[best];
                        order[best] = tmp;
                }
                *status = (sweep < max_sweeps || off_s <= 1e-20 * frob_s) ? 0 : 1;
        }
        __syncthreads();
        for (int e = tid; e < m * m; e += nt) {
                const int i = e % m, j = e / m;
                Z[i + j * ld] = Q[i][order[j]];
        }
        for (int j = tid; j < m; j += nt) w[j] = A[order[j]][order[j]];
}

// ---------------------------------------------------------------------------

struct DavidsonBuffers {
        double *V = nullptr, *VA = nullptr, *t = nullptr, *S = nullptr, *Z = nullptr,
               *w = nullptr, *partials = nullptr, *coef = nullptr, *scal = nullptr;
        double *vin = nullptr, *vout = nullptr;   // fixed matvec operands
        int *status = nullptr;
        int *dm = nullptr;                          // current basis size
        double *host_scal = nullptr;   // pinned
        ~DavidsonBuffers()
        {
                cudaFree(V); cudaFree(VA); cudaFree(t); cudaFree(S); cudaFree(Z); cudaFree(w);
                cudaFree(partials); cudaFree(coef); cudaFree(scal); cudaFree(status);
                cudaFree(vin); cudaFree(vout); cudaFree(dm);
                if (host_scal) cudaFreeHost(host_scal);
        }
};

// Subspace size that fits, shrinking like the reference's max_vecs_to_alloc
// (src/davidson.c:56-78) but against device memory.
static int alloc_basis(DavidsonBuffers &b, int64_t n, int max_vecs)
{
        for (int mv = max_vecs; mv >= 3; --mv) {
                cudaError_t e1 = cudaMalloc(&b.V, sizeof(double) * n * mv);
                cudaError_t e2 = e1 == cudaSuccess ? cudaMalloc(&b.VA, sizeof(double) * n * mv)
                                                    : cudaErrorMemoryAllocation;
                if (e1 == cudaSuccess && e2 == cudaSuccess) {
                        if (mv != max_vecs)
                                printf("Note @davidson: keeping %d instead of %d vectors.\n", mv, max_vecs);
                        return mv;
                }
                cudaGetLastError();
                cudaFree(b.V);
                cudaFree(b.VA);
                b.V = b.VA = nullptr;
        }
        return -1;
}

// y = H x on device vectors, enqueued on the given stream
using DevMatvec = std::function<int(const double *, double *, cudaStream_t)>;

// stall > 0: also stop (returning 2) once the residual is below
// stall_level * max(1, |energy|) -- the region where the split-precision
// matvec's rounding can level it off -- and has not fallen below 0.9 of its
// best value for `stall` iterations.
// mv_err (optional): the matvec kernel's device error status; it is read back
// with the iteration's scalars and a non-zero value ends the solve with
// T3NS_E_DEVICE instead of continuing on a wrong product.
static int davidson_core(int64_t n, const DevMatvec &matvec, double *d_result, double *energy,
                         int max_vecs, int keep, double tol, int max_its, const double *d_diag,
                         t3ns_davidson_info *info, cudaStream_t s, int stall = 0,
                         bool use_graphs = false, const int *mv_err = nullptr,
                         double stall_level = kStallLevel)
{
        const auto t_start = std::chrono::steady_clock::now();
        if (max_vecs > kMaxVecs || keep > 4 || keep < 1 || keep >= max_vecs || max_vecs < 3)
                return set_error(T3NS_E_LIMIT, "davidson: need 1 <= keep_deflate <= 4, "
                                               "keep_deflate < max_vecs <= 32");
        if (n <= 0) return set_error(T3NS_E_ARG, "davidson: empty vector");
        DavidsonBuffers b;
        const int mv = alloc_basis(b, n, max_vecs);
        if (mv < 0) return set_error(T3NS_E_NOMEM, "davidson: cannot allocate the basis");
        T3NS_CUDA_TRY(cudaMalloc(&b.t, sizeof(double) * n));
        T3NS_CUDA_TRY(cudaMalloc(&b.S, sizeof(double) * mv * mv));
        T3NS_CUDA_TRY(cudaMalloc(&b.Z, sizeof(double) * mv * mv));
        T3NS_CUDA_TRY(cudaMalloc(&b.w, sizeof(double) * mv));
        T3NS_CUDA_TRY(cudaMalloc(&b.partials, sizeof(double) * kRedBlocks * 64));
        T3NS_CUDA_TRY(cudaMalloc(&b.coef, sizeof(double) * 64));
        T3NS_CUDA_TRY(cudaMalloc(&b.scal, sizeof(double) * 8));
        T3NS_CUDA_TRY(cudaMalloc(&b.status, sizeof(int)));
        T3NS_CUDA_TRY(cudaMalloc(&b.dm, sizeof(int)));
        T3NS_CUDA_TRY(cudaMalloc(&b.vin, sizeof(double) * n));
        T3NS_CUDA_TRY(cudaMalloc(&b.vout, sizeof(double) * n));
        T3NS_CUDA_TRY(cudaMallocHost(&b.host_scal, sizeof(double) * 8));
        T3NS_CUDA_TRY(cudaMemsetAsync(b.S, 0, sizeof(double) * mv * mv, s));
        T3NS_CUDA_TRY(cudaMemcpyAsync(b.t, d_result, sizeof(double) * n,
                                      cudaMemcpyDeviceToDevice, s));
        const int G = kRedBlocks, T = kRedThreads;
        int m = 0, its = 0, since_best = 0;
        bool stalled = false;
        double res = tol * 10, e_old = 0, d_e = tol * 10, best_res = 0;
        *energy = 0;
        T3NS_CUDA_TRY(cudaMemsetAsync(b.dm, 0, sizeof(int), s));

        // One iteration, with every m-dependent count and column read from
        // b.dm on the device (so it can be captured once and replayed):
        // new search vector (CGS2 + normalise), matvec, new column of S,
        // Rayleigh-Ritz, deflation when the basis is full, Ritz vector and
        // residual, the host's 4 doubles, preconditioner.
        auto column_of_S = [&](const int *dm, int col) {
                // S[i, c] = V_i . VA_c for i <= c, c = m (dm) or col (dm == nullptr)
                dots_kernel<<<G, T, 0, s>>>(b.V, n, dm, dm ? 1 : col + 1,
                                            b.VA + (dm ? 0 : (int64_t) col * n), dm ? 1 : 0, n,
                                            b.partials);
                reduce_partials_kernel<<<1, 64, 0, s>>>(b.partials, G, dm, dm ? 1 : col + 1,
                                                        b.S + (dm ? 0 : (int64_t) col * mv),
                                                        dm ? mv : 0, 1, 1.0);
        };
        auto body = [&](bool deflate) -> int {
                for (int pass = 0; pass < 2; ++pass) {
                        dots_kernel<<<G, T, 0, s>>>(b.V, n, b.dm, 0, b.t, 0, n, b.partials);
                        reduce_partials_kernel<<<1, 64, 0, s>>>(b.partials, G, b.dm, 0, b.coef, 0, 1, 1.0);
                        gs_update_kernel<<<G, T, 0, s>>>(b.V, n, b.dm, b.coef, b.t, n, b.partials);
                }
                normalize_kernel<<<G, T, 0, s>>>(b.t, b.V, n, b.dm, b.vin, n, b.partials, G);
                T3NS_CUDA_TRY(cudaGetLastError());
                T3NS_TRY(matvec(b.vin, b.vout, s));
                store_column_kernel<<<G, T, 0, s>>>(b.vout, b.VA, n, b.dm, n);
                column_of_S(b.dm, 0);
                set_m_kernel<<<1, 1, 0, s>>>(b.dm, 1, -1);
                jacobi_eig_kernel<<<1, 256, 0, s>>>(b.S, mv, b.dm, b.Z, b.w, b.status);
                if (deflate) {
                        deflate_kernel<<<G, T, 0, s>>>(b.V, n, mv, b.Z, mv, keep, n);
                        deflate_kernel<<<G, T, 0, s>>>(b.VA, n, mv, b.Z, mv, keep, n);
                        set_m_kernel<<<1, 1, 0, s>>>(b.dm, 0, keep);
                        for (int c = 0; c < keep; ++c) column_of_S(nullptr, c);
                        jacobi_eig_kernel<<<1, 256, 0, s>>>(b.S, mv, b.dm, b.Z, b.w, b.status);
                }
                ritz_kernel<<<G, T, 0, s>>>(b.V, b.VA, n, b.dm, b.Z, b.w, d_diag, d_result, b.t, n,
                                            b.partials);
                reduce_partials_kernel<<<1, 64, 0, s>>>(b.partials, G, nullptr, 3, b.scal, 0, 1, 1.0);
                T3NS_CUDA_TRY(cudaGetLastError());
                T3NS_CUDA_TRY(cudaMemcpyAsync(b.host_scal, b.scal, sizeof(double) * 3,
                                              cudaMemcpyDeviceToHost, s));
                T3NS_CUDA_TRY(cudaMemcpyAsync(b.host_scal + 3, b.w, sizeof(double),
                                              cudaMemcpyDeviceToHost, s));
                T3NS_CUDA_TRY(cudaMemcpyAsync(b.host_scal + 4, b.status, sizeof(int),
                                              cudaMemcpyDeviceToHost, s));
                if (mv_err)
                        T3NS_CUDA_TRY(cudaMemcpyAsync(b.host_scal + 5, mv_err, sizeof(int),
                                                      cudaMemcpyDeviceToHost, s));
                precond_kernel<<<G, T, 0, s>>>(d_result, b.t, d_diag, b.scal, b.w, n);
                T3NS_CUDA_TRY(cudaGetLastError());
                return T3NS_OK;
        };
        // graph per iteration kind (plain / deflating), captured on first use
        // after one eager iteration has run (the matvec's one-time set-up
        // calls must not happen under capture)
        cudaGraphExec_t gexec[2] = {nullptr, nullptr};
        auto release = [&]() {
                for (auto &g : gexec)
                        if (g) cudaGraphExecDestroy(g);
        };
        auto run_iteration = [&](bool deflate) -> int {
                if (!use_graphs || its == 0) return body(deflate);
                cudaGraphExec_t &ge = gexec[deflate ? 1 : 0];
                if (!ge) {
                        cudaGraph_t g = nullptr;
                        T3NS_CUDA_TRY(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
                        const int rc = body(deflate);
                        const cudaError_t ce = cudaStreamEndCapture(s, &g);
                        if (rc != T3NS_OK) {
                                if (g) cudaGraphDestroy(g);
                                return rc;
                        }
                        if (ce != cudaSuccess)
                                return set_error(T3NS_E_CUDA, std::string("davidson: capture: ") +
                                                                      cudaGetErrorString(ce));
                        const cudaError_t ie = cudaGraphInstantiate(&ge, g, 0);
                        cudaGraphDestroy(g);
                        if (ie != cudaSuccess)
                                return set_error(T3NS_E_CUDA, std::string("davidson: instantiate: ") +
                                                                      cudaGetErrorString(ie));
                }
                T3NS_CUDA_TRY(cudaGraphLaunch(ge, s));
                return T3NS_OK;
        };

        while (res > tol && its < max_its && !stalled) {
                const bool deflate = m + 1 == mv;
                const int rc = run_iteration(deflate);
                if (rc != T3NS_OK) {
                        release();
                        return rc;
                }
                m = deflate ? keep : m + 1;
                const cudaError_t se = cudaStreamSynchronize(s);
                if (se != cudaSuccess) {
                        release();
                        return set_error(T3NS_E_CUDA, std::string("davidson: iteration failed: ") +
                                                              cudaGetErrorString(se));
                }
                int st = 0;
                if (mv_err) {
                        memcpy(&st, b.host_scal + 5, sizeof(int));
                        if (st != 0) {
                                release();
                                return set_error(T3NS_E_DEVICE, "davidson: matvec kernel reported "
                                                                "error status " + std::to_string(st));
                        }
                }
                memcpy(&st, b.host_scal + 4, sizeof(int));
                if (st != 0) {
                        release();
                        return set_error(T3NS_E_EIG, "davidson: subspace eigensolver did not converge");
                }
                res = sqrt(b.host_scal[0]);
                if (its == 0 || res < 0.9 * best_res) {
                        best_res = res;
                        since_best = 0;
                } else if (stall > 0 && ++since_best >= stall &&
                           res < stall_level * std::max(1.0, fabs(b.host_scal[3]))) {
                        stalled = true;
                }
                const double theta = b.host_scal[3];
                d_e = e_old - theta;
                e_old = theta;
                *energy = theta;
                ++its;
        }
        release();
        T3NS_CUDA_TRY(cudaStreamSynchronize(s));
        if (info) {
                info->iterations = its;
                info->max_vecs = mv;
                info->d_energy = d_e;
                info->residual = res;
                info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() -
                                                              t_start).count();
                info->fp64_iterations = its;
        }
        if (res <= tol) return 0;
        return stalled ? 2 : 1;
}

int davidson_run(t3ns_heff *h, double *d_result, double *energy, int max_vecs,
                 int keep, double tol, int max_its, const double *d_diag,
                 t3ns_davidson_info *info, cudaStream_t s)
{
        auto matvec_in = [h](int precision) {
                return DevMatvec([h, precision](const double *x, double *y, cudaStream_t st) {
                        int launches = 0;
                        return launch_heff(h->dp, precision, x, y, st, &launches);
                });
        };
        // iterations replay captured CUDA graphs unless T3NS_B200_GRAPHS=0
        const char *ge = getenv("T3NS_B200_GRAPHS");
        const bool graphs = !ge || strcmp(ge, "0") != 0;
        if (h->precision == T3NS_PREC_FP64)
                return davidson_core(h->hp.size, matvec_in(T3NS_PREC_FP64), d_result, energy,
                                     max_vecs, keep, tol, max_its, d_diag, info, s, 0, graphs,
                                     h->dp.err);
        // split-precision iterations, then FP64 defect correction from their
        // vector; the split phase leaves at least a quarter of the iterations
        // (and 10) to the FP64 phase
        t3ns_davidson_info i1{}, i2{};
        const auto t0 = std::chrono::steady_clock::now();
        int split_its = std::max(1, max_its - std::max(10, max_its / 4));
        // a vector shorter than the basis: the split phase stops before its
        // basis could span the whole space (the next correction would then
        // vanish in the orthogonalisation), the FP64 phase finishes
        if (h->hp.size <= max_vecs) split_its = (int) std::max<int64_t>(1, std::min<int64_t>(split_its, h->hp.size - 2));
        const double level = h->precision == T3NS_PREC_BF16X3 ? kStallLevelBf16 : kStallLevel;
        int rc = davidson_core(h->hp.size, matvec_in(h->precision), d_result, energy, max_vecs,
                               keep, tol, split_its, d_diag, &i1, s, /*stall=*/4, graphs, h->dp.err,
                               level);
        if (rc < 0) return rc;
        rc = davidson_core(h->hp.size, matvec_in(T3NS_PREC_FP64), d_result, energy, max_vecs,
                           keep, tol, std::max(max_its - i1.iterations, 2), d_diag, &i2, s, 0,
                           graphs, h->dp.err);
        if (rc < 0) return rc;
        if (info) {
                *info = i2;
                info->iterations = i1.iterations + i2.iterations;
                info->fp64_iterations = i2.iterations;
                info->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        }
        return rc == 0 ? 0 : 1;
}

}  // namespace t3ns

using namespace t3ns;

extern "C" {

int t3ns_davidson_device(t3ns_heff *h, double *result, double *energy, int max_vecs,
                         int keep_deflate, double tol, int max_its, const double *diagonal,
                         t3ns_davidson_info *info, void *stream)
{
        if (!h || !result || !energy || !diagonal) return set_error(T3NS_E_ARG, "null argument");
        return davidson_run(h, result, energy, max_vecs, keep_deflate, tol, max_its, diagonal,
                            info, (cudaStream_t) stream);
}

int t3ns_davidson_host(t3ns_heff *h, double *result, double *energy, int max_vecs,
                       int keep_deflate, double tol, int max_its, const double *diagonal,
                       t3ns_davidson_info *info)
{
        if (!h || !result || !energy || !diagonal) return set_error(T3NS_E_ARG, "null argument");
        const size_t bytes = sizeof(double) * h->hp.size;
        double *d_res = nullptr, *d_diag = nullptr;
        T3NS_CUDA_TRY(cudaMalloc(&d_res, bytes));
        if (cudaMalloc(&d_diag, bytes) != cudaSuccess) {
                cudaGetLastError();
                cudaFree(d_res);
                return set_error(T3NS_E_NOMEM, "davidson: diagonal buffer");
        }
        int rc = T3NS_OK;
        if (cudaMemcpy(d_res, result, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(d_diag, diagonal, bytes, cudaMemcpyHostToDevice) != cudaSuccess)
                rc = set_error(T3NS_E_CUDA, "davidson: upload");
        if (rc == T3NS_OK)
                rc = davidson_run(h, d_res, energy, max_vecs, keep_deflate, tol, max_its, d_diag,
                                  info, h->stream);
        if (rc >= 0 && cudaMemcpy(result, d_res, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = set_error(T3NS_E_CUDA, "davidson: download");
        cudaFree(d_res);
        cudaFree(d_diag);
        return rc;
}

int t3ns_davidson_callback(int64_t size, void (*matvec)(const double *, double *, void *),
                           void *ctx, double *result, double *energy, int max_vecs,
                           int keep_deflate, double tol, int max_its, const double *diagonal,
                           t3ns_davidson_info *info)
{
        if (!matvec || !result || !energy || !diagonal || size <= 0)
                return set_error(T3NS_E_ARG, "null argument");
        const size_t bytes = sizeof(double) * size;
        double *d_res = nullptr, *d_diag = nullptr, *h_in = nullptr, *h_out = nullptr;
        cudaStream_t s = nullptr;
        int rc = T3NS_OK;
        if (cudaMalloc(&d_res, bytes) != cudaSuccess || cudaMalloc(&d_diag, bytes) != cudaSuccess ||
            cudaMallocHost(&h_in, bytes) != cudaSuccess || cudaMallocHost(&h_out, bytes) != cudaSuccess ||
            cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
                cudaGetLastError();
                rc = set_error(T3NS_E_NOMEM, "davidson: buffers");
        }
        if (rc == T3NS_OK &&
            (cudaMemcpy(d_res, result, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
             cudaMemcpy(d_diag, diagonal, bytes, cudaMemcpyHostToDevice) != cudaSuccess))
                rc = set_error(T3NS_E_CUDA, "davidson: upload");
        if (rc == T3NS_OK) {
                // the caller's matvec runs on the host: the new basis vector
                // goes down, its image comes back up
                DevMatvec mv = [&](const double *x, double *y, cudaStream_t st) {
                        T3NS_CUDA_TRY(cudaMemcpyAsync(h_in, x, bytes, cudaMemcpyDeviceToHost, st));
                        T3NS_CUDA_TRY(cudaStreamSynchronize(st));
                        matvec(h_in, h_out, ctx);
                        T3NS_CUDA_TRY(cudaMemcpyAsync(y, h_out, bytes, cudaMemcpyHostToDevice, st));
                        return T3NS_OK;
                };
                rc = davidson_core(size, mv, d_res, energy, max_vecs, keep_deflate, tol, max_its,
                                   d_diag, info, s);
        }
        if (rc >= 0 && cudaMemcpy(result, d_res, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
                rc = set_error(T3NS_E_CUDA, "davidson: download");
        if (s) cudaStreamDestroy(s);
        cudaFree(d_res);
        cudaFree(d_diag);
        cudaFreeHost(h_in);
        cudaFreeHost(h_out);
        return rc;
}

int t3ns_precondition_host(int64_t size, const double *result, double theta,
                           const double *diagonal, double *vec_t)
{
        if (!result || !diagonal || !vec_t || size <= 0) return set_error(T3NS_E_ARG, "null argument");
        const size_t bytes = sizeof(double) * size;
        double *d = nullptr;
        double *scal = nullptr;
        int rc = T3NS_OK;
        if (cudaMalloc(&d, 3 * bytes + sizeof(double) * (kRedBlocks * 3 + 8)) != cudaSuccess) {
                cudaGetLastError();
                return set_error(T3NS_E_NOMEM, "precondition: buffers");
        }
        double *d_r = d, *d_diag = d + size, *d_t = d + 2 * size;
        double *part = d + 3 * size;
        scal = part + kRedBlocks * 3;
        double *d_theta = scal + 4;
        if (cudaMemcpy(d_r, result, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(d_diag, diagonal, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(d_t, vec_t, bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(d_theta, &theta, sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
                rc = set_error(T3NS_E_CUDA, "precondition: upload");
        if (rc == T3NS_OK) {
                precond_sums_kernel<<<kRedBlocks, kRedThreads>>>(d_r, d_t, d_diag, d_theta, size, part);
                reduce_partials_kernel<<<1, 64>>>(part, kRedBlocks, nullptr, 3, scal, 0, 1, 1.0);
                precond_kernel<<<kRedBlocks, kRedThreads>>>(d_r, d_t, d_diag, scal, d_theta, size);
                if (cudaGetLastError() != cudaSuccess ||
                    cudaMemcpy(vec_t, d_t, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
                        rc = set_error(T3NS_E_CUDA, "precondition: kernels");
        }
        cudaFree(d);
        return rc;
}

}  // extern "C"
