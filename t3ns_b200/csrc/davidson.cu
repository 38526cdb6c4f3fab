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
#include <cstdio>
#include <cstring>
#include <cmath>
#include <functional>
#include <vector>

#include "common.h"
#include "heff_internal.h"

namespace t3ns {

static constexpr int kRedBlocks = 296;   // 2 x 148 SMs
static constexpr int kRedThreads = 256;
static constexpr int kChunk = 8;         // basis columns per register pass
static constexpr double kDiagCutoff = 1e-12;
static constexpr int kMaxVecs = 32;      // largest Davidson subspace

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

// partials[b * ncols + j] = sum over the rows of block b of V[i, j] * t[i]
__global__ void __launch_bounds__(kRedThreads)
dots_kernel(const double *__restrict__ V, int64_t ld, int ncols,
            const double *__restrict__ t, int64_t n, double *__restrict__ partials)
{
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

// out[j * out_stride] = scale * sum_b partials[b * ncols + j]   (fixed order)
__global__ void reduce_partials_kernel(const double *__restrict__ partials, int nblk, int ncols,
                                       double *__restrict__ out, int out_stride, double scale)
{
        for (int j = threadIdx.x; j < ncols; j += blockDim.x) {
                double s = 0;
                for (int b = 0; b < nblk; ++b) s += partials[b * ncols + j];
                out[j * out_stride] = scale * s;
        }
}

// t[i] -= sum_j V[i, j] coef[j]; partials[b] = block sum of t[i]^2 afterwards
__global__ void __launch_bounds__(kRedThreads)
gs_update_kernel(const double *__restrict__ V, int64_t ld, int ncols,
                 const double *__restrict__ coef, double *__restrict__ t, int64_t n,
                 double *__restrict__ partials)
{
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

// out[i] = t[i] / ||t||, with ||t||^2 = sum of the nblk partials (each block
// reduces them itself, in the same order)
__global__ void __launch_bounds__(kRedThreads)
normalize_kernel(const double *__restrict__ t, double *__restrict__ out, int64_t n,
                 const double *__restrict__ partials, int nblk)
{
        __shared__ double inv;
        if (threadIdx.x == 0) {
                double s = 0;
                for (int b = 0; b < nblk; ++b) s += partials[b];
                inv = 1.0 / sqrt(s);
        }
        __syncthreads();
        const double a = inv;
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x)
                out[i] = t[i] * a;
}

// result = V y, t = VA y - theta result; partials[b*3 + {0,1,2}] =
// {sum t^2, sum uK t, sum uK result} with uK = result / (diag - theta)
// (cutoff kDiagCutoff), i.e. calculate_residue and the reductions of the
// preconditioner fused in one pass.
__global__ void __launch_bounds__(kRedThreads)
ritz_kernel(const double *__restrict__ V, const double *__restrict__ VA, int64_t ld, int m,
            const double *__restrict__ y, const double *__restrict__ theta_p,
            const double *__restrict__ diag, double *__restrict__ result,
            double *__restrict__ t, int64_t n, double *__restrict__ partials)
{
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
__global__ void jacobi_eig_kernel(const double *__restrict__ S, int ld, int m,
                                  double *__restrict__ Z, double *__restrict__ w,
                                  int *__restrict__ status)
{
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
        int *status = nullptr;
        double *host_scal = nullptr;   // pinned
        ~DavidsonBuffers()
        {
                cudaFree(V); cudaFree(VA); cudaFree(t); cudaFree(S); cudaFree(Z); cudaFree(w);
                cudaFree(partials); cudaFree(coef); cudaFree(scal); cudaFree(status);
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

// stall > 0: also stop (returning 2) once the residual has not fallen below
// 0.9 of its best value for `stall` iterations (the split-precision phase,
// whose residual levels off at the matvec's rounding).
static int davidson_core(int64_t n, const DevMatvec &matvec, double *d_result, double *energy,
                         int max_vecs, int keep, double tol, int max_its, const double *d_diag,
                         t3ns_davidson_info *info, cudaStream_t s, int stall = 0)
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
        T3NS_CUDA_TRY(cudaMallocHost(&b.host_scal, sizeof(double) * 8));
        T3NS_CUDA_TRY(cudaMemsetAsync(b.S, 0, sizeof(double) * mv * mv, s));
        T3NS_CUDA_TRY(cudaMemcpyAsync(b.t, d_result, sizeof(double) * n,
                                      cudaMemcpyDeviceToDevice, s));
        const int G = kRedBlocks, T = kRedThreads;
        int m = 0, its = 0, since_best = 0;
        bool stalled = false;
        double res = tol * 10, e_old = 0, d_e = tol * 10, best_res = 0;
        *energy = 0;

        auto column_of_S = [&](int col) -> int {
                // S[i, col] = V_i . VA_col, i <= col
                dots_kernel<<<G, T, 0, s>>>(b.V, n, col + 1, b.VA + (int64_t) col * n, n, b.partials);
                reduce_partials_kernel<<<1, 64, 0, s>>>(b.partials, G, col + 1,
                                                        b.S + (int64_t) col * mv, 1, 1.0);
                T3NS_CUDA_TRY(cudaGetLastError());
                return T3NS_OK;
        };
        auto eigsolve = [&](int mm) -> int {
                jacobi_eig_kernel<<<1, 256, 0, s>>>(b.S, mv, mm, b.Z, b.w, b.status);
                T3NS_CUDA_TRY(cudaGetLastError());
                return T3NS_OK;
        };

        while (res > tol && its < max_its && !stalled) {
                double *vm = b.V + (int64_t) m * n;
                if (m > 0) {
                        for (int pass = 0; pass < 2; ++pass) {
                                dots_kernel<<<G, T, 0, s>>>(b.V, n, m, b.t, n, b.partials);
                                reduce_partials_kernel<<<1, 64, 0, s>>>(b.partials, G, m, b.coef, 1, 1.0);
                                gs_update_kernel<<<G, T, 0, s>>>(b.V, n, m, b.coef, b.t, n, b.partials);
                        }
                } else {
                        norm2_kernel<<<G, T, 0, s>>>(b.t, n, b.partials);
                }
                normalize_kernel<<<G, T, 0, s>>>(b.t, vm, n, b.partials, G);
                T3NS_CUDA_TRY(cudaGetLastError());
                T3NS_TRY(matvec(vm, b.VA + (int64_t) m * n, s));
                T3NS_TRY(column_of_S(m));
                ++m;
                T3NS_TRY(eigsolve(m));
                if (m == mv) {
                        deflate_kernel<<<G, T, 0, s>>>(b.V, n, mv, b.Z, mv, keep, n);
                        deflate_kernel<<<G, T, 0, s>>>(b.VA, n, mv, b.Z, mv, keep, n);
                        T3NS_CUDA_TRY(cudaGetLastError());
                        m = 0;
                        while (m < keep) {
                                T3NS_TRY(column_of_S(m));
                                ++m;
                        }
                        T3NS_TRY(eigsolve(m));
                }
                ritz_kernel<<<G, T, 0, s>>>(b.V, b.VA, n, m, b.Z, b.w, d_diag, d_result, b.t, n,
                                            b.partials);
                reduce_partials_kernel<<<1, 64, 0, s>>>(b.partials, G, 3, b.scal, 1, 1.0);
                T3NS_CUDA_TRY(cudaGetLastError());
                T3NS_CUDA_TRY(cudaMemcpyAsync(b.host_scal, b.scal, sizeof(double) * 3,
                                              cudaMemcpyDeviceToHost, s));
                T3NS_CUDA_TRY(cudaMemcpyAsync(b.host_scal + 3, b.w, sizeof(double),
                                              cudaMemcpyDeviceToHost, s));
                T3NS_CUDA_TRY(cudaMemcpyAsync(b.host_scal + 4, b.status, sizeof(int),
                                              cudaMemcpyDeviceToHost, s));
                T3NS_CUDA_TRY(cudaStreamSynchronize(s));
                int st = 0;
                memcpy(&st, b.host_scal + 4, sizeof(int));
                if (st != 0) return set_error(T3NS_E_EIG, "davidson: subspace eigensolver did not converge");
                res = sqrt(b.host_scal[0]);
                if (its == 0 || res < 0.9 * best_res) {
                        best_res = res;
                        since_best = 0;
                } else if (stall > 0 && ++since_best >= stall) {
                        stalled = true;
                }
                const double theta = b.host_scal[3];
                d_e = e_old - theta;
                e_old = theta;
                *energy = theta;
                ++its;
                precond_kernel<<<G, T, 0, s>>>(d_result, b.t, d_diag, b.scal, b.w, n);
                T3NS_CUDA_TRY(cudaGetLastError());
        }
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
        if (h->precision == T3NS_PREC_FP64)
                return davidson_core(h->hp.size, matvec_in(T3NS_PREC_FP64), d_result, energy,
                                     max_vecs, keep, tol, max_its, d_diag, info, s);
        // split-precision iterations, then FP64 defect correction from their vector
        t3ns_davidson_info i1{}, i2{};
        const auto t0 = std::chrono::steady_clock::now();
        int rc = davidson_core(h->hp.size, matvec_in(h->precision), d_result, energy, max_vecs,
                               keep, tol, max_its, d_diag, &i1, s, /*stall=*/4);
        if (rc < 0) return rc;
        rc = davidson_core(h->hp.size, matvec_in(T3NS_PREC_FP64), d_result, energy, max_vecs,
                           keep, tol, std::max(max_its - i1.iterations, 2), d_diag, &i2, s);
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
                reduce_partials_kernel<<<1, 64>>>(part, kRedBlocks, 3, scal, 1, 1.0);
                precond_kernel<<<kRedBlocks, kRedThreads>>>(d_r, d_t, d_diag, scal, d_theta, size);
                if (cudaGetLastError() != cudaSuccess ||
                    cudaMemcpy(vec_t, d_t, bytes, cudaMemcpyDeviceToHost) != cudaSuccess)
                        rc = set_error(T3NS_E_CUDA, "precondition: kernels");
        }
        cudaFree(d);
        return rc;
}

}  // extern "C"
