// CTA-wide FP64 GEMM on the FP64 tensor pipe (mma.sync.m8n8k4.f64), for the
// operator-update kernels: C = alpha * op(A) * op(B) + beta * C with
// column-major operands in global or shared memory, any M, N, K.
// Each warp owns 16x16 output tiles (2x2 mma per k-step of 4).
#pragma once
#include <cstdint>

namespace t3ns {

__device__ __forceinline__ void dmma884(double &d0, double &d1, double a, double b)
{
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                     : "+d"(d0), "+d"(d1)
                     : "d"(a), "d"(b));
}

// op(A)(m,k) = TA ? A[k + m*lda] : A[m + k*lda]
// op(B)(k,n) = TB ? B[n + k*ldb] : B[k + n*ldb]
// beta == 0 never reads C.  All warps of the CTA must call it (it contains
// no barrier; callers separate dependent GEMMs with __syncthreads()).
template <bool TA, bool TB>
__device__ void cta_dgemm(int M, int N, int K, double alpha, const double *A, int64_t lda,
                          const double *B, int64_t ldb, double beta, double *C, int64_t ldc)
{
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int nwarps = blockDim.x >> 5;
        const int lr = lane >> 2, lc = lane & 3;
        const int mt = (M + 15) >> 4, nt = (N + 15) >> 4;
        for (int t = warp; t < mt * nt; t += nwarps) {
                const int m0 = (t % mt) << 4, n0 = (t / mt) << 4;
                double d[2][2][2] = {{{0, 0}, {0, 0}}, {{0, 0}, {0, 0}}};
                const int ma[2] = {m0 + lr, m0 + 8 + lr};
                const int nb[2] = {n0 + lr, n0 + 8 + lr};
                for (int k0 = 0; k0 < K; k0 += 4) {
                        const int k = k0 + lc;
                        double a[2], b[2];
#pragma unroll
                        for (int i = 0; i < 2; ++i) {
                                const bool ok = ma[i] < M && k < K;
                                a[i] = ok ? (TA ? A[k + (int64_t) ma[i] * lda] : A[ma[i] + (int64_t) k * lda]) : 0.0;
                        }
#pragma unroll
                        for (int j = 0; j < 2; ++j) {
                                const bool ok = nb[j] < N && k < K;
                                b[j] = ok ? (TB ? B[nb[j] + (int64_t) k * ldb] : B[k + (int64_t) nb[j] * ldb]) : 0.0;
                        }
#pragma unroll
                        for (int i = 0; i < 2; ++i)
#pragma unroll
                                for (int j = 0; j < 2; ++j) dmma884(d[i][j][0], d[i][j][1], a[i], b[j]);
                }
#pragma unroll
                for (int i = 0; i < 2; ++i) {
                        const int m = m0 + 8 * i + lr;
                        if (m >= M) continue;
#pragma unroll
                        for (int j = 0; j < 2; ++j)
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                        const int n = n0 + 8 * j + 2 * lc + h;
                                        if (n >= N) continue;
                                        double *c = C + m + (int64_t) n * ldc;
                                        const double v = alpha * d[i][j][h];
                                        *c = beta == 0.0 ? v : fma(beta, *c, v);
                                }
                }
        }
}

}  // namespace t3ns
