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
// make_map, src/Heff.c:668-682); blocks are column-major with axis 0
// fastest and operator blocks are (new x old) column-major.  The reference
// applies the three operators one at a time with cblas_dgemm (do_contract,
// src/sparseblocks.c:133-158) in the order chosen per pair by make_cinfo
// (src/Heff.c:629-666).
//
// GPU organisation:
//   * the host flattens the schedule into one term per (pair, instruction)
//     whose three operator blocks are all present (find_operator_tel,
//     src/Heff.c:798-813), grouped by pair, pairs grouped by output block;
//   * an output block becomes one or more work units, tiles along one or two
//     memory axes small enough for a shared-memory accumulator; each tile
//     applies only its own rows of every operator, and the tiling and each
//     pair's contraction order are chosen together by their FLOPs summed over
//     the tiles (a stage that runs before a tiled axis is contracted is
//     repeated for every tile along that axis);
//   * one persistent kernel; each CTA takes units off a global counter
//     (heaviest first), keeps the unit's output tile in shared memory and
//     walks its pairs.  A pair's terms share every block dimension and the
//     contraction order, so G terms at a time go through each stage as one
//     uniform batched small GEMM on the FP64 tensor pipe (mma.m8n8k4,
//     register-blocked warp tiles of up to 32x8 / 16x16 / 8x32); the stage before
//     the last scales by the term prefactor, so the last stage is a plain
//     reduction over the group inside each warp (single owner per output
//     element: no atomics).
#include <cuda_bf16.h>

#include <algorithm>
#include <bitset>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <type_traits>
#include <unordered_map>
#include <vector>

#include "common.h"
#include "heff_internal.h"
#include "heff_v2.cuh"

namespace t3ns {

constexpr int kGMax = 64;         // terms per group
constexpr int kMaxDevices = 64;
constexpr double kPairVisitCost = 4e4;   // FLOP-equivalent of one (unit, pair) visit

// Kernel configurations.  The large one (one 512-thread CTA per SM, 208 KB of
// shared buffers) tiles fewer blocks and hides latency with 16 warps; the
// small one (two 256-thread CTAs per SM) suits steps of many small blocks.
// Both fit the 64K registers of an SM (at most 128 per thread).
struct CfgLarge {
        static constexpr int kThreads = 512, kMinBlocks = 1;
        static constexpr int kOut = 8192, kPsi = 1024, kW = 17408;
};
struct CfgSmall {
        static constexpr int kThreads = 256, kMinBlocks = 2;
        static constexpr int kOut = 3072, kPsi = 1024, kW = 9472;
};
// 24 warps per SM at 80 registers a thread: more warps to hide operand
// latency on large steps, at the price of a few spilled registers
struct CfgWide {
        static constexpr int kThreads = 768, kMinBlocks = 1;
        static constexpr int kOut = 6144, kPsi = 1024, kW = 19456;
};
// Contraction-ordered kernel (heff_v2.cuh): 768 threads with 6,144-element
// output tiles, and 512 threads with 8,192; both stage old blocks of up to
// 4,096 padded elements.
// BF16x3 tilings of the three configurations above: an output tile of FP32
// accumulators and BF16-pair intermediates take half the bytes of FP64
// elements, so the same shared memory holds twice the elements (kOut here
// in FP32 elements; kPsi and kW in FP64-sized slots, two BF16 pairs each).
struct CfgLargeB {
        static constexpr int kThreads = 512, kMinBlocks = 1;
        static constexpr int kOut = 16384, kPsi = 1024, kW = 17408;
};
struct CfgSmallB {
        static constexpr int kThreads = 256, kMinBlocks = 2;
        static constexpr int kOut = 6144, kPsi = 1024, kW = 9472;
};
struct CfgWideB {
        static constexpr int kThreads = 768, kMinBlocks = 1;
        static constexpr int kOut = 12288, kPsi = 1024, kW = 19456;
};
struct CfgV2Wide {
        static constexpr int kThreads = 768, kMinBlocks = 1;
        static constexpr int kOut = 6144, kPsi = 4096, kW = 17408;
};
struct CfgV2Large {
        static constexpr int kThreads = 512, kMinBlocks = 1;
        static constexpr int kOut = 8192, kPsi = 4096, kW = 15360;
};
const KernelCfg kCfgs[kNumCfgs] = {
        {CfgLarge::kThreads, CfgLarge::kMinBlocks, CfgLarge::kOut, CfgLarge::kPsi, CfgLarge::kW,
         "fp64-512x1-out8192", 0},
        {CfgSmall::kThreads, CfgSmall::kMinBlocks, CfgSmall::kOut, CfgSmall::kPsi, CfgSmall::kW,
         "fp64-256x2-out3072", 0},
        {CfgWide::kThreads, CfgWide::kMinBlocks, CfgWide::kOut, CfgWide::kPsi, CfgWide::kW,
         "fp64-768x1-out6144", 0},
        {CfgV2Wide::kThreads, CfgV2Wide::kMinBlocks, CfgV2Wide::kOut, CfgV2Wide::kPsi, CfgV2Wide::kW,
         "fp64-ordered-768x1-out6144", 1},
        {CfgV2Large::kThreads, CfgV2Large::kMinBlocks, CfgV2Large::kOut, CfgV2Large::kPsi,
         CfgV2Large::kW, "fp64-ordered-512x1-out8192", 1},
        // BF16x3 only: plan capacities in BF16 pairs (twice the FP64 slots)
        {CfgLargeB::kThreads, CfgLargeB::kMinBlocks, CfgLargeB::kOut, 2 * CfgLargeB::kPsi,
         2 * CfgLargeB::kW, "bf16-512x1-out16384", 0, 1},
        {CfgSmallB::kThreads, CfgSmallB::kMinBlocks, CfgSmallB::kOut, 2 * CfgSmallB::kPsi,
         2 * CfgSmallB::kW, "bf16-256x2-out6144", 0, 1},
        {CfgWideB::kThreads, CfgWideB::kMinBlocks, CfgWideB::kOut, 2 * CfgWideB::kPsi,
         2 * CfgWideB::kW, "bf16-768x1-out12288", 0, 1},
};

bool cfg_supports(int cfg, int precision)
{
        if (cfg < 0 || cfg >= kNumCfgs) return false;
        if (kCfgs[cfg].bf16) return precision == T3NS_PREC_BF16X3;
        if (kCfgs[cfg].v2) return precision != T3NS_PREC_BF16X3;
        return true;
}


// D(8x8) += A(8x4) * B(4x8) on the FP64 tensor pipe (one warp).  Fragment
// layout (PTX ISA, mma.m8n8k4 .f64): lane l holds A[l/4][l%4], B[l%4][l/4]
// and D[l/4][2*(l%4) + {0,1}].
__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b)
{
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                     : "+d"(d0), "+d"(d1)
                     : "d"(a), "d"(b));
}

// q = a / b, r = a % b for 0 <= a < 2^22 and b > 0, with rb = 1.0f / b: the
// float quotient is off by at most one, which one correction step fixes.
__device__ __forceinline__ int fast_divmod(int a, int b, float rb, int &r)
{
        int q = __float2int_rz(__int2float_rz(a) * rb);
        r = a - q * b;
        if (r < 0) {
                --q;
                r += b;
        } else if (r >= b) {
                ++q;
                r -= b;
        }
        return q;
}

// GEMM row m of a stage -> element offset of its row in A and in C.  A stage
// on memory axis 1 runs its w[2] slices as one GEMM with M = w[0] * w[2]
// (row m = slice m / w[0], row m % w[0] of the slice), so a small w[0] is
// padded once instead of per slice; the other stages have plain rows.
struct RowSplit {
        int div;          // rows per slice (1 << 30 when unsplit)
        float rdiv;
        int64_t a_slice;  // slice stride in A
        int64_t c_slice;  // slice stride in C
        __device__ __forceinline__ int64_t a_off(int m) const
        {
                int r;
                const int q = fast_divmod(m, div, rdiv, r);
                return r + q * a_slice;
        }
        __device__ __forceinline__ int64_t c_off(int m) const
        {
                int r;
                const int q = fast_divmod(m, div, rdiv, r);
                return r + q * c_slice;
        }
};

// Warp tile of (8*RM) x (8*RN) outputs: RM*RN mma per k-step sharing RM A
// fragments and RN B fragments, A(m, k) = Ab[m + k*ak], B(k, n) =
// Bb[k*bk + n*bn]; the next k-step's fragments are loaded before the current
// step's mma are issued.  The K loop runs its full 4-wide steps on pointers
// advanced in place (no per-element index arithmetic or K bound) and a
// predicated tail step.  Loop bounds are warp-uniform (mma.sync needs the
// whole warp); lanes outside M or N read row / column 0 and use zeros.
// Loads of one operand: the operator side (A_OP: A is the operator) reads
// global memory through the read-only path, the other side is the staged
// block or an intermediate in shared memory.
template <bool GLOBAL_RO>
__device__ __forceinline__ double ld_opnd(const double *p)
{
        if constexpr (GLOBAL_RO) return __ldg(p);
        else return *p;
}

template <int RM, int RN, bool A_OP>
__device__ __forceinline__ void warp_tile_mma(double (&d)[RM][RN][2], const double *Ab, int ak,
                                              const RowSplit &rs, const double *Bb, int bk,
                                              int bn, int K, int M, int N, int m0, int n0, int lr,
                                              int lc)
{
        bool mok[RM], nok[RN];
        const double *ap[RM], *bp[RN];
#pragma unroll
        for (int i = 0; i < RM; ++i) {
                const int m = m0 + 8 * i + lr;
                mok[i] = m < M;
                ap[i] = Ab + rs.a_off(mok[i] ? m : 0) + (int64_t) lc * ak;
        }
#pragma unroll
        for (int j = 0; j < RN; ++j) {
                const int n = n0 + 8 * j + lr;
                nok[j] = n < N;
                bp[j] = Bb + (int64_t) (nok[j] ? n : 0) * bn + (int64_t) lc * bk;
        }
        const int64_t astep = 4 * (int64_t) ak, bstep = 4 * (int64_t) bk;
        const int full = K >> 2;
        double a[RM], b[RN];
        auto load_step = [&]() {
#pragma unroll
                for (int i = 0; i < RM; ++i) {
                        a[i] = mok[i] ? ld_opnd<A_OP>(ap[i]) : 0.0;
                        ap[i] += astep;
                }
#pragma unroll
                for (int j = 0; j < RN; ++j) {
                        b[j] = nok[j] ? ld_opnd<!A_OP>(bp[j]) : 0.0;
                        bp[j] += bstep;
                }
        };
        if (full > 0) {
                load_step();
                for (int st = 0; st < full; ++st) {
                        double ca[RM], cb[RN];
#pragma unroll
                        for (int i = 0; i < RM; ++i) ca[i] = a[i];
#pragma unroll
                        for (int j = 0; j < RN; ++j) cb[j] = b[j];
                        if (st + 1 < full) load_step();
#pragma unroll
                        for (int i = 0; i < RM; ++i)
#pragma unroll
                                for (int j = 0; j < RN; ++j)
                                        dmma_8x8x4(d[i][j][0], d[i][j][1], ca[i], cb[j]);
                }
        }
        if (K & 3) {
                const bool kok = lc < (K & 3);
#pragma unroll
                for (int i = 0; i < RM; ++i) a[i] = (mok[i] && kok) ? ld_opnd<A_OP>(ap[i]) : 0.0;
#pragma unroll
                for (int j = 0; j < RN; ++j) b[j] = (nok[j] && kok) ? ld_opnd<!A_OP>(bp[j]) : 0.0;
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int j = 0; j < RN; ++j) dmma_8x8x4(d[i][j][0], d[i][j][1], a[i], b[j]);
        }
}

// The accumulating stage's loop over terms g0, g0 + gstep, ... < g1 of one
// warp tile, as warp_tile_mma per term but pipelined across terms: the K
// loop runs ceil(K/4) steps (the last predicated when K % 4 != 0) and the
// final step of a term already loads the first step of the next term, so a
// term's start does not wait on its operand loads.
template <int RM, int RN, int AX>
__device__ __forceinline__ void warp_tile_mma_terms(double (&d)[RM][RN][2],
                                                    const double *__restrict__ ops,
                                                    const int64_t *opoff, const double *in,
                                                    int in_gs, int g0, int g1, int gstep, int ak,
                                                    const RowSplit &rs, int bk, int bn, int K,
                                                    int M, int N, int m0, int n0, int lr, int lc)
{
        const int S = (K + 3) >> 2, rem = K & 3;
        if (g0 >= g1 || S == 0) return;
        bool mok[RM], nok[RN];
        int64_t ao[RM], bo[RN];
#pragma unroll
        for (int i = 0; i < RM; ++i) {
                const int m = m0 + 8 * i + lr;
                mok[i] = m < M;
                ao[i] = rs.a_off(mok[i] ? m : 0) + (int64_t) lc * ak;
        }
#pragma unroll
        for (int j = 0; j < RN; ++j) {
                const int n = n0 + 8 * j + lr;
                nok[j] = n < N;
                bo[j] = (int64_t) (nok[j] ? n : 0) * bn + (int64_t) lc * bk;
        }
        const int64_t astep = 4 * (int64_t) ak, bstep = 4 * (int64_t) bk;
        const double *ap[RM], *bp[RN];
        auto set_term = [&](int g) {
                const double *op = ops + opoff[g];
                const double *tin = in + (int64_t) g * in_gs;
                const double *Ab = AX == 0 ? op : tin, *Bb = AX == 0 ? tin : op;
#pragma unroll
                for (int i = 0; i < RM; ++i) ap[i] = Ab + ao[i];
#pragma unroll
                for (int j = 0; j < RN; ++j) bp[j] = Bb + bo[j];
        };
        double a[RM], b[RN];
        auto load = [&](int st) {
                const bool kok = st + 1 < S || rem == 0 || lc < rem;
#pragma unroll
                for (int i = 0; i < RM; ++i) {
                        a[i] = (mok[i] && kok) ? ld_opnd<AX == 0>(ap[i]) : 0.0;
                        ap[i] += astep;
                }
#pragma unroll
                for (int j = 0; j < RN; ++j) {
                        b[j] = (nok[j] && kok) ? ld_opnd<AX != 0>(bp[j]) : 0.0;
                        bp[j] += bstep;
                }
        };
        set_term(g0);
        load(0);
        for (int g = g0; g < g1; g += gstep) {
                for (int st = 0; st < S; ++st) {
                        double ca[RM], cb[RN];
#pragma unroll
                        for (int i = 0; i < RM; ++i) ca[i] = a[i];
#pragma unroll
                        for (int j = 0; j < RN; ++j) cb[j] = b[j];
                        if (st + 1 < S) {
                                load(st + 1);
                        } else if (g + gstep < g1) {
                                set_term(g + gstep);
                                load(0);
                        }
#pragma unroll
                        for (int i = 0; i < RM; ++i)
#pragma unroll
                                for (int j = 0; j < RN; ++j)
                                        dmma_8x8x4(d[i][j][0], d[i][j][1], ca[i], cb[j]);
                }
        }
}

// One contraction stage for G terms.  Term g applies rows [row0, row0+rows)
// of the operator block at ops + opoff[g] (leading dimension ldop) on axis ax
// of `in + g * in_gs` (dims w), writing `out + g * out_gs` (scaled by
// scale[g] when scale != nullptr).  With ACC the G results are summed into
// `out` instead (which then has no term stride).  Each warp owns
// (8*RM) x (8*RN) output tiles and runs their K loop on the FP64 tensor
// pipe; with ACC the group reduction stays inside the warp's accumulators.
template <bool ACC, int RM, int RN, int NW, int AX>
__device__ __forceinline__ void grouped_stage_t(const int *w, int rows, int ldop, int G,
                                                const int64_t *opoff,
                                                const double *__restrict__ ops, const double *in,
                                                int in_gs, double *out, int out_gs,
                                                const double *scale, double *scratch,
                                                int scratch_cap, const int *in_idx)
{
        int M, N, K, ak, bk, bn, cn;
        RowSplit rs{1 << 30, 1.0f / (1 << 30), 0, 0};
        // A(m,k) = Ab[rs.a_off(m) + k*ak], B(k,n) = Bb[k*bk + n*bn],
        // C(m,n) = Cb[rs.c_off(m) + n*cn]
        if constexpr (AX == 0) {
                M = rows; N = w[1] * w[2]; K = w[0];
                ak = ldop; bk = 1; bn = K; cn = rows;
        } else if constexpr (AX == 1) {
                M = w[0] * w[2]; N = rows; K = w[1];
                ak = w[0]; bk = ldop; bn = 1; cn = w[0];
                rs = RowSplit{w[0], 1.0f / w[0], (int64_t) w[0] * w[1], (int64_t) w[0] * rows};
        } else {
                M = w[0] * w[1]; N = rows; K = w[2];
                ak = M; bk = ldop; bn = 1; cn = M;
        }
        const int mt = (M + 8 * RM - 1) / (8 * RM), nt = (N + 8 * RN - 1) / (8 * RN);
        const int tiles = mt * nt;
        // The accumulating stage sums the G terms inside each warp.  When its
        // output has fewer tiles than the CTA has warps, the terms are dealt
        // out to P parts (term g to part g % P) so P warps share a tile; the
        // parts' partial tiles go to scratch and are added in part order
        // (deterministic).
        int P = 1;
        const int MN = M * N;
        if (ACC && tiles < NW && G > 1 && scratch) {
                P = min(G, NW / tiles);
                P = min(P, scratch_cap / max(MN, 1));
                if (P < 2) P = 1;
        }
        const int items = (ACC ? P : G) * tiles;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int lr = lane >> 2, lc = lane & 3;
        const float r_tiles = 1.0f / tiles, r_mt = 1.0f / mt;
        for (int it = warp; it < items; it += NW) {
                int tile, tm;
                const int q = fast_divmod(it, tiles, r_tiles, tile);   // term (or part)
                const int g0 = q;
                const int tn = fast_divmod(tile, mt, r_mt, tm);
                const int g1 = ACC ? G : g0 + 1;
                const int gstep = ACC ? P : 1;
                const int m0 = tm * 8 * RM, n0 = tn * 8 * RN;
                double d[RM][RN][2];
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int j = 0; j < RN; ++j) d[i][j][0] = d[i][j][1] = 0.0;
                if constexpr (ACC) {
                        warp_tile_mma_terms<RM, RN, AX>(d, ops, opoff, in, in_gs, g0, g1, gstep, ak,
                                                        rs, bk, bn, K, M, N, m0, n0, lr, lc);
                } else {
                        const double *op = ops + opoff[g0];
                        const double *tin = in + (in_idx ? in_idx[g0] : g0) * in_gs;
                        if constexpr (AX == 0)
                                warp_tile_mma<RM, RN, true>(d, op, ak, rs, tin, bk, bn, K, M, N, m0,
                                                            n0, lr, lc);
                        else
                                warp_tile_mma<RM, RN, false>(d, tin, ak, rs, op, bk, bn, K, M, N, m0,
                                                             n0, lr, lc);
                }
                const double sc = (!ACC && scale) ? scale[g0] : 1.0;
                double *Cb = out + (ACC ? 0 : g0 * out_gs);
#pragma unroll
                for (int i = 0; i < RM; ++i) {
                        const int mc = m0 + 8 * i + lr;
                        if (mc >= M) continue;
                        double *crow = Cb + rs.c_off(mc);
#pragma unroll
                        for (int j = 0; j < RN; ++j) {
                                const int nc0 = n0 + 8 * j + 2 * lc;
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                        if (nc0 + h >= N) continue;
                                        if (ACC && P > 1) {
                                                scratch[(int64_t) q * MN + mc + (nc0 + h) * M] = d[i][j][h];
                                                continue;
                                        }
                                        double *cp = crow + (nc0 + h) * cn;
                                        *cp = ACC ? *cp + d[i][j][h] : sc * d[i][j][h];
                                }
                        }
                }
        }
        if (ACC && P > 1) {
                __syncthreads();
                const float r_m = 1.0f / M;
                for (int e = threadIdx.x; e < MN; e += NW * 32) {
                        int m;
                        const int n = fast_divmod(e, M, r_m, m);
                        double sum = 0.0;
                        for (int p = 0; p < P; ++p) sum += scratch[(int64_t) p * MN + e];
                        out[rs.c_off(m) + (int64_t) n * cn] += sum;
                }
        }
}

// Warp-tile shape per stage: 8x32 when M is small, 32x8 when N is small,
// else 16x16.
template <bool ACC, int NW>
__device__ __forceinline__ void grouped_stage(int ax, const int *w, int rows, int ldop, int G,
                                              const int64_t *opoff,
                                              const double *__restrict__ ops, const double *in,
                                              int in_gs, double *out, int out_gs,
                                              const double *scale, double *scratch = nullptr,
                                              int scratch_cap = 0, const int *in_idx = nullptr)
{
        const int M = ax == 0 ? rows : ax == 1 ? w[0] * w[2] : w[0] * w[1];
        const int N = ax == 0 ? w[1] * w[2] : rows;
        // the stage axis is a template parameter: it fixes which operand is
        // the operator (global) and which the staged data (shared memory)
        auto go = [&](auto axc) {
                constexpr int AX = decltype(axc)::value;
                if (M <= 8)
                        grouped_stage_t<ACC, 1, 4, NW, AX>(w, rows, ldop, G, opoff, ops, in, in_gs, out,
                                                           out_gs, scale, scratch, scratch_cap, in_idx);
                else if (N <= 8)
                        grouped_stage_t<ACC, 4, 1, NW, AX>(w, rows, ldop, G, opoff, ops, in, in_gs, out,
                                                           out_gs, scale, scratch, scratch_cap, in_idx);
                else
                        grouped_stage_t<ACC, 2, 2, NW, AX>(w, rows, ldop, G, opoff, ops, in, in_gs, out,
                                                           out_gs, scale, scratch, scratch_cap, in_idx);
        };
        if (ax == 0) go(std::integral_constant<int, 0>{});
        else if (ax == 1) go(std::integral_constant<int, 1>{});
        else go(std::integral_constant<int, 2>{});
}

// ---------------------------------------------------------------------------
// Split-precision stages: products on the TF32 tensor pipe (mma.m16n8k8) as
// 3xTF32 -- x = hi + lo with hi = tf32(x), lo = tf32(x - hi),
// x*y ~ lo_x*hi_y + hi_x*lo_y + hi_x*hi_y (the lo*lo term, ~2^-22 relative,
// is dropped) -- with FP32 accumulation.  Operands are stored already split,
// as float2 {hi, lo}: the operators once per plan, Psi once per matvec, and
// every intermediate when a stage writes it, so the inner loop loads a pair
// and issues the three products with no conversion.

__device__ __forceinline__ uint32_t to_tf32(float x)
{
        uint32_t r;
        asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
        return r;
}

__device__ __forceinline__ float2 split_tf32(float x)
{
        const uint32_t hi = to_tf32(x);
        return make_float2(__uint_as_float(hi), __uint_as_float(to_tf32(x - __uint_as_float(hi))));
}

// D(16x8) += A(16x8) * B(8x8).  Fragments (PTX ISA, mma.m16n8k8 .tf32), with
// g = lane/4, t = lane%4: a = {A[g][t], A[g+8][t], A[g][t+4], A[g+8][t+4]},
// b = {B[t][g], B[t+4][g]}, d = {D[g][2t], D[g][2t+1], D[g+8][2t], D[g+8][2t+1]}.
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
        asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, "
                     "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                     : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                     : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// Warp tile of (16*RM) x (8*RN) outputs over pre-split operands.
// A(m,k) = Ab[arow(m) + k*ak] and B(k,n) = Bb[k*bk + bcol(n)], where the row
// (column) offsets are the stage's RowSplit offsets on the split side
// (split_a: rows of A, else columns of B) and m*am (n*bn) otherwise, taken
// once per tile.  Loop bounds warp-uniform; lanes outside M, N or K use zeros.
template <int RM, int RN>
__device__ __forceinline__ void warp_tile_tf32x3(float (&d)[RM][RN][4], const float2 *Ab, int am,
                                                 int ak, const float2 *Bb, int bk, int bn,
                                                 const RowSplit &rs, bool split_a, int K, int M,
                                                 int N, int m0, int n0, int g, int t)
{
        // 32-bit element offsets from the tile's bases (a block and its
        // intermediates are far below 2^31 elements); -1 marks a lane outside
        // M or N
        int ao[RM][2], bo[RN];
#pragma unroll
        for (int i = 0; i < RM; ++i)
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                        const int m = m0 + 16 * i + 8 * r + g;
                        ao[i][r] = m < M ? (int) (split_a ? rs.a_off(m) : (int64_t) m * am) + t * ak : -1;
                }
#pragma unroll
        for (int j = 0; j < RN; ++j) {
                const int n = n0 + 8 * j + g;
                bo[j] = n < N ? (int) (split_a ? (int64_t) n * bn : rs.a_off(n)) + t * bk : -1;
        }
        const int a4 = 4 * ak, b4 = 4 * bk;
        const float2 zero = make_float2(0.f, 0.f);
        for (int k0 = 0, ka = 0, kb = 0; k0 < K; k0 += 8, ka += 2 * a4, kb += 2 * b4) {
                const bool k0ok = k0 + t < K, k1ok = k0 + t + 4 < K;
                uint32_t ah[RM][4], al[RM][4], bh[RN][2], bl[RN][2];
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int r = 0; r < 2; ++r) {
                                const bool ok = ao[i][r] >= 0;
                                const float2 v0 = (ok && k0ok) ? Ab[ao[i][r] + ka] : zero;
                                const float2 v1 = (ok && k1ok) ? Ab[ao[i][r] + ka + a4] : zero;
                                ah[i][r] = __float_as_uint(v0.x);
                                al[i][r] = __float_as_uint(v0.y);
                                ah[i][r + 2] = __float_as_uint(v1.x);
                                al[i][r + 2] = __float_as_uint(v1.y);
                        }
#pragma unroll
                for (int j = 0; j < RN; ++j) {
                        const bool ok = bo[j] >= 0;
                        const float2 v0 = (ok && k0ok) ? Bb[bo[j] + kb] : zero;
                        const float2 v1 = (ok && k1ok) ? Bb[bo[j] + kb + b4] : zero;
                        bh[j][0] = __float_as_uint(v0.x);
                        bl[j][0] = __float_as_uint(v0.y);
                        bh[j][1] = __float_as_uint(v1.x);
                        bl[j][1] = __float_as_uint(v1.y);
                }
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int j = 0; j < RN; ++j) {
                                mma_tf32(d[i][j], al[i], bh[j]);
                                mma_tf32(d[i][j], ah[i], bl[j]);
                                mma_tf32(d[i][j], ah[i], bh[j]);
                        }
        }
}

// ---------------------------------------------------------------------------
// BF16x3 stages: x = hi + lo with hi = bf16(x), lo = bf16(x - hi) (16
// significant bits together), x*y ~ lo_x*hi_y + hi_x*lo_y + hi_x*hi_y on the
// BF16 tensor pipe (mma.m16n8k16), FP32 accumulation; the dropped lo*lo term
// and the representation error are ~2^-16 relative.  An element is stored
// as one 32-bit pair (hi in the low half, lo in the high half): half the
// bytes of an FP64 or {hi, lo} TF32 operand, and twice the K of a TF32 MMA.
struct __align__(4) BfPair {
        uint32_t v;
};

__device__ __forceinline__ uint32_t bf16_bits(float x)
{
        return (uint32_t) __bfloat16_as_ushort(__float2bfloat16_rn(x));
}

__device__ __forceinline__ float bf16_value(uint32_t b)
{
        return __uint_as_float(b << 16);
}

__device__ __forceinline__ BfPair split_bf16(float x)
{
        const uint32_t hi = bf16_bits(x);
        return BfPair{hi | (bf16_bits(x - bf16_value(hi)) << 16)};
}

// D(16x8) += A(16x16) * B(16x8).  Fragments (PTX ISA, mma.m16n8k16 .bf16),
// with g = lane/4, t = lane%4, each register two K-consecutive elements
// (the lower K in the low half): a = {A[g][2t..2t+1], A[g+8][2t..2t+1],
// A[g][2t+8..2t+9], A[g+8][2t+8..2t+9]}, b = {B[2t..2t+1][g],
// B[2t+8..2t+9][g]}; d as for the TF32 MMA.
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
        asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, "
                     "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                     : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                     : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// hi (sel 0x5410) or lo (sel 0x7632) halves of two K-consecutive pairs
__device__ __forceinline__ uint32_t pick(uint32_t p0, uint32_t p1, uint32_t sel)
{
        return __byte_perm(p0, p1, sel);
}

// Warp tile of (16*RM) x (8*RN) outputs over BF16 pairs; addressing as
// warp_tile_tf32x3 (A(m,k) = Ab[arow(m) + k*ak], B(k,n) = Bb[k*bk + bcol(n)]).
template <int RM, int RN>
__device__ __forceinline__ void warp_tile_x3(float (&d)[RM][RN][4], const BfPair *Ab, int am,
                                             int ak, const BfPair *Bb, int bk, int bn,
                                             const RowSplit &rs, bool split_a, int K, int M, int N,
                                             int m0, int n0, int g, int t)
{
        int ao[RM][2], bo[RN];
#pragma unroll
        for (int i = 0; i < RM; ++i)
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                        const int m = m0 + 16 * i + 8 * r + g;
                        ao[i][r] = m < M ? (int) (split_a ? rs.a_off(m) : (int64_t) m * am) + 2 * t * ak : -1;
                }
#pragma unroll
        for (int j = 0; j < RN; ++j) {
                const int n = n0 + 8 * j + g;
                bo[j] = n < N ? (int) (split_a ? (int64_t) n * bn : rs.a_off(n)) + 2 * t * bk : -1;
        }
        const uint32_t *A = reinterpret_cast<const uint32_t *>(Ab);
        const uint32_t *B = reinterpret_cast<const uint32_t *>(Bb);
        for (int k0 = 0, ka = 0, kb = 0; k0 < K; k0 += 16, ka += 16 * ak, kb += 16 * bk) {
                // this lane's K indices: k0 + 2t + {0, 1, 8, 9}
                const int kk = k0 + 2 * t;
                const bool q0 = kk < K, q1 = kk + 1 < K, q2 = kk + 8 < K, q3 = kk + 9 < K;
                uint32_t ah[RM][4], al[RM][4], bh[RN][2], bl[RN][2];
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int r = 0; r < 2; ++r) {
                                const bool ok = ao[i][r] >= 0;
                                const int o = ao[i][r] + ka;
                                const uint32_t e0 = (ok && q0) ? A[o] : 0u;
                                const uint32_t e1 = (ok && q1) ? A[o + ak] : 0u;
                                const uint32_t e2 = (ok && q2) ? A[o + 8 * ak] : 0u;
                                const uint32_t e3 = (ok && q3) ? A[o + 9 * ak] : 0u;
                                ah[i][r] = pick(e0, e1, 0x5410);
                                al[i][r] = pick(e0, e1, 0x7632);
                                ah[i][r + 2] = pick(e2, e3, 0x5410);
                                al[i][r + 2] = pick(e2, e3, 0x7632);
                        }
#pragma unroll
                for (int j = 0; j < RN; ++j) {
                        const bool ok = bo[j] >= 0;
                        const int o = bo[j] + kb;
                        const uint32_t f0 = (ok && q0) ? B[o] : 0u;
                        const uint32_t f1 = (ok && q1) ? B[o + bk] : 0u;
                        const uint32_t f2 = (ok && q2) ? B[o + 8 * bk] : 0u;
                        const uint32_t f3 = (ok && q3) ? B[o + 9 * bk] : 0u;
                        bh[j][0] = pick(f0, f1, 0x5410);
                        bl[j][0] = pick(f0, f1, 0x7632);
                        bh[j][1] = pick(f2, f3, 0x5410);
                        bl[j][1] = pick(f2, f3, 0x7632);
                }
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int j = 0; j < RN; ++j) {
                                mma_bf16(d[i][j], al[i], bh[j]);
                                mma_bf16(d[i][j], ah[i], bl[j]);
                                mma_bf16(d[i][j], ah[i], bh[j]);
                        }
        }
}

// The BF16x3 tile with the operator side in the k-paired layout of the
// BF16 operator copy: element (r, k) of an operator block with leading
// dimension ld (the new dim) at (k/2)*2*ld + 2*r + (k%2), an odd K padded
// with a zero column, so the two K-consecutive pairs a lane needs come in
// one 8-byte load.  A_PK / B_PK: which operand is the operator (unit row or
// column stride there, k stride ak / bk = ld); the other is read as in
// warp_tile_x3.  Every paired offset is even (the copy places a block at
// twice its FP64 offset), so the 8-byte loads are aligned.
template <int RM, int RN, bool A_PK, bool B_PK>
__device__ __forceinline__ void warp_tile_x3_pk(float (&d)[RM][RN][4], const BfPair *Ab, int am,
                                                int ak, const BfPair *Bb, int bk, int bn,
                                                const RowSplit &rs, bool split_a, int K, int M,
                                                int N, int m0, int n0, int g, int t)
{
        int ao[RM][2], bo[RN];
#pragma unroll
        for (int i = 0; i < RM; ++i)
#pragma unroll
                for (int r = 0; r < 2; ++r) {
                        const int m = m0 + 16 * i + 8 * r + g;
                        if (A_PK)
                                ao[i][r] = m < M ? 2 * m + 2 * t * ak : -1;
                        else
                                ao[i][r] = m < M ? (int) (split_a ? rs.a_off(m) : (int64_t) m * am) +
                                                           2 * t * ak
                                                 : -1;
                }
#pragma unroll
        for (int j = 0; j < RN; ++j) {
                const int n = n0 + 8 * j + g;
                if (B_PK)
                        bo[j] = n < N ? 2 * n + 2 * t * bk : -1;
                else
                        bo[j] = n < N ? (int) (split_a ? (int64_t) n * bn : rs.a_off(n)) + 2 * t * bk : -1;
        }
        const uint32_t *A = reinterpret_cast<const uint32_t *>(Ab);
        const uint32_t *B = reinterpret_cast<const uint32_t *>(Bb);
        for (int k0 = 0, ka = 0, kb = 0; k0 < K; k0 += 16, ka += 16 * ak, kb += 16 * bk) {
                const int kk = k0 + 2 * t;
                const bool q0 = kk < K, q1 = kk + 1 < K, q2 = kk + 8 < K, q3 = kk + 9 < K;
                uint32_t ah[RM][4], al[RM][4], bh[RN][2], bl[RN][2];
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int r = 0; r < 2; ++r) {
                                const bool ok = ao[i][r] >= 0;
                                const int o = ao[i][r] + ka;
                                uint32_t e0 = 0u, e1 = 0u, e2 = 0u, e3 = 0u;
                                if (A_PK) {
                                        if (ok && q0) {
                                                const uint2 v = *reinterpret_cast<const uint2 *>(A + o);
                                                e0 = v.x;
                                                e1 = v.y;
                                        }
                                        if (ok && q2) {
                                                const uint2 v = *reinterpret_cast<const uint2 *>(A + o + 8 * ak);
                                                e2 = v.x;
                                                e3 = v.y;
                                        }
                                } else {
                                        e0 = (ok && q0) ? A[o] : 0u;
                                        e1 = (ok && q1) ? A[o + ak] : 0u;
                                        e2 = (ok && q2) ? A[o + 8 * ak] : 0u;
                                        e3 = (ok && q3) ? A[o + 9 * ak] : 0u;
                                }
                                ah[i][r] = pick(e0, e1, 0x5410);
                                al[i][r] = pick(e0, e1, 0x7632);
                                ah[i][r + 2] = pick(e2, e3, 0x5410);
                                al[i][r + 2] = pick(e2, e3, 0x7632);
                        }
#pragma unroll
                for (int j = 0; j < RN; ++j) {
                        const bool ok = bo[j] >= 0;
                        const int o = bo[j] + kb;
                        uint32_t f0 = 0u, f1 = 0u, f2 = 0u, f3 = 0u;
                        if (B_PK) {
                                if (ok && q0) {
                                        const uint2 v = *reinterpret_cast<const uint2 *>(B + o);
                                        f0 = v.x;
                                        f1 = v.y;
                                }
                                if (ok && q2) {
                                        const uint2 v = *reinterpret_cast<const uint2 *>(B + o + 8 * bk);
                                        f2 = v.x;
                                        f3 = v.y;
                                }
                        } else {
                                f0 = (ok && q0) ? B[o] : 0u;
                                f1 = (ok && q1) ? B[o + bk] : 0u;
                                f2 = (ok && q2) ? B[o + 8 * bk] : 0u;
                                f3 = (ok && q3) ? B[o + 9 * bk] : 0u;
                        }
                        bh[j][0] = pick(f0, f1, 0x5410);
                        bl[j][0] = pick(f0, f1, 0x7632);
                        bh[j][1] = pick(f2, f3, 0x5410);
                        bl[j][1] = pick(f2, f3, 0x7632);
                }
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int j = 0; j < RN; ++j) {
                                mma_bf16(d[i][j], al[i], bh[j]);
                                mma_bf16(d[i][j], ah[i], bl[j]);
                                mma_bf16(d[i][j], ah[i], bh[j]);
                        }
        }
}

// the 3xTF32 tile under the common name of the split stages
template <int RM, int RN>
__device__ __forceinline__ void warp_tile_x3(float (&d)[RM][RN][4], const float2 *Ab, int am,
                                             int ak, const float2 *Bb, int bk, int bn,
                                             const RowSplit &rs, bool split_a, int K, int M, int N,
                                             int m0, int n0, int g, int t)
{
        warp_tile_tf32x3<RM, RN>(d, Ab, am, ak, Bb, bk, bn, rs, split_a, K, M, N, m0, n0, g, t);
}

__device__ __forceinline__ void store_out(BfPair *p, float v, float sc, bool acc)
{
        *p = split_bf16(sc * v);   // intermediates: split once, here
}

__device__ __forceinline__ void store_out(float2 *p, float v, float sc, bool acc)
{
        *p = split_tf32(sc * v);   // intermediates: split once, here
}

__device__ __forceinline__ void store_out(float *p, float v, float sc, bool acc)
{
        *p = acc ? *p + v : sc * v;   // the output tile accumulates in FP32
}

// The grouped stage of the FP64 path for pre-split operands.  The GEMM is
// taken in the orientation that puts the larger of M and N on the tile's
// 16-row side.
template <bool ACC, int RM, int RN, int NW, class E, class OutT>
__device__ __forceinline__ void grouped_stage_x_t(int ax, const int *w, int rows, int ldop, int G,
                                                  const int64_t *opoff,
                                                  const E *__restrict__ ops,
                                                  const E *in, int in_gs, OutT *out,
                                                  int out_gs, const float *scale, bool swap,
                                                  float *scratch, int scratch_cap,
                                                  const int *in_idx)
{
        int M, N, K, ak, bk, bn, cn;
        RowSplit rs{1 << 30, 1.0f / (1 << 30), 0, 0};
        // A(m,k) = Ab[rs.a_off(m) + k*ak], B(k,n) = Bb[k*bk + n*bn],
        // C(m,n) = Cb[rs.c_off(m) + n*cn]  (axis 1: slices merged into M)
        if (ax == 0) {
                M = rows; N = w[1] * w[2]; K = w[0];
                ak = ldop; bk = 1; bn = K; cn = rows;
        } else if (ax == 1) {
                M = w[0] * w[2]; N = rows; K = w[1];
                ak = w[0]; bk = ldop; bn = 1; cn = w[0];
                rs = RowSplit{w[0], 1.0f / w[0], (int64_t) w[0] * w[1], (int64_t) w[0] * rows};
        } else {
                M = w[0] * w[1]; N = rows; K = w[2];
                ak = M; bk = ldop; bn = 1; cn = M;
        }
        // tile orientation (M', N'): swapped, A'(m', k) = B(k, m') and
        // B'(k, n') = A(n', k), whose split rows become B' columns
        const int Mt = swap ? N : M, Nt = swap ? M : N;
        const int mt = (Mt + 16 * RM - 1) / (16 * RM), nt = (Nt + 8 * RN - 1) / (8 * RN);
        const int tiles = mt * nt;
        // terms of the accumulating stage dealt to P parts when its output
        // has fewer tiles than warps (as in the FP64 stage)
        int P = 1;
        const int MN = M * N;
        if (ACC && tiles < NW && G > 1 && scratch) {
                P = min(G, NW / tiles);
                P = min(P, scratch_cap / max(MN, 1));
                if (P < 2) P = 1;
        }
        const int items = (ACC ? P : G) * tiles;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int g = lane >> 2, t = lane & 3;
        const float r_tiles = 1.0f / tiles, r_mt = 1.0f / mt;
        for (int it = warp; it < items; it += NW) {
                int tile, tm;
                const int g0 = fast_divmod(it, tiles, r_tiles, tile);   // term (or part)
                const int tn = fast_divmod(tile, mt, r_mt, tm);
                const int g1 = ACC ? G : g0 + 1;
                const int gstep = ACC ? P : 1;
                const int m0 = tm * 16 * RM, n0 = tn * 8 * RN;
                float d[RM][RN][4];
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int j = 0; j < RN; ++j)
#pragma unroll
                                for (int q = 0; q < 4; ++q) d[i][j][q] = 0.f;
                for (int gg = g0; gg < g1; gg += gstep) {
                        const E *tin = in + (!ACC && in_idx ? in_idx[gg] : gg) * in_gs;
                        if constexpr (std::is_same<E, BfPair>::value) {
                                // k-paired operator copy, each block at twice its offset
                                const E *op = ops + 2 * opoff[gg];
                                const E *Ab = ax == 0 ? op : tin;
                                const E *Bb = ax == 0 ? tin : op;
                                // the operator is A' exactly when (ax == 0) != swap
                                if (swap) {
                                        if (ax == 0)
                                                warp_tile_x3_pk<RM, RN, false, true>(d, Bb, bn, bk, Ab, ak, 1, rs,
                                                                                     false, K, Mt, Nt, m0, n0, g, t);
                                        else
                                                warp_tile_x3_pk<RM, RN, true, false>(d, Bb, bn, bk, Ab, ak, 1, rs,
                                                                                     false, K, Mt, Nt, m0, n0, g, t);
                                } else {
                                        if (ax == 0)
                                                warp_tile_x3_pk<RM, RN, true, false>(d, Ab, 1, ak, Bb, bk, bn, rs,
                                                                                     true, K, Mt, Nt, m0, n0, g, t);
                                        else
                                                warp_tile_x3_pk<RM, RN, false, true>(d, Ab, 1, ak, Bb, bk, bn, rs,
                                                                                     true, K, Mt, Nt, m0, n0, g, t);
                                }
                        } else {
                                const E *op = ops + opoff[gg];
                                const E *Ab = ax == 0 ? op : tin;
                                const E *Bb = ax == 0 ? tin : op;
                                if (swap)
                                        warp_tile_x3<RM, RN>(d, Bb, bn, bk, Ab, ak, 1, rs, false, K, Mt, Nt,
                                                             m0, n0, g, t);
                                else
                                        warp_tile_x3<RM, RN>(d, Ab, 1, ak, Bb, bk, bn, rs, true, K, Mt, Nt,
                                                             m0, n0, g, t);
                        }
                }
                const float sc = (!ACC && scale) ? scale[g0] : 1.f;
                OutT *Cb = out + (ACC ? 0 : g0 * out_gs);
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int r = 0; r < 2; ++r) {
                                const int mc = m0 + 16 * i + 8 * r + g;
                                if (mc >= Mt) continue;
#pragma unroll
                                for (int j = 0; j < RN; ++j)
#pragma unroll
                                        for (int h = 0; h < 2; ++h) {
                                                const int ncol = n0 + 8 * j + 2 * t + h;
                                                if (ncol >= Nt) continue;
                                                if (ACC && P > 1) {
                                                        // C(m, n) of this part in scratch
                                                        const int m = swap ? ncol : mc, n = swap ? mc : ncol;
                                                        scratch[(int64_t) g0 * MN + m + n * M] = d[i][j][2 * r + h];
                                                        continue;
                                                }
                                                // C(m, n) with (m, n) = swap ? (ncol, mc) : (mc, ncol)
                                                OutT *cp = swap ? Cb + rs.c_off(ncol) + (int64_t) mc * cn
                                                                : Cb + rs.c_off(mc) + (int64_t) ncol * cn;
                                                store_out(cp, d[i][j][2 * r + h], sc, ACC);
                                        }
                        }
        }
        if (ACC && P > 1) {
                __syncthreads();
                const float r_m = 1.0f / M;
                for (int e = threadIdx.x; e < MN; e += NW * 32) {
                        int m;
                        const int n = fast_divmod(e, M, r_m, m);
                        float sum = 0.f;
                        for (int p = 0; p < P; ++p) sum += scratch[(int64_t) p * MN + e];
                        store_out(out + rs.c_off(m) + (int64_t) n * cn, sum, 1.f, true);
                }
        }
}

template <bool ACC, int NW, class E, class OutT>
__device__ __forceinline__ void grouped_stage_split(int ax, const int *w, int rows, int ldop, int G,
                                                    const int64_t *opoff, const E *__restrict__ ops,
                                                    const E *in, int in_gs, OutT *out, int out_gs,
                                                    const float *scale, E *scratch, int scratch_cap,
                                                    const int *in_idx)
{
        // the scratch holds FP32 partial tiles (two per float2 slot, one per
        // BF16 pair)
        float *fs = reinterpret_cast<float *>(scratch);
        const int fcap = scratch_cap * (int) (sizeof(E) / sizeof(float));
        const int M = ax == 0 ? rows : ax == 1 ? w[0] * w[2] : w[0] * w[1];
        const int N = ax == 0 ? w[1] * w[2] : rows;
        // padded work of the two orientations (16 x 8 granules)
        const int64_t pw0 = (int64_t) ((M + 15) / 16) * ((N + 7) / 8);
        const int64_t pw1 = (int64_t) ((N + 15) / 16) * ((M + 7) / 8);
        const bool swap = pw1 < pw0;
        const int Mt = swap ? N : M, Nt = swap ? M : N;
        if (Mt <= 16)
                grouped_stage_x_t<ACC, 1, 4, NW>(ax, w, rows, ldop, G, opoff, ops, in, in_gs, out,
                                                 out_gs, scale, swap, fs, fcap, in_idx);
        else if (Nt <= 8)
                grouped_stage_x_t<ACC, 2, 1, NW>(ax, w, rows, ldop, G, opoff, ops, in, in_gs, out,
                                                 out_gs, scale, swap, fs, fcap, in_idx);
        else
                grouped_stage_x_t<ACC, 2, 2, NW>(ax, w, rows, ldop, G, opoff, ops, in, in_gs, out,
                                                 out_gs, scale, swap, fs, fcap, in_idx);
}

// the split-precision stages for the two operand encodings
template <bool ACC, int NW, class OutT>
__device__ __forceinline__ void grouped_stage(int ax, const int *w, int rows, int ldop, int G,
                                              const int64_t *opoff, const float2 *__restrict__ ops,
                                              const float2 *in, int in_gs, OutT *out, int out_gs,
                                              const float *scale, float2 *scratch = nullptr,
                                              int scratch_cap = 0, const int *in_idx = nullptr)
{
        grouped_stage_split<ACC, NW>(ax, w, rows, ldop, G, opoff, ops, in, in_gs, out, out_gs, scale,
                                     scratch, scratch_cap, in_idx);
}

template <bool ACC, int NW, class OutT>
__device__ __forceinline__ void grouped_stage(int ax, const int *w, int rows, int ldop, int G,
                                              const int64_t *opoff, const BfPair *__restrict__ ops,
                                              const BfPair *in, int in_gs, OutT *out, int out_gs,
                                              const float *scale, BfPair *scratch = nullptr,
                                              int scratch_cap = 0, const int *in_idx = nullptr)
{
        grouped_stage_split<ACC, NW>(ax, w, rows, ldop, G, opoff, ops, in, in_gs, out, out_gs, scale,
                                     scratch, scratch_cap, in_idx);
}

// Element types of the kernel: operand storage T, the output tile's
// accumulator and the term prefactors.
template <class T>
struct Elem;
template <>
struct Elem<double> {
        using Acc = double;
        using Scale = double;
};
template <>
struct Elem<float2> {
        using Acc = float;
        using Scale = float;
};
template <>
struct Elem<BfPair> {
        using Acc = float;
        using Scale = float;
};

// Shared buffer capacities (elements) of a configuration for element type T:
// the output tile is the plan's; the staged block and intermediates take the
// configuration's bytes (a float2 pair is as wide as a double, a BF16 pair
// half as wide, so twice as many fit).
template <class Cfg, class T>
struct Caps {
        static constexpr int kOut = Cfg::kOut;
        static constexpr int kPsi = Cfg::kPsi * (int) (sizeof(double) / sizeof(T));
        static constexpr int kW = Cfg::kW * (int) (sizeof(double) / sizeof(T));
        static_assert(sizeof(double) % sizeof(T) == 0, "operands are 8 or 4 bytes wide");
};

template <class Cfg, class T>
constexpr size_t smem_bytes_t()
{
        return sizeof(typename Elem<T>::Acc) * Caps<Cfg, T>::kOut +
               sizeof(T) * (Caps<Cfg, T>::kPsi + Caps<Cfg, T>::kW) +
               sizeof(typename Elem<T>::Scale) * kGMax + sizeof(int64_t) * 4 * kGMax +
               sizeof(int) * kGMax + 64;
}

template <class Cfg, class T>
__global__ void __launch_bounds__(Cfg::kThreads, Cfg::kMinBlocks)
heff_kernel(const T *__restrict__ x, double *__restrict__ y,
                 const T *__restrict__ ops, const int64_t *__restrict__ blk_off,
                 const int4 *__restrict__ edims, const HeffUnit *__restrict__ units, int n_units,
                 const int *__restrict__ pair_ptr, const HeffPair *__restrict__ pairs,
                 const HeffTask *__restrict__ tasks, int *counter, int *err)
{
        extern __shared__ __align__(16) unsigned char smem_raw[];
        using C = Caps<Cfg, T>;
        using Acc = typename Elem<T>::Acc;
        using Scale = typename Elem<T>::Scale;
        Acc *OUT = reinterpret_cast<Acc *>(smem_raw);
        constexpr int kThreads = Cfg::kThreads, NW = Cfg::kThreads / 32;
        T *PSI = reinterpret_cast<T *>(OUT + C::kOut);
        T *W = PSI + C::kPsi;
        Scale *PREF = reinterpret_cast<Scale *>(W + C::kW);
        int64_t *OPOFF = reinterpret_cast<int64_t *>(PREF + kGMax);   // [3][kGMax]
        int64_t *UOFF = OPOFF + 3 * kGMax;     // distinct first-stage operators of a group
        int *AIDX = reinterpret_cast<int *>(UOFF + kGMax);   // term -> its first-stage result
        int *UNIT = AIDX + kGMax;              // [0] unit, [1] group size, [2] distinct count
        const int tid = threadIdx.x;

        for (;;) {
                if (tid == 0) *UNIT = atomicAdd(counter, 1);
                __syncthreads();
                const int u = *UNIT;
                __syncthreads();
                if (u >= n_units) break;
                const HeffUnit un = units[u];
                const int nb = un.nb;
                const int4 en = edims[nb];
                const int dn[3] = {en.x, en.y, en.z};
                // extent and first row of the tile along each axis
                const int ext[3] = {un.at, un.bt, un.ct};
                const int row0[3] = {un.a0, un.b0, un.c0};
                const int st = ext[0] * ext[1] * ext[2];
                for (int e = tid; e < st; e += kThreads) OUT[e] = Acc(0);
                __syncthreads();
                for (int p = un.p0; p < un.p1; ++p) {
                        const HeffPair pr = pairs[p];
                        const int4 eo = edims[pr.old];
                        const int nst = (pr.axes >> 6) & 3;
                        int ax[3];
                        for (int s = 0; s < 3; ++s) ax[s] = (pr.axes >> (2 * s)) & 3;
                        const int w0[3] = {eo.x, eo.y, eo.z};
                        int w1[3] = {w0[0], w0[1], w0[2]};
                        w1[ax[0]] = ext[ax[0]];
                        int w2[3] = {w1[0], w1[1], w1[2]};
                        w2[ax[1]] = ext[ax[1]];
                        const int s0 = w0[0] * w0[1] * w0[2];
                        const int s1 = w1[0] * w1[1] * w1[2];
                        const int s2 = nst == 3 ? w2[0] * w2[1] * w2[2] : 0;
                        if (s1 + s2 > C::kW) {
                                if (tid == 0) atomicExch(err, 3);
                                return;
                        }
                        const T *xin = x + blk_off[pr.old];
                        const T *in0 = xin;
                        if (s0 <= C::kPsi) {
                                for (int e = tid; e < s0; e += kThreads) PSI[e] = xin[e];
                                in0 = PSI;
                        }
                        const int G = min(kGMax, C::kW / (s1 + s2));
                        T *W1 = W;
                        const int nterm = pr.t1 - pr.t0;
                        for (int t0 = 0, g = 0; t0 < nterm; t0 += g) {
                                const int cand = min(nst == 3 ? kGMax : G, nterm - t0);
                                if (tid < cand) {
                                        const HeffTask &tk = tasks[pr.t0 + t0 + tid];
                                        for (int s = 0; s < 3; ++s)
                                                OPOFF[s * kGMax + tid] = tk.op_off[ax[s]] + row0[ax[s]];
                                        PREF[tid] = (Scale) tk.pref;
                                }
                                // Terms that apply the same first-stage operator share its
                                // result (the host sorts a pair's terms so they sit next to
                                // each other): while the first warps stage the group's
                                // offsets, warp 2 reads the candidates' first-stage
                                // operators itself, numbers their runs and takes the longest
                                // prefix of the candidates whose n1 first-stage results and
                                // g second-stage results fit the intermediate buffer, so one
                                // barrier serves both.
                                if (nst == 3 && (tid >> 5) == 2) {
                                        const int lane = tid & 31;
                                        int base = 0, gsel = 0, n1 = 0;
                                        int64_t carry = -1;
                                        for (int h = 0; h < kGMax / 32; ++h) {
                                                const int t = lane + 32 * h;
                                                const bool in = t < cand;
                                                const int64_t cur =
                                                        in ? tasks[pr.t0 + t0 + t].op_off[ax[0]] + row0[ax[0]] : -2;
                                                int64_t prev = __shfl_up_sync(0xffffffffu, cur, 1);
                                                if (lane == 0) prev = carry;
                                                carry = __shfl_sync(0xffffffffu, cur, 31);
                                                const bool first = in && (t == 0 || cur != prev);
                                                const unsigned fb = __ballot_sync(0xffffffffu, first);
                                                const int incl = base + __popc(fb & (0xffffffffu >> (31 - lane)));
                                                const bool fits = in && (int64_t) incl * s1 +
                                                                        (int64_t) (t + 1) * s2 <= C::kW;
                                                const unsigned ok = __ballot_sync(0xffffffffu, fits);
                                                if (in) AIDX[t] = incl - 1;
                                                if (first) UOFF[incl - 1] = cur;
                                                if (ok) {
                                                        const int last = 31 - __clz(ok);
                                                        gsel = 32 * h + last + 1;
                                                        n1 = __shfl_sync(0xffffffffu, incl, last);
                                                }
                                                base += __popc(fb);
                                        }
                                        if (lane == 0) {
                                                UNIT[1] = gsel;
                                                UNIT[2] = n1;
                                        }
                                }
                                __syncthreads();
                                if (nst == 3) {
                                        g = UNIT[1];
                                        const int n1 = UNIT[2];
                                        T *V2 = W + n1 * s1;
                                        // the first stage reads the staged block (shared memory) or
                                        // the block in global memory: one call site for each, so
                                        // each is compiled for its own address space
                                        if (in0 == PSI)
                                                grouped_stage<false, NW>(ax[0], w0, ext[ax[0]], dn[ax[0]], n1,
                                                                     UOFF, ops, PSI, 0, W1, s1, nullptr);
                                        else
                                                grouped_stage<false, NW>(ax[0], w0, ext[ax[0]], dn[ax[0]], n1,
                                                                     UOFF, ops, xin, 0, W1, s1, nullptr);
                                        __syncthreads();
                                        grouped_stage<false, NW>(ax[1], w1, ext[ax[1]], dn[ax[1]], g,
                                                             OPOFF + kGMax, ops, W1, s1, V2, s2, PREF,
                                                             nullptr, 0, AIDX);
                                        __syncthreads();
                                        // stage 3 reads V2 only: the larger free region (the
                                        // first-stage results or the tail) is its scratch
                                        const int used = n1 * s1 + g * s2;
                                        if (n1 * s1 >= C::kW - used)
                                                grouped_stage<true, NW>(ax[2], w2, ext[ax[2]], dn[ax[2]], g,
                                                                    OPOFF + 2 * kGMax, ops, V2, s2, OUT, 0,
                                                                    nullptr, W1, n1 * s1);
                                        else
                                                grouped_stage<true, NW>(ax[2], w2, ext[ax[2]], dn[ax[2]], g,
                                                                    OPOFF + 2 * kGMax, ops, V2, s2, OUT, 0,
                                                                    nullptr, W + used, C::kW - used);
                                } else {
                                        g = cand;
                                        if (in0 == PSI)
                                                grouped_stage<false, NW>(ax[0], w0, ext[ax[0]], dn[ax[0]], g,
                                                                     OPOFF, ops, PSI, 0, W1, s1, PREF);
                                        else
                                                grouped_stage<false, NW>(ax[0], w0, ext[ax[0]], dn[ax[0]], g,
                                                                     OPOFF, ops, xin, 0, W1, s1, PREF);
                                        __syncthreads();
                                        grouped_stage<true, NW>(ax[1], w1, ext[ax[1]], dn[ax[1]], g,
                                                            OPOFF + kGMax, ops, W1, s1, OUT, 0,
                                                            nullptr, W1 + G * s1, C::kW - G * s1);
                                }
                                __syncthreads();
                        }
                }
                // write the tile back
                double *yn = y + blk_off[nb];
                for (int e = tid; e < st; e += kThreads) {
                        const int a = e % ext[0];
                        const int t = e / ext[0];
                        const int b = t % ext[1];
                        const int c = t / ext[1];
                        double *dst = yn + (row0[0] + a) +
                                      (int64_t) dn[0] * ((row0[1] + b) + (int64_t) dn[1] * (row0[2] + c));
                        if (un.split) atomicAdd(dst, (double) OUT[e]);
                        else *dst = (double) OUT[e];
                }
                __syncthreads();
        }
}

template <class Cfg>
constexpr size_t smem_bytes_v2()
{
        return sizeof(double) * (Cfg::kOut + Cfg::kPsi + Cfg::kW + kGMax) +
               sizeof(int64_t) * 3 * kGMax + 3 * sizeof(v2::Geo) + 64;
}

// The matvec with contraction-ordered layouts (heff_v2.cuh): persistent CTAs
// take units off the counter as heff_kernel does; per pair the old block is
// staged permuted for the pair's sequence, and the stages run on the
// transposed operators ops_t (offsets toff per task and memory axis).  SPLIT:
// 3xTF32 products of {hi, lo} pairs (ops_t holds pairs, the staged block and
// the intermediates too), FP64 output tile.
template <class Cfg, bool SPLIT>
__global__ void __launch_bounds__(Cfg::kThreads, Cfg::kMinBlocks)
heff_v2_kernel(const double *__restrict__ x, double *__restrict__ y,
               const typename std::conditional<SPLIT, float2, double>::type *__restrict__ ops_t,
               const int64_t *__restrict__ blk_off, const int4 *__restrict__ edims,
               const HeffUnit *__restrict__ units, int n_units, const HeffPair *__restrict__ pairs,
               const HeffTask *__restrict__ tasks, const int64_t *__restrict__ toff, int *counter,
               int *err)
{
        using E = typename std::conditional<SPLIT, float2, double>::type;
        extern __shared__ __align__(16) unsigned char smem_raw[];
        constexpr int kThreads = Cfg::kThreads, NW = Cfg::kThreads / 32;
        double *OUT = reinterpret_cast<double *>(smem_raw);
        E *PSI = reinterpret_cast<E *>(OUT + Cfg::kOut);
        E *W = PSI + Cfg::kPsi;
        double *PREF = reinterpret_cast<double *>(W + Cfg::kW);
        int64_t *OPOFF = reinterpret_cast<int64_t *>(PREF + kGMax);   // [3][kGMax]
        v2::Geo *GEO = reinterpret_cast<v2::Geo *>(OPOFF + 3 * kGMax);   // [3]
        int *UNIT = reinterpret_cast<int *>(GEO + 3);
        const int tid = threadIdx.x;

        for (;;) {
                if (tid == 0) *UNIT = atomicAdd(counter, 1);
                __syncthreads();
                const int u = *UNIT;
                __syncthreads();
                if (u >= n_units) break;
                const HeffUnit un = units[u];
                const int nb = un.nb;
                const int4 en = edims[nb];
                const int dn[3] = {en.x, en.y, en.z};
                const int ext[3] = {un.at, un.bt, un.ct};
                const int row0[3] = {un.a0, un.b0, un.c0};
                const int st = ext[0] * ext[1] * ext[2];
                for (int e = tid; e < st; e += kThreads) OUT[e] = 0.0;
                __syncthreads();
                for (int p = un.p0; p < un.p1; ++p) {
                        const HeffPair pr = pairs[p];
                        const int4 eo = edims[pr.old];
                        const int o[3] = {eo.x, eo.y, eo.z};
                        const int nst = (pr.axes >> 6) & 3;
                        int seq[3];
                        seq[0] = pr.axes & 3;
                        seq[1] = (pr.axes >> 2) & 3;
                        seq[2] = nst == 3 ? (pr.axes >> 4) & 3 : 3 - seq[0] - seq[1];
                        const int psz = v2::staged_ld(o[seq[0]]) * o[seq[1]] * o[seq[2]];
                        const bool staged = psz <= Cfg::kPsi;
                        if (!staged && seq[0] != 0) {
                                // the plan starts every sequence of an unstaged block on axis 0
                                if (tid == 0) atomicExch(err, 4);
                                return;
                        }
                        if (tid == 0) {
                                const int ostr[3] = {1, ext[0], ext[0] * ext[1]};
                                v2::make_geos(GEO, nst, seq, o, ext, staged, ostr);
                        }
                        __syncthreads();
                        const int s1 = GEO[0].out_size, s2 = nst == 3 ? GEO[1].out_size : 0;
                        if (s1 + s2 > Cfg::kW) {
                                if (tid == 0) atomicExch(err, 3);
                                return;
                        }
                        const double *xin = x + blk_off[pr.old];
                        if (staged) {
                                // old block -> (s0 padded, s1, s2), padding zeroed
                                const int ld = v2::staged_ld(o[seq[0]]);
                                const int K = o[seq[0]], d1 = o[seq[1]];
                                const int str[3] = {1, o[0], o[0] * o[1]};
                                const int sk = str[seq[0]], s1s = str[seq[1]], s2s = str[seq[2]];
                                const float rld = 1.0f / ld, rd1 = 1.0f / d1;
                                for (int e = tid; e < psz; e += kThreads) {
                                        int k;
                                        const int col = v2::divmod(e, ld, rld, k);
                                        double v = 0.0;
                                        if (k < K) {
                                                int i1;
                                                const int i2 = v2::divmod(col, d1, rd1, i1);
                                                v = xin[k * sk + i1 * s1s + i2 * s2s];
                                        }
                                        if constexpr (SPLIT) PSI[e] = v2::split_pair(v);
                                        else PSI[e] = v;
                                }
                        }
                        const int G = min(kGMax, Cfg::kW / (s1 + s2));
                        E *W1 = W, *W2 = W + G * s1;
                        const int nterm = pr.t1 - pr.t0;
                        for (int t0 = 0; t0 < nterm; t0 += G) {
                                const int gg = min(G, nterm - t0);
                                if (tid < gg) {
                                        const int t = pr.t0 + t0 + tid;
                                        for (int j = 0; j < nst; ++j)
                                                OPOFF[j * kGMax + tid] = toff[3 * (int64_t) t + seq[j]] +
                                                                         (int64_t) row0[seq[j]] * GEO[j].lda;
                                        PREF[tid] = tasks[t].pref;
                                }
                                __syncthreads();
                                const double *sc0 = nst == 3 ? nullptr : PREF;
                                if constexpr (SPLIT) {
                                        float *scr3 = reinterpret_cast<float *>(W1);
                                        float *scr2 = reinterpret_cast<float *>(W1 + G * s1);
                                        if (staged)
                                                v2::stage_x<false, NW, false>(GEO[0], gg, OPOFF, ops_t, PSI, 0, W1,
                                                                              s1, sc0);
                                        else
                                                v2::stage_x<false, NW, true>(GEO[0], gg, OPOFF, ops_t, xin, 0, W1,
                                                                             s1, sc0);
                                        __syncthreads();
                                        if (nst == 3) {
                                                v2::stage_x<false, NW, false>(GEO[1], gg, OPOFF + kGMax, ops_t, W1,
                                                                              s1, W2, s2, PREF);
                                                __syncthreads();
                                                v2::stage_x<true, NW, false>(GEO[2], gg, OPOFF + 2 * kGMax, ops_t,
                                                                             W2, s2, OUT, 0, nullptr, scr3,
                                                                             2 * G * s1);
                                        } else {
                                                v2::stage_x<true, NW, false>(GEO[1], gg, OPOFF + kGMax, ops_t, W1,
                                                                             s1, OUT, 0, nullptr, scr2,
                                                                             2 * (Cfg::kW - G * s1));
                                        }
                                } else {
                                        // the first stage reads the staged block (shared memory) or
                                        // the block in place (global memory): one call site for each
                                        if (staged)
                                                v2::stage<false, NW, false>(GEO[0], gg, OPOFF, ops_t, PSI, 0, W1, s1,
                                                                            sc0);
                                        else
                                                v2::stage<false, NW, true>(GEO[0], gg, OPOFF, ops_t, xin, 0, W1, s1,
                                                                           sc0);
                                        __syncthreads();
                                        if (nst == 3) {
                                                v2::stage<false, NW, false>(GEO[1], gg, OPOFF + kGMax, ops_t, W1, s1,
                                                                            W2, s2, PREF);
                                                __syncthreads();
                                                // the last stage reads W2 only: W1's share is its scratch
                                                v2::stage<true, NW, false>(GEO[2], gg, OPOFF + 2 * kGMax, ops_t, W2,
                                                                           s2, OUT, 0, nullptr, W1, G * s1);
                                        } else {
                                                v2::stage<true, NW, false>(GEO[1], gg, OPOFF + kGMax, ops_t, W1, s1,
                                                                           OUT, 0, nullptr, W1 + G * s1,
                                                                           Cfg::kW - G * s1);
                                        }
                                }
                                __syncthreads();
                        }
                }
                double *yn = y + blk_off[nb];
                for (int e = tid; e < st; e += kThreads) {
                        const int a = e % ext[0];
                        const int t = e / ext[0];
                        const int b = t % ext[1];
                        const int c = t / ext[1];
                        double *dst = yn + (row0[0] + a) +
                                      (int64_t) dn[0] * ((row0[1] + b) + (int64_t) dn[1] * (row0[2] + c));
                        if (un.split) atomicAdd(dst, OUT[e]);
                        else *dst = OUT[e];
                }
                __syncthreads();
        }
}

// {hi, lo} pairs of the transposed operators (split-precision matvec of the
// contraction-ordered configurations).
__global__ void split_pairs_kernel(const double *__restrict__ a, float2 *__restrict__ b, int64_t n)
{
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x)
                b[i] = v2::split_pair(a[i]);
}

// Transposes the referenced operator blocks into the layout of the
// contraction-ordered kernel: job j = {src, dst, rows, cols} of a (rows x
// cols) column-major block at ops[src] -> row-major at opt[dst] with rows of
// v2::op_ld(cols) doubles (the padding zeroed).
__global__ void transpose_ops_kernel(const double *__restrict__ ops, double *__restrict__ opt,
                                     const int64_t *__restrict__ jobs, int64_t njobs, int64_t n_ops,
                                     int64_t n_opt, int *err)
{
        for (int64_t j = blockIdx.x; j < njobs; j += gridDim.x) {
                const int64_t src = jobs[4 * j], dst = jobs[4 * j + 1];
                const int rows = (int) jobs[4 * j + 2], cols = (int) jobs[4 * j + 3];
                const int ld = v2::op_ld(cols);
                const int n = rows * ld;
                // the host checks every job before the launch; a job out of
                // range is recorded and skipped here all the same
                if (rows < 0 || cols < 0 || src < 0 || src + (int64_t) rows * cols > n_ops || dst < 0 ||
                    dst + n > n_opt) {
                        if (threadIdx.x == 0) atomicExch(err, 5);
                        continue;
                }
                for (int e = threadIdx.x; e < n; e += blockDim.x) {
                        const int r = e / ld, k = e - r * ld;
                        opt[dst + e] = k < cols ? ops[src + r + (int64_t) k * rows] : 0.0;
                }
        }
}

int build_transposed_ops(const HostPlan &hp, DevicePlan &dp, const int64_t *d_jobs, cudaStream_t s)
{
        const int64_t njobs = (int64_t) hp.tjobs.size() / 4;
        if (njobs == 0) return T3NS_OK;
        for (int64_t j = 0; j < njobs; ++j) {
                const int64_t *jb = &hp.tjobs[4 * j];
                if (jb[2] < 0 || jb[3] < 0 || jb[0] < 0 || jb[0] + jb[2] * jb[3] > hp.op_elems ||
                    jb[1] < 0 || jb[1] + jb[2] * v2::op_ld((int) jb[3]) > hp.opt_elems)
                        return set_error(T3NS_E_ARG, "transposed operators: job " + std::to_string(j) +
                                                             " out of range");
        }
        const int grid = (int) std::min<int64_t>(njobs, 148 * 16);
        transpose_ops_kernel<<<grid, 256, 0, s>>>(dp.ops, dp.ops_t, d_jobs, njobs, hp.op_elems,
                                                  hp.opt_elems, dp.err);
        T3NS_CUDA_TRY(cudaGetLastError());
        return T3NS_OK;
}

// Diagonal: diag[n](a,b,c) = sum over the terms of the (n, n) pair of
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

// FLOPs of contracting a pair in the order seq, summed over the tiles of
// the output block: ext is the tile extent and nt the number of tiles along
// each axis.  Each tile applies its own rows of every operator, so a stage
// costs 2 * (new rows) * (old dim) * (the other current dims); an axis not
// yet contracted is still at its old extent in every tile, so that stage is
// repeated for every tile along it.  s1, s2: per-tile sizes of the first
// two intermediates.
static double seq_cost(const int *seq, int nst, const int *o, const int *n, const int *ext,
                       const int *nt, int64_t *s1, int64_t *s2, double s1scale = 1.0)
{
        double fl = 0;
        bool done[3] = {false, false, false};
        int64_t wt[3] = {o[0], o[1], o[2]};
        for (int s = 0; s < nst; ++s) {
                const int a = seq[s];
                double f = 2.0 * n[a] * o[a];
                for (int j = 0; j < 3; ++j) {
                        if (j == a) continue;
                        f *= done[j] ? (double) n[j] : (double) o[j] * nt[j];
                }
                fl += s == 0 ? s1scale * f : f;
                done[a] = true;
                wt[a] = ext[a];
                if (s == 0) *s1 = wt[0] * wt[1] * wt[2];
                if (s == 1) *s2 = nst == 3 ? wt[0] * wt[1] * wt[2] : 0;
        }
        return fl;
}

// Tensor-pipe work of the same sequence: each stage as the kernel maps it
// to GEMMs (axis 0: M = rows, N = the other two dims; axis 1: M = dims 0
// and 2, N = rows; axis 2: M = dims 0 and 1, N = rows; K = the old dim),
// with M and N padded to the 8 of an mma.m8n8k4 tile and K to its 4, per
// tile (extent ext) times the number of tiles.  Thin tiles and small dims
// cost what they occupy on the pipe, not their FLOPs.
static double tile_cost(const int *seq, int nst, const int *o, const int *ext, const int *nt,
                        double s1scale = 1.0)
{
        auto p8 = [](int64_t x) { return (double) ((x + 7) / 8 * 8); };
        auto p4 = [](int64_t x) { return (double) ((x + 3) / 4 * 4); };
        int64_t cur[3] = {o[0], o[1], o[2]};
        double c = 0;
        for (int s = 0; s < nst; ++s) {
                const int a = seq[s];
                const int64_t rows = ext[a];
                double m, n;
                if (a == 0) {
                        m = p8(rows);
                        n = p8(cur[1] * cur[2]);
                } else if (a == 1) {
                        m = p8(cur[0] * cur[2]);
                        n = p8(rows);
                } else {
                        m = p8(cur[0] * cur[1]);
                        n = p8(rows);
                }
                c += (s == 0 ? s1scale : 1.0) * 2.0 * m * n * p4(cur[a]);
                cur[a] = rows;
        }
        return c * nt[0] * nt[1] * nt[2];
}

// Cheapest contraction sequence for a pair on a tiling (ext, nt) by
// tensor-pipe work, among those whose intermediates fit the shared buffer;
// fl_out receives its FLOPs and pc_out its tensor-pipe work.  Returns -1 if
// none fits.
// For the contraction-ordered kernel (v2) the intermediates take their padded
// sizes, and an old block larger than psi_cap (padded) is read in place,
// which needs a sequence that starts on memory axis 0.
// Terms sorted by their operator on memory axis dax share the first stage
// when the sequence starts there (three-operator steps, heff_kernel): that
// stage then costs dfrac of its per-term work.
static int choose_seq(int nst, const int *o, const int *n, const int *ext, const int *nt,
                      int w_cap, double *fl_out, double *pc_out, int seq_out[3], bool ordered = false,
                      int psi_cap = 0, int dax = -1, double dfrac = 1.0)
{
        static const int perms3[6][3] = {{0, 1, 2}, {0, 2, 1}, {1, 0, 2},
                                         {1, 2, 0}, {2, 0, 1}, {2, 1, 0}};
        static const int perms2[2][3] = {{0, 1, 2}, {1, 0, 2}};
        const int np = nst == 3 ? 6 : 2;
        int best = -1;
        double bfl = 0, bpc = 0;
        for (int q = 0; q < np; ++q) {
                const int *seq = nst == 3 ? perms3[q] : perms2[q];
                int64_t s1 = 0, s2 = 0;
                const double s1scale = (!ordered && nst == 3 && seq[0] == dax) ? dfrac : 1.0;
                const double fl = seq_cost(seq, nst, o, n, ext, nt, &s1, &s2, s1scale);
                if (ordered) {
                        const int s0 = seq[0], q1 = seq[1], q2 = nst == 3 ? seq[2] : 3 - seq[0] - seq[1];
                        const int64_t psz = (int64_t) v2::staged_ld(o[s0]) * o[q1] * o[q2];
                        if (psz > psi_cap && s0 != 0) continue;
                        s1 = (int64_t) v2::staged_ld(o[q1]) * o[q2] * ext[s0];
                        s2 = nst == 3 ? (int64_t) v2::staged_ld(o[q2]) * ext[s0] * ext[q1] : 0;
                }
                if (s1 + s2 > w_cap) continue;
                const double pc = tile_cost(seq, nst, o, ext, nt, s1scale);
                if (best < 0 || pc < bpc) { best = q; bfl = fl; bpc = pc; }
        }
        if (best < 0) return -1;
        const int *seq = nst == 3 ? perms3[best] : perms2[best];
        for (int s = 0; s < 3; ++s) seq_out[s] = seq[s];
        *fl_out = bfl;
        *pc_out = bpc;
        return 0;
}

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
                // the kernels address elements inside one block (and inside one
                // operator block, whose sizes are 32-bit in the descriptor) with
                // 32-bit offsets; only the offsets of blocks are 64-bit
                if ((int64_t) e[0] * e[1] * e[2] >= ((int64_t) 1 << 31))
                        return set_error(T3NS_E_LIMIT, "block " + std::to_string(b) +
                                                               " has 2^31 or more elements");
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

        // terms, grouped by pair, pairs by new block
        hp.task_ptr.assign(d->nblocks + 1, 0);
        hp.tasks.clear();
        for (auto &tp : hp.tiles) tp = TilePlan();
        double flops_ref = 0;
        int64_t npairs = 0;
        std::vector<std::vector<PairTmp>> blocks_pairs(d->nblocks);
        for (int nb = 0; nb < d->nblocks; ++nb) {
                hp.task_ptr[nb] = (int) hp.tasks.size();
                const int dn[3] = {d->dims[3 * nb], d->dims[3 * nb + 1],
                                   d->isdmrg ? 1 : d->dims[3 * nb + 2]};
                std::vector<PairTmp> ptmp;
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
                        {
                                double wd[3] = {(double) dold[0], (double) dold[1], (double) dold[2]};
                                for (int s = 0; s < nops; ++s) {
                                        fl += 2.0 * wd[0] * wd[1] * wd[2] * dn[o[s]];
                                        wd[o[s]] = dn[o[s]];
                                }
                        }
                        const int t0 = (int) hp.tasks.size();
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
                                        t.axes = nops << 6;
                                        hp.tasks.push_back(t);
                                        flops_ref += fl;
                                }
                        }
                        const int t1 = (int) hp.tasks.size();
                        if (t1 > t0) {
                                const int4 eo4 = hp.edims[ob];
                                int dax = -1;
                                double dfrac = 1.0;
                                if (nops == 3) {
                                        // the axis whose shared first stage gives the
                                        // cheapest untiled sequence (distinct operator
                                        // blocks / terms on it scale that stage); the
                                        // pair's terms sorted by it (stable)
                                        std::vector<int64_t> v(t1 - t0);
                                        const int eo[3] = {eo4.x, eo4.y, eo4.z};
                                        const int en3[3] = {dn[hp.map[0]], dn[hp.map[1]], dn[hp.map[2]]};
                                        const int nt1[3] = {1, 1, 1};
                                        double best = 0;
                                        for (int ax = 0; ax < 3; ++ax) {
                                                for (int t = t0; t < t1; ++t) v[t - t0] = hp.tasks[t].op_off[ax];
                                                std::sort(v.begin(), v.end());
                                                const double fr = (double) (std::unique(v.begin(), v.end()) -
                                                                            v.begin()) / (t1 - t0);
                                                double cost = 0;
                                                for (int q = 0; q < 6; ++q) {
                                                        const int *sq = kOrders3[q];
                                                        int64_t s1, s2;
                                                        const double c = seq_cost(sq, 3, eo, en3, en3, nt1, &s1, &s2,
                                                                                  sq[0] == ax ? fr : 1.0);
                                                        if (q == 0 || c < cost) cost = c;
                                                }
                                                if (dax < 0 || cost < best) {
                                                        dax = ax;
                                                        dfrac = fr;
                                                        best = cost;
                                                }
                                        }
                                        std::stable_sort(hp.tasks.begin() + t0, hp.tasks.begin() + t1,
                                                         [dax](const HeffTask &a, const HeffTask &b) {
                                                                 return a.op_off[dax] < b.op_off[dax];
                                                         });
                                }
                                ptmp.push_back({ob, t0, t1, {eo4.x, eo4.y, eo4.z}, dax, dfrac});
                        }
                }
                blocks_pairs[nb] = std::move(ptmp);
        }
        hp.task_ptr[d->nblocks] = (int) hp.tasks.size();
        if (hp.tasks.size() > (size_t) INT32_MAX)
                return set_error(T3NS_E_LIMIT, "more than 2^31 tasks");
        hp.blocks_pairs = std::move(blocks_pairs);
        hp.npairs = npairs;
        hp.flops_ref = flops_ref;

        // transposed operator buffer of the contraction-ordered kernel
        {
                hp.toff.assign(3 * hp.tasks.size(), 0);
                hp.tjobs.clear();
                std::unordered_map<int64_t, int64_t> tmap;
                tmap.reserve(1 << 16);
                int64_t tot = 0;
                for (int nb = 0; nb < d->nblocks; ++nb)
                        for (int t = hp.task_ptr[nb]; t < hp.task_ptr[nb + 1]; ++t) {
                                const HeffTask &tk = hp.tasks[t];
                                const int4 eo = hp.edims[tk.old], en = hp.edims[nb];
                                const int o3[3] = {eo.x, eo.y, eo.z}, n3[3] = {en.x, en.y, en.z};
                                for (int ax = 0; ax < nops; ++ax) {
                                        auto it = tmap.find(tk.op_off[ax]);
                                        int64_t off;
                                        if (it == tmap.end()) {
                                                off = tot;
                                                tot += ((int64_t) n3[ax] * v2::op_ld(o3[ax]) + 3) & ~(int64_t) 3;
                                                tmap.emplace(tk.op_off[ax], off);
                                                hp.tjobs.insert(hp.tjobs.end(),
                                                                {tk.op_off[ax], off, (int64_t) n3[ax], (int64_t) o3[ax]});
                                        } else {
                                                off = it->second;
                                        }
                                        hp.toff[3 * (size_t) t + ax] = off;
                                }
                        }
                hp.opt_elems = tot;
        }

        // algorithmic bytes: vectors in/out + each referenced operator block once
        {
                std::vector<std::pair<int64_t, int64_t>> blocks;
                blocks.reserve(hp.tasks.size() * nops);
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
                double opbytes = 0;
                for (auto &b : blocks) opbytes += 8.0 * b.second;
                hp.bytes_alg = 16.0 * hp.size + opbytes;
        }
        return tile_plan(hp, 0);
}


int tile_plan(HostPlan &hp, int cfg)
{
        if (cfg < 0 || cfg >= kNumCfgs) return set_error(T3NS_E_ARG, "unknown kernel configuration");
        TilePlan &tp = hp.tiles[cfg];
        if (tp.built) return T3NS_OK;
        const KernelCfg &kc = kCfgs[cfg];
        const int nops = hp.isdmrg ? 2 : 3;
        tp.pair_ptr.assign(hp.nblocks + 1, 0);
        tp.pairs.clear();
        tp.units.clear();
        double flops_exec = 0;
        std::vector<double> unit_work;
        // a unit should not carry more than a small share of the work, so the
        // heaviest-first schedule ends evenly across the CTAs
        const double unit_cap = std::max(hp.flops_ref / (148.0 * kc.ctas_per_sm * 8), 1e6);
        for (int nb = 0; nb < hp.nblocks; ++nb) {
                tp.pair_ptr[nb] = (int) tp.pairs.size();
                auto &ptmp = hp.blocks_pairs[nb];
                if (ptmp.empty()) continue;
                const int4 en4 = hp.edims[nb];
                const int en[3] = {en4.x, en4.y, en4.z};

                // tiling of the output block and a sequence per pair that fits:
                // candidates tile one or two memory axes (halving sizes); the
                // cheapest one whose units stay under the work cap is taken
                struct Cand { int at, bt, ct; };
                std::vector<Cand> cand;
                const int64_t sn = (int64_t) en[0] * en[1] * en[2];
                if (sn <= kc.out_cap) cand.push_back({en[0], en[1], en[2]});
                for (int ax = 0; ax < 3; ++ax) {
                        const int64_t rest = sn / std::max(en[ax], 1);
                        if (rest == 0 || rest > kc.out_cap) continue;
                        for (int t = (int) std::min<int64_t>(en[ax], kc.out_cap / rest); t >= 1; t /= 2) {
                                if (t == en[ax]) continue;
                                Cand c{en[0], en[1], en[2]};
                                (ax == 0 ? c.at : ax == 1 ? c.bt : c.ct) = t;
                                cand.push_back(c);
                        }
                }
                for (int pair = 0; pair < 3; ++pair) {
                        // tile axis p1 with t, axis p2 with 1
                        const int p1 = pair == 2 ? 0 : pair + 1, p2 = pair == 2 ? 1 : (pair == 0 ? 2 : 0);
                        const int other = 3 - p1 - p2;
                        if (en[other] > kc.out_cap || en[p2] <= 1) continue;
                        for (int t = std::min(en[p1], kc.out_cap / std::max(en[other], 1)); t >= 1; t /= 2) {
                                Cand c{en[0], en[1], en[2]};
                                (p1 == 0 ? c.at : p1 == 1 ? c.bt : c.ct) = t;
                                (p2 == 0 ? c.at : p2 == 1 ? c.bt : c.ct) = 1;
                                cand.push_back(c);
                        }
                }
                int best_ci = -1;
                double best_fl = 0, best_cost = 0;
                std::vector<int> best_seqs;
                for (size_t ci = 0; ci < cand.size(); ++ci) {
                        const Cand &cd = cand[ci];
                        const int ext[3] = {cd.at, cd.bt, cd.ct};
                        const int nt[3] = {(en[0] + cd.at - 1) / cd.at, (en[1] + cd.bt - 1) / cd.bt,
                                           (en[2] + cd.ct - 1) / cd.ct};
                        std::vector<int> seqs(ptmp.size());
                        double fl_blk = 0, pc_blk = 0;
                        bool ok = true;
                        for (size_t q = 0; q < ptmp.size() && ok; ++q) {
                                int seq[3];
                                double fl, pc;
                                if (choose_seq(nops, ptmp[q].eo, en, ext, nt, kc.w_cap, &fl, &pc, seq,
                                               kc.v2 != 0, kc.psi_cap, ptmp[q].dax, ptmp[q].dfrac) != 0) {
                                        ok = false;
                                        break;
                                }
                                int axes = nops << 6;
                                for (int st = 0; st < nops; ++st) axes |= seq[st] << (2 * st);
                                seqs[q] = axes;
                                fl_blk += fl * (ptmp[q].t1 - ptmp[q].t0);
                                pc_blk += pc * (ptmp[q].t1 - ptmp[q].t0);
                        }
                        if (!ok) continue;
                        // cost: tensor-pipe work plus a fixed charge per (unit,
                        // pair) visit (staging the old block, group barriers),
                        // which keeps tiles from shrinking for a marginal saving
                        const double nunits = std::ceil((double) en[0] / cd.at) *
                                              std::ceil((double) en[1] / cd.bt) *
                                              std::ceil((double) en[2] / cd.ct);
                        const double cost = pc_blk + kPairVisitCost * nunits * ptmp.size();
                        if (best_ci < 0 || cost < best_cost) {
                                best_ci = (int) ci;
                                best_fl = fl_blk;
                                best_cost = cost;
                                best_seqs = seqs;
                        }
                }
                const bool placed = best_ci >= 0;
                if (placed) {
                        const Cand cd = cand[best_ci];
                        const int ext[3] = {cd.at, cd.bt, cd.ct};
                        const int nt[3] = {(en[0] + cd.at - 1) / cd.at, (en[1] + cd.bt - 1) / cd.bt,
                                           (en[2] + cd.ct - 1) / cd.ct};
                        const int pbase = (int) tp.pairs.size();
                        std::vector<double> pfl(ptmp.size());
                        for (size_t q = 0; q < ptmp.size(); ++q) {
                                tp.pairs.push_back({ptmp[q].ob, best_seqs[q], ptmp[q].t0, ptmp[q].t1});
                                int seq[3];
                                for (int st = 0; st < 3; ++st) seq[st] = (best_seqs[q] >> (2 * st)) & 3;
                                int64_t s1, s2;
                                const double s1scale = (!kc.v2 && nops == 3 && seq[0] == ptmp[q].dax)
                                                               ? ptmp[q].dfrac : 1.0;
                                pfl[q] = seq_cost(seq, nops, ptmp[q].eo, en, ext, nt, &s1, &s2, s1scale) *
                                         (ptmp[q].t1 - ptmp[q].t0);
                        }
                        flops_exec += best_fl;
                        const int nat = (en[0] + cd.at - 1) / cd.at;
                        const int nbt = (en[1] + cd.bt - 1) / cd.bt, nct = (en[2] + cd.ct - 1) / cd.ct;
                        for (int ia = 0; ia < nat; ++ia)
                                for (int ib = 0; ib < nbt; ++ib)
                                        for (int ic = 0; ic < nct; ++ic) {
                                                HeffUnit u{};
                                                u.nb = nb;
                                                u.a0 = ia * cd.at;
                                                u.at = std::min(cd.at, en[0] - u.a0);
                                                u.b0 = ib * cd.bt;
                                                u.bt = std::min(cd.bt, en[1] - u.b0);
                                                u.c0 = ic * cd.ct;
                                                u.ct = std::min(cd.ct, en[2] - u.c0);
                                                const double frac = ((double) u.at * u.bt * u.ct) / (double) sn;
                                                // split the tile's pairs into chunks under the cap
                                                const double tile_work = best_fl * frac;
                                                const bool split = tile_work + kPairVisitCost * ptmp.size() > unit_cap &&
                                                                   ptmp.size() > 1;
                                                size_t q = 0;
                                                while (q < ptmp.size()) {
                                                        double w = 0;
                                                        size_t q1 = q;
                                                        while (q1 < ptmp.size() &&
                                                               (q1 == q || !split ||
                                                                w + pfl[q1] * frac + kPairVisitCost <= unit_cap)) {
                                                                w += pfl[q1] * frac + kPairVisitCost;
                                                                ++q1;
                                                        }
                                                        HeffUnit v = u;
                                                        v.p0 = pbase + (int) q;
                                                        v.p1 = pbase + (int) q1;
                                                        v.split = split ? 1 : 0;
                                                        tp.units.push_back(v);
                                                        unit_work.push_back(w + 1e4 * (q1 - q));
                                                        q = q1;
                                                }
                                        }
                }
                if (!placed)
                        return set_error(T3NS_E_LIMIT, "no tiling of output block " + std::to_string(nb) +
                                                               " fits the shared-memory buffers");
        }
        tp.pair_ptr[hp.nblocks] = (int) tp.pairs.size();
        tp.flops_exec = flops_exec;

        // Blocks in order of their total work, heaviest first, and the tiles
        // of one block next to each other (heaviest first): CTAs that start
        // together then read the same operator rows while they sit in L2.
        std::vector<int> idx(tp.units.size());
        std::iota(idx.begin(), idx.end(), 0);
        std::vector<double> block_work(hp.nblocks, 0.0);
        for (size_t u = 0; u < tp.units.size(); ++u) block_work[tp.units[u].nb] += unit_work[u];
        std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) {
                const int na = tp.units[a].nb, nb = tp.units[b].nb;
                if (na != nb)
                        return block_work[na] != block_work[nb] ? block_work[na] > block_work[nb]
                                                                : na < nb;
                return unit_work[a] > unit_work[b];
        });
        std::vector<HeffUnit> sorted(tp.units.size());
        for (size_t i = 0; i < idx.size(); ++i) sorted[i] = tp.units[idx[i]];
        tp.units.swap(sorted);

        tp.built = true;
        return T3NS_OK;
}

template <class Cfg, bool SPLIT>
static int launch_v2(const DevicePlan &dp, const DeviceTiles &dt, const double *x, double *y,
                     cudaStream_t s)
{
        static std::mutex mu;
        static std::bitset<kMaxDevices> attr_set;
        int dev = 0;
        T3NS_CUDA_TRY(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kMaxDevices) return set_error(T3NS_E_LIMIT, "device ordinal too large");
        {
                std::lock_guard<std::mutex> lk(mu);
                if (!attr_set[dev]) {
                        T3NS_CUDA_TRY(cudaFuncSetAttribute(heff_v2_kernel<Cfg, SPLIT>,
                                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                           (int) smem_bytes_v2<Cfg>()));
                        attr_set[dev] = true;
                }
        }
        const int share = dp.share ? std::max(1, dp.share->load(std::memory_order_relaxed)) : 1;
        const int grid = std::max(1, dt.grid / share);
        if constexpr (SPLIT) {
                if (!dp.ops_t_split || !dp.toff)
                        return set_error(T3NS_E_ARG, "matvec: the split transposed operators are not set up");
                heff_v2_kernel<Cfg, true><<<grid, Cfg::kThreads, smem_bytes_v2<Cfg>(), s>>>(
                        x, y, dp.ops_t_split, dp.blk_off, dp.edims, dt.units, dt.n_units, dt.pairs,
                        dp.tasks, dp.toff, dp.counter, dp.err);
        } else {
                if (!dp.ops_t || !dp.toff)
                        return set_error(T3NS_E_ARG, "matvec: the transposed operators are not set up");
                heff_v2_kernel<Cfg, false><<<grid, Cfg::kThreads, smem_bytes_v2<Cfg>(), s>>>(
                        x, y, dp.ops_t, dp.blk_off, dp.edims, dt.units, dt.n_units, dt.pairs, dp.tasks,
                        dp.toff, dp.counter, dp.err);
        }
        T3NS_CUDA_TRY(cudaGetLastError());
        return T3NS_OK;
}

int convert_to_pairs(const double *a, float2 *b, int64_t n, cudaStream_t s)
{
        if (n <= 0) return T3NS_OK;
        const int grid = (int) std::min<int64_t>((n + 255) / 256, 148 * 16);
        split_pairs_kernel<<<grid, 256, 0, s>>>(a, b, n);
        T3NS_CUDA_TRY(cudaGetLastError());
        return T3NS_OK;
}

template <class Cfg, class T>
static int launch_cfg(const DevicePlan &dp, const DeviceTiles &dt, const T *x, const T *ops,
                      double *y, cudaStream_t s)
{
        // the shared-memory opt-in is a per-device attribute of the kernel:
        // set once per device (per instantiation), under a lock
        static std::mutex mu;
        static std::bitset<kMaxDevices> attr_set;
        int dev = 0;
        T3NS_CUDA_TRY(cudaGetDevice(&dev));
        if (dev < 0 || dev >= kMaxDevices) return set_error(T3NS_E_LIMIT, "device ordinal too large");
        {
                std::lock_guard<std::mutex> lk(mu);
                if (!attr_set[dev]) {
                        T3NS_CUDA_TRY(cudaFuncSetAttribute(heff_kernel<Cfg, T>,
                                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                           (int) smem_bytes_t<Cfg, T>()));
                        attr_set[dev] = true;
                }
        }
        const int share = dp.share ? std::max(1, dp.share->load(std::memory_order_relaxed)) : 1;
        const int grid = std::max(1, dt.grid / share);
        heff_kernel<Cfg, T><<<grid, Cfg::kThreads, smem_bytes_t<Cfg, T>(), s>>>(
                x, y, ops, dp.blk_off, dp.edims, dt.units, dt.n_units, dt.pair_ptr, dt.pairs,
                dp.tasks, dp.counter, dp.err);
        T3NS_CUDA_TRY(cudaGetLastError());
        return T3NS_OK;
}

// b[i] = {hi, lo}: hi = tf32(a[i]), lo = tf32(a[i] - hi), the remainder
// taken in FP64 so lo carries the bits FP32 would round away.
__global__ void split_tf32_kernel(const double *__restrict__ a, float2 *__restrict__ b, int64_t n)
{
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x) {
                const double v = a[i];
                const float hi = __uint_as_float(to_tf32((float) v));
                const float lo = __uint_as_float(to_tf32((float) (v - (double) hi)));
                b[i] = make_float2(hi, lo);
        }
}

// b[i] = {hi, lo}: hi = bf16(a[i]), lo = bf16(a[i] - hi), the remainder
// taken in FP64.
__global__ void split_bf16_kernel(const double *__restrict__ a, BfPair *__restrict__ b, int64_t n)
{
        for (int64_t i = blockIdx.x * (int64_t) blockDim.x + threadIdx.x; i < n;
             i += (int64_t) gridDim.x * blockDim.x) {
                const double v = a[i];
                const uint32_t hi = (uint32_t) __bfloat16_as_ushort(__double2bfloat16(v));
                const uint32_t lo = (uint32_t) __bfloat16_as_ushort(
                        __double2bfloat16(v - (double) bf16_value(hi)));
                b[i] = BfPair{hi | (lo << 16)};
        }
}

// The k-paired BF16 operator copy: job {src, -, rows, cols} (the plan's list
// of referenced operator blocks) writes block (rows x cols, column-major at
// src) at 2*src as (k/2)*2*rows + 2*r + (k%2), an odd cols padded with a
// zero column (the block's doubled slot has room: cols+1 <= 2*cols).
__global__ void pair_bf16_ops_kernel(const double *__restrict__ ops, BfPair *__restrict__ out,
                                     const int64_t *__restrict__ jobs, int64_t njobs, int64_t n_ops,
                                     int *err)
{
        for (int64_t j = blockIdx.x; j < njobs; j += gridDim.x) {
                const int64_t src = jobs[4 * j];
                const int rows = (int) jobs[4 * j + 2], cols = (int) jobs[4 * j + 3];
                const int kp = (cols + 1) & ~1;
                if (rows < 0 || cols < 0 || src < 0 || src + (int64_t) rows * cols > n_ops) {
                        if (threadIdx.x == 0) atomicExch(err, 6);
                        continue;
                }
                const int n = rows * kp;
                for (int p = threadIdx.x; p < n; p += blockDim.x) {
                        const int pi = p / (2 * rows), rem = p - pi * 2 * rows;
                        const int r = rem >> 1, k = 2 * pi + (rem & 1);
                        const double v = k < cols ? ops[src + r + (int64_t) k * rows] : 0.0;
                        const uint32_t hi = (uint32_t) __bfloat16_as_ushort(__double2bfloat16(v));
                        const uint32_t lo = (uint32_t) __bfloat16_as_ushort(
                                __double2bfloat16(v - (double) bf16_value(hi)));
                        out[2 * src + p] = BfPair{hi | (lo << 16)};
                }
        }
}

int build_paired_bf16_ops(const HostPlan &hp, DevicePlan &dp, const int64_t *d_jobs, cudaStream_t s)
{
        const int64_t njobs = (int64_t) hp.tjobs.size() / 4;
        if (njobs == 0) return T3NS_OK;
        for (int64_t j = 0; j < njobs; ++j) {
                const int64_t *jb = &hp.tjobs[4 * j];
                if (jb[2] < 0 || jb[3] < 0 || jb[0] < 0 || jb[0] + jb[2] * jb[3] > hp.op_elems)
                        return set_error(T3NS_E_ARG, "paired operators: job " + std::to_string(j) +
                                                             " out of range");
        }
        const int grid = (int) std::min<int64_t>(njobs, 148 * 16);
        pair_bf16_ops_kernel<<<grid, 256, 0, s>>>(dp.ops, reinterpret_cast<BfPair *>(dp.ops_bf16),
                                                  d_jobs, njobs, hp.op_elems, dp.err);
        T3NS_CUDA_TRY(cudaGetLastError());
        return T3NS_OK;
}

int convert_to_bf16_pairs(const double *a, void *b, int64_t n, cudaStream_t s)
{
        if (n <= 0) return T3NS_OK;
        const int grid = (int) std::min<int64_t>((n + 255) / 256, 148 * 16);
        split_bf16_kernel<<<grid, 256, 0, s>>>(a, reinterpret_cast<BfPair *>(b), n);
        T3NS_CUDA_TRY(cudaGetLastError());
        return T3NS_OK;
}

int convert_to_split(const double *a, float2 *b, int64_t n, cudaStream_t s)
{
        if (n <= 0) return T3NS_OK;
        const int grid = (int) std::min<int64_t>((n + 255) / 256, 148 * 16);
        split_tf32_kernel<<<grid, 256, 0, s>>>(a, b, n);
        T3NS_CUDA_TRY(cudaGetLastError());
        return T3NS_OK;
}

int launch_heff(const DevicePlan &dp, int precision, const double *x, double *y, cudaStream_t s,
                int *launches, bool per_block)
{
        // a BF16x3-only configuration (5-7) runs the other arithmetic modes in
        // the configuration of the same launch shape (0-2), whose tiling the
        // engine builds beside it (FP64 defect correction after BF16x3)
        int act = dp.active;
        if (act >= kBfFirst && !cfg_supports(act, precision) && dp.tiles[act - kBfFirst].built)
                act -= kBfFirst;
        if (per_block) {
                // the same kernel, one launch per output block (its own unit run)
                const DeviceTiles &full = dp.tiles[act];
                if (!full.built) return set_error(T3NS_E_ARG, "matvec: the active configuration has no tiling");
                if (precision != T3NS_PREC_FP64 || !cfg_supports(act, precision))
                        return set_error(T3NS_E_ARG, "matvec: per-block dispatch is FP64 only");
                T3NS_CUDA_TRY(cudaMemsetAsync(y, 0, sizeof(double) * dp.size, s));
                DevicePlan one = dp;
                one.active = act;
                int n = 0;
                for (size_t r = 0; r + 1 < full.block_runs.size(); r += 2) {
                        DeviceTiles &dt = one.tiles[act];
                        dt.units = full.units + full.block_runs[r];
                        dt.n_units = full.block_runs[r + 1] - full.block_runs[r];
                        dt.grid = std::max(1, std::min(dt.n_units, full.grid));
                        T3NS_CUDA_TRY(cudaMemsetAsync(dp.counter, 0, sizeof(int), s));
                        int rc;
                        switch (act) {
                        case 0: rc = launch_cfg<CfgLarge, double>(one, dt, x, dp.ops, y, s); break;
                        case 1: rc = launch_cfg<CfgSmall, double>(one, dt, x, dp.ops, y, s); break;
                        case 2: rc = launch_cfg<CfgWide, double>(one, dt, x, dp.ops, y, s); break;
                        case 3: rc = launch_v2<CfgV2Wide, false>(one, dt, x, y, s); break;
                        default: rc = launch_v2<CfgV2Large, false>(one, dt, x, y, s); break;
                        }
                        T3NS_TRY(rc);
                        ++n;
                }
                if (launches) *launches = n;
                return T3NS_OK;
        }
        const DeviceTiles &dt = dp.tiles[act];
        if (!dt.built) return set_error(T3NS_E_ARG, "matvec: the active configuration has no tiling");
        const bool split = precision == T3NS_PREC_3XTF32;
        const bool bf = precision == T3NS_PREC_BF16X3;
        if (split && !kCfgs[act].v2 && (!dp.ops_split || !dp.x_split))
                return set_error(T3NS_E_ARG, "matvec: split precision is not set up on this plan");
        if (!cfg_supports(act, precision))
                return set_error(T3NS_E_ARG, "matvec: configuration " + std::to_string(act) +
                                                     " does not run this precision");
        if (bf && (!dp.ops_bf16 || !dp.x_bf16))
                return set_error(T3NS_E_ARG, "matvec: BF16x3 is not set up on this plan");
        if (precision != T3NS_PREC_FP64 && !split && !bf)
                return set_error(T3NS_E_ARG, "matvec: unsupported precision");
        T3NS_CUDA_TRY(cudaMemsetAsync(y, 0, sizeof(double) * dp.size, s));
        if (launches) *launches = 0;
        if (dt.n_units == 0) return T3NS_OK;
        // the contraction-ordered kernel splits the staged blocks itself
        if (split && !kCfgs[act].v2) T3NS_TRY(convert_to_split(x, dp.x_split, dp.size, s));
        if (bf) T3NS_TRY(convert_to_bf16_pairs(x, dp.x_bf16, dp.size, s));
        T3NS_CUDA_TRY(cudaMemsetAsync(dp.counter, 0, sizeof(int), s));
        static_assert(kNumCfgs == 8, "one launch branch per configuration");
        int rc;
        if (act == 3) {
                rc = split ? launch_v2<CfgV2Wide, true>(dp, dt, x, y, s)
                           : launch_v2<CfgV2Wide, false>(dp, dt, x, y, s);
        } else if (act == 4) {
                rc = split ? launch_v2<CfgV2Large, true>(dp, dt, x, y, s)
                           : launch_v2<CfgV2Large, false>(dp, dt, x, y, s);
        } else if (bf) {
                const BfPair *xs = reinterpret_cast<const BfPair *>(dp.x_bf16);
                const BfPair *os = reinterpret_cast<const BfPair *>(dp.ops_bf16);
                switch (act) {
                case 0: rc = launch_cfg<CfgLarge, BfPair>(dp, dt, xs, os, y, s); break;
                case 1: rc = launch_cfg<CfgSmall, BfPair>(dp, dt, xs, os, y, s); break;
                case 2: rc = launch_cfg<CfgWide, BfPair>(dp, dt, xs, os, y, s); break;
                case 5: rc = launch_cfg<CfgLargeB, BfPair>(dp, dt, xs, os, y, s); break;
                case 6: rc = launch_cfg<CfgSmallB, BfPair>(dp, dt, xs, os, y, s); break;
                default: rc = launch_cfg<CfgWideB, BfPair>(dp, dt, xs, os, y, s); break;
                }
        } else if (split) {
                const float2 *xs = dp.x_split, *os = dp.ops_split;
                rc = act == 0   ? launch_cfg<CfgLarge, float2>(dp, dt, xs, os, y, s)
                     : act == 1 ? launch_cfg<CfgSmall, float2>(dp, dt, xs, os, y, s)
                                      : launch_cfg<CfgWide, float2>(dp, dt, xs, os, y, s);
        } else {
                rc = act == 0   ? launch_cfg<CfgLarge, double>(dp, dt, x, dp.ops, y, s)
                     : act == 1 ? launch_cfg<CfgSmall, double>(dp, dt, x, dp.ops, y, s)
                                      : launch_cfg<CfgWide, double>(dp, dt, x, dp.ops, y, s);
        }
        T3NS_TRY(rc);
        if (launches) *launches = ((split && !kCfgs[act].v2) || bf) ? 2 : 1;
        return T3NS_OK;
}

int launch_heff_fp64(const DevicePlan &dp, const double *x, double *y, cudaStream_t s,
                     int *launches)
{
        return launch_heff(dp, T3NS_PREC_FP64, x, y, s, launches);
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
