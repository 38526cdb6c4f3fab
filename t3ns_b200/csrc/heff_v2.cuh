// FP64 matvec kernel with contraction-ordered layouts (kernel configurations
// kV2First and up).  Included by heff.cu.
//
// Same work decomposition as heff_kernel (units = output tiles of one new
// block, pairs, groups of terms going through the stages together), but every
// stage contracts the fastest-varying axis of its input:
//
//   * operator blocks are stored on the device transposed from the reference
//     layout: row-major (new index r, old index k) with the row padded with
//     zeros to a multiple of 4 doubles (op_ld), blocks 32-byte aligned, so a
//     tile's rows are one contiguous range and a lane reads its k values in
//     16-byte pairs;
//   * the old block is staged in shared memory permuted to (s0, s1, s2) for
//     the pair's contraction sequence s, the contracted axis padded with zeros
//     (staged_ld); a block too large to stage is read in place from global
//     memory, which the plan allows only for sequences that start on axis 0;
//   * each stage writes its output directly in the layout the next stage
//     contracts: (next axis, remaining axis, new axis), next axis fastest and
//     zero-padded; the last stage accumulates into the output tile.
//
// A stage is then C(m, n) = sum_k A(m, k) B(k, n) with A the operator rows
// (k contiguous) and B the input columns (k contiguous, stride ldb).  In the
// FP64 tensor-core tile (mma.m8n8k4) lane l holds A[l/4][k] and B[k][l/4] for
// one k per step; the sum over k is order-free, so over a chunk of 8 the lane
// with l%4 = q takes k = 2q in the first step and k = 2q+1 in the second and
// loads both with one 16-byte load from each operand.  Rows and columns past
// the stage's M and N read a clamped (valid) row or column and are not
// stored, so the inner loop has no predicates.
#pragma once

namespace t3ns {
namespace v2 {

// Padded length of a contracted axis in shared memory: a multiple of 4; above
// 8, rounded up to 8 mod 16 doubles when that costs at most a quarter more
// (two columns of a quarter-warp's 16-byte loads then fall on disjoint banks).
__host__ __device__ __forceinline__ int staged_ld(int k)
{
        int p = (k + 3) & ~3;
        if (p > 8) {
                const int q = p + ((8 - p % 16) + 16) % 16;
                if (q - p <= p / 4) p = q;
        }
        return p;
}

// q = a / b, r = a % b for 0 <= a < 2^22 and b > 0, given rb = 1.0f / b: the
// float quotient is off by at most one, which one correction step fixes.
__device__ __forceinline__ int divmod(int a, int b, float rb, int &r)
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

// Row length of an operator block in the transposed device buffer.
__host__ __device__ __forceinline__ int op_ld(int k) { return (k + 3) & ~3; }

// Geometry of one stage of a pair on a unit.
// Element offsets inside a block, a tile or a shared buffer fit 32 bits (plan
// build rejects blocks of 2^31 elements or more).
struct Geo {
        int a;            // contracted axis
        int K, Kp;        // old dim of a and its multiple of 4
        int M;            // new rows (tile extent of a)
        int N;            // columns = product of the two other current dims
        int ldb;          // column stride of the input
        int du;           // columns n = iu + du * iv (input layout (a, u, v))
        int c_is_u;       // next stage contracts u (else v); unused by the last stage
        int str_u, str_v, mstride;   // output address = iu*str_u + iv*str_v + m*mstride
        int out_size;     // elements of the output buffer (padded; 0 for the last stage)
        int next_K, next_Kp, next_cols;  // padding of the output: k in [next_K, next_Kp) of each column
        int lda;          // row length of the operator blocks (op_ld(K))
};

// Stage geometries of a pair: old dims o, tile extents ext (memory axes),
// contraction sequence seq (nst stages; seq[2] is the leftover axis of a
// two-stage pair), staged (the old block is staged in shared memory as
// (s0, s1, s2)), output tile strides ostr.
__device__ __forceinline__ void make_geos(Geo *g, int nst, const int (&seq)[3], const int (&o)[3],
                                          const int (&ext)[3], bool staged, const int (&ostr)[3])
{
        int cur[3] = {o[0], o[1], o[2]};
        // input layout of stage 0: (s0, s1, s2) staged, else natural (0, 1, 2)
        int u = staged ? seq[1] : (seq[0] == 0 ? 1 : 0);
        int v = staged ? seq[2] : 3 - seq[0] - u;
        int ldb = staged ? staged_ld(o[seq[0]]) : o[seq[0]];
        for (int j = 0; j < nst; ++j) {
                Geo &s = g[j];
                const int a = seq[j];
                s.a = a;
                s.K = cur[a];
                s.Kp = (s.K + 3) & ~3;
                s.M = ext[a];
                s.N = cur[u] * cur[v];
                s.ldb = ldb;
                s.du = cur[u];
                s.lda = op_ld(s.K);
                cur[a] = ext[a];
                if (j == nst - 1) {
                        s.c_is_u = false;
                        s.str_u = ostr[u];
                        s.str_v = ostr[v];
                        s.mstride = ostr[a];
                        s.out_size = 0;
                        s.next_K = s.next_Kp = s.next_cols = 0;
                } else {
                        const int c = seq[j + 1];
                        const int r = c == u ? v : u;
                        const int ldn = staged_ld(cur[c]);
                        s.c_is_u = c == u;
                        // next layout (c, r, a): address = ic + ldn * (ir + dim_r * m)
                        s.str_u = s.c_is_u ? 1 : ldn;
                        s.str_v = s.c_is_u ? ldn : 1;
                        s.mstride = ldn * cur[r];
                        s.out_size = ldn * cur[r] * cur[a];
                        s.next_K = cur[c];
                        s.next_Kp = (cur[c] + 3) & ~3;
                        s.next_cols = cur[r] * cur[a];
                        // the next stage's input layout
                        u = r;
                        v = a;
                        ldb = ldn;
                }
        }
}

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b)
{
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                     : "+d"(d0), "+d"(d1)
                     : "d"(a), "d"(b));
}

// K loop of one warp tile for one term: A rows ap[i] (global, k contiguous,
// zero-padded to Kp), B columns bp[j] (k contiguous; NATURAL: the unpadded
// old block in global memory, whose k >= K must not be read).
template <int RM, int RN, bool NATURAL>
__device__ __forceinline__ void k_loop(double (&d)[RM][RN][2], const double *const (&ap)[RM],
                                       const double *const (&bp)[RN], int K, int Kp, int lc)
{
        if constexpr (NATURAL) {
#pragma unroll 1
                for (int k = 0; k < Kp; k += 4) {
                        const int kk = k + lc;
                        const bool ok = kk < K;
                        double a[RM], b[RN];
#pragma unroll
                        for (int i = 0; i < RM; ++i) a[i] = __ldg(ap[i] + kk);
#pragma unroll
                        for (int j = 0; j < RN; ++j) b[j] = ok ? __ldg(bp[j] + kk) : 0.0;
#pragma unroll
                        for (int i = 0; i < RM; ++i)
#pragma unroll
                                for (int j = 0; j < RN; ++j) dmma(d[i][j][0], d[i][j][1], a[i], b[j]);
                }
        } else {
                const int full = Kp >> 3;
                const int q = 2 * lc;
#pragma unroll 2
                for (int c = 0; c < full; ++c) {
                        const int k = 8 * c + q;
                        double2 a[RM], b[RN];
#pragma unroll
                        for (int i = 0; i < RM; ++i) a[i] = __ldg(reinterpret_cast<const double2 *>(ap[i] + k));
#pragma unroll
                        for (int j = 0; j < RN; ++j) b[j] = *reinterpret_cast<const double2 *>(bp[j] + k);
#pragma unroll
                        for (int i = 0; i < RM; ++i)
#pragma unroll
                                for (int j = 0; j < RN; ++j) dmma(d[i][j][0], d[i][j][1], a[i].x, b[j].x);
#pragma unroll
                        for (int i = 0; i < RM; ++i)
#pragma unroll
                                for (int j = 0; j < RN; ++j) dmma(d[i][j][0], d[i][j][1], a[i].y, b[j].y);
                }
                if (Kp & 4) {
                        const int kk = 8 * full + lc;
                        double ta[RM], tb[RN];
#pragma unroll
                        for (int i = 0; i < RM; ++i) ta[i] = __ldg(ap[i] + kk);
#pragma unroll
                        for (int j = 0; j < RN; ++j) tb[j] = bp[j][kk];
#pragma unroll
                        for (int i = 0; i < RM; ++i)
#pragma unroll
                                for (int j = 0; j < RN; ++j) dmma(d[i][j][0], d[i][j][1], ta[i], tb[j]);
                }
        }
}

// One stage for G terms (see the file comment).  Term g applies the operator
// rows at ops + opoff[g] (row length lda) to `in + g * in_gs` and writes
// `out + g * out_gs` scaled by scale[g] (scale may be null); with ACC the G
// results are summed into `out` (the output tile).  When an accumulating
// stage has fewer tiles than the CTA has warps, its terms are dealt to P
// parts whose partial tiles go to scratch and are added in part order.
template <bool ACC, int RM, int RN, int NW, bool NATURAL>
__device__ __forceinline__ void stage_t(const Geo &s, int G, const int64_t *opoff,
                                        const double *__restrict__ ops, const double *in, int in_gs,
                                        double *out, int out_gs, const double *scale,
                                        double *scratch, int scratch_cap)
{
        // the geometry lives in shared memory: take what the loops need into
        // registers once (stores to the output buffers could alias it)
        const int M = s.M, N = s.N, lda = s.lda, ldb = s.ldb, K = s.K, Kp = s.Kp;
        const int du = s.du, str_u = s.str_u, str_v = s.str_v, mstride = s.mstride;
        const float rdu = 1.0f / du;
        const int mt = (M + 8 * RM - 1) / (8 * RM), nt = (N + 8 * RN - 1) / (8 * RN);
        const int tiles = mt * nt;
        const float rtiles = 1.0f / tiles, rmt = 1.0f / mt;
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
#pragma unroll 1
        for (int it = warp; it < items; it += NW) {
                int tile, tm;
                const int q = divmod(it, tiles, rtiles, tile);
                const int tn = divmod(tile, mt, rmt, tm);
                const int m0 = tm * 8 * RM, n0 = tn * 8 * RN;
                int arow[RM], bcol[RN];
#pragma unroll
                for (int i = 0; i < RM; ++i) arow[i] = min(m0 + 8 * i + lr, M - 1) * lda;
#pragma unroll
                for (int j = 0; j < RN; ++j) bcol[j] = min(n0 + 8 * j + lr, N - 1) * ldb;
                double d[RM][RN][2];
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int j = 0; j < RN; ++j) d[i][j][0] = d[i][j][1] = 0.0;
                const int g1 = ACC ? G : q + 1;
                const int gstep = ACC ? P : 1;
#pragma unroll 1
                for (int g = q; g < g1; g += gstep) {
                        const double *op = ops + opoff[g];
                        const double *tin = in + (int64_t) g * in_gs;
                        const double *ap[RM];
                        const double *bp[RN];
#pragma unroll
                        for (int i = 0; i < RM; ++i) ap[i] = op + arow[i];
#pragma unroll
                        for (int j = 0; j < RN; ++j) bp[j] = tin + bcol[j];
                        k_loop<RM, RN, NATURAL>(d, ap, bp, K, Kp, lc);
                }
                const double sc = (!ACC && scale) ? scale[q] : 1.0;
                double *Cb = out + (ACC ? 0 : (int64_t) q * out_gs);
                // output offsets of this lane's columns
                int coff[RN][2];
                bool cok[RN][2];
#pragma unroll
                for (int j = 0; j < RN; ++j)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                                const int n = n0 + 8 * j + 2 * lc + h;
                                cok[j][h] = n < N;
                                int iu;
                                const int iv = divmod(n, du, rdu, iu);
                                coff[j][h] = iu * str_u + iv * str_v;
                        }
#pragma unroll
                for (int i = 0; i < RM; ++i) {
                        const int m = m0 + 8 * i + lr;
                        if (m >= M) continue;
                        const int ro = m * mstride;
#pragma unroll
                        for (int j = 0; j < RN; ++j)
#pragma unroll
                                for (int h = 0; h < 2; ++h) {
                                        if (!cok[j][h]) continue;
                                        if (ACC && P > 1) {
                                                const int n = n0 + 8 * j + 2 * lc + h;
                                                scratch[(int64_t) q * MN + m + (int64_t) n * M] = d[i][j][h];
                                                continue;
                                        }
                                        double *cp = Cb + ro + coff[j][h];
                                        *cp = ACC ? *cp + d[i][j][h] : sc * d[i][j][h];
                                }
                }
        }
        if (ACC && P > 1) {
                __syncthreads();
                const float rM = 1.0f / M;
                for (int e = threadIdx.x; e < MN; e += NW * 32) {
                        int m, iu;
                        const int n = divmod(e, M, rM, m);
                        double sum = 0.0;
                        for (int p = 0; p < P; ++p) sum += scratch[(int64_t) p * MN + e];
                        const int iv = divmod(n, du, rdu, iu);
                        out[m * mstride + iu * str_u + iv * str_v] += sum;
                }
        }
        if (!ACC && s.next_Kp > s.next_K) {
                // zero the padding of the next stage's contracted axis: columns of
                // the next layout are ldn apart, k in [next_K, next_Kp)
                const int nk = s.next_K, padw = s.next_Kp - nk;
                const int cols = G * s.next_cols;   // the G outputs are out_gs = cols * ldn apart
                const int ldn = s.c_is_u ? str_v : str_u;
                for (int c = threadIdx.x; c < cols; c += NW * 32)
                        for (int k = 0; k < padw; ++k) out[(int64_t) c * ldn + nk + k] = 0.0;
        }
}

// The stage's geometry is read from shared memory (written once per pair).
template <bool ACC, int NW, bool NATURAL>
__device__ __forceinline__ void stage(const Geo &s, int G, const int64_t *opoff,
                                      const double *__restrict__ ops, const double *in, int in_gs,
                                      double *out, int out_gs, const double *scale,
                                      double *scratch = nullptr, int scratch_cap = 0)
{
        if (s.M <= 8)
                stage_t<ACC, 1, 4, NW, NATURAL>(s, G, opoff, ops, in, in_gs, out, out_gs, scale,
                                                scratch, scratch_cap);
        else if (s.N <= 8)
                stage_t<ACC, 4, 1, NW, NATURAL>(s, G, opoff, ops, in, in_gs, out, out_gs, scale,
                                                scratch, scratch_cap);
        else
                stage_t<ACC, 2, 2, NW, NATURAL>(s, G, opoff, ops, in, in_gs, out, out_gs, scale,
                                                scratch, scratch_cap);
}

// ---------------------------------------------------------------------------
// Split precision (3xTF32) on the same layouts.  Operators, the staged block
// and the intermediates hold {hi, lo} TF32 pairs (float2: hi = tf32(x),
// lo = tf32(x - hi)), the products run on the TF32 tensor pipe
// (mma.m16n8k8) as lo*hi + hi*lo + hi*hi with FP32 accumulation, and the
// output tile accumulates in FP64.  In the m16n8k8 fragments lane (g, t)
// (g = lane / 4, t = lane % 4) holds A[g][t], A[g+8][t], A[g][t+4],
// A[g+8][t+4] and B[t][g], B[t+4][g]: the k slots t and t+4 map to the
// physical k = 2t and 2t+1 of a chunk of 8, so one 16-byte load brings the
// two pairs of a row (or column).

__device__ __forceinline__ uint32_t tf32_bits(float x)
{
        uint32_t r;
        asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(x));
        return r;
}

__device__ __forceinline__ float2 split_pair(float x)
{
        const uint32_t hi = tf32_bits(x);
        return make_float2(__uint_as_float(hi), __uint_as_float(tf32_bits(x - __uint_as_float(hi))));
}

// {hi, lo} of an FP64 value: the remainder is taken in FP64, so lo carries
// the bits that a rounding to FP32 first would lose.
__device__ __forceinline__ float2 split_pair(double x)
{
        const float hi = __uint_as_float(tf32_bits((float) x));
        return make_float2(hi, __uint_as_float(tf32_bits((float) (x - (double) hi))));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&b)[2])
{
        asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, "
                     "{%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
                     : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                     : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One chunk of 8 k (tail: of 4, the lanes with t >= 2 contributing zeros).
// A rows ap[i][r] (pairs, global), B columns bp[j] (pairs in shared memory,
// or with NATURAL the FP64 old block in global memory, unpadded: k >= K read
// as zero and split here).
template <int RM, int RN, bool NATURAL>
__device__ __forceinline__ void x_chunk(float (&d)[RM][RN][4], const float2 *const (&ap)[RM][2],
                                        const void *const (&bpv)[RN], int k, bool tail, int K, int t)
{
        const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
        const bool on = !tail || t < 2;
        uint32_t ah[RM][4], al[RM][4], bh[RN][2], bl[RN][2];
#pragma unroll
        for (int i = 0; i < RM; ++i) {
                float4 v[2];
#pragma unroll
                for (int r = 0; r < 2; ++r)
                        v[r] = on ? __ldg(reinterpret_cast<const float4 *>(ap[i][r] + k)) : z;
                ah[i][0] = __float_as_uint(v[0].x);
                ah[i][1] = __float_as_uint(v[1].x);
                ah[i][2] = __float_as_uint(v[0].z);
                ah[i][3] = __float_as_uint(v[1].z);
                al[i][0] = __float_as_uint(v[0].y);
                al[i][1] = __float_as_uint(v[1].y);
                al[i][2] = __float_as_uint(v[0].w);
                al[i][3] = __float_as_uint(v[1].w);
        }
#pragma unroll
        for (int j = 0; j < RN; ++j) {
                float4 v;
                if constexpr (NATURAL) {
                        const double *bp = static_cast<const double *>(bpv[j]);
                        const float2 p0 = k < K ? split_pair(__ldg(bp + k)) : make_float2(0.f, 0.f);
                        const float2 p1 = k + 1 < K ? split_pair(__ldg(bp + k + 1)) : make_float2(0.f, 0.f);
                        v = make_float4(p0.x, p0.y, p1.x, p1.y);
                } else {
                        v = on ? *reinterpret_cast<const float4 *>(static_cast<const float2 *>(bpv[j]) + k) : z;
                }
                bh[j][0] = __float_as_uint(v.x);
                bh[j][1] = __float_as_uint(v.z);
                bl[j][0] = __float_as_uint(v.y);
                bl[j][1] = __float_as_uint(v.w);
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

// The split-precision stage (as stage_t): warp tiles of RM x RN m16n8
// tiles; non-accumulating stages write {hi, lo} pairs of the scaled result,
// the accumulating stage adds its FP32 group sums into the FP64 tile.
template <bool ACC, int RM, int RN, int NW, bool NATURAL>
__device__ __forceinline__ void stage_x_t(const Geo &s, int G, const int64_t *opoff,
                                          const float2 *__restrict__ ops, const void *in, int in_gs,
                                          void *outv, int out_gs, const double *scale,
                                          float *scratch, int scratch_cap)
{
        const int M = s.M, N = s.N, lda = s.lda, ldb = s.ldb, K = s.K;
        const int du = s.du, str_u = s.str_u, str_v = s.str_v, mstride = s.mstride;
        const float rdu = 1.0f / du;
        const int mt = (M + 16 * RM - 1) / (16 * RM), nt = (N + 8 * RN - 1) / (8 * RN);
        const int tiles = mt * nt;
        const float rtiles = 1.0f / tiles, rmt = 1.0f / mt;
        int P = 1;
        const int MN = M * N;
        if (ACC && tiles < NW && G > 1 && scratch) {
                P = min(G, NW / tiles);
                P = min(P, scratch_cap / max(MN, 1));
                if (P < 2) P = 1;
        }
        const int items = (ACC ? P : G) * tiles;
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        const int gq = lane >> 2, t = lane & 3;
        const int full = s.Kp >> 3;
        const bool tail = (s.Kp & 4) != 0;
#pragma unroll 1
        for (int it = warp; it < items; it += NW) {
                int tile, tm;
                const int q = divmod(it, tiles, rtiles, tile);
                const int tn = divmod(tile, mt, rmt, tm);
                const int m0 = tm * 16 * RM, n0 = tn * 8 * RN;
                int arow[RM][2], bcol[RN];
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int r = 0; r < 2; ++r) arow[i][r] = min(m0 + 16 * i + 8 * r + gq, M - 1) * lda;
#pragma unroll
                for (int j = 0; j < RN; ++j) bcol[j] = min(n0 + 8 * j + gq, N - 1) * ldb;
                float d[RM][RN][4];
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int j = 0; j < RN; ++j)
#pragma unroll
                                for (int e = 0; e < 4; ++e) d[i][j][e] = 0.f;
                const int g1 = ACC ? G : q + 1;
                const int gstep = ACC ? P : 1;
#pragma unroll 1
                for (int g = q; g < g1; g += gstep) {
                        const float2 *op = ops + opoff[g];
                        const float2 *ap[RM][2];
                        const void *bp[RN];
#pragma unroll
                        for (int i = 0; i < RM; ++i)
#pragma unroll
                                for (int r = 0; r < 2; ++r) ap[i][r] = op + arow[i][r];
#pragma unroll
                        for (int j = 0; j < RN; ++j) {
                                if constexpr (NATURAL)
                                        bp[j] = static_cast<const double *>(in) + (int64_t) g * in_gs + bcol[j];
                                else
                                        bp[j] = static_cast<const float2 *>(in) + (int64_t) g * in_gs + bcol[j];
                        }
#pragma unroll 1
                        for (int c = 0; c < full; ++c)
                                x_chunk<RM, RN, NATURAL>(d, ap, bp, 8 * c + 2 * t, false, K, t);
                        if (tail) x_chunk<RM, RN, NATURAL>(d, ap, bp, 8 * full + 2 * t, true, K, t);
                }
                const float sc = (!ACC && scale) ? (float) scale[q] : 1.f;
                int coff[RN][2];
                bool cok[RN][2];
#pragma unroll
                for (int j = 0; j < RN; ++j)
#pragma unroll
                        for (int h = 0; h < 2; ++h) {
                                const int n = n0 + 8 * j + 2 * t + h;
                                cok[j][h] = n < N;
                                int iu;
                                const int iv = divmod(n, du, rdu, iu);
                                coff[j][h] = iu * str_u + iv * str_v;
                        }
#pragma unroll
                for (int i = 0; i < RM; ++i)
#pragma unroll
                        for (int r = 0; r < 2; ++r) {
                                const int m = m0 + 16 * i + 8 * r + gq;
                                if (m >= M) continue;
                                const int ro = m * mstride;
#pragma unroll
                                for (int j = 0; j < RN; ++j)
#pragma unroll
                                        for (int h = 0; h < 2; ++h) {
                                                if (!cok[j][h]) continue;
                                                const float v = d[i][j][2 * r + h];
                                                if constexpr (ACC) {
                                                        if (P > 1) {
                                                                const int n = n0 + 8 * j + 2 * t + h;
                                                                scratch[(int64_t) q * MN + m + (int64_t) n * M] = v;
                                                        } else {
                                                                double *cp = static_cast<double *>(outv) + ro + coff[j][h];
                                                                *cp += (double) v;
                                                        }
                                                } else {
                                                        float2 *cp = static_cast<float2 *>(outv) + (int64_t) q * out_gs +
                                                                     ro + coff[j][h];
                                                        *cp = split_pair(sc * v);
                                                }
                                        }
                        }
        }
        if (ACC && P > 1) {
                __syncthreads();
                double *out = static_cast<double *>(outv);
                const float rM = 1.0f / M;
                for (int e = threadIdx.x; e < MN; e += NW * 32) {
                        int m, iu;
                        const int n = divmod(e, M, rM, m);
                        float sum = 0.f;
                        for (int p = 0; p < P; ++p) sum += scratch[(int64_t) p * MN + e];
                        const int iv = divmod(n, du, rdu, iu);
                        out[m * mstride + iu * str_u + iv * str_v] += (double) sum;
                }
        }
        if (!ACC && s.next_Kp > s.next_K) {
                float2 *out = static_cast<float2 *>(outv);
                const int nk = s.next_K, padw = s.next_Kp - nk;
                const int cols = G * s.next_cols;
                const int ldn = s.c_is_u ? str_v : str_u;
                for (int c = threadIdx.x; c < cols; c += NW * 32)
                        for (int k = 0; k < padw; ++k) out[(int64_t) c * ldn + nk + k] = make_float2(0.f, 0.f);
        }
}

template <bool ACC, int NW, bool NATURAL>
__device__ __forceinline__ void stage_x(const Geo &s, int G, const int64_t *opoff,
                                        const float2 *__restrict__ ops, const void *in, int in_gs,
                                        void *out, int out_gs, const double *scale,
                                        float *scratch = nullptr, int scratch_cap = 0)
{
        if (s.M <= 16)
                stage_x_t<ACC, 1, 4, NW, NATURAL>(s, G, opoff, ops, in, in_gs, out, out_gs, scale,
                                                  scratch, scratch_cap);
        else if (s.N <= 8)
                stage_x_t<ACC, 4, 1, NW, NATURAL>(s, G, opoff, ops, in, in_gs, out, out_gs, scale,
                                                  scratch, scratch_cap);
        else
                stage_x_t<ACC, 2, 2, NW, NATURAL>(s, G, opoff, ops, in, in_gs, out, out_gs, scale,
                                                  scratch, scratch_cap);
}

}  // namespace v2
}  // namespace t3ns
