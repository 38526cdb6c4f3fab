// Internal data structures of the matvec engine (host plan, device plan).
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <cstdint>
#include <vector>

#include "t3ns_b200.h"

namespace t3ns {

// One (new block, old block, instruction) term: op_off[j] is the element
// offset, in the device operator buffer, of the operator block acting on
// memory axis j; `axes` packs the contraction sequence (2 bits per stage,
// stage count in bits 6-7); pref = instruction prefactor * symmetry prefactor.
struct __align__(16) HeffTask {
        int64_t op_off[3];
        double pref;
        int old;
        int axes;
};

// One (new, old) block pair: its terms are tasks[t0, t1); `axes` packs the
// contraction sequence chosen for the pair (same encoding as HeffTask).
struct __align__(16) HeffPair {
        int old;
        int axes;
        int t0, t1;
};

// One unit of kernel work: the output tile [a0,a0+at) x [b0,b0+bt) x
// [c0,c0+ct) of new block nb (memory axes), over pairs [p0, p1) of nb.
// When a tile's pairs are split over several units (split != 0) each adds
// its share into the output with atomics.
struct __align__(16) HeffUnit {
        int nb;
        int b0, bt;
        int c0, ct;
        int a0, at;
        int p0, p1;
        int split;
        int pad[2];
};

// Kernel configurations (launch shape and shared-memory buffers, in
// elements of the compute type); a plan is tiled for one of them.
struct KernelCfg {
        int threads;       // per CTA
        int ctas_per_sm;   // resident CTAs per SM the launch is sized for
        int out_cap;       // output tile
        int psi_cap;       // staged old block
        int w_cap;         // intermediates of a group of terms
        const char *name;
        int v2;            // 1: contraction-ordered layouts (heff_v2_kernel)
        int bf16;          // 1: BF16x3 only, buffers sized in BF16 pairs
};
constexpr int kNumCfgs = 8;
constexpr int kV2First = 3;   // configurations 3, 4 run heff_v2_kernel
constexpr int kBfFirst = 5;   // configurations 5-7: BF16x3 tilings of 0-2

// Whether configuration cfg runs matvecs in arithmetic `precision`.
bool cfg_supports(int cfg, int precision);
extern const KernelCfg kCfgs[kNumCfgs];

// One (new, old) pair before tiling: its terms and the old block's dims.
// The terms are sorted by their operator block on memory axis dax, the axis
// with the fewest distinct operator blocks (dfrac = distinct / terms): a
// sequence that starts on dax computes each distinct first-stage result once.
struct PairTmp {
        int ob;
        int t0, t1;
        int eo[3];
        int dax;
        double dfrac;
};

// The pairs and work units of a plan tiled for one kernel configuration.
struct TilePlan {
        bool built = false;
        std::vector<int> pair_ptr;                // [nblocks + 1] into pairs
        std::vector<HeffPair> pairs;
        std::vector<HeffUnit> units;              // heaviest first
        double flops_exec = 0;
};

struct HostPlan {
        int isdmrg = 0;
        int map[3] = {0, 1, 2};
        int nblocks = 0;
        int64_t size = 0;
        std::vector<int64_t> block_off;
        std::vector<int4> edims;                  // memory-axis dims per block
        std::vector<std::vector<int64_t>> op_base;  // [set][op] element base
        int64_t op_elems = 0;
        std::vector<int> task_ptr;
        std::vector<HeffTask> tasks;
        std::vector<std::vector<PairTmp>> blocks_pairs;   // per new block
        TilePlan tiles[kNumCfgs];
        int64_t npairs = 0;
        double flops_ref = 0, bytes_alg = 0;
        // transposed operator buffer of the contraction-ordered kernel: every
        // referenced operator block row-major (new x old), rows padded with
        // zeros to v2::op_ld(old dim), 32-byte aligned; toff[3 * task + axis]
        // is the block's offset there, tjobs the transposition jobs
        // {reference offset, transposed offset, rows, cols}
        std::vector<int64_t> toff;
        std::vector<int64_t> tjobs;
        int64_t opt_elems = 0;
};

// Device copy of one tiling.
struct DeviceTiles {
        bool built = false;
        int *pair_ptr = nullptr;
        HeffPair *pairs = nullptr;
        HeffUnit *units = nullptr;
        int n_units = 0;
        int grid = 0;
        // runs [block_runs[2i], block_runs[2i+1]) of the units of one output
        // block (the unit list keeps a block's tiles together)
        std::vector<int> block_runs;
};

struct DevicePlan {
        int nblocks = 0;
        int64_t size = 0;
        double *ops = nullptr;
        double *ops_t = nullptr;                  // transposed operators (v2 configurations)
        float2 *ops_t_split = nullptr;            // their {hi, lo} TF32 pairs
        int64_t *toff = nullptr;                  // their offsets per task and axis
        float2 *ops_split = nullptr;              // {hi, lo} TF32 split of the operators
        float2 *x_split = nullptr;                // {hi, lo} split of the matvec input
        uint32_t *ops_bf16 = nullptr;             // k-paired {hi, lo} BF16 copy of the operators
                                                  // (2 * op_elems pairs, block at twice its offset)
        uint32_t *x_bf16 = nullptr;               // and of the matvec input
        int64_t *blk_off = nullptr;
        int4 *edims = nullptr;
        int *task_ptr = nullptr;
        HeffTask *tasks = nullptr;
        DeviceTiles tiles[kNumCfgs];
        int active = 0;                           // configuration the matvec runs
        // when set (by the request loop), the number of solves sharing the
        // GPU: each matvec launch takes that share of the persistent grid, so
        // concurrent solves run side by side instead of queueing for SMs
        const std::atomic<int> *share = nullptr;
        int *counter = nullptr;                   // dynamic unit scheduler
        int *err = nullptr;
};

// Shared part of the plan (terms, block tables) and the tiling for
// configuration 0.
int build_plan(const t3ns_heff_desc *d, HostPlan &hp);
// Tiling of hp for configuration cfg (hp.tiles[cfg]).
int tile_plan(HostPlan &hp, int cfg);
int launch_heff_fp64(const DevicePlan &dp, const double *x, double *y, cudaStream_t s,
                     int *launches);
// The matvec in precision T3NS_PREC_FP64 or T3NS_PREC_3XTF32 (FP64 in and out).
// per_block: one launch per output block over that block's units (the
// per-block dispatch a loop over blocks would issue), for comparison with the
// single persistent launch.
int launch_heff(const DevicePlan &dp, int precision, const double *x, double *y, cudaStream_t s,
                int *launches, bool per_block = false);
int convert_to_split(const double *a, float2 *b, int64_t n, cudaStream_t s);
// {hi, lo} BF16 pairs (hi in the low 16 bits) of n doubles.
int convert_to_bf16_pairs(const double *a, void *b, int64_t n, cudaStream_t s);
// Fills dp.ops_bf16 (2 * op_elems pairs) with the k-paired BF16 copy of every
// referenced operator block (the plan's transposition job list).
int build_paired_bf16_ops(const HostPlan &hp, DevicePlan &dp, const int64_t *d_jobs,
                          cudaStream_t s);
// {hi, lo} pairs of the transposed operators.
int convert_to_pairs(const double *a, float2 *b, int64_t n, cudaStream_t s);
// Fills dp.ops_t from dp.ops with the plan's transposition jobs.
int build_transposed_ops(const HostPlan &hp, DevicePlan &dp, const int64_t *d_jobs,
                         cudaStream_t s);
int launch_heff_diag(const DevicePlan &dp, double *diag, cudaStream_t s);

}  // namespace t3ns

struct t3ns_heff {
        t3ns::HostPlan hp;
        t3ns::DevicePlan dp;
        int precision = T3NS_PREC_FP64;
        int device = 0;
        int last_launches = 0;
        double *stage_x = nullptr;   // device staging for host-buffer calls
        double *stage_y = nullptr;
        cudaStream_t stream = nullptr;
        std::vector<void *> allocs;
};
