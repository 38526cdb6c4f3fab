// C ABI of the engine (include/t3ns_b200.h): plan lifetime, device uploads,
// host/device matvec entry points and error reporting.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "common.h"
#include "heff_internal.h"

namespace t3ns {

static thread_local std::string g_last_error;

int set_error(int code, const std::string &msg)
{
        g_last_error = msg;
        return code;
}

template <class T>
static int dev_alloc(t3ns_heff *h, T **p, size_t n)
{
        *p = nullptr;
        if (n == 0) n = 1;
        cudaError_t e = cudaMalloc((void **) p, sizeof(T) * n);
        if (e != cudaSuccess) {
                cudaGetLastError();
                return set_error(T3NS_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e) +
                                                       " (" + std::to_string(sizeof(T) * n) + " bytes)");
        }
        h->allocs.push_back(*p);
        return T3NS_OK;
}

template <class T>
static int upload(t3ns_heff *h, T **p, const T *src, size_t n)
{
        T3NS_TRY(dev_alloc(h, p, n));
        if (n) T3NS_CUDA_TRY(cudaMemcpy(*p, src, sizeof(T) * n, cudaMemcpyHostToDevice));
        return T3NS_OK;
}

// Autotuner cache: size bucket -> fastest configuration.
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int>, int> g_tune_cache;

static std::tuple<int, int, int, int> size_bucket(const HostPlan &hp, int precision)
{
        int64_t maxblk = 1;
        for (int b = 0; b < hp.nblocks; ++b)
                maxblk = std::max<int64_t>(maxblk, hp.block_off[b + 1] - hp.block_off[b]);
        auto lg = [](double v) { return v > 1 ? (int) std::floor(std::log2(v)) : 0; };
        return {lg((double) hp.size), lg((double) maxblk), lg(hp.flops_ref), precision};
}

static int check_device_error(t3ns_heff *h, cudaStream_t s = nullptr);

// Transposed operators of the contraction-ordered configurations (built on
// the device from the resident operators, on first use).
static int setup_transposed(t3ns_heff *h)
{
        DevicePlan &dp = h->dp;
        if (dp.ops_t) return T3NS_OK;
        const HostPlan &hp = h->hp;
        T3NS_TRY(upload(h, &dp.toff, hp.toff.data(), hp.toff.size()));
        T3NS_TRY(dev_alloc(h, &dp.ops_t, (size_t) hp.opt_elems));
        int64_t *d_jobs = nullptr;
        if (!hp.tjobs.empty()) {
                T3NS_CUDA_TRY(cudaMalloc(&d_jobs, sizeof(int64_t) * hp.tjobs.size()));
                const cudaError_t e = cudaMemcpy(d_jobs, hp.tjobs.data(), sizeof(int64_t) * hp.tjobs.size(),
                                                 cudaMemcpyHostToDevice);
                int rc = e == cudaSuccess ? build_transposed_ops(hp, dp, d_jobs, h->stream)
                                          : set_error(T3NS_E_CUDA, std::string("transposed operators: upload: ") +
                                                                       cudaGetErrorString(e));
                if (rc == T3NS_OK) {
                        const cudaError_t se = cudaStreamSynchronize(h->stream);
                        if (se != cudaSuccess)
                                rc = set_error(T3NS_E_CUDA, std::string("transposed operators: kernel: ") +
                                                                    cudaGetErrorString(se));
                }
                if (rc == T3NS_OK) rc = check_device_error(h);
                cudaFree(d_jobs);
                T3NS_TRY(rc);
        }
        return T3NS_OK;
}

// {hi, lo} pairs of the transposed operators (split precision on the
// contraction-ordered configurations).
static int setup_transposed_split(t3ns_heff *h)
{
        DevicePlan &dp = h->dp;
        if (dp.ops_t_split) return T3NS_OK;
        T3NS_TRY(setup_transposed(h));
        T3NS_TRY(dev_alloc(h, &dp.ops_t_split, (size_t) h->hp.opt_elems));
        T3NS_TRY(convert_to_pairs(dp.ops_t, dp.ops_t_split, h->hp.opt_elems, h->stream));
        T3NS_CUDA_TRY(cudaStreamSynchronize(h->stream));
        return T3NS_OK;
}

// Device copy of the tiling for configuration cfg (tiled on first use).
static int upload_tiles(t3ns_heff *h, int cfg)
{
        if (kCfgs[cfg].v2) {
                T3NS_TRY(setup_transposed(h));
                if (h->precision == T3NS_PREC_3XTF32) T3NS_TRY(setup_transposed_split(h));
        }
        DeviceTiles &dt = h->dp.tiles[cfg];
        if (dt.built) return T3NS_OK;
        T3NS_TRY(tile_plan(h->hp, cfg));
        const TilePlan &tp = h->hp.tiles[cfg];
        T3NS_TRY(upload(h, &dt.pair_ptr, tp.pair_ptr.data(), tp.pair_ptr.size()));
        T3NS_TRY(upload(h, &dt.pairs, tp.pairs.data(), tp.pairs.size()));
        T3NS_TRY(upload(h, &dt.units, tp.units.data(), tp.units.size()));
        dt.n_units = (int) tp.units.size();
        dt.block_runs.clear();
        for (int u = 0; u < dt.n_units; ++u)
                if (u == 0 || tp.units[u].nb != tp.units[u - 1].nb) {
                        if (u) dt.block_runs.push_back(u);
                        dt.block_runs.push_back(u);
                }
        if (dt.n_units) dt.block_runs.push_back(dt.n_units);
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
        dt.grid = std::max(1, std::min(dt.n_units, kCfgs[cfg].ctas_per_sm * sms));
        dt.built = true;
        return T3NS_OK;
}

// Pre-split {hi, lo} operator copy and input staging of the split-precision
// matvec.
static int setup_precision(t3ns_heff *h, int precision)
{
        if (precision != T3NS_PREC_FP64 && precision != T3NS_PREC_3XTF32 &&
            precision != T3NS_PREC_BF16X3)
                return set_error(T3NS_E_ARG, "unknown precision");
        DevicePlan &dp = h->dp;
        if (!cfg_supports(dp.active, precision)) {
                // the active configuration does not run this precision
                // (3, 4: not BF16x3; 5-7: BF16x3 only): fall back to 0
                T3NS_TRY(upload_tiles(h, 0));
                dp.active = 0;
        }
        if (precision == T3NS_PREC_BF16X3) {
                if (!dp.ops_bf16) {
                        const HostPlan &hp = h->hp;
                        T3NS_TRY(dev_alloc(h, &dp.ops_bf16, 2 * (size_t) std::max<int64_t>(hp.op_elems, 1)));
                        T3NS_TRY(dev_alloc(h, &dp.x_bf16, (size_t) hp.size));
                        if (!hp.tjobs.empty()) {
                                int64_t *d_jobs = nullptr;
                                T3NS_CUDA_TRY(cudaMalloc(&d_jobs, sizeof(int64_t) * hp.tjobs.size()));
                                const cudaError_t e = cudaMemcpy(d_jobs, hp.tjobs.data(),
                                                                 sizeof(int64_t) * hp.tjobs.size(),
                                                                 cudaMemcpyHostToDevice);
                                int rc = e == cudaSuccess
                                                 ? build_paired_bf16_ops(hp, dp, d_jobs, h->stream)
                                                 : set_error(T3NS_E_CUDA, std::string("paired operators: upload: ") +
                                                                                  cudaGetErrorString(e));
                                if (rc == T3NS_OK) {
                                        const cudaError_t se = cudaStreamSynchronize(h->stream);
                                        if (se != cudaSuccess)
                                                rc = set_error(T3NS_E_CUDA, std::string("paired operators: kernel: ") +
                                                                                    cudaGetErrorString(se));
                                }
                                if (rc == T3NS_OK) rc = check_device_error(h);
                                cudaFree(d_jobs);
                                T3NS_TRY(rc);
                        }
                }
        }
        if (precision == T3NS_PREC_3XTF32 && !dp.ops_split) {
                T3NS_TRY(dev_alloc(h, &dp.ops_split, (size_t) h->hp.op_elems));
                T3NS_TRY(dev_alloc(h, &dp.x_split, (size_t) h->hp.size));
                T3NS_TRY(convert_to_split(dp.ops, dp.ops_split, h->hp.op_elems, h->stream));
                T3NS_CUDA_TRY(cudaStreamSynchronize(h->stream));
        }
        h->precision = precision;
        if (precision == T3NS_PREC_3XTF32 && dp.ops_t) T3NS_TRY(setup_transposed_split(h));
        return T3NS_OK;
}

static int create_impl(const t3ns_heff_desc *desc, int precision, t3ns_heff *h)
{
        T3NS_CUDA_TRY(cudaGetDevice(&h->device));
        T3NS_TRY(build_plan(desc, h->hp));
        HostPlan &hp = h->hp;
        DevicePlan &dp = h->dp;
        dp.nblocks = hp.nblocks;
        dp.size = hp.size;

        // operators: one buffer, every operator's elements at its base offset
        T3NS_TRY(dev_alloc(h, &dp.ops, (size_t) hp.op_elems));
        const int nops = hp.isdmrg ? 2 : 3;
        for (int i = 0; i < nops; ++i) {
                const t3ns_ropset &rs = desc->ops[i];
                for (int k = 0; k < rs.nrops; ++k) {
                        const int64_t n = rs.op_beginblock[k][rs.op_nblocks[k]];
                        if (n > 0)
                                T3NS_CUDA_TRY(cudaMemcpy(dp.ops + hp.op_base[i][k], rs.op_tel[k],
                                                         sizeof(double) * n, cudaMemcpyHostToDevice));
                }
        }
        T3NS_TRY(upload(h, &dp.blk_off, hp.block_off.data(), hp.block_off.size()));
        T3NS_TRY(upload(h, &dp.edims, hp.edims.data(), hp.edims.size()));
        T3NS_TRY(upload(h, &dp.task_ptr, hp.task_ptr.data(), hp.task_ptr.size()));
        T3NS_TRY(upload(h, &dp.tasks, hp.tasks.data(), hp.tasks.size()));
        int cfg = 0;
        {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                auto it = g_tune_cache.find(size_bucket(hp, precision));
                if (it != g_tune_cache.end()) cfg = it->second;
        }
        // status word, counter and stream first: the tiling of a cached
        // configuration may already launch set-up kernels
        T3NS_TRY(dev_alloc(h, &dp.counter, 1));
        T3NS_TRY(dev_alloc(h, &dp.err, 1));
        T3NS_CUDA_TRY(cudaMemset(dp.err, 0, sizeof(int)));
        T3NS_TRY(dev_alloc(h, &h->stage_x, (size_t) hp.size));
        T3NS_TRY(dev_alloc(h, &h->stage_y, (size_t) hp.size));
        T3NS_CUDA_TRY(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        T3NS_TRY(upload_tiles(h, cfg));
        if (kCfgs[cfg].bf16) T3NS_TRY(upload_tiles(h, cfg - kBfFirst));
        dp.active = cfg;
        return setup_precision(h, precision);
}

// Reads the kernel's error status after the work on stream s (the plan's
// own stream when s is null): the copy is ordered after that work.
static int check_device_error(t3ns_heff *h, cudaStream_t s)
{
        if (!s) s = h->stream;
        int err = 0;
        T3NS_CUDA_TRY(cudaMemcpyAsync(&err, h->dp.err, sizeof(int), cudaMemcpyDeviceToHost, s));
        T3NS_CUDA_TRY(cudaStreamSynchronize(s));
        if (err) {
                T3NS_CUDA_TRY(cudaMemsetAsync(h->dp.err, 0, sizeof(int), s));
                T3NS_CUDA_TRY(cudaStreamSynchronize(s));
                return set_error(T3NS_E_DEVICE, "matvec kernel reported error status " +
                                                         std::to_string(err));
        }
        return T3NS_OK;
}

}  // namespace t3ns

using namespace t3ns;

extern "C" {

int t3ns_heff_create(const t3ns_heff_desc *desc, int precision, t3ns_heff **out)
{
        if (!out) return set_error(T3NS_E_ARG, "out is NULL");
        *out = nullptr;
        if (precision != T3NS_PREC_FP64 && precision != T3NS_PREC_3XTF32 &&
            precision != T3NS_PREC_BF16X3)
                return set_error(T3NS_E_ARG, "unknown precision");
        t3ns_heff *h = new (std::nothrow) t3ns_heff();
        if (!h) return set_error(T3NS_E_NOMEM, "host allocation");
        int r = create_impl(desc, precision, h);
        if (r != T3NS_OK) {
                t3ns_heff_destroy(h);
                return r;
        }
        *out = h;
        return T3NS_OK;
}

int t3ns_heff_matvec_device(t3ns_heff *h, const double *x, double *y, void *stream)
{
        if (!h || !x || !y) return set_error(T3NS_E_ARG, "null argument");
        return launch_heff(h->dp, h->precision, x, y, (cudaStream_t) stream, &h->last_launches);
}

int t3ns_heff_matvec_device_per_block(t3ns_heff *h, const double *x, double *y, void *stream)
{
        if (!h || !x || !y) return set_error(T3NS_E_ARG, "null argument");
        return launch_heff(h->dp, h->precision, x, y, (cudaStream_t) stream, &h->last_launches, true);
}

int t3ns_heff_matvec_host(t3ns_heff *h, const double *x, double *y)
{
        if (!h || !x || !y) return set_error(T3NS_E_ARG, "null argument");
        const size_t bytes = sizeof(double) * h->hp.size;
        T3NS_CUDA_TRY(cudaMemcpyAsync(h->stage_x, x, bytes, cudaMemcpyHostToDevice, h->stream));
        T3NS_TRY(launch_heff(h->dp, h->precision, h->stage_x, h->stage_y, h->stream,
                             &h->last_launches));
        T3NS_CUDA_TRY(cudaMemcpyAsync(y, h->stage_y, bytes, cudaMemcpyDeviceToHost, h->stream));
        T3NS_CUDA_TRY(cudaStreamSynchronize(h->stream));
        return check_device_error(h);
}

int t3ns_heff_check_status(t3ns_heff *h, void *stream)
{
        if (!h) return set_error(T3NS_E_ARG, "null plan");
        if (!stream) {
                // legacy default stream: every blocking stream has drained
                T3NS_CUDA_TRY(cudaStreamSynchronize(nullptr));
                return check_device_error(h);
        }
        return check_device_error(h, (cudaStream_t) stream);
}

int t3ns_heff_diagonal_device(t3ns_heff *h, double *diag, void *stream)
{
        if (!h || !diag) return set_error(T3NS_E_ARG, "null argument");
        return launch_heff_diag(h->dp, diag, (cudaStream_t) stream);
}

int t3ns_heff_diagonal_host(t3ns_heff *h, double *diag)
{
        if (!h || !diag) return set_error(T3NS_E_ARG, "null argument");
        T3NS_TRY(launch_heff_diag(h->dp, h->stage_y, h->stream));
        T3NS_CUDA_TRY(cudaMemcpyAsync(diag, h->stage_y, sizeof(double) * h->hp.size,
                                      cudaMemcpyDeviceToHost, h->stream));
        T3NS_CUDA_TRY(cudaStreamSynchronize(h->stream));
        return T3NS_OK;
}

int t3ns_heff_set_precision(t3ns_heff *h, int precision)
{
        if (!h) return set_error(T3NS_E_ARG, "null plan");
        return setup_precision(h, precision);
}

int t3ns_heff_set_config(t3ns_heff *h, int config)
{
        if (!h) return set_error(T3NS_E_ARG, "null plan");
        if (config < 0 || config >= kNumCfgs) return set_error(T3NS_E_ARG, "unknown configuration");
        if (!cfg_supports(config, h->precision))
                return set_error(T3NS_E_ARG, "configuration " + std::to_string(config) +
                                                     " does not run this precision "
                                                     "(3, 4: FP64 and 3xTF32; 5-7: BF16x3)");
        T3NS_TRY(upload_tiles(h, config));
        // the other modes (FP64 defect correction) run a BF16x3-only
        // configuration's launch shape in its FP64 twin
        if (kCfgs[config].bf16) T3NS_TRY(upload_tiles(h, config - kBfFirst));
        h->dp.active = config;
        return T3NS_OK;
}

int t3ns_heff_get_config(const t3ns_heff *h) { return h ? h->dp.active : -1; }

int t3ns_heff_autotune(t3ns_heff *h, int reps, int force, double *ms_out)
{
        if (!h) return set_error(T3NS_E_ARG, "null plan");
        if (ms_out)
                for (int c = 0; c < kNumCfgs; ++c) ms_out[c] = 0.0;
        const auto key = size_bucket(h->hp, h->precision);
        if (!force) {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                auto it = g_tune_cache.find(key);
                if (it != g_tune_cache.end()) return t3ns_heff_set_config(h, it->second);
        }
        reps = std::max(reps, 1);
        cudaEvent_t e0, e1;
        T3NS_CUDA_TRY(cudaEventCreate(&e0));
        T3NS_CUDA_TRY(cudaEventCreate(&e1));
        int best = h->dp.active;
        double best_ms = 0;
        int rc = T3NS_OK;
        bool first = true;
        for (int c = 0; c < kNumCfgs && rc == T3NS_OK; ++c) {
                if (!cfg_supports(c, h->precision)) continue;
                rc = t3ns_heff_set_config(h, c);
                if (rc != T3NS_OK) break;
                // one untimed run, then `reps` timed ones
                rc = launch_heff(h->dp, h->precision, h->stage_x, h->stage_y, h->stream, nullptr);
                std::vector<float> t;
                for (int r = 0; r < reps && rc == T3NS_OK; ++r) {
                        cudaEventRecord(e0, h->stream);
                        rc = launch_heff(h->dp, h->precision, h->stage_x, h->stage_y, h->stream,
                                         nullptr);
                        cudaEventRecord(e1, h->stream);
                        float ms = 0;
                        if (cudaEventSynchronize(e1) != cudaSuccess ||
                            cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
                                rc = set_error(T3NS_E_CUDA, "autotune: event timing failed");
                        t.push_back(ms);
                }
                if (rc != T3NS_OK) break;
                std::sort(t.begin(), t.end());
                const double med = t[t.size() / 2];
                if (ms_out) ms_out[c] = med;
                if (first || med < best_ms) {
                        best = c;
                        best_ms = med;
                        first = false;
                }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        T3NS_TRY(rc);
        T3NS_TRY(check_device_error(h));
        {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                g_tune_cache[key] = best;
        }
        return t3ns_heff_set_config(h, best);
}

int t3ns_heff_get_stats(const t3ns_heff *h, t3ns_heff_stats *st)
{
        if (!h || !st) return set_error(T3NS_E_ARG, "null argument");
        st->size = h->hp.size;
        st->nblocks = h->hp.nblocks;
        st->npairs = h->hp.npairs;
        st->ntasks = (int64_t) h->hp.tasks.size();
        st->flops_ref = h->hp.flops_ref;
        st->flops_exec = h->hp.tiles[h->dp.active].flops_exec;
        st->bytes_alg = h->hp.bytes_alg;
        st->op_elems = h->hp.op_elems;
        st->scratch_bytes = 0;
        return T3NS_OK;
}

int t3ns_heff_last_launches(const t3ns_heff *h) { return h ? h->last_launches : 0; }

void t3ns_heff_destroy(t3ns_heff *h)
{
        if (!h) return;
        if (h->stream) cudaStreamDestroy(h->stream);
        for (void *p : h->allocs) cudaFree(p);
        delete h;
}

int t3ns_heff_plan_dump(const t3ns_heff_desc *desc, const char *path)
{
        return t3ns_heff_plan_dump_config(desc, 0, path);
}

int t3ns_heff_plan_dump_config(const t3ns_heff_desc *desc, int config, const char *path)
{
        HostPlan hp;
        T3NS_TRY(build_plan(desc, hp));
        if (config < 0 || config >= kNumCfgs) return set_error(T3NS_E_ARG, "unknown configuration");
        T3NS_TRY(tile_plan(hp, config));
        FILE *f = fopen(path, "wb");
        if (!f) return set_error(T3NS_E_ARG, std::string("cannot open ") + path);
        auto put = [&](const char *name, int dtype, int64_t n, const void *a) {
                char nm[48] = {0};
                strncpy(nm, name, sizeof nm - 1);
                int32_t hdr[2] = {dtype, 0};
                fwrite(nm, 1, sizeof nm, f);
                fwrite(hdr, sizeof hdr, 1, f);
                fwrite(&n, sizeof n, 1, f);
                if (n) fwrite(a, dtype == 1 ? 4 : 8, (size_t) n, f);
        };
        fwrite("T3NSCAP1", 1, 8, f);
        std::vector<int> units, pairs, edims;
        const TilePlan &tp = hp.tiles[config];
        for (auto &u : tp.units) { units.insert(units.end(), {u.nb, u.b0, u.bt, u.c0, u.ct, u.a0, u.at, u.p0, u.p1, u.split}); }
        for (auto &p : tp.pairs) { pairs.insert(pairs.end(), {p.old, p.axes, p.t0, p.t1}); }
        for (auto &e : hp.edims) { edims.insert(edims.end(), {e.x, e.y, e.z}); }
        std::vector<int64_t> offs;
        std::vector<double> prefs;
        for (auto &t : hp.tasks) {
                offs.insert(offs.end(), {t.op_off[0], t.op_off[1], t.op_off[2]});
                prefs.push_back(t.pref);
        }
        put("plan.units", 1, (int64_t) units.size(), units.data());
        put("plan.pairs", 1, (int64_t) pairs.size(), pairs.data());
        put("plan.pair_ptr", 1, (int64_t) tp.pair_ptr.size(), tp.pair_ptr.data());
        put("plan.edims", 1, (int64_t) edims.size(), edims.data());
        put("plan.op_off", 2, (int64_t) offs.size(), offs.data());
        put("plan.pref", 3, (int64_t) prefs.size(), prefs.data());
        put("plan.flops", 3, 2, std::vector<double>{hp.flops_ref, tp.flops_exec}.data());
        put("plan.tjobs", 2, (int64_t) hp.tjobs.size(), hp.tjobs.data());
        put("plan.toff", 2, (int64_t) hp.toff.size(), hp.toff.data());
        put("plan.elems", 2, 2, std::vector<int64_t>{hp.op_elems, hp.opt_elems}.data());
        fclose(f);
        return T3NS_OK;
}

const char *t3ns_last_error(void) { return g_last_error.c_str(); }

const char *t3ns_version(void) { return "t3ns_b200 0.1 (sm_100a)"; }

}  // extern "C"
