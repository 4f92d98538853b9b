/*
 * engine.cu -- the batched encode engine behind include/h261b.h.
 *
 * Memory: every open session owns two reconstruction pictures in HBM (they
 * alternate as reference and output) and its denoise state, taken from a
 * size-class slab pool so that opening a session in steady state does not
 * call cudaMalloc.  Queued source pictures sit in a pinned upload arena
 * (copied there by h261b_session_submit, or written there directly by the
 * caller through h261b_session_input); a step moves the whole arena with
 * one copy, runs one launch over the flat (session, MB) work list, and
 * brings the compact results of all sessions back with one copy.
 *
 * Pipelining: steps rotate over NSLOT (3) slots, each with its CUDA stream
 * and its set of arenas.  Within a step the order is upload -> kernel ->
 * download; across steps only the kernels are ordered (step k+1's kernel
 * waits for step k's, whose reconstructions are its references), so step
 * k+1's upload overlaps step k's kernel and step k's download overlaps step
 * k+1's kernel.  Results of step k stay readable until step k+3 is issued,
 * so a caller can issue step k+1 while it has still to read step k-1.
 *
 * Tuning: when warps_per_cta is 0 the first steps try each launch shape on
 * live work (the results do not depend on it) and keep the fastest by CUDA
 * event time.
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "common.h"
#include "copy_pool.h"
#include "h261b_device.h"

namespace h261b {

/* steps in flight at once: step id uses slot id % NSLOT (its stream,
 * arenas, events and graph), so the host can issue a step while the two
 * before it still run and their results are still readable */
constexpr int NSLOT = 3;

static thread_local char g_err[512];

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

void clear_error() { g_err[0] = 0; }

/* ---------------------------------------------------------------- pool */

/* slabs of equal-size device blocks, one slab list per block size */
class DevicePool {
  public:
    ~DevicePool()
    {
        for (void *p : slabs_)
            cudaFree(p);
    }
    int get(size_t bytes, void **out)
    {
        bytes = align_up(bytes, 256);
        auto &fl = free_[bytes];
        if (fl.empty()) {
            const size_t per = std::max<size_t>(1, (size_t)(64u << 20) / bytes);
            void *slab = nullptr;
            cudaError_t err = cudaMalloc(&slab, per * bytes);
            if (err != cudaSuccess) {
                set_error("device pool: cudaMalloc(%zu) failed: %s", per * bytes, cudaGetErrorString(err));
                return H261B_ERR_NOMEM;
            }
            slabs_.push_back(slab);
            held_ += per * bytes;
            for (size_t i = 0; i < per; i++)
                fl.push_back((char *)slab + i * bytes);
        }
        *out = fl.back();
        fl.pop_back();
        return H261B_OK;
    }
    void put(size_t bytes, void *p) { free_[align_up(bytes, 256)].push_back(p); }
    /* at least `count` free blocks of this size, in slabs of up to 1 GiB */
    int reserve(size_t bytes, size_t count)
    {
        bytes = align_up(bytes, 256);
        auto &fl = free_[bytes];
        while (fl.size() < count) {
            const size_t per = std::max<size_t>(1, std::min<size_t>(count - fl.size(), (size_t)(1u << 30) / bytes));
            void *slab = nullptr;
            cudaError_t err = cudaMalloc(&slab, per * bytes);
            if (err != cudaSuccess) {
                set_error("device pool: cudaMalloc(%zu) failed: %s", per * bytes, cudaGetErrorString(err));
                return H261B_ERR_NOMEM;
            }
            slabs_.push_back(slab);
            held_ += per * bytes;
            for (size_t i = 0; i < per; i++)
                fl.push_back((char *)slab + i * bytes);
        }
        return H261B_OK;
    }
    int64_t held() const { return (int64_t)held_; }

  private:
    std::map<size_t, std::vector<void *>> free_;
    std::vector<void *> slabs_;
    size_t held_ = 0;
};

/* pinned host + device buffer pair of one capacity */
struct Mirror {
    uint8_t *host = nullptr;
    uint8_t *dev = nullptr;
    size_t cap = 0;
    /* grow to at least `bytes`; the first `keep` host bytes survive */
    int reserve(size_t bytes, size_t keep = 0)
    {
        if (bytes <= cap)
            return H261B_OK;
        /* doubling: a growing session count reallocates (and syncs) only a
         * few times */
        size_t c = align_up(std::max<size_t>(std::max<size_t>(bytes, 1 << 20), 2 * cap), 4096);
        uint8_t *nh = nullptr, *nd = nullptr;
        cudaError_t e1 = cudaMallocHost(&nh, c);
        cudaError_t e2 = cudaMalloc(&nd, c);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            set_error("arena allocation of %zu bytes failed", c);
            if (nh)
                cudaFreeHost(nh);
            if (nd)
                cudaFree(nd);
            return H261B_ERR_NOMEM;
        }
        if (keep && host)
            memcpy(nh, host, std::min(keep, cap));
        release();
        host = nh;
        dev = nd;
        cap = c;
        return H261B_OK;
    }
    void release()
    {
        if (host)
            cudaFreeHost(host);
        if (dev)
            cudaFree(dev);
        host = dev = nullptr;
        cap = 0;
    }
};

/* everything about a step's launches that a captured graph bakes in */
struct StepKey {
    const void *dm_host, *dm_dev, *um_host, *um_dev, *rm_host, *rm_dev, *bits_dev;
    size_t bits_cap, desc_off, work_off, desc_bytes, upload_bytes, ssd_base, d2h;
    int64_t n;
    int32_t n_work, rc_begin, n_rc, ssd, warps, ctas, phases, waits;
    bool operator==(const StepKey &o) const { return memcmp(this, &o, sizeof(StepKey)) == 0; }
};

struct StepGraph {
    cudaGraphExec_t exec = nullptr;
    StepKey key;
    /* the signature of the last step launched directly on this slot: a
     * graph is captured only for a signature seen twice in a row, so that
     * steps whose sessions keep changing (one stream at a time, serving)
     * do not pay a capture each */
    StepKey last_direct;
    bool has_last_direct = false;
    void reset()
    {
        if (exec)
            cudaGraphExecDestroy(exec);
        exec = nullptr;
    }
};

/* where one step left a session's results */
struct Result {
    int64_t step = -1;
    int32_t frame = 0, type = 0, quant = 0;
    size_t info_off = 0, level_off = 0;
    size_t pic_off = 0;            /* h261b_pic_info_t of a bitstream session */
    bool has_bits = false;
    size_t ssd_off = 0;            /* three uint64 squared-error sums        */
    bool has_ssd = false;
};

/* pinned host memory the device writes into (mapped) */
struct HostArena {
    uint8_t *host = nullptr;
    uint8_t *dev = nullptr;
    size_t cap = 0;
    int reserve(size_t bytes)
    {
        if (bytes <= cap)
            return H261B_OK;
        release();
        uint8_t *h = nullptr;
        void *d = nullptr;
        cudaError_t err = cudaHostAlloc(&h, bytes, cudaHostAllocMapped);
        if (err == cudaSuccess)
            err = cudaHostGetDevicePointer(&d, h, 0);
        if (err != cudaSuccess) {
            if (h)
                cudaFreeHost(h);
            set_error("host bitstream arena of %zu bytes: %s", bytes, cudaGetErrorString(err));
            return H261B_ERR_NOMEM;
        }
        host = h;
        dev = (uint8_t *)d;
        cap = bytes;
        return H261B_OK;
    }
    void release()
    {
        if (host)
            cudaFreeHost(host);
        host = dev = nullptr;
        cap = 0;
    }
};

struct Session {
    bool open = false;
    int32_t w = 0, h = 0, mbw = 0, mbh = 0, nmb = 0;
    int32_t quant = 8, intra_period = 0;
    int32_t frame_index = 0;       /* next picture number                 */
    PictureLayout lay;
    uint8_t *rec[2] = { nullptr, nullptr };
    int rec_cur = 0;               /* holds the latest reconstruction     */
    h261b_denoise_dev_t *dn = nullptr;
    size_t slot_bytes = 0;
    /* bitstream: one device block per step slot (picture, MB scratch,
     * positions, header plans, picture size) */
    bool bitstream = false;
    uint8_t *bits_base[NSLOT] = {};
    h261b_bits_layout_t bits_lay = {};
    std::vector<uint8_t> bits_spill;   /* a picture the host arena missed */
    /* CBR rate control: its state and the mode decisions between the two
     * encode launches of a step */
    bool psnr = false;
    bool rc = false;
    h261b_rc_dev_t *rc_dev = nullptr;
    h261_mb_mode_decision_t *md_dev = nullptr;
    /* queued picture: in the upload arena, or already in device memory */
    bool queued = false;
    size_t src_off = 0;
    const uint8_t *dev_src[3] = { nullptr, nullptr, nullptr };
    int32_t queued_quant = 0;
    Result res[NSLOT];             /* by step slot                        */
};

/* how the encode kernel is launched: the knobs of h261b_engine_config_t */
/* The defaults are the plan measured fastest on the batch64 workload; the
 * tuner keeps them unless a candidate is clearly faster on the device at
 * hand. */
struct LaunchPlan {
    int32_t warps = 8;      /* warps per CTA                                 */
    int32_t ctas = 0;       /* grid cap, 0 = one wave of resident CTAs       */
    int32_t split = 0;      /* 0 one fused kernel, 1 search + encode kernels */
    int32_t tail = 0;       /* items per warp drawn one at a time            */
    int32_t staging = 0;    /* 0 16-byte cp.async, 1 bulk row copies         */
    bool operator==(const LaunchPlan &o) const
    {
        return warps == o.warps && ctas == o.ctas && split == o.split && tail == o.tail && staging == o.staging;
    }
    /* the phases-word bits of h261b_launch_step for this plan */
    int32_t bits() const
    {
        return ((tail + 1) << H261B_TAIL_SHIFT) | (staging ? H261B_STAGE_BULK : 0);
    }
};

/* Tuning on live steps: each stage's candidates run on the engine's next
 * mostly-inter steps (at least half of the step's MBs from inter pictures,
 * whose search dominates), every candidate three times in round-robin
 * order.  A stage keeps its incumbent (candidate 0: the default plan, then
 * stage 1's winner) unless another candidate's median CUDA-event time is at
 * least 3 % below the incumbent's: successive live steps differ by a few per
 * cent in content, and a single lucky step must not move the plan.  Stage 1
 * tries the CTA widths of the fused kernel and of the split kernels; stage 2
 * tries the tail length and the staging variant on the winner. */
struct Tuner {
    static constexpr int kRounds = 3;
    static constexpr float kMargin = 0.97f;
    std::vector<LaunchPlan> cands;
    std::vector<std::vector<float>> ms;   /* per candidate, its rounds' times */
    size_t next = 0;          /* index into cands x kRounds                */
    int stage = 0;            /* 1, 2 while tuning; 0 idle                  */
    /* every candidate measured (plan, ms), for h261b_engine_tuning */
    std::vector<std::pair<LaunchPlan, float>> log;
    bool active() const { return stage != 0 && next < cands.size() * kRounds; }
    const LaunchPlan &current() const { return cands[next % cands.size()]; }
};

} // namespace h261b

using namespace h261b;

struct h261b_engine_s {
    h261b_engine_config_t cfg;
    int sm_count = 0;
    cudaStream_t stream[NSLOT] = {};
    /* per slot: a side stream that records the events marking the encode
     * kernel's end, so that nothing sits between the encode kernel and the
     * bitstream kernel that depends on it (a programmatic dependent launch) */
    cudaStream_t side[NSLOT] = {};
    cudaEvent_t fork_ev[NSLOT] = {}, join_ev[NSLOT] = {};
    DevicePool pool;
    std::vector<Session> sessions;
    int32_t open_count = 0;
    int64_t session_bytes = 0;

    Mirror upload[NSLOT];      /* queued source pictures                  */
    Mirror results[NSLOT];     /* mb info + levels of every session        */
    Mirror desc[NSLOT];        /* session descriptors + work list           */
    size_t upload_used = 0;    /* bytes queued for the next step           */
    bool upload_checked = false;
    int64_t next_step = 0;     /* id of the next step; slot = id % NSLOT    */
    int64_t done_step = -1;    /* every step up to this one has completed   */
    cudaEvent_t h2d_done[NSLOT] = {};
    cudaEvent_t kernel_done[NSLOT] = {};
    cudaEvent_t step_done[NSLOT] = {};
    cudaEvent_t k_start[NSLOT] = {}, k_end[NSLOT] = {};
    cudaEvent_t b_end[NSLOT] = {};         /* after the bitstream kernel */
    cudaEvent_t layout_done[NSLOT] = {};   /* rate control inputs written */
    /* timing of each phase of a step: begin, uploads done, kernels may
     * start (the previous step's encode is done), results downloaded */
    cudaEvent_t t_begin[NSLOT] = {}, t_h2d[NSLOT] = {};
    cudaEvent_t t_ready[NSLOT] = {}, t_end[NSLOT] = {};
    /* step arena bytes asked for by h261b_engine_reserve_step */
    size_t reserved_upload = 0, reserved_results = 0, reserved_desc = 0;
    /* the encode launches' work counters, two per stream (h261b_launch_step) */
    int32_t *sched_dev = nullptr;
    bool step_bits_ran[NSLOT] = {};
    bool in_flight[NSLOT] = {};
    int64_t step_mbs[NSLOT] = {};   /* MB records of the step in each arena */
    int64_t last_h2d = 0, last_d2h = 0;  /* bytes copied by the last step */
    HostArena bits[NSLOT];     /* pictures written by the bitstream kernel */
    size_t bits_want = 0;      /* capacity the arenas grow to              */
    /* slots of closed sessions, returned to the pool once the last step
     * that may use them (second field) has completed */
    struct Retired {
        void *block;
        size_t bytes;
        int64_t last_step;
    };
    std::vector<Retired> retired;
    std::unique_ptr<CopyPool> copier;   /* batched submissions */
    std::vector<CopyJob> copy_jobs;

    /* graph replay of steps (use_graphs) */
    StepGraph graph[NSLOT];
    bool graphs_off = false;
    int64_t graph_captures = 0, graph_replays = 0;

    /* phases-word bits the checking build adds for its tests (0 otherwise) */
    int32_t test_bits = 0;
    int32_t test_codes_extra = 0;   /* checking build: the codes wait's test */
    /* the encode kernel's launch plan, and its tuning */
    LaunchPlan plan;
    Tuner tuner;
    bool tuned = false;
    int shape_source = 0;   /* 0 configured, 1 tuned here, 2 tuned earlier in this process */
};

/* the launch plan tuning chose, per device, for the engines created after
 * it in this process */
static std::mutex g_tuned_mu;
static std::map<int, LaunchPlan> g_tuned;

static const char *k_version = "h261b 0.2 (sm_100a)";

extern "C" const char *h261b_last_error(void) { return g_err; }
extern "C" const char *h261b_version(void) { return k_version; }

extern "C" void h261b_engine_config_default(h261b_engine_config_t *c)
{
    memset(c, 0, sizeof(*c));
    c->device = 0;
    c->max_sessions = 4096;
    c->hbm_budget_bytes = 0;
    c->me_mode = H261B_ME_REFERENCE;
    c->fmad = 1;
    c->warps_per_cta = 0;
    c->max_ctas = 0;
    c->copy_threads = 0;
    c->levels_to_host = 1;
    c->bits_host_bytes = 0;
    c->use_graphs = 1;
}

extern "C" int64_t h261b_session_bytes(int32_t w, int32_t h)
{
    if (w < 16 || h < 16 || (w & 15) || (h & 15))
        return -1;
    return (int64_t)(2 * PictureLayout::of(w, h).bytes + align_up(sizeof(h261b_denoise_dev_t), 256));
}

extern "C" int64_t h261b_session_bits_bytes(int32_t w, int32_t h)
{
    return NSLOT * (int64_t)align_up((size_t)h261b_bits_slot_bytes(w, h), 256);
}

/* rate-control state and one picture's mode decisions */
static int64_t rc_bytes(int32_t w, int32_t h)
{
    return 256 + (int64_t)align_up((size_t)(w / 16) * (h / 16) * sizeof(h261_mb_mode_decision_t), 256);
}

static bool session_config_ok(const h261b_session_config_t *c)
{
    return c && c->width >= 16 && c->height >= 16 && !(c->width & 15) && !(c->height & 15) &&
           (c->width / 16) * (c->height / 16) <= H261B_MAX_MB_PER_SESSION && c->quant >= 1 && c->quant <= 31 &&
           c->intra_period >= 0 && c->denoise >= 0 && (c->bitstream == 0 || c->bitstream == 1) &&
           (c->psnr == 0 || c->psnr == 1) &&
           (c->rate_control == 0 || (c->rate_control == 1 && c->bitstream == 1 && c->bitrate >= 8));
}

extern "C" int64_t h261b_session_config_bytes(const h261b_session_config_t *c)
{
    if (!session_config_ok(c))
        return H261B_ERR_ARG;
    const int64_t bits = c->bitstream ? h261b_session_bits_bytes(c->width, c->height) : 0;
    if (c->bitstream && bits == 0)
        return H261B_ERR_ARG;
    return h261b_session_bytes(c->width, c->height) + bits + (c->rate_control ? rc_bytes(c->width, c->height) : 0);
}

/* return retired session slots whose last step has completed */
static void reclaim(h261b_engine_t *e)
{
    size_t k = 0;
    for (size_t i = 0; i < e->retired.size(); i++) {
        if (e->retired[i].last_step <= e->done_step)
            e->pool.put(e->retired[i].bytes, e->retired[i].block);
        else
            e->retired[k++] = e->retired[i];
    }
    e->retired.resize(k);
}

static int sync_all(h261b_engine_t *e)
{
    for (int p = 0; p < NSLOT; p++)
        H261B_CUDA_TRY(cudaStreamSynchronize(e->stream[p]));
    e->done_step = e->next_step - 1;
    reclaim(e);
    return H261B_OK;
}

/* stage 1: CTA widths of the fused kernel and of the split kernels, for
 * the knobs the configuration leaves open */
static void tuner_stage1(h261b_engine_t *e)
{
    const h261b_engine_config_t &c = e->cfg;
    Tuner &t = e->tuner;
    t.cands.clear();
    /* candidate 0: the engine's plan (defaults and configured knobs) */
    t.cands.push_back(e->plan);
    for (int split = 0; split < 2; split++) {
        if (c.kernel_split > 0 && split != c.kernel_split - 1)
            continue;
        const int widths_fused[3] = { 2, 4, 8 }, widths_split[2] = { 4, 8 };
        const int *wl = split ? widths_split : widths_fused;
        const int nw = split ? 2 : 3;
        for (int i = 0; i < nw; i++) {
            if (c.warps_per_cta > 0 && wl[i] != c.warps_per_cta)
                continue;
            LaunchPlan p = e->plan;
            p.split = split;
            p.warps = wl[i];
            if (!(p == t.cands[0]))
                t.cands.push_back(p);
        }
    }
    t.ms.assign(t.cands.size(), std::vector<float>());
    t.next = 0;
    t.stage = 1;
}

/* stage 2: the tail length and the staging variant on stage 1's winner */
static void tuner_stage2(h261b_engine_t *e, const LaunchPlan &w)
{
    const h261b_engine_config_t &c = e->cfg;
    Tuner &t = e->tuner;
    t.cands.assign(1, w);
    if (c.tail_items == 0)
        for (int tail : { 0, 2, 4 }) {
            if (tail == w.tail)
                continue;
            LaunchPlan p = w;
            p.tail = tail;
            t.cands.push_back(p);
        }
    if (c.staging == 0) {
        LaunchPlan p = w;
        p.staging = 1 - w.staging;
        t.cands.push_back(p);
    }
    t.ms.assign(t.cands.size(), std::vector<float>());
    t.next = 0;
    t.stage = 2;
}

/* record a tuning step's time; move to the next stage or finish */
static void tuner_record(h261b_engine_t *e, float ms)
{
    Tuner &t = e->tuner;
    const size_t i = t.next % t.cands.size();
    t.log.push_back({ t.cands[i], ms });
    t.ms[i].push_back(ms);
    t.next++;
    if (t.next < t.cands.size() * Tuner::kRounds)
        return;
    auto median = [](std::vector<float> v) {
        std::sort(v.begin(), v.end());
        return v[v.size() / 2];
    };
    /* the incumbent (candidate 0) unless a candidate is clearly faster */
    size_t best = 0;
    float best_ms = median(t.ms[0]);
    const float bar = best_ms * Tuner::kMargin;
    for (size_t k = 1; k < t.cands.size(); k++) {
        const float m = median(t.ms[k]);
        if (m < bar && m < best_ms) {
            best = k;
            best_ms = m;
        }
    }
    const LaunchPlan w = t.cands[best];
    if (t.stage == 1 && t.cands.size() >= 1 && (e->cfg.tail_items == 0 || e->cfg.staging == 0)) {
        tuner_stage2(e, w);
        if (t.cands.size() > 1)
            return;
    }
    e->plan = w;
    e->tuned = true;
    e->shape_source = 1;
    t.stage = 0;
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    g_tuned[e->cfg.device] = w;
}

extern "C" int h261b_engine_create(const h261b_engine_config_t *cfg, h261b_engine_t **out)
{
    clear_error();
    if (!cfg || !out || cfg->max_sessions < 1 || cfg->max_sessions > 65536 || cfg->warps_per_cta < 0 ||
        cfg->warps_per_cta > 8 || (cfg->me_mode != 0 && cfg->me_mode != 1) || cfg->copy_threads < 0 ||
        cfg->copy_threads > 64 || cfg->bits_host_bytes < 0 || (cfg->levels_to_host != 0 && cfg->levels_to_host != 1) ||
        cfg->kernel_split < 0 || cfg->kernel_split > 2 || cfg->tail_items < 0 || cfg->tail_items > 15 ||
        cfg->staging < 0 || cfg->staging > 2) {
        set_error("h261b_engine_create: bad configuration");
        return H261B_ERR_ARG;
    }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || cfg->device < 0 || cfg->device >= ndev) {
        set_error("h261b_engine_create: CUDA device %d not available", cfg->device);
        return H261B_ERR_NO_DEVICE;
    }
    H261B_CUDA_TRY(cudaSetDevice(cfg->device));
    h261b_engine_t *e = new h261b_engine_s();
    e->cfg = *cfg;
    e->sessions.resize((size_t)cfg->max_sessions);
    e->bits_want = cfg->bits_host_bytes > 0 ? align_up((size_t)cfg->bits_host_bytes, 4096) : (size_t)8 << 20;
    int copiers = cfg->copy_threads;
    if (copiers == 0)
        copiers = std::max(1, std::min(8, (int)std::thread::hardware_concurrency() / 2));
    e->copier.reset(new CopyPool(copiers - 1));   /* the caller is one of them */
    cudaDeviceProp prop;
    bool ok = cudaGetDeviceProperties(&prop, cfg->device) == cudaSuccess && h261b_set_quant_table() == 0;
    for (int p = 0; p < NSLOT && ok; p++) {
        ok = cudaStreamCreateWithFlags(&e->stream[p], cudaStreamNonBlocking) == cudaSuccess &&
             cudaStreamCreateWithFlags(&e->side[p], cudaStreamNonBlocking) == cudaSuccess &&
             cudaEventCreateWithFlags(&e->fork_ev[p], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&e->join_ev[p], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&e->h2d_done[p], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&e->kernel_done[p], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreateWithFlags(&e->step_done[p], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreate(&e->k_start[p]) == cudaSuccess && cudaEventCreate(&e->k_end[p]) == cudaSuccess &&
             cudaEventCreate(&e->b_end[p]) == cudaSuccess && cudaEventCreate(&e->t_begin[p]) == cudaSuccess &&
             cudaEventCreateWithFlags(&e->layout_done[p], cudaEventDisableTiming) == cudaSuccess &&
             cudaEventCreate(&e->t_h2d[p]) == cudaSuccess && cudaEventCreate(&e->t_ready[p]) == cudaSuccess &&
             cudaEventCreate(&e->t_end[p]) == cudaSuccess;
    }
    ok = ok && cudaMalloc(&e->sched_dev, 2 * NSLOT * sizeof(int32_t)) == cudaSuccess &&
         cudaMemset(e->sched_dev, 0, 2 * NSLOT * sizeof(int32_t)) == cudaSuccess;
    if (!ok) {
        set_error("h261b_engine_create: device setup failed: %s", cudaGetErrorString(cudaGetLastError()));
        h261b_engine_destroy(e);
        return H261B_ERR_CUDA;
    }
    e->sm_count = prop.multiProcessorCount;
    if (cfg->bits_host_bytes > 0) {
        /* a configured host bitstream arena is allocated now, not by the
         * first steps */
        for (int p = 0; p < NSLOT; p++)
            if (e->bits[p].reserve(e->bits_want) != H261B_OK) {
                h261b_engine_destroy(e);
                return H261B_ERR_NOMEM;
            }
    }
    /* the launch plan: configured knobs are fixed; the others come from an
     * earlier tuning on this device in this process, or are tuned on this
     * engine's first mostly-inter steps */
    LaunchPlan &pl = e->plan;
    pl.ctas = cfg->max_ctas;
    if (cfg->warps_per_cta > 0)
        pl.warps = cfg->warps_per_cta;
    if (cfg->kernel_split > 0)
        pl.split = cfg->kernel_split - 1;
    if (cfg->tail_items > 0)
        pl.tail = cfg->tail_items - 1;
    if (cfg->staging > 0)
        pl.staging = cfg->staging - 1;
    const bool all_set = cfg->warps_per_cta > 0 && cfg->kernel_split > 0 && cfg->tail_items > 0 && cfg->staging > 0;
    if (all_set) {
        e->tuned = true;
    } else {
        std::lock_guard<std::mutex> lk(g_tuned_mu);
        auto it = g_tuned.find(cfg->device);
        if (it != g_tuned.end()) {
            /* a tuned plan for the knobs left open */
            const LaunchPlan &t = it->second;
            if (cfg->warps_per_cta == 0)
                pl.warps = t.warps;
            if (cfg->kernel_split == 0)
                pl.split = t.split;
            if (cfg->tail_items == 0)
                pl.tail = t.tail;
            if (cfg->staging == 0)
                pl.staging = t.staging;
            e->tuned = true;
            e->shape_source = 2;
        }
    }
    if (!e->tuned)
        tuner_stage1(e);
#ifdef H261B_DEBUG_CHECKS
    /* the checking build's test of the bounded staging wait: every warp's
     * first bulk staging announces more bytes than it copies */
    if (getenv("H261B_TEST_STAGE_SHORT"))
        e->test_bits |= H261B_STAGE_SHORT;
    /* and of the codes kernel's bounded wait for a picture's MBs */
    if (getenv("H261B_TEST_CODES_WAIT"))
        e->test_codes_extra = 1;
#endif
    *out = e;
    return H261B_OK;
}

extern "C" int h261b_engine_destroy(h261b_engine_t *e)
{
    if (!e)
        return H261B_OK;
    cudaSetDevice(e->cfg.device);
    if (e->copier)
        e->copier->join();
    for (int p = 0; p < NSLOT; p++)
        if (e->stream[p])
            cudaStreamSynchronize(e->stream[p]);
    for (int p = 0; p < NSLOT; p++) {
        e->graph[p].reset();
        e->upload[p].release();
        e->results[p].release();
        e->desc[p].release();
        e->bits[p].release();
        cudaEventDestroy(e->h2d_done[p]);
        cudaEventDestroy(e->kernel_done[p]);
        cudaEventDestroy(e->step_done[p]);
        cudaEventDestroy(e->k_start[p]);
        cudaEventDestroy(e->k_end[p]);
        cudaEventDestroy(e->b_end[p]);
        cudaEventDestroy(e->layout_done[p]);
        cudaEventDestroy(e->t_begin[p]);
        cudaEventDestroy(e->t_h2d[p]);
        cudaEventDestroy(e->t_ready[p]);
        cudaEventDestroy(e->t_end[p]);
        if (e->stream[p])
            cudaStreamDestroy(e->stream[p]);
        if (e->side[p])
            cudaStreamDestroy(e->side[p]);
        cudaEventDestroy(e->fork_ev[p]);
        cudaEventDestroy(e->join_ev[p]);
    }
    if (e->sched_dev)
        cudaFree(e->sched_dev);
    delete e;
    return H261B_OK;
}

static Session *get_session(h261b_engine_t *e, int32_t id)
{
    if (!e || id < 0 || id >= (int32_t)e->sessions.size() || !e->sessions[(size_t)id].open) {
        set_error("invalid session id %d", id);
        return nullptr;
    }
    return &e->sessions[(size_t)id];
}

extern "C" int h261b_session_open(h261b_engine_t *e, const h261b_session_config_t *c, int32_t *id)
{
    clear_error();
    if (!e || !id || !session_config_ok(c)) {
        set_error("h261b_session_open: bad session configuration%s",
                  c && c->rate_control ? " (rate control needs bitstream = 1 and a bitrate)" : "");
        return H261B_ERR_ARG;
    }
    const int64_t bits_need = c->bitstream ? h261b_session_bits_bytes(c->width, c->height) : 0;
    if (c->bitstream && bits_need == 0) {
        set_error("h261b_session_open: H.261 bitstreams exist for 176x144 and 352x288 only, not %dx%d",
                  c->width, c->height);
        return H261B_ERR_ARG;
    }
    const int64_t need = h261b_session_config_bytes(c);
    if (e->cfg.hbm_budget_bytes > 0 && e->session_bytes + need > e->cfg.hbm_budget_bytes) {
        set_error("h261b_session_open: HBM budget %lld exceeded", (long long)e->cfg.hbm_budget_bytes);
        return H261B_ERR_BUDGET;
    }
    int32_t slot = -1;
    for (size_t i = 0; i < e->sessions.size(); i++)
        if (!e->sessions[i].open) {
            slot = (int32_t)i;
            break;
        }
    if (slot < 0) {
        set_error("h261b_session_open: all %d session slots in use", e->cfg.max_sessions);
        return H261B_ERR_BUDGET;
    }
    cudaSetDevice(e->cfg.device);
    reclaim(e);
    void *blk = nullptr;
    int rc = e->pool.get((size_t)need, &blk);
    if (rc != H261B_OK)
        return rc;
    Session &s = e->sessions[(size_t)slot];
    s = Session();
    s.w = c->width;
    s.h = c->height;
    s.mbw = c->width / 16;
    s.mbh = c->height / 16;
    s.nmb = s.mbw * s.mbh;
    s.quant = c->quant;
    s.intra_period = c->intra_period;
    s.psnr = c->psnr != 0;
    s.lay = PictureLayout::of(s.w, s.h);
    s.slot_bytes = (size_t)need;
    uint8_t *base = (uint8_t *)blk;
    s.rec[0] = base;
    s.rec[1] = base + s.lay.bytes;
    s.dn = (h261b_denoise_dev_t *)(base + 2 * s.lay.bytes);
    if (c->bitstream) {
        const size_t sb = align_up((size_t)h261b_bits_slot_bytes(c->width, c->height), 256);
        uint8_t *b0 = base + h261b_session_bytes(c->width, c->height);
        s.bitstream = true;
        s.bits_lay = h261b_bits_layout(c->width, c->height);
        for (int q = 0; q < NSLOT; q++)
            s.bits_base[q] = b0 + q * sb;
    }
    h261b_rc_dev_t rc0;
    if (c->rate_control) {
        uint8_t *r0 = base + h261b_session_bytes(c->width, c->height) + bits_need;
        s.rc = true;
        s.rc_dev = (h261b_rc_dev_t *)r0;
        s.md_dev = (h261_mb_mode_decision_t *)(r0 + 256);
        /* h261_init_ratectrl(ctx, quant, bitrate, bitrate, CBR)
         * (src/h261_ratectrl.c:107-127) */
        memset(&rc0, 0, sizeof(rc0));
        rc0.current_quant = c->quant;
        rc0.prediction_cost[0] = rc0.prediction_cost[1] = 100;
        rc0.prediction_size[0] = rc0.prediction_size[1] = 1;
        rc0.bitrate = c->bitrate / 8;
        rc0.vbv_size = c->bitrate / 8;
        rc0.vbv_fill = rc0.vbv_size;
        rc0.picture_quant = c->quant;
    }
    /* the first reference is black like the reference's zeroed frame
     * (h261_main.c:155-157); denoise state starts at zero
     * (gpu_device.cu:495-508).  No step in flight touches this slot (a
     * closed slot returns to the pool only after its last step), and the
     * clearing goes on the stream of the next step: every later step waits
     * for that one's kernel, so none can read the slot before it is clear.
     * The pageable source of the state copy is staged before the call
     * returns. */
    h261b_denoise_dev_t dn0;
    memset(&dn0, 0, sizeof(dn0));
    dn0.denoise = c->denoise;
    cudaStream_t st = e->stream[e->next_step % NSLOT];
    H261B_CUDA_TRY(cudaMemsetAsync(base, 0, 2 * s.lay.bytes, st));
    for (int q = 0; q < NSLOT && s.bitstream; q++)
        H261B_CUDA_TRY(cudaMemsetAsync(s.bits_base[q] + s.bits_lay.total, 0, 256, st));
    if (s.rc)
        H261B_CUDA_TRY(cudaMemcpyAsync(s.rc_dev, &rc0, sizeof(rc0), cudaMemcpyHostToDevice, st));
    H261B_CUDA_TRY(cudaMemcpyAsync(s.dn, &dn0, sizeof(dn0), cudaMemcpyHostToDevice, st));
    s.open = true;
    e->open_count++;
    e->session_bytes += need;
    *id = slot;
    return H261B_OK;
}

extern "C" int h261b_engine_reserve(h261b_engine_t *e, const h261b_session_config_t *c, int32_t count)
{
    clear_error();
    if (!e || count < 0 || !session_config_ok(c)) {
        set_error("h261b_engine_reserve: bad arguments");
        return H261B_ERR_ARG;
    }
    const int64_t need = h261b_session_config_bytes(c);
    if (need <= 0) {
        set_error("h261b_engine_reserve: bad session configuration");
        return H261B_ERR_ARG;
    }
    cudaSetDevice(e->cfg.device);
    return e->pool.reserve((size_t)need, (size_t)count);
}

static int grow_arenas(h261b_engine_t *e, int p, size_t up, size_t keep, size_t res, size_t desc);

extern "C" int h261b_engine_reserve_step(h261b_engine_t *e, const h261b_session_config_t *c, int32_t pictures)
{
    clear_error();
    if (!e || pictures < 0 || !session_config_ok(c)) {
        set_error("h261b_engine_reserve_step: bad arguments");
        return H261B_ERR_ARG;
    }
    cudaSetDevice(e->cfg.device);
    const PictureLayout lay = PictureLayout::of(c->width, c->height);
    const size_t nmb = (size_t)(c->width / 16) * (c->height / 16), k = (size_t)pictures;
    e->reserved_upload += k * align_up(lay.bytes, 256);
    e->reserved_results += k * (nmb * sizeof(h261b_mb_info_t) + sizeof(h261b_pic_info_t) + 32 +
                                align_up(nmb * 384, 256)) + 1024;
    e->reserved_desc += k * (sizeof(h261b_session_dev_t) + nmb * sizeof(uint32_t)) + 1024;
    for (int p = 0; p < NSLOT; p++) {
        const size_t keep = (p == (int)(e->next_step % NSLOT) && e->upload_checked) ? e->upload_used : 0;
        int rc = grow_arenas(e, p, e->reserved_upload, keep, e->reserved_results, e->reserved_desc);
        if (rc)
            return rc;
    }
    return H261B_OK;
}

extern "C" int h261b_session_close(h261b_engine_t *e, int32_t id)
{
    clear_error();
    Session *s = get_session(e, id);
    if (!s)
        return H261B_ERR_ARG;
    /* steps already issued may still read or write the slot: it goes back
     * to the pool once the last of them has completed */
    e->retired.push_back({ s->rec[0], s->slot_bytes, e->next_step - 1 });
    reclaim(e);
    e->session_bytes -= (int64_t)s->slot_bytes;
    e->open_count--;
    *s = Session();
    return H261B_OK;
}

/* Grow the arenas of slot p to hold `up` upload bytes (the first `keep`
 * of which are queued pictures that survive), `res` result bytes and `desc`
 * descriptor bytes.  Sized by what a step actually holds, not by every open
 * session, so that a server with thousands of open sessions and a few
 * pictures per step keeps small arenas; they grow by doubling, so a
 * growing load reallocates (and waits for the slot's stream) a few times
 * only. */
static int grow_arenas(h261b_engine_t *e, int p, size_t up, size_t keep, size_t res, size_t desc)
{
    if (up <= e->upload[p].cap && res <= e->results[p].cap && desc <= e->desc[p].cap)
        return H261B_OK;
    e->copier->join();   /* copies in flight write into the upload arena */
    H261B_CUDA_TRY(cudaStreamSynchronize(e->stream[p]));
    int rc;
    if ((rc = e->upload[p].reserve(up, keep)) || (rc = e->results[p].reserve(res)) || (rc = e->desc[p].reserve(desc)))
        return rc;
    return H261B_OK;
}

/* room for one picture of session s in the next step's upload arena */
static int reserve_input(h261b_engine_t *e, Session *s, int32_t id, int32_t quant, size_t *off, const char *who)
{
    if (quant > 31) {
        set_error("%s: QUANT %d out of range", who, quant);
        return H261B_ERR_ARG;
    }
    if (s->queued) {
        set_error("%s: session %d already has a queued picture", who, id);
        return H261B_ERR_STATE;
    }
    const int p = (int)(e->next_step % NSLOT);
    if (!e->upload_checked) {
        /* the copy that last read this pinned arena (NSLOT steps ago) must be
         * complete before the host writes into it */
        if (e->in_flight[p])
            H261B_CUDA_TRY(cudaEventSynchronize(e->h2d_done[p]));
        e->upload_checked = true;
        e->upload_used = 0;
    }
    *off = e->upload_used;
    int rc = grow_arenas(e, p, *off + align_up(s->lay.bytes, 256), e->upload_used, 0, 0);
    if (rc)
        return rc;
    if (*off + s->lay.bytes > e->upload[p].cap) {
        set_error("%s: upload arena overflow", who);
        return H261B_ERR_STATE;
    }
    e->upload_used = *off + align_up(s->lay.bytes, 256);
    s->src_off = *off;
    s->queued = true;
    s->queued_quant = quant > 0 ? quant : 0;
    return H261B_OK;
}

extern "C" int h261b_session_submit(h261b_engine_t *e, int32_t id, const uint8_t *y, const uint8_t *cb,
                                    const uint8_t *cr, int32_t quant)
{
    clear_error();
    Session *s = get_session(e, id);
    if (!s || !y || !cb || !cr) {
        if (s)
            set_error("h261b_session_submit: NULL plane");
        return H261B_ERR_ARG;
    }
    size_t off = 0;
    int rc = reserve_input(e, s, id, quant, &off, "h261b_session_submit");
    if (rc)
        return rc;
    uint8_t *dst = e->upload[e->next_step % NSLOT].host + off;
    const size_t ny = (size_t)s->w * s->h, nc = ny / 4;
    memcpy(dst + s->lay.off_y, y, ny);
    memcpy(dst + s->lay.off_cb, cb, nc);
    memcpy(dst + s->lay.off_cr, cr, nc);
    return H261B_OK;
}

extern "C" int h261b_engine_inputs(h261b_engine_t *e, int32_t n, const int32_t *ids, const int32_t *quants,
                                   uint8_t **staging, int64_t *offsets)
{
    clear_error();
    if (!e || n < 0 || (n > 0 && (!ids || !offsets)) || !staging) {
        set_error("h261b_engine_inputs: bad arguments");
        return H261B_ERR_ARG;
    }
    for (int32_t i = 0; i < n; i++)
        if (!get_session(e, ids[i])) {
            set_error("h261b_engine_inputs: session %d is not open", ids[i]);
            return H261B_ERR_ARG;
        }
    /* room for the whole batch at once: one reallocation at most */
    {
        const int p = (int)(e->next_step % NSLOT);
        if (!e->upload_checked) {
            if (e->in_flight[p])
                H261B_CUDA_TRY(cudaEventSynchronize(e->h2d_done[p]));
            e->upload_checked = true;
            e->upload_used = 0;
        }
        size_t need = e->upload_used;
        for (int32_t i = 0; i < n; i++)
            need += align_up(e->sessions[(size_t)ids[i]].lay.bytes, 256);
        int rc = grow_arenas(e, p, need, e->upload_used, 0, 0);
        if (rc)
            return rc;
    }
    const size_t used0 = e->upload_used;
    for (int32_t i = 0; i < n; i++) {
        Session *s = get_session(e, ids[i]);
        size_t off = 0;
        int rc = reserve_input(e, s, ids[i], quants ? quants[i] : 0, &off, "h261b_engine_inputs");
        if (rc) {
            /* undo the reservations of this call */
            for (int32_t j = 0; j < i; j++) {
                Session *t = get_session(e, ids[j]);
                t->queued = false;
                t->queued_quant = 0;
            }
            e->upload_used = used0;
            return rc;
        }
        offsets[3 * i] = (int64_t)(off + s->lay.off_y);
        offsets[3 * i + 1] = (int64_t)(off + s->lay.off_cb);
        offsets[3 * i + 2] = (int64_t)(off + s->lay.off_cr);
    }
    *staging = e->upload[e->next_step % NSLOT].host;
    return H261B_OK;
}

static int submit_batch(h261b_engine_t *e, int32_t n, const int32_t *ids, const uint8_t *const *y,
                        const uint8_t *const *cb, const uint8_t *const *cr, const int32_t *quants, bool async)
{
    clear_error();
    if (!e || n < 0 || (n > 0 && (!ids || !y || !cb || !cr))) {
        set_error("h261b_engine_submit_batch: bad arguments");
        return H261B_ERR_ARG;
    }
    for (int32_t i = 0; i < n; i++)
        if (!y[i] || !cb[i] || !cr[i]) {
            set_error("h261b_engine_submit_batch: NULL plane for picture %d", i);
            return H261B_ERR_ARG;
        }
    NvtxRange range("h261b copy %d pictures%s", n, async ? " (async)" : "");
    e->copier->join();   /* one batch in flight at a time */
    std::vector<int64_t> offs((size_t)n * 3);
    uint8_t *staging = nullptr;
    int rc = h261b_engine_inputs(e, n, ids, quants, &staging, offs.data());
    if (rc)
        return rc;
    std::vector<CopyJob> &jobs = e->copy_jobs;
    jobs.clear();
    for (int32_t i = 0; i < n; i++) {
        const Session &s = e->sessions[(size_t)ids[i]];
        const size_t ny = (size_t)s.w * s.h, nc = ny / 4;
        jobs.push_back({ staging + offs[3 * i], y[i], ny });
        jobs.push_back({ staging + offs[3 * i + 1], cb[i], nc });
        jobs.push_back({ staging + offs[3 * i + 2], cr[i], nc });
    }
    if (async)
        e->copier->start(jobs);
    else
        e->copier->run(jobs);
    return H261B_OK;
}

extern "C" int h261b_engine_submit_batch(h261b_engine_t *e, int32_t n, const int32_t *ids, const uint8_t *const *y,
                                         const uint8_t *const *cb, const uint8_t *const *cr, const int32_t *quants)
{
    return submit_batch(e, n, ids, y, cb, cr, quants, false);
}

extern "C" int h261b_engine_submit_batch_async(h261b_engine_t *e, int32_t n, const int32_t *ids,
                                               const uint8_t *const *y, const uint8_t *const *cb,
                                               const uint8_t *const *cr, const int32_t *quants)
{
    return submit_batch(e, n, ids, y, cb, cr, quants, true);
}

extern "C" int h261b_engine_step_records(h261b_engine_t *e, const h261b_mb_result_t **records, int64_t *count,
                                         int64_t *step)
{
    clear_error();
    if (!e || !records || !count || !step)
        return H261B_ERR_ARG;
    *step = e->done_step;
    if (e->done_step < 0) {
        *records = nullptr;
        *count = 0;
        return H261B_OK;
    }
    const int p = (int)(e->done_step % NSLOT);
    *records = (const h261b_mb_result_t *)e->results[p].host;
    *count = e->step_mbs[p];
    return H261B_OK;
}

extern "C" int h261b_session_input(h261b_engine_t *e, int32_t id, int32_t quant, uint8_t **y, uint8_t **cb,
                                   uint8_t **cr)
{
    clear_error();
    Session *s = get_session(e, id);
    if (!s || !y || !cb || !cr) {
        if (s)
            set_error("h261b_session_input: NULL output pointer");
        return H261B_ERR_ARG;
    }
    size_t off = 0;
    int rc = reserve_input(e, s, id, quant, &off, "h261b_session_input");
    if (rc)
        return rc;
    uint8_t *dst = e->upload[e->next_step % NSLOT].host + off;
    *y = dst + s->lay.off_y;
    *cb = dst + s->lay.off_cb;
    *cr = dst + s->lay.off_cr;
    return H261B_OK;
}

extern "C" int h261b_session_submit_device(h261b_engine_t *e, int32_t id, const uint8_t *y, const uint8_t *cb,
                                           const uint8_t *cr, int32_t quant)
{
    clear_error();
    Session *s = get_session(e, id);
    if (!s || !y || !cb || !cr || quant > 31)
        return H261B_ERR_ARG;
    /* 16-byte luma rows and 8-byte chroma rows are loaded whole */
    if (((uintptr_t)y & 15) || ((uintptr_t)cb & 7) || ((uintptr_t)cr & 7)) {
        set_error("h261b_session_submit_device: planes must be 16 (Y) and 8 (Cb, Cr) byte aligned");
        return H261B_ERR_ARG;
    }
    if (s->queued) {
        set_error("h261b_session_submit_device: session %d already has a queued picture", id);
        return H261B_ERR_STATE;
    }
    s->dev_src[0] = y;
    s->dev_src[1] = cb;
    s->dev_src[2] = cr;
    s->queued = true;
    s->queued_quant = quant > 0 ? quant : 0;
    return H261B_OK;
}

extern "C" int h261b_engine_submit_device_batch(h261b_engine_t *e, int32_t n, const int32_t *ids,
                                                const uint8_t *const *y, const uint8_t *const *cb,
                                                const uint8_t *const *cr, const int32_t *quants)
{
    clear_error();
    if (!e || n < 0 || (n > 0 && (!ids || !y || !cb || !cr))) {
        set_error("h261b_engine_submit_device_batch: bad arguments");
        return H261B_ERR_ARG;
    }
    /* all or nothing: every picture is checked before any is queued */
    std::vector<int32_t> order(ids, ids + n);
    std::sort(order.begin(), order.end());
    if (std::adjacent_find(order.begin(), order.end()) != order.end()) {
        set_error("h261b_engine_submit_device_batch: a session appears twice");
        return H261B_ERR_ARG;
    }
    for (int32_t i = 0; i < n; i++) {
        const Session *s = get_session(e, ids[i]);
        const int32_t q = quants ? quants[i] : 0;
        if (!s || !y[i] || !cb[i] || !cr[i] || q > 31) {
            set_error("h261b_engine_submit_device_batch: picture %d: bad session, plane or QUANT", i);
            return H261B_ERR_ARG;
        }
        if (((uintptr_t)y[i] & 15) || ((uintptr_t)cb[i] & 7) || ((uintptr_t)cr[i] & 7)) {
            set_error("h261b_engine_submit_device_batch: picture %d: planes must be 16 (Y) and 8 (Cb, Cr) byte "
                      "aligned", i);
            return H261B_ERR_ARG;
        }
        if (s->queued) {
            set_error("h261b_engine_submit_device_batch: session %d already has a queued picture", ids[i]);
            return H261B_ERR_STATE;
        }
    }
    for (int32_t i = 0; i < n; i++) {
        Session &s = e->sessions[(size_t)ids[i]];
        const int32_t q = quants ? quants[i] : 0;
        s.dev_src[0] = y[i];
        s.dev_src[1] = cb[i];
        s.dev_src[2] = cr[i];
        s.queued = true;
        s.queued_quant = q > 0 ? q : 0;
    }
    return H261B_OK;
}

/* the plan of the next step: a tuning candidate while the tuner runs and
 * the step is mostly inter (returns 1), else the engine's plan */
static int next_plan(h261b_engine_t *e, bool mostly_inter, LaunchPlan *out)
{
    if (!e->tuned && e->tuner.active() && mostly_inter) {
        *out = e->tuner.current();
        return 1;
    }
    *out = e->plan;
    return 0;
}

static const void *bits_dev_or_null(h261b_engine_t *e, int p, int32_t n_bits)
{
    return n_bits ? (const void *)e->bits[p].dev : nullptr;
}

extern "C" int h261b_engine_step(h261b_engine_t *e)
{
    clear_error();
    if (!e)
        return H261B_ERR_ARG;
    NvtxRange range("h261b step %lld", (long long)e->next_step);
    cudaSetDevice(e->cfg.device);
    const int64_t id = e->next_step;
    const int p = (int)(id % NSLOT);
    const int prev = (int)((id + NSLOT - 1) % NSLOT);   /* the slot of step id - 1 */
    std::vector<int32_t> list;
    for (size_t i = 0; i < e->sessions.size(); i++)
        if (e->sessions[i].open && e->sessions[i].queued)
            list.push_back((int32_t)i);
    if (list.empty())
        return 0;
    /* this step's descriptor and result bytes (the layouts below) */
    {
        int64_t mbs = 0;
        size_t levels = 0;
        for (int32_t sid : list) {
            mbs += e->sessions[(size_t)sid].nmb;
            levels += align_up((size_t)e->sessions[(size_t)sid].nmb * 384, 256);
        }
        const size_t n_list = list.size();
        const size_t res = align_up(align_up(align_up((size_t)mbs * sizeof(h261b_mb_info_t), 256) +
                                                 n_list * sizeof(h261b_pic_info_t),
                                             256) +
                                        n_list * 32,
                                    256) +
                           levels + align_up((size_t)mbs * sizeof(h261_mb_mode_decision_t), 256);
        const size_t desc = sizeof(h261b_step_dev_t) + align_up(n_list * sizeof(h261b_session_dev_t), 256) +
                            (size_t)mbs * sizeof(uint32_t);
        int rc = grow_arenas(e, p, 0, 0, res, desc);
        if (rc)
            return rc;
    }
    int rc;
    /* arenas of this slot were last used by step id - NSLOT */
    if (e->in_flight[p] && id - NSLOT > e->done_step) {
        H261B_CUDA_TRY(cudaEventSynchronize(e->step_done[p]));
        e->done_step = id - NSLOT;
        reclaim(e);
    }

    Mirror &dm = e->desc[p], &rm = e->results[p], &um = e->upload[p];
    const size_t n = list.size();
    /* descriptor arena: step state, session descriptors, work list */
    memset(dm.host, 0, sizeof(h261b_step_dev_t));
    const size_t desc_off = sizeof(h261b_step_dev_t);
    h261b_session_dev_t *desc = (h261b_session_dev_t *)(dm.host + desc_off);
    const size_t work_off = desc_off + align_up(n * sizeof(h261b_session_dev_t), 256);
    uint32_t *work = (uint32_t *)(dm.host + work_off);
    /* results arena: the MB records of all sessions back to back, the
     * picture records of the bitstream writer, then the levels of each
     * session on a 256-byte boundary */
    int64_t total_mb = 0;
    for (int32_t sid : list)
        total_mb += e->sessions[(size_t)sid].nmb;
    size_t info_off = 0;
    const size_t pic_base = align_up((size_t)total_mb * sizeof(h261b_mb_info_t), 256);
    const size_t ssd_base = align_up(pic_base + n * sizeof(h261b_pic_info_t), 256);
    const size_t levels_base = align_up(ssd_base + n * 32, 256);
    size_t res_off = levels_base;
    size_t levels_total = 0;
    for (int32_t sid : list)
        levels_total += align_up((size_t)e->sessions[(size_t)sid].nmb * 384, 256);
    /* the mode decisions a search launch hands to the encode launch (split
     * kernels; device only, after the levels) */
    const size_t md_base = levels_base + levels_total;
    size_t md_off = md_base;
    int64_t inter_mbs = 0;
    int32_t n_work = 0, n_bits = 0, n_rc = 0, rc_begin = 0, n_ssd = 0;
    for (size_t k = 0; k < n; k++) {
        Session &s = e->sessions[(size_t)list[k]];
        if (s.queued_quant > 0)
            s.quant = s.queued_quant;
        const int intra = s.frame_index == 0 || (s.intra_period > 0 && s.frame_index % s.intra_period == 0);
        const uint8_t *src = um.dev + s.src_off;
        const uint8_t *ref = s.rec[s.rec_cur];
        uint8_t *rec = s.rec[s.rec_cur ^ 1];
        h261b_session_dev_t &d = desc[k];
        memset(&d, 0, sizeof(d));
        if (s.dev_src[0]) {
            d.cur_y = s.dev_src[0];
            d.cur_cb = s.dev_src[1];
            d.cur_cr = s.dev_src[2];
        } else {
            d.cur_y = src + s.lay.off_y;
            d.cur_cb = src + s.lay.off_cb;
            d.cur_cr = src + s.lay.off_cr;
        }
        d.ref_y = ref + s.lay.off_y;
        d.ref_cb = ref + s.lay.off_cb;
        d.ref_cr = ref + s.lay.off_cr;
        d.rec_y = rec + s.lay.off_y;
        d.rec_cb = rec + s.lay.off_cb;
        d.rec_cr = rec + s.lay.off_cr;
        d.pitch_y = s.lay.pitch_y;
        d.pitch_c = s.lay.pitch_c;
        d.mbw = s.mbw;
        d.mbh = s.mbh;
        d.frame_type = intra ? H261B_FRAME_TYPE_INTRA : H261B_FRAME_TYPE_INTER;
        d.quant = s.quant;
        d.me_mode = e->cfg.me_mode;
        d.skip_search = intra;
        d.dn = s.dn;
        Result &r = s.res[p];
        r.step = id;
        r.frame = s.frame_index;
        r.type = d.frame_type;
        r.quant = s.quant;
        r.info_off = info_off;
        d.info_out = (h261b_mb_info_t *)(rm.dev + info_off);
        info_off += (size_t)s.nmb * sizeof(h261b_mb_info_t);
        r.level_off = res_off;
        d.level_out = (int8_t *)(rm.dev + res_off);
        res_off += align_up((size_t)s.nmb * 384, 256);
        r.has_bits = s.bitstream;
        r.pic_off = pic_base + k * sizeof(h261b_pic_info_t);
        if (s.bitstream) {
            uint8_t *bb = s.bits_base[p];
            const h261b_bits_layout_t &L = s.bits_lay;
            d.bits_out = (uint32_t *)(bb + L.picture);
            d.bits_cap = (int32_t)(L.scratch - L.picture);
            d.frame_num = s.frame_index;
            d.pic_out = (h261b_pic_info_t *)(rm.dev + r.pic_off);
            d.vlc_scratch = (uint32_t *)(bb + L.scratch);
            d.vlc_pos = (int32_t *)(bb + L.pos);
            d.vlc_plan = (uint32_t *)(bb + L.plan);
            d.vlc_total = (int32_t *)(bb + L.total);
            n_bits++;
        }
        r.has_ssd = s.psnr;
        r.ssd_off = ssd_base + k * 32;
        if (s.psnr) {
            d.ssd_out = (unsigned long long *)(rm.dev + r.ssd_off);
            n_ssd++;
        }
        if (s.rc) {
            d.rc = s.rc_dev;
            d.md_out = s.md_dev;
            d.md_in = s.md_dev;
            n_rc++;
        } else {
            /* read only by an encode launch after a search launch */
            d.md_out = (h261_mb_mode_decision_t *)(rm.dev + md_off);
            d.md_in = d.md_out;
        }
        md_off += (size_t)s.nmb * sizeof(h261_mb_mode_decision_t);
        if (!intra)
            inter_mbs += s.nmb;
    }
    /* work list: the MBs of fixed-QUANT sessions, then those of
     * rate-controlled ones (the second encode launch takes that tail) */
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1)
            rc_begin = n_work;
        for (size_t k = 0; k < n; k++) {
            const Session &s = e->sessions[(size_t)list[k]];
            if ((int)s.rc != pass)
                continue;
            for (int32_t m = 0; m < s.nmb; m++)
                work[n_work++] = ((uint32_t)k << 12) | (uint32_t)m;
        }
    }
    cudaStream_t st = e->stream[p];
    const size_t desc_bytes = work_off + (size_t)n_work * sizeof(uint32_t);
    e->copier->join();   /* pictures of h261b_engine_submit_batch_async */
    LaunchPlan plan;
    const int tuning = next_plan(e, 2 * inter_mbs >= total_mb, &plan);
    const int warps = plan.warps, ctas = plan.ctas;
    /* the arithmetic and the search mode are the engine's, for every launch */
    const int fmad_bit =
        (e->cfg.fmad ? H261B_FMAD_BIT : 0) | (e->cfg.me_mode == H261B_ME_FULL ? H261B_LAUNCH_ME_FULL : 0);
    const int phases = H261B_PHASE_ME | H261B_PHASE_MD | H261B_PHASE_ENCDEC | fmad_bit | plan.bits() |
                       e->test_bits | (plan.split ? H261B_KIND_SEARCH : 0);
    if (!plan.split)
        for (size_t k = 0; k < n; k++)
            if (!desc[k].rc)
            {
                desc[k].md_out = nullptr;   /* the fused kernel hands nothing on */
                desc[k].md_in = nullptr;
            }
    h261b_session_dev_t *desc_dev = (h261b_session_dev_t *)(dm.dev + desc_off);
    const uint32_t *work_dev = (const uint32_t *)(dm.dev + work_off);
    const size_t upload_bytes = e->upload_checked ? e->upload_used : 0;
    /* records and picture records always, levels when asked for */
    const size_t d2h = e->cfg.levels_to_host ? res_off : levels_base;
    if (n_bits && (rc = e->bits[p].reserve(e->bits_want)))
        return rc;

    /* the step's device work: uploads, encode (and rate control), the
     * bitstream kernels, the download, and the events the host and the
     * other stream wait on.  Recorded as external events so that a graph
     * captured from it keeps them visible outside the graph. */
    auto enqueue = [&](bool capturing) -> int {
        const unsigned rf = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
        const unsigned wf = capturing ? cudaEventWaitExternal : cudaEventWaitDefault;
        H261B_CUDA_TRY(cudaEventRecordWithFlags(e->t_begin[p], st, rf));
        if (n_ssd)
            H261B_CUDA_TRY(cudaMemsetAsync(rm.dev + ssd_base, 0, n * 32, st));
        H261B_CUDA_TRY(cudaMemcpyAsync(dm.dev, dm.host, desc_bytes, cudaMemcpyHostToDevice, st));
        if (upload_bytes)
            H261B_CUDA_TRY(cudaMemcpyAsync(um.dev, um.host, upload_bytes, cudaMemcpyHostToDevice, st));
        H261B_CUDA_TRY(cudaEventRecordWithFlags(e->h2d_done[p], st, rf));
        H261B_CUDA_TRY(cudaEventRecordWithFlags(e->t_h2d[p], st, rf));
        /* the previous step's reconstructions are this step's references */
        if (id > 0)
            H261B_CUDA_TRY(cudaStreamWaitEvent(st, e->kernel_done[prev], wf));
        H261B_CUDA_TRY(cudaEventRecordWithFlags(e->t_ready[p], st, rf));
        H261B_CUDA_TRY(cudaEventRecordWithFlags(e->k_start[p], st, rf));
        int32_t *sched = e->sched_dev + 2 * p;
        /* fused: one launch encodes the fixed-QUANT sessions and searches
         * the rate-controlled ones; split: a search launch over every MB
         * (mode decisions into md_out) */
        int lr = h261b_launch_step(desc_dev, work_dev, n_work, phases, warps, ctas, sched, st);
        if (lr == 0 && n_rc) {
            /* rate-controlled sessions: the picture QUANT from this
             * picture's costs and the previous picture's size (written by
             * the layout kernel of the step that held it), then their
             * encode.  That step is one of the other slots' latest (a
             * session may skip steps) or older, on this stream. */
            for (int q = 1; q < NSLOT && q <= id; q++)
                H261B_CUDA_TRY(cudaStreamWaitEvent(st, e->layout_done[(id + NSLOT - q) % NSLOT], wf));
            lr = h261b_launch_ratectrl(desc_dev, (int32_t)n, st);
        }
        if (lr == 0 && plan.split) {
            /* the encode launch over every MB, right after the search launch
             * (a programmatic dependent launch) or after the rate control */
            lr = h261b_launch_step(desc_dev, work_dev, n_work,
                                   H261B_PHASE_ENCDEC | fmad_bit | plan.bits() | e->test_bits | H261B_KIND_ENCODE |
                                       (n_rc ? 0 : H261B_LAUNCH_PDL),
                                   warps, ctas, sched, st);
        } else if (lr == 0 && n_rc) {
            lr = h261b_launch_step(desc_dev, work_dev + rc_begin, n_work - rc_begin,
                                   H261B_PHASE_ENCDEC | fmad_bit | plan.bits() | e->test_bits, warps, ctas, sched, st);
        }
        if (lr != 0) {
            set_error("step launch failed: %s", cudaGetErrorString((cudaError_t)lr));
            return H261B_ERR_CUDA;
        }
        /* the encode kernel's end, marked on the side stream: the next step
         * may start encoding while this one writes bitstreams */
        H261B_CUDA_TRY(cudaEventRecord(e->fork_ev[p], st));
        H261B_CUDA_TRY(cudaStreamWaitEvent(e->side[p], e->fork_ev[p], 0));
        H261B_CUDA_TRY(cudaEventRecordWithFlags(e->k_end[p], e->side[p], rf));
        H261B_CUDA_TRY(cudaEventRecordWithFlags(e->kernel_done[p], e->side[p], rf));
        H261B_CUDA_TRY(cudaEventRecord(e->join_ev[p], e->side[p]));
        if (n_bits) {
            lr = h261b_launch_bitstream(desc_dev, (int32_t)n, work_dev, n_work, (h261b_step_dev_t *)dm.dev,
                                        e->bits[p].dev, (int64_t)e->bits[p].cap, e->sm_count, st,
                                        n_rc ? (void *)e->layout_done[p] : nullptr, e->test_codes_extra);
            if (lr != 0) {
                set_error("bitstream launch failed: %s", cudaGetErrorString((cudaError_t)lr));
                return H261B_ERR_CUDA;
            }
            H261B_CUDA_TRY(cudaEventRecordWithFlags(e->b_end[p], st, rf));
        }
        /* the records download waits for the encode kernel's end: the
         * bitstream kernels may finish first (the codes kernel waits only
         * for the pictures that write a bitstream) */
        H261B_CUDA_TRY(cudaStreamWaitEvent(st, e->join_ev[p], 0));
        H261B_CUDA_TRY(cudaMemcpyAsync(rm.host, rm.dev, d2h, cudaMemcpyDeviceToHost, st));
        H261B_CUDA_TRY(cudaEventRecordWithFlags(e->t_end[p], st, rf));
        H261B_CUDA_TRY(cudaEventRecordWithFlags(e->step_done[p], st, rf));
        return H261B_OK;
    };

    /* Steps whose launches look the same (sizes, arena addresses, launch
     * shape) replay one CUDA graph per slot: the descriptor and work-list
     * contents differ, but they are data in pinned memory that the graph's
     * upload copies.  A signature is captured the second time in a row it
     * comes on its slot.  Tuning steps, an engine's first step and engines
     * with use_graphs = 0 launch directly. */
    const StepKey key = { dm.host, dm.dev, um.host, um.dev, rm.host, rm.dev, bits_dev_or_null(e, p, n_bits),
                          n_bits ? e->bits[p].cap : 0, desc_off, work_off, desc_bytes, upload_bytes, ssd_base,
                          d2h, (int64_t)n, n_work, rc_begin, n_rc, n_ssd ? 1 : 0, warps, ctas, phases,
                          (int32_t)std::min<int64_t>(id, NSLOT - 1) };
    StepGraph &gr = e->graph[p];
    const bool repeated = gr.has_last_direct && gr.last_direct == key;
    const bool capturable = e->cfg.use_graphs && !e->graphs_off && !tuning && id > 0;
    if (capturable && !(gr.exec && gr.key == key) && !repeated) {
        /* a new signature: launch directly, capture if it comes again */
        gr.last_direct = key;
        gr.has_last_direct = true;
        if ((rc = enqueue(false)))
            return rc;
    } else if (capturable && gr.exec && gr.key == key) {
        H261B_CUDA_TRY(cudaGraphLaunch(gr.exec, st));
        e->graph_replays++;
    } else if (capturable && cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        const int erc = enqueue(true);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(st, &g);
        cudaGraphExec_t ex = nullptr;
        if (erc == H261B_OK && ce == cudaSuccess && g)
            ce = cudaGraphInstantiate(&ex, g, 0);
        if (g)
            cudaGraphDestroy(g);
        if (erc != H261B_OK || ce != cudaSuccess || !ex) {
            /* capture did not work here: nothing of it ran; launch directly
             * from now on */
            cudaGetLastError();
            e->graphs_off = true;
            if ((rc = enqueue(false)))
                return rc;
        } else {
            gr.reset();
            gr.exec = ex;
            gr.key = key;
            H261B_CUDA_TRY(cudaGraphLaunch(ex, st));
            e->graph_captures++;
        }
    } else {
        if ((rc = enqueue(false)))
            return rc;
    }
    e->step_bits_ran[p] = n_bits > 0;
    e->last_h2d = (int64_t)desc_bytes + (int64_t)upload_bytes;
    e->last_d2h = (int64_t)d2h;
    e->in_flight[p] = true;
    e->step_mbs[p] = total_mb;

    if (tuning) {
        /* time this candidate before moving on (tuning steps are synchronous) */
        H261B_CUDA_TRY(cudaEventSynchronize(e->k_end[p]));
        float ms = 0.f;
        H261B_CUDA_TRY(cudaEventElapsedTime(&ms, e->k_start[p], e->k_end[p]));
        tuner_record(e, ms);
    }

    for (int32_t sid : list) {
        Session &s = e->sessions[(size_t)sid];
        s.queued = false;
        s.queued_quant = 0;
        s.dev_src[0] = s.dev_src[1] = s.dev_src[2] = nullptr;
        s.rec_cur ^= 1;
        s.frame_index++;
    }
    e->next_step = id + 1;
    e->upload_checked = false;
    e->upload_used = 0;
    return (int)n;
}

/* Wait until every step up to `id` has completed.  Steps do not complete in
 * issue order: step k's stream waits only for step k-1's encode kernel (its
 * references), not for k-1's bitstream kernels and download on the other
 * slot's stream, so each step in (done_step, id] is waited for on its own
 * slot.  Steps older than NSLOT before the next one were waited for when
 * their slot was reused. */
static int wait_step(h261b_engine_t *e, int64_t id)
{
    if (id < 0 || id <= e->done_step)
        return H261B_OK;
    NvtxRange range("h261b wait step %lld", (long long)id);
    for (int64_t k = std::max(e->done_step + 1, id - NSLOT + 1); k <= id; k++)
        H261B_CUDA_TRY(cudaEventSynchronize(e->step_done[k % NSLOT]));
    e->done_step = id;
    reclaim(e);
    return H261B_OK;
}

extern "C" int h261b_engine_sync(h261b_engine_t *e)
{
    clear_error();
    if (!e)
        return H261B_ERR_ARG;
    return wait_step(e, e->next_step - 1);
}

extern "C" int h261b_engine_wait_step(h261b_engine_t *e, int64_t step)
{
    clear_error();
    if (!e)
        return H261B_ERR_ARG;
    if (step >= e->next_step) {
        set_error("h261b_engine_wait_step: step %lld has not been issued", (long long)step);
        return H261B_ERR_STATE;
    }
    if (step < e->next_step - NSLOT) {
        set_error("h261b_engine_wait_step: step %lld is older than the steps in flight", (long long)step);
        return H261B_ERR_STATE;
    }
    return wait_step(e, step);
}

extern "C" int h261b_engine_wait_previous(h261b_engine_t *e)
{
    clear_error();
    if (!e)
        return H261B_ERR_ARG;
    return wait_step(e, e->next_step - 2);
}

extern "C" int h261b_session_result(h261b_engine_t *e, int32_t id, h261b_frame_result_t *out)
{
    clear_error();
    Session *s = get_session(e, id);
    if (!s || !out)
        return H261B_ERR_ARG;
    const Result *best = nullptr;
    for (const Result &r : s->res)
        if (r.step >= 0 && r.step <= e->done_step && (!best || r.step > best->step))
            best = &r;
    if (!best) {
        set_error("h261b_session_result: no completed step for session %d (wait for a step first)", id);
        return H261B_ERR_STATE;
    }
    const int p = (int)(best->step % NSLOT);
    const Mirror &rm = e->results[p];
    out->frame_index = best->frame;
    out->frame_type = best->type;
    out->quant = best->quant;
    out->num_mb = s->nmb;
    out->mbs = (const h261b_mb_result_t *)(rm.host + best->info_off);
    out->levels = e->cfg.levels_to_host ? (const int8_t *)(rm.host + best->level_off) : nullptr;
    out->bits = nullptr;
    out->bits_bytes = 0;
    out->bits_status = 0;
    for (int c = 0; c < 3; c++) {
        out->ssd[c] = 0;
        out->psnr[c] = 0.0;
    }
    if (best->has_ssd) {
        const uint64_t *ssd = (const uint64_t *)(rm.host + best->ssd_off);
        for (int c = 0; c < 3; c++) {
            /* h261_main.c:79-86 */
            const double pels = c == 0 ? (double)s->w * s->h : (double)(s->w / 2) * (s->h / 2);
            out->ssd[c] = ssd[c];
            out->psnr[c] = ssd[c] == 0 ? 100.0 : 10 * log10(255.0 * 255.0 * pels / (double)ssd[c]);
        }
    }
    if (best->has_bits) {
        const h261b_pic_info_t &pi = *(const h261b_pic_info_t *)(rm.host + best->pic_off);
        out->quant = pi.quant;   /* the rate control's choice for CBR sessions */
        if (pi.status != 0) {
            out->bits_status = H261B_ERR_STATE;
        } else if (pi.host_off >= 0) {
            out->bits = e->bits[p].host + pi.host_off;
            out->bits_bytes = pi.bytes;
        } else {
            /* the step's pictures overflowed the host arena: this one is
             * still in the session's device slot (until the step after
             * next); later steps get a larger arena */
            s->bits_spill.resize((size_t)pi.bytes);
            cudaSetDevice(e->cfg.device);
            H261B_CUDA_TRY(cudaMemcpy(s->bits_spill.data(), s->bits_base[p] + s->bits_lay.picture, (size_t)pi.bytes,
                                      cudaMemcpyDeviceToHost));
            out->bits = s->bits_spill.data();
            out->bits_bytes = pi.bytes;
            e->bits_want = std::max(e->bits_want, 2 * e->bits[p].cap);
        }
    }
    return H261B_OK;
}

extern "C" int h261b_engine_step_bits(h261b_engine_t *e, int64_t *bytes, int32_t *pictures)
{
    clear_error();
    if (!e || !bytes)
        return H261B_ERR_ARG;
    *bytes = 0;
    if (pictures)
        *pictures = 0;
    if (e->done_step < 0)
        return H261B_OK;
    const int p = (int)(e->done_step % NSLOT);
    const Mirror &rm = e->results[p];
    for (const Session &s : e->sessions) {
        const Result &r = s.res[p];
        if (!s.open || !r.has_bits || r.step != e->done_step)
            continue;
        const h261b_pic_info_t &pi = *(const h261b_pic_info_t *)(rm.host + r.pic_off);
        if (pi.status == 0) {
            *bytes += pi.bytes;
            if (pictures)
                (*pictures)++;
        }
    }
    return H261B_OK;
}

extern "C" int h261b_session_recon(h261b_engine_t *e, int32_t id, uint8_t *y, uint8_t *cb, uint8_t *cr)
{
    clear_error();
    Session *s = get_session(e, id);
    if (!s || !y || !cb || !cr)
        return H261B_ERR_ARG;
    cudaSetDevice(e->cfg.device);
    int rc = sync_all(e);
    if (rc)
        return rc;
    const uint8_t *rec = s->rec[s->rec_cur];
    const size_t ny = (size_t)s->w * s->h, nc = ny / 4;
    H261B_CUDA_TRY(cudaMemcpy(y, rec + s->lay.off_y, ny, cudaMemcpyDeviceToHost));
    H261B_CUDA_TRY(cudaMemcpy(cb, rec + s->lay.off_cb, nc, cudaMemcpyDeviceToHost));
    H261B_CUDA_TRY(cudaMemcpy(cr, rec + s->lay.off_cr, nc, cudaMemcpyDeviceToHost));
    return H261B_OK;
}

extern "C" int h261b_result_to_abi(const h261b_frame_result_t *r, int32_t width, h261_macroblock_t *mbs)
{
    if (!r || !mbs || width < 16 || (width & 15))
        return H261B_ERR_ARG;
    const int32_t mbw = width / 16;
    for (int32_t i = 0; i < r->num_mb; i++) {
        const h261b_mb_result_t &m = r->mbs[i];
        h261_macroblock_t &o = mbs[i];
        o.i_macroblock_address = 0;
        o.i_macroblock_type = m.type;
        o.i_macroblock_type_flags = m.flags;
        o.i_macroblock_quant = m.quant;
        o.rgi_mv[0] = m.mvx;
        o.rgi_mv[1] = m.mvy;
        o.i_coded_block_pattern = (uint8_t)m.cbp;
        /* compact levels are column-major per block: [b][u][v] */
        const int8_t *lv = r->levels + (size_t)i * 384;
        for (int b = 0; b < 6; b++)
            for (int u = 0; u < 8; u++)
                for (int v = 0; v < 8; v++)
                    o.rgi_tcoeff[b][v * 8 + u] = lv[b * 64 + u * 8 + v];
        if (m.type == H261B_MB_TYPE_INTRA)
            for (int b = 0; b < 6; b++)
                o.rgi_tcoeff[b][0] = (uint8_t)lv[b * 64];
        o.i_mb_x = (i % mbw) * 16;
        o.i_mb_y = (i / mbw) * 16;
    }
    return H261B_OK;
}

extern "C" int h261b_engine_last_kernel_ms(h261b_engine_t *e, float *ms)
{
    if (!e || !ms || e->next_step == 0)
        return H261B_ERR_ARG;
    const int p = (int)((e->next_step - 1) % NSLOT);
    H261B_CUDA_TRY(cudaEventSynchronize(e->k_end[p]));
    H261B_CUDA_TRY(cudaEventElapsedTime(ms, e->k_start[p], e->k_end[p]));
    return H261B_OK;
}

extern "C" int h261b_engine_last_copy_bytes(h261b_engine_t *e, int64_t *h2d, int64_t *d2h)
{
    if (!e || !h2d || !d2h)
        return H261B_ERR_ARG;
    *h2d = e->last_h2d;
    *d2h = e->last_d2h;
    return H261B_OK;
}

extern "C" int h261b_engine_last_bits_ms(h261b_engine_t *e, float *ms)
{
    if (!e || !ms || e->next_step == 0)
        return H261B_ERR_ARG;
    const int p = (int)((e->next_step - 1) % NSLOT);
    *ms = 0.f;
    if (!e->step_bits_ran[p])
        return H261B_OK;
    H261B_CUDA_TRY(cudaEventSynchronize(e->b_end[p]));
    H261B_CUDA_TRY(cudaEventElapsedTime(ms, e->k_end[p], e->b_end[p]));
    return H261B_OK;
}

extern "C" int h261b_engine_step_timing(h261b_engine_t *e, h261b_step_timing_t *t)
{
    clear_error();
    if (!e || !t)
        return H261B_ERR_ARG;
    if (e->done_step < 0) {
        set_error("h261b_engine_step_timing: no step has completed");
        return H261B_ERR_STATE;
    }
    const int p = (int)(e->done_step % NSLOT);
    float a = 0, b = 0, c = 0, d = 0, f = 0;
    H261B_CUDA_TRY(cudaEventElapsedTime(&a, e->t_begin[p], e->t_h2d[p]));
    H261B_CUDA_TRY(cudaEventElapsedTime(&b, e->t_h2d[p], e->t_ready[p]));
    H261B_CUDA_TRY(cudaEventElapsedTime(&c, e->k_start[p], e->k_end[p]));
    if (e->step_bits_ran[p])
        H261B_CUDA_TRY(cudaEventElapsedTime(&d, e->k_end[p], e->b_end[p]));
    H261B_CUDA_TRY(cudaEventElapsedTime(&f, e->t_begin[p], e->t_end[p]));
    t->step = e->done_step;
    t->upload_ms = a;
    t->wait_ms = b;
    t->encode_ms = c;
    t->bitstream_ms = d;
    t->total_ms = f;
    return H261B_OK;
}

extern "C" int h261b_engine_step_pictures(h261b_engine_t *e, int32_t cap, h261b_picture_t *out, int32_t *count,
                                          const uint8_t **arena, int64_t *arena_bytes)
{
    clear_error();
    if (!e || !count || (cap > 0 && !out) || cap < 0)
        return H261B_ERR_ARG;
    *count = 0;
    if (arena)
        *arena = nullptr;
    if (arena_bytes)
        *arena_bytes = 0;
    if (e->done_step < 0)
        return H261B_OK;
    const int p = (int)(e->done_step % NSLOT);
    const Mirror &rm = e->results[p];
    int64_t span = 0;
    int32_t n = 0;
    for (size_t i = 0; i < e->sessions.size(); i++) {
        const Session &s = e->sessions[i];
        const Result &r = s.res[p];
        if (!s.open || !r.has_bits || r.step != e->done_step)
            continue;
        const h261b_pic_info_t &pi = *(const h261b_pic_info_t *)(rm.host + r.pic_off);
        if (pi.status == 0 && pi.host_off >= 0)
            span = std::max<int64_t>(span, (int64_t)pi.host_off + ((pi.bytes + 15) & ~15));
        if (pi.status == 0 && pi.host_off < 0)
            e->bits_want = std::max(e->bits_want, 2 * e->bits[p].cap);   /* later steps fit */
        if (n < cap) {
            h261b_picture_t &o = out[n];
            o.session_id = (int32_t)i;
            o.frame_index = r.frame;
            o.bytes = pi.status == 0 ? pi.bytes : 0;
            o.status = pi.status == 0 ? (pi.host_off >= 0 ? 0 : 1) : H261B_ERR_STATE;
            o.bits = (pi.status == 0 && pi.host_off >= 0) ? e->bits[p].host + pi.host_off : nullptr;
        }
        n++;
    }
    *count = n;
    if (arena)
        *arena = e->bits[p].host;
    if (arena_bytes)
        *arena_bytes = span;
    return H261B_OK;
}

extern "C" int h261b_engine_graph_stats(h261b_engine_t *e, int64_t *captures, int64_t *replays)
{
    if (!e || !captures || !replays)
        return H261B_ERR_ARG;
    *captures = e->graph_captures;
    *replays = e->graph_replays;
    return H261B_OK;
}

extern "C" int h261b_engine_launch_shape(h261b_engine_t *e, int32_t *warps_per_cta, int32_t *max_ctas,
                                         int32_t *source)
{
    if (!e || !warps_per_cta || !max_ctas || !source)
        return H261B_ERR_ARG;
    *warps_per_cta = e->plan.warps;
    *max_ctas = e->plan.ctas;
    *source = e->shape_source;
    return H261B_OK;
}

static h261b_launch_plan_t plan_out(const LaunchPlan &p, int32_t source, int32_t tuning)
{
    h261b_launch_plan_t o;
    memset(&o, 0, sizeof(o));
    o.warps_per_cta = p.warps;
    o.max_ctas = p.ctas;
    o.kernel_split = p.split + 1;
    o.tail_items = p.tail + 1;
    o.staging = p.staging + 1;
    o.source = source;
    o.tuning = tuning;
    return o;
}

extern "C" int h261b_engine_plan(h261b_engine_t *e, h261b_launch_plan_t *plan, int32_t log_cap,
                                 h261b_launch_plan_t *log, float *log_ms, int32_t *log_count)
{
    if (!e || !plan || log_cap < 0 || (log_cap > 0 && (!log || !log_ms)))
        return H261B_ERR_ARG;
    *plan = plan_out(e->plan, e->shape_source, e->tuned ? 0 : 1);
    const std::vector<std::pair<LaunchPlan, float>> &lg = e->tuner.log;
    for (size_t i = 0; i < lg.size() && (int32_t)i < log_cap; i++) {
        log[i] = plan_out(lg[i].first, 1, 0);
        log_ms[i] = lg[i].second;
    }
    if (log_count)
        *log_count = (int32_t)lg.size();
    return H261B_OK;
}

extern "C" int h261b_engine_stats(h261b_engine_t *e, int32_t *open_sessions, int32_t *queued, int64_t *bytes)
{
    if (!e)
        return H261B_ERR_ARG;
    int32_t q = 0;
    for (const Session &s : e->sessions)
        q += s.open && s.queued;
    if (open_sessions)
        *open_sessions = e->open_count;
    if (queued)
        *queued = q;
    if (bytes)
        *bytes = e->pool.held();
    return H261B_OK;
}
