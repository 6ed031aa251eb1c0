// api.cu -- host side of libprzmgpu.so: contexts, the batch engine and the C
// ABI declared in include/przmgpu.h.  All kernels are compiled into this one
// translation unit.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdio>
#include <cstring>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/przmgpu.h"

#include "common.cuh"
#include "entropy.cu"
#include "dists.cu"
#include "fibers.cu"
#include "frame.cu"
#include "decode.cu"
#include "match.cu"
#include "tokenize.cu"
#include "front.cu"
#include "streams.cu"

using namespace pz;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;
static std::atomic<int> g_mock_unavailable{0};
static std::atomic<int> g_mock_match_err{0};

static int32_t fail(int32_t code, const std::string& msg) {
    g_err = msg;
    return code;
}
static int32_t cuda_fail(const char* what, cudaError_t e) {
    return fail(PRZMG_ERR_CUDA, std::string(what) + " failed with CUDA error " + std::to_string((int)e) + " (" +
                                    cudaGetErrorString(e) + ")");
}
#define CK(call)                                               \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_fail(#call, e_);    \
    } while (0)

extern "C" const char* przmg_last_error(void) { return g_err.c_str(); }

// ---------------------------------------------------------------------------
// grow-only device / pinned buffers
// ---------------------------------------------------------------------------
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        // geometric growth: a buffer that keeps growing is reallocated
        // O(log) times (cudaFree synchronises the device)
        size_t want = std::max(bytes + bytes / 8, cap + cap / 2) + 4096;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, want);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

struct HostBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t bytes) {
        if (bytes <= cap && p) return cudaSuccess;
        if (p) cudaFreeHost(p);
        p = nullptr;
        size_t want = std::max(bytes + bytes / 8, cap + cap / 2) + 4096;  // pinning is slow: grow geometrically
        cap = 0;
        cudaError_t e = cudaHostAlloc(&p, want, cudaHostAllocDefault);
        if (e == cudaSuccess) cap = want;
        return e;
    }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        cap = 0;
    }
    template <class T> T* as() const { return reinterpret_cast<T*>(p); }
};

static inline uint64_t align16(uint64_t v) { return (v + 15) & ~15ull; }
static inline uint64_t align64(uint64_t v) { return (v + 63) & ~63ull; }

extern "C" uint64_t przmg_frame_bound(uint64_t n) { return 2 * n + (n >> 13) + 4096; }

// ---------------------------------------------------------------------------
// batch engine
// ---------------------------------------------------------------------------
struct Ctx;

// Launch geometry of one size class (mean input size of a batch), chosen by
// the autotuner (przm_b200/autotune.py); never changes an output byte.
//   front        0: one kernel per front-end stage, 1: the persistent front end
//   ctas_per_sm  resident blocks per SM of the persistent front end
//   verify_chunk radix candidates per verify item of the persistent front end
struct Tuning {
    uint32_t front = 0, ctas_per_sm = 2, verify_chunk = 2048;
};
constexpr int kSizeClasses = 4;
// upper bounds of the mean input size of classes 0..2 (class 3: above)
constexpr uint64_t kClassBound[kSizeClasses - 1] = {64ull << 10, 768ull << 10, 2ull << 20};
static inline bool valid_profile(int32_t p) {
    return p == PRZMG_PROFILE_D2D || p == PRZMG_PROFILE_ANS || p == PRZMG_PROFILE_ANS_DIST || p == PRZMG_PROFILE_ANS_SHEAF;
}
static inline int size_class(uint64_t mean) {
    int k = 0;
    while (k < kSizeClasses - 1 && mean > kClassBound[k]) k++;
    return k;
}

struct przmg_batch {
    Ctx* ctx = nullptr;
    int profile = 1;
    bool force_radix = false;
    bool owned = false;  // created through przmg_batch_create
    uint32_t njobs = 0, ntiles = 0, nsmall = 0, nbig = 0;
    std::vector<Job> jobs;
    std::vector<TileRef> small;
    std::vector<uint32_t> big;
    std::vector<TokTile> tiles;
    std::vector<uint2> asm_items;  // every frame's part 0 first, then the literal parts
    std::vector<uint64_t> in_offs, out_offs, up_offs;
    uint64_t in_bytes = 0, desc_words = 0, stream_bytes = 0, ans_bytes = 0, out_bytes = 0;
    DevBuf d_in, d_jobs, d_small, d_big, d_tiles, d_desc, d_slots, d_tile_lens, d_streams, d_job_lens, d_hist, d_tabs,
        d_infos, d_ans, d_outs, d_plans, d_sizes, d_out, d_misc, d_lists;
    // radix-strike tables (one per finder CTA) and the packed upload/download
    // staging belong to the batch, so batches on different streams never
    // share scratch
    DevBuf d_rtiles, d_rx_toff, d_rx_list, d_rx_pred, d_stage_in, d_stage_out, d_stage_offs, d_up_offs;
    DevBuf d_tile_sched;  // tokenizer tile weights [0, ntiles) and walk order [ntiles, 2 ntiles)
    DevBuf d_asm;         // assembly work items (frame, part)
    DevBuf d_asm_job;     // the same items grouped by input (plain per-input launches)
    DevBuf d_s3, d_s3f;   // P2 and up: per-input Section 3 regions and their S3Frame facts
    DevBuf d_fib;         // P3: per-input fiber regions
    // P2 and up: the Mode 12 chains run on a second stream, forked after the
    // distance codes exist and joined before the plan (graph capture keeps
    // the two branches)
    cudaStream_t aux = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    // per input i, where its items start in each work list ([i + 1] = end)
    std::vector<uint32_t> job_small0, job_rt0, job_big0, job_tile0, job_asm0;
    int launches_plain = 0;
    // persistent front end (used when tune.front == 1 and every input has at
    // most 512 tiles): its work items, tile list and per-input tokenizer targets
    Tuning tune;
    bool front = false;
    uint32_t nfront = 0;
    DevBuf d_fitems, d_ftiles, d_ftarget, d_fctl;  // d_fctl: [0] next item, [16 ...] per-input progress
    HostBuf h_offs;
    std::vector<RxTile> rtiles;
    uint64_t max_big_cand = 0;  // most radix candidates of one frame
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches = 0;
    // the batch holds one input and its match table from a completed
    // one-input call (what the tokenizer-only entry points run on)
    bool staged_single = false;
    ~przmg_batch() {
        drop_graph();
        release();
        if (ev_fork) cudaEventDestroy(ev_fork);
        if (ev_join) cudaEventDestroy(ev_join);
        if (aux) cudaStreamDestroy(aux);
    }
    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    void release() {
        DevBuf* all[] = {&d_in, &d_jobs, &d_small, &d_big, &d_tiles, &d_desc, &d_slots, &d_tile_lens, &d_streams,
                         &d_job_lens, &d_hist, &d_tabs, &d_infos, &d_ans, &d_outs, &d_plans, &d_sizes, &d_out, &d_misc,
                         &d_lists, &d_rtiles, &d_rx_toff, &d_rx_list, &d_rx_pred, &d_stage_in,
                         &d_stage_out, &d_stage_offs, &d_up_offs, &d_tile_sched, &d_asm, &d_asm_job,
                         &d_fitems, &d_ftiles, &d_ftarget, &d_fctl, &d_s3, &d_s3f, &d_fib};
        for (DevBuf* b : all) b->release();
        h_offs.release();
    }
    uint32_t* err_word() const { return d_misc.as<uint32_t>(); }
};

// PinnedBufferPool (gpu/memory.go:91-165): a mutex-guarded stack of pinned
// host buffers of one size, at most max_cap of them kept.
struct przmg_pinned_pool {
    std::mutex mu;
    uint64_t buf_size = 0;
    size_t max_cap = 8;
    std::vector<void*> free_bufs;
    bool ctx_owned = false;  // created by GetPinned: the context frees it
    void free_all() {
        std::lock_guard<std::mutex> lk(mu);
        for (void* p : free_bufs) cudaFreeHost(p);
        free_bufs.clear();
    }
};

struct Ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::mutex mu;
    Tuning tune[kSizeClasses];
    uint64_t front_wait_ns = 1000000000ull;  // limit of one persistent front-end wait
    bool front_unreachable = false;          // test hook: add a wait that nothing ends
    int clock_khz = 1965000;
    std::mutex pools_mu;
    std::unordered_map<uint64_t, przmg_pinned_pool*> pools;  // GetPinned pools by power-of-two size
    cudaDeviceProp prop{};
    int sms = 148;
    DevBuf d_meta8, d_ctxlut;
    DevBuf d_dist12;  // Mode 12 static weights in EncSym form (4 x 64)
    przmg_batch single;  // reused by the one-input calls
    HostBuf h_in, h_out, h_aux;
    DevBuf d_scr_in, d_scr_out, d_scr_aux, d_scr_tab;
    DevBuf d_s3;   // scratch of przmg_package_offsets_batch
    DevBuf d_lit;  // scratch of przmg_package_literals_batch
    // the GPU decoder: static tables, per-frame scratch, jobs, results,
    // entropy tasks; przmg_batch_verify's decoded bytes and comparisons
    DevBuf d_dstatic, d_dscr, d_djobs, d_dinfo, d_dtasks, d_dout, d_ddiff;
    cudaStream_t dec_aux = nullptr;  // the decoder's static-model chains
    cudaEvent_t dec_fork = nullptr, dec_join = nullptr;
    cudaEvent_t ev[8] = {};
};

// Work items of the persistent front end in stage order, inputs largest
// first within a stage (their long rANS chains then start first), with each
// item's progress target: the number of items of its input in earlier
// stages.  Per input, large (radix) frames have nrt count items, 1 scan, nrt
// scatters, kFrontResolveItems resolves, nv verify chunks, then one item per
// tokenizer tile and one gather; small frames one tile-finder item per tile,
// then their tiles and the gather.
static void front_build(const przmg_batch* b, uint32_t chunk, bool unreachable, std::vector<FrontItem>& items,
                        std::vector<TokTile>& ftiles, std::vector<uint32_t>& tok_target) {
    const uint32_t nj = b->njobs;
    std::vector<uint32_t> ord(nj);
    for (uint32_t i = 0; i < nj; i++) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t x, uint32_t y) { return b->jobs[x].n > b->jobs[y].n; });
    items.clear();
    ftiles.clear();
    tok_target.assign(nj, 0);
    auto nrt = [&](uint32_t j) { return b->job_rt0[j + 1] - b->job_rt0[j]; };
    auto nv = [&](uint32_t j) { return (rx_ncand(b->jobs[j].n) + chunk - 1) / chunk; };
    auto big = [&](uint32_t j) { return b->job_big0[j + 1] > b->job_big0[j]; };
    for (uint32_t j : ord)
        for (uint32_t t = b->job_rt0[j]; t < b->job_rt0[j + 1]; t++) items.push_back({FS_RX_SORT, j, t, 0});
    for (uint32_t j : ord)
        for (uint32_t t = b->job_small0[j]; t < b->job_small0[j + 1]; t++) items.push_back({FS_TILE_FIND, j, t, 0});
    for (uint32_t j : ord)
        if (big(j))
            for (uint32_t g = 0; g < kFrontResolveItems; g++)
                items.push_back({FS_RX_RESOLVE, j, g * kFrontWarps, nrt(j)});
    for (uint32_t j : ord)
        if (big(j))
            for (uint32_t c = 0; c < nv(j); c++)
                items.push_back({FS_RX_VERIFY, j, c * chunk, nrt(j) + kFrontResolveItems});
    for (uint32_t j : ord) {
        const uint32_t nt = b->job_tile0[j + 1] - b->job_tile0[j];
        tok_target[j] = big(j) ? nrt(j) + kFrontResolveItems + nv(j) : nt;
        for (uint32_t t = b->job_tile0[j]; t < b->job_tile0[j + 1]; t++) ftiles.push_back(b->tiles[t]);
    }
    for (uint32_t t = 0; t < ftiles.size(); t += kFrontWarps)
        items.push_back({FS_TOKENIZE, std::min<uint32_t>(kFrontWarps, (uint32_t)ftiles.size() - t), t, 0});
    for (uint32_t j : ord) {
        const uint32_t nt = b->job_tile0[j + 1] - b->job_tile0[j];
        items.push_back({FS_GATHER, j, j, nt ? tok_target[j] + nt : 0});
    }
    if (unreachable && nj) items.push_back({FS_NOP, 0, 0, 0xFFFFFFFFu});
}

// Lay out a batch for the given input sizes; (re)allocates only when a
// buffer is too small, so repeated calls of similar size reuse memory.
static int32_t batch_prepare(przmg_batch* b, const uint64_t* sizes, uint32_t njobs, int profile, bool force_radix,
                             cudaStream_t setup = nullptr) {
    b->drop_graph();
    b->staged_single = false;
    b->profile = profile;
    b->force_radix = force_radix;
    b->njobs = njobs;
    b->jobs.assign(njobs, Job{});
    b->small.clear();
    b->big.clear();
    b->tiles.clear();
    b->rtiles.clear();
    b->max_big_cand = 0;
    b->in_offs.assign(njobs, 0);
    b->out_offs.assign(njobs, 0);
    uint64_t in = 0, desc = 0, str = 0, ans = 0, out = 0, s3 = 0, fib = 0;
    uint32_t tile0 = 0;
    for (auto* v : {&b->job_small0, &b->job_rt0, &b->job_big0, &b->job_tile0, &b->job_asm0}) v->assign(njobs + 1, 0);
    for (uint32_t i = 0; i < njobs; i++) {
        b->job_small0[i] = (uint32_t)b->small.size();
        b->job_rt0[i] = (uint32_t)b->rtiles.size();
        b->job_big0[i] = (uint32_t)b->big.size();
        b->job_tile0[i] = (uint32_t)b->tiles.size();
        Job& j = b->jobs[i];
        const uint64_t n = sizes[i];
        if (n >= (1ull << 32) - 4096) return fail(PRZMG_ERR_EXCEEDS_MAX_BLOCK, "input too large for one frame");
        j.n = (uint32_t)n;
        j.kind = (force_radix || n > kSmallMax) ? 1 : 0;
        j.ntiles = (uint32_t)std::max<uint64_t>(1, (n + kTile - 1) / kTile);
        j.tile0 = tile0;
        j.profile = (uint32_t)profile;
        j.in_off = in;
        b->in_offs[i] = in;
        in = align16(in + n + 64);
        j.desc_off = desc;
        const uint64_t ncand = n >= 8 ? (n - 8) / 8 + 1 : 0;
        desc += j.kind == 0 ? align16(n + 1) : align16(ncand + 1);
        j.cmd_cap = j.ntiles * kSlotCmd;
        j.off_cap = j.ntiles * kSlotOff;
        j.lit_cap = j.ntiles * kSlotLit;
        j.str_off = str;
        str += align16(stream_region_bytes(j));
        if (profile >= 2) {
            j.dist_cap = (uint32_t)(n / 4 + 64);
            j.s3_off = s3;
            s3 += align16(s3_region_bytes(j));
        }
        if (profile >= 3) {
            j.fib_off = fib;
            fib += align16(fib_region_bytes(j));
        }
        j.ans_off = ans;
        if (profile >= 1) ans += align16(ans_region_bytes(j));
        j.out_cap = (uint32_t)std::min<uint64_t>(przmg_frame_bound(n), 0xFFFFFFF0u);
        j.out_off = out;
        b->out_offs[i] = out;
        out = align16(out + j.out_cap);
        if (n > 0) {
            if (j.kind == 0) {
                for (uint32_t t = 0; t < j.ntiles; t++) b->small.push_back({i, t});
            } else {
                b->big.push_back(i);
                b->max_big_cand = std::max<uint64_t>(b->max_big_cand, ncand);
                const uint32_t nct = (uint32_t)((ncand + kCandPerTile - 1) / kCandPerTile);
                for (uint32_t t = 0; t < nct; t++) b->rtiles.push_back({i, t});
            }
            for (uint32_t t = 0; t < j.ntiles; t++) b->tiles.push_back({i, t});
        }
        tile0 += j.ntiles;
    }
    b->ntiles = tile0;
    b->nsmall = (uint32_t)b->small.size();
    b->nbig = (uint32_t)b->big.size();
    b->job_small0[njobs] = b->nsmall;
    b->job_rt0[njobs] = (uint32_t)b->rtiles.size();
    b->job_big0[njobs] = b->nbig;
    b->job_tile0[njobs] = (uint32_t)b->tiles.size();
    b->in_bytes = in + 64;
    b->asm_items.clear();
    for (uint32_t i = 0; i < njobs; i++) b->asm_items.push_back(make_uint2(i, 0));
    for (uint32_t i = 0; i < njobs; i++)
        for (uint32_t k = 0, np = asm_lit_parts(b->jobs[i]); k < np; k++) b->asm_items.push_back(make_uint2(i, k + 1));
    // the same items grouped by input, for per-input launches
    std::vector<uint2> asm_job;
    asm_job.reserve(b->asm_items.size());
    for (uint32_t i = 0; i < njobs; i++) {
        b->job_asm0[i] = (uint32_t)asm_job.size();
        for (uint32_t k = 0, np = asm_lit_parts(b->jobs[i]); k <= np; k++) asm_job.push_back(make_uint2(i, k));
    }
    b->job_asm0[njobs] = (uint32_t)asm_job.size();
    // launch geometry of this batch's size class; the persistent front end
    // needs every input within 512 tiles (its gather's shared tile offsets)
    uint64_t total_n = 0;
    uint32_t max_tiles = 0;
    for (uint32_t i = 0; i < njobs; i++) { total_n += b->jobs[i].n; max_tiles = std::max(max_tiles, b->jobs[i].ntiles); }
    b->tune = b->ctx->tune[size_class(njobs ? total_n / njobs : 0)];
    b->front = b->tune.front == 1 && njobs > 0 && max_tiles <= 512 && !force_radix;
    std::vector<FrontItem> fitems;
    std::vector<TokTile> ftiles;
    std::vector<uint32_t> ftarget;
    if (b->front)
        front_build(b, std::max<uint32_t>(256, b->tune.verify_chunk), b->ctx->front_unreachable, fitems, ftiles, ftarget);
    b->nfront = (uint32_t)fitems.size();
    b->desc_words = desc + 16;
    b->stream_bytes = str + 64;
    b->ans_bytes = ans + 64;
    b->out_bytes = out + 64;
    CK(b->d_in.ensure(b->in_bytes));
    CK(b->d_jobs.ensure(sizeof(Job) * std::max<uint32_t>(njobs, 1)));
    CK(b->d_small.ensure(sizeof(TileRef) * std::max<uint32_t>(b->nsmall, 1)));
    CK(b->d_big.ensure(sizeof(uint32_t) * std::max<uint32_t>(b->nbig, 1)));
    CK(b->d_tiles.ensure(sizeof(TokTile) * std::max<size_t>(b->tiles.size(), 1)));
    CK(b->d_tile_sched.ensure(2 * sizeof(uint32_t) * std::max<size_t>(b->tiles.size(), 1)));
    CK(b->d_asm.ensure(sizeof(uint2) * std::max<size_t>(b->asm_items.size(), 1)));
    CK(b->d_asm_job.ensure(sizeof(uint2) * std::max<size_t>(asm_job.size(), 1)));
    if (b->front) {
        CK(b->d_fitems.ensure(sizeof(FrontItem) * fitems.size()));
        CK(b->d_ftiles.ensure(sizeof(TokTile) * std::max<size_t>(ftiles.size(), 1)));
        CK(b->d_ftarget.ensure(4ull * njobs));
        CK(b->d_fctl.ensure(64 + 4ull * njobs));
    }
    CK(b->d_desc.ensure(b->desc_words * 4));
    CK(b->d_slots.ensure((size_t)b->ntiles * kSlotStride));
    CK(b->d_tile_lens.ensure((size_t)b->ntiles * S_COUNT * 4));
    CK(b->d_streams.ensure(b->stream_bytes));
    CK(b->d_job_lens.ensure((size_t)njobs * S_COUNT * 4 + 16));
    CK(b->d_hist.ensure((size_t)njobs * 1024 * 4 + 16));
    CK(b->d_tabs.ensure((size_t)njobs * kModels * 256 * sizeof(EncSym) + 16));
    CK(b->d_infos.ensure((size_t)njobs * kModels * sizeof(TableInfo) + 16));
    CK(b->d_s3.ensure(s3 + 64));
    CK(b->d_s3f.ensure(sizeof(S3Frame) * std::max<uint32_t>(njobs, 1)));
    CK(b->d_fib.ensure(fib + 64));
    if (profile >= 2 && !b->aux) {
        CK(cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking));
        CK(cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming));
    }
    CK(b->d_ans.ensure(b->ans_bytes));
    CK(b->d_outs.ensure((size_t)njobs * T_COUNT * sizeof(TaskOut) + 16));
    CK(b->d_plans.ensure((size_t)njobs * sizeof(Plan) + 16));
    CK(b->d_sizes.ensure((size_t)njobs * 4 + 16));
    CK(b->d_out.ensure(b->out_bytes));
    CK(b->d_misc.ensure(64));
    CK(b->d_lists.ensure((size_t)2 * kModels * std::max<uint32_t>(njobs, 1) * sizeof(TaskDesc) + 64));
    CK(b->d_up_offs.ensure(8ull * std::max<uint32_t>(njobs, 1) + 64));
    if (b->nbig) {
        CK(b->d_rtiles.ensure(sizeof(RxTile) * std::max<size_t>(b->rtiles.size(), 1)));
        CK(b->d_rx_toff.ensure((size_t)b->ntiles * kRxParts * 4 + 64));
        CK(b->d_rx_list.ensure(b->desc_words * 4));
        CK(b->d_rx_pred.ensure(b->desc_words * 4));
    }
    b->up_offs.assign(njobs, 0);
    for (uint32_t i = 1; i < njobs; i++) b->up_offs[i] = b->up_offs[i - 1] + b->jobs[i - 1].n;
    cudaStream_t s = setup ? setup : b->ctx->stream;
    if (njobs) CK(cudaMemcpyAsync(b->d_up_offs.p, b->up_offs.data(), 8ull * njobs, cudaMemcpyHostToDevice, s));
    if (!b->rtiles.empty())
        CK(cudaMemcpyAsync(b->d_rtiles.p, b->rtiles.data(), sizeof(RxTile) * b->rtiles.size(), cudaMemcpyHostToDevice, s));
    CK(cudaMemcpyAsync(b->d_jobs.p, b->jobs.data(), sizeof(Job) * njobs, cudaMemcpyHostToDevice, s));
    if (b->nsmall) CK(cudaMemcpyAsync(b->d_small.p, b->small.data(), sizeof(TileRef) * b->nsmall, cudaMemcpyHostToDevice, s));
    if (b->nbig) CK(cudaMemcpyAsync(b->d_big.p, b->big.data(), sizeof(uint32_t) * b->nbig, cudaMemcpyHostToDevice, s));
    if (!b->tiles.empty())
        CK(cudaMemcpyAsync(b->d_tiles.p, b->tiles.data(), sizeof(TokTile) * b->tiles.size(), cudaMemcpyHostToDevice, s));
    if (!b->asm_items.empty())
        CK(cudaMemcpyAsync(b->d_asm.p, b->asm_items.data(), sizeof(uint2) * b->asm_items.size(), cudaMemcpyHostToDevice, s));
    if (!asm_job.empty())
        CK(cudaMemcpyAsync(b->d_asm_job.p, asm_job.data(), sizeof(uint2) * asm_job.size(), cudaMemcpyHostToDevice, s));
    if (b->front) {
        CK(cudaMemcpyAsync(b->d_fitems.p, fitems.data(), sizeof(FrontItem) * fitems.size(), cudaMemcpyHostToDevice, s));
        if (!ftiles.empty())
            CK(cudaMemcpyAsync(b->d_ftiles.p, ftiles.data(), sizeof(TokTile) * ftiles.size(), cudaMemcpyHostToDevice, s));
        CK(cudaMemcpyAsync(b->d_ftarget.p, ftarget.data(), 4ull * njobs, cudaMemcpyHostToDevice, s));
    }
    CK(cudaMemsetAsync(b->d_sizes.p, 0, (size_t)njobs * 4 + 16, s));
    CK(cudaMemsetAsync(b->d_job_lens.p, 0, (size_t)njobs * S_COUNT * 4 + 16, s));
    // the host-side vectors above must stay alive until the copies ran
    CK(cudaStreamSynchronize(s));
    return PRZMG_OK;
}

// Stages of one enqueue.  stop_after: 0 match only, 1 through tokenize +
// gather, 2 the full frame pipeline.
static const char* const kStageNames[] = {"tile_find", "radix_find", "tokenize", "gather", "front",
                                          "normalize", "rans", "plan", "assemble"};
constexpr int kStages = 9;

// The part of a batch one launch sequence covers: inputs [j0, j0 + nj) and
// the matching runs of the batch's work lists (every list is ordered by
// input, so one input's items are contiguous).
struct Range {
    uint32_t j0, nj;
    uint32_t small0, nsmall;  // tile-finder tiles
    uint32_t rt0, nrt;        // radix tiles
    uint32_t big0, nbig;      // radix frames
    uint32_t tile0, nt;       // tokenizer tiles
    uint32_t asm0, nasm;      // assembly items (of d_asm, or of d_asm_job for one input)
    const uint2* asm_list;
    uint32_t maxtiles;
    uint64_t max_big_cand;
};

static Range whole_range(const przmg_batch* b) {
    Range r{};
    r.j0 = 0;
    r.nj = b->njobs;
    r.nsmall = b->nsmall;
    r.nrt = (uint32_t)b->rtiles.size();
    r.nbig = b->nbig;
    r.nt = (uint32_t)b->tiles.size();
    r.nasm = (uint32_t)b->asm_items.size();
    r.asm_list = b->d_asm.as<uint2>();
    r.maxtiles = 1;
    for (const Job& j : b->jobs) r.maxtiles = std::max(r.maxtiles, j.ntiles);
    r.max_big_cand = b->max_big_cand;
    return r;
}

static Range job_range(const przmg_batch* b, uint32_t i) {
    Range r{};
    r.j0 = i;
    r.nj = 1;
    r.small0 = b->job_small0[i];
    r.nsmall = b->job_small0[i + 1] - r.small0;
    r.rt0 = b->job_rt0[i];
    r.nrt = b->job_rt0[i + 1] - r.rt0;
    r.big0 = b->job_big0[i];
    r.nbig = b->job_big0[i + 1] - r.big0;
    r.tile0 = b->job_tile0[i];
    r.nt = b->job_tile0[i + 1] - r.tile0;
    r.asm0 = b->job_asm0[i];
    r.nasm = b->job_asm0[i + 1] - r.asm0;
    r.asm_list = b->d_asm_job.as<uint2>();
    r.maxtiles = std::max<uint32_t>(1, b->jobs[i].ntiles);
    r.max_big_cand = rx_ncand(b->jobs[i].n);
    return r;
}

// ev (optional): kStages + 1 events; ev[0] before the first kernel and
// ev[k + 1] after stage k (stages that do not run record back to back).
// skip_match: the match table is already in d_desc (tokenizer-only runs).
// use_front: match, tokenize and gather of the whole batch in one launch of
// the persistent front end (stages 0-3 then record back to back).
static int32_t launch_range(przmg_batch* b, cudaStream_t s, int stop_after, const Range& R, cudaEvent_t* ev,
                            bool skip_match, bool use_front, int& launches) {
    Ctx* c = b->ctx;
    auto mark = [&](int k) -> cudaError_t { return ev ? cudaEventRecord(ev[k], s) : cudaSuccess; };
    CK(mark(0));
    if (use_front) {
        for (int k = 1; k <= 4; k++) CK(mark(k));
        CK(cudaMemsetAsync(b->d_fctl.p, 0, 64 + 4ull * b->njobs, s));
        FrontArgs a;
        a.in = b->d_in.as<uint8_t>();
        a.jobs = b->d_jobs.as<Job>();
        a.items = b->d_fitems.as<FrontItem>();
        a.nitems = b->nfront;
        a.head = b->d_fctl.as<uint32_t>();
        a.progress = b->d_fctl.as<uint32_t>() + 16;
        a.err = b->err_word();
        a.tok_target = b->d_ftarget.as<uint32_t>();
        a.wait_cycles = (long long)((double)c->front_wait_ns * c->clock_khz / 1e6);
        a.small = b->d_small.as<TileRef>();
        a.rtiles = b->d_rtiles.as<RxTile>();
        a.tiles = b->d_ftiles.as<TokTile>();
        a.ntiles = (uint32_t)b->tiles.size();
        a.verify_chunk = std::max<uint32_t>(256, b->tune.verify_chunk);
        a.desc = b->d_desc.as<uint32_t>();
        a.rx_toff = b->d_rx_toff.as<uint32_t>();
        a.rx_list = b->d_rx_list.as<uint32_t>();
        a.rx_pred = b->d_rx_pred.as<uint32_t>();
        a.slots = b->d_slots.as<uint8_t>();
        a.tile_lens = b->d_tile_lens.as<uint32_t>();
        a.streams = b->d_streams.as<uint8_t>();
        a.job_lens = b->d_job_lens.as<uint32_t>();
        a.hist = b->d_hist.as<uint32_t>();
        const uint32_t grid = std::max<uint32_t>(1, std::min<uint32_t>(b->nfront, std::max<uint32_t>(1, b->tune.ctas_per_sm) * c->sms));
        k_front<<<grid, kFrontThreads, kFrontSmem, s>>>(a);
        CK(cudaGetLastError());
        launches++;
        CK(mark(5));
    } else {
    if (R.nsmall && !skip_match) {
        const uint32_t grid = std::min<uint32_t>(R.nsmall, 8u * c->sms);
        k_tile_find<<<grid, 256, kTileFindSmem, s>>>(b->d_in.as<uint8_t>(), b->d_jobs.as<Job>(),
                                                     b->d_small.as<TileRef>() + R.small0, R.nsmall,
                                                     b->d_desc.as<uint32_t>(), b->err_word());
        CK(cudaGetLastError());
        launches++;
    }
    CK(mark(1));
    if (R.nbig && R.nrt && !skip_match) {
        const uint32_t gt = std::min<uint32_t>(R.nrt, 16u * c->sms);
        const RxTile* rt = b->d_rtiles.as<RxTile>() + R.rt0;
        const uint32_t* big = b->d_big.as<uint32_t>() + R.big0;
        k_rx_sort<<<gt, 256, 0, s>>>(b->d_in.as<uint8_t>(), b->d_jobs.as<Job>(), rt, R.nrt, b->d_rx_toff.as<uint32_t>(),
                                     b->d_rx_list.as<uint32_t>());
        CK(cudaGetLastError());
        const uint32_t nwarps = R.nbig * kRxParts;
        // one block per 8 partitions: partitions differ in size, so the
        // hardware's block scheduling balances the SMs (3 blocks fit per SM)
        const uint32_t gr = (nwarps + kRxResolveWarps - 1) / kRxResolveWarps;
        k_rx_resolve<<<gr, kRxResolveWarps * 32, kRxResolveSmem, s>>>(
            b->d_jobs.as<Job>(), big, R.nbig, b->d_rx_toff.as<uint32_t>(), b->d_rx_list.as<uint32_t>(),
            b->d_rx_pred.as<uint32_t>());
        CK(cudaGetLastError());
        const uint32_t vx = std::max<uint32_t>(1, std::min<uint32_t>(64u, (uint32_t)((R.max_big_cand + 255) / 256)));
        k_rx_verify<<<dim3(vx, std::min<uint32_t>(R.nbig, 65535u)), 256, 0, s>>>(
            b->d_in.as<uint8_t>(), b->d_jobs.as<Job>(), big, b->d_rx_list.as<uint32_t>(), b->d_rx_pred.as<uint32_t>(),
            R.nbig, b->d_desc.as<uint32_t>());
        CK(cudaGetLastError());
        launches += 3;
    }
    CK(mark(2));
    if (stop_after >= 1 && R.nt) {
        const uint32_t nt = R.nt;
        uint32_t* tile_w = b->d_tile_sched.as<uint32_t>() + R.tile0;
        uint32_t* tile_order = b->d_tile_sched.as<uint32_t>() + b->tiles.size() + R.tile0;
        const TokTile* tiles = b->d_tiles.as<TokTile>() + R.tile0;
        k_tile_weight<<<std::min<uint32_t>(nt, 16u * c->sms), 256, 0, s>>>(b->d_jobs.as<Job>(), tiles, nt,
                                                                          b->d_desc.as<uint32_t>(), tile_w);
        CK(cudaGetLastError());
        k_tile_order<<<1, 1024, 0, s>>>(tile_w, nt, tile_order);
        CK(cudaGetLastError());
        k_tokenize<<<(nt + kTokWarps - 1) / kTokWarps, kTokWarps * 32, 0, s>>>(
            b->d_in.as<uint8_t>(), b->d_jobs.as<Job>(), tiles, nt, tile_order, b->d_desc.as<uint32_t>(),
            b->d_slots.as<uint8_t>(), b->d_tile_lens.as<uint32_t>(), b->err_word());
        CK(cudaGetLastError());
        CK(mark(3));
        k_gather<<<std::min<uint32_t>(R.nj, 16u * c->sms), kGatherThreads, (R.maxtiles + 1) * 4, s>>>(
            b->d_jobs.as<Job>(), R.j0, R.nj, b->d_slots.as<uint8_t>(), b->d_tile_lens.as<uint32_t>(),
            b->d_streams.as<uint8_t>(), b->d_job_lens.as<uint32_t>(), b->d_hist.as<uint32_t>(), b->err_word());
        CK(cudaGetLastError());
        launches += 4;
    } else {
        CK(mark(3));
    }
    CK(mark(4));
    CK(mark(5));
    }
    if (stop_after >= 2 && R.nj) {
        if (b->profile >= 1) {
            if (b->profile >= 2) {  // Section 3: the distances' codes, extra bits and histogram
                k_s3_frame<<<R.nj, kS3Threads, 0, s>>>(b->d_jobs.as<Job>(), R.j0, b->d_job_lens.as<uint32_t>(),
                                                      b->d_streams.as<uint8_t>(), b->d_s3.as<uint8_t>(),
                                                      b->d_s3f.as<S3Frame>(), b->err_word());
                CK(cudaGetLastError());
                launches++;
                // the Mode 12 chains (one thread per frame, serial by the
                // format) on the second stream, beside the rANS launch
                CK(cudaEventRecord(b->ev_fork, s));
                CK(cudaStreamWaitEvent(b->aux, b->ev_fork, 0));
                k_s3_chain<<<(R.nj + 31) / 32, 32, 0, b->aux>>>(b->d_jobs.as<Job>(), R.j0, R.nj, b->d_s3.as<uint8_t>(),
                                                               b->d_s3f.as<S3Frame>(), c->d_dist12.as<EncSym>());
                CK(cudaGetLastError());
                CK(cudaEventRecord(b->ev_join, b->aux));
                launches++;
            }
            if (b->profile >= 3) {  // Section 4: the literals' four foliations
                k_frame_fibers<<<dim3(R.nj, 4), kFibThreads, 0, s>>>(b->d_jobs.as<Job>(), R.j0, b->d_job_lens.as<uint32_t>(),
                                                             b->d_streams.as<uint8_t>(), b->d_fib.as<uint8_t>());
                CK(cudaGetLastError());
                launches++;
            }
            k_normalize<<<R.nj, 32 * kModels, 0, s>>>(b->d_jobs.as<Job>(), R.j0, b->d_hist.as<uint32_t>(),
                                                      b->d_s3.as<uint8_t>(), b->d_s3f.as<S3Frame>(),
                                                      b->d_fib.as<uint8_t>(), b->d_tabs.as<EncSym>(),
                                                      b->d_infos.as<TableInfo>());
            CK(cudaGetLastError());
            CK(mark(6));
            const uint32_t list_cap = kModels * b->njobs;
            TaskDesc* lists = b->d_lists.as<TaskDesc>();
            uint32_t* counts = reinterpret_cast<uint32_t*>(lists + 2 * list_cap);
            k_task_list<<<1, 1024, 0, s>>>(b->d_jobs.as<Job>(), R.j0, R.nj, b->d_job_lens.as<uint32_t>(),
                                           b->d_s3f.as<S3Frame>(), b->d_streams.as<uint8_t>(), b->d_s3.as<uint8_t>(),
                                           b->d_fib.as<uint8_t>(), b->d_ans.as<uint8_t>(), lists, list_cap, counts);
            CK(cudaGetLastError());
            const uint32_t nad = (b->profile >= 3 ? kModels : b->profile >= 2 ? 5 : 4) * R.nj;  // adaptive tasks at most
            const uint32_t nb_ad = (nad + 8 * kRansWarps - 1) / (8 * kRansWarps);
            const uint32_t nb_m8 = (3 * R.nj + 8 * kRansWarps - 1) / (8 * kRansWarps);
            k_rans<<<nb_ad + nb_m8, kRansWarps * 32, kRansSmem, s>>>(lists, list_cap, counts, nb_ad,
                                                                    b->d_tabs.as<EncSym>(), c->d_meta8.as<EncSym>(),
                                                                    c->d_ctxlut.as<uint8_t>(), b->d_outs.as<TaskOut>());
            CK(cudaGetLastError());
            launches += 3;
            if (b->profile >= 2) CK(cudaStreamWaitEvent(s, b->ev_join, 0));  // the Mode 12 chains
            CK(mark(7));
        } else {
            CK(mark(6));
            CK(mark(7));
        }
        k_plan<<<(R.nj + 127) / 128, 128, 0, s>>>(b->d_jobs.as<Job>(), R.j0, R.nj, b->d_job_lens.as<uint32_t>(),
                                                  b->d_infos.as<TableInfo>(), b->d_outs.as<TaskOut>(),
                                                  b->d_streams.as<uint8_t>(), b->d_s3f.as<S3Frame>(),
                                                  b->d_fib.as<uint8_t>(), b->d_plans.as<Plan>(),
                                                  b->d_sizes.as<uint32_t>());
        CK(cudaGetLastError());
        CK(mark(8));
        k_assemble<<<std::max<uint32_t>(1, std::min<uint32_t>(R.nasm, 1u << 20)), kAsmThreads, 0, s>>>(
            b->d_in.as<uint8_t>(), b->d_jobs.as<Job>(), R.asm_list + R.asm0, R.nasm, b->d_job_lens.as<uint32_t>(),
            b->d_plans.as<Plan>(), b->d_infos.as<TableInfo>(), b->d_outs.as<TaskOut>(), b->d_streams.as<uint8_t>(),
            b->d_ans.as<uint8_t>(), b->d_s3.as<uint8_t>(), b->d_s3f.as<S3Frame>(), b->d_fib.as<uint8_t>(),
            b->d_out.as<uint8_t>());
        CK(cudaGetLastError());
        launches += 2;
        CK(mark(9));
    } else {
        for (int k = 6; k <= 9; k++) CK(mark(k));
    }
    return PRZMG_OK;
}

// The whole batch as one launch sequence.
static int32_t batch_launch(przmg_batch* b, cudaStream_t s, int stop_after, cudaEvent_t* ev = nullptr,
                            bool skip_match = false) {
    CK(cudaMemsetAsync(b->d_misc.p, 0, 16, s));
    int launches = 0;
    const bool use_front = b->front && stop_after >= 1 && !skip_match;
    int32_t r = launch_range(b, s, stop_after, whole_range(b), ev, skip_match, use_front, launches);
    b->launches = launches;
    return r;
}

// Plain per-input launches: the same pipeline once per input, one input
// after another on one stream (what a caller without batching does).
static int32_t batch_launch_plain(przmg_batch* b, cudaStream_t s) {
    CK(cudaMemsetAsync(b->d_misc.p, 0, 16, s));
    int launches = 0;
    for (uint32_t i = 0; i < b->njobs; i++) {
        if (b->jobs[i].n == 0) continue;
        int32_t r = launch_range(b, s, 2, job_range(b, i), nullptr, false, false, launches);
        if (r) return r;
    }
    b->launches_plain = launches;
    return PRZMG_OK;
}

static int32_t device_error(uint32_t err) {
    if (err & E_COPY_TIMEOUT)
        return fail(PRZMG_ERR_DEVICE, "a bulk copy into shared memory did not complete within its wait limit (error bits " +
                                          std::to_string(err) + ")");
    if (err & E_SCHED_TIMEOUT)
        return fail(PRZMG_ERR_DEVICE, "a wait of the persistent front end ran past its limit (error bits " +
                                          std::to_string(err) + "); the batch's frames are not valid");
    return fail(PRZMG_ERR_DEVICE, "device bound violation, error bits " + std::to_string(err));
}

static int32_t batch_check(przmg_batch* b) {
    uint32_t err = 0;
    CK(cudaMemcpyAsync(&err, b->err_word(), 4, cudaMemcpyDeviceToHost, b->ctx->stream));
    CK(cudaStreamSynchronize(b->ctx->stream));
    if (err) return device_error(err);
    return PRZMG_OK;
}

// ---------------------------------------------------------------------------
// context lifetime
// ---------------------------------------------------------------------------
static std::mutex g_global_mu;
static Ctx* g_global = nullptr;

extern "C" int32_t przmg_is_available(void) {
    if (g_mock_unavailable.load()) return 0;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) return 0;
    for (int i = 0; i < n; i++) {
        int major = 0;
        if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, i) == cudaSuccess && major >= 10) return 1;
    }
    return 0;
}

static int32_t ctx_setup(Ctx* c) {
    CK(cudaSetDevice(c->device));
    CK(cudaGetDeviceProperties(&c->prop, c->device));
    if (c->prop.major < 10) return fail(PRZMG_ERR_UNAVAILABLE, "compute capability 10.x (B200, sm_100a) required");
    c->sms = c->prop.multiProcessorCount;
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    for (auto& e : c->ev) CK(cudaEventCreate(&e));
    CK(cudaFuncSetAttribute(k_tile_find, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileFindSmem));
    CK(cudaFuncSetAttribute(k_rx_resolve, cudaFuncAttributeMaxDynamicSharedMemorySize, kRxResolveSmem));
    CK(cudaFuncSetAttribute(k_rans, cudaFuncAttributeMaxDynamicSharedMemorySize, kRansSmem));
    CK(cudaFuncSetAttribute(k_front, cudaFuncAttributeMaxDynamicSharedMemorySize, kFrontSmem));
    CK(cudaDeviceGetAttribute(&c->clock_khz, cudaDevAttrClockRate, c->device));
    CK(cudaFuncSetAttribute(k_stream_rans, cudaFuncAttributeMaxDynamicSharedMemorySize, kRansSmem));
    CK(c->d_meta8.ensure(8 * 256 * sizeof(EncSym)));
    CK(c->d_ctxlut.ensure(256));
    {
        std::vector<EncSym> tab(8 * 256);
        std::vector<uint8_t> lut(256);
        build_meta8_tables(tab.data(), lut.data());
        CK(cudaMemcpy(c->d_meta8.p, tab.data(), tab.size() * sizeof(EncSym), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(c->d_ctxlut.p, lut.data(), 256, cudaMemcpyHostToDevice));
        std::vector<EncSym> t12(4 * 64);
        for (int k = 0; k < 4; k++)
            for (uint32_t sym = 0, cum = 0; sym < 64; sym++) {
                t12[k * 64 + sym] = make_encsym(przm_dist_freq4[k][sym], cum);
                cum += przm_dist_freq4[k][sym];
            }
        CK(c->d_dist12.ensure(t12.size() * sizeof(EncSym)));
        CK(cudaMemcpy(c->d_dist12.p, t12.data(), t12.size() * sizeof(EncSym), cudaMemcpyHostToDevice));
    }
    c->single.ctx = c;
    CK(cudaStreamSynchronize(c->stream));
    return PRZMG_OK;
}

extern "C" int32_t przmg_init(int32_t device, przmg_ctx** out) {
    if (!out) return fail(PRZMG_ERR_INVALID_ARG, "null output pointer");
    *out = nullptr;
    if (!przmg_is_available()) return fail(PRZMG_ERR_UNAVAILABLE, "cuda gpu acceleration not available");
    Ctx* c = new Ctx();
    c->device = device;
    int32_t r = ctx_setup(c);
    if (r) {
        delete c;
        return r;
    }
    *out = reinterpret_cast<przmg_ctx*>(c);
    return PRZMG_OK;
}

extern "C" int32_t przmg_close(przmg_ctx* h) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c) return PRZMG_OK;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
        c->single.drop_graph();
        c->single.release();
        DevBuf* bufs[] = {&c->d_meta8, &c->d_ctxlut, &c->d_dist12, &c->d_scr_in, &c->d_scr_out, &c->d_scr_aux,
                          &c->d_scr_tab, &c->d_s3, &c->d_lit, &c->d_dstatic, &c->d_dscr, &c->d_djobs,
                          &c->d_dinfo, &c->d_dtasks, &c->d_dout, &c->d_ddiff};
        for (DevBuf* b : bufs) b->release();
        c->h_in.release();
        c->h_out.release();
        c->h_aux.release();
        for (auto& e : c->ev) if (e) cudaEventDestroy(e);
        if (c->dec_fork) cudaEventDestroy(c->dec_fork);
        if (c->dec_join) cudaEventDestroy(c->dec_join);
        if (c->dec_aux) cudaStreamDestroy(c->dec_aux);
        cudaStreamDestroy(c->stream);
    }
    {
        std::lock_guard<std::mutex> lk(c->pools_mu);
        for (auto& kv : c->pools) {
            kv.second->free_all();
            delete kv.second;
        }
        c->pools.clear();
    }
    {
        std::lock_guard<std::mutex> g(g_global_mu);
        if (g_global == c) g_global = nullptr;
    }
    delete c;
    return PRZMG_OK;
}

extern "C" int32_t przmg_get_global(przmg_ctx** out) {
    if (!out) return fail(PRZMG_ERR_INVALID_ARG, "null output pointer");
    std::lock_guard<std::mutex> g(g_global_mu);
    if (g_global) { *out = reinterpret_cast<przmg_ctx*>(g_global); return PRZMG_OK; }
    if (!przmg_is_available()) return fail(PRZMG_ERR_UNAVAILABLE, "cuda gpu acceleration not available or compute capability < 10.0");
    przmg_ctx* c = nullptr;
    g_global_mu.unlock();
    int32_t r = przmg_init(0, &c);
    g_global_mu.lock();
    if (r) return r;
    if (g_global) {  // another thread won the race
        g_global_mu.unlock();
        przmg_close(c);
        g_global_mu.lock();
    } else {
        g_global = reinterpret_cast<Ctx*>(c);
    }
    *out = reinterpret_cast<przmg_ctx*>(g_global);
    return PRZMG_OK;
}

extern "C" void przmg_reset_global_for_test(void) {
    Ctx* c;
    {
        std::lock_guard<std::mutex> g(g_global_mu);
        c = g_global;
        g_global = nullptr;
    }
    if (c) przmg_close(reinterpret_cast<przmg_ctx*>(c));
}

extern "C" void przmg_set_mock_unavailable(int32_t v) { g_mock_unavailable.store(v ? 1 : 0); }
extern "C" void przmg_set_mock_match_error(int32_t code) { g_mock_match_err.store(code); }

static int32_t mock_check() {
    int m = g_mock_match_err.load();
    if (m) return fail(PRZMG_ERR_MOCK, "mock match error " + std::to_string(m));
    return PRZMG_OK;
}

extern "C" int32_t przmg_device_info(przmg_ctx* h, int32_t* major, int32_t* minor, char* name, size_t name_cap,
                                     int32_t* sm_count, uint64_t* total_vram) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c) return fail(PRZMG_ERR_INVALID_ARG, "null context");
    if (major) *major = c->prop.major;
    if (minor) *minor = c->prop.minor;
    if (name && name_cap) { std::snprintf(name, name_cap, "%s", c->prop.name); }
    if (sm_count) *sm_count = c->sms;
    if (total_vram) *total_vram = c->prop.totalGlobalMem;
    return PRZMG_OK;
}

static void fill_profile(Ctx* c, przmg_profile_t* p) {
    if (!p) return;
    std::snprintf(p->device_name, sizeof p->device_name, "%.127s", c->prop.name);
    p->sm_count = c->sms;
    p->total_vram_bytes = c->prop.totalGlobalMem;
    if (p->pipelined_chunks == 0) p->pipelined_chunks = 1;
}

static float ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}
static double gbps(double bytes, double ms) { return ms > 0 ? bytes / (ms / 1000.0) / 1e9 : 0; }

#define LOCKED(c)                                  \
    std::lock_guard<std::mutex> lk_((c)->mu);      \
    CK(cudaSetDevice((c)->device))

// ---------------------------------------------------------------------------
// one-input compress / tokenize
// ---------------------------------------------------------------------------
static int32_t single_run(Ctx* c, const uint8_t* src, uint64_t n, int profile, int stop_after, bool force_radix,
                          przmg_profile_t* prof) {
    przmg_batch* b = &c->single;
    int32_t r = batch_prepare(b, &n, 1, profile, force_radix);
    if (r) return r;
    CK(c->h_in.ensure(n + 64));
    std::memcpy(c->h_in.p, src, n);
    CK(cudaEventRecord(c->ev[0], c->stream));
    CK(cudaMemcpyAsync(b->d_in.p, c->h_in.p, n, cudaMemcpyHostToDevice, c->stream));
    CK(cudaEventRecord(c->ev[1], c->stream));
    r = batch_launch(b, c->stream, stop_after);
    if (r) return r;
    CK(cudaEventRecord(c->ev[2], c->stream));
    r = batch_check(b);
    if (r) return r;
    b->staged_single = true;
    if (prof) {
        *prof = przmg_profile_t{};
        prof->ingress_dma_bytes = n;
        prof->ingress_dma_time_ms = ev_ms(c->ev[0], c->ev[1]);
        prof->ingress_dma_bandwidth_gbps = gbps((double)n, prof->ingress_dma_time_ms);
        prof->kernel_time_ms = ev_ms(c->ev[1], c->ev[2]);
        prof->internal_vram_bandwidth_gbps = gbps((double)n, prof->kernel_time_ms);
    }
    return PRZMG_OK;
}

static int32_t compress_one(Ctx* c, const uint8_t* src, uint64_t n, int profile, uint8_t* dst, uint64_t cap,
                            uint64_t* out_len, przmg_profile_t* prof) {
    if (out_len) *out_len = 0;
    if (n == 0) { if (prof) { *prof = przmg_profile_t{}; fill_profile(c, prof); } return PRZMG_OK; }
    if (!src || !dst || !out_len) return fail(PRZMG_ERR_INVALID_ARG, "null buffer");
    if (profile >= PRZMG_PROFILE_ANS && n >= (1u << 24))
        return fail(PRZMG_ERR_EXCEEDS_MAX_BLOCK, "the frame header holds 24-bit sizes: input must be < 16 MiB");
    int32_t r = single_run(c, src, n, profile, 2, false, prof);
    if (r) return r;
    przmg_batch* b = &c->single;
    uint32_t size = 0;
    CK(cudaMemcpyAsync(&size, b->d_sizes.p, 4, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (size > cap) return fail(PRZMG_ERR_BUFFER_TOO_SMALL, "destination too small for the frame");
    CK(c->h_out.ensure(size + 16));
    CK(cudaEventRecord(c->ev[3], c->stream));
    CK(cudaMemcpyAsync(c->h_out.p, b->d_out.p, size, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaEventRecord(c->ev[4], c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memcpy(dst, c->h_out.p, size);
    *out_len = size;
    if (prof) {
        prof->egress_dma_bytes = size;
        prof->egress_dma_time_ms = ev_ms(c->ev[3], c->ev[4]);
        prof->egress_dma_bandwidth_gbps = gbps((double)size, prof->egress_dma_time_ms);
        prof->total_round_trip_ms = ev_ms(c->ev[0], c->ev[4]);
        prof->end_to_end_bandwidth_gbps = gbps((double)n, prof->total_round_trip_ms);
        if (prof->total_round_trip_ms > 0)
            prof->pcie_overhead_percent = 100.0 * (prof->ingress_dma_time_ms + prof->egress_dma_time_ms) / prof->total_round_trip_ms;
        fill_profile(c, prof);
    }
    return PRZMG_OK;
}

extern "C" int32_t przmg_compress_d2d(przmg_ctx* h, const uint8_t* src, uint64_t n, uint8_t* dst, uint64_t cap,
                                      uint64_t* out_len, przmg_profile_t* prof) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c) return fail(PRZMG_ERR_INVALID_ARG, "null context");
    if (int32_t m = mock_check()) return m;
    LOCKED(c);
    return compress_one(c, src, n, PRZMG_PROFILE_D2D, dst, cap, out_len, prof);
}

extern "C" int32_t przmg_compress(przmg_ctx* h, const uint8_t* src, uint64_t n, int32_t profile, uint8_t* dst,
                                  uint64_t cap, uint64_t* out_len, przmg_profile_t* prof) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c) return fail(PRZMG_ERR_INVALID_ARG, "null context");
    if (!valid_profile(profile)) return fail(PRZMG_ERR_INVALID_ARG, "unknown profile");
    if (int32_t m = mock_check()) return m;
    LOCKED(c);
    return compress_one(c, src, n, profile, dst, cap, out_len, prof);
}

// src != null: stage src and run match + tokenize; src == null: tokenize
// again the input and match table staged by the last one-input call
// (TokenizeDeviceOnly, gpu/bridge.go:1915-1940).
static int32_t tokenize_common(Ctx* c, const uint8_t* src, uint64_t n, przmg_tokenizer_profile_t* prof, uint32_t lens6[6]) {
    przmg_batch* b = &c->single;
    if (src) {
        int32_t r = single_run(c, src, n, PRZMG_PROFILE_D2D, 1, false, nullptr);
        if (r) return r;
    } else {
        if (!b->staged_single || b->njobs != 1 || b->jobs[0].n != n)
            return fail(PRZMG_ERR_INVALID_ARG, "no staged input of " + std::to_string(n) +
                                                   " bytes: the tokenizer-only calls run on the input of the last "
                                                   "one-input call (przmg_tokenize, przmg_match_table, ...)");
        CK(cudaEventRecord(c->ev[0], c->stream));
        CK(cudaEventRecord(c->ev[1], c->stream));
        int32_t r = batch_launch(b, c->stream, 1, nullptr, true);
        if (r) return r;
        CK(cudaEventRecord(c->ev[2], c->stream));
        r = batch_check(b);
        if (r) return r;
    }
    CK(cudaMemcpyAsync(lens6, b->d_job_lens.p, 24, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (prof) {
        *prof = przmg_tokenizer_profile_t{};
        prof->kernel_time_ms = ev_ms(c->ev[1], c->ev[2]);
        prof->pass1_ms = prof->kernel_time_ms;
        prof->total_round_trip_ms = ev_ms(c->ev[0], c->ev[2]);
        prof->throughput_gbps = gbps((double)n, prof->kernel_time_ms);
        prof->cmd_bytes = lens6[S_CMD];
        prof->offset_bytes = lens6[S_OFF];
        prof->literal_bytes = lens6[S_LIT];
        prof->num_chunks = (n + kTile - 1) / kTile;
    }
    return PRZMG_OK;
}

static int32_t tokenize_to_host(Ctx* c, const uint8_t* src, uint64_t n, uint8_t* cmd, uint64_t cmd_cap, uint8_t* off,
                                uint64_t off_cap, uint8_t* lit, uint64_t lit_cap, uint64_t lens[3],
                                przmg_tokenizer_profile_t* prof);
static int32_t tokenize_to_device(Ctx* c, const uint8_t* src, uint64_t n, przmg_device_streams_t* out,
                                  przmg_tokenizer_profile_t* prof);

extern "C" int32_t przmg_tokenize(przmg_ctx* h, const uint8_t* src, uint64_t n, uint8_t* cmd, uint64_t cmd_cap,
                                  uint8_t* off, uint64_t off_cap, uint8_t* lit, uint64_t lit_cap, uint64_t lens[3],
                                  przmg_tokenizer_profile_t* prof) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || !lens) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    if (int32_t m = mock_check()) return m;
    lens[0] = lens[1] = lens[2] = 0;
    if (prof) *prof = przmg_tokenizer_profile_t{};
    if (n == 0) return PRZMG_OK;
    if (!src) return fail(PRZMG_ERR_INVALID_ARG, "null source");
    LOCKED(c);
    return tokenize_to_host(c, src, n, cmd, cmd_cap, off, off_cap, lit, lit_cap, lens, prof);
}

extern "C" int32_t przmg_tokenize_device_only(przmg_ctx* h, uint64_t n, uint8_t* cmd, uint64_t cmd_cap, uint8_t* off,
                                              uint64_t off_cap, uint8_t* lit, uint64_t lit_cap, uint64_t lens[3],
                                              przmg_tokenizer_profile_t* prof) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || !lens) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    lens[0] = lens[1] = lens[2] = 0;
    if (prof) *prof = przmg_tokenizer_profile_t{};
    if (n == 0) return PRZMG_OK;
    LOCKED(c);
    return tokenize_to_host(c, nullptr, n, cmd, cmd_cap, off, off_cap, lit, lit_cap, lens, prof);
}

static int32_t tokenize_to_host(Ctx* c, const uint8_t* src, uint64_t n, uint8_t* cmd, uint64_t cmd_cap, uint8_t* off,
                                uint64_t off_cap, uint8_t* lit, uint64_t lit_cap, uint64_t lens[3],
                                przmg_tokenizer_profile_t* prof) {
    uint32_t l6[6];
    int32_t r = tokenize_common(c, src, n, prof, l6);
    if (r) return r;
    if (l6[S_CMD] > cmd_cap || l6[S_OFF] > off_cap || l6[S_LIT] > lit_cap)
        return fail(PRZMG_ERR_BUFFER_TOO_SMALL, "stream buffers too small");
    if ((l6[S_CMD] && !cmd) || (l6[S_OFF] && !off) || (l6[S_LIT] && !lit))
        return fail(PRZMG_ERR_INVALID_ARG, "null stream buffer");
    przmg_batch* b = &c->single;
    const Job& j = b->jobs[0];
    const uint8_t* base = b->d_streams.as<uint8_t>() + j.str_off;
    if (l6[S_CMD]) CK(cudaMemcpyAsync(cmd, base + stream_base(j, S_CMD), l6[S_CMD], cudaMemcpyDeviceToHost, c->stream));
    if (l6[S_OFF]) CK(cudaMemcpyAsync(off, base + stream_base(j, S_OFF), l6[S_OFF], cudaMemcpyDeviceToHost, c->stream));
    if (l6[S_LIT]) CK(cudaMemcpyAsync(lit, base + stream_base(j, S_LIT), l6[S_LIT], cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    lens[0] = l6[S_CMD];
    lens[1] = l6[S_OFF];
    lens[2] = l6[S_LIT];
    return PRZMG_OK;
}

extern "C" int32_t przmg_tokenize_device(przmg_ctx* h, const uint8_t* src, uint64_t n, przmg_device_streams_t* out,
                                         przmg_tokenizer_profile_t* prof) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || !out) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    if (int32_t m = mock_check()) return m;
    *out = przmg_device_streams_t{};
    if (prof) *prof = przmg_tokenizer_profile_t{};
    if (n == 0) return PRZMG_OK;
    if (!src) return fail(PRZMG_ERR_INVALID_ARG, "null source");
    LOCKED(c);
    return tokenize_to_device(c, src, n, out, prof);
}

extern "C" int32_t przmg_tokenize_pointers_device_only(przmg_ctx* h, uint64_t n, przmg_device_streams_t* out,
                                                       przmg_tokenizer_profile_t* prof) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || !out) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    *out = przmg_device_streams_t{};
    if (prof) *prof = przmg_tokenizer_profile_t{};
    if (n == 0) return PRZMG_OK;
    LOCKED(c);
    return tokenize_to_device(c, nullptr, n, out, prof);
}

static int32_t tokenize_to_device(Ctx* c, const uint8_t* src, uint64_t n, przmg_device_streams_t* out,
                                  przmg_tokenizer_profile_t* prof) {
    uint32_t l6[6];
    int32_t r = tokenize_common(c, src, n, prof, l6);
    if (r) return r;
    przmg_batch* b = &c->single;
    const Job& j = b->jobs[0];
    uint8_t* base = b->d_streams.as<uint8_t>() + j.str_off;
    // {cmd, off, lit} totals, as dTotals (przm_tokenizer.cuh:512-514)
    uint32_t tot[3] = {l6[S_CMD], l6[S_OFF], l6[S_LIT]};
    uint32_t* d_tot = b->d_misc.as<uint32_t>() + 4;
    CK(cudaMemcpyAsync(d_tot, tot, 12, cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out->d_final_cmds = (uint64_t)(uintptr_t)(base + stream_base(j, S_CMD));
    out->d_final_offs = (uint64_t)(uintptr_t)(base + stream_base(j, S_OFF));
    out->d_final_lits = (uint64_t)(uintptr_t)(base + stream_base(j, S_LIT));
    out->d_totals = (uint64_t)(uintptr_t)d_tot;
    out->cmd_len = l6[S_CMD];
    out->off_len = l6[S_OFF];
    out->lit_len = l6[S_LIT];
    out->num_chunks = j.ntiles;
    out->stream = (uint64_t)(uintptr_t)c->stream;
    return PRZMG_OK;
}

// Per-position match table of Tokenize/CompressD2D (the slot's dMatch after
// launchMatchSearch, gpu/bridge.go:924-950): tile finder for n <= 64 KiB,
// radix strike otherwise (non-8-aligned positions are 0).
extern "C" int32_t przmg_match_table(przmg_ctx* h, const uint8_t* src, uint64_t n, uint32_t* desc) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c) return fail(PRZMG_ERR_INVALID_ARG, "null context");
    if (int32_t m = mock_check()) return m;
    if (n == 0) return PRZMG_OK;
    if (!src || !desc) return fail(PRZMG_ERR_INVALID_ARG, "null buffer");
    LOCKED(c);
    int32_t r = single_run(c, src, n, PRZMG_PROFILE_D2D, 0, false, nullptr);
    if (r) return r;
    przmg_batch* b = &c->single;
    const Job& j = b->jobs[0];
    const uint32_t* d = b->d_desc.as<uint32_t>() + j.desc_off;
    if (j.kind == 0) {
        CK(cudaMemcpyAsync(desc, d, 4 * n, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        return PRZMG_OK;
    }
    const uint64_t nd = n >= 8 ? (n - 8) / 8 + 1 : 0;
    CK(c->h_out.ensure(4 * nd + 16));
    if (nd) CK(cudaMemcpyAsync(c->h_out.p, d, 4 * nd, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    std::memset(desc, 0, 4 * n);
    for (uint64_t k = 0; k < nd; k++) desc[8 * k] = c->h_out.as<uint32_t>()[k];
    return PRZMG_OK;
}

extern "C" int32_t przmg_download_device_bytes(przmg_ctx* h, uint64_t d_ptr, uint64_t size, uint8_t* dst) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c) return fail(PRZMG_ERR_INVALID_ARG, "null context");
    if (size == 0) return PRZMG_OK;
    if (!d_ptr || !dst) return fail(PRZMG_ERR_INVALID_ARG, "null pointer");
    LOCKED(c);
    CK(cudaMemcpyAsync(dst, (const void*)(uintptr_t)d_ptr, size, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return PRZMG_OK;
}

// EncodeD2D: flat sections and header from device-resident streams
// (encodeD2DLocked, gpu/bridge.go:2287-2458).
extern "C" int32_t przmg_encode_d2d(przmg_ctx* h, const przmg_device_streams_t* st, uint32_t usize, int32_t window_log,
                                    uint8_t* dst, uint64_t cap, uint64_t* out_len, przmg_profile_t* prof) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || !st || !out_len) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    *out_len = 0;
    if (usize == 0) return PRZMG_OK;
    LOCKED(c);
    const uint32_t l2 = st->cmd_len + 5, l3 = st->off_len + 5;
    uint32_t wl = (uint32_t)window_log;
    if (wl == 0) wl = d2d_wlog(usize);
    const bool ext = usize > 65535 || l2 > 65535 || l3 > 65535 || wl > 16;
    const uint32_t hdr = 8 + (ext ? 6 : 4) + 8;
    const uint64_t total = (uint64_t)hdr + l2 + l3 + st->lit_len;
    if (total > cap) return fail(PRZMG_ERR_BUFFER_TOO_SMALL, "destination too small for the frame");
    CK(c->d_scr_out.ensure(total + 64));
    CK(c->h_out.ensure(total + 64));
    uint8_t* hb = c->h_out.as<uint8_t>();
    uint8_t head[40];
    uint32_t w = 0;
    head[w++] = 'P'; head[w++] = 'R'; head[w++] = 'Z'; head[w++] = 'M';
    head[w++] = ext ? 0x08 : 0;
    head[w++] = (uint8_t)usize; head[w++] = (uint8_t)(usize >> 8); head[w++] = (uint8_t)(usize >> 16);
    if (!ext) {
        head[w++] = (uint8_t)l2; head[w++] = (uint8_t)(l2 >> 8); head[w++] = (uint8_t)l3; head[w++] = (uint8_t)(l3 >> 8);
    } else {
        head[w++] = (uint8_t)l2; head[w++] = (uint8_t)(l2 >> 8); head[w++] = (uint8_t)(l2 >> 16);
        head[w++] = (uint8_t)l3; head[w++] = (uint8_t)(l3 >> 8); head[w++] = (uint8_t)(l3 >> 16);
    }
    for (int k = 0; k < 8; k++) head[w++] = 0;
    head[hdr - 7] = (uint8_t)wl;
    head[w++] = 0;
    for (int k = 0; k < 4; k++) head[w++] = (uint8_t)(st->cmd_len >> (8 * k));
    std::memcpy(hb, head, w);
    uint8_t* d = c->d_scr_out.as<uint8_t>();
    cudaStream_t s = c->stream;
    CK(cudaEventRecord(c->ev[0], s));
    CK(cudaMemcpyAsync(d, hb, w, cudaMemcpyHostToDevice, s));
    if (st->cmd_len) CK(cudaMemcpyAsync(d + hdr + 5, (const void*)(uintptr_t)st->d_final_cmds, st->cmd_len, cudaMemcpyDeviceToDevice, s));
    uint8_t h3[5] = {0, (uint8_t)st->off_len, (uint8_t)(st->off_len >> 8), (uint8_t)(st->off_len >> 16), (uint8_t)(st->off_len >> 24)};
    std::memcpy(hb + 64, h3, 5);
    CK(cudaMemcpyAsync(d + hdr + l2, hb + 64, 5, cudaMemcpyHostToDevice, s));
    if (st->off_len) CK(cudaMemcpyAsync(d + hdr + l2 + 5, (const void*)(uintptr_t)st->d_final_offs, st->off_len, cudaMemcpyDeviceToDevice, s));
    if (st->lit_len) CK(cudaMemcpyAsync(d + hdr + l2 + l3, (const void*)(uintptr_t)st->d_final_lits, st->lit_len, cudaMemcpyDeviceToDevice, s));
    CK(cudaEventRecord(c->ev[1], s));
    CK(cudaStreamSynchronize(s));
    CK(cudaMemcpyAsync(hb, d, total, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(c->ev[2], s));
    CK(cudaStreamSynchronize(s));
    std::memcpy(dst, hb, total);
    *out_len = total;
    if (prof) {
        *prof = przmg_profile_t{};
        prof->kernel_time_ms = ev_ms(c->ev[0], c->ev[1]);
        prof->internal_vram_bandwidth_gbps = gbps((double)usize, prof->kernel_time_ms);
        prof->egress_dma_bytes = total;
        prof->total_round_trip_ms = ev_ms(c->ev[0], c->ev[2]);
        fill_profile(c, prof);
    }
    return PRZMG_OK;
}

// ---------------------------------------------------------------------------
// many inputs per call
// ---------------------------------------------------------------------------
extern "C" int32_t przmg_compress_batch(przmg_ctx* h, przmg_job_t* jobs, uint64_t njobs, int32_t profile,
                                        int32_t batched, przmg_profile_t* prof) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || (!jobs && njobs)) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    if (!valid_profile(profile)) return fail(PRZMG_ERR_INVALID_ARG, "unknown profile");
    if (int32_t m = mock_check()) return m;
    LOCKED(c);
    for (uint64_t i = 0; i < njobs; i++) {
        jobs[i].out_len = 0;
        jobs[i].status = PRZMG_OK;
        if (profile >= PRZMG_PROFILE_ANS && jobs[i].n >= (1u << 24)) jobs[i].status = PRZMG_ERR_EXCEEDS_MAX_BLOCK;
    }
    if (!batched) {
        for (uint64_t i = 0; i < njobs; i++) {
            if (jobs[i].status || jobs[i].n == 0) continue;
            uint64_t len = 0;
            int32_t r = compress_one(c, jobs[i].src, jobs[i].n, profile, jobs[i].dst, jobs[i].cap, &len, nullptr);
            jobs[i].status = r;
            jobs[i].out_len = len;
        }
        if (prof) { *prof = przmg_profile_t{}; prof->pipelined_chunks = (int32_t)njobs; fill_profile(c, prof); }
        return PRZMG_OK;
    }
    std::vector<uint64_t> sizes(njobs);
    uint64_t total = 0;
    for (uint64_t i = 0; i < njobs; i++) { sizes[i] = jobs[i].status ? 0 : jobs[i].n; total += sizes[i]; }
    przmg_batch* b = &c->single;
    int32_t r = batch_prepare(b, sizes.data(), (uint32_t)njobs, profile, false);
    if (r) return r;
    CK(c->h_in.ensure(b->in_bytes));
    for (uint64_t i = 0; i < njobs; i++)
        if (sizes[i]) std::memcpy(c->h_in.as<uint8_t>() + b->in_offs[i], jobs[i].src, sizes[i]);
    cudaStream_t s = c->stream;
    CK(cudaEventRecord(c->ev[0], s));
    CK(cudaMemcpyAsync(b->d_in.p, c->h_in.p, b->in_bytes - 64, cudaMemcpyHostToDevice, s));
    CK(cudaEventRecord(c->ev[1], s));
    r = batch_launch(b, s, 2);
    if (r) return r;
    CK(cudaEventRecord(c->ev[2], s));
    r = batch_check(b);
    if (r) return r;
    std::vector<uint32_t> fs(njobs);
    CK(cudaMemcpyAsync(fs.data(), b->d_sizes.p, 4 * njobs, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    CK(c->h_out.ensure(b->out_bytes));
    CK(cudaMemcpyAsync(c->h_out.p, b->d_out.p, b->out_bytes - 64, cudaMemcpyDeviceToHost, s));
    CK(cudaEventRecord(c->ev[3], s));
    CK(cudaStreamSynchronize(s));
    uint64_t egress = 0;
    for (uint64_t i = 0; i < njobs; i++) {
        if (jobs[i].status || sizes[i] == 0) continue;
        if (fs[i] > jobs[i].cap) { jobs[i].status = PRZMG_ERR_BUFFER_TOO_SMALL; continue; }
        std::memcpy(jobs[i].dst, c->h_out.as<uint8_t>() + b->out_offs[i], fs[i]);
        jobs[i].out_len = fs[i];
        egress += fs[i];
    }
    if (prof) {
        *prof = przmg_profile_t{};
        prof->ingress_dma_bytes = total;
        prof->ingress_dma_time_ms = ev_ms(c->ev[0], c->ev[1]);
        prof->kernel_time_ms = ev_ms(c->ev[1], c->ev[2]);
        prof->egress_dma_bytes = egress;
        prof->total_round_trip_ms = ev_ms(c->ev[0], c->ev[3]);
        prof->end_to_end_bandwidth_gbps = gbps((double)total, prof->total_round_trip_ms);
        prof->internal_vram_bandwidth_gbps = gbps((double)total, prof->kernel_time_ms);
        prof->pipelined_chunks = (int32_t)njobs;
        fill_profile(c, prof);
    }
    return PRZMG_OK;
}

extern "C" int32_t przmg_batch_create(przmg_ctx* h, const uint64_t* sizes, uint64_t njobs, int32_t profile,
                                      przmg_batch** out) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || !out || (!sizes && njobs)) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    if (!valid_profile(profile)) return fail(PRZMG_ERR_INVALID_ARG, "unknown profile");
    for (uint64_t i = 0; i < njobs; i++)
        if (profile >= PRZMG_PROFILE_ANS && sizes[i] >= (1u << 24))
            return fail(PRZMG_ERR_EXCEEDS_MAX_BLOCK, "the frame header holds 24-bit sizes: inputs must be < 16 MiB");
    LOCKED(c);
    przmg_batch* b = new przmg_batch();
    b->ctx = c;
    b->owned = true;
    int32_t r = batch_prepare(b, sizes, (uint32_t)njobs, profile, false);
    if (r) { delete b; return r; }
    *out = b;
    return PRZMG_OK;
}

extern "C" int32_t przmg_batch_inputs(przmg_batch* b, uint64_t* d_in, uint64_t* offsets) {
    if (!b) return fail(PRZMG_ERR_INVALID_ARG, "null batch");
    if (d_in) *d_in = (uint64_t)(uintptr_t)b->d_in.p;
    if (offsets) std::copy(b->in_offs.begin(), b->in_offs.end(), offsets);
    return PRZMG_OK;
}

extern "C" int32_t przmg_batch_outputs(przmg_batch* b, uint64_t* d_out, uint64_t* offsets) {
    if (!b) return fail(PRZMG_ERR_INVALID_ARG, "null batch");
    if (d_out) *d_out = (uint64_t)(uintptr_t)b->d_out.p;
    if (offsets) std::copy(b->out_offs.begin(), b->out_offs.end(), offsets);
    return PRZMG_OK;
}

extern "C" int32_t przmg_batch_enqueue(przmg_batch* b, uint64_t stream, int32_t use_graph) {
    if (!b) return fail(PRZMG_ERR_INVALID_ARG, "null batch");
    Ctx* c = b->ctx;
    LOCKED(c);
    cudaStream_t s = stream ? (cudaStream_t)(uintptr_t)stream : c->stream;
    if (!use_graph) return batch_launch(b, s, 2);
    if (!b->exec) {
        cudaStream_t cap_s;
        CK(cudaStreamCreateWithFlags(&cap_s, cudaStreamNonBlocking));
        CK(cudaStreamBeginCapture(cap_s, cudaStreamCaptureModeThreadLocal));
        int32_t r = batch_launch(b, cap_s, 2);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(cap_s, &g);
        cudaStreamDestroy(cap_s);
        if (r) { if (g) cudaGraphDestroy(g); return r; }
        if (e != cudaSuccess) return cuda_fail("cudaStreamEndCapture", e);
        b->graph = g;
        CK(cudaGraphInstantiate(&b->exec, g, 0));
    }
    CK(cudaGraphLaunch(b->exec, s));
    return PRZMG_OK;
}

extern "C" int32_t przmg_batch_sizes(przmg_batch* b, uint32_t* sizes) {
    if (!b) return fail(PRZMG_ERR_INVALID_ARG, "null batch");
    Ctx* c = b->ctx;
    LOCKED(c);
    CK(cudaDeviceSynchronize());
    int32_t r = batch_check(b);
    if (r) return r;
    if (sizes && b->njobs) {
        CK(cudaMemcpy(sizes, b->d_sizes.p, 4ull * b->njobs, cudaMemcpyDeviceToHost));
    }
    return PRZMG_OK;
}

extern "C" int32_t przmg_batch_launch_count(przmg_batch* b) { return b ? b->launches : 0; }

extern "C" int32_t przmg_size_class(uint64_t mean_input_bytes) { return size_class(mean_input_bytes); }

extern "C" int32_t przmg_set_tuning(przmg_ctx* h, int32_t cls, int32_t front, int32_t ctas_per_sm, int32_t verify_chunk) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c) return fail(PRZMG_ERR_INVALID_ARG, "null context");
    if (cls < 0 || cls >= kSizeClasses || front < 0 || front > 1 || ctas_per_sm < 1 || ctas_per_sm > 3 ||
        verify_chunk < 256 || verify_chunk > (1 << 16) || (verify_chunk & 255))
        return fail(PRZMG_ERR_INVALID_ARG, "tuning out of range (class 0-3, front 0/1, 1-3 blocks per SM, "
                                           "verify chunk a multiple of 256 in [256, 65536])");
    std::lock_guard<std::mutex> lk(c->mu);
    c->tune[cls].front = (uint32_t)front;
    c->tune[cls].ctas_per_sm = (uint32_t)ctas_per_sm;
    c->tune[cls].verify_chunk = (uint32_t)verify_chunk;
    return PRZMG_OK;
}

extern "C" int32_t przmg_get_tuning(przmg_ctx* h, int32_t cls, int32_t* front, int32_t* ctas_per_sm,
                                    int32_t* verify_chunk) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || cls < 0 || cls >= kSizeClasses) return fail(PRZMG_ERR_INVALID_ARG, "null context or unknown class");
    std::lock_guard<std::mutex> lk(c->mu);
    if (front) *front = (int32_t)c->tune[cls].front;
    if (ctas_per_sm) *ctas_per_sm = (int32_t)c->tune[cls].ctas_per_sm;
    if (verify_chunk) *verify_chunk = (int32_t)c->tune[cls].verify_chunk;
    return PRZMG_OK;
}

extern "C" int32_t przmg_set_front_wait(przmg_ctx* h, uint64_t limit_ns, int32_t add_unreachable_wait) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c) return fail(PRZMG_ERR_INVALID_ARG, "null context");
    if (limit_ns == 0 || limit_ns > 60ull * 1000000000ull) return fail(PRZMG_ERR_INVALID_ARG, "limit out of range");
    std::lock_guard<std::mutex> lk(c->mu);
    c->front_wait_ns = limit_ns;
    c->front_unreachable = add_unreachable_wait != 0;
    return PRZMG_OK;
}

extern "C" int32_t przmg_batch_info(przmg_batch* b, uint32_t info[4]) {
    if (!b || !info) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    uint64_t total = 0;
    for (const Job& j : b->jobs) total += j.n;
    info[0] = b->front ? 1u : 0u;
    info[1] = (uint32_t)size_class(b->njobs ? total / b->njobs : 0);
    info[2] = b->tune.ctas_per_sm;
    info[3] = b->tune.verify_chunk;
    return PRZMG_OK;
}

extern "C" int32_t przmg_batch_enqueue_plain(przmg_batch* b, uint64_t stream, int32_t* launches) {
    if (!b) return fail(PRZMG_ERR_INVALID_ARG, "null batch");
    Ctx* c = b->ctx;
    LOCKED(c);
    int32_t r = batch_launch_plain(b, stream ? (cudaStream_t)(uintptr_t)stream : c->stream);
    if (launches) *launches = b->launches_plain;
    return r;
}

// Scatter of back-to-back inputs into the padded per-frame layout, and the
// inverse gather of the frames into back-to-back output.
__global__ void k_scatter_inputs(const uint8_t* __restrict__ packed, const uint64_t* __restrict__ src_off,
                                 const Job* __restrict__ jobs, uint32_t njobs, uint8_t* __restrict__ in) {
    for (uint32_t j = blockIdx.y; j < njobs; j += gridDim.y) {
        const uint32_t n = jobs[j].n;
        const uint32_t chunk = ((n + gridDim.x - 1) / gridDim.x + 15) & ~15u;  // 16-byte aligned slice per block
        const uint32_t lo = min(n, blockIdx.x * chunk), hi = min(n, lo + chunk);
        if (lo < hi) block_copy(in + jobs[j].in_off + lo, packed + src_off[j] + lo, hi - lo);
    }
}

__global__ void k_gather_frames(const uint8_t* __restrict__ out, const Job* __restrict__ jobs,
                                const uint32_t* __restrict__ sizes, const uint64_t* __restrict__ dst_off, uint32_t njobs,
                                uint8_t* __restrict__ packed) {
    for (uint32_t j = blockIdx.y; j < njobs; j += gridDim.y) {
        const uint32_t n = sizes[j];
        const uint32_t chunk = ((n + gridDim.x - 1) / gridDim.x + 15) & ~15u;
        const uint32_t lo = min(n, blockIdx.x * chunk), hi = min(n, lo + chunk);
        if (lo < hi) block_copy(packed + dst_off[j] + lo, out + jobs[j].out_off + lo, hi - lo);
    }
}

static int32_t batch_upload_packed(przmg_batch* b, const uint8_t* host, cudaStream_t s) {
    uint64_t total = 0;
    for (uint32_t i = 0; i < b->njobs; i++) total += b->jobs[i].n;
    CK(b->d_stage_in.ensure(total + 64));
    if (total) CK(cudaMemcpyAsync(b->d_stage_in.p, host, total, cudaMemcpyHostToDevice, s));
    if (b->njobs) {
        // b->d_up_offs holds the packed input offsets, written by batch_prepare
        k_scatter_inputs<<<dim3(64, std::min<uint32_t>(b->njobs, 4096)), 256, 0, s>>>(
            b->d_stage_in.as<uint8_t>(), b->d_up_offs.as<uint64_t>(), b->d_jobs.as<Job>(), b->njobs, b->d_in.as<uint8_t>());
        CK(cudaGetLastError());
    }
    return PRZMG_OK;
}

static int32_t batch_download_packed(przmg_batch* b, uint8_t* host, uint64_t cap, uint64_t* total, uint32_t* sizes,
                                     cudaStream_t s) {
    std::vector<uint32_t> fs(b->njobs);
    if (b->njobs) CK(cudaMemcpyAsync(fs.data(), b->d_sizes.p, 4ull * b->njobs, cudaMemcpyDeviceToHost, s));
    uint32_t err = 0;
    CK(cudaMemcpyAsync(&err, b->err_word(), 4, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    if (err) return device_error(err);
    std::vector<uint64_t> offs(b->njobs);
    uint64_t t = 0;
    for (uint32_t i = 0; i < b->njobs; i++) { offs[i] = t; t += fs[i]; }
    if (sizes) std::copy(fs.begin(), fs.end(), sizes);
    *total = t;
    if (t > cap) return fail(PRZMG_ERR_BUFFER_TOO_SMALL, "output buffer too small for the frames");
    CK(b->d_stage_out.ensure(t + 64));
    CK(b->d_stage_offs.ensure(8ull * b->njobs + 64));
    CK(b->h_offs.ensure(8ull * b->njobs + 64));
    std::memcpy(b->h_offs.p, offs.data(), 8ull * b->njobs);
    CK(cudaMemcpyAsync(b->d_stage_offs.p, b->h_offs.p, 8ull * b->njobs, cudaMemcpyHostToDevice, s));
    if (b->njobs) {
        k_gather_frames<<<dim3(64, std::min<uint32_t>(b->njobs, 4096)), 256, 0, s>>>(
            b->d_out.as<uint8_t>(), b->d_jobs.as<Job>(), b->d_sizes.as<uint32_t>(), b->d_stage_offs.as<uint64_t>(), b->njobs,
            b->d_stage_out.as<uint8_t>());
        CK(cudaGetLastError());
    }
    if (t) CK(cudaMemcpyAsync(host, b->d_stage_out.p, t, cudaMemcpyDeviceToHost, s));
    CK(cudaStreamSynchronize(s));
    return PRZMG_OK;
}

extern "C" int32_t przmg_batch_upload(przmg_batch* b, const uint8_t* host, uint64_t stream) {
    if (!b || (!host && b->njobs)) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    Ctx* c = b->ctx;
    LOCKED(c);
    return batch_upload_packed(b, host, stream ? (cudaStream_t)(uintptr_t)stream : c->stream);
}

extern "C" int32_t przmg_batch_download(przmg_batch* b, uint8_t* host, uint64_t cap, uint64_t* total, uint32_t* sizes,
                                        uint64_t stream) {
    if (!b || !total) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    Ctx* c = b->ctx;
    LOCKED(c);
    return batch_download_packed(b, host, cap, total, sizes, stream ? (cudaStream_t)(uintptr_t)stream : c->stream);
}

extern "C" int32_t przmg_batch_stage_times(przmg_batch* b, float* ms, int32_t cap, int32_t* count) {
    if (!b || !ms || !count) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    Ctx* c = b->ctx;
    LOCKED(c);
    cudaEvent_t ev[kStages + 1];
    for (auto& e : ev) CK(cudaEventCreate(&e));
    int32_t r = batch_launch(b, c->stream, 2, ev);
    if (r == 0) {
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) r = cuda_fail("cudaStreamSynchronize", e);
    }
    const int n = std::min<int>(cap, kStages);
    for (int k = 0; k < n && r == 0; k++) ms[k] = ev_ms(ev[k], ev[k + 1]);
    for (auto& e : ev) cudaEventDestroy(e);
    *count = n;
    return r;
}

// Totals of the last run of a batch (synchronises):
//   [0] input bytes   [1] frame bytes   [2] literal bytes   [3] command bytes
//   [4] offset bytes  [5] rANS symbols of the active tasks
//   [6] bytes the rANS lanes emitted   [7] frames stored uncompressed
extern "C" int32_t przmg_batch_stats(przmg_batch* b, uint64_t stats[8]) {
    if (!b || !stats) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    Ctx* c = b->ctx;
    LOCKED(c);
    for (int k = 0; k < 8; k++) stats[k] = 0;
    const uint32_t nj = b->njobs;
    std::vector<uint32_t> lens((size_t)nj * S_COUNT + 1), sizes(nj + 1);
    std::vector<TaskOut> outs((size_t)nj * T_COUNT + 1);
    std::vector<Plan> plans(nj + 1);
    std::vector<S3Frame> s3f(nj + 1);
    std::vector<uint32_t> fls(16 * (size_t)nj + 16, 0);
    if (nj) {
        CK(cudaMemcpyAsync(lens.data(), b->d_job_lens.p, 4ull * nj * S_COUNT, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(sizes.data(), b->d_sizes.p, 4ull * nj, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaMemcpyAsync(plans.data(), b->d_plans.p, sizeof(Plan) * nj, cudaMemcpyDeviceToHost, c->stream));
        if (b->profile >= 1)
            CK(cudaMemcpyAsync(outs.data(), b->d_outs.p, sizeof(TaskOut) * nj * T_COUNT, cudaMemcpyDeviceToHost, c->stream));
        if (b->profile >= 2)
            CK(cudaMemcpyAsync(s3f.data(), b->d_s3f.p, sizeof(S3Frame) * nj, cudaMemcpyDeviceToHost, c->stream));
        if (b->profile >= 3)
            for (uint32_t j = 0; j < nj; j++)
                CK(cudaMemcpyAsync(&fls[16 * (size_t)j], b->d_fib.as<uint8_t>() + b->jobs[j].fib_off, 64,
                                   cudaMemcpyDeviceToHost, c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    for (uint32_t j = 0; j < nj; j++) {
        const uint32_t* l = &lens[(size_t)j * S_COUNT];
        stats[0] += b->jobs[j].n;
        stats[1] += sizes[j];
        stats[2] += l[S_LIT];
        stats[3] += l[S_CMD];
        stats[4] += l[S_OFF];
        stats[7] += plans[j].uncompressed;
        if (b->profile < 1) continue;
        for (int t = 0; t < T_COUNT; t++) {
            const uint32_t nd = t == T_S3 && b->profile >= 2 ? s3_task_nd(s3f[j]) : 0u;
            const uint32_t* fl = b->profile >= 3 ? &fls[16 * (size_t)j] : nullptr;
            if (!task_active(b->jobs[j], l, t, nd, fl)) continue;
            stats[5] += task_len(l, t, nd, fl);
            const TaskOut& o = outs[(size_t)j * T_COUNT + t];
            stats[6] += (uint64_t)o.count[0] + o.count[1] + o.count[2] + o.count[3];
        }
    }
    return PRZMG_OK;
}

extern "C" const char* przmg_stage_name(int32_t k) { return (k >= 0 && k < kStages) ? kStageNames[k] : ""; }

extern "C" int32_t przmg_compress_packed(przmg_ctx* h, const uint8_t* host_in, const uint64_t* sizes, uint64_t njobs,
                                         int32_t profile, uint8_t* host_out, uint64_t out_cap, uint32_t* out_sizes,
                                         uint64_t* out_total) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || !sizes || !out_total || (njobs && (!host_in || !host_out))) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    if (!valid_profile(profile)) return fail(PRZMG_ERR_INVALID_ARG, "unknown profile");
    for (uint64_t i = 0; i < njobs; i++)
        if (profile >= PRZMG_PROFILE_ANS && sizes[i] >= (1u << 24))
            return fail(PRZMG_ERR_EXCEEDS_MAX_BLOCK, "the frame header holds 24-bit sizes: inputs must be < 16 MiB");
    if (int32_t m = mock_check()) return m;
    LOCKED(c);
    przmg_batch* b = &c->single;
    int32_t r = batch_prepare(b, sizes, (uint32_t)njobs, profile, false);
    if (r) return r;
    r = batch_upload_packed(b, host_in, c->stream);
    if (r) return r;
    r = batch_launch(b, c->stream, 2);
    if (r) return r;
    return batch_download_packed(b, host_out, out_cap, out_total, out_sizes, c->stream);
}


extern "C" int32_t przmg_batch_stream_lens(przmg_batch* b, uint32_t* lens, uint64_t cap) {
    if (!b || (!lens && b->njobs)) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    if (cap < (uint64_t)b->njobs * S_COUNT) return fail(PRZMG_ERR_BUFFER_TOO_SMALL, "lens needs 6 entries per input");
    Ctx* c = b->ctx;
    LOCKED(c);
    if (b->njobs) {
        CK(cudaMemcpyAsync(lens, b->d_job_lens.p, 4ull * b->njobs * S_COUNT, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
    }
    return PRZMG_OK;
}

extern "C" int32_t przmg_batch_destroy(przmg_batch* b) {
    if (!b) return PRZMG_OK;
    Ctx* c = b->ctx;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        cudaSetDevice(c->device);
        cudaStreamSynchronize(c->stream);
    }
    if (b->owned) delete b;
    return PRZMG_OK;
}

// ---------------------------------------------------------------------------
// MatchLZ77
// ---------------------------------------------------------------------------
static int32_t match_chunks(Ctx* c, const uint8_t* src, uint64_t n, uint64_t chunk, przmg_match_t* out, uint64_t cap,
                            uint64_t* n_out, przmg_profile_t* prof) {
    *n_out = 0;
    if (prof) *prof = przmg_profile_t{};
    if (n == 0) { fill_profile(c, prof); return PRZMG_OK; }
    if (!src || !out) return fail(PRZMG_ERR_INVALID_ARG, "null buffer");
    std::vector<uint64_t> sizes;
    for (uint64_t base = 0; base < n; base += chunk) sizes.push_back(std::min<uint64_t>(chunk, n - base));
    przmg_batch* b = &c->single;
    int32_t r = batch_prepare(b, sizes.data(), (uint32_t)sizes.size(), PRZMG_PROFILE_D2D, true);
    if (r) return r;
    CK(c->h_in.ensure(b->in_bytes));
    uint64_t base = 0;
    for (size_t i = 0; i < sizes.size(); i++) {
        std::memcpy(c->h_in.as<uint8_t>() + b->in_offs[i], src + base, sizes[i]);
        base += sizes[i];
    }
    cudaStream_t s = c->stream;
    CK(cudaEventRecord(c->ev[0], s));
    CK(cudaMemcpyAsync(b->d_in.p, c->h_in.p, b->in_bytes - 64, cudaMemcpyHostToDevice, s));
    CK(cudaEventRecord(c->ev[1], s));
    r = batch_launch(b, s, 0);
    if (r) return r;
    // compaction per chunk into pos/desc arrays
    uint64_t maxd = 0;
    for (auto sz : sizes) maxd = std::max<uint64_t>(maxd, sz >= 8 ? (sz - 8) / 8 + 1 : 0);
    const uint32_t nb_max = (uint32_t)((maxd + 1023) / 1024 + 1);
    CK(c->d_scr_aux.ensure((size_t)(nb_max + 16) * 4 * sizes.size()));
    CK(c->d_scr_out.ensure((size_t)2 * 4 * (n / 8 + 16)));
    uint32_t* d_pos = c->d_scr_out.as<uint32_t>();
    uint32_t* d_dsc = d_pos + (n / 8 + 16);
    std::vector<uint32_t> totals(sizes.size(), 0);
    uint64_t pos_base = 0;
    for (size_t i = 0; i < sizes.size(); i++) {
        const Job& j = b->jobs[i];
        const uint32_t nd = j.n >= 8 ? (j.n - 8) / 8 + 1 : 0;
        if (nd) {
            const uint32_t nbk = (nd + 1023) / 1024;
            uint32_t* cnt = c->d_scr_aux.as<uint32_t>() + i * (nb_max + 16);
            uint32_t* tot = cnt + nb_max + 8;
            const uint32_t* d8 = b->d_desc.as<uint32_t>() + j.desc_off;
            k_compact_count<<<nbk, 1024, 0, s>>>(d8, nd, cnt);
            k_compact_scan<<<1, 1024, 0, s>>>(cnt, nbk, tot);
            CK(cudaMemcpyAsync(&totals[i], tot, 4, cudaMemcpyDeviceToHost, s));
            CK(cudaStreamSynchronize(s));
            k_compact_scatter<<<nbk, 1024, 0, s>>>(d8, nd, cnt, (uint32_t)pos_base, d_pos + *n_out, d_dsc + *n_out);
            CK(cudaGetLastError());
            *n_out += totals[i];
        }
        pos_base += sizes[i];
    }
    CK(cudaEventRecord(c->ev[2], s));
    const uint64_t m = *n_out;
    if (m > cap) return fail(PRZMG_ERR_BUFFER_TOO_SMALL, "match buffer too small");
    CK(c->h_out.ensure(8 * m + 64));
    uint32_t* hp = c->h_out.as<uint32_t>();
    if (m) {
        CK(cudaMemcpyAsync(hp, d_pos, 4 * m, cudaMemcpyDeviceToHost, s));
        CK(cudaMemcpyAsync(hp + m, d_dsc, 4 * m, cudaMemcpyDeviceToHost, s));
    }
    CK(cudaEventRecord(c->ev[3], s));
    CK(cudaStreamSynchronize(s));
    for (uint64_t k = 0; k < m; k++) {
        out[k].position = hp[k];
        out[k].offset = hp[m + k] & 0xFFFFFu;
        out[k].length = (uint16_t)(hp[m + k] >> 20);
        out[k].literal = 0;
        out[k].reserved = 0;
    }
    if (prof) {
        prof->ingress_dma_bytes = n;
        prof->ingress_dma_time_ms = ev_ms(c->ev[0], c->ev[1]);
        prof->ingress_dma_bandwidth_gbps = gbps((double)n, prof->ingress_dma_time_ms);
        prof->kernel_time_ms = ev_ms(c->ev[1], c->ev[2]);
        prof->internal_vram_bandwidth_gbps = gbps((double)n, prof->kernel_time_ms);
        prof->egress_dma_bytes = 8 * m;
        prof->egress_dma_time_ms = ev_ms(c->ev[2], c->ev[3]);
        prof->egress_dma_bandwidth_gbps = gbps(8.0 * m, prof->egress_dma_time_ms);
        prof->total_round_trip_ms = ev_ms(c->ev[0], c->ev[3]);
        prof->end_to_end_bandwidth_gbps = gbps((double)n, prof->total_round_trip_ms);
        if (prof->total_round_trip_ms > 0)
            prof->pcie_overhead_percent = 100.0 * (prof->ingress_dma_time_ms + prof->egress_dma_time_ms) / prof->total_round_trip_ms;
        prof->pipelined_chunks = (int32_t)sizes.size();
        fill_profile(c, prof);
    }
    return PRZMG_OK;
}

extern "C" int32_t przmg_match_lz77(przmg_ctx* h, const uint8_t* src, uint64_t n, przmg_match_t* out, uint64_t cap,
                                    uint64_t* n_out, przmg_profile_t* prof) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || !n_out) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    if (int32_t m = mock_check()) return m;
    LOCKED(c);
    // > 16 MiB streams in 8 MiB chunks (gpu/bridge.go:1494-1496)
    return match_chunks(c, src, n, n > (16ull << 20) ? (8ull << 20) : std::max<uint64_t>(n, 1), out, cap, n_out, prof);
}

extern "C" int32_t przmg_match_lz77_streaming(przmg_ctx* h, const uint8_t* src, uint64_t n, int64_t chunk,
                                              przmg_match_t* out, uint64_t cap, uint64_t* n_out, przmg_profile_t* prof) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || !n_out) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    if (int32_t m = mock_check()) return m;
    LOCKED(c);
    // chunk rule of matchLZ77StreamingLocked, gpu/bridge.go:1222-1233
    uint64_t cs = chunk > 0 ? (uint64_t)chunk : std::max<uint64_t>(n / 2, 16ull << 20);
    cs = std::min<uint64_t>(cs, 64ull << 20);
    if ((n + cs - 1) / std::max<uint64_t>(cs, 1) <= 1) cs = std::max<uint64_t>(n, 1);
    return match_chunks(c, src, n, cs, out, cap, n_out, prof);
}

// ---------------------------------------------------------------------------
// histogram / flat pack / V-ANS single-stream APIs and the stream batch
// ---------------------------------------------------------------------------
#include "api_streams.inc"

// ---------------------------------------------------------------------------
// Section 3 distance coding of many distance arrays
// ---------------------------------------------------------------------------
#include "offsets.inc"

// ---------------------------------------------------------------------------
// Section 4 selection (V-ANS or a sheaf foliation) of many literal streams
// ---------------------------------------------------------------------------
#include "literals.inc"

// ---------------------------------------------------------------------------
// serving: continuous batching of submitted requests
// ---------------------------------------------------------------------------
#include "serve.inc"

// ---------------------------------------------------------------------------
// the GPU decoder
// ---------------------------------------------------------------------------
#include "decode.inc"

// ---------------------------------------------------------------------------
// allocation-free single-stream V-ANS (static device scratch)
// ---------------------------------------------------------------------------
#include "noalloc.inc"

// ---------------------------------------------------------------------------
// pinned memory
// ---------------------------------------------------------------------------
extern "C" int32_t przmg_alloc_pinned_host(uint64_t size, void** out) {
    if (!out) return fail(PRZMG_ERR_INVALID_ARG, "null output pointer");
    *out = nullptr;
    if (size == 0) return PRZMG_OK;
    CK(cudaHostAlloc(out, size, cudaHostAllocDefault));
    return PRZMG_OK;
}

extern "C" int32_t przmg_free_pinned_host(void* p) {
    if (!p) return PRZMG_OK;
    CK(cudaFreeHost(p));
    return PRZMG_OK;
}

// NewPinnedBufferPool, gpu/memory.go:108-124
extern "C" int32_t przmg_pinned_pool_create(uint64_t buf_size, int32_t initial_cap, przmg_pinned_pool** out) {
    if (!out) return fail(PRZMG_ERR_INVALID_ARG, "null output pointer");
    *out = nullptr;
    if (buf_size == 0 || initial_cap < 0) return fail(PRZMG_ERR_INVALID_ARG, "invalid pool size");
    auto* p = new przmg_pinned_pool();
    p->buf_size = buf_size;
    p->max_cap = std::max<size_t>((size_t)initial_cap, 8);
    for (int32_t i = 0; i < initial_cap; i++) {
        void* b = nullptr;
        cudaError_t e = cudaHostAlloc(&b, buf_size, cudaHostAllocDefault);
        if (e != cudaSuccess) {
            p->free_all();
            delete p;
            return cuda_fail("cudaHostAlloc", e);
        }
        p->free_bufs.push_back(b);
    }
    *out = p;
    return PRZMG_OK;
}

// PinnedBufferPool.Get, gpu/memory.go:127-141
extern "C" int32_t przmg_pinned_pool_get(przmg_pinned_pool* p, void** buf) {
    if (!p || !buf) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    *buf = nullptr;
    {
        std::lock_guard<std::mutex> lk(p->mu);
        if (!p->free_bufs.empty()) {
            *buf = p->free_bufs.back();
            p->free_bufs.pop_back();
            return PRZMG_OK;
        }
    }
    CK(cudaHostAlloc(buf, p->buf_size, cudaHostAllocDefault));
    return PRZMG_OK;
}

// PinnedBufferPool.Put, gpu/memory.go:144-155
extern "C" void przmg_pinned_pool_put(przmg_pinned_pool* p, void* buf, uint64_t len) {
    if (!p || !buf || len != p->buf_size) return;
    {
        std::lock_guard<std::mutex> lk(p->mu);
        if (p->free_bufs.size() < p->max_cap) {
            p->free_bufs.push_back(buf);
            return;
        }
    }
    cudaFreeHost(buf);
}

// PinnedBufferPool.Close, gpu/memory.go:158-165
extern "C" int32_t przmg_pinned_pool_close(przmg_pinned_pool* p) {
    if (!p) return PRZMG_OK;
    p->free_all();
    if (!p->ctx_owned) delete p;
    return PRZMG_OK;
}

extern "C" uint64_t przmg_pinned_pool_buf_size(const przmg_pinned_pool* p) { return p ? p->buf_size : 0; }

extern "C" uint64_t przmg_pinned_pool_pooled(przmg_pinned_pool* p) {
    if (!p) return 0;
    std::lock_guard<std::mutex> lk(p->mu);
    return p->free_bufs.size();
}

// GetPinned, gpu/bridge.go:452-471: pools keyed by the next power of two
extern "C" int32_t przmg_get_pinned(przmg_ctx* h, uint64_t size, void** buf, przmg_pinned_pool** pool) {
    Ctx* c = reinterpret_cast<Ctx*>(h);
    if (!c || !buf || !pool) return fail(PRZMG_ERR_INVALID_ARG, "null argument");
    *buf = nullptr;
    *pool = nullptr;
    if (size == 0 || size > (1ull << 62)) return fail(PRZMG_ERR_INVALID_ARG, "invalid size");
    uint64_t alloc = 1;
    while (alloc < size) alloc <<= 1;
    przmg_pinned_pool* p = nullptr;
    {
        std::lock_guard<std::mutex> lk(c->pools_mu);
        auto it = c->pools.find(alloc);
        if (it == c->pools.end()) {
            int32_t r = przmg_pinned_pool_create(alloc, 0, &p);
            if (r) return r;
            p->ctx_owned = true;
            c->pools[alloc] = p;
        } else {
            p = it->second;
        }
    }
    *pool = p;
    return przmg_pinned_pool_get(p, buf);
}
