// front.cu -- the persistent front end: one launch that runs the match
// finders, the tokenizer and the gather for every input of a batch.
//
// The work of a batch is a list of items in stage order (radix tile sorts
// and tile-finder tiles, partition resolves, verify chunks, tokenizer tiles,
// gathers), built on the host when the batch is laid
// out.  Blocks stay resident and take the next item from a device counter
// (atomicAdd), so a block that finishes a short item -- a 1 KiB input's
// tile, a 2048-candidate verify chunk -- takes another at once, and inputs of
// very different sizes share one launch with no per-stage grid or tail.
//
// Each input has a progress counter: every item of the input adds one when
// it is done, and an item waits until its input's counter reaches the number
// of items of that input in earlier stages (its target).  Items are claimed
// in list order and a block finishes its item before claiming the next, so
// every item an item waits for was claimed earlier by a block that is
// running: the waits always end.  They are bounded anyway: a wait that
// exceeds its limit sets E_SCHED_TIMEOUT in the batch's error word, and every
// block stops taking items once that bit is set (the host then reports
// PRZMG_ERR_DEVICE).  The output bytes do not depend on which block runs
// which item.
//
// An item's progress is published with a fence and an atomic add after the
// block's barrier, and a waiting item reads it with ld.acquire.gpu before its
// block's barrier.  Data that other blocks of the same launch wrote
// (descriptors, radix lists, run starts and predecessors, tokenizer slots
// and tile lengths) is read with ld.global.cg, which goes to L2, never through the non-coherent
// read-only path, whose contents are only valid for data that no block of
// the running kernel writes.
#include "common.cuh"

namespace pz {

enum FrontStage : uint32_t {
    FS_TILE_FIND = 0,  // idx = small tile (TileRef list)
    FS_RX_SORT,        // idx = radix tile (RxTile list)
    FS_RX_RESOLVE,     // idx = first partition (8 per item, one per warp)
    FS_RX_VERIFY,      // idx = first candidate of the chunk
    FS_TOKENIZE,       // idx = first tile (tile list), up to 8 tiles (one per warp)
    FS_GATHER,         // idx = input
    FS_NOP,            // a wait and nothing else (the wait-limit test)
};

// job: the input whose progress the item adds to (for FS_TOKENIZE: the
// number of tiles of the item); target: the progress the item waits for
// (for FS_TOKENIZE the per-tile targets are in tok_target).
struct FrontItem { uint32_t stage, job, idx, target; };

constexpr uint32_t kFrontThreads = 256;
constexpr uint32_t kFrontWarps = kFrontThreads / 32;
constexpr uint32_t kFrontResolveItems = kRxParts / kFrontWarps;  // resolve items per large frame
constexpr uint32_t kFrontGatherSmem = 4 * 4 * 256 * 4 + (512 + 4) * 4;  // histograms + tile offsets (<= 512 tiles)
constexpr uint32_t kFrontSmem = (kTileFindSmem > kRxResolveSmem ? kTileFindSmem : kRxResolveSmem) >
                                        kFrontWarps * sizeof(TokSmem)
                                    ? (kTileFindSmem > kRxResolveSmem ? kTileFindSmem : kRxResolveSmem)
                                    : (uint32_t)(kFrontWarps * sizeof(TokSmem));
static_assert(kFrontSmem >= kFrontGatherSmem && kFrontSmem >= sizeof(RxSortSmem), "front shared memory");
static_assert(kRxResolveWarps == kFrontWarps, "a resolve item is one partition per warp");

constexpr uint32_t E_SCHED_TIMEOUT = 16;  // a front-end wait ran out (error word bit)

struct FrontArgs {
    const uint8_t* in;
    const Job* jobs;
    const FrontItem* items;
    uint32_t nitems;
    uint32_t* head;       // next item to claim
    uint32_t* progress;   // per input
    uint32_t* err;        // the batch's error word
    const uint32_t* tok_target;  // per input: progress before its tokenizer tiles
    long long wait_cycles;       // limit of one wait, in SM clock cycles
    const TileRef* small;
    const RxTile* rtiles;
    const TokTile* tiles;
    uint32_t ntiles;
    uint32_t verify_chunk;
    uint32_t* desc;
    uint32_t* rx_toff;
    uint32_t* rx_list;
    uint32_t* rx_pred;
    uint8_t* slots;
    uint32_t* tile_lens;
    uint8_t* streams;
    uint32_t* job_lens;
    uint32_t* hist;
};

__device__ __forceinline__ uint32_t ld_acquire_gpu(const uint32_t* p) {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Waits until *p >= target; false (and E_SCHED_TIMEOUT set) when the wait
// runs past `limit` cycles, false at once when another wait already failed.
__device__ bool front_wait(const uint32_t* p, uint32_t target, uint32_t* err, long long limit) {
    if (ld_acquire_gpu(p) >= target) return true;
    const long long t0 = clock64();
    for (;;) {
        __nanosleep(128);
        if (ld_acquire_gpu(p) >= target) return true;
        if (ld_acquire_gpu(err) & E_SCHED_TIMEOUT) return false;
        if (clock64() - t0 > limit) {
            atomicOr(err, E_SCHED_TIMEOUT);
            return false;
        }
    }
}

__device__ __forceinline__ void front_signal(uint32_t* p) {
    __threadfence();
    atomicAdd(p, 1u);
}

__global__ void __launch_bounds__(kFrontThreads, 3) k_front(const FrontArgs a) {
    extern __shared__ __align__(16) uint8_t smem_f[];
    __shared__ uint32_t s_item;
    __shared__ uint32_t s_go;
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        __syncthreads();  // the previous item no longer reads shared memory
        if (tid == 0) s_item = (ld_acquire_gpu(a.err) & E_SCHED_TIMEOUT) ? a.nitems : atomicAdd(a.head, 1u);
        __syncthreads();
        const uint32_t it = s_item;
        if (it >= a.nitems) return;
        const FrontItem fi = a.items[it];
        if (fi.stage == FS_TOKENIZE) {
            // one tile per warp, each waiting for its own input's match table
            const uint32_t t = fi.idx + warp;
            if (warp < fi.job && t < a.ntiles) {
                const TokTile tt = a.tiles[t];
                uint32_t go = 0;
                if (lane == 0) go = front_wait(a.progress + tt.job, a.tok_target[tt.job], a.err, a.wait_cycles) ? 1u : 0u;
                go = __shfl_sync(0xFFFFFFFFu, go, 0);
                if (go) {
                    tokenize_tile<true>(a.in, a.jobs, tt, a.desc, a.slots, a.tile_lens, a.err,
                                  reinterpret_cast<TokSmem*>(smem_f)[warp]);
                    __syncwarp();
                    if (lane == 0) front_signal(a.progress + tt.job);
                }
            }
            continue;
        }
        if (tid == 0) s_go = front_wait(a.progress + fi.job, fi.target, a.err, a.wait_cycles) ? 1u : 0u;
        __syncthreads();
        if (!s_go) continue;
        switch (fi.stage) {
            case FS_TILE_FIND:
                tile_find_item(a.in, a.jobs, a.small[fi.idx], a.desc, smem_f, a.err);
                break;
            case FS_RX_SORT:
                rx_sort_item(a.in, a.jobs, a.rtiles[fi.idx], a.rx_toff, a.rx_list, *reinterpret_cast<RxSortSmem*>(smem_f));
                break;
            case FS_RX_RESOLVE:
                rx_resolve_warp<true>(a.jobs, fi.job, fi.idx + warp, a.rx_toff, a.rx_list, a.rx_pred,
                                reinterpret_cast<uint32_t*>(smem_f) + warp * kRxKeys);
                break;
            case FS_RX_VERIFY: {
                const Job job = a.jobs[fi.job];
                const uint32_t hi = min(rx_ncand(job.n), fi.idx + a.verify_chunk);
                rx_verify_range<true>(a.in, job, a.rx_list, a.rx_pred, a.desc, fi.idx, hi, tid, kFrontThreads);
                break;
            }
            case FS_GATHER:
                gather_item<true>(a.jobs, fi.idx, a.slots, a.tile_lens, a.streams, a.job_lens, a.hist, a.err,
                            reinterpret_cast<uint32_t*>(smem_f) + 4 * 4 * 256,
                            reinterpret_cast<uint32_t(*)[4][256]>(smem_f));
                break;
            default:
                break;
        }
        __syncthreads();
        if (tid == 0) front_signal(a.progress + fi.job);
    }
}

}  // namespace pz
