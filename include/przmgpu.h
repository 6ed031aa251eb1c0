/*
 * przmgpu.h -- C ABI of the B200 PRZM compression path (libprzmgpu.so).
 *
 * Drop-in boundary for the reference's Go `gpu` package (Lemon4ksan/przm,
 * gpu/bridge.go, gpu/types.go, gpu/memory.go).  Every entry point below
 * names the reference function it replaces.  A Go caller binds these through
 * cgo; Python tests bind them through ctypes.
 *
 * Conventions
 *   - status: int32, 0 = OK, negative = error (PRZMG_ERR_*); the numeric
 *     values of the shared codes follow include/przm_dec.h of the reference;
 *   - the caller owns every host buffer; the library owns device memory of a
 *     context (grow-only pools, like ensureSlotCap, gpu/bridge.go:807-922);
 *   - device pointers and CUDA streams travel as uint64_t (the reference
 *     passes uint64 device pointers and uintptr streams);
 *   - a context serialises its calls with an internal mutex, as every
 *     GPUCompressor method does (for example gpu/bridge.go:1487-1488);
 *   - empty inputs succeed with zero-length results (gpu/bridge.go:1089-1091).
 */
#ifndef PRZMGPU_H
#define PRZMGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PRZMG_OK 0
#define PRZMG_ERR_INVALID_ARG (-1)       /* same value as PRZM_ERR_CORRUPTED_FRAME */
#define PRZMG_ERR_BUFFER_TOO_SMALL (-4)  /* PRZM_ERR_BUFFER_TOO_SMALL */
#define PRZMG_ERR_EXCEEDS_MAX_BLOCK (-5) /* PRZM_ERR_EXCEEDS_MAX_BLOCK */
#define PRZMG_ERR_CUDA (-10)             /* a CUDA runtime call failed (cuCheck, gpu/bridge.go:24-29) */
#define PRZMG_ERR_UNAVAILABLE (-11)      /* no usable device (IsAvailable() == false) */
#define PRZMG_ERR_MOCK (-12)             /* SetMockMatchErrorForTest is armed */
#define PRZMG_ERR_DEVICE (-13)           /* a kernel reported an internal bound violation */
#define PRZMG_ERR_NOT_FOUND (-14)        /* serving: unknown request id */
#define PRZMG_ERR_BUSY (-15)             /* serving: admission refused (budget or queue full) */
/* decoder status codes: the reference decoder's own values (przm_dec.h) */
#define PRZMG_ERR_CORRUPTED_FRAME (-1)   /* PRZM_ERR_CORRUPTED_FRAME (also PRZMG_ERR_INVALID_ARG) */
#define PRZMG_ERR_INVALID_MAGIC (-2)     /* PRZM_ERR_INVALID_MAGIC */
#define PRZMG_ERR_UNSUPPORTED_MODE (-6)  /* PRZM_ERR_UNSUPPORTED_MODE: a frame feature the GPU decoder does not take */

#define PRZMG_PROFILE_D2D 0   /* CompressD2D frame: flat sections, raw literals */
#define PRZMG_PROFILE_ANS 1   /* match + tokenize + ANS frame (Mode 8 + V-ANS)   */
/* PRZMG_PROFILE_ANS with Section 3 as the CPU compressor writes it
 * (PackageOffsetsSection, core/distance/distance.go:825-849, called from
 * compress.go:956): the frame's distances as a distance-prefix container
 * (Mode 12 or adaptive V-ANS codes + MSB-first extra bits) or 0x09 + LEB128
 * varints, and an empty Section 3 when the frame has no distance.  No GPU
 * entry point of the reference writes this frame; its decoders read it. */
#define PRZMG_PROFILE_ANS_DIST 2
/* PRZMG_PROFILE_ANS_DIST with Section 4 as the CPU compressor writes it
 * (PackageLiteralsSection, core/literals/literals.go:664-693, called from
 * compress.go:957): the smallest of the raw literals, their adaptive V-ANS
 * container and the four étale-sheaf foliations (core/literals/sheaf.go),
 * raw under PRZMG_PROFILE_ANS's decodability rule.  No GPU entry point of
 * the reference writes this frame; its decoders read it. */
#define PRZMG_PROFILE_ANS_SHEAF 3

#define PRZMG_NORM_GO 0       /* gpu.NormalizeFreq, container flag 0x01 */
#define PRZMG_NORM_CPU 1      /* literals.NormalizeFrequencies, flag 0x00 */

typedef struct przmg_ctx przmg_ctx;
typedef struct przmg_batch przmg_batch;

/* GPUProfile, gpu/types.go:55-71 */
typedef struct {
    uint64_t ingress_dma_bytes;
    double ingress_dma_time_ms;
    double ingress_dma_bandwidth_gbps;
    double kernel_time_ms;
    double internal_vram_bandwidth_gbps;
    uint64_t egress_dma_bytes;
    double egress_dma_time_ms;
    double egress_dma_bandwidth_gbps;
    double total_round_trip_ms;
    double end_to_end_bandwidth_gbps;
    double pcie_overhead_percent;
    char device_name[128];
    int32_t sm_count;
    int32_t pipelined_chunks;
    uint64_t total_vram_bytes;
} przmg_profile_t;

/* TokenizerProfile, gpu/types.go:74-85 */
typedef struct {
    double kernel_time_ms;
    double pass1_ms;
    double pass2_ms;
    double pass3_ms;
    double total_round_trip_ms;
    double throughput_gbps;
    int64_t cmd_bytes;
    int64_t offset_bytes;
    int64_t literal_bytes;
    int64_t num_chunks;
} przmg_tokenizer_profile_t;

/* DeviceTokenStreams, gpu/types.go:90-100 (pointers borrowed from the
 * context; the next call on the context invalidates them, gpu/bridge.go:2122) */
typedef struct {
    uint64_t d_final_cmds;
    uint64_t d_final_offs;
    uint64_t d_final_lits;
    uint64_t d_totals;
    uint32_t cmd_len;
    uint32_t off_len;
    uint32_t lit_len;
    uint32_t num_chunks;
    uint64_t stream;
} przmg_device_streams_t;

/* LZ77Match, gpu/types.go:19-24 */
typedef struct {
    uint32_t position;
    uint32_t offset;
    uint16_t length;
    uint8_t literal;
    uint8_t reserved;
} przmg_match_t;

/* One input of a batch call (host buffers). */
typedef struct {
    const uint8_t* src;
    uint64_t n;
    uint8_t* dst;
    uint64_t cap;
    uint64_t out_len;   /* out: frame size */
    int32_t status;     /* out */
    int32_t reserved;
} przmg_job_t;

/* ---- discovery and lifetime ------------------------------------------- */
int32_t przmg_is_available(void);                              /* IsAvailable, gpu/bridge.go:61 */
int32_t przmg_init(int32_t device, przmg_ctx** out);            /* NewGPUCompressor, gpu/bridge.go:291 */
int32_t przmg_get_global(przmg_ctx** out);                      /* GetGlobalCompressor, gpu/bridge.go:96 */
void przmg_reset_global_for_test(void);                         /* ResetGlobalCompressorForTest, :117 */
/* (*GPUCompressor).Close, :513.  Batches (przmg_batch_create) and serving
 * engines (przmg_serve_create) use their context until they are destroyed:
 * destroy them first. */
int32_t przmg_close(przmg_ctx* ctx);
void przmg_set_mock_unavailable(int32_t unavailable);           /* SetMockUnavailableForTest, :45 */
void przmg_set_mock_match_error(int32_t code);                  /* SetMockMatchErrorForTest, :50 (0 clears) */
/* ComputeMajor/ComputeMinor/DeviceName/SMCount/TotalVRAMBytes fields, :283-287 */
int32_t przmg_device_info(przmg_ctx* ctx, int32_t* major, int32_t* minor, char* name, size_t name_cap,
                          int32_t* sm_count, uint64_t* total_vram);
const char* przmg_last_error(void);                             /* message of the calling thread's last error */

/* ---- match finding ------------------------------------------------------ */
/* MatchLZ77, gpu/bridge.go:1480 (radix strike for every size; > 16 MiB is
 * streamed in 8 MiB chunks).  out must hold n entries. */
int32_t przmg_match_lz77(przmg_ctx* ctx, const uint8_t* src, uint64_t n, przmg_match_t* out, uint64_t cap,
                         uint64_t* n_out, przmg_profile_t* prof);
/* Per-position match descriptors that Tokenize/CompressD2D consume: the
 * slot's dMatch after launchMatchSearch, gpu/bridge.go:924-950 (tile finder
 * for n <= 64 KiB, radix strike above; packing of gpu/types.go:27-33).
 * desc must hold n entries. */
int32_t przmg_match_table(przmg_ctx* ctx, const uint8_t* src, uint64_t n, uint32_t* desc);
/* MatchLZ77Streaming, gpu/bridge.go:1461 (chunk <= 0 picks the default) */
int32_t przmg_match_lz77_streaming(przmg_ctx* ctx, const uint8_t* src, uint64_t n, int64_t chunk,
                                   przmg_match_t* out, uint64_t cap, uint64_t* n_out, przmg_profile_t* prof);

/* ---- tokenization ------------------------------------------------------- */
/* Tokenize, gpu/bridge.go:1895: lens[0..2] = cmd/off/lit bytes written. */
int32_t przmg_tokenize(przmg_ctx* ctx, const uint8_t* src, uint64_t n, uint8_t* cmd, uint64_t cmd_cap, uint8_t* off,
                       uint64_t off_cap, uint8_t* lit, uint64_t lit_cap, uint64_t lens[3],
                       przmg_tokenizer_profile_t* prof);
/* TokenizeDevice / TokenizeDeviceZeroCopy, gpu/bridge.go:2139, 2247 */
int32_t przmg_tokenize_device(przmg_ctx* ctx, const uint8_t* src, uint64_t n, przmg_device_streams_t* out,
                              przmg_tokenizer_profile_t* prof);
/* TokenizeDeviceOnly, gpu/bridge.go:1915: runs only the tokenizer (parse,
 * scan and gather) again on the input and match table the context staged in
 * device memory for its last one-input call (przmg_tokenize,
 * przmg_tokenize_device, przmg_match_table, przmg_compress...), and copies
 * the streams out as przmg_tokenize does.  n must equal that input's size
 * (the reference reads whatever its slot holds; here a call with nothing
 * staged, or with another n, fails with PRZMG_ERR_INVALID_ARG).  n == 0
 * succeeds with empty streams. */
int32_t przmg_tokenize_device_only(przmg_ctx* ctx, uint64_t n, uint8_t* cmd, uint64_t cmd_cap, uint8_t* off,
                                   uint64_t off_cap, uint8_t* lit, uint64_t lit_cap, uint64_t lens[3],
                                   przmg_tokenizer_profile_t* prof);
/* TokenizePointersDeviceOnly, gpu/bridge.go:2163: the same tokenizer-only
 * run, returning borrowed device pointers like przmg_tokenize_device. */
int32_t przmg_tokenize_pointers_device_only(przmg_ctx* ctx, uint64_t n, przmg_device_streams_t* out,
                                            przmg_tokenizer_profile_t* prof);
/* DownloadDeviceBytes, gpu/bridge.go:2253 */
int32_t przmg_download_device_bytes(przmg_ctx* ctx, uint64_t d_ptr, uint64_t size, uint8_t* dst);

/* ---- frames ------------------------------------------------------------- */
uint64_t przmg_frame_bound(uint64_t n);                         /* capacity a frame of n input bytes needs */
/* EncodeD2D, gpu/bridge.go:2466 (window_log 0 picks 16/20/23 by size) */
int32_t przmg_encode_d2d(przmg_ctx* ctx, const przmg_device_streams_t* streams, uint32_t usize, int32_t window_log,
                         uint8_t* dst, uint64_t cap, uint64_t* out_len, przmg_profile_t* prof);
/* CompressD2D, gpu/bridge.go:2486 */
int32_t przmg_compress_d2d(przmg_ctx* ctx, const uint8_t* src, uint64_t n, uint8_t* dst, uint64_t cap,
                           uint64_t* out_len, przmg_profile_t* prof);
/* Compress with GPUAcceleration (api.go:15/32 + options.go:85): PRZMG_PROFILE_ANS
 * is the entropy-coded frame; n must stay below 16 MiB (24-bit uSize). */
int32_t przmg_compress(przmg_ctx* ctx, const uint8_t* src, uint64_t n, int32_t profile, uint8_t* dst, uint64_t cap,
                       uint64_t* out_len, przmg_profile_t* prof);
/* Many inputs in one call (no reference counterpart; the reference compresses
 * one input per call).  batched = 1: one launch sequence for all inputs;
 * batched = 0: one launch sequence and one synchronisation per input. */
int32_t przmg_compress_batch(przmg_ctx* ctx, przmg_job_t* jobs, uint64_t njobs, int32_t profile, int32_t batched,
                             przmg_profile_t* prof);

/* Many inputs laid back to back in host memory (pinned for full speed):
 * frames come back back to back in host_out; out_sizes (optional, njobs)
 * receives each frame's size.  No reference counterpart. */
int32_t przmg_compress_packed(przmg_ctx* ctx, const uint8_t* host_in, const uint64_t* sizes, uint64_t njobs,
                              int32_t profile, uint8_t* host_out, uint64_t out_cap, uint32_t* out_sizes,
                              uint64_t* out_total);

/* Device-resident batches (inputs already in HBM; used for throughput runs). */
int32_t przmg_batch_create(przmg_ctx* ctx, const uint64_t* sizes, uint64_t njobs, int32_t profile,
                           przmg_batch** out);
/* device base of the packed inputs and the per-input byte offsets (njobs) */
int32_t przmg_batch_inputs(przmg_batch* b, uint64_t* d_in, uint64_t* offsets);
/* device base of the frames and their byte offsets (njobs) */
int32_t przmg_batch_outputs(przmg_batch* b, uint64_t* d_out, uint64_t* offsets);
/* enqueue the whole pipeline on `stream` (0: the context stream); use_graph
 * replays a captured CUDA graph of the same sequence */
int32_t przmg_batch_enqueue(przmg_batch* b, uint64_t stream, int32_t use_graph);
/* synchronise and read back frame sizes (njobs) and the kernel error word */
int32_t przmg_batch_sizes(przmg_batch* b, uint32_t* sizes);
/* kernels a single enqueue launches (for launch accounting) */
int32_t przmg_batch_launch_count(przmg_batch* b);
/* Plain per-input launches of the same batch: the pipeline enqueued once per
 * input, input after input on `stream`, each launch sized for that input
 * alone -- what a caller of the reference's one-input API gets
 * (gpu/bridge.go:2486-2544 compresses one input per call).  The frames are
 * byte-identical to przmg_batch_enqueue's; *launches (optional) = kernels
 * launched.  For comparisons of batched against plain launches. */
int32_t przmg_batch_enqueue_plain(przmg_batch* b, uint64_t stream, int32_t* launches);

/* ---- launch geometry per size class (no reference counterpart: the
 * reference launches fixed grids, gpu/bridge.go:924-1068) ------------------
 * A batch belongs to size class przmg_size_class(mean input bytes): 0 up to
 * 64 KiB, 1 up to 768 KiB, 2 up to 2 MiB, 3 above.  Per class: front = 1 runs
 * the match finders, tokenizer and gather as ONE persistent launch whose
 * blocks take work items (tiles, verify chunks, frames) from a device queue,
 * front = 0 one kernel per stage; ctas_per_sm (1-3) and verify_chunk (radix
 * candidates per work item, a multiple of 256) shape the persistent launch.
 * The values come from the autotuner (przm_b200/autotune.py); none changes an
 * output byte.  A batch takes its class's values when it is laid out
 * (przmg_batch_create, or each one-input / many-input call). */
int32_t przmg_size_class(uint64_t mean_input_bytes);
int32_t przmg_set_tuning(przmg_ctx* ctx, int32_t size_class, int32_t front, int32_t ctas_per_sm, int32_t verify_chunk);
int32_t przmg_get_tuning(przmg_ctx* ctx, int32_t size_class, int32_t* front, int32_t* ctas_per_sm,
                         int32_t* verify_chunk);
/* info[0] = 1 if the batch runs the persistent front end, [1] size class,
 * [2] blocks per SM, [3] verify chunk */
int32_t przmg_batch_info(przmg_batch* b, uint32_t info[4]);
/* Every wait of the persistent front end (an item waiting for the earlier
 * stages of its input) gives up after limit_ns (default 1 s), sets an error
 * bit and stops the launch; the call then returns PRZMG_ERR_DEVICE and the
 * context stays usable.  add_unreachable_wait = 1 appends to batches laid
 * out afterwards one item whose wait never ends (for testing that path). */
int32_t przmg_set_front_wait(przmg_ctx* ctx, uint64_t limit_ns, int32_t add_unreachable_wait);
/* copy back-to-back host inputs (sum of the sizes, pinned for full PCIe
 * speed) into the batch's inputs, asynchronously on `stream` */
int32_t przmg_batch_upload(przmg_batch* b, const uint8_t* host, uint64_t stream);
/* synchronise, then copy the frames back to back into host (capacity cap);
 * total = bytes written, sizes (optional) = per-frame sizes */
int32_t przmg_batch_download(przmg_batch* b, uint8_t* host, uint64_t cap, uint64_t* total, uint32_t* sizes,
                             uint64_t stream);
/* one enqueue with CUDA events between the stages; ms[k] = device time of
 * stage k (names from przmg_stage_name), count = stages reported */
int32_t przmg_batch_stage_times(przmg_batch* b, float* ms, int32_t cap, int32_t* count);
const char* przmg_stage_name(int32_t k);
/* totals of the last run (synchronises): input, frame, literal, command and
 * offset bytes, rANS symbols and emitted bytes, uncompressed frames */
int32_t przmg_batch_stats(przmg_batch* b, uint64_t stats[8]);
/* per-input stream lengths of the last run (synchronises): lens[6 i + s] for
 * s = commands, op, meta, var substreams, offsets, literals; cap = entries */
int32_t przmg_batch_stream_lens(przmg_batch* b, uint32_t* lens, uint64_t cap);
int32_t przmg_batch_destroy(przmg_batch* b);

/* ---- serving: continuous batching (no reference counterpart; the reference
 * has no request loop, the north-star serving pattern) ---------------------
 * przmg_serve_create starts an engine on a context: up to max_inflight
 * batches run at once, each on its own stream with its own resident device
 * buffers, each laid out within mem_budget / max_inflight device bytes (and
 * max_batch_bytes of input, 0 = 256 MiB).  Requests are copied at submit;
 * requests that arrive while batches run join the next batch.  A request's
 * frame is byte-identical to a one-input przmg_compress of the same input and
 * profile.  poll returns 1 when the frame is copied out (the request is then
 * released), 0 while pending (wait = 0), < 0 on error; t_submit_ns/t_done_ns
 * are steady-clock stamps of submission and of completion (frame on the
 * host).  Status codes: PRZMG_ERR_BUSY (queue full), PRZMG_ERR_NOT_FOUND
 * (unknown or released id), PRZMG_ERR_EXCEEDS_MAX_BLOCK (n >= 16 MiB for
 * PRZMG_PROFILE_ANS), PRZMG_ERR_BUFFER_TOO_SMALL (dst smaller than the frame;
 * the request stays pollable). */
typedef struct przmg_server przmg_server;
int32_t przmg_serve_create(przmg_ctx* ctx, int32_t profile, uint64_t mem_budget, int32_t max_inflight,
                           uint64_t max_batch_bytes, przmg_server** out);
int32_t przmg_serve_submit(przmg_server* s, const uint8_t* src, uint64_t n, uint64_t* id);
int32_t przmg_serve_poll(przmg_server* s, uint64_t id, int32_t wait, uint8_t* dst, uint64_t cap, uint64_t* out_len,
                         uint64_t* t_submit_ns, uint64_t* t_done_ns);
/* stats[8]: batches launched, requests finished, input bytes, frame bytes,
 * largest batch (requests), most batches in flight at once, requests pending,
 * requests not yet polled */
int32_t przmg_serve_stats(przmg_server* s, uint64_t stats[8]);
/* t[6]: per-batch host times in ms, summed and largest: {sum launch, sum
 * wait, sum out, max launch, max wait, max out}; launch = lay out, stage,
 * upload and enqueue; wait = launched -> complete on the device; out =
 * download and hand the frames to their requests */
int32_t przmg_serve_timing(przmg_server* s, double t[6]);
/* finishes the batches in flight, then frees the engine */
int32_t przmg_serve_destroy(przmg_server* s);

/* ---- histogram / flat pack / V-ANS ------------------------------------- */
/* ComputeHistogramGPU, gpu/bridge.go:2890 */
int32_t przmg_compute_histogram_gpu(przmg_ctx* ctx, uint64_t d_in, uint64_t n, uint64_t stream, uint32_t counts[256],
                                    double* ms, double* gbps);
/* ComputeHistogramHost, gpu/bridge.go:2961 */
int32_t przmg_compute_histogram_host(przmg_ctx* ctx, const uint8_t* src, uint64_t n, uint32_t counts[256],
                                     przmg_profile_t* prof);
/* PackStreamFlatGPU, gpu/bridge.go:3033 (out_len = n + 5) */
int32_t przmg_pack_stream_flat_gpu(przmg_ctx* ctx, uint64_t d_in, uint64_t d_out, uint64_t n, uint64_t stream,
                                   uint64_t* out_len, double* ms, double* gbps);
/* PackStreamFlatHost, gpu/bridge.go:3079 */
int32_t przmg_pack_stream_flat_host(przmg_ctx* ctx, const uint8_t* src, uint64_t n, uint8_t* dst, uint64_t cap,
                                    uint64_t* out_len, przmg_profile_t* prof);
/* VANSEncode4xGPU, gpu/bridge.go:3161 (container flag 0x01) */
int32_t przmg_vans_encode4x_gpu(przmg_ctx* ctx, uint64_t d_in, uint64_t d_out, uint64_t n, const uint16_t freq[256],
                                const uint16_t cdf[257], const uint8_t* mat, uint32_t mat_len, uint64_t stream,
                                uint64_t* out_len, double* ms, double* gbps);
/* VANSEncode4xHost, gpu/bridge.go:3233 */
int32_t przmg_vans_encode4x_host(przmg_ctx* ctx, const uint8_t* src, uint64_t n, uint8_t* dst, uint64_t cap,
                                 uint64_t* out_len, przmg_profile_t* prof);
/* Histogram + normalise + V-ANS of many device streams in one launch sequence
 * (no reference counterpart: the reference encodes one stream per call).
 * norm: PRZMG_NORM_GO (NormalizeFreq, flag 0x01) or PRZMG_NORM_CPU
 * (NormalizeFrequencies, EncodeAdaptiveVANS4x, flag 0x00).  out_offs[i] must
 * leave room for 1024 + 2 * lens[i] bytes. */
int32_t przmg_vans_encode_batch(przmg_ctx* ctx, uint64_t d_in, const uint64_t* in_offs, const uint32_t* lens,
                                uint64_t count, int32_t norm, uint64_t d_out, const uint64_t* out_offs,
                                uint32_t* out_lens, uint64_t stream);
/* PackageOffsetsSection, core/distance/distance.go:825-849, for many
 * distance arrays in one call: the Section 3 bytes the reference's CPU
 * compressor writes for each (a distance-prefix container 0x0B/0x0A/0x06 whose
 * code stream is Mode 12 or the codes' adaptive V-ANS container, or 0x09 +
 * LEB128 varints; nothing for an empty array).  d_dist + 4 * dist_offs[i]
 * holds counts[i] <= 2^21 uint32 distances; section i goes to
 * d_out + out_offs[i], whose out_caps[i] bytes must hold 1 + 5 * counts[i]
 * in the worst case; out_lens[i] receives its size.  Synchronises the stream.
 * PRZMG_ERR_EXCEEDS_MAX_BLOCK for an array above 2^21 distances (nothing
 * runs), PRZMG_ERR_BUFFER_TOO_SMALL when a section does not fit its capacity
 * (that section is left empty with out_lens[i] = 0; the others are written). */
int32_t przmg_package_offsets_batch(przmg_ctx* ctx, uint64_t d_dist, const uint64_t* dist_offs, const uint32_t* counts,
                                    uint64_t count, uint64_t d_out, const uint64_t* out_offs, const uint64_t* out_caps,
                                    uint64_t* out_lens, uint64_t stream);
/* PackageLiteralsSection, core/literals/literals.go:664-693, for many
 * literal streams in one call: the Section 4 bytes the reference's CPU
 * compressor writes for each -- the smallest of the adaptive V-ANS container
 * and the four étale-sheaf foliations (literals.go:600-662, sheaf.go) when
 * one is smaller than the literals, else the literals themselves -- and its
 * flag nibble (nibbles[i] = 0x80 for a container, 0 for raw).  Stream i is
 * lens[i] <= 4 MiB bytes at d_in + in_offs[i]; its section goes to
 * d_out + out_offs[i] (out_caps[i] >= lens[i] always suffices).  At most
 * 65535 streams per call.  Synchronises the stream.
 * PRZMG_ERR_EXCEEDS_MAX_BLOCK for a stream above 4 MiB (nothing runs),
 * PRZMG_ERR_BUFFER_TOO_SMALL when a section does not fit its capacity (that
 * section is left empty with out_lens[i] = 0; the others are written). */
int32_t przmg_package_literals_batch(przmg_ctx* ctx, uint64_t d_in, const uint64_t* in_offs, const uint32_t* lens,
                                     uint64_t count, uint64_t d_out, const uint64_t* out_offs, const uint64_t* out_caps,
                                     uint64_t* out_lens, uint8_t* nibbles, uint64_t stream);

/* ---- allocation-free V-ANS encode: no counterpart in the reference -------
 * Histogram + normalise + V-ANS of ONE device stream: the same launch
 * sequence and the same container bytes as przmg_vans_encode_batch with
 * count == 1, for callers that must not allocate device memory (a serving
 * loop whose device-memory budget is spent, an out-of-memory recovery path,
 * or a stream that must not meet the device-wide synchronisation of
 * cudaFree).  It allocates nothing: no cudaMalloc/cudaFree, no host staging
 * copy, no context; all scratch is one file-scope __device__ array of about
 * 2.3 MiB per device, so n is limited to PRZMG_NOALLOC_MAX_N symbols.
 *   n > PRZMG_NOALLOC_MAX_N           -> PRZMG_ERR_EXCEEDS_MAX_BLOCK
 *   out_cap < 1024 + 2 * n            -> PRZMG_ERR_BUFFER_TOO_SMALL
 *   unknown norm, null address, or
 *   d_out_len not 4-byte aligned      -> PRZMG_ERR_INVALID_ARG
 * (nothing is launched on these errors; przmg_last_error() says why).  A
 * CUDA error pending from earlier work is returned (PRZMG_ERR_CUDA) before
 * anything is queued.  A CUDA error raised by one of the call's own launches
 * returns PRZMG_ERR_CUDA with part of the sequence already queued; d_out and
 * d_out_len are then undefined.
 * Runs on the CURRENT device, asynchronously on `stream` (0 = the legacy
 * default stream); the container length is written as a u32 to the device
 * address d_out_len (4-byte aligned) when the stream reaches it.  The first
 * call on each device does setup (cudaGetSymbolAddress of the scratch with
 * that device current, which may load the module, and the rANS kernel's
 * shared-memory attribute): make one call on every device before capturing a
 * stream.  The scratch address is looked up once per device and process:
 * after cudaDeviceReset of a device this entry point must not be called on
 * that device again in the same process (the cached address belonged to the
 * destroyed context).
 * Nothing in the scratch has to start at zero: each call clears the 1 KiB
 * histogram it counts into and overwrites the rest before reading it.
 * All calls on one device share the one scratch, so calls that overlap in
 * time (on two streams, or from two host threads) race and corrupt each
 * other's output: serialise them (one stream, or a lock around the call
 * and a wait for the stream). */
#define PRZMG_NOALLOC_MAX_N (1u << 20)
int32_t przmg_vans_encode_noalloc(uint64_t d_in, uint32_t n, int32_t norm, uint64_t d_out, uint64_t out_cap,
                                  uint64_t d_out_len, uint64_t stream);

/* host helpers */
void przmg_normalize_freq(const uint32_t counts[256], uint32_t target_m, uint16_t freq[256]); /* NormalizeFreq, :2777 */
void przmg_normalize_frequencies(const uint32_t counts[256], uint16_t freq[256]); /* literals.NormalizeFrequencies */
void przmg_build_cdf(const uint16_t freq[256], uint16_t cdf[257]);                 /* BuildCDF, :2832 */
uint32_t przmg_serialize_matrix(const uint16_t freq[256], uint8_t* out);          /* SerializeMatrix, :2844 (out >= 546) */

/* ---- benchmarks ---------------------------------------------------------- */
int32_t przmg_benchmark_vram_bandwidth(przmg_ctx* ctx, int32_t size_mb, int32_t iterations, double* gbps); /* :2674 */
int32_t przmg_benchmark_d2d_entropy(przmg_ctx* ctx, int32_t size_mb, int32_t iterations, double* gbps);     /* :2547 */
int32_t przmg_benchmark_entropy_vram(przmg_ctx* ctx, int32_t size_mb, int32_t iterations, double* gbps);   /* :3325 */

/* ---- pinned host memory (gpu/memory.go:51-165) --------------------------- */
int32_t przmg_alloc_pinned_host(uint64_t size, void** out); /* AllocPinnedHost */
int32_t przmg_free_pinned_host(void* p);                    /* FreePinnedHost */

/* PinnedBufferPool, gpu/memory.go:91-165: thread-safe reuse of pinned host
 * buffers of one size.  create = NewPinnedBufferPool(buf_size, initial_cap)
 * (initial_cap buffers allocated up front; the pool keeps at most
 * max(initial_cap, 8)); get = Get (a pooled buffer, else a new one); put =
 * Put (len must equal the pool's buffer size, else the buffer is ignored, as
 * in the reference; a full pool frees it); close = Close (frees the pooled
 * buffers, then the pool, unless the pool belongs to a context -- see
 * przmg_get_pinned -- in which case the context frees it in przmg_close). */
typedef struct przmg_pinned_pool przmg_pinned_pool;
int32_t przmg_pinned_pool_create(uint64_t buf_size, int32_t initial_cap, przmg_pinned_pool** out);
int32_t przmg_pinned_pool_get(przmg_pinned_pool* pool, void** buf);
void przmg_pinned_pool_put(przmg_pinned_pool* pool, void* buf, uint64_t len);
int32_t przmg_pinned_pool_close(przmg_pinned_pool* pool);
uint64_t przmg_pinned_pool_buf_size(const przmg_pinned_pool* pool);
uint64_t przmg_pinned_pool_pooled(przmg_pinned_pool* pool); /* buffers held (for tests) */
/* GetPinned, gpu/bridge.go:452: leases a buffer of at least size bytes from
 * the context's pool of the next power-of-two size (created on first use,
 * owned by the context).  *pool receives that pool: return the buffer with
 * przmg_pinned_pool_put(pool, buf, przmg_pinned_pool_buf_size(pool)). */
int32_t przmg_get_pinned(przmg_ctx* ctx, uint64_t size, void** buf, przmg_pinned_pool** pool);

/* ---- the GPU decoder (decompress.go:380-700, src/przm_dec.c:741-1529) -----
 * The reference's gpu package has no decoder: these decode PRZM frames on
 * the device with the semantics of its CPU decoder, for every frame this
 * library writes (profiles 0-3) and the frames of the same format written
 * elsewhere.  Frames that use an external dictionary, the base64
 * normalisation flag, delta-masked matches, the nibble-plane literal form or
 * the dictionary-word opcodes return PRZMG_ERR_UNSUPPORTED_MODE (decode those
 * on the host). */
/* Decompress (api.go:44): one frame from host memory into dst (dst_cap >=
 * the frame's size); *out_len = decoded bytes.  An empty src gives 0 bytes. */
int32_t przmg_decompress(przmg_ctx* ctx, const uint8_t* src, uint64_t src_len, uint8_t* dst, uint64_t dst_cap,
                         uint64_t* out_len);
/* count device-resident frames (d_src + src_offs[i], src_lens[i] bytes) into
 * d_dst + dst_offs[i] (dst_caps[i] bytes): status[i] (PRZMG_OK or the frame's
 * error) and out_lens[i] per frame; waits for the work (enqueued on
 * `stream`, 0 = the context's).  The return value is the call's own status. */
int32_t przmg_decompress_batch_device(przmg_ctx* ctx, uint64_t d_src, const uint64_t* src_offs,
                                      const uint32_t* src_lens, uint64_t count, uint64_t d_dst,
                                      const uint64_t* dst_offs, const uint32_t* dst_caps, int32_t* status,
                                      uint64_t* out_lens, uint64_t stream);
/* Every frame of the batch's last run decoded on the device and compared
 * with its input there; *bad = the frames that do not decode or differ.
 * Synchronises the device first. */
int32_t przmg_batch_verify(przmg_batch* b, uint64_t* bad);

#ifdef __cplusplus
}
#endif

#endif /* PRZMGPU_H */
