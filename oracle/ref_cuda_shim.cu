// Test-only host shim around the reference's own CUDA kernels.
//
// The reference compiles gpu/kernel/przm_lz77.cu (which #includes
// przm_tokenizer.cuh and przm_ans.cu) into one module and launches its
// kernels from Go with cuLaunchKernel.  This file is compiled together with
// that source (oracle/Makefile, -I<checkout>/gpu/kernel) and adds C entry
// points for the kernels that have no host wrapper of their own, with the
// launch shapes the Go bridge uses:
//   histogram: clear <<<1,256>>> + przm_byte_histogram_kernel <<<224,256>>>
//              (gpu/bridge.go:2904-2934)
//   V-ANS:     przm_vans_encode4x_kernel <<<1,256>>> (gpu/bridge.go:3206-3211)
// The host wrappers that already exist in the reference source
// (cuda_lz77_match_batch, cuda_lz77_radix_strike_batch,
// cuda_lz77_compact_stream, cuda_lz77_tokenize_stream) are exported as they are.
#include "przm_lz77.cu"

extern "C" int ref_histogram(const uint8_t* d_in, uint32_t n, uint32_t* d_hist, uint32_t* d_meta, void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    przm_clear_histogram_kernel<<<1, 256, 0, s>>>(d_hist, d_meta);
    przm_byte_histogram_kernel<<<224, 256, 0, s>>>(d_in, n, d_hist, d_meta);
    return (int)cudaGetLastError();
}

extern "C" int ref_vans_encode4x(const uint8_t* d_in, uint32_t n, const uint16_t* d_freq, const uint16_t* d_cdf,
                                 const uint8_t* d_mat, uint32_t mat_len, uint8_t* d_out, uint32_t* d_out_len,
                                 uint8_t* d_temp, void* stream) {
    przm_vans_encode4x_kernel<<<1, 256, 0, (cudaStream_t)stream>>>(d_in, n, d_freq, d_cdf, d_mat, mat_len, d_out,
                                                                   d_out_len, d_temp);
    return (int)cudaGetLastError();
}

// Tokenizer with the Go bridge's launch shape (one warp per 32 KiB tile,
// gpu/bridge.go:1693-1702), followed by the reference scan and gather.
extern "C" int ref_tokenize(const uint8_t* d_in, uint64_t n, const uint32_t* d_matches, uint8_t* d_chunk_cmds,
                            uint8_t* d_chunk_offs, uint8_t* d_chunk_lits, uint32_t* d_lens /* 6 * chunks */,
                            uint32_t* d_totals, uint8_t* d_cmds, uint8_t* d_offs, uint8_t* d_lits, uint32_t num_chunks,
                            void* stream) {
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t* cl = d_lens;
    uint32_t* ol = d_lens + num_chunks;
    uint32_t* ll = d_lens + 2 * num_chunks;
    uint32_t* co = d_lens + 3 * num_chunks;
    uint32_t* oo = d_lens + 4 * num_chunks;
    uint32_t* lo = d_lens + 5 * num_chunks;
    przm_fused_tokenizer_kernel<<<num_chunks, 32, 0, s>>>(d_in, n, d_matches, d_chunk_cmds, d_chunk_offs, d_chunk_lits,
                                                          cl, ol, ll, PRZM_TOKENIZER_TILE_SIZE, PRZM_MAX_TILE_CMD_BYTES,
                                                          PRZM_MAX_TILE_OFF_BYTES, PRZM_MAX_TILE_LIT_BYTES, num_chunks);
    przm_tokenizer_scan_kernel<<<1, 96, 0, s>>>(cl, ol, ll, co, oo, lo, d_totals, num_chunks);
    uint32_t g = num_chunks < 256 ? num_chunks : 256;
    przm_tokenizer_gather_kernel<<<g, 256, 0, s>>>(d_chunk_cmds, d_chunk_offs, d_chunk_lits, cl, ol, ll, co, oo, lo,
                                                    d_cmds, d_offs, d_lits, PRZM_MAX_TILE_CMD_BYTES,
                                                    PRZM_MAX_TILE_OFF_BYTES, PRZM_MAX_TILE_LIT_BYTES, num_chunks);
    return (int)cudaGetLastError();
}
