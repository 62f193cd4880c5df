// kernels.h — launch interface of the sm_100a kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "image.h"

// Resident CTAs of 256 threads per SM the sampling kernels are compiled for
// (it caps registers at 65536 / (256 * n)); the W > 4 batch kernel uses 1.
#ifndef KSIM_SAMPLE_MIN_CTAS
#define KSIM_SAMPLE_MIN_CTAS 2
#endif

// Shots one thread of the sampling kernels carries for parameter vectors of
// W words: two for W <= 4 (each column record is decoded once for both, and
// the two shots are independent dependency chains), one for wider vectors.
#ifndef KSIM_SHOTS_PER_THREAD
#define KSIM_SHOTS_PER_THREAD 2
#endif

namespace ksim {

__host__ __device__ constexpr int shots_per_thread(int W) { return W <= 4 ? KSIM_SHOTS_PER_THREAD : 1; }

// Shared memory of the warp-sliced parity rows (sample_tile.cuh): per warp one
// ballot word per parameter bit plus two zero words, per thread and shot
// ROW_WORDS row-parity words (the blocks of one term and one spare).
constexpr int ROW_WORDS = 9;
__host__ __device__ constexpr int ballot_words_per_warp(int W) { return 64 * W + 2; }
__host__ __device__ constexpr size_t sliced_smem_bytes(int W, int threads)
{
    return (size_t)(threads / 32) * (size_t)ballot_words_per_warp(W) * 8u +
           (size_t)ROW_WORDS * (size_t)shots_per_thread(W) * (size_t)threads * 4u;
}

// One sampling job: a component image, its input rows and output placement.
struct SampleJob {
    const uint8_t *image;      // device program image
    const GraphDir *gdir;      // = image
    const ChunkDir *cdir;      // device chunk directory for slot_bytes
    int32_t n_chunks, n_graphs, F, n_out;
    int32_t slot_bytes, rng_mode;
    const uint8_t *f;          // rows of f bytes
    int64_t f_stride;          // bytes between rows
    const int32_t *f_sel;      // nullable: column j of the component = f[row][f_sel[j]]
    uint8_t *out;              // output bytes
    int64_t out_stride, out_col0;
    const int32_t *out_cols;   // nullable: output i goes to column out_cols[i]
    double *amp;               // nullable: (B, n_out+1) |A_k|
    int64_t B, shot_offset;
    uint64_t seed;
    uint32_t *status;          // KSIM_FLAG_* accumulator
    int64_t wait_limit;        // > 0: a staging wait gives up after this many test_wait polls
    int64_t reserved;
};

struct LaunchCfg {
    int threads = 256;   // shots per CTA (one shot per thread)
    int staged = 1;      // stage term chunks in shared memory with TMA bulk copies
    int slot_bytes = 16384;
    int paths = 0;       // term paths the program uses: 0 all, 1 32-bit only, 2 32-bit and hybrid
                         // (the kernels compiled without the others)
};

// Launch the plain (one component per launch) sampler.
cudaError_t launch_sample(const SampleJob &job, int W, const LaunchCfg &cfg, cudaStream_t st);

enum EvalMode { EVAL_COMPLEX = 0, EVAL_ABS = 1, EVAL_TERMS = 2 };

struct EvalJob {
    const uint8_t *image;
    const GraphDir *gdir;
    int32_t graph;
    const uint8_t *params;   // (B, P) bytes
    int64_t B, P;
    int32_t mode;
    void *out;               // complex: (B,2) f64; abs: (B,) f64; terms: (B,G,5) i64
    uint32_t *status;
};

cudaError_t launch_eval(const EvalJob &job, int W, cudaStream_t st);

// Bit-packed rows (bit c of a row = byte c/8, bit c%8) <-> one byte per bit.
cudaError_t launch_unpack_bits(const uint8_t *packed, int64_t rows, int64_t packed_row, int64_t n_cols,
                               uint8_t *out, cudaStream_t st);
cudaError_t launch_pack_bits(const uint8_t *bytes, int64_t rows, int64_t n_cols, int64_t packed_row,
                             uint8_t *out, cudaStream_t st);

// The noise draw of a noise model (noise.cu): f rows of num_f bytes.
cudaError_t launch_noise(const ksim_noise *n, int64_t B, int64_t shot_offset, uint64_t seed, uint8_t *f,
                         int64_t f_stride, cudaStream_t st);

int noise_device(const ksim_noise *n);

// Shared-memory bytes of the staging ring (barriers + two slots).
size_t staged_smem_bytes(int slot_bytes);

// Shared-memory bytes of a sampling CTA: barriers, the staging slots when
// staged, then the sliced-parity scratch for W-word vectors.
inline size_t sample_smem_bytes(int slot_bytes, bool staged, int W, int threads)
{
    return (staged ? staged_smem_bytes(slot_bytes) : (size_t)128) + sliced_smem_bytes(W, threads);
}

}  // namespace ksim
