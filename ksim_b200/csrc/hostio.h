// hostio.h — the chunk plan of a host-buffer sampling call (host code only).
//
// A call on host buffers (ksim_program_sample and its packed and noisy
// forms) samples B shots in chunks so that copies overlap sampling.  The
// plan is kept here, free of CUDA, so the CPU tests check it directly.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

namespace ksim {

// Chunk boundaries of a host call over B shots whose rows move row_bytes
// across PCIe (input and output together).  Only the first chunk's input
// copy and the last chunk's output copy are not hidden behind sampling, so
// the chunks ramp: u, 2u, then chunks of about 4u, then 2u, u, with u about
// B / 32 shots — at least 16 Ki shots and 256 KiB of copies (a chunk costs
// a few microseconds of launches and events, which a smaller copy does not
// repay), a multiple of 4 Ki.  Returns 0 = b_0 < b_1 < ... < b_n = B.
inline std::vector<int64_t> host_chunk_bounds(int64_t B, int64_t row_bytes)
{
    const int64_t by_bytes = ((int64_t)1 << 18) / std::max<int64_t>(row_bytes, 1);
    const int64_t u = (std::max<int64_t>({(int64_t)1 << 14, B / 32, by_bytes}) + 4095) / 4096 * 4096;
    std::vector<int64_t> b = {0};
    if (B <= 6 * u) {  // too few shots to ramp: chunks of u
        for (int64_t x = u; x < B; x += u) b.push_back(x);
        b.push_back(B);
        return b;
    }
    b.push_back(u);
    b.push_back(3 * u);
    const int64_t body = B - 6 * u, n_body = (body + 4 * u - 1) / (4 * u);
    const int64_t step = (body / n_body + 4095) / 4096 * 4096;
    for (int64_t k = 1; k < n_body; ++k) b.push_back(3 * u + k * step);
    b.push_back(B - 3 * u);
    b.push_back(B - u);
    b.push_back(B);
    return b;
}

// How many chunks behind the sampling a call issues each chunk's output
// copy: one wave of sampling CTAs (wave_shots) over the largest chunk,
// between 1 and max_lag (the compute streams).  Into page-locked memory the
// copies are asynchronous anyway; into pageable memory each one holds the
// host until it is done, and the lag keeps about a wave queued meanwhile
// without leaving many copies for after the last chunk.
inline int host_copy_lag(const std::vector<int64_t> &bounds, int64_t wave_shots, int max_lag)
{
    int64_t largest = 1;
    for (size_t i = 0; i + 1 < bounds.size(); ++i) largest = std::max(largest, bounds[i + 1] - bounds[i]);
    return (int)std::min<int64_t>(max_lag, std::max<int64_t>(1, (wave_shots + largest - 1) / largest));
}

}  // namespace ksim
