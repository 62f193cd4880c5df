// noise.cu — the per-shot noise draw (the f parameters) on the device.
//
// Reference: ChannelSampler (src/python/ksim/compile/channels.py:503-658).
// A noise model is a list of channels; channel i has 2^k_i outcome
// probabilities over its k_i error bits e, and error_transform (num_f x num_e,
// GF(2)) maps error bits to f parameters.  The reference draws, per channel,
// the shots where it fires by geometric skips along the shot axis and an
// outcome by searchsorted on the conditional CDF, then XORs the outcome's f
// pattern into those rows (channels.py:624-658), with numpy's PCG64 stream.
//
// Here one thread owns one shot and walks all channels in order:
//   fire    iff  u32(shot, channel) < thr_fire  (thr_fire = floor(p_fire 2^32))
//   outcome =    first o with u32'(shot, channel) < thr_cdf[o] (last otherwise)
//   f      ^=    pattern[outcome]          (packed 64-bit words of f bits)
// with counter-based Philox4x32-10 draws keyed by (seed, shot), so any shot
// range can be drawn alone and the CPU restatement in the oracle reproduces
// every bit.  Per channel, P(fire) and each P(outcome | fire) equal the
// reference's to within 2^-32 (integer thresholds); channels are independent,
// as in the reference, so the distribution of f is the reference's up to that
// quantisation.  The reference's channel simplification (merging, absorbing,
// folding) only regroups independent channels and does not change the
// distribution of f, so it is not repeated.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/ksim_b200.h"
#include "kernels.h"
#include "runtime.h"
#include "zring.cuh"

namespace ksim {

struct NoiseChan {
    uint32_t thr_fire;  // fire iff draw < thr_fire
    uint32_t n_out;     // outcomes other than the identity
    uint32_t cdf_off;   // n_out - 1 thresholds in the cdf array
    uint32_t pat_off;   // n_out patterns of W words in the pattern array
};

constexpr uint32_t NOISE_TAG_FIRE = 0x4E4F4953u;
constexpr uint32_t NOISE_TAG_OUTCOME = 0x4F55544Bu;

namespace {

template <int W>
__global__ void __launch_bounds__(256) k_noise(const NoiseChan *__restrict__ ch, const uint32_t *__restrict__ cdf,
                                               const uint64_t *__restrict__ pat, int n_ch, int num_f, int64_t B,
                                               int64_t shot_offset, uint64_t seed, uint8_t *__restrict__ f,
                                               int64_t f_stride)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B) return;
    const uint64_t shot = (uint64_t)(shot_offset + s);
    uint64_t acc[W];
#pragma unroll
    for (int w = 0; w < W; ++w) acc[w] = 0;
    for (int blk = 0; 4 * blk < n_ch; ++blk) {
        uint32_t x[4] = {(uint32_t)shot, (uint32_t)(shot >> 32), (uint32_t)blk, NOISE_TAG_FIRE};
        philox4x32_10(x, seed);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int c = 4 * blk + i;
            if (c >= n_ch) break;
            const NoiseChan cc = ch[c];
            if (x[i] >= cc.thr_fire) continue;
            uint32_t y[4] = {(uint32_t)shot, (uint32_t)(shot >> 32), (uint32_t)c, NOISE_TAG_OUTCOME};
            philox4x32_10(y, seed);
            uint32_t o = 0;
            while (o + 1 < cc.n_out && y[0] >= cdf[cc.cdf_off + o]) ++o;
            const uint64_t *pp = pat + cc.pat_off + (size_t)o * W;
#pragma unroll
            for (int w = 0; w < W; ++w) acc[w] ^= pp[w];
        }
    }
    uint8_t *row = f + s * f_stride;
    for (int j = 0; j < num_f; ++j) row[j] = (uint8_t)((acc[j >> 6] >> (j & 63)) & 1u);
}

template <int W>
cudaError_t launch_noise_w(const ksim_noise *n, int64_t B, int64_t shot_offset, uint64_t seed, uint8_t *f,
                           int64_t f_stride, cudaStream_t st);

}  // namespace
}  // namespace ksim

struct ksim_noise {
    int device = 0;
    int num_f = 0, num_e = 0, W = 1;
    int n_ch = 0;           // channels that can fire
    int64_t n_outcomes = 0; // patterns stored
    uint8_t *d_buf = nullptr;
    const ksim::NoiseChan *d_ch = nullptr;
    const uint32_t *d_cdf = nullptr;
    const uint64_t *d_pat = nullptr;
    size_t bytes = 0;
};

namespace ksim {
namespace {

template <int W>
cudaError_t launch_noise_w(const ksim_noise *n, int64_t B, int64_t shot_offset, uint64_t seed, uint8_t *f,
                           int64_t f_stride, cudaStream_t st)
{
    const int64_t blocks = (B + 255) / 256;
    if (blocks > 0x7FFFFFFF) return cudaErrorInvalidConfiguration;
    k_noise<W><<<(unsigned)blocks, 256, 0, st>>>(n->d_ch, n->d_cdf, n->d_pat, n->n_ch, n->num_f, B, shot_offset,
                                                 seed, f, f_stride);
    return cudaGetLastError();
}

// u in [0, 1] -> floor(u * 2^32), clamped to [0, 2^32 - 1]
uint32_t threshold32(double u)
{
    if (!(u > 0.0)) return 0u;
    const double t = std::floor(std::ldexp(u, 32));
    return t >= 4294967295.0 ? 4294967295u : (uint32_t)t;
}

}  // namespace

cudaError_t launch_noise(const ksim_noise *n, int64_t B, int64_t shot_offset, uint64_t seed, uint8_t *f,
                         int64_t f_stride, cudaStream_t st)
{
    if (B <= 0 || n->num_f == 0) return cudaSuccess;
    switch (n->W) {
    case 1: return launch_noise_w<1>(n, B, shot_offset, seed, f, f_stride, st);
    case 2: return launch_noise_w<2>(n, B, shot_offset, seed, f, f_stride, st);
    case 3: return launch_noise_w<3>(n, B, shot_offset, seed, f, f_stride, st);
    case 4: return launch_noise_w<4>(n, B, shot_offset, seed, f, f_stride, st);
    case 5: return launch_noise_w<5>(n, B, shot_offset, seed, f, f_stride, st);
    case 6: return launch_noise_w<6>(n, B, shot_offset, seed, f, f_stride, st);
    case 8: return launch_noise_w<8>(n, B, shot_offset, seed, f, f_stride, st);
    case 10: return launch_noise_w<10>(n, B, shot_offset, seed, f, f_stride, st);
    case 12: return launch_noise_w<12>(n, B, shot_offset, seed, f, f_stride, st);
    case 16: return launch_noise_w<16>(n, B, shot_offset, seed, f, f_stride, st);
    default: return cudaErrorInvalidValue;
    }
}

int noise_device(const ksim_noise *n) { return n->device; }

}  // namespace ksim

using namespace ksim;

extern "C" {

ksim_status ksim_noise_create(const double *probs, const int32_t *n_bits, int32_t n_channels,
                              const uint8_t *error_transform, int32_t num_f, int32_t num_e, int32_t device,
                              ksim_noise **out)
{
    if (!out) return fail(KSIM_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (n_channels < 0 || num_f < 0 || num_e < 0 || (n_channels > 0 && (!probs || !n_bits)) ||
        (num_f > 0 && num_e > 0 && !error_transform))
        return fail(KSIM_ERR_INVALID_ARGUMENT, "bad noise model arguments");
    if (num_f > 64 * 16) return fail(KSIM_ERR_UNSUPPORTED, "more than 1024 f parameters");
    if (ksim_device_count() <= 0) return fail(KSIM_ERR_NO_DEVICE, "no CUDA device is visible");
    const int W = supported_words(std::max(1, (num_f + 63) / 64));
    int64_t e_total = 0, p_total = 0;
    for (int i = 0; i < n_channels; ++i) {
        if (n_bits[i] < 0 || n_bits[i] > 16)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "channel " + std::to_string(i) + " has " +
                                                       std::to_string(n_bits[i]) + " bits (0..16 supported)");
        e_total += n_bits[i];
        p_total += (int64_t)1 << n_bits[i];
    }
    if (e_total != num_e)
        return fail(KSIM_ERR_INVALID_ARGUMENT, "channels carry " + std::to_string(e_total) +
                                                   " error bits; error_transform has " + std::to_string(num_e));
    for (int64_t i = 0; i < (int64_t)num_f * num_e; ++i)
        if (error_transform[i] > 1) return fail(KSIM_ERR_INVALID_ARGUMENT, "error_transform holds a byte other than 0/1");
    // f pattern of every error bit (column of error_transform), packed
    std::vector<uint64_t> col((size_t)std::max(num_e, 1) * W, 0);
    for (int fi = 0; fi < num_f; ++fi)
        for (int e = 0; e < num_e; ++e)
            if (error_transform[(size_t)fi * num_e + e]) col[(size_t)e * W + (fi >> 6)] |= 1ull << (fi & 63);

    std::vector<NoiseChan> chans;
    std::vector<uint32_t> cdf;
    std::vector<uint64_t> pat;
    const double *pp = probs;
    int e_off = 0;
    for (int i = 0; i < n_channels; ++i) {
        const int k = n_bits[i];
        const int64_t n = (int64_t)1 << k;
        const double *pr = pp;
        pp += n;
        double sum = 0;
        for (int64_t o = 0; o < n; ++o) {
            if (!(pr[o] >= -1e-6 && pr[o] <= 1.0 + 1e-6))
                return fail(KSIM_ERR_INVALID_ARGUMENT, "channel " + std::to_string(i) + ": probability out of [0, 1]");
            sum += pr[o];
        }
        if (std::fabs(sum - 1.0) > 1e-6)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "channel " + std::to_string(i) + ": probabilities do not sum to 1");
        const double p_fire = 1.0 - pr[0];
        if (!(p_fire > 1e-15) || n <= 1) {  // never fires (channels.py:599-600)
            e_off += k;
            continue;
        }
        NoiseChan c;
        c.thr_fire = threshold32(p_fire);
        c.n_out = (uint32_t)(n - 1);
        c.cdf_off = (uint32_t)cdf.size();
        c.pat_off = (uint32_t)pat.size();
        // conditional CDF over the non-identity outcomes, normalised by its
        // last entry (channels.py:602-603)
        std::vector<double> cum((size_t)(n - 1));
        double run = 0;
        for (int64_t o = 1; o < n; ++o) {
            run += std::max(pr[o], 0.0) / p_fire;
            cum[(size_t)(o - 1)] = run;
        }
        for (int64_t o = 0; o + 1 < n - 1; ++o) cdf.push_back(threshold32(cum[(size_t)o] / cum[(size_t)(n - 2)]));
        for (int64_t o = 1; o < n; ++o) {
            for (int w = 0; w < W; ++w) {
                uint64_t x = 0;
                for (int b = 0; b < k; ++b)
                    if ((o >> b) & 1) x ^= col[(size_t)(e_off + b) * W + w];
                pat.push_back(x);
            }
        }
        chans.push_back(c);
        e_off += k;
    }
    if (chans.size() > 0x7FFFFFFF || cdf.size() > 0xFFFFFFFFull || pat.size() > 0xFFFFFFFFull)
        return fail(KSIM_ERR_UNSUPPORTED, "noise model too large");

    std::unique_ptr<ksim_noise> nm(new ksim_noise());
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(KSIM_ERR_NO_DEVICE, "cudaGetDevice failed");
    nm->device = device;
    nm->num_f = num_f;
    nm->num_e = num_e;
    nm->W = W;
    nm->n_ch = (int)chans.size();
    nm->n_outcomes = (int64_t)pat.size() / W;
    const size_t b_ch = sizeof(NoiseChan) * std::max<size_t>(chans.size(), 1);
    const size_t b_cdf = ((sizeof(uint32_t) * std::max<size_t>(cdf.size(), 1)) + 15) & ~size_t(15);
    const size_t b_pat = sizeof(uint64_t) * std::max<size_t>(pat.size(), 1);
    std::vector<uint8_t> host(b_ch + b_cdf + b_pat, 0);
    if (!chans.empty()) std::memcpy(host.data(), chans.data(), sizeof(NoiseChan) * chans.size());
    if (!cdf.empty()) std::memcpy(host.data() + b_ch, cdf.data(), sizeof(uint32_t) * cdf.size());
    if (!pat.empty()) std::memcpy(host.data() + b_ch + b_cdf, pat.data(), sizeof(uint64_t) * pat.size());
    DeviceGuard g(device);
    if (!g.ok) return fail(KSIM_ERR_INVALID_ARGUMENT, "cannot select device " + std::to_string(device));
    cudaError_t e = cudaMalloc(&nm->d_buf, host.size());
    if (e == cudaSuccess) e = cudaMemcpy(nm->d_buf, host.data(), host.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        ksim_noise_destroy(nm.release());
        return cuda_fail(e, "noise model upload");
    }
    nm->bytes = host.size();
    nm->d_ch = (const NoiseChan *)nm->d_buf;
    nm->d_cdf = (const uint32_t *)(nm->d_buf + b_ch);
    nm->d_pat = (const uint64_t *)(nm->d_buf + b_ch + b_cdf);
    *out = nm.release();
    return KSIM_OK;
}

void ksim_noise_destroy(ksim_noise *n)
{
    if (!n) return;
    DeviceGuard g(n->device);
    if (n->d_buf) cudaFree(n->d_buf);
    delete n;
}

int32_t ksim_noise_num_f(const ksim_noise *n) { return n ? n->num_f : -1; }
int32_t ksim_noise_num_channels(const ksim_noise *n) { return n ? n->n_ch : -1; }

ksim_status ksim_noise_sample_device(ksim_noise *n, int64_t B, int64_t shot_offset, uint64_t seed, uint8_t *d_f,
                                     int64_t f_stride, void *stream)
{
    if (!n) return fail(KSIM_ERR_INVALID_ARGUMENT, "noise model is NULL");
    if (B < 0 || shot_offset < 0) return fail(KSIM_ERR_INVALID_ARGUMENT, "B and shot_offset must be >= 0");
    if (B == 0 || n->num_f == 0) return KSIM_OK;
    if (!d_f || f_stride < n->num_f) return fail(KSIM_ERR_INVALID_ARGUMENT, "f is NULL or f_stride < num_f");
    DeviceGuard g(n->device);
    cudaError_t e = launch_noise(n, B, shot_offset, seed, d_f, f_stride, (cudaStream_t)stream);
    if (e != cudaSuccess) return cuda_fail(e, "noise kernel launch");
    return KSIM_OK;
}

ksim_status ksim_noise_sample(ksim_noise *n, int64_t B, int64_t shot_offset, uint64_t seed, uint8_t *f_host)
{
    if (!n) return fail(KSIM_ERR_INVALID_ARGUMENT, "noise model is NULL");
    if (B < 0 || shot_offset < 0) return fail(KSIM_ERR_INVALID_ARGUMENT, "B and shot_offset must be >= 0");
    if (B == 0 || n->num_f == 0) return KSIM_OK;
    if (!f_host) return fail(KSIM_ERR_INVALID_ARGUMENT, "f is NULL");
    DeviceGuard g(n->device);
    uint8_t *d = nullptr;
    cudaError_t e = cudaMalloc(&d, (size_t)(B * n->num_f));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(noise rows)");
    e = launch_noise(n, B, shot_offset, seed, d, n->num_f, nullptr);
    if (e == cudaSuccess) e = cudaMemcpy(f_host, d, (size_t)(B * n->num_f), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "noise sample");
    return KSIM_OK;
}

}  // extern "C"
