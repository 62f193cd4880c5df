// noise.cu — the per-shot noise draw (the f parameters) on the device.
//
// Reference: ChannelSampler (src/python/ksim/compile/channels.py:503-658).
// A noise model is a list of channels; channel i has 2^k_i outcome
// probabilities over its k_i error bits e, and error_transform (num_f x num_e,
// GF(2)) maps error bits to f parameters.  The reference simplifies the
// channels (channels.py:480-500: merging channels over identical error-bit
// signatures by XOR convolution, among other steps), then draws, per channel,
// the shots where it fires by geometric skips along the shot axis and an
// outcome by searchsorted on the conditional CDF, and XORs the outcome's f
// pattern into those rows (channels.py:624-658), with numpy's PCG64 stream.
//
// Here, on the host at model creation:
//   * channels that never fire are dropped, and channels whose error bits
//     have identical f patterns (same count, same patterns in order) are
//     merged by XOR convolution of their outcome probabilities, in order of
//     first appearance (the reference's merge_identical_channels);
//   * the merged channels are ordered by firing probability (descending,
//     ties in merged order) and cut into runs of equal probability p; each
//     run gets the skip table T_k = floor((1 - p)^k 2^32), k = 1, 2, ...
//     (until it reaches 0 or the run's length).
// On the device one thread owns one shot and, per run, jumps from firing
// channel to firing channel: from position j the next firing channel is
// j + 1 + #{k : u < T_k} for a fresh 32-bit draw u, since P(no fire in the
// next k channels) = (1 - p)^k: the count starts from the logarithm's guess
// log2(u 2^-32) / log2(1 - p) and one or two table reads make it exact (the
// walks from the guess end at the count whatever the guess); an outcome is
// then the first whose conditional-CDF threshold exceeds a second draw, and
// its f pattern is XORed in.  Work per shot is proportional to the channels
// that fire, not to the channels of the model.  Rows are written as 16-byte
// pieces of 0/1 bytes where they start on 16-byte boundaries.  The draws
// are one counter-based Philox4x32-10 stream per shot (key = seed, counter =
// (shot, block, 0, tag), four draws a block, consumed in order), so any shot
// range can be drawn alone and the oracle's CPU restatement reproduces every
// bit.  All thresholds are integers, so host and oracle tables agree bit for
// bit.  Per channel, P(fire) and each P(outcome | fire) equal the
// reference's to within 2^-32 per table entry, and channels stay
// independent, so the distribution of f is the reference's up to that
// quantisation.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "../../include/ksim_b200.h"
#include "kernels.h"
#include "runtime.h"
#include "zring.cuh"

namespace ksim {

struct NoiseChan {
    uint32_t n_out;    // outcomes other than the identity
    uint32_t cdf_off;  // n_out - 1 thresholds in the cdf array
    uint32_t pat_off;  // n_out patterns of W words in the pattern array
    uint32_t pad;
};

struct NoiseRun {
    uint32_t first;     // first channel of the run
    uint32_t n;         // channels in the run
    uint32_t skip_off;  // its skip table T_1.. in the skip array
    uint32_t skip_len;
    float inv_log2q;    // 1 / log2(1 - p): the skip's first guess
    uint32_t pad[3];
};

constexpr uint32_t NOISE_TAG = 0x4E4F4953u;

namespace {

// The shot's stream of 32-bit draws: Philox4x32-10 blocks of counter
// (shot lo, shot hi, block, tag), four draws each, in order.
struct DrawStream {
    uint64_t shot, seed;
    uint32_t blk, pos, b0, b1, b2, b3;  // named, not an array: selects keep them in registers
    __device__ __forceinline__ uint32_t next()
    {
        if (pos == 4) {
            uint32_t x[4] = {(uint32_t)shot, (uint32_t)(shot >> 32), blk++, NOISE_TAG};
            philox4x32_10(x, seed);
            b0 = x[0]; b1 = x[1]; b2 = x[2]; b3 = x[3];
            pos = 0;
        }
        const uint32_t r = pos == 0 ? b0 : pos == 1 ? b1 : pos == 2 ? b2 : b3;
        ++pos;
        return r;
    }
};

template <int W>
__global__ void __launch_bounds__(256) k_noise(const NoiseRun *__restrict__ runs, int n_runs,
                                               const NoiseChan *__restrict__ ch, const uint32_t *__restrict__ cdf,
                                               const uint64_t *__restrict__ pat, const uint32_t *__restrict__ skip,
                                               int num_f, int64_t B, int64_t shot_offset, uint64_t seed,
                                               uint8_t *__restrict__ f, int64_t f_stride, bool vec_rows)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= B) return;
    DrawStream st;
    st.shot = (uint64_t)(shot_offset + s);
    st.seed = seed;
    st.blk = 0;
    st.pos = 4;
    uint64_t acc[W];
#pragma unroll
    for (int w = 0; w < W; ++w) acc[w] = 0;
    for (int r = 0; r < n_runs; ++r) {
        const NoiseRun R = runs[r];
        const uint32_t *T = skip + R.skip_off;
        int64_t j = -1;  // last channel of the run visited
        for (;;) {
            // k* = #{k in 1..skip_len : u < T_k}, T decreasing: the first
            // index i of T (T[i] = T_{i+1}) with u >= T[i], or skip_len.
            // First guess from u < (1 - p)^k 2^32 <=> k < log2(u 2^-32) /
            // log2(1 - p); the two walks then make it exact whatever the
            // guess (within one or two of k* here, so a table read or two)
            const uint32_t u = st.next();
            const float g = (__log2f((float)u + 0.5f) - 32.0f) * R.inv_log2q;
            uint32_t k = g <= 0.0f ? 0u : g >= (float)R.skip_len ? R.skip_len : (uint32_t)g;
            while (k < R.skip_len && u < __ldg(T + k)) ++k;
            while (k > 0 && u >= __ldg(T + k - 1)) --k;
            j += (int64_t)k + 1;  // every step advances: at most n steps per run
            if (j >= (int64_t)R.n) break;
            const NoiseChan c = ch[R.first + (uint32_t)j];
            const uint32_t v = st.next();
            uint32_t o = 0;
            while (o + 1 < c.n_out && v >= __ldg(cdf + c.cdf_off + o)) ++o;
            const uint64_t *pp = pat + c.pat_off + (size_t)o * W;
#pragma unroll
            for (int w = 0; w < W; ++w) acc[w] ^= __ldg(pp + w);
        }
    }
    uint8_t *row = f + s * f_stride;
    // 16-byte rows of 0/1 bytes where the rows allow it: a nibble n spreads
    // to four bytes as (n * 0x00204081) & 0x01010101 (its copies shifted by
    // 0, 7, 14, 21 do not overlap, and byte k keeps bit k)
    const int vec16 = vec_rows ? num_f >> 4 : 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {  // static word indices keep acc in registers
        const int q0 = 4 * w, q1 = min(4 * w + 4, vec16);
        for (int q = q0; q < q1; ++q) {
            const uint32_t h = (uint32_t)(acc[w] >> (16 * (q - q0)));
            uint4 v;
            v.x = ((h & 0xFu) * 0x00204081u) & 0x01010101u;
            v.y = (((h >> 4) & 0xFu) * 0x00204081u) & 0x01010101u;
            v.z = (((h >> 8) & 0xFu) * 0x00204081u) & 0x01010101u;
            v.w = (((h >> 12) & 0xFu) * 0x00204081u) & 0x01010101u;
            *(uint4 *)(row + 16 * q) = v;
        }
        const int lim = min(64, num_f - 64 * w);
        for (int b = max(16 * (q1 - q0), 0); b < lim; ++b) row[64 * w + b] = (uint8_t)((acc[w] >> b) & 1u);
    }
}

template <int W>
cudaError_t launch_noise_w(const ksim_noise *n, int64_t B, int64_t shot_offset, uint64_t seed, uint8_t *f,
                           int64_t f_stride, cudaStream_t st);

}  // namespace
}  // namespace ksim

struct ksim_noise {
    int device = 0;
    int num_f = 0, num_e = 0, W = 1;
    int n_ch = 0;           // channels that can fire, after merging
    int n_runs = 0;         // runs of equal firing probability
    int64_t n_outcomes = 0; // patterns stored
    uint8_t *d_buf = nullptr;
    const ksim::NoiseRun *d_runs = nullptr;
    const ksim::NoiseChan *d_ch = nullptr;
    const uint32_t *d_cdf = nullptr;
    const uint64_t *d_pat = nullptr;
    const uint32_t *d_skip = nullptr;
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
    // rows start on 16-byte boundaries: whole 16-byte pieces are stored at once
    const bool vec_rows = ((uintptr_t)f & 15u) == 0 && (f_stride & 15) == 0;
    k_noise<W><<<(unsigned)blocks, 256, 0, st>>>(n->d_runs, n->n_runs, n->d_ch, n->d_cdf, n->d_pat, n->d_skip,
                                                 n->num_f, B, shot_offset, seed, f, f_stride, vec_rows);
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

namespace {

// One channel on the host: k error bits, 2^k outcome probabilities and the
// f pattern (W words) of each error bit.
struct HostChan {
    int k = 0;
    std::vector<double> p;
    std::vector<uint64_t> bits;
};

// P(o) = sum over o1 ^ o2 = o of a(o1) b(o2), in the order i, then j.
std::vector<double> xor_convolve(const std::vector<double> &a, const std::vector<double> &b)
{
    std::vector<double> out(a.size(), 0.0);
    for (size_t i = 0; i < a.size(); ++i)
        for (size_t j = 0; j < b.size(); ++j) out[i ^ j] += a[i] * b[j];
    return out;
}

}  // namespace

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
    int64_t e_total = 0;
    for (int i = 0; i < n_channels; ++i) {
        if (n_bits[i] < 0 || n_bits[i] > 16)
            return fail(KSIM_ERR_INVALID_ARGUMENT, "channel " + std::to_string(i) + " has " +
                                                       std::to_string(n_bits[i]) + " bits (0..16 supported)");
        e_total += n_bits[i];
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

    // validate, drop never-firing channels (channels.py:599-600), merge
    // channels over identical error-bit patterns
    std::vector<HostChan> merged;
    std::map<std::vector<uint64_t>, size_t> by_sig;
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
        const int eo = e_off;
        e_off += k;
        if (!(1.0 - pr[0] > 1e-15) || n <= 1) continue;
        std::vector<uint64_t> sig(1, (uint64_t)k);
        for (int b = 0; b < k; ++b)
            for (int w = 0; w < W; ++w) sig.push_back(col[(size_t)(eo + b) * W + w]);
        std::vector<double> pv(pr, pr + n);
        auto it = by_sig.find(sig);
        if (it != by_sig.end()) {
            merged[it->second].p = xor_convolve(merged[it->second].p, pv);
        } else {
            HostChan c;
            c.k = k;
            c.p = pv;
            c.bits.assign(sig.begin() + 1, sig.end());
            by_sig.emplace(sig, merged.size());
            merged.push_back(std::move(c));
        }
    }
    // channels by firing probability (descending, ties in merged order), cut
    // into runs of equal probability
    std::vector<size_t> order;
    for (size_t i = 0; i < merged.size(); ++i)
        if (1.0 - merged[i].p[0] > 1e-15) order.push_back(i);
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        const double pa = 1.0 - merged[a].p[0], pb = 1.0 - merged[b].p[0];
        return pa != pb ? pa > pb : a < b;
    });
    std::vector<NoiseRun> runs;
    std::vector<NoiseChan> chans;
    std::vector<uint32_t> cdf, skip;
    std::vector<uint64_t> pat;
    for (size_t r0 = 0; r0 < order.size();) {
        const double p_fire = 1.0 - merged[order[r0]].p[0];
        size_t r1 = r0;
        while (r1 < order.size() && 1.0 - merged[order[r1]].p[0] == p_fire) ++r1;
        NoiseRun run;
        run.first = (uint32_t)chans.size();
        run.n = (uint32_t)(r1 - r0);
        run.skip_off = (uint32_t)skip.size();
        const double q = 1.0 - p_fire;
        double t = 1.0;
        for (uint32_t k = 1; k <= run.n; ++k) {
            t *= q;
            const uint32_t thr = threshold32(t);
            if (thr == 0) break;
            skip.push_back(thr);
        }
        run.skip_len = (uint32_t)skip.size() - run.skip_off;
        run.inv_log2q = q > 0.0 ? (float)(1.0 / std::log2(q)) : 0.0f;
        run.pad[0] = run.pad[1] = run.pad[2] = 0;
        runs.push_back(run);
        for (size_t x = r0; x < r1; ++x) {
            const HostChan &hc = merged[order[x]];
            const int64_t n = (int64_t)1 << hc.k;
            NoiseChan c;
            c.n_out = (uint32_t)(n - 1);
            c.cdf_off = (uint32_t)cdf.size();
            c.pat_off = (uint32_t)pat.size();
            c.pad = 0;
            // conditional CDF over the non-identity outcomes, normalised by its
            // last entry (channels.py:602-603)
            std::vector<double> cum((size_t)(n - 1));
            double run_sum = 0;
            for (int64_t o = 1; o < n; ++o) {
                run_sum += std::max(hc.p[(size_t)o], 0.0) / p_fire;
                cum[(size_t)(o - 1)] = run_sum;
            }
            for (int64_t o = 0; o + 1 < n - 1; ++o) cdf.push_back(threshold32(cum[(size_t)o] / cum[(size_t)(n - 2)]));
            for (int64_t o = 1; o < n; ++o)
                for (int w = 0; w < W; ++w) {
                    uint64_t xw = 0;
                    for (int b = 0; b < hc.k; ++b)
                        if ((o >> b) & 1) xw ^= hc.bits[(size_t)b * W + w];
                    pat.push_back(xw);
                }
            chans.push_back(c);
        }
        r0 = r1;
    }
    if (chans.size() > 0x7FFFFFFF || cdf.size() > 0xFFFFFFFFull || pat.size() > 0xFFFFFFFFull ||
        skip.size() > 0xFFFFFFFFull)
        return fail(KSIM_ERR_UNSUPPORTED, "noise model too large");

    std::unique_ptr<ksim_noise> nm(new ksim_noise());
    if (device < 0 && cudaGetDevice(&device) != cudaSuccess) return fail(KSIM_ERR_NO_DEVICE, "cudaGetDevice failed");
    nm->device = device;
    nm->num_f = num_f;
    nm->num_e = num_e;
    nm->W = W;
    nm->n_ch = (int)chans.size();
    nm->n_runs = (int)runs.size();
    nm->n_outcomes = (int64_t)pat.size() / W;
    auto pad16 = [](size_t b) { return (std::max<size_t>(b, 16) + 15) & ~size_t(15); };
    const size_t b_run = pad16(sizeof(NoiseRun) * runs.size());
    const size_t b_ch = pad16(sizeof(NoiseChan) * chans.size());
    const size_t b_cdf = pad16(sizeof(uint32_t) * cdf.size());
    const size_t b_skip = pad16(sizeof(uint32_t) * skip.size());
    const size_t b_pat = pad16(sizeof(uint64_t) * pat.size());
    std::vector<uint8_t> host(b_run + b_ch + b_cdf + b_skip + b_pat, 0);
    size_t off = 0;
    auto put = [&](const void *src, size_t bytes, size_t span) {
        if (bytes) std::memcpy(host.data() + off, src, bytes);
        const size_t at = off;
        off += span;
        return at;
    };
    const size_t o_run = put(runs.data(), sizeof(NoiseRun) * runs.size(), b_run);
    const size_t o_ch = put(chans.data(), sizeof(NoiseChan) * chans.size(), b_ch);
    const size_t o_cdf = put(cdf.data(), sizeof(uint32_t) * cdf.size(), b_cdf);
    const size_t o_skip = put(skip.data(), sizeof(uint32_t) * skip.size(), b_skip);
    const size_t o_pat = put(pat.data(), sizeof(uint64_t) * pat.size(), b_pat);
    DeviceGuard g(device);
    if (!g.ok) return fail(KSIM_ERR_INVALID_ARGUMENT, "cannot select device " + std::to_string(device));
    cudaError_t e = cudaMalloc(&nm->d_buf, host.size());
    if (e == cudaSuccess) e = cudaMemcpy(nm->d_buf, host.data(), host.size(), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
        ksim_noise_destroy(nm.release());
        return cuda_fail(e, "noise model upload");
    }
    nm->bytes = host.size();
    nm->d_runs = (const NoiseRun *)(nm->d_buf + o_run);
    nm->d_ch = (const NoiseChan *)(nm->d_buf + o_ch);
    nm->d_cdf = (const uint32_t *)(nm->d_buf + o_cdf);
    nm->d_skip = (const uint32_t *)(nm->d_buf + o_skip);
    nm->d_pat = (const uint64_t *)(nm->d_buf + o_pat);
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
