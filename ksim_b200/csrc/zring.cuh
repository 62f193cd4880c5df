// zring.cuh — exact Z[w] term evaluation over the packed program image.
//
// w = e^{i pi/4}.  Elements are (a, b, c, d) in the basis (1, w, i, conj w),
// the representation of the reference (zx_eval.hpp:25-47), held as uint64 so
// every add and multiply wraps exactly like the reference's int64.
//
// Multiplying by w^j is a signed rotation of the coefficients:
//   w^0: ( a,  b,  c,  d)      w^1: ( d,  a,  b, -c)
//   w^2: (-c,  d,  a, -b)      w^3: (-b, -c,  d, -a)      w^(j+4) = -w^j
// HalfPi and the phase index are rotations and PiProducts a sign; the fast
// path sums them into one rotation, applied with the floatfactor as one
// product with a tabulated ff * w^k.
//
// NodePhases need no per-column arithmetic at all.  A column's factor is
// 1 + s w^j (s = +-1 from the parity), and 1 - x = (1 + x) u with a unit u:
//   j = 2: u = w^6,   j = 1: u = w^6 / lambda,   j = 3: u = w^6 lambda,
// lambda = 1 + sqrt2 = 1 + w + conj w.  With m_j the number of columns of
// class j whose sign is -1, the block's product is
//   2^n0 (1 + i)^n2 (1 + w)^n1 (1 + w^3)^n3 * w^(6 (m1 + m2 + m3)) * lambda^(m3 - m1)
// or 0 if a class-0 column (factor 1 + s = 2 or 0) has s = -1.  Every factor
// has (1 - w)-adic valuation <= 4 and the reference halves at most once per
// factor, so it divides the product by 2^H, H = floor(sum nu / 4), whatever
// the signs.  The host folds the all-plus product / 2^H into one constant C
// per term; a shot counts its m_j, reads lambda^(m3 - m1) from a table and
// makes one product, and the rotation joins the deferred one at the end.
//
// Renormalisation ("halve when all four are even and not all zero",
// zx_eval.hpp:35-41) is decided without looking at the coefficients: for
// nonzero z, all four are even  <=>  nu(z) >= 4, where nu is the
// (1 - w)-adic valuation (2 = unit * (1 - w)^4), and nu is additive under
// products.  PhasePairs factors 1 + w^a + w^b - w^(a+b) depend on the shot's
// parities; the host tabulates each factor's nu per sign pair, so a shot
// tracks nu(z) and runs two columns at a time: their two halving decisions,
// one product with the tabulated pair product, one shift.  This reproduces the reference's (a, b, c, d, pw)
// exactly whenever no coefficient leaves the int64 range (all the fast path's
// arithmetic wraps like the reference's, and only a halving or the end needs
// the true value); the host proves that per term from an embedding-norm bound
// (|coefficient| <= max_k |sigma_k(z)|), and terms it cannot prove safe are
// evaluated by eval_term_exact, the reference's step-by-step arithmetic
// including the explicit evenness test and int64 wrap.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define KS_HD __host__ __device__ __forceinline__
#define KS_CE __host__ __device__ constexpr
#else
#define KS_HD inline
#define KS_CE constexpr
#endif

namespace ksim {

// ---- image record layout (shared with image.cpp) --------------------------
// TF_SLOW: evaluate step by step (no proof the fast path stays in range);
// TF_NARROW: every value the fast path must know exactly (at each halving
// and at the end) is proven below 2^31, so it runs on 32-bit coefficients.
// TF_HYBRID: the NodePhases block is proven below 2^31 and runs on 32-bit
// words, the rest on 64-bit words.
// TF_EXP: every scale 2^(pw + power2) the fast term can reach (pw from the
// NodePhases halvings or a kill's dead_pw, plus at most two halvings per
// PhasePairs pair and one renormalisation) is a normal double, so the scale
// is built from its exponent bits without pow2i's range tests.
enum : uint32_t { TF_SLOW = 1u, TF_APX = 2u, TF_NARROW = 4u, TF_HYBRID = 8u, TF_EXP = 16u };
constexpr int TERM_HDR_BYTES = 96;
constexpr int TERM_APX_BYTES = 16;
// NodePhases / HalfPi column: W mask words + 1 constant word, padded to 16 B
KS_HD constexpr int rec1_words(int W) { return (W + 2) & ~1; }
// PiProducts / PhasePairs column: 2W mask words + 1 constant word, padded
KS_HD constexpr int rec2_words(int W) { return (2 * W + 2) & ~1; }
// lambda^e for |e| <= LAM_MAX; a fast term has max(n1, n3) <= LAM_MAX
constexpr int LAM_MAX = 127;
constexpr uint32_t NU_ZERO = 15u;  // PhasePairs factor is exactly zero

// Coefficients as unsigned words, so every add and multiply wraps like the
// reference's int64 (T = uint64_t) or, on the narrow path, like int32.
template <typename T>
struct Zr { T a, b, c, d; };
using Zu = Zr<uint64_t>;
using Zn = Zr<uint32_t>;

template <typename T>
KS_HD T sneg(T x, T m) { return (x ^ m) - m; }  // m = 0: x, m = ~0: -x

// acc + (m ? -x : x).  64-bit: xor/subtract on the integer ALU; 32-bit: one
// multiply-add by +-1, which runs on the FMA pipe and leaves the ALU free.
KS_HD uint64_t cadd(uint64_t acc, uint64_t x, uint64_t m) { return acc + sneg(x, m); }
KS_HD uint32_t cadd(uint32_t acc, uint32_t x, uint32_t m) { return acc + (m | 1u) * x; }

// Arithmetic shift right of the signed value held in x.
KS_HD uint64_t sshr(uint64_t x, uint32_t n) { return (uint64_t)((int64_t)x >> n); }
KS_HD uint32_t sshr(uint32_t x, uint32_t n) { return (uint32_t)((int32_t)x >> n); }

KS_HD uint32_t popc64(uint64_t x)
{
#if defined(__CUDA_ARCH__)
    return (uint32_t)__popc((uint32_t)x ^ (uint32_t)(x >> 32));
#else
    return (uint32_t)__builtin_popcountll(x);
#endif
}

template <int W>
KS_HD uint32_t parity(const uint64_t *m, const uint64_t (&v)[W])
{
    uint64_t x = m[0] & v[0];
#pragma unroll
    for (int w = 1; w < W; ++w) x ^= m[w] & v[w];
    return popc64(x) & 1u;
}

// IEEE double ops that the compiler may not contract into FMAs.
KS_HD double dadd(double x, double y)
{
#if defined(__CUDA_ARCH__)
    return __dadd_rn(x, y);
#else
    return x + y;
#endif
}
KS_HD double dsub(double x, double y)
{
#if defined(__CUDA_ARCH__)
    return __dsub_rn(x, y);
#else
    return x - y;
#endif
}
KS_HD double dmul(double x, double y)
{
#if defined(__CUDA_ARCH__)
    return __dmul_rn(x, y);
#else
    return x * y;
#endif
}
KS_HD double bits_to_double(uint64_t u)
{
#if defined(__CUDA_ARCH__)
    return __longlong_as_double((long long)u);
#else
    double d;
    __builtin_memcpy(&d, &u, 8);
    return d;
#endif
}

// 2^n exactly (the value exp2 returns for an integer argument, including the
// subnormal range and the 0 / +inf ends).
KS_HD double pow2i(int64_t n)
{
    if (n > 1023) return bits_to_double(0x7FF0000000000000ull);
    if (n >= -1022) return bits_to_double((uint64_t)(n + 1023) << 52);
    if (n >= -1074) return bits_to_double(1ull << (n + 1074));
    return 0.0;
}

// 2^n for n in [-1022, 1023] (a normal double: exponent field n + 1023).
KS_HD double pow2_normal(int32_t n)
{
#if defined(__CUDA_ARCH__)
    return __hiloint2double((n + 1023) << 20, 0);
#else
    return bits_to_double((uint64_t)(n + 1023) << 52);
#endif
}

// z * w^k for a per-shot k in 0..7 (selects, no branches).
template <typename T>
KS_HD Zr<T> rot_var(Zr<T> z, uint32_t k)
{
    const bool k1 = k & 1u, k2 = k & 2u;
    Zr<T> r;
    r.a = k1 ? z.d : z.a;
    r.b = k1 ? z.a : z.b;
    r.c = k1 ? z.b : z.c;
    r.d = k1 ? (T)(0 - z.c) : z.d;
    Zr<T> q;
    q.a = k2 ? (T)(0 - r.c) : r.a;
    q.b = k2 ? r.d : r.b;
    q.c = k2 ? r.a : r.c;
    q.d = k2 ? (T)(0 - r.b) : r.d;
    const T m = (T)0 - (T)((k >> 2) & 1u);
    q.a = sneg(q.a, m); q.b = sneg(q.b, m); q.c = sneg(q.c, m); q.d = sneg(q.d, m);
    return q;
}

// The sign (-1)^p in the form the signed adds use, for both orientations:
// 32-bit words multiply by +-1 (one multiply-add each), 64-bit words
// xor / subtract with a 0 / ~0 mask.
template <typename T>
struct Sign { T pos, neg; };
KS_HD Sign<uint32_t> sign_of(uint32_t p, uint32_t) { return {1u - 2u * p, 2u * p - 1u}; }
KS_HD Sign<uint64_t> sign_of(uint32_t p, uint64_t)
{
    const uint64_t m = 0 - (uint64_t)p;
    return {m, ~m};
}
KS_HD uint32_t sadd(uint32_t acc, uint32_t x, uint32_t s) { return acc + s * x; }
KS_HD uint64_t sadd(uint64_t acc, uint64_t x, uint64_t m) { return acc + sneg(x, m); }

// acc += (-1)^p * R_j(t), j in 0..3 the same for all shots.
template <typename T>
KS_HD void add_rot(Zr<T> &acc, const Zr<T> &t, uint32_t j, uint32_t p)
{
    const Sign<T> g = sign_of(p, T());
    const T m = g.pos, n = g.neg;
    switch (j & 3u) {
    case 0: acc.a = sadd(acc.a, t.a, m); acc.b = sadd(acc.b, t.b, m); acc.c = sadd(acc.c, t.c, m); acc.d = sadd(acc.d, t.d, m); break;
    case 1: acc.a = sadd(acc.a, t.d, m); acc.b = sadd(acc.b, t.a, m); acc.c = sadd(acc.c, t.b, m); acc.d = sadd(acc.d, t.c, n); break;
    case 2: acc.a = sadd(acc.a, t.c, n); acc.b = sadd(acc.b, t.d, m); acc.c = sadd(acc.c, t.a, m); acc.d = sadd(acc.d, t.b, n); break;
    default: acc.a = sadd(acc.a, t.b, n); acc.b = sadd(acc.b, t.c, n); acc.c = sadd(acc.c, t.d, m); acc.d = sadd(acc.d, t.a, n); break;
    }
}

// Full product (zx_eval.hpp:27-33 formula, basis (1, w, i, conj w)).
template <typename T>
KS_HD Zr<T> zmul(const Zr<T> &x, const Zr<T> &y)
{
    Zr<T> r;
    r.a = x.a * y.a + x.b * y.d - x.c * y.c + x.d * y.b;
    r.b = x.a * y.b + x.b * y.a + x.c * y.d + x.d * y.c;
    r.c = x.a * y.c + x.b * y.b + x.c * y.a - x.d * y.d;
    r.d = x.a * y.d - x.b * y.c - x.c * y.b + x.d * y.a;
    return r;
}

template <typename T>
KS_HD void shr_all(Zr<T> &z, uint32_t n)
{
    z.a = sshr(z.a, n); z.b = sshr(z.b, n); z.c = sshr(z.c, n); z.d = sshr(z.d, n);
}

KS_HD void shr1_all(Zu &z) { shr_all(z, 1u); }

// One renormalisation step with the explicit test (zx_eval.hpp:35-41).
template <typename T, typename P>
KS_HD void zreduce(Zr<T> &z, P &pw)
{
    const T o = z.a | z.b | z.c | z.d;
    if (o != 0 && (o & 1u) == 0) {
        shr_all(z, 1u);
        pw += 1;
    }
}

// Sign-extend a narrow element to the 64-bit representation.
KS_HD Zu widen(const Zn &z)
{
    Zu r;
    r.a = (uint64_t)(int64_t)(int32_t)z.a;
    r.b = (uint64_t)(int64_t)(int32_t)z.b;
    r.c = (uint64_t)(int64_t)(int32_t)z.c;
    r.d = (uint64_t)(int64_t)(int32_t)z.d;
    return r;
}

KS_HD bool over62(const Zu &z)
{
    const uint64_t k = 1ull << 62, lim = 1ull << 63;
    return (z.a + k) > lim || (z.b + k) > lim || (z.c + k) > lim || (z.d + k) > lim;
}

struct TermHdr {
    uint32_t n_np, n_hp, n_pp, n_ph;
    uint32_t pf_idx, flags;
    int32_t power2;
    Zu ff;
    uint32_t n_cls[4];  // NodePhases columns per rotation class, in run order j = 0, 2, 1, 3
    int32_t np_pw;      // halvings of the NodePhases block (a term that survives it)
    uint32_t rec_bytes; // the whole term record
    uint32_t nb;          // 32-row parity blocks (fast terms)
    // fast terms: byte offsets of the record's parts (written by the packer
    // from the layout_* functions below, so a shot reads them instead of
    // deriving them from the counts), the first PhasePairs row and the
    // valuation of the NodePhases result mod 4
    uint32_t off_meta, off_tab, off_step, off_npl, off_blk, ph_row0, nu0;
};
// The NodePhases constant C (4 x 64-bit words, mod 2^64) follows the header
// fields at this offset.
constexpr int TERM_NPC_OFF = 48;
// A fast term has at most this many 32-row parity blocks.
constexpr int NB_MAX = 8;

// The parameter vector's top bit (bit 63 of word W-1) is the constant 1; a
// column mask that includes it has its constant folded into its parity.
template <int W>
KS_HD void set_one_bit(uint64_t (&v)[W])
{
    v[W - 1] |= 1ull << 63;
}

KS_HD TermHdr load_hdr(const uint8_t *p)
{
    uint32_t u[12], nb, lay[3];
#if defined(__CUDA_ARCH__)
    const uint4 *q = (const uint4 *)p;  // records are 16-byte aligned
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const uint4 x = q[i];
        u[4 * i] = x.x; u[4 * i + 1] = x.y; u[4 * i + 2] = x.z; u[4 * i + 3] = x.w;
    }
    const uint4 t = q[5];
    nb = t.x; lay[0] = t.y; lay[1] = t.z; lay[2] = t.w;
#else
    const uint32_t *q = (const uint32_t *)p;
    for (int i = 0; i < 12; ++i) u[i] = q[i];
    nb = q[20];
    lay[0] = q[21]; lay[1] = q[22]; lay[2] = q[23];
#endif
    TermHdr h;
    h.n_np = u[0] & 0xFFFFu; h.n_hp = u[0] >> 16;
    h.n_pp = u[1] & 0xFFFFu; h.n_ph = u[1] >> 16;
    h.pf_idx = u[2] & 7u; h.flags = (u[2] >> 16) & 0xFFu;
    h.power2 = (int32_t)u[3];
    h.ff.a = (uint64_t)(int64_t)(int32_t)u[4]; h.ff.b = (uint64_t)(int64_t)(int32_t)u[5];
    h.ff.c = (uint64_t)(int64_t)(int32_t)u[6]; h.ff.d = (uint64_t)(int64_t)(int32_t)u[7];
    h.n_cls[0] = u[8] & 0xFFFFu; h.n_cls[1] = u[8] >> 16;
    h.n_cls[2] = u[9] & 0xFFFFu; h.n_cls[3] = u[9] >> 16;
    h.np_pw = (int32_t)u[10];
    h.rec_bytes = u[11];
    h.nb = nb;
    h.off_tab = (lay[0] & 0xFFFFu) << 4;
    h.off_step = (lay[0] >> 16) << 4;
    h.off_npl = (lay[1] & 0xFFFFu) << 4;
    h.off_blk = (lay[1] >> 16) << 4;
    h.ph_row0 = lay[2] & 0xFFFFu;
    h.nu0 = (lay[2] >> 16) & 3u;
    h.off_meta = (lay[2] >> 18) << 4;
    return h;
}

// ---- powers of lambda = 1 + sqrt2 = (1, 1, 0, 1), a unit of Z[w] ----------
// lambda^-1 = sqrt2 - 1 = (-1, 1, 0, 1).  Entry e + LAM_MAX holds lambda^e
// mod 2^64 (the low halves are lambda^e mod 2^32).
struct LamTable { uint64_t z[2 * LAM_MAX + 1][4]; };
struct alignas(16) LamTable32 { uint32_t z[2 * LAM_MAX + 1][4]; };

KS_CE void lam_step(uint64_t (&z)[4], const uint64_t (&y)[4])
{
    const uint64_t a = z[0] * y[0] + z[1] * y[3] - z[2] * y[2] + z[3] * y[1];
    const uint64_t b = z[0] * y[1] + z[1] * y[0] + z[2] * y[3] + z[3] * y[2];
    const uint64_t c = z[0] * y[2] + z[1] * y[1] + z[2] * y[0] - z[3] * y[3];
    const uint64_t d = z[0] * y[3] - z[1] * y[2] - z[2] * y[1] + z[3] * y[0];
    z[0] = a; z[1] = b; z[2] = c; z[3] = d;
}

KS_CE LamTable make_lam_table()
{
    LamTable t{};
    const uint64_t up[4] = {1, 1, 0, 1}, dn[4] = {~0ull, 1, 0, 1};
    uint64_t p[4] = {1, 0, 0, 0}, n[4] = {1, 0, 0, 0};
    for (int k = 0; k < 4; ++k) t.z[LAM_MAX][k] = p[k];
    for (int e = 1; e <= LAM_MAX; ++e) {
        lam_step(p, up);
        lam_step(n, dn);
        for (int k = 0; k < 4; ++k) {
            t.z[LAM_MAX + e][k] = p[k];
            t.z[LAM_MAX - e][k] = n[k];
        }
    }
    return t;
}

KS_CE LamTable32 make_lam_table32()
{
    const LamTable t = make_lam_table();
    LamTable32 r{};
    for (int e = 0; e < 2 * LAM_MAX + 1; ++e)
        for (int k = 0; k < 4; ++k) r.z[e][k] = (uint32_t)t.z[e][k];
    return r;
}

#if defined(__CUDACC__)
static __device__ const LamTable kLamDev = make_lam_table();
static __device__ const LamTable32 kLam32Dev = make_lam_table32();
#endif
static constexpr LamTable kLamHost = make_lam_table();

// lambda^e, |e| <= LAM_MAX, in the word type of the path.
KS_HD Zr<uint64_t> lam_pow(int e, uint64_t)
{
#if defined(__CUDA_ARCH__)
    const ulonglong2 *q = (const ulonglong2 *)&kLamDev.z[e + LAM_MAX][0];
    const ulonglong2 x = __ldg(q), y = __ldg(q + 1);
    return {x.x, x.y, y.x, y.y};
#else
    const uint64_t *z = kLamHost.z[e + LAM_MAX];
    return {z[0], z[1], z[2], z[3]};
#endif
}
KS_HD Zr<uint32_t> lam_pow(int e, uint32_t)
{
#if defined(__CUDA_ARCH__)
    const uint4 x = __ldg((const uint4 *)&kLam32Dev.z[e + LAM_MAX][0]);
    return {x.x, x.y, x.z, x.w};
#else
    const uint64_t *z = kLamHost.z[e + LAM_MAX];
    return {(uint32_t)z[0], (uint32_t)z[1], (uint32_t)z[2], (uint32_t)z[3]};
#endif
}

KS_HD int term_bytes(const TermHdr &h, int) { return (int)h.rec_bytes; }

// Load R 64-bit words of a 16-byte aligned record with 16-byte vector loads.
template <int R>
KS_HD void load_rec(const uint64_t *rec, uint64_t (&r)[R])
{
#if defined(__CUDA_ARCH__)
    const ulonglong2 *q = (const ulonglong2 *)rec;
#pragma unroll
    for (int i = 0; i < R / 2; ++i) {
        ulonglong2 x = q[i];
        r[2 * i] = x.x;
        r[2 * i + 1] = x.y;
    }
#else
    for (int i = 0; i < R; ++i) r[i] = rec[i];
#endif
}

struct TermOut {
    Zu z;
    int64_t pw;
    int32_t power2;
    uint32_t risk;  // KSIM_FLAG_INT64_RISK raised by the exact path
};

// ---- fast terms: parity rows -------------------------------------------------
// A fast term's columns are parity rows over the parameter vector, each
// stored as the list of its set bits.  Row order (term-relative position):
//   NodePhases class 0 in column order | the other NodePhases rows, the
//   HalfPi rows and the PiProducts (psi, phi) pairs (each pair at an even
//   position, a zero row where needed), the rows with the most set bits
//   first | (zero rows to a multiple of 4: the header's ph_row0) |
//   PhasePairs (alpha, beta) pairs in column order
// After the header (and approximation) the term's constants: the floatfactor
// times w^(k + phase index) for k = 0..7 (8 x 4 i32, so the final rotation
// and the floatfactor are one table read and one product), u16 dead_pw per
// class-0 row, padded to 16 bytes; the PhasePairs pair tables and valuation
// words (see layout_pair_tab_off), each part padded to 16 bytes; then nb
// blocks of 32 rows, each a 32-byte head
//   u32 n_pairs, u32 masks P1, P2, P4, E3, E1, PP, K0 (bit i = row 32b + i)
// and n_pairs x 32 u32 words of two u16 byte offsets (8 x bit index; word
// [i][r] holds the set bits 2i and 2i + 1 of row r of the block, 8 x 64W,
// the zero word, where it has fewer).
// Every sum the term needs is linear in the row bits w of a block:
//   rotation  += popc(w & P1) + 2 popc(w & P2) + 4 popc(w & (P4 | PP & w >> 1))
//     (P2 and P4 hold the NodePhases classes 1-3, whose sign count enters as
//     w^6 per -1; P1 / P2 / P4 the HalfPi rows by coefficient bit; PP the psi
//     rows, whose pair product psi * phi is a sign, w^4)
//   lambda exponent += popc((w & E3) | (~w & E1)), minus n1 at the end
//     (= m3 - m1 with E3 / E1 the class-3 / class-1 rows)
//   kill: the first row of w & K0 (class 0) with its dead_pw.
constexpr int BLOCK_HEAD_BYTES = 32;
constexpr int TERM_FFK_BYTES = 128;
// PhasePairs columns 2p and 2p + 1 run as one pair (an odd last column
// pairs with the factor 1, its sign bits being rows past the end, which are
// zero): a table of the 16 products (4 x i8 each, combo c = pa | pb << 1 |
// pa' << 2 | pb' << 3), then per pair a 256-byte step table: entry 16 c + nu,
// for the state nu of z before the pair — its valuation (0..14; a factor can
// have nu up to 6, so nu can grow, and the packer sends terms that can leave
// that range to the exact path) or NU_DEAD once z is zero (a class-0 kill or
// a zero factor) — holds the pair's halvings (bits 0-1) and the state after
// it (bits 2-5).  NU_DEAD absorbs and takes no halvings.
constexpr uint32_t NU_DEAD = 15;
// NodePhases products C lambda^e, e = -n1 .. n3, follow for terms with
// class-1 or class-3 columns (n_cls[2], n_cls[3] in run order): 4 x u32 per
// entry on the 32-bit NodePhases paths, 4 x u64 otherwise; entry i is
// e = i - n1.
//
// The layout from the counts (the packer places the parts with these and
// stores the offsets in the header) ...
KS_HD int layout_meta_off(const TermHdr &h) { return TERM_HDR_BYTES + ((h.flags & TF_APX) ? TERM_APX_BYTES : 0); }
KS_HD uint32_t layout_ph_pairs(const TermHdr &h) { return (h.n_ph + 1) >> 1; }
KS_HD int layout_pair_tab_off(const TermHdr &h)
{
    return layout_meta_off(h) + TERM_FFK_BYTES + ((2 * (int)h.n_cls[0] + 15) & ~15);
}
KS_HD int layout_pair_step_off(const TermHdr &h) { return layout_pair_tab_off(h) + 64 * (int)layout_ph_pairs(h); }
KS_HD bool layout_np_odd(const TermHdr &h) { return (h.n_cls[2] | h.n_cls[3]) != 0; }
KS_HD int layout_npl_off(const TermHdr &h) { return layout_pair_step_off(h) + 256 * (int)layout_ph_pairs(h); }
KS_HD int layout_npl_bytes(const TermHdr &h)
{
    if (!layout_np_odd(h)) return 0;
    const int entry = (h.flags & (TF_NARROW | TF_HYBRID)) ? 16 : 32;
    return ((int)(h.n_cls[2] + h.n_cls[3] + 1) * entry + 15) & ~15;
}
KS_HD int layout_blocks_off(const TermHdr &h) { return layout_npl_off(h) + layout_npl_bytes(h); }
// Valuation mod 4 of the NodePhases result: (2 n2 + n1 + n3) mod 4.
KS_HD uint32_t layout_nu0(const TermHdr &h) { return (2u * h.n_cls[1] + h.n_cls[2] + h.n_cls[3]) & 3u; }

// ... and as a record's reader takes it from the header.
KS_HD int term_meta_off(const TermHdr &h) { return (int)h.off_meta; }
KS_HD int term_pair_tab_off(const TermHdr &h) { return (int)h.off_tab; }
KS_HD int term_pair_step_off(const TermHdr &h) { return (int)h.off_step; }
KS_HD uint32_t term_ph_pairs(const TermHdr &h) { return (h.off_npl - h.off_step) >> 8; }  // 256 step bytes a pair
KS_HD int term_npl_off(const TermHdr &h) { return (int)h.off_npl; }
KS_HD bool term_np_odd(const TermHdr &h) { return h.off_blk != h.off_npl; }
KS_HD int term_blocks_off(const TermHdr &h) { return (int)h.off_blk; }
KS_HD int term_ph_row0(const TermHdr &h) { return (int)h.ph_row0; }

// Entry i of a term's lambda table in the word type of its NodePhases block.
KS_HD Zr<uint32_t> load_npl(const uint8_t *tab, uint32_t i, uint32_t)
{
#if defined(__CUDA_ARCH__)
    const uint4 x = *(const uint4 *)(tab + 16 * (size_t)i);
    return {x.x, x.y, x.z, x.w};
#else
    const uint32_t *q = (const uint32_t *)(tab + 16 * (size_t)i);
    return {q[0], q[1], q[2], q[3]};
#endif
}
KS_HD Zr<uint64_t> load_npl(const uint8_t *tab, uint32_t i, uint64_t)
{
#if defined(__CUDA_ARCH__)
    const ulonglong2 *q = (const ulonglong2 *)(tab + 32 * (size_t)i);
    const ulonglong2 x = q[0], y = q[1];
    return {x.x, x.y, y.x, y.y};
#else
    const uint64_t *q = (const uint64_t *)(tab + 32 * (size_t)i);
    return {q[0], q[1], q[2], q[3]};
#endif
}
KS_HD void load_i32x4(const uint8_t *p, int32_t (&r)[4])
{
#if defined(__CUDA_ARCH__)
    const int4 x = *(const int4 *)p;
    r[0] = x.x; r[1] = x.y; r[2] = x.z; r[3] = x.w;
#else
    const int32_t *q = (const int32_t *)p;
    r[0] = q[0]; r[1] = q[1]; r[2] = q[2]; r[3] = q[3];
#endif
}

// Byte B of x as a signed 32-bit value.  On the device one byte permute:
// a selector nibble with its top bit set copies the sign bit of the byte it
// names into every bit of the result byte (PTX prmt, default mode).
template <int B>
KS_HD int32_t sext_byte(uint32_t x)
{
#if defined(__CUDA_ARCH__)
    constexpr uint32_t sel = (uint32_t)B | ((uint32_t)(8 | B) * 0x1110u);
    uint32_t r;
    asm("prmt.b32 %0, %1, 0, %2;" : "=r"(r) : "r"(x), "n"(sel));
    return (int32_t)r;
#else
    return (int32_t)(x << (24 - 8 * B)) >> 24;
#endif
}

KS_HD uint32_t popc32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
    return (uint32_t)__popc(x);
#else
    return (uint32_t)__builtin_popcount(x);
#endif
}
KS_HD int ffs32(uint32_t x)
{
#if defined(__CUDA_ARCH__)
    return __ffs((int)x) - 1;
#else
    return __builtin_ctz(x);
#endif
}

// Row-parity words of one shot: word b holds rows 32b..32b+31 (bit i = row
// 32b + i), `stride` words apart (shared memory, one column per thread) or
// contiguous (a local array).
struct RowBits {
    const uint32_t *w;
    int stride;
    KS_HD uint32_t word(int b) const { return w[b * stride]; }
};

// Parity-row words of one shot from the block records, bit by bit (the
// per-shot form; the sampling kernels build them for a warp at once).
template <int W>
KS_HD void term_words_shot(const uint8_t *p, const TermHdr &h, const uint64_t (&v)[W], uint32_t (&out)[NB_MAX + 1])
{
    const uint8_t *blk = p + term_blocks_off(h);
    for (int b = 0; b <= NB_MAX; ++b) out[b] = 0;
    for (uint32_t b = 0; b < h.nb; ++b) {
        const uint32_t n_pairs = *(const uint32_t *)blk;
        const uint32_t *ix = (const uint32_t *)(blk + BLOCK_HEAD_BYTES);
        uint32_t word = 0;
        for (int r = 0; r < 32; ++r) {
            uint32_t par = 0;
            for (uint32_t i = 0; i < 2 * n_pairs; ++i) {
                const uint32_t k = ((ix[(i >> 1) * 32 + r] >> (16 * (i & 1u))) & 0xFFFFu) >> 3;
                uint64_t bit = 0;
#pragma unroll
                for (int w = 0; w < W; ++w) bit |= ((uint32_t)w == (k >> 6)) ? (v[w] >> (k & 63u)) & 1u : 0u;
                par ^= (uint32_t)bit;
            }
            word |= par << r;
        }
        out[b] = word;
        blk += BLOCK_HEAD_BYTES + 128 * n_pairs;
    }
}

// Fast path: exact when the host proved every coefficient stays below 2^62
// (T = uint64_t) or that every value it must know exactly stays below 2^31
// (T = uint32_t, TF_NARROW): adds and multiplies wrap, so intermediate sums
// may leave the narrow range, but the values at each halving, at the
// widening and at the end are the true ones.  S shots at once, from their
// parity-row bits.
// TN: word of the NodePhases block, T: word of the rest (TN = uint32_t, T =
// uint64_t is the hybrid path: NodePhases proven below 2^31, the rest not).
// The head of a parity block: index-pair count and the seven role masks.
struct BlockHead {
    uint32_t n_pairs, P1, P2, P4, E3, E1, PP, K0;
};
KS_HD BlockHead load_block_head(const uint8_t *blk)
{
    BlockHead m;
#if defined(__CUDA_ARCH__)
    const uint4 x = *(const uint4 *)blk, y = *(const uint4 *)(blk + 16);
    m.n_pairs = x.x; m.P1 = x.y; m.P2 = x.z; m.P4 = x.w;
    m.E3 = y.x; m.E1 = y.y; m.PP = y.z; m.K0 = y.w;
#else
    const uint32_t *u = (const uint32_t *)blk;
    m.n_pairs = u[0]; m.P1 = u[1]; m.P2 = u[2]; m.P4 = u[3];
    m.E3 = u[4]; m.E1 = u[5]; m.PP = u[6]; m.K0 = u[7];
#endif
    return m;
}

// A shot's running sums over a fast term's blocks: rotation (mod 8), lambda
// exponent (+ n1), and the class-0 kill with its pw.
struct RowSums {
    uint32_t rot, lam, alive;
    int32_t pw;  // halvings within one term stay far below 2^31
};
KS_HD void row_sums_init(RowSums &a, const TermHdr &h)
{
    a.rot = 0;
    a.lam = 0;
    a.alive = 1;
    a.pw = h.np_pw;
}
// Block b with row-parity word w.
KS_HD void row_sums_add(RowSums &a, uint32_t w, const BlockHead &m, uint32_t b, const uint16_t *dead_pw)
{
    if (m.K0) {
        const uint32_t k = w & m.K0;
        if (k != 0 && a.alive) {
            a.pw = (int32_t)dead_pw[32 * b + (uint32_t)ffs32(k)];
            a.alive = 0;
        }
    }
    a.rot += popc32(w & m.P1) + 2u * popc32(w & m.P2) + 4u * popc32(w & (m.P4 | (m.PP & (w >> 1))));
    a.lam += popc32((w & m.E3) | (~w & m.E1));
}
KS_HD const uint16_t *term_dead_pw(const uint8_t *p, const TermHdr &h)
{
    return (const uint16_t *)(p + term_meta_off(h) + TERM_FFK_BYTES);
}

// The rest of a fast term from its block sums (a) and its row-parity bits
// (read for the PhasePairs rows).
template <typename TN, typename T, int S>
KS_HD const uint8_t *eval_term_rows(const uint8_t *p, const TermHdr &h, const RowSums (&sums)[S],
                                    const RowBits (&bits)[S], TermOut (&o)[S])
{
    const uint8_t *meta = p + term_meta_off(h);
    uint32_t rot[S], lam[S], alive[S];
    int32_t pw[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        rot[s] = sums[s].rot;
        lam[s] = sums[s].lam;
        alive[s] = sums[s].alive;
        pw[s] = sums[s].pw;
    }
    // NodePhases: C * lambda^(m3 - m1); its rotation w^(6 (m1 + m2 + m3)) is
    // in rot with the HalfPi and PiProducts ones (units: they change no
    // valuation and commute with the PhasePairs factors, so they join the
    // prefactor's w^idx at the end; the reference's renormalisation after
    // HalfPi cannot fire)
    const uint64_t *cp = (const uint64_t *)(p + TERM_NPC_OFF);
    const Zr<TN> c = {(TN)cp[0], (TN)cp[1], (TN)cp[2], (TN)cp[3]};
    const bool odd = term_np_odd(h);
    const uint8_t *npl = p + term_npl_off(h);
    Zr<T> z[S];
#pragma unroll
    for (int s = 0; s < S; ++s) {
        // C lambda^(m3 - m1), tabulated per term: lam = m3 + (n1 - m1)
        Zr<TN> zn = c;
        if (odd) zn = load_npl(npl, lam[s], TN());
        const TN keep = (TN)0 - (TN)alive[s];
        zn.a &= keep; zn.b &= keep; zn.c &= keep; zn.d &= keep;
        if constexpr (sizeof(TN) == sizeof(T)) {
            z[s].a = (T)zn.a; z[s].b = (T)zn.b; z[s].c = (T)zn.c; z[s].d = (T)zn.d;
        } else {
            z[s] = widen(zn);  // sign-extend to the 64-bit words of the rest
        }
    }
    const int ph0 = term_ph_row0(h);
    // PhasePairs in pairs: the valuation of z (known per shot: the
    // NodePhases result has nu = (2 n2 + n1 + n3) mod 4, and each factor's nu
    // is fixed by its signs) decides the reference's two halvings, so one
    // product with the tabulated F F' and one shift replace two factors and
    // two evenness tests; the pair's step table gives the halvings, the next
    // nu and whether a zero factor ended the halvings, from (signs, nu).
    {
        const uint32_t n_pair = term_ph_pairs(h);
        const uint8_t *ptab = p + term_pair_tab_off(h);
        const uint8_t *pstep = p + term_pair_step_off(h);
        uint32_t nu[S];
#pragma unroll
        for (int s = 0; s < S; ++s) nu[s] = alive[s] ? h.nu0 : NU_DEAD;  // a class-0 kill: no halvings
        for (uint32_t q = 0; q < n_pair; ++q) {
            const int pos = ph0 + 4 * (int)q;
#pragma unroll
            for (int s = 0; s < S; ++s) {
                const uint32_t c = (bits[s].word(pos >> 5) >> (pos & 31)) & 15u;
                const uint32_t e = pstep[256 * q + 16 * c + nu[s]];
                const uint32_t hh = e & 3u;
                nu[s] = e >> 2;
                const uint32_t fw = *(const uint32_t *)(ptab + 64 * q + 4 * c);  // 4 x i8
                const Zr<T> F = {(T)(int64_t)sext_byte<0>(fw), (T)(int64_t)sext_byte<1>(fw),
                                 (T)(int64_t)sext_byte<2>(fw), (T)(int64_t)sext_byte<3>(fw)};
                z[s] = zmul(z[s], F);
                shr_all(z[s], hh);
                pw[s] += (int32_t)hh;
            }
        }
    }
    // prefactor: w^(NodePhases + HalfPi + PiProducts + idx) times the exact
    // floatfactor (one product with the tabulated ff * w^k), then one
    // renormalisation
#pragma unroll
    for (int s = 0; s < S; ++s) {
        int32_t f[4];
        load_i32x4(meta + 16 * (rot[s] & 7u), f);
        const Zr<T> ffk = {(T)(int64_t)f[0], (T)(int64_t)f[1], (T)(int64_t)f[2], (T)(int64_t)f[3]};
        Zr<T> zz = zmul(z[s], ffk);
        zreduce(zz, pw[s]);
        if constexpr (sizeof(T) == 8) {
            o[s].z = zz;
        } else {
            o[s].z = widen(zz);
        }
        o[s].pw = (int64_t)pw[s];
        o[s].power2 = h.power2;
        o[s].risk = 0;
    }
    return p + h.rec_bytes;
}

// A fast term on the path its header selects.
template <int S>
KS_HD const uint8_t *eval_term_rows_any(const uint8_t *p, const TermHdr &h, const RowSums (&sums)[S],
                                        const RowBits (&bits)[S], TermOut (&o)[S])
{
    if (h.flags & TF_NARROW) return eval_term_rows<uint32_t, uint32_t, S>(p, h, sums, bits, o);
    if (h.flags & TF_HYBRID) return eval_term_rows<uint32_t, uint64_t, S>(p, h, sums, bits, o);
    return eval_term_rows<uint64_t, uint64_t, S>(p, h, sums, bits, o);
}

// Exact path: the reference's step-by-step arithmetic (zx_eval.hpp:101-165),
// int64 wrap included, over the same records.
template <int W>
KS_HD const uint8_t *eval_term_exact(const uint8_t *p, const TermHdr &h, const uint64_t (&v)[W],
                                     TermOut &o)
{
    constexpr int R1 = rec1_words(W), R2 = rec2_words(W);
    const uint64_t *q = (const uint64_t *)(p + TERM_HDR_BYTES + ((h.flags & TF_APX) ? TERM_APX_BYTES : 0));
    const Zu one = {1, 0, 0, 0};
    Zu z = one;
    int64_t pw = 0;
    uint32_t risk = 0;
    for (uint32_t t = 0; t < h.n_np; ++t, q += R1) {
        // phase + 4 par (mod 8) = (phase & 3) + 4 (par ^ phase bit 2): the mask
        // carries bit 2 of the phase in the constant bit
        const uint32_t cw = (uint32_t)q[W];
        const uint32_t k = ((parity<W>(q, v) << 2) | (cw & 3u)) & 7u;
        Zu u = rot_var(one, k);
        u.a += 1;
        risk |= over62(z);
        z = zmul(z, u);
        zreduce(z, pw);
    }
    {
        uint32_t tot = 0;
        for (uint32_t t = 0; t < h.n_hp; ++t, q += R1)
            tot += (parity<W>(q, v) * (uint32_t)q[W]) & 7u;
        risk |= over62(z);
        z = zmul(z, rot_var(one, tot & 7u));
        zreduce(z, pw);
    }
    {
        uint32_t e = 0;
        for (uint32_t t = 0; t < h.n_pp; ++t, q += R2) {
            const uint32_t psi = parity<W>(q, v), phi = parity<W>(q + W, v);  // constants folded in
            e ^= psi & phi;
        }
        if (e) { z.a = 0 - z.a; z.b = 0 - z.b; z.c = 0 - z.c; z.d = 0 - z.d; }
    }
    for (uint32_t t = 0; t < h.n_ph; ++t, q += R2) {
        const uint32_t cw = (uint32_t)q[2 * W];
        const uint32_t al = ((cw & 3u) | (parity<W>(q, v) << 2)) & 7u;
        const uint32_t be = (((cw >> 3) & 3u) | (parity<W>(q + W, v) << 2)) & 7u;
        const Zu u = rot_var(one, al), x = rot_var(one, be), y = rot_var(one, (al + be) & 7u);
        Zu term = {1 + u.a + x.a - y.a, u.b + x.b - y.b, u.c + x.c - y.c, u.d + x.d - y.d};
        risk |= over62(z);
        z = zmul(z, term);
        zreduce(z, pw);
    }
    risk |= over62(z);
    z = zmul(z, rot_var(one, h.pf_idx));
    risk |= over62(z);
    z = zmul(z, h.ff);
    zreduce(z, pw);
    o.z = z;
    o.pw = pw;
    o.power2 = h.power2;
    o.risk = risk ? 1u : 0u;
    return (const uint8_t *)q;
}

constexpr double SQ = 0.70710678118654752440;  // cos(pi/4)

// Complex value of a finished term (zx_eval.hpp:166-176), no FMA contraction.
KS_HD void term_complex(const TermOut &o, const uint8_t *hdr_ptr, uint32_t flags, double &re, double &im)
{
    const double A = (double)(int64_t)o.z.a, Bv = (double)(int64_t)o.z.b;
    const double C = (double)(int64_t)o.z.c, D = (double)(int64_t)o.z.d;
    re = dadd(A, dmul(dadd(Bv, D), SQ));
    im = dadd(C, dmul(dsub(Bv, D), SQ));
    const double s = (flags & TF_EXP) ? pow2_normal((int32_t)o.pw + o.power2) : pow2i(o.pw + (int64_t)o.power2);
    re = dmul(re, s);
    im = dmul(im, s);
    if (flags & TF_APX) {
        const double *ap = (const double *)(hdr_ptr + TERM_HDR_BYTES);
        const double ar = ap[0], ai = ap[1];
        const double r2 = dsub(dmul(re, ar), dmul(im, ai));
        im = dadd(dmul(re, ai), dmul(im, ar));
        re = r2;
    }
}

// One term for S shots on the path its header selects (per-shot parity rows).
// Returns the next record.
template <int W, int S>
KS_HD const uint8_t *eval_term_s(const uint8_t *p, const TermHdr &h, const uint64_t (&v)[S][W],
                                 TermOut (&o)[S])
{
    if (h.flags & TF_SLOW) {
#pragma unroll
        for (int s = 0; s < S; ++s) eval_term_exact<W>(p, h, v[s], o[s]);
        return p + h.rec_bytes;
    }
    uint32_t words[S][NB_MAX + 1];
    RowBits bits[S];
    RowSums sums[S];
    const uint16_t *dead_pw = term_dead_pw(p, h);
#pragma unroll
    for (int s = 0; s < S; ++s) {
        term_words_shot<W>(p, h, v[s], words[s]);
        bits[s].w = words[s];
        bits[s].stride = 1;
        row_sums_init(sums[s], h);
        const uint8_t *blk = p + term_blocks_off(h);
        for (uint32_t b = 0; b < h.nb; ++b) {
            const BlockHead m = load_block_head(blk);
            row_sums_add(sums[s], words[s][b], m, b, dead_pw);
            blk += BLOCK_HEAD_BYTES + 128 * m.n_pairs;
        }
    }
    return eval_term_rows_any<S>(p, h, sums, bits, o);
}

// One term for one shot.
template <int W>
KS_HD const uint8_t *eval_term(const uint8_t *p, const TermHdr &h, const uint64_t (&v)[W], TermOut &o)
{
    return eval_term_s<W, 1>(p, h, reinterpret_cast<const uint64_t(&)[1][W]>(v),
                             reinterpret_cast<TermOut(&)[1]>(o));
}

// Evaluate `n_terms` consecutive term records starting at p for S shots,
// adding each term's complex value to (sum_re[s], sum_im[s]) in order.
// Risk flags count only for the shots set in `live`.  Returns the end pointer.
template <int W, int S>
KS_HD const uint8_t *eval_terms_s(const uint8_t *p, uint32_t n_terms, const uint64_t (&v)[S][W],
                                  double (&sum_re)[S], double (&sum_im)[S], uint32_t &risk,
                                  uint32_t live = ~0u)
{
    for (uint32_t t = 0; t < n_terms; ++t) {
        const TermHdr h = load_hdr(p);
        TermOut o[S];
        const uint8_t *next = eval_term_s<W, S>(p, h, v, o);
#pragma unroll
        for (int s = 0; s < S; ++s) {
            double re, im;
            term_complex(o[s], p, h.flags, re, im);
            sum_re[s] = dadd(sum_re[s], re);
            sum_im[s] = dadd(sum_im[s], im);
            risk |= o[s].risk & (live >> s);
        }
        p = next;
    }
    return p;
}

// The same for one shot.
template <int W>
KS_HD const uint8_t *eval_terms(const uint8_t *p, uint32_t n_terms, const uint64_t (&v)[W], double &sum_re,
                                double &sum_im, uint32_t &risk)
{
    return eval_terms_s<W, 1>(p, n_terms, reinterpret_cast<const uint64_t(&)[1][W]>(v),
                              reinterpret_cast<double(&)[1]>(sum_re), reinterpret_cast<double(&)[1]>(sum_im),
                              risk);
}

// Parameter-vector masks: bits [lo, hi) of word w.
KS_HD uint64_t bit_range(int w, int64_t lo, int64_t hi)
{
    const int64_t b0 = (int64_t)w * 64, b1 = b0 + 64;
    const int64_t s = lo > b0 ? lo : b0, e = hi < b1 ? hi : b1;
    if (e <= s) return 0;
    const int n = (int)(e - s), o = (int)(s - b0);
    const uint64_t m = n == 64 ? ~0ull : ((1ull << n) - 1);
    return m << o;
}

// ---- uniform streams --------------------------------------------------------
KS_HD uint64_t xorshift_init(uint64_t seed, uint64_t shot)
{
    uint64_t r = seed ^ (shot * 0x9e3779b97f4a7c15ull);
    r ^= r >> 30;
    r *= 0xbf58476d1ce4e5b9ull;
    r ^= r >> 27;
    return r ? r : 1ull;
}

KS_HD double xorshift_uniform(uint64_t &s)
{
    s ^= s << 13;
    s ^= s >> 7;
    s ^= s << 17;
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
}

KS_HD uint32_t mulhi32(uint32_t a, uint32_t b)
{
#if defined(__CUDA_ARCH__)
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 10 rounds of the
// multiply-xor S-box with Weyl key schedule.  c: counter in, block out.
KS_HD void philox4x32_10(uint32_t (&c)[4], uint64_t seed)
{
    uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r) { k0 += 0x9E3779B9u; k1 += 0xBB67AE85u; }
        const uint32_t h0 = mulhi32(0xD2511F53u, c[0]), l0 = 0xD2511F53u * c[0];
        const uint32_t h1 = mulhi32(0xCD9E8D57u, c[2]), l1 = 0xCD9E8D57u * c[2];
        const uint32_t n0 = h1 ^ c[1] ^ k0, n2 = h0 ^ c[3] ^ k1;
        c[0] = n0; c[1] = l1; c[2] = n2; c[3] = l0;
    }
}

// Uniform of (shot, output): counter (shot lo, shot hi, output, 0), key = seed.
KS_HD double philox_uniform(uint64_t seed, uint64_t shot, uint32_t output)
{
    uint32_t c[4] = {(uint32_t)shot, (uint32_t)(shot >> 32), output, 0u};
    philox4x32_10(c, seed);
    const uint64_t bits = ((uint64_t)c[1] << 32) | c[0];
    return (double)(bits >> 11) * (1.0 / 9007199254740992.0);
}

}  // namespace ksim
