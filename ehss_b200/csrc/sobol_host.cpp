// Host-side scrambled-Sobol set-up: bit-exact to scipy's
// qmc.Sobol(d, scramble=True, seed=seed), which the reference calls at
// src/support_exchange_transport/ehss_state.py:44 (impact disk) and
// ccs_cli.py:148 (adaptive PA directions).
//
// scipy draws its scrambling bits from numpy.random.default_rng(seed), i.e. a
// PCG64 generator seeded through numpy's SeedSequence, as integers(2, size,
// dtype=uint32): first d*30 shift bits (LSB-first), then d*30*30 bits of
// lower-triangular matrices whose diagonal is forced to one; each direction
// number's MSB-first 30-digit vector is multiplied by its dimension's matrix
// over GF(2) (Matousek's linear matrix scramble).  The published algorithms
// restated here:
//   * SeedSequence entropy pool and state generation (numpy, after O'Neill's
//     seed_seq_fe): 4-word pool, hash/mix constants as published;
//   * PCG64 = 128-bit LCG with XSL-RR 128/64 output; next_uint32 returns the
//     low then the high half of one 64-bit output;
//   * bounded uint32 draws by Lemire's multiply-shift; for the range {0, 1}
//     this is the top bit of each 32-bit word and never rejects;
//   * Joe--Kuo direction numbers (new-joe-kuo-6.21201), dimensions 1..8.
#include <cstdint>
#include <cstring>

namespace ehss {

namespace {

constexpr uint32_t kInitA = 0x43b0d7e5u, kMultA = 0x931e8875u;
constexpr uint32_t kInitB = 0x8b51f9ddu, kMultB = 0x58f38dedu;
constexpr uint32_t kMixL = 0xca01f9ddu, kMixR = 0x4973f715u;

struct SeedSequence {
    uint32_t pool[4];
    explicit SeedSequence(uint64_t seed) {
        uint32_t entropy[2];
        int n = 0;
        do { entropy[n++] = (uint32_t)(seed & 0xffffffffu); seed >>= 32; } while (seed != 0 && n < 2);
        uint32_t hash_const = kInitA;
        auto hashmix = [&hash_const](uint32_t v) {
            v ^= hash_const;
            hash_const *= kMultA;
            v *= hash_const;
            v ^= v >> 16;
            return v;
        };
        auto mix = [](uint32_t x, uint32_t y) {
            uint32_t r = kMixL * x - kMixR * y;
            r ^= r >> 16;
            return r;
        };
        for (int i = 0; i < 4; ++i) pool[i] = hashmix(i < n ? entropy[i] : 0u);
        for (int s = 0; s < 4; ++s)
            for (int d = 0; d < 4; ++d)
                if (s != d) pool[d] = mix(pool[d], hashmix(pool[s]));
        // entropy longer than the pool does not occur for seeds < 2^64
    }
    void generate(uint32_t* out, int n_words) const {
        uint32_t hash_const = kInitB;
        for (int i = 0; i < n_words; ++i) {
            uint32_t v = pool[i % 4];
            v ^= hash_const;
            hash_const *= kMultB;
            v *= hash_const;
            v ^= v >> 16;
            out[i] = v;
        }
    }
};

struct PCG64 {
    unsigned __int128 state, inc;
    bool has32 = false;
    uint32_t buf32 = 0;
    static unsigned __int128 mult() {
        return ((unsigned __int128)0x2360ED051FC65DA4ull << 64) | 0x4385DF649FCCF645ull;
    }
    explicit PCG64(uint64_t seed) {
        uint32_t w[8];
        SeedSequence(seed).generate(w, 8);
        uint64_t u[4];
        for (int i = 0; i < 4; ++i) u[i] = (uint64_t)w[2 * i] | ((uint64_t)w[2 * i + 1] << 32);
        unsigned __int128 s = ((unsigned __int128)u[0] << 64) | u[1];
        unsigned __int128 q = ((unsigned __int128)u[2] << 64) | u[3];
        state = 0;
        inc = (q << 1) | 1u;
        step();
        state += s;
        step();
    }
    void step() { state = state * mult() + inc; }
    uint64_t next64() {
        step();
        uint64_t x = (uint64_t)(state >> 64) ^ (uint64_t)state;
        unsigned rot = (unsigned)(state >> 122);
        return (x >> rot) | (x << ((64u - rot) & 63u));
    }
    uint32_t next32() {
        if (has32) { has32 = false; return buf32; }
        uint64_t v = next64();
        has32 = true;
        buf32 = (uint32_t)(v >> 32);
        return (uint32_t)v;
    }
    uint32_t bit() { return next32() >> 31; }   // Lemire bounded draw on {0, 1}
};

// (degree s, coefficient a, m_1..m_s) for dimensions 2..8
struct JK { int s, a; uint32_t m[5]; };
const JK kJoeKuo[7] = {
    {1, 0, {1}}, {2, 1, {1, 3}}, {3, 1, {1, 3, 1}}, {3, 2, {1, 1, 1}},
    {4, 1, {1, 1, 3, 3}}, {4, 4, {1, 3, 5, 13}}, {5, 2, {1, 1, 5, 5, 17}},
};

}  // namespace

constexpr int kBits = 30;
constexpr int kMaxDim = 8;

void sobol_direction_numbers(int dim, uint32_t* v /* [dim*30] */) {
    for (int k = 0; k < kBits; ++k) v[k] = 1u << (kBits - 1 - k);
    for (int j = 1; j < dim; ++j) {
        const JK& p = kJoeKuo[j - 1];
        uint32_t* row = v + j * kBits;
        for (int k = 0; k < kBits; ++k) {
            if (k < p.s) {
                row[k] = p.m[k] << (kBits - 1 - k);
            } else {
                uint32_t x = row[k - p.s] ^ (row[k - p.s] >> p.s);
                for (int t = 1; t < p.s; ++t)
                    if ((p.a >> (p.s - 1 - t)) & 1) x ^= row[k - t];
                row[k] = x;
            }
        }
    }
}

bool sobol_scramble(int dim, uint64_t seed, uint32_t* sv, uint32_t* shift) {
    if (dim < 1 || dim > kMaxDim) return false;
    PCG64 rng(seed);
    for (int j = 0; j < dim; ++j) {
        uint32_t s = 0;
        for (int k = 0; k < kBits; ++k) s |= rng.bit() << k;
        shift[j] = s;
    }
    // L[j][i][l], i = row (output digit, MSB-first), l = column; tril + unit diagonal
    static thread_local uint8_t L[kMaxDim][kBits][kBits];
    for (int j = 0; j < dim; ++j)
        for (int i = 0; i < kBits; ++i)
            for (int l = 0; l < kBits; ++l) {
                uint8_t b = (uint8_t)rng.bit();
                L[j][i][l] = (l < i) ? b : (l == i ? 1 : 0);
            }
    uint32_t v[kMaxDim * kBits];
    sobol_direction_numbers(dim, v);
    for (int j = 0; j < dim; ++j)
        for (int k = 0; k < kBits; ++k) {
            uint32_t in = v[j * kBits + k], out = 0;
            for (int i = 0; i < kBits; ++i) {
                uint32_t acc = 0;
                for (int l = 0; l <= i; ++l) acc ^= L[j][i][l] & ((in >> (kBits - 1 - l)) & 1u);
                out |= acc << (kBits - 1 - i);
            }
            sv[j * kBits + k] = out;
        }
    return true;
}

}  // namespace ehss
