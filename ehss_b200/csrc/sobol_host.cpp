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
    // Row i of dimension j's matrix (output digit i, MSB-first; tril + unit
    // diagonal) as a mask over the input word: column l <-> bit 29 - l, so
    // digit i of the product is the parity of (row & input).  Every bit is
    // drawn, in numpy's order, including those above the diagonal.
    uint32_t rows[kMaxDim][kBits];
    for (int j = 0; j < dim; ++j)
        for (int i = 0; i < kBits; ++i) {
            uint32_t m = 0;
            for (int l = 0; l < kBits; ++l) {
                uint32_t b = rng.bit();
                if (l < i) m |= b << (kBits - 1 - l);
            }
            rows[j][i] = m | (1u << (kBits - 1 - i));
        }
    uint32_t v[kMaxDim * kBits];
    sobol_direction_numbers(dim, v);
    for (int j = 0; j < dim; ++j)
        for (int k = 0; k < kBits; ++k) {
            const uint32_t in = v[j * kBits + k];
            uint32_t out = 0;
            for (int i = 0; i < kBits; ++i)
                out |= (uint32_t)(__builtin_popcount(rows[j][i] & in) & 1) << (kBits - 1 - i);
            sv[j * kBits + k] = out;
        }
    return true;
}

}  // namespace ehss

namespace ehss {

// Coherent enumeration of one block's 2^m Sobol(4) points.
//
// Point n is q(n) = shift ^ XOR_k n_k D[k] with D[k] = sv[k] ^ sv[k-1] (the
// Gray-code recurrence written on the bits of n).  Rows "bit b of dimension
// j" of this linear map are taken greedily, coarsest digits first and the
// four dimensions in turn, keeping each row that is independent of those
// already taken, until m rows form an invertible matrix A (always possible:
// the leading m digits of dimension 0 alone are a bijection).  Position p is
// given the point whose selected digits equal the bits of p (first row = most
// significant bit of p): n = A^-1 (p ^ s), so consecutive positions differ
// only in the finest selected digits and a warp's rays have nearby directions
// and impact points.  The positions 0..2^m-1 enumerate exactly the same point
// set as the indices 0..2^m-1.  Output: point(p) = base ^ XOR_{bit e of p}
// basis[e] (dimension-major: basis[e*4 + j]).
bool sobol_coherent_order(int m, const uint32_t* sv /* [4*30] dim-major */, const uint32_t* shift /* [4] */,
                          uint32_t* basis /* [30*4] */, uint32_t* base /* [4] */) {
    if (m < 0 || m > 30) return false;
    constexpr int kDims = 4;
    uint32_t D[kDims][kBits];
    for (int j = 0; j < kDims; ++j)
        for (int k = 0; k < kBits; ++k) D[j][k] = sv[j * kBits + k] ^ (k > 0 ? sv[j * kBits + k - 1] : 0u);
    // candidate rows in preferred order; row = m-bit mask over n's bits
    uint32_t rows[kBits];        // selected rows as bit masks over n (bit k <-> n_k)
    uint32_t rshift[kBits];      // shift bit of each selected row
    uint32_t echelon[kBits];     // reduced copies for the independence test
    int pivot[kBits];
    int taken = 0;
    for (int b = 0; b < kBits && taken < m; ++b)
        for (int j = 0; j < kDims && taken < m; ++j) {
            uint32_t row = 0;
            for (int k = 0; k < m; ++k) row |= ((D[j][k] >> (kBits - 1 - b)) & 1u) << k;
            uint32_t red = row;
            for (int t = 0; t < taken; ++t)
                if ((red >> pivot[t]) & 1u) red ^= echelon[t];
            if (!red) continue;
            int pv = 31 - __builtin_clz(red);
            echelon[taken] = red;
            pivot[taken] = pv;
            rows[taken] = row;
            rshift[taken] = (shift[j] >> (kBits - 1 - b)) & 1u;
            ++taken;
        }
    if (taken < m) return false;
    // invert A (rows[t] . n = y_t) by Gauss-Jordan on [A | I]
    uint32_t a[kBits], inv[kBits];
    for (int t = 0; t < m; ++t) { a[t] = rows[t]; inv[t] = 1u << t; }
    for (int col = 0; col < m; ++col) {
        int r = col;
        while (r < m && !((a[r] >> col) & 1u)) ++r;
        if (r == m) return false;
        uint32_t ta = a[r], ti = inv[r];
        a[r] = a[col]; inv[r] = inv[col]; a[col] = ta; inv[col] = ti;
        for (int q = 0; q < m; ++q)
            if (q != col && ((a[q] >> col) & 1u)) { a[q] ^= a[col]; inv[q] ^= inv[col]; }
    }
    // now n_k = XOR_t inv[k]_t y_t ; y_t = bit (m-1-t) of p ^ rshift[t]
    auto apply = [&](uint32_t nbits, uint32_t* out) {      // out[j] = XOR_k n_k D[j][k]
        for (int j = 0; j < kDims; ++j) {
            uint32_t v = 0;
            for (int k = 0; k < m; ++k)
                if ((nbits >> k) & 1u) v ^= D[j][k];
            out[j] = v;
        }
    };
    auto n_of_y = [&](uint32_t ybits) {                    // ybits bit t = y_t
        uint32_t n = 0;
        for (int k = 0; k < m; ++k)
            n |= (uint32_t)(__builtin_popcount(inv[k] & ybits) & 1) << k;
        return n;
    };
    uint32_t s = 0;
    for (int t = 0; t < m; ++t) s |= rshift[t] << t;
    uint32_t c[kDims];
    apply(n_of_y(s), c);
    for (int j = 0; j < kDims; ++j) base[j] = shift[j] ^ c[j];
    for (int e = 0; e < kBits; ++e) {
        uint32_t col[kDims] = {0, 0, 0, 0};
        if (e < m) apply(n_of_y(1u << (m - 1 - e)), col);
        for (int j = 0; j < kDims; ++j) basis[e * kDims + j] = col[j];
    }
    return true;
}

}  // namespace ehss
