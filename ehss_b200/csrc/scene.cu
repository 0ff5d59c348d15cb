// Device LBVH scene builder (batched over structures).
//
// Replaces the reference's static preparation (PreparedStaticCPUEHSS,
// src/support_exchange_transport/ehss_static.py:62-101: median groups,
// implicit topology, padded leaf bounds, parent unions) and the PA index
// build (SphereIndex / build_tree, pa_spatial.py:38-75, 157-160).  The tree
// differs by design -- results do not depend on it, because every traversal
// keeps the reference's (distance, atom id) minimum and prunes only boxes
// that provably contain no nearer entry.
//
// Pipeline (one launch each, all structures of a batch at once):
//   1. k_stats     per structure: scene header (layout offsets), sequential
//                  FP64 mean of the centres (the order numpy's mean(axis=0)
//                  uses), enclosing radius R, scale S, largest radius, centre
//                  bounds, input validation
//   2. k_morton    per atom: 30-bit Morton code of the centre in its
//                  structure's centre box; key = structure << 31 | buried << 30
//                  | code (buried only in the second pass of an exterior build)
//   3. stable sort of (key, atom) pairs, so equal codes keep atom order:
//                  per structure in one CTA (k_morton_segsort, steps 2-3 in one
//                  launch) when every structure holds at most 8192 atoms, else
//                  a device-wide LSD radix sort over the key's significant bits
//                  (k_radix_count / k_radix_scan / k_radix_scatter, 8 bits a pass)
//   4. k_karras    per internal node: Karras (2012) range / split search
//                  within the structure's segment of tree atoms
//   5. k_refit     per atom: FP32 boxes rounded outward, unioned bottom-up
//                  with one atomic arrival counter per internal node
//   6. k_emit_*    per internal node: 128-byte 4-wide record built from the
//                  binary node's children and grandchildren (boxes expanded
//                  by eps_box; subtrees of at most leaf_size atoms collapsed
//                  into leaf references); per atom: FP32 and FP64 records in
//                  leaf order, id maps.
// Exterior builds (EHSS_BUILD_EXTERIOR) then run k_exposure on that tree and
// repeat steps 2-6 with the buried atoms sorted behind the exposed ones and
// left out of the tree.
#include <cub/block/block_radix_sort.cuh>
#include <cub/block/block_scan.cuh>
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <vector>
#include "ehss_internal.cuh"

namespace ehss {

struct BuildDesc {
    const double* xyz;
    const double* radii;
    char* scene;
    int64_t n;
    int64_t atom0;       // first global atom index
    int64_t inner0;      // first global internal-node index
    int32_t leaf_size;
    int32_t exterior;
    int64_t n_active;          // atoms in the tree (exterior scenes: the exposed atoms)
    double cmin[3], cext[3];   // centre box relative to the scene centre (filled by k_stats)
    int32_t refit;             // 1: new coordinates for an existing full scene (tree kept)
    int32_t pad;
};

// Header status codes (0 = valid scene).
constexpr int32_t kStatusBadInput = 1;     // non-positive or non-finite radius, non-finite coordinate
constexpr int32_t kStatusRefitMismatch = 3;   // refit of a scene that is not a full scene of n atoms
constexpr int32_t kStatusCorrupt = 4;      // refit found a malformed node record

struct BuildWork {
    BuildDesc* descs;
    int32_t* atom_scene;     // [N] structure of each global atom
    uint64_t* keys_in;       // [N]
    uint64_t* keys_out;      // [N]
    int32_t* vals_in;        // [N]
    int32_t* vals_out;       // [N]
    int32_t* inner_child;    // [2*I] child refs of Karras internal nodes (>=0 inner local idx, <0 ~leaf)
    int32_t* inner_range;    // [2*I] first/last sorted position (local)
    int32_t* parent_inner;   // [I]   parent local inner index of each internal node (-1 root)
    int32_t* parent_leaf;    // [N]   parent local inner index of each leaf
    float* inner_box;        // [6*I]
    float* leaf_box;         // [6*N]
    int32_t* inner_height;   // [I]
    uint32_t* arrivals;      // [I]
    uint8_t* culled;         // [N] 1 = buried atom (exterior builds)
    uint32_t* radix_counts;  // [256 * tiles] per-tile digit counts of the device-wide sort
    uint32_t* radix_offsets; // [256 * tiles] their exclusive scan (digit-major)
};

// --------------------------------------------------------------------------
__global__ void k_stats(BuildDesc* descs, int n_scenes) {
    int s = blockIdx.x;
    if (s >= n_scenes) return;
    BuildDesc& D = descs[s];
    SceneHeader* H = reinterpret_cast<SceneHeader*>(D.scene);
    const int64_t n = D.n;
    __shared__ double center[3];
    __shared__ int bad;
    if (D.refit) {
        // refit: the tree fields stay; the scene must be a valid full scene of n atoms
        __shared__ int mismatch;
        if (threadIdx.x == 0) {
            uint64_t on, oa, o64, oi, orr, total;
            scene_layout(n, &on, &oa, &o64, &oi, &orr, &total);
            mismatch = !(H->magic == kSceneMagic && H->status == 0 && H->exterior == 0 && H->n_atoms == n &&
                         H->n_active == n && H->n_nodes >= 1 && H->n_nodes <= (n > 1 ? n - 1 : 1) &&
                         H->off_nodes == on && H->off_atoms == oa && H->off_atoms64 == o64 && H->off_ids == oi &&
                         H->off_rank == orr && H->bytes == total);
            if (mismatch) H->status = kStatusRefitMismatch;
            bad = 0;
        }
        __syncthreads();
        if (mismatch) return;
    } else {
        // header: zeroed, then the layout offsets (the rest is filled below and by k_emit_nodes)
        if (threadIdx.x < sizeof(SceneHeader) / 4) reinterpret_cast<uint32_t*>(H)[threadIdx.x] = 0u;
        __syncthreads();
        if (threadIdx.x == 0) {
            bad = 0;
            scene_layout(n, &H->off_nodes, &H->off_atoms, &H->off_atoms64, &H->off_ids, &H->off_rank, &H->bytes);
        }
    }
    __syncthreads();
    // Sequential sum, one lane per coordinate: numpy's mean(axis=0) adds the
    // rows in order and divides by n (ehss_state.py:46).
    if (threadIdx.x < 3) {
        int c = threadIdx.x;
        double acc = 0.;
        int64_t i = 0;
        for (; i + 8 <= n; i += 8) {         // loads ahead of the (sequential) sum
            double v[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) v[k] = D.xyz[(i + k) * 3 + c];
#pragma unroll
            for (int k = 0; k < 8; ++k) acc = dadd(acc, v[k]);
        }
        for (; i < n; ++i) acc = dadd(acc, D.xyz[i * 3 + c]);
        center[c] = ddiv(acc, (double)n);
    }
    // validation and radii extrema
    double rmax = 0.;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        double r = D.radii[i];
        double x = D.xyz[i * 3], y = D.xyz[i * 3 + 1], z = D.xyz[i * 3 + 2];
        if (!(r > 0.) || !isfinite(r) || !isfinite(x) || !isfinite(y) || !isfinite(z)) bad = 1;
        rmax = fmax(rmax, r);
    }
    __syncthreads();
    // R = max(|c_j - center| + r_j) * (1 + 1e-9) (ehss_state.py:47); norm as
    // numpy's linalg.norm(axis=1): sqrt((x*x + y*y) + z*z).
    double smax = 0.;
    double lo[3] = {CUDART_INF, CUDART_INF, CUDART_INF}, hi[3] = {-CUDART_INF, -CUDART_INF, -CUDART_INF};
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
        double x = dsub(D.xyz[i * 3], center[0]);
        double y = dsub(D.xyz[i * 3 + 1], center[1]);
        double z = dsub(D.xyz[i * 3 + 2], center[2]);
        double len = dadd(dsqrt(dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z))), D.radii[i]);
        smax = fmax(smax, len);
        lo[0] = fmin(lo[0], x); lo[1] = fmin(lo[1], y); lo[2] = fmin(lo[2], z);
        hi[0] = fmax(hi[0], x); hi[1] = fmax(hi[1], y); hi[2] = fmax(hi[2], z);
    }
    // block-wide maxima (order-independent): warp shuffles, then one warp
    __shared__ double partial[8][32];
    __shared__ double result[8];
    double vals[8] = {rmax, smax, -lo[0], -lo[1], -lo[2], hi[0], hi[1], hi[2]};
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int k = 0; k < 8; ++k) {
        double m = vals[k];
        for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
        if (lane == 0) partial[k][warp] = m;
    }
    __syncthreads();
    if (warp == 0) {
        for (int k = 0; k < 8; ++k) {
            double m = lane < nwarps ? partial[k][lane] : -CUDART_INF;
            for (int off = 16; off > 0; off >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, off));
            if (lane == 0) result[k] = m;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        H->magic = kSceneMagic;
        H->status = bad ? kStatusBadInput : 0;
        H->n_atoms = (int32_t)n;
        if (!D.refit) H->leaf_size = D.leaf_size;
        for (int c = 0; c < 3; ++c) H->center[c] = center[c];
        H->rmax = result[0];
        H->scale = result[1];
        H->radius = dmul(result[1], 1.000000001);
        H->scale_f = __double2float_ru(result[1]);
        H->rmax_f = __double2float_ru(result[0]);
        // FP32 box expansion: 2^-14 S covers the FP32 rounding of any ray
        // whose origin lies within 3 S of the centre (the traversal sends
        // farther origins to the FP64 all-atom search).
        H->eps_box = __double2float_ru(result[1] * 0x1p-14);
        for (int c = 0; c < 3; ++c) {
            D.cmin[c] = -result[2 + c];
            D.cext[c] = result[5 + c] + result[2 + c];
        }
    }
}

__device__ __forceinline__ uint32_t spread10(uint32_t v) {
    v &= 0x3ffu;
    v = (v | (v << 16)) & 0x030000FFu;
    v = (v | (v << 8)) & 0x0300F00Fu;
    v = (v | (v << 4)) & 0x030C30C3u;
    v = (v | (v << 2)) & 0x09249249u;
    return v;
}

// Morton key of atom i of structure D (low 31 bits: buried flag << 30 | 30-bit
// code of the centre in the structure's centre box).
__device__ __forceinline__ uint32_t morton_key31(const BuildDesc& D, const SceneHeader* H, int64_t i, bool buried) {
    uint32_t q[3];
    for (int c = 0; c < 3; ++c) {
        double rel = (D.xyz[i * 3 + c] - H->center[c]) - D.cmin[c];
        double e = D.cext[c];
        double u = e > 0. ? rel / e : 0.;
        u = fmin(fmax(u, 0.), 1.);
        q[c] = (uint32_t)fmin(u * 1024.0, 1023.0);
    }
    uint32_t code = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
    return (buried ? (1u << 30) : 0u) | code;
}

__global__ void k_morton(const BuildDesc* descs, const int32_t* atom_scene, int64_t N, const uint8_t* culled,
                         uint64_t* keys, int32_t* vals) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= N) return;
    int s = atom_scene[g];
    const BuildDesc& D = descs[s];
    const SceneHeader* H = reinterpret_cast<const SceneHeader*>(D.scene);
    int64_t i = g - D.atom0;
    // buried atoms of an exterior build sort after every exposed atom of their structure
    const bool buried = culled && D.exterior && culled[g];
    keys[g] = ((uint64_t)s << 31) | morton_key31(D, H, i, buried);
    vals[g] = (int32_t)i;
}

// Batches whose structures all hold at most kSegSortMax atoms: keys made and
// sorted per structure by one CTA (stable block radix sort in shared memory),
// one launch instead of the device-wide sort's several.  Keys never cross
// structures, so the result equals the device-wide stable sort of k_morton's
// keys element for element.  Two sizes: 256 x 8 keys (structures of at most
// 2048 atoms) and 512 x 16 (8192).
constexpr int kSegSortMax = 8192, kSegSortSmall = 2048;

template <int THREADS, int ITEMS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_morton_segsort(const BuildDesc* descs,
                                                                          const uint8_t* culled,
                                                                          uint64_t* keys_out, int32_t* vals_out) {
    using SegSort = cub::BlockRadixSort<uint32_t, THREADS, ITEMS, int32_t>;
    static_assert(sizeof(typename SegSort::TempStorage) <= 48 * 1024, "segment sort storage fits static shared memory");
    __shared__ typename SegSort::TempStorage temp;
    const int s = blockIdx.x;
    const BuildDesc& D = descs[s];
    const SceneHeader* H = reinterpret_cast<const SceneHeader*>(D.scene);
    const int n = D.n < THREADS * ITEMS ? (int)D.n : THREADS * ITEMS;     // the host sends no larger structure
    uint32_t key[ITEMS];
    int32_t val[ITEMS];
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const int i = threadIdx.x * ITEMS + k;              // blocked: item order = atom order
        val[k] = i;
        key[k] = i < n ? morton_key31(D, H, i, culled && D.exterior && culled[D.atom0 + i]) : 0xffffffffu;
    }
    SegSort(temp).Sort(key, val, 0, 32);
#pragma unroll
    for (int k = 0; k < ITEMS; ++k) {
        const int j = threadIdx.x * ITEMS + k;
        if (j < n) {
            keys_out[D.atom0 + j] = ((uint64_t)s << 31) | key[k];
            vals_out[D.atom0 + j] = val[k];
        }
    }
}

// --------------------------------------------------------------------------
// Device-wide stable LSD radix sort of (uint64 key, int32 value) pairs, for
// batches with a structure above kSegSortMax atoms.  Each pass sorts by one
// 8-bit digit in three launches:
//   k_radix_count    per tile of kRadixTile keys: digit histogram, stored
//                    digit-major (counts[digit * tiles + tile]);
//   k_radix_scan     one CTA: exclusive scan of the counts in that order, so
//                    offsets[digit * tiles + tile] is where the tile's keys
//                    of that digit start in the output;
//   k_radix_scatter  per tile: the tile's pairs are sorted by the digit in
//                    shared memory (stable block radix sort of the blocked
//                    arrangement, which is input order), and each pair goes
//                    to its digit's offset plus its rank among the tile's
//                    pairs of that digit.
// Every pass is stable, so the result is the stable sort by the key's low
// end_bit bits, element for element what any stable sort gives.
// --------------------------------------------------------------------------
constexpr int kRadixThreads = 256, kRadixItems = 8, kRadixTile = kRadixThreads * kRadixItems, kRadixBins = 256;
static_assert(kRadixThreads == kRadixBins, "one thread per digit in the histogram steps");

__host__ __device__ inline int64_t radix_tiles(int64_t n) { return (n + kRadixTile - 1) / kRadixTile; }

__global__ void __launch_bounds__(kRadixThreads) k_radix_count(const uint64_t* keys, int64_t n, int shift,
                                                              uint32_t* counts, int64_t tiles) {
    __shared__ uint32_t h[kRadixBins];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kRadixTile;
#pragma unroll
    for (int k = 0; k < kRadixItems; ++k) {
        const int64_t i = base + k * kRadixThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(unsigned)(keys[i] >> shift) & (kRadixBins - 1)], 1u);
    }
    __syncthreads();
    counts[(int64_t)threadIdx.x * tiles + blockIdx.x] = h[threadIdx.x];
}

__global__ void __launch_bounds__(1024) k_radix_scan(const uint32_t* counts, uint32_t* offsets, int64_t m) {
    // the counts add up to the batch's atom count (< 2^31), so 32-bit sums suffice
    using Scan = cub::BlockScan<uint32_t, 1024>;
    __shared__ typename Scan::TempStorage tmp;
    const int64_t per = (m + 1023) / 1024;
    const int64_t b = threadIdx.x * per, e = b + per < m ? b + per : m;
    uint32_t sum = 0;
    for (int64_t i = b; i < e; ++i) sum += counts[i];
    uint32_t pre;
    Scan(tmp).ExclusiveSum(sum, pre);
    for (int64_t i = b; i < e; ++i) {
        const uint32_t c = counts[i];
        offsets[i] = pre;
        pre += c;
    }
}

__global__ void __launch_bounds__(kRadixThreads) k_radix_scatter(const uint64_t* keys_in, const int32_t* vals_in,
                                                                uint64_t* keys_out, int32_t* vals_out, int64_t n,
                                                                int shift, const uint32_t* counts,
                                                                const uint32_t* offsets, int64_t tiles) {
    using Sort = cub::BlockRadixSort<uint64_t, kRadixThreads, kRadixItems, int32_t>;
    using Scan = cub::BlockScan<uint32_t, kRadixThreads>;
    __shared__ union {
        typename Sort::TempStorage sort;
        typename Scan::TempStorage scan;
    } tmp;
    __shared__ uint32_t start[kRadixBins], dest[kRadixBins];
    const int64_t base = (int64_t)blockIdx.x * kRadixTile;
    uint64_t key[kRadixItems];
    int32_t val[kRadixItems];
#pragma unroll
    for (int k = 0; k < kRadixItems; ++k) {
        const int64_t i = base + threadIdx.x * kRadixItems + k;     // blocked: item order = input order
        const bool in = i < n;
        key[k] = in ? keys_in[i] : ~0ull;                           // padding sorts behind every real key
        val[k] = in ? vals_in[i] : -1;
    }
    // where this tile's keys of each digit start, in the tile and in the output
    const int64_t slot = (int64_t)threadIdx.x * tiles + blockIdx.x;
    uint32_t first;
    Scan(tmp.scan).ExclusiveSum(counts[slot], first);
    start[threadIdx.x] = first;
    dest[threadIdx.x] = offsets[slot];
    __syncthreads();
    Sort(tmp.sort).Sort(key, val, shift, shift + 8 < 64 ? shift + 8 : 64);
#pragma unroll
    for (int k = 0; k < kRadixItems; ++k) {
        if (val[k] < 0) continue;                                   // padding (last tile only)
        const unsigned d = (unsigned)(key[k] >> shift) & (kRadixBins - 1);
        const uint32_t pos = threadIdx.x * kRadixItems + k;           // rank in the sorted tile
        const int64_t o = (int64_t)dest[d] + (pos - start[d]);
        keys_out[o] = key[k];
        vals_out[o] = val[k];
    }
}

// Passes of the device-wide sort over bits [0, end_bit).
__host__ __device__ inline int radix_passes(int end_bit) { return (end_bit + 7) / 8; }

// Sorts n pairs; the input must be in (keys_a, vals_a) when the pass count is
// odd and in (keys_b, vals_b) when it is even, so that the result always
// lands in (keys_b, vals_b).
static int radix_sort_pairs(uint64_t* keys_a, int32_t* vals_a, uint64_t* keys_b, int32_t* vals_b, int64_t n,
                            int end_bit, uint32_t* counts, uint32_t* offsets, cudaStream_t stream) {
    const int64_t tiles = radix_tiles(n);
    const int passes = radix_passes(end_bit);
    uint64_t* kin = passes % 2 ? keys_a : keys_b;
    int32_t* vin = passes % 2 ? vals_a : vals_b;
    uint64_t* kout = passes % 2 ? keys_b : keys_a;
    int32_t* vout = passes % 2 ? vals_b : vals_a;
    for (int p = 0; p < passes; ++p) {
        const int shift = 8 * p;
        k_radix_count<<<(unsigned)tiles, kRadixThreads, 0, stream>>>(kin, n, shift, counts, tiles);
        k_radix_scan<<<1, 1024, 0, stream>>>(counts, offsets, (int64_t)kRadixBins * tiles);
        k_radix_scatter<<<(unsigned)tiles, kRadixThreads, 0, stream>>>(kin, vin, kout, vout, n, shift, counts,
                                                                        offsets, tiles);
        uint64_t* tk = kin; kin = kout; kout = tk;
        int32_t* tv = vin; vin = vout; vout = tv;
    }
    return cuda_status(cudaGetLastError(), "LBVH key sort");
}

// Karras (2012), "Maximizing parallelism in the construction of BVHs,
// octrees, and k-d trees": internal node i of a segment of n sorted keys.
__device__ __forceinline__ int delta(const uint64_t* k, int64_t base, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint64_t a = k[base + i], b = k[base + j];
    if (a == b) return 64 + __clz((uint32_t)(i ^ j));
    return __clzll(a ^ b);
}

__global__ void k_karras(const BuildDesc* descs, int n_scenes, int64_t I_total, const uint64_t* keys,
                         int32_t* inner_child, int32_t* inner_range, int32_t* parent_inner, int32_t* parent_leaf) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= I_total) return;
    // structure owning inner node g: last s with inner0 <= g (binary search)
    int lo = 0, hi = n_scenes - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (descs[mid].inner0 <= g) lo = mid; else hi = mid - 1;
    }
    const BuildDesc& D = descs[lo];
    int n = (int)D.n_active;
    int i = (int)(g - D.inner0);
    if (i >= n - 1) return;   // structures with one (active) atom own no internal node
    int64_t base = D.atom0;
    int d = (delta(keys, base, n, i, i + 1) - delta(keys, base, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(keys, base, n, i, i - d);
    int lmax = 2;
    while (delta(keys, base, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, base, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(keys, base, n, i, j);
    int s = 0;
    int span = l;
    for (int t = (span + 1) >> 1;; t = (t + 1) >> 1) {
        if (delta(keys, base, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
    }
    int gamma = i + s * d + (d < 0 ? d : 0);
    int first = i < j ? i : j, last = i < j ? j : i;
    int64_t gi = D.inner0 + i;
    inner_range[2 * gi] = first;
    inner_range[2 * gi + 1] = last;
    int left = (first == gamma) ? ~gamma : gamma;
    int right = (last == gamma + 1) ? ~(gamma + 1) : gamma + 1;
    inner_child[2 * gi] = left;
    inner_child[2 * gi + 1] = right;
    if (left < 0) parent_leaf[base + gamma] = i; else parent_inner[D.inner0 + left] = i;
    if (right < 0) parent_leaf[base + gamma + 1] = i; else parent_inner[D.inner0 + right] = i;
    if (i == 0) parent_inner[gi] = -1;
}

__device__ __forceinline__ void atom_box(const BuildDesc& D, const SceneHeader* H, int64_t atom, float* b) {
    double r = D.radii[atom];
    for (int c = 0; c < 3; ++c) {
        double rel = D.xyz[atom * 3 + c] - H->center[c];
        b[c] = __double2float_rd(rel - r);
        b[3 + c] = __double2float_ru(rel + r);
    }
}

__global__ void k_refit(const BuildDesc* descs, const int32_t* atom_scene, int64_t N, const int32_t* vals_sorted,
                        const int32_t* inner_child, const int32_t* parent_inner, const int32_t* parent_leaf,
                        float* inner_box, float* leaf_box, int32_t* inner_height, uint32_t* arrivals) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= N) return;
    const BuildDesc& D = descs[atom_scene[g]];
    const SceneHeader* H = reinterpret_cast<const SceneHeader*>(D.scene);
    float b[6];
    atom_box(D, H, vals_sorted[g], b);
    for (int k = 0; k < 6; ++k) leaf_box[6 * g + k] = b[k];
    if (D.n_active == 1 || g - D.atom0 >= D.n_active) return;    // no tree above, or a buried atom
    int node = parent_leaf[g];
    __threadfence();
    // a walk longer than any LBVH depth (Morton bits + duplicate bits) means a malformed link
    for (int hops = 0; node >= 0 && node < D.n_active - 1 && hops < 128; ++hops) {
        int64_t gi = D.inner0 + node;
        if (atomicAdd(&arrivals[gi], 1u) == 0) return;   // the sibling subtree is not finished yet
        __threadfence();
        float u[6] = {CUDART_INF_F, CUDART_INF_F, CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F};
        int h = 0;
        for (int side = 0; side < 2; ++side) {
            int c = inner_child[2 * gi + side];
            const float* src;
            int hc;
            if (c < 0 ? (~c >= D.n_active) : (c >= D.n_active - 1)) return;   // malformed link: leave the node unset
            if (c < 0) { src = leaf_box + 6 * (D.atom0 + ~c); hc = 0; }
            else { src = inner_box + 6 * (D.inner0 + c); hc = __ldcg(inner_height + D.inner0 + c); }
            for (int k = 0; k < 3; ++k) {
                u[k] = fminf(u[k], __ldcg(src + k));
                u[3 + k] = fmaxf(u[3 + k], __ldcg(src + 3 + k));
            }
            h = max(h, hc);
        }
        for (int k = 0; k < 6; ++k) inner_box[6 * gi + k] = u[k];
        inner_height[gi] = h + 1;
        __threadfence();
        node = parent_inner[gi];
    }
}

// 4-wide node record i (see ehss_internal.cuh) from up to four child slots.
__device__ __forceinline__ void write_node4(float4* nodes, int64_t i, const float (*box)[6], const int* ref, int n,
                                            float eps) {
    float v[6][4];
    int r[4];
    for (int c = 0; c < 4; ++c) {
        bool used = c < n;
        for (int k = 0; k < 3; ++k) {
            // lo and hi rounded outward; an unused slot's box is empty (lo = +inf, hi = -inf)
            v[2 * k][c] = used ? __fsub_rd(box[c][k], eps) : CUDART_INF_F;
            v[2 * k + 1][c] = used ? __fadd_ru(box[c][3 + k], eps) : -CUDART_INF_F;
        }
        r[c] = used ? ref[c] : kEmptyChild;
    }
    float4* nd = nodes + 8 * i;
    for (int f = 0; f < 6; ++f) nd[f] = make_float4(v[f][0], v[f][1], v[f][2], v[f][3]);
    nd[6] = make_float4(__int_as_float(r[0]), __int_as_float(r[1]), __int_as_float(r[2]), __int_as_float(r[3]));
    nd[7] = make_float4(0.f, 0.f, 0.f, 0.f);
}

__global__ void k_emit_nodes(const BuildDesc* descs, int n_scenes, int64_t I_total, const int32_t* inner_child,
                             const int32_t* inner_range, const float* inner_box, const float* leaf_box,
                             const int32_t* inner_height) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    // one extra thread per structure handles the single-leaf case (n <= leaf_size)
    if (g >= I_total + n_scenes) return;
    if (g >= I_total) {
        const BuildDesc& D = descs[g - I_total];
        SceneHeader* H = reinterpret_cast<SceneHeader*>(D.scene);
        H->n_active = (int32_t)D.n_active;
        H->exterior = D.exterior;
        if (D.n_active > D.leaf_size) {
            H->depth = inner_height[D.inner0];
            H->n_nodes = (int32_t)(D.n_active - 1);
            return;
        }
        // whole structure in one leaf below a single node
        float4* nodes = reinterpret_cast<float4*>(D.scene + H->off_nodes);
        float u[1][6] = {{CUDART_INF_F, CUDART_INF_F, CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F}};
        for (int64_t a = 0; a < D.n_active; ++a)
            for (int k = 0; k < 3; ++k) {
                u[0][k] = fminf(u[0][k], leaf_box[6 * (D.atom0 + a) + k]);
                u[0][3 + k] = fmaxf(u[0][3 + k], leaf_box[6 * (D.atom0 + a) + 3 + k]);
            }
        int ref = ~((0 << kLeafBits) | (int)(D.n_active - 1));
        write_node4(nodes, 0, u, &ref, 1, H->eps_box);
        H->depth = 1;
        H->n_nodes = 1;
        return;
    }
    int lo = 0, hi = n_scenes - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (descs[mid].inner0 <= g) lo = mid; else hi = mid - 1;
    }
    const BuildDesc& D = descs[lo];
    int i = (int)(g - D.inner0);
    if (i >= D.n_active - 1 || D.n_active <= D.leaf_size) return;
    SceneHeader* H = reinterpret_cast<SceneHeader*>(D.scene);
    float4* nodes = reinterpret_cast<float4*>(D.scene + H->off_nodes);
    // slot of a binary child: leaf reference when it is an atom or a subtree
    // of at most leaf_size atoms, else the node index (expanded once more)
    auto classify = [&](int c, int& ref, const float*& box) -> bool {   // true: expandable internal node
        if (c < 0) {
            box = leaf_box + 6 * (D.atom0 + ~c);
            ref = ~((~c) << kLeafBits);
            return false;
        }
        box = inner_box + 6 * (D.inner0 + c);
        int first = inner_range[2 * (D.inner0 + c)], last = inner_range[2 * (D.inner0 + c) + 1];
        int count = last - first + 1;
        if (count <= D.leaf_size) { ref = ~((first << kLeafBits) | (count - 1)); return false; }
        ref = c;
        return true;
    };
    int refs[4];
    float boxes[4][6];
    int n = 0;
    for (int side = 0; side < 2; ++side) {
        int c = inner_child[2 * g + side];
        int ref;
        const float* box;
        if (!classify(c, ref, box)) {
            refs[n] = ref;
            for (int k = 0; k < 6; ++k) boxes[n][k] = box[k];
            ++n;
            continue;
        }
        for (int side2 = 0; side2 < 2; ++side2) {          // grandchildren
            int gc = inner_child[2 * (D.inner0 + c) + side2];
            int ref2;
            const float* box2;
            classify(gc, ref2, box2);
            refs[n] = ref2;
            for (int k = 0; k < 6; ++k) boxes[n][k] = box2[k];
            ++n;
        }
    }
    write_node4(nodes, i, boxes, refs, n, H->eps_box);
}

__global__ void k_emit_atoms(const BuildDesc* descs, const int32_t* atom_scene, int64_t N, const int32_t* vals_sorted) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= N) return;
    const BuildDesc& D = descs[atom_scene[g]];
    SceneHeader* H = reinterpret_cast<SceneHeader*>(D.scene);
    int64_t j = g - D.atom0;               // leaf-order position
    int64_t a = vals_sorted[g];            // input atom id
    float4* atoms = reinterpret_cast<float4*>(D.scene + H->off_atoms);
    double4* atoms64 = reinterpret_cast<double4*>(D.scene + H->off_atoms64);
    int32_t* ids = reinterpret_cast<int32_t*>(D.scene + H->off_ids);
    int32_t* rank = reinterpret_cast<int32_t*>(D.scene + H->off_rank);
    double x = D.xyz[a * 3], y = D.xyz[a * 3 + 1], z = D.xyz[a * 3 + 2], r = D.radii[a];
    atoms[j] = make_float4(__double2float_rn(x - H->center[0]), __double2float_rn(y - H->center[1]),
                           __double2float_rn(z - H->center[2]), __double2float_rn(r));
    atoms64[j] = make_double4(x, y, z, r);
    ids[j] = (int32_t)a;
    rank[a] = (int32_t)j;
}

__global__ void k_fill_scene_index(const BuildDesc* descs, int n_scenes, int32_t* atom_scene) {
    int s = blockIdx.x;
    if (s >= n_scenes) return;
    const BuildDesc& D = descs[s];
    for (int64_t i = threadIdx.x; i < D.n; i += blockDim.x) atom_scene[D.atom0 + i] = s;
}

// --------------------------------------------------------------------------
// Refit: new coordinates for a full scene, tree topology kept (the reference's
// SphereIndex.refit / _refit, pa_spatial.py:78-95, 166-170).  k_stats (refit
// mode) rewrites the header from the new coordinates; then
//   k_refit_atoms   per leaf-order slot: FP32/FP64 records of the atom it
//                   holds (ids unchanged) and its outward-rounded box
//   k_node_links    per 4-wide node: parent link of each node child, count
//                   of node children
//   k_refit_nodes   per 4-wide node without node children: child boxes from
//                   the atom boxes, then up the parent links; the last child
//                   to finish a node (atomic arrival count) fits the node
// A node child's slot box is the union of that node's slot boxes before the
// eps_box expansion, i.e. the union of all its atoms' boxes, which is exactly
// the box a build with this topology computes.  Node indices of structure s
// start at descs[s].inner0 (sum of max(n - 1, 1) over the structures before).
// --------------------------------------------------------------------------
__device__ __forceinline__ bool refit_live(const BuildDesc& D) {
    const SceneHeader* H = reinterpret_cast<const SceneHeader*>(D.scene);
    return D.refit && H->status == 0;
}

__global__ void k_refit_atoms(const BuildDesc* descs, const int32_t* atom_scene, int64_t N, float* leaf_box) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= N) return;
    const BuildDesc& D = descs[atom_scene[g]];
    if (!refit_live(D)) return;
    SceneHeader* H = reinterpret_cast<SceneHeader*>(D.scene);
    const int64_t j = g - D.atom0;
    const int32_t* ids = reinterpret_cast<const int32_t*>(D.scene + H->off_ids);
    const int64_t a = ids[j];
    if (a < 0 || a >= D.n) { H->status = kStatusCorrupt; return; }
    float4* atoms = reinterpret_cast<float4*>(D.scene + H->off_atoms);
    double4* atoms64 = reinterpret_cast<double4*>(D.scene + H->off_atoms64);
    double x = D.xyz[a * 3], y = D.xyz[a * 3 + 1], z = D.xyz[a * 3 + 2], r = D.radii[a];
    atoms[j] = make_float4(__double2float_rn(x - H->center[0]), __double2float_rn(y - H->center[1]),
                           __double2float_rn(z - H->center[2]), __double2float_rn(r));
    atoms64[j] = make_double4(x, y, z, r);
    float b[6];
    atom_box(D, H, a, b);
    for (int k = 0; k < 6; ++k) leaf_box[6 * g + k] = b[k];
}

// Structure owning global node index g (last s with inner0 <= g).
__device__ __forceinline__ int node_owner(const BuildDesc* descs, int n_scenes, int64_t g) {
    int lo = 0, hi = n_scenes - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (descs[mid].inner0 <= g) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__global__ void k_node_links(const BuildDesc* descs, int n_scenes, int64_t nodes_total, int32_t* parent,
                             int32_t* node_children) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= nodes_total) return;
    const BuildDesc& D = descs[node_owner(descs, n_scenes, g)];
    if (!refit_live(D)) return;
    SceneHeader* H = reinterpret_cast<SceneHeader*>(D.scene);
    const int i = (int)(g - D.inner0), n_nodes = H->n_nodes;
    if (i >= n_nodes) return;
    const float4 rf = reinterpret_cast<const float4*>(D.scene + H->off_nodes)[8 * (int64_t)i + 6];
    const int ref[4] = {__float_as_int(rf.x), __float_as_int(rf.y), __float_as_int(rf.z), __float_as_int(rf.w)};
    int count = 0;
    for (int c = 0; c < 4; ++c) {
        if (ref[c] == kEmptyChild) break;                  // used slots form a prefix
        if (ref[c] < 0) continue;                          // leaf slot
        if (ref[c] == i || ref[c] >= n_nodes) { H->status = kStatusCorrupt; return; }
        parent[D.inner0 + ref[c]] = i;
        ++count;
    }
    node_children[g] = count;
}

__global__ void k_refit_nodes(const BuildDesc* descs, int n_scenes, int64_t nodes_total, const int32_t* parent,
                              const int32_t* node_children, const float* leaf_box, float* node_box,
                              uint32_t* arrivals) {
    int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (g >= nodes_total) return;
    const BuildDesc& D = descs[node_owner(descs, n_scenes, g)];
    if (!refit_live(D)) return;
    SceneHeader* H = reinterpret_cast<SceneHeader*>(D.scene);
    const int n_nodes = H->n_nodes;
    int node = (int)(g - D.inner0);
    if (node >= n_nodes || node_children[g] != 0) return;   // walks start at nodes whose slots are all leaves
    float4* nodes = reinterpret_cast<float4*>(D.scene + H->off_nodes);
    const float eps = H->eps_box;
    // a walk longer than any tree depth means a malformed link
    for (int hops = 0; hops < 128; ++hops) {
        const int64_t gi = D.inner0 + node;
        const float4 rf = nodes[8 * (int64_t)node + 6];
        int ref[4] = {__float_as_int(rf.x), __float_as_int(rf.y), __float_as_int(rf.z), __float_as_int(rf.w)};
        float box[4][6];
        float u[6] = {CUDART_INF_F, CUDART_INF_F, CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F};
        int used = 0;
        for (int c = 0; c < 4; ++c) {
            if (ref[c] == kEmptyChild) break;              // used slots form a prefix
            float b[6] = {CUDART_INF_F, CUDART_INF_F, CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F, -CUDART_INF_F};
            if (ref[c] < 0) {
                const int code = ~ref[c];
                const int first = code >> kLeafBits, cnt = (code & (kMaxLeaf - 1)) + 1;
                if (first + cnt > D.n) { H->status = kStatusCorrupt; return; }
                for (int a = first; a < first + cnt; ++a)
                    for (int k = 0; k < 3; ++k) {
                        b[k] = fminf(b[k], leaf_box[6 * (D.atom0 + a) + k]);
                        b[3 + k] = fmaxf(b[3 + k], leaf_box[6 * (D.atom0 + a) + 3 + k]);
                    }
            } else {
                if (ref[c] >= n_nodes) { H->status = kStatusCorrupt; return; }
                const float* src = node_box + 6 * (D.inner0 + ref[c]);
                for (int k = 0; k < 6; ++k) b[k] = __ldcg(src + k);
            }
            for (int k = 0; k < 6; ++k) box[c][k] = b[k];
            for (int k = 0; k < 3; ++k) { u[k] = fminf(u[k], b[k]); u[3 + k] = fmaxf(u[3 + k], b[3 + k]); }
            ++used;
        }
        if (used == 0) { H->status = kStatusCorrupt; return; }
        write_node4(nodes, node, box, ref, used, eps);
        for (int k = 0; k < 6; ++k) node_box[6 * gi + k] = u[k];
        __threadfence();
        const int up = parent[gi];
        if (up < 0) return;                                // the root, or a node no record references
        const int64_t gu = D.inner0 + up;
        if (atomicAdd(&arrivals[gu], 1u) + 1u < (uint32_t)node_children[gu]) return;   // siblings still running
        __threadfence();
        node = up;
    }
    H->status = kStatusCorrupt;
}

// --------------------------------------------------------------------------
// Exterior scenes: atoms that no ray starting outside the union can reach.
//
// A sphere B whose every surface point lies inside some other sphere at depth
// >= m > 0 is never the nearest entry of a ray that starts outside the union
// of the spheres or on its boundary (the impact disk and every bounce point
// of the EHSS path): to reach B's surface the ray must cross the surface of
// a covering sphere C at least m earlier, so C wins the (distance, id)
// comparison strictly; and such a ray hits some other sphere whenever it hits
// B, so any-hit results keep too.  Buried spheres are left out of the tree of
// an exterior scene; outcomes are unchanged.
//
// Test (one warp per atom B, radius r).  Each neighbour C overlapping B gives
// a cap on B's unit sphere, {s : |r s - (c_C - c_B)| <= r_C - h - mu}, i.e.
// s.u_C >= cos(alpha_C) with u_C the unit direction to C.  The samples are
// the vertices of the geodesic (icosahedral) spheres of 162, 642 and 2562
// vertices (levels A, B, C; each level's vertices start with the previous
// level's).  Their covering radii rho_L -- the largest distance from a point
// of the sphere to the nearest vertex, computed on the host from the
// triangulation (the circumradius of each triangle, or half its longest
// edge when the circumcentre falls outside) -- bound every surface point's
// chord distance to its nearest level-L sample by r rho_L.  A sample of level
// L is "covered" when it lies in some cap with h = r rho_L: every surface
// point within rho_L of it is then inside C at depth >= mu.  B is buried when
// every surface point is certified that way:
//   level A: every vertex is tested; the uncovered ones are kept open.
//   level B, C: only the vertices within rho_prev + rho_L of an open vertex
//            of the previous level are tested (every point within rho_prev
//            of that vertex has its nearest level-L vertex among them, from
//            host-made neighbour lists); the uncovered ones become the open
//            vertices.  None open: buried.
// More than kMaxOpen open vertices, or any left at level C, keep the atom.
// mu = 1e-4 (r + d + r_C) + 2e-6 S bounds the FP32 error of the cap test (at
// most 1e-5 (r + d + r_C) for the caps used, whose shrunk radius is >= 0.05
// (r + d + r_C)), of the FP32 atom records and of the FP32 vertex directions
// ten times over.  Dropping a neighbour, or declaring an atom exposed, only
// keeps atoms, so the fixed-size lists below never make a wrong cut.
// --------------------------------------------------------------------------
constexpr int kIcoA = 162, kIcoB = 642, kIcoC = 2562;
constexpr int kIcoNbr = 24;            // neighbour list width (at most 17 used: checked on the host)
constexpr int kExposureWarps = 8;
constexpr int kMaxCaps = 96;
constexpr int kFrontier = 64;
constexpr int kLeafList = 64;
constexpr int kMaxOpen = 8;
constexpr int kMaskWords = (kIcoC + 31) / 32;
constexpr int kCandList = 256;         // distinct candidate vertices of one refinement level

// geodesic sphere vertices (levels A, B, C are prefixes), level A -> B and
// B -> C neighbour lists, covering radii (uploaded by build_scenes)
__device__ float4 g_ico_dirs[kIcoC];
__device__ uint16_t g_ico_nbr[(kIcoA + kIcoB) * kIcoNbr];
__device__ uint8_t g_ico_nnbr[kIcoA + kIcoB];
__device__ float g_ico_rho[3];

struct ExposureWarp {
    float4 cap[kMaxCaps];              // (u, cos alpha at the current lattice)
    float2 dr[kMaxCaps];               // (distance, radius of C)
    int front[2][kFrontier];
    int leaves[kLeafList];
    int open[2][kMaxOpen];             // open vertices of the last two levels
    unsigned mask[kMaskWords];         // candidate vertices of the current refinement level
    int cand[kCandList];
    int n_front[2];
    int n_leaves, n_caps, whole;
};

__device__ __forceinline__ float cap_cos(float r, float d, float rc_full, float h, float mS) {
    const float L = r + d + rc_full;
    const float rc = rc_full - h - 1e-4f * L - mS;     // shrunk radius of C
    if (rc < 0.05f * L || d >= r + rc) return 3.f;    // too thin to count, or no cap
    return (r * r + d * d - rc * rc) / (2.f * r * d);
}

// Caps for lattice spacing h; true when one cap alone holds the whole sphere.
__device__ __forceinline__ bool set_caps(ExposureWarp& W, int nc, float r, float h, float mS, int lane) {
    bool whole = false;
    for (int i = lane; i < nc; i += 32) {
        const float2 dr = W.dr[i];
        const float c = cap_cos(r, dr.x, dr.y, h, mS);
        W.cap[i].w = c;
        whole = whole || c <= -1.f;
    }
    __syncwarp();
    return __any_sync(0xffffffffu, whole);
}

__device__ __forceinline__ bool in_some_cap(const ExposureWarp& W, int nc, float sx, float sy, float sz) {
    int c = 0;
    for (; c + 4 <= nc; c += 4) {          // four caps per step: their loads overlap
        const float4 u0 = W.cap[c], u1 = W.cap[c + 1], u2 = W.cap[c + 2], u3 = W.cap[c + 3];
        const bool h = (sx * u0.x + sy * u0.y + sz * u0.z >= u0.w) | (sx * u1.x + sy * u1.y + sz * u1.z >= u1.w) |
                       (sx * u2.x + sy * u2.y + sz * u2.z >= u2.w) | (sx * u3.x + sy * u3.y + sz * u3.z >= u3.w);
        if (h) return true;
    }
    for (; c < nc; ++c) {
        const float4 u = W.cap[c];
        if (sx * u.x + sy * u.y + sz * u.z >= u.w) return true;
    }
    return false;
}

__global__ void __launch_bounds__(32 * kExposureWarps, 4) k_exposure(BuildDesc* descs, const int32_t* atom_scene,
                                                                  int64_t N, uint8_t* culled) {
    __shared__ float4 dirs_a[kIcoA];
    __shared__ ExposureWarp wsm[kExposureWarps];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu, below = (1u << lane) - 1u;
    for (int t = threadIdx.x; t < kIcoA; t += blockDim.x) dirs_a[t] = g_ico_dirs[t];
    __syncthreads();
    const float rho_a = g_ico_rho[0], rho_b = g_ico_rho[1], rho_c = g_ico_rho[2];
    ExposureWarp& W = wsm[warp];
    for (int64_t g = blockIdx.x * (int64_t)kExposureWarps + warp; g < N; g += (int64_t)gridDim.x * kExposureWarps) {
        BuildDesc& D = descs[atom_scene[g]];
        const SceneView S = scene_view(D.scene);
        const int j = (int)(g - D.atom0);          // leaf-order position: neighbouring warps share subtrees
        const float4 b = S.atoms[j];
        const float mS = 2e-6f * S.h->scale_f;
        const float h_fine = b.w * rho_c;
        if (lane == 0) {
            W.front[0][0] = 0;
            W.n_front[0] = 1;
            W.n_leaves = W.n_caps = W.whole = 0;
        }
        __syncwarp();
        // 1. leaves whose boxes meet B's box (breadth first, one node per lane)
        const float lo[3] = {b.x - b.w, b.y - b.w, b.z - b.w}, hi[3] = {b.x + b.w, b.y + b.w, b.z + b.w};
        const int n_nodes = S.h->n_nodes;
        int cur = 0;
        for (int level = 0; level < 64; ++level) {
            const int nf = min(W.n_front[cur], kFrontier);
            __syncwarp();
            if (nf == 0) break;
            if (lane == 0) W.n_front[cur ^ 1] = 0;
            __syncwarp();
            for (int k = lane; k < nf; k += 32) {
                const int node = W.front[cur][k];
                if (node < 0 || node >= n_nodes) continue;       // malformed: drop (keeps atoms)
                const float4* nd = S.nodes + 8 * (int64_t)node;
                const float4 lx = nd[0], hx = nd[1], ly = nd[2], hy = nd[3], lz = nd[4], hz = nd[5], rf = nd[6];
                const float cl[3][4] = {{lx.x, lx.y, lx.z, lx.w}, {ly.x, ly.y, ly.z, ly.w}, {lz.x, lz.y, lz.z, lz.w}};
                const float ch[3][4] = {{hx.x, hx.y, hx.z, hx.w}, {hy.x, hy.y, hy.z, hy.w}, {hz.x, hz.y, hz.z, hz.w}};
                const int refs[4] = {__float_as_int(rf.x), __float_as_int(rf.y), __float_as_int(rf.z),
                                     __float_as_int(rf.w)};
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    if (refs[c] == kEmptyChild) continue;
                    bool hit = true;
#pragma unroll
                    for (int a = 0; a < 3; ++a) hit = hit && cl[a][c] <= hi[a] && ch[a][c] >= lo[a];
                    if (!hit) continue;
                    if (refs[c] >= 0) {
                        int slot = atomicAdd(&W.n_front[cur ^ 1], 1);
                        if (slot < kFrontier) W.front[cur ^ 1][slot] = refs[c];
                    } else {
                        int slot = atomicAdd(&W.n_leaves, 1);
                        if (slot < kLeafList) W.leaves[slot] = refs[c];
                    }
                }
            }
            __syncwarp();
            cur ^= 1;
        }
        // 2. neighbours with a cap on the finest lattice: the atoms of all listed leaves, one per lane
        const int nl = min(W.n_leaves, kLeafList);
        int* leaf_end = W.front[0];                 // free after the walk: running atom counts of the leaves
        int n_cand = 0;
        for (int base = 0; base < nl; base += 32) {
            const int l = base + lane;
            const int c = l < nl ? ((~W.leaves[l]) & (kMaxLeaf - 1)) + 1 : 0;
            int incl = c;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int v = __shfl_up_sync(full, incl, o);
                if (lane >= o) incl += v;
            }
            if (l < nl) leaf_end[l] = n_cand + incl;
            n_cand += __shfl_sync(full, incl, 31);
        }
        __syncwarp();
        for (int t = lane; t < n_cand; t += 32) {
            int lo_l = 0, hi_l = nl - 1;                // leaf of candidate t: first with leaf_end > t
            while (lo_l < hi_l) {
                const int mid = (lo_l + hi_l) >> 1;
                if (leaf_end[mid] > t) hi_l = mid; else lo_l = mid + 1;
            }
            const int k = ((~W.leaves[lo_l]) >> kLeafBits) + t - (lo_l ? leaf_end[lo_l - 1] : 0);
            if (k >= S.h->n_atoms || k == j) continue;
            const float4 a = S.atoms[k];
            const float dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
            const float d = sqrtf(dx * dx + dy * dy + dz * dz);
            if (d + b.w <= a.w - 1e-4f * (b.w + d + a.w) - mS) { W.whole = 1; continue; }   // C alone holds B
            const float key = cap_cos(b.w, d, a.w, h_fine, mS);
            if (!(key < 1.f)) continue;
            if (key <= -1.f) { W.whole = 1; continue; }
            const int slot = atomicAdd(&W.n_caps, 1);
            if (slot < kMaxCaps) {
                W.cap[slot] = make_float4(dx / d, dy / d, dz / d, key);
                W.dr[slot] = make_float2(d, a.w);
            }
        }
        __syncwarp();
        const int nc = min(W.n_caps, kMaxCaps);
        bool buried = W.whole != 0;
        // caps wider than a hemisphere first: most samples then stop at the first few
        if (!buried && nc > 32) {
            float4 mc[3];
            float2 md[3];
            bool big[3];
            int n_big = 0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int i = lane + 32 * q;
                big[q] = false;
                if (i < nc) { mc[q] = W.cap[i]; md[q] = W.dr[i]; big[q] = mc[q].w < 0.f; }
                n_big += __popc(__ballot_sync(full, big[q]));
            }
            __syncwarp();
            int before_big = 0, before_small = 0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
                const int i = lane + 32 * q;
                const unsigned mb = __ballot_sync(full, big[q]), ms = __ballot_sync(full, i < nc && !big[q]);
                if (i < nc) {
                    const int at = big[q] ? before_big + __popc(mb & below) : n_big + before_small + __popc(ms & below);
                    W.cap[at] = mc[q];
                    W.dr[at] = md[q];
                }
                before_big += __popc(mb);
                before_small += __popc(ms);
            }
            __syncwarp();
        }
        bool exposed = nc == 0 && !buried;
        // 3a. level A: every vertex; the uncovered ones stay open
        int n_open = 0;
        if (!buried && !exposed) {
            buried = set_caps(W, nc, b.w, b.w * rho_a, mS, lane);
            for (int base = 0; base < kIcoA && !buried && !exposed; base += 32) {
                const int t = base + lane;
                bool miss = false;
                if (t < kIcoA) {
                    const float4 s = dirs_a[t];
                    miss = !in_some_cap(W, nc, s.x, s.y, s.z);
                }
                const unsigned m = __ballot_sync(full, miss);
                const int at = n_open + __popc(m & below);
                if (miss && at < kMaxOpen) W.open[0][at] = t;
                n_open += __popc(m);
                exposed = n_open > kMaxOpen;
            }
            __syncwarp();
            if (!buried && !exposed && n_open == 0) buried = true;
        }
        // 3b. levels B and C: the distinct neighbours of the open vertices, each tested once
        int side = 0;
        for (int lv = 1; lv <= 2 && !buried && !exposed; ++lv) {
            const int n_lv = lv == 1 ? kIcoB : kIcoC, words = (n_lv + 31) >> 5;
            const int nbr0 = lv == 1 ? 0 : kIcoA;           // neighbour lists of the previous level's vertices
            if (set_caps(W, nc, b.w, b.w * (lv == 1 ? rho_b : rho_c), mS, lane)) { buried = true; break; }
            for (int w = lane; w < words; w += 32) W.mask[w] = 0u;
            __syncwarp();
            for (int u = 0; u < n_open; ++u) {
                const int v = W.open[side][u];
                const int cnt = g_ico_nnbr[nbr0 + v];
                if (lane < cnt) {
                    const int idx = g_ico_nbr[(nbr0 + v) * kIcoNbr + lane];
                    atomicOr(&W.mask[idx >> 5], 1u << (idx & 31));
                }
            }
            __syncwarp();
            // compact the marked vertices into W.cand, in index order
            int total = 0;
            for (int wb = 0; wb < words; wb += 32) {
                const int w = wb + lane;
                unsigned bits = w < words ? W.mask[w] : 0u;
                const int c = __popc(bits);
                int incl = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int v = __shfl_up_sync(full, incl, o);
                    if (lane >= o) incl += v;
                }
                int at = total + incl - c;
                while (bits) {
                    const int bit = __ffs(bits) - 1;
                    bits &= bits - 1;
                    if (at < kCandList) W.cand[at] = (w << 5) + bit;
                    ++at;
                }
                total += __shfl_sync(full, incl, 31);
            }
            __syncwarp();
            if (total > kCandList) { exposed = true; break; }   // too many to test: keep the atom
            int n_next = 0;
            for (int base = 0; base < total && !exposed; base += 32) {
                const int t = base + lane;
                bool miss = false;
                int id = 0;
                if (t < total) {
                    id = W.cand[t];
                    const float4 s = g_ico_dirs[id];
                    miss = !in_some_cap(W, nc, s.x, s.y, s.z);
                }
                const unsigned m = __ballot_sync(full, miss);
                const int at = n_next + __popc(m & below);
                if (miss && at < kMaxOpen) W.open[side ^ 1][at] = id;
                n_next += __popc(m);
                exposed = n_next > kMaxOpen;
            }
            __syncwarp();
            if (exposed) break;
            if (n_next == 0) buried = true;
            else if (lv == 2) exposed = true;
            n_open = n_next;
            side ^= 1;
        }
        if (lane == 0) {
            culled[D.atom0 + S.ids[j]] = buried ? 1 : 0;
            if (buried) atomicAdd(reinterpret_cast<unsigned long long*>(&D.n_active), ~0ull);   // -1
        }
        __syncwarp();
    }
}

// A structure whose atoms all tested buried (impossible for a bounded union:
// its boundary lies on some exposed sphere) falls back to the full tree.
__global__ void k_finish_exposure(BuildDesc* descs, int n_scenes) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_scenes) return;
    if (descs[s].n_active < 1) { descs[s].n_active = descs[s].n; descs[s].exterior = 0; }
}

// --------------------------------------------------------------------------
// Host side
// --------------------------------------------------------------------------
namespace {

// Geodesic spheres of the exposure test: the icosahedron subdivided 2, 3 and 4
// times (162, 642, 2562 vertices; each level's vertices come first in the
// next), their covering radii and the level A -> B, B -> C neighbour lists.
struct IcoTables {
    float4 dirs[kIcoC];
    uint16_t nbr[(kIcoA + kIcoB) * kIcoNbr];
    uint8_t nnbr[kIcoA + kIcoB];
    float rho[3];
    bool ok = false;
};

using Vec3 = std::array<double, 3>;
Vec3 sub3(const Vec3& a, const Vec3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
double dot3(const Vec3& a, const Vec3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
Vec3 cross3(const Vec3& a, const Vec3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
Vec3 unit3(const Vec3& a) { double n = std::sqrt(dot3(a, a)); return {a[0] / n, a[1] / n, a[2] / n}; }
double angle3(const Vec3& a, const Vec3& b) { return std::acos(std::max(-1.0, std::min(1.0, dot3(a, b)))); }

// Largest distance from a point of the sphere to the nearest vertex: over the
// triangles, the circumradius when the circumcentre lies in the triangle,
// else half the longest edge.
double covering_radius(const std::vector<Vec3>& v, const std::vector<std::array<int, 3>>& faces) {
    double worst = 0.;
    for (const auto& f : faces) {
        const Vec3 &A = v[f[0]], &B = v[f[1]], &C = v[f[2]];
        Vec3 n = unit3(cross3(sub3(B, A), sub3(C, A)));
        if (dot3(n, A) < 0) n = {-n[0], -n[1], -n[2]};
        const bool inside = dot3(cross3(A, B), n) >= -1e-15 && dot3(cross3(B, C), n) >= -1e-15 &&
                            dot3(cross3(C, A), n) >= -1e-15;
        double r = inside ? angle3(n, A)
                          : 0.5 * std::max(angle3(A, B), std::max(angle3(B, C), angle3(C, A)));
        worst = std::max(worst, r);
    }
    return worst + 1e-9;
}

const IcoTables& ico_tables() {
    static IcoTables T;
    static std::once_flag once;
    std::call_once(once, [] {
        const double t = (1. + std::sqrt(5.)) / 2.;
        const double base[12][3] = {{-1, t, 0}, {1, t, 0}, {-1, -t, 0}, {1, -t, 0}, {0, -1, t}, {0, 1, t},
                                    {0, -1, -t}, {0, 1, -t}, {t, 0, -1}, {t, 0, 1}, {-t, 0, -1}, {-t, 0, 1}};
        std::vector<Vec3> v;
        for (const auto& p : base) v.push_back(unit3({p[0], p[1], p[2]}));
        std::vector<std::array<int, 3>> f = {{0, 11, 5}, {0, 5, 1}, {0, 1, 7}, {0, 7, 10}, {0, 10, 11}, {1, 5, 9},
                                             {5, 11, 4}, {11, 10, 2}, {10, 7, 6}, {7, 1, 8}, {3, 9, 4}, {3, 4, 2},
                                             {3, 2, 6}, {3, 6, 8}, {3, 8, 9}, {4, 9, 5}, {2, 4, 11}, {6, 2, 10},
                                             {8, 6, 7}, {9, 8, 1}};
        double rho[3];
        for (int level = 1; level <= 4; ++level) {
            std::map<std::pair<int, int>, int> mid;
            auto midpoint = [&](int a, int b) {
                auto key = std::make_pair(std::min(a, b), std::max(a, b));
                auto it = mid.find(key);
                if (it != mid.end()) return it->second;
                const Vec3 m = {v[a][0] + v[b][0], v[a][1] + v[b][1], v[a][2] + v[b][2]};
                v.push_back(unit3(m));
                mid[key] = (int)v.size() - 1;
                return (int)v.size() - 1;
            };
            std::vector<std::array<int, 3>> next;
            for (const auto& q : f) {
                const int ab = midpoint(q[0], q[1]), bc = midpoint(q[1], q[2]), ca = midpoint(q[2], q[0]);
                next.push_back({q[0], ab, ca});
                next.push_back({q[1], bc, ab});
                next.push_back({q[2], ca, bc});
                next.push_back({ab, bc, ca});
            }
            f.swap(next);
            if (level >= 2) rho[level - 2] = covering_radius(v, f);
        }
        if ((int)v.size() != kIcoC) return;
        for (int i = 0; i < kIcoC; ++i)
            T.dirs[i] = make_float4((float)v[i][0], (float)v[i][1], (float)v[i][2], 0.f);
        for (int l = 0; l < 3; ++l) {
            float r = (float)rho[l];
            if ((double)r < rho[l]) r = std::nextafter(r, 1.f);
            T.rho[l] = r;
        }
        // level A -> B, B -> C: vertices of the finer level within rho_coarse + rho_fine
        for (int lv = 0; lv < 2; ++lv) {
            const int n_from = lv == 0 ? kIcoA : kIcoB, n_to = lv == 0 ? kIcoB : kIcoC, off = lv == 0 ? 0 : kIcoA;
            const double lim = std::cos(rho[lv] + rho[lv + 1] + 1e-6);
            for (int u = 0; u < n_from; ++u) {
                int c = 0;
                for (int w = 0; w < n_to; ++w) {
                    if (dot3(v[u], v[w]) < lim) continue;
                    if (c == kIcoNbr) return;                    // table too narrow: T.ok stays false
                    T.nbr[(off + u) * kIcoNbr + c++] = (uint16_t)w;
                }
                T.nnbr[off + u] = (uint8_t)c;
            }
        }
        T.ok = true;
    });
    return T;
}

// Once per device and process: a copy from pageable memory waits for the
// stream to drain, which in the middle of a build would leave the GPU idle
// while the host issues the rest of the build.  The first upload completes
// before any build proceeds, so builds on other streams see the tables.
int upload_ico_tables(cudaStream_t stream) {
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static bool uploaded[kMaxDevices] = {};
    int dev = -1;
    int rc = cuda_status(cudaGetDevice(&dev), "exposure table upload");
    if (rc) return rc;
    std::lock_guard<std::mutex> lock(mu);
    if (dev >= 0 && dev < kMaxDevices && uploaded[dev]) return EHSS_OK;
    const IcoTables& T = ico_tables();
    if (!T.ok) { set_error("exposure test tables could not be made"); return EHSS_ERR_VALUE; }
    rc = cuda_status(cudaMemcpyToSymbolAsync(g_ico_dirs, T.dirs, sizeof(T.dirs), 0, cudaMemcpyHostToDevice, stream),
                     "exposure table upload");
    if (!rc) rc = cuda_status(cudaMemcpyToSymbolAsync(g_ico_nbr, T.nbr, sizeof(T.nbr), 0, cudaMemcpyHostToDevice, stream),
                              "exposure table upload");
    if (!rc) rc = cuda_status(cudaMemcpyToSymbolAsync(g_ico_nnbr, T.nnbr, sizeof(T.nnbr), 0, cudaMemcpyHostToDevice,
                                                      stream), "exposure table upload");
    if (!rc) rc = cuda_status(cudaMemcpyToSymbolAsync(g_ico_rho, T.rho, sizeof(T.rho), 0, cudaMemcpyHostToDevice, stream),
                              "exposure table upload");
    if (!rc) rc = cuda_status(cudaStreamSynchronize(stream), "exposure table upload");
    if (!rc && dev >= 0 && dev < kMaxDevices) uploaded[dev] = true;
    return rc;
}

}  // namespace
// Workspace for a batch with N atoms over S structures.
uint64_t build_workspace_bytes(int64_t N, int S) {
    int64_t I = N > 0 ? N : 1;
    uint64_t b = 0;
    b += align256(sizeof(BuildDesc) * (uint64_t)S);
    b += align256(4ull * N);            // atom_scene
    b += 2 * align256(8ull * N);        // keys
    b += 2 * align256(4ull * N);        // vals
    b += align256(8ull * I);            // inner_child
    b += align256(8ull * I);            // inner_range
    b += align256(4ull * I);            // parent_inner
    b += align256(4ull * N);            // parent_leaf
    b += align256(24ull * I);           // inner_box
    b += align256(24ull * N);           // leaf_box
    b += align256(4ull * I);            // inner_height
    b += align256(4ull * I);            // arrivals
    b += align256(1ull * N);            // culled
    b += 2 * align256(4ull * kRadixBins * (uint64_t)radix_tiles(N));   // radix counts, offsets
    return b + 256;
}

int build_scenes(int S, const double* const* xyz, const double* const* radii, const int64_t* n, int leaf_size,
                 void* const* scenes, const uint64_t* scene_bytes, void* workspace, uint64_t workspace_bytes,
                 cudaStream_t stream, bool exterior) {
    if (S < 1) { set_error("at least one structure required"); return EHSS_ERR_VALUE; }
    if (leaf_size < 1 || leaf_size > kMaxLeaf) { set_error("leaf_size must be 1..%d", kMaxLeaf); return EHSS_ERR_VALUE; }
    int64_t N = 0, I = 0, max_n = 0;
    BuildDesc* host = new BuildDesc[S];
    for (int s = 0; s < S; ++s) {
        if (n[s] < 1 || n[s] > (1 << 27)) {
            delete[] host;
            set_error("structure %d: atom count %lld outside 1..2^27", s, (long long)n[s]);
            return EHSS_ERR_VALUE;
        }
        uint64_t on, oa, o64, oi, orr, total;
        scene_layout(n[s], &on, &oa, &o64, &oi, &orr, &total);
        if (scene_bytes[s] < total) {
            delete[] host;
            set_error("structure %d: scene buffer holds %llu bytes, %llu required", s,
                      (unsigned long long)scene_bytes[s], (unsigned long long)total);
            return EHSS_ERR_CAPACITY;
        }
        if (((uintptr_t)scenes[s] & 255u) != 0) {
            delete[] host;
            set_error("structure %d: scene buffer must be 256-byte aligned", s);
            return EHSS_ERR_VALUE;
        }
        BuildDesc& D = host[s];
        D.xyz = xyz[s]; D.radii = radii[s]; D.scene = (char*)scenes[s];
        D.n = n[s]; D.atom0 = N; D.inner0 = I; D.leaf_size = leaf_size; D.exterior = exterior ? 1 : 0;
        D.n_active = n[s];
        D.refit = 0; D.pad = 0;
        if (n[s] > max_n) max_n = n[s];
        N += n[s];
        I += n[s] - 1;
    }
    if (N > (int64_t)INT32_MAX) {          // the key sort counts items in int
        delete[] host;
        set_error("a batch holds at most %d atoms, got %lld", INT32_MAX, (long long)N);
        return EHSS_ERR_VALUE;
    }
    uint64_t need = build_workspace_bytes(N, S);
    if (workspace_bytes < need) {
        delete[] host;
        set_error("build workspace holds %llu bytes, %llu required", (unsigned long long)workspace_bytes,
                  (unsigned long long)need);
        return EHSS_ERR_CAPACITY;
    }
    char* p = (char*)(((uintptr_t)workspace + 255u) & ~(uintptr_t)255u);
    BuildWork W;
    int64_t Ia = I > 0 ? I : 1;
    W.descs = (BuildDesc*)p; p += align256(sizeof(BuildDesc) * (uint64_t)S);
    W.atom_scene = (int32_t*)p; p += align256(4ull * N);
    W.keys_in = (uint64_t*)p; p += align256(8ull * N);
    W.keys_out = (uint64_t*)p; p += align256(8ull * N);
    W.vals_in = (int32_t*)p; p += align256(4ull * N);
    W.vals_out = (int32_t*)p; p += align256(4ull * N);
    W.inner_child = (int32_t*)p; p += align256(8ull * Ia);
    W.inner_range = (int32_t*)p; p += align256(8ull * Ia);
    W.parent_inner = (int32_t*)p; p += align256(4ull * Ia);
    W.parent_leaf = (int32_t*)p; p += align256(4ull * N);
    W.inner_box = (float*)p; p += align256(24ull * Ia);
    W.leaf_box = (float*)p; p += align256(24ull * N);
    W.inner_height = (int32_t*)p; p += align256(4ull * Ia);
    W.arrivals = (uint32_t*)p; p += align256(4ull * Ia);
    W.culled = (uint8_t*)p; p += align256(1ull * N);
    W.radix_counts = (uint32_t*)p; p += align256(4ull * kRadixBins * (uint64_t)radix_tiles(N));
    W.radix_offsets = (uint32_t*)p;

    // The headers are written on the device (k_stats); the descriptors are the
    // only upload.  A copy from pageable host memory has staged its source
    // when the call returns, so the host descriptors may go now.
    int rc = cuda_status(cudaMemcpyAsync(W.descs, host, sizeof(BuildDesc) * S, cudaMemcpyHostToDevice, stream),
                         "build descriptor upload");
    delete[] host;
    if (rc) return rc;

    const int T = 256;
    auto blocks = [&](int64_t count) { return (unsigned)((count + T - 1) / T); };
    k_fill_scene_index<<<S, 256, 0, stream>>>(W.descs, S, W.atom_scene);
    k_stats<<<S, 256, 0, stream>>>(W.descs, S);
    int end_bit = 31;
    while ((1ll << (end_bit - 31)) < S) ++end_bit;
    const bool segsort = max_n <= kSegSortMax;
    // one pass: Morton keys -> sort -> Karras hierarchy -> refit -> node and atom records
    auto tree_pass = [&](const uint8_t* culled) -> int {
        int r;
        if (segsort) {
            if (max_n <= kSegSortSmall)
                k_morton_segsort<256, 8><<<S, 256, 0, stream>>>(W.descs, culled, W.keys_out, W.vals_out);
            else
                k_morton_segsort<512, 16><<<S, 512, 0, stream>>>(W.descs, culled, W.keys_out, W.vals_out);
            r = cuda_status(cudaGetLastError(), "LBVH key sort");
        } else {
            // the keys start in the buffer from which an odd or even number of passes ends in keys_out
            const bool odd = radix_passes(end_bit) % 2 != 0;
            k_morton<<<blocks(N), T, 0, stream>>>(W.descs, W.atom_scene, N, culled, odd ? W.keys_in : W.keys_out,
                                                  odd ? W.vals_in : W.vals_out);
            r = radix_sort_pairs(W.keys_in, W.vals_in, W.keys_out, W.vals_out, N, end_bit, W.radix_counts,
                                 W.radix_offsets, stream);
        }
        if (r) return r;
        // parent links start at -1 so that a missing link ends a refit walk
        r = cuda_status(cudaMemsetAsync(W.parent_leaf, 0xff, 4ull * N, stream), "LBVH parent reset");
        if (r) return r;
        if (I > 0) {
            r = cuda_status(cudaMemsetAsync(W.arrivals, 0, 4ull * I, stream), "LBVH arrival reset");
            if (!r) r = cuda_status(cudaMemsetAsync(W.parent_inner, 0xff, 4ull * I, stream), "LBVH parent reset");
            if (r) return r;
            k_karras<<<blocks(I), T, 0, stream>>>(W.descs, S, I, W.keys_out, W.inner_child, W.inner_range,
                                                  W.parent_inner, W.parent_leaf);
        }
        k_refit<<<blocks(N), T, 0, stream>>>(W.descs, W.atom_scene, N, W.vals_out, W.inner_child, W.parent_inner,
                                             W.parent_leaf, W.inner_box, W.leaf_box, W.inner_height, W.arrivals);
        k_emit_nodes<<<blocks(I + S), T, 0, stream>>>(W.descs, S, I, W.inner_child, W.inner_range, W.inner_box,
                                                      W.leaf_box, W.inner_height);
        k_emit_atoms<<<blocks(N), T, 0, stream>>>(W.descs, W.atom_scene, N, W.vals_out);
        return cuda_status(cudaGetLastError(), "LBVH build launch");
    };
    rc = tree_pass(nullptr);
    if (rc || !exterior) return rc;
    // exterior scenes: mark buried atoms with the full tree, then rebuild over the exposed ones
    rc = upload_ico_tables(stream);
    if (rc) return rc;
    {
        int64_t want = (N + kExposureWarps - 1) / kExposureWarps;
        static const int per_sm = [] {
            int b = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_exposure, 32 * kExposureWarps, 0) != cudaSuccess || b < 1)
                b = 1;
            return b;
        }();
        int64_t cap = (int64_t)per_sm * sm_count();
        unsigned grid = (unsigned)(want < cap ? want : cap);
        k_exposure<<<grid, 32 * kExposureWarps, 0, stream>>>(W.descs, W.atom_scene, N, W.culled);
    }
    k_finish_exposure<<<(S + 127) / 128, 128, 0, stream>>>(W.descs, S);
    rc = cuda_status(cudaGetLastError(), "exposure launch");
    if (rc) return rc;
    return tree_pass(W.culled);
}

int refit_scenes(int S, const double* const* xyz, const double* const* radii, const int64_t* n, void* const* scenes,
                 void* workspace, uint64_t workspace_bytes, cudaStream_t stream) {
    if (S < 1) { set_error("at least one structure required"); return EHSS_ERR_VALUE; }
    int64_t N = 0, nodes_total = 0;
    std::vector<BuildDesc> host(S);
    for (int s = 0; s < S; ++s) {
        if (n[s] < 1 || n[s] > (1 << 27)) {
            set_error("structure %d: atom count %lld outside 1..2^27", s, (long long)n[s]);
            return EHSS_ERR_VALUE;
        }
        if (((uintptr_t)scenes[s] & 255u) != 0) {
            set_error("structure %d: scene buffer must be 256-byte aligned", s);
            return EHSS_ERR_VALUE;
        }
        BuildDesc& D = host[s];
        std::memset(&D, 0, sizeof(D));
        D.xyz = xyz[s]; D.radii = radii[s]; D.scene = (char*)scenes[s];
        D.n = n[s]; D.atom0 = N; D.inner0 = nodes_total; D.n_active = n[s];
        D.refit = 1;
        N += n[s];
        nodes_total += n[s] > 1 ? n[s] - 1 : 1;        // node records of a full scene (ehss_scene_bytes layout)
    }
    if (N > (int64_t)INT32_MAX) {
        set_error("a batch holds at most %d atoms, got %lld", INT32_MAX, (long long)N);
        return EHSS_ERR_VALUE;
    }
    uint64_t need = build_workspace_bytes(N, S);
    if (workspace_bytes < need) {
        set_error("refit workspace holds %llu bytes, %llu required", (unsigned long long)workspace_bytes,
                  (unsigned long long)need);
        return EHSS_ERR_CAPACITY;
    }
    // the build workspace's regions, reused: nodes_total <= N, so the per-node arrays fit the inner-node ones
    char* p = (char*)(((uintptr_t)workspace + 255u) & ~(uintptr_t)255u);
    const int64_t Ia = N > 0 ? N : 1;
    BuildDesc* descs = (BuildDesc*)p; p += align256(sizeof(BuildDesc) * (uint64_t)S);
    int32_t* atom_scene = (int32_t*)p; p += align256(4ull * N);
    p += 2 * align256(8ull * N) + 2 * align256(4ull * N);           // keys, vals (unused)
    int32_t* node_children = (int32_t*)p; p += align256(8ull * Ia);
    p += align256(8ull * Ia);                                       // inner_range (unused)
    int32_t* parent = (int32_t*)p; p += align256(4ull * Ia);
    p += align256(4ull * N);                                        // parent_leaf (unused)
    float* node_box = (float*)p; p += align256(24ull * Ia);
    float* leaf_box = (float*)p; p += align256(24ull * N);
    p += align256(4ull * Ia);                                       // inner_height (unused)
    uint32_t* arrivals = (uint32_t*)p;

    int rc = cuda_status(cudaMemcpyAsync(descs, host.data(), sizeof(BuildDesc) * S, cudaMemcpyHostToDevice, stream),
                         "refit descriptor upload");
    if (!rc) rc = cuda_status(cudaMemsetAsync(parent, 0xff, 4ull * nodes_total, stream), "refit parent reset");
    if (!rc) rc = cuda_status(cudaMemsetAsync(node_children, 0, 4ull * nodes_total, stream), "refit link reset");
    if (!rc) rc = cuda_status(cudaMemsetAsync(arrivals, 0, 4ull * nodes_total, stream), "refit arrival reset");
    if (rc) return rc;
    const int T = 256;
    auto blocks = [&](int64_t count) { return (unsigned)((count + T - 1) / T); };
    k_fill_scene_index<<<S, 256, 0, stream>>>(descs, S, atom_scene);
    k_stats<<<S, 256, 0, stream>>>(descs, S);
    k_refit_atoms<<<blocks(N), T, 0, stream>>>(descs, atom_scene, N, leaf_box);
    k_node_links<<<blocks(nodes_total), T, 0, stream>>>(descs, S, nodes_total, parent, node_children);
    k_refit_nodes<<<blocks(nodes_total), T, 0, stream>>>(descs, S, nodes_total, parent, node_children, leaf_box,
                                                         node_box, arrivals);
    return cuda_status(cudaGetLastError(), "refit launch");
}

}  // namespace ehss
