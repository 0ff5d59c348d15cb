// Internal declarations shared by the ehss_b200 CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include <cstdint>
#include <cfloat>
#include <cstddef>
#include "../../include/ehss_b200.h"

namespace ehss {

// ---------------------------------------------------------------------------
// Scene buffer layout (one structure, device resident, 256-byte aligned).
//
//   SceneHeader                              256 B
//   nodes   float4[8 * n_nodes]              4-wide nodes (below), child boxes in FP32
//   atoms   float4[n]      (x, y, z, r)      FP32, centre relative to header.center,
//                                            in leaf order
//   atoms64 double4[n]     (x, y, z, r)      FP64 reference values, leaf order
//   ids     int32[n]       leaf order -> input atom id
//   rank    int32[n]       input atom id -> leaf order
//
// Node record (128 B, eight float4): a 4-wide node, structure of arrays over
// its children c = 0..3:
//   f[0] = lo.x[c]  f[1] = hi.x[c]  f[2] = lo.y[c]  f[3] = hi.y[c]
//   f[4] = lo.z[c]  f[5] = hi.z[c]  f[6] = child ref[c] (int bits)  f[7] = unused
// child >= 0: node index; child < 0: leaf ~(first << kLeafBits | (count - 1));
// kEmptyChild marks an unused slot, whose box is empty: lo = +inf, hi = -inf.  Node i is built from binary LBVH node i
// with its grandchildren as children (children that are leaves, or subtrees
// of at most leaf_size atoms, stay single slots), so only binary nodes at
// even depth are ever referenced.
// ---------------------------------------------------------------------------
constexpr uint32_t kSceneMagic = 0x45485353u;  // "EHSS"
constexpr int kLeafBits = 4;                 // leaf reference: atom count - 1 in the low bits
constexpr int kMaxLeaf = 1 << kLeafBits;
constexpr int kEmptyChild = INT32_MIN;
constexpr int kStackDepth = 96;   // >= 3 x the deepest 4-wide tree (binary LBVH height <= 55)
constexpr int kMaxWorkParts = 512;
// Fixed point of the angle sums: a ray adds at most 2 * 2^36, so a block of up
// to 2^26 rays sums below 2^63 (ehss_blocks_prepare enforces the bound).
constexpr double kFxScale = 0x1p36;
constexpr int kMaxBlockLog2 = 26;    // per-SM work ranges of the persistent kernel (workspace 4 KiB)

struct alignas(256) SceneHeader {
    uint32_t magic;
    int32_t status;        // 0 ok; nonzero: build failure code
    int32_t n_atoms;
    int32_t n_nodes;
    int32_t leaf_size;
    int32_t depth;
    double center[3];
    double radius;         // impact-disk radius R = max(|c - center| + r) * (1 + 1e-9)
    double scale;          // S = max(|c - center| + r)
    double rmax;
    float eps_box;         // absolute FP32 box expansion
    float scale_f;
    float rmax_f;
    float pad0;
    int32_t n_active;      // atoms in the tree: all of them, or the exposed ones of an exterior scene
    int32_t exterior;      // 1: buried atoms left out of the tree (valid for rays starting outside)
    uint64_t off_nodes, off_atoms, off_atoms64, off_ids, off_rank;
    uint64_t bytes;
};
static_assert(sizeof(SceneHeader) == 256, "scene header is one 256-byte line");
static_assert(sizeof(ehss_residual) == 88 && offsetof(ehss_residual, block) == 72, "residual ray record layout");
static_assert(sizeof(ehss_block) == 560 && offsetof(ehss_block, basis) == 0 && offsetof(ehss_block, base) == 480,
              "block descriptors are read with 16-byte vector loads");

struct SceneView {
    const SceneHeader* h;
    const float4* nodes;
    const float4* atoms;
    const double4* atoms64;
    const int32_t* ids;
    const int32_t* rank;
};

__host__ __device__ inline uint64_t align256(uint64_t x) { return (x + 255u) & ~uint64_t(255); }

__host__ __device__ inline void scene_layout(int64_t n, uint64_t* off_nodes, uint64_t* off_atoms, uint64_t* off_atoms64,
                         uint64_t* off_ids, uint64_t* off_rank, uint64_t* total) {
    int64_t nodes = n > 1 ? n - 1 : 1;
    uint64_t o = 256;
    *off_nodes = o; o = align256(o + (uint64_t)nodes * 128);
    *off_atoms = o; o = align256(o + (uint64_t)n * 16);
    *off_atoms64 = o; o = align256(o + (uint64_t)n * 32);
    *off_ids = o; o = align256(o + (uint64_t)n * 4);
    *off_rank = o; o = align256(o + (uint64_t)n * 4);
    *total = o;
}

__device__ inline SceneView scene_view(const void* p) {
    SceneView v;
    const char* b = reinterpret_cast<const char*>(p);
    v.h = reinterpret_cast<const SceneHeader*>(b);
    v.nodes = reinterpret_cast<const float4*>(b + v.h->off_nodes);
    v.atoms = reinterpret_cast<const float4*>(b + v.h->off_atoms);
    v.atoms64 = reinterpret_cast<const double4*>(b + v.h->off_atoms64);
    v.ids = reinterpret_cast<const int32_t*>(b + v.h->off_ids);
    v.rank = reinterpret_cast<const int32_t*>(b + v.h->off_rank);
    return v;
}

// ---------------------------------------------------------------------------
// FP64 arithmetic in the reference's exact operation order.  Every operation
// is an explicitly rounded intrinsic so that no multiply-add is contracted:
// the reference runs Numba without fastmath and g++ without FMA, so its
// products and sums are each rounded once.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ double dsqrt(double a) { return __dsqrt_rn(a); }
__device__ __forceinline__ double dmax0(double a) { return a > 0. ? a : 0.; }

// entry_scalar (src/support_exchange_transport/ehss_cpu.py:12-24) ==
// entry_distance (ehss_reference.py:8-23) == entry (src/native/ehss_cpu.cpp:7-17).
__device__ __forceinline__ double entry64(double o0, double o1, double o2, double d0, double d1, double d2,
                                          double c0, double c1, double c2, double radius) {
    double x0 = dsub(o0, c0), x1 = dsub(o1, c1), x2 = dsub(o2, c2);
    double aa = dadd(dadd(dmul(d0, d0), dmul(d1, d1)), dmul(d2, d2));
    double projection = ddiv(dadd(dadd(dmul(x0, d0), dmul(x1, d1)), dmul(x2, d2)), aa);
    double p0 = dsub(x0, dmul(projection, d0));
    double p1 = dsub(x1, dmul(projection, d1));
    double p2 = dsub(x2, dmul(projection, d2));
    double disc = dsub(dmul(radius, radius), dadd(dadd(dmul(p0, p0), dmul(p1, p1)), dmul(p2, p2)));
    if (disc < 0. || projection >= 0.) return CUDART_INF;
    double near_ = dsub(-projection, dsqrt(ddiv(dmax0(disc), aa)));
    if (near_ < dmul(-64.0 * DBL_EPSILON, radius)) return CUDART_INF;
    return dmax0(near_);
}

// sphere_hit (inside_out_pa.py:93-101).
__device__ __forceinline__ bool sphere_hit64(double o0, double o1, double o2, double d0, double d1, double d2,
                                             double c0, double c1, double c2, double r) {
    double x = dsub(o0, c0), y = dsub(o1, c1), z = dsub(o2, c2);
    double b = dadd(dadd(dmul(x, d0), dmul(y, d1)), dmul(z, d2));
    double cc = dsub(dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z)), dmul(r, r));
    double disc = dsub(dmul(b, b), cc);
    return disc >= 0 && dadd(-b, dsqrt(dmax0(disc))) > 0;
}

// reflect_scalar (ehss_cpu.py:27-40) == reflect (src/native/ehss_cpu.cpp:31-40).
__device__ __forceinline__ void reflect64(double& o0, double& o1, double& o2, double& d0, double& d1, double& d2,
                                          double c0, double c1, double c2, double r, double distance) {
    double n0 = dsub(dadd(o0, dmul(distance, d0)), c0);
    double n1 = dsub(dadd(o1, dmul(distance, d1)), c1);
    double n2 = dsub(dadd(o2, dmul(distance, d2)), c2);
    double norm = dsqrt(dadd(dadd(dmul(n0, n0), dmul(n1, n1)), dmul(n2, n2)));
    n0 = ddiv(n0, norm); n1 = ddiv(n1, norm); n2 = ddiv(n2, norm);
    o0 = dadd(c0, dmul(r, n0)); o1 = dadd(c1, dmul(r, n1)); o2 = dadd(c2, dmul(r, n2));
    double dot = dadd(dadd(dmul(d0, n0), dmul(d1, n1)), dmul(d2, n2));
    double two_dot = dmul(2.0, dot);
    d0 = dsub(d0, dmul(two_dot, n0)); d1 = dsub(d1, dmul(two_dot, n1)); d2 = dsub(d2, dmul(two_dot, n2));
    norm = dsqrt(dadd(dadd(dmul(d0, d0), dmul(d1, d1)), dmul(d2, d2)));
    d0 = ddiv(d0, norm); d1 = ddiv(d1, norm); d2 = ddiv(d2, norm);
}

// clip(1 - incoming . outgoing, 0, 2) of EHSSResult.contributions
// (ehss_state.py:84-87); numpy sums the three products left to right.
__device__ __forceinline__ double scatter_angle(double i0, double i1, double i2, double o0, double o1, double o2) {
    double dot = dadd(dadd(dmul(i0, o0), dmul(i1, o1)), dmul(i2, o2));
    double a = dsub(1.0, dot);
    return a < 0. ? 0. : (a > 2. ? 2. : a);
}

// ---------------------------------------------------------------------------
// Sobol on the device: point n of a (shift, sv[bit][dim]) scramble.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 sobol4(const uint4* sv, uint4 shift, uint32_t n) {
    uint32_t g = n ^ (n >> 1);
    uint4 q = shift;
    while (g) {
        int k = __ffs(g) - 1;
        g &= g - 1;
        uint4 v = sv[k];
        q.x ^= v.x; q.y ^= v.y; q.z ^= v.z; q.w ^= v.w;
    }
    return q;
}

// Scrambles passed by value as kernel parameters.
struct SobolParams { uint32_t sv[8 * 30]; uint32_t shift[8]; };   // [dim][bit]
struct Sobol4Params { uint4 sv[30]; uint4 shift; };               // [bit][dim]

struct Ray64 { double o[3], d[3]; };

// external_source mapping (ehss_state.py:45-52, inside_out_pa.py:45-58) of one
// Sobol point; center/radius are the scene's.  Transcendentals are CUDA's
// double cos/sin/sqrt (sqrt is correctly rounded; cos/sin within 2 ulp).
__device__ __forceinline__ Ray64 impact_ray(uint4 q, const double* center, double radius) {
    const double s = 0x1p-30;
    double u0 = q.x * s, u1 = q.y * s, u2 = q.z * s, u3 = q.w * s;
    const double two_pi = 2.0 * 3.141592653589793;
    double z = dsub(1.0, dmul(2.0, u0));
    double phi = dmul(two_pi, u1);
    double rho = dsqrt(dmax0(dsub(1.0, dmul(z, z))));
    double sp, cp;
    sincos(phi, &sp, &cp);
    double d0 = dmul(rho, cp), d1 = dmul(rho, sp), d2 = z;
    // tangent_frames: axis = e_z unless |d_z| > 0.9, then e_x; t = axis x d / |.|; b = d x t
    double a0 = 0., a1 = 0., a2 = 1.;
    if (fabs(d2) > .9) { a0 = 1.; a2 = 0.; }
    double t0 = dsub(dmul(a1, d2), dmul(a2, d1));
    double t1 = dsub(dmul(a2, d0), dmul(a0, d2));
    double t2 = dsub(dmul(a0, d1), dmul(a1, d0));
    double tn = dsqrt(dadd(dadd(dmul(t0, t0), dmul(t1, t1)), dmul(t2, t2)));
    t0 = ddiv(t0, tn); t1 = ddiv(t1, tn); t2 = ddiv(t2, tn);
    double b0 = dsub(dmul(d1, t2), dmul(d2, t1));
    double b1 = dsub(dmul(d2, t0), dmul(d0, t2));
    double b2 = dsub(dmul(d0, t1), dmul(d1, t0));
    double rr = dmul(radius, dsqrt(u2));
    double ps, pc;
    sincos(dmul(two_pi, u3), &ps, &pc);
    Ray64 ray;
    ray.o[0] = dadd(dsub(center[0], dmul(radius, d0)), dmul(rr, dadd(dmul(pc, t0), dmul(ps, b0))));
    ray.o[1] = dadd(dsub(center[1], dmul(radius, d1)), dmul(rr, dadd(dmul(pc, t1), dmul(ps, b1))));
    ray.o[2] = dadd(dsub(center[2], dmul(radius, d2)), dmul(rr, dadd(dmul(pc, t2), dmul(ps, b2))));
    ray.d[0] = d0; ray.d[1] = d1; ray.d[2] = d2;
    return ray;
}

// ---------------------------------------------------------------------------
// Host helpers
// ---------------------------------------------------------------------------
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);
bool sobol_scramble(int dim, uint64_t seed, uint32_t* sv, uint32_t* shift);
bool sobol_coherent_order(int m, const uint32_t* sv, const uint32_t* shift, uint32_t* basis, uint32_t* base);
void sobol_direction_numbers(int dim, uint32_t* v);
int sm_count();
void sobol4_params(uint64_t seed, Sobol4Params* p);
uint64_t build_workspace_bytes(int64_t N, int S);
int build_scenes(int S, const double* const* xyz, const double* const* radii, const int64_t* n, int leaf_size,
                 void* const* scenes, const uint64_t* scene_bytes, void* workspace, uint64_t workspace_bytes,
                 cudaStream_t stream, bool exterior = false);
int refit_scenes(int S, const double* const* xyz, const double* const* radii, const int64_t* n, void* const* scenes,
                 void* workspace, uint64_t workspace_bytes, cudaStream_t stream);
int launch_trace_rays(const void* scene, int64_t n, int cap, int precision, double* P, double* D,
                      const int64_t* last, int64_t* bounces, uint8_t* esc, uint8_t* unres, int32_t* hist,
                      uint64_t* stats, cudaStream_t stream);
int launch_pa_rays(const void* scene, int64_t n, const double* P, const double* D, const int64_t* owners,
                   uint8_t* blocked, uint64_t* stats, cudaStream_t stream);
int launch_sobol_points(int dim, const SobolParams& p, int64_t first, int64_t n, uint32_t* q, cudaStream_t stream);
int launch_source_rays(const void* scene, const Sobol4Params& p, int64_t first, int64_t n, double* O, double* D,
                       cudaStream_t stream);
uint64_t grid_workspace_bytes(int64_t n_atoms, int n_dirs, int n);
int launch_grid_pa(const void* scene, int64_t n_atoms, int n_dirs, uint64_t seed, int n, unsigned long long* counts,
                   double* spacing_out, double* xy_out, void* workspace, uint64_t ws_bytes, cudaStream_t stream);
int launch_compact_rays(const ehss_boundary& B, const SobolParams& p, int dim, int64_t first, int64_t n,
                        double inv_count, double* O, double* D, double* W, cudaStream_t stream);
int launch_extend(const ehss_block* blocks, int nb, const int32_t* row, int rows, const ehss_residual* in,
                  int64_t n_in, int new_cap, ehss_extension* ext, uint64_t* hist, uint64_t* ledger,
                  ehss_residual* out, int64_t out_capacity, unsigned long long* out_count, uint64_t* stats,
                  cudaStream_t stream);
int launch_blocks(const ehss_block* blocks, int nb, int64_t chunk_first, int64_t total_chunks, const ehss_launch& L,
                  ehss_block_result* results, uint64_t* hist, uint64_t* ledger, unsigned long long* work,
                  cudaStream_t stream, ehss_residual* residual = nullptr, int64_t residual_capacity = 0,
                  unsigned long long* residual_count = nullptr);

}  // namespace ehss
