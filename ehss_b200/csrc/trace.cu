// EHSS and PA kernels: nearest-entry query over the device LBVH, specular
// bounce loop, any-hit PA, and the fused Sobol -> trace -> reduction blocks.
//
// Reference behaviour restated (paths relative to the reference project):
//   nearest_scalar        src/support_exchange_transport/ehss_cpu.py:43-63
//   _trace_loop           ehss_cpu.py:66-100, src/native/ehss_cpu.cpp:54-78
//   entry_scalar/reflect  ehss_cpu.py:12-40 (see ehss_internal.cuh)
//   tree_blocked / _one   pa_spatial.py:114-142 with sphere_hit inside_out_pa.py:93-101
//   readout               ehss_state.py:84-103, ccs_cli.py:209-219
//
// Query design.  The reference walks a median-split tree in pre-order and
// keeps the lexicographic (distance, atom id) minimum of the FP64 entry
// distances.  Here the 4-wide LBVH is walked near-child-first with a
// per-thread stack; node boxes are FP32, rounded outward and expanded by eps_box, so a
// box is culled only when it provably holds no entry at or before the
// current bound U.  Two sphere-test precisions share the walk:
//   EXACT (EHSS_PREC_FP64): every reached sphere is tested with the
//     reference's FP64 formula; U is the running best distance rounded up.
//   FILTER (EHSS_PREC_FP32): spheres are tested in FP32 with the
//     cancellation-free perpendicular-distance discriminant
//     disc = r^2 - |v - (v.d) d|^2 (the fused kernel: the shorter
//     b^2 + (r^2 - |v|^2) under a widened bound) and a per-ray error bound
//     (Ep on projections, Edisc on the discriminant).  Certain misses are dropped;
//     certain hits give an interval [t - Et, t + Et] and lower U to t + Et;
//     every sphere whose lower bound is <= U (certain or near-tangent) is
//     kept in a 2-entry candidate list, re-tested in FP64 at the end with the
//     reference formula and the (distance, id) rule.  The reached candidates
//     always contain the FP64 winner, so outcomes equal EXACT's; a full list
//     re-runs the query in EXACT mode.
// Ray origins farther than 3 S from the structure centre (never produced by
// the impact-disk source) use an FP64 all-atom search instead.
#include <cstdio>
#include "ehss_internal.cuh"

namespace ehss {

constexpr float kU32 = 5.9604645e-08f;   // 2^-24
// Candidate slots per query.  A slot whose lower bound exceeds the current U is
// reused, so two slots overflow only when three spheres are within the error
// band of each other (89 of 124 M queries on the mixed 256-globule batch).  Each
// slot is two registers of the fused kernel, which runs at its 64-register
// bound: 2 slots trace that batch in 27.9 ms, 3 in 28.8, 4 in 29.7, while 1
// slot sends every grazing query to the FP64 re-run (1e5 fallbacks, 29.0 ms).
constexpr int kCand = 2;
constexpr int kSmemBins = 16;

struct LocalStats {
    uint32_t box, sphere, queries, grazing, fallback, fp64, errors;
    __device__ LocalStats() : box(0), sphere(0), queries(0), grazing(0), fallback(0), fp64(0), errors(0) {}
};

struct RayF {
    float ox, oy, oz, dx, dy, dz, ix, iy, iz, Ep, Edisc;
};

// Inverse direction component for the box tests, from the fast quotient
// (within 2 ulp for these arguments, whose magnitude lies in [1e-20, 1]).  A
// relative error e in inv moves a slab crossing along the ray by |t| e; with
// t below 6 S (origins within 3 S, boxes within S) that is under 1.5e-6 S
// even with the slab's own roundings, well inside the 2^-14 S (6.1e-5 S) by
// which every node box is widened, and the sign, which picks the near plane,
// is exact.
__device__ __forceinline__ float safe_rcp(float x) {
    float a = fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x;
    return __fdividef(1.0f, a);
}

// FP32 copy of an FP64 ray in the scene frame; false when the origin is too
// far from the centre for the FP32 error bounds (or not finite).  widen > 0
// adds widen * (rmax^2 + A^2) to the discriminant bound, for the fused
// kernel's shorter discriminant (kWidenShortDisc below).
__device__ __forceinline__ bool setup_ray(const SceneHeader* H, const double* o, const double* d, RayF& r,
                                          float widen = 0.0f) {
    r.ox = __double2float_rn(o[0] - H->center[0]);
    r.oy = __double2float_rn(o[1] - H->center[1]);
    r.oz = __double2float_rn(o[2] - H->center[2]);
    r.dx = __double2float_rn(d[0]); r.dy = __double2float_rn(d[1]); r.dz = __double2float_rn(d[2]);
    float S = H->scale_f;
    float a = sqrtf(fmaf(r.ox, r.ox, fmaf(r.oy, r.oy, r.oz * r.oz)));
    if (!(a <= 3.0f * S)) return false;
    r.ix = safe_rcp(r.dx); r.iy = safe_rcp(r.dy); r.iz = safe_rcp(r.dz);
    float A = a + S;
    r.Ep = A * (32.0f * kU32);
    float rm = H->rmax_f;
    r.Edisc = (8.0f * kU32) * rm * rm + 2.5f * rm * r.Ep + 8.0f * r.Ep * r.Ep;
    if (widen > 0.0f) r.Edisc += widen * (rm * rm + A * A);
    return true;
}

// The fused kernel's FILTER leaf test forms disc = b^2 + (r^2 - |v|^2)
// (two operations fewer, and a dependency chain three shorter, than
// r^2 - |v - b d|^2; v = c - o, b = v.d, both computed as in the
// cancellation-free form).  In exact arithmetic on the FP32 values the two
// differ by 2 b db + b^2 (|d|^2 - 1), db the rounding of b (<= 3u |v|) and
// | |d|^2 - 1 | <= 2.1u: at most 8.2u |v|^2.  Rounding r^2 - |v|^2 costs at
// most 4u (|v|^2 + r^2) and the last fma u |disc|; the cancellation-free
// value's own roundings, already inside Edisc, are at most 5.1u |v - b d|^2 +
// u |disc| again, and where a classification depends on them (true disc >= 0,
// or computed disc >= 2 Edisc) |v - b d|^2 <= rmax^2 + 2 Edisc.  With
// |v| <= |o| + S <= A (1 + 4u) the difference stays below 12.3u A^2 + 11.1u
// rmax^2, so adding 16u (rmax^2 + A^2) to Edisc keeps every certain miss,
// certain-hit interval and grazing lower bound as sound as before (u = 2^-24).
constexpr float kWidenShortDisc = 16.0f * kU32;

// sqrt(disc) of a certain hit (computed disc >= 2 Edisc) and the error bound Et
// of its entry and exit distances b -/+ sqrt(disc), from one reciprocal square
// root: s = disc * y and Edisc / s = Edisc * y.  rsqrtf is within 2 ulp of 1/sqrt(disc) (the CUDA
// math library's stated bound; at most 2.09 u measured over every float in
// [2^-14, 2^8)), so s is within 5.01 u of sqrt(disc) and Edisc * y within
// 5.01 u of Edisc / sqrt(disc).  With the roundings of s and of b -/+ s the
// distance error stays below Ep + Edisc / sqrt(disc) + 6.01 u (|b| + s), which Et
// covers with a factor-2 margin on its first two terms, as the correctly
// rounded square root and quotient did before (u = 2^-24).
__device__ __forceinline__ float certain_sqrt(float b, float disc, const RayF& r, float& Et) {
    const float y = rsqrtf(disc);
    const float s = disc * y;
    Et = 2.0f * (r.Ep + r.Edisc * y) + 8.0f * kU32 * (fabsf(b) + s);
    return s;
}

__device__ __forceinline__ float max3f(float a, float b, float c) {
    float d;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}
__device__ __forceinline__ float min3f(float a, float b, float c) {
    float d;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
    return d;
}

// Slab test of one child box against [0, U]; returns entry distance or +inf.
// The planes come as near (n*) and far (f*) per axis: with inv >= 0 the low
// plane is met first, and fma(lo, inv, -oi) <= fma(hi, inv, -oi) because
// rounding is monotone, so the near plane's distance is the slab minimum the
// textbook test forms with fminf, bit for bit.  An unused slot holds the box
// lo = +inf, hi = -inf, whose near distance is +inf on every axis, so it
// misses without a check of its reference.  oi = o * inv per axis, formed
// once per node visit (held per lane it would cost three registers of the
// fused kernel).
__device__ __forceinline__ float box_enter(const RayF& r, float oix, float oiy, float oiz, float nx, float fx, float ny,
                                           float fy, float nz, float fz, float U) {
    float tnx = fmaf(nx, r.ix, -oix), tfx = fmaf(fx, r.ix, -oix);
    float tny = fmaf(ny, r.iy, -oiy), tfy = fmaf(fy, r.iy, -oiy);
    float tnz = fmaf(nz, r.iz, -oiz), tfz = fmaf(fz, r.iz, -oiz);
    float tmin = max3f(tnx, tny, fmaxf(tnz, 0.0f));
    float tmax = min3f(tfx, tfy, fminf(tfz, U));
    return tmin <= tmax ? tmin : CUDART_INF_F;
}

// One 4-wide node: entry distances of the children that the ray meets within
// [0, U], sorted ascending (misses and empty slots last, at +inf).
struct Hits4 {
    int ref[4];
    float t[4];
    int n;
};

__device__ __forceinline__ void cswap(Hits4& h, int a, int b) {
    bool s = h.t[b] < h.t[a];
    float ta = s ? h.t[b] : h.t[a], tb = s ? h.t[a] : h.t[b];
    int ra = s ? h.ref[b] : h.ref[a], rb = s ? h.ref[a] : h.ref[b];
    h.t[a] = ta; h.t[b] = tb; h.ref[a] = ra; h.ref[b] = rb;
}

__device__ __forceinline__ Hits4 visit4(const float4* nodes, int node, const RayF& r, float U) {
    const float4* nd = nodes + 8 * (int64_t)node;
    // near and far plane rows by the direction's sign per axis (the node stores lo, hi)
    const int sx = __float_as_uint(r.ix) >> 31, sy = __float_as_uint(r.iy) >> 31, sz = __float_as_uint(r.iz) >> 31;
    float4 nx = __ldg(nd + sx), fx = __ldg(nd + (1 - sx)), ny = __ldg(nd + (2 + sy)), fy = __ldg(nd + (3 - sy));
    float4 nz = __ldg(nd + (4 + sz)), fz = __ldg(nd + (5 - sz)), rf = __ldg(nd + 6);
    Hits4 h;
    h.ref[0] = __float_as_int(rf.x); h.ref[1] = __float_as_int(rf.y);
    h.ref[2] = __float_as_int(rf.z); h.ref[3] = __float_as_int(rf.w);
    const float oix = r.ox * r.ix, oiy = r.oy * r.iy, oiz = r.oz * r.iz;
    h.t[0] = box_enter(r, oix, oiy, oiz, nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, U);
    h.t[1] = box_enter(r, oix, oiy, oiz, nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, U);
    h.t[2] = box_enter(r, oix, oiy, oiz, nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, U);
    h.t[3] = box_enter(r, oix, oiy, oiz, nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, U);
    cswap(h, 0, 1); cswap(h, 2, 3); cswap(h, 0, 2); cswap(h, 1, 3); cswap(h, 1, 2);
    h.n = (h.t[0] != CUDART_INF_F) + (h.t[1] != CUDART_INF_F) + (h.t[2] != CUDART_INF_F) + (h.t[3] != CUDART_INF_F);
    return h;
}

// Reference rule of nearest_scalar (ehss_cpu.py:60): strictly nearer, or
// equally near with a smaller input atom id.
__device__ __forceinline__ bool better(double dist, int id, double best, int best_id) {
    return dist < best || (dist == best && isfinite(dist) && (best_id < 0 || id < best_id));
}

// FP64 all-atom nearest search (origins far from the structure).
__device__ __noinline__ int nearest_flat(const SceneView& S, const double* o, const double* d, int last_rank, double& best_out,
                            LocalStats& st) {
    int n = S.h->n_atoms;
    double best = CUDART_INF;
    int best_rank = -1, best_id = -1;
    for (int k = 0; k < n; ++k) {
        if (k == last_rank) continue;
        double4 a = S.atoms64[k];
        double t = entry64(o[0], o[1], o[2], d[0], d[1], d[2], a.x, a.y, a.z, a.w);
        ++st.sphere; ++st.fp64;
        int id = S.ids[k];
        if (better(t, id, best, best_id)) { best = t; best_rank = k; best_id = id; }
    }
    best_out = best;
    return best_rank;
}

// Nearest entry: returns the leaf-order rank of the collider (or -1) and its
// FP64 entry distance, identical to the reference's choice.  The explicit-ray
// kernels and the fused kernel's overflow fallback use it; it restates the
// Walker's FP32 filter in a self-contained form because the fused kernel's
// local-memory frame includes this function's, and a Walker-based version
// (with a LaneRay copy) measured 0.9 % slower on the batched trace.
template <bool EXACT>
__device__ __noinline__ int nearest(const SceneView& S, const double* o, const double* d, int last_rank,
                                    double& best_out, LocalStats& st) {
    ++st.queries;
    RayF r;
    if (!setup_ray(S.h, o, d, r)) return nearest_flat(S, o, d, last_rank, best_out, st);
    float U = CUDART_INF_F;
    double best = CUDART_INF;
    int best_rank = -1, best_id = -1;
    int cand_rank[kCand];
    float cand_lo[kCand];
#pragma unroll
    for (int e = 0; e < kCand; ++e) { cand_rank[e] = -1; cand_lo[e] = CUDART_INF_F; }
    bool overflow = false, grazing = false;

    int stack_ref[kStackDepth];
    float stack_t[kStackDepth];
    int sp = 0;
    int cur = 0;
    const int n_nodes = S.h->n_nodes, n_atoms = S.h->n_atoms;
    // each node and leaf is entered at most once per query; more steps mean a malformed tree
    for (int steps = 0;; ++steps) {
        if (cur >= n_nodes || steps > 2 * n_nodes + 2) { ++st.errors; break; }
        if (cur >= 0) {
            Hits4 h = visit4(S.nodes, cur, r, U);
            st.box += 4;
            if (h.n > 0) {
                for (int k = h.n - 1; k >= 1; --k) {
                    if (sp < kStackDepth) { stack_ref[sp] = h.ref[k]; stack_t[sp] = h.t[k]; ++sp; }
                    else { ++st.errors; }
                }
                cur = h.ref[0];
                continue;
            }
        } else {
            int code = ~cur;
            int first = code >> kLeafBits, cnt = (code & (kMaxLeaf - 1)) + 1;
            if (first + cnt > n_atoms) { ++st.errors; cnt = 0; }
            for (int k = first; k < first + cnt; ++k) {
                if (k == last_rank) continue;
                ++st.sphere;
                if (EXACT) {
                    double4 a = S.atoms64[k];
                    double t = entry64(o[0], o[1], o[2], d[0], d[1], d[2], a.x, a.y, a.z, a.w);
                    ++st.fp64;
                    int id = __ldg(S.ids + k);
                    if (better(t, id, best, best_id)) {
                        best = t; best_rank = k; best_id = id;
                        U = __double2float_ru(best);
                    }
                } else {
                    float4 a = __ldg(S.atoms + k);
                    float vx = a.x - r.ox, vy = a.y - r.oy, vz = a.z - r.oz;
                    float b = fmaf(vx, r.dx, fmaf(vy, r.dy, vz * r.dz));
                    float px = fmaf(-b, r.dx, vx), py = fmaf(-b, r.dy, vy), pz = fmaf(-b, r.dz, vz);
                    float q = fmaf(px, px, fmaf(py, py, pz * pz));
                    float disc = fmaf(a.w, a.w, -q);
                    if (disc < -r.Edisc || b < -r.Ep) continue;          // certain miss
                    float lo;
                    bool certain = false;
                    if (disc >= 2.0f * r.Edisc) {
                        float Et;
                        const float t = b - certain_sqrt(b, disc, r, Et);
                        if (t < -2.0f * Et) continue;                    // origin inside: no entry ahead
                        if (t > Et) {
                            certain = true;
                            lo = t - Et;
                            float up = t + Et;
                            if (up < U) U = up;
                        }
                    }
                    if (!certain) {
                        lo = fmaxf(0.0f, (b - r.Ep - sqrtf(fmaxf(disc, 0.0f) + r.Edisc)) * (1.0f - 8.0f * kU32));
                        grazing = true;
                    }
                    if (lo <= U) {
                        bool placed = false;
#pragma unroll
                        for (int e = 0; e < kCand; ++e) {
                            bool free_slot = cand_rank[e] < 0 || cand_lo[e] > U;
                            if (!placed && free_slot) { cand_rank[e] = k; cand_lo[e] = lo; placed = true; }
                        }
                        if (!placed) overflow = true;
                    }
                }
            }
        }
        // pop the nearest pending subtree that can still hold an entry <= U
        bool found = false;
        while (sp > 0) {
            --sp;
            if (stack_t[sp] <= U) { cur = stack_ref[sp]; found = true; break; }
        }
        if (!found) break;
    }
    if (!EXACT) {
        if (grazing) ++st.grazing;
        if (overflow) {
            ++st.fallback;
            --st.queries;
            return nearest<true>(S, o, d, last_rank, best_out, st);
        }
#pragma unroll
        for (int e = 0; e < kCand; ++e) {
            if (cand_rank[e] >= 0 && cand_lo[e] <= U) {
                int k = cand_rank[e];
                double4 a = S.atoms64[k];
                double t = entry64(o[0], o[1], o[2], d[0], d[1], d[2], a.x, a.y, a.z, a.w);
                ++st.fp64;
                int id = __ldg(S.ids + k);
                if (better(t, id, best, best_id)) { best = t; best_rank = k; best_id = id; }
            }
        }
    }
    best_out = best;
    return best_rank;
}

// Any-hit PA query (pa_spatial._one with sphere_hit): true when the ray
// meets any sphere other than owner_rank.
__device__ __noinline__ bool anyhit(const SceneView& S, const double* o, const double* d, int owner_rank,
                                    LocalStats& st) {
    ++st.queries;
    RayF r;
    if (!setup_ray(S.h, o, d, r)) {
        int n = S.h->n_atoms;
        for (int k = 0; k < n; ++k) {
            if (k == owner_rank) continue;
            double4 a = S.atoms64[k];
            ++st.sphere; ++st.fp64;
            if (sphere_hit64(o[0], o[1], o[2], d[0], d[1], d[2], a.x, a.y, a.z, a.w)) return true;
        }
        return false;
    }
    int stack_ref[kStackDepth];
    int sp = 0;
    int cur = 0;
    const float U = CUDART_INF_F;
    const int n_nodes = S.h->n_nodes, n_atoms = S.h->n_atoms;
    for (int steps = 0;; ++steps) {
        if (cur >= n_nodes || steps > 2 * n_nodes + 2) { ++st.errors; break; }
        if (cur >= 0) {
            Hits4 h = visit4(S.nodes, cur, r, U);
            st.box += 4;
            if (h.n > 0) {
                for (int k = h.n - 1; k >= 1; --k) {
                    if (sp < kStackDepth) stack_ref[sp++] = h.ref[k]; else ++st.errors;
                }
                cur = h.ref[0];
                continue;
            }
        } else {
            int code = ~cur;
            int first = code >> kLeafBits, cnt = (code & (kMaxLeaf - 1)) + 1;
            if (first + cnt > n_atoms) { ++st.errors; cnt = 0; }
            for (int k = first; k < first + cnt; ++k) {
                if (k == owner_rank) continue;
                ++st.sphere;
                float4 a = __ldg(S.atoms + k);
                float vx = a.x - r.ox, vy = a.y - r.oy, vz = a.z - r.oz;
                float b = fmaf(vx, r.dx, fmaf(vy, r.dy, vz * r.dz));
                float px = fmaf(-b, r.dx, vx), py = fmaf(-b, r.dy, vy), pz = fmaf(-b, r.dz, vz);
                float q = fmaf(px, px, fmaf(py, py, pz * pz));
                float disc = fmaf(a.w, a.w, -q);
                if (disc < -r.Edisc) continue;
                if (disc >= 2.0f * r.Edisc) {
                    float Et;
                    // far root: the reference's -b + sqrt(disc) with b = x.d = -(v.d)
                    const float exitp = b + certain_sqrt(b, disc, r, Et);
                    if (exitp > Et) return true;
                    if (exitp < -2.0f * Et) continue;
                } else if (b + sqrtf(fmaxf(disc, 0.0f) + r.Edisc) < -2.0f * r.Ep) {
                    continue;
                }
                double4 a64 = S.atoms64[k];
                ++st.fp64;
                if (sphere_hit64(o[0], o[1], o[2], d[0], d[1], d[2], a64.x, a64.y, a64.z, a64.w)) return true;
            }
        }
        if (sp == 0) break;
        cur = stack_ref[--sp];
    }
    return false;
}

struct TraceOut {
    int64_t bounces;
    bool escaped, unresolved;
};

// _trace_loop body for one ray (ehss_cpu.py:72-98).  o/d are updated in
// place; history (may be null) receives input atom ids.
__device__ __forceinline__ TraceOut trace_ray(const SceneView& S, double* o, double* d, int last_rank,
                                              int64_t count, int cap, bool exact, int32_t* history,
                                              LocalStats& st) {
    TraceOut out;
    out.escaped = out.unresolved = false;
    while (true) {
        double best;
        int k = exact ? nearest<true>(S, o, d, last_rank, best, st) : nearest<false>(S, o, d, last_rank, best, st);
        if (k < 0) { out.escaped = true; break; }
        if (count >= cap) { out.unresolved = true; break; }
        double4 a = S.atoms64[k];
        reflect64(o[0], o[1], o[2], d[0], d[1], d[2], a.x, a.y, a.z, a.w, best);
        if (history) history[count] = S.ids[k];
        ++count;
        last_rank = k;
    }
    out.bounces = count;
    return out;
}

__device__ __forceinline__ void flush_stats(const LocalStats& st, uint64_t* stats) {
    if (!stats) return;
    unsigned v[7] = {st.box, st.sphere, st.queries, st.grazing, st.fallback, st.fp64, st.errors};
    const int slot[7] = {EHSS_STAT_BOX_TESTS, EHSS_STAT_SPHERE_TESTS, EHSS_STAT_QUERIES, EHSS_STAT_GRAZING,
                         EHSS_STAT_FALLBACK, EHSS_STAT_FP64_TESTS, EHSS_STAT_ERRORS};
    unsigned lane = threadIdx.x & 31;
#pragma unroll
    for (int i = 0; i < 7; ++i) {
        // 64-bit warp sum (per-thread counts can exceed 2^32 / 32 on long runs)
        unsigned long long x = v[i];
        for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
        if (lane == 0 && x) atomicAdd((unsigned long long*)&stats[slot[i]], x);
    }
}

// --------------------------------------------------------------------------
// Explicit-ray kernels
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_trace_rays(const void* scene, int64_t n, int cap, int exact, double* P,
                                                    double* D, const int64_t* last_atom, int64_t* bounces,
                                                    uint8_t* escaped, uint8_t* unresolved, int32_t* history,
                                                    uint64_t* stats) {
    SceneView S = scene_view(scene);
    LocalStats st;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t first = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    // exterior scenes hold only the atoms reachable from outside the union: not for arbitrary rays
    bool ok = S.h->magic == kSceneMagic && S.h->status == 0 && S.h->exterior == 0;
    for (int64_t i = first; i < n; i += stride) {
        double o[3] = {P[3 * i], P[3 * i + 1], P[3 * i + 2]};
        double d[3] = {D[3 * i], D[3 * i + 1], D[3 * i + 2]};
        int64_t count = bounces[i];
        int64_t last_id = last_atom[i];
        int32_t* h = history ? history + i * (int64_t)cap : nullptr;
        if (!ok || last_id < -1 || last_id >= S.h->n_atoms || count < 0 || count > 1 ||
            (count == 1 && last_id < 0)) {
            ++st.errors;
            escaped[i] = 0; unresolved[i] = 0;
            continue;
        }
        int last_rank = last_id >= 0 ? S.rank[last_id] : -1;
        if (h && count == 1) h[0] = (int32_t)last_id;
        TraceOut t = trace_ray(S, o, d, last_rank, count, cap, exact != 0, h, st);
        P[3 * i] = o[0]; P[3 * i + 1] = o[1]; P[3 * i + 2] = o[2];
        D[3 * i] = d[0]; D[3 * i + 1] = d[1]; D[3 * i + 2] = d[2];
        bounces[i] = t.bounces;
        escaped[i] = t.escaped;
        unresolved[i] = t.unresolved;
    }
    flush_stats(st, stats);
}

__global__ void __launch_bounds__(128) k_pa_rays(const void* scene, int64_t n, const double* P, const double* D,
                                                 const int64_t* owners, uint8_t* blocked, uint64_t* stats) {
    SceneView S = scene_view(scene);
    LocalStats st;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    // exterior scenes hold only the atoms reachable from outside the union: not for arbitrary rays
    bool ok = S.h->magic == kSceneMagic && S.h->status == 0 && S.h->exterior == 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
        double o[3] = {P[3 * i], P[3 * i + 1], P[3 * i + 2]};
        double d[3] = {D[3 * i], D[3 * i + 1], D[3 * i + 2]};
        int64_t owner = owners ? owners[i] : -1;
        if (!ok || owner < -1 || owner >= S.h->n_atoms) { ++st.errors; blocked[i] = 0; continue; }
        blocked[i] = anyhit(S, o, d, owner >= 0 ? S.rank[owner] : -1, st);
    }
    flush_stats(st, stats);
}

__global__ void k_sobol_points(int dim, SobolParams p, int64_t first, int64_t n, uint32_t* q) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t idx = (uint32_t)(first + i);
    uint32_t g = idx ^ (idx >> 1);
    for (int j = 0; j < dim; ++j) {
        uint32_t v = p.shift[j];
        uint32_t gg = g;
        while (gg) {
            int k = __ffs(gg) - 1;
            gg &= gg - 1;
            v ^= p.sv[j * 30 + k];
        }
        q[i * dim + j] = v;
    }
}

__global__ void k_source_rays(const void* scene, Sobol4Params p, int64_t first, int64_t n, double* O, double* Dd) {
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    SceneView S = scene_view(scene);
    uint4 q = sobol4(p.sv, p.shift, (uint32_t)(first + i));
    Ray64 ray = impact_ray(q, S.h->center, S.h->radius);
    for (int c = 0; c < 3; ++c) { O[3 * i + c] = ray.o[c]; Dd[3 * i + c] = ray.d[c]; }
}

// --------------------------------------------------------------------------
// Fused blocks (persistent): Sobol -> impact disk -> EHSS / PA -> reduction
//
// One warp takes one chunk (chunk_rays consecutive positions of one block's
// coherent Sobol enumeration) at a time.  Lanes are refilled with the chunk's
// next rays, kNewRayBatch or more at a time.  Each warp alternates two phases:
//   traverse  while-while walk for every lane whose query is open: inner
//             nodes until each lane holds a leaf (a lane holding one walks on
//             to its next), then one leaf per lane, all lanes together;
//             repeated until at least `resolve_batch` lanes have finished
//             their query or wait for a new ray, or none is left traversing;
//   resolve   for all finished lanes together: FP64 candidate re-test,
//             escape / cap / reflection, and new rays once enough lanes
//             wait for one.
// Batching the FP64 work keeps most lanes of the warp busy in both phases.
// The FP64 ray state (position, direction, incoming direction) waits in
// shared memory while the lane traverses in FP32.
// --------------------------------------------------------------------------
// Per-warp accumulators of the chunk in shared memory (updated once per ray
// or per query, so registers stay free for the traversal).
struct WarpAcc {
    unsigned count[kSmemBins];
    unsigned long long ledger[kSmemBins];
    unsigned long long angle_fx;
    unsigned hits, unresolved, escaped, pa;
    unsigned queries, grazing, fallback, fp64, errors, pad;
    unsigned long long box, sphere;
    unsigned long long hits_fx, unres_fx, pa_fx;   // weighted sums of ray blocks
    uint4 q0;
};

struct LaneRay {
    double o[3], d[3], din[3];
};

// The fused kernel's dynamic shared memory: per-warp accumulators, per-lane
// FP64 ray state, then the lanes' traversal-stack columns (and, for ray
// blocks, the lanes' ray weights).
extern __shared__ __align__(16) unsigned char smem_raw[];

// Byte offset of the stack columns.  Recomputed from blockDim wherever a
// stack entry is addressed, so no lane keeps a pointer to its column in
// registers (the fused kernel runs at its 64-register bound: holding the
// pointer and the column stride cost 24 bytes of spills per thread and 1.8 %
// of trace time on the mixed 256-globule batch).
__device__ __forceinline__ unsigned stack_off() {
    return (unsigned)(sizeof(WarpAcc) * (blockDim.x >> 5) + sizeof(LaneRay) * blockDim.x);
}

__device__ __forceinline__ unsigned long long warp_sum64(unsigned long long x) {
    for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
    return x;
}

// Point at position p of a block's coherent enumeration.
__device__ __forceinline__ uint4 block_point(const uint4* basis, uint4 base, uint32_t p) {
    uint4 q = base;
    while (p) {
        int e = __ffs(p) - 1;
        p &= p - 1;
        uint4 v = __ldg(basis + e);
        q.x ^= v.x; q.y ^= v.y; q.z ^= v.z; q.w ^= v.w;
    }
    return q;
}

constexpr int kIdle = 0, kTraverse = 1, kDone = 2, kNeedRay = 3;
// Lanes whose ray has finished wait for a new one until this many of a warp
// do (16 of 32: the 256-globule batch traces in 23.9 ms against 24.6 with a
// new ray at once, 24.2 with 8 and 24.2 with 24).
constexpr int kNewRayBatch = 16;
constexpr int kSentinel = INT32_MAX - 1;   // stack exhausted
constexpr int kNoLeaf = INT32_MAX;

// Traversal stack: the top kSmemStack entries of each lane live in shared
// memory (entry i of lane t at smem_stack[i * blockDim + t], conflict-free);
// deeper entries, rare for an LBVH walked near-child first, go to a
// per-lane local array.
constexpr int kSmemStackMax = 32;

template <bool EXACT, bool COUNT>
struct Walker {
    RayF r;
    float U;
    int cur, leaf, sp, steps;
    int cand_rank[kCand];
    float cand_lo[kCand];
    bool overflow, grazing, error;
    double best;
    int best_rank, best_id;
    unsigned box, sphere;
    // shared-memory stack entry i of this lane
    __device__ __forceinline__ int2* slot(int i) const {
        return reinterpret_cast<int2*>(smem_raw + stack_off()) + i * blockDim.x + threadIdx.x;
    }
    int deep_ref[kStackDepth];
    float deep_t[kStackDepth];

    __device__ __forceinline__ void push(int ref, float t, int sdepth) {
        if (sp < sdepth) *slot(sp) = make_int2(ref, __float_as_int(t));
        else if (sp < kStackDepth) { deep_ref[sp - sdepth] = ref; deep_t[sp - sdepth] = t; }
        else { error = true; return; }
        ++sp;
    }

    __device__ __forceinline__ void reset() {
        U = CUDART_INF_F;
        cur = 0; leaf = kNoLeaf; sp = 0; steps = 0;
#pragma unroll
        for (int e = 0; e < kCand; ++e) { cand_rank[e] = -1; cand_lo[e] = CUDART_INF_F; }
        overflow = grazing = error = false;
        if (EXACT) { best = CUDART_INF; best_rank = -1; best_id = -1; }
    }
    __device__ __forceinline__ int pop(int sdepth) {
        while (sp > 0) {
            --sp;
            int ref;
            float t;
            if (sp < sdepth) { int2 e = *slot(sp); ref = e.x; t = __int_as_float(e.y); }
            else { ref = deep_ref[sp - sdepth]; t = deep_t[sp - sdepth]; }
            if (t <= U) return ref;
        }
        return kSentinel;
    }
    __device__ __forceinline__ int visit(const float4* nodes, int node, int sdepth) {
        Hits4 h = visit4(nodes, node, r, U);
        if (COUNT) box += 4;
        // the distances are sorted with misses at +inf
        if (h.t[0] == CUDART_INF_F) return pop(sdepth);
        if (h.t[3] != CUDART_INF_F) push(h.ref[3], h.t[3], sdepth);
        if (h.t[2] != CUDART_INF_F) push(h.ref[2], h.t[2], sdepth);
        if (h.t[1] != CUDART_INF_F) push(h.ref[1], h.t[1], sdepth);
        return h.ref[0];
    }
    __device__ __forceinline__ void add_candidate(int k, float lo) {
        if (lo > U) return;
        bool placed = false;
#pragma unroll
        for (int e = 0; e < kCand; ++e) {
            bool free_slot = cand_rank[e] < 0 || cand_lo[e] > U;
            if (!placed && free_slot) { cand_rank[e] = k; cand_lo[e] = lo; placed = true; }
        }
        if (!placed) overflow = true;
    }
    __device__ __forceinline__ void leaf_tests(const SceneView& S, int ref, int last_rank, const LaneRay& L) {
        int code = ~ref;
        int first = code >> kLeafBits, cnt = (code & (kMaxLeaf - 1)) + 1;
        if (first + cnt > S.h->n_atoms) { error = true; return; }
        for (int k = first; k < first + cnt; ++k) {
            // FILTER: the start atom is excluded after the cheap reject below, which a ray
            // leaving that atom's surface (moving away from its centre) nearly always takes
            if (EXACT || COUNT) {
                if (k == last_rank) continue;
                if (COUNT) ++sphere;
            }
            if (EXACT) {
                double4 a = S.atoms64[k];
                double t = entry64(L.o[0], L.o[1], L.o[2], L.d[0], L.d[1], L.d[2], a.x, a.y, a.z, a.w);
                int id = __ldg(S.ids + k);
                if (better(t, id, best, best_id)) {
                    best = t; best_rank = k; best_id = id;
                    U = __double2float_ru(best);
                }
            } else {
                float4 a = __ldg(S.atoms + k);
                float vx = a.x - r.ox, vy = a.y - r.oy, vz = a.z - r.oz;
                float b = fmaf(vx, r.dx, fmaf(vy, r.dy, vz * r.dz));
                // the short discriminant; r.Edisc is widened for it (kWidenShortDisc)
                float w = fmaf(-vx, vx, fmaf(-vy, vy, fmaf(-vz, vz, a.w * a.w)));
                float disc = fmaf(b, b, w);
                if (disc < -r.Edisc || b < -r.Ep) continue;
                if (!COUNT && k == last_rank) continue;
                if (disc >= 2.0f * r.Edisc) {
                    float Et;
                    const float t = b - certain_sqrt(b, disc, r, Et);
                    if (t < -2.0f * Et) continue;
                    if (t > Et) {
                        float up = t + Et;
                        if (up < U) U = up;
                        add_candidate(k, t - Et);
                        continue;
                    }
                }
                grazing = true;
                add_candidate(k, fmaxf(0.0f, (b - r.Ep - sqrtf(fmaxf(disc, 0.0f) + r.Edisc)) * (1.0f - 8.0f * kU32)));
            }
        }
    }
};

// FP64 resolution of a finished FILTER query: re-test the candidates with the
// reference formula and the (distance, id) rule.
template <bool COUNT>
__device__ __forceinline__ int resolve_candidates(const SceneView& S, const Walker<false, COUNT>& W, const LaneRay& L,
                                                  double& best, unsigned& fp64) {
    best = CUDART_INF;
    int k = -1, best_id = -1;
#pragma unroll
    for (int e = 0; e < kCand; ++e) {
        if (W.cand_rank[e] >= 0 && W.cand_lo[e] <= W.U) {
            int kk = W.cand_rank[e];
            double4 a = S.atoms64[kk];
            double t = entry64(L.o[0], L.o[1], L.o[2], L.d[0], L.d[1], L.d[2], a.x, a.y, a.z, a.w);
            ++fp64;
            int id = __ldg(S.ids + kk);
            if (better(t, id, best, best_id)) { best = t; k = kk; best_id = id; }
        }
    }
    return k;
}

// Rare path of k_blocks, kept out of line so that it costs the hot loop no registers.
__device__ __noinline__ void save_residual(ehss_residual* residual, long long capacity, unsigned long long* count,
                                           const LaneRay& L, int block, int last_rank, int bounces) {
    unsigned long long at = atomicAdd(count, 1ull);
    if (at >= (unsigned long long)capacity) return;
    ehss_residual& R = residual[at];
    for (int i = 0; i < 3; ++i) { R.o[i] = L.o[i]; R.d[i] = L.d[i]; R.din[i] = L.din[i]; }
    R.block = block;
    R.last_rank = last_rank;
    R.bounces = bounces;
    R.reserved = 0;
}

// Work distribution: the chunk list is cut into one contiguous range per SM
// (partition = %smid mod n_parts) so that the warps of an SM trace the same
// structure, and neighbouring regions of its ray space, at the same time and
// share their L1.  A warp whose range is used up takes chunks from the next
// ranges in turn.  counters[p] counts the chunks handed out from range p.
// Only the window [first, first + total) of the chunk list is traced (the
// whole list, or one GPU's share of it).
__device__ __forceinline__ bool next_chunk(unsigned long long* counters, int n_parts, int& scan, int64_t first,
                                           int64_t total, long long& chunk) {
    for (; scan < n_parts; ++scan) {
        unsigned smid;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        int p = (int)((smid + (unsigned)scan) % (unsigned)n_parts);
        int64_t begin = total * p / n_parts, end = total * (p + 1) / n_parts;
        if (begin >= end) continue;
        unsigned long long t = atomicAdd(counters + p, 1ull);
        if (begin + (int64_t)t < end) { chunk = first + begin + (int64_t)t; return true; }
    }
    return false;
}

// RAYS: the instance for blocks with EHSS_BLOCK_RAYS (caller-made weighted rays);
// each instance skips the other kind's chunks, like the precision instances.
template <bool EXACT, bool COUNT, bool RAYS>
__global__ void __launch_bounds__(128, 8) k_blocks(const ehss_block* blocks, int nb, int64_t chunk_first,
                                                   int64_t total_chunks, int chunk_rays, int resolve_batch,
                                                   ehss_block_result* results,
                                                   uint64_t* hist, uint64_t* ledger, unsigned long long* work,
                                                   int n_parts, int smem_stack, ehss_residual* residual,
                                                   long long residual_capacity, unsigned long long* residual_count) {
    const unsigned lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    WarpAcc& A = reinterpret_cast<WarpAcc*>(smem_raw)[warp];
    LaneRay& L = reinterpret_cast<LaneRay*>(smem_raw + sizeof(WarpAcc) * nwarps)[threadIdx.x];
    int2* stack_base = reinterpret_cast<int2*>(smem_raw + sizeof(WarpAcc) * nwarps + sizeof(LaneRay) * blockDim.x);
    // RAYS: each lane's ray weight relative to the block's largest, after the stack
    double* rho_lane = reinterpret_cast<double*>(stack_base + smem_stack * blockDim.x) + threadIdx.x;
    const unsigned lt_mask = (1u << lane) - 1u;
    Walker<EXACT, COUNT> W;
    int scan = 0;
    while (true) {
        long long c = 0;
        int have = 0;
        if (lane == 0) have = next_chunk(work, n_parts, scan, chunk_first, total_chunks, c);
        have = __shfl_sync(0xffffffffu, have, 0);
        if (!have) break;
        c = __shfl_sync(0xffffffffu, c, 0);
        int bi = 0, hi = nb - 1;
        while (bi < hi) {
            int mid = (bi + hi + 1) >> 1;
            if (blocks[mid].chunk_begin <= c) bi = mid; else hi = mid - 1;
        }
        const ehss_block* B = blocks + bi;
        if ((B->precision == EHSS_PREC_FP64) != EXACT) continue;     // the other instantiation's chunk
        if (((B->flags & EHSS_BLOCK_RAYS) != 0) != RAYS) continue;
        const int64_t ray0 = (c - B->chunk_begin) * (int64_t)chunk_rays;
        const int cnt = (int)min((long long)chunk_rays, (long long)((1ll << B->log2_rays) - ray0));
        // only the scene's base stays live across the phases; each phase rebuilds the view
        // it needs from the (L1-resident) header, which keeps the traversal's registers free
        const void* const sbase = B->scene;
        const bool ok = scene_view(sbase).h->magic == kSceneMagic && scene_view(sbase).h->status == 0;
        if (lane < kSmemBins) { A.count[lane] = 0; A.ledger[lane] = 0; }
        if (lane == 0) {
            const uint4 b0 = make_uint4(B->base[0], B->base[1], B->base[2], B->base[3]);
            A.q0 = block_point(reinterpret_cast<const uint4*>(B->basis), b0, (uint32_t)ray0);
            A.angle_fx = 0; A.hits = A.unresolved = A.escaped = A.pa = 0;
            A.queries = A.grazing = A.fallback = A.fp64 = 0;
            A.errors = ok ? 0 : 1;
            A.box = A.sphere = 0;
            A.hits_fx = A.unres_fx = A.pa_fx = 0;
        }
        __syncwarp();
        if (COUNT) { W.box = 0; W.sphere = 0; }
        int status = ok ? kNeedRay : kIdle;
        int pool = 0, bounces = 0, last_rank = -1;
        while (true) {
            // ---- resolve finished queries (FP64) ----
            if (status == kDone) {
                const SceneView S = scene_view(sbase);
                int k;
                double best;
                if (W.error) {
                    atomicAdd(&A.errors, 1u);
                    k = -1; best = CUDART_INF;
                } else if (EXACT) {
                    k = W.best_rank; best = W.best;
                    atomicAdd(&A.fp64, 1u);
                } else {
                    if (W.grazing) atomicAdd(&A.grazing, 1u);
                    if (W.overflow) {
                        LocalStats fst;
                        k = nearest<true>(S, L.o, L.d, last_rank, best, fst);
                        atomicAdd(&A.fallback, 1u);
                        atomicAdd(&A.fp64, fst.fp64);
                    } else {
                        unsigned f = 0;
                        k = resolve_candidates<COUNT>(S, reinterpret_cast<const Walker<false, COUNT>&>(W), L, best, f);
                        atomicAdd(&A.fp64, f);
                    }
                }
                if (k < 0 || bounces >= __ldg(&B->cap)) {
                    bool escaped = k < 0;
                    unsigned long long fx = 0;
                    if (escaped) {
                        double a = scatter_angle(L.din[0], L.din[1], L.din[2], L.d[0], L.d[1], L.d[2]);
                        fx = __double2ull_rn((RAYS ? a * *rho_lane : a) * kFxScale);
                        atomicAdd(&A.escaped, 1u);
                        if (fx) atomicAdd(&A.angle_fx, fx);
                    } else {
                        atomicAdd(&A.unresolved, 1u);
                        if (RAYS) atomicAdd(&A.unres_fx, __double2ull_rn(*rho_lane * kFxScale));
                        // save the state for a later cap extension
                        if (residual) save_residual(residual, residual_capacity, residual_count, L, bi, last_rank, bounces);
                    }
                    if (bounces > 0 || !escaped) {
                        atomicAdd(&A.hits, 1u);
                        if (RAYS) atomicAdd(&A.hits_fx, __double2ull_rn(*rho_lane * kFxScale));
                    }
                    if (bounces < kSmemBins) {
                        atomicAdd(&A.count[bounces], 1u);
                        if (fx) atomicAdd(&A.ledger[bounces], fx);
                    } else {
                        atomicAdd((unsigned long long*)&hist[B->hist_offset + bounces], 1ull);
                        if (fx) atomicAdd((unsigned long long*)&ledger[B->hist_offset + bounces], fx);
                    }
                    status = kNeedRay;
                } else {
                    double4 a = S.atoms64[k];
                    reflect64(L.o[0], L.o[1], L.o[2], L.d[0], L.d[1], L.d[2], a.x, a.y, a.z, a.w, best);
                    ++bounces;
                    last_rank = k;
                    W.reset();
                    if (!setup_ray(S.h, L.o, L.d, W.r, EXACT ? 0.0f : kWidenShortDisc)) W.error = true;   // bounce points lie within S
                    atomicAdd(&A.queries, 1u);
                    status = kTraverse;
                }
            }
            // ---- new rays for lanes whose ray finished ----
            // made once kNewRayBatch lanes wait for one (or the chunk is used up, or no
            // lane traverses), so that the FP64 impact-disk work runs at warp width
            unsigned need = __ballot_sync(0xffffffffu, status == kNeedRay);
            if (need && (__popc(need) >= kNewRayBatch || pool >= cnt || !__any_sync(0xffffffffu, status == kTraverse))) {
                const SceneView S = scene_view(sbase);
                if (status == kNeedRay) {
                    int p = pool + __popc(need & lt_mask);
                    if (p < cnt) {
                        if (RAYS) {
                            // caller-made rays: origins [3n], directions [3n], weights [n]
                            const int64_t n = 1ll << B->log2_rays, r = ray0 + p;
                            const double* R = B->rays;
#pragma unroll
                            for (int i = 0; i < 3; ++i) {
                                L.o[i] = R[3 * r + i];
                                L.d[i] = L.din[i] = R[3 * n + 3 * r + i];
                            }
                            *rho_lane = R[6 * n + r] * B->ray_scale;
                        } else {
                            // ray0 is a multiple of the chunk size, so point(ray0 + p) = point(ray0) ^ B(p)
                            uint4 q = block_point(reinterpret_cast<const uint4*>(B->basis), A.q0, (uint32_t)p);
                            Ray64 ray = impact_ray(q, S.h->center, S.h->radius);
#pragma unroll
                            for (int i = 0; i < 3; ++i) { L.o[i] = ray.o[i]; L.d[i] = ray.d[i]; L.din[i] = ray.d[i]; }
                        }
                        if (__ldg(&B->flags) & EHSS_BLOCK_PA) {
                            LocalStats pst;
                            if (anyhit(S, L.o, L.d, -1, pst)) {
                                atomicAdd(&A.pa, 1u);
                                if (RAYS) atomicAdd(&A.pa_fx, __double2ull_rn(*rho_lane * kFxScale));
                            }
                            // the counting instance adds the any-hit tests to the block's counters
                            if (COUNT) { W.box += pst.box; W.sphere += pst.sphere; }
                        }
                        bounces = 0;
                        last_rank = -1;
                        if (__ldg(&B->flags) & EHSS_BLOCK_EHSS) {
                            W.reset();
                            if (!setup_ray(S.h, L.o, L.d, W.r, EXACT ? 0.0f : kWidenShortDisc)) W.error = true;
                            atomicAdd(&A.queries, 1u);
                            status = kTraverse;
                        }
                    } else {
                        status = kIdle;
                    }
                }
                pool += __popc(need);
                if (__any_sync(0xffffffffu, status == kNeedRay)) continue;   // PA-only lanes refill again
            }
            if (!__any_sync(0xffffffffu, status == kTraverse)) break;
            // ---- traverse until enough queries are finished ----
            const SceneView S = scene_view(sbase);
            while (true) {
                if (status == kTraverse) {
                    // inner nodes; the first leaf reached is held while the lane walks on
                    while (W.cur >= 0 && W.cur != kSentinel) {
                        const int n_nodes = __ldg(&S.h->n_nodes);
                        if (W.cur >= n_nodes || ++W.steps > 2 * n_nodes + 2) { W.error = true; W.cur = kSentinel; break; }
                        W.cur = W.visit(S.nodes, W.cur, smem_stack);
                        if (W.cur < 0 && W.leaf == kNoLeaf) {
                            W.leaf = W.cur;
                            W.cur = W.pop(smem_stack);
                        }
                        if (!__any_sync(__activemask(), W.leaf == kNoLeaf)) break;
                    }
                    // one leaf per lane and phase: a lane's next leaf joins the next phase
                    if (W.leaf != kNoLeaf) {
                        W.leaf_tests(S, W.leaf, last_rank, L);
                        W.leaf = kNoLeaf;
                        if (W.cur < 0) {
                            W.leaf = W.cur;
                            W.cur = W.pop(smem_stack);
                        }
                    }
                    if (W.cur == kSentinel && W.leaf == kNoLeaf) status = kDone;
                }
                // lanes waiting for a new ray count towards the resolve batch
                unsigned done = __ballot_sync(0xffffffffu, status == kDone || status == kNeedRay);
                unsigned trav = __ballot_sync(0xffffffffu, status == kTraverse);
                if (!trav || __popc(done) >= resolve_batch) break;
            }
        }
        if (COUNT) {
            unsigned long long b = warp_sum64(W.box), sp = warp_sum64(W.sphere);
            if (lane == 0) { A.box = b; A.sphere = sp; }
        }
        __syncwarp();
        // one atomic per field into the block result
        ehss_block_result* R = results + bi;
        if (lane == 0) {
            if (A.angle_fx) atomicAdd((unsigned long long*)&R->angle_fx, A.angle_fx);
            if (A.hits) atomicAdd((unsigned long long*)&R->hits, (unsigned long long)A.hits);
            if (A.unresolved) atomicAdd((unsigned long long*)&R->unresolved, (unsigned long long)A.unresolved);
            if (A.escaped) atomicAdd((unsigned long long*)&R->escaped, (unsigned long long)A.escaped);
            if (A.pa) atomicAdd((unsigned long long*)&R->pa_blocked, (unsigned long long)A.pa);
            if (A.hits_fx) atomicAdd((unsigned long long*)&R->hits_fx, A.hits_fx);
            if (A.unres_fx) atomicAdd((unsigned long long*)&R->unresolved_fx, A.unres_fx);
            if (A.pa_fx) atomicAdd((unsigned long long*)&R->pa_fx, A.pa_fx);
            unsigned long long v[7] = {A.box, A.sphere, A.queries, A.grazing, A.fallback, A.fp64, A.errors};
            const int slot[7] = {EHSS_STAT_BOX_TESTS, EHSS_STAT_SPHERE_TESTS, EHSS_STAT_QUERIES, EHSS_STAT_GRAZING,
                                 EHSS_STAT_FALLBACK, EHSS_STAT_FP64_TESTS, EHSS_STAT_ERRORS};
            for (int i = 0; i < 7; ++i)
                if (v[i]) atomicAdd((unsigned long long*)&R->stats[slot[i]], v[i]);
        }
        if (lane < kSmemBins && lane <= B->cap) {
            if (A.count[lane])
                atomicAdd((unsigned long long*)&hist[B->hist_offset + lane], (unsigned long long)A.count[lane]);
            if (A.ledger[lane]) atomicAdd((unsigned long long*)&ledger[B->hist_offset + lane], A.ledger[lane]);
        }
        __syncwarp();
    }
}

// --------------------------------------------------------------------------
// Host launchers
// --------------------------------------------------------------------------
static unsigned grid_for(int64_t n, int threads) {
    int64_t want = (n + threads - 1) / threads;
    int64_t cap = (int64_t)sm_count() * 16;
    if (want > cap) want = cap;
    return (unsigned)(want > 0 ? want : 1);
}

int launch_trace_rays(const void* scene, int64_t n, int cap, int precision, double* P, double* D,
                      const int64_t* last, int64_t* bounces, uint8_t* esc, uint8_t* unres, int32_t* hist,
                      uint64_t* stats, cudaStream_t stream) {
    if (n == 0) return EHSS_OK;
    k_trace_rays<<<grid_for(n, 128), 128, 0, stream>>>(scene, n, cap, precision == EHSS_PREC_FP64, P, D, last,
                                                       bounces, esc, unres, hist, stats);
    return cuda_status(cudaGetLastError(), "trace launch");
}

int launch_pa_rays(const void* scene, int64_t n, const double* P, const double* D, const int64_t* owners,
                   uint8_t* blocked, uint64_t* stats, cudaStream_t stream) {
    if (n == 0) return EHSS_OK;
    k_pa_rays<<<grid_for(n, 128), 128, 0, stream>>>(scene, n, P, D, owners, blocked, stats);
    return cuda_status(cudaGetLastError(), "PA launch");
}

int launch_sobol_points(int dim, const SobolParams& p, int64_t first, int64_t n, uint32_t* q, cudaStream_t stream) {
    if (n == 0) return EHSS_OK;
    k_sobol_points<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(dim, p, first, n, q);
    return cuda_status(cudaGetLastError(), "Sobol launch");
}

int launch_source_rays(const void* scene, const Sobol4Params& p, int64_t first, int64_t n, double* O, double* D,
                       cudaStream_t stream) {
    if (n == 0) return EHSS_OK;
    k_source_rays<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(scene, p, first, n, O, D);
    return cuda_status(cudaGetLastError(), "source launch");
}

int launch_blocks(const ehss_block* blocks, int nb, int64_t chunk_first, int64_t total_chunks, const ehss_launch& L,
                  ehss_block_result* results, uint64_t* hist, uint64_t* ledger, unsigned long long* work,
                  cudaStream_t stream, ehss_residual* residual, int64_t residual_capacity,
                  unsigned long long* residual_count) {
    int warps = L.block_threads / 32;
    const int sdepth = L.smem_stack > 0 ? L.smem_stack : 16;
    const size_t smem = sizeof(WarpAcc) * (size_t)warps + sizeof(LaneRay) * (size_t)L.block_threads +
                        sizeof(int2) * sdepth * (size_t)L.block_threads;
    const size_t smem_rays = smem + sizeof(double) * (size_t)L.block_threads;
    unsigned grid = (unsigned)(sm_count() * L.ctas_per_sm);
    int batch = L.resolve_batch > 0 ? L.resolve_batch : 1;
    const bool count = (L.options & EHSS_LAUNCH_COUNT_TESTS) != 0;
    // one launch per precision and ray kind present; each skips the other blocks' chunks
    const int mask = L.precisions ? L.precisions : 3;
    const int kinds = (L.options & EHSS_LAUNCH_RAY_BLOCKS) ? ((L.options & EHSS_LAUNCH_NO_DISK_BLOCKS) ? 2 : 3) : 1;
    bool first = true;
    for (int exact = 1; exact >= 0; --exact) {
        if (!((mask >> (exact ? EHSS_PREC_FP64 : EHSS_PREC_FP32)) & 1)) continue;
        for (int rays = 0; rays <= 1; ++rays) {
            if (!((kinds >> rays) & 1)) continue;
            if (!first) {
                int rc = cuda_status(cudaMemsetAsync(work, 0, sizeof(unsigned long long) * kMaxWorkParts, stream),
                                     "work counter reset");
                if (rc) return rc;
            }
            first = false;
            const int n_parts = sm_count() < kMaxWorkParts ? sm_count() : kMaxWorkParts;
#define EHSS_LAUNCH_BLOCKS(E, C, R) \
            k_blocks<E, C, R><<<grid, L.block_threads, R ? smem_rays : smem, stream>>>( \
                blocks, nb, chunk_first, total_chunks, L.chunk_rays, batch, results, hist, ledger, work, n_parts, sdepth, \
                residual, residual_capacity, residual_count)
            if (exact) {
                if (rays) { if (count) EHSS_LAUNCH_BLOCKS(true, true, true); else EHSS_LAUNCH_BLOCKS(true, false, true); }
                else { if (count) EHSS_LAUNCH_BLOCKS(true, true, false); else EHSS_LAUNCH_BLOCKS(true, false, false); }
            } else {
                if (rays) { if (count) EHSS_LAUNCH_BLOCKS(false, true, true); else EHSS_LAUNCH_BLOCKS(false, false, true); }
                else { if (count) EHSS_LAUNCH_BLOCKS(false, true, false); else EHSS_LAUNCH_BLOCKS(false, false, false); }
            }
#undef EHSS_LAUNCH_BLOCKS
            int rc = cuda_status(cudaGetLastError(), "blocks launch");
            if (rc) return rc;
        }
    }
    return EHSS_OK;
}

// --------------------------------------------------------------------------
// Cap extension: continue saved unresolved rays (one thread per ray) from
// their exact state, so each follows the path it would have followed with
// the larger cap from the start.  Sums are the same integers k_blocks uses.
// --------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_extend(const ehss_block* blocks, int nb, const int32_t* row_of, int rows,
                                                const ehss_residual* in, int64_t n_in, int new_cap,
                                                ehss_extension* ext, uint64_t* hist, uint64_t* ledger,
                                                ehss_residual* out, int64_t out_capacity,
                                                unsigned long long* out_count, uint64_t* stats) {
    LocalStats st;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_in; i += stride) {
        const ehss_residual R = in[i];
        if (R.block < 0 || R.block >= nb) { ++st.errors; continue; }
        const int row = row_of[R.block];
        if (row < 0) continue;
        if (row >= rows) { ++st.errors; continue; }
        const ehss_block* B = blocks + R.block;
        const SceneView S = scene_view(B->scene);
        if ((B->flags & EHSS_BLOCK_RAYS) || S.h->magic != kSceneMagic || S.h->status != 0 || R.bounces >= new_cap || R.last_rank < -1 ||
            R.last_rank >= S.h->n_atoms) {
            ++st.errors;
            continue;
        }
        const bool exact = B->precision == EHSS_PREC_FP64;
        double o[3] = {R.o[0], R.o[1], R.o[2]}, d[3] = {R.d[0], R.d[1], R.d[2]};
        int last_rank = R.last_rank, count = R.bounces;
        bool escaped = false;
        double so[3], sd[3];
        int s_last = last_rank;
        while (true) {
            double best;
            const int k = exact ? nearest<true>(S, o, d, last_rank, best, st) : nearest<false>(S, o, d, last_rank, best, st);
            if (k < 0) { escaped = true; break; }
            if (count >= new_cap) {
                for (int c = 0; c < 3; ++c) { so[c] = o[c]; sd[c] = d[c]; }
                s_last = last_rank;
                break;
            }
            const double4 a = S.atoms64[k];
            reflect64(o[0], o[1], o[2], d[0], d[1], d[2], a.x, a.y, a.z, a.w, best);
            ++count;
            last_rank = k;
        }
        ehss_extension& E = ext[row];
        uint64_t* h = hist + (int64_t)row * (new_cap + 1);
        uint64_t* l = ledger + (int64_t)row * (new_cap + 1);
        atomicAdd((unsigned long long*)&E.continued, 1ull);
        atomicAdd((unsigned long long*)&h[count], 1ull);
        if (escaped) {
            const double ang = scatter_angle(R.din[0], R.din[1], R.din[2], d[0], d[1], d[2]);
            const unsigned long long fx = __double2ull_rn(ang * kFxScale);
            atomicAdd((unsigned long long*)&E.escaped, 1ull);
            if (fx) {
                atomicAdd((unsigned long long*)&E.angle_fx, fx);
                atomicAdd((unsigned long long*)&l[count], fx);
            }
        } else {
            atomicAdd((unsigned long long*)&E.unresolved, 1ull);
            const unsigned long long at = atomicAdd(out_count, 1ull);
            if (at < (unsigned long long)out_capacity) {
                ehss_residual& Q = out[at];
                for (int c = 0; c < 3; ++c) { Q.o[c] = so[c]; Q.d[c] = sd[c]; Q.din[c] = R.din[c]; }
                Q.block = R.block;
                Q.last_rank = s_last;
                Q.bounces = count;
                Q.reserved = 0;
            }
        }
    }
    flush_stats(st, stats);
}

int launch_extend(const ehss_block* blocks, int nb, const int32_t* row, int rows, const ehss_residual* in,
                  int64_t n_in, int new_cap, ehss_extension* ext, uint64_t* hist, uint64_t* ledger,
                  ehss_residual* out, int64_t out_capacity, unsigned long long* out_count, uint64_t* stats,
                  cudaStream_t stream) {
    if (n_in == 0) return EHSS_OK;
    k_extend<<<grid_for(n_in, 128), 128, 0, stream>>>(blocks, nb, row, rows, in, n_in, new_cap, ext, hist, ledger,
                                                      out, out_capacity, out_count, stats);
    return cuda_status(cudaGetLastError(), "cap extension launch");
}

}  // namespace ehss
