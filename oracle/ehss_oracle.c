/*
 * TEST INFRASTRUCTURE — CPU oracle, not part of the product.
 *
 * Plain-C restatement of the SCIMMS/EHSS reference's FP64 CPU algorithm for
 * the PA + EHSS cross-section path.  Only the test suite, the smoke check and
 * the CPU-baseline leg of the benchmark load this library, and only as the
 * checker or the timed CPU baseline; the CUDA library never calls it.
 *
 * Every function names the reference file:line it restates (paths relative to
 * the reference project root).  Arithmetic keeps the reference's operation
 * order and parenthesisation; the build uses -ffp-contract=off so that no
 * multiply-add is fused, matching Numba without fastmath (which the reference
 * runs with) bit for bit.  Parity is pinned by tests/golden fixtures produced
 * from the reference itself (tests/golden/make_golden.py).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#define EPS64 DBL_EPSILON

/* ---------------------------------------------------------------------- */
/* Stable argsort helper (numpy kind='mergesort'/'stable' semantics).      */
/* ---------------------------------------------------------------------- */
typedef struct { double v; int64_t pos; int64_t id; } keyed_t;

static int keyed_cmp(const void* a, const void* b) {
    const keyed_t* x = (const keyed_t*)a;
    const keyed_t* y = (const keyed_t*)b;
    if (x->v < y->v) return -1;
    if (x->v > y->v) return 1;
    return (x->pos < y->pos) ? -1 : (x->pos > y->pos);
}

/* Sort ids[0..n) stably by key(ids[k]) = vals[ids[k]*3+axis]. */
static void stable_sort_ids(int64_t* ids, int64_t n, const double* vals, int axis, keyed_t* tmp) {
    for (int64_t k = 0; k < n; ++k) {
        tmp[k].v = vals[ids[k] * 3 + axis];
        tmp[k].pos = k;
        tmp[k].id = ids[k];
    }
    qsort(tmp, (size_t)n, sizeof(keyed_t), keyed_cmp);
    for (int64_t k = 0; k < n; ++k) ids[k] = tmp[k].id;
}

/* ---------------------------------------------------------------------- */
/* Static EHSS BVH preparation.                                            */
/* ---------------------------------------------------------------------- */

/* Box centres exactly as static_spatial_groups forms them:
 * lo = c - r, hi = c + r, centre = (lo + hi) / 2  (ehss_static.py:53-59). */
void oracle_box_centres(int64_t n, const double* centers, const double* radii, double* out) {
    for (int64_t i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) {
            double lo = centers[i * 3 + c] - radii[i];
            double hi = centers[i * 3 + c] + radii[i];
            out[i * 3 + c] = (lo + hi) / 2;
        }
}

/* _median_groups (ehss_static.py:16-50): depth-first median split on the
 * axis of largest centre span; leaves at <= leaf_size atoms, depth 24 or zero
 * span; groups numbered in left-first DFS order.  Returns the group count. */
int64_t oracle_median_groups(int64_t n, const double* box_centres, int64_t leaf_size, int64_t* groups) {
    int64_t* ids = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
    keyed_t* tmp = (keyed_t*)malloc(sizeof(keyed_t) * (size_t)(n > 0 ? n : 1));
    for (int64_t i = 0; i < n; ++i) ids[i] = i;
    int64_t starts[64], stops[64], depths[64];
    starts[0] = 0; stops[0] = n; depths[0] = 0;
    int64_t pending = 1, group = 0;
    while (pending) {
        pending -= 1;
        int64_t a = starts[pending], b = stops[pending], depth = depths[pending];
        double span[3];
        for (int c = 0; c < 3; ++c) {
            double low = INFINITY, high = -INFINITY;
            for (int64_t k = a; k < b; ++k) {
                double v = box_centres[ids[k] * 3 + c];
                low = v < low ? v : low;
                high = v > high ? v : high;
            }
            span[c] = high - low;
        }
        int axis = 0;
        for (int c = 1; c < 3; ++c) if (span[c] > span[axis]) axis = c;
        if (b - a <= leaf_size || depth >= 24 || span[axis] == 0) {
            for (int64_t k = a; k < b; ++k) groups[ids[k]] = group;
            group += 1;
            continue;
        }
        stable_sort_ids(ids + a, b - a, box_centres, axis, tmp);
        int64_t mid = a + (b - a) / 2;
        starts[pending] = mid; stops[pending] = b; depths[pending] = depth + 1;
        starts[pending + 1] = a; stops[pending + 1] = mid; depths[pending + 1] = depth + 1;
        pending += 2;
    }
    free(ids); free(tmp);
    return group;
}

/* topology (ehss_cpu_geometry.py:19-38): implicit balanced binary tree over
 * group index ranges, 2G-1 nodes in pre-order, end[] = skip pointer. */
void oracle_topology(int64_t ng, int64_t* left, int64_t* right, int64_t* end, int64_t* parent,
                     int64_t* leaf, int64_t* leaf_node) {
    int64_t nodes = 2 * ng - 1;
    int64_t* begin = (int64_t*)calloc((size_t)nodes, sizeof(int64_t));
    int64_t* stop = (int64_t*)calloc((size_t)nodes, sizeof(int64_t));
    for (int64_t i = 0; i < nodes; ++i) { left[i] = right[i] = parent[i] = leaf[i] = -1; }
    stop[0] = ng;
    for (int64_t node = 0; node < nodes; ++node) {
        int64_t a = begin[node], b = stop[node];
        end[node] = node + 2 * (b - a) - 1;
        if (b - a == 1) {
            leaf[node] = a; leaf_node[a] = node;
        } else {
            int64_t mid = a + (b - a) / 2;
            int64_t l = node + 1, r = node + 2 * (mid - a);
            left[node] = l; right[node] = r;
            begin[l] = a; stop[l] = mid; begin[r] = mid; stop[r] = b;
            parent[l] = node; parent[r] = node;
        }
    }
    free(begin); free(stop);
}

/* Full static preparation (PreparedStaticCPUEHSS.__init__, ehss_static.py:62-91):
 * groups -> topology -> offsets/ids (cumsum of bincount, stable argsort) ->
 * padded leaf bounds (leaf_serial, ehss_cpu_geometry.py:41-54, pad =
 * 1e-10*max(1, max r), ehss_static.py:86) -> parent unions (parents,
 * ehss_cpu_geometry.py:58-71).  Output arrays are sized by the caller:
 * nodes = 2*ng-1 where ng = oracle_median_groups(...). */
void oracle_static_tree(int64_t n, const double* centers, const double* radii, const int64_t* groups,
                        int64_t ng, double* lo, double* hi, int64_t* end, int64_t* leaf_group,
                        int64_t* offsets, int64_t* ids) {
    int64_t nodes = 2 * ng - 1;
    int64_t* left = (int64_t*)malloc(sizeof(int64_t) * (size_t)nodes);
    int64_t* right = (int64_t*)malloc(sizeof(int64_t) * (size_t)nodes);
    int64_t* parent = (int64_t*)malloc(sizeof(int64_t) * (size_t)nodes);
    int64_t* leaf_node = (int64_t*)malloc(sizeof(int64_t) * (size_t)ng);
    oracle_topology(ng, left, right, end, parent, leaf_group, leaf_node);
    memset(offsets, 0, sizeof(int64_t) * (size_t)(ng + 1));
    for (int64_t i = 0; i < n; ++i) offsets[groups[i] + 1] += 1;
    for (int64_t g = 0; g < ng; ++g) offsets[g + 1] += offsets[g];
    int64_t* fill = (int64_t*)malloc(sizeof(int64_t) * (size_t)ng);
    memcpy(fill, offsets, sizeof(int64_t) * (size_t)ng);
    for (int64_t i = 0; i < n; ++i) ids[fill[groups[i]]++] = i;   /* stable argsort of groups */
    double rmax = radii[0];
    for (int64_t i = 1; i < n; ++i) rmax = radii[i] > rmax ? radii[i] : rmax;
    double pad = 1e-10 * (1. > rmax ? 1. : rmax);
    for (int64_t g = 0; g < ng; ++g) {
        int64_t node = leaf_node[g];
        for (int c = 0; c < 3; ++c) {
            double low = INFINITY, high = -INFINITY;
            for (int64_t k = offsets[g]; k < offsets[g + 1]; ++k) {
                int64_t atom = ids[k];
                double a = centers[atom * 3 + c] - radii[atom];
                double b = centers[atom * 3 + c] + radii[atom];
                low = a < low ? a : low;
                high = b > high ? b : high;
            }
            lo[node * 3 + c] = low - pad;
            hi[node * 3 + c] = high + pad;
        }
    }
    for (int64_t node = nodes - 1; node >= 0; --node) {
        if (left[node] >= 0) {
            for (int c = 0; c < 3; ++c) {
                double a = lo[left[node] * 3 + c], b = lo[right[node] * 3 + c];
                lo[node * 3 + c] = a < b ? a : b;
                a = hi[left[node] * 3 + c]; b = hi[right[node] * 3 + c];
                hi[node * 3 + c] = a > b ? a : b;
            }
        }
    }
    free(left); free(right); free(parent); free(leaf_node); free(fill);
}

/* ---------------------------------------------------------------------- */
/* EHSS trace.                                                             */
/* ---------------------------------------------------------------------- */

/* entry_scalar (ehss_cpu.py:12-24) == entry_distance (ehss_reference.py:8-23). */
double oracle_entry(const double* o, const double* d, const double* c, double radius) {
    double x0 = o[0] - c[0], x1 = o[1] - c[1], x2 = o[2] - c[2];
    double aa = (d[0] * d[0] + d[1] * d[1]) + d[2] * d[2];
    double projection = ((x0 * d[0] + x1 * d[1]) + x2 * d[2]) / aa;
    double p0 = x0 - projection * d[0], p1 = x1 - projection * d[1], p2 = x2 - projection * d[2];
    double disc = radius * radius - ((p0 * p0 + p1 * p1) + p2 * p2);
    if (disc < 0. || projection >= 0.) return INFINITY;
    double near = -projection - sqrt((disc > 0. ? disc : 0.) / aa);
    if (near < -64 * EPS64 * radius) return INFINITY;
    return near > 0. ? near : 0.;
}

/* box_interval (ehss_support_tree.py:19-31); returns 1 when the node is
 * visited (not pruned) under nearest_scalar's rule near > best or far < 0. */
static int box_visit(const double* o, const double* d, const double* lo, const double* hi, double best) {
    double near = 0., far = INFINITY;
    for (int k = 0; k < 3; ++k) {
        if (d[k] == 0.) {
            if (o[k] < lo[k] || o[k] > hi[k]) return 0;
        } else {
            double a = (lo[k] - o[k]) / d[k], b = (hi[k] - o[k]) / d[k];
            double mn = a < b ? a : b, mx = a > b ? a : b;
            near = mn > near ? mn : near;
            far = mx < far ? mx : far;
        }
    }
    if (far < near) return 0;
    return !(near > best || far < 0.);
}

/* reflect_scalar (ehss_cpu.py:27-40). */
static void reflect(double* o, double* d, const double* c, double r, double distance) {
    double n0 = o[0] + distance * d[0] - c[0];
    double n1 = o[1] + distance * d[1] - c[1];
    double n2 = o[2] + distance * d[2] - c[2];
    double norm = sqrt((n0 * n0 + n1 * n1) + n2 * n2);
    n0 /= norm; n1 /= norm; n2 /= norm;
    o[0] = c[0] + r * n0; o[1] = c[1] + r * n1; o[2] = c[2] + r * n2;
    double dot = (d[0] * n0 + d[1] * n1) + d[2] * n2;
    d[0] = d[0] - 2 * dot * n0; d[1] = d[1] - 2 * dot * n1; d[2] = d[2] - 2 * dot * n2;
    norm = sqrt((d[0] * d[0] + d[1] * d[1]) + d[2] * d[2]);
    d[0] /= norm; d[1] /= norm; d[2] /= norm;
}

/* nearest_scalar (ehss_cpu.py:43-63): stackless pre-order walk, skip `last`,
 * lexicographic (distance, atom id) minimum. */
static int64_t nearest(const double* o, const double* d, int64_t last, int64_t nn,
                       const double* lo, const double* hi, const int64_t* end, const int64_t* leaf_group,
                       const int64_t* offsets, const int64_t* ids, const double* world, const double* radii,
                       double* best_out, int64_t* boxes, int64_t* spheres) {
    int64_t node = 0, atom = -1;
    double best = INFINITY;
    while (node < nn) {
        *boxes += 1;
        if (!box_visit(o, d, lo + 3 * node, hi + 3 * node, best)) { node = end[node]; continue; }
        int64_t g = leaf_group[node];
        if (g >= 0) {
            for (int64_t k = offsets[g]; k < offsets[g + 1]; ++k) {
                int64_t wanted = ids[k];
                if (wanted == last) continue;
                *spheres += 1;
                double distance = oracle_entry(o, d, world + 3 * wanted, radii[wanted]);
                if (distance < best || (distance == best && isfinite(distance) && (atom < 0 || wanted < atom))) {
                    atom = wanted; best = distance;
                }
            }
        }
        node += 1;
    }
    *best_out = best;
    return atom;
}

/* _trace_loop (ehss_cpu.py:66-100): bounce until escape; a hit found once the
 * ray already has `cap` collisions marks it unresolved.  p/d are updated in
 * place (the caller passes copies, as CPUEHSSTransport.trace does). */
void oracle_trace(int64_t nr, int64_t nn, int64_t cap, int record, int threads,
                  double* p, double* d, const int64_t* lasts, int64_t* counts,
                  uint8_t* escaped, uint8_t* unresolved, int32_t* history,
                  const double* lo, const double* hi, const int64_t* end, const int64_t* leaf_group,
                  const int64_t* offsets, const int64_t* ids, const double* world, const double* radii,
                  int64_t* counters, int64_t* per_ray_boxes, int64_t* per_ray_spheres) {
    int64_t boxes = 0, spheres = 0;
    (void)threads;
#pragma omp parallel for schedule(dynamic, 64) reduction(+:boxes, spheres) num_threads(threads > 0 ? threads : 1)
    for (int64_t ray = 0; ray < nr; ++ray) {
        double* o = p + 3 * ray;
        double* v = d + 3 * ray;
        int64_t last = lasts[ray];
        int64_t nb = 0, ns = 0;
        escaped[ray] = 0; unresolved[ray] = 0;
        if (record && counts[ray] == 1) history[ray * cap] = (int32_t)last;
        while (1) {
            double best;
            int64_t atom = nearest(o, v, last, nn, lo, hi, end, leaf_group, offsets, ids, world, radii,
                                   &best, &nb, &ns);
            if (atom < 0) { escaped[ray] = 1; break; }
            if (counts[ray] >= cap) { unresolved[ray] = 1; break; }
            reflect(o, v, world + 3 * atom, radii[atom], best);
            if (record) history[ray * cap + counts[ray]] = (int32_t)atom;
            counts[ray] += 1;
            last = atom;
        }
        if (per_ray_boxes) per_ray_boxes[ray] = nb;
        if (per_ray_spheres) per_ray_spheres[ray] = ns;
        boxes += nb; spheres += ns;
    }
    counters[0] = boxes; counters[1] = spheres;
}

/* trace_all (ehss_reference.py:40-64): the independent all-atom search
 * (nearest_all :26-37, strict distance < best in atom order). */
void oracle_trace_flat(int64_t nr, int64_t n, int64_t cap, double* p, double* d, const int64_t* lasts,
                       int64_t* counts, uint8_t* escaped, uint8_t* unresolved, int32_t* ledger,
                       const double* centers, const double* radii) {
    for (int64_t ray = 0; ray < nr; ++ray) {
        double* o = p + 3 * ray;
        double* v = d + 3 * ray;
        int64_t last = lasts[ray];
        escaped[ray] = 0; unresolved[ray] = 0;
        if (counts[ray] == 1) ledger[ray * cap] = (int32_t)last;
        while (1) {
            double best = INFINITY; int64_t atom = -1;
            for (int64_t j = 0; j < n; ++j) {
                if (j == last) continue;
                double t = oracle_entry(o, v, centers + 3 * j, radii[j]);
                if (t < best) { best = t; atom = j; }
            }
            if (atom < 0) { escaped[ray] = 1; break; }
            if (counts[ray] >= cap) { unresolved[ray] = 1; break; }
            double q[3];
            for (int c = 0; c < 3; ++c) q[c] = o[c] + best * v[c];
            double nrm[3] = {q[0] - centers[3 * atom], q[1] - centers[3 * atom + 1], q[2] - centers[3 * atom + 2]};
            double len = sqrt((nrm[0] * nrm[0] + nrm[1] * nrm[1]) + nrm[2] * nrm[2]);
            for (int c = 0; c < 3; ++c) nrm[c] /= len;
            for (int c = 0; c < 3; ++c) o[c] = centers[3 * atom + c] + radii[atom] * nrm[c];
            double dot = (v[0] * nrm[0] + v[1] * nrm[1]) + v[2] * nrm[2];
            for (int c = 0; c < 3; ++c) v[c] = v[c] - 2 * dot * nrm[c];
            len = sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
            for (int c = 0; c < 3; ++c) v[c] /= len;
            ledger[ray * cap + counts[ray]] = (int32_t)atom;
            counts[ray] += 1;
            last = atom;
        }
    }
}

/* ---------------------------------------------------------------------- */
/* BVH any-hit PA.                                                         */
/* ---------------------------------------------------------------------- */

/* build_tree, kind 'bvh' (pa_spatial.py:38-75): recursive stable median
 * split over primitive-box centres; node bounds are the unpadded union of
 * the primitive boxes; pre-order with end[] skip pointers. */
typedef struct {
    const double *plo, *phi, *ctr;
    int64_t leaf_size;
    double *lo, *hi;
    int64_t *end, *first, *count, *ids;
    int64_t nodes, nids;
    keyed_t* tmp;
} pa_builder;

static void pa_visit(pa_builder* B, int64_t* idx, int64_t m, int64_t depth) {
    int64_t index = B->nodes++;
    for (int c = 0; c < 3; ++c) {
        double low = INFINITY, high = -INFINITY;
        for (int64_t k = 0; k < m; ++k) {
            double a = B->plo[idx[k] * 3 + c], b = B->phi[idx[k] * 3 + c];
            low = a < low ? a : low;
            high = b > high ? b : high;
        }
        B->lo[index * 3 + c] = low; B->hi[index * 3 + c] = high;
    }
    B->end[index] = 0; B->first[index] = B->nids; B->count[index] = 0;
    double ptp[3];
    for (int c = 0; c < 3; ++c) {
        double low = INFINITY, high = -INFINITY;
        for (int64_t k = 0; k < m; ++k) {
            double v = B->ctr[idx[k] * 3 + c];
            low = v < low ? v : low;
            high = v > high ? v : high;
        }
        ptp[c] = high - low;
    }
    if (m <= B->leaf_size || depth >= 24 || (ptp[0] == 0 && ptp[1] == 0 && ptp[2] == 0)) {
        B->count[index] = m;
        for (int64_t k = 0; k < m; ++k) B->ids[B->nids++] = idx[k];
    } else {
        int axis = 0;
        for (int c = 1; c < 3; ++c) if (ptp[c] > ptp[axis]) axis = c;
        stable_sort_ids(idx, m, B->ctr, axis, B->tmp);
        int64_t middle = m / 2;
        pa_visit(B, idx, middle, depth + 1);
        pa_visit(B, idx + middle, m - middle, depth + 1);
    }
    B->end[index] = B->nodes;
}

/* Returns the node count; arrays must hold 2n nodes (the tree has at most
 * 2n-1).  plo/phi are the primitive boxes c -/+ r (SphereIndex.__init__,
 * pa_spatial.py:158-160). */
int64_t oracle_pa_tree(int64_t n, const double* plo, const double* phi, int64_t leaf_size,
                       double* lo, double* hi, int64_t* end, int64_t* first, int64_t* count, int64_t* ids) {
    pa_builder B;
    double* ctr = (double*)malloc(sizeof(double) * 3 * (size_t)n);
    for (int64_t i = 0; i < 3 * n; ++i) ctr[i] = (plo[i] + phi[i]) / 2;
    int64_t* idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    for (int64_t i = 0; i < n; ++i) idx[i] = i;
    B.plo = plo; B.phi = phi; B.ctr = ctr; B.leaf_size = leaf_size;
    B.lo = lo; B.hi = hi; B.end = end; B.first = first; B.count = count; B.ids = ids;
    B.nodes = 0; B.nids = 0;
    B.tmp = (keyed_t*)malloc(sizeof(keyed_t) * (size_t)n);
    pa_visit(&B, idx, n, 0);
    free(ctr); free(idx); free(B.tmp);
    return B.nodes;
}

/* box_hit (pa_spatial.py:98-111). */
static int pa_box_hit(const double* o, const double* d, const double* lo, const double* hi) {
    double near = 0., far = INFINITY;
    for (int axis = 0; axis < 3; ++axis) {
        if (d[axis] == 0) {
            if (o[axis] < lo[axis] || o[axis] > hi[axis]) return 0;
        } else {
            double a = (lo[axis] - o[axis]) / d[axis], b = (hi[axis] - o[axis]) / d[axis];
            double mn = a < b ? a : b, mx = a > b ? a : b;
            near = near > mn ? near : mn;
            far = far < mx ? far : mx;
            if (far < near) return 0;
        }
    }
    return 1;
}

/* sphere_hit (inside_out_pa.py:93-101). */
int oracle_sphere_hit(const double* o, const double* d, const double* c, double r) {
    double x = o[0] - c[0], y = o[1] - c[1], z = o[2] - c[2];
    double b = x * d[0] + y * d[1] + z * d[2];
    double cc = x * x + y * y + z * z - r * r;
    double disc = b * b - cc;
    return disc >= 0 && -b + sqrt(disc > 0. ? disc : 0.) > 0;
}

/* tree_blocked / _one (pa_spatial.py:114-142): first hit of any sphere other
 * than the ray's owner. */
void oracle_pa_blocked(int64_t nr, const double* origins, const double* dirs, const int64_t* owners,
                       const double* centers, const double* radii, int64_t nn, const double* lo, const double* hi,
                       const int64_t* end, const int64_t* first, const int64_t* count, const int64_t* ids,
                       uint8_t* blocked, int64_t* counters, int threads) {
    int64_t boxes = 0, tests = 0;
    (void)threads;
#pragma omp parallel for schedule(dynamic, 64) reduction(+:boxes, tests) num_threads(threads > 0 ? threads : 1)
    for (int64_t i = 0; i < nr; ++i) {
        const double* o = origins + 3 * i;
        const double* d = dirs + 3 * i;
        int64_t node = 0, stop = end[0], hit = 0;
        while (node < stop && !hit) {
            boxes += 1;
            if (!pa_box_hit(o, d, lo + 3 * node, hi + 3 * node)) { node = end[node]; continue; }
            for (int64_t k = first[node]; k < first[node] + count[node]; ++k) {
                int64_t j = ids[k];
                if (j != owners[i]) {
                    tests += 1;
                    if (oracle_sphere_hit(o, d, centers + 3 * j, radii[j])) { hit = 1; break; }
                }
            }
            node += 1;
        }
        blocked[i] = (uint8_t)hit;
    }
    (void)nn;
    counters[0] = boxes; counters[1] = tests;
}

/* ---------------------------------------------------------------------- */
/* Adaptive finite-grid PA.                                                */
/* ---------------------------------------------------------------------- */

/* row_span (pa_dyadic_bitmask.py:50-61): covered pixels [lo, hi) of row y
 * for the disk (cx, cy, r); pixel i has midpoint lower + (i + 0.5) spacing and
 * is covered when (x_mid - cx)^2 <= r^2 - (y_mid - cy)^2. */
static void row_span(double cx, double cy, double r, double lower0, double lower1, double spacing, int64_t y,
                     int64_t n, int64_t* lo_out, int64_t* hi_out) {
    double dy = lower1 + (y + .5) * spacing - cy;
    double rem = r * r - dy * dy;
    *lo_out = 0; *hi_out = 0;
    if (rem < 0) return;
    double half = sqrt(rem);
    double a = ceil((cx - half - lower0) / spacing - .5);
    double b = floor((cx + half - lower0) / spacing - .5);
    int64_t lo = (int64_t)a, hi = (int64_t)b + 1;
    lo = lo < n ? lo : n; lo = lo > 0 ? lo : 0;
    hi = hi < n ? hi : n; hi = hi > 0 ? hi : 0;
    while (lo > 0) { double t = lower0 + (lo - .5) * spacing - cx; if (t * t <= rem) lo -= 1; else break; }
    while (lo < hi) { double t = lower0 + (lo + .5) * spacing - cx; if (t * t > rem) lo += 1; else break; }
    while (hi < n) { double t = lower0 + (hi + .5) * spacing - cx; if (t * t <= rem) hi += 1; else break; }
    while (hi > lo) { double t = lower0 + (hi - .5) * spacing - cx; if (t * t > rem) hi -= 1; else break; }
    *lo_out = lo; *hi_out = hi;
}

/* row_bounds (pa_dyadic_bitmask.py:63-68). */
static void row_bounds(double cy, double r, double lower1, double spacing, int64_t n, int64_t* lo, int64_t* hi) {
    int64_t a = (int64_t)ceil((cy - r - lower1) / spacing - .5) - 1;
    int64_t b = (int64_t)floor((cy + r - lower1) / spacing - .5) + 2;
    a = a < n ? a : n; a = a > 0 ? a : 0;
    b = b < n ? b : n; b = b > 0 ? b : 0;
    *lo = a; *hi = b;
}

/* Pixels of the n x n midpoint grid covered by the union of the disks
 * (the quantity block_count(block_disks(...)) counts, pa_sparse_blocks.py:134-166);
 * bits: caller-provided n*ceil(n/64) uint64 words. */
int64_t oracle_union_count(int64_t m, const double* xy, const double* radii, double lower0, double lower1,
                           double spacing, int64_t n, uint64_t* bits) {
    int64_t words = (n + 63) / 64;
    memset(bits, 0, sizeof(uint64_t) * (size_t)(n * words));
    for (int64_t a = 0; a < m; ++a) {
        int64_t y0, y1;
        row_bounds(xy[2 * a + 1], radii[a], lower1, spacing, n, &y0, &y1);
        for (int64_t y = y0; y < y1; ++y) {
            int64_t lo, hi;
            row_span(xy[2 * a], xy[2 * a + 1], radii[a], lower0, lower1, spacing, y, n, &lo, &hi);
            for (int64_t x = lo; x < hi; ++x) bits[y * words + x / 64] |= (uint64_t)1 << (x % 64);
        }
    }
    int64_t count = 0;
    for (int64_t i = 0; i < n * words; ++i) count += __builtin_popcountll(bits[i]);
    return count;
}
