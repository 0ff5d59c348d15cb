// Adaptive finite-grid PA on the device.
//
// Replaces ccs_cli.adaptive_pa (src/support_exchange_transport/ccs_cli.py:142-160):
// for each of n_dirs directions drawn from Sobol(2, seed) through unit_sphere
// (inside_out_pa.py:45-49), project the atom centres on the plane normal to
// the direction (project_grid, pa_walsh_geometry.py:171-180), lay an n x n
// grid of pixel midpoints over the enclosing square and count the pixels that
// lie in the union of the atom disks -- the quantity the reference's sparse
// quadtree (block_disks / block_count, pa_sparse_blocks.py:134-166) counts
// with the exact row inequality of row_span (pa_dyadic_bitmask.py:50-61).
//
// Device layout per direction: projected coordinates xy[atom][2] (FP64),
// frame/extent record, and a bitmask of n rows x ceil(n/64) 64-bit words.
//   k_grid_project  one CTA per direction: direction frame, projections, extent
//   k_grid_raster   one thread per (direction, atom): exact row spans -> atomicOr
//   k_grid_count    one CTA per direction: popcount of the bitmask
// Counts are integers, so a direction's count equals the reference's count
// whenever the projected coordinates are the same.
#include <cstdio>
#include "ehss_internal.cuh"

namespace ehss {

struct GridDir {
    double u[3], v[3];
    double lower, spacing;     // lower = -extent (both axes), spacing = 2 extent / n
};

struct Sobol2Params { uint32_t sv[2][30]; uint32_t shift[2]; };

__device__ __forceinline__ double dot3(const double* a, const double* b) {
    return dadd(dadd(dmul(a[0], b[0]), dmul(a[1], b[1])), dmul(a[2], b[2]));
}

__global__ void k_grid_project(const void* scene, const double* xyz, Sobol2Params sob, int n_dirs, int n,
                               GridDir* dirs, double* xy) {
    const int dir = blockIdx.x;
    if (dir >= n_dirs) return;
    SceneView S = scene_view(scene);
    const int m = S.h->n_atoms;
    __shared__ double frame[6];
    __shared__ double partial[32];
    if (threadIdx.x == 0) {
        // unit_sphere of Sobol(2) point `dir` (the reference's direction list order)
        uint32_t g = (uint32_t)dir ^ ((uint32_t)dir >> 1);
        uint32_t q0 = sob.shift[0], q1 = sob.shift[1];
        while (g) {
            int k = __ffs(g) - 1;
            g &= g - 1;
            q0 ^= sob.sv[0][k];
            q1 ^= sob.sv[1][k];
        }
        double u0 = q0 * 0x1p-30, u1 = q1 * 0x1p-30;
        double z = dsub(1.0, dmul(2.0, u0));
        double phi = dmul(2.0 * 3.141592653589793, u1);
        double rho = dsqrt(dmax0(dsub(1.0, dmul(z, z))));
        double sp, cp;
        sincos(phi, &sp, &cp);
        double d[3] = {dmul(rho, cp), dmul(rho, sp), z};
        // project_grid: normalise, frame axis e_z unless |d_z| >= 0.9 (then e_x)
        double nd = dsqrt(dot3(d, d));
        for (int c = 0; c < 3; ++c) d[c] = ddiv(d[c], nd);
        double a[3] = {0., 0., 1.};
        if (!(fabs(d[2]) < .9)) { a[0] = 1.; a[2] = 0.; }
        double u[3] = {dsub(dmul(a[1], d[2]), dmul(a[2], d[1])), dsub(dmul(a[2], d[0]), dmul(a[0], d[2])),
                       dsub(dmul(a[0], d[1]), dmul(a[1], d[0]))};
        double nu = dsqrt(dot3(u, u));
        for (int c = 0; c < 3; ++c) u[c] = ddiv(u[c], nu);
        double v[3] = {dsub(dmul(d[1], u[2]), dmul(d[2], u[1])), dsub(dmul(d[2], u[0]), dmul(d[0], u[2])),
                       dsub(dmul(d[0], u[1]), dmul(d[1], u[0]))};
        for (int c = 0; c < 3; ++c) { frame[c] = u[c]; frame[3 + c] = v[c]; }
    }
    __syncthreads();
    const double u[3] = {frame[0], frame[1], frame[2]}, v[3] = {frame[3], frame[4], frame[5]};
    double ext = 0.;
    double* out = xy + (int64_t)dir * m * 2;
    for (int i = threadIdx.x; i < m; i += blockDim.x) {
        // input order: atoms64 is in leaf order, the rank map gives input id -> leaf
        double4 a = S.atoms64[S.rank[i]];
        double c[3] = {dsub(a.x, S.h->center[0]), dsub(a.y, S.h->center[1]), dsub(a.z, S.h->center[2])};
        double x = dot3(c, u), y = dot3(c, v);
        out[2 * i] = x;
        out[2 * i + 1] = y;
        ext = fmax(ext, fmax(dadd(fabs(x), a.w), dadd(fabs(y), a.w)));
    }
    (void)xyz;
    for (int off = 16; off > 0; off >>= 1) ext = fmax(ext, __shfl_xor_sync(0xffffffffu, ext, off));
    if ((threadIdx.x & 31) == 0) partial[threadIdx.x >> 5] = ext;
    __syncthreads();
    if (threadIdx.x < 32) {
        double e = threadIdx.x < (blockDim.x >> 5) ? partial[threadIdx.x] : 0.;
        for (int off = 16; off > 0; off >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, off));
        if (threadIdx.x == 0) {
            double extent = dmul(e, 1.0000000001);
            GridDir& D = dirs[dir];
            for (int c = 0; c < 3; ++c) { D.u[c] = u[c]; D.v[c] = v[c]; }
            D.lower = -extent;
            D.spacing = ddiv(dmul(2.0, extent), (double)n);
        }
    }
}

// row_span (pa_dyadic_bitmask.py:50-61) in FP64 without contraction.
__device__ __forceinline__ void row_span(double cx, double cy, double r, double lower, double spacing, int y, int n,
                                         int& lo_out, int& hi_out) {
    lo_out = hi_out = 0;
    double dy = dsub(dadd(lower, dmul((double)y + .5, spacing)), cy);
    double rem = dsub(dmul(r, r), dmul(dy, dy));
    if (rem < 0) return;
    double half = dsqrt(rem);
    double a = ceil(dsub(ddiv(dsub(dsub(cx, half), lower), spacing), .5));
    double b = floor(dsub(ddiv(dsub(dadd(cx, half), lower), spacing), .5));
    long long lo = (long long)a, hi = (long long)b + 1;
    lo = lo < n ? lo : n; lo = lo > 0 ? lo : 0;
    hi = hi < n ? hi : n; hi = hi > 0 ? hi : 0;
    for (int it = 0; it < 4 && lo > 0; ++it) {
        double t = dsub(dadd(lower, dmul((double)lo - .5, spacing)), cx);
        if (dmul(t, t) <= rem) --lo; else break;
    }
    for (int it = 0; it < 4 && lo < hi; ++it) {
        double t = dsub(dadd(lower, dmul((double)lo + .5, spacing)), cx);
        if (dmul(t, t) > rem) ++lo; else break;
    }
    for (int it = 0; it < 4 && hi < n; ++it) {
        double t = dsub(dadd(lower, dmul((double)hi + .5, spacing)), cx);
        if (dmul(t, t) <= rem) ++hi; else break;
    }
    for (int it = 0; it < 4 && hi > lo; ++it) {
        double t = dsub(dadd(lower, dmul((double)hi - .5, spacing)), cx);
        if (dmul(t, t) > rem) --hi; else break;
    }
    lo_out = (int)lo;
    hi_out = (int)hi;
}

__global__ void k_grid_raster(const void* scene, int n_dirs, int n, const GridDir* dirs, const double* xy,
                              unsigned long long* bits, unsigned long long* errors) {
    const int dir = blockIdx.y;
    SceneView S = scene_view(scene);
    const int m = S.h->n_atoms;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (dir >= n_dirs || i >= m) return;
    const GridDir D = dirs[dir];
    const double cx = xy[((int64_t)dir * m + i) * 2], cy = xy[((int64_t)dir * m + i) * 2 + 1];
    const double r = S.atoms64[S.rank[i]].w;
    const int words = (n + 63) >> 6;
    unsigned long long* mask = bits + (int64_t)dir * n * words;
    // row_bounds (pa_dyadic_bitmask.py:63-68): one extra row each side, rows
    // outside the disk give empty spans
    long long y0 = (long long)ceil(dsub(ddiv(dsub(dsub(cy, r), D.lower), D.spacing), .5)) - 1;
    long long y1 = (long long)floor(dsub(ddiv(dsub(dadd(cy, r), D.lower), D.spacing), .5)) + 2;
    y0 = y0 < n ? y0 : n; y0 = y0 > 0 ? y0 : 0;
    y1 = y1 < n ? y1 : n; y1 = y1 > 0 ? y1 : 0;
    for (long long y = y0; y < y1; ++y) {
        int lo, hi;
        row_span(cx, cy, r, D.lower, D.spacing, (int)y, n, lo, hi);
        if (hi <= lo) continue;
        for (int k = lo >> 6; k <= (hi - 1) >> 6; ++k) {
            int left = lo - 64 * k, right = hi - 64 * k;
            left = left > 0 ? left : 0;
            right = right < 64 ? right : 64;
            unsigned long long hib = right >= 64 ? ~0ull : ((1ull << right) - 1ull);
            unsigned long long lob = left >= 64 ? ~0ull : ((1ull << left) - 1ull);
            if (k < words) atomicOr(mask + y * words + k, hib ^ lob);
            else atomicAdd(errors, 1ull);
        }
    }
}

__global__ void k_grid_count(int n_dirs, int n, const unsigned long long* bits, unsigned long long* counts) {
    const int dir = blockIdx.x;
    if (dir >= n_dirs) return;
    const int words = (n + 63) >> 6;
    const unsigned long long* mask = bits + (int64_t)dir * n * words;
    unsigned long long c = 0;
    for (int64_t w = threadIdx.x; w < (int64_t)n * words; w += blockDim.x) c += __popcll(mask[w]);
    for (int off = 16; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
    __shared__ unsigned long long part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
        counts[dir] = t;
    }
}

uint64_t grid_workspace_bytes(int64_t n_atoms, int n_dirs, int n) {
    uint64_t words = (uint64_t)((n + 63) / 64);
    return align256(sizeof(GridDir) * (uint64_t)n_dirs) + align256(16ull * n_atoms * n_dirs) +
           align256(8ull * n_dirs * n * words) + 256 + 256;
}

int launch_grid_pa(const void* scene, int64_t n_atoms, int n_dirs, uint64_t seed, int n, unsigned long long* counts,
                   double* spacing_out, double* xy_out, void* workspace, uint64_t ws_bytes, cudaStream_t stream) {
    uint64_t need = grid_workspace_bytes(n_atoms, n_dirs, n);
    if (ws_bytes < need) {
        set_error("adaptive PA workspace holds %llu bytes, %llu required", (unsigned long long)ws_bytes,
                  (unsigned long long)need);
        return EHSS_ERR_CAPACITY;
    }
    char* p = (char*)(((uintptr_t)workspace + 255u) & ~(uintptr_t)255u);
    GridDir* dirs = (GridDir*)p; p += align256(sizeof(GridDir) * (uint64_t)n_dirs);
    double* xy = (double*)p; p += align256(16ull * n_atoms * n_dirs);
    unsigned long long* bits = (unsigned long long*)p;
    uint64_t words = (uint64_t)((n + 63) / 64);
    p += align256(8ull * n_dirs * n * words);
    unsigned long long* errors = (unsigned long long*)p;
    Sobol2Params sob;
    uint32_t sv[2 * 30], shift[2];
    sobol_scramble(2, seed, sv, shift);
    for (int j = 0; j < 2; ++j) {
        for (int k = 0; k < 30; ++k) sob.sv[j][k] = sv[j * 30 + k];
        sob.shift[j] = shift[j];
    }
    int rc = cuda_status(cudaMemsetAsync(bits, 0, 8ull * n_dirs * n * words, stream), "grid reset");
    if (!rc) rc = cuda_status(cudaMemsetAsync(errors, 0, 8, stream), "grid reset");
    if (rc) return rc;
    k_grid_project<<<n_dirs, 256, 0, stream>>>(scene, nullptr, sob, n_dirs, n, dirs, xy);
    dim3 grid((unsigned)((n_atoms + 127) / 128), (unsigned)n_dirs);
    k_grid_raster<<<grid, 128, 0, stream>>>(scene, n_dirs, n, dirs, xy, bits, errors);
    k_grid_count<<<n_dirs, 256, 0, stream>>>(n_dirs, n, bits, counts);
    if (spacing_out)
        rc = cuda_status(cudaMemcpy2DAsync(spacing_out, sizeof(double), &dirs[0].spacing, sizeof(GridDir),
                                           sizeof(double), (size_t)n_dirs, cudaMemcpyDeviceToDevice, stream),
                         "grid spacing copy");
    if (!rc && xy_out)
        rc = cuda_status(cudaMemcpyAsync(xy_out, xy, 16ull * n_atoms * n_dirs, cudaMemcpyDeviceToDevice, stream),
                         "grid xy copy");
    if (rc) return rc;
    return cuda_status(cudaGetLastError(), "adaptive PA launch");
}

}  // namespace ehss
