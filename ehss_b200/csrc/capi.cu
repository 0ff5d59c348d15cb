// extern "C" entry points of libehss_b200.so (declared in include/ehss_b200.h).
// Host-side validation mirrors the reference's ValueError checks; every
// failure sets a thread-local message and returns a nonzero status.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <cmath>
#include "ehss_internal.cuh"

namespace ehss {

static thread_local char g_error[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_error, sizeof(g_error), fmt, ap);
    va_end(ap);
}

static const char* error_text() { return g_error; }
static void clear_error() { g_error[0] = '\0'; }

int cuda_status(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return EHSS_OK;
    set_error("%s: %s", what, cudaGetErrorString(e));
    return EHSS_ERR_CUDA;
}

int sm_count() {
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!cached[dev]) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cached[dev] = n > 0 ? n : 148;
    }
    return cached[dev];
}

void sobol4_params(uint64_t seed, Sobol4Params* p) {
    uint32_t sv[4 * 30], shift[4];
    sobol_scramble(4, seed, sv, shift);
    for (int k = 0; k < 30; ++k) p->sv[k] = make_uint4(sv[k], sv[30 + k], sv[60 + k], sv[90 + k]);
    p->shift = make_uint4(shift[0], shift[1], shift[2], shift[3]);
}

}  // namespace ehss

using namespace ehss;

static cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

extern "C" {

const char* ehss_last_error(void) { return error_text(); }

int ehss_abi_version(void) { return EHSS_ABI_VERSION; }

int ehss_sobol_scramble(int dim, uint64_t seed, uint32_t* sv_host, uint32_t* shift_host) {
    clear_error();
    if (!sv_host || !shift_host) { set_error("null output pointer"); return EHSS_ERR_VALUE; }
    if (!sobol_scramble(dim, seed, sv_host, shift_host)) {
        set_error("Sobol dimension must be 1..8, got %d", dim);
        return EHSS_ERR_VALUE;
    }
    return EHSS_OK;
}

int ehss_sobol_points(int dim, uint64_t seed, int64_t first, int64_t n, uint32_t* q_dev, void* stream) {
    clear_error();
    if (dim < 1 || dim > 8) { set_error("Sobol dimension must be 1..8, got %d", dim); return EHSS_ERR_VALUE; }
    if (first < 0 || n < 0 || first + n > (1ll << 30)) {
        set_error("Sobol point range [%lld, %lld) outside 0..2^30", (long long)first, (long long)(first + n));
        return EHSS_ERR_VALUE;
    }
    if (n > 0 && !q_dev) { set_error("null output pointer"); return EHSS_ERR_VALUE; }
    SobolParams p;
    memset(&p, 0, sizeof(p));
    sobol_scramble(dim, seed, p.sv, p.shift);
    return launch_sobol_points(dim, p, first, n, q_dev, as_stream(stream));
}

int ehss_compact_source_rays(const ehss_boundary* boundary_host, int log2n, uint64_t seed, int64_t first, int64_t n,
                             double* origins_dev, double* directions_dev, double* weights_dev, void* stream) {
    clear_error();
    if (!boundary_host) { set_error("null boundary"); return EHSS_ERR_VALUE; }
    const ehss_boundary& B = *boundary_host;
    if (B.kind != EHSS_BOUNDARY_SPHERE && B.kind != EHSS_BOUNDARY_ELLIPSOID && B.kind != EHSS_BOUNDARY_BOX) {
        set_error("Boundary must be sphere, ellipsoid, or box");
        return EHSS_ERR_VALUE;
    }
    for (int k = 0; k < 3; ++k)
        if (!(B.axes[k] > 0.) || !std::isfinite(B.axes[k]) || !std::isfinite(B.center[k])) {
            set_error("boundary centre must be finite and its semi-axes positive and finite");
            return EHSS_ERR_VALUE;
        }
    for (int k = 0; k < 9; ++k)
        if (!std::isfinite(B.rotation[k])) { set_error("boundary rotation must be finite"); return EHSS_ERR_VALUE; }
    if (log2n < 0 || log2n > 30) { set_error("log2n must be 0..30"); return EHSS_ERR_VALUE; }
    if (first < 0 || n < 0 || first + n > (1ll << log2n)) { set_error("ray range outside the sequence"); return EHSS_ERR_VALUE; }
    if (n > 0 && (!origins_dev || !directions_dev || !weights_dev)) { set_error("null output pointer"); return EHSS_ERR_VALUE; }
    const int dim = B.kind == EHSS_BOUNDARY_BOX ? 5 : 4;
    SobolParams p;
    memset(&p, 0, sizeof(p));
    sobol_scramble(dim, seed, p.sv, p.shift);
    return launch_compact_rays(B, p, dim, first, n, 1.0 / (double)(1ll << log2n), origins_dev, directions_dev,
                               weights_dev, as_stream(stream));
}

int ehss_enclosing_radius(int64_t n_atoms, const double* xyz, const double* radii, double* radius) {
    clear_error();
    if (n_atoms < 1 || !xyz || !radii || !radius) { set_error("invalid arguments"); return EHSS_ERR_VALUE; }
    // k_stats' operations: sequential column sums divided by n, then max of |c - centre| + r
    // (norm as sqrt((x*x + y*y) + z*z)), times 1.000000001; each operation rounded once
    volatile double acc[3] = {0., 0., 0.};
    for (int64_t i = 0; i < n_atoms; ++i)
        for (int c = 0; c < 3; ++c) acc[c] = acc[c] + xyz[3 * i + c];
    double center[3];
    for (int c = 0; c < 3; ++c) center[c] = acc[c] / (double)n_atoms;
    double smax = 0.;
    bool nan = false;
    for (int64_t i = 0; i < n_atoms; ++i) {
        volatile double x = xyz[3 * i] - center[0], y = xyz[3 * i + 1] - center[1], z = xyz[3 * i + 2] - center[2];
        volatile double xx = x * x, yy = y * y, zz = z * z;
        volatile double s = xx + yy;
        s = s + zz;
        volatile double len = std::sqrt((double)s);
        len = len + radii[i];
        if (std::isnan((double)len)) nan = true;
        else if (len > smax) smax = len;
    }
    *radius = nan ? NAN : smax * 1.000000001;
    return EHSS_OK;
}

int ehss_scene_bytes(int64_t n_atoms, int leaf_size, uint64_t* scene_bytes, uint64_t* workspace_bytes) {
    clear_error();
    if (n_atoms < 1 || n_atoms > (1 << 27)) {
        set_error("atom count %lld outside 1..2^27", (long long)n_atoms);
        return EHSS_ERR_VALUE;
    }
    if (leaf_size < 1 || leaf_size > kMaxLeaf) { set_error("leaf_size must be 1..%d", kMaxLeaf); return EHSS_ERR_VALUE; }
    uint64_t a, b, c, d, e, total;
    scene_layout(n_atoms, &a, &b, &c, &d, &e, &total);
    if (scene_bytes) *scene_bytes = total;
    if (workspace_bytes) *workspace_bytes = build_workspace_bytes(n_atoms, 1);
    return EHSS_OK;
}

int ehss_scene_build(int64_t n_atoms, const double* xyz_dev, const double* radii_dev, int leaf_size, void* scene_dev,
                     uint64_t scene_bytes, void* workspace_dev, uint64_t workspace_bytes, void* stream) {
    clear_error();
    if (!xyz_dev || !radii_dev || !scene_dev || !workspace_dev) { set_error("null pointer"); return EHSS_ERR_VALUE; }
    return build_scenes(1, &xyz_dev, &radii_dev, &n_atoms, leaf_size, &scene_dev, &scene_bytes, workspace_dev,
                        workspace_bytes, as_stream(stream));
}

int ehss_scenes_workspace_bytes(int n_scenes, const int64_t* n_atoms_host, uint64_t* workspace_bytes) {
    clear_error();
    if (n_scenes < 1 || !n_atoms_host || !workspace_bytes) { set_error("invalid arguments"); return EHSS_ERR_VALUE; }
    int64_t N = 0;
    for (int s = 0; s < n_scenes; ++s) {
        if (n_atoms_host[s] < 1) { set_error("structure %d has no atoms", s); return EHSS_ERR_VALUE; }
        N += n_atoms_host[s];
    }
    if (N > (int64_t)INT32_MAX) { set_error("a batch holds at most %d atoms", INT32_MAX); return EHSS_ERR_VALUE; }
    *workspace_bytes = build_workspace_bytes(N, n_scenes);
    return EHSS_OK;
}

int ehss_scenes_build(int n_scenes, const double* const* xyz_dev, const double* const* radii_dev,
                      const int64_t* n_atoms_host, int leaf_size, void* const* scenes_dev,
                      const uint64_t* scene_bytes_host, void* workspace_dev, uint64_t workspace_bytes, void* stream) {
    clear_error();
    if (n_scenes < 1 || !xyz_dev || !radii_dev || !n_atoms_host || !scenes_dev || !scene_bytes_host ||
        !workspace_dev) {
        set_error("invalid arguments");
        return EHSS_ERR_VALUE;
    }
    return build_scenes(n_scenes, xyz_dev, radii_dev, n_atoms_host, leaf_size, scenes_dev, scene_bytes_host,
                        workspace_dev, workspace_bytes, as_stream(stream));
}

int ehss_scenes_build_ex(int n_scenes, const double* const* xyz_dev, const double* const* radii_dev,
                         const int64_t* n_atoms_host, int leaf_size, void* const* scenes_dev,
                         const uint64_t* scene_bytes_host, void* workspace_dev, uint64_t workspace_bytes,
                         uint32_t flags, void* stream) {
    clear_error();
    if (n_scenes < 1 || !xyz_dev || !radii_dev || !n_atoms_host || !scenes_dev || !scene_bytes_host ||
        !workspace_dev) {
        set_error("invalid arguments");
        return EHSS_ERR_VALUE;
    }
    if (flags & ~EHSS_BUILD_EXTERIOR) { set_error("unknown build flags 0x%x", flags); return EHSS_ERR_VALUE; }
    return build_scenes(n_scenes, xyz_dev, radii_dev, n_atoms_host, leaf_size, scenes_dev, scene_bytes_host,
                        workspace_dev, workspace_bytes, as_stream(stream), (flags & EHSS_BUILD_EXTERIOR) != 0);
}

int ehss_scenes_refit(int n_scenes, const double* const* xyz_dev, const double* const* radii_dev,
                      const int64_t* n_atoms_host, void* const* scenes_dev, void* workspace_dev,
                      uint64_t workspace_bytes, void* stream) {
    clear_error();
    if (n_scenes < 1 || !xyz_dev || !radii_dev || !n_atoms_host || !scenes_dev || !workspace_dev) {
        set_error("invalid arguments");
        return EHSS_ERR_VALUE;
    }
    return refit_scenes(n_scenes, xyz_dev, radii_dev, n_atoms_host, scenes_dev, workspace_dev, workspace_bytes,
                        as_stream(stream));
}

int ehss_scene_info_get(const void* scene_dev, ehss_scene_info* info, void* stream) {
    clear_error();
    if (!scene_dev || !info) { set_error("null pointer"); return EHSS_ERR_VALUE; }
    SceneHeader h;
    int rc = cuda_status(cudaMemcpyAsync(&h, scene_dev, sizeof(h), cudaMemcpyDeviceToHost, as_stream(stream)),
                         "scene header read");
    if (rc) return rc;
    rc = cuda_status(cudaStreamSynchronize(as_stream(stream)), "scene header read");
    if (rc) return rc;
    if (h.magic != kSceneMagic) { set_error("not a built scene buffer"); return EHSS_ERR_VALUE; }
    if (h.status == 3) { set_error("refit requires a full (non-exterior) scene with the same atom count"); return EHSS_ERR_VALUE; }
    if (h.status == 4) { set_error("refit found a malformed node record"); return EHSS_ERR_VALUE; }
    if (h.status != 0) { set_error("scene input has a non-positive or non-finite radius or coordinate"); return EHSS_ERR_VALUE; }
    info->n_atoms = h.n_atoms;
    info->n_nodes = h.n_nodes;
    info->leaf_size = h.leaf_size;
    info->depth = h.depth;
    for (int c = 0; c < 3; ++c) info->center[c] = h.center[c];
    info->radius = h.radius;
    info->scale = h.scale;
    info->rmax = h.rmax;
    info->bytes = h.bytes;
    info->n_active = h.n_active;
    info->exterior = h.exterior;
    info->reserved = 0;
    return EHSS_OK;
}

int ehss_source_rays(const void* scene_dev, int log2n, uint64_t seed, int64_t first, int64_t n, double* origins_dev,
                     double* directions_dev, void* stream) {
    clear_error();
    if (!scene_dev) { set_error("null scene"); return EHSS_ERR_VALUE; }
    if (log2n < 0 || log2n > 30) { set_error("log2n must be 0..30"); return EHSS_ERR_VALUE; }
    if (first < 0 || n < 0 || first + n > (1ll << log2n)) { set_error("ray range outside the sequence"); return EHSS_ERR_VALUE; }
    if (n > 0 && (!origins_dev || !directions_dev)) { set_error("null output pointer"); return EHSS_ERR_VALUE; }
    Sobol4Params p;
    sobol4_params(seed, &p);
    return launch_source_rays(scene_dev, p, first, n, origins_dev, directions_dev, as_stream(stream));
}

int ehss_trace(const void* scene_dev, int64_t n_rays, int cap, int precision, double* positions_dev,
               double* directions_dev, const int64_t* last_atom_dev, int64_t* bounces_dev, uint8_t* escaped_dev,
               uint8_t* unresolved_dev, int32_t* history_dev, uint64_t* stats_dev, void* stream) {
    clear_error();
    if (cap < 1) { set_error("Positive cap and zero/one initial collision required"); return EHSS_ERR_VALUE; }
    if (precision != EHSS_PREC_FP64 && precision != EHSS_PREC_FP32) { set_error("unknown precision %d", precision); return EHSS_ERR_VALUE; }
    if (n_rays < 0) { set_error("negative ray count"); return EHSS_ERR_VALUE; }
    if (n_rays > 0 && (!scene_dev || !positions_dev || !directions_dev || !last_atom_dev || !bounces_dev ||
                       !escaped_dev || !unresolved_dev)) {
        set_error("null pointer");
        return EHSS_ERR_VALUE;
    }
    return launch_trace_rays(scene_dev, n_rays, cap, precision, positions_dev, directions_dev, last_atom_dev,
                             bounces_dev, escaped_dev, unresolved_dev, history_dev, stats_dev, as_stream(stream));
}

int ehss_pa_anyhit(const void* scene_dev, int64_t n_rays, const double* origins_dev, const double* directions_dev,
                   const int64_t* owners_dev, uint8_t* blocked_dev, uint64_t* stats_dev, void* stream) {
    clear_error();
    if (n_rays < 0) { set_error("negative ray count"); return EHSS_ERR_VALUE; }
    if (n_rays > 0 && (!scene_dev || !origins_dev || !directions_dev || !blocked_dev)) {
        set_error("null pointer");
        return EHSS_ERR_VALUE;
    }
    return launch_pa_rays(scene_dev, n_rays, origins_dev, directions_dev, owners_dev, blocked_dev, stats_dev,
                          as_stream(stream));
}

static bool pow2_in(int64_t v, int64_t lo, int64_t hi) { return v >= lo && v <= hi && (v & (v - 1)) == 0; }

int ehss_pa_grid_workspace_bytes(int64_t n_atoms, int n_dirs, int n, uint64_t* bytes) {
    clear_error();
    if (!bytes || n_atoms < 1 || !pow2_in(n_dirs, 1, 1 << 16) || !pow2_in(n, 8, 8192)) {
        set_error("need n_atoms >= 1, n_dirs a power of two in 1..65536 and n a power of two in 8..8192");
        return EHSS_ERR_VALUE;
    }
    *bytes = grid_workspace_bytes(n_atoms, n_dirs, n);
    return EHSS_OK;
}

int ehss_pa_grid(const void* scene_dev, int64_t n_atoms, int n_dirs, uint64_t seed, int n, uint64_t* counts_dev,
                 double* spacing_dev, double* xy_dev, void* workspace_dev, uint64_t workspace_bytes, void* stream) {
    clear_error();
    if (!scene_dev || !counts_dev || !workspace_dev) { set_error("null pointer"); return EHSS_ERR_VALUE; }
    if (n_atoms < 1 || !pow2_in(n_dirs, 1, 1 << 16) || !pow2_in(n, 8, 8192)) {
        set_error("need n_atoms >= 1, n_dirs a power of two in 1..65536 and n a power of two in 8..8192");
        return EHSS_ERR_VALUE;
    }
    return launch_grid_pa(scene_dev, n_atoms, n_dirs, seed, n, reinterpret_cast<unsigned long long*>(counts_dev),
                          spacing_dev, xy_dev, workspace_dev, workspace_bytes, as_stream(stream));
}

int ehss_blocks_prepare(ehss_block* blocks, int n_blocks, const uint64_t* seeds, int chunk_rays, int64_t* total_chunks) {
    clear_error();
    if (!blocks || !seeds || !total_chunks || n_blocks < 1) { set_error("invalid arguments"); return EHSS_ERR_VALUE; }
    if (chunk_rays < 32 || chunk_rays > 4096 || (chunk_rays & (chunk_rays - 1))) {
        set_error("chunk_rays must be a power of two in 32..4096");
        return EHSS_ERR_VALUE;
    }
    int64_t total = 0, hist = 0;
    for (int b = 0; b < n_blocks; ++b) {
        ehss_block& B = blocks[b];
        if (!B.scene) { set_error("block %d: null scene", b); return EHSS_ERR_VALUE; }
        if (B.log2_rays < 3 || B.log2_rays > kMaxBlockLog2) {
            set_error("block %d: log2_rays must be 3..%d", b, kMaxBlockLog2);
            return EHSS_ERR_VALUE;
        }
        if (B.cap < 1 || B.cap > 100000) { set_error("block %d: cap must be 1..100000", b); return EHSS_ERR_VALUE; }
        if (B.precision != EHSS_PREC_FP64 && B.precision != EHSS_PREC_FP32) { set_error("block %d: unknown precision", b); return EHSS_ERR_VALUE; }
        if (!(B.flags & (EHSS_BLOCK_EHSS | EHSS_BLOCK_PA))) { set_error("block %d: no work flags", b); return EHSS_ERR_VALUE; }
        if (B.hist_offset < 0) B.hist_offset = hist;
        hist = B.hist_offset + B.cap + 1;
        uint32_t sv[4 * 30], shift[4];
        sobol_scramble(4, seeds[b], sv, shift);
        if (!sobol_coherent_order(B.log2_rays, sv, shift, &B.basis[0][0], B.base)) {
            set_error("block %d: no coherent enumeration", b);
            return EHSS_ERR_VALUE;
        }
        if (B.flags & EHSS_BLOCK_RAYS) {
            if (!B.rays || !(B.ray_scale > 0.) || !std::isfinite(B.ray_scale)) {
                set_error("block %d: ray blocks need a ray buffer and a positive ray_scale", b);
                return EHSS_ERR_VALUE;
            }
        } else {
            B.rays = nullptr;
            B.ray_scale = 0.;
        }
        if (B.flags & ~(EHSS_BLOCK_EHSS | EHSS_BLOCK_PA | EHSS_BLOCK_RAYS)) { set_error("block %d: unknown flags", b); return EHSS_ERR_VALUE; }
        B.reserved = 0;
        B.chunk_begin = total;
        int64_t n = 1ll << B.log2_rays;
        total += (n + chunk_rays - 1) / chunk_rays;
    }
    *total_chunks = total;
    return EHSS_OK;
}

int ehss_blocks_workspace_bytes(int n_blocks, uint64_t* bytes) {
    clear_error();
    if (n_blocks < 1 || !bytes) { set_error("invalid arguments"); return EHSS_ERR_VALUE; }
    *bytes = sizeof(unsigned long long) * kMaxWorkParts;
    return EHSS_OK;
}

static int trace_blocks_impl(const ehss_block* blocks_dev, int n_blocks, int64_t total_chunks,
                             ehss_block_result* results_dev, uint64_t* hist_dev, uint64_t* ledger_dev,
                             int64_t hist_entries, void* workspace_dev, uint64_t workspace_bytes,
                             const ehss_launch* launch, ehss_residual* residual_dev, int64_t residual_capacity,
                             unsigned long long* residual_count_dev, void* stream, int64_t chunk_first = 0,
                             int64_t chunk_end = -1) {
    if (!blocks_dev || n_blocks < 1 || !results_dev || !hist_dev || !ledger_dev || !workspace_dev || !launch) {
        set_error("invalid arguments");
        return EHSS_ERR_VALUE;
    }
    if (chunk_end < 0) chunk_end = total_chunks;
    if (total_chunks < 0 || chunk_first < 0 || chunk_first > chunk_end || chunk_end > total_chunks) {
        set_error("chunk window [%lld, %lld) outside the %lld prepared chunks", (long long)chunk_first,
                  (long long)chunk_end, (long long)total_chunks);
        return EHSS_ERR_VALUE;
    }
    if (workspace_bytes < sizeof(unsigned long long) * kMaxWorkParts) {
        set_error("blocks workspace must hold %zu bytes", sizeof(unsigned long long) * kMaxWorkParts);
        return EHSS_ERR_CAPACITY;
    }
    const ehss_launch& L = *launch;
    if (L.smem_stack < 0 || L.smem_stack > 32) { set_error("smem_stack must be 0..32"); return EHSS_ERR_VALUE; }
    if (L.block_threads != 64 && L.block_threads != 128) {
        set_error("block_threads must be 64 or 128");
        return EHSS_ERR_VALUE;
    }
    if (L.ctas_per_sm < 1 || L.ctas_per_sm > 16) { set_error("ctas_per_sm must be 1..16"); return EHSS_ERR_VALUE; }
    if (L.chunk_rays < 32 || L.chunk_rays > 4096 || (L.chunk_rays & (L.chunk_rays - 1))) {
        set_error("chunk_rays must be a power of two in 32..4096");
        return EHSS_ERR_VALUE;
    }
    if (L.resolve_batch < 1 || L.resolve_batch > 32) { set_error("resolve_batch must be 1..32"); return EHSS_ERR_VALUE; }
    if (L.precisions < 0 || L.precisions > 3) { set_error("precisions must be a mask of 1 and 2 (0 = both)"); return EHSS_ERR_VALUE; }
    if (L.options & ~(EHSS_LAUNCH_COUNT_TESTS | EHSS_LAUNCH_RAY_BLOCKS | EHSS_LAUNCH_NO_DISK_BLOCKS)) {
        set_error("unknown launch options 0x%x", L.options);
        return EHSS_ERR_VALUE;
    }
    cudaStream_t s = as_stream(stream);
    int rc = cuda_status(cudaMemsetAsync(results_dev, 0, sizeof(ehss_block_result) * (size_t)n_blocks, s), "result reset");
    if (!rc && hist_entries > 0) rc = cuda_status(cudaMemsetAsync(hist_dev, 0, 8ull * hist_entries, s), "hist reset");
    if (!rc && hist_entries > 0) rc = cuda_status(cudaMemsetAsync(ledger_dev, 0, 8ull * hist_entries, s), "ledger reset");
    if (!rc) rc = cuda_status(cudaMemsetAsync(workspace_dev, 0, sizeof(unsigned long long) * kMaxWorkParts, s),
                              "work counter reset");
    if (rc) return rc;
    if (residual_count_dev) {
        rc = cuda_status(cudaMemsetAsync(residual_count_dev, 0, sizeof(unsigned long long), s), "residual count reset");
        if (rc) return rc;
    }
    if (chunk_end == chunk_first) return EHSS_OK;
    return launch_blocks(blocks_dev, n_blocks, chunk_first, chunk_end - chunk_first, L, results_dev, hist_dev, ledger_dev,
                         reinterpret_cast<unsigned long long*>(workspace_dev), s, residual_dev, residual_capacity,
                         residual_count_dev);
}

int ehss_trace_blocks(const ehss_block* blocks_dev, int n_blocks, int64_t total_chunks, ehss_block_result* results_dev,
                      uint64_t* hist_dev, uint64_t* ledger_dev, int64_t hist_entries, void* workspace_dev,
                      uint64_t workspace_bytes, const ehss_launch* launch, void* stream) {
    clear_error();
    return trace_blocks_impl(blocks_dev, n_blocks, total_chunks, results_dev, hist_dev, ledger_dev, hist_entries,
                             workspace_dev, workspace_bytes, launch, nullptr, 0, nullptr, stream);
}

int ehss_trace_blocks_window(const ehss_block* blocks_dev, int n_blocks, int64_t total_chunks, int64_t chunk_first,
                             int64_t chunk_end, ehss_block_result* results_dev, uint64_t* hist_dev,
                             uint64_t* ledger_dev, int64_t hist_entries, void* workspace_dev, uint64_t workspace_bytes,
                             const ehss_launch* launch, void* stream) {
    clear_error();
    return trace_blocks_impl(blocks_dev, n_blocks, total_chunks, results_dev, hist_dev, ledger_dev, hist_entries,
                             workspace_dev, workspace_bytes, launch, nullptr, 0, nullptr, stream, chunk_first,
                             chunk_end);
}

int ehss_trace_blocks_residual(const ehss_block* blocks_dev, int n_blocks, int64_t total_chunks,
                               ehss_block_result* results_dev, uint64_t* hist_dev, uint64_t* ledger_dev,
                               int64_t hist_entries, void* workspace_dev, uint64_t workspace_bytes,
                               const ehss_launch* launch, ehss_residual* residual_dev, int64_t residual_capacity,
                               unsigned long long* residual_count_dev, void* stream) {
    clear_error();
    if (!residual_dev || residual_capacity < 1 || !residual_count_dev) {
        set_error("residual buffer, capacity >= 1 and count pointer required");
        return EHSS_ERR_VALUE;
    }
    return trace_blocks_impl(blocks_dev, n_blocks, total_chunks, results_dev, hist_dev, ledger_dev, hist_entries,
                             workspace_dev, workspace_bytes, launch, residual_dev, residual_capacity,
                             residual_count_dev, stream);
}

int ehss_extend_blocks(const ehss_block* blocks_dev, int n_blocks, const int32_t* row_dev, int rows,
                       const ehss_residual* in_dev, int64_t n_in, int new_cap, ehss_extension* ext_dev,
                       uint64_t* hist_dev, uint64_t* ledger_dev, ehss_residual* out_dev, int64_t out_capacity,
                       unsigned long long* out_count_dev, uint64_t* stats_dev, void* stream) {
    clear_error();
    if (!blocks_dev || n_blocks < 1 || !row_dev || rows < 1 || n_in < 0 || (n_in > 0 && !in_dev) || !ext_dev ||
        !hist_dev || !ledger_dev || !out_dev || out_capacity < 1 || !out_count_dev) {
        set_error("invalid arguments");
        return EHSS_ERR_VALUE;
    }
    if (new_cap < 2 || new_cap > 100000) { set_error("new_cap must be 2..100000"); return EHSS_ERR_VALUE; }
    cudaStream_t s = as_stream(stream);
    const size_t per = (size_t)(new_cap + 1) * (size_t)rows;
    int rc = cuda_status(cudaMemsetAsync(ext_dev, 0, sizeof(ehss_extension) * (size_t)rows, s), "extension reset");
    if (!rc) rc = cuda_status(cudaMemsetAsync(hist_dev, 0, 8 * per, s), "extension hist reset");
    if (!rc) rc = cuda_status(cudaMemsetAsync(ledger_dev, 0, 8 * per, s), "extension ledger reset");
    if (!rc) rc = cuda_status(cudaMemsetAsync(out_count_dev, 0, sizeof(unsigned long long), s), "residual count reset");
    if (rc) return rc;
    return launch_extend(blocks_dev, n_blocks, row_dev, rows, in_dev, n_in, new_cap, ext_dev, hist_dev, ledger_dev,
                         out_dev, out_capacity, out_count_dev, stats_dev, s);
}

}  // extern "C"
