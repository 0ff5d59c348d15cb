/*
 * ehss_b200 — C ABI of the B200 (sm_100a) PA + EHSS cross-section library.
 *
 * Every entry point returns an int status (EHSS_OK = 0) and never aborts;
 * ehss_last_error() gives the message of the calling thread's last failure.
 * Array arguments named *_dev are device pointers (any allocator: PyTorch,
 * cudaMalloc, a pool); *_host are host pointers.  `stream` is a cudaStream_t
 * passed as void* (NULL = legacy default stream).  Work is enqueued on that
 * stream; nothing synchronises unless the comment says so.
 *
 * The reference (SCIMMS/EHSS, package support_exchange_transport) exposes
 * this path as Python objects plus one native C entry point; each function
 * below names the reference interface it replaces (paths relative to the
 * reference project root).
 */
#ifndef EHSS_B200_H
#define EHSS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define EHSS_ABI_VERSION 1

/* Status codes.  EHSS_ERR_VALUE corresponds to the reference's ValueError. */
#define EHSS_OK 0
#define EHSS_ERR_VALUE 1    /* invalid argument (size, cap, identity, layout) */
#define EHSS_ERR_CUDA 2     /* a CUDA runtime call failed */
#define EHSS_ERR_CAPACITY 3 /* a buffer or workspace is too small */
#define EHSS_ERR_DEVICE 4   /* a kernel reported a bounded failure (stack/loop limit) */

/* Precision of the nearest-entry search. */
#define EHSS_PREC_FP64 0    /* every sphere test in FP64, bit-identical to the reference */
#define EHSS_PREC_FP32 1    /* FP32 traversal + tests, FP64 re-test of every candidate that
                               can be nearest (same outcomes as FP64 by construction) */

/* Per-call statistics slots (uint64 array of EHSS_NSTATS, accumulated). */
#define EHSS_STAT_BOX_TESTS 0
#define EHSS_STAT_SPHERE_TESTS 1
#define EHSS_STAT_QUERIES 2
#define EHSS_STAT_GRAZING 3      /* queries whose FP32 tangency/order margin was below the
                                    error bound, resolved by the FP64 re-test */
#define EHSS_STAT_FALLBACK 4     /* queries re-run entirely in FP64 (candidate list full) */
#define EHSS_STAT_FP64_TESTS 5   /* FP64 sphere evaluations */
#define EHSS_STAT_ERRORS 6       /* bounded device failures (must stay 0) */
#define EHSS_NSTATS 8

/* Message of the calling thread's last failed call ("" if none). */
const char* ehss_last_error(void);
int ehss_abi_version(void);

/* ------------------------------------------------------------------------ */
/* Scrambled Sobol (host).  Replaces scipy qmc.Sobol(dim, scramble=True,
 * seed=seed) as called by ehss_state.external_source
 * (src/support_exchange_transport/ehss_state.py:44) and ccs_cli.adaptive_pa
 * (ccs_cli.py:148): sv[dim*30] receives the LMS-scrambled direction numbers
 * (row j = dimension j), shift[dim] the random digital shift; point n is
 * (shift ^ XOR_{bit k of gray(n)} sv[k]) * 2^-30.  1 <= dim <= 8,
 * seed < 2^64. */
int ehss_sobol_scramble(int dim, uint64_t seed, uint32_t* sv_host, uint32_t* shift_host);

/* The same points generated on the device: q_dev[n*dim] (uint32, row-major)
 * for point indices [first, first+n).  Bit-exact to scipy's sequence. */
int ehss_sobol_points(int dim, uint64_t seed, int64_t first, int64_t n, uint32_t* q_dev, void* stream);

/* ------------------------------------------------------------------------ */
/* Scene: one structure's atoms plus a device LBVH, resident in a caller-
 * owned device buffer.  Replaces PreparedStaticCPUEHSS.__init__
 * (ehss_static.py:62-101) and SphereIndex.__init__ (pa_spatial.py:157-160):
 * the scene owns a copy of the coordinates (as the reference scene does,
 * ehss_static.py:68-69).  Results never depend on the tree.  leaf_size 1..16
 * is the LBVH leaf bound (the reference's --leaf-size only shapes its own
 * tree and has no effect on results). */
typedef struct ehss_scene_info {
    int64_t n_atoms;
    int64_t n_nodes;
    int32_t leaf_size;
    int32_t depth;            /* LBVH depth (root = 1) */
    double center[3];         /* sequential mean of the centres (ehss_state.py:46) */
    double radius;            /* impact-disk radius R (ehss_state.py:47) */
    double scale;             /* max |c_j - center| + r_j */
    double rmax;              /* largest radius */
    uint64_t bytes;           /* bytes used in the scene buffer */
    int64_t n_active;         /* atoms in the tree: n_atoms, or the exposed atoms of an exterior scene */
    int32_t exterior;         /* 1: built with EHSS_BUILD_EXTERIOR */
    int32_t reserved;
} ehss_scene_info;

/* Impact-disk radius R = max_i(|c_i - mean(c)| + r_i) * (1 + 1e-9) of host
 * arrays xyz_host[n*3], radii_host[n], computed with the operations and order
 * of the device builder (and of external_source, ehss_state.py:46-47), so a
 * caller can weight block results (pi R^2 / n per ray) without reading the
 * scene header back.  Host only. */
int ehss_enclosing_radius(int64_t n_atoms, const double* xyz_host, const double* radii_host, double* radius);

/* Bytes of the scene buffer and of the build workspace for n_atoms. */
int ehss_scene_bytes(int64_t n_atoms, int leaf_size, uint64_t* scene_bytes, uint64_t* workspace_bytes);

/* Build a scene from device arrays xyz_dev[n*3] and radii_dev[n] (float64,
 * Angstrom).  scene_dev and workspace_dev must be 256-byte aligned.  Radii
 * must be positive and finite (checked on the device; failures are reported
 * by ehss_scene_info). */
int ehss_scene_build(int64_t n_atoms, const double* xyz_dev, const double* radii_dev, int leaf_size,
                     void* scene_dev, uint64_t scene_bytes, void* workspace_dev, uint64_t workspace_bytes,
                     void* stream);

/* Scene build that allocates nothing.  No counterpart in the reference (its
 * CPU path never allocates device memory).  For callers that cannot call
 * cudaMalloc -- a plugin inside a runtime that owns the device's memory pool,
 * a process under a fixed memory budget -- it builds a scene like
 * ehss_scene_build but takes the builder's workspace from one fixed 4 MiB
 * array in device memory declared by the library (held by every GPU that
 * loads the library until exit).  The caller still passes the inputs and the
 * scene buffer.  At most EHSS_NOALLOC_MAX_ATOMS atoms (larger: EHSS_ERR_VALUE).
 * All calls on a device share the array: calls whose work overlaps on the GPU
 * race, so order them on one stream.  The first call on a device looks up the
 * array's address; make it before any stream capture. */
#define EHSS_NOALLOC_MAX_ATOMS 20000
int ehss_scene_build_noalloc(int64_t n_atoms, const double* xyz_dev, const double* radii_dev, int leaf_size,
                             void* scene_dev, uint64_t scene_bytes, void* stream);

/* Batched build: n_scenes structures in one pass of the builder kernels
 * (the batched/served forms build every admitted structure at once).
 * Arrays of device pointers and sizes are host arrays of length n_scenes. */
int ehss_scenes_workspace_bytes(int n_scenes, const int64_t* n_atoms_host, uint64_t* workspace_bytes);
int ehss_scenes_build(int n_scenes, const double* const* xyz_dev, const double* const* radii_dev,
                      const int64_t* n_atoms_host, int leaf_size, void* const* scenes_dev,
                      const uint64_t* scene_bytes_host, void* workspace_dev, uint64_t workspace_bytes,
                      void* stream);

/* Batched build with options.  No counterpart in the reference.
 * EHSS_BUILD_EXTERIOR leaves buried atoms out of the tree: an atom whose
 * whole surface lies inside other atoms (tested on geodesic sample lattices whose
 * covering radius is added to the required depth) is never the nearest entry
 * of a ray that starts outside the union of the spheres, which every
 * impact-disk ray and every EHSS bounce point does, so the fused block trace
 * (ehss_trace_blocks) gives the same outcomes on an exterior scene with fewer
 * tests.  ehss_trace and ehss_pa_anyhit take arbitrary rays and report every
 * ray of an exterior scene as an error (EHSS_STAT_ERRORS).  flags = 0 is
 * ehss_scenes_build.  The first exterior build on a device uploads the
 * sample lattices and synchronises `stream`: make it outside stream capture. */
#define EHSS_BUILD_EXTERIOR 1u
int ehss_scenes_build_ex(int n_scenes, const double* const* xyz_dev, const double* const* radii_dev,
                         const int64_t* n_atoms_host, int leaf_size, void* const* scenes_dev,
                         const uint64_t* scene_bytes_host, void* workspace_dev, uint64_t workspace_bytes,
                         uint32_t flags, void* stream);

/* Refit: new coordinates (and radii) for scenes built without
 * EHSS_BUILD_EXTERIOR, same atom count and identities, tree topology kept.
 * Replaces SphereIndex.refit (pa_spatial.py:166-170, which raises
 * ValueError('Refit requires fixed primitive identities.') for another atom
 * count) and the bottom-up box refit (_refit, pa_spatial.py:78-95;
 * parents, ehss_cpu_geometry.py:58-71).  The header (centre, R, S, rmax,
 * eps_box) and the FP32/FP64 atom records are recomputed exactly as a build
 * of the new coordinates computes them; every node box becomes the outward-
 * rounded union of its atoms' boxes under the old topology, so traversals
 * return the same (distance, id) choices as on a rebuilt scene (the tree may
 * be looser after large moves).  Same workspace as ehss_scenes_build.
 * Asynchronous like the build: a scene that is not a full scene of n_atoms
 * atoms, or new inputs with a non-positive or non-finite radius or a
 * non-finite coordinate, leave the scene invalid, reported by
 * ehss_scene_info_get. */
int ehss_scenes_refit(int n_scenes, const double* const* xyz_dev, const double* const* radii_dev,
                      const int64_t* n_atoms_host, void* const* scenes_dev, void* workspace_dev,
                      uint64_t workspace_bytes, void* stream);

/* Copy the scene header to the host (synchronises `stream`).  Fails with
 * EHSS_ERR_VALUE when the build found a non-positive or non-finite radius or
 * a non-finite coordinate, or a refit found a scene it cannot refit. */
int ehss_scene_info_get(const void* scene_dev, ehss_scene_info* info_host, void* stream);

/* ------------------------------------------------------------------------ */
/* Impact-disk source on the device.  Replaces ehss_state.external_source
 * (ehss_state.py:42-53): 2^log2n rays from Sobol(4, seed); writes origins and
 * directions (float64 [n*3]) for ray indices [first, first+n).  Each ray's
 * weight is pi*R*R/2^log2n with R from ehss_scene_info. */
int ehss_source_rays(const void* scene_dev, int log2n, uint64_t seed, int64_t first, int64_t n,
                     double* origins_dev, double* directions_dev, void* stream);

/* ------------------------------------------------------------------------ */
/* Incidence on a compact enclosing boundary.  Replaces CompactBoundary.source
 * (src/support_exchange_transport/ehss_compact_source.py:47-87): directions
 * uniform on S2 from Sobol dimensions 0-1; origins uniform over the
 * boundary's projection perpendicular to the direction, upstream of the
 * boundary (Sobol dimensions 2-3, and 4 for the box); weight = projected
 * area / 2^log2n.  The boundary (centre, rotation, semi-axes) is the one
 * CompactBoundary.fit computes (ehss_compact_source.py:24-45); the sphere
 * boundary is the impact disk of ehss_source_rays.  Writes origins and
 * directions [n*3] and weights [n] (float64) for ray indices [first, first+n). */
#define EHSS_BOUNDARY_SPHERE 0
#define EHSS_BOUNDARY_ELLIPSOID 1
#define EHSS_BOUNDARY_BOX 2
typedef struct ehss_boundary {
    int32_t kind;             /* EHSS_BOUNDARY_* */
    int32_t reserved;
    double center[3];
    double rotation[9];       /* row major; columns are the local axes */
    double axes[3];           /* semi-axes (sphere: radius in axes[0]) */
} ehss_boundary;
int ehss_compact_source_rays(const ehss_boundary* boundary_host, int log2n, uint64_t seed, int64_t first, int64_t n,
                             double* origins_dev, double* directions_dev, double* weights_dev, void* stream);

/* ------------------------------------------------------------------------ */
/* EHSS trace of explicit rays.  Replaces the reference's native entry point
 * ehss_trace (src/native/ehss_cpu.cpp:42-82) and CPUEHSSTransport.trace
 * (ehss_cpu.py:118-142): positions_dev/directions_dev [n*3] hold the source
 * origins/directions on entry and the final positions/outgoing directions on
 * return; bounces_dev holds the initial bounce count (0 or 1) on entry and the
 * collision count on return; last_atom_dev is the initial collider (-1 for
 * none).  escaped/unresolved are 0/1 bytes.  history_dev is NULL or an
 * int32 [n*cap] array that receives collider ids (-1 filled), as
 * record_history does.  stats_dev (NULL or uint64[EHSS_NSTATS]) is
 * accumulated.  cap >= 1. */
int ehss_trace(const void* scene_dev, int64_t n_rays, int cap, int precision,
               double* positions_dev, double* directions_dev, const int64_t* last_atom_dev,
               int64_t* bounces_dev, uint8_t* escaped_dev, uint8_t* unresolved_dev, int32_t* history_dev,
               uint64_t* stats_dev, void* stream);

/* BVH any-hit PA of explicit rays.  Replaces SphereIndex.query / tree_blocked
 * (pa_spatial.py:133-142, 162-164) with sphere_hit semantics
 * (inside_out_pa.py:93-101): blocked_dev[i] = 1 when ray i meets a sphere
 * other than owners_dev[i] (NULL = no owner). */
int ehss_pa_anyhit(const void* scene_dev, int64_t n_rays, const double* origins_dev, const double* directions_dev,
                   const int64_t* owners_dev, uint8_t* blocked_dev, uint64_t* stats_dev, void* stream);

/* ------------------------------------------------------------------------ */
/* Adaptive finite-grid PA.  Replaces ccs_cli.adaptive_pa (ccs_cli.py:142-160)
 * with project_grid (pa_walsh_geometry.py:171-180) and the sparse quadtree
 * count block_disks/block_count (pa_sparse_blocks.py:134-166): for direction
 * k of the n_dirs Sobol(2, seed) directions, counts_dev[k] receives the
 * number of pixels of the n x n midpoint grid covered by the union of the
 * projected atom disks (row_span's exact inequality, pa_dyadic_bitmask.py:
 * 50-61) and spacing_dev[k] (or NULL) the pixel size; the direction's area is
 * counts * spacing^2 and the PA is their mean.  xy_dev (NULL or float64
 * [n_dirs * n_atoms * 2]) receives the projected centres.  n_atoms must be
 * the scene's atom count; n_dirs and n are powers of two. */
int ehss_pa_grid_workspace_bytes(int64_t n_atoms, int n_dirs, int n, uint64_t* workspace_bytes);
int ehss_pa_grid(const void* scene_dev, int64_t n_atoms, int n_dirs, uint64_t seed, int n, uint64_t* counts_dev,
                 double* spacing_dev, double* xy_dev, void* workspace_dev, uint64_t workspace_bytes, void* stream);

/* ------------------------------------------------------------------------ */
/* Fused blocks: Sobol -> impact disk -> trace -> (1 - cos chi) reduction,
 * with no per-ray HBM traffic.  One block = one replicate of one structure
 * (the body of ccs_cli.solve_frame's repeat loop, ccs_cli.py:189-219).  The
 * same entry point serves one structure (plain path) and many structures of
 * uneven size in one persistent launch (batched path).
 *
 * Sums are kept in integer fixed point so that every block's result is
 * independent of scheduling and of what else runs in the launch:
 *   omega     = w * angle_fx * 2^-36        (w = pi R^2 / 2^log2_rays)
 *   pa (same rays) = w * hits ;  tail bound = 2 * w * unresolved
 * hist/ledger rows have cap+1 entries (bincount of bounces, unweighted and
 * weighted by the contribution in 2^-36 units). */
#define EHSS_BLOCK_EHSS 1u      /* trace EHSS */
#define EHSS_BLOCK_PA 2u        /* any-hit PA on the same rays */
#define EHSS_BLOCK_RAYS 4u      /* rays from `rays` (origins [3n], directions [3n], weights [n],
                                   float64, n = 2^log2_rays; e.g. ehss_compact_source_rays) instead
                                   of the scene's impact disk: every ray then adds its weight
                                   times ray_scale (<= 1 + 1e-9) to the weighted sums hits_fx,
                                   unresolved_fx, pa_fx and to angle_fx, and
                                   omega = angle_fx * 2^-36 / ray_scale etc. */

/* 560 bytes, a multiple of 16: the device reads basis/base as 16-byte
 * vectors, so a device array of blocks must start on a 16-byte boundary.
 * ehss_blocks_prepare fills basis/base with the block's 2^log2_rays Sobol(4)
 * points of `seed` in a spatially coherent enumeration: position p carries
 * the point (base ^ XOR_{bit e of p} basis[e]) * 2^-30.  The positions
 * 0..2^log2_rays-1 enumerate exactly the scipy point set of (seed,
 * log2_rays), reordered so that neighbouring positions share their leading
 * digits (nearby directions and impact points); block sums do not depend on
 * the order. */
typedef struct ehss_block {
    uint32_t basis[30][4];    /* per position bit, [bit][dim] (offset 0) */
    uint32_t base[4];         /* offset 480 */
    const void* scene;        /* device scene buffer */
    int32_t log2_rays;        /* 3..26 (the angle sum stays below 2^63) */
    int32_t cap;              /* collision cap >= 1 */
    int32_t precision;        /* EHSS_PREC_* */
    uint32_t flags;           /* EHSS_BLOCK_* */
    int64_t hist_offset;      /* first hist/ledger entry of this block (-1: next free) */
    int64_t chunk_begin;      /* filled by ehss_blocks_prepare */
    const double* rays;       /* EHSS_BLOCK_RAYS: device ray buffer, else NULL */
    double ray_scale;         /* EHSS_BLOCK_RAYS: 1 / (largest ray weight), else 0 */
    int64_t reserved;         /* 0 */
} ehss_block;

typedef struct ehss_block_result {
    uint64_t angle_fx;        /* sum of clip(1 - d_in.d_out, 0, 2) over escaped rays, 2^-36 units */
    uint64_t hits;            /* rays with bounces > 0 or unresolved */
    uint64_t unresolved;
    uint64_t escaped;
    uint64_t pa_blocked;      /* any-hit PA count (EHSS_BLOCK_PA) */
    uint64_t hits_fx;         /* EHSS_BLOCK_RAYS: weighted hits, unresolved rays and PA hits, */
    uint64_t unresolved_fx;   /*   each ray adding weight * ray_scale in 2^-36 units */
    uint64_t pa_fx;
    uint64_t stats[EHSS_NSTATS];
} ehss_block_result;

/* Fill seeds' scrambles and chunk offsets of host block descriptors; returns
 * the total chunk count.  chunk_rays is a power of two (32..4096). */
int ehss_blocks_prepare(ehss_block* blocks_host, int n_blocks, const uint64_t* seeds_host, int chunk_rays,
                        int64_t* total_chunks);

/* Workspace bytes for ehss_trace_blocks. */
int ehss_blocks_workspace_bytes(int n_blocks, uint64_t* bytes);

/* Launch configuration chosen by the caller or the autotuner. */
typedef struct ehss_launch {
    int32_t block_threads;    /* 64 or 128 */
    int32_t ctas_per_sm;      /* persistent CTAs per SM (grid = SMs * ctas_per_sm) */
    int32_t chunk_rays;       /* rays per work item (as passed to ehss_blocks_prepare) */
    int32_t resolve_batch;    /* a warp leaves its traversal phase once this many lanes have a
                                 finished query, and resolves them together (1..32) */
    int32_t precisions;       /* bit mask of the EHSS_PREC_* values present among the blocks
                                 (1 << EHSS_PREC_FP64 | 1 << EHSS_PREC_FP32); 0 = both */
    int32_t options;          /* EHSS_LAUNCH_* bits */
    int32_t smem_stack;       /* traversal-stack entries per lane kept in shared memory
                                 (0 = 16, max 32); deeper entries go to local memory */
    int32_t reserved;         /* 0 */
} ehss_launch;
#define EHSS_LAUNCH_COUNT_TESTS 1   /* count box and sphere tests into the block stats (slower); a block
                                       with EHSS_BLOCK_PA adds its any-hit tests to the same counters */
#define EHSS_LAUNCH_RAY_BLOCKS 2    /* some blocks have EHSS_BLOCK_RAYS (adds a launch of that kernel instance) */
#define EHSS_LAUNCH_NO_DISK_BLOCKS 4  /* with EHSS_LAUNCH_RAY_BLOCKS: every block has EHSS_BLOCK_RAYS */

/* Run all blocks in one persistent launch.  blocks_dev: device copy of the
 * prepared descriptors; results_dev[n_blocks], hist_dev/ledger_dev
 * [sum of (cap+1)] are zeroed by this call before accumulation. */
int ehss_trace_blocks(const ehss_block* blocks_dev, int n_blocks, int64_t total_chunks,
                      ehss_block_result* results_dev, uint64_t* hist_dev, uint64_t* ledger_dev,
                      int64_t hist_entries, void* workspace_dev, uint64_t workspace_bytes,
                      const ehss_launch* launch, void* stream);

/* ehss_trace_blocks over the window [chunk_first, chunk_end) of the prepared
 * chunk list only (0 <= chunk_first <= chunk_end <= total_chunks): the
 * several-GPU form of one batch.  Each GPU traces a disjoint window of the
 * same blocks; its results/hist/ledger hold the integer sums of its rays, and
 * the element-wise sum over GPUs equals the single-launch results exactly.
 * Replaces the reference's parallel loop over the rays of one structure
 * (prange, src/support_exchange_transport/ehss_cpu.py:72; OpenMP,
 * src/native/ehss_cpu.cpp:49-53) at the scale of several devices. */
int ehss_trace_blocks_window(const ehss_block* blocks_dev, int n_blocks, int64_t total_chunks, int64_t chunk_first,
                             int64_t chunk_end, ehss_block_result* results_dev, uint64_t* hist_dev,
                             uint64_t* ledger_dev, int64_t hist_entries, void* workspace_dev, uint64_t workspace_bytes,
                             const ehss_launch* launch, void* stream);

/* ------------------------------------------------------------------------ */
/* Cap extension.  The reference's production runs start at cap 512 and
 * retrace the same rays at caps 1024, 2048 and 4096 while a run's sampled
 * tail bound exceeds 0.05 % of its CCS (manuscript, Methods; the wrapper
 * itself is not in the reference tree).  Here the rays left unresolved at a
 * block's cap are saved with their full state, and only they are continued:
 * a ray continued from its saved state follows the path it would have
 * followed with the larger cap from the start, so merged totals equal a run
 * at the larger cap, bit for bit. */
typedef struct ehss_residual {
    double o[3];          /* last bounce point */
    double d[3];          /* direction leaving it */
    double din[3];        /* the ray's incoming direction */
    int32_t block;        /* index of its block in the blocks array */
    int32_t last_rank;    /* leaf-order index of the last collider */
    int32_t bounces;      /* collisions so far (the cap it stopped at) */
    int32_t reserved;
} ehss_residual;

typedef struct ehss_extension {   /* one row per extended block */
    uint64_t angle_fx;    /* angle sum (2^-36 units) of the continued rays that escaped */
    uint64_t escaped;     /* continued rays that escaped */
    uint64_t unresolved;  /* continued rays still unresolved at the new cap */
    uint64_t continued;   /* continued rays */
} ehss_extension;

/* ehss_trace_blocks that also appends every ray left unresolved to
 * residual_dev[0 .. residual_capacity) and counts them in
 * *residual_count_dev (zeroed by the call; a count above the capacity means
 * the extra rays were not saved). */
int ehss_trace_blocks_residual(const ehss_block* blocks_dev, int n_blocks, int64_t total_chunks,
                               ehss_block_result* results_dev, uint64_t* hist_dev, uint64_t* ledger_dev,
                               int64_t hist_entries, void* workspace_dev, uint64_t workspace_bytes,
                               const ehss_launch* launch, ehss_residual* residual_dev, int64_t residual_capacity,
                               unsigned long long* residual_count_dev, void* stream);

/* Continue saved rays to new_cap.  row_dev[n_blocks] (device int32) maps a
 * block to its row in ext_dev / hist_dev / ledger_dev, or -1 to leave that
 * block's rays alone.  ext_dev[rows] and hist_dev/ledger_dev[rows *
 * (new_cap + 1)] are zeroed by the call; a continued ray that escapes adds
 * its angle to its row and counts at hist[row * (new_cap + 1) + bounces], one
 * still unresolved counts at bounces = new_cap and is appended to out_dev
 * (count in *out_count_dev, zeroed by the call).  new_cap must exceed the
 * bounce count of every continued ray.  stats_dev: NULL or uint64[EHSS_NSTATS]. */
int ehss_extend_blocks(const ehss_block* blocks_dev, int n_blocks, const int32_t* row_dev, int rows,
                       const ehss_residual* in_dev, int64_t n_in, int new_cap, ehss_extension* ext_dev,
                       uint64_t* hist_dev, uint64_t* ledger_dev, ehss_residual* out_dev, int64_t out_capacity,
                       unsigned long long* out_count_dev, uint64_t* stats_dev, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EHSS_B200_H */
