// Scene build that allocates nothing: for callers that may not call
// cudaMalloc.
//
// Some hosts of this library cannot allocate device memory on their own: a
// plugin running inside another runtime whose memory pool owns the device, a
// process under a strict memory budget set by its host application, or code
// that must not allocate while a CUDA graph is being recorded elsewhere.  They
// can still pass their own input arrays (coordinates, radii) and their own
// output buffer (the scene), but not the builder's workspace.  This variant
// takes that workspace from one fixed array in device memory that the library
// declares at file scope: every GPU that loads the library holds it (4 MiB)
// until the process exits.
//
// Limits and sharing rules:
//   * at most EHSS_NOALLOC_MAX_ATOMS atoms per call; larger structures are
//     rejected with EHSS_ERR_VALUE and a message (use ehss_scene_build);
//   * every call on a device uses the same array, which keeps what the last
//     call left there; the builder resets what must start at a known value
//     (arrival counters to zero, parent links to -1) on every call;
//   * two calls whose work overlaps on the GPU (different streams, or
//     different host threads without ordering) race on that array: order
//     them on one stream;
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins.  The address is kept per device and
//     per CUDA context: after the context is torn down (cudaDeviceReset) the
//     next call notices the new context and looks the address up again, so
//     that call, too, belongs before any capture.
#include <mutex>
#include "ehss_internal.cuh"

namespace ehss {

constexpr uint64_t kNoAllocScratchBytes = 4ull << 20;

// One fixed workspace per device.  In host code this name is only a handle
// for the runtime, not a device address: the address comes from
// cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_ptr[kMaxDevices] = {nullptr};
unsigned long long g_noalloc_ctx[kMaxDevices] = {0};

// The address belongs to the device's context at the time of the lookup.  A
// context that is torn down (cudaDeviceReset, or a driver-API caller
// destroying it) takes the mapping with it, and the next context may map the
// array elsewhere.  Each call therefore compares the current context's id
// (cuCtxGetId: unique within the process, never reused) with the id recorded
// at the lookup and looks the address up again when they differ.  Both driver
// functions come through the runtime's entry-point query, so the library
// does not link the driver library itself; without them every call looks the
// address up.
using CtxGetCurrentFn = int (*)(void**);
using CtxGetIdFn = int (*)(void*, unsigned long long*);

bool current_context_id(unsigned long long* id) {
    static bool tried = false;
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!tried) {
        tried = true;
        cudaDriverEntryPointQueryResult q1, q2;
        const bool ok1 = cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", (void**)&get_current, 12000,
                                                          cudaEnableDefault, &q1) == cudaSuccess &&
                         q1 == cudaDriverEntryPointSuccess;
        const bool ok2 = cudaGetDriverEntryPointByVersion("cuCtxGetId", (void**)&get_id, 12000, cudaEnableDefault,
                                                          &q2) == cudaSuccess &&
                         q2 == cudaDriverEntryPointSuccess;
        if (!ok1 || !ok2) {
            get_current = nullptr;
            get_id = nullptr;
            cudaGetLastError();   // a failed query is not the caller's error
        }
    }
    void* ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx) return false;
    return get_id(ctx, id) == 0 && *id != 0;
}

// Device address of the scratch array for the current device: looked up
// with that device current, at the device's first call and again after its
// context has changed.
int noalloc_scratch(void** out) {
    int dev = 0;
    int rc = cuda_status(cudaGetDevice(&dev), "current device");
    if (rc) return rc;
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device ordinal %d outside 0..%d", dev, kMaxDevices - 1);
        return EHSS_ERR_VALUE;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    unsigned long long id = 0;
    const bool known = current_context_id(&id);
    if (!known || !g_noalloc_ptr[dev] || g_noalloc_ctx[dev] != id) {
        void* p = nullptr;
        rc = cuda_status(cudaGetSymbolAddress(&p, g_noalloc_scratch), "scratch symbol address");
        if (rc) return rc;
        g_noalloc_ptr[dev] = p;
        // the lookup creates the primary context when none was current yet
        g_noalloc_ctx[dev] = current_context_id(&id) ? id : 0;
    }
    *out = g_noalloc_ptr[dev];
    return EHSS_OK;
}
}  // namespace

}  // namespace ehss

using namespace ehss;

extern "C" int ehss_scene_build_noalloc(int64_t n_atoms, const double* xyz_dev, const double* radii_dev,
                                        int leaf_size, void* scene_dev, uint64_t scene_bytes, void* stream) {
    set_error("%s", "");
    if (!xyz_dev || !radii_dev || !scene_dev) {
        set_error("null pointer");
        return EHSS_ERR_VALUE;
    }
    if (n_atoms < 1 || n_atoms > EHSS_NOALLOC_MAX_ATOMS) {
        set_error("ehss_scene_build_noalloc takes 1..%d atoms, got %lld; use ehss_scene_build for larger structures",
                  EHSS_NOALLOC_MAX_ATOMS, (long long)n_atoms);
        return EHSS_ERR_VALUE;
    }
    uint64_t need = build_workspace_bytes(n_atoms, 1);
    if (need > kNoAllocScratchBytes) {
        set_error("build of %lld atoms needs %llu bytes of scratch, the fixed array holds %llu", (long long)n_atoms,
                  (unsigned long long)need, (unsigned long long)kNoAllocScratchBytes);
        return EHSS_ERR_VALUE;
    }
    void* scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    return build_scenes(1, &xyz_dev, &radii_dev, &n_atoms, leaf_size, &scene_dev, &scene_bytes, scratch,
                        kNoAllocScratchBytes, reinterpret_cast<cudaStream_t>(stream));
}
