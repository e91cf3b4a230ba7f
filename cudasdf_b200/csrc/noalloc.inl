// Allocation-free active-block scout (included at the end of sdfmesh.cu).
//
// launchScoutActiveBlocks obtains its working memory (per-block flags, the compaction's scan status
// words, a diagnostics word) from cudaMalloc the first time it sees a grid of a given size. Some
// callers cannot let a library allocate: a renderer's per-frame loop or a plugin host that forbids
// device allocation while it runs (cudaMalloc and cudaFree synchronise the whole device and can fail
// when the host application owns a fixed memory budget), or an application that routes every device
// allocation through its own allocator. sdf_scout_active_blocks_static gives them the same scout with
// its working memory in one statically sized device array that lives in this library's module.
//
// Properties a caller has to know:
//  * The array holds at most kStaticScoutMaxBlocks blocks; larger grids are rejected with
//    SDF_ERR_CAPACITY before anything is launched.
//  * Each device that loads the library keeps the array (a little over 4 MiB) until the process exits.
//  * The first call on a device looks the array up for that device (cudaGetSymbolAddress, with that
//    device current); make that first call before any stream capture on that device. The address is
//    kept for the life of the process: after cudaDeviceReset on a device the module is loaded again
//    and the kept address is stale, so this entry point must not be called on that device again in
//    the same process (the library's other device memory, like every caller's, is gone too).
//  * All calls share the one array and it keeps the last call's contents; each call clears the parts
//    that must start at zero. Calls whose work overlaps on the GPU (two streams, two host threads
//    without ordering) race on the array: order them.
//  * It allocates nothing: no cudaMalloc, no cudaFree, no allocating library call.

namespace sdfb {

constexpr unsigned kStaticScoutMaxBlocks = SDF_SCOUT_STATIC_MAX_BLOCKS;  // 1,048,576 8^3 blocks, e.g. 1024 x 1024 x 512
static_assert(kStaticScoutMaxBlocks == (1u << 20), "the header's stated limit");
constexpr unsigned kStaticScoutTiles = (kStaticScoutMaxBlocks + SCAN_TILE - 1) / SCAN_TILE;
constexpr size_t kStaticStatusBytes = (size_t)(kStaticScoutTiles + 1) * sizeof(unsigned long long);
constexpr size_t kStaticDiagOffset = (kStaticStatusBytes + 255) & ~size_t(255);
constexpr size_t kStaticFlagsOffset = (kStaticDiagOffset + sizeof(Diag) + 255) & ~size_t(255);
constexpr size_t kStaticScoutBytes = kStaticFlagsOffset + (size_t)kStaticScoutMaxBlocks * sizeof(unsigned);

// The working memory. In host code this name is only a stand-in for the symbol: its device address
// comes from cudaGetSymbolAddress below, once per device.
static __device__ __align__(256) unsigned char g_static_scout_scratch[kStaticScoutBytes];

static unsigned char* g_static_scout_base[16];  // device address of the array, per device

}  // namespace sdfb

extern "C" sdf_status sdf_scout_active_blocks_static(sdf_grid* grid, float time) {
    using namespace sdfb;
    if (!grid || !grid->d_activeBlocks || !grid->d_activeBlockCount) return SDF_ERR_INVALID;
    const long long nblocks = (long long)grid->blocksDim[0] * grid->blocksDim[1] * grid->blocksDim[2];
    if (nblocks <= 0) return SDF_ERR_INVALID;
    if (nblocks > (long long)kStaticScoutMaxBlocks) return SDF_ERR_CAPACITY;
    std::lock_guard<std::mutex> lk(g_mutex);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        record(e);
        return SDF_ERR_CUDA;
    }
    if (dev < 0 || dev >= 16) return SDF_ERR_INVALID;
    if (!g_static_scout_base[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_static_scout_scratch);
        if (e != cudaSuccess || !p) {
            record(e);
            return SDF_ERR_CUDA;
        }
        g_static_scout_base[dev] = static_cast<unsigned char*>(p);
    }
    unsigned char* base = g_static_scout_base[dev];
    g_scratch[dev & 15].rows_valid = false;  // the active list is rewritten: drop-in field rows are stale
    unsigned long long* status = reinterpret_cast<unsigned long long*>(base);
    Diag* diag = reinterpret_cast<Diag*>(base + kStaticDiagOffset);
    unsigned* flags = reinterpret_cast<unsigned*>(base + kStaticFlagsOffset);
    // the scan's ticket and status words are cleared inside run_scout_compact; the diagnostics here
    e = cudaMemsetAsync(diag, 0, sizeof(Diag), 0);
    if (e != cudaSuccess) {
        record(e);
        return SDF_ERR_CUDA;
    }
    // run_scout_compact reports the first error of its two launches and its memset (a refused launch
    // leaves the active list and count unwritten)
    e = run_scout_compact(grid_view(*grid), scene_view(*grid), time, flags, status, grid->d_activeBlocks,
                          grid->d_activeBlockCount, diag, 0);
    return e == cudaSuccess ? SDF_OK : SDF_ERR_CUDA;
}
