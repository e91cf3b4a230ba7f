// sdf_engine: the fused extraction pipeline (included at the end of sdfmesh.cu).
//
// Marching cubes:   scout -> compact -> block field (+ per-block vertex totals) -> scan of the block
//                   totals -> emission from the stored fields
// Dual contouring:  scout -> compact -> block map -> mark (+ stored fields) -> scan of has-vertex ->
//                   solve -> count quads (+ block totals) -> scan of block totals -> quads
// All stages run back to back on one stream; the active count stays on the device (persistent CTAs
// read it), so the only host synchronisation is the final read-back of the counts.
#include <chrono>

namespace sdfb {

// control block on the device, zeroed by one memset per extraction
struct Ctrl {
    int active_count;
    unsigned tickets[12];
    unsigned total_vertices;
    unsigned dc_vertices;
    unsigned halo_misses;  // listed halo samples of the block field (k_field_plan)
    unsigned welded_vertices;  // indexed marching-cubes output: vertices (one per owned crossed edge)
    unsigned herm[2];          // dual contouring: Hermite samples and representatives listed (k_dc_hermite_reps)
    Diag diag;
};

// learned-surrogate state of an engine (device parameters, optimiser moments, work buffers)
struct SurrogateState {
    float* theta = nullptr;
    float* m1 = nullptr;
    float* m2 = nullptr;
    __nv_bfloat16* wbf = nullptr;
    float* freq = nullptr;
    float* partial = nullptr;       // per-CTA gradient partials
    int partial_rows = 0;
    float* loss_partial = nullptr;
    float* grad = nullptr;
    int* error = nullptr;
    float* coarse_f = nullptr;      // f_net at the coarse block centres
    size_t coarse_cap = 0;
    unsigned long long* counters = nullptr;  // audit counters
    float io[7] = {0.f, 0.f, 0.f, 1.f, 1.f, 1.f, 0.25f};
    bool has_params = false;
    bool certified = false;
    bool enabled = false;
    bool exact_coarse = false;      // cull by the exact map() at the coarse centres, not by f_net
    float exact_extra = 0.f;        // the exact mode's margin beyond the reach
    float eps = 0.f;
    float slack_cells = 2.f;

    ~SurrogateState() {
        void* ptrs[] = {theta, m1, m2, wbf, freq, partial, loss_partial, grad, error, coarse_f, counters};
        for (void* p : ptrs)
            if (p) cudaFree(p);
    }
    sur::NetView view() const {
        sur::NetView v;
        v.theta = theta;
        v.wbf = wbf;
        v.freq = freq;
        v.cx = io[0]; v.cy = io[1]; v.cz = io[2];
        v.sx = io[3]; v.sy = io[4]; v.sz = io[5];
        v.clamp = io[6];
        return v;
    }
};

// coarse blocks of the culled scout: 4 x 4 x 4 blocks of 8^3 cells (32^3 cells), two scout bricks
constexpr int SUR_SPAN_BLOCKS = 4;
constexpr int SUR_SPAN_CELLS = 8 * SUR_SPAN_BLOCKS;

struct EngineImpl {
    int device = 0;
    sdf_config cfg;
    bool configured = false;
    GridView gv;
    int nblocks = 0;
    // scene
    std::vector<sdf_primitive> sorted;
    std::vector<sdf_bvh_node> nodes;
    int nbvh = 0;
    int depth = 0;
    int nprims = 0;                      // primitives on the device (sorted: unions first)
    int nnodes = 0;                      // BVH nodes on the device
    bool device_scene = false;           // the scene was built on the GPU (no host copy)
    unsigned char* bvh_work = nullptr;   // GPU BVH build: work arrays and control block
    size_t bvh_work_cap = 0;             // primitives the work arrays hold
    sdfb::bvhd::Ctl* h_bvh_ctl = nullptr;  // pinned read-back of the build's control block
    sdf_primitive* d_prims = nullptr;
    size_t prims_cap = 0;
    sdf_bvh_node* d_nodes = nullptr;
    size_t nodes_cap = 0;
    // pipeline
    unsigned* flags = nullptr;
    int* list = nullptr;
    float* fields = nullptr;
    unsigned* block_totals = nullptr;
    unsigned* block_offsets = nullptr;
    unsigned* packet_counts = nullptr;   // per cell: MC debug output / DC has-vertex + quad counts
    unsigned* packet_offsets = nullptr;  // per cell: MC debug output
    int* b2a = nullptr;
    unsigned char* masks = nullptr;
    unsigned* dc_voff = nullptr;
    ushort4* dc_verts = nullptr;
    short4* dc_norms = nullptr;
    size_t dc_cap = 0;
    float4* dc_qef = nullptr;              // debug bit 1: mass-point QEF vertices before projection
    size_t dc_qef_cap = 0;
    float4* dc_proj = nullptr;             // mass-point projection records (k_dc_project), 2 per vertex
    float4* dc_proj_nsum = nullptr;        //   and the Hermite normal sums when cell normals are kept
    size_t dc_proj_cap = 0, dc_proj_nsum_cap = 0;
    unsigned last_dc_vertices = 0;         // DC vertices of the last collected extraction
    // Hermite normals across blocks: per sample its representative, per representative the edge point
    // and the normal, per active block the first sample and representative
    unsigned* dc_hsamp = nullptr;
    float4* dc_hreps = nullptr;
    float4* dc_hnorm = nullptr;
    int4* dc_hbase = nullptr;
    size_t dc_hsamp_cap = 0, dc_hrep_cap = 0, dc_hbase_cap = 0;
    unsigned last_herm[2] = {0u, 0u};
    // quads' winding normals across blocks: per counted quad (active block, cell << 2 | axis) and normal
    uint2* dc_qrec = nullptr;
    float4* dc_qnorm = nullptr;
    size_t dc_qcap = 0;
    unsigned last_total_vertices = 0;
    unsigned char* ctrl_region = nullptr;  // Ctrl, then the three scan regions
    size_t ctrl_bytes = 0;
    size_t scanA_off = 0, scanB_off = 0, scanD_off = 0, scanC_off = 0;
    // indexed marching-cubes output: per active block, owned-edge bitmaps, word prefixes, totals, bases
    unsigned* weld_bits = nullptr;
    unsigned short* weld_prefix = nullptr;
    unsigned* weld_totals = nullptr;
    unsigned* weld_base = nullptr;
    size_t weld_cap = 0;
    Ctrl* h_ctrl = nullptr;                // pinned read-back, one Ctrl per extraction slot
    // extractions in flight (sdf_engine_extract_async): each slot owns a read-back Ctrl and an event
    struct Pending {
        bool used = false;
        uint64_t ticket = 0;
        cudaEvent_t done = nullptr;
        int nb = 0;
        int rows_cap = 0;                  // active blocks the per-block buffers held
        bool dc = false, welded = false, culled = false;
        uint32_t max_vertices = 0;
        size_t dc_cap = 0;
        std::chrono::high_resolution_clock::time_point t0;
        // what to run again when the extraction finds more active blocks than rows_cap
        sdf_outputs out{};
        float time = 0.f;
        cudaStream_t stream = nullptr;
    };
    static constexpr int ASYNC_SLOTS = 4;
    Pending pend[ASYNC_SLOTS];
    uint64_t next_ticket = 0;
    // pinned image of the uploaded scene (sdf_engine_set_scene_async uploads from it in stream order)
    sdf_primitive* h_scene_prims = nullptr;
    size_t h_scene_prims_cap = 0;
    sdf_bvh_node* h_scene_nodes = nullptr;
    size_t h_scene_nodes_cap = 0;
    cudaEvent_t scene_ev = nullptr;        // the last upload from the image
    bool scene_ev_pending = false;
    uint64_t scene_gen = 0;                // host scene builds so far
    uint64_t image_gen = ~0ull;            // the build the pinned image holds
    bool timing = false;
    int debug = 0;
    // active blocks the per-active-block buffers hold (block-field rows, halo-miss list, cell words,
    // per-cell DC arrays, weld bitmaps); grown after an extraction that found more (engine_grow_rows)
    int rows_cap = 0;
    cudaEvent_t ev[8] = {};
    // the halo misses run on a second stream beside the own samples (they write other row entries and
    // both need only the plan): the miss kernel's CTAs take the SMs the own-sample kernel's last wave frees
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    size_t packet_cap = 0;
    unsigned* miss = nullptr;          // listed halo samples, capacity nblocks * HALO_N
    size_t miss_cap = 0;
    unsigned* cell_words = nullptr;    // flat emission: one word per cell of every active block
    size_t cell_words_cap = 0;
    Diag* eval_diag = nullptr;
    std::vector<sdf_primitive> scene;  // the primitives as given (the surrogate's surface run uses them)
    SurrogateState* sur = nullptr;

    ~EngineImpl() { release(); }

    void release() {
        void* ptrs[] = {d_prims, d_nodes, flags, list, fields, block_totals, block_offsets, packet_counts,
                        packet_offsets, b2a, masks, dc_voff, dc_verts, dc_norms, ctrl_region, eval_diag, miss,
                        cell_words, bvh_work, weld_bits, weld_prefix, weld_totals, weld_base, dc_qef,
                        dc_proj, dc_proj_nsum, dc_hsamp, dc_hreps, dc_hnorm, dc_hbase, dc_qrec, dc_qnorm};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        d_prims = nullptr; d_nodes = nullptr; flags = nullptr; list = nullptr; fields = nullptr;
        block_totals = nullptr; block_offsets = nullptr; packet_counts = nullptr; packet_offsets = nullptr;
        b2a = nullptr; masks = nullptr; dc_voff = nullptr; dc_verts = nullptr; dc_norms = nullptr;
        ctrl_region = nullptr;
        eval_diag = nullptr;
        miss = nullptr;
        cell_words = nullptr;
        bvh_work = nullptr;
        weld_bits = nullptr; weld_prefix = nullptr; weld_totals = nullptr; weld_base = nullptr;
        weld_cap = 0;
        dc_qef = nullptr;
        dc_qef_cap = 0;
        dc_proj = dc_proj_nsum = nullptr;
        dc_proj_cap = dc_proj_nsum_cap = 0;
        dc_hsamp = nullptr;
        dc_hreps = dc_hnorm = nullptr;
        dc_hbase = nullptr;
        dc_hsamp_cap = dc_hrep_cap = dc_hbase_cap = 0;
        dc_qrec = nullptr;
        dc_qnorm = nullptr;
        dc_qcap = 0;
        prims_cap = nodes_cap = dc_cap = packet_cap = miss_cap = cell_words_cap = bvh_work_cap = 0;
        if (h_bvh_ctl) cudaFreeHost(h_bvh_ctl);
        h_bvh_ctl = nullptr;
        if (h_ctrl) cudaFreeHost(h_ctrl);
        h_ctrl = nullptr;
        for (auto& pd : pend)
            if (pd.done) { cudaEventDestroy(pd.done); pd.done = nullptr; pd.used = false; }
        if (h_scene_prims) cudaFreeHost(h_scene_prims);
        if (h_scene_nodes) cudaFreeHost(h_scene_nodes);
        h_scene_prims = nullptr; h_scene_nodes = nullptr;
        h_scene_prims_cap = h_scene_nodes_cap = 0;
        if (scene_ev) { cudaEventDestroy(scene_ev); scene_ev = nullptr; }
        scene_ev_pending = false;
        for (auto& e : ev)
            if (e) { cudaEventDestroy(e); e = nullptr; }
        if (fork_ev) { cudaEventDestroy(fork_ev); fork_ev = nullptr; }
        if (join_ev) { cudaEventDestroy(join_ev); join_ev = nullptr; }
        if (side) { cudaStreamDestroy(side); side = nullptr; }
        delete sur;
        sur = nullptr;
    }
};

template <class T>
static sdf_status dev_alloc(T*& p, size_t count) {
    if (p) cudaFree(p);
    p = nullptr;
    if (count == 0) count = 1;
    if (cudaMalloc((void**)&p, count * sizeof(T)) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        return SDF_ERR_NOMEM;
    }
    return SDF_OK;
}

}  // namespace sdfb

struct sdf_engine {
    sdfb::EngineImpl impl;
};

using sdfb::EngineImpl;

static sdf_status engine_ensure_packets(EngineImpl& E, size_t cells) {
    if (E.packet_cap >= cells) return SDF_OK;
    sdf_status s = sdfb::dev_alloc(E.packet_counts, cells);
    if (s == SDF_OK) s = sdfb::dev_alloc(E.packet_offsets, cells);
    if (s == SDF_OK) s = sdfb::dev_alloc(E.masks, cells);
    if (s == SDF_OK) s = sdfb::dev_alloc(E.dc_voff, cells);
    E.packet_cap = s == SDF_OK ? cells : 0;
    return s;
}

// the grid-dependent part K of the cull margin: coarse half-diagonal + scout radius + slack
static float surrogate_reach(const EngineImpl& E, float slack_cells) {
    using namespace sdfb;
    const float cell = E.gv.cell;
    const float r_scout = (8 * 0.5f * 1.73205f + 2.0f) * cell;
    return 0.5f * (float)SUR_SPAN_CELLS * 1.7320508f * cell + r_scout + slack_cells * cell;
}

// the cull threshold on |f| at a coarse centre: the certified error plus the reach, or the reach alone
// when the coarse field is the exact map()
static float surrogate_margin(const EngineImpl& E) {
    return (E.sur->exact_coarse ? E.sur->exact_extra : E.sur->eps) + surrogate_reach(E, E.sur->slack_cells);
}

// the block field with shared halos (plan -> evaluation -> gather, see mc_kernels.cuh) and the block totals
template <bool COUNT>
static sdf_status run_block_field(EngineImpl& E, const sdfb::SceneView& sv, float time, const sdfb::ActiveView& av,
                                  sdfb::Ctrl* ctrl, unsigned* packet_counts, cudaStream_t st,
                                  unsigned* cell_words = nullptr, bool counts = true) {
    using namespace sdfb;
    const size_t need = (size_t)E.rows_cap * HALO_N;
    if (E.miss_cap < need) {
        if (dev_alloc(E.miss, need) != SDF_OK) {
            E.miss_cap = 0;
            return SDF_ERR_NOMEM;
        }
        E.miss_cap = need;
    }
    k_field_plan<<<num_sms() * 8, 256, 0, st>>>(E.gv, av, E.flags, E.fields, E.b2a, E.miss, &ctrl->halo_misses);
    check_launch();
    // own samples on the extraction's stream, then the halo misses beside them on the second stream
    const bool fork = E.side && E.fork_ev && E.join_ev;
    if (fork) {
        record(cudaEventRecord(E.fork_ev, st));
        record(cudaStreamWaitEvent(E.side, E.fork_ev, 0));
    }
    k_field_own<COUNT><<<persistent_grid(k_field_own<COUNT>, BLK_THREADS, E.rows_cap), BLK_THREADS, 0, st>>>(
        E.gv, sv, time, av, E.fields, &ctrl->tickets[0], &ctrl->diag);
    check_launch();
    k_field_miss<COUNT><<<persistent_grid(k_field_miss<COUNT>, BLK_THREADS, 1 << 30), BLK_THREADS, 0,
                          fork ? E.side : st>>>(E.gv, sv, time, av, E.fields, E.miss, &ctrl->halo_misses,
                                                &ctrl->tickets[4], &ctrl->diag);
    check_launch();
    if (fork) {
        record(cudaEventRecord(E.join_ev, E.side));
        record(cudaStreamWaitEvent(st, E.join_ev, 0));
    }
    if (E.timing) cudaEventRecord(E.ev[5], st);  // the gather: halos, case codes, counts
    k_field_gather<<<persistent_grid(k_field_gather, BLK_THREADS, (E.rows_cap + GATHER_WARPS - 1) / GATHER_WARPS),
                     BLK_THREADS, 0, st>>>(E.gv, av, E.fields, E.b2a, E.flags,
                                           (COUNT || !counts) ? nullptr : E.block_totals, packet_counts, cell_words);
    check_launch();
    return SDF_OK;
}

static void coarse_dims(const EngineImpl& E, int& cx, int& cy, int& cz) {
    using namespace sdfb;
    cx = (E.gv.bx + SUR_SPAN_BLOCKS - 1) / SUR_SPAN_BLOCKS;
    cy = (E.gv.by + SUR_SPAN_BLOCKS - 1) / SUR_SPAN_BLOCKS;
    cz = (E.gv.bz + SUR_SPAN_BLOCKS - 1) / SUR_SPAN_BLOCKS;
}

static sdfb::SceneView engine_scene_view(EngineImpl& E) {
    sdfb::SceneView sv;
    sv.prims = reinterpret_cast<const float4*>(E.d_prims);
    sv.nodes = reinterpret_cast<const float4*>(E.d_nodes);
    sv.nprims = E.nprims;
    sv.nbvh = E.nbvh;
    sv.nnodes = E.nnodes;
    return sv;
}

// the exact map() at the coarse block centres (the culling without the network)
__global__ void __launch_bounds__(sdfb::BLK_THREADS) k_coarse_exact(sdfb::SceneView sc, sur::CoarseCentres cc,
                                                                     float time, float* __restrict__ out,
                                                                     sdfb::Diag* diag) {
    using namespace sdfb;
    const int warps_total = (gridDim.x * blockDim.x) >> 5;
    const int lane = threadIdx.x & 31;
    for (int base = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; base < cc.n; base += warps_total * 32) {
        const int i = base + lane;
        const bool valid = i < cc.n;
        const float3 p = valid ? cc(i) : f3(0.f, 0.f, 0.f);
        MapState<false> st;
        map_warp<false>(sc, p, valid, time, st, diag);
        if (valid) out[i] = st.d;
    }
}

// f_net (or, in the exact mode, map()) at the coarse block centres into E.sur->coarse_f
static sdf_status surrogate_coarse_eval(EngineImpl& E, cudaStream_t st, float time = 0.f) {
    using namespace sdfb;
    SurrogateState& S = *E.sur;
    int cx, cy, cz;
    coarse_dims(E, cx, cy, cz);
    const size_t nc = (size_t)cx * cy * cz;
    if (S.coarse_cap < nc) {
        if (dev_alloc(S.coarse_f, nc) != SDF_OK) return SDF_ERR_NOMEM;
        S.coarse_cap = nc;
    }
    sur::CoarseCentres cc;
    cc.ox = E.gv.ox; cc.oy = E.gv.oy; cc.oz = E.gv.oz; cc.cell = E.gv.cell;
    cc.cx = cx; cc.cy = cy; cc.cz = cz; cc.span = SUR_SPAN_CELLS;
    cc.n = (int)nc;
    if (S.exact_coarse) {
        const int warps = (int)((nc + 31) / 32);
        k_coarse_exact<<<std::max(1, std::min((warps + 7) / 8, num_sms() * 8)), BLK_THREADS, 0, st>>>(
            engine_scene_view(E), cc, time, S.coarse_f, &reinterpret_cast<Ctrl*>(E.ctrl_region)->diag);
        check_launch();
        return SDF_OK;
    }
    const size_t smem = sizeof(sur::InferSmem);
    const int tiles = (int)((nc + sur::TILE - 1) / sur::TILE);
    sur::k_sur_infer<sur::CoarseCentres><<<persistent_grid(sur::k_sur_infer<sur::CoarseCentres>, sur::TILE, tiles, smem),
                                      sur::TILE, smem, st>>>(S.view(), cc, S.coarse_f, S.error);
    check_launch();
    return SDF_OK;
}

// the scout of run_scout_compact, skipping the coarse blocks the surrogate culls
static void run_culled_scout_compact(EngineImpl& E, const sdfb::SceneView& sv, float time, unsigned long long* status,
                                     sdfb::Ctrl* ctrl, cudaStream_t st) {
    using namespace sdfb;
    const GridView& gv = E.gv;
    surrogate_coarse_eval(E, st, time);
    const int nbricks = scout_single_bricks(gv);
    const int warps_per_cta = BLK_THREADS / 32;
    k_scout_t<true><<<persistent_grid(k_scout_t<true>, BLK_THREADS, (nbricks + warps_per_cta - 1) / warps_per_cta),
                      BLK_THREADS, 0, st>>>(gv, sv, time, E.flags, &ctrl->diag, E.sur->coarse_f, surrogate_margin(E),
                                            &ctrl->tickets[10]);
    check_launch();
    const unsigned tiles = scan_tiles((unsigned)E.nblocks);
    k_compact<<<std::max(1u, tiles), SCAN_THREADS, 0, st>>>(E.flags, (unsigned)E.nblocks, E.list, &ctrl->active_count,
                                                          scan_state(status), &ctrl->diag);
    check_launch();
}

extern "C" {

sdf_status sdf_engine_create(sdf_engine** out, int device) {
    if (!out) return SDF_ERR_INVALID;
    *out = nullptr;
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return SDF_ERR_CUDA;
    sdf_engine* e = new sdf_engine();
    cudaGetDevice(&e->impl.device);
    if (cudaMallocHost(&e->impl.h_ctrl, sizeof(sdfb::Ctrl) * EngineImpl::ASYNC_SLOTS) != cudaSuccess) {
        delete e;
        return SDF_ERR_NOMEM;
    }
    for (auto& ev : e->impl.ev) cudaEventCreate(&ev);
    for (auto& pd : e->impl.pend) cudaEventCreateWithFlags(&pd.done, cudaEventDisableTiming);
    cudaEventCreateWithFlags(&e->impl.scene_ev, cudaEventDisableTiming);
    // without the second stream or its events the halo misses run after the own samples on one stream
    if (cudaStreamCreateWithFlags(&e->impl.side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->impl.fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->impl.join_ev, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        if (e->impl.side) cudaStreamDestroy(e->impl.side);
        e->impl.side = nullptr;
    }
    *out = e;
    return SDF_OK;
}

void sdf_engine_destroy(sdf_engine* e) {
    if (!e) return;
    cudaSetDevice(e->impl.device);
    delete e;
}

void sdf_engine_set_timing(sdf_engine* e, int enabled) {
    if (e) e->impl.timing = enabled != 0;
}

// debug bit 0: also write the per-cell counts/offsets of the drop-in layout (marching cubes);
// debug bit 1: keep each mass-point QEF vertex before its projection steps (buffer 11, float4 per DC
// vertex, w = 1 where the cell was solved in FP64); debug bit 2: dual contouring with cross-block lists
// of a few hundred entries (tests of the in-block paths beside the listed ones)
void sdf_engine_set_debug(sdf_engine* e, int flags) {
    if (e) e->impl.debug = flags;
}

sdf_status sdf_engine_configure(sdf_engine* e, const sdf_config* cfg) {
    if (!e || !cfg) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    cudaSetDevice(E.device);
    if (!(cfg->cell_size > 0.f)) return SDF_ERR_INVALID;
    float size[3];
    for (int k = 0; k < 3; ++k) {
        size[k] = cfg->bounds_max[k] - cfg->bounds_min[k];
        if (!(size[k] > 0.f)) return SDF_ERR_INVALID;
    }
    // CudaSDFMesh::Initialize (CudaSDFMesh.cpp:107-129): samples per axis and blocks per axis
    const unsigned w = (unsigned)ceilf(size[0] / cfg->cell_size);
    const unsigned h = (unsigned)ceilf(size[1] / cfg->cell_size);
    const unsigned d = (unsigned)ceilf(size[2] / cfg->cell_size);
    if ((unsigned long long)w * h * d > 8589934592ULL) return SDF_ERR_INVALID;
    sdfb::GridView gv;
    gv.w = (int)w; gv.h = (int)h; gv.d = (int)d;
    gv.bx = (int)((w + 7) / 8); gv.by = (int)((h + 7) / 8); gv.bz = (int)((d + 7) / 8);
    gv.ox = cfg->bounds_min[0]; gv.oy = cfg->bounds_min[1]; gv.oz = cfg->bounds_min[2];
    gv.cell = cfg->cell_size;
    const long long nb = (long long)gv.bx * gv.by * gv.bz;
    if (nb * 512 >= (1LL << 32)) return SDF_ERR_INVALID;  // packed cell indices are 32-bit
    const bool same_grid = E.configured && E.nblocks == (int)nb;
    E.cfg = *cfg;
    E.gv = gv;
    E.configured = true;
    if (same_grid) return SDF_OK;
    E.nblocks = (int)nb;
    sdf_status s = SDF_OK;
    if (s == SDF_OK) s = sdfb::dev_alloc(E.flags, nb);
    if (s == SDF_OK) s = sdfb::dev_alloc(E.list, nb);
    if (s == SDF_OK) s = sdfb::dev_alloc(E.block_totals, nb);
    if (s == SDF_OK) s = sdfb::dev_alloc(E.block_offsets, nb);
    if (s == SDF_OK) s = sdfb::dev_alloc(E.b2a, nb);
    // the per-active-block buffers start at a sixteenth of the blocks (a surface touches a few percent
    // of them) and grow when an extraction finds more active blocks
    E.rows_cap = (int)std::min<long long>(nb, std::max<long long>(4096, nb / 16));
    if (s == SDF_OK) s = sdfb::dev_alloc(E.fields, (size_t)E.rows_cap * sdfb::FIELD_STRIDE);
    if (s != SDF_OK) return s;
    // a block's map entry is read only where its scout flag is set; blocks past rows_cap keep -1
    cudaMemset(E.b2a, 0xFF, (size_t)nb * sizeof(int));
    // control block + scan regions (word 0 of a region is its ticket)
    const size_t tA = sdfb::scan_tiles((unsigned)nb) + 1;
    const size_t tC = sdfb::scan_tiles((unsigned)(nb * 512)) + 1;
    E.scanA_off = (sizeof(sdfb::Ctrl) + 255) & ~size_t(255);
    E.scanB_off = E.scanA_off + tA * 8;
    E.scanD_off = E.scanB_off + tA * 8;
    E.scanC_off = E.scanD_off + tA * 8;
    E.ctrl_bytes = E.scanC_off + tC * 8;
    s = sdfb::dev_alloc(E.ctrl_region, E.ctrl_bytes);
    // per-cell buffers are allocated on first use
    E.packet_cap = 0;
    return s;
}

// The host part of a scene change (CudaSDFMesh::UpdateBVH): an unchanged scene (byte-identical
// primitives) keeps its host BVH and its trained surrogate; the upload that follows still runs.
static sdf_status scene_prepare(EngineImpl& E, const sdf_primitive* prims, int count) {
    const bool same = count > 0 && !E.device_scene && E.scene.size() == (size_t)count && E.d_prims &&
                      memcmp(E.scene.data(), prims, (size_t)count * sizeof(sdf_primitive)) == 0;
    if (!same) {
        E.scene.assign(prims, prims + count);
        if (E.sur) {  // a new scene needs a new surrogate; the exact coarse culling stays valid
            E.sur->certified = false;
            if (!E.sur->exact_coarse) E.sur->enabled = false;
        }
        E.nbvh = sdfb::prepare_scene(prims, count, E.sorted, E.nodes);
        E.depth = sdfb::bvh_depth(E.nodes);
        ++E.scene_gen;
    }
    if (E.depth + 1 > sdfb::MAP_STACK) return SDF_ERR_STACK;
    if (E.prims_cap < E.sorted.size()) {
        if (sdfb::dev_alloc(E.d_prims, E.sorted.size() * 2) != SDF_OK) return SDF_ERR_NOMEM;
        E.prims_cap = E.sorted.size() * 2;
    }
    if (E.nodes_cap < E.nodes.size()) {
        if (sdfb::dev_alloc(E.d_nodes, E.nodes.size() * 2) != SDF_OK) return SDF_ERR_NOMEM;
        E.nodes_cap = E.nodes.size() * 2;
    }
    return SDF_OK;
}

sdf_status sdf_engine_set_scene_async(sdf_engine* e, const sdf_primitive* prims, int count, void* stream) {
    if (!e || count < 0 || (count > 0 && !prims)) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    cudaSetDevice(E.device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const sdf_status s = scene_prepare(E, prims, count);
    if (s != SDF_OK) return s;
    // refresh the pinned image when the scene changed (after the last upload from it has left)
    if (E.image_gen != E.scene_gen || !E.h_scene_prims) {
        if (E.scene_ev_pending) cudaEventSynchronize(E.scene_ev);
        E.scene_ev_pending = false;
        if (E.h_scene_prims_cap < E.sorted.size()) {
            if (E.h_scene_prims) cudaFreeHost(E.h_scene_prims);
            E.h_scene_prims = nullptr;
            E.h_scene_prims_cap = 0;
            if (cudaMallocHost(&E.h_scene_prims, std::max<size_t>(1, E.sorted.size()) * sizeof(sdf_primitive)) !=
                cudaSuccess)
                return SDF_ERR_NOMEM;
            E.h_scene_prims_cap = std::max<size_t>(1, E.sorted.size());
        }
        if (E.h_scene_nodes_cap < E.nodes.size() || !E.h_scene_nodes) {
            if (E.h_scene_nodes) cudaFreeHost(E.h_scene_nodes);
            E.h_scene_nodes = nullptr;
            E.h_scene_nodes_cap = 0;
            if (cudaMallocHost(&E.h_scene_nodes, std::max<size_t>(1, E.nodes.size()) * sizeof(sdf_bvh_node)) !=
                cudaSuccess)
                return SDF_ERR_NOMEM;
            E.h_scene_nodes_cap = std::max<size_t>(1, E.nodes.size());
        }
        if (!E.sorted.empty()) memcpy(E.h_scene_prims, E.sorted.data(), E.sorted.size() * sizeof(sdf_primitive));
        if (!E.nodes.empty()) memcpy(E.h_scene_nodes, E.nodes.data(), E.nodes.size() * sizeof(sdf_bvh_node));
        E.image_gen = E.scene_gen;
    }
    if (!E.sorted.empty() && cudaMemcpyAsync(E.d_prims, E.h_scene_prims, E.sorted.size() * sizeof(sdf_primitive),
                                             cudaMemcpyHostToDevice, st) != cudaSuccess)
        return SDF_ERR_CUDA;
    if (!E.nodes.empty() && cudaMemcpyAsync(E.d_nodes, E.h_scene_nodes, E.nodes.size() * sizeof(sdf_bvh_node),
                                            cudaMemcpyHostToDevice, st) != cudaSuccess)
        return SDF_ERR_CUDA;
    cudaEventRecord(E.scene_ev, st);
    E.scene_ev_pending = true;
    E.nprims = (int)E.sorted.size();
    E.nnodes = (int)E.nodes.size();
    E.device_scene = false;
    return SDF_OK;
}

sdf_status sdf_engine_set_scene(sdf_engine* e, const sdf_primitive* prims, int count) {
    if (!e || count < 0 || (count > 0 && !prims)) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    cudaSetDevice(E.device);
    const sdf_status s = scene_prepare(E, prims, count);
    if (s != SDF_OK) return s;
    if (!E.sorted.empty() &&
        cudaMemcpy(E.d_prims, E.sorted.data(), E.sorted.size() * sizeof(sdf_primitive), cudaMemcpyHostToDevice) !=
            cudaSuccess)
        return SDF_ERR_CUDA;
    if (!E.nodes.empty() &&
        cudaMemcpy(E.d_nodes, E.nodes.data(), E.nodes.size() * sizeof(sdf_bvh_node), cudaMemcpyHostToDevice) !=
            cudaSuccess)
        return SDF_ERR_CUDA;
    E.nprims = (int)E.sorted.size();
    E.nnodes = (int)E.nodes.size();
    E.device_scene = false;
    return SDF_OK;
}

sdf_status sdf_engine_set_scene_device(sdf_engine* e, const sdf_primitive* prims, int count, void* stream_ptr) {
    using namespace sdfb;
    if (!e || count < 0 || (count > 0 && !prims)) return SDF_ERR_INVALID;
    if (reinterpret_cast<uintptr_t>(prims) & 15) return SDF_ERR_INVALID;  // rows are read as float4
    EngineImpl& E = e->impl;
    cudaSetDevice(E.device);
    cudaStream_t st = static_cast<cudaStream_t>(stream_ptr);
    // the scene changes: the host copy, the host-built nodes and the surrogate no longer apply
    E.scene.clear();
    E.sorted.clear();
    E.nodes.clear();
    if (E.sur) {
        E.sur->certified = false;
        if (!E.sur->exact_coarse) E.sur->enabled = false;
    }
    E.nprims = E.nbvh = E.nnodes = E.depth = 0;
    E.device_scene = true;
    if (count == 0) return SDF_OK;
    const size_t n = (size_t)count;
    if (E.prims_cap < n) {
        if (dev_alloc(E.d_prims, n) != SDF_OK) return SDF_ERR_NOMEM;
        E.prims_cap = n;
    }
    if (E.nodes_cap < 2 * n) {
        if (dev_alloc(E.d_nodes, 2 * n) != SDF_OK) return SDF_ERR_NOMEM;
        E.nodes_cap = 2 * n;
    }
    // work arrays: 9 floats, 3 ints and 2 segments per primitive, then the control block
    const size_t seg_bytes = 2 * n * sizeof(bvhd::Seg);
    const size_t work_bytes = n * (9 * sizeof(float) + 3 * sizeof(int)) + seg_bytes +
                              bvhd::PREP_CTAS * sizeof(int) + sizeof(bvhd::Ctl) + 256;
    if (E.bvh_work_cap < n) {
        if (dev_alloc(E.bvh_work, work_bytes) != SDF_OK) return SDF_ERR_NOMEM;
        E.bvh_work_cap = n;
    }
    if (!E.h_bvh_ctl && cudaMallocHost(&E.h_bvh_ctl, sizeof(bvhd::Ctl)) != cudaSuccess) {
        E.h_bvh_ctl = nullptr;
        return SDF_ERR_NOMEM;
    }
    bvhd::Work w;
    const size_t cap = E.bvh_work_cap;
    unsigned char* q = E.bvh_work;
    w.cap = (int)cap;
    w.box = reinterpret_cast<float*>(q);                 q += 6 * cap * sizeof(float);
    w.cent = reinterpret_cast<float*>(q);                q += 3 * cap * sizeof(float);
    w.idx[0] = reinterpret_cast<int*>(q);                q += cap * sizeof(int);
    w.idx[1] = reinterpret_cast<int*>(q);                q += cap * sizeof(int);
    w.hist = reinterpret_cast<int*>(q);                  q += cap * sizeof(int);
    w.seg[0] = reinterpret_cast<bvhd::Seg*>(q);          q += cap * sizeof(bvhd::Seg);
    w.seg[1] = reinterpret_cast<bvhd::Seg*>(q);          q += cap * sizeof(bvhd::Seg);
    w.cta_count = reinterpret_cast<int*>(q);             q += bvhd::PREP_CTAS * sizeof(int);
    q = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(q) + 255) & ~uintptr_t(255));
    w.ctl = reinterpret_cast<bvhd::Ctl*>(q);
    cudaGetLastError();
    const int ctas = (int)std::min<size_t>(bvhd::PREP_CTAS, (n + bvhd::PREP_THREADS - 1) / bvhd::PREP_THREADS);
    const int per = (int)((n + ctas - 1) / ctas);
    bvhd::k_bvh_count<<<ctas, bvhd::PREP_THREADS, 0, st>>>(prims, count, per, w);
    bvhd::k_bvh_scatter<<<ctas, bvhd::PREP_THREADS, 0, st>>>(prims, count, per, E.d_prims, E.d_nodes, w);
    // levels in batches; after each batch the next level's segment count says whether to go on
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, E.device);
    const int smem_cap = (int)std::min<size_t>(n, bvhd::SMEM_HIST);
    const size_t smem = (size_t)smem_cap * sizeof(int);
    if (cudaFuncSetAttribute(bvhd::k_bvh_big, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return SDF_ERR_CUDA;
    const int grid_big = (int)std::max<size_t>(1, std::min<size_t>((size_t)sms, n / 33));
    const int grid_small = (int)std::max<size_t>(1, std::min<size_t>((size_t)sms * 8, n / 64));
    constexpr int BATCH = 8;
    for (int level = 0; level < bvhd::MAX_LEVELS; level += BATCH) {
        const int last = std::min(level + BATCH, bvhd::MAX_LEVELS);
        for (int l = level; l < last; ++l) {
            bvhd::k_bvh_big<<<grid_big, bvhd::BIG_THREADS, smem, st>>>(w, E.d_nodes, l, smem_cap);
            bvhd::k_bvh_small<<<grid_small, bvhd::SMALL_THREADS, 0, st>>>(w, E.d_nodes, l);
        }
        if (cudaMemcpyAsync(E.h_bvh_ctl, w.ctl, sizeof(bvhd::Ctl), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
            return SDF_ERR_CUDA;
        if (last >= bvhd::MAX_LEVELS || E.h_bvh_ctl->nseg[last] == 0) break;
    }
    if (cudaGetLastError() != cudaSuccess) return SDF_ERR_CUDA;
    const bvhd::Ctl& c = *E.h_bvh_ctl;
    E.nprims = count;
    E.nbvh = c.nu;
    E.nnodes = c.nu > 0 ? 2 * c.nu - 1 : 0;
    E.depth = c.depth;
    if (c.overflow || E.depth + 1 > MAP_STACK) {
        E.nbvh = E.nnodes = 0;
        return SDF_ERR_STACK;
    }
    return SDF_OK;
}

int sdf_engine_get_bvh(sdf_engine* e, sdf_bvh_node* nodes_out, int capacity, int* num_bvh_primitives) {
    if (!e) return -1;
    EngineImpl& E = e->impl;
    if (num_bvh_primitives) *num_bvh_primitives = E.nbvh;
    if (nodes_out && E.device_scene) {
        const int k = std::min(E.nnodes, capacity);
        if (k > 0 && cudaMemcpy(nodes_out, E.d_nodes, (size_t)k * sizeof(sdf_bvh_node), cudaMemcpyDeviceToHost) !=
                         cudaSuccess)
            return -1;
    } else if (nodes_out) {
        for (int i = 0; i < (int)E.nodes.size() && i < capacity; ++i) nodes_out[i] = E.nodes[i];
    }
    return E.nnodes;
}

int sdf_build_bvh_host(const sdf_primitive* prims, int count, sdf_primitive* sorted_out, sdf_bvh_node* nodes_out,
                       int capacity, int* num_bvh_primitives) {
    if (count < 0 || (count > 0 && (!prims || !sorted_out))) return -1;
    std::vector<sdf_primitive> sorted;
    std::vector<sdf_bvh_node> nodes;
    int nbvh = 0;
    try {
        nbvh = sdfb::prepare_scene(prims, count, sorted, nodes);
    } catch (...) {
        return -1;  // out of host memory
    }
    if (!nodes.empty() && (!nodes_out || capacity < (int)nodes.size())) return -1;
    for (int i = 0; i < count; ++i) sorted_out[i] = sorted[i];
    for (size_t i = 0; i < nodes.size(); ++i) nodes_out[i] = nodes[i];
    if (num_bvh_primitives) *num_bvh_primitives = nbvh;
    return (int)nodes.size();
}

// Enqueues one extraction on `st` (no host synchronisation): the final counts are copied into the
// slot's pinned Ctrl and the slot's event is recorded after them.
static sdf_status engine_enqueue(EngineImpl& E, float time, const sdf_outputs* out, cudaStream_t st,
                                 EngineImpl::Pending& P, sdfb::Ctrl* h_slot) {
    using namespace sdfb;
    const unsigned failures_before = g_launch_failures;
    const sdf_config& C = E.cfg;
    const bool dc = C.technique == SDF_TECH_DUAL_CONTOURING;
    const int cap = E.rows_cap;  // active blocks the per-block buffers hold
    if (dc || (E.debug & 1)) {
        const sdf_status s = engine_ensure_packets(E, (size_t)cap * 512);
        if (s != SDF_OK) return s;
    }
    if (dc) {
        const size_t want = std::min<size_t>((size_t)cap * 512, (size_t)1 << 28);
        if (E.dc_cap < want) {
            if (dev_alloc(E.dc_verts, want) != SDF_OK || dev_alloc(E.dc_norms, want) != SDF_OK) return SDF_ERR_NOMEM;
            E.dc_cap = want;
        }
        if ((E.debug & 2) && E.dc_qef_cap < E.dc_cap) {
            if (dev_alloc(E.dc_qef, E.dc_cap) != SDF_OK) return SDF_ERR_NOMEM;
            E.dc_qef_cap = E.dc_cap;
        }
        // the Hermite lists: sized by the last extraction's counts (a quarter and an eighth of the cells at
        // first); blocks whose samples do not fit evaluate their normals inside k_dc_solve
        {
            const size_t ws = std::min<size_t>(E.dc_cap, std::max<size_t>(E.dc_cap / 4, (size_t)E.last_herm[0] +
                                                                                        E.last_herm[0] / 4));
            const size_t wr = std::min<size_t>(E.dc_cap, std::max<size_t>(E.dc_cap / 8, (size_t)E.last_herm[1] +
                                                                                        E.last_herm[1] / 4));
            auto grow = [](auto*& p, size_t& cap, size_t want) {
                if (cap >= want) return;
                if (p) cudaFree(p);
                p = nullptr;
                cap = 0;
                if (dev_alloc(p, want) == SDF_OK) cap = want;
                cudaGetLastError();
            };
            grow(E.dc_hsamp, E.dc_hsamp_cap, ws);
            size_t rc = E.dc_hrep_cap, rc2 = E.dc_hrep_cap;
            if (rc < wr) {
                grow(E.dc_hreps, rc, wr);
                grow(E.dc_hnorm, rc2, wr);
                E.dc_hrep_cap = std::min(rc, rc2);
            }
            grow(E.dc_hbase, E.dc_hbase_cap, (size_t)cap);
            const size_t wq = std::min<size_t>(E.dc_cap, std::max<size_t>(E.dc_cap / 16, (size_t)E.last_total_vertices / 6 +
                                                                                         E.last_total_vertices / 24));
            if (E.dc_qcap < wq) {
                size_t c1 = E.dc_qcap, c2 = E.dc_qcap;
                grow(E.dc_qrec, c1, wq);
                grow(E.dc_qnorm, c2, wq);
                E.dc_qcap = std::min(c1, c2);
            }
        }
        // projection records for k_dc_project: sized by the last extraction's vertices (an eighth of the
        // cells at first); vertices beyond them are projected inside k_dc_solve, so no size is wrong
        if (C.dc_solver == SDF_DC_SOLVER_MASSPOINT && C.projection_iters > 0) {
            const size_t pw = std::min<size_t>(E.dc_cap, std::max<size_t>(E.dc_cap / 8, (size_t)E.last_dc_vertices +
                                                                                          E.last_dc_vertices / 4));
            if (E.dc_proj_cap < pw) {
                if (E.dc_proj) cudaFree(E.dc_proj);
                E.dc_proj = nullptr;
                E.dc_proj_cap = 0;
                if (dev_alloc(E.dc_proj, 2 * pw) == SDF_OK) E.dc_proj_cap = pw;
                cudaGetLastError();  // without records every vertex is projected in k_dc_solve
            }
            if ((E.debug & 1) && E.dc_proj_nsum_cap < E.dc_proj_cap) {
                if (E.dc_proj_nsum) cudaFree(E.dc_proj_nsum);
                E.dc_proj_nsum = nullptr;
                E.dc_proj_nsum_cap = 0;
                if (dev_alloc(E.dc_proj_nsum, E.dc_proj_cap) == SDF_OK) E.dc_proj_nsum_cap = E.dc_proj_cap;
                cudaGetLastError();
            }
        }
    }
    cudaGetLastError();
    auto t0 = std::chrono::high_resolution_clock::now();
    Ctrl* ctrl = reinterpret_cast<Ctrl*>(E.ctrl_region);
    unsigned long long* scanA = reinterpret_cast<unsigned long long*>(E.ctrl_region + E.scanA_off);
    unsigned long long* scanB = reinterpret_cast<unsigned long long*>(E.ctrl_region + E.scanB_off);
    unsigned long long* scanC = reinterpret_cast<unsigned long long*>(E.ctrl_region + E.scanC_off);
    // only the parts of the scan regions this extraction can touch need zeroing
    const size_t zero_bytes = dc ? E.ctrl_bytes : E.scanC_off;
    record(cudaMemsetAsync(E.ctrl_region, 0, zero_bytes, st));
    if (E.timing) cudaEventRecord(E.ev[0], st);

    SceneView sv;
    sv.prims = reinterpret_cast<const float4*>(E.d_prims);
    sv.nodes = reinterpret_cast<const float4*>(E.d_nodes);
    sv.nprims = E.nprims;
    sv.nbvh = E.nbvh;
    sv.nnodes = E.nnodes;
    const GridView gv = E.gv;
    Diag* diag = &ctrl->diag;
    const int nb = E.nblocks;
    const bool culled = E.sur && E.sur->enabled;
    if (culled)
        run_culled_scout_compact(E, sv, time, scanA, ctrl, st);
    else if (run_scout_compact(gv, sv, time, E.flags, scanA, E.list, &ctrl->active_count, diag, st) != cudaSuccess)
        return SDF_ERR_CUDA;
    if (E.timing) cudaEventRecord(E.ev[1], st);
    ActiveView av{E.list, &ctrl->active_count, cap};  // the kernels take at most cap active blocks
    MeshOut mo;
    mo.verts = reinterpret_cast<float4*>(out->vertices);
    mo.colors = reinterpret_cast<float4*>(out->colors);
    mo.indices = out->indices;
    mo.uvs = reinterpret_cast<float2*>(out->uvs);
    mo.primids = out->primitive_ids;
    mo.normals = reinterpret_cast<float4*>(out->normals);
    mo.maxV = out->max_vertices;
    unsigned mask = C.out_mask;
    if (!out->colors) mask &= ~OUT_COLORS;
    if (!out->indices) mask &= ~OUT_INDICES;
    if (!out->uvs) mask &= ~OUT_UVS;
    if (!out->primitive_ids) mask &= ~OUT_PRIMIDS;
    if (!out->normals) mask &= ~OUT_NORMALS;

    const bool welded = (C.out_mask & OUT_WELDED) != 0;
    if (welded && (!out->indices || (mask & (OUT_COLORS | OUT_UVS | OUT_PRIMIDS | OUT_NORMALS))))
        return SDF_ERR_INVALID;  // an indexed mesh has per-vertex positions only, and needs its indices
    if (!dc) {
        // positions and indices only (no per-cell debug layout): the flat per-cell emission
        const bool flat = !(mask & (OUT_COLORS | OUT_UVS | OUT_PRIMIDS | OUT_NORMALS)) && (!(E.debug & 1) || welded);
        if (welded && E.weld_cap < (size_t)cap) {
            E.weld_cap = 0;
            if (dev_alloc(E.weld_bits, (size_t)cap * WELD_STRIDE) != SDF_OK ||
                dev_alloc(E.weld_prefix, (size_t)cap * WELD_STRIDE) != SDF_OK ||
                dev_alloc(E.weld_totals, (size_t)cap) != SDF_OK || dev_alloc(E.weld_base, (size_t)cap) != SDF_OK)
                return SDF_ERR_NOMEM;
            E.weld_cap = (size_t)cap;
        }
        if (flat && E.cell_words_cap < (size_t)cap * 512) {
            if (dev_alloc(E.cell_words, (size_t)cap * 512) != SDF_OK) {
                E.cell_words_cap = 0;
                return SDF_ERR_NOMEM;
            }
            E.cell_words_cap = (size_t)cap * 512;
        }
        if (run_block_field<false>(E, sv, time, av, ctrl, (E.debug & 1) ? E.packet_counts : nullptr, st,
                                   flat ? E.cell_words : nullptr) != SDF_OK)
            return SDF_ERR_NOMEM;
        if (E.timing) cudaEventRecord(E.ev[2], st);
        k_exclusive_scan<<<std::max(1u, scan_tiles((unsigned)cap)), SCAN_THREADS, 0, st>>>(
            E.block_totals, E.block_offsets, (unsigned)cap, &ctrl->active_count, 1, scan_state(scanB),
            &ctrl->total_vertices, diag);
        check_launch();
        if (E.timing) cudaEventRecord(E.ev[3], st);
        if (welded) {
            WeldBuffers wb;
            wb.bits = E.weld_bits;
            wb.prefix = E.weld_prefix;
            wb.totals = E.weld_totals;
            wb.base = E.weld_base;
            wb.flags = E.flags;
            wb.block_to_active = E.b2a;
            const int wblocks = (cap + WELD_WARPS - 1) / WELD_WARPS;
            k_weld_mark<<<persistent_grid(k_weld_mark, WELD_WARPS * 32, wblocks), WELD_WARPS * 32, 0, st>>>(gv, av,
                                                                                                     E.fields, wb);
            check_launch();
            unsigned long long* scanD = reinterpret_cast<unsigned long long*>(E.ctrl_region + E.scanD_off);
            k_exclusive_scan<<<std::max(1u, scan_tiles((unsigned)cap)), SCAN_THREADS, 0, st>>>(
                E.weld_totals, E.weld_base, (unsigned)cap, &ctrl->active_count, 1, scan_state(scanD),
                &ctrl->welded_vertices, diag);
            check_launch();
            k_weld_vertices<<<persistent_grid(k_weld_vertices, WELD_WARPS * 32, wblocks), WELD_WARPS * 32, 0, st>>>(
                gv, av, E.fields, wb, mo.verts, mo.maxV);
            check_launch();
            k_weld_indices<<<persistent_grid(k_weld_indices, WELD_WARPS * 32, wblocks), WELD_WARPS * 32, 0, st>>>(
                gv, av, E.cell_words, E.block_offsets, wb, mo.indices, mo.maxV);
        } else if (flat) {
            k_mc_emit_cells<<<persistent_grid(k_mc_emit_cells, EMIT_WARPS * 32, (cap + EMIT_WARPS - 1) / EMIT_WARPS),
                              EMIT_WARPS * 32, 0, st>>>(
                gv, av, E.fields, E.cell_words, E.block_offsets, mo, mask, diag);
        } else {
            k_mc_emit<<<persistent_grid(k_mc_emit, BLK_THREADS, cap), BLK_THREADS, 0, st>>>(
                gv, sv, time, av, E.fields, E.block_offsets, nullptr, (E.debug & 1) ? E.packet_offsets : nullptr, mo,
                mask, &ctrl->tickets[1], diag);
        }
        check_launch();
        if (E.timing) cudaEventRecord(E.ev[4], st);
    } else {
        DcBuffers B;
        B.block_to_active = E.b2a;
        B.masks = E.masks;
        B.vert_offsets = E.dc_voff;
        B.cell_verts = E.dc_verts;
        B.cell_normals = (E.debug & 1) ? E.dc_norms : nullptr;  // no output reads them; debug keeps them
        B.cell_normals_tmp = nullptr;
        B.counts = E.packet_counts;
        B.offsets = E.packet_offsets;
        B.qef_debug = (E.debug & 2) ? E.dc_qef : nullptr;
        const bool project = C.dc_solver == SDF_DC_SOLVER_MASSPOINT && C.projection_iters > 0 && E.dc_proj &&
                             (!B.cell_normals || E.dc_proj_nsum_cap >= E.dc_proj_cap);
        B.proj = project ? E.dc_proj : nullptr;
        B.proj_nsum = project && B.cell_normals ? E.dc_proj_nsum : nullptr;
        // debug bit 2: lists of a few hundred entries, so most blocks, passes and vertices take the
        // in-block paths next to listed ones (the results are the same either way)
        const bool small_lists = (E.debug & 4) != 0;
        auto list_cap = [&](size_t c, size_t small) {
            return (unsigned)std::min<size_t>(small_lists ? std::min(c, small) : c, 0xFFFFFFFFu);
        };
        B.proj_cap = project ? list_cap(E.dc_proj_cap, 256) : 0u;
        const bool herm = E.dc_hsamp && E.dc_hreps && E.dc_hnorm && E.dc_hbase && E.dc_hbase_cap >= (size_t)cap &&
                          E.dc_hsamp_cap > 0 && E.dc_hrep_cap > 0;
        B.hbase = herm ? E.dc_hbase : nullptr;
        B.hsample_rep = herm ? E.dc_hsamp : nullptr;
        B.hnormals = herm ? E.dc_hnorm : nullptr;
        const bool qlist = E.dc_qrec && E.dc_qnorm && E.dc_qcap > 0;
        B.qnormals = qlist ? E.dc_qnorm : nullptr;
        B.qcap = qlist ? list_cap(E.dc_qcap, 512) : 0u;
        record(cudaMemsetAsync(E.b2a, 0xFF, (size_t)nb * sizeof(int), st));
        k_dc_block_map<<<(cap + 255) / 256, 256, 0, st>>>(E.list, &ctrl->active_count, cap, nb, E.b2a);
        check_launch();
        // the block rows by the shared-halo block field (own samples two per lane, halos copied from
        // active neighbours), then the cells classified from the finished rows
        if (run_block_field<false>(E, sv, time, av, ctrl, nullptr, st, nullptr, false) != SDF_OK) return SDF_ERR_NOMEM;
        k_dc_mark<<<persistent_grid(k_dc_mark, BLK_THREADS, cap), BLK_THREADS, 0, st>>>(gv, sv, time, av, E.fields, B,
                                                                                      &ctrl->tickets[5], diag, true);
        check_launch();
        const unsigned ncells_max = (unsigned)cap * 512u;
        k_exclusive_scan<<<std::max(1u, scan_tiles(ncells_max)), SCAN_THREADS, 0, st>>>(
            E.packet_counts, E.dc_voff, (unsigned)cap, &ctrl->active_count, 512, scan_state(scanC),
            &ctrl->dc_vertices, diag);
        check_launch();
        if (E.timing) cudaEventRecord(E.ev[2], st);
        DcSolveParams sp;
        sp.max_cell_vertices = (unsigned)E.dc_cap;
        sp.qef_blend = C.qef_blend;
        sp.solver = C.dc_solver;
        sp.projection_iters = C.dc_solver == SDF_DC_SOLVER_MASSPOINT ? C.projection_iters : 0;
        sp.cond_threshold = C.cond_threshold > 0.f ? C.cond_threshold : 1e4f;
        if (herm) {
            const size_t hsmem = sizeof(HermSmem);
            k_dc_hermite_reps<<<persistent_grid(k_dc_hermite_reps, SOLVE_THREADS, cap, hsmem), SOLVE_THREADS, hsmem, st>>>(
                gv, av, E.fields, B, sp, ctrl->herm, E.dc_hsamp, E.dc_hreps, list_cap(E.dc_hsamp_cap, 512),
                list_cap(E.dc_hrep_cap, 256), &ctrl->tickets[7]);
            k_dc_hermite_normals<<<persistent_grid(k_dc_hermite_normals, BLK_THREADS,
                                                   std::max(1, (int)(E.dc_hrep_cap / 256))),
                                   BLK_THREADS, 0, st>>>(gv, sv, time, av, E.dc_hreps, ctrl->herm,
                                                         list_cap(E.dc_hrep_cap, 256), E.dc_hnorm, &ctrl->tickets[8],
                                                         diag);
            check_launch();
        }
        const size_t solve_smem = sizeof(SolveSmem);
        k_dc_solve<<<persistent_grid(k_dc_solve, SOLVE_THREADS, cap, solve_smem), SOLVE_THREADS, solve_smem, st>>>(
            gv, sv, time, av, E.fields, B, sp, &ctrl->tickets[1], diag);
        check_launch();
        if (project) {
            k_dc_project<<<persistent_grid(k_dc_project, BLK_THREADS, std::max(1, (int)(B.proj_cap / 256))), BLK_THREADS,
                           0, st>>>(gv, sv, time, av, B, sp, &ctrl->dc_vertices, &ctrl->tickets[6], diag);
            check_launch();
        }
        if (E.timing) cudaEventRecord(E.ev[3], st);
        k_dc_count_quads<<<std::min(cap, num_sms() * 4), 512, 0, st>>>(gv, av, B, E.packet_counts, E.block_totals);
        check_launch();
        k_exclusive_scan<<<std::max(1u, scan_tiles((unsigned)cap)), SCAN_THREADS, 0, st>>>(
            E.block_totals, E.block_offsets, (unsigned)cap, &ctrl->active_count, 1, scan_state(scanB),
            &ctrl->total_vertices, diag);
        check_launch();
        DcQuadParams qp;
        qp.adaptive_diagonal = (C.dc_solver == SDF_DC_SOLVER_MASSPOINT) ? C.adaptive_diagonal : 0;
        if (qlist) {
            k_dc_quad_list<<<std::min(cap, num_sms() * 8), BLK_THREADS, 0, st>>>(gv, av, B, E.packet_counts,
                                                                                   E.block_offsets, E.dc_qrec, B.qcap);
            k_dc_quad_normals<<<persistent_grid(k_dc_quad_normals, BLK_THREADS, std::max(1, (int)(B.qcap / 256))),
                                BLK_THREADS, 0, st>>>(gv, sv, time, av, B, E.dc_qrec, &ctrl->total_vertices, B.qcap,
                                                      mo.maxV, E.dc_qnorm, &ctrl->tickets[9], diag, &ctrl->dc_vertices,
                                                      mo, mask, qp);
            check_launch();
        }
        const size_t quad_smem = sizeof(QuadSmem);
        k_dc_quads<<<persistent_grid(k_dc_quads, BLK_THREADS, cap, quad_smem), BLK_THREADS, quad_smem, st>>>(
            gv, sv, time, av, B, nullptr, E.packet_counts, E.block_offsets, mo, mask, qp, &ctrl->tickets[2], diag,
            &ctrl->total_vertices, &ctrl->dc_vertices);
        check_launch();
        if (welded) {  // indexed output: the cell vertices themselves
            k_dc_weld_vertices<<<persistent_grid(k_dc_weld_vertices, 256, cap * 2), 256, 0, st>>>(
                gv, av, B, (unsigned)E.dc_cap, mo.verts, mo.maxV);
            check_launch();
        }
        if (E.timing) cudaEventRecord(E.ev[4], st);
    }
    check_launch();
    if (g_launch_failures != failures_before) return SDF_ERR_CUDA;  // a kernel was not launched
    record(cudaMemcpyAsync(h_slot, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    if (cudaEventRecord(P.done, st) != cudaSuccess) return SDF_ERR_CUDA;
    P.nb = nb;
    P.rows_cap = cap;
    P.out = *out;
    P.time = time;
    P.stream = st;
    P.dc = dc;
    P.welded = welded;
    P.culled = culled;
    P.max_vertices = out->max_vertices;
    P.dc_cap = E.dc_cap;
    P.t0 = t0;
    return SDF_OK;
}

// Grows the per-active-block buffers to hold `need` active blocks (a quarter more, at most every block)
// after an extraction found more active blocks than they held. Waits for the device first: other
// extractions in flight may still use the buffers the next enqueue reallocates.
static sdf_status engine_grow_rows(EngineImpl& E, long long need) {
    using namespace sdfb;
    const long long cap = std::min<long long>(E.nblocks, need + need / 4 + 1024);
    if (cap <= E.rows_cap) return SDF_OK;
    const cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        record(e);
        return SDF_ERR_CUDA;
    }
    if (dev_alloc(E.fields, (size_t)cap * FIELD_STRIDE) != SDF_OK) {
        E.rows_cap = 0;
        return SDF_ERR_NOMEM;
    }
    E.rows_cap = (int)cap;  // the miss list, cell words, weld and DC arrays follow on their next use
    return SDF_OK;
}

// Waits for the extraction of a slot and turns its read-back into stats and a status. The stage
// times are the engine's timing events, valid for the most recent extraction only. *rows_need > 0:
// the extraction found more active blocks than its per-block buffers held (its outputs are not
// valid; engine_grow_rows and a second run follow).
static sdf_status engine_collect(EngineImpl& E, int slot, sdf_stats* stats, bool stage_times,
                                 long long* rows_need = nullptr) {
    using namespace sdfb;
    EngineImpl::Pending& P = E.pend[slot];
    const cudaError_t err = cudaEventSynchronize(P.done);
    auto t1 = std::chrono::high_resolution_clock::now();
    P.used = false;
    if (err != cudaSuccess) {
        record(err);
        return SDF_ERR_CUDA;
    }
    const Ctrl& h = E.h_ctrl[slot];
    if (rows_need) *rows_need = h.active_count > P.rows_cap ? (long long)h.active_count : 0;
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->total_blocks = P.nb;
        stats->active_blocks = h.active_count;
        stats->total_vertices = h.total_vertices;
        stats->written_vertices = std::min<int64_t>(h.total_vertices, P.max_vertices);
        stats->dc_cell_vertices = h.dc_vertices;
        if (P.dc) {
            E.last_dc_vertices = h.dc_vertices;
            E.last_herm[0] = h.herm[0];
            E.last_herm[1] = h.herm[1];
            E.last_total_vertices = h.total_vertices;
        }
        stats->bvh_cap_hits = (int64_t)h.diag.cap_hits;
        stats->scouted_blocks = P.culled ? (int64_t)h.diag.scouted : (int64_t)P.nb;
        stats->dc_fp64_cells = (int64_t)h.diag.fp64_cells;
        stats->welded_vertices = P.welded ? (int64_t)(P.dc ? h.dc_vertices : h.welded_vertices) : 0;
        stats->ms_total = std::chrono::duration<float, std::milli>(t1 - P.t0).count();
        if (E.timing && stage_times) {
            cudaEventElapsedTime(&stats->ms_scout, E.ev[0], E.ev[1]);
            cudaEventElapsedTime(&stats->ms_field, E.ev[1], E.ev[2]);
            cudaEventElapsedTime(&stats->ms_scan, E.ev[2], E.ev[3]);
            cudaEventElapsedTime(&stats->ms_emit, E.ev[3], E.ev[4]);
            if (!P.dc) cudaEventElapsedTime(&stats->ms_classify, E.ev[5], E.ev[2]);
        }
    }
    if (h.diag.timeout) return SDF_ERR_TIMEOUT;
    if (h.diag.stack_overflow) return SDF_ERR_STACK;
    if (h.diag.inconsistent) return SDF_ERR_CUDA;
    if (h.total_vertices > P.max_vertices || (P.dc && h.dc_vertices > P.dc_cap) ||
        (P.welded && (P.dc ? h.dc_vertices : h.welded_vertices) > P.max_vertices))
        return SDF_ERR_CAPACITY;
    return SDF_OK;
}

sdf_status sdf_engine_extract_async(sdf_engine* e, float time, const sdf_outputs* out, void* stream,
                                    uint64_t* ticket) {
    if (!e || !out || !out->vertices || !ticket) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    if (!E.configured) return SDF_ERR_INVALID;
    cudaSetDevice(E.device);
    const int slot = (int)(E.next_ticket % EngineImpl::ASYNC_SLOTS);
    EngineImpl::Pending& P = E.pend[slot];
    if (P.used) {  // the oldest extraction still holds the slot: it must finish first
        cudaEventSynchronize(P.done);
        P.used = false;
    }
    const sdf_status s = engine_enqueue(E, time, out, static_cast<cudaStream_t>(stream), P, &E.h_ctrl[slot]);
    if (s != SDF_OK) return s;
    P.used = true;
    P.ticket = E.next_ticket;
    *ticket = E.next_ticket++;
    return SDF_OK;
}

sdf_status sdf_engine_extract_wait(sdf_engine* e, uint64_t ticket, sdf_stats* stats) {
    if (!e) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    cudaSetDevice(E.device);
    const int slot = (int)(ticket % EngineImpl::ASYNC_SLOTS);
    if (!E.pend[slot].used || E.pend[slot].ticket != ticket) return SDF_ERR_INVALID;  // unknown or collected
    const bool last = ticket + 1 == E.next_ticket;
    long long need = 0;
    sdf_status s = engine_collect(E, slot, stats, last, &need);
    if (need == 0) return s;
    // more active blocks than the per-block buffers held: grow them and run this extraction again
    // (synchronously, on its stream; the same scene and time cannot need more the second time)
    s = engine_grow_rows(E, need);
    if (s != SDF_OK) return s;
    EngineImpl::Pending& P = E.pend[slot];
    const sdf_outputs out = P.out;
    s = engine_enqueue(E, P.time, &out, P.stream, P, &E.h_ctrl[slot]);
    if (s != SDF_OK) return s;
    P.used = true;
    return engine_collect(E, slot, stats, last, &need);
}

sdf_status sdf_engine_extract(sdf_engine* e, float time, const sdf_outputs* out, void* stream, sdf_stats* stats) {
    uint64_t t = 0;
    const sdf_status s = sdf_engine_extract_async(e, time, out, stream, &t);
    if (s != SDF_OK) return s;
    return sdf_engine_extract_wait(e, t, stats);
}

const void* sdf_engine_buffer(sdf_engine* e, int which, size_t* bytes) {
    if (!e) return nullptr;
    EngineImpl& E = e->impl;
    const size_t cells = (size_t)E.rows_cap * 512;
    const void* p = nullptr;
    size_t b = 0;
    switch (which) {
        case 0: p = E.list; b = (size_t)E.nblocks * 4; break;
        case 1: p = E.packet_counts; b = E.packet_cap ? cells * 4 : 0; break;
        case 2: p = E.packet_offsets; b = E.packet_cap ? cells * 4 : 0; break;
        case 3: p = E.masks; b = E.packet_cap ? cells : 0; break;
        case 4: p = E.dc_voff; b = E.packet_cap ? cells * 4 : 0; break;
        case 5: p = E.dc_verts; b = E.dc_cap * 8; break;
        case 6: p = E.dc_norms; b = E.dc_cap * 8; break;
        case 7: p = E.block_totals; b = (size_t)E.nblocks * 4; break;
        case 8: p = E.fields; b = (size_t)E.rows_cap * sdfb::FIELD_STRIDE * 4; break;
        case 9: p = E.d_prims; b = (size_t)E.nprims * sizeof(sdf_primitive); break;
        case 10: p = E.d_nodes; b = (size_t)E.nnodes * sizeof(sdf_bvh_node); break;
        case 11: p = E.dc_qef; b = E.dc_qef_cap * 16; break;
        default: break;
    }
    if (bytes) *bytes = b;
    return p;
}

sdf_status sdf_engine_eval_normals(sdf_engine* e, const float* d_points, int n, float time, float cell,
                                   float* d_out, void* stream) {
    using namespace sdfb;
    if (!e || n < 0 || (n > 0 && (!d_points || !d_out))) return SDF_ERR_INVALID;
    if (n == 0) return SDF_OK;
    EngineImpl& E = e->impl;
    cudaSetDevice(E.device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!E.eval_diag && cudaMalloc(&E.eval_diag, sizeof(Diag)) != cudaSuccess) return SDF_ERR_NOMEM;
    const int warps = (n + 31) / 32;
    const int blocks = std::min((warps + 7) / 8, num_sms() * 8);
    k_eval_normals<<<blocks, BLK_THREADS, 0, st>>>(engine_scene_view(E), d_points, n, time, cell, d_out,
                                                   E.eval_diag);
    return cudaGetLastError() == cudaSuccess ? SDF_OK : SDF_ERR_CUDA;
}

sdf_status sdf_engine_eval_distance(sdf_engine* e, const float* d_points, int n, float time, float* d_out,
                                    void* stream) {
    using namespace sdfb;
    if (!e || n < 0 || (n > 0 && (!d_points || !d_out))) return SDF_ERR_INVALID;
    if (n == 0) return SDF_OK;
    EngineImpl& E = e->impl;
    cudaSetDevice(E.device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!E.eval_diag && cudaMalloc(&E.eval_diag, sizeof(Diag)) != cudaSuccess) return SDF_ERR_NOMEM;
    const int warps = (n + 31) / 32;
    const int blocks = std::min((warps + 7) / 8, num_sms() * 8);
    k_eval_distance<<<blocks, BLK_THREADS, 0, st>>>(engine_scene_view(E), d_points, n, time, d_out, E.eval_diag);
    return cudaGetLastError() == cudaSuccess ? SDF_OK : SDF_ERR_CUDA;
}

sdf_status sdf_engine_eval(sdf_engine* e, const float* d_points, int n, float time, float* d_out, void* stream) {
    using namespace sdfb;
    if (!e || n < 0 || (n > 0 && (!d_points || !d_out))) return SDF_ERR_INVALID;
    if (n == 0) return SDF_OK;
    EngineImpl& E = e->impl;
    cudaSetDevice(E.device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (!E.eval_diag && cudaMalloc(&E.eval_diag, sizeof(Diag)) != cudaSuccess) return SDF_ERR_NOMEM;
    record(cudaMemsetAsync(E.eval_diag, 0, sizeof(Diag), st));
    SceneView sv;
    sv.prims = reinterpret_cast<const float4*>(E.d_prims);
    sv.nodes = reinterpret_cast<const float4*>(E.d_nodes);
    sv.nprims = E.nprims;
    sv.nbvh = E.nbvh;
    sv.nnodes = E.nnodes;
    const int warps = (n + 31) / 32;
    const int blocks = std::min((warps + 7) / 8, num_sms() * 8);
    k_eval_points<<<blocks, BLK_THREADS, 0, st>>>(sv, d_points, n, time, d_out, E.eval_diag);
    const cudaError_t err = cudaGetLastError();
    return err == cudaSuccess ? SDF_OK : SDF_ERR_CUDA;
}

sdf_status sdf_engine_count_work(sdf_engine* e, unsigned long long out[8]) {
    using namespace sdfb;
    if (!e || !out) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    if (!E.configured) return SDF_ERR_INVALID;
    cudaSetDevice(E.device);
    Ctrl* ctrl = reinterpret_cast<Ctrl*>(E.ctrl_region);
    unsigned long long* scanA = reinterpret_cast<unsigned long long*>(E.ctrl_region + E.scanA_off);
    record(cudaMemsetAsync(E.ctrl_region, 0, E.scanC_off, 0));
    SceneView sv;
    sv.prims = reinterpret_cast<const float4*>(E.d_prims);
    sv.nodes = reinterpret_cast<const float4*>(E.d_nodes);
    sv.nprims = E.nprims;
    sv.nbvh = E.nbvh;
    sv.nnodes = E.nnodes;
    if (run_scout_compact(E.gv, sv, 0.f, E.flags, scanA, E.list, &ctrl->active_count, &ctrl->diag, 0) != cudaSuccess)
        return SDF_ERR_CUDA;
    int count = 0;
    if (cudaMemcpy(&count, &ctrl->active_count, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return SDF_ERR_CUDA;
    if (count > E.rows_cap && engine_grow_rows(E, count) != SDF_OK) return SDF_ERR_NOMEM;
    record(cudaMemsetAsync(&ctrl->diag, 0, sizeof(Diag), 0));
    ActiveView av{E.list, &ctrl->active_count, E.rows_cap};
    // the engine's block-field stage (own samples, then the halos no active block owns) with counters on
    if (run_block_field<true>(E, sv, 0.f, av, ctrl, nullptr, 0) != SDF_OK) return SDF_ERR_NOMEM;
    Ctrl h;
    if (cudaMemcpy(&h, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost) != cudaSuccess) return SDF_ERR_CUDA;
    out[0] = h.diag.node_pops;
    out[1] = h.diag.leaf_evals;
    out[2] = h.diag.points;
    out[3] = (unsigned long long)h.active_count;
    out[4] = h.diag.warp_pops;
    out[5] = h.diag.warp_tests;
    out[6] = h.diag.warp_leaves;
    out[7] = 0;
    return SDF_OK;
}

sdf_status sdf_measure_fp32_peak(double* tflops) {
    using namespace sdfb;
    if (!tflops) return SDF_ERR_INVALID;
    float* dummy = nullptr;
    if (cudaMalloc(&dummy, 256 * sizeof(float)) != cudaSuccess) return SDF_ERR_NOMEM;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const int blocks = num_sms() * 8, iters = 4096;
    k_fma_peak<<<blocks, 256>>>(dummy, iters, 0.9999f, 1e-7f);  // warm-up
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(a);
        k_fma_peak<<<blocks, 256>>>(dummy, iters, 0.9999f, 1e-7f);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        best = std::min(best, ms);
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(dummy);
    if (cudaGetLastError() != cudaSuccess) return SDF_ERR_CUDA;
    const double flops = 2.0 * 8 * 16 * (double)iters * blocks * 256;
    *tflops = flops / (best * 1e-3) / 1e12;
    return SDF_OK;
}

sdf_status sdf_engine_read_buffer(sdf_engine* e, int which, void* host_dst, size_t bytes) {
    size_t have = 0;
    const void* p = sdf_engine_buffer(e, which, &have);
    if (!p || !host_dst || bytes > have) return SDF_ERR_INVALID;
    cudaSetDevice(e->impl.device);
    if (cudaDeviceSynchronize() != cudaSuccess) return SDF_ERR_CUDA;
    return cudaMemcpy(host_dst, p, bytes, cudaMemcpyDeviceToHost) == cudaSuccess ? SDF_OK : SDF_ERR_CUDA;
}

sdf_status sdf_extract(const sdf_primitive* prims, int count, const sdf_config* cfg, float time,
                       const sdf_outputs* out, void* stream, sdf_stats* stats) {
    sdf_engine* e = nullptr;
    sdf_status s = sdf_engine_create(&e, -1);
    if (s != SDF_OK) return s;
    s = sdf_engine_configure(e, cfg);
    if (s == SDF_OK) s = sdf_engine_set_scene(e, prims, count);
    if (s == SDF_OK) s = sdf_engine_extract(e, time, out, stream, stats);
    sdf_engine_destroy(e);
    return s;
}

}  // extern "C"
