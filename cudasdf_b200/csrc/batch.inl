// sdf_batch: many scenes meshed together (included at the end of sdfmesh.cu, after engine.inl).
//
// The scenes of one technique form a group. A group numbers the blocks of all its scenes globally
// (scene s owns [block_base_s, block_base_s + blocks_s)), uploads every scene's primitives and BVH
// into one array each (a scene's SceneView points at its part), and runs the engine's stages once
// for the whole group: scout over the global bricks, one compaction (the active list is then sorted
// by scene), the block field / DC stages with each work item resolving its scene, one scan of the
// block totals, and one emission into the group's concatenated output. k_batch_scene_first turns
// the scan into each scene's first output vertex.
#include <cstring>

namespace sdfb {

struct BatchGroup {
    int technique = 0;
    std::vector<int> scenes;            // batch indices of the group's scenes, in group order
    std::vector<SceneDesc> desc_host;
    SceneDesc* desc = nullptr;
    int n = 0;
    long long total_blocks = 0, total_bricks = 0;
    sdf_primitive* prims = nullptr;
    sdf_bvh_node* nodes = nullptr;
    unsigned* flags = nullptr;
    int* list = nullptr;
    float* fields = nullptr;
    unsigned* block_totals = nullptr;
    unsigned* block_offsets = nullptr;
    int* b2a = nullptr;
    unsigned* miss = nullptr;
    unsigned* cell_words = nullptr;     // flat emission (no attribute outputs)
    unsigned* first = nullptr;          // n + 1 first vertices
    unsigned char* ctrl_region = nullptr;
    size_t scanA_off = 0, scanB_off = 0, scanC_off = 0, ctrl_bytes = 0;
    // dual contouring
    unsigned* packet_counts = nullptr;
    unsigned* packet_offsets = nullptr;
    unsigned char* masks = nullptr;
    unsigned* dc_voff = nullptr;
    ushort4* dc_verts = nullptr;
    size_t dc_cap = 0;
    DcSolveParams sp{};
    DcQuadParams qp{};
    // dual contouring, the lists of the cross-block kernels (sized by the last run's counts; blocks and
    // quads past them are handled inside k_dc_solve / k_dc_quads): Hermite samples and representatives,
    // quads, projection records
    unsigned* hsamp = nullptr;
    float4* hreps = nullptr;
    float4* hnorm = nullptr;
    int4* hbase = nullptr;
    uint2* qrec = nullptr;
    float4* qnorm = nullptr;
    float4* proj = nullptr;
    size_t hsamp_cap = 0, hrep_cap = 0, q_cap = 0, proj_cap = 0;
    unsigned last_herm[2] = {0u, 0u};
    unsigned last_total = 0, last_dc = 0;
    // pinned read-back
    Ctrl* h_ctrl = nullptr;
    unsigned* h_first = nullptr;

    void release() {
        void* ptrs[] = {desc, prims, nodes, flags, list, fields, block_totals, block_offsets, b2a, miss, cell_words, first,
                        ctrl_region, packet_counts, packet_offsets, masks, dc_voff, dc_verts, hsamp, hreps, hnorm,
                        hbase, qrec, qnorm, proj};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        if (h_ctrl) cudaFreeHost(h_ctrl);
        if (h_first) cudaFreeHost(h_first);
        *this = BatchGroup();
    }
    Ctrl* ctrl() const { return reinterpret_cast<Ctrl*>(ctrl_region); }
    unsigned long long* scan(size_t off) const { return reinterpret_cast<unsigned long long*>(ctrl_region + off); }
    ActiveView active() const { return ActiveView{list, &ctrl()->active_count, (int)total_blocks, desc, n}; }
};

// persistent grid of `kernel` with at most `cap` CTAs per SM (0: as many as fit)
template <class K>
static int capped_grid(K kernel, int threads, long long items, size_t smem, int cap) {
    int per_sm = 0;
    opt_in_smem(kernel, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
    if (per_sm < 1) per_sm = 1;
    if (cap > 0 && cap < per_sm) per_sm = cap;
    return (int)std::max(1LL, std::min<long long>((long long)num_sms() * per_sm, items));
}

// launch shapes of one extraction, fixed before any capture
struct BatchGrids {
    int own, miss, gather, emit, mark, solve, quads, count_quads, emit_cells, herm_reps, flat;
};

static BatchGrids batch_grids(long long blocks, const int ctas[4]) {
    BatchGrids G;
    G.own = capped_grid(k_field_own<false>, BLK_THREADS, blocks, 0, ctas[0]);
    G.miss = capped_grid(k_field_miss<false>, BLK_THREADS, 1LL << 30, 0, ctas[0]);
    G.gather = capped_grid(k_field_gather, BLK_THREADS, (blocks + GATHER_WARPS - 1) / GATHER_WARPS, 0, 0);
    G.emit = capped_grid(k_mc_emit, BLK_THREADS, blocks, 0, ctas[1]);
    G.mark = capped_grid(k_dc_mark, BLK_THREADS, blocks, 0, ctas[0]);
    G.solve = capped_grid(k_dc_solve, SOLVE_THREADS, blocks, sizeof(SolveSmem), ctas[2]);
    G.quads = capped_grid(k_dc_quads, BLK_THREADS, blocks, sizeof(QuadSmem), ctas[3]);
    G.count_quads = (int)std::min<long long>(std::max(1LL, blocks), (long long)num_sms() * 4);
    G.emit_cells = capped_grid(k_mc_emit_cells, EMIT_WARPS * 32, (blocks + EMIT_WARPS - 1) / EMIT_WARPS, 0, 0);
    G.herm_reps = capped_grid(k_dc_hermite_reps, SOLVE_THREADS, blocks, sizeof(HermSmem), 0);
    // the flat DC kernels (Hermite normals, projection, quad normals) claim 32-item tasks: one full wave
    G.flat = capped_grid(k_dc_quad_normals, BLK_THREADS, 1LL << 30, 0, 0);
    return G;
}

static MeshOut mesh_out(const sdf_outputs* o) {
    MeshOut m{};
    if (!o) return m;
    m.verts = reinterpret_cast<float4*>(o->vertices);
    m.colors = reinterpret_cast<float4*>(o->colors);
    m.indices = o->indices;
    m.uvs = reinterpret_cast<float2*>(o->uvs);
    m.primids = o->primitive_ids;
    m.normals = reinterpret_cast<float4*>(o->normals);
    m.maxV = o->max_vertices;
    return m;
}

static unsigned out_mask_for(const sdf_outputs* o, unsigned mask) {
    if (!o) return 0;
    if (!o->colors) mask &= ~OUT_COLORS;
    if (!o->indices) mask &= ~OUT_INDICES;
    if (!o->uvs) mask &= ~OUT_UVS;
    if (!o->primitive_ids) mask &= ~OUT_PRIMIDS;
    if (!o->normals) mask &= ~OUT_NORMALS;
    return mask;
}

// every kernel of one group's extraction, on stream st (no host synchronisation)
static void enqueue_group(BatchGroup& B, const BatchGrids& G, float time, const sdf_outputs* out, unsigned mask,
                          cudaStream_t st) {
    if (B.n == 0) return;
    const bool dc = B.technique == SDF_TECH_DUAL_CONTOURING;
    Ctrl* ctrl = B.ctrl();
    Diag* diag = &ctrl->diag;
    const GridView g0 = B.desc_host[0].g;
    const SceneView sc0 = B.desc_host[0].sc;
    const ActiveView av = B.active();
    const unsigned nb = (unsigned)B.total_blocks;
    const MeshOut mo = mesh_out(out);
    const unsigned m = out_mask_for(out, mask);
    record(cudaMemsetAsync(B.ctrl_region, 0, dc ? B.ctrl_bytes : B.scanC_off, st));
    k_scout_batch<<<(unsigned)((B.total_bricks + BLK_THREADS / 32 - 1) / (BLK_THREADS / 32)), BLK_THREADS, 0, st>>>(
        B.desc, B.n, (unsigned)B.total_bricks, time, B.flags, diag);
    k_compact<<<std::max(1u, scan_tiles(nb)), SCAN_THREADS, 0, st>>>(B.flags, nb, B.list, &ctrl->active_count,
                                                                     scan_state(B.scan(B.scanA_off)), diag);
    if (!dc) {
        k_field_plan<<<num_sms() * 8, 256, 0, st>>>(g0, av, B.flags, B.fields, B.b2a, B.miss, &ctrl->halo_misses);
        k_field_own<false><<<G.own, BLK_THREADS, 0, st>>>(g0, sc0, time, av, B.fields, &ctrl->tickets[0], diag);
        k_field_miss<false><<<G.miss, BLK_THREADS, 0, st>>>(g0, sc0, time, av, B.fields, B.miss, &ctrl->halo_misses,
                                                            &ctrl->tickets[4], diag);
        const bool flat = B.cell_words && !(m & (OUT_COLORS | OUT_UVS | OUT_PRIMIDS | OUT_NORMALS));
        k_field_gather<<<G.gather, BLK_THREADS, 0, st>>>(g0, av, B.fields, B.b2a, B.flags, B.block_totals, nullptr,
                                                         flat ? B.cell_words : nullptr);
        k_exclusive_scan<<<std::max(1u, scan_tiles(nb)), SCAN_THREADS, 0, st>>>(
            B.block_totals, B.block_offsets, nb, &ctrl->active_count, 1, scan_state(B.scan(B.scanB_off)),
            &ctrl->total_vertices, diag);
        if (flat)
            k_mc_emit_cells<<<G.emit_cells, EMIT_WARPS * 32, 0, st>>>(g0, av, B.fields, B.cell_words, B.block_offsets,
                                                                      mo, m, diag);
        else
            k_mc_emit<<<G.emit, BLK_THREADS, 0, st>>>(g0, sc0, time, av, B.fields, B.block_offsets, nullptr, nullptr, mo,
                                                      m, &ctrl->tickets[1], diag);
    } else {
        DcBuffers D;
        D.block_to_active = B.b2a;
        D.masks = B.masks;
        D.vert_offsets = B.dc_voff;
        D.cell_verts = B.dc_verts;
        D.cell_normals = nullptr;  // the per-cell normals feed no output
        D.cell_normals_tmp = nullptr;
        D.counts = B.packet_counts;
        D.offsets = B.packet_offsets;
        D.qef_debug = nullptr;
        const bool project = B.sp.solver == SDF_DC_SOLVER_MASSPOINT && B.sp.projection_iters > 0 && B.proj_cap > 0;
        D.proj = project ? B.proj : nullptr;
        D.proj_nsum = nullptr;  // no cell normals
        D.proj_cap = project ? (unsigned)std::min<size_t>(B.proj_cap, 0xFFFFFFFFu) : 0u;
        const bool herm = B.hsamp_cap > 0 && B.hrep_cap > 0 && B.hbase;
        D.hbase = herm ? B.hbase : nullptr;
        D.hsample_rep = herm ? B.hsamp : nullptr;
        D.hnormals = herm ? B.hnorm : nullptr;
        const bool qlist = B.q_cap > 0;
        D.qnormals = qlist ? B.qnorm : nullptr;
        D.qcap = qlist ? (unsigned)std::min<size_t>(B.q_cap, 0xFFFFFFFFu) : 0u;
        record(cudaMemsetAsync(B.b2a, 0xFF, (size_t)nb * sizeof(int), st));
        k_dc_block_map<<<(nb + 255) / 256, 256, 0, st>>>(B.list, &ctrl->active_count, (int)nb, (int)nb, B.b2a);
        // block rows by the shared-halo block field, then the cells classified from the rows
        k_field_plan<<<num_sms() * 8, 256, 0, st>>>(g0, av, B.flags, B.fields, B.b2a, B.miss, &ctrl->halo_misses);
        k_field_own<false><<<G.own, BLK_THREADS, 0, st>>>(g0, sc0, time, av, B.fields, &ctrl->tickets[3], diag);
        k_field_miss<false><<<G.miss, BLK_THREADS, 0, st>>>(g0, sc0, time, av, B.fields, B.miss, &ctrl->halo_misses,
                                                            &ctrl->tickets[4], diag);
        k_field_gather<<<G.gather, BLK_THREADS, 0, st>>>(g0, av, B.fields, B.b2a, B.flags, nullptr, nullptr, nullptr);
        k_dc_mark<<<G.mark, BLK_THREADS, 0, st>>>(g0, sc0, time, av, B.fields, D, &ctrl->tickets[0], diag, true);
        k_exclusive_scan<<<std::max(1u, scan_tiles(nb * 512u)), SCAN_THREADS, 0, st>>>(
            B.packet_counts, B.dc_voff, nb, &ctrl->active_count, 512, scan_state(B.scan(B.scanC_off)),
            &ctrl->dc_vertices, diag);
        DcSolveParams sp = B.sp;
        sp.max_cell_vertices = (unsigned)B.dc_cap;
        if (herm) {
            k_dc_hermite_reps<<<G.herm_reps, SOLVE_THREADS, sizeof(HermSmem), st>>>(
                g0, av, B.fields, D, sp, ctrl->herm, B.hsamp, B.hreps, (unsigned)std::min<size_t>(B.hsamp_cap, 0xFFFFFFFFu),
                (unsigned)std::min<size_t>(B.hrep_cap, 0xFFFFFFFFu), &ctrl->tickets[7]);
            k_dc_hermite_normals<<<G.flat, BLK_THREADS, 0, st>>>(g0, sc0, time, av, B.hreps, ctrl->herm,
                                                                 (unsigned)std::min<size_t>(B.hrep_cap, 0xFFFFFFFFu),
                                                                 B.hnorm, &ctrl->tickets[8], diag);
        }
        k_dc_solve<<<G.solve, SOLVE_THREADS, sizeof(SolveSmem), st>>>(g0, sc0, time, av, B.fields, D, sp,
                                                                    &ctrl->tickets[1], diag);
        if (project)
            k_dc_project<<<G.flat, BLK_THREADS, 0, st>>>(g0, sc0, time, av, D, sp, &ctrl->dc_vertices,
                                                         &ctrl->tickets[6], diag);
        k_dc_count_quads<<<G.count_quads, 512, 0, st>>>(g0, av, D, B.packet_counts, B.block_totals);
        k_exclusive_scan<<<std::max(1u, scan_tiles(nb)), SCAN_THREADS, 0, st>>>(
            B.block_totals, B.block_offsets, nb, &ctrl->active_count, 1, scan_state(B.scan(B.scanB_off)),
            &ctrl->total_vertices, diag);
        if (qlist) {
            k_dc_quad_list<<<G.count_quads, BLK_THREADS, 0, st>>>(g0, av, D, B.packet_counts, B.block_offsets, B.qrec,
                                                                 D.qcap);
            k_dc_quad_normals<<<G.flat, BLK_THREADS, 0, st>>>(g0, sc0, time, av, D, B.qrec, &ctrl->total_vertices,
                                                              D.qcap, mo.maxV, B.qnorm, &ctrl->tickets[9], diag,
                                                              &ctrl->dc_vertices, mo, m, B.qp);
        }
        k_dc_quads<<<G.quads, BLK_THREADS, sizeof(QuadSmem), st>>>(g0, sc0, time, av, D, nullptr, B.packet_counts,
                                                                   B.block_offsets, mo, m, B.qp, &ctrl->tickets[2],
                                                                   diag, &ctrl->total_vertices, &ctrl->dc_vertices);
    }
    k_batch_scene_first<<<(B.n + 1 + 127) / 128, 128, 0, st>>>(B.desc, B.n, av, B.block_offsets,
                                                                &ctrl->total_vertices, B.first);
    record(cudaMemcpyAsync(B.h_ctrl, ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, st));
    record(cudaMemcpyAsync(B.h_first, B.first, (B.n + 1) * sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    check_launch();
}

struct BatchImpl {
    int device = 0;
    unsigned out_mask = 0;
    int nscenes = 0;
    std::vector<int> group_of, index_in_group;
    BatchGroup g[2];  // marching cubes, dual contouring
    int ctas[4] = {0, 0, 0, 0};
    cudaStream_t cap_stream = nullptr;
    // the dual-contouring group runs on side_stream, concurrently with the marching-cubes group: the two
    // groups share no data, so one group's small stages and tails overlap the other's heavy stages
    cudaStream_t side_stream = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    sdf_outputs graph_out[2]{};
    float graph_time = 0.f;

    void drop_graph() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~BatchImpl() {
        drop_graph();
        g[0].release();
        g[1].release();
        if (cap_stream) cudaStreamDestroy(cap_stream);
        if (side_stream) cudaStreamDestroy(side_stream);
        if (fork_ev) cudaEventDestroy(fork_ev);
        if (join_ev) cudaEventDestroy(join_ev);
    }
};

// both groups' kernels: marching cubes on st, dual contouring on the side stream forked from st and
// joined back into it (in a capture this records two parallel branches of the graph)
static void enqueue_both(BatchImpl& I, const BatchGrids& G, float time, const sdf_outputs* mc_out,
                         const sdf_outputs* dc_out, cudaStream_t st) {
    const bool both = I.g[0].n && I.g[1].n;
    if (both) {
        record(cudaEventRecord(I.fork_ev, st));
        record(cudaStreamWaitEvent(I.side_stream, I.fork_ev, 0));
    }
    enqueue_group(I.g[0], G, time, mc_out, I.out_mask, st);
    enqueue_group(I.g[1], G, time, dc_out, I.out_mask, both ? I.side_stream : st);
    if (both) {
        record(cudaEventRecord(I.join_ev, I.side_stream));
        record(cudaStreamWaitEvent(st, I.join_ev, 0));
    }
}

static bool same_outputs(const sdf_outputs* a, const sdf_outputs& b) {
    sdf_outputs z{};
    return memcmp(a ? a : &z, &b, sizeof(sdf_outputs)) == 0;
}

static sdf_status build_group(BatchGroup& B, const sdf_batch_scene* scenes, unsigned out_mask) {
    using namespace sdfb;
    std::vector<sdf_primitive> prims;
    std::vector<sdf_bvh_node> nodes;
    std::vector<size_t> prim_off, node_off;
    B.desc_host.clear();
    long long blocks = 0, bricks = 0;
    for (int i : B.scenes) {
        const sdf_batch_scene& S = scenes[i];
        const sdf_config& c = S.config;
        GridView gv;
        const float sx = c.bounds_max[0] - c.bounds_min[0], sy = c.bounds_max[1] - c.bounds_min[1],
                    sz = c.bounds_max[2] - c.bounds_min[2];
        if (!(c.cell_size > 0.f) || !(sx > 0.f) || !(sy > 0.f) || !(sz > 0.f)) return SDF_ERR_INVALID;
        gv.w = (int)ceilf(sx / c.cell_size);
        gv.h = (int)ceilf(sy / c.cell_size);
        gv.d = (int)ceilf(sz / c.cell_size);
        gv.bx = (gv.w + 7) / 8; gv.by = (gv.h + 7) / 8; gv.bz = (gv.d + 7) / 8;
        gv.ox = c.bounds_min[0]; gv.oy = c.bounds_min[1]; gv.oz = c.bounds_min[2];
        gv.cell = c.cell_size;
        std::vector<sdf_primitive> sorted;
        std::vector<sdf_bvh_node> nd;
        const int nbvh = prepare_scene(S.prims, S.count, sorted, nd);
        if (bvh_depth(nd) + 1 > MAP_STACK) return SDF_ERR_STACK;
        SceneDesc d;
        d.g = gv;
        d.sc.prims = nullptr;  // patched after the upload
        d.sc.nodes = nullptr;
        d.sc.nprims = (int)sorted.size();
        d.sc.nbvh = nbvh;
        d.sc.nnodes = (int)nd.size();
        d.block_base = (unsigned)blocks;
        d.brick_base = (unsigned)bricks;
        blocks += (long long)gv.bx * gv.by * gv.bz;
        bricks += (long long)sdfb::scout_pair_bricks(gv);
        prim_off.push_back(prims.size());
        node_off.push_back(nodes.size());
        prims.insert(prims.end(), sorted.begin(), sorted.end());
        nodes.insert(nodes.end(), nd.begin(), nd.end());
        B.desc_host.push_back(d);
    }
    if (blocks * 512 >= (1LL << 32) || blocks >= (1LL << 24)) return SDF_ERR_INVALID;  // 32-bit cells, miss list
    B.n = (int)B.desc_host.size();
    B.total_blocks = blocks;
    B.total_bricks = bricks;
    sdf_status s = SDF_OK;
    if (s == SDF_OK) s = dev_alloc(B.prims, std::max<size_t>(prims.size(), 1));
    if (s == SDF_OK) s = dev_alloc(B.nodes, std::max<size_t>(nodes.size(), 1));
    if (s != SDF_OK) return s;
    for (int k = 0; k < B.n; ++k) {
        B.desc_host[k].sc.prims = reinterpret_cast<const float4*>(B.prims + prim_off[k]);
        B.desc_host[k].sc.nodes = reinterpret_cast<const float4*>(B.nodes + node_off[k]);
    }
    if (!prims.empty() && cudaMemcpy(B.prims, prims.data(), prims.size() * sizeof(sdf_primitive),
                                     cudaMemcpyHostToDevice) != cudaSuccess)
        return SDF_ERR_CUDA;
    if (!nodes.empty() && cudaMemcpy(B.nodes, nodes.data(), nodes.size() * sizeof(sdf_bvh_node),
                                     cudaMemcpyHostToDevice) != cudaSuccess)
        return SDF_ERR_CUDA;
    if (s == SDF_OK) s = dev_alloc(B.desc, B.n);
    if (s == SDF_OK && cudaMemcpy(B.desc, B.desc_host.data(), B.n * sizeof(SceneDesc), cudaMemcpyHostToDevice) !=
                           cudaSuccess)
        s = SDF_ERR_CUDA;
    const size_t nb = (size_t)blocks;
    if (s == SDF_OK) s = dev_alloc(B.flags, nb);
    if (s == SDF_OK) s = dev_alloc(B.list, nb);
    if (s == SDF_OK) s = dev_alloc(B.fields, nb * FIELD_STRIDE);
    if (s == SDF_OK) s = dev_alloc(B.block_totals, nb);
    if (s == SDF_OK) s = dev_alloc(B.block_offsets, nb);
    if (s == SDF_OK) s = dev_alloc(B.b2a, nb);
    if (s == SDF_OK) s = dev_alloc(B.first, (size_t)B.n + 1);
    if (s != SDF_OK) return s;
    const bool dc = B.technique == SDF_TECH_DUAL_CONTOURING;
    s = dev_alloc(B.miss, nb * HALO_N);  // the shared-halo block field of both techniques
    if (!dc) {
        if (s == SDF_OK && !(out_mask & (OUT_COLORS | OUT_UVS | OUT_PRIMIDS | OUT_NORMALS)))
            s = dev_alloc(B.cell_words, nb * 512);
    } else {
        const size_t cells = nb * 512;
        if (s == SDF_OK) s = dev_alloc(B.packet_counts, cells);
        if (s == SDF_OK) s = dev_alloc(B.packet_offsets, cells);
        if (s == SDF_OK) s = dev_alloc(B.masks, cells);
        if (s == SDF_OK) s = dev_alloc(B.dc_voff, cells);
        B.dc_cap = std::min<size_t>(cells, (size_t)1 << 28);
        if (s == SDF_OK) s = dev_alloc(B.dc_verts, B.dc_cap);
    }
    if (s != SDF_OK) return s;
    const size_t tA = scan_tiles((unsigned)nb) + 1, tC = scan_tiles((unsigned)(nb * 512)) + 1;
    B.scanA_off = (sizeof(Ctrl) + 255) & ~size_t(255);
    B.scanB_off = B.scanA_off + tA * 8;
    B.scanC_off = B.scanB_off + tA * 8;
    B.ctrl_bytes = B.scanC_off + (dc ? tC * 8 : 8);
    s = dev_alloc(B.ctrl_region, B.ctrl_bytes);
    if (s != SDF_OK) return s;
    if (cudaMallocHost(&B.h_ctrl, sizeof(Ctrl)) != cudaSuccess ||
        cudaMallocHost(&B.h_first, ((size_t)B.n + 1) * sizeof(unsigned)) != cudaSuccess)
        return SDF_ERR_NOMEM;
    return SDF_OK;
}

}  // namespace sdfb

struct sdf_batch {
    sdfb::BatchImpl impl;
};

extern "C" {

sdf_status sdf_batch_create(sdf_batch** out, int device) {
    if (!out) return SDF_ERR_INVALID;
    *out = nullptr;
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return SDF_ERR_CUDA;
    sdf_batch* b = new sdf_batch();
    cudaGetDevice(&b->impl.device);
    if (cudaStreamCreateWithFlags(&b->impl.cap_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->impl.side_stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->impl.fork_ev, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->impl.join_ev, cudaEventDisableTiming) != cudaSuccess) {
        delete b;
        return SDF_ERR_CUDA;
    }
    *out = b;
    return SDF_OK;
}

void sdf_batch_destroy(sdf_batch* b) {
    if (!b) return;
    cudaSetDevice(b->impl.device);
    delete b;
}

sdf_status sdf_batch_set_scenes(sdf_batch* b, const sdf_batch_scene* scenes, int n, uint32_t out_mask) {
    using namespace sdfb;
    if (!b || n <= 0 || !scenes) return SDF_ERR_INVALID;
    BatchImpl& I = b->impl;
    cudaSetDevice(I.device);
    I.drop_graph();
    I.g[0].release();
    I.g[1].release();
    I.g[0].technique = SDF_TECH_MARCHING_CUBES;
    I.g[1].technique = SDF_TECH_DUAL_CONTOURING;
    I.group_of.assign(n, 0);
    I.index_in_group.assign(n, 0);
    const sdf_config* dc_ref = nullptr;
    for (int i = 0; i < n; ++i) {
        const sdf_config& c = scenes[i].config;
        if (scenes[i].count < 0 || (scenes[i].count > 0 && !scenes[i].prims)) return SDF_ERR_INVALID;
        if (c.technique != SDF_TECH_MARCHING_CUBES && c.technique != SDF_TECH_DUAL_CONTOURING) return SDF_ERR_INVALID;
        const int k = c.technique == SDF_TECH_DUAL_CONTOURING ? 1 : 0;
        if (k == 1) {  // one set of DC options per batch
            if (!dc_ref) dc_ref = &c;
            if (c.dc_solver != dc_ref->dc_solver || c.projection_iters != dc_ref->projection_iters ||
                c.adaptive_diagonal != dc_ref->adaptive_diagonal || c.cond_threshold != dc_ref->cond_threshold ||
                c.qef_blend != dc_ref->qef_blend)
                return SDF_ERR_INVALID;
        }
        I.group_of[i] = k;
        I.index_in_group[i] = (int)I.g[k].scenes.size();
        I.g[k].scenes.push_back(i);
    }
    if (dc_ref) {
        BatchGroup& D = I.g[1];
        D.sp.qef_blend = dc_ref->qef_blend;
        D.sp.solver = dc_ref->dc_solver;
        D.sp.projection_iters = dc_ref->dc_solver == SDF_DC_SOLVER_MASSPOINT ? dc_ref->projection_iters : 0;
        D.sp.cond_threshold = dc_ref->cond_threshold > 0.f ? dc_ref->cond_threshold : 1e4f;
        D.qp.adaptive_diagonal = dc_ref->dc_solver == SDF_DC_SOLVER_MASSPOINT ? dc_ref->adaptive_diagonal : 0;
    }
    for (int k = 0; k < 2; ++k) {
        if (I.g[k].scenes.empty()) continue;
        const sdf_status s = build_group(I.g[k], scenes, out_mask);
        if (s != SDF_OK) {
            I.g[0].release();
            I.g[1].release();
            return s;
        }
    }
    I.nscenes = n;
    I.out_mask = out_mask;
    return SDF_OK;
}

// Grows the dual-contouring group's lists to the last run's counts plus a quarter (fractions of the cells
// before any run); true when a buffer moved. Called outside any capture.
static bool batch_size_lists(sdfb::BatchGroup& B) {
    using namespace sdfb;
    if (B.technique != SDF_TECH_DUAL_CONTOURING || B.n == 0) return false;
    bool moved = false;
    auto grow = [&](auto*& p, size_t& cap, size_t want) {
        if (cap >= want) return;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        moved = true;
        if (dev_alloc(p, want) == SDF_OK) cap = want;
        cudaGetLastError();  // without a list the kernels fall back to their in-block paths
    };
    auto want = [&](unsigned last, size_t div) {
        return std::min<size_t>(B.dc_cap, std::max<size_t>(B.dc_cap / div, (size_t)last + last / 4));
    };
    size_t hb = B.hbase ? (size_t)B.total_blocks : 0;
    grow(B.hbase, hb, (size_t)B.total_blocks);
    if (!B.hbase) B.hsamp_cap = B.hrep_cap = 0;
    grow(B.hsamp, B.hsamp_cap, want(B.last_herm[0], 4));
    {
        const size_t w = want(B.last_herm[1], 8);
        size_t c1 = B.hrep_cap, c2 = B.hrep_cap;
        if (c1 < w) {
            grow(B.hreps, c1, w);
            grow(B.hnorm, c2, w);
            B.hrep_cap = std::min(c1, c2);
        }
    }
    {
        const size_t w = want(B.last_total / 6, 16);
        size_t c1 = B.q_cap, c2 = B.q_cap;
        if (c1 < w) {
            grow(B.qrec, c1, w);
            grow(B.qnorm, c2, w);
            B.q_cap = std::min(c1, c2);
        }
    }
    if (B.sp.solver == SDF_DC_SOLVER_MASSPOINT && B.sp.projection_iters > 0) {
        const size_t w = want(B.last_dc, 8);
        if (B.proj_cap < w) {
            if (B.proj) cudaFree(B.proj);
            B.proj = nullptr;
            B.proj_cap = 0;
            moved = true;
            if (dev_alloc(B.proj, 2 * w) == SDF_OK) B.proj_cap = w;
            cudaGetLastError();
        }
    }
    return moved;
}

// the counts the lists are sized by, from the last read-back of the group's control block
static void batch_note_counts(sdfb::BatchGroup& B) {
    if (B.n == 0 || !B.h_ctrl) return;
    B.last_herm[0] = B.h_ctrl->herm[0];
    B.last_herm[1] = B.h_ctrl->herm[1];
    B.last_total = B.h_ctrl->total_vertices;
    B.last_dc = B.h_ctrl->dc_vertices;
}

static sdf_status batch_finish(sdfb::BatchImpl& I, const sdf_outputs* out[2], int64_t* first_vertex,
                               int64_t* vertex_count, sdf_batch_stats* stats, float ms, int graph) {
    using namespace sdfb;
    sdf_status status = SDF_OK;
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->scenes = I.nscenes;
        stats->ms_total = ms;
        stats->graph = graph;
        for (int k = 0; k < 4; ++k) stats->tuned_ctas[k] = I.ctas[k];
    }
    for (int k = 0; k < 2; ++k) {
        BatchGroup& B = I.g[k];
        if (B.n == 0) continue;
        const Ctrl& h = *B.h_ctrl;
        batch_note_counts(B);
        if (h.diag.timeout) status = SDF_ERR_TIMEOUT;
        if (h.diag.inconsistent && status == SDF_OK) status = SDF_ERR_CUDA;
        if (h.diag.stack_overflow && status == SDF_OK) status = SDF_ERR_STACK;
        const unsigned cap = out[k] ? out[k]->max_vertices : 0u;
        if (status == SDF_OK && (h.total_vertices > cap || (k == 1 && h.dc_vertices > B.dc_cap)))
            status = SDF_ERR_CAPACITY;
        if (stats) {
            stats->total_blocks += B.total_blocks;
            stats->active_blocks += h.active_count;
            (k == 0 ? stats->mc_vertices : stats->dc_vertices) = h.total_vertices;
        }
        for (int j = 0; j < B.n; ++j) {
            const int i = B.scenes[j];
            if (first_vertex) first_vertex[i] = B.h_first[j];
            if (vertex_count) vertex_count[i] = (int64_t)B.h_first[j + 1] - (int64_t)B.h_first[j];
        }
    }
    return status;
}

sdf_status sdf_batch_extract(sdf_batch* b, float time, const sdf_outputs* mc_out, const sdf_outputs* dc_out,
                             void* stream, int64_t* first_vertex, int64_t* vertex_count, sdf_batch_stats* stats) {
    using namespace sdfb;
    if (!b || b->impl.nscenes == 0) return SDF_ERR_INVALID;
    BatchImpl& I = b->impl;
    if ((I.g[0].n && (!mc_out || !mc_out->vertices)) || (I.g[1].n && (!dc_out || !dc_out->vertices)))
        return SDF_ERR_INVALID;
    cudaSetDevice(I.device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaGetLastError();
    auto t0 = std::chrono::high_resolution_clock::now();
    const bool replay = I.exec && time == I.graph_time && same_outputs(mc_out, I.graph_out[0]) &&
                        same_outputs(dc_out, I.graph_out[1]);
    const unsigned failures_before = g_launch_failures;
    if (replay) {
        record(cudaGraphLaunch(I.exec, st));
    } else {
        if (batch_size_lists(I.g[1])) I.drop_graph();  // the graph holds the old lists
        const BatchGrids G = batch_grids(std::max(I.g[0].total_blocks, I.g[1].total_blocks), I.ctas);
        enqueue_both(I, G, time, mc_out, dc_out, st);
    }
    const cudaError_t err = cudaStreamSynchronize(st);
    if (g_launch_failures != failures_before) return SDF_ERR_CUDA;  // a kernel was not launched
    auto t1 = std::chrono::high_resolution_clock::now();
    if (err != cudaSuccess) {
        record(err);
        return SDF_ERR_CUDA;
    }
    const sdf_outputs* outs[2] = {mc_out, dc_out};
    return batch_finish(I, outs, first_vertex, vertex_count, stats,
                        std::chrono::duration<float, std::milli>(t1 - t0).count(), replay ? 1 : 0);
}

sdf_status sdf_batch_capture(sdf_batch* b, float time, const sdf_outputs* mc_out, const sdf_outputs* dc_out,
                             void* stream, int tune) {
    using namespace sdfb;
    if (!b || b->impl.nscenes == 0) return SDF_ERR_INVALID;
    BatchImpl& I = b->impl;
    if ((I.g[0].n && (!mc_out || !mc_out->vertices)) || (I.g[1].n && (!dc_out || !dc_out->vertices)))
        return SDF_ERR_INVALID;
    cudaSetDevice(I.device);
    cudaStream_t st = I.cap_stream;
    I.drop_graph();
    const long long blocks = std::max(I.g[0].total_blocks, I.g[1].total_blocks);
    batch_size_lists(I.g[1]);
    if (tune) {
        // coordinate descent over the CTAs per SM of the block field, the emission, the DC solve and
        // the DC quads: each candidate is timed on one direct extraction after a warm-up run
        const int cand[4][3] = {{0, 4, 2}, {0, 4, 2}, {0, 2, 1}, {0, 2, 1}};
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        for (int k = 0; k < 4; ++k) {
            if ((k == 1 && I.g[0].n == 0) || (k >= 2 && I.g[1].n == 0)) continue;
            float best = 1e30f;
            int best_v = 0;
            for (int v : cand[k]) {
                I.ctas[k] = v;
                const BatchGrids G = batch_grids(blocks, I.ctas);
                float ms = 0.f;
                for (int rep = 0; rep < 2; ++rep) {
                    cudaEventRecord(e0, st);
                    enqueue_both(I, G, time, mc_out, dc_out, st);
                    cudaEventRecord(e1, st);
                    if (cudaStreamSynchronize(st) != cudaSuccess) {
                        cudaEventDestroy(e0);
                        cudaEventDestroy(e1);
                        return SDF_ERR_CUDA;
                    }
                    cudaEventElapsedTime(&ms, e0, e1);
                    batch_note_counts(I.g[1]);
                }
                if (ms < best) {
                    best = ms;
                    best_v = v;
                }
            }
            I.ctas[k] = best_v;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    const BatchGrids G = batch_grids(blocks, I.ctas);  // attributes set before the capture
    if (!tune) {  // one direct run gives the counts the lists are sized by
        enqueue_both(I, G, time, mc_out, dc_out, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return SDF_ERR_CUDA;
        batch_note_counts(I.g[1]);
    }
    batch_size_lists(I.g[1]);
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return SDF_ERR_CUDA;
    enqueue_both(I, G, time, mc_out, dc_out, st);
    if (cudaStreamEndCapture(st, &I.graph) != cudaSuccess || !I.graph) {
        I.graph = nullptr;
        cudaGetLastError();
        return SDF_ERR_CUDA;
    }
    if (cudaGraphInstantiate(&I.exec, I.graph, 0) != cudaSuccess) {
        I.drop_graph();
        cudaGetLastError();
        return SDF_ERR_CUDA;
    }
    sdf_outputs z{};
    I.graph_out[0] = mc_out ? *mc_out : z;
    I.graph_out[1] = dc_out ? *dc_out : z;
    I.graph_time = time;
    return SDF_OK;
}

sdf_status sdf_batch_read_buffer(sdf_batch* b, int technique, int which, void* host_dst, size_t* bytes) {
    using namespace sdfb;
    if (!b || !bytes || (technique != SDF_TECH_MARCHING_CUBES && technique != SDF_TECH_DUAL_CONTOURING))
        return SDF_ERR_INVALID;
    BatchImpl& I = b->impl;
    BatchGroup& B = I.g[technique == SDF_TECH_DUAL_CONTOURING ? 1 : 0];
    if (B.n == 0 || !B.h_ctrl) return SDF_ERR_INVALID;
    const size_t act = (size_t)std::min<long long>(B.h_ctrl->active_count, B.total_blocks);
    const void* src = nullptr;
    size_t have = 0;
    switch (which) {
        case 0: src = B.list; have = act * sizeof(int); break;
        case 1: src = B.block_totals; have = act * sizeof(unsigned); break;
        case 2: src = B.packet_counts; have = B.packet_counts ? act * 512 * sizeof(unsigned) : 0; break;
        case 3: src = B.masks; have = B.masks ? act * 512 : 0; break;
        case 4: src = B.dc_voff; have = B.dc_voff ? act * 512 * sizeof(unsigned) : 0; break;
        case 5:
            src = B.dc_verts;
            have = B.dc_verts ? (size_t)std::min<unsigned long long>(B.h_ctrl->dc_vertices, B.dc_cap) * sizeof(ushort4)
                              : 0;
            break;
        default: return SDF_ERR_INVALID;
    }
    const size_t want = std::min(*bytes, have);
    *bytes = have;
    if (!host_dst || want == 0) return SDF_OK;
    cudaSetDevice(I.device);
    const cudaError_t e = cudaMemcpy(host_dst, src, want, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        record(e);
        return SDF_ERR_CUDA;
    }
    return SDF_OK;
}

}  // extern "C"
