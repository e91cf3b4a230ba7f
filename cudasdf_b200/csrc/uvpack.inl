// UV atlas packing: the host side of the reference's GridUVPacker steps (GridUVPacker.cu:833-1547).
// Included by sdfmesh.cu after the other entry points (uses ensure_buffer, check_launch, num_sms).
//
// Per step, the host does what the reference's host does that decides a result: the island bounds
// from the chart table (float arithmetic as GridUVPacker.cu:916-925), std::sort of the islands by
// area (not stable; its permutation depends only on the comparisons, so sorting these records gives
// the reference's order, GridUVPacker.cu:1052-1058), the attempt seeds from srand / rand
// (GridUVPacker.cu:1117-1122) and the shelf width (GridUVPacker.cu:1126-1138). Everything else runs
// on the device, with one read-back per step that needs its size.

struct sdf_uv_atlas {
    // charts
    int64_t T = 0;   // triangles of the last extraction
    int R = 0;       // primitive id range: largest id + 1
    std::vector<sdf_uv_chart> charts;
    int* d_small = nullptr;   // [0] largest id, [1] chart count
    unsigned* d_cnt = nullptr;
    size_t cnt_cap = 0;
    unsigned* d_keys = nullptr;
    size_t keys_cap = 0;
    int* d_chart_of_id = nullptr;
    size_t coi_cap = 0;
    sdf_uv_chart* d_charts = nullptr;
    size_t charts_cap = 0;
    int* d_tri_chart = nullptr;
    size_t tri_cap = 0;
    bool have_charts = false;
    // islands
    std::vector<sdf_uv_island> islands;   // packing order
    int64_t words = 0, rb_n = 0, prof_n = 0;
    sdf_uv_island* d_isl = nullptr;
    size_t isl_cap = 0;
    int* d_slot = nullptr;
    size_t slot_cap = 0;
    int64_t* d_pre = nullptr;
    size_t pre_cap = 0;
    uint32_t* d_words = nullptr;
    size_t words_cap = 0;
    uint16_t* d_rb = nullptr;
    size_t rb_cap = 0;
    int32_t* d_prof = nullptr;
    size_t prof_cap = 0;
    bool have_islands = false;
    // packing
    int num_solutions = 0, n_order = 0;
    std::vector<int32_t> seeds;
    int32_t* d_seeds = nullptr;
    size_t seeds_cap = 0;
    uint32_t* d_boards = nullptr;
    size_t boards_cap = 0;
    sdf_uv_solution* d_sols = nullptr;
    size_t sols_cap = 0;
    sdf_uv_placement* d_pl = nullptr;
    size_t pl_cap = 0;
    sdf_uv_placement* d_best = nullptr;
    size_t best_cap = 0;
    uvp::ChartPlace* d_cp = nullptr;
    size_t cp_cap = 0;
    uvp::AtlasResult* d_res = nullptr;
    sdf_uv_atlas_info info{};
    std::vector<sdf_uv_placement> best;
    bool have_pack = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

namespace {

// (int)f as x86-64 converts it; the reference's host code relies on it for out-of-range values
int uv_host_f2i(float f) { return (f >= -2147483648.0f && f < 2147483648.0f) ? (int)f : INT_MIN; }

int uv_grid(int64_t items, int threads = 256) {
    const int64_t cap = (int64_t)num_sms() * 8;
    const int64_t need = (items + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min(cap, need));
}

sdf_status uv_cuda(cudaError_t e) {
    if (e == cudaSuccess) return SDF_OK;
    record(e);
    return SDF_ERR_CUDA;
}

}  // namespace

extern "C" {

void sdf_uv_pack_default_config(sdf_uv_pack_config* c) {
    if (!c) return;
    // PackingConfig() (GridUVPacker.cuh:135-140)
    c->grid_size = 128;
    c->grid_resolution = 64;
    c->max_iterations = 500;
    c->margin_cells = 2;
    c->enable_rotation = 1;
    c->x_alignment = 8;
    c->max_candidates_per_island = 32;
    c->max_drop_steps = 0;
    c->shuffle_order_per_attempt = 1;
    c->random_seed = 0;
}

sdf_status sdf_uv_atlas_create(sdf_uv_atlas** out) {
    if (!out) return SDF_ERR_INVALID;
    *out = nullptr;
    sdf_uv_atlas* a = new (std::nothrow) sdf_uv_atlas();
    if (!a) return SDF_ERR_NOMEM;
    if (cudaMalloc(&a->d_small, 2 * sizeof(int)) != cudaSuccess ||
        cudaMalloc(&a->d_res, sizeof(uvp::AtlasResult)) != cudaSuccess ||
        cudaEventCreate(&a->ev0) != cudaSuccess || cudaEventCreate(&a->ev1) != cudaSuccess) {
        cudaGetLastError();
        sdf_uv_atlas_destroy(a);
        return SDF_ERR_NOMEM;
    }
    *out = a;
    return SDF_OK;
}

void sdf_uv_atlas_destroy(sdf_uv_atlas* a) {
    if (!a) return;
    void* bufs[] = {a->d_small, a->d_cnt,    a->d_keys, a->d_chart_of_id, a->d_charts, a->d_tri_chart,
                    a->d_isl,   a->d_slot,   a->d_pre,  a->d_words,       a->d_rb,     a->d_prof,
                    a->d_seeds, a->d_boards, a->d_sols, a->d_pl,          a->d_best,   a->d_cp,
                    a->d_res};
    for (void* p : bufs)
        if (p) cudaFree(p);
    if (a->ev0) cudaEventDestroy(a->ev0);
    if (a->ev1) cudaEventDestroy(a->ev1);
    delete a;
}

sdf_status sdf_uv_atlas_extract_charts(sdf_uv_atlas* a, const sdf_float2* d_uvs, const float* d_primitive_ids,
                                       int64_t num_vertices, void* stream, int32_t* num_charts) {
    if (!a || num_vertices < 0 || (num_vertices >= 3 && (!d_uvs || !d_primitive_ids))) return SDF_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    a->have_charts = a->have_islands = a->have_pack = false;
    a->charts.clear();
    a->R = 0;
    const int64_t T = num_vertices / 3;
    a->T = T;
    if (num_charts) *num_charts = 0;
    if (!ensure_buffer(a->d_tri_chart, a->tri_cap, (size_t)std::max<int64_t>(T, 1))) return SDF_ERR_NOMEM;
    int max_id = -1;
    if (T > 0) {
        cudaMemsetAsync(a->d_small, 0xff, sizeof(int), s);
        uvp::k_uv_max_id<<<uv_grid(T), 256, 0, s>>>(d_primitive_ids, T, a->d_small);
        if (check_launch() != cudaSuccess) return SDF_ERR_CUDA;
        cudaMemcpyAsync(&max_id, a->d_small, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (sdf_status st = uv_cuda(cudaStreamSynchronize(s))) return st;
    }
    if (max_id >= (1 << 24)) return SDF_ERR_INVALID;
    const int R = max_id + 1;
    a->R = R;
    if (R > 0) {
        if (!ensure_buffer(a->d_cnt, a->cnt_cap, (size_t)R) || !ensure_buffer(a->d_keys, a->keys_cap, 4 * (size_t)R) ||
            !ensure_buffer(a->d_chart_of_id, a->coi_cap, (size_t)R) ||
            !ensure_buffer(a->d_charts, a->charts_cap, (size_t)R))
            return SDF_ERR_NOMEM;
        uvp::k_uv_hist_init<<<uv_grid(R), 256, 0, s>>>(a->d_cnt, a->d_keys, R);
        uvp::k_uv_hist<<<uv_grid(T), 256, 0, s>>>(d_uvs, d_primitive_ids, T, R, a->d_cnt, a->d_keys);
        uvp::k_uv_chart_compact<<<1, 1024, 0, s>>>(a->d_cnt, a->d_keys, R, a->d_chart_of_id, a->d_charts, a->d_small + 1);
    }
    if (T > 0) uvp::k_uv_tri_chart<<<uv_grid(T), 256, 0, s>>>(d_primitive_ids, T, R, a->d_chart_of_id, a->d_tri_chart);
    if (check_launch() != cudaSuccess) return SDF_ERR_CUDA;
    int nc = 0;
    if (R > 0) {
        cudaMemcpyAsync(&nc, a->d_small + 1, sizeof(int), cudaMemcpyDeviceToHost, s);
        if (sdf_status st = uv_cuda(cudaStreamSynchronize(s))) return st;
        a->charts.resize((size_t)nc);
        if (nc > 0) {
            cudaMemcpyAsync(a->charts.data(), a->d_charts, sizeof(sdf_uv_chart) * (size_t)nc, cudaMemcpyDeviceToHost, s);
            if (sdf_status st = uv_cuda(cudaStreamSynchronize(s))) return st;
        }
    }
    a->have_charts = true;
    if (num_charts) *num_charts = nc;
    return SDF_OK;
}

sdf_status sdf_uv_atlas_create_islands(sdf_uv_atlas* a, const sdf_float2* d_uvs, int32_t grid_resolution,
                                       int32_t margin_cells, void* stream) {
    if (!a || !a->have_charts || margin_cells > 1024 || (a->T > 0 && !d_uvs)) return SDF_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    a->have_islands = a->have_pack = false;
    const int nc = (int)a->charts.size();
    std::vector<sdf_uv_island> isl((size_t)nc);
    for (int i = 0; i < nc; i++) {
        const sdf_uv_chart& c = a->charts[(size_t)i];
        const float fr = (float)grid_resolution;
        const int64_t minX = (int64_t)uv_host_f2i(floorf(c.uv_min.x * fr)) - margin_cells;
        const int64_t minY = (int64_t)uv_host_f2i(floorf(c.uv_min.y * fr)) - margin_cells;
        const int64_t maxX = (int64_t)uv_host_f2i(ceilf(c.uv_max.x * fr)) + margin_cells;
        const int64_t maxY = (int64_t)uv_host_f2i(ceilf(c.uv_max.y * fr)) + margin_cells;
        if (minX < INT_MIN || minY < INT_MIN || maxX > INT_MAX || maxY > INT_MAX) return SDF_ERR_INVALID;
        const int64_t w = std::max<int64_t>(1, maxX - minX), h = std::max<int64_t>(1, maxY - minY);
        if (w > 65536 || h > 65536 || w * h > (int64_t)1 << 30) return SDF_ERR_INVALID;
        sdf_uv_island& d = isl[(size_t)i];
        memset(&d, 0, sizeof(d));
        d.island_index = i;
        d.primitive_id = c.primitive_id;
        d.num_triangles = c.num_triangles;
        d.min_cell_x = (int32_t)minX;
        d.min_cell_y = (int32_t)minY;
        d.width = (int32_t)w;
        d.height = (int32_t)h;
    }
    std::sort(isl.begin(), isl.end(),
              [](const sdf_uv_island& x, const sdf_uv_island& y) { return x.width * x.height > y.width * y.height; });
    std::vector<int> slot((size_t)std::max(nc, 1), -1);
    std::vector<int64_t> pre(3 * ((size_t)nc + 1), 0);
    int64_t words = 0, rbn = 0, prn = 0;
    for (int i = 0; i < nc; i++) {
        sdf_uv_island& d = isl[(size_t)i];
        slot[(size_t)d.island_index] = i;
        const int w = d.width, h = d.height, s0 = (w + 31) / 32, s9 = (h + 31) / 32;
        sdf_uv_grid* gs[4] = {&d.mask, &d.collision, &d.mask90, &d.collision90};
        for (int k = 0; k < 4; k++) {
            const bool rot = k >= 2;
            gs[k]->width = rot ? h : w;
            gs[k]->height = rot ? w : h;
            gs[k]->stride = rot ? s9 : s0;
            gs[k]->word_offset = words;
            words += (int64_t)gs[k]->stride * gs[k]->height;
        }
        d.row_bounds = rbn;
        rbn += 2 * (int64_t)h;
        d.row_bounds90 = rbn;
        rbn += 2 * (int64_t)w;
        d.profile = prn;
        prn += 2 * (int64_t)w;
        d.profile90 = prn;
        prn += 2 * (int64_t)h;
        pre[(size_t)i + 1] = pre[(size_t)i] + (int64_t)s0 * h;                                       // dilation
        pre[(size_t)nc + 1 + i + 1] = pre[(size_t)nc + 1 + i] + 2 * (int64_t)s9 * w;                 // rotation
        pre[2 * ((size_t)nc + 1) + i + 1] = pre[2 * ((size_t)nc + 1) + i] + 2 * ((int64_t)w + h);    // bounds
    }
    if (!ensure_buffer(a->d_isl, a->isl_cap, (size_t)std::max(nc, 1)) ||
        !ensure_buffer(a->d_slot, a->slot_cap, slot.size()) || !ensure_buffer(a->d_pre, a->pre_cap, pre.size()) ||
        !ensure_buffer(a->d_words, a->words_cap, (size_t)std::max<int64_t>(words, 1)) ||
        !ensure_buffer(a->d_rb, a->rb_cap, (size_t)std::max<int64_t>(rbn, 1)) ||
        !ensure_buffer(a->d_prof, a->prof_cap, (size_t)std::max<int64_t>(prn, 1)))
        return SDF_ERR_NOMEM;
    a->islands = isl;
    a->words = words;
    a->rb_n = rbn;
    a->prof_n = prn;
    if (nc > 0) {
        cudaMemcpyAsync(a->d_isl, isl.data(), sizeof(sdf_uv_island) * (size_t)nc, cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(a->d_slot, slot.data(), sizeof(int) * slot.size(), cudaMemcpyHostToDevice, s);
        cudaMemcpyAsync(a->d_pre, pre.data(), sizeof(int64_t) * pre.size(), cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(a->d_words, 0, sizeof(uint32_t) * (size_t)words, s);
        if (a->T > 0)
            uvp::k_uv_raster<<<uv_grid(a->T), 256, 0, s>>>(d_uvs, a->T, a->d_tri_chart, a->d_slot, a->d_isl,
                                                             a->d_words, grid_resolution);
        uvp::k_uv_dilate<<<uv_grid(pre[(size_t)nc]), 256, 0, s>>>(a->d_isl, nc, a->d_pre, a->d_words, margin_cells);
        uvp::k_uv_rotate<<<uv_grid(pre[2 * (size_t)nc + 1]), 256, 0, s>>>(a->d_isl, nc, a->d_pre + nc + 1, a->d_words);
        uvp::k_uv_bounds<<<uv_grid(pre[3 * (size_t)nc + 2]), 256, 0, s>>>(a->d_isl, nc, a->d_pre + 2 * (nc + 1),
                                                                        a->d_words, a->d_rb, a->d_prof);
        if (check_launch() != cudaSuccess) return SDF_ERR_CUDA;
    }
    a->have_islands = true;
    return SDF_OK;
}

sdf_status sdf_uv_atlas_pack(sdf_uv_atlas* a, const sdf_uv_pack_config* c, void* stream, sdf_uv_atlas_info* info) {
    if (!a || !c || !a->have_islands || c->grid_size < 1 || c->grid_size > 16384) return SDF_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    a->have_pack = false;
    a->best.clear();
    sdf_uv_atlas_info& r = a->info;
    memset(&r, 0, sizeof(r));
    r.scaling_factor = 1.0f;
    r.best_solution = -1;
    r.num_charts = (int32_t)a->charts.size();
    r.num_islands = (int32_t)a->islands.size();
    const int G = c->grid_size;
    const int nisl = (int)a->islands.size();
    bool packable = nisl > 0;   // "No islands to pack" (GridUVPacker.cu:1069-1073)
    for (const sdf_uv_island& d : a->islands)   // an island larger than the board (GridUVPacker.cu:1080-1096)
        if (d.width > G || d.height > G) packable = false;
    const int nsol = std::min(c->max_iterations, 256);
    if (nsol <= 0) packable = false;   // the reference's launch of zero attempts fails
    if (!packable) {
        a->have_pack = true;
        if (info) *info = r;
        return SDF_OK;
    }
    // seeds (GridUVPacker.cu:1117-1122)
    a->seeds.assign((size_t)nsol, 0);
    srand(c->random_seed == 0 ? (unsigned int)time(nullptr) : (unsigned int)c->random_seed);
    for (int i = 0; i < nsol; i++) a->seeds[(size_t)i] = rand();
    // shelf width (GridUVPacker.cu:1126-1138)
    int maxW = 0;
    int64_t total = 0;
    for (const sdf_uv_island& d : a->islands) {
        maxW = std::max(maxW, d.width);
        total += (int64_t)d.width * d.height;
    }
    if (total > INT_MAX) return SDF_ERR_INVALID;
    const int target = uv_host_f2i(sqrtf((float)(int)total * 1.3f));
    const int shelf = std::max(maxW * 2 + maxW / 2, std::min(target, G));
    uvp::PackArgs pa;
    pa.G = G;
    pa.bs = (G + 31) / 32;
    pa.align = std::max(1, c->x_alignment);
    pa.shelf_max = std::min(G, uvp::align_down(std::max(1, shelf), pa.align));
    pa.budget = std::max(4, std::min(uvp::kMaxCand, c->max_candidates_per_island));
    pa.drop_cap = c->max_drop_steps;
    pa.n = std::min(nisl, uvp::kMaxOrder);
    pa.num_islands = nisl;
    pa.rotation = c->enable_rotation != 0;
    pa.shuffle = c->shuffle_order_per_attempt != 0;
    const size_t board_words = (size_t)nsol * G * pa.bs;
    if (!ensure_buffer(a->d_seeds, a->seeds_cap, (size_t)nsol) || !ensure_buffer(a->d_boards, a->boards_cap, board_words) ||
        !ensure_buffer(a->d_sols, a->sols_cap, (size_t)nsol) ||
        !ensure_buffer(a->d_pl, a->pl_cap, (size_t)nsol * pa.n) || !ensure_buffer(a->d_best, a->best_cap, (size_t)pa.n))
        return SDF_ERR_NOMEM;
    a->num_solutions = nsol;
    a->n_order = pa.n;
    cudaMemcpyAsync(a->d_seeds, a->seeds.data(), sizeof(int32_t) * (size_t)nsol, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(a->d_boards, 0, sizeof(uint32_t) * board_words, s);
    cudaEventRecord(a->ev0, s);
    uvp::k_uv_pack<<<nsol, uvp::kPackThreads, sizeof(unsigned short) * (size_t)G, s>>>(
        a->d_isl, pa, a->d_seeds, a->d_words, a->d_rb, a->d_prof, a->d_boards, a->d_sols, a->d_pl);
    cudaEventRecord(a->ev1, s);
    uvp::k_uv_select<<<1, 32, 0, s>>>(a->d_sols, nsol, nisl, G, a->d_pl, pa.n, a->d_best, a->d_res);
    if (check_launch() != cudaSuccess) return SDF_ERR_CUDA;
    uvp::AtlasResult res;
    cudaMemcpyAsync(&res, a->d_res, sizeof(res), cudaMemcpyDeviceToHost, s);
    if (sdf_status st = uv_cuda(cudaStreamSynchronize(s))) return st;
    a->best.resize((size_t)std::max(res.placed, 0));
    if (res.placed > 0) {
        cudaMemcpyAsync(a->best.data(), a->d_best, sizeof(sdf_uv_placement) * (size_t)res.placed, cudaMemcpyDeviceToHost, s);
        if (sdf_status st = uv_cuda(cudaStreamSynchronize(s))) return st;
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a->ev0, a->ev1);
    r.success = res.success;
    r.atlas_width = res.width;
    r.atlas_height = res.height;
    r.num_placed = res.placed;
    r.fitness = res.fitness;
    r.scaling_factor = res.scaling;
    r.num_solutions = nsol;
    r.best_solution = res.best;
    r.shelf_width = shelf;
    r.candidate_loop_open = res.open ? 1 : 0;
    r.ms_pack = ms;
    a->have_pack = true;
    if (info) *info = r;
    return SDF_OK;
}

namespace {
sdf_status uv_remap(sdf_uv_atlas* a, sdf_float2* d_uvs, const float* d_prim, int64_t nv, int res,
                    const sdf_uv_placement* d_pl, int np, int atlas_w, int atlas_h, cudaStream_t s) {
    const int nc = (int)a->charts.size();
    if (!ensure_buffer(a->d_cp, a->cp_cap, (size_t)std::max(nc, 1))) return SDF_ERR_NOMEM;
    const int nisl = (int)a->islands.size();
    uvp::k_uv_remap_init<<<uv_grid(nisl), 256, 0, s>>>(a->d_isl, nisl, a->d_cp);
    uvp::k_uv_remap_place<<<uv_grid(np), 256, 0, s>>>(d_pl, np, nc, a->d_cp);
    const float denom = (float)std::max(atlas_w, atlas_h);
    if (nv > 0)
        uvp::k_uv_remap<<<uv_grid(nv), 256, 0, s>>>(d_uvs, d_prim, nv, a->d_chart_of_id, a->R, a->d_cp, res, denom);
    return check_launch() == cudaSuccess ? SDF_OK : SDF_ERR_CUDA;
}
}  // namespace

sdf_status sdf_uv_atlas_remap(sdf_uv_atlas* a, sdf_float2* d_uvs, const float* d_primitive_ids, int64_t num_vertices,
                              int32_t grid_resolution, void* stream) {
    if (!a || num_vertices < 0 || (num_vertices > 0 && (!d_uvs || !d_primitive_ids))) return SDF_ERR_INVALID;
    // "Cannot remap UVs - invalid atlas" (GridUVPacker.cu:1450-1453): the UVs stay as they are
    if (!a->have_pack || !a->info.success || a->best.empty()) return SDF_OK;
    return uv_remap(a, d_uvs, d_primitive_ids, num_vertices, grid_resolution, a->d_best, (int)a->best.size(),
                    a->info.atlas_width, a->info.atlas_height, (cudaStream_t)stream);
}

sdf_status sdf_uv_atlas_remap_placements(sdf_uv_atlas* a, sdf_float2* d_uvs, const float* d_primitive_ids,
                                         int64_t num_vertices, int32_t grid_resolution,
                                         const sdf_uv_placement* placements, int32_t num_placements,
                                         int32_t success, int32_t atlas_width, int32_t atlas_height, void* stream) {
    if (!a || num_vertices < 0 || num_placements < 0 || (num_vertices > 0 && (!d_uvs || !d_primitive_ids)) ||
        (num_placements > 0 && !placements) || !a->have_islands)
        return SDF_ERR_INVALID;
    if (!success || num_placements == 0) return SDF_OK;
    cudaStream_t s = (cudaStream_t)stream;
    if (!ensure_buffer(a->d_best, a->best_cap, (size_t)num_placements)) return SDF_ERR_NOMEM;
    cudaMemcpyAsync(a->d_best, placements, sizeof(sdf_uv_placement) * (size_t)num_placements, cudaMemcpyHostToDevice, s);
    return uv_remap(a, d_uvs, d_primitive_ids, num_vertices, grid_resolution, a->d_best, num_placements, atlas_width,
                    atlas_height, s);
}

sdf_status sdf_uv_atlas_run(sdf_uv_atlas* a, sdf_float2* d_uvs, const float* d_primitive_ids, int64_t num_vertices,
                            const sdf_uv_pack_config* c, void* stream, sdf_uv_atlas_info* info) {
    if (!c) return SDF_ERR_INVALID;
    int32_t nc = 0;
    if (sdf_status st = sdf_uv_atlas_extract_charts(a, d_uvs, d_primitive_ids, num_vertices, stream, &nc)) return st;
    if (sdf_status st = sdf_uv_atlas_create_islands(a, d_uvs, c->grid_resolution, c->margin_cells, stream)) return st;
    if (sdf_status st = sdf_uv_atlas_pack(a, c, stream, info)) return st;
    return sdf_uv_atlas_remap(a, d_uvs, d_primitive_ids, num_vertices, c->grid_resolution, stream);
}

sdf_status sdf_uv_atlas_read(sdf_uv_atlas* a, int which, void* host_dst, size_t* bytes) {
    if (!a || !bytes) return SDF_ERR_INVALID;
    const void* src = nullptr;
    size_t n = 0;
    bool dev = true;
    switch (which) {
        case 0: src = a->charts.data(); n = sizeof(sdf_uv_chart) * a->charts.size(); dev = false; break;
        case 1: src = a->d_tri_chart; n = a->have_charts ? sizeof(int) * (size_t)a->T : 0; break;
        case 2: src = a->islands.data(); n = sizeof(sdf_uv_island) * a->islands.size(); dev = false; break;
        case 3: src = a->d_words; n = a->have_islands ? sizeof(uint32_t) * (size_t)a->words : 0; break;
        case 4: src = a->d_rb; n = a->have_islands ? sizeof(uint16_t) * (size_t)a->rb_n : 0; break;
        case 5: src = a->d_prof; n = a->have_islands ? sizeof(int32_t) * (size_t)a->prof_n : 0; break;
        case 6: src = a->seeds.data(); n = a->have_pack ? sizeof(int32_t) * a->seeds.size() : 0; dev = false; break;
        case 7: src = a->d_sols; n = a->have_pack && a->num_solutions > 0 ? sizeof(sdf_uv_solution) * (size_t)a->num_solutions : 0; break;
        case 8: src = a->d_pl; n = a->have_pack && a->num_solutions > 0 ? sizeof(sdf_uv_placement) * (size_t)a->num_solutions * a->n_order : 0; break;
        case 9: src = a->best.data(); n = a->have_pack ? sizeof(sdf_uv_placement) * a->best.size() : 0; dev = false; break;
        default: return SDF_ERR_INVALID;
    }
    const size_t cap = *bytes;
    *bytes = n;
    if (!host_dst || n == 0) return SDF_OK;
    if (cap < n) return SDF_ERR_CAPACITY;
    if (!dev) {
        memcpy(host_dst, src, n);
        return SDF_OK;
    }
    return uv_cuda(cudaMemcpy(host_dst, src, n, cudaMemcpyDeviceToHost));
}

sdf_status sdf_uv_pack_random_draws(const int32_t* seeds, int32_t num_seeds, int32_t per_seed, uint32_t* host_out) {
    if (!seeds || !host_out || num_seeds < 0 || per_seed < 0) return SDF_ERR_INVALID;
    if (num_seeds == 0 || per_seed == 0) return SDF_OK;
    int32_t* d_s = nullptr;
    uint32_t* d_o = nullptr;
    const size_t n = (size_t)num_seeds * per_seed;
    if (cudaMalloc(&d_s, sizeof(int32_t) * num_seeds) != cudaSuccess || cudaMalloc(&d_o, sizeof(uint32_t) * n) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(d_s);
        cudaFree(d_o);
        return SDF_ERR_NOMEM;
    }
    cudaMemcpy(d_s, seeds, sizeof(int32_t) * num_seeds, cudaMemcpyHostToDevice);
    uvp::k_uv_draws<<<(num_seeds + 127) / 128, 128>>>(d_s, num_seeds, per_seed, d_o);
    cudaError_t e = check_launch();
    if (e == cudaSuccess) e = cudaMemcpy(host_out, d_o, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost);
    cudaFree(d_s);
    cudaFree(d_o);
    return uv_cuda(e);
}

}  // extern "C"
