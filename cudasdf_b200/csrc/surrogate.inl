// Learned surrogate: training, certification, culling control and audit (included at the end of
// sdfmesh.cu, after engine.inl). The kernels are in surrogate.cuh.
#include <cmath>
#include <random>

namespace sdfb {

// f_net error of every exact-active block whose coarse block was culled, and the culled coarse blocks
__global__ void k_sur_audit(const unsigned* __restrict__ flags, int bx, int by, int bz,
                            const float* __restrict__ coarse_f, int cx, int cy, int cz, float margin,
                            unsigned long long* __restrict__ counters) {
    const long long nb = (long long)bx * by * bz, nc = (long long)cx * cy * cz;
    const long long n = nb > nc ? nb : nc;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        if (i < nb && flags[i]) {
            const int x = (int)(i % bx), t = (int)(i / bx), y = t % by, z = t / by;
            const long long c = x / SUR_SPAN_BLOCKS + (long long)cx * (y / SUR_SPAN_BLOCKS + (long long)cy * (z / SUR_SPAN_BLOCKS));
            if (fabsf(coarse_f[c]) > margin) atomicAdd(&counters[0], 1ull);
        }
        if (i < nc && fabsf(coarse_f[i]) > margin) atomicAdd(&counters[1], 1ull);
    }
}

static sdf_status surrogate_state(EngineImpl& E) {
    if (E.sur) return SDF_OK;
    SurrogateState* S = new SurrogateState();
    sdf_status s = SDF_OK;
    if (s == SDF_OK) s = dev_alloc(S->theta, sur::NPARAM);
    if (s == SDF_OK) s = dev_alloc(S->m1, sur::NPARAM);
    if (s == SDF_OK) s = dev_alloc(S->m2, sur::NPARAM);
    if (s == SDF_OK) s = dev_alloc(S->grad, sur::NPARAM);
    if (s == SDF_OK) s = dev_alloc(S->wbf, sur::NW);
    if (s == SDF_OK) s = dev_alloc(S->freq, sur::NF * 3);
    if (s == SDF_OK) s = dev_alloc(S->error, 1);
    if (s == SDF_OK) s = dev_alloc(S->counters, 2);
    if (s == SDF_OK) {
        S->partial_rows = num_sms();
        s = dev_alloc(S->partial, (size_t)S->partial_rows * sur::PART_STRIDE);
    }
    if (s == SDF_OK) s = dev_alloc(S->loss_partial, S->partial_rows);
    if (s != SDF_OK) {
        delete S;
        return s;
    }
    cudaMemset(S->error, 0, sizeof(int));
    E.sur = S;
    return SDF_OK;
}

static int train_grid(int tiles) {
    int per_sm = 0;
    cudaFuncSetAttribute(sur::k_sur_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(sur::TrainSmem));
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sur::k_sur_train, sur::TILE, sizeof(sur::TrainSmem));
    // the kernel holds all 512 tensor-memory columns of its SM: one CTA per SM
    return std::max(1, std::min(num_sms(), tiles));
}

// one forward + backward pass over n samples; leaves the per-CTA partials in S.partial and returns
// the grid used
static int surrogate_pass(SurrogateState& S, const float* pts, const float* tgt, int n, cudaStream_t st) {
    const int tiles = (n + sur::TILE - 1) / sur::TILE;
    const int grid = std::min(train_grid(tiles), S.partial_rows);
    sur::k_sur_train<<<grid, sur::TILE, sizeof(sur::TrainSmem), st>>>(S.view(), pts, tgt, n, 1.f / (float)n, S.partial,
                                                                      S.loss_partial, S.error);
    check_launch();
    return grid;
}

// Smallest eps with |f_net - clamp(f)| <= eps at every sample where |f_net| > eps + reach: the samples
// sorted by decreasing |f_net|, the running maximum of their errors, then a bisection on eps (the
// condition only gets easier as eps grows, since fewer samples qualify and the bound is larger).
static float conditional_certificate(const std::vector<float>& fnet, const std::vector<float>& f, float clampv,
                                     float reach) {
    const size_t n = fnet.size();
    std::vector<std::pair<float, float>> v(n);  // (|f_net|, error)
    float emax = 0.f;
    for (size_t i = 0; i < n; ++i) {
        const float t = std::min(std::max(f[i], -clampv), clampv);
        v[i] = {std::fabs(fnet[i]), std::fabs(fnet[i] - t)};
        emax = std::max(emax, v[i].second);
    }
    std::sort(v.begin(), v.end(), [](const std::pair<float, float>& a, const std::pair<float, float>& b) {
        return a.first > b.first;
    });
    std::vector<float> runmax(n + 1, 0.f);  // runmax[k] = max error of the k largest |f_net|
    for (size_t k = 0; k < n; ++k) runmax[k + 1] = std::max(runmax[k], v[k].second);
    auto ok = [&](float eps) {
        // number of samples with |f_net| > eps + reach
        size_t lo = 0, hi = n;
        while (lo < hi) {
            const size_t mid = (lo + hi) / 2;
            if (v[mid].first > eps + reach) lo = mid + 1; else hi = mid;
        }
        return runmax[lo] <= eps;
    };
    if (ok(0.f)) return 0.f;
    float lo = 0.f, hi = emax;  // ok(emax) holds
    for (int it = 0; it < 40; ++it) {
        const float mid = 0.5f * (lo + hi);
        if (ok(mid)) hi = mid; else lo = mid;
    }
    return hi;
}

static bool surrogate_error(SurrogateState& S) {
    int err = 0;
    cudaMemcpy(&err, S.error, sizeof(int), cudaMemcpyDeviceToHost);
    if (err) cudaMemset(S.error, 0, sizeof(int));
    return err != 0;
}

}  // namespace sdfb

extern "C" {

int sdf_surrogate_num_params(void) { return sdfb::sur::NPARAM; }

void sdf_surrogate_default_config(sdf_surrogate_config* c) {
    if (!c) return;
    c->samples = 2000000;
    c->validation = 262144;
    c->steps = 1500;
    c->batch = 65536;
    c->lr = 2e-3f;
    c->freq_sigma = 2.f;
    c->surface_sigma = 0.01f;
    c->clamp = 0.25f;
    c->surface_res = 128;
    c->slack_cells = 2.f;
    c->time = 0.f;
    c->seed = 1u;
}

sdf_status sdf_surrogate_set_params(sdf_engine* e, const float* theta, const float* freq, const float io[7]) {
    using namespace sdfb;
    if (!e || !theta || !freq || !io) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    cudaSetDevice(E.device);
    sdf_status s = surrogate_state(E);
    if (s != SDF_OK) return s;
    SurrogateState& S = *E.sur;
    if (cudaMemcpy(S.theta, theta, sur::NPARAM * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(S.freq, freq, sur::NF * 3 * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
        return SDF_ERR_CUDA;
    for (int k = 0; k < 7; ++k) S.io[k] = io[k];
    sur::k_sur_pack_weights<<<(sur::NW + 255) / 256, 256>>>(S.theta, S.wbf);
    cudaMemset(S.m1, 0, sur::NPARAM * sizeof(float));
    cudaMemset(S.m2, 0, sur::NPARAM * sizeof(float));
    S.has_params = true;
    S.certified = S.enabled = false;
    return cudaDeviceSynchronize() == cudaSuccess ? SDF_OK : SDF_ERR_CUDA;
}

sdf_status sdf_surrogate_get_params(sdf_engine* e, float* theta, float* freq, float io[7]) {
    using namespace sdfb;
    if (!e || !e->impl.sur || !e->impl.sur->has_params) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    cudaSetDevice(E.device);
    SurrogateState& S = *E.sur;
    if (theta && cudaMemcpy(theta, S.theta, sur::NPARAM * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SDF_ERR_CUDA;
    if (freq && cudaMemcpy(freq, S.freq, sur::NF * 3 * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SDF_ERR_CUDA;
    if (io)
        for (int k = 0; k < 7; ++k) io[k] = S.io[k];
    return SDF_OK;
}

sdf_status sdf_surrogate_forward(sdf_engine* e, const float* d_points, int n, float* d_out, void* stream) {
    using namespace sdfb;
    if (!e || n < 0 || (n > 0 && (!d_points || !d_out))) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    if (!E.sur || !E.sur->has_params) return SDF_ERR_INVALID;
    if (n == 0) return SDF_OK;
    cudaSetDevice(E.device);
    SurrogateState& S = *E.sur;
    sur::PointArray pa{d_points, n};
    const size_t smem = sizeof(sur::InferSmem);
    const int tiles = (n + sur::TILE - 1) / sur::TILE;
    sur::k_sur_infer<sur::PointArray><<<persistent_grid(sur::k_sur_infer<sur::PointArray>, sur::TILE, tiles, smem),
                                        sur::TILE, smem, static_cast<cudaStream_t>(stream)>>>(S.view(), pa, d_out,
                                                                                              S.error);
    return cudaGetLastError() == cudaSuccess ? SDF_OK : SDF_ERR_CUDA;
}

sdf_status sdf_surrogate_gradient(sdf_engine* e, const float* d_points, const float* d_targets, int n, float* h_grad,
                                  float* h_loss) {
    using namespace sdfb;
    if (!e || n <= 0 || !d_points || !d_targets) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    if (!E.sur || !E.sur->has_params) return SDF_ERR_INVALID;
    cudaSetDevice(E.device);
    SurrogateState& S = *E.sur;
    const int grid = surrogate_pass(S, d_points, d_targets, n, 0);
    sur::k_sur_adam<<<(sur::NPARAM + 255) / 256, 256>>>(S.theta, S.m1, S.m2, S.partial, grid, S.grad, 0.f, 0.f, 0.f,
                                                       0.f, 1.f, 1.f, 0, S.wbf);
    const cudaError_t err = cudaDeviceSynchronize();
    if (err != cudaSuccess) {
        record(err);
        return SDF_ERR_CUDA;
    }
    if (surrogate_error(S)) return SDF_ERR_TIMEOUT;
    if (h_grad && cudaMemcpy(h_grad, S.grad, sur::NPARAM * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
        return SDF_ERR_CUDA;
    if (h_loss) {
        std::vector<float> lp(grid);
        if (cudaMemcpy(lp.data(), S.loss_partial, grid * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess)
            return SDF_ERR_CUDA;
        double sum = 0.0;
        for (float v : lp) sum += v;
        *h_loss = (float)(sum / n);
    }
    return SDF_OK;
}

sdf_status sdf_surrogate_train(sdf_engine* e, const sdf_surrogate_config* cfg_in, sdf_surrogate_stats* stats) {
    using namespace sdfb;
    if (!e) return SDF_ERR_INVALID;
    sdf_surrogate_config C;
    if (cfg_in)
        C = *cfg_in;
    else
        sdf_surrogate_default_config(&C);
    if (C.batch <= 0 || C.samples < C.batch || C.steps < 0 || C.validation <= 0 || C.surface_res < 8 ||
        !(C.clamp > 0.f) || !(C.lr >= 0.f) || !(C.slack_cells >= 0.f))
        return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    if (!E.configured) return SDF_ERR_INVALID;
    cudaSetDevice(E.device);
    sdf_status s = surrogate_state(E);
    if (s != SDF_OK) return s;
    SurrogateState& S = *E.sur;
    S.certified = S.enabled = false;

    // ---- initial parameters: frequencies N(0, sigma^2); layers U(-1/sqrt(fan_in), 1/sqrt(fan_in))
    {
        std::mt19937 rng(C.seed);
        std::normal_distribution<float> nd(0.f, C.freq_sigma);
        std::uniform_real_distribution<float> ud(-0.125f, 0.125f);
        std::vector<float> theta(sur::NPARAM), freq(sur::NF * 3);
        for (float& f : freq) f = nd(rng);
        for (float& t : theta) t = ud(rng);
        float io[7];
        for (int k = 0; k < 3; ++k) {
            io[k] = 0.5f * (E.cfg.bounds_min[k] + E.cfg.bounds_max[k]);
            io[3 + k] = 2.f / (E.cfg.bounds_max[k] - E.cfg.bounds_min[k]);
        }
        io[6] = C.clamp;
        s = sdf_surrogate_set_params(e, theta.data(), freq.data(), io);
        if (s != SDF_OK) return s;
    }
    cudaEvent_t ev[4];
    for (auto& x : ev) cudaEventCreate(&x);
    cudaEventRecord(ev[0]);

    // ---- surface points: a coarse marching-cubes run of the same scene over the same bounds
    const int nt = C.samples, nv = C.validation;
    float* pts = nullptr;
    float* tgt = nullptr;
    float* fnet = nullptr;
    sdf_float4* verts = nullptr;
    unsigned* maxbits = nullptr;
    const uint32_t vcap = 1u << 22;
    int64_t nverts = 0;
    auto cleanup = [&]() {
        void* ptrs[] = {pts, tgt, fnet, verts, maxbits};
        for (void* p : ptrs)
            if (p) cudaFree(p);
        for (auto& x : ev) cudaEventDestroy(x);
    };
    if (dev_alloc(pts, (size_t)(nt + nv) * 3) != SDF_OK || dev_alloc(tgt, (size_t)(nt + nv)) != SDF_OK ||
        dev_alloc(fnet, (size_t)nv) != SDF_OK || dev_alloc(verts, vcap) != SDF_OK || dev_alloc(maxbits, 1) != SDF_OK) {
        cleanup();
        return SDF_ERR_NOMEM;
    }
    {
        sdf_engine* tmp = nullptr;
        s = sdf_engine_create(&tmp, E.device);
        if (s == SDF_OK) {
            sdf_config cc = E.cfg;
            float ext = 0.f;
            for (int k = 0; k < 3; ++k) ext = std::max(ext, E.cfg.bounds_max[k] - E.cfg.bounds_min[k]);
            cc.cell_size = ext / (float)C.surface_res;
            cc.technique = SDF_TECH_MARCHING_CUBES;
            cc.out_mask = 0;
            sdf_outputs o;
            memset(&o, 0, sizeof(o));
            o.vertices = verts;
            o.max_vertices = vcap;
            sdf_stats st;
            s = sdf_engine_configure(tmp, &cc);
            // a scene built on the GPU has no host copy: its sorted primitives give the same BVH
            std::vector<sdf_primitive> host_scene;
            const std::vector<sdf_primitive>* scene = &E.scene;
            if (E.device_scene) {
                host_scene.resize((size_t)E.nprims);
                if (E.nprims > 0 && cudaMemcpy(host_scene.data(), E.d_prims, host_scene.size() * sizeof(sdf_primitive),
                                               cudaMemcpyDeviceToHost) != cudaSuccess)
                    s = SDF_ERR_CUDA;
                scene = &host_scene;
            }
            if (s == SDF_OK) s = sdf_engine_set_scene(tmp, scene->data(), (int)scene->size());
            if (s == SDF_OK) {
                s = sdf_engine_extract(tmp, C.time, &o, nullptr, &st);
                if (s == SDF_ERR_CAPACITY) s = SDF_OK;  // a subset of the surface is enough
                nverts = std::min<int64_t>(st.total_vertices, vcap);
            }
            sdf_engine_destroy(tmp);
            cudaSetDevice(E.device);
        }
        if (s != SDF_OK) {
            cleanup();
            return s;
        }
    }
    // ---- samples and their exact distances (training set, then the held-out set)
    const float* bmin = E.cfg.bounds_min;
    const float* bmax = E.cfg.bounds_max;
    sur::k_sur_samples<<<(nt + 255) / 256, 256>>>(reinterpret_cast<const float4*>(verts), (unsigned)nverts, nt, nt / 2,
                                                  C.seed * 2654435761u + 1u, bmin[0], bmin[1], bmin[2], bmax[0], bmax[1],
                                                  bmax[2], C.surface_sigma, pts);
    sur::k_sur_samples<<<(nv + 255) / 256, 256>>>(reinterpret_cast<const float4*>(verts), (unsigned)nverts, nv, nv / 2,
                                                  C.seed * 2654435761u + 0x51ED27u, bmin[0], bmin[1], bmin[2], bmax[0],
                                                  bmax[1], bmax[2], C.surface_sigma, pts + (size_t)3 * nt);
    check_launch();
    s = sdf_engine_eval_distance(e, pts, nt + nv, C.time, tgt, nullptr);
    if (s != SDF_OK) {
        cleanup();
        return s;
    }
    cudaEventRecord(ev[1]);

    // ---- Adam steps over contiguous batches, cosine-decayed learning rate
    const int nbatches = nt / C.batch;
    const float b1 = 0.9f, b2 = 0.999f;
    double bc1 = 1.0, bc2 = 1.0;
    int grid = 1;
    for (int step = 0; step < C.steps; ++step) {
        const size_t off = (size_t)(step % nbatches) * C.batch;
        grid = surrogate_pass(S, pts + 3 * off, tgt + off, C.batch, 0);
        bc1 *= b1;
        bc2 *= b2;
        const double frac = C.steps > 1 ? (double)step / (double)(C.steps - 1) : 1.0;
        const float lr = (float)(C.lr * (0.02 + 0.98 * 0.5 * (1.0 + cos(M_PI * frac))));
        sur::k_sur_adam<<<(sur::NPARAM + 255) / 256, 256>>>(S.theta, S.m1, S.m2, S.partial, grid, nullptr, lr, b1, b2,
                                                           1e-8f, (float)(1.0 - bc1), (float)(1.0 - bc2), 1, S.wbf);
    }
    check_launch();
    cudaEventRecord(ev[2]);

    // ---- certificate over the held-out samples
    cudaMemset(maxbits, 0, sizeof(unsigned));
    s = sdf_surrogate_forward(e, pts + (size_t)3 * nt, nv, fnet, nullptr);
    if (s == SDF_OK) {
        sur::k_sur_max_err<<<std::min((nv + 255) / 256, num_sms() * 8), 256>>>(fnet, tgt + nt, nv, C.clamp, maxbits);
        cudaEventRecord(ev[3]);
        if (cudaDeviceSynchronize() != cudaSuccess) s = SDF_ERR_CUDA;
    }
    if (s == SDF_OK && surrogate_error(S)) s = SDF_ERR_TIMEOUT;
    unsigned bits = 0;
    float loss = 0.f, eps_cert = 0.f;
    if (s == SDF_OK) {
        cudaMemcpy(&bits, maxbits, sizeof(unsigned), cudaMemcpyDeviceToHost);
        std::vector<float> hf(nv), ht(nv);
        cudaMemcpy(hf.data(), fnet, nv * sizeof(float), cudaMemcpyDeviceToHost);
        cudaMemcpy(ht.data(), tgt + nt, nv * sizeof(float), cudaMemcpyDeviceToHost);
        eps_cert = conditional_certificate(hf, ht, C.clamp, surrogate_reach(E, C.slack_cells));
        if (C.steps > 0) {
            std::vector<float> lp(grid);
            cudaMemcpy(lp.data(), S.loss_partial, grid * sizeof(float), cudaMemcpyDeviceToHost);
            double sum = 0.0;
            for (float v : lp) sum += v;
            loss = (float)(sum / C.batch);
        }
    }
    float eps = 0.f;
    memcpy(&eps, &bits, sizeof(float));
    if (s == SDF_OK && !(std::isfinite(eps) && std::isfinite(eps_cert))) s = SDF_ERR_CUDA;
    if (s == SDF_OK) {
        S.eps = eps_cert;
        S.slack_cells = C.slack_cells;
        S.certified = true;
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        stats->final_loss = loss;
        stats->eps_max = eps;
        stats->eps_cert = eps_cert;
        stats->margin = s == SDF_OK ? surrogate_margin(E) : 0.f;
        stats->surface_points = (int32_t)nverts;
        if (s == SDF_OK) {
            cudaEventElapsedTime(&stats->ms_samples, ev[0], ev[1]);
            cudaEventElapsedTime(&stats->ms_train, ev[1], ev[2]);
            cudaEventElapsedTime(&stats->ms_certify, ev[2], ev[3]);
        }
    }
    cleanup();
    return s;
}

sdf_status sdf_surrogate_enable(sdf_engine* e, int enabled) {
    if (!e) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    if (enabled && (!E.sur || !E.sur->certified)) return SDF_ERR_INVALID;
    if (E.sur) {
        E.sur->enabled = enabled != 0;
        E.sur->exact_coarse = false;
    }
    return SDF_OK;
}

sdf_status sdf_engine_set_coarse_cull(sdf_engine* e, int mode, float extra_margin) {
    using namespace sdfb;
    if (!e || mode < SDF_CULL_NONE || mode > SDF_CULL_EXACT || !(extra_margin >= 0.f)) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    if (mode == SDF_CULL_SURROGATE) return sdf_surrogate_enable(e, 1);
    if (mode == SDF_CULL_NONE) {
        if (E.sur) E.sur->enabled = E.sur->exact_coarse = false;
        return SDF_OK;
    }
    cudaSetDevice(E.device);
    const sdf_status s = surrogate_state(E);  // the coarse-field buffer and the audit counters
    if (s != SDF_OK) return s;
    E.sur->exact_coarse = true;
    E.sur->exact_extra = extra_margin;
    E.sur->enabled = true;
    return SDF_OK;
}

sdf_status sdf_surrogate_audit(sdf_engine* e, float time, int64_t* violations, int64_t* culled, int64_t* coarse) {
    using namespace sdfb;
    if (!e) return SDF_ERR_INVALID;
    EngineImpl& E = e->impl;
    if (!E.configured || !E.sur || !(E.sur->certified || E.sur->exact_coarse)) return SDF_ERR_INVALID;
    cudaSetDevice(E.device);
    SurrogateState& S = *E.sur;
    Ctrl* ctrl = reinterpret_cast<Ctrl*>(E.ctrl_region);
    record(cudaMemsetAsync(&ctrl->diag, 0, sizeof(Diag), 0));
    const SceneView sv = engine_scene_view(E);
    const GridView& gv = E.gv;
    const int nbricks = scout_pair_bricks(gv);
    k_scout_t<false><<<(nbricks + BLK_THREADS / 32 - 1) / (BLK_THREADS / 32), BLK_THREADS>>>(gv, sv, time, E.flags,
                                                                                            &ctrl->diag, nullptr, 0.f, nullptr);
    sdf_status s = surrogate_coarse_eval(E, 0, time);
    if (s != SDF_OK) return s;
    int cx, cy, cz;
    coarse_dims(E, cx, cy, cz);
    cudaMemset(S.counters, 0, 2 * sizeof(unsigned long long));
    k_sur_audit<<<num_sms() * 4, 256>>>(E.flags, gv.bx, gv.by, gv.bz, S.coarse_f, cx, cy, cz, surrogate_margin(E),
                                       S.counters);
    unsigned long long h[2] = {0, 0};
    if (cudaDeviceSynchronize() != cudaSuccess) return SDF_ERR_CUDA;
    if (surrogate_error(S)) return SDF_ERR_TIMEOUT;
    cudaMemcpy(h, S.counters, sizeof(h), cudaMemcpyDeviceToHost);
    if (violations) *violations = (int64_t)h[0];
    if (culled) *culled = (int64_t)h[1];
    if (coarse) *coarse = (int64_t)cx * cy * cz;
    return SDF_OK;
}

}  // extern "C"
