// Learned surrogate of the composite distance: a Fourier-feature MLP evaluated and trained on the
// 5th-generation tensor cores (tcgen05.mma, operands in shared memory, accumulators in tensor memory).
//
//   x_n  = (p - centre) * inv_half                      (grid bounds mapped to [-1, 1]^3)
//   g    = [sin(2 pi B x_n), cos(2 pi B x_n)]           B: 32 x 3 fixed Gaussian frequencies -> 64 features
//   h_l  = SiLU(W_l h_{l-1} + b_l),  l = 1..4            W_l: 64 x 64, BF16 operands, FP32 accumulation
//   f    = w5 . h_4 + b5                                 FP32 on the CUDA cores
//
// One CTA of 128 threads owns a tile of 128 samples: thread t holds sample row t, which is also
// tensor-memory lane t of every accumulator (M = 128, cta_group::1). Every 64 x 64 layer is four
// tcgen05.mma of K = 16 issued by thread 0 and tracked by one mbarrier; the epilogue (bias, SiLU,
// conversion to BF16) runs on the CUDA cores after tcgen05.ld and writes the next layer's operand
// back to shared memory. Training runs the same forward pass, keeps the four pre-activations in tensor
// memory and runs the backward pass with two more MMAs per layer: dW_l += dZ_l^T H_{l-1} (K = the 128
// samples of the tile, accumulated in tensor memory over all tiles of the CTA) and
// dH_{l-1} = dZ_l W_l. Per-CTA gradient partials go to global memory; k_sur_adam reduces them.
//
// Shared-memory operand layout (no swizzle, K-major): 8-row x 16-byte core matrices, the eight (or
// sixteen) K-chunks of one 8-row group stored next to each other:
//     offset(row, k) = ((row / 8) * KCH + k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2,   KCH = K / 8
// so the leading-dimension byte offset (between K-chunks) is 128 and the stride byte offset (between
// 8-row groups) is KCH * 128; the K = 16 step of one MMA advances the start address by 256 bytes.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

namespace sdfb {
namespace sur {

constexpr int NF = 32;                        // Fourier frequencies
constexpr int W = 64;                         // layer width (= feature count)
constexpr int NL = 4;                         // hidden layers
constexpr int TILE = 128;                     // samples per tile (MMA M)
constexpr int NW = NL * W * W;                // hidden weights
constexpr int NPARAM = NW + NL * W + W + 1;   // trainable parameters: W, b, w5, b5
constexpr int OFF_B = NW;                     // biases b_l
constexpr int OFF_W5 = NW + NL * W;           // output weights
constexpr int OFF_B5 = OFF_W5 + W;            // output bias
constexpr int PART_STRIDE = (NPARAM + 3) & ~3; // row stride of the per-CTA partials (16-byte rows)
constexpr unsigned IDESC_M128_N64 =           // kind::f16 instruction descriptor
    (1u << 4)                                 // D: FP32
    | (1u << 7) | (1u << 10)                  // A, B: BF16
    | ((uint32_t)(W >> 3) << 17)              // N = 64
    | ((uint32_t)(TILE >> 4) << 24);          // M = 128
constexpr long long WAIT_CYCLES = 4000000000LL;  // about two seconds at the boost clock

// Network view passed to the kernels (device pointers).
struct NetView {
    const float* theta;            // NPARAM fp32 master parameters
    const __nv_bfloat16* wbf;      // NL x 64 x 64 BF16 copies of the hidden weights
    const float* freq;             // NF x 3 frequencies
    float cx, cy, cz;              // input centre
    float sx, sy, sz;              // input scale (1 / half extent)
    float clamp;                   // training targets are clamped to [-clamp, clamp]
};

// ------------------------------------------------------------------------------------------------
// PTX wrappers
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Waits for the phase with the given parity to complete; gives up after WAIT_CYCLES and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity) {
    if (mbar_test(bar, parity)) return true;
    const long long t0 = clock64();
    for (;;) {
        if (mbar_test(bar, parity)) return true;
        if (clock64() - t0 > WAIT_CYCLES) return false;
        __nanosleep(64);
    }
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(dst)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void async_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(IDESC_M128_N64), "r"(accumulate)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

// One warp reads 32 consecutive FP32 columns of its 32 lanes (thread i <- lane base + i).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// ------------------------------------------------------------------------------------------------
// activation: SiLU(v) = v * sigmoid(v), sigmoid(v) = 0.5 + 0.5 tanh(v / 2) (hardware tanh)
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ float tanh_hw(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float sigmoid_hw(float v) { return fmaf(0.5f, tanh_hw(0.5f * v), 0.5f); }

// ------------------------------------------------------------------------------------------------
// operand layout helpers
// ------------------------------------------------------------------------------------------------
template <int KCH>
__device__ __forceinline__ uint32_t op_off(int row, int k) {
    return (uint32_t)(((row >> 3) * KCH + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// writes a 64-wide FP32 row as BF16 into a K = 64 operand (row = sample)
__device__ __forceinline__ void put_row64(unsigned char* buf, int row, const float* v) {
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        __nv_bfloat162 p0 = __floats2bfloat162_rn(v[8 * c + 0], v[8 * c + 1]);
        __nv_bfloat162 p1 = __floats2bfloat162_rn(v[8 * c + 2], v[8 * c + 3]);
        __nv_bfloat162 p2 = __floats2bfloat162_rn(v[8 * c + 4], v[8 * c + 5]);
        __nv_bfloat162 p3 = __floats2bfloat162_rn(v[8 * c + 6], v[8 * c + 7]);
        uint4 q;
        q.x = *reinterpret_cast<uint32_t*>(&p0);
        q.y = *reinterpret_cast<uint32_t*>(&p1);
        q.z = *reinterpret_cast<uint32_t*>(&p2);
        q.w = *reinterpret_cast<uint32_t*>(&p3);
        *reinterpret_cast<uint4*>(buf + op_off<8>(row, 8 * c)) = q;
    }
}

// writes a 64-wide FP32 row as BF16 into column `col` of a K = 128 operand whose rows are features
__device__ __forceinline__ void put_col128(unsigned char* buf, int col, const float* v) {
#pragma unroll
    for (int k = 0; k < 64; ++k)
        *reinterpret_cast<__nv_bfloat16*>(buf + op_off<16>(k, col)) = __float2bfloat16_rn(v[k]);
}

// ------------------------------------------------------------------------------------------------
// Fourier features of one point
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ void features(const float* s_freq, float x, float y, float z, float* g) {
#pragma unroll
    for (int j = 0; j < NF; ++j) {
        const float t = 2.f * fmaf(s_freq[3 * j + 2], z, fmaf(s_freq[3 * j + 1], y, s_freq[3 * j] * x));
        float sn, cs;
        sincospif(t, &sn, &cs);
        g[j] = sn;
        g[NF + j] = cs;
    }
}

// Sums v[0..63] over the 32 lanes of a warp by recursive halving (62 shuffles); lane L receives the
// sums of elements 2L and 2L + 1. v is overwritten.
__device__ __forceinline__ float2 warp_sum64(float* v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 16, half = 32; o > 0; o >>= 1, half >>= 1) {
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int j = 0; j < half; ++j) {
            const float keep = up ? v[half + j] : v[j];
            const float send = up ? v[j] : v[half + j];
            v[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return make_float2(v[0], v[1]);
}

// loads the hidden weights (BF16, [layer][out][in]) into K-major operands; if `transposed`, also the
// transposed copies of layers 2..4 used by the backward pass
__device__ void load_weights(const __nv_bfloat16* __restrict__ wbf, unsigned char* s_w, unsigned char* s_wt) {
    for (int i = threadIdx.x; i < NL * W * W / 8; i += blockDim.x) {
        const int l = i / (W * W / 8), r = (i / 8) % W, c = i % 8;
        const uint4 q = reinterpret_cast<const uint4*>(wbf)[i];
        *reinterpret_cast<uint4*>(s_w + l * 8192 + op_off<8>(r, 8 * c)) = q;
        if (s_wt && l > 0) {
            const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&q);
#pragma unroll
            for (int j = 0; j < 8; ++j)
                *reinterpret_cast<__nv_bfloat16*>(s_wt + (l - 1) * 8192 + op_off<8>(8 * c + j, r)) = e[j];
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Inference: f_net at n points. POINTS supplies point i (see the two sources below).
// ------------------------------------------------------------------------------------------------
struct PointArray {
    const float* p;  // xyz, stride 3
    int n;
    __device__ float3 operator()(int i) const { return make_float3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
};

// centres of the coarse blocks of `span` x `span` x `span` cells of a grid
struct CoarseCentres {
    float ox, oy, oz, cell;
    int cx, cy, cz, span;
    int n;
    __device__ float3 operator()(int i) const {
        const int x = i % cx, t = i / cx, y = t % cy, z = t / cy;
        const float h = 0.5f * (float)span;
        return make_float3(ox + ((float)(x * span) + h) * cell, oy + ((float)(y * span) + h) * cell,
                           oz + ((float)(z * span) + h) * cell);
    }
};

struct InferSmem {
    unsigned char w[NL * 8192];   // K-major hidden weights
    unsigned char a[TILE * 128];  // activation operand (128 x 64 BF16)
    float bias[NL * W];
    float w5[W];
    float freq[NF * 3];
    float b5;
    uint64_t bar;
    uint32_t tmem;
    int fail;
};

template <class POINTS>
__global__ void __launch_bounds__(TILE) k_sur_infer(NetView net, POINTS pts, float* __restrict__ out,
                                                  int* __restrict__ error) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    InferSmem& S = *reinterpret_cast<InferSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5;
    load_weights(net.wbf, S.w, nullptr);
    for (int i = tid; i < NL * W; i += TILE) S.bias[i] = net.theta[OFF_B + i];
    if (tid < W) S.w5[tid] = net.theta[OFF_W5 + tid];
    if (tid < NF * 3) S.freq[tid] = net.freq[tid];
    if (tid == 0) {
        S.b5 = net.theta[OFF_B5];
        S.fail = 0;
        mbar_init(&S.bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(&S.tmem, 64);
    async_fence();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = S.tmem;
    const uint32_t my_lanes = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t a_addr = saddr(S.a), w_addr = saddr(S.w);
    unsigned phase = 0;
    const int ntiles = (pts.n + TILE - 1) / TILE;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int i = tile * TILE + tid;
        float v[64];
        {
            float3 p = i < pts.n ? pts(i) : make_float3(0.f, 0.f, 0.f);
            features(S.freq, (p.x - net.cx) * net.sx, (p.y - net.cy) * net.sy, (p.z - net.cz) * net.sz, v);
        }
        put_row64(S.a, tid, v);
        float f = S.b5;
        for (int l = 0; l < NL; ++l) {
            async_fence();
            tc_before_sync();
            __syncthreads();
            tc_after_sync();
            if (tid == 0) {
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    mma_bf16(tmem, smem_desc(a_addr + 256 * s, 128, 1024), smem_desc(w_addr + l * 8192 + 256 * s, 128, 1024),
                             s > 0);
                mma_commit(&S.bar);
            }
            if (!mbar_wait(&S.bar, phase)) S.fail = 1;
            phase ^= 1;
            tc_after_sync();
            tmem_ld32(my_lanes, v);
            tmem_ld32(my_lanes + 32, v + 32);
#pragma unroll
            for (int j = 0; j < 64; ++j) {
                const float z = v[j] + S.bias[l * W + j];
                v[j] = z * sigmoid_hw(z);
            }
            if (l + 1 < NL) {
                put_row64(S.a, tid, v);
            } else {
#pragma unroll
                for (int j = 0; j < 64; ++j) f = fmaf(S.w5[j], v[j], f);
            }
            tc_before_sync();
            __syncthreads();
            if (S.fail) break;
        }
        if (S.fail) break;
        if (i < pts.n) out[i] = f;
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (S.fail && tid == 0) atomicExch(error, 1);
    if (warp == 0) tmem_dealloc(tmem, 64);
}

// ------------------------------------------------------------------------------------------------
// Training: one pass over n samples (forward + backward), gradient partials per CTA.
// ------------------------------------------------------------------------------------------------
struct TrainSmem {
    unsigned char w[NL * 8192];        // W_l, K-major over inputs   (forward B operand)
    unsigned char wt[(NL - 1) * 8192]; // W_l^T for l = 2..4         (backward dH B operand)
    unsigned char a[TILE * 128];       // H_{l-1}, row = sample       (forward A operand)
    unsigned char ht[NL][W * 256];     // H_{l-1}^T, row = feature, K = 128 samples (dW B operand)
    unsigned char dz[TILE * 128];      // dZ_l, row = sample          (dH A operand)
    unsigned char dzt[TILE * 256];     // dZ_l^T, rows 0..63 = feature, 64..127 unused (dW A operand)
    float bias[NL * W];
    float w5[W];
    float freq[NF * 3];
    float gbias[NL * W];               // bias gradients of this CTA
    float gw5[W];
    float red[2][TILE / 32];           // b5 gradient and loss, per warp
    float b5;
    uint64_t bar;
    uint32_t tmem;
    int fail;
};

// tensor-memory columns: Z_l (and later dH_{l-1}) at 64 (l - 1); dW_l at 256 + 64 (l - 1)
__global__ void __launch_bounds__(TILE, 1) k_sur_train(NetView net, const float* __restrict__ pts,
                                                     const float* __restrict__ target, int n, float inv_n,
                                                     float* __restrict__ partial, float* __restrict__ loss_partial,
                                                     int* __restrict__ error) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    TrainSmem& S = *reinterpret_cast<TrainSmem*>(smem_raw);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    load_weights(net.wbf, S.w, S.wt);
    for (int i = tid; i < NL * W; i += TILE) {
        S.bias[i] = net.theta[OFF_B + i];
        S.gbias[i] = 0.f;
    }
    if (tid < W) {
        S.w5[tid] = net.theta[OFF_W5 + tid];
        S.gw5[tid] = 0.f;
    }
    if (tid < NF * 3) S.freq[tid] = net.freq[tid];
    // rows 64..127 of the dZ^T operand only feed accumulator rows that are never read; keep them finite
    for (int i = tid; i < TILE * 256 / 16; i += TILE) reinterpret_cast<uint4*>(S.dzt)[i] = make_uint4(0, 0, 0, 0);
    if (tid == 0) {
        S.b5 = net.theta[OFF_B5];
        S.fail = 0;
        mbar_init(&S.bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(&S.tmem, 512);
    async_fence();
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    const uint32_t tmem = S.tmem;
    const uint32_t my_lanes = tmem + ((uint32_t)(warp * 32) << 16);
    const uint32_t a_addr = saddr(S.a), w_addr = saddr(S.w), wt_addr = saddr(S.wt), dz_addr = saddr(S.dz),
                   dzt_addr = saddr(S.dzt);
    unsigned phase = 0;
    float gb5 = 0.f, loss = 0.f;
    bool first = true;
    const int ntiles = (n + TILE - 1) / TILE;
    auto sync_mma = [&]() {
        // all threads: publish shared-memory operands, order prior tensor-memory reads
        async_fence();
        tc_before_sync();
        __syncthreads();
        tc_after_sync();
    };
    auto wait_mma = [&]() {  // every thread waits; the barrier makes S.fail uniform
        if (!mbar_wait(&S.bar, phase)) S.fail = 1;
        phase ^= 1;
        __syncthreads();
        tc_after_sync();
    };
    for (int tile = blockIdx.x; tile < ntiles && !S.fail; tile += gridDim.x) {
        const int i = tile * TILE + tid;
        const bool valid = i < n;
        float v[64];
        {
            const float x = valid ? pts[3 * i] : 0.f, y = valid ? pts[3 * i + 1] : 0.f, z = valid ? pts[3 * i + 2] : 0.f;
            features(S.freq, (x - net.cx) * net.sx, (y - net.cy) * net.sy, (z - net.cz) * net.sz, v);
        }
        put_row64(S.a, tid, v);
        put_col128(S.ht[0], tid, v);
        float f = S.b5;
        // ---------------- forward ----------------
        for (int l = 0; l < NL; ++l) {
            sync_mma();
            if (tid == 0) {
#pragma unroll
                for (int s = 0; s < 4; ++s)
                    mma_bf16(tmem + 64 * l, smem_desc(a_addr + 256 * s, 128, 1024),
                             smem_desc(w_addr + l * 8192 + 256 * s, 128, 1024), s > 0);
                mma_commit(&S.bar);
            }
            wait_mma();
            if (S.fail) break;
            tmem_ld32(my_lanes + 64 * l, v);
            tmem_ld32(my_lanes + 64 * l + 32, v + 32);
#pragma unroll
            for (int j = 0; j < 64; ++j) {
                const float zz = v[j] + S.bias[l * W + j];
                v[j] = zz * sigmoid_hw(zz);
            }
            if (l + 1 < NL) {
                tc_before_sync();
                __syncthreads();  // the layer's MMA has completed; S.a may be overwritten
                put_row64(S.a, tid, v);
                put_col128(S.ht[l + 1], tid, v);
            }
        }
        if (S.fail) break;
        // ---------------- output layer and loss ----------------
#pragma unroll
        for (int j = 0; j < 64; ++j) f = fmaf(S.w5[j], v[j], f);
        const float t = valid ? fminf(fmaxf(target[i], -net.clamp), net.clamp) : 0.f;
        const float e = valid ? f - t : 0.f;
        loss = fmaf(e, e, loss);
        const float g = 2.f * e * inv_n;  // dLoss/df for the mean squared error
        gb5 += g;
        float dh[64];
#pragma unroll
        for (int j = 0; j < 64; ++j) v[j] *= g;
        {
            const float2 r = warp_sum64(v);
            atomicAdd(&S.gw5[2 * lane], r.x);
            atomicAdd(&S.gw5[2 * lane + 1], r.y);
        }
#pragma unroll
        for (int j = 0; j < 64; ++j) dh[j] = g * S.w5[j];
        // ---------------- backward ----------------
        for (int l = NL - 1; l >= 0; --l) {
            if (l < NL - 1) {  // dH_l was produced into the columns of Z_{l+1}
                tmem_ld32(my_lanes + 64 * (l + 1), dh);
                tmem_ld32(my_lanes + 64 * (l + 1) + 32, dh + 32);
            }
            tmem_ld32(my_lanes + 64 * l, v);
            tmem_ld32(my_lanes + 64 * l + 32, v + 32);
#pragma unroll
            for (int j = 0; j < 64; ++j) {
                const float zz = v[j] + S.bias[l * W + j];
                const float s = sigmoid_hw(zz);
                v[j] = valid ? dh[j] * s * fmaf(zz, 1.f - s, 1.f) : 0.f;
            }
            put_row64(S.dz, tid, v);
            put_col128(S.dzt, tid, v);
            {
                const float2 r = warp_sum64(v);
                atomicAdd(&S.gbias[l * W + 2 * lane], r.x);
                atomicAdd(&S.gbias[l * W + 2 * lane + 1], r.y);
            }
            sync_mma();
            if (tid == 0) {
                // dW_l += dZ^T H_{l-1}: K = 128 samples, eight steps of 16
#pragma unroll
                for (int s = 0; s < 8; ++s)
                    mma_bf16(tmem + 256 + 64 * l, smem_desc(dzt_addr + 256 * s, 128, 2048),
                             smem_desc(saddr(S.ht[l]) + 256 * s, 128, 2048), (!first || s > 0) ? 1u : 0u);
                if (l > 0) {
                    // dH_{l-1} = dZ W_l into the columns of Z_l (read above)
#pragma unroll
                    for (int s = 0; s < 4; ++s)
                        mma_bf16(tmem + 64 * l, smem_desc(dz_addr + 256 * s, 128, 1024),
                                 smem_desc(wt_addr + (l - 1) * 8192 + 256 * s, 128, 1024), s > 0);
                }
                mma_commit(&S.bar);
            }
            wait_mma();
            if (S.fail) break;
        }
        first = false;
        tc_before_sync();
        __syncthreads();
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    float* mine = partial + (size_t)blockIdx.x * PART_STRIDE;
    if (!S.fail) {
        // dW rows 0..63 live in lanes 0..63: warps 0 and 1
        if (warp < 2) {
            for (int l = 0; l < NL; ++l) {
                float w[64];
                if (first) {
#pragma unroll
                    for (int j = 0; j < 64; ++j) w[j] = 0.f;
                } else {
                    tmem_ld32(my_lanes + 256 + 64 * l, w);
                    tmem_ld32(my_lanes + 256 + 64 * l + 32, w + 32);
                }
                float4* dst = reinterpret_cast<float4*>(mine + l * W * W + tid * W);
#pragma unroll
                for (int j = 0; j < 16; ++j) dst[j] = make_float4(w[4 * j], w[4 * j + 1], w[4 * j + 2], w[4 * j + 3]);
            }
        }
        for (int i = tid; i < NL * W; i += TILE) mine[OFF_B + i] = S.gbias[i];
        if (tid < W) mine[OFF_W5 + tid] = S.gw5[tid];
    }
    // b5 gradient and loss: warp sums then one thread
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        gb5 += __shfl_xor_sync(0xffffffffu, gb5, o);
        loss += __shfl_xor_sync(0xffffffffu, loss, o);
    }
    if (lane == 0) {
        S.red[0][warp] = gb5;
        S.red[1][warp] = loss;
    }
    tc_before_sync();
    __syncthreads();
    tc_after_sync();
    if (tid == 0) {
        float a = 0.f, b = 0.f;
        for (int k = 0; k < TILE / 32; ++k) {
            a += S.red[0][k];
            b += S.red[1][k];
        }
        mine[OFF_B5] = S.fail ? 0.f : a;
        loss_partial[blockIdx.x] = b;
        if (S.fail) atomicExch(error, 1);
    }
    if (warp == 0) tmem_dealloc(tmem, 512);
}

// Sums the per-CTA partials of parameter i; optionally applies one Adam step and refreshes the BF16
// copies of the hidden weights.
__global__ void k_sur_adam(float* __restrict__ theta, float* __restrict__ m1, float* __restrict__ m2,
                           const float* __restrict__ partial, int nparts, float* __restrict__ grad_out, float lr,
                           float beta1, float beta2, float eps, float bc1, float bc2, int apply,
                           __nv_bfloat16* __restrict__ wbf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= NPARAM) return;
    float g = 0.f;
    for (int c = 0; c < nparts; ++c) g += partial[(size_t)c * PART_STRIDE + i];
    if (grad_out) grad_out[i] = g;
    if (!apply) return;
    const float a = beta1 * m1[i] + (1.f - beta1) * g;
    const float b = beta2 * m2[i] + (1.f - beta2) * g * g;
    m1[i] = a;
    m2[i] = b;
    const float th = theta[i] - lr * (a / bc1) / (sqrtf(b / bc2) + eps);
    theta[i] = th;
    if (i < NW) wbf[i] = __float2bfloat16_rn(th);
}

__global__ void k_sur_pack_weights(const float* __restrict__ theta, __nv_bfloat16* __restrict__ wbf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < NW) wbf[i] = __float2bfloat16_rn(theta[i]);
}

// ------------------------------------------------------------------------------------------------
// Training samples: the first half uniform in the box, the second half at mesh vertices plus an
// isotropic Gaussian offset (counter-based hash generator, Box-Muller).
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}
__device__ __forceinline__ float unit01(uint32_t h) { return ((float)(h >> 8) + 0.5f) * (1.f / 16777216.f); }

__global__ void k_sur_samples(const float4* __restrict__ verts, unsigned nverts, int n, int n_uniform, uint32_t seed,
                              float bx0, float by0, float bz0, float bx1, float by1, float bz1, float sigma,
                              float* __restrict__ pts) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t k = hash32(seed ^ hash32((uint32_t)i * 0x9E3779B9u));
    float x, y, z;
    if (i < n_uniform || nverts == 0) {
        x = bx0 + (bx1 - bx0) * unit01(hash32(k + 1));
        y = by0 + (by1 - by0) * unit01(hash32(k + 2));
        z = bz0 + (bz1 - bz0) * unit01(hash32(k + 3));
    } else {
        const float4 v = verts[hash32(k + 4) % nverts];
        const float u1 = unit01(hash32(k + 5)), u2 = unit01(hash32(k + 6));
        const float u3 = unit01(hash32(k + 7)), u4 = unit01(hash32(k + 8));
        const float r1 = sqrtf(-2.f * logf(u1)), r2 = sqrtf(-2.f * logf(u3));
        float s1, c1, s2, c2;
        sincospif(2.f * u2, &s1, &c1);
        sincospif(2.f * u4, &s2, &c2);
        x = v.x + sigma * r1 * c1;
        y = v.y + sigma * r1 * s1;
        z = v.z + sigma * r2 * c2;
    }
    pts[3 * i] = x;
    pts[3 * i + 1] = y;
    pts[3 * i + 2] = z;
}

// max |f_net - clamp(f)| over n points (f_net and f given), as an ordered-int atomic max
__global__ void k_sur_max_err(const float* __restrict__ fnet, const float* __restrict__ f, int n, float clampv,
                              unsigned* __restrict__ out_bits) {
    float m = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float t = fminf(fmaxf(f[i], -clampv), clampv);
        m = fmaxf(m, fabsf(fnet[i] - t));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out_bits, __float_as_uint(m));  // non-negative floats order as uints
}

}  // namespace sur
}  // namespace sdfb
