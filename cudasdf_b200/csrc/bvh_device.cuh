// Scene preparation on the GPU: the primitives reordered unions first and the BVH over the unions,
// with the same sorted array, node order, boxes and leaf assignment as the host builder in bvh_host.h
// (which restates CudaSDFMesh::UpdateBVH, CudaSDFMesh.cpp:216-249, getPrimitiveAABB,
// CudaSDFUtil.h:507-542, and buildBVHRecursive, CudaSDFUtil.h:544-603).
//
// The recursion is run level by level. A segment is a range [start, start + count) of the index
// array with the id of the node it becomes; ids follow the host's pre-order numbering, which is
// fixed by the segment sizes alone (a subtree over m primitives has 2m - 1 nodes, so the left child
// of node id is id + 1 and the right child id + 2 mid). One CTA takes one segment (one warp a segment
// of at most 32):
//   bounds   min / max over the segment (order-free, a block reduction)
//   centroid the host's running sum in index order, kept sequential (one warp adds in order) so that
//            every rounding is the host's; only the axis the split uses is summed
//   split    the host's in-place partition (swap each primitive left of the split with the first
//            primitive right of it) gives: left part = the left primitives in order; right part = a
//            queue that receives each right primitive at its end and, at each left primitive met
//            after the first right one, moves its front element to its end. Entry j of that queue's
//            history is either a right primitive or a copy of entry r (r = moves before it), so the
//            final order follows from two block scans and pointer jumping over the history
//            instead of a sequential loop.
#pragma once

#include "sdf_device.cuh"

namespace sdfb {
namespace bvhd {

constexpr int PREP_THREADS = 1024;
constexpr int BIG_THREADS = 1024;
constexpr int SMALL_THREADS = 256;
constexpr int PREP_CTAS = 1024;            // at most one count per thread of k_bvh_scatter's scan
constexpr int SMEM_HIST = 32768;           // segments up to this size keep their history on chip
constexpr int MAX_LEVELS = MAP_STACK + 1;  // deeper trees are refused by the traversal anyway

struct Seg {
    int start, count, node;
};

struct Ctl {
    int nseg[MAX_LEVELS + 1];  // segments per level
    int nu;                    // primitives in the BVH (unions)
    int depth;                 // levels of the finished tree (the host's bvh_depth)
    int overflow;              // a level beyond MAX_LEVELS was needed
};

// Work arrays, `cap` entries each (cap >= number of unions).
struct Work {
    float* box;   // 6 x cap: min x, y, z, max x, y, z (struct of arrays)
    float* cent;  // 3 x cap: (min + max) * 0.5 per axis
    int* idx[2];  // index arrays of even / odd levels
    int* hist;    // per segment: the right part's queue history (segments too large for shared memory)
    Seg* seg[2];  // segment lists of even / odd levels
    int* cta_count;  // PREP_CTAS: unions per CTA of the partition
    Ctl* ctl;
    int cap;
};

__device__ __forceinline__ bool is_union(int op) { return op == OP_UNION || op == OP_UNION_BLEND; }

// rotateVector as the host build computes it: separate roundings, reference operand order
__device__ __forceinline__ float3 host_rotate_dev(float3 v, float4 q) {
    const float duv = ADD(ADD(MUL(q.x, v.x), MUL(q.y, v.y)), MUL(q.z, v.z));
    const float duu = ADD(ADD(MUL(q.x, q.x), MUL(q.y, q.y)), MUL(q.z, q.z));
    const float a = MUL(2.0f, duv), b = SUB(MUL(q.w, q.w), duu), c = MUL(2.0f, q.w);
    const float3 cr = f3(SUB(MUL(q.y, v.z), MUL(q.z, v.y)), SUB(MUL(q.z, v.x), MUL(q.x, v.z)),
                         SUB(MUL(q.x, v.y), MUL(q.y, v.x)));
    return f3(ADD(ADD(MUL(a, q.x), MUL(b, v.x)), MUL(c, cr.x)), ADD(ADD(MUL(a, q.y), MUL(b, v.y)), MUL(c, cr.y)),
              ADD(ADD(MUL(a, q.z), MUL(b, v.z)), MUL(c, cr.z)));
}

// getPrimitiveAABB (CudaSDFUtil.h:507-542) with the host build's roundings
__device__ __forceinline__ void primitive_box_dev(const sdf_primitive& p, float3& mn, float3& mx) {
    float pad = 0.1f;
    if (p.displacement != 0) pad = ADD(pad, 0.5f);
    float3 dims = f3(1.f, 1.f, 1.f);
    if (p.type == P_SPHERE) dims = f3(p.params[0], p.params[0], p.params[0]);
    else if (p.type == P_BOX || p.type == P_RBOX) dims = f3(p.params[0], p.params[1], p.params[2]);
    else if (p.type == P_TORUS) {
        const float r = ADD(p.params[0], p.params[1]);
        dims = f3(r, p.params[1], r);
    }
    dims = f3(ADD(dims.x, pad), ADD(dims.y, pad), ADD(dims.z, pad));
    const float4 q = make_float4(p.rotation[0], p.rotation[1], p.rotation[2], p.rotation[3]);
    mn = f3(1e10f, 1e10f, 1e10f);
    mx = f3(-1e10f, -1e10f, -1e10f);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const float3 c = f3((i & 1) ? dims.x : -dims.x, (i & 2) ? dims.y : -dims.y, (i & 4) ? dims.z : -dims.z);
        float3 w = host_rotate_dev(f3(MUL(c.x, p.scale[0]), MUL(c.y, p.scale[1]), MUL(c.z, p.scale[2])), q);
        w = f3(ADD(w.x, p.position[0]), ADD(w.y, p.position[1]), ADD(w.z, p.position[2]));
        mn = f3(fminf(mn.x, w.x), fminf(mn.y, w.y), fminf(mn.z, w.z));
        mx = f3(fmaxf(mx.x, w.x), fmaxf(mx.y, w.y), fmaxf(mx.z, w.z));
    }
}

// Stable partition of the primitives (unions first, then the rest, each in input order), the
// unions' boxes and centroids, the identity index array and the root segment, in two grid-wide
// passes: k_bvh_count counts each CTA's unions, k_bvh_scatter places them. CTA b owns primitives
// [b * per, (b + 1) * per).
__global__ void __launch_bounds__(PREP_THREADS) k_bvh_count(const sdf_primitive* __restrict__ in, int n, int per,
                                                           Work w) {
    __shared__ unsigned s_warp[PREP_THREADS / 32];
    const int lo = blockIdx.x * per, hi = min(n, lo + per);
    unsigned cnt = 0;
    for (int i = lo + (int)threadIdx.x; i < hi; i += PREP_THREADS) cnt += is_union(in[i].operation) ? 1u : 0u;
    unsigned tot = 0;
    block_exclusive<PREP_THREADS>(cnt, s_warp, &tot);
    if (threadIdx.x == 0) w.cta_count[blockIdx.x] = (int)tot;
}

__global__ void __launch_bounds__(PREP_THREADS) k_bvh_scatter(const sdf_primitive* __restrict__ in, int n, int per,
                                                             sdf_primitive* __restrict__ sorted,
                                                             sdf_bvh_node* __restrict__ nodes, Work w) {
    __shared__ unsigned s_warp[PREP_THREADS / 32];
    // unions before this CTA's range and in total (gridDim.x <= PREP_THREADS)
    const unsigned c = threadIdx.x < gridDim.x ? (unsigned)w.cta_count[threadIdx.x] : 0u;
    unsigned nu = 0;
    const unsigned before = block_exclusive<PREP_THREADS>(c, s_warp, &nu);
    __shared__ unsigned s_base;
    if (threadIdx.x == blockIdx.x) s_base = before;
    __syncthreads();
    const int lo = blockIdx.x * per, hi = min(n, lo + per);
    unsigned carry_u = s_base, carry_o = (unsigned)lo - s_base;
    for (int base = lo; base < hi; base += PREP_THREADS) {
        const int i = base + (int)threadIdx.x;
        const bool valid = i < hi;
        const bool u = valid && is_union(in[i].operation);
        unsigned tot_u = 0;
        const unsigned pre_u = block_exclusive<PREP_THREADS>(u ? 1u : 0u, s_warp, &tot_u);
        if (valid) {
            const unsigned pre_o = threadIdx.x - pre_u;  // other primitives before i in this chunk
            const unsigned dst = u ? carry_u + pre_u : nu + carry_o + pre_o;
            const float4* src = reinterpret_cast<const float4*>(in + i);
            float4* out = reinterpret_cast<float4*>(sorted + dst);
#pragma unroll
            for (int k = 0; k < PRIM_ROWS; ++k) out[k] = src[k];
            if (u) {
                float3 mn, mx;
                primitive_box_dev(in[i], mn, mx);
                const int cp = w.cap;
                w.box[dst] = mn.x; w.box[cp + dst] = mn.y; w.box[2 * cp + dst] = mn.z;
                w.box[3 * cp + dst] = mx.x; w.box[4 * cp + dst] = mx.y; w.box[5 * cp + dst] = mx.z;
                w.cent[dst] = MUL(ADD(mn.x, mx.x), 0.5f);
                w.cent[cp + dst] = MUL(ADD(mn.y, mx.y), 0.5f);
                w.cent[2 * cp + dst] = MUL(ADD(mn.z, mx.z), 0.5f);
                w.idx[0][dst] = (int)dst;
                if (nu == 1) {  // the whole tree is one leaf
                    sdf_bvh_node nd;
                    nd.min[0] = fminf(1e10f, mn.x); nd.min[1] = fminf(1e10f, mn.y); nd.min[2] = fminf(1e10f, mn.z);
                    nd.max[0] = fmaxf(-1e10f, mx.x); nd.max[1] = fmaxf(-1e10f, mx.y); nd.max[2] = fmaxf(-1e10f, mx.z);
                    nd.left = 0;
                    nd.right = -1;
                    nodes[0] = nd;
                }
            }
        }
        carry_u += tot_u;
        carry_o += (unsigned)min(PREP_THREADS, hi - base) - tot_u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        Ctl& ct = *w.ctl;
        for (int l = 0; l <= MAX_LEVELS; ++l) ct.nseg[l] = 0;
        ct.nu = (int)nu;
        ct.overflow = 0;
        ct.depth = nu > 0 ? 1 : 0;
        if (nu > 1) {
            w.seg[0][0] = Seg{0, (int)nu, 0};
            ct.nseg[0] = 1;
        }
    }
}

__device__ __forceinline__ float block_min(float v, float* s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fminf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s[warp] = v;
    __syncthreads();
    float r = s[0];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = fminf(r, s[k]);
    return r;
}
__device__ __forceinline__ float block_max(float v, float* s) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) s[warp] = v;
    __syncthreads();
    float r = s[0];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) r = fmaxf(r, s[k]);
    return r;
}

__device__ __forceinline__ void write_leaf(const Work& w, sdf_bvh_node* nodes, int id, int prim) {
    sdf_bvh_node nd;
    nd.min[0] = fminf(1e10f, w.box[prim]);
    nd.min[1] = fminf(1e10f, w.box[w.cap + prim]);
    nd.min[2] = fminf(1e10f, w.box[2 * w.cap + prim]);
    nd.max[0] = fmaxf(-1e10f, w.box[3 * w.cap + prim]);
    nd.max[1] = fmaxf(-1e10f, w.box[4 * w.cap + prim]);
    nd.max[2] = fmaxf(-1e10f, w.box[5 * w.cap + prim]);
    nd.left = prim;
    nd.right = -1;
    nodes[id] = nd;
}

// The node of a split segment and its children: children of one primitive become leaves, larger
// ones go to the next level's list.
__device__ __forceinline__ void finish_segment(const Work& w, sdf_bvh_node* nodes, const int* dst, int level,
                                               const Seg& sg, int mid, const float* mn, const float* mx) {
    Ctl& ctl = *w.ctl;
    const int id = sg.node;
    sdf_bvh_node nd;
    nd.min[0] = mn[0]; nd.min[1] = mn[1]; nd.min[2] = mn[2];
    nd.max[0] = mx[0]; nd.max[1] = mx[1]; nd.max[2] = mx[2];
    nd.left = id + 1;
    nd.right = id + 2 * mid;
    nodes[id] = nd;
    const Seg kids[2] = {Seg{sg.start, mid, id + 1}, Seg{sg.start + mid, sg.count - mid, id + 2 * mid}};
    for (int k = 0; k < 2; ++k) {
        if (kids[k].count == 1) {
            write_leaf(w, nodes, kids[k].node, dst[kids[k].start]);
        } else if (level + 1 < MAX_LEVELS) {
            const int slot = atomicAdd(&ctl.nseg[level + 1], 1);
            w.seg[(level + 1) & 1][slot] = kids[k];
        } else {
            ctl.overflow = 1;
        }
    }
    atomicMax(&ctl.depth, level + 2);
}

// Segments of more than 32 primitives, one CTA (BIG_THREADS) each. The segment's centroids along
// the split axis and then its queue history live in `hist`: dynamic shared memory for segments of
// up to `smem_cap` primitives, else the segment's range of w.hist.
__global__ void __launch_bounds__(BIG_THREADS) k_bvh_big(Work w, sdf_bvh_node* __restrict__ nodes, int level,
                                                        int smem_cap) {
    extern __shared__ int s_dyn[];
    __shared__ float s_red[32];
    __shared__ unsigned s_warp[BIG_THREADS / 32];
    __shared__ float s_split;
    __shared__ int s_more;
    Ctl& ctl = *w.ctl;
    const int nseg = ctl.nseg[level];
    const int* __restrict__ src = w.idx[level & 1];
    int* __restrict__ dst = w.idx[(level + 1) & 1];
    const Seg* __restrict__ segs = w.seg[level & 1];
    const int c6 = w.cap;
    const unsigned FULL = 0xffffffffu;
    for (int s = blockIdx.x; s < nseg; s += gridDim.x) {
        const Seg sg = segs[s];
        const int start = sg.start, count = sg.count;
        if (count <= 32) continue;  // the same for the whole CTA
        int* hist = count <= smem_cap ? s_dyn : w.hist + start;
        // bounds (fminf / fmaxf are order-free)
        float mn[3] = {1e10f, 1e10f, 1e10f}, mx[3] = {-1e10f, -1e10f, -1e10f};
        for (int i = threadIdx.x; i < count; i += blockDim.x) {
            const int p = src[start + i];
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                mn[k] = fminf(mn[k], w.box[k * c6 + p]);
                mx[k] = fmaxf(mx[k], w.box[(3 + k) * c6 + p]);
            }
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = block_min(mn[k], s_red);
            mx[k] = block_max(mx[k], s_red);
        }
        const float ex = SUB(mx[0], mn[0]), ey = SUB(mx[1], mn[1]), ez = SUB(mx[2], mn[2]);
        int axis = 0;
        if (ey > ex) axis = 1;
        if (ez > ey && ez > ex) axis = 2;
        const float* __restrict__ cent = w.cent + axis * c6;
        for (int i = threadIdx.x; i < count; i += blockDim.x) hist[i] = __float_as_int(cent[src[start + i]]);
        __syncthreads();
        // the centroid sum in index order by warp 0: 32 values per step, added in order (every lane
        // adds the same values in the same order)
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            float cc = 0.f;
            int b = 0;
            for (; b + 32 <= count; b += 32) {
                const float v = __int_as_float(hist[b + lane]);
#pragma unroll
                for (int q = 0; q < 32; ++q) cc = ADD(cc, __shfl_sync(FULL, v, q));
            }
            const float v = b + lane < count ? __int_as_float(hist[b + lane]) : 0.f;
            for (int q = 0; q < count - b; ++q) cc = ADD(cc, __shfl_sync(FULL, v, q));
            if (lane == 0) s_split = MUL(cc, DIV(1.0f, (float)count));
        }
        __syncthreads();
        const float split = s_split;
        // partition: left primitives keep their order; the right part is the queue history's tail.
        // A step writes history entry j <= its own index, so the centroids of later chunks survive.
        unsigned carry_l = 0, carry_r = 0;  // left primitives / queue moves so far
        for (int b = 0; b < count; b += blockDim.x) {
            const int i = b + (int)threadIdx.x;
            const bool valid = i < count;
            const int p = valid ? src[start + i] : 0;
            const bool left = valid && __int_as_float(hist[i < count ? i : 0]) < split;
            unsigned tl = 0;
            const unsigned pl = carry_l + block_exclusive<BIG_THREADS>(left ? 1u : 0u, s_warp, &tl);
            const unsigned rights_before = (unsigned)i - pl;  // right primitives before i
            const bool move = left && rights_before > 0;      // the queue is not empty
            unsigned tr = 0;
            const unsigned pr = carry_r + block_exclusive<BIG_THREADS>(move ? 1u : 0u, s_warp, &tr);
            if (valid) {
                if (left) dst[start + (int)pl] = p;
                const unsigned j = rights_before + pr;  // history entry of this step
                if (!left) hist[j] = p;
                else if (move) hist[j] = -(int)pr - 1;  // a copy of entry pr
            }
            carry_l += tl;
            carry_r += tr;
        }
        const int nleft = (int)carry_l, moves = (int)carry_r;
        const int nright = count - nleft;
        const int hlen = nright + moves;
        // resolve copies by pointer jumping (each entry points to an earlier one; chains halve per round)
        for (int round = 0; round < 64; ++round) {
            __syncthreads();
            if (threadIdx.x == 0) s_more = 0;
            __syncthreads();
            for (int j = threadIdx.x; j < hlen; j += blockDim.x) {
                const int v = hist[j];
                if (v < 0) {
                    const int t = hist[-v - 1];
                    hist[j] = t;
                    if (t < 0) s_more = 1;
                }
            }
            __syncthreads();
            if (!s_more) break;
        }
        for (int k = threadIdx.x; k < nright; k += blockDim.x) {
            const int v = hist[moves + k];
            dst[start + nleft + k] = v < 0 ? 0 : v;
            if (v < 0) ctl.overflow = 2;  // unresolved copy (cannot happen)
        }
        __syncthreads();
        int mid = nleft;
        if (mid == 0 || mid == count) mid = count / 2;
        if (threadIdx.x == 0) finish_segment(w, nodes, dst, level, sg, mid, mn, mx);
        __syncthreads();
    }
}

// Segments of at most 32 primitives: one warp each, lane i on the segment's primitive i, the queue
// history in registers.
__global__ void __launch_bounds__(SMALL_THREADS) k_bvh_small(Work w, sdf_bvh_node* __restrict__ nodes, int level) {
    __shared__ int s_hist[SMALL_THREADS / 32][32];
    Ctl& ctl = *w.ctl;
    const int nseg = ctl.nseg[level];
    const int* __restrict__ src = w.idx[level & 1];
    int* __restrict__ dst = w.idx[(level + 1) & 1];
    const Seg* __restrict__ segs = w.seg[level & 1];
    const int c6 = w.cap;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const unsigned FULL = 0xffffffffu;
    for (int s = blockIdx.x * wpb + warp; s < nseg; s += gridDim.x * wpb) {
        const Seg sg = segs[s];
        const int start = sg.start, count = sg.count;
        if (count > 32) continue;  // the same for the whole warp
        const bool has = lane < count;
        const int p = has ? src[start + lane] : 0;
        float mn[3], mx[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            mn[k] = has ? fminf(1e10f, w.box[k * c6 + p]) : 1e10f;
            mx[k] = has ? fmaxf(-1e10f, w.box[(3 + k) * c6 + p]) : -1e10f;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                mn[k] = fminf(mn[k], __shfl_xor_sync(FULL, mn[k], o));
                mx[k] = fmaxf(mx[k], __shfl_xor_sync(FULL, mx[k], o));
            }
        }
        const float ex = SUB(mx[0], mn[0]), ey = SUB(mx[1], mn[1]), ez = SUB(mx[2], mn[2]);
        int axis = 0;
        if (ey > ex) axis = 1;
        if (ez > ey && ez > ex) axis = 2;
        const float c = has ? w.cent[axis * c6 + p] : 0.f;
        float cc = 0.f;
        for (int q = 0; q < count; ++q) cc = ADD(cc, __shfl_sync(FULL, c, q));
        const float split = MUL(cc, DIV(1.0f, (float)count));
        const bool left = has && c < split;
        const unsigned below = (1u << lane) - 1u;
        const unsigned bl = __ballot_sync(FULL, left);
        const int pl = __popc(bl & below);
        const int rb = lane - pl;
        const bool move = left && rb > 0;
        const unsigned bm = __ballot_sync(FULL, move);
        const int pr = __popc(bm & below);
        const int nleft = __popc(bl), moves = __popc(bm), nright = count - nleft;
        if (has && (!left || move)) s_hist[warp][rb + pr] = left ? -pr - 1 : p;
        __syncwarp();
        int h = lane < nright + moves ? s_hist[warp][lane] : 0;
        for (int round = 0; round < 32 && __any_sync(FULL, h < 0); ++round) {
            const int v = __shfl_sync(FULL, h, h < 0 ? -h - 1 : lane);
            if (h < 0) h = v;
        }
        const int right_elem = __shfl_sync(FULL, h, (moves + lane) & 31);
        if (left) dst[start + pl] = p;
        if (lane < nright) dst[start + nleft + lane] = right_elem < 0 ? 0 : right_elem;
        if (lane < nright && right_elem < 0) ctl.overflow = 2;  // unresolved (cannot happen)
        __syncwarp();
        int mid = nleft;
        if (mid == 0 || mid == count) mid = count / 2;
        if (lane == 0) finish_segment(w, nodes, dst, level, sg, mid, mn, mx);
        __syncwarp();
    }
}

}  // namespace bvhd
}  // namespace sdfb
