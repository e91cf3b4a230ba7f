// Host-side scene preparation, restating the reference's BVH construction so that node order,
// boxes and leaf assignment are identical (the node order is part of the parity contract: map()
// visits nodes in this order and its 256-pop cap depends on it).
//   CudaSDFMesh::UpdateBVH   CudaSDFMesh.cpp:216-249  (unions first, BVH over unions only)
//   getPrimitiveAABB         CudaSDFUtil.h:507-542    (tight box for sphere/box/torus, else +-1)
//   buildBVHRecursive        CudaSDFUtil.h:544-603    (mean-centroid split on the longest axis)
// The reference compiles this as host code without fused multiply-adds; this file is built with
// -ffp-contract=off so that every operation rounds the same way.
#pragma once

#include <math.h>

#include <thread>
#include <vector>

#include "../../include/sdfmesh_b200.h"

namespace sdfb {

// fminf / fmaxf as the C library computes them (a NaN operand ignored, of two equal values the second),
// inline: under strict IEEE compilation the library functions are calls, most of the build's time
inline float hmin(float a, float b) { return (b != b) ? a : ((a != a) ? b : (a < b ? a : b)); }
inline float hmax(float a, float b) { return (b != b) ? a : ((a != a) ? b : (a > b ? a : b)); }

struct HostV3 {
    float x, y, z;
};

inline HostV3 hv(float x, float y, float z) { return HostV3{x, y, z}; }

// rotateVector (Commons.cuh:264-273), separate roundings, reference operand order
inline HostV3 host_rotate(HostV3 v, const float* q) {
    const HostV3 u = hv(q[0], q[1], q[2]);
    const float s = q[3];
    const float duv = (u.x * v.x + u.y * v.y) + u.z * v.z;
    const float duu = (u.x * u.x + u.y * u.y) + u.z * u.z;
    const float a = 2.0f * duv, b = s * s - duu, c = 2.0f * s;
    const HostV3 cr = hv(u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x);
    return hv((a * u.x + b * v.x) + c * cr.x, (a * u.y + b * v.y) + c * cr.y, (a * u.z + b * v.z) + c * cr.z);
}

inline void primitive_box(const sdf_primitive& p, HostV3& mn, HostV3& mx) {
    float pad = 0.1f;
    if (p.displacement != DISP_NONE) pad += 0.5f;
    HostV3 dims = hv(1.f, 1.f, 1.f);
    if (p.type == SDF_SPHERE) dims = hv(p.params[0], p.params[0], p.params[0]);
    else if (p.type == SDF_BOX || p.type == SDF_ROUNDED_BOX) dims = hv(p.params[0], p.params[1], p.params[2]);
    else if (p.type == SDF_TORUS) dims = hv(p.params[0] + p.params[1], p.params[1], p.params[0] + p.params[1]);
    dims = hv(dims.x + pad, dims.y + pad, dims.z + pad);
    mn = hv(1e10f, 1e10f, 1e10f);
    mx = hv(-1e10f, -1e10f, -1e10f);
    for (int i = 0; i < 8; ++i) {
        const HostV3 c = hv((i & 1) ? dims.x : -dims.x, (i & 2) ? dims.y : -dims.y, (i & 4) ? dims.z : -dims.z);
        HostV3 w = host_rotate(hv(c.x * p.scale[0], c.y * p.scale[1], c.z * p.scale[2]), p.rotation);
        w = hv(w.x + p.position[0], w.y + p.position[1], w.z + p.position[2]);
        mn = hv(hmin(mn.x, w.x), hmin(mn.y, w.y), hmin(mn.z, w.z));
        mx = hv(hmax(mx.x, w.x), hmax(mx.y, w.y), hmax(mx.z, w.z));
    }
}

struct HostBox {
    HostV3 mn, mx;
};

// The recursion of buildBVHRecursive. The reference recomputes getPrimitiveAABB for every primitive
// at every level (twice); the box is a pure function of the primitive, so it is computed once per
// primitive here and looked up, which gives the same nodes in O(n) box evaluations. Nodes are numbered
// in the reference's pre-order (a node, then its left subtree, then its right one), and a subtree over
// m primitives always has 2m - 1 nodes (leaves hold one primitive, inner nodes two children), so the
// node `cur` of `count` primitives has its left child at cur + 1 and its right child at cur + 2 mid:
// the two subtrees can be built at once, the left one on another thread while `threads` allows.
inline void build_node(int* idx, int count, const std::vector<HostBox>& boxes, sdf_bvh_node* nodes, int cur,
                       int threads) {
    sdf_bvh_node node;
    node.min[0] = node.min[1] = node.min[2] = 1e10f;
    node.max[0] = node.max[1] = node.max[2] = -1e10f;
    HostV3 cc = hv(0.f, 0.f, 0.f);
    for (int i = 0; i < count; ++i) {
        const HostV3 a = boxes[idx[i]].mn, b = boxes[idx[i]].mx;
        node.min[0] = hmin(node.min[0], a.x); node.min[1] = hmin(node.min[1], a.y); node.min[2] = hmin(node.min[2], a.z);
        node.max[0] = hmax(node.max[0], b.x); node.max[1] = hmax(node.max[1], b.y); node.max[2] = hmax(node.max[2], b.z);
        cc = hv(cc.x + (a.x + b.x) * 0.5f, cc.y + (a.y + b.y) * 0.5f, cc.z + (a.z + b.z) * 0.5f);
    }
    const float inv = 1.0f / (float)count;
    cc = hv(cc.x * inv, cc.y * inv, cc.z * inv);
    if (count <= 1) {
        node.left = idx[0];
        node.right = -1;
        nodes[cur] = node;
        return;
    }
    int axis = 0;
    const HostV3 ext = hv(node.max[0] - node.min[0], node.max[1] - node.min[1], node.max[2] - node.min[2]);
    if (ext.y > ext.x) axis = 1;
    if (ext.z > ext.y && ext.z > ext.x) axis = 2;
    const float split = axis == 0 ? cc.x : (axis == 1 ? cc.y : cc.z);
    int mid = 0;
    for (int i = 0; i < count; ++i) {
        const HostV3 a = boxes[idx[i]].mn, b = boxes[idx[i]].mx;
        const float c = axis == 0 ? (a.x + b.x) * 0.5f : (axis == 1 ? (a.y + b.y) * 0.5f : (a.z + b.z) * 0.5f);
        if (c < split) {
            const int t = idx[i];
            idx[i] = idx[mid];
            idx[mid] = t;
            ++mid;
        }
    }
    if (mid == 0 || mid == count) mid = count / 2;
    node.left = cur + 1;
    node.right = cur + 2 * mid;
    nodes[cur] = node;
    // the left subtree on a thread of its own when it is large and threads remain; if a thread cannot
    // be started, both subtrees are built here (the same nodes)
    if (threads > 1 && count >= 4096) {
        const int tl = threads / 2;
        try {
            std::thread t(build_node, idx, mid, std::cref(boxes), nodes, cur + 1, tl);
            build_node(idx + mid, count - mid, boxes, nodes, cur + 2 * mid, threads - tl);
            t.join();
            return;
        } catch (...) {
        }
    }
    build_node(idx, mid, boxes, nodes, cur + 1, 1);
    build_node(idx + mid, count - mid, boxes, nodes, cur + 2 * mid, 1);
}

// the host threads the scene build uses (at most 16)
inline int build_threads() {
    const unsigned h = std::thread::hardware_concurrency();
    return h == 0 ? 1 : (h > 16 ? 16 : (int)h);
}

// Reorders `prims` (unions first, stable) and builds the BVH over the unions.
// Returns the number of BVH primitives.
inline int prepare_scene(const sdf_primitive* in, int n, std::vector<sdf_primitive>& sorted,
                         std::vector<sdf_bvh_node>& nodes) {
    sorted.clear();
    nodes.clear();
    for (int i = 0; i < n; ++i)
        if (in[i].operation == SDF_UNION || in[i].operation == SDF_UNION_BLEND) sorted.push_back(in[i]);
    const int nu = (int)sorted.size();
    for (int i = 0; i < n; ++i)
        if (!(in[i].operation == SDF_UNION || in[i].operation == SDF_UNION_BLEND)) sorted.push_back(in[i]);
    if (nu > 0) {
        std::vector<HostBox> boxes(nu);
        const int threads = nu >= 4096 ? build_threads() : 1;
        auto box_range = [&](int i0, int i1) {
            for (int i = i0; i < i1; ++i) primitive_box(sorted[i], boxes[i].mn, boxes[i].mx);
        };
        std::vector<std::thread> pool;
        if (threads > 1) {
            const int chunk = (nu + threads - 1) / threads;
            try {
                for (int t = 1; t < threads; ++t) {
                    const int i0 = t * chunk, i1 = i0 + chunk < nu ? i0 + chunk : nu;
                    if (i0 >= nu) break;
                    pool.emplace_back(box_range, i0, i1);
                }
            } catch (...) {
            }
            const int done = (int)pool.size();  // ranges 1 .. done went to threads
            box_range(0, chunk < nu ? chunk : nu);
            for (auto& th : pool) th.join();
            // ranges whose thread could not be started
            for (int t = done + 1; t < threads; ++t) {
                const int i0 = t * chunk, i1 = i0 + chunk < nu ? i0 + chunk : nu;
                if (i0 < nu) box_range(i0, i1);
            }
        } else {
            box_range(0, nu);
        }
        std::vector<int> idx(nu);
        for (int i = 0; i < nu; ++i) idx[i] = i;
        nodes.resize(2 * (size_t)nu - 1);
        build_node(idx.data(), nu, boxes, nodes.data(), 0, threads);
    }
    return nu;
}

inline int bvh_depth(const std::vector<sdf_bvh_node>& nodes, int i = 0) {
    if (nodes.empty()) return 0;
    if (nodes[i].right == -1) return 1;
    const int l = bvh_depth(nodes, nodes[i].left), r = bvh_depth(nodes, nodes[i].right);
    return 1 + (l > r ? l : r);
}

}  // namespace sdfb
