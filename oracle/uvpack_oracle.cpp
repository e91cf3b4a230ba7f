// CPU oracle for the UV atlas packer: TEST INFRASTRUCTURE, not part of the product.
// Restates mite51/CudaSDF src/SDFMesh/GridUVPacker.cu; see uvpack_oracle.h for the conventions.
#include "uvpack_oracle.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <map>
#include <vector>

namespace {

struct V2 { float x, y; };

// (int)f as the reference's x86-64 host code converts it (cvttss2si): NaN and out-of-range give INT_MIN.
int host_f2i(float f) { return (f >= -2147483648.0f && f < 2147483648.0f) ? (int)f : INT_MIN; }
// (int)f in the reference's device code (round toward zero, saturating, NaN -> 0).
int dev_f2i(float f) {
    if (f != f) return 0;
    if (f >= 2147483648.0f) return INT_MAX;
    if (f <= -2147483648.0f) return INT_MIN;
    return (int)f;
}

struct Grid {
    uint32_t* c;
    int w, h, s;
};
struct CGrid {
    const uint32_t* c;
    int w, h, s;
};

// getGridCell / setGridCell (GridUVPacker.cu:14-35)
bool get_cell(const CGrid& g, int x, int y) {
    if (x < 0 || y < 0 || x >= g.w || y >= g.h) return false;
    return (g.c[(int64_t)y * g.s + (x >> 5)] >> (x & 31)) & 1u;
}
void set_cell(Grid& g, int x, int y) {
    if (x < 0 || y < 0 || x >= g.w || y >= g.h) return;
    g.c[(int64_t)y * g.s + (x >> 5)] |= 1u << (x & 31);
}

// triangleArea2D (GridUVPacker.cu:41-43). Where its difference of products is fused, the compiled code
// is fma(t1, t2, -(t3 * t4)); where both products are shared with other calls it rounds both.
float area2d(V2 a, V2 b, V2 c, bool fused) {
    float t1 = b.x - a.x, t2 = c.y - a.y, t3 = c.x - a.x, t4 = b.y - a.y;
    return 0.5f * fabsf(fused ? fmaf(t1, t2, -(t3 * t4)) : (t1 * t2) - (t3 * t4));
}

// pointInTriangle (GridUVPacker.cu:56-64) as called alone: every area fused.
bool point_in_triangle(V2 p, V2 a, V2 b, V2 c) {
    float total = area2d(a, b, c, true);
    float a1 = area2d(p, b, c, true), a2 = area2d(a, p, c, true), a3 = area2d(a, b, p, true);
    return fabsf(total - ((a1 + a2) + a3)) < 1e-6f;
}

// pointInTriangle as compiled inside triangleOverlapsCell (GridUVPacker.cu:131-136). There the four
// corner tests share products: each product of area(a, p, c) and area(a, b, p) involves only the
// corner's x or only its y, so corners with the same x or y form it too, and the compiled code rounds
// both products of those two areas on their own; the total and area(p, b, c) stay fused. (Pinned
// against the reference's compiled triangleOverlapsCell on the GPU.)
bool corner_in_triangle(V2 p, V2 a, V2 b, V2 c) {
    float total = area2d(a, b, c, true);
    float a1 = area2d(p, b, c, true), a2 = area2d(a, p, c, false), a3 = area2d(a, b, p, false);
    return fabsf(total - ((a1 + a2) + a3)) < 1e-6f;
}

V2 sub2(V2 a, V2 b) { return V2{a.x - b.x, a.y - b.y}; }
float cross2(V2 a, V2 b) { return fmaf(a.x, b.y, -(a.y * b.x)); }

// onSegment / orientSign / segmentsIntersect (GridUVPacker.cu:74-105)
bool on_segment(V2 a, V2 b, V2 p) {
    float minX = fminf(a.x, b.x) - 1e-6f, maxX = fmaxf(a.x, b.x) + 1e-6f;
    float minY = fminf(a.y, b.y) - 1e-6f, maxY = fmaxf(a.y, b.y) + 1e-6f;
    return p.x >= minX && p.x <= maxX && p.y >= minY && p.y <= maxY;
}
int orient_sign(V2 a, V2 b, V2 c) {
    float v = cross2(sub2(b, a), sub2(c, a));
    if (v > 1e-6f) return 1;
    if (v < -1e-6f) return -1;
    return 0;
}
bool segments_intersect(V2 a, V2 b, V2 c, V2 d) {
    int o1 = orient_sign(a, b, c), o2 = orient_sign(a, b, d), o3 = orient_sign(c, d, a), o4 = orient_sign(c, d, b);
    if (o1 != o2 && o3 != o4) return true;
    if (o1 == 0 && on_segment(a, b, c)) return true;
    if (o2 == 0 && on_segment(a, b, d)) return true;
    if (o3 == 0 && on_segment(c, d, a)) return true;
    if (o4 == 0 && on_segment(c, d, b)) return true;
    return false;
}

bool in_box(V2 v, float x0, float y0, float x1, float y1) { return v.x >= x0 && v.x <= x1 && v.y >= y0 && v.y <= y1; }

// triangleOverlapsCell (GridUVPacker.cu:107-165)
bool triangle_overlaps_cell(V2 v0, V2 v1, V2 v2, int cx, int cy) {
    float x0 = (float)cx, y0 = (float)cy, x1 = (float)(cx + 1), y1 = (float)(cy + 1);
    V2 corners[4] = {{x0, y0}, {x1, y0}, {x1, y1}, {x0, y1}};
    if (in_box(v0, x0, y0, x1, y1) || in_box(v1, x0, y0, x1, y1) || in_box(v2, x0, y0, x1, y1)) return true;
    for (int i = 0; i < 4; i++)
        if (corner_in_triangle(corners[i], v0, v1, v2)) return true;
    V2 ta[3] = {v0, v1, v2}, tb[3] = {v1, v2, v0};
    for (int e = 0; e < 3; e++)
        for (int r = 0; r < 4; r++)
            if (segments_intersect(ta[e], tb[e], corners[r], corners[(r + 1) & 3])) return true;
    V2 ctr{((v0.x + v1.x) + v2.x) / 3.0f, ((v0.y + v1.y) + v2.y) / 3.0f};
    return in_box(ctr, x0, y0, x1, y1);
}

// rasterizeIslandKernel, one triangle (GridUVPacker.cu:171-225)
void rasterize_triangle(const float* uvs, int64_t t, int minx, int miny, int res, Grid& g) {
    V2 p[3];
    for (int v = 0; v < 3; v++) {
        const float* uv = uvs + 2 * (3 * t + v);
        p[v] = V2{fmaf(uv[0], (float)res, -(float)minx), fmaf(uv[1], (float)res, -(float)miny)};
    }
    float minU = fminf(fminf(p[0].x, p[1].x), p[2].x), maxU = fmaxf(fmaxf(p[0].x, p[1].x), p[2].x);
    float minV = fminf(fminf(p[0].y, p[1].y), p[2].y), maxV = fmaxf(fmaxf(p[0].y, p[1].y), p[2].y);
    int xMin = dev_f2i(floorf(minU)), xMax = dev_f2i(ceilf(maxU));
    int yMin = dev_f2i(floorf(minV)), yMax = dev_f2i(ceilf(maxV));
    xMin = std::max(0, std::min(xMin, g.w - 1));
    xMax = std::max(0, std::min(xMax, g.w));
    yMin = std::max(0, std::min(yMin, g.h - 1));
    yMax = std::max(0, std::min(yMax, g.h));
    for (int y = yMin; y < yMax; y++)
        for (int x = xMin; x < xMax; x++)
            if (triangle_overlaps_cell(p[0], p[1], p[2], x, y)) set_cell(g, x, y);
}

// dilateGridKernel (GridUVPacker.cu:227-257)
void dilate(const CGrid& in, Grid& out, int r) {
    for (int y = 0; y < out.h; y++)
        for (int x = 0; x < out.w; x++) {
            bool hit = false;
            for (int dy = -r; dy <= r && !hit; dy++)
                for (int dx = -r; dx <= r; dx++) {
                    if (dx * dx + dy * dy > r * r) continue;
                    if (get_cell(in, x + dx, y + dy)) { hit = true; break; }
                }
            if (hit) set_cell(out, x, y);
        }
}

// rotateGridKernel, rotation 1 = 90 degrees clockwise (GridUVPacker.cu:259-298)
void rotate90(const CGrid& in, Grid& out) {
    for (int y = 0; y < out.h; y++)
        for (int x = 0; x < out.w; x++)
            if (get_cell(in, y, in.h - 1 - x)) set_cell(out, x, y);
}

// computeRowWordBoundsKernel (GridUVPacker.cu:300-339)
void row_bounds(const CGrid& g, uint16_t* mn, uint16_t* mx) {
    for (int y = 0; y < g.h; y++) {
        int lo = g.s, hi = -1;
        for (int w = 0; w < g.s; w++)
            if (g.c[(int64_t)y * g.s + w] != 0) { lo = std::min(lo, w); hi = std::max(hi, w); }
        if (hi < 0) { mn[y] = 0xFFFF; mx[y] = 0; }
        else { mn[y] = (uint16_t)lo; mx[y] = (uint16_t)hi; }
    }
}

int align_down(int v, int a) { return a <= 1 ? v : v - (v % a); }

// checkIslandCollisionBitsAlignedRanged (GridUVPacker.cu:341-386)
bool collides(const uint32_t* board, int G, int bs, const CGrid& isl, const uint16_t* mn, const uint16_t* mx, int ox,
              int oy) {
    if (ox < 0 || oy < 0) return true;
    if (ox + isl.w > G) return true;
    if (oy + isl.h > G) return true;
    int ws = ox >> 5, bsh = ox & 31;
    for (int y = 0; y < isl.h; y++) {
        uint16_t lo = mn[y];
        if (lo == 0xFFFF) continue;
        uint16_t hi = mx[y];
        const uint32_t* ir = isl.c + (int64_t)y * isl.s + lo;
        const uint32_t* br = board + (int64_t)(oy + y) * bs + ws + lo;
        int wc = (int)hi - (int)lo + 1;
        if (bsh == 0) {
            for (int w = 0; w < wc; w++)
                if (br[w] & ir[w]) return true;
        } else {
            uint32_t carry = 0;
            for (int w = 0; w < wc; w++) {
                uint32_t cur = ir[w];
                uint32_t sh = (cur << bsh) | carry;
                carry = cur >> (32 - bsh);
                if (br[w] & sh) return true;
            }
            if (carry != 0 && (ws + lo + wc) < bs && (br[wc] & carry)) return true;
        }
    }
    return false;
}

// writeIslandToMaskBitsAlignedRanged (GridUVPacker.cu:388-425)
void write_island(uint32_t* board, int bs, const CGrid& isl, const uint16_t* mn, const uint16_t* mx, int ox, int oy) {
    int ws = ox >> 5, bsh = ox & 31;
    for (int y = 0; y < isl.h; y++) {
        uint16_t lo = mn[y];
        if (lo == 0xFFFF) continue;
        uint16_t hi = mx[y];
        const uint32_t* ir = isl.c + (int64_t)y * isl.s + lo;
        uint32_t* br = board + (int64_t)(oy + y) * bs + ws + lo;
        int wc = (int)hi - (int)lo + 1;
        if (bsh == 0) {
            for (int w = 0; w < wc; w++) br[w] |= ir[w];
        } else {
            uint32_t carry = 0;
            for (int w = 0; w < wc; w++) {
                uint32_t cur = ir[w];
                br[w] |= (cur << bsh) | carry;
                carry = cur >> (32 - bsh);
            }
            if (carry != 0 && (ws + lo + wc) < bs) br[wc] |= carry;
        }
    }
}

CGrid cgrid(const uint32_t* words, int64_t off, int w, int h, int s) { return CGrid{words + off, w, h, s}; }

}  // namespace

extern "C" {

// ExtractCharts (GridUVPacker.cu:833-896): triangles grouped by the primitive id of their first vertex,
// charts in ascending id order (std::map), UV bounds over the triangles' three vertices. Only complete
// triangles are read (the reference also reads past a partial last one).
int64_t uvo_extract_charts(const float* uvs, const float* prim_ids, int64_t num_vertices, int32_t* tri_chart,
                           int32_t* chart_prim, int32_t* chart_ntris, float* chart_bounds, int64_t max_charts) {
    int64_t T = num_vertices / 3;
    std::map<int, std::vector<int64_t>> by_prim;
    for (int64_t t = 0; t < T; t++) {
        int id = host_f2i(prim_ids[3 * t] + 0.5f);
        tri_chart[t] = -1;
        if (id >= 0) by_prim[id].push_back(t);
    }
    if ((int64_t)by_prim.size() > max_charts) return -1;
    int64_t c = 0;
    for (auto& kv : by_prim) {
        float mnx = 1e10f, mny = 1e10f, mxx = -1e10f, mxy = -1e10f;
        for (int64_t t : kv.second) {
            tri_chart[t] = (int32_t)c;
            for (int v = 0; v < 3; v++) {
                const float* uv = uvs + 2 * (3 * t + v);
                mnx = fminf(mnx, uv[0]);
                mny = fminf(mny, uv[1]);
                mxx = fmaxf(mxx, uv[0]);
                mxy = fmaxf(mxy, uv[1]);
            }
        }
        chart_prim[c] = kv.first;
        chart_ntris[c] = (int32_t)kv.second.size();
        chart_bounds[4 * c + 0] = mnx;
        chart_bounds[4 * c + 1] = mny;
        chart_bounds[4 * c + 2] = mxx;
        chart_bounds[4 * c + 3] = mxy;
        c++;
    }
    return c;
}

// Island bounds of CreateIslands (GridUVPacker.cu:916-925) and the oracle's arena layout.
int uvo_island_plan(int num_charts, const int32_t* chart_prim, const int32_t* chart_ntris,
                    const float* chart_bounds, int grid_resolution, int margin_cells, UvoIsland* out,
                    int64_t* total_words, int64_t* total_rb) {
    int64_t words = 0, rb = 0;
    for (int i = 0; i < num_charts; i++) {
        const float* b = chart_bounds + 4 * i;
        int minX = host_f2i(floorf(b[0] * (float)grid_resolution)) - margin_cells;
        int minY = host_f2i(floorf(b[1] * (float)grid_resolution)) - margin_cells;
        int maxX = host_f2i(ceilf(b[2] * (float)grid_resolution)) + margin_cells;
        int maxY = host_f2i(ceilf(b[3] * (float)grid_resolution)) + margin_cells;
        UvoIsland& d = out[i];
        memset(&d, 0, sizeof(d));
        d.island_index = i;
        d.primitive_id = chart_prim[i];
        d.num_triangles = chart_ntris[i];
        d.min_x = minX;
        d.min_y = minY;
        d.w = std::max(1, maxX - minX);
        d.h = std::max(1, maxY - minY);
        if (d.w > 65536 || d.h > 65536) return -1;
        d.stride = (d.w + 31) / 32;
        d.stride90 = (d.h + 31) / 32;
        d.off_mask = words;
        words += (int64_t)d.stride * d.h;
        d.off_coll = words;
        words += (int64_t)d.stride * d.h;
        d.off_mask90 = words;
        words += (int64_t)d.stride90 * d.w;
        d.off_coll90 = words;
        words += (int64_t)d.stride90 * d.w;
        d.off_rb = rb;
        rb += 2 * (int64_t)d.h;
        d.off_rb90 = rb;
        rb += 2 * (int64_t)d.w;
    }
    *total_words = words;
    *total_rb = rb;
    return 0;
}

// The masks of CreateIslands (GridUVPacker.cu:942-1049): rasterise, dilate by the margin (or copy),
// rotate both by 90 degrees, row word bounds of both collision masks.
int uvo_island_build(const float* uvs, int64_t num_vertices, const int32_t* tri_chart, int num_charts,
                     const UvoIsland* islands, int grid_resolution, int margin_cells, uint32_t* words,
                     uint16_t* rb) {
    int64_t T = num_vertices / 3;
    std::vector<std::vector<int64_t>> tris(num_charts);
    for (int64_t t = 0; t < T; t++)
        if (tri_chart[t] >= 0 && tri_chart[t] < num_charts) tris[tri_chart[t]].push_back(t);
    for (int i = 0; i < num_charts; i++) {
        const UvoIsland& d = islands[i];
        int64_t n0 = (int64_t)d.stride * d.h, n9 = (int64_t)d.stride90 * d.w;
        memset(words + d.off_mask, 0, 4 * n0);
        memset(words + d.off_coll, 0, 4 * n0);
        memset(words + d.off_mask90, 0, 4 * n9);
        memset(words + d.off_coll90, 0, 4 * n9);
        Grid mask{words + d.off_mask, d.w, d.h, d.stride};
        Grid coll{words + d.off_coll, d.w, d.h, d.stride};
        Grid mask90{words + d.off_mask90, d.h, d.w, d.stride90};
        Grid coll90{words + d.off_coll90, d.h, d.w, d.stride90};
        for (int64_t t : tris[i]) rasterize_triangle(uvs, t, d.min_x, d.min_y, grid_resolution, mask);
        if (margin_cells > 0) dilate(CGrid{mask.c, mask.w, mask.h, mask.s}, coll, margin_cells);
        else memcpy(coll.c, mask.c, 4 * n0);
        rotate90(CGrid{mask.c, mask.w, mask.h, mask.s}, mask90);
        rotate90(CGrid{coll.c, coll.w, coll.h, coll.s}, coll90);
        row_bounds(CGrid{coll.c, coll.w, coll.h, coll.s}, rb + d.off_rb, rb + d.off_rb + d.h);
        row_bounds(CGrid{coll90.c, coll90.w, coll90.h, coll90.s}, rb + d.off_rb90, rb + d.off_rb90 + d.w);
    }
    (void)num_vertices;
    return 0;
}

// std::sort of the islands by mask area, largest first (GridUVPacker.cu:1052-1058). std::sort is not
// stable; its permutation depends only on the comparisons, so sorting the records gives the reference's.
void uvo_island_sort(int n, const UvoIsland* islands, int32_t* order) {
    std::vector<UvoIsland> v(islands, islands + n);
    std::sort(v.begin(), v.end(), [](const UvoIsland& a, const UvoIsland& b) { return a.w * a.h > b.w * b.h; });
    for (int i = 0; i < n; i++) order[i] = v[i].island_index;
}

// The attempt seeds of PackIslands (GridUVPacker.cu:1117-1122): srand(seed or time), rand() per attempt.
void uvo_seeds(int random_seed, int n, int32_t* out) {
    srand(random_seed == 0 ? (unsigned int)time(nullptr) : (unsigned int)random_seed);
    for (int i = 0; i < n; i++) out[i] = rand();
}

// The shelf width of PackIslands (GridUVPacker.cu:1126-1138).
int uvo_shelf_width(int n, const UvoIsland* sorted, int grid_size) {
    int maxW = 0, total = 0;
    for (int i = 0; i < n; i++) {
        maxW = std::max(maxW, sorted[i].w);
        total += sorted[i].w * sorted[i].h;
    }
    int target = host_f2i(sqrtf((float)total * 1.3f));
    int minShelf = maxW * 2 + maxW / 2;
    return std::max(minShelf, std::min(target, grid_size));
}

// 1 when every candidate loop of packSolutionKernel (GridUVPacker.cu:660-665) can fill its budget:
// for each island and rotation that passes the size checks, the aligned columns of [0, maxX] must be
// at least the candidate budget, otherwise the reference's loop draws forever.
int uvo_candidate_loops_end(int n, const UvoIsland* sorted, const int32_t* cfg, int shelf_width) {
    int G = cfg[UVO_GRID_SIZE], A = std::max(1, cfg[UVO_X_ALIGN]);
    int shelfMax = std::min(G, align_down(std::max(1, shelf_width), A));
    int budget = std::max(4, std::min(64, cfg[UVO_MAX_CAND]));
    int nrot = cfg[UVO_ROTATION] ? 2 : 1;
    for (int i = 0; i < std::min(n, 256); i++)
        for (int rot = 0; rot < nrot; rot++) {
            int iw = rot ? sorted[i].h : sorted[i].w, ih = rot ? sorted[i].w : sorted[i].h;
            if (iw > G || ih > G) continue;
            int maxX = std::min(shelfMax, G) - iw;
            if (maxX < 0) continue;
            if (maxX / A + 1 < budget) return 0;
        }
    return 1;
}

// The helpers on n records of (a, b, c, p) with a cell each: triangleArea2D(a, b, c),
// pointInTriangle(p, a, b, c), orientSign(a, b, c), segmentsIntersect(a, b, c, p),
// triangleOverlapsCell(a, b, c, cell) (GridUVPacker.cu:41-165), as the reference's probes return them.
void uvo_probe(const float* rec, const int32_t* cells, int64_t n, float* area, int32_t* pit, int32_t* orient,
               int32_t* seg, int32_t* overlap) {
    for (int64_t i = 0; i < n; i++) {
        const float* r = rec + 8 * i;
        V2 a{r[0], r[1]}, b{r[2], r[3]}, c{r[4], r[5]}, p{r[6], r[7]};
        area[i] = area2d(a, b, c, true);
        pit[i] = point_in_triangle(p, a, b, c) ? 1 : 0;
        orient[i] = orient_sign(a, b, c);
        seg[i] = segments_intersect(a, b, c, p) ? 1 : 0;
        overlap[i] = triangle_overlaps_cell(a, b, c, cells[2 * i], cells[2 * i + 1]) ? 1 : 0;
    }
}

// packSolutionKernel (GridUVPacker.cu:585-777), one attempt per solution, fed with that attempt's
// recorded draws. Where the reference's candidate loop could not end (fewer aligned columns than the
// budget) the loop stops once every column is listed and the attempt is flagged UVO_CANDIDATE_LOOP_OPEN.
// sol_info per attempt: placed, utilized width, utilized height, status bits, draws used.
int uvo_pack(int num_islands, const UvoIsland* sorted, const uint32_t* words, const uint16_t* rb,
             const int32_t* cfg, int shelf_width, int num_solutions, const uint32_t* draws,
             int64_t draws_per_solution, int32_t* sol_info, float* sol_fitness, int32_t* placements,
             int nthreads) {
    const int G = cfg[UVO_GRID_SIZE];
    const int bs = (G + 31) / 32;
    const int A = std::max(1, cfg[UVO_X_ALIGN]);
    const int shelfMax = std::min(G, align_down(std::max(1, shelf_width), A));
    const int budget = std::max(4, std::min(64, cfg[UVO_MAX_CAND]));
    const int dropCap = cfg[UVO_MAX_DROP];
    const int n = std::min(num_islands, 256);
    const bool rot_on = cfg[UVO_ROTATION] != 0;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads > 0 ? nthreads : 1)
    for (int s = 0; s < num_solutions; s++) {
        std::vector<uint32_t> board((size_t)bs * G, 0u);
        const uint32_t* dr = draws + (int64_t)s * draws_per_solution;
        int64_t k = 0;
        int status = 0;
        auto draw = [&]() -> uint32_t {
            if (k >= draws_per_solution) { status |= UVO_DRAWS_EXHAUSTED; return 0u; }
            return dr[k++];
        };
        int uW = 0, uH = 0, placed = 0;
        std::vector<int> order(n);
        for (int i = 0; i < n; i++) order[i] = i;
        if (cfg[UVO_SHUFFLE] && n > 1)
            for (int i = n - 1; i > 0; i--) {
                int j = (int)(draw() % (unsigned)(i + 1));
                std::swap(order[i], order[j]);
            }
        int32_t* pl = placements + (int64_t)s * n * 4;
        for (int oi = 0; oi < n; oi++) {
            const UvoIsland& isl = sorted[order[oi]];
            int nrot = rot_on ? 2 : 1;
            int rotOrder = rot_on ? (int)(draw() & 1u) : 0;
            float bestScore = 1e30f;
            int bestX = -1, bestY = -1, bestRot = 0, bestW = 0, bestH = 0;
            for (int rr = 0; rr < nrot; rr++) {
                int rotation = rr ^ rotOrder;
                CGrid g = rotation ? cgrid(words, isl.off_coll90, isl.h, isl.w, isl.stride90)
                                   : cgrid(words, isl.off_coll, isl.w, isl.h, isl.stride);
                const uint16_t* mn = rb + (rotation ? isl.off_rb90 : isl.off_rb);
                const uint16_t* mx = mn + g.h;
                if (g.w > G || g.h > G) continue;
                int maxX = std::min(shelfMax, G) - g.w;
                if (maxX < 0) continue;
                int cand[64], cc = 0;
                auto push = [&](int x) {
                    if (cc >= budget) return;
                    x = std::max(0, std::min(maxX, x));
                    x = align_down(x, A);
                    for (int q = 0; q < cc; q++)
                        if (cand[q] == x) return;
                    cand[cc++] = x;
                };
                push(0);
                push(align_down(uW - g.w, A));
                push(align_down(maxX, A));
                const int columns = maxX / A + 1;
                while (cc < budget) {
                    if (cc >= columns) { status |= UVO_CANDIDATE_LOOP_OPEN; break; }
                    unsigned r = draw();
                    push((int)(r % (unsigned)(maxX + 1)));
                    if (status & UVO_DRAWS_EXHAUSTED) break;
                }
                for (int ci = 0; ci < cc; ci++) {
                    int x = cand[ci];
                    int y = std::min(uH, G - g.h);
                    if (y < 0) continue;
                    while (y <= G - g.h && collides(board.data(), G, bs, g, mn, mx, x, y)) y++;
                    if (y > G - g.h) continue;
                    int steps = 0;
                    while (y > 0) {
                        if (dropCap > 0 && steps >= dropCap) break;
                        if (collides(board.data(), G, bs, g, mn, mx, x, y - 1)) break;
                        y--;
                        steps++;
                    }
                    int newW = std::max(uW, x + g.w), newH = std::max(uH, y + g.h);
                    int maxDim = std::max(newW, newH);
                    float score = fmaf(0.01f, (float)(maxDim * maxDim), (float)(newW * newH));
                    if (score < bestScore) {
                        bestScore = score;
                        bestX = x; bestY = y; bestRot = rotation; bestW = g.w; bestH = g.h;
                    }
                }
            }
            if (bestX < 0) break;
            CGrid g = bestRot ? cgrid(words, isl.off_coll90, isl.h, isl.w, isl.stride90)
                              : cgrid(words, isl.off_coll, isl.w, isl.h, isl.stride);
            const uint16_t* mn = rb + (bestRot ? isl.off_rb90 : isl.off_rb);
            write_island(board.data(), bs, g, mn, mn + g.h, bestX, bestY);
            pl[4 * placed + 0] = isl.island_index;
            pl[4 * placed + 1] = bestX;
            pl[4 * placed + 2] = bestY;
            pl[4 * placed + 3] = bestRot;
            placed++;
            uW = std::max(uW, bestX + bestW);
            uH = std::max(uH, bestY + bestH);
        }
        float fit = 0.0f;
        if (placed > 0 && uW > 0 && uH > 0) {
            float ratio = (float)placed / (float)num_islands;
            int maxDim = std::max(uW, uH);
            float sq = (float)(uW * uH) / (float)(maxDim * maxDim);
            fit = ratio * sq;
        }
        sol_info[5 * s + 0] = placed;
        sol_info[5 * s + 1] = uW;
        sol_info[5 * s + 2] = uH;
        sol_info[5 * s + 3] = status;
        sol_info[5 * s + 4] = (int32_t)k;
        sol_fitness[s] = fit;
    }
    return 0;
}

// The choice of PackIslands (GridUVPacker.cu:1188-1214, 1403-1420): most islands placed, then the
// higher fitness, first attempt on ties; the atlas is squared. atlas_i: success, width, height,
// placed, best attempt (-1 when nothing was placed); atlas_f: fitness, scaling factor.
int uvo_select(int num_solutions, const int32_t* sol_info, const float* sol_fitness, int num_islands,
               int grid_size, int32_t* atlas_i, float* atlas_f) {
    int best = -1, most = 0;
    float bestFit = 0.0f;
    for (int i = 0; i < num_solutions; i++) {
        int p = sol_info[5 * i];
        if (p > most) { most = p; best = i; bestFit = sol_fitness[i]; }
        else if (p == most && sol_fitness[i] > bestFit) { best = i; bestFit = sol_fitness[i]; }
    }
    atlas_i[0] = 0; atlas_i[1] = 0; atlas_i[2] = 0; atlas_i[3] = 0; atlas_i[4] = -1;
    atlas_f[0] = 0.0f; atlas_f[1] = 1.0f;
    if (best < 0 || most == 0) return 0;
    int w = sol_info[5 * best + 1], h = sol_info[5 * best + 2];
    int m = std::max(w, h);
    atlas_i[0] = (sol_info[5 * best] == num_islands) ? 1 : 0;
    atlas_i[1] = m;
    atlas_i[2] = m;
    atlas_i[3] = sol_info[5 * best];
    atlas_i[4] = best;
    atlas_f[0] = sol_fitness[best];
    atlas_f[1] = m > 0 ? (float)grid_size / (float)m : 1.0f;
    return 1;
}

// RemapUVsToAtlas + remapUVsKernel (GridUVPacker.cu:779-831, 1441-1547). The caller skips it when
// the atlas is not a success, as the reference does.
void uvo_remap(float* uvs, const float* prim_ids, int64_t num_vertices, int num_charts,
               const int32_t* chart_prim, const UvoIsland* islands_chart_order, const int32_t* placements,
               int num_placements, int atlas_width, int atlas_height, int grid_resolution) {
    std::vector<int> byChart(4 * (size_t)num_charts, 0);
    for (int c = 0; c < num_charts; c++) byChart[4 * c] = -1;
    for (int i = 0; i < num_placements; i++) {
        int idx = placements[4 * i];
        if (idx >= 0 && idx < num_charts)
            for (int q = 0; q < 4; q++) byChart[4 * idx + q] = placements[4 * i + q];
    }
    int maxPrim = -1;
    for (int c = 0; c < num_charts; c++) maxPrim = std::max(maxPrim, chart_prim[c]);
    std::vector<int> primToChart(std::max(maxPrim + 1, 1), -1);
    for (int c = 0; c < num_charts; c++)
        if (chart_prim[c] >= 0 && chart_prim[c] < (int)primToChart.size()) primToChart[chart_prim[c]] = c;
    const int size = (int)primToChart.size();
    const float denom = (float)std::max(atlas_width, atlas_height);
    for (int64_t v = 0; v < num_vertices; v++) {
        int id = dev_f2i(prim_ids[v] + 0.5f);
        if (id < 0) continue;
        int c = id < size ? primToChart[id] : -1;
        if (c < 0) continue;
        const int* p = &byChart[4 * c];
        if (p[0] < 0) continue;
        const UvoIsland& isl = islands_chart_order[c];
        float* uv = uvs + 2 * v;
        float cx = fmaf(uv[0], (float)grid_resolution, -(float)isl.min_x);
        float cy = fmaf(uv[1], (float)grid_resolution, -(float)isl.min_y);
        if (p[3] == 1) {
            float t = cx;
            cx = cy;
            cy = (float)(isl.w - 1) - t;
        }
        float ax = (float)p[1] + cx, ay = (float)p[2] + cy;
        if (denom <= 0.0f) continue;
        uv[0] = ax / denom;
        uv[1] = ay / denom;
    }
}

}  // extern "C"
