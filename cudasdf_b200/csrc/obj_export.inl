// Wavefront OBJ export of an extracted mesh, in the format of the reference's ExportMeshToOBJ
// (main.cpp:1043-1119): two comment lines and a blank line, one "v x y z" line per vertex, a blank
// line, optionally one "vt u v" line per vertex and a blank line, then one face line per triangle with
// 1-based indices ("f a b c", or "f a/a b/b c/c" with UVs). Numbers are written as the reference's
// std::ofstream writes a float by default: six significant digits, %g. The reference writes the soup
// (face k is vertices 3k..3k+2); with an index buffer the faces use it (the indexed output). As in the
// reference (main.cpp:1066-1070), a mesh without vertices leaves a file holding the header only and is
// reported as an error.
//
// The text is formatted in parallel (one chunk of lines per host thread) and written in order.

#include <thread>

namespace sdfb {

// formats lines [lo, hi) of one kind into `out`
template <class F>
static void obj_lines(std::string& out, uint64_t lo, uint64_t hi, F line) {
    char buf[160];
    out.clear();
    out.reserve((size_t)(hi - lo) * 36);
    for (uint64_t i = lo; i < hi; ++i) {
        const int n = line(i, buf);
        out.append(buf, (size_t)n);
    }
}

// all lines [0, count) of one kind, formatted by `threads` host threads and appended to the file
template <class F>
static bool obj_block(FILE* f, uint64_t count, int threads, F line) {
    if (count == 0) return true;
    const int nt = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)threads, count / 4096 + 1));
    std::vector<std::string> parts((size_t)nt);
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t) {
        const uint64_t lo = count * (uint64_t)t / (uint64_t)nt, hi = count * (uint64_t)(t + 1) / (uint64_t)nt;
        pool.emplace_back([&parts, t, lo, hi, &line] { obj_lines(parts[(size_t)t], lo, hi, line); });
    }
    for (auto& th : pool) th.join();
    for (const auto& s : parts)
        if (!s.empty() && fwrite(s.data(), 1, s.size(), f) != s.size()) return false;
    return true;
}

}  // namespace sdfb

extern "C" sdf_status sdf_write_obj(const char* path, const sdf_float4* vertices, uint64_t num_vertices,
                                    const uint32_t* indices, uint64_t num_indices, const sdf_float2* uvs) {
    using namespace sdfb;
    if (!path || (num_vertices && !vertices)) return SDF_ERR_INVALID;
    const uint64_t nfaces = (indices ? num_indices : num_vertices) / 3;
    if (indices)
        for (uint64_t i = 0; i < nfaces * 3; ++i)
            if (indices[i] >= num_vertices) return SDF_ERR_INVALID;  // a face names a missing vertex
    FILE* f = fopen(path, "wb");
    if (!f) return SDF_ERR_INVALID;
    const char* base = strrchr(path, '/');
    base = base ? base + 1 : path;
    bool ok = fprintf(f, "# Exported from CudaSDF\n# Generated: %s\n\n", base) > 0;
    if (num_vertices == 0) {
        fclose(f);
        return SDF_ERR_INVALID;
    }
    const int threads = (int)std::max(1u, std::thread::hardware_concurrency());
    ok = ok && obj_block(f, num_vertices, threads, [&](uint64_t i, char* b) {
        return snprintf(b, 160, "v %g %g %g\n", (double)vertices[i].x, (double)vertices[i].y, (double)vertices[i].z);
    });
    ok = ok && fputs("\n", f) >= 0;
    if (uvs) {
        ok = ok && obj_block(f, num_vertices, threads, [&](uint64_t i, char* b) {
            return snprintf(b, 160, "vt %g %g\n", (double)uvs[i].x, (double)uvs[i].y);
        });
        ok = ok && fputs("\n", f) >= 0;
    }
    ok = ok && obj_block(f, nfaces, threads, [&](uint64_t k, char* b) {
        const unsigned long long a = (indices ? indices[3 * k] : 3 * k) + 1ull;
        const unsigned long long c = (indices ? indices[3 * k + 1] : 3 * k + 1) + 1ull;
        const unsigned long long d = (indices ? indices[3 * k + 2] : 3 * k + 2) + 1ull;
        return uvs ? snprintf(b, 160, "f %llu/%llu %llu/%llu %llu/%llu\n", a, a, c, c, d, d)
                   : snprintf(b, 160, "f %llu %llu %llu\n", a, c, d);
    });
    if (fclose(f) != 0) ok = false;
    return ok ? SDF_OK : SDF_ERR_INVALID;
}
