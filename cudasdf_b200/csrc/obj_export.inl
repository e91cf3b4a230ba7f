// Wavefront OBJ export of an extracted mesh, in the format of the reference's ExportMeshToOBJ
// (main.cpp:1043-1119): two comment lines and a blank line, one "v x y z" line per vertex, a blank
// line, optionally one "vt u v" line per vertex and a blank line, then one face line per triangle with
// 1-based indices ("f a b c", or "f a/a b/b c/c" with UVs). Numbers are written as the reference's
// std::ofstream writes a float by default: six significant digits, %g. The reference writes the soup
// (face k is vertices 3k..3k+2); with an index buffer the faces use it (the indexed output). As in the
// reference (main.cpp:1066-1070), a mesh without vertices leaves a file holding the header only and is
// reported as an error.
//
// The text is formatted in parallel (one chunk of lines per host thread) and written in order. Numbers
// go through std::to_chars, which formats as printf does in the "C" locale whatever the process's
// LC_NUMERIC is (the reference's std::ofstream also uses the classic locale), so a host application
// that sets a comma-decimal locale still gets "v 0.5 1.25 ..." lines.

#include <charconv>
#include <new>
#include <system_error>
#include <thread>

namespace sdfb {

// "%g" of a float (six significant digits), locale-independent
static inline char* obj_float(char* p, char* end, float v) {
    return std::to_chars(p, end, (double)v, std::chars_format::general, 6).ptr;
}
static inline char* obj_uint(char* p, char* end, unsigned long long v) { return std::to_chars(p, end, v).ptr; }
static inline char* obj_str(char* p, const char* s) {
    while (*s) *p++ = *s++;
    return p;
}

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

// all lines [0, count) of one kind, formatted by `threads` host threads and appended to the file.
// No exception leaves a worker thread (an escaping one would end the process): a chunk whose
// formatting failed marks the block as failed, and a chunk that got no thread is formatted here.
template <class F>
static bool obj_block(FILE* f, uint64_t count, int threads, F line) {
    if (count == 0) return true;
    const int nt = (int)std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)threads, count / 4096 + 1));
    std::vector<std::string> parts((size_t)nt);
    std::vector<char> started((size_t)nt, 0), failed((size_t)nt, 0);
    std::vector<std::thread> pool;
    pool.reserve((size_t)nt);  // no reallocation (hence no exception) once threads run
    auto chunk = [&](int t) {
        const uint64_t lo = count * (uint64_t)t / (uint64_t)nt, hi = count * (uint64_t)(t + 1) / (uint64_t)nt;
        try {
            obj_lines(parts[(size_t)t], lo, hi, line);
        } catch (...) {
            failed[(size_t)t] = 1;
        }
    };
    for (int t = 0; t < nt; ++t) {
        try {
            pool.emplace_back(chunk, t);
            started[(size_t)t] = 1;
        } catch (...) {
            // no thread for this chunk (std::system_error, or no memory for its state): the calling
            // thread formats it below
        }
    }
    for (auto& th : pool) th.join();
    for (int t = 0; t < nt; ++t)
        if (!started[(size_t)t]) chunk(t);
    for (int t = 0; t < nt; ++t)
        if (failed[(size_t)t]) throw std::bad_alloc();
    for (const auto& s : parts)
        if (!s.empty() && fwrite(s.data(), 1, s.size(), f) != s.size()) return false;
    return true;
}

// closes the file on every path out of the writer, exceptions included
struct ObjFile {
    FILE* f;
    explicit ObjFile(FILE* file) : f(file) {}
    ~ObjFile() {
        if (f) fclose(f);
    }
    bool close() {
        const bool ok = fclose(f) == 0;
        f = nullptr;
        return ok;
    }
};

static sdf_status write_obj_impl(const char* path, const sdf_float4* vertices, uint64_t num_vertices,
                                 const uint32_t* indices, uint64_t num_indices, const sdf_float2* uvs) {
    if (!path || (num_vertices && !vertices)) return SDF_ERR_INVALID;
    const uint64_t nfaces = (indices ? num_indices : num_vertices) / 3;
    if (indices)
        for (uint64_t i = 0; i < nfaces * 3; ++i)
            if (indices[i] >= num_vertices) return SDF_ERR_INVALID;  // a face names a missing vertex
    ObjFile file(fopen(path, "wb"));
    FILE* f = file.f;
    if (!f) return SDF_ERR_INVALID;
    const char* base = strrchr(path, '/');
    base = base ? base + 1 : path;
    bool ok = fprintf(f, "# Exported from CudaSDF\n# Generated: %s\n\n", base) > 0;
    if (num_vertices == 0) {
        file.close();
        return SDF_ERR_INVALID;
    }
    const int threads = (int)std::max(1u, std::thread::hardware_concurrency());
    // a line is at most 3 x 13 characters of "%g" or 3 x 2 x 20 digits of indices plus separators,
    // well inside the 160-byte line buffer
    ok = ok && obj_block(f, num_vertices, threads, [&](uint64_t i, char* b) {
        char* e = b + 160;
        char* p = obj_str(b, "v ");
        p = obj_float(p, e, vertices[i].x);
        *p++ = ' ';
        p = obj_float(p, e, vertices[i].y);
        *p++ = ' ';
        p = obj_float(p, e, vertices[i].z);
        *p++ = '\n';
        return (int)(p - b);
    });
    ok = ok && fputs("\n", f) >= 0;
    if (uvs) {
        ok = ok && obj_block(f, num_vertices, threads, [&](uint64_t i, char* b) {
            char* e = b + 160;
            char* p = obj_str(b, "vt ");
            p = obj_float(p, e, uvs[i].x);
            *p++ = ' ';
            p = obj_float(p, e, uvs[i].y);
            *p++ = '\n';
            return (int)(p - b);
        });
        ok = ok && fputs("\n", f) >= 0;
    }
    ok = ok && obj_block(f, nfaces, threads, [&](uint64_t k, char* b) {
        const unsigned long long v[3] = {(indices ? indices[3 * k] : 3 * k) + 1ull,
                                         (indices ? indices[3 * k + 1] : 3 * k + 1) + 1ull,
                                         (indices ? indices[3 * k + 2] : 3 * k + 2) + 1ull};
        char* e = b + 160;
        char* p = obj_str(b, "f");
        for (int j = 0; j < 3; ++j) {
            *p++ = ' ';
            p = obj_uint(p, e, v[j]);
            if (uvs) {
                *p++ = '/';
                p = obj_uint(p, e, v[j]);
            }
        }
        *p++ = '\n';
        return (int)(p - b);
    });
    if (!file.close()) ok = false;
    return ok ? SDF_OK : SDF_ERR_INVALID;
}

}  // namespace sdfb

// Exceptions (a failed allocation while formatting) never cross the C boundary: they become
// SDF_ERR_NOMEM, or SDF_ERR_INVALID for anything else.
extern "C" sdf_status sdf_write_obj(const char* path, const sdf_float4* vertices, uint64_t num_vertices,
                                    const uint32_t* indices, uint64_t num_indices, const sdf_float2* uvs) {
    try {
        return sdfb::write_obj_impl(path, vertices, num_vertices, indices, num_indices, uvs);
    } catch (const std::bad_alloc&) {
        return SDF_ERR_NOMEM;
    } catch (...) {
        return SDF_ERR_INVALID;
    }
}
