// Mesh and scene files.
//
// PLY: smallgwn's tests and benchmarks read triangle meshes from PLY files through libigl
// (tests/test_mesh_io.cpp:43-92: positions as doubles narrowed to float, non-finite positions and
// out-of-range indices refused, empty meshes refused). This reader parses the format itself --
// ASCII and binary of either byte order, any numeric property types, the x/y/z vertex properties
// and the face index list (other elements and properties are skipped); polygons are split into a
// triangle fan (v0, vk, vk+1). The writer emits float positions and uint32 indices.
//
// Scene files: geometry, BVH4 (nodes, primitive order, leaf-ordered records, root, stack bounds) and
// optionally the smallgwn-layout moment nodes of each order, so a later process skips the build.
// Layout (little-endian): 8-byte magic, u32 version, u32 moment-order mask, u64 vertex, triangle,
// node and primitive counts, the 32-byte root child, u32 internal and packed stack bounds, then the
// arrays x, y, z, i0, i1, i2, nodes, primitive order, records, the moment nodes of each order in the
// mask, and a 64-bit checksum of everything before it. Loading uploads geometry and BVH under a new
// revision and refits the moments of each saved order (deterministic, so bit-equal to the saved
// nodes, which is checked); the refit also rebuilds the library's derived state for queries.
#include "gwnb_internal.cuh"

#include <algorithm>
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <sstream>
#include <string>
#include <vector>

namespace gwnb {
namespace {

// ---- PLY ----------------------------------------------------------------------------------------

enum class ply_type { none, i8, u8, i16, u16, i32, u32, f32, f64 };

ply_type parse_type(std::string const &t) {
    if (t == "char" || t == "int8")
        return ply_type::i8;
    if (t == "uchar" || t == "uint8")
        return ply_type::u8;
    if (t == "short" || t == "int16")
        return ply_type::i16;
    if (t == "ushort" || t == "uint16")
        return ply_type::u16;
    if (t == "int" || t == "int32")
        return ply_type::i32;
    if (t == "uint" || t == "uint32")
        return ply_type::u32;
    if (t == "float" || t == "float32")
        return ply_type::f32;
    if (t == "double" || t == "float64")
        return ply_type::f64;
    return ply_type::none;
}

std::size_t type_size(ply_type t) {
    switch (t) {
    case ply_type::i8:
    case ply_type::u8:
        return 1;
    case ply_type::i16:
    case ply_type::u16:
        return 2;
    case ply_type::i32:
    case ply_type::u32:
    case ply_type::f32:
        return 4;
    case ply_type::f64:
        return 8;
    default:
        return 0;
    }
}

struct ply_property {
    std::string name;
    ply_type type = ply_type::none;
    bool list = false;
    ply_type count_type = ply_type::none;
};

struct ply_element {
    std::string name;
    std::uint64_t count = 0;
    std::vector<ply_property> props;
};

enum class ply_format { ascii, binary_le, binary_be };

// Values of one body, read in file order.
class ply_body {
public:
    ply_body(std::vector<char> const &data, std::size_t pos, ply_format fmt) : d_(data), pos_(pos), fmt_(fmt) {}

    bool read(ply_type t, double &out) {
        if (fmt_ == ply_format::ascii)
            return read_ascii(out);
        std::size_t const n = type_size(t);
        if (n == 0 || pos_ + n > d_.size())
            return false;
        unsigned char b[8];
        std::memcpy(b, d_.data() + pos_, n);
        pos_ += n;
        if (fmt_ == ply_format::binary_be)
            for (std::size_t i = 0; i < n / 2; ++i)
                std::swap(b[i], b[n - 1 - i]);
        switch (t) {
        case ply_type::i8: out = static_cast<std::int8_t>(b[0]); break;
        case ply_type::u8: out = b[0]; break;
        case ply_type::i16: { std::int16_t v; std::memcpy(&v, b, 2); out = v; break; }
        case ply_type::u16: { std::uint16_t v; std::memcpy(&v, b, 2); out = v; break; }
        case ply_type::i32: { std::int32_t v; std::memcpy(&v, b, 4); out = v; break; }
        case ply_type::u32: { std::uint32_t v; std::memcpy(&v, b, 4); out = v; break; }
        case ply_type::f32: { float v; std::memcpy(&v, b, 4); out = v; break; }
        case ply_type::f64: { double v; std::memcpy(&v, b, 8); out = v; break; }
        default: return false;
        }
        return true;
    }

    // Bytes left in the body, and the fewest bytes one value of type t can take (a digit and a
    // separator in ASCII): counts in the header are checked against them before any allocation.
    std::size_t remaining() const { return pos_ < d_.size() ? d_.size() - pos_ : 0; }
    std::size_t min_bytes(ply_type t) const { return fmt_ == ply_format::ascii ? 2 : type_size(t); }

private:
    bool read_ascii(double &out) {
        while (pos_ < d_.size() && std::isspace(static_cast<unsigned char>(d_[pos_])))
            ++pos_;
        if (pos_ >= d_.size())
            return false;
        std::size_t end = pos_;
        while (end < d_.size() && !std::isspace(static_cast<unsigned char>(d_[end])))
            ++end;
        std::string const tok(d_.data() + pos_, end - pos_);
        pos_ = end;
        char *stop = nullptr;
        out = std::strtod(tok.c_str(), &stop);
        return stop != tok.c_str() && *stop == '\0';
    }

    std::vector<char> const &d_;
    std::size_t pos_;
    ply_format fmt_;
};

int ply_fail(std::string const &path, std::string const &why) {
    return set_error(GWNB_INVALID_ARGUMENT, "ply: " + path + ": " + why);
}

int read_ply(std::string const &path, std::vector<float> &x, std::vector<float> &y, std::vector<float> &z,
             std::vector<std::uint32_t> &i0, std::vector<std::uint32_t> &i1, std::vector<std::uint32_t> &i2) {
    std::ifstream in(path, std::ios::binary);
    if (!in)
        return ply_fail(path, "cannot open the file");
    std::vector<char> data((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    // header, line by line
    std::size_t pos = 0;
    auto next_line = [&](std::string &line) -> bool {
        if (pos >= data.size())
            return false;
        std::size_t end = pos;
        while (end < data.size() && data[end] != '\n')
            ++end;
        line.assign(data.data() + pos, end - pos);
        if (!line.empty() && line.back() == '\r')
            line.pop_back();
        pos = end < data.size() ? end + 1 : end;
        return true;
    };
    std::string line;
    if (!next_line(line) || line != "ply")
        return ply_fail(path, "missing the 'ply' magic line");
    ply_format fmt = ply_format::ascii;
    bool have_format = false, ended = false;
    std::vector<ply_element> elements;
    while (next_line(line)) {
        std::istringstream ls(line);
        std::string key;
        ls >> key;
        if (key.empty() || key == "comment" || key == "obj_info")
            continue;
        if (key == "format") {
            std::string f;
            ls >> f;
            if (f == "ascii")
                fmt = ply_format::ascii;
            else if (f == "binary_little_endian")
                fmt = ply_format::binary_le;
            else if (f == "binary_big_endian")
                fmt = ply_format::binary_be;
            else
                return ply_fail(path, "unknown format '" + f + "'");
            have_format = true;
        } else if (key == "element") {
            ply_element e;
            if (!(ls >> e.name >> e.count))
                return ply_fail(path, "malformed element line");
            elements.push_back(e);
        } else if (key == "property") {
            if (elements.empty())
                return ply_fail(path, "property before any element");
            ply_property p;
            std::string t;
            ls >> t;
            if (t == "list") {
                std::string ct, it;
                ls >> ct >> it >> p.name;
                p.list = true;
                p.count_type = parse_type(ct);
                p.type = parse_type(it);
                if (p.count_type == ply_type::none || p.type == ply_type::none)
                    return ply_fail(path, "unknown list property types");
            } else {
                p.type = parse_type(t);
                ls >> p.name;
                if (p.type == ply_type::none)
                    return ply_fail(path, "unknown property type '" + t + "'");
            }
            elements.back().props.push_back(p);
        } else if (key == "end_header") {
            ended = true;
            break;
        } else {
            return ply_fail(path, "unknown header line '" + line + "'");
        }
    }
    if (!have_format || !ended)
        return ply_fail(path, "incomplete header");
    ply_body body(data, pos, fmt);
    x.clear(), y.clear(), z.clear(), i0.clear(), i1.clear(), i2.clear();
    std::uint64_t vertex_count = 0;
    bool have_vertices = false;
    for (ply_element const &e : elements) {
        bool const is_vertex = e.name == "vertex";
        bool const is_face = e.name == "face";
        int ix = -1, iy = -1, iz = -1, iface = -1;
        for (std::size_t k = 0; k < e.props.size(); ++k) {
            ply_property const &p = e.props[k];
            if (is_vertex && !p.list) {
                if (p.name == "x")
                    ix = static_cast<int>(k);
                else if (p.name == "y")
                    iy = static_cast<int>(k);
                else if (p.name == "z")
                    iz = static_cast<int>(k);
            }
            if (is_face && p.list && (p.name == "vertex_indices" || p.name == "vertex_index"))
                iface = static_cast<int>(k);
        }
        if (is_face && iface < 0)
            for (std::size_t k = 0; k < e.props.size(); ++k)
                if (e.props[k].list) {
                    iface = static_cast<int>(k);
                    break;
                }
        if (is_vertex) {
            if (ix < 0 || iy < 0 || iz < 0)
                return ply_fail(path, "vertex element without x, y and z");
            if (e.count > 0xffffffffull)
                return ply_fail(path, "more vertices than 32-bit indices address");
        }
        if (is_face && !have_vertices)
            return ply_fail(path, "face element before the vertex element");
        std::size_t record_bytes = 0;
        for (ply_property const &p : e.props)
            record_bytes += body.min_bytes(p.list ? p.count_type : p.type);
        if (record_bytes > 0 && e.count > body.remaining() / record_bytes)
            return ply_fail(path, "truncated element '" + e.name + "'");
        if (is_vertex)
            x.reserve(e.count), y.reserve(e.count), z.reserve(e.count);
        std::vector<double> poly;
        for (std::uint64_t r = 0; r < e.count; ++r) {
            double xyz[3] = {0.0, 0.0, 0.0};
            for (std::size_t k = 0; k < e.props.size(); ++k) {
                ply_property const &p = e.props[k];
                if (p.list) {
                    double cnt = 0.0;
                    if (!body.read(p.count_type, cnt) || cnt < 0.0)
                        return ply_fail(path, "truncated list in element '" + e.name + "'");
                    auto const n = static_cast<std::uint64_t>(cnt);
                    if (n > body.remaining() / std::max<std::size_t>(1, body.min_bytes(p.type)))
                        return ply_fail(path, "truncated list in element '" + e.name + "'");
                    bool const keep = is_face && static_cast<int>(k) == iface;
                    if (keep)
                        poly.assign(n, 0.0);
                    for (std::uint64_t j = 0; j < n; ++j) {
                        double v;
                        if (!body.read(p.type, v))
                            return ply_fail(path, "truncated list in element '" + e.name + "'");
                        if (keep)
                            poly[j] = v;
                    }
                } else {
                    double v;
                    if (!body.read(p.type, v))
                        return ply_fail(path, "truncated element '" + e.name + "'");
                    if (is_vertex && static_cast<int>(k) == ix)
                        xyz[0] = v;
                    else if (is_vertex && static_cast<int>(k) == iy)
                        xyz[1] = v;
                    else if (is_vertex && static_cast<int>(k) == iz)
                        xyz[2] = v;
                }
            }
            if (is_vertex) {
                if (!std::isfinite(xyz[0]) || !std::isfinite(xyz[1]) || !std::isfinite(xyz[2]))
                    return ply_fail(path, "non-finite vertex position");
                x.push_back(static_cast<float>(xyz[0]));
                y.push_back(static_cast<float>(xyz[1]));
                z.push_back(static_cast<float>(xyz[2]));
            } else if (is_face && iface >= 0) {
                if (poly.size() < 3)
                    return ply_fail(path, "face with fewer than three vertices");
                for (double const v : poly)
                    if (!(v >= 0.0) || v >= static_cast<double>(vertex_count) || v != std::floor(v))
                        return ply_fail(path, "face index out of range");
                for (std::size_t j = 1; j + 1 < poly.size(); ++j) {
                    i0.push_back(static_cast<std::uint32_t>(poly[0]));
                    i1.push_back(static_cast<std::uint32_t>(poly[j]));
                    i2.push_back(static_cast<std::uint32_t>(poly[j + 1]));
                }
            }
        }
        if (is_vertex) {
            vertex_count = e.count;
            have_vertices = true;
        }
    }
    if (x.empty() || i0.empty())
        return ply_fail(path, "no vertices or no triangles");
    return GWNB_OK;
}

template <class T> T *copy_out(std::vector<T> const &v) {
    auto *p = static_cast<T *>(std::malloc(std::max<std::size_t>(v.size(), 1) * sizeof(T)));
    if (p != nullptr && !v.empty())
        std::memcpy(p, v.data(), v.size() * sizeof(T));
    return p;
}

// ---- scene files ----------------------------------------------------------------------------------

constexpr char k_scene_magic[8] = {'G', 'W', 'N', 'B', 'S', 'C', 'N', '1'};
constexpr std::uint32_t k_scene_version = 1;

struct scene_header {
    char magic[8];
    std::uint32_t version;
    std::uint32_t moment_mask;
    std::uint64_t vertex_count, triangle_count, node_count, primitive_count;
    gwnb_child_f32 root;
    std::uint32_t internal_stack_bound, packed_stack_bound;
};
static_assert(sizeof(scene_header) == 88);

// 64-bit checksum: FNV-1a over 8-byte words (then the tail bytes).
std::uint64_t checksum(unsigned char const *p, std::size_t n, std::uint64_t h = 0xcbf29ce484222325ull) {
    constexpr std::uint64_t prime = 0x100000001b3ull;
    std::size_t i = 0;
    for (; i + 8 <= n; i += 8) {
        std::uint64_t w;
        std::memcpy(&w, p + i, 8);
        h = (h ^ w) * prime;
    }
    for (; i < n; ++i)
        h = (h ^ p[i]) * prime;
    return h;
}

// The saved hierarchy is a tree the kernels can walk: a leaf root comes with no nodes; an internal
// root is node 0; every other node is the internal child of exactly one node with a smaller index
// (so no cycles); leaf ranges lie inside the primitive order; primitive ids name triangles.
bool scene_topology_ok(unsigned char const *node_bytes, std::size_t N, std::size_t P, std::size_t T,
                       std::uint32_t const *prims, std::uint64_t root) {
    for (std::size_t i = 0; i < P; ++i)
        if (prims[i] >= T)
            return false;
    if (ref_leaf(root))
        return N == 0 && ref_offset(root) <= P && ref_count(root) <= P - ref_offset(root);
    if (!ref_internal(root) || ref_offset(root) != 0 || N == 0)
        return false;
    std::vector<unsigned char> parents(N, 0);
    for (std::size_t n = 0; n < N; ++n) {
        node4 node;
        std::memcpy(&node, node_bytes + n * sizeof(node4), sizeof(node4));
        for (child const &c : node.c) {
            std::uint64_t const r = c.reference;
            if (!ref_valid(r))
                continue;
            std::uint64_t const off = ref_offset(r);
            if (ref_internal(r)) {
                if (off <= n || off >= N || parents[off]++ != 0)
                    return false;
            } else if (off > P || ref_count(r) > P - off) {
                return false;
            }
        }
    }
    for (std::size_t n = 1; n < N; ++n)
        if (parents[n] != 1)
            return false;
    return true;
}

int copy_to_host(void *dst, void const *src, std::size_t bytes, cudaStream_t s) {
    if (bytes == 0)
        return GWNB_OK;
    GWNB_CUDA_TRY(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    return GWNB_OK;
}

} // namespace
} // namespace gwnb

using namespace gwnb;

extern "C" {

int gwnb_mesh_read_ply(const char *path, gwnb_host_mesh_f32 *out) try {
    if (path == nullptr || out == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "ply: null path or output.");
    std::vector<float> x, y, z;
    std::vector<std::uint32_t> i0, i1, i2;
    GWNB_TRY(read_ply(path, x, y, z, i0, i1, i2));
    gwnb_host_mesh_f32 m{};
    m.x = copy_out(x);
    m.y = copy_out(y);
    m.z = copy_out(z);
    m.i0 = copy_out(i0);
    m.i1 = copy_out(i1);
    m.i2 = copy_out(i2);
    m.vertex_count = x.size();
    m.triangle_count = i0.size();
    if (!m.x || !m.y || !m.z || !m.i0 || !m.i1 || !m.i2) {
        gwnb_host_mesh_free(&m);
        return set_error(GWNB_INTERNAL_ERROR, "ply: out of host memory.");
    }
    *out = m;
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

void gwnb_host_mesh_free(gwnb_host_mesh_f32 *m) {
    if (m == nullptr)
        return;
    std::free(m->x);
    std::free(m->y);
    std::free(m->z);
    std::free(m->i0);
    std::free(m->i1);
    std::free(m->i2);
    *m = gwnb_host_mesh_f32{};
}

int gwnb_mesh_write_ply(const char *path, const gwnb_host_mesh_f32 *m, int binary) try {
    if (path == nullptr || m == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "ply: null path or mesh.");
    if (!has_storage(m->x, m->vertex_count) || !has_storage(m->y, m->vertex_count) ||
        !has_storage(m->z, m->vertex_count) || !has_storage(m->i0, m->triangle_count) ||
        !has_storage(m->i1, m->triangle_count) || !has_storage(m->i2, m->triangle_count))
        return set_error(GWNB_INVALID_ARGUMENT, "ply: mesh arrays must be non-null when non-empty.");
    std::ofstream o(path, std::ios::binary);
    if (!o)
        return set_error(GWNB_INVALID_ARGUMENT, std::string("ply: cannot create ") + path);
    o << "ply\nformat " << (binary ? "binary_little_endian" : "ascii") << " 1.0\n"
      << "element vertex " << m->vertex_count << "\nproperty float x\nproperty float y\nproperty float z\n"
      << "element face " << m->triangle_count << "\nproperty list uchar uint vertex_indices\nend_header\n";
    if (binary) {
        for (std::uint64_t v = 0; v < m->vertex_count; ++v) {
            float const p[3] = {m->x[v], m->y[v], m->z[v]};
            o.write(reinterpret_cast<char const *>(p), sizeof(p));
        }
        for (std::uint64_t t = 0; t < m->triangle_count; ++t) {
            unsigned char const three = 3;
            std::uint32_t const f[3] = {m->i0[t], m->i1[t], m->i2[t]};
            o.write(reinterpret_cast<char const *>(&three), 1);
            o.write(reinterpret_cast<char const *>(f), sizeof(f));
        }
    } else {
        char buf[128];
        for (std::uint64_t v = 0; v < m->vertex_count; ++v) {
            std::snprintf(buf, sizeof(buf), "%.9g %.9g %.9g\n", m->x[v], m->y[v], m->z[v]);
            o << buf;
        }
        for (std::uint64_t t = 0; t < m->triangle_count; ++t)
            o << "3 " << m->i0[t] << ' ' << m->i1[t] << ' ' << m->i2[t] << '\n';
    }
    if (!o)
        return set_error(GWNB_INTERNAL_ERROR, std::string("ply: write failed for ") + path);
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_scene_save_f32(const char *path, const gwnb_geometry_f32 *g, const gwnb_bvh4_f32 *b,
                        const gwnb_moment4_f32 *const *moments, int moment_count, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::scene_save");
    if (path == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "scene: null path.");
    if (!geometry_valid(g) || g->triangle_count == 0)
        return set_error(GWNB_INVALID_ARGUMENT, "Geometry object contains no queryable data.");
    if (!bvh_valid(b))
        return set_error(GWNB_INVALID_ARGUMENT, "BVH object contains no queryable data.");
    if (b->primitive_count != g->triangle_count)
        return set_error(GWNB_INVALID_ARGUMENT, "Geometry and BVH triangle counts differ.");
    if (moment_count < 0 || moment_count > 3 || (moment_count > 0 && moments == nullptr))
        return set_error(GWNB_INVALID_ARGUMENT, "scene: at most one moment object per order (0, 1, 2).");
    scene_header h{};
    std::memcpy(h.magic, k_scene_magic, 8);
    h.version = k_scene_version;
    for (int k = 0; k < moment_count; ++k) {
        gwnb_moment4_f32 const *m = moments[k];
        if (!moment_valid_for(m, b) || m->order < 0 || m->order > 2)
            return set_error(GWNB_INVALID_ARGUMENT, "scene: a moment object is not aligned with the BVH.");
        if (h.moment_mask & (1u << m->order))
            return set_error(GWNB_INVALID_ARGUMENT, "scene: two moment objects of the same order.");
        h.moment_mask |= 1u << m->order;
    }
    h.vertex_count = g->vertex_count;
    h.triangle_count = g->triangle_count;
    h.node_count = b->node_count;
    h.primitive_count = b->primitive_count;
    h.root = b->root;
    h.internal_stack_bound = b->internal_stack_bound;
    h.packed_stack_bound = b->packed_stack_bound;
    std::size_t const V = g->vertex_count, T = g->triangle_count, N = b->node_count, P = b->primitive_count;
    std::vector<unsigned char> blob(sizeof(h));
    std::memcpy(blob.data(), &h, sizeof(h));
    std::size_t total = sizeof(h) + 3 * V * 4 + 3 * T * 4 + N * 128 + P * 4 + P * 36;
    for (int o = 0; o < 3; ++o)
        if (h.moment_mask & (1u << o))
            total += N * gwnb_moment_node_bytes(o);
    blob.resize(total);
    cudaStream_t const s = as_cuda(stream);
    unsigned char *w = blob.data() + sizeof(h);
    auto put = [&](void const *src, std::size_t bytes) -> int {
        int const rc = copy_to_host(w, src, bytes, s);
        w += bytes;
        return rc;
    };
    GWNB_TRY(put(g->vertex_x, V * 4));
    GWNB_TRY(put(g->vertex_y, V * 4));
    GWNB_TRY(put(g->vertex_z, V * 4));
    GWNB_TRY(put(g->tri_i0, T * 4));
    GWNB_TRY(put(g->tri_i1, T * 4));
    GWNB_TRY(put(g->tri_i2, T * 4));
    GWNB_TRY(put(b->nodes, N * 128));
    GWNB_TRY(put(b->primitive_indices, P * 4));
    GWNB_TRY(put(b->triangles, P * 36));
    for (int o = 0; o < 3; ++o)
        for (int k = 0; k < moment_count; ++k)
            if (moments[k]->order == o)
                GWNB_TRY(put(moments[k]->nodes, N * gwnb_moment_node_bytes(o)));
    GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    std::uint64_t const sum = checksum(blob.data(), blob.size());
    std::ofstream out(path, std::ios::binary);
    if (!out)
        return set_error(GWNB_INVALID_ARGUMENT, std::string("scene: cannot create ") + path);
    out.write(reinterpret_cast<char const *>(blob.data()), static_cast<std::streamsize>(blob.size()));
    out.write(reinterpret_cast<char const *>(&sum), sizeof(sum));
    if (!out)
        return set_error(GWNB_INTERNAL_ERROR, std::string("scene: write failed for ") + path);
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

int gwnb_scene_load_f32(const char *path, gwnb_geometry_f32 *g_out, gwnb_bvh4_f32 *b_out, gwnb_moment4_f32 *m_out,
                        int *moment_mask, gwnb_stream_t stream) try {
    GWNB_NVTX("gwnb::scene_load");
    if (path == nullptr || g_out == nullptr || b_out == nullptr || m_out == nullptr)
        return set_error(GWNB_INVALID_ARGUMENT, "scene: null path or output.");
    std::ifstream in(path, std::ios::binary);
    if (!in)
        return set_error(GWNB_INVALID_ARGUMENT, std::string("scene: cannot open ") + path);
    std::vector<unsigned char> blob((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
    if (blob.size() < sizeof(scene_header) + 8)
        return set_error(GWNB_INVALID_ARGUMENT, "scene: file too short.");
    scene_header h;
    std::memcpy(&h, blob.data(), sizeof(h));
    if (std::memcmp(h.magic, k_scene_magic, 8) != 0)
        return set_error(GWNB_INVALID_ARGUMENT, "scene: not a scene file (bad magic).");
    if (h.version != k_scene_version)
        return set_error(GWNB_INVALID_ARGUMENT, "scene: unsupported version " + std::to_string(h.version) + ".");
    std::uint64_t stored;
    std::memcpy(&stored, blob.data() + blob.size() - 8, 8);
    if (checksum(blob.data(), blob.size() - 8) != stored)
        return set_error(GWNB_INVALID_ARGUMENT, "scene: checksum mismatch (corrupt or truncated file).");
    std::size_t const V = h.vertex_count, T = h.triangle_count, N = h.node_count, P = h.primitive_count;
    if (V > blob.size() || T > blob.size() || N > blob.size() || P > blob.size()) // keeps the sum below exact
        return set_error(GWNB_INVALID_ARGUMENT, "scene: inconsistent counts in the header.");
    std::size_t total = sizeof(h) + 3 * V * 4 + 3 * T * 4 + N * 128 + P * 4 + P * 36 + 8;
    for (int o = 0; o < 3; ++o)
        if (h.moment_mask & (1u << o))
            total += N * gwnb_moment_node_bytes(o);
    if ((h.moment_mask & ~7u) != 0 || total != blob.size() || P != T || T == 0)
        return set_error(GWNB_INVALID_ARGUMENT, "scene: inconsistent counts in the header.");
    unsigned char const *r = blob.data() + sizeof(h);
    auto take = [&](std::size_t bytes) {
        unsigned char const *p = r;
        r += bytes;
        return p;
    };
    auto const *x = reinterpret_cast<float const *>(take(V * 4));
    auto const *y = reinterpret_cast<float const *>(take(V * 4));
    auto const *z = reinterpret_cast<float const *>(take(V * 4));
    auto const *i0 = reinterpret_cast<std::uint32_t const *>(take(T * 4));
    auto const *i1 = reinterpret_cast<std::uint32_t const *>(take(T * 4));
    auto const *i2 = reinterpret_cast<std::uint32_t const *>(take(T * 4));
    unsigned char const *nodes = take(N * 128);
    unsigned char const *prims = take(P * 4);
    unsigned char const *tris = take(P * 36);
    std::vector<std::uint32_t> prim_ids(P);
    std::memcpy(prim_ids.data(), prims, P * 4);
    if (!scene_topology_ok(nodes, N, P, T, prim_ids.data(), h.root.reference))
        return set_error(GWNB_INVALID_ARGUMENT, "scene: the saved hierarchy is not a valid BVH4 tree.");
    cudaStream_t const s = as_cuda(stream);
    gwnb_geometry_f32 g{};
    GWNB_TRY(gwnb_geometry_upload_f32(&g, x, y, z, V, i0, i1, i2, T, stream));
    gwnb_bvh4_f32 b{};
    auto fail = [&](int rc) {
        gwnb_bvh4_release_f32(&b, stream);
        gwnb_geometry_release_f32(&g, stream);
        return rc;
    };
    int rc;
    if ((rc = alloc(reinterpret_cast<node4 **>(&b.nodes), N, s)) != GWNB_OK ||
        (rc = alloc(&b.primitive_indices, P, s)) != GWNB_OK ||
        (rc = alloc(reinterpret_cast<triangle **>(&b.triangles), P, s)) != GWNB_OK)
        return fail(rc);
    b.node_count = N;
    b.node_capacity = N;
    b.primitive_count = P;
    b.root = h.root;
    b.internal_stack_bound = h.internal_stack_bound;
    b.packed_stack_bound = h.packed_stack_bound;
    cudaError_t e = cudaSuccess;
    if (N > 0)
        e = cudaMemcpyAsync(b.nodes, nodes, N * 128, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b.primitive_indices, prims, P * 4, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(b.triangles, tris, P * 36, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess)
        return fail(set_cuda_error(e, "scene upload"));
    b.revision = reserve_revision();
    if (!bvh_valid(&b))
        return fail(set_error(GWNB_INVALID_ARGUMENT, "scene: the BVH in the file is not queryable."));
    if ((rc = ensure_bvh_aux(&b, s)) != GWNB_OK)
        return fail(rc);
    gwnb_moment4_f32 loaded[3] = {};
    auto fail_all = [&](int code) {
        for (int o = 0; o < 3; ++o)
            gwnb_moment4_release_f32(&loaded[o], stream);
        return fail(code);
    };
    for (int o = 0; o < 3; ++o) {
        loaded[o].order = o;
        if (!(h.moment_mask & (1u << o)))
            continue;
        std::size_t const bytes = N * gwnb_moment_node_bytes(o);
        unsigned char const *saved = take(bytes);
        if ((rc = gwnb_moment4_refit_f32(&b, o, &loaded[o], stream)) != GWNB_OK)
            return fail_all(rc);
        std::vector<unsigned char> now(bytes);
        if (bytes > 0) {
            if ((e = cudaMemcpyAsync(now.data(), loaded[o].nodes, bytes, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
                (e = cudaStreamSynchronize(s)) != cudaSuccess)
                return fail_all(set_cuda_error(e, "scene moment check"));
            if (std::memcmp(now.data(), saved, bytes) != 0)
                return fail_all(set_error(GWNB_INVALID_ARGUMENT, "scene: saved order-" + std::to_string(o) +
                                                                     " moments differ from a refit of the saved BVH."));
        }
    }
    GWNB_CUDA_TRY(cudaStreamSynchronize(s));
    *g_out = g;
    *b_out = b;
    for (int o = 0; o < 3; ++o)
        m_out[o] = loaded[o];
    if (moment_mask != nullptr)
        *moment_mask = static_cast<int>(h.moment_mask);
    return GWNB_OK;
} catch (...) {
    return host_exception();
}

} // extern "C"
