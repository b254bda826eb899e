// ply.cpp - reads triangle meshes from PLY files as Shape/PlyMesh.swift does:
// format binary_little_endian or binary_big_endian 1.0; a vertex element of
// float properties x y z, optionally followed by u v, nx ny nz, nx ny nz u v
// (or s t) or u v nx ny nz; a face element with a "list uchar|uint int"
// vertex_indices property and an optional "int face_indices".  Faces must be
// triangles (the reference warns and appends any other count, which
// misaligns every later face; here it is an error).  The arrays are packed
// for the device ingestion path: float x3 points, int32 x3 indices.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "gzg_internal.h"

namespace gzg {
namespace {

struct Reader {
        const uint8_t *p;
        size_t n, pos = 0;
        bool big = false;
        bool line(std::string *out) {
                out->clear();
                while (pos < n && p[pos] != '\n') out->push_back((char)p[pos++]);
                if (pos >= n) return false;
                ++pos;
                if (!out->empty() && out->back() == '\r') out->pop_back();
                return true;
        }
        template <class T>
        bool get(T *v) {
                if (n - pos < sizeof(T) || pos > n) return false;
                uint8_t b[sizeof(T)];
                std::memcpy(b, p + pos, sizeof(T));
                if (big)
                        for (size_t i = 0; i < sizeof(T) / 2; ++i) std::swap(b[i], b[sizeof(T) - 1 - i]);
                std::memcpy(v, b, sizeof(T));
                pos += sizeof(T);
                return true;
        }
};

gzg_status bad(const std::string &m) { return set_error(GZG_ERR_BAD_SCENE, "gzg_ply_parse: " + m); }

}  // namespace
}  // namespace gzg

using namespace gzg;

struct gzg_ply_owned {
        gzg_ply_mesh mesh{};
        std::vector<float> points, normals, uvs;
        std::vector<int32_t> indices, face_indices;
};

namespace {

gzg_status parse_ply(const uint8_t *data, size_t size, gzg_ply_mesh **out) {
        Reader r{data, size};
        std::string ln;
        if (!r.line(&ln) || ln != "ply") return bad("the first line must be \"ply\"");
        enum { kNone, kVertex, kFace } state = kNone;
        int64_t nv = -1, nf = -1;
        std::vector<std::string> props;
        int list_bits = 8;
        bool has_face_indices = false, have_list = false;
        for (;;) {
                if (!r.line(&ln)) return bad("header without end_header");
                std::istringstream ws(ln);
                std::vector<std::string> w;
                for (std::string t; ws >> t;) w.push_back(t);
                if (w.empty()) return bad("empty header line");
                if (w[0] == "comment" || w[0] == "obj_info") continue;
                if (w[0] == "format") {
                        if (w.size() < 3 || w[2] != "1.0") return bad("format version must be 1.0");
                        if (w[1] == "binary_little_endian")
                                r.big = false;
                        else if (w[1] == "binary_big_endian")
                                r.big = true;
                        else
                                return bad("unsupported format " + w[1]);
                } else if (w[0] == "element") {
                        if (w.size() < 3) return bad("bad element line");
                        char *end = nullptr;
                        const long long c = std::strtoll(w[2].c_str(), &end, 10);
                        if (!end || *end || c < 0) return bad("bad element count");
                        if (w[1] == "vertex") {
                                state = kVertex;
                                nv = c;
                        } else if (w[1] == "face") {
                                state = kFace;
                                nf = c;
                        } else {
                                return bad("unknown element " + w[1]);
                        }
                } else if (w[0] == "property") {
                        if (w.size() < 3) return bad("bad property line");
                        if (w[1] == "float" || w[1] == "float32") {
                                if (state != kVertex) return bad("float property outside the vertex element");
                                props.push_back(w[2]);
                        } else if (w[1] == "list") {
                                if (state != kFace || w.size() < 5) return bad("list property outside the face element");
                                if (w[2] == "uint" || w[2] == "uint32")
                                        list_bits = 32;
                                else if (w[2] == "uchar" || w[2] == "uint8")
                                        list_bits = 8;
                                else
                                        return bad("unsupported list count type " + w[2]);
                                if (w[3] != "int" && w[3] != "int32") return bad("list indices must be int");
                                have_list = true;
                        } else if (w[1] == "int" || w[1] == "int32") {
                                if (state != kFace || w[2] != "face_indices") return bad("unknown int property " + w[2]);
                                has_face_indices = true;
                        } else {
                                return bad("unknown property type " + w[1]);
                        }
                } else if (w[0] == "end_header") {
                        break;
                } else {
                        return bad("unknown header word " + w[0]);
                }
        }
        if (nv < 0) return bad("no vertex element");
        if (nf < 0) nf = 0;
        if (nf > 0 && !have_list) return bad("face element without vertex_indices");
        // vertex layouts of PlyMesh.readVertices
        auto is = [&](std::initializer_list<const char *> names) {
                if (props.size() != names.size()) return false;
                size_t i = 0;
                for (const char *nm : names)
                        if (props[i++] != nm) return false;
                return true;
        };
        enum { kP, kPUV, kPN, kPNUV, kPUVN } layout;
        if (is({"x", "y", "z"}))
                layout = kP;
        else if (is({"x", "y", "z", "u", "v"}))
                layout = kPUV;
        else if (is({"x", "y", "z", "nx", "ny", "nz"}))
                layout = kPN;
        else if (is({"x", "y", "z", "nx", "ny", "nz", "u", "v"}) || is({"x", "y", "z", "nx", "ny", "nz", "s", "t"}))
                layout = kPNUV;
        else if (is({"x", "y", "z", "u", "v", "nx", "ny", "nz"}))
                layout = kPUVN;
        else
                return bad("unsupported vertex properties");
        const size_t per = props.size() * 4;
        if ((uint64_t)nv > (r.n - r.pos) / per) return bad("file shorter than its vertices");
        if (nv > INT32_MAX || nf > INT32_MAX) return set_error(GZG_ERR_LIMIT, "gzg_ply_parse: more than 2^31 vertices or faces");
        auto o = std::make_unique<gzg_ply_owned>();
        o->points.resize((size_t)nv * 3);
        const bool has_n = layout == kPN || layout == kPNUV || layout == kPUVN;
        const bool has_uv = layout == kPUV || layout == kPNUV || layout == kPUVN;
        if (has_n) o->normals.resize((size_t)nv * 3);
        if (has_uv) o->uvs.resize((size_t)nv * 2);
        for (int64_t i = 0; i < nv; ++i) {
                float v[8];
                for (size_t k = 0; k < props.size(); ++k) r.get(&v[k]);
                std::memcpy(&o->points[3 * i], v, 12);
                if (layout == kPUV) std::memcpy(&o->uvs[2 * i], v + 3, 8);
                if (layout == kPN) std::memcpy(&o->normals[3 * i], v + 3, 12);
                if (layout == kPNUV) {
                        std::memcpy(&o->normals[3 * i], v + 3, 12);
                        std::memcpy(&o->uvs[2 * i], v + 6, 8);
                }
                if (layout == kPUVN) {
                        std::memcpy(&o->uvs[2 * i], v + 3, 8);
                        std::memcpy(&o->normals[3 * i], v + 5, 12);
                }
        }
        o->indices.resize((size_t)nf * 3);
        if (has_face_indices) o->face_indices.resize((size_t)nf);
        for (int64_t f = 0; f < nf; ++f) {
                uint32_t cnt = 0;
                bool ok;
                if (list_bits == 8) {
                        uint8_t c8 = 0;
                        ok = r.get(&c8);
                        cnt = c8;
                } else {
                        ok = r.get(&cnt);
                }
                if (!ok) return bad("file shorter than its faces");
                if (cnt != 3) return bad("face " + std::to_string(f) + " has " + std::to_string(cnt) + " indices, not 3");
                for (int k = 0; k < 3; ++k) {
                        int32_t ix;
                        if (!r.get(&ix)) return bad("file shorter than its faces");
                        if (ix < 0 || ix >= nv) return bad("face " + std::to_string(f) + " index out of range");
                        o->indices[3 * f + k] = ix;
                }
                if (has_face_indices) {
                        int32_t fi;
                        if (!r.get(&fi)) return bad("file shorter than its faces");
                        o->face_indices[f] = fi;
                }
        }
        gzg_ply_mesh &m = o->mesh;
        m.vertex_count = nv;
        m.face_count = nf;
        m.points = o->points.data();
        m.normals = has_n ? o->normals.data() : nullptr;
        m.uvs = has_uv ? o->uvs.data() : nullptr;
        m.indices = o->indices.data();
        m.face_indices = has_face_indices ? o->face_indices.data() : nullptr;
        m.owner = o.get();
        *out = &o.release()->mesh;
        return clear_error();
}

}  // namespace

GZG_API gzg_status gzg_ply_parse(const void *data, int64_t size, gzg_ply_mesh **out) {
        if (!out || (!data && size > 0) || size < 0) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_ply_parse: bad arguments");
        *out = nullptr;
        return parse_ply(reinterpret_cast<const uint8_t *>(data), (size_t)size, out);
}

GZG_API gzg_status gzg_ply_read(const char *path, gzg_ply_mesh **out) {
        if (!path || !out) return set_error(GZG_ERR_INVALID_ARGUMENT, "gzg_ply_read: null argument");
        *out = nullptr;
        std::FILE *f = std::fopen(path, "rb");
        if (!f) return set_error(GZG_ERR_INVALID_ARGUMENT, std::string("gzg_ply_read: cannot open ") + path);
        std::vector<uint8_t> buf;
        uint8_t chunk[1 << 16];
        size_t got;
        while ((got = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + got);
        std::fclose(f);
        return parse_ply(buf.data(), buf.size(), out);
}

GZG_API gzg_status gzg_ply_free(gzg_ply_mesh *mesh) {
        if (mesh) delete static_cast<gzg_ply_owned *>(mesh->owner);
        return clear_error();
}
