// Scene ingestion and film output: Wavefront OBJ meshes, Radiance .hdr
// images, PFM images.  Replaces the reference's delegates, which call assimp
// (src/delegate/meshimporter.cpp:41-120) and stb_image
// (src/delegate/imageutil.cpp:98-139); both are third-party code absent from
// the reference tree, so the behaviour below is restated from their
// documented processing (assimp's aiProcess_Triangulate | GenSmoothNormals |
// FlipUVs | CalcTangentSpace, stb_image's RGBE decoding) in code of our own.
// Host code only: parsing runs on the CPU, the results go through
// cl_build_meshes / cl_build_emitters like any caller-owned data.
#include "../../include/colvillea_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <new>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

namespace clb
{
void setLastError(const std::string& msg);
}

namespace
{
struct V3
{
    double x, y, z;
};
V3     sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3     add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
V3     mul(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
V3     cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
bool   normalizeInPlace(V3& a)
{
    double l = std::sqrt(dot(a, a));
    if (!(l > 0.0) || !std::isfinite(l)) return false;
    a = mul(a, 1.0 / l);
    return true;
}
// Any unit vector perpendicular to n (the larger of two candidates).
V3 perpendicular(V3 n)
{
    V3 t = std::fabs(n.x) > std::fabs(n.y) ? V3{-n.z, 0.0, n.x} : V3{0.0, n.z, -n.y};
    if (!normalizeInPlace(t)) t = {1.0, 0.0, 0.0};
    return t;
}

cl_status fail(cl_status s, const std::string& msg)
{
    clb::setLastError(msg);
    return s;
}
} // namespace

// One OBJ group: arrays in cl_mesh_desc layout, owned here.
struct ObjMesh
{
    std::string           name;
    std::vector<float>    pos, nrm, tan, uv;
    std::vector<uint32_t> idx;
    bool                  hasUV = false;
};

struct cl_obj
{
    std::vector<ObjMesh> meshes;
};

namespace
{
// Face vertex reference (1-based OBJ indices resolved to 0-based, -1 = absent).
struct Ref
{
    long v = -1, t = -1, n = -1;
    bool operator<(const Ref& o) const { return std::tie(v, t, n) < std::tie(o.v, o.t, o.n); }
};

bool parseIndex(const std::string& s, long count, long* out)
{
    if (s.empty()) return false;
    char* end = nullptr;
    long  i   = std::strtol(s.c_str(), &end, 10);
    if (*end != '\0' || i == 0) return false;
    *out = i > 0 ? i - 1 : count + i; // negative: relative to the end
    return *out >= 0 && *out < count;
}

struct Group
{
    std::string             name;
    std::vector<Ref>        corners; // 3 per triangle
};

// Builds the mesh of one group: vertices unified per (v, vt, vn) triple;
// normals from vn when every corner has one, else smooth normals (sum of
// the area-weighted face normals of the faces that share the position);
// uvs from vt with v flipped (1 - v) when every corner has one; tangents
// from the uv derivatives (dP/du summed over the faces of the vertex,
// orthogonalised against the normal), or any perpendicular without uvs.
cl_status buildMesh(const Group& g, const std::vector<V3>& P, const std::vector<std::pair<double, double>>& T,
                    const std::vector<V3>& N, ObjMesh* out)
{
    bool allN = true, allT = true;
    for (const Ref& r : g.corners)
    {
        allN &= r.n >= 0;
        allT &= r.t >= 0;
    }
    std::map<Ref, uint32_t> ids;
    std::vector<Ref>        verts;
    std::vector<uint32_t>   idx;
    idx.reserve(g.corners.size());
    for (Ref r : g.corners)
    {
        if (!allN) r.n = -1;
        if (!allT) r.t = -1;
        auto it = ids.find(r);
        if (it == ids.end())
        {
            it = ids.emplace(r, uint32_t(verts.size())).first;
            verts.push_back(r);
        }
        idx.push_back(it->second);
    }
    const size_t nv = verts.size(), nt = idx.size() / 3;
    std::vector<V3> nrm(nv, V3{0, 0, 0}), tan(nv, V3{0, 0, 0});
    if (allN)
        for (size_t i = 0; i < nv; ++i) nrm[i] = N[size_t(verts[i].n)];
    else
    {
        // Smooth normals per position index.
        std::map<long, V3> acc;
        for (size_t f = 0; f < nt; ++f)
        {
            const Ref &a = verts[idx[3 * f]], &b = verts[idx[3 * f + 1]], &c = verts[idx[3 * f + 2]];
            V3 fn = cross(sub(P[b.v], P[a.v]), sub(P[c.v], P[a.v]));
            for (const Ref* r : {&a, &b, &c}) acc[r->v] = add(acc[r->v], fn);
        }
        for (size_t i = 0; i < nv; ++i) nrm[i] = acc[verts[i].v];
    }
    for (size_t i = 0; i < nv; ++i)
        if (!normalizeInPlace(nrm[i])) nrm[i] = {0.0, 1.0, 0.0};
    if (allT)
    {
        for (size_t f = 0; f < nt; ++f)
        {
            const uint32_t i0 = idx[3 * f], i1 = idx[3 * f + 1], i2 = idx[3 * f + 2];
            const Ref &a = verts[i0], &b = verts[i1], &c = verts[i2];
            V3     e1 = sub(P[b.v], P[a.v]), e2 = sub(P[c.v], P[a.v]);
            double du1 = T[b.t].first - T[a.t].first, dv1 = T[b.t].second - T[a.t].second;
            double du2 = T[c.t].first - T[a.t].first, dv2 = T[c.t].second - T[a.t].second;
            double det = du1 * dv2 - du2 * dv1;
            if (!(std::fabs(det) > 0.0)) continue;
            V3 t = mul(sub(mul(e1, dv2), mul(e2, dv1)), 1.0 / det);
            for (uint32_t k : {i0, i1, i2}) tan[k] = add(tan[k], t);
        }
    }
    for (size_t i = 0; i < nv; ++i)
    {
        V3 t = sub(tan[i], mul(nrm[i], dot(nrm[i], tan[i])));
        if (!normalizeInPlace(t)) t = perpendicular(nrm[i]);
        tan[i] = t;
    }
    out->name = g.name;
    out->pos.resize(3 * nv);
    out->nrm.resize(3 * nv);
    out->tan.resize(3 * nv);
    out->hasUV = allT;
    if (allT) out->uv.resize(2 * nv);
    for (size_t i = 0; i < nv; ++i)
    {
        const V3& p = P[size_t(verts[i].v)];
        out->pos[3 * i] = float(p.x), out->pos[3 * i + 1] = float(p.y), out->pos[3 * i + 2] = float(p.z);
        out->nrm[3 * i] = float(nrm[i].x), out->nrm[3 * i + 1] = float(nrm[i].y), out->nrm[3 * i + 2] = float(nrm[i].z);
        out->tan[3 * i] = float(tan[i].x), out->tan[3 * i + 1] = float(tan[i].y), out->tan[3 * i + 2] = float(tan[i].z);
        if (allT)
        {
            out->uv[2 * i]     = float(T[size_t(verts[i].t)].first);
            out->uv[2 * i + 1] = float(1.0 - T[size_t(verts[i].t)].second);
        }
    }
    out->idx = std::move(idx);
    return CL_OK;
}

cl_status parseObj(std::istream& in, cl_obj* obj, std::string* err)
{
    std::vector<V3>                        P, N;
    std::vector<std::pair<double, double>> T;
    std::vector<Group>                     groups(1);
    std::string                            line, pending;
    size_t                                 lineNo = 0;
    auto newGroup = [&](const std::string& name) {
        if (!groups.back().corners.empty()) groups.emplace_back();
        groups.back().name = name;
    };
    while (std::getline(in, line))
    {
        ++lineNo;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        if (!line.empty() && line.back() == '\\') // continuation
        {
            pending += line.substr(0, line.size() - 1) + " ";
            continue;
        }
        line = pending + line;
        pending.clear();
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        std::istringstream ls(line);
        std::string        tag;
        if (!(ls >> tag)) continue;
        auto bad = [&](const char* what) {
            *err = "OBJ line " + std::to_string(lineNo) + ": " + what;
            return CL_ERR_INVALID_ARG;
        };
        if (tag == "v")
        {
            V3 p;
            if (!(ls >> p.x >> p.y >> p.z)) return bad("vertex needs 3 coordinates");
            P.push_back(p);
        }
        else if (tag == "vt")
        {
            double u = 0.0, v = 0.0;
            if (!(ls >> u)) return bad("texture coordinate needs u");
            ls >> v;
            T.emplace_back(u, v);
        }
        else if (tag == "vn")
        {
            V3 n;
            if (!(ls >> n.x >> n.y >> n.z)) return bad("normal needs 3 components");
            N.push_back(n);
        }
        else if (tag == "f")
        {
            std::vector<Ref> face;
            std::string      tok;
            while (ls >> tok)
            {
                Ref               r;
                std::string       parts[3];
                int               k = 0;
                for (char ch : tok)
                {
                    if (ch == '/')
                    {
                        if (++k > 2) return bad("face vertex with more than 3 fields");
                    }
                    else
                        parts[k] += ch;
                }
                if (!parseIndex(parts[0], long(P.size()), &r.v)) return bad("bad vertex index");
                if (k >= 1 && !parts[1].empty() && !parseIndex(parts[1], long(T.size()), &r.t))
                    return bad("bad texture-coordinate index");
                if (k >= 2 && !parts[2].empty() && !parseIndex(parts[2], long(N.size()), &r.n))
                    return bad("bad normal index");
                face.push_back(r);
            }
            if (face.size() < 3) return bad("face with fewer than 3 vertices");
            for (size_t i = 1; i + 1 < face.size(); ++i) // fan triangulation
            {
                groups.back().corners.push_back(face[0]);
                groups.back().corners.push_back(face[i]);
                groups.back().corners.push_back(face[i + 1]);
            }
        }
        else if (tag == "o" || tag == "g" || tag == "usemtl")
        {
            std::string name;
            std::getline(ls, name);
            name.erase(0, name.find_first_not_of(" \t"));
            newGroup(name);
        }
        // s, mtllib, l, p and other statements carry nothing the renderer uses.
    }
    for (const Group& g : groups)
    {
        if (g.corners.empty()) continue;
        obj->meshes.emplace_back();
        cl_status s = buildMesh(g, P, T, N, &obj->meshes.back());
        if (s != CL_OK) return s;
    }
    if (obj->meshes.empty())
    {
        *err = "OBJ file has no faces";
        return CL_ERR_INVALID_ARG;
    }
    return CL_OK;
}

// Radiance RGBE: value = byte * 2^(e - 136) for e != 0, else 0; alpha 1
// (stb_image's conversion for 4 requested components).
void rgbeToFloat(const uint8_t* q, float* out)
{
    if (q[3] != 0)
    {
        const float f = std::ldexp(1.0f, int(q[3]) - 136);
        out[0] = float(q[0]) * f, out[1] = float(q[1]) * f, out[2] = float(q[2]) * f;
    }
    else
        out[0] = out[1] = out[2] = 0.0f;
    out[3] = 1.0f;
}

struct Reader
{
    const std::vector<uint8_t>& b;
    size_t                      p = 0;
    bool get(uint8_t* v)
    {
        if (p >= b.size()) return false;
        *v = b[p++];
        return true;
    }
    bool line(std::string* s)
    {
        s->clear();
        while (p < b.size() && b[p] != '\n') s->push_back(char(b[p++]));
        if (p >= b.size()) return false;
        ++p;
        return true;
    }
};

// Header ("#?RADIANCE" or "#?RGBE", FORMAT=32-bit_rle_rgbe, blank line), the
// resolution line "-Y h +X w" (top-to-bottom rows, the orientation the
// reference's loader accepts), then per scanline either the new-style
// run-length encoding (2, 2, width hi, width lo, then the four channels each
// as runs: count > 128 repeats the next byte count - 128 times, otherwise
// count literal bytes) or flat RGBE quads.
cl_status decodeHdr(const std::vector<uint8_t>& data, std::vector<float>* rgba, uint32_t* w, uint32_t* h,
                    std::string* err)
{
    Reader      r{data};
    std::string ln;
    if (!r.line(&ln) || (ln.rfind("#?RADIANCE", 0) != 0 && ln.rfind("#?RGBE", 0) != 0))
    {
        *err = "not a Radiance HDR file (no #?RADIANCE header)";
        return CL_ERR_INVALID_ARG;
    }
    bool fmt = false;
    for (;;)
    {
        if (!r.line(&ln))
        {
            *err = "HDR header not terminated";
            return CL_ERR_INVALID_ARG;
        }
        if (!ln.empty() && ln.back() == '\r') ln.pop_back();
        if (ln.empty()) break;
        if (ln == "FORMAT=32-bit_rle_rgbe") fmt = true;
        if (ln.rfind("FORMAT=", 0) == 0 && ln != "FORMAT=32-bit_rle_rgbe")
        {
            *err = "unsupported HDR format: " + ln;
            return CL_ERR_INVALID_ARG;
        }
    }
    if (!fmt)
    {
        *err = "HDR header lacks FORMAT=32-bit_rle_rgbe";
        return CL_ERR_INVALID_ARG;
    }
    if (!r.line(&ln))
    {
        *err = "HDR file lacks a resolution line";
        return CL_ERR_INVALID_ARG;
    }
    int  H = 0, W = 0;
    char ya[3] = {}, xa[3] = {};
    if (std::sscanf(ln.c_str(), "%2s %d %2s %d", ya, &H, xa, &W) != 4 || std::strcmp(ya, "-Y") != 0 ||
        std::strcmp(xa, "+X") != 0 || W <= 0 || H <= 0 || W > (1 << 16) || H > (1 << 16))
    {
        *err = "unsupported HDR resolution line (only \"-Y h +X w\"): " + ln;
        return CL_ERR_INVALID_ARG;
    }
    rgba->assign(size_t(W) * H * 4, 0.0f);
    std::vector<uint8_t> scan(size_t(W) * 4);
    auto truncated = [&]() {
        *err = "HDR pixel data truncated";
        return CL_ERR_INVALID_ARG;
    };
    for (int y = 0; y < H; ++y)
    {
        uint8_t q[4];
        for (int k = 0; k < 4; ++k)
            if (!r.get(&q[k])) return truncated();
        const bool rle = W >= 8 && W < 32768 && q[0] == 2 && q[1] == 2 && !(q[2] & 0x80);
        if (!rle)
        {
            // Flat scanline: the four bytes read are the first pixel.
            std::memcpy(&scan[0], q, 4);
            for (int x = 1; x < W; ++x)
                for (int k = 0; k < 4; ++k)
                    if (!r.get(&scan[4 * size_t(x) + k])) return truncated();
        }
        else
        {
            if ((int(q[2]) << 8 | q[3]) != W)
            {
                *err = "HDR scanline width mismatch";
                return CL_ERR_INVALID_ARG;
            }
            for (int c = 0; c < 4; ++c)
            {
                int x = 0;
                while (x < W)
                {
                    uint8_t cnt;
                    if (!r.get(&cnt)) return truncated();
                    if (cnt > 128)
                    {
                        uint8_t v;
                        if (!r.get(&v)) return truncated();
                        int n = cnt - 128;
                        if (x + n > W)
                        {
                            *err = "HDR run exceeds the scanline";
                            return CL_ERR_INVALID_ARG;
                        }
                        for (int i = 0; i < n; ++i) scan[4 * size_t(x++) + c] = v;
                    }
                    else
                    {
                        if (cnt == 0 || x + cnt > W)
                        {
                            *err = "bad HDR literal run";
                            return CL_ERR_INVALID_ARG;
                        }
                        for (int i = 0; i < cnt; ++i)
                            if (!r.get(&scan[4 * size_t(x++) + c])) return truncated();
                    }
                }
            }
        }
        for (int x = 0; x < W; ++x) rgbeToFloat(&scan[4 * size_t(x)], &(*rgba)[(size_t(y) * W + x) * 4]);
    }
    *w = uint32_t(W);
    *h = uint32_t(H);
    return CL_OK;
}

bool readFile(const char* path, std::vector<uint8_t>* out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    out->assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return true;
}

template <class F> cl_status guardedIo(F&& f)
{
    std::string err;
    cl_status   s;
    try
    {
        s = f(&err);
    }
    catch (const std::bad_alloc&)
    {
        err = "host allocation failed";
        s   = CL_ERR_OOM;
    }
    catch (const std::exception& e)
    {
        err = e.what();
        s   = CL_ERR_STATE;
    }
    if (s != CL_OK) clb::setLastError(err.empty() ? "error " + std::to_string(s) : err);
    return s;
}
} // namespace

extern "C" {

cl_status cl_obj_load(const char* path, cl_obj** out)
{
    if (!path || !out) return fail(CL_ERR_INVALID_ARG, "path or out is null");
    *out = nullptr;
    return guardedIo([&](std::string* e) -> cl_status {
        std::ifstream f(path);
        if (!f)
        {
            *e = std::string("cannot open ") + path;
            return CL_ERR_INVALID_ARG;
        }
        std::unique_ptr<cl_obj> o(new cl_obj());
        cl_status               s = parseObj(f, o.get(), e);
        if (s == CL_OK) *out = o.release();
        return s;
    });
}

cl_status cl_obj_mesh_count(const cl_obj* obj, uint32_t* count)
{
    if (!obj || !count) return fail(CL_ERR_INVALID_ARG, "obj or count is null");
    *count = uint32_t(obj->meshes.size());
    return CL_OK;
}

cl_status cl_obj_get_mesh(const cl_obj* obj, uint32_t index, cl_mesh_desc* mesh)
{
    if (!obj || !mesh) return fail(CL_ERR_INVALID_ARG, "obj or mesh is null");
    if (index >= obj->meshes.size()) return fail(CL_ERR_INVALID_ARG, "mesh index out of range");
    const ObjMesh& m    = obj->meshes[index];
    mesh->positions     = m.pos.data();
    mesh->normals       = m.nrm.data();
    mesh->tangents      = m.tan.data();
    mesh->uvs           = m.hasUV ? m.uv.data() : nullptr;
    mesh->num_vertices  = uint32_t(m.pos.size() / 3);
    mesh->indices       = m.idx.data();
    mesh->num_triangles = uint32_t(m.idx.size() / 3);
    return CL_OK;
}

cl_status cl_obj_free(cl_obj* obj)
{
    delete obj;
    return CL_OK;
}

cl_status cl_image_load_hdr(const char* path, float** rgba, uint32_t* width, uint32_t* height)
{
    if (!path || !rgba || !width || !height) return fail(CL_ERR_INVALID_ARG, "null argument");
    *rgba = nullptr;
    return guardedIo([&](std::string* e) -> cl_status {
        std::vector<uint8_t> data;
        if (!readFile(path, &data))
        {
            *e = std::string("cannot open ") + path;
            return CL_ERR_INVALID_ARG;
        }
        std::vector<float> px;
        cl_status s = decodeHdr(data, &px, width, height, e);
        if (s != CL_OK) return s;
        float* buf = static_cast<float*>(std::malloc(px.size() * sizeof(float)));
        if (!buf)
        {
            *e = "host allocation failed";
            return CL_ERR_OOM;
        }
        std::memcpy(buf, px.data(), px.size() * sizeof(float));
        *rgba = buf;
        return CL_OK;
    });
}

cl_status cl_image_free(float* rgba)
{
    std::free(rgba);
    return CL_OK;
}

// PFM: "PF\n<w> <h>\n-1\n" (negative scale: little endian), then RGB float32
// scanlines from the bottom row up; the image rows are top to bottom.
cl_status cl_image_write_pfm(const char* path, const float* rgba, uint32_t width, uint32_t height)
{
    if (!path || !rgba || width == 0 || height == 0) return fail(CL_ERR_INVALID_ARG, "null argument or empty image");
    return guardedIo([&](std::string* e) -> cl_status {
        std::ofstream f(path, std::ios::binary);
        if (!f)
        {
            *e = std::string("cannot write ") + path;
            return CL_ERR_INVALID_ARG;
        }
        f << "PF\n" << width << " " << height << "\n-1\n";
        std::vector<float> row(size_t(width) * 3);
        for (uint32_t y = height; y-- > 0;)
        {
            for (uint32_t x = 0; x < width; ++x)
                for (int c = 0; c < 3; ++c) row[3 * size_t(x) + c] = rgba[(size_t(y) * width + x) * 4 + c];
            f.write(reinterpret_cast<const char*>(row.data()), std::streamsize(row.size() * sizeof(float)));
        }
        if (!f)
        {
            *e = std::string("write failed: ") + path;
            return CL_ERR_STATE;
        }
        return CL_OK;
    });
}

cl_status cl_image_read_pfm(const char* path, float** rgba, uint32_t* width, uint32_t* height)
{
    if (!path || !rgba || !width || !height) return fail(CL_ERR_INVALID_ARG, "null argument");
    *rgba = nullptr;
    return guardedIo([&](std::string* e) -> cl_status {
        std::vector<uint8_t> data;
        if (!readFile(path, &data))
        {
            *e = std::string("cannot open ") + path;
            return CL_ERR_INVALID_ARG;
        }
        Reader      r{data};
        std::string magic, dims, scale;
        if (!r.line(&magic) || !r.line(&dims) || !r.line(&scale) || (magic != "PF" && magic != "Pf"))
        {
            *e = "not a PFM file";
            return CL_ERR_INVALID_ARG;
        }
        const int ch = magic == "PF" ? 3 : 1;
        int       W = 0, H = 0;
        if (std::sscanf(dims.c_str(), "%d %d", &W, &H) != 2 || W <= 0 || H <= 0 || W > (1 << 16) || H > (1 << 16))
        {
            *e = "bad PFM size";
            return CL_ERR_INVALID_ARG;
        }
        const double s      = std::atof(scale.c_str());
        const bool   little = s < 0.0;
        const size_t need   = size_t(W) * H * ch * 4;
        if (data.size() - r.p < need)
        {
            *e = "PFM pixel data truncated";
            return CL_ERR_INVALID_ARG;
        }
        float* buf = static_cast<float*>(std::malloc(size_t(W) * H * 4 * sizeof(float)));
        if (!buf)
        {
            *e = "host allocation failed";
            return CL_ERR_OOM;
        }
        for (int y = 0; y < H; ++y) // file row y is image row H-1-y
            for (int x = 0; x < W; ++x)
            {
                float* o = buf + (size_t(H - 1 - y) * W + x) * 4;
                for (int c = 0; c < ch; ++c)
                {
                    uint8_t b4[4];
                    std::memcpy(b4, &data[r.p + ((size_t(y) * W + x) * ch + c) * 4], 4);
                    if (!little) std::swap(b4[0], b4[3]), std::swap(b4[1], b4[2]);
                    std::memcpy(&o[c], b4, 4);
                }
                if (ch == 1) o[1] = o[2] = o[0];
                o[3] = 1.0f;
            }
        *rgba   = buf;
        *width  = uint32_t(W);
        *height = uint32_t(H);
        return CL_OK;
    });
}

} // extern "C"
