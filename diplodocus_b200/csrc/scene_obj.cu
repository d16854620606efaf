// OBJ scene loading on the host: the reference's ObjSceneLoader, restated so a scene file reaches the engine
// with the same triangles, in the same order and with the same float bits as the reference's Scene.
//
// Replaces ObjSceneLoader::Load / LoadObj / LoadMetadata (src/io/scene/obj_scene_loader.cc:20-205) and the
// parts of its vendored tinyobjloader 2.0 (third-party/tinyobjloader/tiny_obj_loader.h) that decide which
// triangles come out:
//   * numbers: the longest decimal prefix of a token (or a nan / inf literal), string -> double -> float;
//   * faces: 1-based indices, negative ones relative to the vertices read so far; faces are triangulated when
//     the pending group is flushed (a usemtl that changes the material, g, o, end of file);
//   * a quad is split along its shorter diagonal (float32), larger polygons by ear clipping (projection plane
//     from the first corner with a cross-product component above FLT_EPSILON, ear test by the signs of the
//     edge cross product and a corner area term, point-in-triangle by crossings);
//   * MTL: Ka, Kd, Ks, Kt/Tf, Ke, Ni, Ns, d, Tr (1 - Tr unless d was given), map_Kd before Kd gives diffuse 0.6;
//     duplicate names keep the first index; of the files one mtllib line names, the first that loads.
// Each triangle gets RecomputeTriangleGeometricNormal (scene.cc:18-21), and an emissive material makes it an
// area light with CalculateTriangleSurfaceArea (triangle.h:28-34), both in float in the reference's order.
//
// Deliberate differences: an out-of-range vertex or normal index fails the load (the reference reads out of
// bounds); a .meta value must be one complete number token.
//
// Attribution: the quad split, the ear-clipping loop and its point-in-polygon test follow the rules of
// tinyobjloader (MIT licence, Copyright (c) 2012-present Syoyo Fujita and contributors), which the reference
// vendors; the point-in-polygon crossing test is W. Randolph Franklin's PNPOLY (BSD-style licence,
// Copyright (c) 1970-2003 Wm. Randolph Franklin). They are restated here so the triangles match the reference's.
#include <cctype>
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <new>
#include <set>
#include <sstream>
#include <string>
#include <thread>
#include <vector>
#include <algorithm>

#include "internal.h"

struct dipl_obj_scene {
    std::vector<float> positions;  // 9 per triangle
    std::vector<float> normals;    // 9 per triangle (0 where absent)
    std::vector<float> geom;       // 3 per triangle
    std::vector<int32_t> material_ids;
    std::vector<uint8_t> has_normals;
    struct Mat {
        std::string name;
        float v[19];  // ambient, diffuse, specular, transmittance, emission, shininess, ior, r_ior, dissolve
    };
    std::vector<Mat> materials;
    std::vector<int32_t> area_ids;
    std::vector<float> area_colors;  // 3 per light
    std::vector<float> area_areas;
    std::vector<float> point_lights;  // 7 per light
    float camera[11] = {0};           // pos, dir, up, fov, far
};

namespace dipl {
namespace {

struct LoadError {
    std::string msg;
};

[[noreturn]] void fail(const std::string& m) { throw LoadError{m}; }

// ---- tokens ---------------------------------------------------------------------------------------------------
bool is_space(char c) { return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f'; }

std::vector<std::string> split(const std::string& line) {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < line.size()) {
        while (i < line.size() && is_space(line[i])) ++i;
        size_t j = i;
        while (j < line.size() && !is_space(line[j])) ++j;
        if (j > i) out.emplace_back(line.substr(i, j - i));
        i = j;
    }
    return out;
}

bool ieq_prefix(const char* s, const char* lit) {
    for (; *lit; ++s, ++lit)
        if (std::tolower((unsigned char)*s) != *lit) return false;
    return true;
}

// A number token of an OBJ / MTL file: the longest decimal prefix ([+-] digits [. digits] | [+-] . digits, then
// an optional exponent with digits), or nan / inf; out of range fails.
float obj_number(const std::string& tok) {
    const char* s = tok.c_str();
    const char* p = s;
    if (*p == '+' || *p == '-') ++p;
    if (ieq_prefix(p, "nan")) return std::nanf("") * (s[0] == '-' ? -1.0f : 1.0f);
    if (ieq_prefix(p, "inf")) return s[0] == '-' ? -INFINITY : INFINITY;
    const char* q = p;
    bool digits = false;
    while (*q >= '0' && *q <= '9') ++q, digits = true;
    if (*q == '.') {
        ++q;
        while (*q >= '0' && *q <= '9') ++q, digits = true;
    }
    if (!digits) fail("expected number, got '" + tok + "'");
    if (*q == 'e' || *q == 'E') {
        const char* e = q + 1;
        if (*e == '+' || *e == '-') ++e;
        if (*e >= '0' && *e <= '9') {
            while (*e >= '0' && *e <= '9') ++e;
            q = e;
        }
    }
    const std::string prefix(s, q);
    errno = 0;
    const double d = std::strtod(prefix.c_str(), nullptr);  // correctly rounded
    if (std::isinf(d)) fail("number out of range: '" + tok + "'");
    return static_cast<float>(d);
}

// The same reading for a token [s, e) of a file buffer, without copies: Clinger's exact fast path (a mantissa of
// at most 2^53 times or over an exactly representable power of ten is one correctly rounded operation), else
// the general path above.
constexpr double kPow10[23] = {1e0,  1e1,  1e2,  1e3,  1e4,  1e5,  1e6,  1e7,  1e8,  1e9,  1e10, 1e11,
                               1e12, 1e13, 1e14, 1e15, 1e16, 1e17, 1e18, 1e19, 1e20, 1e21, 1e22};

bool fast_number(const char* s, const char* e, float* out) {
    const char* p = s;
    bool neg = false;
    if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
    uint64_t mant = 0;
    int sig = 0, exp10 = 0;
    bool digits = false;
    while (p < e && *p >= '0' && *p <= '9') {
        digits = true;
        if (mant || *p != '0') {
            if (++sig > 19) return false;
            mant = mant * 10 + (uint64_t)(*p - '0');
        }
        ++p;
    }
    if (p < e && *p == '.') {
        ++p;
        while (p < e && *p >= '0' && *p <= '9') {
            digits = true;
            if (mant || *p != '0') {
                if (++sig > 19) return false;
                mant = mant * 10 + (uint64_t)(*p - '0');
            }
            --exp10;
            ++p;
        }
    }
    if (!digits) return false;
    if (p < e && (*p == 'e' || *p == 'E')) {
        const char* q = p + 1;
        bool eneg = false;
        if (q < e && (*q == '+' || *q == '-')) eneg = *q++ == '-';
        if (q < e && *q >= '0' && *q <= '9') {
            int x = 0;
            while (q < e && *q >= '0' && *q <= '9') {
                if (x < 100000) x = x * 10 + (*q - '0');
                ++q;
            }
            exp10 += eneg ? -x : x;
        }
    }
    if (mant > (1ull << 53) || exp10 < -22 || exp10 > 22) return false;
    double d = (double)mant;
    d = exp10 >= 0 ? d * kPow10[exp10] : d / kPow10[-exp10];
    *out = static_cast<float>(neg ? -d : d);
    return true;
}

float number(const char* s, const char* e) {
    float f;
    if (fast_number(s, e, &f)) return f;
    return obj_number(std::string(s, e));
}

// A .meta value: exactly one decimal token.
float meta_number(const std::string& tok) {
    const char* s = tok.c_str();
    char* end = nullptr;
    const char* p = s + ((s[0] == '+' || s[0] == '-') ? 1 : 0);
    if (!((*p >= '0' && *p <= '9') || (*p == '.' && p[1] >= '0' && p[1] <= '9'))) fail("expected number '" + tok + "'");
    for (const char* c = p; *c; ++c)
        if (!((*c >= '0' && *c <= '9') || *c == '.' || *c == 'e' || *c == 'E' || *c == '+' || *c == '-'))
            fail("expected number '" + tok + "'");
    const double d = std::strtod(s, &end);
    if (end == s || *end != '\0') fail("expected number '" + tok + "'");
    return static_cast<float>(d);
}

// ---- float32 geometry in the reference's order ----------------------------------------------------------------
struct V3 {
    float x, y, z;
};
V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
float length(V3 v) { return std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z); }

V3 geom_normal(V3 p0, V3 p1, V3 p2) {
    const V3 c = cross(sub(p1, p0), sub(p2, p0));
    const float len = length(c);
    if (len <= 1e-6f) return {0.0f, 0.0f, 0.0f};
    return {c.x / len, c.y / len, c.z / len};
}

float surface_area(V3 p0, V3 p1, V3 p2) {
    const float m = length(cross(sub(p1, p0), sub(p2, p0)));
    return static_cast<float>(0.5 * m);
}

// ---- polygon triangulation --------------------------------------------------------------------------------
struct Corner {
    int v, vt, vn;
};

bool pnpoly3(const float* vx, const float* vy, float tx, float ty) {
    bool c = false;
    for (int i = 0, j = 2; i < 3; j = i++) {
        if (((vy[i] > ty) != (vy[j] > ty)) && (tx < (vx[j] - vx[i]) * (ty - vy[i]) / (vy[j] - vy[i]) + vx[i])) c = !c;
    }
    return c;
}

// Triangles (corner positions within the face) of one polygon, given the vertex positions read so far.
void triangulate(const Corner* face, int n, const float* v, long nv, std::vector<int>& out) {
    auto ok = [&](int k) { return face[k].v >= 0 && face[k].v < nv; };
    auto P = [&](int k) { return V3{v[3 * face[k].v], v[3 * face[k].v + 1], v[3 * face[k].v + 2]}; };
    if (n < 3) return;  // degenerate face: skipped
    if (n == 3) {
        out.insert(out.end(), {0, 1, 2});
        return;
    }
    if (n == 4) {
        for (int k = 0; k < 4; ++k)
            if (!ok(k)) return;  // face with an invalid vertex index: skipped
        const V3 e02 = sub(P(2), P(0)), e13 = sub(P(3), P(1));
        const float sqr02 = e02.x * e02.x + e02.y * e02.y + e02.z * e02.z;
        const float sqr13 = e13.x * e13.x + e13.y * e13.y + e13.z * e13.z;
        if (sqr02 < sqr13) out.insert(out.end(), {0, 1, 2, 0, 2, 3});
        else out.insert(out.end(), {0, 1, 3, 1, 2, 3});
        return;
    }
    int axes[2] = {1, 2};
    const float feps = 1.1920928955078125e-07f;
    for (int k = 0; k < n; ++k) {
        const int a = k % n, b = (k + 1) % n, c = (k + 2) % n;
        if (!ok(a) || !ok(b) || !ok(c)) continue;
        const V3 e0 = sub(P(b), P(a)), e1 = sub(P(c), P(b));
        const float cx = std::fabs(e0.y * e1.z - e0.z * e1.y);
        const float cy = std::fabs(e0.z * e1.x - e0.x * e1.z);
        const float cz = std::fabs(e0.x * e1.y - e0.y * e1.x);
        if (cx > feps || cy > feps || cz > feps) {
            if (!(cx > cy && cx > cz)) {
                axes[0] = 0;
                if (cz > cx && cz > cy) axes[1] = 1;
            }
            break;
        }
    }
    auto proj = [&](int k, float& x, float& y) {
        if (!ok(k)) {
            x = y = 0.0f;
            return;
        }
        const float* p = &v[3 * face[k].v];
        x = p[axes[0]];
        y = p[axes[1]];
    };
    std::vector<int> rem(n);
    for (int k = 0; k < n; ++k) rem[k] = k;
    int guess = 0, iterations = n, previous = n;
    while ((int)rem.size() > 3 && iterations > 0) {
        const int m = (int)rem.size();
        if (guess >= m) guess -= m;
        if (previous != m) {
            previous = m;
            iterations = m;
        } else {
            --iterations;
        }
        int ind[3];
        float vx[3], vy[3];
        for (int k = 0; k < 3; ++k) {
            ind[k] = rem[(guess + k) % m];
            proj(ind[k], vx[k], vy[k]);
        }
        const float e0x = vx[1] - vx[0], e0y = vy[1] - vy[0];
        const float e1x = vx[2] - vx[1], e1y = vy[2] - vy[1];
        const float cr = e0x * e1y - e0y * e1x;
        const float area = (vx[0] * vy[1] - vy[0] * vx[1]) * 0.5f;
        if (cr * area < 0.0f) {
            guess += 1;
            continue;
        }
        bool overlap = false;
        for (int other = 3; other < m; ++other) {
            const int k = rem[(guess + other) % m];
            if (!ok(k)) continue;
            float tx, ty;
            proj(k, tx, ty);
            if (pnpoly3(vx, vy, tx, ty)) {
                overlap = true;
                break;
            }
        }
        if (overlap) {
            guess += 1;
            continue;
        }
        out.insert(out.end(), {ind[0], ind[1], ind[2]});
        rem.erase(rem.begin() + (guess + 1) % m);
    }
    if ((int)rem.size() == 3) out.insert(out.end(), {rem[0], rem[1], rem[2]});
}

// ---- MTL ---------------------------------------------------------------------------------------------------
struct MtlState {
    dipl_obj_scene::Mat m;
    bool has_d = false, has_kd = false;
};

void init_mat(MtlState& s) {
    s = MtlState{};
    for (float& x : s.m.v) x = 0.0f;
    s.m.v[15] = 1.0f;  // shininess
    s.m.v[16] = 1.0f;  // ior
    s.m.v[18] = 1.0f;  // dissolve
}

bool load_mtl(const std::string& path, std::vector<dipl_obj_scene::Mat>& mats, std::map<std::string, int>& map) {
    std::ifstream in(path);
    if (!in) return false;
    MtlState cur;
    init_mat(cur);
    auto flush = [&]() {
        if (!cur.m.name.empty()) {
            map.insert({cur.m.name, (int)mats.size()});
            mats.push_back(cur.m);
        }
    };
    auto rgb = [&](const std::vector<std::string>& t, int at) {
        for (int i = 0; i < 3; ++i) cur.m.v[at + i] = (size_t)(i + 1) < t.size() ? obj_number(t[i + 1]) : 0.0f;
    };
    auto one = [&](const std::vector<std::string>& t) { return t.size() > 1 ? obj_number(t[1]) : 0.0f; };
    std::string line;
    try {
        while (std::getline(in, line)) {
            if (line.size() >= 3 && (unsigned char)line[0] == 0xEF && (unsigned char)line[1] == 0xBB &&
                (unsigned char)line[2] == 0xBF)
                line = line.substr(3);
            const std::vector<std::string> t = split(line);
            if (t.empty() || t[0][0] == '#') continue;
            const std::string& k = t[0];
            if (k == "newmtl") {
                flush();
                init_mat(cur);
                cur.m.name = t.size() > 1 ? t[1] : "";
            } else if (k == "Ka") {
                rgb(t, 0);
            } else if (k == "Kd") {
                rgb(t, 3);
                cur.has_kd = true;
            } else if (k == "Ks") {
                rgb(t, 6);
            } else if (k == "Kt" || k == "Tf") {
                rgb(t, 9);
            } else if (k == "Ke") {
                rgb(t, 12);
            } else if (k == "Ns") {
                cur.m.v[15] = one(t);
            } else if (k == "Ni") {
                cur.m.v[16] = one(t);
            } else if (k == "d") {
                cur.m.v[18] = one(t);
                cur.has_d = true;
            } else if (k == "Tr") {
                if (!cur.has_d) cur.m.v[18] = 1.0f - one(t);
            } else if (k == "map_Kd") {
                if (!cur.has_kd) cur.m.v[3] = cur.m.v[4] = cur.m.v[5] = 0.6f;
            }
        }
    } catch (const LoadError&) {
        return false;  // materials completed before the error stay
    }
    flush();
    return true;
}

// ---- OBJ: chunks of lines parsed in parallel, then merged in file order -------------------------------------
struct FaceRec {
    uint32_t first, count;        // corners [first, first + count) of the chunk's corner array
    uint32_t nv, nvt, nvn;        // vertices / texcoords / normals of the chunk before this line
};
struct EventRec {
    size_t order;                 // faces of the chunk before this event
    uint32_t nv;                  // vertices of the chunk before this event
    std::vector<std::string> tok; // the line's tokens
};
struct Chunk {
    std::vector<float> v, vn;
    uint32_t nvt = 0;
    std::vector<int64_t> corners;  // raw v, vt, vn indices per corner (0 = absent)
    std::vector<FaceRec> faces;
    std::vector<EventRec> events;
    std::string error;
};

const char* skip_ws(const char* p, const char* e) {
    while (p < e && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f')) ++p;
    return p;
}
const char* token_end(const char* p, const char* e) {
    while (p < e && !(*p == ' ' || *p == '\t' || *p == '\r' || *p == '\v' || *p == '\f')) ++p;
    return p;
}

int64_t parse_int(const char* s, const char* e) {
    const char* p = s;
    bool neg = false;
    if (p < e && (*p == '+' || *p == '-')) neg = *p++ == '-';
    if (p >= e || *p < '0' || *p > '9') fail("bad index '" + std::string(s, e) + "'");
    int64_t x = 0;
    while (p < e && *p >= '0' && *p <= '9') {
        if (x < (int64_t)1 << 40) x = x * 10 + (*p - '0');
        ++p;
    }
    if (x == 0) fail("zero index");
    return neg ? -x : x;
}

void parse_chunk(const char* b, const char* e, Chunk& c) {
    try {
        while (b < e) {
            const char* nl = static_cast<const char*>(std::memchr(b, '\n', (size_t)(e - b)));
            const char* le = nl ? nl : e;
            const char* hash = static_cast<const char*>(std::memchr(b, '#', (size_t)(le - b)));
            const char* end = hash ? hash : le;
            const char* p = skip_ws(b, end);
            b = nl ? nl + 1 : e;
            if (p >= end) continue;
            const char* ke = token_end(p, end);
            const size_t kl = (size_t)(ke - p);
            if (kl == 1 && *p == 'v') {
                const char* q = ke;
                for (int i = 0; i < 3; ++i) {
                    q = skip_ws(q, end);
                    const char* te = token_end(q, end);
                    c.v.push_back(q < te ? number(q, te) : 0.0f);
                    q = te;
                }
            } else if (kl == 2 && p[0] == 'v' && p[1] == 'n') {
                const char* q = ke;
                for (int i = 0; i < 3; ++i) {
                    q = skip_ws(q, end);
                    const char* te = token_end(q, end);
                    c.vn.push_back(q < te ? number(q, te) : 0.0f);
                    q = te;
                }
            } else if (kl == 2 && p[0] == 'v' && p[1] == 't') {
                ++c.nvt;
            } else if (kl == 1 && *p == 'f') {
                FaceRec f{(uint32_t)(c.corners.size() / 3), 0, (uint32_t)(c.v.size() / 3), c.nvt,
                          (uint32_t)(c.vn.size() / 3)};
                const char* q = skip_ws(ke, end);
                while (q < end) {
                    const char* te = token_end(q, end);
                    const char* s1 = static_cast<const char*>(std::memchr(q, '/', (size_t)(te - q)));
                    int64_t vi = parse_int(q, s1 ? s1 : te), ti = 0, ni = 0;
                    if (s1) {
                        const char* s2 = static_cast<const char*>(std::memchr(s1 + 1, '/', (size_t)(te - s1 - 1)));
                        const char* t_end = s2 ? s2 : te;
                        if (t_end > s1 + 1) ti = parse_int(s1 + 1, t_end);
                        if (s2 && s2 + 1 < te) ni = parse_int(s2 + 1, te);
                    }
                    c.corners.insert(c.corners.end(), {vi, ti, ni});
                    ++f.count;
                    q = skip_ws(te, end);
                }
                c.faces.push_back(f);
            } else if ((kl == 6 && (std::memcmp(p, "usemtl", 6) == 0 || std::memcmp(p, "mtllib", 6) == 0)) ||
                       (kl == 1 && (*p == 'g' || *p == 'o'))) {
                EventRec ev{c.faces.size(), (uint32_t)(c.v.size() / 3), split(std::string(p, end))};
                c.events.push_back(std::move(ev));
            }
        }
    } catch (const LoadError& err) {
        c.error = err.msg;
    }
}

int resolve(int64_t raw, int64_t count) {
    if (raw > 0) return (int)(raw - 1);
    if (raw < 0) return (int)(count + raw);
    return -1;  // absent
}

void load_obj(const std::string& path, dipl_obj_scene& sc) {
    std::FILE* fp = std::fopen(path.c_str(), "rb");
    if (!fp) fail("cannot read " + path);
    std::string buf;
    std::fseek(fp, 0, SEEK_END);
    const long size = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    buf.resize(size > 0 ? (size_t)size : 0);
    const size_t got = buf.empty() ? 0 : std::fread(&buf[0], 1, buf.size(), fp);
    std::fclose(fp);
    if (got != buf.size()) fail("cannot read " + path);
    const size_t slash = path.find_last_of('/');
    const std::string base = slash == std::string::npos ? std::string(".") : path.substr(0, slash);

    // chunks at line starts; one per hardware thread, at least 4 MB each
    const size_t want = std::max<size_t>(1, std::min<size_t>(std::max(1u, std::thread::hardware_concurrency()),
                                                                buf.size() / (4u << 20) + 1));
    std::vector<size_t> cut{0};
    for (size_t k = 1; k < want; ++k) {
        size_t at = buf.size() * k / want;
        const void* nl = std::memchr(buf.data() + at, '\n', buf.size() - at);
        at = nl ? (size_t)(static_cast<const char*>(nl) - buf.data()) + 1 : buf.size();
        if (at > cut.back()) cut.push_back(at);
    }
    cut.push_back(buf.size());
    const size_t nc = cut.size() - 1;
    std::vector<Chunk> chunks(nc);
    {
        std::vector<std::thread> th;
        for (size_t k = 1; k < nc; ++k)
            th.emplace_back(parse_chunk, buf.data() + cut[k], buf.data() + cut[k + 1], std::ref(chunks[k]));
        parse_chunk(buf.data() + cut[0], buf.data() + cut[1], chunks[0]);
        for (auto& t : th) t.join();
    }
    for (const Chunk& c : chunks)
        if (!c.error.empty()) fail(c.error);

    // all positions and normals, in file order
    std::vector<float> v, vn;
    std::vector<uint32_t> v0(nc), vt0(nc), vn0(nc);
    uint32_t tv = 0, tvt = 0, tvn = 0;
    for (size_t k = 0; k < nc; ++k) {
        v0[k] = tv, vt0[k] = tvt, vn0[k] = tvn;
        tv += (uint32_t)(chunks[k].v.size() / 3), tvt += chunks[k].nvt, tvn += (uint32_t)(chunks[k].vn.size() / 3);
    }
    v.reserve(3 * (size_t)tv);
    vn.reserve(3 * (size_t)tvn);
    for (const Chunk& c : chunks) {
        v.insert(v.end(), c.v.begin(), c.v.end());
        vn.insert(vn.end(), c.vn.begin(), c.vn.end());
    }

    // faces and events in file order: materials, flush points, triangulation
    std::map<std::string, int> material_map;
    std::set<std::string> loaded;
    int material = -1;
    struct Pending {
        size_t chunk, face;
        int mat;
    };
    std::vector<Pending> pending;
    struct OutTri {
        Corner c[3];
        int mat;
    };
    std::vector<OutTri> tris;
    std::vector<int> idx;
    std::vector<Corner> face;
    auto flush = [&](long nv_now) {
        for (const Pending& pf : pending) {
            const Chunk& c = chunks[pf.chunk];
            const FaceRec& f = c.faces[pf.face];
            face.clear();
            for (uint32_t j = 0; j < f.count; ++j) {
                const int64_t* r = &c.corners[3 * ((size_t)f.first + j)];
                face.push_back({resolve(r[0], (int64_t)v0[pf.chunk] + f.nv),
                                resolve(r[1], (int64_t)vt0[pf.chunk] + f.nvt),
                                resolve(r[2], (int64_t)vn0[pf.chunk] + f.nvn)});
            }
            idx.clear();
            triangulate(face.data(), (int)face.size(), v.data(), nv_now, idx);
            for (size_t k = 0; k + 2 < idx.size(); k += 3)
                tris.push_back({{face[idx[k]], face[idx[k + 1]], face[idx[k + 2]]}, pf.mat});
        }
        pending.clear();
    };
    for (size_t k = 0; k < nc; ++k) {
        const Chunk& c = chunks[k];
        size_t fi = 0;
        for (const EventRec& ev : c.events) {
            for (; fi < ev.order; ++fi) pending.push_back({k, fi, material});
            const long nv_now = (long)v0[k] + ev.nv;
            const std::string& key = ev.tok[0];
            if (key == "usemtl") {
                const std::string name = ev.tok.size() > 1 ? ev.tok[1] : "";
                auto it = material_map.find(name);
                const int id = it == material_map.end() ? -1 : it->second;
                if (id != material) {
                    flush(nv_now);
                    material = id;
                }
            } else if (key == "mtllib") {
                for (size_t i = 1; i < ev.tok.size(); ++i) {
                    if (loaded.count(ev.tok[i])) continue;
                    if (load_mtl(base + "/" + ev.tok[i], sc.materials, material_map)) {
                        loaded.insert(ev.tok[i]);
                        break;
                    }
                }
            } else {
                flush(nv_now);  // g, o
            }
        }
        for (; fi < c.faces.size(); ++fi) pending.push_back({k, fi, material});
    }
    flush((long)tv);
    chunks.clear();

    const long nv = (long)tv, nn = (long)tvn;
    const size_t n = tris.size();
    sc.positions.assign(9 * n, 0.0f);
    sc.normals.assign(9 * n, 0.0f);
    sc.geom.assign(3 * n, 0.0f);
    sc.material_ids.assign(n, -1);
    sc.has_normals.assign(n, 0);
    for (size_t i = 0; i < n; ++i) {
        const OutTri& tr = tris[i];
        V3 p[3];
        for (int k = 0; k < 3; ++k) {
            const int vi = tr.c[k].v;
            if (vi < 0 || vi >= nv) fail("vertex index out of range");
            p[k] = {v[3 * (size_t)vi], v[3 * (size_t)vi + 1], v[3 * (size_t)vi + 2]};
            sc.positions[9 * i + 3 * k + 0] = p[k].x;
            sc.positions[9 * i + 3 * k + 1] = p[k].y;
            sc.positions[9 * i + 3 * k + 2] = p[k].z;
        }
        if (tr.c[0].vn >= 0 && tr.c[1].vn >= 0 && tr.c[2].vn >= 0) {
            for (int k = 0; k < 3; ++k) {
                const int ni = tr.c[k].vn;
                if (ni >= nn) fail("normal index out of range");
                for (int j = 0; j < 3; ++j) sc.normals[9 * i + 3 * k + j] = vn[3 * (size_t)ni + j];
            }
            sc.has_normals[i] = 1;
        }
        const V3 g = geom_normal(p[0], p[1], p[2]);
        sc.geom[3 * i + 0] = g.x;
        sc.geom[3 * i + 1] = g.y;
        sc.geom[3 * i + 2] = g.z;
        sc.material_ids[i] = tr.mat;
        if (tr.mat >= 0) {
            const float* em = &sc.materials[tr.mat].v[12];
            if (em[0] != 0.0f || em[1] != 0.0f || em[2] != 0.0f) {
                sc.area_ids.push_back((int32_t)i);
                sc.area_colors.insert(sc.area_colors.end(), {em[0], em[1], em[2]});
                sc.area_areas.push_back(surface_area(p[0], p[1], p[2]));
            }
        }
    }
    for (auto& m : sc.materials) m.v[17] = 1.0f / m.v[16];  // r_ior
}

void load_meta(const std::string& path, dipl_obj_scene& sc) {
    std::ifstream in(path);
    if (!in) fail("cannot read " + path);
    std::stringstream ss;
    ss << in.rdbuf();
    const std::vector<std::string> t = split(ss.str());
    size_t i = 0;
    auto take = [&](float* dst, int k) {
        if (i + k > t.size()) fail("missing metadata value");
        for (int j = 0; j < k; ++j) dst[j] = meta_number(t[i + j]);
        i += k;
    };
    while (i < t.size()) {
        const std::string tok = t[i++];
        if (tok == "cam_pos") take(sc.camera + 0, 3);
        else if (tok == "cam_dir") take(sc.camera + 3, 3);
        else if (tok == "cam_up") take(sc.camera + 6, 3);
        else if (tok == "cam_fov") take(sc.camera + 9, 1);
        else if (tok == "cam_far") take(sc.camera + 10, 1);
        else if (tok == "point_light") {
            float pl[7];
            take(pl, 7);
            sc.point_lights.insert(sc.point_lights.end(), pl, pl + 7);
        } else {
            fail("unrecognized metadata token '" + tok + "'");
        }
    }
}

}  // namespace
}  // namespace dipl

using namespace dipl;

extern "C" dipl_status dipl_obj_scene_load(const char* dirpath, const char* name, dipl_obj_scene** out) {
    DIPL_CHECK_ARG(dirpath && name && out, "dirpath, name and out must be non-NULL");
    *out = nullptr;
    auto* sc = new (std::nothrow) dipl_obj_scene();
    if (!sc) return DIPL_ERR_OUT_OF_MEMORY;
    const std::string base = std::string(dirpath) + "/" + name;
    try {
        load_meta(base + ".meta", *sc);  // the reference reads the metadata first (obj_scene_loader.cc:200-201)
        load_obj(base + ".obj", *sc);
    } catch (const LoadError& e) {
        delete sc;
        set_last_error("dipl_obj_scene_load: " + e.msg);
        return DIPL_ERR_IO;
    } catch (const std::bad_alloc&) {
        delete sc;
        return DIPL_ERR_OUT_OF_MEMORY;
    }
    *out = sc;
    return DIPL_OK;
}

extern "C" dipl_status dipl_obj_scene_get_info(const dipl_obj_scene* sc, dipl_obj_scene_info* info) {
    DIPL_CHECK_ARG(sc && info, "scene and info must be non-NULL");
    info->num_triangles = (int64_t)sc->material_ids.size();
    info->num_materials = (int64_t)sc->materials.size();
    info->num_area_lights = (int64_t)sc->area_ids.size();
    info->num_point_lights = (int64_t)(sc->point_lights.size() / 7);
    std::memcpy(info->camera, sc->camera, sizeof(sc->camera));
    return DIPL_OK;
}

extern "C" dipl_status dipl_obj_scene_get_triangles(const dipl_obj_scene* sc, float* positions, float* normals,
                                                    float* geom_normals, int32_t* material_ids,
                                                    uint8_t* has_vertex_normals) {
    DIPL_CHECK_ARG(sc, "scene must be non-NULL");
    const size_t n = sc->material_ids.size();
    if (positions) std::memcpy(positions, sc->positions.data(), 9 * n * sizeof(float));
    if (normals) std::memcpy(normals, sc->normals.data(), 9 * n * sizeof(float));
    if (geom_normals) std::memcpy(geom_normals, sc->geom.data(), 3 * n * sizeof(float));
    if (material_ids) std::memcpy(material_ids, sc->material_ids.data(), n * sizeof(int32_t));
    if (has_vertex_normals) std::memcpy(has_vertex_normals, sc->has_normals.data(), n);
    return DIPL_OK;
}

extern "C" dipl_status dipl_obj_scene_get_soa(const dipl_obj_scene* sc, float* v0, float* v1, float* v2) {
    DIPL_CHECK_ARG(sc && v0 && v1 && v2, "scene and v0/v1/v2 must be non-NULL");
    const size_t n = sc->material_ids.size();
    float* dst[3] = {v0, v1, v2};
    for (size_t i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) std::memcpy(dst[k] + 3 * i, &sc->positions[9 * i + 3 * k], 3 * sizeof(float));
    return DIPL_OK;
}

extern "C" dipl_status dipl_obj_scene_get_materials(const dipl_obj_scene* sc, float* values, char* names) {
    DIPL_CHECK_ARG(sc, "scene must be non-NULL");
    for (size_t i = 0; i < sc->materials.size(); ++i) {
        if (values) std::memcpy(values + 19 * i, sc->materials[i].v, 19 * sizeof(float));
        if (names) {
            std::memset(names + 64 * i, 0, 64);
            std::strncpy(names + 64 * i, sc->materials[i].name.c_str(), 63);
        }
    }
    return DIPL_OK;
}

extern "C" dipl_status dipl_obj_scene_get_lights(const dipl_obj_scene* sc, int32_t* area_triangle_ids,
                                                 float* area_colors, float* area_surface_areas,
                                                 float* point_lights) {
    DIPL_CHECK_ARG(sc, "scene must be non-NULL");
    const size_t na = sc->area_ids.size();
    if (area_triangle_ids) std::memcpy(area_triangle_ids, sc->area_ids.data(), na * sizeof(int32_t));
    if (area_colors) std::memcpy(area_colors, sc->area_colors.data(), 3 * na * sizeof(float));
    if (area_surface_areas) std::memcpy(area_surface_areas, sc->area_areas.data(), na * sizeof(float));
    if (point_lights) std::memcpy(point_lights, sc->point_lights.data(), sc->point_lights.size() * sizeof(float));
    return DIPL_OK;
}

extern "C" void dipl_obj_scene_destroy(dipl_obj_scene* sc) { delete sc; }
