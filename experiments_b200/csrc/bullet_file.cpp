// .bullet scene files: btBulletDataExtractor::convertAllObjects
// (P2/BulletDataExtractor.cpp:456-721) over this library's own reader of the
// format that bullet2's btDefaultSerializer writes (LinearMath/btSerializer.h)
// and bParse's btBulletFile reads (BulletSerialize/BulletFileLoader).
//
// The format: a 12-byte header ("BULLET", 'f' or 'd' precision, '-' for
// 8-byte or '_' for 4-byte pointers, 'v' little or 'V' big endian, a
// version), then chunks of {code, length, old pointer, struct index, count}
// followed by their bytes. Pointers inside a chunk are the old pointers of
// other chunks. The "DNA1" chunk is the struct catalogue: names, type names,
// type sizes and, per struct, its (type, name) fields in order, from which
// the field offsets follow. Fields are found by name, as bParse does, so a
// file need not match this build's structs byte for byte.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "b3_internal.h"
#include "b3_world.h"
#include "hull.h"

namespace {

struct Field {
    int type;     // type index
    std::string name;
    int offset;
    int size;     // bytes of the whole field (arrays included)
    bool pointer;
};

struct Catalog {
    std::vector<std::string> types;
    std::vector<int> typeSize;
    std::vector<int> structType;  // per struct: its type index
    std::vector<std::vector<Field>> fields;
    std::map<int, int> structOfType;
    int ptrSize = 8;
};

struct Chunk {
    uint32_t code;
    const unsigned char* data;
    int length;
    uint64_t oldPtr;
    int dna;
    int count;
};

std::string base_name(const std::string& n) {
    // "*m_ptr", "m_floats[4]", "(*m_fn)()" -> "m_ptr", "m_floats", "m_fn"
    std::string s;
    for (char ch : n) {
        if (ch == '[') break;
        if (ch != '*' && ch != '(' && ch != ')') s += ch;
    }
    return s;
}

int array_len(const std::string& n) {
    int len = 1;
    for (size_t i = 0; i < n.size(); ++i)
        if (n[i] == '[') len *= std::atoi(n.c_str() + i + 1);
    return len;
}

bool parse_dna(const unsigned char* d, int len, int ptrSize, Catalog& C, std::string& err) {
    int p = 0;
    auto need = [&](int n) { return p + n <= len; };
    auto tag = [&](const char* t) {
        if (!need(4) || std::memcmp(d + p, t, 4) != 0) return false;
        p += 4;
        return true;
    };
    auto i32 = [&]() {
        int v;
        std::memcpy(&v, d + p, 4);
        p += 4;
        return v;
    };
    auto i16 = [&]() {
        short v;
        std::memcpy(&v, d + p, 2);
        p += 2;
        return (int)v;
    };
    auto align4 = [&]() { p = (p + 3) & ~3; };
    auto strings = [&](std::vector<std::string>& out) {
        if (!need(4)) return false;
        const int n = i32();
        for (int i = 0; i < n; ++i) {
            const int s = p;
            while (p < len && d[p]) ++p;
            if (p >= len) return false;
            out.emplace_back((const char*)d + s, p - s);
            ++p;
        }
        align4();
        return true;
    };
    std::vector<std::string> names;
    if (!tag("SDNA") || !tag("NAME") || !strings(names) || !tag("TYPE") || !strings(C.types)) {
        err = "malformed DNA1 names or types";
        return false;
    }
    if (!tag("TLEN") || !need(2 * (int)C.types.size())) {
        err = "malformed DNA1 type sizes";
        return false;
    }
    for (size_t i = 0; i < C.types.size(); ++i) C.typeSize.push_back(i16());
    align4();
    if (!tag("STRC") || !need(4)) {
        err = "malformed DNA1 structs";
        return false;
    }
    const int ns = i32();
    for (int s = 0; s < ns; ++s) {
        if (!need(4)) {
            err = "truncated DNA1 struct list";
            return false;
        }
        const int t = i16(), nf = i16();
        if (t < 0 || t >= (int)C.types.size() || !need(4 * nf)) {
            err = "malformed DNA1 struct";
            return false;
        }
        std::vector<Field> fs;
        int off = 0;
        for (int f = 0; f < nf; ++f) {
            const int ft = i16(), fn = i16();
            if (ft < 0 || ft >= (int)C.types.size() || fn < 0 || fn >= (int)names.size()) {
                err = "malformed DNA1 field";
                return false;
            }
            Field F;
            F.type = ft;
            F.name = names[fn];
            F.pointer = F.name[0] == '*' || F.name[0] == '(';
            F.offset = off;
            F.size = (F.pointer ? ptrSize : C.typeSize[ft]) * array_len(F.name);
            off += F.size;
            fs.push_back(F);
        }
        C.structType.push_back(t);
        C.structOfType[t] = s;
        C.fields.push_back(fs);
    }
    return true;
}

// Byte offset of a dotted field path inside struct s (-1 when absent), and
// the field's record.
int field_offset(const Catalog& C, int s, const std::string& path, Field* out) {
    int off = 0;
    size_t at = 0;
    while (true) {
        const size_t dot = path.find('.', at);
        const std::string part = path.substr(at, dot == std::string::npos ? std::string::npos : dot - at);
        const Field* hit = nullptr;
        for (const Field& f : C.fields[s])
            if (base_name(f.name) == part) {
                hit = &f;
                break;
            }
        if (!hit) return -1;
        off += hit->offset;
        if (dot == std::string::npos) {
            if (out) *out = *hit;
            return off;
        }
        auto it = C.structOfType.find(hit->type);
        if (it == C.structOfType.end() || hit->pointer) return -1;
        s = it->second;
        at = dot + 1;
    }
}

struct File {
    std::vector<unsigned char> bytes;
    Catalog cat;
    std::vector<Chunk> chunks;
    std::map<uint64_t, size_t> byPtr;

    const Chunk* chunk_at(uint64_t ptr) const {
        auto it = byPtr.find(ptr);
        return it == byPtr.end() ? nullptr : &chunks[it->second];
    }
    bool has(const Chunk& c, const char* path) const { return field_offset(cat, c.dna, path, nullptr) >= 0; }
    float f32(const Chunk& c, const char* path, int k = 0) const {
        Field f;
        const int o = field_offset(cat, c.dna, path, &f);
        float v = 0.f;
        if (o >= 0 && o + 4 * (k + 1) <= c.length) std::memcpy(&v, c.data + o + 4 * k, 4);
        return v;
    }
    int i32(const Chunk& c, const char* path) const {
        const int o = field_offset(cat, c.dna, path, nullptr);
        int v = 0;
        if (o >= 0 && o + 4 <= c.length) std::memcpy(&v, c.data + o, 4);
        return v;
    }
    uint64_t ptr(const Chunk& c, const char* path) const {
        const int o = field_offset(cat, c.dna, path, nullptr);
        uint64_t v = 0;
        if (o >= 0 && o + cat.ptrSize <= c.length) std::memcpy(&v, c.data + o, cat.ptrSize);
        return v;
    }
};

uint32_t code4(const char* s) { return (uint32_t)s[0] | (uint32_t)s[1] << 8 | (uint32_t)s[2] << 16 | (uint32_t)s[3] << 24; }

bool read_file(const char* path, File& F, std::string& err) {
    FILE* fp = std::fopen(path, "rb");
    if (!fp) {
        err = std::string("cannot open ") + path;
        return false;
    }
    std::fseek(fp, 0, SEEK_END);
    const long n = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    F.bytes.resize(n > 0 ? (size_t)n : 0);
    const size_t got = n > 0 ? std::fread(F.bytes.data(), 1, (size_t)n, fp) : 0;
    std::fclose(fp);
    if ((long)got != n || n < 12 || std::memcmp(F.bytes.data(), "BULLET", 6) != 0) {
        err = "not a .bullet file";
        return false;
    }
    const unsigned char* h = F.bytes.data();
    if (h[6] != 'f') {
        err = "double-precision .bullet files are not supported (as in the reference demo)";
        return false;
    }
    if (h[8] != 'v') {
        err = "big-endian .bullet files are not supported";
        return false;
    }
    F.cat.ptrSize = h[7] == '-' ? 8 : 4;
    const int hdr = 16 + F.cat.ptrSize;  // code, length, old pointer, struct index, count
    size_t p = 12;
    const Chunk* dna = nullptr;
    while (p + hdr <= F.bytes.size()) {
        Chunk c;
        int len;
        std::memcpy(&c.code, h + p, 4);
        std::memcpy(&len, h + p + 4, 4);
        c.oldPtr = 0;
        std::memcpy(&c.oldPtr, h + p + 8, F.cat.ptrSize);
        std::memcpy(&c.dna, h + p + 8 + F.cat.ptrSize, 4);
        std::memcpy(&c.count, h + p + 12 + F.cat.ptrSize, 4);
        if (c.code == code4("ENDB")) break;
        if (len < 0 || p + hdr + (size_t)len > F.bytes.size()) {
            err = "truncated chunk";
            return false;
        }
        c.length = len;
        c.data = h + p + hdr;
        F.chunks.push_back(c);
        p += hdr + (size_t)len;
    }
    for (size_t i = 0; i < F.chunks.size(); ++i) {
        F.byPtr[F.chunks[i].oldPtr] = i;
        if (F.chunks[i].code == code4("DNA1")) dna = &F.chunks[i];
    }
    if (!dna) {
        err = "no DNA1 chunk";
        return false;
    }
    if (!parse_dna(dna->data, dna->length, F.cat.ptrSize, F.cat, err)) return false;
    for (const Chunk& c : F.chunks)
        if (c.code != code4("DNA1") && (c.dna < 0 || c.dna >= (int)F.cat.fields.size())) {
            err = "chunk with an unknown struct";
            return false;
        }
    return true;
}

// btMatrix3x3::getRotation (bullet2/LinearMath/btMatrix3x3.h:395-460), the
// published trace method: rows r of the basis, quaternion (x, y, z, w)
void basis_to_quat(const double r[3][3], float q[4]) {
    const double tr = r[0][0] + r[1][1] + r[2][2];
    double x, y, z, w;
    if (tr > 0.0) {
        const double s = std::sqrt(tr + 1.0);
        w = 0.5 * s;
        const double t = 0.5 / s;
        x = (r[2][1] - r[1][2]) * t;
        y = (r[0][2] - r[2][0]) * t;
        z = (r[1][0] - r[0][1]) * t;
    } else {
        int i = r[0][0] < r[1][1] ? (r[1][1] < r[2][2] ? 2 : 1) : (r[0][0] < r[2][2] ? 2 : 0);
        const int j = (i + 1) % 3, k = (i + 2) % 3;
        const double s = std::sqrt(r[i][i] - r[j][j] - r[k][k] + 1.0);
        double v[3];
        v[i] = 0.5 * s;
        const double t = 0.5 / s;
        w = (r[k][j] - r[j][k]) * t;
        v[j] = (r[j][i] + r[i][j]) * t;
        v[k] = (r[k][i] + r[i][k]) * t;
        x = v[0];
        y = v[1];
        z = v[2];
    }
    q[0] = (float)x;
    q[1] = (float)y;
    q[2] = (float)z;
    q[3] = (float)w;
}

// shape types of the reference's broadphase proxy enum
// (P2/BulletDataExtractor.cpp:529-577)
constexpr int kBoxShape = 0;
constexpr int kConvexHullShape = 4;
constexpr int kSphereShape = 8;
constexpr int kStaticPlaneShape = 28;
// most points a convex hull record of a file may hold
constexpr int64_t kMaxFileHullPoints = 1 << 16;

// A shape or body of the file, read and checked before anything registers.
struct ShapeRec {
    uint64_t oldPtr;
    int kind = 0;               // 0 convex hull, 1 sphere, 2 static plane
    std::vector<float> points;  // hull: xyz triples, final scale applied
    float radius = 0.f;         // sphere
    float plane[4] = {};        // static plane: normal, constant
};
struct BodyRec {
    int shape;  // index into the shape records
    float mass, pos[3], quat[4];
};

}  // namespace

extern "C" int b3_load_bullet_file(b3World w, const char* path, int keepStaticObjects, int* numBodiesOut) {
    return b3_load_bullet_file_ex(w, path, keepStaticObjects ? B3_BULLET_KEEP_STATIC_OBJECTS : 0, numBodiesOut);
}

extern "C" int b3_load_bullet_file_ex(b3World w, const char* path, int flags, int* numBodiesOut) {
    if (!w || !path) return B3_ERR_INVALID_ARG;
    if (flags & ~(B3_BULLET_KEEP_STATIC_OBJECTS | B3_BULLET_SPHERES_AND_PLANES)) return B3_ERR_INVALID_ARG;
    const bool keepStaticObjects = (flags & B3_BULLET_KEEP_STATIC_OBJECTS) != 0;
    const bool spheresPlanes = (flags & B3_BULLET_SPHERES_AND_PLANES) != 0;
    File F;
    std::string err;
    if (!read_file(path, F, err)) {
        b3_set_error("%s: %s", path, err.c_str());
        return B3_ERR_INVALID_ARG;
    }
    // Pass 1 reads and checks every record; nothing is registered unless
    // the whole file is usable, so a failed load leaves the world as it was.
    // Shapes in file order (convertCollisionShape :723-840): boxes and
    // convex hulls; spheres, planes and the rest are skipped, as there
    // (createSphereShape and createPlaneShape return -1, :999-1010), unless
    // B3_BULLET_SPHERES_AND_PLANES asks for this library's sphere and plane
    // shapes.
    std::vector<ShapeRec> shapes;
    for (const Chunk& c : F.chunks) {
        if (c.code != code4("SHAP")) continue;
        // a convex hull's record nests the convex-internal part
        const bool hull = F.has(c, "m_convexInternalShapeData");
        const std::string in = hull ? "m_convexInternalShapeData." : "";
        const int stype = F.i32(c, (in + "m_collisionShapeData.m_shapeType").c_str());
        float scale[3];
        for (int k = 0; k < 3; ++k) scale[k] = F.f32(c, (in + "m_localScaling.m_floats").c_str(), k);
        ShapeRec r;
        r.oldPtr = c.oldPtr;
        if (spheresPlanes && stype == kSphereShape && !hull) {
            // btSphereShape: radius = implicitShapeDimensions.x * localScaling.x
            if (!F.has(c, "m_implicitShapeDimensions")) continue;
            r.kind = 1;
            r.radius = F.f32(c, "m_implicitShapeDimensions.m_floats", 0) * scale[0];
            if (!(r.radius > 0.f) || !std::isfinite(r.radius)) {
                b3_set_error("%s: sphere of radius %g", path, (double)r.radius);
                return B3_ERR_INVALID_ARG;
            }
            shapes.push_back(std::move(r));
            continue;
        }
        if (spheresPlanes && stype == kStaticPlaneShape && !hull) {
            // btStaticPlaneShape: the plane n . x = constant (its local
            // scaling changes only its bounding box)
            if (!F.has(c, "m_planeNormal") || !F.has(c, "m_planeConstant")) continue;
            r.kind = 2;
            for (int k = 0; k < 3; ++k) r.plane[k] = F.f32(c, "m_planeNormal.m_floats", k);
            r.plane[3] = F.f32(c, "m_planeConstant");
            const float len2 = r.plane[0] * r.plane[0] + r.plane[1] * r.plane[1] + r.plane[2] * r.plane[2];
            if (!(len2 > 0.f) || !std::isfinite(len2) || !std::isfinite(r.plane[3])) {
                b3_set_error("%s: static plane without a normal", path);
                return B3_ERR_INVALID_ARG;
            }
            shapes.push_back(std::move(r));
            continue;
        }
        if (stype == kBoxShape && !hull) {
            // createBoxShape (:969-997): the unit cube scaled by
            // halfDimensions * localScaling + margin
            if (!F.has(c, "m_implicitShapeDimensions")) continue;
            const float margin = F.f32(c, "m_collisionMargin");
            float he[3];
            for (int k = 0; k < 3; ++k) he[k] = F.f32(c, "m_implicitShapeDimensions.m_floats", k) * scale[k] + margin;
            for (int i = 0; i < 8; ++i) {
                r.points.push_back((i & 1) ? he[0] : -he[0]);
                r.points.push_back((i & 2) ? he[1] : -he[1]);
                r.points.push_back((i & 4) ? he[2] : -he[2]);
            }
        } else if (stype == kConvexHullShape && hull) {
            // the points times localScaling (:757-787)
            const int64_t n = F.i32(c, "m_numUnscaledPoints");
            const Chunk* pts = F.chunk_at(F.ptr(c, "m_unscaledPointsFloatPtr"));
            if (n < 4 || !pts || (int64_t)pts->length < 16 * n) {
                b3_set_error("%s: convex hull without its points", path);
                return B3_ERR_INVALID_ARG;
            }
            if (n > kMaxFileHullPoints) {
                b3_set_error("%s: convex hull of %lld points (at most %lld)", path, (long long)n,
                             (long long)kMaxFileHullPoints);
                return B3_ERR_CAPACITY;
            }
            r.points.resize(3 * (size_t)n);
            for (int64_t i = 0; i < n; ++i)
                for (int k = 0; k < 3; ++k) {
                    float v;
                    std::memcpy(&v, pts->data + 16 * i + 4 * k, 4);
                    r.points[3 * i + k] = v * scale[k];
                }
        } else {
            continue;
        }
        // the same hull construction registration runs: a point set it
        // refuses fails the load here, before anything is registered
        b3hull::Polyhedron P;
        std::string herr;
        if (!b3hull::compute_polyhedron(r.points.data(), (int)(r.points.size() / 3), P, &herr)) {
            b3_set_error("%s: convex hull: %s", path, herr.c_str());
            return B3_ERR_INVALID_ARG;
        }
        shapes.push_back(std::move(r));
    }
    // bodies grouped by shape, shapes in order, file order inside a group
    // (:614-666); mass 1 / inverseMass, friction 1 (registerRigidBody,
    // P1/btGpuNarrowPhaseAndSolver.cpp:577); static bodies only when kept
    std::vector<BodyRec> bodies;
    for (size_t g = 0; g < shapes.size(); ++g) {
        for (const Chunk& c : F.chunks) {
            if (c.code != code4("RBDY")) continue;
            if (F.ptr(c, "m_collisionObjectData.m_collisionShape") != shapes[g].oldPtr) continue;
            const float invMass = F.f32(c, "m_inverseMass");
            if (!keepStaticObjects && invMass == 0.f) continue;
            double r[3][3];
            for (int row = 0; row < 3; ++row)
                for (int k = 0; k < 3; ++k)
                    r[row][k] = F.f32(c, "m_collisionObjectData.m_worldTransform.m_basis.m_el", 4 * row + k);
            BodyRec b;
            b.shape = (int)g;
            b.mass = invMass == 0.f ? 0.f : 1.f / invMass;
            basis_to_quat(r, b.quat);
            for (int k = 0; k < 3; ++k) b.pos[k] = F.f32(c, "m_collisionObjectData.m_worldTransform.m_origin.m_floats", k);
            bodies.push_back(b);
        }
    }
    const int64_t extra = keepStaticObjects ? 0 : 50 * 50;
    if ((int64_t)w->bodies.size() + (int64_t)bodies.size() + extra > (int64_t)w->cfg.maxBodies) {
        b3_set_error("%s: %lld bodies do not fit the world (capacity %d, %d registered)", path,
                     (long long)(bodies.size() + extra), w->cfg.maxBodies, (int)w->bodies.size());
        return B3_ERR_CAPACITY;
    }
    // Pass 2: register.
    std::vector<int> shapeCol(shapes.size(), -1);
    const float unit[3] = {1.f, 1.f, 1.f};
    for (size_t g = 0; g < shapes.size(); ++g) {
        const ShapeRec& r = shapes[g];
        int rc;
        if (r.kind == 1) rc = b3_register_sphere(w, r.radius, &shapeCol[g]);
        else if (r.kind == 2) rc = b3_register_plane(w, r.plane, r.plane[3], &shapeCol[g]);
        else rc = b3_register_convex_hull(w, r.points.data(), (int)(r.points.size() / 3), 12, unit, &shapeCol[g]);
        if (rc != B3_OK) return rc;
    }
    int count = 0;
    for (const BodyRec& b : bodies) {
        int body;
        const int rc = b3_register_body(w, b.mass, b.pos, b.quat, shapeCol[b.shape], 1.f, 0.f, 0, &body);
        if (rc != B3_OK) return rc;
        ++count;
    }
    if (!keepStaticObjects) {
        // the demo's replacement ground: 50 x 50 static tiles, an inverted
        // square pyramid scaled (2.5, 2, 2.5), 5.01 m apart (:678-708)
        const float tile[15] = {-1.f, 0.f, -1.f, -1.f, 0.f, 1.f, 1.f, 0.f, 1.f, 1.f, 0.f, -1.f, 0.f, -1.f, 0.f};
        const float scaling[3] = {2.5f, 2.f, 2.5f};
        int col;
        int rc = b3_register_convex_hull(w, tile, 5, 12, scaling, &col);
        if (rc != B3_OK) return rc;
        const float q[4] = {0.f, 0.f, 0.f, 1.f};
        for (int i = 0; i < 50; ++i)
            for (int j = 0; j < 50; ++j) {
                const float pos[3] = {(float)(i * 5.01 - 120.0), 0.f, (float)(j * 5.01 - 120.0)};
                int body;
                rc = b3_register_body(w, 0.f, pos, q, col, 1.f, 0.f, 0, &body);
                if (rc != B3_OK) return rc;
                ++count;
            }
    }
    if (numBodiesOut) *numBodiesOut = count;
    return B3_OK;
}
