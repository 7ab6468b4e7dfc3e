// core.cpp — PropertyList, object factory, transforms, XML scene loading and
// file loaders of the C++17 Nori host (reference: include/proplist.h,
// include/object.h, src/cpu/parser.cpp, include/dpdf.h of
// gracejinsotrue/PBRT-renderer-).
#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <set>
#include <sstream>

#include "nori/nori.h"

namespace nori {

// ---------------------------------------------------------------------------
// Color / Transform
// ---------------------------------------------------------------------------
std::string Color3f::toString() const {
    char b[96];
    std::snprintf(b, sizeof(b), "[%f, %f, %f]", c[0], c[1], c[2]);
    return b;
}

static void ident(float m[4][4]) {
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) m[i][j] = i == j ? 1.0f : 0.0f;
}
// General 4x4 inverse (Gauss-Jordan with partial pivoting, in double).
static bool invert4(const float a[4][4], float out[4][4]) {
    double m[4][8];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 8; j++) m[i][j] = j < 4 ? a[i][j] : (j - 4 == i ? 1.0 : 0.0);
    for (int c = 0; c < 4; c++) {
        int p = c;
        for (int r = c + 1; r < 4; r++)
            if (std::fabs(m[r][c]) > std::fabs(m[p][c])) p = r;
        if (std::fabs(m[p][c]) < 1e-300) return false;
        if (p != c)
            for (int j = 0; j < 8; j++) std::swap(m[p][j], m[c][j]);
        double d = m[c][c];
        for (int j = 0; j < 8; j++) m[c][j] /= d;
        for (int r = 0; r < 4; r++)
            if (r != c) {
                double f = m[r][c];
                for (int j = 0; j < 8; j++) m[r][j] -= f * m[c][j];
            }
    }
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) out[i][j] = (float)m[i][j + 4];
    return true;
}
Transform::Transform() { ident(m); ident(inv); }
Transform::Transform(const float mat[4][4]) {
    std::memcpy(m, mat, sizeof(m));
    if (!invert4(m, inv)) throw NoriException("Transform: singular matrix");
}
Transform Transform::inverse() const {
    Transform t;
    std::memcpy(t.m, inv, sizeof(inv));
    std::memcpy(t.inv, m, sizeof(m));
    return t;
}
Transform Transform::operator*(const Transform &t) const {
    float r[4][4], ri[4][4];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            float s = 0, si = 0;
            for (int k = 0; k < 4; k++) { s += m[i][k] * t.m[k][j]; si += t.inv[i][k] * inv[k][j]; }
            r[i][j] = s;
            ri[i][j] = si;
        }
    Transform o;
    std::memcpy(o.m, r, sizeof(r));
    std::memcpy(o.inv, ri, sizeof(ri));
    return o;
}
Point3f Transform::point(const Point3f &p) const {
    float r[4];
    for (int i = 0; i < 4; i++) r[i] = m[i][0] * p[0] + m[i][1] * p[1] + m[i][2] * p[2] + m[i][3];
    return Point3f(r[0] / r[3], r[1] / r[3], r[2] / r[3]);
}
Vector3f Transform::vector(const Vector3f &v) const {
    return Vector3f(m[0][0] * v[0] + m[0][1] * v[1] + m[0][2] * v[2], m[1][0] * v[0] + m[1][1] * v[1] + m[1][2] * v[2],
                    m[2][0] * v[0] + m[2][1] * v[1] + m[2][2] * v[2]);
}
Normal3f Transform::normal(const Normal3f &n) const {
    return Normal3f(inv[0][0] * n[0] + inv[1][0] * n[1] + inv[2][0] * n[2],
                    inv[0][1] * n[0] + inv[1][1] * n[1] + inv[2][1] * n[2],
                    inv[0][2] * n[0] + inv[1][2] * n[1] + inv[2][2] * n[2]);
}
std::string Transform::toString() const {
    std::ostringstream os;
    os << "[";
    for (int i = 0; i < 4; i++) {
        for (int j = 0; j < 4; j++) os << m[i][j] << (j < 3 ? ", " : "");
        os << (i < 3 ? "; " : "]");
    }
    return os.str();
}

// ---------------------------------------------------------------------------
// PropertyList (src/cpu/proplist.cpp): typed values, getters throw on a
// missing name (no default) or on a type mismatch.
// ---------------------------------------------------------------------------
void PropertyList::put(const std::string &name, Property p) {
    if (m_props.count(name)) std::fprintf(stderr, "Property \"%s\" was specified multiple times!\n", name.c_str());
    m_props[name] = std::move(p);
}
const PropertyList::Property *PropertyList::find(const std::string &name, Type type, bool required) const {
    auto it = m_props.find(name);
    if (it == m_props.end()) {
        if (required) throw NoriException("Property '" + name + "' is missing!");
        return nullptr;
    }
    if (it->second.type != type) throw NoriException("Property '" + name + "' has the wrong type!");
    return &it->second;
}
#define NORI_PROP(Name, T, TypeTag, field)                                                             \
    void PropertyList::set##Name(const std::string &name, T value) {                                   \
        Property p;                                                                                    \
        p.type = TypeTag;                                                                              \
        p.field = value;                                                                               \
        put(name, p);                                                                                  \
    }
NORI_PROP(Boolean, bool, Boolean, b)
NORI_PROP(Integer, int, Integer, i)
NORI_PROP(Float, float, Float, f)
NORI_PROP(String, const std::string &, String, s)
NORI_PROP(Color, const Color3f &, Color, c)
NORI_PROP(Point, const Point3f &, Point, p)
NORI_PROP(Vector, const Vector3f &, Vector, p)
NORI_PROP(Transform, const Transform &, TransformT, t)
#undef NORI_PROP
bool PropertyList::getBoolean(const std::string &n) const { return find(n, Boolean, true)->b; }
bool PropertyList::getBoolean(const std::string &n, bool d) const { auto p = find(n, Boolean, false); return p ? p->b : d; }
int PropertyList::getInteger(const std::string &n) const { return find(n, Integer, true)->i; }
int PropertyList::getInteger(const std::string &n, int d) const { auto p = find(n, Integer, false); return p ? p->i : d; }
float PropertyList::getFloat(const std::string &n) const { return find(n, Float, true)->f; }
float PropertyList::getFloat(const std::string &n, float d) const { auto p = find(n, Float, false); return p ? p->f : d; }
std::string PropertyList::getString(const std::string &n) const { return find(n, String, true)->s; }
std::string PropertyList::getString(const std::string &n, const std::string &d) const {
    auto p = find(n, String, false);
    return p ? p->s : d;
}
Color3f PropertyList::getColor(const std::string &n) const { return find(n, Color, true)->c; }
Color3f PropertyList::getColor(const std::string &n, const Color3f &d) const { auto p = find(n, Color, false); return p ? p->c : d; }
Point3f PropertyList::getPoint(const std::string &n) const { return find(n, Point, true)->p; }
Point3f PropertyList::getPoint(const std::string &n, const Point3f &d) const { auto p = find(n, Point, false); return p ? p->p : d; }
Vector3f PropertyList::getVector(const std::string &n) const { return find(n, Vector, true)->p; }
Vector3f PropertyList::getVector(const std::string &n, const Vector3f &d) const { auto p = find(n, Vector, false); return p ? p->p : d; }
Transform PropertyList::getTransform(const std::string &n) const { return find(n, TransformT, true)->t; }
Transform PropertyList::getTransform(const std::string &n, const Transform &d) const {
    auto p = find(n, TransformT, false);
    return p ? p->t : d;
}

Color3f readScalarOrColor(const PropertyList &propList, const std::string &name, float scalarDefault) {  // include/medium.h:14-27
    try { return propList.getColor(name); } catch (const NoriException &) {}
    try { return Color3f(propList.getFloat(name)); } catch (const NoriException &) {}
    return Color3f(scalarDefault);
}

// ---------------------------------------------------------------------------
// Object registry (src/cpu/object.cpp)
// ---------------------------------------------------------------------------
static std::map<std::string, NoriObjectFactory::Constructor> &constructors() {
    static std::map<std::string, NoriObjectFactory::Constructor> m;
    return m;
}
void NoriObjectFactory::registerClass(const std::string &name, const Constructor &c) { constructors()[name] = c; }
NoriObject *NoriObjectFactory::createInstance(const std::string &name, const PropertyList &propList) {
    auto it = constructors().find(name);
    if (it == constructors().end()) throw NoriException("A constructor for class \"" + name + "\" could not be found!");
    return it->second(propList);
}
std::vector<std::string> NoriObjectFactory::registeredClasses() {
    std::vector<std::string> v;
    for (auto &kv : constructors()) v.push_back(kv.first);
    return v;
}
void NoriObject::addChild(NoriObject *) {
    throw NoriException("NoriObject::addChild() is not implemented for objects of type '" +
                        classTypeName(getClassType()) + "'!");
}
std::string NoriObject::classTypeName(EClassType type) {
    switch (type) {
        case EScene: return "scene";
        case EMesh: return "mesh";
        case EBSDF: return "bsdf";
        case EEmitter: return "emitter";
        case ECamera: return "camera";
        case EIntegrator: return "integrator";
        case ESampler: return "sampler";
        case ETest: return "test";
        case EMedium: return "medium";
        default: return "<unknown>";
    }
}

// ---------------------------------------------------------------------------
// DiscretePDF (include/dpdf.h)
// ---------------------------------------------------------------------------
float DiscretePDF::normalize() {
    sum = cdf.back();
    if (sum > 0) {
        normalization = 1.0f / sum;
        for (size_t i = 1; i < cdf.size(); ++i) cdf[i] *= normalization;
        cdf.back() = 1.0f;
        normalized = true;
    } else {
        normalization = 0.0f;
    }
    return sum;
}
size_t DiscretePDF::sample(float u) const {
    auto it = std::lower_bound(cdf.begin(), cdf.end(), u);
    size_t idx = (size_t)std::max((ptrdiff_t)0, (ptrdiff_t)(it - cdf.begin()) - 1);
    return std::min(idx, size() - 1);
}
size_t DiscretePDF::sampleReuse(float &u) const {
    size_t i = sample(u);
    u = (u - cdf[i]) / (cdf[i + 1] - cdf[i]);
    return i;
}

// ---------------------------------------------------------------------------
// File resolution + loaders
// ---------------------------------------------------------------------------
static std::vector<std::string> &searchPaths() {
    static std::vector<std::string> v;
    return v;
}
void pushSearchPath(const std::string &dir) { searchPaths().insert(searchPaths().begin(), dir); }
void popSearchPath() {
    if (!searchPaths().empty()) searchPaths().erase(searchPaths().begin());
}
std::string resolvePath(const std::string &name, const std::string &baseDir) {
    if (!name.empty() && name[0] == '/') return name;
    auto readable = [](const std::string &p) { return std::ifstream(p).good(); };
    if (!baseDir.empty() && readable(baseDir + "/" + name)) return baseDir + "/" + name;
    for (const std::string &d : searchPaths()) {
        std::string p = d.empty() ? name : d + "/" + name;
        if (readable(p)) return p;
    }
    return name;
}

// Radiance RGBE (.hdr), flat or new-style run-length encoded scanlines.
bool loadHDR(const std::string &path, std::vector<float> &rgb, uint32_t &w, uint32_t &h) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    std::string line;
    if (!std::getline(f, line) || line.rfind("#?", 0) != 0) return false;
    while (std::getline(f, line) && !line.empty()) {
    }
    if (!std::getline(f, line)) return false;
    char ya[3], xa[3];
    int H, W;
    if (std::sscanf(line.c_str(), "%2s %d %2s %d", ya, &H, xa, &W) != 4 || W <= 0 || H <= 0) return false;
    w = (uint32_t)W;
    h = (uint32_t)H;
    rgb.assign((size_t)W * H * 3, 0.0f);
    std::vector<unsigned char> scan((size_t)W * 4);
    for (int y = 0; y < H; y++) {
        unsigned char hdr[4];
        if (!f.read((char *)hdr, 4)) return false;
        if (hdr[0] == 2 && hdr[1] == 2 && (hdr[2] & 0x80) == 0 && W >= 8 && W < 32768) {
            if (((int)hdr[2] << 8 | hdr[3]) != W) return false;
            for (int c = 0; c < 4; c++) {
                int x = 0;
                while (x < W) {
                    unsigned char cnt;
                    if (!f.read((char *)&cnt, 1)) return false;
                    if (cnt > 128) {
                        unsigned char v;
                        if (!f.read((char *)&v, 1)) return false;
                        for (int k = 0; k < cnt - 128 && x < W; k++) scan[(size_t)x++ * 4 + c] = v;
                    } else {
                        for (int k = 0; k < cnt && x < W; k++) {
                            unsigned char v;
                            if (!f.read((char *)&v, 1)) return false;
                            scan[(size_t)x++ * 4 + c] = v;
                        }
                    }
                }
            }
        } else {
            std::memcpy(scan.data(), hdr, 4);
            if (!f.read((char *)scan.data() + 4, (size_t)W * 4 - 4)) return false;
        }
        for (int x = 0; x < W; x++) {
            const unsigned char *p = &scan[(size_t)x * 4];
            float s = p[3] ? std::ldexp(1.0f, (int)p[3] - 136) : 0.0f;
            float *o = &rgb[((size_t)y * W + x) * 3];
            o[0] = p[0] * s; o[1] = p[1] * s; o[2] = p[2] * s;
        }
    }
    return true;
}

bool loadVol(const std::string &path, std::vector<float> &data, uint32_t &w, uint32_t &h, uint32_t &d) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    char magic[4];
    f.read(magic, 4);
    if (!f || std::memcmp(magic, "VOL1", 4) != 0) return false;
    f.read((char *)&w, 4);
    f.read((char *)&h, 4);
    f.read((char *)&d, 4);
    float bbox[6];
    f.read((char *)bbox, sizeof(bbox));
    if (!f || !w || !h || !d) return false;
    data.resize((size_t)w * h * d);
    f.read((char *)data.data(), data.size() * 4);
    return (bool)f;
}

// ---------------------------------------------------------------------------
// XML scene loading (src/cpu/parser.cpp): tag table, nesting rules,
// instantiate -> addChild/setParent -> activate, transform operations.
// ---------------------------------------------------------------------------
namespace {

struct XNode {
    std::string name;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<XNode> children;
    size_t offset = 0;
    const std::string *attr(const std::string &k) const {
        for (auto &a : attrs)
            if (a.first == k) return &a.second;
        return nullptr;
    }
};

class XmlReader {
public:
    XmlReader(const std::string &text, const std::string &file) : s(text), fn(file) {}
    XNode parseDocument() {
        skipMisc();
        if (pos >= s.size() || s[pos] != '<') fail("expected a root element");
        XNode root = parseElement();
        skipMisc();
        if (pos < s.size()) fail("content after the root element");
        return root;
    }
    std::string where(size_t off) const {
        int line = 1, col = 1;
        for (size_t i = 0; i < off && i < s.size(); i++) {
            if (s[i] == '\n') { line++; col = 1; } else col++;
        }
        return "line " + std::to_string(line) + ", col " + std::to_string(col);
    }

private:
    const std::string &s;
    const std::string fn;
    size_t pos = 0;
    [[noreturn]] void fail(const std::string &m) const {
        throw NoriException("Error while parsing \"" + fn + "\": " + m + " (at " + where(pos) + ")");
    }
    bool starts(const char *p) const { return s.compare(pos, std::strlen(p), p) == 0; }
    void skipWs() { while (pos < s.size() && std::isspace((unsigned char)s[pos])) pos++; }
    void skipMisc() {
        for (;;) {
            skipWs();
            if (starts("<!--")) {
                size_t e = s.find("-->", pos + 4);
                if (e == std::string::npos) fail("unterminated comment");
                pos = e + 3;
            } else if (starts("<?")) {
                size_t e = s.find("?>", pos + 2);
                if (e == std::string::npos) fail("unterminated declaration");
                pos = e + 2;
            } else {
                return;
            }
        }
    }
    std::string name() {
        size_t b = pos;
        while (pos < s.size() && (std::isalnum((unsigned char)s[pos]) || s[pos] == '_' || s[pos] == '-' ||
                                  s[pos] == ':' || s[pos] == '.'))
            pos++;
        if (b == pos) fail("expected a name");
        return s.substr(b, pos - b);
    }
    static std::string unescape(const std::string &v) {
        std::string o;
        for (size_t i = 0; i < v.size(); i++) {
            if (v[i] == '&') {
                size_t e = v.find(';', i);
                std::string ent = e == std::string::npos ? "" : v.substr(i + 1, e - i - 1);
                if (ent == "lt") o += '<'; else if (ent == "gt") o += '>'; else if (ent == "amp") o += '&';
                else if (ent == "quot") o += '"'; else if (ent == "apos") o += '\'';
                else { o += v[i]; continue; }
                i = e;
            } else {
                o += v[i];
            }
        }
        return o;
    }
    XNode parseElement() {
        XNode n;
        n.offset = pos;
        pos++;  // '<'
        n.name = name();
        for (;;) {
            skipWs();
            if (starts("/>")) { pos += 2; return n; }
            if (starts(">")) { pos++; break; }
            std::string k = name();
            skipWs();
            if (pos >= s.size() || s[pos] != '=') fail("expected '=' after attribute " + k);
            pos++;
            skipWs();
            char q = pos < s.size() ? s[pos] : 0;
            if (q != '"' && q != '\'') fail("expected a quoted attribute value");
            size_t e = s.find(q, pos + 1);
            if (e == std::string::npos) fail("unterminated attribute value");
            n.attrs.push_back({k, unescape(s.substr(pos + 1, e - pos - 1))});
            pos = e + 1;
        }
        for (;;) {
            skipMisc();
            if (pos >= s.size()) fail("unterminated element <" + n.name + ">");
            if (starts("</")) {
                pos += 2;
                std::string e = name();
                if (e != n.name) fail("mismatched closing tag </" + e + ">");
                skipWs();
                if (pos >= s.size() || s[pos] != '>') fail("expected '>'");
                pos++;
                return n;
            }
            if (s[pos] == '<') n.children.push_back(parseElement());
            else fail("unexpected content");
        }
    }
};

std::vector<std::string> tokenize(const std::string &v) {
    std::vector<std::string> out;
    std::string cur;
    for (char c : v) {
        if (c == ',' || std::isspace((unsigned char)c)) {
            if (!cur.empty()) out.push_back(cur);
            cur.clear();
        } else {
            cur += c;
        }
    }
    if (!cur.empty()) out.push_back(cur);
    return out;
}
float toFloat(const std::string &v) {
    char *end = nullptr;
    float f = std::strtof(v.c_str(), &end);
    if (end == v.c_str() || *end != '\0') throw NoriException("Could not parse floating point value \"" + v + "\"");
    return f;
}
int toInt(const std::string &v) {
    char *end = nullptr;
    long i = std::strtol(v.c_str(), &end, 10);
    if (end == v.c_str() || *end != '\0') throw NoriException("Could not parse integer value \"" + v + "\"");
    return (int)i;
}
bool toBool(const std::string &v) {
    std::string l = v;
    for (char &c : l) c = (char)std::tolower((unsigned char)c);
    if (l == "true") return true;
    if (l == "false") return false;
    throw NoriException("Could not parse boolean value \"" + v + "\"");
}
Vec3 toVector3f(const std::string &v) {
    auto t = tokenize(v);
    if (t.size() != 3) throw NoriException("Expected 3 values");
    return Vec3(toFloat(t[0]), toFloat(t[1]), toFloat(t[2]));
}
Transform fromMatrix(const float m[4][4]) { return Transform(m); }

enum ETag {
    TScene = NoriObject::EScene, TMesh = NoriObject::EMesh, TBSDF = NoriObject::EBSDF,
    TPhase = NoriObject::EPhaseFunction, TEmitter = NoriObject::EEmitter, TMedium = NoriObject::EMedium,
    TCamera = NoriObject::ECamera, TIntegrator = NoriObject::EIntegrator, TSampler = NoriObject::ESampler,
    TTest = NoriObject::ETest, TRFilter = NoriObject::EReconstructionFilter,
    TBoolean = NoriObject::EClassTypeCount, TInteger, TFloat, TString, TPoint, TVector, TColor, TTransform,
    TTranslate, TMatrix, TRotate, TScale, TLookAt, TInvalid
};

struct Loader {
    XmlReader &xr;
    std::string fn;
    Transform transform;
    std::map<std::string, ETag> tags{
        {"scene", TScene}, {"mesh", TMesh}, {"bsdf", TBSDF}, {"emitter", TEmitter}, {"camera", TCamera},
        {"medium", TMedium}, {"phase", TPhase}, {"integrator", TIntegrator}, {"sampler", TSampler},
        {"rfilter", TRFilter}, {"test", TTest}, {"boolean", TBoolean}, {"integer", TInteger}, {"float", TFloat},
        {"string", TString}, {"point", TPoint}, {"vector", TVector}, {"color", TColor}, {"transform", TTransform},
        {"translate", TTranslate}, {"matrix", TMatrix}, {"rotate", TRotate}, {"scale", TScale}, {"lookat", TLookAt}};

    void check_attributes(const XNode &n, std::set<std::string> want) {
        for (auto &a : n.attrs) {
            auto it = want.find(a.first);
            if (it == want.end())
                throw NoriException("Error while parsing \"" + fn + "\": unexpected attribute \"" + a.first +
                                    "\" in \"" + n.name + "\" at " + xr.where(n.offset));
            want.erase(it);
        }
        if (!want.empty())
            throw NoriException("Error while parsing \"" + fn + "\": missing attribute \"" + *want.begin() +
                                "\" in \"" + n.name + "\" at " + xr.where(n.offset));
    }
    const std::string &attr(const XNode &n, const char *k) { return *n.attr(k); }

    NoriObject *parse(const XNode &node, PropertyList &list, int parentTag) {
        auto it = tags.find(node.name);
        if (it == tags.end())
            throw NoriException("Error while parsing \"" + fn + "\": unexpected tag \"" + node.name + "\" at " +
                                xr.where(node.offset));
        int tag = it->second;
        // The format's nesting rules: the document element is a scene
        // object; a <transform> holds transform steps and nothing else, and
        // a transform step appears only there; every other element sits
        // inside a scene object.
        enum Kind { KObject, KStep, KOther };
        auto kind = [](int t) {
            if (t < NoriObject::EClassTypeCount) return KObject;
            if (t == TTranslate || t == TRotate || t == TScale || t == TLookAt || t == TMatrix) return KStep;
            return KOther;
        };
        const Kind self = kind(tag);
        const char *misplaced = nullptr;
        if (parentTag == TInvalid) {
            if (self != KObject) misplaced = "is not a scene object, so it cannot be the document element";
        } else if (parentTag == TTransform) {
            if (self != KStep) misplaced = "cannot appear inside <transform>, which holds transform steps only";
        } else if (self == KStep) {
            misplaced = "is a transform step and must appear inside <transform>";
        } else if (kind(parentTag) != KObject) {
            misplaced = "must appear inside a scene object";
        }
        if (misplaced)
            throw NoriException("Error while parsing \"" + fn + "\": <" + node.name + "> " + misplaced + " (at " +
                                xr.where(node.offset) + ")");
        const bool currentIsObject = self == KObject;
        if (tag == TTransform) transform = Transform();
        PropertyList propList;
        std::vector<NoriObject *> children;
        for (const XNode &ch : node.children) {
            NoriObject *c = parse(ch, propList, tag);
            if (c) children.push_back(c);
        }
        NoriObject *result = nullptr;
        try {
            if (currentIsObject) {
                std::string type = tag == TScene ? "scene" : "";
                if (tag == TScene) {
                    for (auto &a : node.attrs)
                        if (a.first != "type")
                            throw NoriException("unexpected attribute \"" + a.first + "\" in \"scene\"");
                } else {
                    check_attributes(node, {"type"});
                    type = attr(node, "type");
                }
                result = NoriObjectFactory::createInstance(type, propList);
                if ((int)result->getClassType() != tag)
                    throw NoriException("Unexpectedly constructed an object of type <" +
                                        NoriObject::classTypeName(result->getClassType()) + "> (expected type <" +
                                        NoriObject::classTypeName((NoriObject::EClassType)tag) + ">): " +
                                        result->toString());
                for (NoriObject *ch : children) {
                    result->addChild(ch);
                    ch->setParent(result);
                }
                result->activate();
            } else {
                switch (tag) {
                    case TString: check_attributes(node, {"name", "value"}); list.setString(attr(node, "name"), attr(node, "value")); break;
                    case TFloat: check_attributes(node, {"name", "value"}); list.setFloat(attr(node, "name"), toFloat(attr(node, "value"))); break;
                    case TInteger: check_attributes(node, {"name", "value"}); list.setInteger(attr(node, "name"), toInt(attr(node, "value"))); break;
                    case TBoolean: check_attributes(node, {"name", "value"}); list.setBoolean(attr(node, "name"), toBool(attr(node, "value"))); break;
                    case TPoint: check_attributes(node, {"name", "value"}); list.setPoint(attr(node, "name"), toVector3f(attr(node, "value"))); break;
                    case TVector: check_attributes(node, {"name", "value"}); list.setVector(attr(node, "name"), toVector3f(attr(node, "value"))); break;
                    case TColor: {
                        check_attributes(node, {"name", "value"});
                        Vec3 v = toVector3f(attr(node, "value"));
                        list.setColor(attr(node, "name"), Color3f(v[0], v[1], v[2]));
                        break;
                    }
                    case TTransform: check_attributes(node, {"name"}); list.setTransform(attr(node, "name"), transform); break;
                    case TTranslate: {
                        check_attributes(node, {"value"});
                        Vec3 v = toVector3f(attr(node, "value"));
                        float m[4][4]; ident(m);
                        m[0][3] = v[0]; m[1][3] = v[1]; m[2][3] = v[2];
                        transform = fromMatrix(m) * transform;
                        break;
                    }
                    case TMatrix: {
                        check_attributes(node, {"value"});
                        auto t = tokenize(attr(node, "value"));
                        if (t.size() != 16) throw NoriException("Expected 16 values");
                        float m[4][4];
                        for (int i = 0; i < 4; ++i)
                            for (int j = 0; j < 4; ++j) m[i][j] = toFloat(t[i * 4 + j]);
                        transform = fromMatrix(m) * transform;
                        break;
                    }
                    case TScale: {
                        check_attributes(node, {"value"});
                        Vec3 v = toVector3f(attr(node, "value"));
                        float m[4][4]; ident(m);
                        m[0][0] = v[0]; m[1][1] = v[1]; m[2][2] = v[2];
                        transform = fromMatrix(m) * transform;
                        break;
                    }
                    case TRotate: {
                        check_attributes(node, {"angle", "axis"});
                        float a = degToRad(toFloat(attr(node, "angle")));
                        Vec3 ax = toVector3f(attr(node, "axis")).normalized();
                        float c = std::cos(a), s = std::sin(a), t = 1 - c;
                        float x = ax[0], y = ax[1], z = ax[2];
                        float m[4][4] = {{t * x * x + c, t * x * y - s * z, t * x * z + s * y, 0},
                                         {t * x * y + s * z, t * y * y + c, t * y * z - s * x, 0},
                                         {t * x * z - s * y, t * y * z + s * x, t * z * z + c, 0},
                                         {0, 0, 0, 1}};
                        transform = fromMatrix(m) * transform;
                        break;
                    }
                    case TLookAt: {
                        check_attributes(node, {"origin", "target", "up"});
                        Vec3 o = toVector3f(attr(node, "origin")), t = toVector3f(attr(node, "target")),
                             up = toVector3f(attr(node, "up"));
                        Vec3 dir = (t - o).normalized();
                        Vec3 left = up.normalized().cross(dir).normalized();
                        Vec3 newUp = dir.cross(left).normalized();
                        float m[4][4] = {{left[0], newUp[0], dir[0], o[0]},
                                         {left[1], newUp[1], dir[1], o[1]},
                                         {left[2], newUp[2], dir[2], o[2]},
                                         {0, 0, 0, 1}};
                        transform = fromMatrix(m) * transform;
                        break;
                    }
                    default: throw NoriException("Unhandled element \"" + node.name + "\"");
                }
            }
        } catch (const NoriException &e) {
            throw NoriException("Error while parsing \"" + fn + "\": " + e.what() + " (at " + xr.where(node.offset) + ")");
        }
        return result;
    }
};

}  // namespace

NoriObject *loadFromXML(const std::string &filename) {
    std::ifstream f(filename, std::ios::binary);
    if (!f) throw NoriException("Error while parsing \"" + filename + "\": unable to open file");
    std::stringstream ss;
    ss << f.rdbuf();
    std::string text = ss.str();
    size_t slash = filename.find_last_of('/');
    const std::string dir = slash == std::string::npos ? std::string(".") : filename.substr(0, slash);
    // The scene's directory is searched first while its own files load (the
    // reference's resolver prepends it, src/cpu/parser.cpp), and only then:
    // a later scene in the same process must not find this one's files.
    struct Scoped {
        explicit Scoped(const std::string &d) { pushSearchPath(d); }
        ~Scoped() { popSearchPath(); }
    } scoped(dir);
    XmlReader xr(text, filename);
    XNode root = xr.parseDocument();
    Loader L{xr, filename};
    PropertyList list;
    NoriObject *obj = L.parse(root, list, TInvalid);
    // files the scene names but reads later (envmap, textures, volume grids)
    // resolve against its directory too
    if (obj && obj->getClassType() == NoriObject::EScene) static_cast<Scene *>(obj)->setBaseDir(dir);
    return obj;
}

}  // namespace nori
