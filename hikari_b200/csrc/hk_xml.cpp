// Plugin layer: XML loader, object factory and the plugin classes of the
// pathMIS path, plus a minimal OpenEXR reader/writer.  Mirrors the reference's
// src/core/{Parser,Object,PropertyList}.cpp behaviour (tag set, property
// types, child-first construction, AddChild -> SetParent -> Activate order,
// HikariException messages) and ends in the C ABI: a parsed Scene uploads
// itself through hk_scene_* and builds (Integrator::Preprocess).
#include "hk_xml.h"
#include "hk_obj.h"

#include <zlib.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <sstream>
#include <unordered_map>

namespace hikari {

// ------------------------------------------------------------ factory
namespace {
std::map<std::string, ObjectFactory::Constructor> &registry() {
    static std::map<std::string, ObjectFactory::Constructor> r;
    return r;
}
const char *class_name(EClassType t) {
    switch (t) {
    case EClassType::EScene: return "scene";
    case EClassType::EMesh: return "mesh";
    case EClassType::EBSDF: return "bsdf";
    case EClassType::EEmitter: return "emitter";
    case EClassType::ECamera: return "camera";
    case EClassType::EIntegrator: return "integrator";
    case EClassType::ESampler: return "sampler";
    case EClassType::EReconstructionFilter: return "rfilter";
    case EClassType::EAcceleration: return "acceleration";
    case EClassType::ETest: return "test";
    case EClassType::ETexture: return "texture";
    }
    return "unknown";
}
}  // namespace

void Object::AddChild(Object *child, const std::string &name) {
    throw HikariException(std::string("AddChild(<") + class_name(child->GetClassType()) + ">, <" + name +
                          ">) is not supported for " + type_name);
}
void ObjectFactory::RegisterClass(const std::string &name, const Constructor &c) { registry()[name] = c; }
bool ObjectFactory::Exists(const std::string &name) { return registry().count(name) != 0; }
Object *ObjectFactory::CreateInstance(const std::string &name, const PropertyList &props) {
    auto it = registry().find(name);
    if (it == registry().end())
        throw HikariException("A constructor for class \"" + name + "\" could not be found!");
    Object *o = it->second(props);
    o->type_name = name;
    return o;
}
// REGISTER_CLASS (include/core/Object.hpp:137): static-initialiser registration
#define HK_REGISTER_CLASS(Cls, Name)                                                                      \
    static struct Cls##Registrar {                                                                        \
        Cls##Registrar() {                                                                                \
            ObjectFactory::RegisterClass(Name, [](const PropertyList &p) -> Object * { return new Cls(p); }); \
        }                                                                                                 \
    } Cls##_registrar;

// ------------------------------------------------------------ math helpers
namespace {
Matrix4f identity4() { return {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1}; }
Matrix4f mul4(const Matrix4f &a, const Matrix4f &b) {
    Matrix4f r{};
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            float s = 0;
            for (int k = 0; k < 4; k++) s += a[4 * i + k] * b[4 * k + j];
            r[4 * i + j] = s;
        }
    return r;
}
bool inverse4(const Matrix4f &m, Matrix4f &out) {
    double a[4][8];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 8; j++) a[i][j] = j < 4 ? m[4 * i + j] : (j - 4 == i ? 1.0 : 0.0);
    for (int c = 0; c < 4; c++) {
        int p = c;
        for (int r = c + 1; r < 4; r++)
            if (std::fabs(a[r][c]) > std::fabs(a[p][c])) p = r;
        if (a[p][c] == 0.0) return false;
        for (int j = 0; j < 8; j++) std::swap(a[c][j], a[p][j]);
        double inv = 1.0 / a[c][c];
        for (int j = 0; j < 8; j++) a[c][j] *= inv;
        for (int r = 0; r < 4; r++)
            if (r != c) {
                double f = a[r][c];
                for (int j = 0; j < 8; j++) a[r][j] -= f * a[c][j];
            }
    }
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) out[4 * i + j] = (float)a[i][j + 4];
    return true;
}
Color3f normalized(Color3f v) {
    float n = std::sqrt(v[0] * v[0] + (v[1] * v[1] + v[2] * v[2]));
    return n > 0 ? Color3f{v[0] / n, v[1] / n, v[2] / n} : v;
}
Color3f cross3(Color3f a, Color3f b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}

std::vector<std::string> tokenize(const std::string &s, const std::string &delim = ", \t\r\n") {
    std::vector<std::string> out;
    size_t i = 0;
    while (i < s.size()) {
        size_t j = s.find_first_of(delim, i);
        if (j == std::string::npos) j = s.size();
        if (j > i) out.push_back(s.substr(i, j - i));
        i = j + 1;
    }
    return out;
}
float to_float(const std::string &s) {   // ToFloat (src/core/Common.cpp:97)
    char *end = nullptr;
    float r = std::strtof(s.c_str(), &end);
    if (*end != '\0') throw HikariException("Could not parse floating point value \"" + s + "\"");
    return r;
}
int to_int(const std::string &s) {
    char *end = nullptr;
    long r = std::strtol(s.c_str(), &end, 10);
    if (*end != '\0') throw HikariException("Could not parse integer value \"" + s + "\"");
    return (int)r;
}
bool to_bool(const std::string &s) {
    std::string v = s;
    std::transform(v.begin(), v.end(), v.begin(), ::tolower);
    if (v == "true") return true;
    if (v == "false") return false;
    throw HikariException("Could not parse boolean value \"" + s + "\"");
}
Color3f to_vec3(const std::string &s) {   // ToVector3f (src/core/Common.cpp:108)
    auto t = tokenize(s);
    if (t.size() != 3) throw HikariException("Expected 3 values");
    return {to_float(t[0]), to_float(t[1]), to_float(t[2])};
}

// ------------------------------------------------------------ XML tree
struct XNode {
    std::string name;
    std::vector<std::pair<std::string, std::string>> attrs;
    std::vector<XNode> children;
    int line = 0;
    const std::string *attr(const std::string &n) const {
        for (auto &a : attrs)
            if (a.first == n) return &a.second;
        return nullptr;
    }
};

class XmlReader {
public:
    XmlReader(const std::string &text, const std::string &fn) : s_(text), fn_(fn) {}
    XNode parse_document() {
        skip_misc();
        XNode root = parse_element();
        skip_misc();
        if (i_ < s_.size()) err("unexpected content after the root element");
        return root;
    }

private:
    const std::string &s_;
    std::string fn_;
    size_t i_ = 0;
    [[noreturn]] void err(const std::string &m) {
        int line = 1 + (int)std::count(s_.begin(), s_.begin() + std::min(i_, s_.size()), '\n');
        throw HikariException("Error while parsing \"" + fn_ + "\": " + m + " (at line " + std::to_string(line) + ")");
    }
    bool starts(const char *p) const { return s_.compare(i_, std::strlen(p), p) == 0; }
    void skip_ws() { while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_; }
    void skip_misc() {
        for (;;) {
            skip_ws();
            if (starts("<?")) {
                size_t j = s_.find("?>", i_);
                if (j == std::string::npos) err("unterminated declaration");
                i_ = j + 2;
            } else if (starts("<!--")) {
                size_t j = s_.find("-->", i_);
                if (j == std::string::npos) err("unterminated comment");
                i_ = j + 3;
            } else {
                return;
            }
        }
    }
    std::string name() {
        size_t b = i_;
        while (i_ < s_.size() && (std::isalnum((unsigned char)s_[i_]) || s_[i_] == '_' || s_[i_] == '-' ||
                                  s_[i_] == ':' || s_[i_] == '.'))
            ++i_;
        if (b == i_) err("expected a name");
        return s_.substr(b, i_ - b);
    }
    static std::string unescape(const std::string &v) {
        std::string o;
        for (size_t k = 0; k < v.size(); ++k) {
            if (v[k] == '&') {
                size_t e = v.find(';', k);
                std::string ent = v.substr(k + 1, e - k - 1);
                if (ent == "lt") o += '<'; else if (ent == "gt") o += '>'; else if (ent == "amp") o += '&';
                else if (ent == "quot") o += '"'; else if (ent == "apos") o += '\''; else o += "&" + ent + ";";
                k = e;
            } else {
                o += v[k];
            }
        }
        return o;
    }
    XNode parse_element() {
        if (!starts("<")) err("expected an element");
        XNode n;
        n.line = 1 + (int)std::count(s_.begin(), s_.begin() + i_, '\n');
        ++i_;
        n.name = name();
        for (;;) {
            skip_ws();
            if (starts("/>")) { i_ += 2; return n; }
            if (starts(">")) { ++i_; break; }
            std::string an = name();
            skip_ws();
            if (!starts("=")) err("expected '='");
            ++i_;
            skip_ws();
            char q = s_[i_];
            if (q != '"' && q != '\'') err("expected a quoted attribute value");
            size_t e = s_.find(q, i_ + 1);
            if (e == std::string::npos) err("unterminated attribute value");
            n.attrs.emplace_back(an, unescape(s_.substr(i_ + 1, e - i_ - 1)));
            i_ = e + 1;
        }
        for (;;) {
            skip_misc();
            if (starts("</")) {
                i_ += 2;
                std::string cn = name();
                if (cn != n.name) err("mismatched closing tag </" + cn + ">");
                skip_ws();
                if (!starts(">")) err("expected '>'");
                ++i_;
                return n;
            }
            if (starts("<")) { n.children.push_back(parse_element()); continue; }
            if (i_ >= s_.size()) err("unterminated element <" + n.name + ">");
            // text content is not part of the scene format
            size_t j = s_.find('<', i_);
            std::string txt = s_.substr(i_, j - i_);
            if (txt.find_first_not_of(" \t\r\n") != std::string::npos) err("unexpected content");
            i_ = j;
        }
    }
};

enum class Tag { Object, Boolean, Integer, Float, String, Point, Vector, Color, Transform, Translate, Matrix, Rotate,
                 Scale, LookAt };
const std::map<std::string, EClassType> &object_tags() {
    static const std::map<std::string, EClassType> m = {
        {"scene", EClassType::EScene}, {"mesh", EClassType::EMesh}, {"bsdf", EClassType::EBSDF},
        {"emitter", EClassType::EEmitter}, {"camera", EClassType::ECamera}, {"integrator", EClassType::EIntegrator},
        {"sampler", EClassType::ESampler}, {"rfilter", EClassType::EReconstructionFilter},
        {"acceleration", EClassType::EAcceleration}, {"test", EClassType::ETest}, {"texture", EClassType::ETexture}};
    return m;
}
const std::map<std::string, Tag> &prop_tags() {
    static const std::map<std::string, Tag> m = {
        {"boolean", Tag::Boolean}, {"integer", Tag::Integer}, {"float", Tag::Float}, {"string", Tag::String},
        {"point", Tag::Point}, {"vector", Tag::Vector}, {"color", Tag::Color}, {"transform", Tag::Transform},
        {"translate", Tag::Translate}, {"matrix", Tag::Matrix}, {"rotate", Tag::Rotate}, {"scale", Tag::Scale},
        {"lookat", Tag::LookAt}};
    return m;
}

struct ParseCtx {
    std::string filename, base_dir;
    Matrix4f trans = identity4();
};
thread_local std::string g_base_dir;   // OBJ/EXR paths resolve against the scene directory

std::string req(const XNode &n, const char *a) {
    const std::string *v = n.attr(a);
    if (!v) throw HikariException(std::string("missing attribute \"") + a + "\" in <" + n.name + ">");
    return *v;
}

// ParseTagFunc (src/core/Parser.cpp:157): children first, then the object, then
// AddChild/SetParent for each child and Activate.
Object *parse_tag(const XNode &n, PropertyList &props, bool parent_is_transform, ParseCtx &ctx) {
    auto ot = object_tags().find(n.name);
    if (ot != object_tags().end()) {
        if (parent_is_transform) throw HikariException("transform nodes can only contain transform operations");
        PropertyList child_props;
        std::vector<std::unique_ptr<Object>> kids;
        std::vector<std::string> names;
        for (auto &c : n.children) {
            Object *o = parse_tag(c, child_props, false, ctx);
            if (o) {
                kids.emplace_back(o);
                const std::string *nm = c.attr("name");
                names.push_back(nm ? *nm : "");
            }
        }
        std::string type = n.name == "scene" ? "scene" : req(n, "type");
        std::unique_ptr<Object> obj(ObjectFactory::CreateInstance(type, child_props));
        if (obj->GetClassType() != ot->second)
            throw HikariException("Unexpectedly constructed an object of type <" +
                                  std::string(class_name(obj->GetClassType())) + "> (expected type <" +
                                  class_name(ot->second) + ">)");
        for (size_t k = 0; k < kids.size(); ++k) {
            Object *c = kids[k].release();
            obj->AddChild(c, names[k]);   // the parent owns the child from here on
            const std::string *nm = n.attr("name");
            c->SetParent(obj.get(), nm ? *nm : "");
        }
        obj->Activate();
        return obj.release();
    }
    auto pt = prop_tags().find(n.name);
    if (pt == prop_tags().end()) throw HikariException("unexpected tag \"" + n.name + "\"");
    Tag t = pt->second;
    bool is_op = t == Tag::Translate || t == Tag::Matrix || t == Tag::Rotate || t == Tag::Scale || t == Tag::LookAt;
    if (parent_is_transform != is_op) throw HikariException("transform nodes can only contain transform operations");
    switch (t) {
    case Tag::Boolean: props.SetBoolean(req(n, "name"), to_bool(req(n, "value"))); break;
    case Tag::Integer: props.SetInteger(req(n, "name"), to_int(req(n, "value"))); break;
    case Tag::Float: props.SetFloat(req(n, "name"), to_float(req(n, "value"))); break;
    case Tag::String: props.SetString(req(n, "name"), req(n, "value")); break;
    case Tag::Point: props.SetPoint(req(n, "name"), to_vec3(req(n, "value"))); break;
    case Tag::Vector: props.SetVector(req(n, "name"), to_vec3(req(n, "value"))); break;
    case Tag::Color: props.SetColor(req(n, "name"), to_vec3(req(n, "value"))); break;
    case Tag::Transform: {
        ctx.trans = identity4();
        PropertyList dummy;
        for (auto &c : n.children) parse_tag(c, dummy, true, ctx);
        props.SetTransform(req(n, "name"), ctx.trans);
        break;
    }
    case Tag::Translate: {
        Color3f v = to_vec3(req(n, "value"));
        Matrix4f M = identity4();
        M[3] = v[0]; M[7] = v[1]; M[11] = v[2];
        ctx.trans = mul4(M, ctx.trans);
        break;
    }
    case Tag::Scale: {
        Color3f v = to_vec3(req(n, "value"));
        Matrix4f M = identity4();
        M[0] = v[0]; M[5] = v[1]; M[10] = v[2];
        ctx.trans = mul4(M, ctx.trans);
        break;
    }
    case Tag::Matrix: {
        auto tk = tokenize(req(n, "value"));
        if (tk.size() != 16) throw HikariException("Expected 16 values");
        Matrix4f M;
        for (int k = 0; k < 16; k++) M[k] = to_float(tk[k]);
        ctx.trans = mul4(M, ctx.trans);
        break;
    }
    case Tag::Rotate: {   // Eigen::AngleAxis with the axis as given
        float ang = to_float(req(n, "angle")) * (3.14159265358979323846f / 180.0f);
        Color3f a = to_vec3(req(n, "axis"));
        float c = std::cos(ang), s = std::sin(ang), C = 1 - c;
        float x = a[0], y = a[1], z = a[2];
        Matrix4f M = {x * x * C + c, x * y * C - z * s, x * z * C + y * s, 0, y * x * C + z * s, y * y * C + c,
                      y * z * C - x * s, 0, z * x * C - y * s, z * y * C + x * s, z * z * C + c, 0, 0, 0, 0, 1};
        ctx.trans = mul4(M, ctx.trans);
        break;
    }
    case Tag::LookAt: {   // src/core/Parser.cpp:353
        Color3f o = to_vec3(req(n, "origin")), tg = to_vec3(req(n, "target")), up = to_vec3(req(n, "up"));
        Color3f dir = normalized({tg[0] - o[0], tg[1] - o[1], tg[2] - o[2]});
        Color3f left = normalized(cross3(normalized(up), dir));
        Color3f nup = normalized(cross3(dir, left));
        Matrix4f M = {left[0], nup[0], dir[0], o[0], left[1], nup[1], dir[1], o[1],
                      left[2], nup[2], dir[2], o[2], 0, 0, 0, 1};
        ctx.trans = mul4(M, ctx.trans);
        break;
    }
    default: break;
    }
    return nullptr;
}
}  // namespace

std::unique_ptr<Object> LoadFromXML(const std::string &filename) {
    std::ifstream f(filename, std::ios::binary);
    if (!f) throw HikariException("Unable to open file \"" + filename + "\"");
    std::stringstream ss;
    ss << f.rdbuf();
    std::string text = ss.str();
    XmlReader rd(text, filename);
    XNode root = rd.parse_document();
    ParseCtx ctx;
    ctx.filename = filename;
    size_t slash = filename.find_last_of('/');
    std::string prev = g_base_dir;
    g_base_dir = slash == std::string::npos ? "." : filename.substr(0, slash);
    PropertyList props;
    std::unique_ptr<Object> obj;
    try {
        obj.reset(parse_tag(root, props, false, ctx));
    } catch (const HikariException &e) {
        g_base_dir = prev;
        throw HikariException("Error while parsing \"" + filename + "\": " + e.what());
    }
    g_base_dir = prev;
    if (!obj) throw HikariException("root element must be an object");
    return obj;
}

// ------------------------------------------------------------ OpenEXR
namespace {
float half_to_float(uint16_t h) {
    uint32_t s = (h >> 15) & 1, e = (h >> 10) & 31, m = h & 1023, o;
    if (e == 0) {
        if (m == 0) o = s << 31;
        else {
            int k = -1;
            do { k++; m <<= 1; } while (!(m & 1024));
            m &= 1023;
            o = (s << 31) | ((uint32_t)(127 - 15 - k) << 23) | (m << 13);
        }
    } else if (e == 31) {
        o = (s << 31) | (0xffu << 23) | (m << 13);
    } else {
        o = (s << 31) | ((e - 15 + 127) << 23) | (m << 13);
    }
    float r;
    std::memcpy(&r, &o, 4);
    return r;
}
}  // namespace

void ReadEXR(const std::string &fn, int &W, int &H, std::vector<float> &rgb) {
    std::ifstream f(fn, std::ios::binary);
    if (!f) throw HikariException("Unable to open EXR \"" + fn + "\"");
    std::vector<unsigned char> b((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
    size_t p = 0;
    auto need = [&](size_t n) { if (p + n > b.size()) throw HikariException("truncated EXR \"" + fn + "\""); };
    auto rd32 = [&]() { need(4); int32_t v; std::memcpy(&v, &b[p], 4); p += 4; return v; };
    need(8);
    uint32_t magic;
    std::memcpy(&magic, &b[0], 4);
    if (magic != 20000630u) throw HikariException("not an OpenEXR file: \"" + fn + "\"");
    uint32_t ver;
    std::memcpy(&ver, &b[4], 4);
    if ((ver & 0xff) != 2 || (ver & 0x1e00)) throw HikariException("only single-part scanline EXR is supported");
    p = 8;
    struct Ch { std::string name; int type; };
    std::vector<Ch> chans;
    int comp = -1, x0 = 0, y0 = 0, x1 = -1, y1 = -1;
    for (;;) {
        need(1);
        if (b[p] == 0) { ++p; break; }
        std::string an((const char *)&b[p]);
        p += an.size() + 1;
        need(1);
        std::string at((const char *)&b[p]);
        p += at.size() + 1;
        int32_t sz = rd32();
        need(sz);
        size_t q = p;
        if (an == "channels") {
            while (b[q] != 0) {
                std::string cn((const char *)&b[q]);
                q += cn.size() + 1;
                int32_t pt;
                std::memcpy(&pt, &b[q], 4);
                chans.push_back({cn, pt});
                q += 16;
            }
        } else if (an == "compression") {
            comp = b[q];
        } else if (an == "dataWindow") {
            std::memcpy(&x0, &b[q], 4); std::memcpy(&y0, &b[q + 4], 4);
            std::memcpy(&x1, &b[q + 8], 4); std::memcpy(&y1, &b[q + 12], 4);
        }
        p += sz;
    }
    W = x1 - x0 + 1;
    H = y1 - y0 + 1;
    if (W <= 0 || H <= 0) throw HikariException("EXR has an empty data window");
    if (comp != 0 && comp != 2 && comp != 3)
        throw HikariException("EXR compression not supported (use NONE, ZIPS or ZIP): \"" + fn + "\"");
    int lines_per_chunk = comp == 3 ? 16 : 1;
    int nchunks = (H + lines_per_chunk - 1) / lines_per_chunk;
    std::vector<uint64_t> offs(nchunks);
    need(8ull * nchunks);
    std::memcpy(offs.data(), &b[p], 8ull * nchunks);
    int ci[3] = {-1, -1, -1};
    size_t bpp = 0;
    for (size_t k = 0; k < chans.size(); ++k) {
        if (chans[k].type != 1 && chans[k].type != 2) throw HikariException("EXR channel type must be HALF or FLOAT");
        bpp += chans[k].type == 1 ? 2 : 4;
        if (chans[k].name == "R") ci[0] = (int)k;
        if (chans[k].name == "G") ci[1] = (int)k;
        if (chans[k].name == "B") ci[2] = (int)k;
    }
    if (ci[0] < 0 || ci[1] < 0 || ci[2] < 0) throw HikariException("EXR needs R, G and B channels");
    rgb.assign((size_t)W * H * 3, 0.0f);
    std::vector<unsigned char> raw, tmp;
    for (int c = 0; c < nchunks; ++c) {
        p = offs[c];
        int32_t y = rd32(), n = rd32();
        need(n);
        int ly = std::min(lines_per_chunk, y1 - y + 1);
        size_t expect = (size_t)ly * W * bpp;
        const unsigned char *data = &b[p];
        if (comp != 0 && (size_t)n < expect) {
            tmp.resize(expect);
            uLongf dl = (uLongf)expect;
            if (uncompress(tmp.data(), &dl, data, (uLong)n) != Z_OK || dl != expect)
                throw HikariException("EXR zlib decompression failed");
            for (size_t k = 1; k < expect; ++k) tmp[k] = (unsigned char)(tmp[k - 1] + tmp[k] - 128);
            raw.resize(expect);
            size_t half = (expect + 1) / 2;
            for (size_t k = 0; k < expect; ++k) raw[k] = (k & 1) ? tmp[half + k / 2] : tmp[k / 2];
            data = raw.data();
        } else if ((size_t)n != expect) {
            throw HikariException("EXR chunk has an unexpected size");
        }
        size_t off = 0;
        for (int l = 0; l < ly; ++l) {
            int row = y + l - y0;
            for (size_t k = 0; k < chans.size(); ++k) {
                int target = k == (size_t)ci[0] ? 0 : k == (size_t)ci[1] ? 1 : k == (size_t)ci[2] ? 2 : -1;
                for (int x = 0; x < W; ++x) {
                    float v;
                    if (chans[k].type == 1) { uint16_t h; std::memcpy(&h, data + off, 2); off += 2; v = half_to_float(h); }
                    else { std::memcpy(&v, data + off, 4); off += 4; }
                    if (target >= 0) rgb[3 * ((size_t)row * W + x) + target] = v;
                }
            }
        }
    }
}

void WriteEXR(const std::string &fn, int W, int H, const float *rgb) {
    std::vector<unsigned char> o;
    auto put = [&](const void *d, size_t n) { const unsigned char *c = (const unsigned char *)d; o.insert(o.end(), c, c + n); };
    auto put32 = [&](int32_t v) { put(&v, 4); };
    auto attr = [&](const char *name, const char *type, const std::vector<unsigned char> &val) {
        put(name, std::strlen(name) + 1);
        put(type, std::strlen(type) + 1);
        put32((int32_t)val.size());
        put(val.data(), val.size());
    };
    uint32_t magic = 20000630u, ver = 2;
    put(&magic, 4);
    put(&ver, 4);
    std::vector<unsigned char> ch;
    for (const char *n : {"B", "G", "R"}) {
        ch.insert(ch.end(), n, n + 2);
        int32_t v[4] = {2, 0, 1, 1};   // FLOAT, pLinear+reserved, xSampling, ySampling
        ch.insert(ch.end(), (unsigned char *)v, (unsigned char *)v + 16);
    }
    ch.push_back(0);
    attr("channels", "chlist", ch);
    attr("compression", "compression", {0});
    int32_t win[4] = {0, 0, W - 1, H - 1};
    std::vector<unsigned char> w((unsigned char *)win, (unsigned char *)win + 16);
    attr("dataWindow", "box2i", w);
    attr("displayWindow", "box2i", w);
    attr("lineOrder", "lineOrder", {0});
    float par = 1.0f, ssw = 1.0f, swc[2] = {0, 0};
    attr("pixelAspectRatio", "float", std::vector<unsigned char>((unsigned char *)&par, (unsigned char *)&par + 4));
    attr("screenWindowCenter", "v2f", std::vector<unsigned char>((unsigned char *)swc, (unsigned char *)swc + 8));
    attr("screenWindowWidth", "float", std::vector<unsigned char>((unsigned char *)&ssw, (unsigned char *)&ssw + 4));
    o.push_back(0);
    uint64_t table = o.size(), line_bytes = 8 + 12ull * W;
    o.resize(o.size() + 8ull * H);
    for (int y = 0; y < H; ++y) {
        uint64_t off = table + 8ull * H + y * line_bytes;
        std::memcpy(&o[table + 8ull * y], &off, 8);
    }
    for (int y = 0; y < H; ++y) {
        put32(y);
        put32(12 * W);
        for (int c = 2; c >= 0; --c)
            for (int x = 0; x < W; ++x) put(&rgb[3 * ((size_t)y * W + x) + c], 4);
    }
    std::ofstream f(fn, std::ios::binary);
    if (!f) throw HikariException("Unable to write EXR \"" + fn + "\"");
    f.write((const char *)o.data(), (std::streamsize)o.size());
}

// ------------------------------------------------------------ plugins
namespace {

std::string resolve(const std::string &f) {
    if (!f.empty() && f[0] == '/') return f;
    return g_base_dir + "/" + f;
}

// Texture plugins (src/texture/{Checkerboard,Grid,Scale,Bitmap,Wireframe,Curvature}Texture.cpp),
// defaults of include/core/Common.hpp:425-462
class TexturePlugin : public Object {
public:
    hk_texture_desc d{};
    std::unique_ptr<TexturePlugin> nested;
    std::vector<uint8_t> pixels;   // bitmap: decoded 8-bit pixels (row 0 = top)
    int32_t width = 0, height = 0;
    TexturePlugin(const PropertyList &p, int kind) {
        std::memset(&d, 0, sizeof d);
        d.kind = kind;
        d.nested = -1;
        d.uv_scale[0] = p.GetFloat("uScale", 1.0f);
        d.uv_scale[1] = p.GetFloat("vScale", 1.0f);
        d.uv_offset[0] = p.GetFloat("uOffset", 0.0f);
        d.uv_offset[1] = p.GetFloat("vOffset", 0.0f);
        auto setc = [](float *dst, const Color3f &c) { dst[0] = c[0]; dst[1] = c[1]; dst[2] = c[2]; };
        if (kind == HK_TEX_CHECKERBOARD) {
            d.count = p.GetInteger("blocks", 10);
            setc(d.a, p.GetColor("colorA", {0.4f, 0.4f, 0.4f}));
            setc(d.b, p.GetColor("colorB", {0.2f, 0.2f, 0.2f}));
        } else if (kind == HK_TEX_GRID) {
            d.count = p.GetInteger("lines", 10);
            setc(d.a, p.GetColor("lineColor", {0.4f, 0.4f, 0.4f}));
            setc(d.b, p.GetColor("backgroundColor", {0.2f, 0.2f, 0.2f}));
            d.width = p.GetFloat("lineWidth", 0.01f);
        } else if (kind == HK_TEX_BITMAP) {
            load_bitmap(p);
            return;
        } else if (kind == HK_TEX_WIREFRAME) {   // WireframeTexture ctor (src/texture/WireframeTexture.cpp:10)
            setc(d.a, p.GetColor("interiorColor", {0.5f, 0.5f, 0.5f}));
            setc(d.b, p.GetColor("edgeColor", {0.1f, 0.1f, 0.1f}));
            d.width = p.GetFloat("edgeWidth", 0.0f);
            d.scale = p.GetFloat("transitionWidth", 0.5f);
            return;
        } else if (kind == HK_TEX_CURVATURE) {   // CurvatureTexture ctor (src/texture/CurvatureTexture.cpp:9)
            setc(d.a, p.GetColor("positiveColor", {1.0f, 0.0f, 0.0f}));
            setc(d.b, p.GetColor("negativeColor", {0.0f, 0.0f, 1.0f}));
            d.scale = p.GetFloat("scale", 1.0f);
            const std::string ct = p.GetString("curvatureType");
            if (ct == "gaussian") d.count = 1;
            else if (ct == "mean") d.count = 0;
            else throw HikariException("Unexpected curvature type <" + ct + ">.");
            return;
        } else {
            d.scale = p.GetFloat("scale");
        }
        if (kind != HK_TEX_SCALE && d.count <= 0) throw HikariException("texture block / line count must be positive");
    }
    // BitmapTexture ctor (src/texture/BitmapTexture.cpp:7): the image decoded
    // like stbi_load (hk_image_load), wrap / filter / channel names as there
    void load_bitmap(const PropertyList &p) {
        const std::string fn = resolve(p.GetString("filename"));
        d.gamma = p.GetFloat("gamma", 1.0f);
        auto wrap_of = [](const std::string &w) {
            if (w == "repeat") return HK_WRAP_REPEAT;
            if (w == "clamp") return HK_WRAP_CLAMP;
            if (w == "black") return HK_WRAP_BLACK;
            throw HikariException("Illegal wrap mode [" + w + "].");
        };
        const std::string both = p.GetString("wrapMode", "");
        if (!both.empty()) {
            d.wrap_u = d.wrap_v = wrap_of(both);
        } else {
            d.wrap_u = wrap_of(p.GetString("uWrapMode", "repeat"));
            d.wrap_v = wrap_of(p.GetString("vWrapMode", "repeat"));
        }
        const std::string ft = p.GetString("filterType", "ewa");
        if (ft == "nearest") d.filter = HK_FILTER_NEAREST;
        else if (ft == "bilinear") d.filter = HK_FILTER_BILINEAR;
        else if (ft == "trilinear") d.filter = HK_FILTER_TRILINEAR;
        else if (ft == "ewa") d.filter = HK_FILTER_EWA;
        else throw HikariException("Illegal filter type [" + ft + "].");
        d.max_anisotropy = p.GetFloat("maxAnisotropy", 20.0f);
        const std::string chn = p.GetString("channel", "rgb");
        if (chn == "r") d.channels = 1;
        else if (chn == "rgb") d.channels = 3;
        else throw HikariException("Illegal channel [" + chn + "].");
        uint8_t *buf = nullptr;
        if (hk_image_load(fn.c_str(), d.channels, &width, &height, &buf) != HK_OK)
            throw HikariException(std::string("Load texture \"") + fn + "\" failed. Reason : [" + hk_last_error() + "]");
        pixels.assign(buf, buf + (size_t)width * height * d.channels);
        hk_image_free(buf);
    }
    EClassType GetClassType() const override { return EClassType::ETexture; }
    void AddChild(Object *c, const std::string &name) override {
        if (d.kind == HK_TEX_SCALE && c->GetClassType() == EClassType::ETexture && !nested) {
            nested.reset((TexturePlugin *)c);
            return;
        }
        delete c;
        throw HikariException("ScaleTexture: tried to specify multiple nested textures");
    }
    void Activate() override {
        if (d.kind == HK_TEX_SCALE && !nested) throw HikariException("ScaleTexture needs a nested texture");
    }
};
struct CheckerboardTexture : TexturePlugin { CheckerboardTexture(const PropertyList &p) : TexturePlugin(p, HK_TEX_CHECKERBOARD) {} };
struct GridTexture : TexturePlugin { GridTexture(const PropertyList &p) : TexturePlugin(p, HK_TEX_GRID) {} };
struct ScaleTexture : TexturePlugin { ScaleTexture(const PropertyList &p) : TexturePlugin(p, HK_TEX_SCALE) {} };
struct BitmapTexture : TexturePlugin { BitmapTexture(const PropertyList &p) : TexturePlugin(p, HK_TEX_BITMAP) {} };
struct WireframeTexture : TexturePlugin { WireframeTexture(const PropertyList &p) : TexturePlugin(p, HK_TEX_WIREFRAME) {} };
struct CurvatureTexture : TexturePlugin { CurvatureTexture(const PropertyList &p) : TexturePlugin(p, HK_TEX_CURVATURE) {} };
HK_REGISTER_CLASS(CheckerboardTexture, "checkerboard")
HK_REGISTER_CLASS(GridTexture, "grid")
HK_REGISTER_CLASS(ScaleTexture, "scale")
HK_REGISTER_CLASS(BitmapTexture, "bitmap")
HK_REGISTER_CLASS(WireframeTexture, "wireframe")
HK_REGISTER_CLASS(CurvatureTexture, "curvature")

// The texture slot (hk_bsdf_desc.tex) of a named BSDF texture child, -1 if the
// BSDF takes no texture of that name (the plugins' AddChild)
int texture_slot(int type, const std::string &name) {
    switch (type) {
    case HK_BSDF_DIFFUSE: return name == "albedo" ? 0 : -1;
    case HK_BSDF_ROUGH_DIFFUSE: return name == "albedo" ? 0 : (name == "alpha" ? 4 : -1);
    case HK_BSDF_CONDUCTOR: return name == "ks" ? 1 : -1;
    case HK_BSDF_DIELECTRIC: return name == "ksReflect" ? 1 : (name == "ksRefract" ? 2 : -1);
    case HK_BSDF_PLASTIC: return name == "kd" ? 0 : (name == "ks" ? 1 : -1);
    case HK_BSDF_ROUGH_PLASTIC: return name == "kd" ? 0 : (name == "ks" ? 1 : (name == "alpha" ? 4 : -1));
    case HK_BSDF_ROUGH_CONDUCTOR:
        return name == "ks" ? 1 : (name == "alpha" || name == "alphaU" ? 4 : (name == "alphaV" ? 5 : -1));
    case HK_BSDF_ROUGH_DIELECTRIC:
        return name == "ksReflect" ? 1 : name == "ksRefract" ? 2 : (name == "alpha" || name == "alphaU") ? 4
                                                                   : name == "alphaV" ? 5 : -1;
    case HK_BSDF_ROUGH_COATING: return name == "ks" ? 1 : (name == "sigmaA" ? 3 : (name == "alpha" ? 4 : -1));
    case HK_BSDF_COATING: return name == "ks" ? 1 : (name == "sigmaA" ? 3 : -1);
    default: return -1;
    }
}

// BSDF plugins: one class per reference type; properties and defaults of
// include/core/Common.hpp:331-392 and the plugin constructors.
class BSDFPlugin : public Object {
public:
    hk_bsdf_desc d{};
    std::unique_ptr<BSDFPlugin> nested;    // roughCoating's BSDF, twoSided's front BSDF
    std::unique_ptr<BSDFPlugin> nested2;   // twoSided's back BSDF
    std::unique_ptr<TexturePlugin> tex[6]; // textured parameters by slot
    BSDFPlugin(const PropertyList &p, int type) {
        std::memset(&d, 0, sizeof d);
        d.type = type;
        d.nested = -1;
        d.nested2 = -1;
        const float air = 1.000277f;
        std::string dist = p.GetString("type", "beckmann");
        if (type >= HK_BSDF_ROUGH_CONDUCTOR && type <= HK_BSDF_ROUGH_COATING) {
            if (dist == "beckmann") d.distribution = HK_BECKMANN;
            else if (dist == "ggx") d.distribution = HK_GGX;
            else throw HikariException("Unexpected distribution type : " + dist);
        }
        auto setc = [](float *dst, const Color3f &c) { dst[0] = c[0]; dst[1] = c[1]; dst[2] = c[2]; };
        Color3f one{1, 1, 1}, half{0.5f, 0.5f, 0.5f}, zero{0, 0, 0};
        d.thickness = 1.0f;
        switch (type) {
        case HK_BSDF_DIFFUSE:
            setc(d.kd, p.GetColor("albedo", half));
            break;
        case HK_BSDF_ROUGH_CONDUCTOR:
            d.int_ior = p.GetFloat("intIOR", 1.5046f);
            d.ext_ior = p.GetFloat("extIOR", air);
            setc(d.k, p.GetColor("k", one));
            setc(d.ks, p.GetColor("ks", one));
            break;
        case HK_BSDF_ROUGH_DIELECTRIC:
            d.int_ior = p.GetFloat("intIOR", 1.5046f);
            d.ext_ior = p.GetFloat("extIOR", air);
            setc(d.ks, p.GetColor("ksReflect", one));
            setc(d.ks_refract, p.GetColor("ksRefract", one));
            break;
        case HK_BSDF_ROUGH_PLASTIC:
            d.int_ior = p.GetFloat("intIOR", 1.49f);
            d.ext_ior = p.GetFloat("extIOR", air);
            setc(d.ks, p.GetColor("ks", one));
            setc(d.kd, p.GetColor("kd", half));
            d.nonlinear = p.GetBoolean("nonlinear", false);
            break;
        case HK_BSDF_ROUGH_COATING:
            d.int_ior = p.GetFloat("intIOR", 1.49f);
            d.ext_ior = p.GetFloat("extIOR", air);
            setc(d.ks, p.GetColor("ks", one));
            setc(d.sigma_a, p.GetColor("sigmaA", zero));
            d.thickness = p.GetFloat("thickness", 1.0f);
            break;
        case HK_BSDF_CONDUCTOR:   // src/bsdf/ConductorBSDF.cpp:9-19
            d.int_ior = p.GetFloat("intIOR", 1.5046f);
            d.ext_ior = p.GetFloat("extIOR", air);
            setc(d.k, p.GetColor("k", one));
            setc(d.ks, p.GetColor("ks", one));
            break;
        case HK_BSDF_DIELECTRIC:   // src/bsdf/DielectricBSDF.cpp:9-20
            d.int_ior = p.GetFloat("intIOR", 1.5046f);
            d.ext_ior = p.GetFloat("extIOR", air);
            setc(d.ks, p.GetColor("ksReflect", one));
            setc(d.ks_refract, p.GetColor("ksRefract", one));
            break;
        case HK_BSDF_PLASTIC:   // src/bsdf/PlasticBSDF.cpp:10-28
            d.int_ior = p.GetFloat("intIOR", 1.5046f);
            d.ext_ior = p.GetFloat("extIOR", air);
            setc(d.ks, p.GetColor("ks", one));
            setc(d.kd, p.GetColor("kd", half));
            d.nonlinear = p.GetBoolean("nonlinear", false);
            break;
        case HK_BSDF_COATING:   // src/bsdf/CoatingBSDF.cpp:9-23
            d.int_ior = p.GetFloat("intIOR", 1.49f);
            d.ext_ior = p.GetFloat("extIOR", air);
            d.thickness = p.GetFloat("thickness", 1.0f);
            setc(d.sigma_a, p.GetColor("sigmaA", zero));
            setc(d.ks, p.GetColor("ks", one));
            break;
        case HK_BSDF_ROUGH_DIFFUSE:   // src/bsdf/RoughDiffuseBSDF.cpp:10-17
            setc(d.kd, p.GetColor("albedo", half));
            d.fast_approx = p.GetBoolean("fastApprox", false);
            break;
        default:   // mirror, twoSided: no properties
            d.int_ior = d.ext_ior = 1.0f;
            break;
        }
        if (type == HK_BSDF_ROUGH_CONDUCTOR || type == HK_BSDF_ROUGH_DIELECTRIC) d.anisotropic = p.GetBoolean("as", false);
        auto clampa = [](float a) { return a < 5e-4f ? 5e-4f : (a > 1.0f ? 1.0f : a); };
        if (d.anisotropic) {
            d.alpha_u = clampa(p.GetFloat("alphaU", 0.1f));
            d.alpha_v = clampa(p.GetFloat("alphaV", 0.1f));
        } else {
            d.alpha_u = d.alpha_v = clampa(p.GetFloat("alpha", type == HK_BSDF_ROUGH_DIFFUSE ? 0.2f : 0.1f));
        }
        float e = d.ext_ior != 0.0f ? d.int_ior / d.ext_ior : 0.0f;
        d.eta[0] = d.eta[1] = d.eta[2] = e;
    }
    EClassType GetClassType() const override { return EClassType::EBSDF; }
    void AddChild(Object *c, const std::string &name) override {
        const bool wrap = d.type == HK_BSDF_BUMP_MAP || d.type == HK_BSDF_NORMAL_MAP;
        if (wrap) {   // BumpMapBSDF / NormalMapBSDF::AddChild: one BSDF, one map texture (any name)
            const bool is_tex = c->GetClassType() == EClassType::ETexture;
            if (is_tex ? (bool)tex[0] : (bool)nested || c->GetClassType() != EClassType::EBSDF) {
                delete c;
                throw HikariException(type_name + (is_tex ? ": tried to specify multiple map textures"
                                                          : ": tried to specify multiple nested BSDF"));
            }
            if (is_tex) tex[0].reset((TexturePlugin *)c);
            else nested.reset((BSDFPlugin *)c);
            return;
        }
        if (c->GetClassType() == EClassType::ETexture) {
            const int slot = texture_slot(d.type, name);
            if (slot < 0 || tex[slot]) {
                delete c;
                throw HikariException(type_name + ": a texture named \"" + name + "\" is not supported");
            }
            tex[slot].reset((TexturePlugin *)c);
            return;
        }
        if ((d.type == HK_BSDF_ROUGH_COATING || d.type == HK_BSDF_COATING) && c->GetClassType() == EClassType::EBSDF) {
            if (nested) {
                delete c;
                throw HikariException(std::string(d.type == HK_BSDF_COATING ? "CoatingBSDF" : "RoughCoatingBSDF") +
                                      ": tried to specify multiple nested BSDF");
            }
            nested.reset((BSDFPlugin *)c);
            return;
        }
        if (d.type == HK_BSDF_TWO_SIDED && c->GetClassType() == EClassType::EBSDF) {   // TwoSidedBSDF.cpp:75
            if (!nested) nested.reset((BSDFPlugin *)c);
            else if (!nested2) nested2.reset((BSDFPlugin *)c);
            else {
                delete c;
                throw HikariException("TwoSidedBSDF: tried to specify the third nested BSDF");
            }
            return;
        }
        delete c;
        throw HikariException(type_name + "::AddChild(<" + class_name(c->GetClassType()) + ">, <" + name +
                              ">) is not supported!");
    }
    void Activate() override {
        if (d.type == HK_BSDF_ROUGH_COATING && !nested) throw HikariException("RoughCoatingBSDF needs a nested BSDF!");
        if (d.type == HK_BSDF_COATING && !nested) throw HikariException("CoatingBSDF needs a nested BSDF!");
        if ((d.type == HK_BSDF_BUMP_MAP || d.type == HK_BSDF_NORMAL_MAP) && (!nested || !tex[0]))
            throw HikariException(type_name + " needs a nested BSDF and a map texture");
        if (d.type == HK_BSDF_TWO_SIDED) {   // TwoSidedBSDF::Activate :98
            if (!nested) throw HikariException("TwoSidedBSDF needs at least one nested BSDF!");
            if (nested->transmits() || (nested2 && nested2->transmits()))
                throw HikariException("Only BSDF without transmission can be nested!");
        }
    }
    bool transmits() const {
        if (d.type == HK_BSDF_ROUGH_DIELECTRIC || d.type == HK_BSDF_DIELECTRIC) return true;
        return (nested && nested->transmits()) || (nested2 && nested2->transmits());
    }
};
struct DiffuseBSDF : BSDFPlugin { DiffuseBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_DIFFUSE) {} };
struct RoughConductorBSDF : BSDFPlugin { RoughConductorBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_ROUGH_CONDUCTOR) {} };
struct RoughDielectricBSDF : BSDFPlugin { RoughDielectricBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_ROUGH_DIELECTRIC) {} };
struct RoughPlasticBSDF : BSDFPlugin { RoughPlasticBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_ROUGH_PLASTIC) {} };
struct RoughCoatingBSDF : BSDFPlugin { RoughCoatingBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_ROUGH_COATING) {} };
HK_REGISTER_CLASS(DiffuseBSDF, "diffuse")
HK_REGISTER_CLASS(RoughConductorBSDF, "roughConductor")
HK_REGISTER_CLASS(RoughDielectricBSDF, "roughDielectric")
HK_REGISTER_CLASS(RoughPlasticBSDF, "roughPlastic")
HK_REGISTER_CLASS(RoughCoatingBSDF, "roughCoating")
struct MirrorBSDF : BSDFPlugin { MirrorBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_MIRROR) {} };
struct ConductorBSDF : BSDFPlugin { ConductorBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_CONDUCTOR) {} };
struct DielectricBSDF : BSDFPlugin { DielectricBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_DIELECTRIC) {} };
struct PlasticBSDF : BSDFPlugin { PlasticBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_PLASTIC) {} };
struct TwoSidedBSDF : BSDFPlugin { TwoSidedBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_TWO_SIDED) {} };
struct BumpMapBSDF : BSDFPlugin { BumpMapBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_BUMP_MAP) {} };
struct NormalMapBSDF : BSDFPlugin { NormalMapBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_NORMAL_MAP) {} };
HK_REGISTER_CLASS(BumpMapBSDF, "bumpMap")
HK_REGISTER_CLASS(NormalMapBSDF, "normalMap")
HK_REGISTER_CLASS(MirrorBSDF, "mirror")
HK_REGISTER_CLASS(ConductorBSDF, "conductor")
HK_REGISTER_CLASS(DielectricBSDF, "dielectric")
HK_REGISTER_CLASS(PlasticBSDF, "plastic")
HK_REGISTER_CLASS(TwoSidedBSDF, "twoSided")
struct CoatingBSDF : BSDFPlugin { CoatingBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_COATING) {} };
struct RoughDiffuseBSDF : BSDFPlugin { RoughDiffuseBSDF(const PropertyList &p) : BSDFPlugin(p, HK_BSDF_ROUGH_DIFFUSE) {} };
HK_REGISTER_CLASS(CoatingBSDF, "coating")
HK_REGISTER_CLASS(RoughDiffuseBSDF, "roughDiffuse")

class Mesh;
// Emitters: AreaLight (src/emitter/AreaLight.cpp:8), EnvironmentLight (src/emitter/EnvironmentLight.cpp:8)
class AreaLight : public Object {
public:
    Color3f radiance;
    Object *mesh = nullptr;
    explicit AreaLight(const PropertyList &p) : radiance(p.GetColor("radiance")) {}
    EClassType GetClassType() const override { return EClassType::EEmitter; }
    void SetParent(Object *parent, const std::string &) override {
        if (parent->GetClassType() != EClassType::EMesh)
            throw HikariException("AreaLight::SetParent(<" + std::string(class_name(parent->GetClassType())) +
                                  ">) is not supported!");
        mesh = parent;
    }
};
HK_REGISTER_CLASS(AreaLight, "area")

class EnvironmentLight : public Object {
public:
    float scale;
    Matrix4f to_world;
    int w = 0, h = 0;
    std::vector<float> rgb;
    explicit EnvironmentLight(const PropertyList &p) {
        scale = p.GetFloat("scale", 1.0f);
        to_world = p.GetTransform("toWorld", identity4());
        ReadEXR(resolve(p.GetString("filename")), w, h, rgb);
    }
    EClassType GetClassType() const override { return EClassType::EEmitter; }
};
HK_REGISTER_CLASS(EnvironmentLight, "env")

// ConstantLight (src/emitter/ConstantLight.cpp:8): an environment emitter of one radiance
class ConstantLight : public Object {
public:
    Color3f radiance;
    explicit ConstantLight(const PropertyList &p) : radiance(p.GetColor("radiance")) {}
    EClassType GetClassType() const override { return EClassType::EEmitter; }
};
HK_REGISTER_CLASS(ConstantLight, "constant")

// PointLight (src/emitter/PointLight.cpp:8) and DirectionalLight (src/emitter/DirectionalLight.cpp:8)
class DeltaLight : public Object {
public:
    bool directional;
    Color3f color, vec;   // power and position, or irradiance and direction
    DeltaLight(const PropertyList &p, bool dir)
        : directional(dir), color(p.GetColor(dir ? "irradiance" : "power")),
          vec(dir ? p.GetVector("direction") : p.GetPoint("position")) {}
    EClassType GetClassType() const override { return EClassType::EEmitter; }
};
struct PointLight : DeltaLight { explicit PointLight(const PropertyList &p) : DeltaLight(p, false) {} };
struct DirectionalLight : DeltaLight { explicit DirectionalLight(const PropertyList &p) : DeltaLight(p, true) {} };
HK_REGISTER_CLASS(PointLight, "point")
HK_REGISTER_CLASS(DirectionalLight, "directional")

// WavefrontObjMesh (src/mesh/WavefrontObjMesh.cpp:10-152)
class Mesh : public Object {
public:
    std::vector<float> pos, nrm, uv;
    std::vector<uint32_t> idx;
    std::unique_ptr<BSDFPlugin> bsdf;
    std::unique_ptr<AreaLight> emitter;
    explicit Mesh(const PropertyList &p) {
        std::string fn = resolve(p.GetString("filename"));
        Matrix4f M = p.GetTransform("toWorld", identity4());
        Matrix4f Minv;
        if (!inverse4(M, Minv)) throw HikariException("mesh toWorld is singular");
        try {
            ObjMesh m = load_obj(fn, M.data(), Minv.data());
            pos.swap(m.pos);
            nrm.swap(m.nrm);
            uv.swap(m.uv);
            idx.swap(m.idx);
        } catch (const std::runtime_error &e) {
            throw HikariException(e.what());
        }
    }
    EClassType GetClassType() const override { return EClassType::EMesh; }
    void AddChild(Object *c, const std::string &name) override {
        if (c->GetClassType() == EClassType::EBSDF) {
            if (bsdf) throw HikariException("Mesh: tried to register multiple BSDF instances!");
            bsdf.reset((BSDFPlugin *)c);
        } else if (c->GetClassType() == EClassType::EEmitter) {
            AreaLight *a = dynamic_cast<AreaLight *>(c);
            if (!a) { delete c; throw HikariException("Mesh: only area emitters attach to meshes"); }
            if (emitter) throw HikariException("Mesh: tried to register multiple Emitter instances!");
            emitter.reset(a);
        } else {
            delete c;
            throw HikariException("Mesh::AddChild(<" + std::string(class_name(c->GetClassType())) + ">, <" + name +
                                  ">) is not supported!");
        }
    }
    void Activate() override {
        if (!bsdf) bsdf.reset(new DiffuseBSDF(PropertyList()));   // DEFAULT_MESH_BSDF (Mesh.cpp:235)
    }
};
HK_REGISTER_CLASS(Mesh, "obj")

// PerspectiveCamera + reconstruction filters
class Filter : public Object {
public:
    int kind;
    float radius, p0, p1;
    Filter(const PropertyList &p, int k) : kind(k) {
        if (k == 0) { radius = 0.5f; p0 = p1 = 0; }
        else if (k == 1) { radius = 1.0f; p0 = p1 = 0; }
        else if (k == 2) { radius = p.GetFloat("radius", 2.0f); p0 = p.GetFloat("stddev", 0.5f); p1 = 0; }
        else { radius = p.GetFloat("radius", 2.0f); p0 = p.GetFloat("B", 1.0f / 3.0f); p1 = p.GetFloat("C", 1.0f / 3.0f); }
    }
    EClassType GetClassType() const override { return EClassType::EReconstructionFilter; }
};
struct BoxFilter : Filter { BoxFilter(const PropertyList &p) : Filter(p, 0) {} };
struct TentFilter : Filter { TentFilter(const PropertyList &p) : Filter(p, 1) {} };
struct GaussianFilter : Filter { GaussianFilter(const PropertyList &p) : Filter(p, 2) {} };
struct MitchellNetravaliFilter : Filter { MitchellNetravaliFilter(const PropertyList &p) : Filter(p, 3) {} };
HK_REGISTER_CLASS(BoxFilter, "box")
HK_REGISTER_CLASS(TentFilter, "tent")
HK_REGISTER_CLASS(GaussianFilter, "gaussian")
HK_REGISTER_CLASS(MitchellNetravaliFilter, "mitchell")

class PerspectiveCamera : public Object {
public:
    int width, height;
    Matrix4f to_world;
    float fov, near_clip, far_clip;
    std::unique_ptr<Filter> filter;
    explicit PerspectiveCamera(const PropertyList &p) {
        width = p.GetInteger("width", 1280);
        height = p.GetInteger("height", 720);
        to_world = p.GetTransform("toWorld", identity4());
        fov = p.GetFloat("fov", 30.0f);
        near_clip = p.GetFloat("nearClip", 1e-4f);
        far_clip = p.GetFloat("farClip", 1e4f);
    }
    EClassType GetClassType() const override { return EClassType::ECamera; }
    void AddChild(Object *c, const std::string &name) override {
        if (c->GetClassType() != EClassType::EReconstructionFilter) {
            delete c;
            throw HikariException("Camera::AddChild(<" + std::string(class_name(c->GetClassType())) + ">, <" + name +
                                  ">) is not supported!");
        }
        if (filter) throw HikariException("Camera: tried to register multiple reconstruction filters!");
        filter.reset((Filter *)c);
    }
    void Activate() override {
        if (!filter) filter.reset(new GaussianFilter(PropertyList()));   // DEFAULT_CAMERA_RFILTER
    }
};
HK_REGISTER_CLASS(PerspectiveCamera, "perspective")

class IndependentSampler : public Object {
public:
    int sample_count;
    explicit IndependentSampler(const PropertyList &p) : sample_count(p.GetInteger("sampleCount", 1)) {}
    EClassType GetClassType() const override { return EClassType::ESampler; }
};
HK_REGISTER_CLASS(IndependentSampler, "independent")

// pathMIS (src/integrator/PathMISIntegrator.cpp:11): "depth" is required.
// "pathMISCuda" is the same integrator under the name of the CUDA drop-in.
class PathMISIntegrator : public Object {
public:
    int depth;
    explicit PathMISIntegrator(const PropertyList &p) : depth(p.GetInteger("depth")) {}
    EClassType GetClassType() const override { return EClassType::EIntegrator; }
};
HK_REGISTER_CLASS(PathMISIntegrator, "pathMIS")
struct PathMISCudaIntegrator : PathMISIntegrator { PathMISCudaIntegrator(const PropertyList &p) : PathMISIntegrator(p) {} };
HK_REGISTER_CLASS(PathMISCudaIntegrator, "pathMISCuda")
// The reference's other estimators parse (their XML files mix them with
// pathMIS scenes) but do not run on the CUDA core.
class ParseOnlyIntegrator : public Object {
public:
    explicit ParseOnlyIntegrator(const PropertyList &) {}
    EClassType GetClassType() const override { return EClassType::EIntegrator; }
};
struct PathEMSIntegrator : ParseOnlyIntegrator { PathEMSIntegrator(const PropertyList &p) : ParseOnlyIntegrator(p) {} };
struct PathMATSIntegrator : ParseOnlyIntegrator { PathMATSIntegrator(const PropertyList &p) : ParseOnlyIntegrator(p) {} };
HK_REGISTER_CLASS(PathEMSIntegrator, "pathEMS")
HK_REGISTER_CLASS(PathMATSIntegrator, "pathMATS")

// Accelerations are accepted and ignored: the CUDA core builds its own BVH.
class AccelPlugin : public Object {
public:
    explicit AccelPlugin(const PropertyList &) {}
    EClassType GetClassType() const override { return EClassType::EAcceleration; }
};
struct BrutoAccel : AccelPlugin { BrutoAccel(const PropertyList &p) : AccelPlugin(p) {} };
struct BVHAccel : AccelPlugin { BVHAccel(const PropertyList &p) : AccelPlugin(p) {} };
struct HLBVHAccel : AccelPlugin { HLBVHAccel(const PropertyList &p) : AccelPlugin(p) {} };
HK_REGISTER_CLASS(BrutoAccel, "bruto")
HK_REGISTER_CLASS(BVHAccel, "bvh")
HK_REGISTER_CLASS(HLBVHAccel, "hlbvh")

// Scene (src/core/Scene.cpp): AddChild order fixes the emitter order.
class Scene : public Object {
public:
    Color3f background;
    bool force_background;
    std::vector<std::unique_ptr<Mesh>> meshes;
    std::unique_ptr<EnvironmentLight> env;
    std::unique_ptr<ConstantLight> env_constant;
    int env_position = -1;   // emitter index of the environment (map or constant)
    std::vector<std::pair<int, std::unique_ptr<DeltaLight>>> delta_lights;   // (emitter index, light)
    int n_emitters = 0;
    std::unique_ptr<PerspectiveCamera> camera;
    std::unique_ptr<PathMISIntegrator> integrator;
    std::unique_ptr<Object> other_integrator;   // parsed, not runnable on the CUDA core
    std::unique_ptr<IndependentSampler> sampler;
    std::unique_ptr<Object> accel;
    explicit Scene(const PropertyList &p) {
        background = p.GetColor("background", {0, 0, 0});
        force_background = p.GetBoolean("forceBackground", false);
    }
    EClassType GetClassType() const override { return EClassType::EScene; }
    void AddChild(Object *c, const std::string &name) override {
        switch (c->GetClassType()) {
        case EClassType::EMesh:
            meshes.emplace_back((Mesh *)c);
            if (meshes.back()->emitter) n_emitters++;
            break;
        case EClassType::EEmitter: {
            if (DeltaLight *d = dynamic_cast<DeltaLight *>(c)) {   // Scene.cpp:186: point and directional
                delta_lights.emplace_back(n_emitters++, std::unique_ptr<DeltaLight>(d));
                break;
            }
            EnvironmentLight *e = dynamic_cast<EnvironmentLight *>(c);
            ConstantLight *k = dynamic_cast<ConstantLight *>(c);
            if (!e && !k) { delete c; throw HikariException("Scene::AddChild(): You need to implement this for emitters"); }
            if (env || env_constant) { delete c; throw HikariException("Scene::AddChild(): Only one environment emiiter is allowed for the entire scene"); }
            if (e) env.reset(e);
            else env_constant.reset(k);
            env_position = n_emitters++;
            break;
        }
        case EClassType::ECamera:
            if (camera) { delete c; throw HikariException("There can only be one camera per scene!"); }
            camera.reset((PerspectiveCamera *)c);
            break;
        case EClassType::EIntegrator:
            if (integrator) { delete c; throw HikariException("There can only be one integrator per scene!"); }
            if (dynamic_cast<PathMISIntegrator *>(c)) integrator.reset((PathMISIntegrator *)c);
            else other_integrator.reset(c);
            break;
        case EClassType::ESampler:
            if (sampler) { delete c; throw HikariException("There can only be one sampler per scene!"); }
            sampler.reset((IndependentSampler *)c);
            break;
        case EClassType::EAcceleration:
            if (accel) { delete c; throw HikariException("There can only be one acceleration per scene!"); }
            accel.reset(c);
            break;
        default:
            delete c;
            throw HikariException("Scene::AddChild(<" + std::string(class_name(c->GetClassType())) + ">, <" + name +
                                  ">) is not supported!");
        }
    }
    void Activate() override {   // Scene::Activate (src/core/Scene.cpp:128)
        if (!integrator && !other_integrator) throw HikariException("No integrator was specified!");
        if (!camera) throw HikariException("No camera was specified!");
        if (!sampler) sampler.reset(new IndependentSampler(PropertyList()));
    }
};
HK_REGISTER_CLASS(Scene, "scene")

// <test type="ttest"> holding scenes (src/core/StudentTTest.cpp) -- parsed for
// its scenes; the statistics run in the test harness.
class TTest : public Object {
public:
    std::vector<std::unique_ptr<Scene>> scenes;
    std::vector<float> references;
    explicit TTest(const PropertyList &p) {
        for (auto &t : tokenize(p.GetString("references", ""))) references.push_back(to_float(t));
    }
    EClassType GetClassType() const override { return EClassType::ETest; }
    void AddChild(Object *c, const std::string &) override {
        if (c->GetClassType() != EClassType::EScene) { delete c; throw HikariException("ttest children must be scenes"); }
        scenes.emplace_back((Scene *)c);
    }
};
HK_REGISTER_CLASS(TTest, "ttest")

// Upload a parsed Scene through the C ABI (Integrator::Preprocess).
int upload_scene(const Scene &sc, const std::string &data_dir, hk_scene *h) {
    int rc;
    for (int dist = 0; dist < 2; ++dist) {
        std::string fn = data_dir + (dist ? "/GGXRFTData.bin" : "/BeckmannRFTData.bin");
        std::ifstream f(fn, std::ios::binary);
        if (!f) throw HikariException("Load rough fresnel transmittance data \"" + fn + "\" failed.");
        std::vector<char> bytes((std::istreambuf_iterator<char>(f)), std::istreambuf_iterator<char>());
        if ((rc = hk_scene_set_rft(h, dist, bytes.data(), bytes.size())) != HK_OK) return rc;
    }
    // nested BSDFs first, so that the parent can name their ids
    std::function<int32_t(const TexturePlugin &)> add_texture = [&](const TexturePlugin &t) -> int32_t {
        hk_texture_desc d = t.d;
        if (t.nested) d.nested = add_texture(*t.nested);
        int32_t id;
        rc = d.kind == HK_TEX_BITMAP ? hk_scene_add_bitmap(h, &d, t.pixels.data(), t.width, t.height, &id)
                                     : hk_scene_add_texture(h, &d, &id);
        if (rc != HK_OK) throw HikariException(hk_last_error());
        return id;
    };
    std::function<int32_t(const BSDFPlugin &)> add_bsdf = [&](const BSDFPlugin &b) -> int32_t {
        hk_bsdf_desc d = b.d;
        if (b.nested) d.nested = add_bsdf(*b.nested);
        if (b.nested2) d.nested2 = add_bsdf(*b.nested2);
        for (int k = 0; k < 6; k++)
            if (b.tex[k]) d.tex[k] = 1 + add_texture(*b.tex[k]);
        int32_t id;
        if ((rc = hk_scene_add_bsdf(h, &d, &id)) != HK_OK) throw HikariException(hk_last_error());
        return id;
    };
    // non-mesh emitters go in before the mesh emitter they precede (Scene::AddChild order)
    int emitted = 0;
    bool env_done = false;
    size_t next_delta = 0;
    auto add_pending = [&](bool all) {
        for (;;) {
            if ((sc.env || sc.env_constant) && !env_done && (all || emitted == sc.env_position) &&
                (next_delta == sc.delta_lights.size() || sc.env_position < sc.delta_lights[next_delta].first)) {
                if (sc.env) {
                    const EnvironmentLight &e = *sc.env;
                    rc = hk_scene_set_envmap(h, e.rgb.data(), (uint32_t)e.w, (uint32_t)e.h, e.to_world.data(), e.scale);
                } else {
                    rc = hk_scene_set_constant_light(h, sc.env_constant->radiance.data());
                }
                if (rc != HK_OK) throw HikariException(hk_last_error());
                env_done = true;
                emitted++;
            } else if (next_delta < sc.delta_lights.size() && (all || emitted == sc.delta_lights[next_delta].first)) {
                const DeltaLight &l = *sc.delta_lights[next_delta].second;
                rc = l.directional ? hk_scene_add_directional_light(h, l.color.data(), l.vec.data())
                                   : hk_scene_add_point_light(h, l.color.data(), l.vec.data());
                if (rc != HK_OK) throw HikariException(hk_last_error());
                next_delta++;
                emitted++;
            } else {
                break;
            }
        }
    };
    for (auto &m : sc.meshes) {
        add_pending(false);
        int32_t bid = add_bsdf(*m->bsdf);
        const float *rad = m->emitter ? m->emitter->radiance.data() : nullptr;
        int32_t mid = -1;
        if ((rc = hk_scene_add_mesh(h, m->pos.data(), (uint32_t)(m->pos.size() / 3), m->idx.data(),
                                    (uint32_t)(m->idx.size() / 3), m->nrm.empty() ? nullptr : m->nrm.data(), bid, rad,
                                    &mid)) != HK_OK)
            throw HikariException(hk_last_error());
        if (!m->uv.empty() && (rc = hk_scene_set_mesh_uv(h, mid, m->uv.data())) != HK_OK)
            throw HikariException(hk_last_error());
        if (rad) emitted++;
    }
    add_pending(true);
    const PerspectiveCamera &c = *sc.camera;
    if ((rc = hk_scene_set_camera(h, (uint32_t)c.width, (uint32_t)c.height, c.to_world.data(), c.fov, c.near_clip,
                                  c.far_clip)) != HK_OK)
        throw HikariException(hk_last_error());
    if ((rc = hk_scene_set_filter(h, c.filter->kind, c.filter->radius, c.filter->p0, c.filter->p1)) != HK_OK)
        throw HikariException(hk_last_error());
    if ((rc = hk_scene_set_background(h, sc.background.data(), sc.force_background)) != HK_OK)
        throw HikariException(hk_last_error());
    return HK_OK;
}

thread_local std::string g_xml_error;

}  // namespace
}  // namespace hikari

extern "C" int hk_scene_load_xml_impl(const char *path, const char *data_dir, hk_scene **out, int32_t *depth,
                                      int32_t *spp, int build, std::string *err) {
    using namespace hikari;
    hk_scene *h = nullptr;
    try {
        std::unique_ptr<Object> root = LoadFromXML(path);
        Scene *sc = dynamic_cast<Scene *>(root.get());
        if (!sc) throw HikariException("root element of \"" + std::string(path) + "\" is not a <scene>");
        if (!sc->integrator) throw HikariException("only the pathMIS integrator runs on the CUDA core");
        int rc = hk_scene_create(&h);
        if (rc != HK_OK) return rc;
        rc = upload_scene(*sc, data_dir ? data_dir : ".", h);
        if (rc == HK_OK && build) rc = hk_scene_build(h);
        if (rc != HK_OK) { *err = hk_last_error(); hk_scene_destroy(h); return rc; }
        if (depth) *depth = sc->integrator->depth;
        if (spp) *spp = sc->sampler->sample_count;
        *out = h;
        return HK_OK;
    } catch (const std::exception &e) {
        if (h) hk_scene_destroy(h);
        *err = e.what();
        return HK_ERR_INVALID;
    }
}

extern "C" int hk_exr_read_impl(const char *path, int *w, int *h, std::vector<float> *rgb, std::string *err) {
    try {
        hikari::ReadEXR(path, *w, *h, *rgb);
        return HK_OK;
    } catch (const std::exception &e) {
        *err = e.what();
        return HK_ERR_IO;
    }
}
extern "C" int hk_exr_write_impl(const char *path, int w, int h, const float *rgb, std::string *err) {
    try {
        hikari::WriteEXR(path, w, h, rgb);
        return HK_OK;
    } catch (const std::exception &e) {
        *err = e.what();
        return HK_ERR_IO;
    }
}

namespace hikari {
bool invert4(const float *m, float *out) {
    Matrix4f a, b;
    std::memcpy(a.data(), m, sizeof a);
    if (!inverse4(a, b)) return false;
    std::memcpy(out, b.data(), sizeof b);
    return true;
}
}  // namespace hikari
