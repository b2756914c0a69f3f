// C++ plugin layer mirroring Hikari's object model (include/core/Object.hpp,
// include/core/PropertyList.hpp, src/core/Parser.cpp): a string-keyed object
// factory, typed property lists, the XML loader and the plugin classes of the
// pathMIS path.  A parsed Scene uploads itself to the CUDA core through the C
// ABI of include/hikari_b200.h (the Integrator::Preprocess hook).
#pragma once
#include <array>
#include <functional>
#include <map>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/hikari_b200.h"

namespace hikari {

class HikariException : public std::runtime_error {
public:
    explicit HikariException(const std::string &m) : std::runtime_error(m) {}
};

using Color3f = std::array<float, 3>;
using Matrix4f = std::array<float, 16>;   // row-major

// PropertyList (include/core/PropertyList.hpp:13-125): typed name -> value map;
// a getter without default throws when the property is missing, every getter
// throws on a type mismatch.
class PropertyList {
public:
    void SetBoolean(const std::string &n, bool v) { set(n, Value{kBool, v, 0, 0.0f, {}, {}, {}}); }
    void SetInteger(const std::string &n, int v) { set(n, Value{kInt, false, v, 0.0f, {}, {}, {}}); }
    void SetFloat(const std::string &n, float v) { set(n, Value{kFloat, false, 0, v, {}, {}, {}}); }
    void SetString(const std::string &n, const std::string &v) { set(n, Value{kString, false, 0, 0.0f, v, {}, {}}); }
    void SetColor(const std::string &n, const Color3f &v) { set(n, Value{kColor, false, 0, 0.0f, {}, v, {}}); }
    void SetPoint(const std::string &n, const Color3f &v) { set(n, Value{kPoint, false, 0, 0.0f, {}, v, {}}); }
    void SetVector(const std::string &n, const Color3f &v) { set(n, Value{kVector, false, 0, 0.0f, {}, v, {}}); }
    void SetTransform(const std::string &n, const Matrix4f &v) { set(n, Value{kTransform, false, 0, 0.0f, {}, {}, v}); }

    bool GetBoolean(const std::string &n) const { return get(n, kBool).b; }
    bool GetBoolean(const std::string &n, bool d) const { return has(n) ? get(n, kBool).b : d; }
    int GetInteger(const std::string &n) const { return get(n, kInt).i; }
    int GetInteger(const std::string &n, int d) const { return has(n) ? get(n, kInt).i : d; }
    float GetFloat(const std::string &n) const { return get(n, kFloat).f; }
    float GetFloat(const std::string &n, float d) const { return has(n) ? get(n, kFloat).f : d; }
    std::string GetString(const std::string &n) const { return get(n, kString).s; }
    std::string GetString(const std::string &n, const std::string &d) const { return has(n) ? get(n, kString).s : d; }
    Color3f GetColor(const std::string &n) const { return get(n, kColor).c; }
    Color3f GetColor(const std::string &n, const Color3f &d) const { return has(n) ? get(n, kColor).c : d; }
    Color3f GetPoint(const std::string &n) const { return get(n, kPoint).c; }
    Color3f GetVector(const std::string &n) const { return get(n, kVector).c; }
    Matrix4f GetTransform(const std::string &n, const Matrix4f &d) const { return has(n) ? get(n, kTransform).m : d; }
    bool has(const std::string &n) const { return m_.count(n) != 0; }

private:
    enum Kind { kBool, kInt, kFloat, kString, kColor, kPoint, kVector, kTransform };
    struct Value {
        Kind k;
        bool b;
        int i;
        float f;
        std::string s;
        Color3f c;
        Matrix4f m;
    };
    void set(const std::string &n, Value v) {
        if (m_.count(n)) throw HikariException("Property \"" + n + "\" was specified multiple times!");
        m_[n] = std::move(v);
    }
    const Value &get(const std::string &n, Kind k) const {
        auto it = m_.find(n);
        if (it == m_.end()) throw HikariException("Property '" + n + "' is missing!");
        if (it->second.k != k) throw HikariException("Property '" + n + "' has the wrong type!");
        return it->second;
    }
    std::map<std::string, Value> m_;
};

enum class EClassType { EScene, EMesh, EBSDF, EEmitter, ECamera, EIntegrator, ESampler, EReconstructionFilter,
                        EAcceleration, ETest, ETexture };

// Object (include/core/Object.hpp:26): lifecycle ctor -> AddChild -> SetParent -> Activate
class Object {
public:
    virtual ~Object() = default;
    virtual EClassType GetClassType() const = 0;
    virtual void AddChild(Object *child, const std::string &name);
    virtual void SetParent(Object *, const std::string &) {}
    virtual void Activate() {}
    std::string type_name;
};

// ObjectFactory (include/core/Object.hpp:92-149): string-keyed constructors
class ObjectFactory {
public:
    using Constructor = std::function<Object *(const PropertyList &)>;
    static void RegisterClass(const std::string &name, const Constructor &c);
    static Object *CreateInstance(const std::string &name, const PropertyList &props);
    static bool Exists(const std::string &name);
};

// LoadFromXML (src/core/Parser.cpp:9): returns the root object (owned by the caller)
std::unique_ptr<Object> LoadFromXML(const std::string &filename);

// Read an RGB(A) OpenEXR scanline image (NONE / ZIPS / ZIP compression, HALF or
// FLOAT channels) into H*W*3 floats (src/core/Bitmap.cpp:14).
void ReadEXR(const std::string &filename, int &width, int &height, std::vector<float> &rgb);
// Write H*W*3 floats as an uncompressed FLOAT RGB OpenEXR (src/core/Bitmap.cpp:76).
void WriteEXR(const std::string &filename, int width, int height, const float *rgb);

}  // namespace hikari
