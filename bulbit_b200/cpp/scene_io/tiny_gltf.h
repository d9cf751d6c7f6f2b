// glTF 2.0 reader for the reference CLI's model loader (cli/model_loader.cpp:
// LoadGLTF, LoadMaterials, LoadMesh, ProcessNode), which is written against
// tinygltf's API (tinygltf v2.9.6, fetched by the reference's
// cli/CMakeLists.txt and not part of this image). This header declares the
// model types, the Value type of extension data and the TinyGLTF loader with
// the same names, fields, defaults and numeric constants; gltf_reader.cpp
// implements them with a JSON reader of this project's own.
//
// What is read: .gltf (JSON with buffers given as relative files or base64
// data URIs) and .glb (binary container: JSON chunk plus BIN chunk, which a
// buffer without a uri refers to); asset, scene, scenes, nodes (matrix and
// TRS), meshes and primitives (attributes, indices, material, mode), accessors,
// bufferViews, buffers, materials (PBR metallic-roughness, normal, occlusion
// and emissive textures, alpha mode, extensions as Values), textures, images
// (uri, bufferView, mimeType; their bytes go to the image loader callback when
// there are any) and samplers. Unlike tinygltf, the reader also refuses a file
// whose indices or byte ranges reach outside its arrays or buffers (accessor
// -> bufferView -> buffer, primitive / material / node / scene / texture
// indices) or whose node hierarchy has a cycle, so that code walking a loaded
// Model without checks stays in bounds; -1 keeps its glTF meaning of "absent"
// where the format allows it. Skins, animations, cameras, lights and sparse
// accessors are not read.
#pragma once

#include <cstddef>
#include <functional>
#include <map>
#include <string>
#include <vector>

// Data types and modes, as glTF numbers them.
#define TINYGLTF_MODE_POINTS (0)
#define TINYGLTF_MODE_LINE (1)
#define TINYGLTF_MODE_LINE_LOOP (2)
#define TINYGLTF_MODE_LINE_STRIP (3)
#define TINYGLTF_MODE_TRIANGLES (4)
#define TINYGLTF_MODE_TRIANGLE_STRIP (5)
#define TINYGLTF_MODE_TRIANGLE_FAN (6)

#define TINYGLTF_COMPONENT_TYPE_BYTE (5120)
#define TINYGLTF_COMPONENT_TYPE_UNSIGNED_BYTE (5121)
#define TINYGLTF_COMPONENT_TYPE_SHORT (5122)
#define TINYGLTF_COMPONENT_TYPE_UNSIGNED_SHORT (5123)
#define TINYGLTF_COMPONENT_TYPE_INT (5124)
#define TINYGLTF_COMPONENT_TYPE_UNSIGNED_INT (5125)
#define TINYGLTF_COMPONENT_TYPE_FLOAT (5126)
#define TINYGLTF_COMPONENT_TYPE_DOUBLE (5130)

// Accessor element types (the reader maps glTF's "SCALAR", "VEC3", ... names
// to these numbers, as tinygltf does).
#define TINYGLTF_TYPE_VEC2 (2)
#define TINYGLTF_TYPE_VEC3 (3)
#define TINYGLTF_TYPE_VEC4 (4)
#define TINYGLTF_TYPE_MAT2 (32 + 2)
#define TINYGLTF_TYPE_MAT3 (32 + 3)
#define TINYGLTF_TYPE_MAT4 (32 + 4)
#define TINYGLTF_TYPE_SCALAR (64 + 1)
#define TINYGLTF_TYPE_VECTOR (64 + 4)
#define TINYGLTF_TYPE_MATRIX (64 + 16)

#define TINYGLTF_TARGET_ARRAY_BUFFER (34962)
#define TINYGLTF_TARGET_ELEMENT_ARRAY_BUFFER (34963)

namespace tinygltf
{

enum Type
{
    NULL_TYPE,
    REAL_TYPE,
    INT_TYPE,
    BOOL_TYPE,
    STRING_TYPE,
    ARRAY_TYPE,
    BINARY_TYPE,
    OBJECT_TYPE
};

// Bytes per component of a TINYGLTF_COMPONENT_TYPE_*, -1 if unknown.
int GetComponentSizeInBytes(unsigned int component_type);
// Components per element of a TINYGLTF_TYPE_*, -1 if unknown.
int GetNumComponentsInType(unsigned int ty);

// A JSON value (extension and extras data). An integer also reads as a real.
class Value
{
public:
    typedef std::vector<Value> Array;
    typedef std::map<std::string, Value> Object;

    Value() = default;
    explicit Value(bool b)
        : type_(BOOL_TYPE)
        , boolean_value_(b)
    {
    }
    explicit Value(int i)
        : type_(INT_TYPE)
        , int_value_(i)
        , real_value_(i)
    {
    }
    explicit Value(double n)
        : type_(REAL_TYPE)
        , real_value_(n)
    {
    }
    explicit Value(const std::string& s)
        : type_(STRING_TYPE)
        , string_value_(s)
    {
    }
    explicit Value(Array a)
        : type_(ARRAY_TYPE)
        , array_value_(std::move(a))
    {
    }
    explicit Value(Object o)
        : type_(OBJECT_TYPE)
        , object_value_(std::move(o))
    {
    }

    char Type() const { return static_cast<char>(type_); }
    bool IsBool() const { return type_ == BOOL_TYPE; }
    bool IsInt() const { return type_ == INT_TYPE; }
    bool IsReal() const { return type_ == REAL_TYPE; }
    bool IsNumber() const { return type_ == INT_TYPE || type_ == REAL_TYPE; }
    bool IsString() const { return type_ == STRING_TYPE; }
    bool IsArray() const { return type_ == ARRAY_TYPE; }
    bool IsObject() const { return type_ == OBJECT_TYPE; }

    double GetNumberAsDouble() const { return type_ == INT_TYPE ? double(int_value_) : real_value_; }
    // A real outside the int range (or NaN) reads as INT_MIN, which no
    // index or count accepts.
    int GetNumberAsInt() const
    {
        if (type_ != REAL_TYPE)
        {
            return int_value_;
        }
        return (real_value_ >= -2147483648.0 && real_value_ <= 2147483647.0) ? int(real_value_) : (-2147483647 - 1);
    }

    // Array element / object member, or a shared null Value.
    const Value& Get(int idx) const;
    const Value& Get(const std::string& key) const;
    bool Has(const std::string& key) const { return type_ == OBJECT_TYPE && object_value_.count(key) != 0; }
    size_t ArrayLen() const { return type_ == ARRAY_TYPE ? array_value_.size() : 0; }
    std::vector<std::string> Keys() const;
    size_t Size() const { return type_ == ARRAY_TYPE ? array_value_.size() : object_value_.size(); }

    template <typename T>
    const T& Get() const;
    template <typename T>
    T& Get();

private:
    tinygltf::Type type_ = NULL_TYPE;
    int int_value_ = 0;
    double real_value_ = 0;
    std::string string_value_;
    Array array_value_;
    Object object_value_;
    bool boolean_value_ = false;
};

template <>
inline const bool& Value::Get<bool>() const
{
    return boolean_value_;
}
template <>
inline const double& Value::Get<double>() const
{
    return real_value_;
}
template <>
inline const int& Value::Get<int>() const
{
    return int_value_;
}
template <>
inline const std::string& Value::Get<std::string>() const
{
    return string_value_;
}
template <>
inline const Value::Array& Value::Get<Value::Array>() const
{
    return array_value_;
}
template <>
inline const Value::Object& Value::Get<Value::Object>() const
{
    return object_value_;
}
template <>
inline bool& Value::Get<bool>()
{
    return boolean_value_;
}
template <>
inline double& Value::Get<double>()
{
    return real_value_;
}
template <>
inline int& Value::Get<int>()
{
    return int_value_;
}
template <>
inline std::string& Value::Get<std::string>()
{
    return string_value_;
}
template <>
inline Value::Array& Value::Get<Value::Array>()
{
    return array_value_;
}
template <>
inline Value::Object& Value::Get<Value::Object>()
{
    return object_value_;
}

typedef std::map<std::string, Value> ExtensionMap;

struct TextureInfo
{
    int index = -1;
    int texCoord = 0;
    ExtensionMap extensions;
};

struct NormalTextureInfo
{
    int index = -1;
    int texCoord = 0;
    double scale = 1.0;
    ExtensionMap extensions;
};

struct OcclusionTextureInfo
{
    int index = -1;
    int texCoord = 0;
    double strength = 1.0;
    ExtensionMap extensions;
};

struct PbrMetallicRoughness
{
    std::vector<double> baseColorFactor{ 1.0, 1.0, 1.0, 1.0 };
    TextureInfo baseColorTexture;
    double metallicFactor = 1.0;
    double roughnessFactor = 1.0;
    TextureInfo metallicRoughnessTexture;
    ExtensionMap extensions;
};

struct Material
{
    std::string name;
    std::vector<double> emissiveFactor{ 0.0, 0.0, 0.0 };
    std::string alphaMode = "OPAQUE";
    double alphaCutoff = 0.5;
    bool doubleSided = false;
    PbrMetallicRoughness pbrMetallicRoughness;
    NormalTextureInfo normalTexture;
    OcclusionTextureInfo occlusionTexture;
    TextureInfo emissiveTexture;
    ExtensionMap extensions;
    Value extras;
};

struct Image
{
    std::string name;
    int width = -1;
    int height = -1;
    int component = -1;
    int bits = -1;
    int pixel_type = -1;
    std::vector<unsigned char> image;
    int bufferView = -1;
    std::string mimeType;
    std::string uri;
    ExtensionMap extensions;
};

struct Sampler
{
    std::string name;
    int minFilter = -1;
    int magFilter = -1;
    int wrapS = 10497; // REPEAT
    int wrapT = 10497;
};

struct Texture
{
    std::string name;
    int sampler = -1;
    int source = -1;
    ExtensionMap extensions;
};

struct Buffer
{
    std::string name;
    std::vector<unsigned char> data;
    std::string uri;
};

struct BufferView
{
    std::string name;
    int buffer = -1;
    size_t byteOffset = 0;
    size_t byteLength = 0;
    size_t byteStride = 0; // 0: tightly packed
    int target = 0;
};

struct Accessor
{
    std::string name;
    int bufferView = -1;
    size_t byteOffset = 0;
    bool normalized = false;
    int componentType = -1;
    size_t count = 0;
    int type = -1;
    std::vector<double> minValues;
    std::vector<double> maxValues;
};

struct Primitive
{
    std::map<std::string, int> attributes; // e.g. "POSITION" -> accessor index
    int material = -1;
    int indices = -1;
    int mode = TINYGLTF_MODE_TRIANGLES;
    ExtensionMap extensions;
};

struct Mesh
{
    std::string name;
    std::vector<Primitive> primitives;
    std::vector<double> weights;
};

struct Node
{
    std::string name;
    int camera = -1;
    int skin = -1;
    int mesh = -1;
    std::vector<int> children;
    std::vector<double> rotation;    // quaternion x, y, z, w, or empty
    std::vector<double> scale;       // or empty
    std::vector<double> translation; // or empty
    std::vector<double> matrix;      // 16 values, column-major, or empty
    std::vector<double> weights;
};

struct Scene
{
    std::string name;
    std::vector<int> nodes;
};

struct Asset
{
    std::string version = "2.0";
    std::string generator;
    std::string minVersion;
    std::string copyright;
};

struct Model
{
    std::vector<Accessor> accessors;
    std::vector<BufferView> bufferViews;
    std::vector<Buffer> buffers;
    std::vector<Material> materials;
    std::vector<Mesh> meshes;
    std::vector<Node> nodes;
    std::vector<Texture> textures;
    std::vector<Image> images;
    std::vector<Sampler> samplers;
    std::vector<Scene> scenes;
    int defaultScene = -1; // the file's "scene", -1 when it names none
    std::vector<std::string> extensionsUsed;
    std::vector<std::string> extensionsRequired;
    Asset asset;
};

enum SectionCheck
{
    NO_REQUIRE = 0x00,
    REQUIRE_VERSION = 0x01,
    REQUIRE_SCENE = 0x02,
    REQUIRE_SCENES = 0x04,
    REQUIRE_NODES = 0x08,
    REQUIRE_ACCESSORS = 0x10,
    REQUIRE_BUFFERS = 0x20,
    REQUIRE_BUFFER_VIEWS = 0x40,
    REQUIRE_ALL = 0x7f
};

// Decodes (or, as the CLI's loader does, discards) one image's bytes.
using LoadImageDataFunction = std::function<bool(Image* image, const int image_idx, std::string* err,
                                                 std::string* warn, int req_width, int req_height,
                                                 const unsigned char* bytes, int size, void* user_data)>;

class TinyGLTF
{
public:
    TinyGLTF() = default;

    // Without a loader, image bytes are kept undecoded in Image::image.
    void SetImageLoader(LoadImageDataFunction loader, void* user_data)
    {
        image_loader_ = std::move(loader);
        image_user_data_ = user_data;
    }

    bool LoadASCIIFromFile(Model* model, std::string* err, std::string* warn, const std::string& filename,
                           unsigned int check_sections = REQUIRE_VERSION);
    bool LoadASCIIFromString(Model* model, std::string* err, std::string* warn, const char* str, unsigned int length,
                             const std::string& base_dir, unsigned int check_sections = REQUIRE_VERSION);
    bool LoadBinaryFromFile(Model* model, std::string* err, std::string* warn, const std::string& filename,
                            unsigned int check_sections = REQUIRE_VERSION);
    bool LoadBinaryFromMemory(Model* model, std::string* err, std::string* warn, const unsigned char* bytes,
                              unsigned int length, const std::string& base_dir = "",
                              unsigned int check_sections = REQUIRE_VERSION);

private:
    bool Load(Model* model, std::string* err, std::string* warn, const char* json, size_t json_size,
              const std::string& base_dir, const unsigned char* bin, size_t bin_size, bool has_bin,
              unsigned int check_sections);

    LoadImageDataFunction image_loader_;
    void* image_user_data_ = nullptr;
};

} // namespace tinygltf
