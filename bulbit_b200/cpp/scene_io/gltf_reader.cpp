// The glTF reader behind tiny_gltf.h: a JSON reader that builds tinygltf's
// Value tree, the .glb container reader, and the conversion of the JSON tree
// into a Model with every cross-reference checked.

#include "tiny_gltf.h"

#include <charconv>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <limits>
#include <sstream>

namespace tinygltf
{

int GetComponentSizeInBytes(unsigned int component_type)
{
    switch (component_type)
    {
    case TINYGLTF_COMPONENT_TYPE_BYTE:
    case TINYGLTF_COMPONENT_TYPE_UNSIGNED_BYTE: return 1;
    case TINYGLTF_COMPONENT_TYPE_SHORT:
    case TINYGLTF_COMPONENT_TYPE_UNSIGNED_SHORT: return 2;
    case TINYGLTF_COMPONENT_TYPE_INT:
    case TINYGLTF_COMPONENT_TYPE_UNSIGNED_INT:
    case TINYGLTF_COMPONENT_TYPE_FLOAT: return 4;
    case TINYGLTF_COMPONENT_TYPE_DOUBLE: return 8;
    default: return -1;
    }
}

int GetNumComponentsInType(unsigned int ty)
{
    switch (ty)
    {
    case TINYGLTF_TYPE_SCALAR: return 1;
    case TINYGLTF_TYPE_VEC2: return 2;
    case TINYGLTF_TYPE_VEC3: return 3;
    case TINYGLTF_TYPE_VEC4: return 4;
    case TINYGLTF_TYPE_MAT2: return 4;
    case TINYGLTF_TYPE_MAT3: return 9;
    case TINYGLTF_TYPE_MAT4: return 16;
    default: return -1;
    }
}

namespace
{

const Value& NullValue()
{
    static const Value null_value;
    return null_value;
}

} // namespace

const Value& Value::Get(int idx) const
{
    if (type_ == ARRAY_TYPE && idx >= 0 && size_t(idx) < array_value_.size())
    {
        return array_value_[size_t(idx)];
    }
    return NullValue();
}

const Value& Value::Get(const std::string& key) const
{
    if (type_ == OBJECT_TYPE)
    {
        auto it = object_value_.find(key);
        if (it != object_value_.end())
        {
            return it->second;
        }
    }
    return NullValue();
}

std::vector<std::string> Value::Keys() const
{
    std::vector<std::string> keys;
    for (const auto& kv : object_value_)
    {
        keys.push_back(kv.first);
    }
    return keys;
}

namespace
{

// ------------------------------------------------------------------ JSON

class JsonReader
{
public:
    JsonReader(const char* data, size_t size)
        : begin_(data)
        , s_(data)
        , end_(data + size)
    {
    }

    bool Parse(Value* out, std::string* err)
    {
        SkipSpace();
        if (!ParseValue(out, 0))
        {
            *err += "JSON error at byte " + std::to_string(s_ - begin_) + ": " + error_ + "\n";
            return false;
        }
        SkipSpace();
        if (s_ != end_)
        {
            *err += "JSON error at byte " + std::to_string(s_ - begin_) + ": text after the top-level value\n";
            return false;
        }
        return true;
    }

private:
    static constexpr int kMaxDepth = 512;

    bool Fail(const char* what)
    {
        error_ = what;
        return false;
    }

    void SkipSpace()
    {
        while (s_ < end_ && (*s_ == ' ' || *s_ == '\t' || *s_ == '\n' || *s_ == '\r'))
        {
            ++s_;
        }
    }

    bool Literal(const char* lit)
    {
        size_t n = std::strlen(lit);
        if (size_t(end_ - s_) < n || std::memcmp(s_, lit, n) != 0)
        {
            return Fail("invalid literal");
        }
        s_ += n;
        return true;
    }

    bool ParseValue(Value* out, int depth)
    {
        if (depth > kMaxDepth)
        {
            return Fail("nesting too deep");
        }
        if (s_ >= end_)
        {
            return Fail("unexpected end of input");
        }
        switch (*s_)
        {
        case '{': return ParseObject(out, depth);
        case '[': return ParseArray(out, depth);
        case '"':
        {
            std::string str;
            if (!ParseString(&str))
            {
                return false;
            }
            *out = Value(str);
            return true;
        }
        case 't':
            *out = Value(true);
            return Literal("true");
        case 'f':
            *out = Value(false);
            return Literal("false");
        case 'n':
            *out = Value();
            return Literal("null");
        default: return ParseNumber(out);
        }
    }

    bool ParseObject(Value* out, int depth)
    {
        ++s_; // '{'
        Value::Object obj;
        SkipSpace();
        if (s_ < end_ && *s_ == '}')
        {
            ++s_;
            *out = Value(std::move(obj));
            return true;
        }
        for (;;)
        {
            SkipSpace();
            if (s_ >= end_ || *s_ != '"')
            {
                return Fail("expected a member name");
            }
            std::string key;
            if (!ParseString(&key))
            {
                return false;
            }
            SkipSpace();
            if (s_ >= end_ || *s_ != ':')
            {
                return Fail("expected ':'");
            }
            ++s_;
            SkipSpace();
            Value v;
            if (!ParseValue(&v, depth + 1))
            {
                return false;
            }
            obj[key] = std::move(v); // a repeated member keeps the last value
            SkipSpace();
            if (s_ < end_ && *s_ == ',')
            {
                ++s_;
                continue;
            }
            if (s_ < end_ && *s_ == '}')
            {
                ++s_;
                *out = Value(std::move(obj));
                return true;
            }
            return Fail("expected ',' or '}'");
        }
    }

    bool ParseArray(Value* out, int depth)
    {
        ++s_; // '['
        Value::Array arr;
        SkipSpace();
        if (s_ < end_ && *s_ == ']')
        {
            ++s_;
            *out = Value(std::move(arr));
            return true;
        }
        for (;;)
        {
            SkipSpace();
            Value v;
            if (!ParseValue(&v, depth + 1))
            {
                return false;
            }
            arr.push_back(std::move(v));
            SkipSpace();
            if (s_ < end_ && *s_ == ',')
            {
                ++s_;
                continue;
            }
            if (s_ < end_ && *s_ == ']')
            {
                ++s_;
                *out = Value(std::move(arr));
                return true;
            }
            return Fail("expected ',' or ']'");
        }
    }

    static void PutUtf8(std::string* out, uint32_t cp)
    {
        if (cp < 0x80)
        {
            *out += char(cp);
        }
        else if (cp < 0x800)
        {
            *out += char(0xC0 | (cp >> 6));
            *out += char(0x80 | (cp & 0x3F));
        }
        else if (cp < 0x10000)
        {
            *out += char(0xE0 | (cp >> 12));
            *out += char(0x80 | ((cp >> 6) & 0x3F));
            *out += char(0x80 | (cp & 0x3F));
        }
        else
        {
            *out += char(0xF0 | (cp >> 18));
            *out += char(0x80 | ((cp >> 12) & 0x3F));
            *out += char(0x80 | ((cp >> 6) & 0x3F));
            *out += char(0x80 | (cp & 0x3F));
        }
    }

    bool Hex4(uint32_t* out)
    {
        if (end_ - s_ < 4)
        {
            return Fail("truncated \\u escape");
        }
        uint32_t v = 0;
        for (int k = 0; k < 4; ++k)
        {
            char c = *s_++;
            v <<= 4;
            if (c >= '0' && c <= '9') v |= uint32_t(c - '0');
            else if (c >= 'a' && c <= 'f') v |= uint32_t(c - 'a' + 10);
            else if (c >= 'A' && c <= 'F') v |= uint32_t(c - 'A' + 10);
            else return Fail("malformed \\u escape");
        }
        *out = v;
        return true;
    }

    bool ParseString(std::string* out)
    {
        ++s_; // '"'
        while (s_ < end_)
        {
            unsigned char c = static_cast<unsigned char>(*s_++);
            if (c == '"')
            {
                return true;
            }
            if (c < 0x20)
            {
                return Fail("control character in string");
            }
            if (c != '\\')
            {
                *out += char(c);
                continue;
            }
            if (s_ >= end_)
            {
                break;
            }
            char e = *s_++;
            switch (e)
            {
            case '"': *out += '"'; break;
            case '\\': *out += '\\'; break;
            case '/': *out += '/'; break;
            case 'b': *out += '\b'; break;
            case 'f': *out += '\f'; break;
            case 'n': *out += '\n'; break;
            case 'r': *out += '\r'; break;
            case 't': *out += '\t'; break;
            case 'u':
            {
                uint32_t cp;
                if (!Hex4(&cp))
                {
                    return false;
                }
                if (cp >= 0xD800 && cp <= 0xDBFF)
                {
                    uint32_t lo;
                    if (end_ - s_ < 2 || s_[0] != '\\' || s_[1] != 'u')
                    {
                        return Fail("unpaired surrogate");
                    }
                    s_ += 2;
                    if (!Hex4(&lo) || lo < 0xDC00 || lo > 0xDFFF)
                    {
                        return Fail("unpaired surrogate");
                    }
                    cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                }
                else if (cp >= 0xDC00 && cp <= 0xDFFF)
                {
                    return Fail("unpaired surrogate");
                }
                PutUtf8(out, cp);
                break;
            }
            default: return Fail("unknown escape");
            }
        }
        return Fail("unterminated string");
    }

    // JSON number grammar; integers that fit an int become INT values (which
    // also read as reals), everything else a REAL.
    bool ParseNumber(Value* out)
    {
        const char* start = s_;
        if (s_ < end_ && *s_ == '-')
        {
            ++s_;
        }
        if (s_ >= end_ || !(*s_ >= '0' && *s_ <= '9'))
        {
            return Fail("unexpected character");
        }
        if (*s_ == '0')
        {
            ++s_;
        }
        else
        {
            while (s_ < end_ && *s_ >= '0' && *s_ <= '9') ++s_;
        }
        bool integral = true;
        if (s_ < end_ && *s_ == '.')
        {
            integral = false;
            ++s_;
            if (s_ >= end_ || !(*s_ >= '0' && *s_ <= '9'))
            {
                return Fail("malformed number");
            }
            while (s_ < end_ && *s_ >= '0' && *s_ <= '9') ++s_;
        }
        if (s_ < end_ && (*s_ == 'e' || *s_ == 'E'))
        {
            integral = false;
            ++s_;
            if (s_ < end_ && (*s_ == '+' || *s_ == '-')) ++s_;
            if (s_ >= end_ || !(*s_ >= '0' && *s_ <= '9'))
            {
                return Fail("malformed number");
            }
            while (s_ < end_ && *s_ >= '0' && *s_ <= '9') ++s_;
        }
        if (integral)
        {
            long long v = 0;
            auto r = std::from_chars(start, s_, v);
            if (r.ec == std::errc() && v >= std::numeric_limits<int>::min() && v <= std::numeric_limits<int>::max())
            {
                *out = Value(int(v));
                return true;
            }
        }
        double d = 0;
        auto r = std::from_chars(start, s_, d);
        if (r.ec != std::errc() && r.ec != std::errc::result_out_of_range)
        {
            return Fail("malformed number");
        }
        *out = Value(d);
        return true;
    }

    const char* begin_;
    const char* s_;
    const char* end_;
    const char* error_ = "";
};

// --------------------------------------------------------------- helpers

bool ReadFile(const std::string& path, std::vector<unsigned char>* out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f)
    {
        return false;
    }
    std::ostringstream ss;
    ss << f.rdbuf();
    const std::string& s = ss.str();
    out->assign(s.begin(), s.end());
    return true;
}

std::string DirectoryOf(const std::string& path)
{
    size_t slash = path.find_last_of('/');
    return slash == std::string::npos ? std::string() : path.substr(0, slash + 1);
}

std::string JoinPath(const std::string& dir, const std::string& name)
{
    if (dir.empty() || (!name.empty() && name[0] == '/'))
    {
        return name;
    }
    return dir.back() == '/' ? dir + name : dir + "/" + name;
}

std::string PercentDecode(const std::string& uri)
{
    std::string out;
    for (size_t i = 0; i < uri.size(); ++i)
    {
        auto hex = [](char c) {
            return (c >= '0' && c <= '9') ? c - '0' : (c >= 'a' && c <= 'f') ? c - 'a' + 10 : (c >= 'A' && c <= 'F') ? c - 'A' + 10 : -1;
        };
        if (uri[i] == '%' && i + 2 < uri.size() && hex(uri[i + 1]) >= 0 && hex(uri[i + 2]) >= 0)
        {
            out += char(hex(uri[i + 1]) * 16 + hex(uri[i + 2]));
            i += 2;
        }
        else
        {
            out += uri[i];
        }
    }
    return out;
}

bool IsDataUri(const std::string& uri)
{
    return uri.compare(0, 5, "data:") == 0;
}

// The payload of a base64 data URI ("data:<type>;base64,<payload>").
bool DecodeDataUri(const std::string& uri, std::vector<unsigned char>* out)
{
    size_t comma = uri.find(',');
    if (comma == std::string::npos || uri.rfind(";base64", comma) == std::string::npos)
    {
        return false;
    }
    out->clear();
    uint32_t acc = 0;
    int bits = 0;
    for (size_t i = comma + 1; i < uri.size(); ++i)
    {
        char c = uri[i];
        int v;
        if (c >= 'A' && c <= 'Z') v = c - 'A';
        else if (c >= 'a' && c <= 'z') v = c - 'a' + 26;
        else if (c >= '0' && c <= '9') v = c - '0' + 52;
        else if (c == '+') v = 62;
        else if (c == '/') v = 63;
        else if (c == '=') break;
        else return false;
        acc = (acc << 6) | uint32_t(v);
        bits += 6;
        if (bits >= 8)
        {
            bits -= 8;
            out->push_back(static_cast<unsigned char>((acc >> bits) & 0xFF));
        }
    }
    return true;
}

int Int(const Value& o, const char* key, int def)
{
    const Value& v = o.Get(key);
    return v.IsNumber() ? v.GetNumberAsInt() : def;
}

// A byte count or offset; a negative one keeps the default, one beyond 2^53
// (or NaN) reads as SIZE_MAX, which every range check rejects.
size_t Size(const Value& o, const char* key, size_t def)
{
    const Value& v = o.Get(key);
    if (!v.IsNumber())
    {
        return def;
    }
    const double d = v.GetNumberAsDouble();
    if (d < 0)
    {
        return def;
    }
    return d <= 9007199254740992.0 ? size_t(d) : std::numeric_limits<size_t>::max();
}

double Num(const Value& o, const char* key, double def)
{
    const Value& v = o.Get(key);
    return v.IsNumber() ? v.GetNumberAsDouble() : def;
}

bool Bool(const Value& o, const char* key, bool def)
{
    const Value& v = o.Get(key);
    return v.IsBool() ? v.Get<bool>() : def;
}

std::string Str(const Value& o, const char* key)
{
    const Value& v = o.Get(key);
    return v.IsString() ? v.Get<std::string>() : std::string();
}

std::vector<double> Nums(const Value& o, const char* key, std::vector<double> def = {})
{
    const Value& v = o.Get(key);
    if (!v.IsArray())
    {
        return def;
    }
    std::vector<double> out;
    for (const Value& e : v.Get<Value::Array>())
    {
        out.push_back(e.GetNumberAsDouble());
    }
    return out;
}

std::vector<int> Ints(const Value& o, const char* key)
{
    std::vector<int> out;
    const Value& v = o.Get(key);
    if (v.IsArray())
    {
        for (const Value& e : v.Get<Value::Array>())
        {
            out.push_back(e.GetNumberAsInt());
        }
    }
    return out;
}

ExtensionMap Extensions(const Value& o)
{
    const Value& v = o.Get("extensions");
    return v.IsObject() ? v.Get<Value::Object>() : ExtensionMap();
}

const Value::Array& Items(const Value& root, const char* key)
{
    static const Value::Array empty;
    const Value& v = root.Get(key);
    return v.IsArray() ? v.Get<Value::Array>() : empty;
}

TextureInfo ReadTextureInfo(const Value& o)
{
    TextureInfo t;
    t.index = Int(o, "index", -1);
    t.texCoord = Int(o, "texCoord", 0);
    t.extensions = Extensions(o);
    return t;
}

int AccessorType(const std::string& s)
{
    if (s == "SCALAR") return TINYGLTF_TYPE_SCALAR;
    if (s == "VEC2") return TINYGLTF_TYPE_VEC2;
    if (s == "VEC3") return TINYGLTF_TYPE_VEC3;
    if (s == "VEC4") return TINYGLTF_TYPE_VEC4;
    if (s == "MAT2") return TINYGLTF_TYPE_MAT2;
    if (s == "MAT3") return TINYGLTF_TYPE_MAT3;
    if (s == "MAT4") return TINYGLTF_TYPE_MAT4;
    return -1;
}

// True when index is -1 (absent, where that is allowed) or names an element.
bool ValidIndex(int index, size_t count, bool allow_absent)
{
    return (allow_absent && index == -1) || (index >= 0 && size_t(index) < count);
}

uint32_t ReadU32(const unsigned char* p)
{
    return uint32_t(p[0]) | (uint32_t(p[1]) << 8) | (uint32_t(p[2]) << 16) | (uint32_t(p[3]) << 24);
}

} // namespace

// ---------------------------------------------------------------- loader

bool TinyGLTF::Load(Model* model, std::string* err, std::string* warn, const char* json, size_t json_size,
                    const std::string& base_dir, const unsigned char* bin, size_t bin_size, bool has_bin,
                    unsigned int check_sections)
{
    std::string local_err, local_warn;
    std::string& e = err ? *err : local_err;
    std::string& w = warn ? *warn : local_warn;
    *model = Model();

    Value root;
    if (!JsonReader(json, json_size).Parse(&root, &e))
    {
        return false;
    }
    if (!root.IsObject())
    {
        e += "the top-level JSON value is not an object\n";
        return false;
    }
    auto fail = [&](const std::string& what) {
        e += what + "\n";
        return false;
    };

    const Value& asset = root.Get("asset");
    if ((check_sections & REQUIRE_VERSION) && !asset.Get("version").IsString())
    {
        return fail("asset.version is missing");
    }
    model->asset.version = Str(asset, "version");
    model->asset.generator = Str(asset, "generator");
    model->asset.minVersion = Str(asset, "minVersion");
    model->asset.copyright = Str(asset, "copyright");
    const struct
    {
        unsigned bit;
        const char* key;
    } kRequired[] = { { REQUIRE_SCENE, "scene" },           { REQUIRE_SCENES, "scenes" },
                      { REQUIRE_NODES, "nodes" },           { REQUIRE_ACCESSORS, "accessors" },
                      { REQUIRE_BUFFERS, "buffers" },       { REQUIRE_BUFFER_VIEWS, "bufferViews" } };
    for (const auto& r : kRequired)
    {
        if ((check_sections & r.bit) && !root.Has(r.key))
        {
            return fail(std::string("required section '") + r.key + "' is missing");
        }
    }
    for (const Value& v : Items(root, "extensionsUsed"))
    {
        model->extensionsUsed.push_back(v.IsString() ? v.Get<std::string>() : std::string());
    }
    for (const Value& v : Items(root, "extensionsRequired"))
    {
        model->extensionsRequired.push_back(v.IsString() ? v.Get<std::string>() : std::string());
    }

    // Buffers: a data URI, a file next to the model, or the .glb BIN chunk.
    const Value::Array& buffers = Items(root, "buffers");
    for (size_t i = 0; i < buffers.size(); ++i)
    {
        const Value& b = buffers[i];
        Buffer buf;
        buf.name = Str(b, "name");
        buf.uri = Str(b, "uri");
        const double declared = Num(b, "byteLength", -1);
        if (!(declared >= 0 && declared <= 9007199254740992.0))
        {
            return fail("buffer " + std::to_string(i) + ": byteLength is missing or out of range");
        }
        const size_t length = size_t(declared);
        if (buf.uri.empty())
        {
            if (!has_bin || i != 0)
            {
                return fail("buffer " + std::to_string(i) + " has no uri and is not the .glb BIN chunk");
            }
            buf.data.assign(bin, bin + bin_size);
        }
        else if (IsDataUri(buf.uri))
        {
            if (!DecodeDataUri(buf.uri, &buf.data))
            {
                return fail("buffer " + std::to_string(i) + ": malformed data URI");
            }
        }
        else if (!ReadFile(JoinPath(base_dir, PercentDecode(buf.uri)), &buf.data))
        {
            return fail("buffer " + std::to_string(i) + ": cannot read '" + buf.uri + "'");
        }
        if (buf.data.size() < length)
        {
            return fail("buffer " + std::to_string(i) + ": " + std::to_string(buf.data.size()) +
                        " bytes, byteLength " + std::to_string(length));
        }
        buf.data.resize(length);
        model->buffers.push_back(std::move(buf));
    }

    const Value::Array& views = Items(root, "bufferViews");
    for (size_t i = 0; i < views.size(); ++i)
    {
        const Value& v = views[i];
        BufferView bv;
        bv.name = Str(v, "name");
        bv.buffer = Int(v, "buffer", -1);
        bv.byteOffset = Size(v, "byteOffset", 0);
        bv.byteLength = Size(v, "byteLength", 0);
        bv.byteStride = Size(v, "byteStride", 0);
        bv.target = Int(v, "target", 0);
        if (!ValidIndex(bv.buffer, model->buffers.size(), false) ||
            bv.byteOffset > model->buffers[size_t(bv.buffer)].data.size() ||
            bv.byteLength > model->buffers[size_t(bv.buffer)].data.size() - bv.byteOffset)
        {
            return fail("bufferView " + std::to_string(i) + " reaches outside its buffer");
        }
        if (bv.byteStride != 0 && (bv.byteStride < 4 || bv.byteStride > 252))
        {
            return fail("bufferView " + std::to_string(i) + ": byteStride out of [4, 252]");
        }
        model->bufferViews.push_back(bv);
    }

    const Value::Array& accessors = Items(root, "accessors");
    for (size_t i = 0; i < accessors.size(); ++i)
    {
        const Value& a = accessors[i];
        Accessor acc;
        acc.name = Str(a, "name");
        acc.bufferView = Int(a, "bufferView", -1);
        acc.byteOffset = Size(a, "byteOffset", 0);
        acc.normalized = Bool(a, "normalized", false);
        acc.componentType = Int(a, "componentType", -1);
        acc.count = Size(a, "count", 0);
        acc.type = AccessorType(Str(a, "type"));
        acc.minValues = Nums(a, "min");
        acc.maxValues = Nums(a, "max");
        const std::string where = "accessor " + std::to_string(i);
        const int comp = GetComponentSizeInBytes(unsigned(acc.componentType));
        const int ncomp = GetNumComponentsInType(unsigned(acc.type));
        if (comp < 0 || ncomp < 0)
        {
            return fail(where + ": unknown componentType or type");
        }
        if (!ValidIndex(acc.bufferView, model->bufferViews.size(), false))
        {
            return fail(where + ": no valid bufferView (sparse or zero-filled accessors are not read)");
        }
        const BufferView& bv = model->bufferViews[size_t(acc.bufferView)];
        const size_t elem = size_t(comp) * size_t(ncomp);
        const size_t stride = bv.byteStride ? bv.byteStride : elem;
        if (acc.count > 0)
        {
            // Last element's end, checked without overflow.
            if (acc.count - 1 > (std::numeric_limits<size_t>::max() - elem - acc.byteOffset) / stride ||
                acc.byteOffset + (acc.count - 1) * stride + elem > bv.byteLength)
            {
                return fail(where + " reaches outside its bufferView");
            }
        }
        model->accessors.push_back(acc);
    }

    const Value::Array& images = Items(root, "images");
    const Value::Array& samplers = Items(root, "samplers");
    const Value::Array& textures = Items(root, "textures");
    for (const Value& s : samplers)
    {
        Sampler smp;
        smp.name = Str(s, "name");
        smp.minFilter = Int(s, "minFilter", -1);
        smp.magFilter = Int(s, "magFilter", -1);
        smp.wrapS = Int(s, "wrapS", 10497);
        smp.wrapT = Int(s, "wrapT", 10497);
        model->samplers.push_back(smp);
    }
    for (size_t i = 0; i < textures.size(); ++i)
    {
        const Value& t = textures[i];
        Texture tex;
        tex.name = Str(t, "name");
        tex.sampler = Int(t, "sampler", -1);
        tex.source = Int(t, "source", -1);
        tex.extensions = Extensions(t);
        if (!ValidIndex(tex.sampler, samplers.size(), true) || !ValidIndex(tex.source, images.size(), true))
        {
            return fail("texture " + std::to_string(i) + ": sampler or source out of range");
        }
        model->textures.push_back(tex);
    }
    for (size_t i = 0; i < images.size(); ++i)
    {
        const Value& im = images[i];
        Image img;
        img.name = Str(im, "name");
        img.uri = Str(im, "uri");
        img.mimeType = Str(im, "mimeType");
        img.bufferView = Int(im, "bufferView", -1);
        img.extensions = Extensions(im);
        if (!ValidIndex(img.bufferView, model->bufferViews.size(), true))
        {
            return fail("image " + std::to_string(i) + ": bufferView out of range");
        }
        std::vector<unsigned char> bytes;
        bool have = false;
        if (img.bufferView >= 0)
        {
            const BufferView& bv = model->bufferViews[size_t(img.bufferView)];
            const auto& data = model->buffers[size_t(bv.buffer)].data;
            bytes.assign(data.begin() + std::ptrdiff_t(bv.byteOffset),
                         data.begin() + std::ptrdiff_t(bv.byteOffset + bv.byteLength));
            have = true;
        }
        else if (IsDataUri(img.uri))
        {
            have = DecodeDataUri(img.uri, &bytes);
            if (!have)
            {
                return fail("image " + std::to_string(i) + ": malformed data URI");
            }
        }
        else if (!img.uri.empty())
        {
            have = ReadFile(JoinPath(base_dir, PercentDecode(img.uri)), &bytes);
            if (!have)
            {
                w += "image " + std::to_string(i) + ": cannot read '" + img.uri + "'\n";
            }
        }
        if (have)
        {
            if (image_loader_)
            {
                if (!image_loader_(&img, int(i), &e, &w, 0, 0, bytes.data(), int(bytes.size()), image_user_data_))
                {
                    return fail("image " + std::to_string(i) + ": the image loader failed");
                }
            }
            else
            {
                img.image = std::move(bytes);
            }
        }
        model->images.push_back(std::move(img));
    }

    const Value::Array& materials = Items(root, "materials");
    for (size_t i = 0; i < materials.size(); ++i)
    {
        const Value& m = materials[i];
        Material mat;
        mat.name = Str(m, "name");
        mat.emissiveFactor = Nums(m, "emissiveFactor", { 0.0, 0.0, 0.0 });
        mat.alphaMode = m.Get("alphaMode").IsString() ? Str(m, "alphaMode") : std::string("OPAQUE");
        mat.alphaCutoff = Num(m, "alphaCutoff", 0.5);
        mat.doubleSided = Bool(m, "doubleSided", false);
        const Value& pbr = m.Get("pbrMetallicRoughness");
        mat.pbrMetallicRoughness.baseColorFactor = Nums(pbr, "baseColorFactor", { 1.0, 1.0, 1.0, 1.0 });
        mat.pbrMetallicRoughness.metallicFactor = Num(pbr, "metallicFactor", 1.0);
        mat.pbrMetallicRoughness.roughnessFactor = Num(pbr, "roughnessFactor", 1.0);
        mat.pbrMetallicRoughness.baseColorTexture = ReadTextureInfo(pbr.Get("baseColorTexture"));
        mat.pbrMetallicRoughness.metallicRoughnessTexture = ReadTextureInfo(pbr.Get("metallicRoughnessTexture"));
        mat.pbrMetallicRoughness.extensions = Extensions(pbr);
        const Value& nt = m.Get("normalTexture");
        mat.normalTexture.index = Int(nt, "index", -1);
        mat.normalTexture.texCoord = Int(nt, "texCoord", 0);
        mat.normalTexture.scale = Num(nt, "scale", 1.0);
        mat.normalTexture.extensions = Extensions(nt);
        const Value& ot = m.Get("occlusionTexture");
        mat.occlusionTexture.index = Int(ot, "index", -1);
        mat.occlusionTexture.texCoord = Int(ot, "texCoord", 0);
        mat.occlusionTexture.strength = Num(ot, "strength", 1.0);
        mat.occlusionTexture.extensions = Extensions(ot);
        mat.emissiveTexture = ReadTextureInfo(m.Get("emissiveTexture"));
        mat.extensions = Extensions(m);
        mat.extras = m.Get("extras");
        const size_t nt_count = model->textures.size();
        if (mat.pbrMetallicRoughness.baseColorFactor.size() != 4 || mat.emissiveFactor.size() != 3 ||
            !ValidIndex(mat.pbrMetallicRoughness.baseColorTexture.index, nt_count, true) ||
            !ValidIndex(mat.pbrMetallicRoughness.metallicRoughnessTexture.index, nt_count, true) ||
            !ValidIndex(mat.normalTexture.index, nt_count, true) ||
            !ValidIndex(mat.occlusionTexture.index, nt_count, true) ||
            !ValidIndex(mat.emissiveTexture.index, nt_count, true))
        {
            return fail("material " + std::to_string(i) + ": malformed factor or texture index out of range");
        }
        model->materials.push_back(std::move(mat));
    }

    const Value::Array& meshes = Items(root, "meshes");
    for (size_t i = 0; i < meshes.size(); ++i)
    {
        const Value& m = meshes[i];
        Mesh mesh;
        mesh.name = Str(m, "name");
        mesh.weights = Nums(m, "weights");
        for (const Value& p : Items(m, "primitives"))
        {
            Primitive prim;
            prim.indices = Int(p, "indices", -1);
            prim.material = Int(p, "material", -1);
            prim.mode = Int(p, "mode", TINYGLTF_MODE_TRIANGLES);
            prim.extensions = Extensions(p);
            const Value& attrs = p.Get("attributes");
            if (attrs.IsObject())
            {
                for (const auto& kv : attrs.Get<Value::Object>())
                {
                    prim.attributes[kv.first] = kv.second.GetNumberAsInt();
                }
            }
            bool ok = ValidIndex(prim.indices, model->accessors.size(), true) &&
                      ValidIndex(prim.material, model->materials.size(), true);
            for (const auto& kv : prim.attributes)
            {
                ok = ok && ValidIndex(kv.second, model->accessors.size(), false);
            }
            if (!ok)
            {
                return fail("mesh " + std::to_string(i) + ": primitive index out of range");
            }
            mesh.primitives.push_back(std::move(prim));
        }
        model->meshes.push_back(std::move(mesh));
    }

    const Value::Array& nodes = Items(root, "nodes");
    std::vector<int> parent_of(nodes.size(), -1);
    for (size_t i = 0; i < nodes.size(); ++i)
    {
        const Value& n = nodes[i];
        Node node;
        node.name = Str(n, "name");
        node.camera = Int(n, "camera", -1);
        node.skin = Int(n, "skin", -1);
        node.mesh = Int(n, "mesh", -1);
        node.children = Ints(n, "children");
        node.rotation = Nums(n, "rotation");
        node.scale = Nums(n, "scale");
        node.translation = Nums(n, "translation");
        node.matrix = Nums(n, "matrix");
        node.weights = Nums(n, "weights");
        const std::string where = "node " + std::to_string(i);
        if (!ValidIndex(node.mesh, model->meshes.size(), true) || (!node.matrix.empty() && node.matrix.size() != 16) ||
            (!node.rotation.empty() && node.rotation.size() != 4) || (!node.scale.empty() && node.scale.size() != 3) ||
            (!node.translation.empty() && node.translation.size() != 3))
        {
            return fail(where + ": mesh out of range or malformed transform");
        }
        for (int c : node.children)
        {
            if (!ValidIndex(c, nodes.size(), false) || parent_of[size_t(c)] != -1)
            {
                return fail(where + ": child out of range or with two parents");
            }
            parent_of[size_t(c)] = int(i);
        }
        model->nodes.push_back(std::move(node));
    }
    // The hierarchy must be a forest: following parents from any node ends.
    for (size_t i = 0; i < nodes.size(); ++i)
    {
        size_t steps = 0;
        for (int p = parent_of[i]; p != -1; p = parent_of[size_t(p)])
        {
            if (++steps > nodes.size())
            {
                return fail("node " + std::to_string(i) + " is its own ancestor");
            }
        }
    }

    const Value::Array& scenes = Items(root, "scenes");
    for (size_t i = 0; i < scenes.size(); ++i)
    {
        Scene sc;
        sc.name = Str(scenes[i], "name");
        sc.nodes = Ints(scenes[i], "nodes");
        for (int nd : sc.nodes)
        {
            if (!ValidIndex(nd, model->nodes.size(), false))
            {
                return fail("scene " + std::to_string(i) + ": node out of range");
            }
        }
        model->scenes.push_back(std::move(sc));
    }
    model->defaultScene = Int(root, "scene", -1);
    if (!ValidIndex(model->defaultScene, model->scenes.size(), true))
    {
        return fail("scene index out of range");
    }
    return true;
}

bool TinyGLTF::LoadASCIIFromString(Model* model, std::string* err, std::string* warn, const char* str,
                                   unsigned int length, const std::string& base_dir, unsigned int check_sections)
{
    return Load(model, err, warn, str, length, base_dir, nullptr, 0, false, check_sections);
}

bool TinyGLTF::LoadASCIIFromFile(Model* model, std::string* err, std::string* warn, const std::string& filename,
                                 unsigned int check_sections)
{
    std::vector<unsigned char> data;
    if (!ReadFile(filename, &data))
    {
        if (err)
        {
            *err += "cannot read '" + filename + "'\n";
        }
        return false;
    }
    return Load(model, err, warn, reinterpret_cast<const char*>(data.data()), data.size(), DirectoryOf(filename),
                nullptr, 0, false, check_sections);
}

bool TinyGLTF::LoadBinaryFromMemory(Model* model, std::string* err, std::string* warn, const unsigned char* bytes,
                                    unsigned int length, const std::string& base_dir, unsigned int check_sections)
{
    auto fail = [&](const char* what) {
        if (err)
        {
            *err += std::string(".glb: ") + what + "\n";
        }
        return false;
    };
    // 12-byte header (magic "glTF", version 2, total length), then chunks of
    // (length, type, payload): JSON first, an optional BIN second.
    if (length < 20 || ReadU32(bytes) != 0x46546C67u)
    {
        return fail("not a binary glTF file");
    }
    if (ReadU32(bytes + 4) != 2)
    {
        return fail("unsupported container version");
    }
    const size_t total = ReadU32(bytes + 8);
    if (total > length || total < 20)
    {
        return fail("declared length exceeds the file");
    }
    const size_t json_len = ReadU32(bytes + 12);
    if (ReadU32(bytes + 16) != 0x4E4F534Au || json_len > total - 20)
    {
        return fail("first chunk is not a JSON chunk inside the file");
    }
    const char* json = reinterpret_cast<const char*>(bytes + 20);
    size_t at = 20 + json_len;
    const unsigned char* bin = nullptr;
    size_t bin_len = 0;
    bool has_bin = false;
    if (total - at >= 8)
    {
        bin_len = ReadU32(bytes + at);
        if (ReadU32(bytes + at + 4) == 0x004E4942u)
        {
            if (bin_len > total - at - 8)
            {
                return fail("BIN chunk exceeds the file");
            }
            bin = bytes + at + 8;
            has_bin = true;
        }
    }
    return Load(model, err, warn, json, json_len, base_dir, bin, has_bin ? bin_len : 0, has_bin, check_sections);
}

bool TinyGLTF::LoadBinaryFromFile(Model* model, std::string* err, std::string* warn, const std::string& filename,
                                  unsigned int check_sections)
{
    std::vector<unsigned char> data;
    if (!ReadFile(filename, &data))
    {
        if (err)
        {
            *err += "cannot read '" + filename + "'\n";
        }
        return false;
    }
    if (data.size() > std::numeric_limits<unsigned int>::max())
    {
        if (err)
        {
            *err += "'" + filename + "' is too large\n";
        }
        return false;
    }
    return LoadBinaryFromMemory(model, err, warn, data.data(), unsigned(data.size()), DirectoryOf(filename),
                                check_sections);
}

} // namespace tinygltf
