// The OBJ / MTL reader behind tiny_obj_loader.h: a line-oriented reader that
// fills tinyobjloader's attrib / shape / material structures. Numbers are
// parsed with std::from_chars (locale-independent, correctly rounded to
// float). A colour statement with one value sets all three channels, as the
// MTL format specifies.

#include "tiny_obj_loader.h"

#include <charconv>
#include <fstream>
#include <functional>
#include <sstream>
#include <string_view>

namespace tinyobj
{

namespace
{

bool IsBlank(char c)
{
    return c == ' ' || c == '\t' || c == '\r' || c == '\n' || c == '\v' || c == '\f';
}

std::vector<std::string_view> Split(std::string_view line)
{
    std::vector<std::string_view> out;
    size_t i = 0;
    while (i < line.size())
    {
        while (i < line.size() && IsBlank(line[i]))
        {
            ++i;
        }
        size_t start = i;
        while (i < line.size() && !IsBlank(line[i]))
        {
            ++i;
        }
        if (i > start)
        {
            out.push_back(line.substr(start, i - start));
        }
    }
    return out;
}

// The line after its first token, without surrounding blanks.
std::string Rest(std::string_view line)
{
    size_t i = 0;
    while (i < line.size() && IsBlank(line[i]))
    {
        ++i;
    }
    while (i < line.size() && !IsBlank(line[i]))
    {
        ++i;
    }
    while (i < line.size() && IsBlank(line[i]))
    {
        ++i;
    }
    size_t end = line.size();
    while (end > i && IsBlank(line[end - 1]))
    {
        --end;
    }
    return std::string(line.substr(i, end - i));
}

bool ParseReal(std::string_view t, real_t* out)
{
    if (!t.empty() && t[0] == '+')
    {
        t.remove_prefix(1);
    }
    auto r = std::from_chars(t.data(), t.data() + t.size(), *out);
    return r.ec == std::errc() && r.ptr == t.data() + t.size();
}

bool ParseInt(std::string_view t, long long* out)
{
    if (!t.empty() && t[0] == '+')
    {
        t.remove_prefix(1);
    }
    auto r = std::from_chars(t.data(), t.data() + t.size(), *out);
    return r.ec == std::errc() && r.ptr == t.data() + t.size();
}

bool ReadText(const std::string& path, std::string* out)
{
    std::ifstream f(path, std::ios::binary);
    if (!f)
    {
        return false;
    }
    std::ostringstream ss;
    ss << f.rdbuf();
    *out = ss.str();
    return true;
}

std::string JoinPath(const std::string& dir, const std::string& name)
{
    if (dir.empty() || (!name.empty() && name[0] == '/'))
    {
        return name;
    }
    return dir.back() == '/' ? dir + name : dir + "/" + name;
}

std::string DirectoryOf(const std::string& path)
{
    size_t slash = path.find_last_of('/');
    return slash == std::string::npos ? std::string() : path.substr(0, slash + 1);
}

// Fetches the text of a material library named by an mtllib statement.
using MtlSource = std::function<bool(const std::string& name, std::string* text)>;

class ObjParser
{
public:
    ObjParser(const ObjReaderConfig& config, const MtlSource& mtl, attrib_t* attrib, std::vector<shape_t>* shapes,
              std::vector<material_t>* materials, std::string* warn, std::string* err)
        : config_(config)
        , mtl_(mtl)
        , attrib_(*attrib)
        , shapes_(*shapes)
        , materials_(*materials)
        , warn_(*warn)
        , err_(*err)
    {
        for (size_t i = 0; i < materials_.size(); ++i)
        {
            material_map_.emplace(materials_[i].name, int(i));
        }
    }

    bool Run(std::istream& in)
    {
        std::string line;
        while (std::getline(in, line))
        {
            ++line_no_;
            if (!Line(line))
            {
                return false;
            }
        }
        FlushShape();
        if (!any_color_ || !config_.vertex_color)
        {
            attrib_.colors.clear();
        }
        return true;
    }

private:
    bool Fail(const std::string& what)
    {
        err_ += "line " + std::to_string(line_no_) + ": " + what + "\n";
        return false;
    }

    void Warn(const std::string& what) { warn_ += "line " + std::to_string(line_no_) + ": " + what + "\n"; }

    bool HasElements() const
    {
        return !shape_.mesh.indices.empty() || !shape_.lines.indices.empty() || !shape_.points.indices.empty();
    }

    void FlushShape()
    {
        if (HasElements())
        {
            shapes_.push_back(std::move(shape_));
        }
        shape_ = shape_t();
    }

    // One 1-based (or negative, relative) index into a list of count
    // elements, as a 0-based index.
    bool Resolve(std::string_view t, size_t count, const char* what, int* out)
    {
        long long v = 0;
        if (!ParseInt(t, &v))
        {
            return Fail(std::string("malformed ") + what + " index '" + std::string(t) + "'");
        }
        long long i = v > 0 ? v - 1 : (long long)count + v;
        if (v == 0 || i < 0 || i >= (long long)count)
        {
            return Fail(std::string(what) + " index " + std::to_string(v) + " out of range (" + std::to_string(count) +
                        " read)");
        }
        *out = int(i);
        return true;
    }

    // "v", "v/vt", "v//vn" or "v/vt/vn".
    bool Corner(std::string_view t, index_t* out)
    {
        size_t s1 = t.find('/');
        std::string_view v = t.substr(0, s1);
        if (!Resolve(v, attrib_.vertices.size() / 3, "vertex", &out->vertex_index))
        {
            return false;
        }
        if (s1 == std::string_view::npos)
        {
            return true;
        }
        std::string_view rest = t.substr(s1 + 1);
        size_t s2 = rest.find('/');
        std::string_view vt = rest.substr(0, s2);
        if (!vt.empty() && !Resolve(vt, attrib_.texcoords.size() / 2, "texture coordinate", &out->texcoord_index))
        {
            return false;
        }
        if (s2 != std::string_view::npos)
        {
            std::string_view vn = rest.substr(s2 + 1);
            if (!vn.empty() && !Resolve(vn, attrib_.normals.size() / 3, "normal", &out->normal_index))
            {
                return false;
            }
        }
        return true;
    }

    bool Reals(const std::vector<std::string_view>& tok, size_t first, size_t count, real_t* out)
    {
        for (size_t k = 0; k < count; ++k)
        {
            if (!ParseReal(tok[first + k], &out[k]))
            {
                return Fail("malformed number '" + std::string(tok[first + k]) + "'");
            }
        }
        return true;
    }

    void PushFace(const index_t* c, unsigned int n)
    {
        for (unsigned int k = 0; k < n; ++k)
        {
            shape_.mesh.indices.push_back(c[k]);
        }
        shape_.mesh.num_face_vertices.push_back(n);
        shape_.mesh.material_ids.push_back(material_id_);
        shape_.mesh.smoothing_group_ids.push_back(smoothing_group_);
    }

    real_t Dist2(int a, int b) const
    {
        real_t d = 0;
        for (int k = 0; k < 3; ++k)
        {
            real_t e = attrib_.vertices[3 * size_t(a) + k] - attrib_.vertices[3 * size_t(b) + k];
            d += e * e;
        }
        return d;
    }

    bool Face(const std::vector<std::string_view>& tok)
    {
        std::vector<index_t> c(tok.size() - 1);
        for (size_t k = 1; k < tok.size(); ++k)
        {
            if (!Corner(tok[k], &c[k - 1]))
            {
                return false;
            }
        }
        if (c.size() < 3)
        {
            Warn("face with fewer than 3 corners skipped");
            return true;
        }
        if (!config_.triangulate || c.size() == 3)
        {
            PushFace(c.data(), unsigned(c.size()));
        }
        else if (c.size() == 4)
        {
            if (Dist2(c[0].vertex_index, c[2].vertex_index) <= Dist2(c[1].vertex_index, c[3].vertex_index))
            {
                const index_t t0[3] = { c[0], c[1], c[2] }, t1[3] = { c[0], c[2], c[3] };
                PushFace(t0, 3);
                PushFace(t1, 3);
            }
            else
            {
                const index_t t0[3] = { c[0], c[1], c[3] }, t1[3] = { c[1], c[2], c[3] };
                PushFace(t0, 3);
                PushFace(t1, 3);
            }
        }
        else
        {
            for (size_t k = 1; k + 1 < c.size(); ++k)
            {
                const index_t t[3] = { c[0], c[k], c[k + 1] };
                PushFace(t, 3);
            }
        }
        return true;
    }

    bool Line(std::string& raw)
    {
        std::vector<std::string_view> tok = Split(raw);
        if (tok.empty() || tok[0][0] == '#')
        {
            return true;
        }
        std::string_view key = tok[0];
        if (key == "v")
        {
            if (tok.size() < 4)
            {
                return Fail("vertex needs 3 coordinates");
            }
            real_t p[3];
            if (!Reals(tok, 1, 3, p))
            {
                return false;
            }
            attrib_.vertices.insert(attrib_.vertices.end(), p, p + 3);
            real_t rgb[3] = { 1, 1, 1 };
            if (tok.size() >= 7)
            {
                if (!Reals(tok, 4, 3, rgb))
                {
                    return false;
                }
                any_color_ = true;
            }
            attrib_.colors.insert(attrib_.colors.end(), rgb, rgb + 3);
        }
        else if (key == "vn")
        {
            if (tok.size() < 4)
            {
                return Fail("normal needs 3 components");
            }
            real_t n[3];
            if (!Reals(tok, 1, 3, n))
            {
                return false;
            }
            attrib_.normals.insert(attrib_.normals.end(), n, n + 3);
        }
        else if (key == "vt")
        {
            if (tok.size() < 2)
            {
                return Fail("texture coordinate needs a component");
            }
            real_t uv[2] = { 0, 0 };
            if (!Reals(tok, 1, tok.size() >= 3 ? 2 : 1, uv))
            {
                return false;
            }
            attrib_.texcoords.insert(attrib_.texcoords.end(), uv, uv + 2);
        }
        else if (key == "f")
        {
            return Face(tok);
        }
        else if (key == "l")
        {
            for (size_t k = 1; k < tok.size(); ++k)
            {
                index_t c;
                if (!Corner(tok[k], &c))
                {
                    return false;
                }
                shape_.lines.indices.push_back(c);
            }
            shape_.lines.num_line_vertices.push_back(int(tok.size() - 1));
        }
        else if (key == "p")
        {
            for (size_t k = 1; k < tok.size(); ++k)
            {
                index_t c;
                if (!Corner(tok[k], &c))
                {
                    return false;
                }
                shape_.points.indices.push_back(c);
            }
        }
        else if (key == "o" || key == "g")
        {
            FlushShape();
            shape_.name = Rest(raw);
        }
        else if (key == "usemtl")
        {
            std::string name = Rest(raw);
            auto it = material_map_.find(name);
            if (it == material_map_.end())
            {
                Warn("material '" + name + "' not found in the material libraries");
                material_id_ = -1;
            }
            else
            {
                material_id_ = it->second;
            }
        }
        else if (key == "mtllib")
        {
            bool loaded = false;
            for (size_t k = 1; k < tok.size(); ++k)
            {
                std::string text;
                if (mtl_ && mtl_(std::string(tok[k]), &text))
                {
                    std::istringstream in(text);
                    LoadMtl(&material_map_, &materials_, &in, &warn_, &err_);
                    loaded = true;
                }
            }
            if (!loaded)
            {
                Warn("material library '" + Rest(raw) + "' not found");
            }
        }
        else if (key == "s")
        {
            long long g = 0;
            if (tok.size() >= 2 && tok[1] != "off" && !ParseInt(tok[1], &g))
            {
                return Fail("malformed smoothing group '" + std::string(tok[1]) + "'");
            }
            smoothing_group_ = unsigned(g < 0 ? 0 : g);
        }
        return true; // other statements (vp, curves, ...) are not read
    }

    const ObjReaderConfig& config_;
    const MtlSource& mtl_;
    attrib_t& attrib_;
    std::vector<shape_t>& shapes_;
    std::vector<material_t>& materials_;
    std::string& warn_;
    std::string& err_;
    std::map<std::string, int> material_map_;
    shape_t shape_;
    int material_id_ = -1;
    unsigned smoothing_group_ = 0;
    bool any_color_ = false;
    long line_no_ = 0;
};

bool ParseObj(std::istream& in, const ObjReaderConfig& config, const MtlSource& mtl, attrib_t* attrib,
              std::vector<shape_t>* shapes, std::vector<material_t>* materials, std::string* warn, std::string* err)
{
    *attrib = attrib_t();
    shapes->clear();
    materials->clear();
    return ObjParser(config, mtl, attrib, shapes, materials, warn, err).Run(in);
}

} // namespace

void LoadMtl(std::map<std::string, int>* material_map, std::vector<material_t>* materials, std::istream* in,
             std::string* warning, std::string* err)
{
    (void)err; // a malformed value is skipped with a warning, never an error
    material_t cur;
    bool open = false;
    auto close = [&]() {
        if (open)
        {
            material_map->emplace(cur.name, int(materials->size()));
            materials->push_back(cur);
        }
    };
    auto real = [&](const std::vector<std::string_view>& tok, real_t* out) {
        if (tok.size() < 2 || !ParseReal(tok[1], out))
        {
            *warning += "material '" + cur.name + "': malformed " + std::string(tok[0]) + "\n";
        }
    };
    auto color = [&](const std::vector<std::string_view>& tok, real_t* out) {
        real_t c[3];
        bool ok = tok.size() >= 2 && ParseReal(tok[1], &c[0]);
        if (ok && tok.size() >= 4)
        {
            ok = ParseReal(tok[2], &c[1]) && ParseReal(tok[3], &c[2]);
        }
        else if (ok)
        {
            c[1] = c[2] = c[0];
        }
        if (!ok)
        {
            *warning += "material '" + cur.name + "': malformed " + std::string(tok[0]) + "\n";
            return;
        }
        out[0] = c[0];
        out[1] = c[1];
        out[2] = c[2];
    };

    std::string line;
    while (std::getline(*in, line))
    {
        std::vector<std::string_view> tok = Split(line);
        if (tok.empty() || tok[0][0] == '#')
        {
            continue;
        }
        std::string key(tok[0]);
        if (key == "newmtl")
        {
            close();
            cur = material_t();
            cur.name = Rest(line);
            open = true;
            continue;
        }
        if (!open)
        {
            *warning += "MTL statement '" + key + "' before any newmtl ignored\n";
            continue;
        }
        const std::string tex = tok.size() >= 2 ? std::string(tok.back()) : std::string();
        if (key == "Ka") color(tok, cur.ambient);
        else if (key == "Kd") color(tok, cur.diffuse);
        else if (key == "Ks") color(tok, cur.specular);
        else if (key == "Kt" || key == "Tf") color(tok, cur.transmittance);
        else if (key == "Ke") color(tok, cur.emission);
        else if (key == "Ns") real(tok, &cur.shininess);
        else if (key == "Ni") real(tok, &cur.ior);
        else if (key == "d") real(tok, &cur.dissolve);
        else if (key == "Tr")
        {
            real_t tr = 0;
            real(tok, &tr);
            cur.dissolve = 1 - tr;
        }
        else if (key == "illum")
        {
            long long v = 0;
            if (tok.size() >= 2 && ParseInt(tok[1], &v)) cur.illum = int(v);
        }
        else if (key == "Pr") real(tok, &cur.roughness);
        else if (key == "Pm") real(tok, &cur.metallic);
        else if (key == "Ps") real(tok, &cur.sheen);
        else if (key == "Pc") real(tok, &cur.clearcoat_thickness);
        else if (key == "Pcr") real(tok, &cur.clearcoat_roughness);
        else if (key == "aniso") real(tok, &cur.anisotropy);
        else if (key == "anisor") real(tok, &cur.anisotropy_rotation);
        else if (key == "map_Ka") cur.ambient_texname = tex;
        else if (key == "map_Kd") cur.diffuse_texname = tex;
        else if (key == "map_Ks") cur.specular_texname = tex;
        else if (key == "map_Ns") cur.specular_highlight_texname = tex;
        else if (key == "map_bump" || key == "map_Bump" || key == "bump") cur.bump_texname = tex;
        else if (key == "disp") cur.displacement_texname = tex;
        else if (key == "map_d") cur.alpha_texname = tex;
        else if (key == "refl") cur.reflection_texname = tex;
        else if (key == "map_Pr") cur.roughness_texname = tex;
        else if (key == "map_Pm") cur.metallic_texname = tex;
        else if (key == "map_Ps") cur.sheen_texname = tex;
        else if (key == "map_Ke") cur.emissive_texname = tex;
        else if (key == "norm") cur.normal_texname = tex;
        else cur.unknown_parameter[key] = Rest(line);
    }
    close();
}

bool ObjReader::ParseFromFile(const std::string& filename, const ObjReaderConfig& config)
{
    warning_.clear();
    error_.clear();
    std::ifstream in(filename, std::ios::binary);
    if (!in)
    {
        error_ = "cannot open file '" + filename + "'\n";
        valid_ = false;
        return false;
    }
    const std::string dir = config.mtl_search_path.empty() ? DirectoryOf(filename) : config.mtl_search_path;
    MtlSource mtl = [&](const std::string& name, std::string* text) { return ReadText(JoinPath(dir, name), text); };
    valid_ = ParseObj(in, config, mtl, &attrib_, &shapes_, &materials_, &warning_, &error_);
    return valid_;
}

bool ObjReader::ParseFromString(const std::string& obj_text, const std::string& mtl_text,
                                const ObjReaderConfig& config)
{
    warning_.clear();
    error_.clear();
    std::istringstream in(obj_text);
    MtlSource mtl = [&](const std::string&, std::string* text) {
        *text = mtl_text;
        return true;
    };
    valid_ = ParseObj(in, config, mtl, &attrib_, &shapes_, &materials_, &warning_, &error_);
    return valid_;
}

bool LoadObj(attrib_t* attrib, std::vector<shape_t>* shapes, std::vector<material_t>* materials, std::string* warn,
             std::string* err, const char* filename, const char* mtl_basedir, bool triangulate,
             bool default_vcols_fallback)
{
    ObjReaderConfig config;
    config.triangulate = triangulate;
    config.vertex_color = default_vcols_fallback;
    config.mtl_search_path = mtl_basedir ? mtl_basedir : "";
    ObjReader reader;
    bool ok = reader.ParseFromFile(filename, config);
    *attrib = reader.GetAttrib();
    *shapes = reader.GetShapes();
    *materials = reader.GetMaterials();
    if (warn)
    {
        *warn += reader.Warning();
    }
    if (err)
    {
        *err += reader.Error();
    }
    return ok;
}

} // namespace tinyobj
