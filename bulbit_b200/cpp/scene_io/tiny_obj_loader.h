// Wavefront OBJ / MTL reader for the reference CLI's model loader
// (cli/model_loader.cpp: LoadOBJ, CreateOBJMaterial), which is written
// against tinyobjloader's v2 API (tinyobjloader 7dbc543d, fetched by the
// reference's cli/CMakeLists.txt and not part of this image). This header
// declares that API's reader classes and data types with the same names and
// meaning; obj_reader.cpp implements them with a reader of this project's own.
//
// What is read: v (with optional RGB vertex colour), vn, vt, f (v, v/vt,
// v//vn, v/vt/vn; negative indices count back from the last element read), l,
// p, o / g (a new shape starts once the current one holds elements), usemtl
// (per-face material ids, -1 for none or an unknown name, with a warning), s
// (smoothing groups; "off" is 0), mtllib (files looked up in the config's
// mtl_search_path; a missing file is a warning). With triangulation on,
// quads are split along their shorter diagonal (0-2 on a tie) and larger
// polygons into a fan from their first corner. MTL statements: newmtl, Ka,
// Kd, Ks, Kt / Tf, Ke, Ns, Ni, d, Tr, illum, Pr, Pm, Ps, Pc, Pcr, aniso, anisor
// and the map_* / bump / disp / refl / norm texture names (the last token of
// the line, after any texture options). An index of 0, or one past the
// elements read so far, fails the parse with an error naming the line.
#pragma once

#include <istream>
#include <map>
#include <string>
#include <vector>

namespace tinyobj
{

typedef float real_t;

struct material_t
{
    std::string name;

    real_t ambient[3] = { 0, 0, 0 };
    real_t diffuse[3] = { 0, 0, 0 };
    real_t specular[3] = { 0, 0, 0 };
    real_t transmittance[3] = { 0, 0, 0 };
    real_t emission[3] = { 0, 0, 0 };
    real_t shininess = 1;
    real_t ior = 1;
    real_t dissolve = 1; // 1 = opaque
    int illum = 0;

    std::string ambient_texname;            // map_Ka
    std::string diffuse_texname;            // map_Kd
    std::string specular_texname;           // map_Ks
    std::string specular_highlight_texname; // map_Ns
    std::string bump_texname;               // map_bump, map_Bump, bump
    std::string displacement_texname;       // disp
    std::string alpha_texname;              // map_d
    std::string reflection_texname;         // refl

    // Physically based extension.
    real_t roughness = 0;           // Pr
    real_t metallic = 0;            // Pm
    real_t sheen = 0;               // Ps
    real_t clearcoat_thickness = 0; // Pc
    real_t clearcoat_roughness = 0; // Pcr
    real_t anisotropy = 0;          // aniso
    real_t anisotropy_rotation = 0; // anisor
    std::string roughness_texname;  // map_Pr
    std::string metallic_texname;   // map_Pm
    std::string sheen_texname;      // map_Ps
    std::string emissive_texname;   // map_Ke
    std::string normal_texname;     // norm

    std::map<std::string, std::string> unknown_parameter;
};

struct index_t
{
    int vertex_index = -1;
    int normal_index = -1;   // -1 when the corner has no normal
    int texcoord_index = -1; // -1 when the corner has no texture coordinate
};

struct mesh_t
{
    std::vector<index_t> indices;                  // corners of all faces, face after face
    std::vector<unsigned int> num_face_vertices;   // corners per face (3 when triangulated)
    std::vector<int> material_ids;                 // per face, -1 for none
    std::vector<unsigned int> smoothing_group_ids; // per face, 0 for none
};

struct lines_t
{
    std::vector<index_t> indices;
    std::vector<int> num_line_vertices;
};

struct points_t
{
    std::vector<index_t> indices;
};

struct shape_t
{
    std::string name;
    mesh_t mesh;
    lines_t lines;
    points_t points;
};

struct attrib_t
{
    std::vector<real_t> vertices;  // 3 per position
    std::vector<real_t> normals;   // 3 per normal
    std::vector<real_t> texcoords; // 2 per texture coordinate
    std::vector<real_t> colors;    // 3 per position when any vertex carries a colour, else empty

    const std::vector<real_t>& GetVertices() const { return vertices; }
};

struct ObjReaderConfig
{
    bool triangulate = true;
    std::string triangulation_method = "simple";
    bool vertex_color = true;
    std::string mtl_search_path; // directory of the .mtl files (with or without a trailing '/')
};

class ObjReader
{
public:
    ObjReader() = default;

    bool ParseFromFile(const std::string& filename, const ObjReaderConfig& config = ObjReaderConfig());
    // OBJ text plus the text of the one material library it may name.
    bool ParseFromString(const std::string& obj_text, const std::string& mtl_text,
                         const ObjReaderConfig& config = ObjReaderConfig());

    bool Valid() const { return valid_; }
    const attrib_t& GetAttrib() const { return attrib_; }
    const std::vector<shape_t>& GetShapes() const { return shapes_; }
    const std::vector<material_t>& GetMaterials() const { return materials_; }
    const std::string& Warning() const { return warning_; }
    const std::string& Error() const { return error_; }

private:
    bool valid_ = false;
    attrib_t attrib_;
    std::vector<shape_t> shapes_;
    std::vector<material_t> materials_;
    std::string warning_;
    std::string error_;
};

// The library's older entry point: reads filename with materials looked up
// in mtl_basedir; warnings and errors are appended to *warn / *err.
bool LoadObj(attrib_t* attrib, std::vector<shape_t>* shapes, std::vector<material_t>* materials, std::string* warn,
             std::string* err, const char* filename, const char* mtl_basedir = nullptr, bool triangulate = true,
             bool default_vcols_fallback = true);

// Reads an MTL stream into materials, registering each name in material_map.
void LoadMtl(std::map<std::string, int>* material_map, std::vector<material_t>* materials, std::istream* in,
             std::string* warning, std::string* err);

} // namespace tinyobj
