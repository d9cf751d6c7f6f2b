// Checks of the scene-file readers in bulbit_b200/cpp/scene_io (XML through
// the pugixml API, OBJ / MTL through the tinyobjloader API, glTF / GLB
// through the tinygltf API), the libraries the reference CLI's scene and
// model loaders are written against. Each check prints a line on failure;
// the exit status is the number of failed checks (0 = all passed).
//
//   scene_io_test <scratch directory>

#include "pugixml.hpp"
#include "tiny_gltf.h"
#include "tiny_obj_loader.h"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

namespace
{

int g_failures = 0;
int g_checks = 0;

#define CHECK(cond)                                                                                                   \
    do                                                                                                                \
    {                                                                                                                 \
        ++g_checks;                                                                                                   \
        if (!(cond))                                                                                                  \
        {                                                                                                             \
            ++g_failures;                                                                                             \
            std::printf("FAILED %s:%d: %s\n", __FILE__, __LINE__, #cond);                                             \
        }                                                                                                             \
    } while (0)

bool Eq(const char* a, const char* b)
{
    return std::strcmp(a, b) == 0;
}

pugi::xml_parse_status Status(const char* text)
{
    pugi::xml_document doc;
    return doc.load_string(text).status;
}

void XmlDocumentTree()
{
    pugi::xml_document doc;
    const char* text = "\xEF\xBB\xBF<?xml version=\"1.0\" encoding=\"utf-8\"?>\n"
                       "<!-- a comment with <tags> -->\n"
                       "<scene version=\"3.0\">\n"
                       "  <default name=\"spp\" value=\"16\"/>\n"
                       "  <shape type='sphere' id = \"ball\">\n"
                       "    <float name=\"radius\" value=\"2.5\"/>\n"
                       "    <!-- inside -->\n"
                       "    <point name=\"center\" x=\"1\" y=\"-2\" z=\"3e1\"/>\n"
                       "  </shape>\n"
                       "  text &amp; more\r\nlines\n"
                       "  <![CDATA[<raw> & \"kept\"]]>\n"
                       "</scene>\n";
    pugi::xml_parse_result r = doc.load_string(text);
    CHECK(r);
    CHECK(r.status == pugi::status_ok);
    CHECK(Eq(r.description(), "No error"));

    pugi::xml_node scene = doc.child("scene");
    CHECK(scene);
    CHECK(scene == doc.document_element());
    CHECK(scene.parent() == doc);
    CHECK(Eq(scene.attribute("version").value(), "3.0"));
    CHECK(scene.attribute("version").as_float() == 3.0f);

    std::vector<std::string> names;
    std::vector<pugi::xml_node_type> types;
    for (auto child : scene.children())
    {
        names.push_back(child.name());
        types.push_back(child.type());
    }
    CHECK(names.size() == 4);
    if (names.size() == 4)
    {
        CHECK(names[0] == "default" && names[1] == "shape" && names[2].empty() && names[3].empty());
        CHECK(types[2] == pugi::node_pcdata && types[3] == pugi::node_cdata);
    }
    pugi::xml_node text_node = scene.child("shape").next_sibling();
    CHECK(text_node.type() == pugi::node_pcdata);
    CHECK(std::string(text_node.value()) == "\n  text & more\nlines\n  ");
    CHECK(Eq(text_node.next_sibling().value(), "<raw> & \"kept\""));
    CHECK(Eq(scene.child_value(), "\n  text & more\nlines\n  "));

    pugi::xml_node shape = scene.child("shape");
    CHECK(Eq(shape.attribute("type").value(), "sphere"));
    CHECK(Eq(shape.attribute("id").value(), "ball"));
    CHECK(Eq(shape.child("float").attribute("value").value(), "2.5"));
    pugi::xml_node point = shape.child("point");
    CHECK(point.attribute("z").as_double() == 30.0);
    CHECK(point.attribute("y").as_int() == -2);
    CHECK(point.previous_sibling() == shape.child("float")); // the comment is dropped
    CHECK(point.next_sibling().empty());

    // Missing things are empty handles with "" names and values.
    pugi::xml_attribute none = scene.attribute("missing");
    CHECK(!none);
    CHECK(none.empty());
    CHECK(Eq(none.value(), "") && Eq(none.name(), ""));
    CHECK(none.as_int(7) == 7);
    pugi::xml_node nothing = scene.child("nope");
    CHECK(!nothing && nothing.empty());
    CHECK(Eq(nothing.attribute("x").value(), ""));
    CHECK(Eq(nothing.name(), ""));
    CHECK(nothing.children().begin() == nothing.children().end());

    // Attribute iteration keeps document order.
    std::string attrs;
    for (pugi::xml_attribute a : point.attributes())
    {
        attrs += std::string(a.name()) + "=" + a.value() + ";";
    }
    CHECK(attrs == "name=center;x=1;y=-2;z=3e1;");
    CHECK(point.first_attribute().next_attribute().next_attribute() == point.attribute("y"));
    CHECK(point.last_attribute().previous_attribute() == point.attribute("y"));
}

void XmlNamedChildren()
{
    pugi::xml_document doc;
    CHECK(doc.load_string("<r><a i='1'/><b/><a i='2'/>t<a i='3'/></r>"));
    std::string seen;
    for (auto a : doc.child("r").children("a"))
    {
        seen += a.attribute("i").value();
    }
    CHECK(seen == "123");
    CHECK(Eq(doc.child("r").child("a").next_sibling("a").attribute("i").value(), "2"));
    CHECK(Eq(doc.child("r").last_child().previous_sibling("a").attribute("i").value(), "2"));
}

void XmlEscapes()
{
    pugi::xml_document doc;
    CHECK(doc.load_string("<a v=\"&lt;&gt;&amp;&quot;&apos;&#65;&#x42;&#x263A;&#128512;\" w='x\ty\r\nz\nq'"
                          " u='&unknown; &#xZZ; & &amp'>&#x3C;b&#62;</a>"));
    pugi::xml_node a = doc.child("a");
    CHECK(std::string(a.attribute("v").value()) == "<>&\"'AB\xE2\x98\xBA\xF0\x9F\x98\x80");
    CHECK(std::string(a.attribute("w").value()) == "x y z q");
    CHECK(std::string(a.attribute("u").value()) == "&unknown; &#xZZ; & &amp");
    CHECK(std::string(a.child_value()) == "<b>");
}

void XmlErrors()
{
    CHECK(Status("<a></b>") == pugi::status_end_element_mismatch);
    CHECK(Status("<a><b></a></b>") == pugi::status_end_element_mismatch);
    CHECK(Status("<a>") == pugi::status_end_element_mismatch);
    CHECK(Status("</a>") == pugi::status_end_element_mismatch);
    CHECK(Status("<a b=c/>") == pugi::status_bad_attribute);
    CHECK(Status("<a b='c/>") == pugi::status_bad_attribute);
    CHECK(Status("<a b/>") == pugi::status_bad_attribute);
    CHECK(Status("<a b='1'c='2'/>") == pugi::status_bad_attribute);
    CHECK(Status("<a/ >") == pugi::status_bad_start_element);
    CHECK(Status("<a") == pugi::status_bad_start_element);
    CHECK(Status("<a></a x>") == pugi::status_bad_end_element);
    CHECK(Status("<a><!-- x</a>") == pugi::status_bad_comment);
    CHECK(Status("<a><![CDATA[x</a>") == pugi::status_bad_cdata);
    CHECK(Status("<?xml version='1.0'") == pugi::status_bad_pi);
    CHECK(Status("<!DOCTYPE a [<!ENTITY e 'x'>") == pugi::status_bad_doctype);
    CHECK(Status("<a><1/></a>") == pugi::status_unrecognized_tag);
    CHECK(Status("<a>1 < 2</a>") == pugi::status_unrecognized_tag);
    CHECK(Status("") == pugi::status_no_document_element);
    CHECK(Status("  <!-- only a comment -->  ") == pugi::status_no_document_element);
    CHECK(Status("<!DOCTYPE x [ <!ENTITY e \"v>\"> ]><x/>") == pugi::status_ok);

    pugi::xml_document doc;
    pugi::xml_parse_result r = doc.load_string("<a>\n<b></c></a>");
    CHECK(!r && r.offset == 7); // at the "</c>"
    CHECK(Eq(r.description(), "Start and end tags do not match"));
    CHECK(doc.child("a").child("b")); // the nodes read before the error stay
    r = doc.load_file("/nonexistent/dir/scene.xml");
    CHECK(r.status == pugi::status_file_not_found);
    CHECK(Eq(r.description(), "File was not found"));
    CHECK(!doc.document_element());
}

// ------------------------------------------------------------------ OBJ

const char* kMtl = "# materials\n"
                   "newmtl red\n"
                   "Kd 0.8 0.1 0.1\n"
                   "Ke 2\n"
                   "Ns 10\nNi 1.45\nTr 0.25\nillum 2\n"
                   "map_Kd -bm 0.5 -o 1 1 1 textures/red.png\n"
                   "Pr 0.3\nPm 0.9\n"
                   "Xy custom value\n"
                   "newmtl blue\r\n"
                   "Kd 0.1 0.1 0.9\r\n";

const char* kObj = "# two shapes\n"
                   "mtllib scene.mtl\n"
                   "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\n"
                   "v 0 0 1 0.5 0.25 1\n"
                   "vt 0 0\nvt 1 0\nvt 1 1\nvt 0.5\n"
                   "vn 0 0 1\n"
                   "o quad\n"
                   "usemtl red\n"
                   "s 1\n"
                   "f 1/1/1 2/2/1 3/3/1 4/4/1\n"
                   "usemtl missing\n"
                   "f -5//1 -4//1 -1//1\n"
                   "g second\n"
                   "usemtl blue\n"
                   "s off\n"
                   "f 1 2 3 4 5\n"
                   "l 1 2 3\n"
                   "p 4\n";

void ObjFromString()
{
    tinyobj::ObjReader reader;
    CHECK(reader.ParseFromString(kObj, kMtl));
    CHECK(reader.Valid());
    const auto& attrib = reader.GetAttrib();
    const auto& shapes = reader.GetShapes();
    const auto& mats = reader.GetMaterials();
    CHECK(attrib.vertices.size() == 15 && attrib.normals.size() == 3 && attrib.texcoords.size() == 8);
    CHECK(attrib.colors.size() == 15); // one vertex carries a colour: all get one (1 by default)
    CHECK(attrib.colors[12] == 0.5f && attrib.colors[13] == 0.25f && attrib.colors[0] == 1.0f);
    CHECK(attrib.texcoords[6] == 0.5f && attrib.texcoords[7] == 0.0f);

    CHECK(mats.size() == 2);
    if (mats.size() == 2)
    {
        CHECK(mats[0].name == "red" && mats[1].name == "blue");
        CHECK(mats[0].diffuse[0] == 0.8f && mats[0].diffuse[2] == 0.1f);
        CHECK(mats[0].emission[0] == 2 && mats[0].emission[1] == 2 && mats[0].emission[2] == 2);
        CHECK(mats[0].shininess == 10 && mats[0].ior == 1.45f && mats[0].dissolve == 0.75f && mats[0].illum == 2);
        CHECK(mats[0].diffuse_texname == "textures/red.png");
        CHECK(mats[0].roughness == 0.3f && mats[0].metallic == 0.9f);
        CHECK(mats[0].unknown_parameter.count("Xy") && mats[0].unknown_parameter.at("Xy") == "custom value");
        CHECK(mats[1].diffuse[2] == 0.9f);
    }

    CHECK(shapes.size() == 2);
    if (shapes.size() != 2)
    {
        return;
    }
    const tinyobj::mesh_t& q = shapes[0].mesh;
    CHECK(shapes[0].name == "quad");
    // The square's diagonals tie: split along 0-2. Then the relative triangle.
    CHECK(q.num_face_vertices.size() == 3);
    CHECK(q.indices.size() == 9);
    if (q.indices.size() == 9)
    {
        const int want[9] = { 0, 1, 2, 0, 2, 3, 0, 1, 4 };
        bool same = true;
        for (int k = 0; k < 9; ++k)
        {
            same = same && q.indices[size_t(k)].vertex_index == want[k];
        }
        CHECK(same);
        CHECK(q.indices[1].texcoord_index == 1 && q.indices[1].normal_index == 0);
        CHECK(q.indices[6].texcoord_index == -1 && q.indices[6].normal_index == 0);
    }
    CHECK(q.material_ids.size() == 3 && q.material_ids[0] == 0 && q.material_ids[1] == 0 && q.material_ids[2] == -1);
    CHECK(q.smoothing_group_ids[0] == 1);
    CHECK(reader.Warning().find("missing") != std::string::npos);

    const tinyobj::shape_t& s = shapes[1];
    CHECK(s.name == "second");
    CHECK(s.mesh.num_face_vertices.size() == 3); // pentagon fan
    CHECK(s.mesh.indices.size() == 9 && s.mesh.indices[3].vertex_index == 0 && s.mesh.indices[8].vertex_index == 4);
    CHECK(s.mesh.material_ids[2] == 1 && s.mesh.smoothing_group_ids[2] == 0);
    CHECK(s.lines.indices.size() == 3 && s.lines.num_line_vertices.size() == 1);
    CHECK(s.points.indices.size() == 1 && s.points.indices[0].vertex_index == 3);
}

void ObjQuadDiagonal()
{
    // A long thin quad whose 1-3 diagonal is the shorter one.
    tinyobj::ObjReader reader;
    CHECK(reader.ParseFromString("v 0 0 0\nv 4 0 0\nv 5 1 0\nv 1 1 0\nf 1 2 3 4\n", ""));
    const auto& m = reader.GetShapes().at(0).mesh;
    CHECK(m.indices.size() == 6 && m.indices[2].vertex_index == 3 && m.indices[3].vertex_index == 1);
    CHECK(reader.GetShapes().at(0).name.empty());

    tinyobj::ObjReaderConfig keep;
    keep.triangulate = false;
    CHECK(reader.ParseFromString("v 0 0 0\nv 4 0 0\nv 5 1 0\nv 1 1 0\nf 1 2 3 4\n", "", keep));
    CHECK(reader.GetShapes().at(0).mesh.num_face_vertices.at(0) == 4);
}

void ObjErrors()
{
    tinyobj::ObjReader reader;
    CHECK(!reader.ParseFromString("v 0 0 0\nv 1 0 0\nv 1 1 0\nf 0 1 2\n", ""));
    CHECK(!reader.Valid());
    CHECK(reader.Error().find("line 4") != std::string::npos);
    CHECK(!reader.ParseFromString("v 0 0 0\nv 1 0 0\nv 1 1 0\nf 1 2 4\n", ""));
    CHECK(!reader.ParseFromString("v 0 0 0\nv 1 0 0\nv 1 1 0\nf 1 2 -4\n", ""));
    CHECK(!reader.ParseFromString("v 0 0 0\nv 1 0 0\nv 1 1 0\nf 1/2 2 3\n", ""));
    CHECK(!reader.ParseFromString("v 0 0 zero\n", ""));
    CHECK(!reader.ParseFromFile("/nonexistent/model.obj"));
    CHECK(reader.ParseFromString("v 0 0 0\nv 1 0 0\nf 1 2\n", "")); // degenerate face: a warning
    CHECK(reader.GetShapes().empty() && !reader.Warning().empty());
}

void ObjFromFile(const std::string& dir)
{
    {
        std::ofstream(dir + "/m.obj") << "mtllib m.mtl other.mtl\nv 0 0 0\nv 1 0 0\nv 0 1 0\nusemtl only\nf 1 2 3\n";
        std::ofstream(dir + "/m.mtl") << "newmtl only\nKd 0.5 0.5 0.5\n";
    }
    tinyobj::ObjReader reader;
    CHECK(reader.ParseFromFile(dir + "/m.obj"));
    CHECK(reader.GetMaterials().size() == 1);
    CHECK(reader.GetShapes().size() == 1 && reader.GetShapes()[0].mesh.material_ids[0] == 0);

    tinyobj::attrib_t attrib;
    std::vector<tinyobj::shape_t> shapes;
    std::vector<tinyobj::material_t> mats;
    std::string warn, err;
    CHECK(tinyobj::LoadObj(&attrib, &shapes, &mats, &warn, &err, (dir + "/m.obj").c_str(), (dir + "/").c_str()));
    CHECK(attrib.vertices.size() == 9 && mats.size() == 1 && err.empty());
}

// ----------------------------------------------------------------- glTF

std::string Base64(const std::vector<unsigned char>& bytes)
{
    static const char* kAlphabet = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    std::string out;
    size_t i = 0;
    for (; i + 2 < bytes.size(); i += 3)
    {
        uint32_t v = (uint32_t(bytes[i]) << 16) | (uint32_t(bytes[i + 1]) << 8) | bytes[i + 2];
        out += kAlphabet[(v >> 18) & 63];
        out += kAlphabet[(v >> 12) & 63];
        out += kAlphabet[(v >> 6) & 63];
        out += kAlphabet[v & 63];
    }
    if (i + 1 == bytes.size())
    {
        uint32_t v = uint32_t(bytes[i]) << 16;
        out += kAlphabet[(v >> 18) & 63];
        out += kAlphabet[(v >> 12) & 63];
        out += "==";
    }
    else if (i + 2 == bytes.size())
    {
        uint32_t v = (uint32_t(bytes[i]) << 16) | (uint32_t(bytes[i + 1]) << 8);
        out += kAlphabet[(v >> 18) & 63];
        out += kAlphabet[(v >> 12) & 63];
        out += kAlphabet[(v >> 6) & 63];
        out += '=';
    }
    return out;
}

template <typename T>
void Put(std::vector<unsigned char>* out, const T& v)
{
    const unsigned char* p = reinterpret_cast<const unsigned char*>(&v);
    out->insert(out->end(), p, p + sizeof(T));
}

// One triangle: 3 positions, 3 normals, 3 texcoords (floats), 3 u16 indices.
std::vector<unsigned char> TriangleBytes()
{
    std::vector<unsigned char> b;
    const float pos[9] = { 0, 0, 0, 1, 0, 0, 0, 1, 0 };
    const float nrm[9] = { 0, 0, 1, 0, 0, 1, 0, 0, 1 };
    const float uv[6] = { 0, 0, 1, 0, 0, 1 };
    for (float f : pos) Put(&b, f);
    for (float f : nrm) Put(&b, f);
    for (float f : uv) Put(&b, f);
    for (uint16_t i : { uint16_t(0), uint16_t(1), uint16_t(2) }) Put(&b, i);
    return b; // 36 + 36 + 24 + 6 = 102 bytes
}

std::string TriangleJson(const std::string& buffer_uri_member, size_t index_count = 3, const char* extra_node = "")
{
    return std::string("{\"asset\":{\"version\":\"2.0\",\"generator\":\"t\\u00e9st \\ud83d\\ude00\"},\"scene\":0,"
                       "\"scenes\":[{\"nodes\":[0]}],"
                       "\"nodes\":[{\"mesh\":0,\"children\":[1],\"matrix\":[1,0,0,0,0,1,0,0,0,0,1,0,2,0,0,1]},"
                       "{\"translation\":[0,1,0]}") +
           extra_node +
           "],"
           "\"meshes\":[{\"primitives\":[{\"attributes\":{\"POSITION\":0,\"NORMAL\":1,\"TEXCOORD_0\":2},"
           "\"indices\":3,\"material\":0}]}],"
           "\"materials\":[{\"name\":\"m\",\"pbrMetallicRoughness\":{\"baseColorFactor\":[0.5,0.25,1,1],"
           "\"metallicFactor\":0},\"extensions\":{\"KHR_materials_ior\":{\"ior\":1.33},"
           "\"KHR_materials_anisotropy\":{\"anisotropyStrength\":1,\"anisotropyTexture\":{\"index\":0}}}}],"
           "\"accessors\":["
           "{\"bufferView\":0,\"componentType\":5126,\"count\":3,\"type\":\"VEC3\",\"max\":[1,1,0],\"min\":[0,0,0]},"
           "{\"bufferView\":0,\"byteOffset\":36,\"componentType\":5126,\"count\":3,\"type\":\"VEC3\"},"
           "{\"bufferView\":0,\"byteOffset\":72,\"componentType\":5126,\"count\":3,\"type\":\"VEC2\"},"
           "{\"bufferView\":1,\"componentType\":5123,\"count\":" +
           std::to_string(index_count) +
           ",\"type\":\"SCALAR\"}],"
           "\"bufferViews\":[{\"buffer\":0,\"byteLength\":96},{\"buffer\":0,\"byteOffset\":96,\"byteLength\":6}],"
           "\"buffers\":[{\"byteLength\":102" +
           buffer_uri_member + "}]}";
}

void CheckTriangleModel(const tinygltf::Model& m)
{
    CHECK(m.asset.version == "2.0");
    CHECK(m.asset.generator == "t\xC3\xA9st \xF0\x9F\x98\x80");
    CHECK(m.defaultScene == 0 && m.scenes.size() == 1 && m.scenes[0].nodes.size() == 1);
    CHECK(m.nodes.size() == 2 && m.nodes[0].matrix.size() == 16 && m.nodes[0].matrix[12] == 2.0);
    CHECK(m.nodes[0].children.size() == 1 && m.nodes[1].translation.size() == 3 && m.nodes[1].mesh == -1);
    CHECK(m.meshes.size() == 1 && m.meshes[0].primitives.size() == 1);
    const tinygltf::Primitive& p = m.meshes[0].primitives[0];
    CHECK(p.mode == TINYGLTF_MODE_TRIANGLES && p.indices == 3 && p.material == 0);
    CHECK(p.attributes.at("POSITION") == 0 && p.attributes.at("TEXCOORD_0") == 2);
    CHECK(m.accessors.size() == 4);
    CHECK(m.accessors[0].type == TINYGLTF_TYPE_VEC3 && m.accessors[3].type == TINYGLTF_TYPE_SCALAR);
    CHECK(tinygltf::GetComponentSizeInBytes(unsigned(m.accessors[3].componentType)) == 2);
    CHECK(tinygltf::GetNumComponentsInType(unsigned(m.accessors[2].type)) == 2);
    CHECK(m.accessors[0].maxValues.size() == 3 && m.accessors[0].maxValues[1] == 1.0);
    CHECK(m.buffers.size() == 1 && m.buffers[0].data == TriangleBytes());
    float y1 = 0;
    std::memcpy(&y1, m.buffers[0].data.data() + m.bufferViews[0].byteOffset + m.accessors[0].byteOffset + 7 * 4, 4);
    CHECK(y1 == 1.0f);

    const tinygltf::Material& mat = m.materials.at(0);
    CHECK(mat.name == "m" && mat.pbrMetallicRoughness.baseColorFactor[1] == 0.25);
    CHECK(mat.pbrMetallicRoughness.metallicFactor == 0 && mat.pbrMetallicRoughness.roughnessFactor == 1);
    CHECK(mat.emissiveFactor.size() == 3 && mat.emissiveFactor[0] == 0 && mat.normalTexture.index == -1);
    CHECK(mat.extensions.count("KHR_materials_ior") == 1);
    const tinygltf::Value& ior = mat.extensions.at("KHR_materials_ior");
    CHECK(ior.Has("ior") && std::fabs(ior.Get("ior").Get<double>() - 1.33) < 1e-12);
    const tinygltf::Value& an = mat.extensions.at("KHR_materials_anisotropy");
    CHECK(an.Get("anisotropyStrength").Get<double>() == 1.0); // an integer reads as a real too
    CHECK(an.Get("anisotropyTexture").Get("index").Get<int>() == 0);
    CHECK(!an.Has("nothing") && an.Get("nothing").Type() == tinygltf::NULL_TYPE);
}

void GltfAscii(const std::string& dir)
{
    const std::vector<unsigned char> bytes = TriangleBytes();
    tinygltf::TinyGLTF loader;
    tinygltf::Model m;
    std::string err, warn;

    std::string json = TriangleJson(",\"uri\":\"data:application/octet-stream;base64," + Base64(bytes) + "\"");
    CHECK(loader.LoadASCIIFromString(&m, &err, &warn, json.c_str(), unsigned(json.size()), ""));
    CHECK(err.empty());
    CheckTriangleModel(m);

    // The same buffer as a file next to the .gltf, with a space in its name.
    {
        std::ofstream f(dir + "/tri data.bin", std::ios::binary);
        f.write(reinterpret_cast<const char*>(bytes.data()), std::streamsize(bytes.size()));
        std::ofstream(dir + "/tri.gltf") << TriangleJson(",\"uri\":\"tri%20data.bin\"");
    }
    tinygltf::Model m2;
    CHECK(loader.LoadASCIIFromFile(&m2, &err, &warn, dir + "/tri.gltf"));
    CheckTriangleModel(m2);
}

void GltfBinary()
{
    const std::vector<unsigned char> bytes = TriangleBytes();
    std::string json = TriangleJson("");
    while (json.size() % 4) json += ' ';
    std::vector<unsigned char> bin = bytes;
    while (bin.size() % 4) bin.push_back(0);
    std::vector<unsigned char> glb;
    Put(&glb, uint32_t(0x46546C67));
    Put(&glb, uint32_t(2));
    Put(&glb, uint32_t(12 + 8 + json.size() + 8 + bin.size()));
    Put(&glb, uint32_t(json.size()));
    Put(&glb, uint32_t(0x4E4F534A));
    glb.insert(glb.end(), json.begin(), json.end());
    Put(&glb, uint32_t(bin.size()));
    Put(&glb, uint32_t(0x004E4942));
    glb.insert(glb.end(), bin.begin(), bin.end());

    tinygltf::TinyGLTF loader;
    tinygltf::Model m;
    std::string err, warn;
    CHECK(loader.LoadBinaryFromMemory(&m, &err, &warn, glb.data(), unsigned(glb.size())));
    CheckTriangleModel(m); // the padded BIN chunk is cut to byteLength

    std::vector<unsigned char> cut(glb.begin(), glb.begin() + 40);
    CHECK(!loader.LoadBinaryFromMemory(&m, &err, &warn, cut.data(), unsigned(cut.size())));
    std::vector<unsigned char> text(json.begin(), json.end());
    CHECK(!loader.LoadBinaryFromMemory(&m, &err, &warn, text.data(), unsigned(text.size())));
}

void GltfImagesAndErrors()
{
    const std::vector<unsigned char> bytes = TriangleBytes();
    const std::string uri = ",\"uri\":\"data:application/octet-stream;base64," + Base64(bytes) + "\"";
    tinygltf::TinyGLTF loader;
    tinygltf::Model m;
    std::string err, warn;

    // An embedded image goes to the image loader; without one its bytes are kept.
    std::string with_image = TriangleJson(uri);
    with_image.insert(with_image.size() - 1, ",\"images\":[{\"uri\":\"data:image/png;base64,AAEC\"}],"
                                             "\"textures\":[{\"source\":0}]");
    int calls = 0, seen_size = -1;
    loader.SetImageLoader(
        [&](tinygltf::Image* img, const int, std::string*, std::string*, int, int, const unsigned char*, int size,
            void* user) {
            ++calls;
            seen_size = size;
            img->width = 1;
            return user == &calls;
        },
        &calls);
    CHECK(loader.LoadASCIIFromString(&m, &err, &warn, with_image.c_str(), unsigned(with_image.size()), ""));
    CHECK(calls == 1 && seen_size == 3 && m.images.size() == 1 && m.images[0].width == 1);
    tinygltf::TinyGLTF plain;
    CHECK(plain.LoadASCIIFromString(&m, &err, &warn, with_image.c_str(), unsigned(with_image.size()), ""));
    CHECK(m.images.size() == 1 && m.images[0].image.size() == 3 && m.images[0].image[2] == 2);

    auto fails = [&](const std::string& json, const char* needle) {
        std::string e, w;
        tinygltf::Model mm;
        bool ok = plain.LoadASCIIFromString(&mm, &e, &w, json.c_str(), unsigned(json.size()), "");
        return !ok && e.find(needle) != std::string::npos;
    };
    CHECK(fails(TriangleJson(uri, 4), "accessor 3")); // 4 indices in a 6-byte view
    CHECK(fails(TriangleJson(uri, 3, ",{\"children\":[2]}"), "own ancestor"));
    CHECK(fails(TriangleJson(uri, 3, ",{\"children\":[1]}"), "two parents"));
    CHECK(fails(TriangleJson(""), "no uri"));
    CHECK(fails(TriangleJson(",\"uri\":\"missing.bin\""), "cannot read"));
    CHECK(fails("{\"asset\":{\"version\":\"2.0\"},\"nodes\":[{\"mesh\":0}]}", "node 0"));
    CHECK(fails("{\"asset\":{\"version\":\"2.0\"},\"nodes\":[{\"mesh\":1e10}]}", "node 0"));
    CHECK(fails("{\"asset\":{\"version\":\"2.0\"},\"buffers\":[{\"byteLength\":1e300}]}", "byteLength"));
    CHECK(fails("{\"asset\":{}}", "asset.version"));
    CHECK(fails("{\"asset\":{\"version\":\"2.0\"},}", "JSON error"));
    CHECK(fails("{\"asset\":{\"version\":\"2.0\"}} x", "JSON error"));
    CHECK(fails("[1,2]", "not an object"));
    CHECK(fails("{\"a\":\"\\ud800\"}", "surrogate"));
    CHECK(!loader.LoadASCIIFromFile(&m, &err, &warn, "/nonexistent/model.gltf"));
}

} // namespace

int main(int argc, char** argv)
{
    const std::string dir = argc > 1 ? argv[1] : ".";
    XmlDocumentTree();
    XmlNamedChildren();
    XmlEscapes();
    XmlErrors();
    ObjFromString();
    ObjQuadDiagonal();
    ObjErrors();
    ObjFromFile(dir);
    GltfAscii(dir);
    GltfBinary();
    GltfImagesAndErrors();
    std::printf("%d of %d checks passed\n", g_checks - g_failures, g_checks);
    return g_failures;
}
