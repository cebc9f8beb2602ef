#include "ply_io.hpp"

#include <cstring>
#include <fstream>
#include <sstream>

namespace ply {
namespace {

enum class T { I8, U8, I16, U16, I32, U32, F32, F64, None };

T parse_type(const std::string& s) {
    if (s == "char" || s == "int8") return T::I8;
    if (s == "uchar" || s == "uint8") return T::U8;
    if (s == "short" || s == "int16") return T::I16;
    if (s == "ushort" || s == "uint16") return T::U16;
    if (s == "int" || s == "int32") return T::I32;
    if (s == "uint" || s == "uint32") return T::U32;
    if (s == "float" || s == "float32") return T::F32;
    if (s == "double" || s == "float64") return T::F64;
    return T::None;
}

size_t type_size(T t) {
    switch (t) {
        case T::I8: case T::U8: return 1;
        case T::I16: case T::U16: return 2;
        case T::I32: case T::U32: case T::F32: return 4;
        case T::F64: return 8;
        default: return 0;
    }
}

struct Prop {
    std::string name;
    T type = T::None;
    bool list = false;
    T count_type = T::None;
};

struct Element {
    std::string name;
    size_t count = 0;
    std::vector<Prop> props;
};

enum class Fmt { Ascii, LE, BE };

struct Reader {
    std::istream& in;
    Fmt fmt;
    bool ok = true;

    double value(T t) {
        if (fmt == Fmt::Ascii) {
            double v = 0;
            if (!(in >> v)) ok = false;
            return v;
        }
        unsigned char b[8];
        size_t n = type_size(t);
        if (!in.read(reinterpret_cast<char*>(b), (std::streamsize)n)) { ok = false; return 0; }
        if (fmt == Fmt::BE)
            for (size_t i = 0; i < n / 2; i++) std::swap(b[i], b[n - 1 - i]);
        switch (t) {
            case T::I8: { int8_t v; std::memcpy(&v, b, 1); return v; }
            case T::U8: { uint8_t v; std::memcpy(&v, b, 1); return v; }
            case T::I16: { int16_t v; std::memcpy(&v, b, 2); return v; }
            case T::U16: { uint16_t v; std::memcpy(&v, b, 2); return v; }
            case T::I32: { int32_t v; std::memcpy(&v, b, 4); return v; }
            case T::U32: { uint32_t v; std::memcpy(&v, b, 4); return v; }
            case T::F32: { float v; std::memcpy(&v, b, 4); return v; }
            case T::F64: { double v; std::memcpy(&v, b, 8); return v; }
            default: ok = false; return 0;
        }
    }
};

int find(const Element& e, std::initializer_list<const char*> names) {
    for (size_t i = 0; i < e.props.size(); i++)
        for (const char* n : names)
            if (e.props[i].name == n) return (int)i;
    return -1;
}

}  // namespace

bool read(const std::string& path, Mesh& m, std::string& err) {
    std::ifstream f(path, std::ios::binary);
    if (!f) { err = "cannot open " + path; return false; }
    std::string line;
    std::getline(f, line);
    if (line.rfind("ply", 0) != 0) { err = "not a PLY file"; return false; }
    Fmt fmt = Fmt::Ascii;
    std::vector<Element> elems;
    while (std::getline(f, line)) {
        if (!line.empty() && line.back() == '\r') line.pop_back();
        std::istringstream ls(line);
        std::string w;
        ls >> w;
        if (w == "format") {
            std::string fm;
            ls >> fm;
            if (fm == "ascii") fmt = Fmt::Ascii;
            else if (fm == "binary_little_endian") fmt = Fmt::LE;
            else if (fm == "binary_big_endian") fmt = Fmt::BE;
            else { err = "unknown format " + fm; return false; }
        } else if (w == "element") {
            Element e;
            ls >> e.name >> e.count;
            elems.push_back(e);
        } else if (w == "property") {
            if (elems.empty()) { err = "property before element"; return false; }
            Prop p;
            std::string t;
            ls >> t;
            if (t == "list") {
                std::string ct, it;
                ls >> ct >> it >> p.name;
                p.list = true;
                p.count_type = parse_type(ct);
                p.type = parse_type(it);
            } else {
                p.type = parse_type(t);
                ls >> p.name;
            }
            if (p.type == T::None || (p.list && p.count_type == T::None)) { err = "bad property type"; return false; }
            elems.back().props.push_back(p);
        } else if (w == "end_header") {
            break;
        }
    }
    Reader rd{f, fmt};
    m = Mesh();
    for (const Element& e : elems) {
        const bool vert = e.name == "vertex", face = e.name == "face";
        int ix = -1, iy = -1, iz = -1, inx = -1, iny = -1, inz = -1, ir = -1, ig = -1, ib = -1, il = -1;
        if (vert) {
            ix = find(e, {"x"}); iy = find(e, {"y"}); iz = find(e, {"z"});
            if (ix < 0 || iy < 0 || iz < 0) { err = "vertex element without x,y,z"; return false; }
            inx = find(e, {"nx"}); iny = find(e, {"ny"}); inz = find(e, {"nz"});
            ir = find(e, {"red", "r"}); ig = find(e, {"green", "g"}); ib = find(e, {"blue", "b"});
            m.xyz.resize(3 * e.count);
            if (inx >= 0 && iny >= 0 && inz >= 0) m.normals.resize(3 * e.count);
            if (ir >= 0 && ig >= 0 && ib >= 0) m.rgb.resize(3 * e.count);
        }
        if (face) il = find(e, {"vertex_indices", "vertex_index"});
        std::vector<double> vals(e.props.size());
        for (size_t r = 0; r < e.count; r++) {
            for (size_t pi = 0; pi < e.props.size(); pi++) {
                const Prop& p = e.props[pi];
                if (!p.list) { vals[pi] = rd.value(p.type); continue; }
                size_t cnt = (size_t)rd.value(p.count_type);
                uint32_t idx[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
                for (size_t c = 0; c < cnt; c++) {
                    double v = rd.value(p.type);
                    if (c < 3) idx[c] = (uint32_t)(int64_t)v;
                }
                if (face && (int)pi == il) {
                    m.tris.push_back(idx[0]); m.tris.push_back(idx[1]); m.tris.push_back(idx[2]);
                }
            }
            if (!rd.ok) { err = "truncated " + e.name + " data"; return false; }
            if (vert) {
                m.xyz[3 * r] = (float)vals[ix]; m.xyz[3 * r + 1] = (float)vals[iy]; m.xyz[3 * r + 2] = (float)vals[iz];
                if (!m.normals.empty()) {
                    m.normals[3 * r] = (float)vals[inx]; m.normals[3 * r + 1] = (float)vals[iny];
                    m.normals[3 * r + 2] = (float)vals[inz];
                }
                if (!m.rgb.empty()) {
                    m.rgb[3 * r] = (uint8_t)vals[ir]; m.rgb[3 * r + 1] = (uint8_t)vals[ig]; m.rgb[3 * r + 2] = (uint8_t)vals[ib];
                }
            }
        }
    }
    return true;
}

bool write(const std::string& path, const Mesh& m, std::string& err) {
    std::ofstream f(path, std::ios::binary | std::ios::out | std::ios::trunc);
    if (!f) { err = "cannot write " + path; return false; }
    const size_t nv = m.nV(), nf = m.nF();
    const bool hasN = m.normals.size() == 3 * nv && nv > 0;
    const bool hasC = m.rgb.size() == 3 * nv && nv > 0;
    f << "ply\n" << "format binary_little_endian 1.0\n" << "element vertex " << nv << "\n";
    f << "property float x\n" << "property float y\n" << "property float z\n";
    if (hasN) f << "property float nx\n" << "property float ny\n" << "property float nz\n";
    if (hasC) f << "property uchar red\n" << "property uchar green\n" << "property uchar blue\n";
    if (nf) f << "element face " << nf << "\n" << "property list uchar uint vertex_indices\n";
    f << "end_header\n";
    for (size_t i = 0; i < nv; i++) {
        f.write(reinterpret_cast<const char*>(&m.xyz[3 * i]), 12);
        if (hasN) f.write(reinterpret_cast<const char*>(&m.normals[3 * i]), 12);
        if (hasC) f.write(reinterpret_cast<const char*>(&m.rgb[3 * i]), 3);
    }
    const unsigned char three = 3;
    for (size_t i = 0; i < nf; i++) {
        f.write(reinterpret_cast<const char*>(&three), 1);
        f.write(reinterpret_cast<const char*>(&m.tris[3 * i]), 12);
    }
    if (!f) { err = "write failed"; return false; }
    return true;
}

}  // namespace ply
