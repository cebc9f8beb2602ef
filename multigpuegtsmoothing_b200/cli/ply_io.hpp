// Minimal PLY reader/writer for the KNNCUDA command line.
//
// Reads what the reference reads through miniply (MeshPLY.cpp:8-53): vertex
// positions x,y,z (any numeric type), optional normals nx,ny,nz and colours
// red,green,blue, and the first three indices of every face list
// (vertex_indices / vertex_index).  ASCII, binary little- and big-endian input.
// Writes exactly the reference's output layout (MeshPLY.cpp:67-127): binary
// little-endian, float x y z [nx ny nz] [uchar red green blue], faces as
// "list uchar uint vertex_indices".
//
// Large files: the input is mapped into memory, and the common layouts are
// decoded in parallel on the host cores -- binary elements without lists
// (fixed-size records), binary face lists that hold only triangles, and ASCII
// vertex and face elements written one record per line.  Any other layout (a
// record spread over several lines, polygons other than triangles, lists
// inside the vertex element) is read sequentially with the same value
// conversions, so every layout gives the same result.  The output is laid out
// in memory in parallel and written with one call.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace ply {

struct Mesh {
    std::vector<float> xyz;      // 3 per vertex
    std::vector<float> normals;  // 3 per vertex, or empty
    std::vector<uint8_t> rgb;    // 3 per vertex, or empty
    std::vector<uint32_t> tris;  // 3 per face
    size_t nV() const { return xyz.size() / 3; }
    size_t nF() const { return tris.size() / 3; }
};

// Returns false and sets err on failure.
bool read(const std::string& path, Mesh& m, std::string& err);
bool write(const std::string& path, const Mesh& m, std::string& err);

}  // namespace ply
