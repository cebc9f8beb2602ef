#include "ply_io.hpp"

#include <algorithm>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <thread>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

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

// One binary value at p, converted through double: every property reaches
// its destination type by the same double -> target conversion, whatever its
// stored type and byte order.
double load(const unsigned char* p, T t, bool swap) {
    unsigned char b[8];
    const size_t n = type_size(t);
    std::memcpy(b, p, n);
    if (swap)
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
        default: return 0;
    }
}

bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\r' || c == '\v' || c == '\f'; }

// Parses one decimal number starting at or after p (skipping whitespace);
// returns the position after it, or nullptr when none is there.
const char* parse_number(const char* p, const char* end, double& v) {
    while (p < end && is_space(*p)) p++;
    if (p == end) return nullptr;
    const char* s = p;
    if (*s == '+') s++;  // from_chars takes no leading '+'
    const auto r = std::from_chars(s, end, v);
    if (r.ec != std::errc()) return nullptr;
    return r.ptr;
}

int find(const Element& e, std::initializer_list<const char*> names) {
    for (size_t i = 0; i < e.props.size(); i++)
        for (const char* n : names)
            if (e.props[i].name == n) return (int)i;
    return -1;
}

unsigned worker_count(size_t items) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    return (unsigned)std::max<size_t>(1, std::min<size_t>(hw, items / 65536));
}

// Runs fn(begin, end) over [0, n) in contiguous ranges, one per worker.
template <class F>
void parallel_ranges(size_t n, F fn) {
    const unsigned w = worker_count(n);
    if (w <= 1) { fn(size_t(0), n); return; }
    std::vector<std::thread> pool;
    for (unsigned t = 0; t < w; t++) {
        const size_t b = n * t / w, e = n * (t + 1) / w;
        pool.emplace_back([=] { fn(b, e); });
    }
    for (auto& th : pool) th.join();
}

// Where the vertex properties the mesh keeps sit among an element's
// properties, and the destination arrays.
struct VertexMap {
    int ix = -1, iy = -1, iz = -1, inx = -1, iny = -1, inz = -1, ir = -1, ig = -1, ib = -1;
    bool normals = false, rgb = false;
};

void store_vertex(Mesh& m, const VertexMap& vm, size_t r, const double* vals) {
    m.xyz[3 * r] = (float)vals[vm.ix];
    m.xyz[3 * r + 1] = (float)vals[vm.iy];
    m.xyz[3 * r + 2] = (float)vals[vm.iz];
    if (vm.normals) {
        m.normals[3 * r] = (float)vals[vm.inx];
        m.normals[3 * r + 1] = (float)vals[vm.iny];
        m.normals[3 * r + 2] = (float)vals[vm.inz];
    }
    if (vm.rgb) {
        m.rgb[3 * r] = (uint8_t)vals[vm.ir];
        m.rgb[3 * r + 1] = (uint8_t)vals[vm.ig];
        m.rgb[3 * r + 2] = (uint8_t)vals[vm.ib];
    }
}

// Sequential reader of one element's records, for any layout: binary records
// with lists, or ASCII tokens with records spread over lines in any way.
struct Cursor {
    const unsigned char* p;
    const unsigned char* end;
    Fmt fmt;
    bool ok = true;

    double value(T t) {
        if (fmt == Fmt::Ascii) {
            double v = 0;
            const char* q = parse_number(reinterpret_cast<const char*>(p), reinterpret_cast<const char*>(end), v);
            if (!q) { ok = false; return 0; }
            p = reinterpret_cast<const unsigned char*>(q);
            return v;
        }
        const size_t n = type_size(t);
        if ((size_t)(end - p) < n) { ok = false; return 0; }
        const double v = load(p, t, fmt == Fmt::BE);
        p += n;
        return v;
    }
};

// Reads the records of element e one at a time through the cursor.
bool read_sequential(Cursor& cur, const Element& e, Mesh& m, const VertexMap* vm, int list_face, size_t first) {
    std::vector<double> vals(e.props.size());
    for (size_t r = first; r < e.count; r++) {
        for (size_t pi = 0; pi < e.props.size(); pi++) {
            const Prop& p = e.props[pi];
            if (!p.list) { vals[pi] = cur.value(p.type); continue; }
            const size_t cnt = (size_t)cur.value(p.count_type);
            if (!cur.ok) break;
            uint32_t idx[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
            for (size_t c = 0; c < cnt && cur.ok; c++) {
                const double v = cur.value(p.type);
                if (c < 3) idx[c] = (uint32_t)(int64_t)v;
            }
            if ((int)pi == list_face) {
                m.tris.push_back(idx[0]); m.tris.push_back(idx[1]); m.tris.push_back(idx[2]);
            }
        }
        if (!cur.ok) return false;
        if (vm) store_vertex(m, *vm, r, vals.data());
    }
    return true;
}

// Binary element without lists: fixed-size records, decoded in parallel.
bool read_binary_fixed(const unsigned char*& p, const unsigned char* end, const Element& e, Fmt fmt, Mesh& m,
                       const VertexMap* vm) {
    size_t stride = 0;
    std::vector<size_t> offs(e.props.size());
    for (size_t i = 0; i < e.props.size(); i++) {
        offs[i] = stride;
        stride += type_size(e.props[i].type);
    }
    if (stride == 0) return true;  // records without properties occupy no bytes
    if (e.count && (size_t)(end - p) / stride < e.count) return false;
    if (vm) {
        const unsigned char* base = p;
        const bool swap = fmt == Fmt::BE;
        const int used[9] = {vm->ix, vm->iy, vm->iz, vm->inx, vm->iny, vm->inz, vm->ir, vm->ig, vm->ib};
        bool direct = !swap;  // little-endian float positions and normals: plain 4-byte copies
        for (int j = 0; j < 6; j++)
            if (used[j] >= 0 && e.props[used[j]].type != T::F32) direct = false;
        parallel_ranges(e.count, [&](size_t b, size_t en) {
            std::vector<double> vals(e.props.size());
            for (size_t r = b; r < en; r++) {
                const unsigned char* rec = base + r * stride;
                if (direct) {
                    for (int j = 0; j < 3; j++) std::memcpy(&m.xyz[3 * r + j], rec + offs[used[j]], 4);
                    if (vm->normals)
                        for (int j = 0; j < 3; j++) std::memcpy(&m.normals[3 * r + j], rec + offs[used[3 + j]], 4);
                    if (vm->rgb)
                        for (int j = 0; j < 3; j++)
                            m.rgb[3 * r + j] = (uint8_t)load(rec + offs[used[6 + j]], e.props[used[6 + j]].type, false);
                    continue;
                }
                for (int k : used)
                    if (k >= 0) vals[k] = load(rec + offs[k], e.props[k].type, swap);
                store_vertex(m, *vm, r, vals.data());
            }
        });
    }
    p += e.count * stride;
    return true;
}

// Binary element whose only property is the face list: when every record
// holds three indices, records are fixed-size and are decoded in parallel.
// Returns false (and leaves p unchanged) when some face is not a triangle or
// the data are short; the caller then reads the element sequentially.
bool read_binary_triangles(const unsigned char*& p, const unsigned char* end, const Element& e, Fmt fmt,
                           Mesh& m) {
    const Prop& lp = e.props[0];
    const size_t cs = type_size(lp.count_type), is = type_size(lp.type), stride = cs + 3 * is;
    if (e.count && (size_t)(end - p) / stride < e.count) return false;
    const unsigned char* base = p;
    const bool swap = fmt == Fmt::BE;
    std::vector<char> bad(worker_count(e.count) + 1, 0);
    std::vector<uint32_t> tris(3 * e.count);
    const unsigned w = worker_count(e.count);
    std::vector<std::thread> pool;
    auto work = [&](unsigned t) {
        const size_t b = e.count * t / w, en = e.count * (t + 1) / w;
        for (size_t r = b; r < en; r++) {
            const unsigned char* rec = base + r * stride;
            if (load(rec, lp.count_type, swap) != 3.0) { bad[t] = 1; return; }
            for (int c = 0; c < 3; c++) tris[3 * r + c] = (uint32_t)(int64_t)load(rec + cs + c * is, lp.type, swap);
        }
    };
    if (w <= 1) work(0);
    else {
        for (unsigned t = 0; t < w; t++) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
    }
    for (char b : bad)
        if (b) return false;
    m.tris.insert(m.tris.end(), tris.begin(), tris.end());
    p += e.count * stride;
    return true;
}

// ASCII element without lists, one record per line (the usual layout):
// lines are located in one pass, then parsed in parallel.  Returns false
// (p unchanged) when some line does not hold exactly one record; the caller
// then reads the element sequentially.
// Start of each of the element's `count` lines (blank lines skipped), and
// the position after the last; false when the data end first.
bool line_starts(const char* s, const char* se, size_t count, std::vector<const char*>& starts) {
    starts.clear();
    starts.reserve(count + 1);
    const char* q = s;
    for (size_t r = 0; r < count; r++) {
        while (q < se && is_space(*q)) q++;  // blank lines and leading spaces
        if (q == se) return false;
        starts.push_back(q);
        const void* nl = std::memchr(q, '\n', (size_t)(se - q));
        q = nl ? static_cast<const char*>(nl) + 1 : se;
    }
    starts.push_back(q);
    return true;
}

// True when only whitespace remains in [c, le).
bool line_done(const char* c, const char* le) {
    while (c < le && is_space(*c)) c++;
    return c == le;
}

bool read_ascii_lines(const unsigned char*& p, const unsigned char* end, const Element& e, Mesh& m,
                      const VertexMap* vm) {
    std::vector<const char*> starts;
    if (!line_starts(reinterpret_cast<const char*>(p), reinterpret_cast<const char*>(end), e.count, starts))
        return false;
    const unsigned w = worker_count(e.count);
    std::vector<char> bad(w + 1, 0);
    auto work = [&](unsigned t) {
        const size_t b = e.count * t / w, en = e.count * (t + 1) / w;
        std::vector<double> vals(e.props.size());
        for (size_t r = b; r < en; r++) {
            const char* c = starts[r];
            const char* le = starts[r + 1];
            for (size_t pi = 0; pi < e.props.size(); pi++) {
                c = parse_number(c, le, vals[pi]);
                if (!c) { bad[t] = 1; return; }
            }
            if (!line_done(c, le)) { bad[t] = 1; return; }  // more than one record on the line
            if (vm) store_vertex(m, *vm, r, vals.data());
        }
    };
    if (w <= 1) work(0);
    else {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < w; t++) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
    }
    for (char b : bad)
        if (b) return false;
    p = reinterpret_cast<const unsigned char*>(starts.back());
    return true;
}

// ASCII face element whose only property is the index list, one face per
// line: parsed in parallel like read_ascii_lines, keeping the first three
// indices of each face (0xffffffff for a face with fewer).  Returns false
// (p and m unchanged) when some line does not hold exactly one face.
bool read_ascii_faces(const unsigned char*& p, const unsigned char* end, const Element& e, Mesh& m) {
    std::vector<const char*> starts;
    if (!line_starts(reinterpret_cast<const char*>(p), reinterpret_cast<const char*>(end), e.count, starts))
        return false;
    std::vector<uint32_t> tris(3 * e.count);
    const unsigned w = worker_count(e.count);
    std::vector<char> bad(w + 1, 0);
    auto work = [&](unsigned t) {
        const size_t b = e.count * t / w, en = e.count * (t + 1) / w;
        for (size_t r = b; r < en; r++) {
            const char* c = starts[r];
            const char* le = starts[r + 1];
            double v = 0;
            c = parse_number(c, le, v);
            if (!c) { bad[t] = 1; return; }
            const size_t cnt = (size_t)v;
            uint32_t idx[3] = {0xffffffffu, 0xffffffffu, 0xffffffffu};
            for (size_t j = 0; j < cnt; j++) {
                c = parse_number(c, le, v);
                if (!c) { bad[t] = 1; return; }
                if (j < 3) idx[j] = (uint32_t)(int64_t)v;
            }
            if (!line_done(c, le)) { bad[t] = 1; return; }
            tris[3 * r] = idx[0]; tris[3 * r + 1] = idx[1]; tris[3 * r + 2] = idx[2];
        }
    };
    if (w <= 1) work(0);
    else {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < w; t++) pool.emplace_back(work, t);
        for (auto& th : pool) th.join();
    }
    for (char b : bad)
        if (b) return false;
    m.tris.insert(m.tris.end(), tris.begin(), tris.end());
    p = reinterpret_cast<const unsigned char*>(starts.back());
    return true;
}

// The file's bytes, mapped read-only (falls back to reading into memory
// where the file cannot be mapped).
struct FileBytes {
    const unsigned char* data = nullptr;
    size_t size = 0;
    void* map = nullptr;
    std::vector<unsigned char> copy;
    FileBytes() = default;
    FileBytes(const FileBytes&) = delete;
    FileBytes& operator=(const FileBytes&) = delete;
    ~FileBytes() {
        if (map) munmap(map, size);
    }
};

bool slurp(const std::string& path, FileBytes& fb, std::string& err) {
    const int fd = ::open(path.c_str(), O_RDONLY);
    if (fd < 0) { err = "cannot open " + path; return false; }
    struct stat st;
    if (fstat(fd, &st) != 0) { ::close(fd); err = "cannot read " + path; return false; }
    fb.size = (size_t)st.st_size;
    if (fb.size == 0) { ::close(fd); fb.data = fb.copy.data(); return true; }
    void* mp = mmap(nullptr, fb.size, PROT_READ, MAP_PRIVATE | MAP_POPULATE, fd, 0);
    if (mp != MAP_FAILED) {
        fb.map = mp;
        fb.data = static_cast<const unsigned char*>(mp);
        ::close(fd);
        return true;
    }
    fb.copy.resize(fb.size);
    size_t got = 0;
    while (got < fb.size) {
        const ssize_t r = ::read(fd, fb.copy.data() + got, fb.size - got);
        if (r <= 0) break;
        got += (size_t)r;
    }
    ::close(fd);
    if (got != fb.size) { err = "cannot read " + path; return false; }
    fb.data = fb.copy.data();
    return true;
}

}  // namespace

bool read(const std::string& path, Mesh& m, std::string& err) {
    FileBytes buf;
    if (!slurp(path, buf, err)) return false;
    const unsigned char* p = buf.data;
    const unsigned char* end = p + buf.size;
    auto next_line = [&](std::string& line) {
        if (p >= end) return false;
        const void* nl = std::memchr(p, '\n', (size_t)(end - p));
        const unsigned char* le = nl ? static_cast<const unsigned char*>(nl) : end;
        line.assign(reinterpret_cast<const char*>(p), (size_t)(le - p));
        p = nl ? le + 1 : end;
        if (!line.empty() && line.back() == '\r') line.pop_back();
        return true;
    };
    std::string line;
    if (!next_line(line) || line.rfind("ply", 0) != 0) { err = "not a PLY file"; return false; }
    Fmt fmt = Fmt::Ascii;
    std::vector<Element> elems;
    bool header_done = false;
    while (next_line(line)) {
        char w[64] = {0}, a[64] = {0}, b[64] = {0}, c[256] = {0};
        const int nf = std::sscanf(line.c_str(), "%63s %63s %63s %255s", w, a, b, c);
        if (nf < 1) continue;
        const std::string word = w;
        if (word == "format") {
            const std::string fm = a;
            if (fm == "ascii") fmt = Fmt::Ascii;
            else if (fm == "binary_little_endian") fmt = Fmt::LE;
            else if (fm == "binary_big_endian") fmt = Fmt::BE;
            else { err = "unknown format " + fm; return false; }
        } else if (word == "element") {
            Element e;
            e.name = a;
            e.count = nf >= 3 ? (size_t)std::strtoull(b, nullptr, 10) : 0;
            elems.push_back(e);
        } else if (word == "property") {
            if (elems.empty()) { err = "property before element"; return false; }
            Prop pr;
            const std::string t = a;
            if (t == "list") {
                char ct[64] = {0}, it[64] = {0}, nm[256] = {0};
                std::sscanf(line.c_str(), "%*s %*s %63s %63s %255s", ct, it, nm);
                pr.list = true;
                pr.count_type = parse_type(ct);
                pr.type = parse_type(it);
                pr.name = nm;
            } else {
                pr.type = parse_type(t);
                pr.name = b;
            }
            if (pr.type == T::None || (pr.list && pr.count_type == T::None)) { err = "bad property type"; return false; }
            elems.back().props.push_back(pr);
        } else if (word == "end_header") {
            header_done = true;
            break;
        }
    }
    if (!header_done) { err = "PLY header without end_header"; return false; }
    m = Mesh();
    for (const Element& e : elems) {
        const bool vert = e.name == "vertex", face = e.name == "face";
        VertexMap vm;
        int il = -1;
        if (vert) {
            vm.ix = find(e, {"x"}); vm.iy = find(e, {"y"}); vm.iz = find(e, {"z"});
            if (vm.ix < 0 || vm.iy < 0 || vm.iz < 0) { err = "vertex element without x,y,z"; return false; }
            vm.inx = find(e, {"nx"}); vm.iny = find(e, {"ny"}); vm.inz = find(e, {"nz"});
            vm.ir = find(e, {"red", "r"}); vm.ig = find(e, {"green", "g"}); vm.ib = find(e, {"blue", "b"});
            vm.normals = vm.inx >= 0 && vm.iny >= 0 && vm.inz >= 0;
            vm.rgb = vm.ir >= 0 && vm.ig >= 0 && vm.ib >= 0;
            if (!vm.normals) vm.inx = vm.iny = vm.inz = -1;
            if (!vm.rgb) vm.ir = vm.ig = vm.ib = -1;
            m.xyz.resize(3 * e.count);
            if (vm.normals) m.normals.resize(3 * e.count);
            if (vm.rgb) m.rgb.resize(3 * e.count);
        }
        if (face) il = find(e, {"vertex_indices", "vertex_index"});
        const bool has_list = std::any_of(e.props.begin(), e.props.end(), [](const Prop& x) { return x.list; });
        const VertexMap* vmp = vert ? &vm : nullptr;
        bool done = false;
        if (fmt != Fmt::Ascii && !has_list) {
            if (!read_binary_fixed(p, end, e, fmt, m, vmp)) { err = "truncated " + e.name + " data"; return false; }
            done = true;
        } else if (fmt != Fmt::Ascii && face && il == 0 && e.props.size() == 1) {
            done = read_binary_triangles(p, end, e, fmt, m);
        } else if (fmt == Fmt::Ascii && !has_list && !e.props.empty()) {
            done = read_ascii_lines(p, end, e, m, vmp);
        } else if (fmt == Fmt::Ascii && face && il == 0 && e.props.size() == 1) {
            done = read_ascii_faces(p, end, e, m);
        }
        if (!done) {
            Cursor cur{p, end, fmt};
            if (!read_sequential(cur, e, m, vmp, face ? il : -1, 0)) { err = "truncated " + e.name + " data"; return false; }
            p = cur.p;
        }
    }
    return true;
}

bool write(const std::string& path, const Mesh& m, std::string& err) {
    const size_t nv = m.nV(), nf = m.nF();
    const bool hasN = m.normals.size() == 3 * nv && nv > 0;
    const bool hasC = m.rgb.size() == 3 * nv && nv > 0;
    std::string hdr = "ply\nformat binary_little_endian 1.0\nelement vertex " + std::to_string(nv) + "\n";
    hdr += "property float x\nproperty float y\nproperty float z\n";
    if (hasN) hdr += "property float nx\nproperty float ny\nproperty float nz\n";
    if (hasC) hdr += "property uchar red\nproperty uchar green\nproperty uchar blue\n";
    if (nf) hdr += "element face " + std::to_string(nf) + "\nproperty list uchar uint vertex_indices\n";
    hdr += "end_header\n";
    const size_t vrec = 12 + (hasN ? 12 : 0) + (hasC ? 3 : 0), frec = 13;
    const size_t total = hdr.size() + nv * vrec + nf * frec;
    auto fill = [&](unsigned char* out) {
        std::memcpy(out, hdr.data(), hdr.size());
        unsigned char* vbase = out + hdr.size();
        parallel_ranges(nv, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; i++) {
                unsigned char* r = vbase + i * vrec;
                std::memcpy(r, &m.xyz[3 * i], 12);
                if (hasN) std::memcpy(r + 12, &m.normals[3 * i], 12);
                if (hasC) std::memcpy(r + (hasN ? 24 : 12), &m.rgb[3 * i], 3);
            }
        });
        unsigned char* fbase = vbase + nv * vrec;
        parallel_ranges(nf, [&](size_t b, size_t e) {
            for (size_t i = b; i < e; i++) {
                unsigned char* r = fbase + i * frec;
                r[0] = 3;
                std::memcpy(r + 1, &m.tris[3 * i], 12);
            }
        });
    };
    // the whole file is laid out in memory in parallel, then written at once
    const int fd = ::open(path.c_str(), O_WRONLY | O_CREAT | O_TRUNC, 0644);
    if (fd < 0) { err = "cannot write " + path; return false; }
    std::unique_ptr<unsigned char[]> out(new unsigned char[total]);
    fill(out.get());
    size_t put = 0;
    while (put < total) {
        const ssize_t r = ::pwrite(fd, out.get() + put, total - put, (off_t)put);
        if (r <= 0) break;
        put += (size_t)r;
    }
    if (::close(fd) != 0 || put != total) { err = "write failed"; return false; }
    return true;
}

}  // namespace ply
