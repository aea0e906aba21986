// Exodus II mesh files (the reference's "Input Mesh", read there through Omega_h /
// SEACAS; src/EngineMesh.cpp, src/OmegaHMesh.cpp) in the netCDF classic encodings: CDF-1
// (32-bit offsets), CDF-2 (64-bit offsets) and CDF-5 (64-bit data).  netCDF-4 files are HDF5
// containers and are refused.  What is read: coordinates (coordx/coordy/coordz or coord),
// every element block's connectivity (connect<k>, 1-based, 4-node tetrahedra), node sets
// (node_ns<k>, names from ns_names, else "nodelist_<id>" from ns_prop1) and side sets
// (elem_ss<k>, side_ss<k>, names from ss_names, else "sideset_<id>").  Exodus numbers the
// sides of a tetrahedron 1: (1,2,4), 2: (2,3,4), 3: (1,4,3), 4: (1,3,2) in local node order.
#include <cstdint>
#include <cstring>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "deck.hpp"
#include "plato_b200.h"

namespace {

using plato::deck::DeckError;

enum NcType { NC_BYTE = 1, NC_CHAR = 2, NC_SHORT = 3, NC_INT = 4, NC_FLOAT = 5, NC_DOUBLE = 6, NC_UBYTE = 7,
              NC_USHORT = 8, NC_UINT = 9, NC_INT64 = 10, NC_UINT64 = 11 };

int type_size(int t) {
    switch (t) {
        case NC_BYTE: case NC_CHAR: case NC_UBYTE: return 1;
        case NC_SHORT: case NC_USHORT: return 2;
        case NC_INT: case NC_FLOAT: case NC_UINT: return 4;
        case NC_DOUBLE: case NC_INT64: case NC_UINT64: return 8;
        default: throw DeckError("netCDF: unknown data type " + std::to_string(t));
    }
}

struct NcVar {
    std::vector<int64_t> dims;
    int type = 0;
    uint64_t begin = 0;
    bool record = false;
    std::map<std::string, std::string> text_attrs;
};

class NcFile {
public:
    explicit NcFile(const std::string& path) : buf_(plato::deck::read_file(path)) {
        if (buf_.size() >= 8 && std::memcmp(buf_.data(), "\x89HDF", 4) == 0)
            throw DeckError("'" + path + "' is a netCDF-4 (HDF5) file; write it in a classic netCDF format");
        if (buf_.size() < 4 || std::memcmp(buf_.data(), "CDF", 3) != 0)
            throw DeckError("'" + path + "' is not a netCDF classic file");
        version_ = buf_[3];
        if (version_ != 1 && version_ != 2 && version_ != 5) throw DeckError("netCDF: unsupported version");
        p_ = 4;
        numrecs_ = version_ == 5 ? u64() : u32();
        // dimensions
        uint32_t tag = u32();
        uint64_t n = count();
        if (tag != 0x0A && !(tag == 0 && n == 0)) throw DeckError("netCDF: malformed dimension list");
        for (uint64_t i = 0; i < n; ++i) {
            const std::string name = str();
            const uint64_t len = count();
            dim_names_.push_back(name);
            dim_len_.push_back(len);
            if (len == 0) record_dim_ = int64_t(i);
        }
        skip_attrs(nullptr);
        tag = u32();
        n = count();
        if (tag != 0x0B && !(tag == 0 && n == 0)) throw DeckError("netCDF: malformed variable list");
        for (uint64_t i = 0; i < n; ++i) {
            const std::string name = str();
            NcVar v;
            const uint64_t nd = count();
            for (uint64_t k = 0; k < nd; ++k) {
                const uint64_t id = count();
                if (id >= dim_len_.size()) throw DeckError("netCDF: bad dimension id");
                v.dims.push_back(int64_t(id));
            }
            skip_attrs(&v.text_attrs);
            v.type = int(u32());
            (void)(version_ == 5 ? u64() : u32());  // vsize
            v.begin = version_ == 1 ? u32() : u64();
            v.record = !v.dims.empty() && v.dims[0] == record_dim_;
            vars_[name] = v;
        }
    }

    bool has(const std::string& v) const { return vars_.count(v) != 0; }
    bool has_dim(const std::string& d) const {
        for (const auto& s : dim_names_)
            if (s == d) return true;
        return false;
    }
    uint64_t dim(const std::string& d) const {
        for (size_t i = 0; i < dim_names_.size(); ++i)
            if (dim_names_[i] == d) return dim_len_[i];
        throw DeckError("Exodus: dimension '" + d + "' missing");
    }
    const NcVar& var(const std::string& name) const {
        auto it = vars_.find(name);
        if (it == vars_.end()) throw DeckError("Exodus: variable '" + name + "' missing");
        return it->second;
    }
    // element count of a variable; no variable holds more elements than the file has bytes,
    // so a product beyond that is a corrupt header (and is stopped before it can overflow)
    uint64_t size(const NcVar& v) const {
        uint64_t n = 1;
        for (int64_t d : v.dims) {
            const uint64_t len = dim_len_[size_t(d)];
            if (len != 0 && n > buf_.size() / len) throw DeckError("netCDF: variable larger than the file");
            n *= len;
        }
        return n;
    }
    // a fixed-size variable as doubles / int64 (any numeric type)
    std::vector<double> doubles(const std::string& name) const {
        const NcVar& v = var(name);
        check_range(v, size(v));  // before the allocation: the size comes from the file
        std::vector<double> out(size(v));
        for (size_t i = 0; i < out.size(); ++i) out[i] = value(v, i);
        return out;
    }
    std::vector<int64_t> ints(const std::string& name) const {
        const NcVar& v = var(name);
        check_range(v, size(v));
        std::vector<int64_t> out(size(v));
        for (size_t i = 0; i < out.size(); ++i) out[i] = int64_t(value(v, i));
        return out;
    }
    // rows of a [n][len] char variable as trimmed strings
    std::vector<std::string> strings(const std::string& name) const {
        const NcVar& v = var(name);
        if (v.type != NC_CHAR || v.dims.size() != 2) throw DeckError("Exodus: '" + name + "' is not a name table");
        const uint64_t rows = dim_len_[size_t(v.dims[0])], len = dim_len_[size_t(v.dims[1])];
        check_range(v, size(v));
        std::vector<std::string> out;
        for (uint64_t r = 0; r < rows; ++r) {
            const char* s = buf_.data() + v.begin + r * len;
            size_t k = 0;
            while (k < len && s[k] != '\0') ++k;
            std::string t(s, k);
            while (!t.empty() && t.back() == ' ') t.pop_back();
            out.push_back(t);
        }
        return out;
    }

private:
    void need(uint64_t n) const {
        if (p_ > buf_.size() || n > buf_.size() - p_) throw DeckError("netCDF: header runs past the end of the file");
    }
    uint32_t u32() {
        need(4);
        const auto* b = reinterpret_cast<const unsigned char*>(buf_.data() + p_);
        p_ += 4;
        return (uint32_t(b[0]) << 24) | (uint32_t(b[1]) << 16) | (uint32_t(b[2]) << 8) | uint32_t(b[3]);
    }
    uint64_t u64() {
        const uint64_t hi = u32();
        return (hi << 32) | u32();
    }
    uint64_t count() { return version_ == 5 ? u64() : u32(); }
    std::string str() {
        const uint64_t n = count();
        need(n);
        std::string s = buf_.substr(p_, n);
        p_ += (n + 3) & ~uint64_t(3);
        return s;
    }
    void skip_attrs(std::map<std::string, std::string>* text) {
        const uint32_t tag = u32();
        const uint64_t n = count();
        if (tag != 0x0C && !(tag == 0 && n == 0)) throw DeckError("netCDF: malformed attribute list");
        for (uint64_t i = 0; i < n; ++i) {
            const std::string name = str();
            const int t = int(u32());
            const uint64_t m = count();
            if (m > buf_.size()) throw DeckError("netCDF: header runs past the end of the file");
            const uint64_t bytes = m * uint64_t(type_size(t));  // at most 8 x the file size: no overflow
            need(bytes);
            if (text && t == NC_CHAR) (*text)[name] = buf_.substr(p_, m);
            p_ += (bytes + 3) & ~uint64_t(3);
        }
    }
    void check_range(const NcVar& v, uint64_t n) const {
        if (v.record) throw DeckError("Exodus: record variables are not read");
        const uint64_t ts = uint64_t(type_size(v.type));
        if (v.begin > buf_.size() || n > (buf_.size() - v.begin) / ts)
            throw DeckError("netCDF: variable past the end of the file");
    }
    double value(const NcVar& v, uint64_t i) const {
        if (i == 0) check_range(v, size(v));
        const auto* b = reinterpret_cast<const unsigned char*>(buf_.data() + v.begin) + i * uint64_t(type_size(v.type));
        auto be = [&](int n) {
            uint64_t x = 0;
            for (int k = 0; k < n; ++k) x = (x << 8) | b[k];
            return x;
        };
        switch (v.type) {
            case NC_BYTE: return double(int8_t(b[0]));
            case NC_UBYTE: return double(b[0]);
            case NC_SHORT: return double(int16_t(be(2)));
            case NC_USHORT: return double(uint16_t(be(2)));
            case NC_INT: return double(int32_t(be(4)));
            case NC_UINT: return double(uint32_t(be(4)));
            case NC_INT64: return double(int64_t(be(8)));
            case NC_UINT64: return double(be(8));
            case NC_FLOAT: { const uint32_t x = uint32_t(be(4)); float f; std::memcpy(&f, &x, 4); return double(f); }
            case NC_DOUBLE: { const uint64_t x = be(8); double d; std::memcpy(&d, &x, 8); return d; }
            default: throw DeckError("netCDF: variable is not numeric");
        }
    }

    std::string buf_;
    uint64_t p_ = 0;
    int version_ = 0;
    uint64_t numrecs_ = 0;
    int64_t record_dim_ = -1;
    std::vector<std::string> dim_names_;
    std::vector<uint64_t> dim_len_;
    std::map<std::string, NcVar> vars_;
};

const int32_t kTetSide[4][3] = {{0, 1, 3}, {1, 2, 3}, {0, 3, 2}, {0, 2, 1}};

}  // namespace

struct plato_mesh_file {
    std::vector<double> coords;  // node-major
    std::vector<int32_t> conn;
    std::vector<std::string> ns_names, ss_names;
    std::vector<std::vector<int32_t>> node_sets;
    std::vector<std::vector<int32_t>> ss_cells, ss_local;
    std::string error;
};

namespace {

void load(plato_mesh_file& m, const std::string& path) {
    NcFile f(path);
    const uint64_t nn = f.dim("num_nodes");
    const uint64_t ndim = f.dim("num_dim");
    if (ndim != 3) throw DeckError("Exodus: only 3D meshes are read");
    if (nn > uint64_t(INT32_MAX)) throw DeckError("Exodus: too many nodes");
    m.coords.assign(3 * nn, 0.0);
    if (f.has("coordx")) {
        const char* names[3] = {"coordx", "coordy", "coordz"};
        for (int d = 0; d < 3; ++d) {
            const auto c = f.doubles(names[d]);
            if (c.size() != nn) throw DeckError("Exodus: coordinate length");
            for (uint64_t i = 0; i < nn; ++i) m.coords[3 * i + d] = c[i];
        }
    } else {
        const auto c = f.doubles("coord");  // [num_dim][num_nodes]
        if (c.size() != 3 * nn) throw DeckError("Exodus: coordinate length");
        for (uint64_t i = 0; i < nn; ++i)
            for (int d = 0; d < 3; ++d) m.coords[3 * i + d] = c[d * nn + i];
    }
    const uint64_t nblk = f.dim("num_el_blk");
    for (uint64_t b = 1; b <= nblk; ++b) {
        const std::string cv = "connect" + std::to_string(b);
        const NcVar& v = f.var(cv);
        auto it = v.text_attrs.find("elem_type");
        std::string type = it == v.text_attrs.end() ? std::string() : it->second;
        type = type.substr(0, type.find('\0'));
        for (char& ch : type) ch = char(std::toupper(static_cast<unsigned char>(ch)));
        const uint64_t npe = f.dim("num_nod_per_el" + std::to_string(b));
        if (npe != 4 || (type.rfind("TET", 0) != 0 && !type.empty()))
            throw DeckError("Exodus: element block " + std::to_string(b) + " is '" + type +
                            "'; only 4-node tetrahedra are built");
        const auto c = f.ints(cv);
        for (int64_t id : c) {
            if (id < 1 || uint64_t(id) > nn) throw DeckError("Exodus: connectivity out of range");
            m.conn.push_back(int32_t(id - 1));
        }
    }
    const uint64_t nc = m.conn.size() / 4;
    if (f.has_dim("num_node_sets")) {
        const uint64_t ns = f.dim("num_node_sets");
        std::vector<std::string> names = f.has("ns_names") ? f.strings("ns_names") : std::vector<std::string>();
        std::vector<int64_t> ids = f.has("ns_prop1") ? f.ints("ns_prop1") : std::vector<int64_t>();
        for (uint64_t k = 0; k < ns; ++k) {
            std::string name = k < names.size() ? names[k] : std::string();
            if (name.empty()) name = "nodelist_" + std::to_string(k < ids.size() ? ids[k] : int64_t(k + 1));
            std::vector<int32_t> nodes;
            for (int64_t id : f.ints("node_ns" + std::to_string(k + 1))) {
                if (id < 1 || uint64_t(id) > nn) throw DeckError("Exodus: node set entry out of range");
                nodes.push_back(int32_t(id - 1));
            }
            m.ns_names.push_back(name);
            m.node_sets.push_back(std::move(nodes));
        }
    }
    if (f.has_dim("num_side_sets")) {
        const uint64_t ss = f.dim("num_side_sets");
        std::vector<std::string> names = f.has("ss_names") ? f.strings("ss_names") : std::vector<std::string>();
        std::vector<int64_t> ids = f.has("ss_prop1") ? f.ints("ss_prop1") : std::vector<int64_t>();
        for (uint64_t k = 0; k < ss; ++k) {
            std::string name = k < names.size() ? names[k] : std::string();
            if (name.empty()) name = "sideset_" + std::to_string(k < ids.size() ? ids[k] : int64_t(k + 1));
            const auto el = f.ints("elem_ss" + std::to_string(k + 1));
            const auto sd = f.ints("side_ss" + std::to_string(k + 1));
            if (el.size() != sd.size()) throw DeckError("Exodus: side set lengths differ");
            std::vector<int32_t> cells, local;
            for (size_t i = 0; i < el.size(); ++i) {
                if (el[i] < 1 || uint64_t(el[i]) > nc) throw DeckError("Exodus: side set element out of range");
                if (sd[i] < 1 || sd[i] > 4) throw DeckError("Exodus: tetrahedron side number out of range");
                cells.push_back(int32_t(el[i] - 1));
                for (int a = 0; a < 3; ++a) local.push_back(kTetSide[sd[i] - 1][a]);
            }
            m.ss_names.push_back(name);
            m.ss_cells.push_back(std::move(cells));
            m.ss_local.push_back(std::move(local));
        }
    }
}

thread_local std::string g_open_error;

void copy_name(const std::string& s, char* buf, int64_t cap) {
    if (!buf || cap <= 0) return;
    const size_t n = std::min<size_t>(s.size(), size_t(cap - 1));
    std::memcpy(buf, s.data(), n);
    buf[n] = '\0';
}

}  // namespace

extern "C" {

int plato_mesh_file_open(const char* path, plato_mesh_file** out) {
    if (!out) return PLATO_BAD_INPUT;
    *out = nullptr;
    if (!path) {
        g_open_error = "null path";
        return PLATO_BAD_INPUT;
    }
    auto m = std::make_unique<plato_mesh_file>();
    try {
        load(*m, path);
    } catch (const std::bad_alloc&) {
        g_open_error = "host allocation failed";
        return PLATO_OUT_OF_MEMORY;
    } catch (const std::exception& e) {
        g_open_error = e.what();
        return PLATO_BAD_INPUT;
    }
    *out = m.release();
    return PLATO_OK;
}

const char* plato_mesh_file_last_error(void) { return g_open_error.c_str(); }

int plato_mesh_file_close(plato_mesh_file* m) {
    delete m;
    return PLATO_OK;
}

int plato_mesh_file_info(const plato_mesh_file* m, int32_t* num_nodes, int32_t* num_cells, int32_t* num_node_sets,
                         int32_t* num_side_sets) {
    if (!m) return PLATO_BAD_INPUT;
    if (num_nodes) *num_nodes = int32_t(m->coords.size() / 3);
    if (num_cells) *num_cells = int32_t(m->conn.size() / 4);
    if (num_node_sets) *num_node_sets = int32_t(m->node_sets.size());
    if (num_side_sets) *num_side_sets = int32_t(m->ss_cells.size());
    return PLATO_OK;
}

int plato_mesh_file_mesh(const plato_mesh_file* m, double* coords, int32_t* connectivity) {
    if (!m) return PLATO_BAD_INPUT;
    if (coords) std::memcpy(coords, m->coords.data(), m->coords.size() * sizeof(double));
    if (connectivity) std::memcpy(connectivity, m->conn.data(), m->conn.size() * sizeof(int32_t));
    return PLATO_OK;
}

int plato_mesh_file_node_set(const plato_mesh_file* m, int32_t index, char* name, int64_t name_capacity,
                             int32_t* nodes, int32_t* count) {
    if (!m || !count || index < 0 || size_t(index) >= m->node_sets.size()) return PLATO_BAD_INPUT;
    copy_name(m->ns_names[size_t(index)], name, name_capacity);
    const auto& v = m->node_sets[size_t(index)];
    *count = int32_t(v.size());
    if (nodes) std::memcpy(nodes, v.data(), v.size() * sizeof(int32_t));
    return PLATO_OK;
}

int plato_mesh_file_side_set(const plato_mesh_file* m, int32_t index, char* name, int64_t name_capacity,
                             int32_t* cells, int32_t* local_nodes, int32_t* count) {
    if (!m || !count || index < 0 || size_t(index) >= m->ss_cells.size()) return PLATO_BAD_INPUT;
    copy_name(m->ss_names[size_t(index)], name, name_capacity);
    const auto& c = m->ss_cells[size_t(index)];
    const auto& l = m->ss_local[size_t(index)];
    *count = int32_t(c.size());
    if (cells) std::memcpy(cells, c.data(), c.size() * sizeof(int32_t));
    if (local_nodes) std::memcpy(local_nodes, l.data(), l.size() * sizeof(int32_t));
    return PLATO_OK;
}

}  // extern "C"
