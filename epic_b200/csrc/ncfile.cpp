// netCDF classic-format (CDF-1 / CDF-2 / CDF-5) reader and writer for the
// reference's parcel and field files.  Written from the published format
// description: a big-endian header (magic "CDF" + version, number of
// records, dimension list, global attributes, variables with their
// attributes, type, size and file offset), then the data of the fixed-size
// variables one after the other and the records, each record holding one
// slab of every record variable.  CDF-5 widens every count, length and size
// field to 64 bits; CDF-2 widens only the offsets.
#include "ncfile.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <memory>

namespace ncio {
namespace {

enum : int32_t { T_BYTE = 1, T_CHAR = 2, T_SHORT = 3, T_INT = 4, T_FLOAT = 5, T_DOUBLE = 6,
                 T_UBYTE = 7, T_USHORT = 8, T_UINT = 9, T_INT64 = 10, T_UINT64 = 11 };
enum : uint32_t { TAG_DIM = 10, TAG_VAR = 11, TAG_ATT = 12 };
constexpr int64_t CDF2_MAX_VSIZE = 4294967292LL;   // 2^32 - 4

int type_size(int32_t t) {
    switch (t) {
        case T_BYTE: case T_CHAR: case T_UBYTE: return 1;
        case T_SHORT: case T_USHORT: return 2;
        case T_INT: case T_FLOAT: case T_UINT: return 4;
        case T_DOUBLE: case T_INT64: case T_UINT64: return 8;
    }
    throw Error("netCDF: unknown type " + std::to_string(t));
}

int64_t round4(int64_t v) { return (v + 3) & ~int64_t(3); }

struct Att {
    std::string name;
    int32_t type = T_CHAR;
    int64_t nelems = 0;
    std::vector<uint8_t> raw;   // values in file byte order, unpadded
};
struct Dim {
    std::string name;
    int64_t len;   // 0: the record dimension
};
// Fills buf[0 .. count) with elements [start, start + count) of a variable
// (of one record), in the variable's C order.
using Source = std::function<void(int64_t start, int64_t count, double* buf)>;
struct Var {
    std::string name;
    std::vector<int64_t> dims;
    std::vector<Att> atts;
    int32_t type = T_DOUBLE;
    int64_t vsize = 0, begin = 0;
    Source src;   // writer only
};
struct Header {
    int version = 2;
    int64_t numrecs = 0;
    std::vector<Dim> dims;
    std::vector<Att> gatts;
    std::vector<Var> vars;
    int64_t recsize = 0;
    int rec_dim = -1;
};

void put_be(uint8_t* p, uint64_t v, int bytes) {
    for (int k = bytes - 1; k >= 0; --k) { p[k] = uint8_t(v & 0xff); v >>= 8; }
}
uint64_t get_be(const uint8_t* p, int bytes) {
    uint64_t v = 0;
    for (int k = 0; k < bytes; ++k) v = (v << 8) | p[k];
    return v;
}

Att att_text(const std::string& name, const std::string& s) {
    Att a;
    a.name = name;
    a.type = T_CHAR;
    a.nelems = (int64_t)s.size();
    a.raw.assign(s.begin(), s.end());
    return a;
}
Att att_ints(const std::string& name, const int32_t* v, int n) {
    Att a;
    a.name = name;
    a.type = T_INT;
    a.nelems = n;
    a.raw.resize(4 * n);
    for (int k = 0; k < n; ++k) put_be(&a.raw[4 * k], (uint32_t)v[k], 4);
    return a;
}
Att att_doubles(const std::string& name, const double* v, int n) {
    Att a;
    a.name = name;
    a.type = T_DOUBLE;
    a.nelems = n;
    a.raw.resize(8 * n);
    for (int k = 0; k < n; ++k) {
        uint64_t u;
        std::memcpy(&u, &v[k], 8);
        put_be(&a.raw[8 * k], u, 8);
    }
    return a;
}

// Element k of an attribute as a double (numeric types).
double att_value(const Att& a, int64_t k) {
    const int s = type_size(a.type);
    if (k >= a.nelems) throw Error("netCDF: attribute " + a.name + " too short");
    const uint8_t* p = &a.raw[s * k];
    const uint64_t u = get_be(p, s);
    switch (a.type) {
        case T_BYTE: return (double)(int8_t)u;
        case T_UBYTE: return (double)(uint8_t)u;
        case T_SHORT: return (double)(int16_t)u;
        case T_USHORT: return (double)(uint16_t)u;
        case T_INT: return (double)(int32_t)u;
        case T_UINT: return (double)(uint32_t)u;
        case T_INT64: return (double)(int64_t)u;
        case T_UINT64: return (double)u;
        case T_FLOAT: { uint32_t w = (uint32_t)u; float f; std::memcpy(&f, &w, 4); return f; }
        case T_DOUBLE: { double d; std::memcpy(&d, &u, 8); return d; }
    }
    throw Error("netCDF: attribute " + a.name + " is not numeric");
}

// ---- header serialisation -------------------------------------------------
struct Out {
    std::vector<uint8_t> b;
    int ver;
    void u32(uint64_t v) { size_t i = b.size(); b.resize(i + 4); put_be(&b[i], v, 4); }
    void u64(uint64_t v) { size_t i = b.size(); b.resize(i + 8); put_be(&b[i], v, 8); }
    void nonneg(int64_t v) {
        if (ver == 5) { u64((uint64_t)v); return; }
        if (v < 0 || v > 0x7fffffffLL) throw Error("netCDF: count too large for CDF-2");
        u32((uint64_t)v);
    }
    void offset(int64_t v) { if (ver == 1) u32((uint64_t)v); else u64((uint64_t)v); }
    void pad4() { while (b.size() % 4) b.push_back(0); }
    void name(const std::string& s) { nonneg((int64_t)s.size()); b.insert(b.end(), s.begin(), s.end()); pad4(); }
    void atts(const std::vector<Att>& a) {
        if (a.empty()) { u32(0); nonneg(0); return; }
        u32(TAG_ATT);
        nonneg((int64_t)a.size());
        for (const Att& x : a) {
            name(x.name);
            u32((uint32_t)x.type);
            nonneg(x.nelems);
            b.insert(b.end(), x.raw.begin(), x.raw.end());
            pad4();
        }
    }
};

std::vector<uint8_t> serialise(const Header& h) {
    Out o{{}, h.version};
    o.b = {'C', 'D', 'F', (uint8_t)h.version};
    o.nonneg(h.numrecs);
    if (h.dims.empty()) { o.u32(0); o.nonneg(0); }
    else {
        o.u32(TAG_DIM);
        o.nonneg((int64_t)h.dims.size());
        for (const Dim& d : h.dims) { o.name(d.name); o.nonneg(d.len); }
    }
    o.atts(h.gatts);
    if (h.vars.empty()) { o.u32(0); o.nonneg(0); }
    else {
        o.u32(TAG_VAR);
        o.nonneg((int64_t)h.vars.size());
        for (const Var& v : h.vars) {
            o.name(v.name);
            o.nonneg((int64_t)v.dims.size());
            for (int64_t d : v.dims) o.nonneg(d);
            o.atts(v.atts);
            o.u32((uint32_t)v.type);
            if (h.version == 5) o.u64((uint64_t)v.vsize);
            else o.u32((uint64_t)std::min<int64_t>(v.vsize, 0xffffffffLL));
            o.offset(v.begin);
        }
    }
    return o.b;
}

bool is_record(const Header& h, const Var& v) { return !v.dims.empty() && v.dims[0] == h.rec_dim; }

// Elements of one record of v (of the whole variable if fixed-size); a
// product beyond 2^56 elements (a corrupt header) is an error.
int64_t slab_elems(const Header& h, const Var& v) {
    int64_t n = 1;
    for (size_t k = is_record(h, v) ? 1 : 0; k < v.dims.size(); ++k) {
        const int64_t len = h.dims[v.dims[k]].len;
        if (len < 0 || (len > 0 && n > (int64_t(1) << 56) / len)) throw Error("netCDF: variable too large");
        n *= len;
    }
    return n;
}

// vsize, begin and the record size; the version is raised to 5 when a
// variable does not fit the 32-bit sizes of CDF-2.
void layout(Header& h, int force_version) {
    h.rec_dim = -1;
    for (size_t k = 0; k < h.dims.size(); ++k)
        if (h.dims[k].len == 0) h.rec_dim = (int)k;
    bool big = false;
    for (Var& v : h.vars) {
        v.vsize = round4(slab_elems(h, v) * type_size(v.type));
        if (v.vsize > CDF2_MAX_VSIZE) big = true;
    }
    for (const Dim& d : h.dims) if (d.len > 0x7fffffffLL) big = true;
    h.version = force_version ? force_version : (big ? 5 : 2);
    if (h.version != 5 && big) throw Error("netCDF: data too large for CDF-2");
    int64_t off = (int64_t)serialise(h).size();
    for (Var& v : h.vars) if (!is_record(h, v)) { v.begin = off; off += v.vsize; }
    h.recsize = 0;
    int nrec = 0;
    for (Var& v : h.vars) if (is_record(h, v)) { v.begin = off; off += v.vsize; h.recsize += v.vsize; ++nrec; }
    if (nrec == 1)   // a single record variable is not padded
        for (Var& v : h.vars) if (is_record(h, v)) h.recsize = slab_elems(h, v) * type_size(v.type);
}

struct FileCloser { void operator()(FILE* f) const { if (f) std::fclose(f); } };
using FilePtr = std::unique_ptr<FILE, FileCloser>;

void write_file(const std::string& path, Header& h, int force_version) {
    if (!force_version) {
        const char* e = std::getenv("EPIC_NC_VERSION");
        if (e && std::string(e) == "5") force_version = 5;
    }
    layout(h, force_version);
    const std::vector<uint8_t> head = serialise(h);
    FilePtr f(std::fopen(path.c_str(), "wb"));
    if (!f) throw Error("netCDF: cannot create " + path);
    auto put = [&](const void* p, size_t n) {
        if (n && std::fwrite(p, 1, n, f.get()) != n) throw Error("netCDF: write failed: " + path);
    };
    put(head.data(), head.size());
    constexpr int64_t CH = 1 << 20;
    std::vector<double> buf(CH);
    std::vector<uint8_t> be(CH * 8);
    auto write_slab = [&](const Var& v) {
        const int64_t n = slab_elems(h, v);
        const int s = type_size(v.type);
        for (int64_t i = 0; i < n; i += CH) {
            const int64_t m = std::min(CH, n - i);
            v.src(i, m, buf.data());
            for (int64_t k = 0; k < m; ++k) {
                if (v.type == T_DOUBLE) {
                    uint64_t u;
                    std::memcpy(&u, &buf[k], 8);
                    put_be(&be[8 * k], u, 8);
                } else if (v.type == T_INT) {
                    put_be(&be[4 * k], (uint32_t)(int32_t)std::llround(buf[k]), 4);
                } else if (v.type == T_INT64) {
                    put_be(&be[8 * k], (uint64_t)(int64_t)std::llround(buf[k]), 8);
                } else {
                    throw Error("netCDF: the writer supports int and double variables");
                }
            }
            put(be.data(), (size_t)(m * s));
        }
        const int64_t pad = v.vsize - n * s;
        if (pad > 0 && !(is_record(h, v) && h.recsize == n * s)) {
            const uint8_t z[4] = {0, 0, 0, 0};
            put(z, (size_t)pad);
        }
    };
    for (const Var& v : h.vars) if (!is_record(h, v)) write_slab(v);
    for (int64_t r = 0; r < h.numrecs; ++r)
        for (const Var& v : h.vars) if (is_record(h, v)) write_slab(v);
}

// ---- header parsing -------------------------------------------------------
struct In {
    std::vector<uint8_t> b;
    size_t i = 0;
    int ver = 1;
    const uint8_t* take(size_t n) {
        if (i + n > b.size()) throw Error("netCDF: truncated header");
        const uint8_t* p = &b[i];
        i += n;
        return p;
    }
    uint64_t u32() { return get_be(take(4), 4); }
    uint64_t u64() { return get_be(take(8), 8); }
    int64_t nonneg() { return ver == 5 ? (int64_t)u64() : (int64_t)u32(); }
    int64_t offset() { return ver == 1 ? (int64_t)u32() : (int64_t)u64(); }
    std::string name() {
        const int64_t n = nonneg();
        if (n < 0 || n > (1 << 20)) throw Error("netCDF: bad name length");
        const uint8_t* p = take((size_t)round4(n));
        return std::string(reinterpret_cast<const char*>(p), (size_t)n);
    }
    std::vector<Att> atts() {
        std::vector<Att> out;
        const uint32_t tag = (uint32_t)u32();
        const int64_t n = nonneg();
        if (tag == 0 && n == 0) return out;
        if (tag != TAG_ATT) throw Error("netCDF: bad attribute list");
        for (int64_t k = 0; k < n; ++k) {
            Att a;
            a.name = name();
            a.type = (int32_t)u32();
            a.nelems = nonneg();
            const int ts = type_size(a.type);
            if (a.nelems < 0 || a.nelems > (int64_t)(b.size() - i) / ts) throw Error("netCDF: bad attribute length");
            const int64_t bytes = a.nelems * ts;
            const uint8_t* p = take((size_t)round4(bytes));
            a.raw.assign(p, p + bytes);
            out.push_back(std::move(a));
        }
        return out;
    }
};

struct Reader {
    std::string path;
    FilePtr f;
    Header h;
    int64_t file_size = 0;

    explicit Reader(const std::string& p) : path(p), f(std::fopen(p.c_str(), "rb")) {
        if (!f) throw Error("netCDF: cannot open " + p);
        std::fseek(f.get(), 0, SEEK_END);
        file_size = (int64_t)std::ftell(f.get());
        std::fseek(f.get(), 0, SEEK_SET);
        In in;
        in.b.resize((size_t)std::min<int64_t>(file_size, 16 << 20));
        if (!in.b.empty() && std::fread(in.b.data(), 1, in.b.size(), f.get()) != in.b.size())
            throw Error("netCDF: read failed: " + p);
        const uint8_t* m = in.take(4);
        if (m[0] != 'C' || m[1] != 'D' || m[2] != 'F' || (m[3] != 1 && m[3] != 2 && m[3] != 5))
            throw Error("netCDF: " + p + " is not a netCDF classic file (netCDF-4 / HDF5 files are not read)");
        in.ver = h.version = m[3];
        const uint64_t nr = h.version == 5 ? in.u64() : in.u32();
        const bool streaming = h.version == 5 ? nr == ~0ull : nr == 0xffffffffull;
        h.numrecs = streaming ? -1 : (int64_t)nr;
        uint32_t tag = (uint32_t)in.u32();
        int64_t n = in.nonneg();
        if (!(tag == 0 && n == 0)) {
            if (tag != TAG_DIM) throw Error("netCDF: bad dimension list");
            for (int64_t k = 0; k < n; ++k) {
                Dim d;
                d.name = in.name();
                d.len = in.nonneg();
                if (d.len < 0) throw Error("netCDF: bad dimension length");
                h.dims.push_back(d);
            }
        }
        h.gatts = in.atts();
        tag = (uint32_t)in.u32();
        n = in.nonneg();
        if (!(tag == 0 && n == 0)) {
            if (tag != TAG_VAR) throw Error("netCDF: bad variable list");
            for (int64_t k = 0; k < n; ++k) {
                Var v;
                v.name = in.name();
                const int64_t nd = in.nonneg();
                for (int64_t d = 0; d < nd; ++d) {
                    const int64_t id = in.nonneg();
                    if (id < 0 || id >= (int64_t)h.dims.size()) throw Error("netCDF: bad dimension id");
                    v.dims.push_back(id);
                }
                v.atts = in.atts();
                v.type = (int32_t)in.u32();
                v.vsize = h.version == 5 ? (int64_t)in.u64() : (int64_t)in.u32();
                v.begin = in.offset();
                if (v.begin < 0 || v.begin > file_size) throw Error("netCDF: bad variable offset");
                type_size(v.type);   // an unknown type is an error here
                h.vars.push_back(std::move(v));
            }
        }
        h.rec_dim = -1;
        for (size_t k = 0; k < h.dims.size(); ++k)
            if (h.dims[k].len == 0) h.rec_dim = (int)k;
        // record size from the slabs (the vsize of a > 4 GiB CDF-2 variable is clipped)
        h.recsize = 0;
        int nrec = 0;
        int64_t first_rec = -1;
        for (const Var& v : h.vars)
            if (is_record(h, v)) {
                h.recsize += round4(slab_elems(h, v) * type_size(v.type));
                if (h.recsize > (int64_t(1) << 60)) throw Error("netCDF: record too large");
                if (first_rec < 0) first_rec = v.begin;
                ++nrec;
            }
        if (nrec == 1)
            for (const Var& v : h.vars) if (is_record(h, v)) h.recsize = slab_elems(h, v) * type_size(v.type);
        if (h.numrecs < 0) h.numrecs = (h.recsize > 0 && first_rec >= 0) ? (file_size - first_rec) / h.recsize : 0;
    }

    const Var* var(const std::string& name) const {
        for (const Var& v : h.vars) if (v.name == name) return &v;
        return nullptr;
    }
    const Att* gatt(const std::string& name) const {
        for (const Att& a : h.gatts) if (a.name == name) return &a;
        return nullptr;
    }
    int64_t dim_len(const std::string& name) const {
        for (const Dim& d : h.dims) if (d.name == name) return d.len == 0 ? h.numrecs : d.len;
        return -1;
    }

    // Elements [start, start + count) of record r of v (r ignored for a
    // fixed-size variable), converted to double.
    void read(const Var& v, int64_t r, int64_t start, int64_t count, double* out) {
        const int s = type_size(v.type);
        if (v.type == T_CHAR) throw Error("netCDF: " + v.name + " is not numeric");
        if (start < 0 || start + count > slab_elems(h, v)) throw Error("netCDF: read outside " + v.name);
        int64_t off = v.begin + start * s;
        if (is_record(h, v)) {
            if (r < 0 || r >= h.numrecs) throw Error("netCDF: record out of range in " + v.name);
            if (h.recsize > 0 && r > file_size / h.recsize) throw Error("netCDF: " + path + " is truncated");
            off += r * h.recsize;
        }
        if (off + count * s > file_size) throw Error("netCDF: " + path + " is truncated");
        constexpr int64_t CH = 1 << 20;
        std::vector<uint8_t> buf((size_t)(std::min(CH, count) * s));
        for (int64_t i = 0; i < count; i += CH) {
            const int64_t m = std::min(CH, count - i);
            if (std::fseek(f.get(), (long)(off + i * s), SEEK_SET) != 0 ||
                std::fread(buf.data(), 1, (size_t)(m * s), f.get()) != (size_t)(m * s))
                throw Error("netCDF: read failed: " + path);
            for (int64_t k = 0; k < m; ++k) {
                const uint64_t u = get_be(&buf[(size_t)(k * s)], s);
                double d;
                switch (v.type) {
                    case T_DOUBLE: std::memcpy(&d, &u, 8); break;
                    case T_FLOAT: { uint32_t w = (uint32_t)u; float g; std::memcpy(&g, &w, 4); d = g; break; }
                    case T_INT: d = (double)(int32_t)u; break;
                    case T_UINT: d = (double)(uint32_t)u; break;
                    case T_SHORT: d = (double)(int16_t)u; break;
                    case T_USHORT: d = (double)(uint16_t)u; break;
                    case T_BYTE: d = (double)(int8_t)u; break;
                    case T_UBYTE: d = (double)(uint8_t)u; break;
                    case T_INT64: d = (double)(int64_t)u; break;
                    default: d = (double)u; break;
                }
                out[i + k] = d;
            }
        }
    }
};

Box read_box(const Reader& rd) {
    Box b;
    const Att* nc = rd.gatt("ncells");
    const Att* ex = rd.gatt("extent");
    const Att* og = rd.gatt("origin");
    if (!nc || !ex || !og) throw Error("netCDF: " + rd.path + " lacks the ncells / extent / origin attributes");
    for (int k = 0; k < 3; ++k) {
        b.ncells[k] = (int32_t)att_value(*nc, k);
        b.extent[k] = att_value(*ex, k);
        b.origin[k] = att_value(*og, k);
    }
    return b;
}

std::string att_string(const Att& a) {
    if (a.type != T_CHAR) throw Error("netCDF: attribute " + a.name + " is not text");
    std::string s(a.raw.begin(), a.raw.end());
    while (!s.empty() && (s.back() == '\0' || s.back() == ' ')) s.pop_back();
    return s;
}

void global_atts(Header& h, const Box& box, const std::string& type, const int32_t zeta[2]) {
    h.gatts.push_back(att_text("file_type", type));
    h.gatts.push_back(att_text("Conventions", "CF-1.8"));
    h.gatts.push_back(att_ints("ncells", box.ncells, 3));
    h.gatts.push_back(att_doubles("extent", box.extent, 3));
    h.gatts.push_back(att_doubles("origin", box.origin, 3));
    // The reference keeps these two in a netCDF-4 group "parameters"
    // (parameters.f90:220-265); the classic format has no groups, so they are
    // global attributes here (the reference then keeps its defaults).
    h.gatts.push_back(att_text("l_lower_boundry_zeta_zero", zeta && zeta[0] ? "true" : "false"));
    h.gatts.push_back(att_text("l_upper_boundry_zeta_zero", zeta && zeta[1] ? "true" : "false"));
}

Var dataset(const std::string& name, const std::string& long_name, const std::string& std_name,
            const std::string& unit, int32_t type, std::vector<int64_t> dims, Source src) {
    Var v;
    v.name = name;
    v.type = type;
    v.dims = std::move(dims);
    v.atts.push_back(att_text("units", unit));
    if (!long_name.empty()) v.atts.push_back(att_text("long_name", long_name));
    if (!std_name.empty()) v.atts.push_back(att_text("standard_name", std_name));
    v.src = std::move(src);
    return v;
}

// the time axis (netcdf_writer.f90: define_netcdf_temporal_dimension)
Var time_var(int64_t tdim, double t) {
    Var v = dataset("t", "time ", "time", "seconds since 1970-01-01", T_DOUBLE, {tdim},
                    [t](int64_t, int64_t m, double* b) { std::fill(b, b + m, t); });
    v.atts.push_back(att_text("axis", "T"));
    v.atts.push_back(att_text("calendar", "proleptic_gregorian"));
    return v;
}

}  // namespace

void check_box(const Box& got, const Box& want, const std::string& path) {
    for (int k = 0; k < 3; ++k) {
        const double tol = 1e-12 * std::max(1.0, std::fabs(want.extent[k]));
        if (got.ncells[k] != want.ncells[k] || std::fabs(got.extent[k] - want.extent[k]) > tol ||
            std::fabs(got.origin[k] - want.origin[k]) > tol)
            throw Error("netCDF: the box of " + path + " (ncells, extent, origin) differs from the context's");
    }
}

Info info(const std::string& path) {
    Reader rd(path);
    Info out;
    out.version = rd.h.version;
    const Att* ft = rd.gatt("file_type");
    if (!ft) throw Error("netCDF: " + path + " has no file_type attribute");
    out.file_type = att_string(*ft);
    out.box = read_box(rd);
    out.n_parcels = std::max<int64_t>(0, rd.dim_len("n_parcels"));
    out.n_steps = rd.h.numrecs;
    if (const Var* t = rd.var("t"))
        if (out.n_steps > 0) rd.read(*t, out.n_steps - 1, 0, 1, &out.t);
    const Att* lo = rd.gatt("l_lower_boundry_zeta_zero");
    const Att* hi = rd.gatt("l_upper_boundry_zeta_zero");
    if (lo && hi) {
        out.has_zeta = true;
        out.zeta[0] = att_string(*lo) == "true";
        out.zeta[1] = att_string(*hi) == "true";
    }
    return out;
}

void write_parcels(const std::string& path, const Box& box, const int32_t zeta[2], double t, int64_t n,
                   const double* pos, const double* vor, const double* B, const double* vol,
                   const double* buoy, const double* hum, int force_version, const int64_t* label,
                   const double* dil) {
    if (n < 0 || (n > 0 && (!pos || !vor || !B || !vol || !buoy))) throw Error("netCDF: bad parcel arrays");
    // a dimension of length 0 is the record dimension in the classic format
    if (n == 0) throw Error("netCDF: a parcel file needs at least one parcel");
    Header h;
    h.numrecs = 1;
    global_atts(h, box, "parcels", zeta);
    h.dims = {{"n_parcels", n}, {"world%size", 1}, {"t", 0}};
    h.vars.push_back(time_var(2, t));
    // the box of the single writer (parcel_netcdf.f90:256-290; 0-based cell indices)
    const int32_t box_vals[5] = {1, 0, box.ncells[0] - 1, 0, box.ncells[1] - 1};
    const char* box_names[5] = {"start_index", "xlo", "xhi", "ylo", "yhi"};
    for (int k = 0; k < 5; ++k) {
        const double v = box_vals[k];
        h.vars.push_back(dataset(box_names[k], "", "", "1", T_INT, {1},
                                 [v](int64_t, int64_t m, double* b) { std::fill(b, b + m, v); }));
    }
    auto comp = [](const double* a, int stride, int c) {
        return Source([a, stride, c](int64_t s, int64_t m, double* b) {
            for (int64_t k = 0; k < m; ++k) b[k] = a[(s + k) * stride + c];
        });
    };
    auto zeros = Source([](int64_t, int64_t m, double* b) { std::fill(b, b + m, 0.0); });
    const std::vector<int64_t> pd = {2, 0};
    const char* xyz[3] = {"x", "y", "z"};
    for (int c = 0; c < 3; ++c)
        h.vars.push_back(dataset(std::string(xyz[c]) + "_position", std::string(xyz[c]) + " position component",
                                 "", "m", T_DOUBLE, pd, comp(pos, 3, c)));
    const char* bn[5] = {"B11", "B12", "B13", "B22", "B23"};
    for (int c = 0; c < 5; ++c)
        h.vars.push_back(dataset(bn[c], std::string(bn[c]) + " element of shape matrix", "", "m^2", T_DOUBLE, pd,
                                 comp(B, 5, c)));
    h.vars.push_back(dataset("volume", "parcel volume", "", "m^3", T_DOUBLE, pd, comp(vol, 1, 0)));
    for (int c = 0; c < 3; ++c)
        h.vars.push_back(dataset(std::string(xyz[c]) + "_vorticity", std::string(xyz[c]) + " vorticity component",
                                 "", "1/s", T_DOUBLE, pd, comp(vor, 3, c)));
    h.vars.push_back(dataset("buoyancy", "parcel buoyancy", "", "m/s^2", T_DOUBLE, pd, comp(buoy, 1, 0)));
    h.vars.push_back(dataset("humidity", "parcel humidity", "", "1", T_DOUBLE, pd, hum ? comp(hum, 1, 0) : zeros));
    if (label) {
        // parcel_netcdf.f90:971-982; 64-bit integers need CDF-5
        h.vars.push_back(dataset("label", "parcel label", "", "1", T_INT64, pd,
                                 [label](int64_t s, int64_t m, double* b) {
                                     for (int64_t k = 0; k < m; ++k) b[k] = (double)label[s + k];
                                 }));
        h.vars.push_back(dataset("dilution", "parcel log dilution", "", "1", T_DOUBLE, pd,
                                 dil ? comp(dil, 1, 0) : zeros));
        force_version = 5;
    }
    write_file(path, h, force_version);
}

void read_parcels(const std::string& path, int64_t cap, int64_t* n, double* pos, double* vor, double* B,
                  double* vol, double* buoy, double* hum) {
    Reader rd(path);
    const Att* ft = rd.gatt("file_type");
    if (!ft || att_string(*ft) != "parcels") throw Error("netCDF: " + path + " is not a parcel file");
    const int64_t np = rd.dim_len("n_parcels");
    if (np < 0) throw Error("netCDF: " + path + " has no n_parcels dimension");
    if (n) *n = np;
    if (np > cap) throw Error("netCDF: more parcels in " + path + " than the arrays hold");
    std::vector<double> tmp((size_t)std::min<int64_t>(np, 1 << 20));
    auto get = [&](const char* name, double* dst, int stride, int c, bool required) -> bool {
        const Var* v = rd.var(name);
        if (!v) {
            if (required) throw Error(std::string("netCDF: ") + name + " must be present in " + path);
            if (dst) for (int64_t k = 0; k < np; ++k) dst[k * stride + c] = 0.0;
            return false;
        }
        if (slab_elems(rd.h, *v) != np) throw Error(std::string("netCDF: ") + name + " does not span n_parcels");
        if (!dst) return true;
        for (int64_t s = 0; s < np; s += (int64_t)tmp.size()) {
            const int64_t m = std::min<int64_t>((int64_t)tmp.size(), np - s);
            rd.read(*v, 0, s, m, tmp.data());
            for (int64_t k = 0; k < m; ++k) dst[(s + k) * stride + c] = tmp[(size_t)k];
        }
        return true;
    };
    const char* bn[5] = {"B11", "B12", "B13", "B22", "B23"};
    for (int c = 0; c < 5; ++c) get(bn[c], B, 5, c, true);
    get("x_position", pos, 3, 0, true);
    get("y_position", pos, 3, 1, true);
    get("z_position", pos, 3, 2, true);
    get("volume", vol, 1, 0, true);
    bool valid = false;
    valid |= get("x_vorticity", vor, 3, 0, false);
    valid |= get("y_vorticity", vor, 3, 1, false);
    valid |= get("z_vorticity", vor, 3, 2, false);
    valid |= get("buoyancy", buoy, 1, 0, false);
    valid |= get("humidity", hum, 1, 0, false);
    if (!valid) throw Error("netCDF: " + path + " holds neither vorticity, buoyancy nor humidity");
}

void write_fields(const std::string& path, const Box& box, const int32_t zeta[2], double t,
                  const std::vector<FieldOut>& fields, int force_version) {
    const int64_t nx = box.ncells[0], ny = box.ncells[1], nz = box.ncells[2];
    Header h;
    h.numrecs = 1;
    global_atts(h, box, "fields", zeta);
    h.dims = {{"x", nx}, {"y", ny}, {"z", nz + 1}, {"t", 0}};
    const double dx[3] = {box.extent[0] / nx, box.extent[1] / ny, box.extent[2] / nz};
    const char* axes[3] = {"X", "Y", "Z"};
    const char* names[3] = {"x", "y", "z"};
    for (int k = 0; k < 3; ++k) {
        const double o = box.origin[k], d = dx[k];
        Var v = k < 2 ? dataset(names[k], std::string(names[k]) + "-coordinate in projected coordinate system",
                                std::string("projection_") + names[k] + "_coordinate", "m", T_DOUBLE, {k},
                                [o, d](int64_t s, int64_t m, double* b) { for (int64_t i = 0; i < m; ++i) b[i] = o + double(s + i) * d; })
                      : dataset("z", "height coordinate in projected coordinate system", "height", "m", T_DOUBLE, {k},
                                [o, d](int64_t s, int64_t m, double* b) { for (int64_t i = 0; i < m; ++i) b[i] = o + double(s + i) * d; });
        v.atts.push_back(att_text("axis", axes[k]));
        h.vars.push_back(std::move(v));
    }
    h.vars.push_back(time_var(3, t));
    for (const FieldOut& fo : fields) {
        const double* a = fo.data;
        // file element (z, y, x), x fastest <- field layout (x, y, z + 1), z fastest
        Source src = [a, nx, ny, nz](int64_t s, int64_t m, double* b) {
            for (int64_t k = 0; k < m; ++k) {
                const int64_t e = s + k;
                const int64_t x = e % nx, y = (e / nx) % ny, z = e / (nx * ny);
                b[k] = a[(x * ny + y) * (nz + 3) + z + 1];
            }
        };
        h.vars.push_back(dataset(fo.name, fo.long_name, "", fo.unit, fo.integer ? T_INT : T_DOUBLE, {3, 2, 1, 0}, src));
    }
    write_file(path, h, force_version);
}

int64_t read_variable(const std::string& path, const std::string& name, int64_t record, int64_t cap, double* out) {
    Reader rd(path);
    const Var* v = rd.var(name);
    if (!v) throw Error("netCDF: no variable " + name + " in " + path);
    const int64_t n = slab_elems(rd.h, *v);
    if (!out) return n;
    if (n > cap) throw Error("netCDF: " + name + " has more elements than the buffer holds");
    rd.read(*v, record, 0, n, out);
    return n;
}

bool read_field(const std::string& path, const std::string& name, int64_t step, const Box& expect, double* out) {
    Reader rd(path);
    check_box(read_box(rd), expect, path);
    const Var* v = rd.var(name);
    if (!v) return false;
    const int64_t nx = expect.ncells[0], ny = expect.ncells[1], nz = expect.ncells[2];
    if (slab_elems(rd.h, *v) != nx * ny * (nz + 1)) throw Error("netCDF: " + name + " is not an (nz+1, ny, nx) field");
    int64_t r = 0;
    if (is_record(rd.h, *v)) {
        r = step < 0 ? rd.h.numrecs - 1 : step;
        if (r < 0 || r >= rd.h.numrecs) throw Error("netCDF: step out of range in " + path);
    }
    std::vector<double> plane((size_t)(nx * ny));
    for (int64_t z = 0; z <= nz; ++z) {
        rd.read(*v, r, z * nx * ny, nx * ny, plane.data());
        for (int64_t y = 0; y < ny; ++y)
            for (int64_t x = 0; x < nx; ++x) out[(x * ny + y) * (nz + 3) + z + 1] = plane[(size_t)(y * nx + x)];
    }
    return true;
}

}  // namespace ncio

// ---- host-level C entry points (include/epic_nc.h) --------------------------
#include "../../include/epic_nc.h"

namespace {
thread_local std::string nc_err;

template <class F>
int nc_call(F&& f) {
    try {
        f();
        nc_err.clear();
        return EPIC_OK;
    } catch (const ncio::Error& e) {
        nc_err = e.what();
        return EPIC_ERR_IO;
    } catch (const std::exception& e) {
        nc_err = e.what();
        return EPIC_ERR_IO;
    }
}

ncio::Box make_box(const int32_t ncells[3], const double origin[3], const double extent[3]) {
    if (!ncells || !origin || !extent) throw ncio::Error("netCDF: null box");
    ncio::Box b;
    for (int k = 0; k < 3; ++k) {
        if (ncells[k] <= 0) throw ncio::Error("netCDF: ncells must be positive");
        b.ncells[k] = ncells[k];
        b.origin[k] = origin[k];
        b.extent[k] = extent[k];
    }
    return b;
}
}  // namespace

extern "C" const char* epic_nc_last_error(void) { return nc_err.c_str(); }

extern "C" int epic_nc_info(const char* path, char file_type[16], int32_t ncells[3], double origin[3],
                            double extent[3], int64_t* n_parcels, int64_t* n_steps, double* t,
                            int32_t zeta_flags[2]) {
    return nc_call([&] {
        if (!path) throw ncio::Error("netCDF: null path");
        const ncio::Info in = ncio::info(path);
        if (file_type) {
            std::memset(file_type, 0, 16);
            std::strncpy(file_type, in.file_type.c_str(), 15);
        }
        for (int k = 0; k < 3; ++k) {
            if (ncells) ncells[k] = in.box.ncells[k];
            if (origin) origin[k] = in.box.origin[k];
            if (extent) extent[k] = in.box.extent[k];
        }
        if (n_parcels) *n_parcels = in.n_parcels;
        if (n_steps) *n_steps = in.n_steps;
        if (t) *t = in.t;
        if (zeta_flags) {
            zeta_flags[0] = in.has_zeta ? in.zeta[0] : -1;
            zeta_flags[1] = in.has_zeta ? in.zeta[1] : -1;
        }
    });
}

extern "C" int epic_nc_write_parcels(const char* path, const int32_t ncells[3], const double origin[3],
                                     const double extent[3], const int32_t zeta_flags[2], double t, int64_t n,
                                     const double* pos, const double* vor, const double* B, const double* vol,
                                     const double* buoy, const double* hum) {
    return nc_call([&] {
        if (!path) throw ncio::Error("netCDF: null path");
        ncio::write_parcels(path, make_box(ncells, origin, extent), zeta_flags, t, n, pos, vor, B, vol, buoy, hum);
    });
}

extern "C" int epic_nc_read_parcels(const char* path, int64_t cap, int64_t* n, double* pos, double* vor,
                                    double* B, double* vol, double* buoy, double* hum) {
    int64_t m = 0;
    const int rc = nc_call([&] {
        if (!path) throw ncio::Error("netCDF: null path");
        ncio::read_parcels(path, cap, &m, pos, vor, B, vol, buoy, hum);
    });
    if (n) *n = m;
    if (rc != EPIC_OK && m > cap) return EPIC_ERR_ARG;
    return rc;
}

extern "C" int epic_nc_read_field(const char* path, const char* name, int64_t step, const int32_t ncells[3],
                                  const double origin[3], const double extent[3], double* out) {
    return nc_call([&] {
        if (!path || !name || !out) throw ncio::Error("netCDF: null argument");
        if (!ncio::read_field(path, name, step, make_box(ncells, origin, extent), out))
            throw ncio::Error(std::string("netCDF: no variable ") + name + " in " + path);
    });
}

extern "C" int epic_nc_write_field_file(const char* path, const int32_t ncells[3], const double origin[3],
                                        const double extent[3], const int32_t zeta_flags[2], double t, int nfields,
                                        const char* const* names, const char* const* units,
                                        const double* const* data) {
    return nc_call([&] {
        if (!path || nfields < 0 || (nfields > 0 && (!names || !data))) throw ncio::Error("netCDF: null argument");
        std::vector<ncio::FieldOut> out;
        for (int k = 0; k < nfields; ++k) {
            if (!names[k] || !data[k]) throw ncio::Error("netCDF: null field");
            out.push_back({names[k], "", units && units[k] ? units[k] : "1", data[k], false});
        }
        ncio::write_fields(path, make_box(ncells, origin, extent), zeta_flags, t, out);
    });
}

extern "C" int epic_nc_read_variable(const char* path, const char* name, int64_t record, int64_t cap, int64_t* n,
                                     double* out) {
    int64_t m = 0;
    const int rc = nc_call([&] {
        if (!path || !name) throw ncio::Error("netCDF: null argument");
        m = ncio::read_variable(path, name, record, cap, out);
    });
    if (n) *n = m;
    return rc;
}
