// Checkpoint / restart and particle writers of one vector (host side).
//
// save / load (vector_dist.hpp:2459-2476) write and read the domain particles --
// positions, global ids and every property -- in this library's own binary
// format (the reference's HDF5_writer/HDF5_reader live in openfpm_io, which is not
// part of the reference tree, and HDF5 is not a dependency here):
//
//   offset  size         field
//   0       8            magic "PDVDIST1"
//   8       4 x 4        version (1), dim (3), dtype (PD_F32 / PD_F64), nprops
//   24      8            n (domain particles)
//   32      9 x 8        lo[3], hi[3], ghost[3] (double)
//   104     4 x 4        bc[3], 0
//   120     nprops x 8   (type, ncomp) per property (int32 each)
//   ...     n x 3 x St   positions, particle-major (x, y, z)
//   ...     n x 4        global ids (int32)
//   ...     per property, component-major: ncomp x n x element
//   end     8            FNV-1a 64 of every byte after the header's property table
//
// load replaces the vector's particles (ghosts dropped); the vector must have the
// file's dtype, and either no properties (they are added) or the file's list.
//
// write / write_frame (vector_dist.hpp:2498-2721) emit the domain particles as VTK
// XML PolyData (`<out>_0.vtp`, ASCII or base64 binary) or CSV (`<out>_0.csv`);
// openfpm_io's writers are not in the reference tree, so the layouts are the
// standard VTK XML PolyData and a one-header-line CSV, with properties named
// attr<k> like the reference's default property names.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "pd_internal.cuh"

namespace pd {

static const char MAGIC[8] = {'P', 'D', 'V', 'D', 'I', 'S', 'T', '1'};

struct Fnv {
    unsigned long long h = 1469598103934665603ull;
    void add(const void* p, size_t n) {
        const unsigned char* b = (const unsigned char*)p;
        for (size_t i = 0; i < n; ++i) {
            h ^= b[i];
            h *= 1099511628211ull;
        }
    }
};

struct File {
    FILE* f = nullptr;
    explicit File(const char* path, const char* mode) { f = fopen(path, mode); }
    ~File() {
        if (f) fclose(f);
    }
};

static bool wr(FILE* f, const void* p, size_t n, Fnv* h = nullptr) {
    if (h) h->add(p, n);
    return n == 0 || fwrite(p, 1, n, f) == n;
}
static bool rd(FILE* f, void* p, size_t n, Fnv* h = nullptr) {
    if (n && fread(p, 1, n, f) != n) return false;
    if (h) h->add(p, n);
    return true;
}

// domain particles on the host: xyz (St), gids, property columns (component-major)
struct HostCopy {
    std::vector<unsigned char> pos;
    std::vector<int> gid;
    std::vector<std::vector<unsigned char>> prop;
};

static int fetch(pd_vd h, HostCopy& c) {
    const long n = h->n_real;
    const size_t es = h->dtype == PD_F64 ? 8 : 4;
    c.pos.resize(es * 3 * (size_t)n);
    std::vector<long> g((size_t)n);
    if (n) {
        PD_TRY(pd_d2h_pos(h, c.pos.data(), 0, n, nullptr));
        PD_TRY(pd_d2h_gid(h, g.data(), 0, n, nullptr));
    }
    c.gid.assign(g.begin(), g.end());
    c.prop.resize(h->props.size());
    for (size_t p = 0; p < h->props.size(); ++p) {
        const Prop& P = h->props[p];
        c.prop[p].resize((size_t)P.esize * P.ncomp * n);
        if (n) PD_TRY(pd_d2h_prop(h, (int)p, c.prop[p].data(), 0, n, nullptr));
    }
    return PD_OK;
}

static const char* vtk_type(int t) {
    switch (t) {
        case PD_F32: return "Float32";
        case PD_F64: return "Float64";
        case PD_I32: return "Int32";
        case PD_U32: return "UInt32";
        default: return "Int64";
    }
}

static void put_value(std::string& s, const unsigned char* base, int type, size_t i) {
    char buf[64];
    switch (type) {
        case PD_F32: snprintf(buf, sizeof(buf), "%.9g", (double)((const float*)base)[i]); break;
        case PD_F64: snprintf(buf, sizeof(buf), "%.17g", ((const double*)base)[i]); break;
        case PD_I32: snprintf(buf, sizeof(buf), "%d", ((const int*)base)[i]); break;
        case PD_U32: snprintf(buf, sizeof(buf), "%u", ((const unsigned int*)base)[i]); break;
        default: snprintf(buf, sizeof(buf), "%lld", ((const long long*)base)[i]); break;
    }
    s += buf;
}

static void base64(std::string& out, const unsigned char* p, size_t n) {
    static const char T[] = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
    size_t i = 0;
    for (; i + 2 < n; i += 3) {
        const unsigned v = (p[i] << 16) | (p[i + 1] << 8) | p[i + 2];
        out += T[v >> 18];
        out += T[(v >> 12) & 63];
        out += T[(v >> 6) & 63];
        out += T[v & 63];
    }
    if (i < n) {
        const unsigned v = (p[i] << 16) | ((i + 1 < n ? p[i + 1] : 0) << 8);
        out += T[v >> 18];
        out += T[(v >> 12) & 63];
        out += i + 1 < n ? T[(v >> 6) & 63] : '=';
        out += '=';
    }
}

// one DataArray: `vals` holds n tuples of ncomp elements of `type`, tuple-major
static void data_array(std::string& s, const char* name, int type, int ncomp, const std::vector<unsigned char>& vals,
                       size_t n, bool binary) {
    s += "<DataArray type=\"";
    s += vtk_type(type);
    s += "\" Name=\"";
    s += name;
    s += "\" NumberOfComponents=\"" + std::to_string(ncomp) + "\" format=\"" + (binary ? "binary" : "ascii") + "\">\n";
    const size_t es = (size_t)type_size(type);
    if (binary) {
        // base64 of a 32-bit byte count followed by the raw values (VTK XML binary, no compression)
        const unsigned int nb = (unsigned int)(n * ncomp * es);
        std::vector<unsigned char> blk(4 + (size_t)nb);
        memcpy(blk.data(), &nb, 4);
        if (nb) memcpy(blk.data() + 4, vals.data(), nb);
        base64(s, blk.data(), blk.size());
        s += "\n";
    } else {
        for (size_t i = 0; i < n; ++i) {
            for (int c = 0; c < ncomp; ++c) {
                if (c) s += ' ';
                put_value(s, vals.data(), type, i * ncomp + c);
            }
            s += '\n';
        }
    }
    s += "</DataArray>\n";
}

// property p of the host copy (component-major), re-laid tuple-major
static std::vector<unsigned char> tuples(const std::vector<unsigned char>& cm, int esize, int ncomp, size_t n) {
    std::vector<unsigned char> t(cm.size());
    for (int k = 0; k < ncomp; ++k)
        for (size_t i = 0; i < n; ++i)
            memcpy(&t[(i * ncomp + k) * esize], &cm[((size_t)k * n + i) * esize], esize);
    return t;
}

static int write_vtp(pd_vd h, const HostCopy& c, const std::string& path, const char* meta, bool binary) {
    const size_t n = (size_t)h->n_real;
    std::string s;
    s.reserve(256 + n * 64);
    s += "<?xml version=\"1.0\"?>\n<VTKFile type=\"PolyData\" version=\"1.0\" byte_order=\"LittleEndian\" "
         "header_type=\"UInt32\">\n<PolyData>\n";
    if (meta && *meta) {
        // "name = value" meta information becomes a one-value FieldData array
        std::string m(meta), name = m, val = "0";
        size_t eq = m.find('=');
        if (eq != std::string::npos) {
            name = m.substr(0, eq);
            val = m.substr(eq + 1);
        }
        auto trim = [](std::string& x) {
            size_t a = x.find_first_not_of(" \t"), b = x.find_last_not_of(" \t");
            x = a == std::string::npos ? std::string() : x.substr(a, b - a + 1);
        };
        trim(name);
        trim(val);
        s += "<FieldData>\n<DataArray type=\"Float64\" Name=\"" + name +
             "\" NumberOfTuples=\"1\" format=\"ascii\">\n" + val + "\n</DataArray>\n</FieldData>\n";
    }
    s += "<Piece NumberOfPoints=\"" + std::to_string(n) + "\" NumberOfVerts=\"" + std::to_string(n) +
         "\" NumberOfLines=\"0\" NumberOfStrips=\"0\" NumberOfPolys=\"0\">\n<Points>\n";
    data_array(s, "Points", h->dtype, 3, c.pos, n, binary);
    s += "</Points>\n<Verts>\n";
    std::vector<unsigned char> conn(sizeof(long long) * n), offs(sizeof(long long) * n);
    for (size_t i = 0; i < n; ++i) {
        long long a = (long long)i, b = (long long)i + 1;
        memcpy(&conn[i * 8], &a, 8);
        memcpy(&offs[i * 8], &b, 8);
    }
    data_array(s, "connectivity", PD_I64, 1, conn, n, binary);
    data_array(s, "offsets", PD_I64, 1, offs, n, binary);
    s += "</Verts>\n<PointData>\n";
    for (size_t p = 0; p < h->props.size(); ++p) {
        const Prop& P = h->props[p];
        const std::string name = "attr" + std::to_string(p);
        data_array(s, name.c_str(), P.type, P.ncomp, tuples(c.prop[p], P.esize, P.ncomp, n), n, binary);
    }
    s += "</PointData>\n</Piece>\n</PolyData>\n</VTKFile>\n";
    File f(path.c_str(), "wb");
    if (!f.f || !wr(f.f, s.data(), s.size())) {
        set_error("write: cannot write %s", path.c_str());
        return PD_EIO;
    }
    return PD_OK;
}

static int write_csv(pd_vd h, const HostCopy& c, const std::string& path) {
    const size_t n = (size_t)h->n_real;
    std::string s = "x[0],x[1],x[2]";
    for (size_t p = 0; p < h->props.size(); ++p)
        for (int k = 0; k < h->props[p].ncomp; ++k)
            s += h->props[p].ncomp == 1 ? ",attr" + std::to_string(p)
                                        : ",attr" + std::to_string(p) + "[" + std::to_string(k) + "]";
    s += '\n';
    for (size_t i = 0; i < n; ++i) {
        for (int d = 0; d < 3; ++d) {
            if (d) s += ',';
            put_value(s, c.pos.data(), h->dtype, i * 3 + d);
        }
        for (size_t p = 0; p < h->props.size(); ++p)
            for (int k = 0; k < h->props[p].ncomp; ++k) {
                s += ',';
                put_value(s, c.prop[p].data(), h->props[p].type, (size_t)k * n + i);
            }
        s += '\n';
    }
    File f(path.c_str(), "wb");
    if (!f.f || !wr(f.f, s.data(), s.size())) {
        set_error("write: cannot write %s", path.c_str());
        return PD_EIO;
    }
    return PD_OK;
}

static int write_any(pd_vd h, const std::string& path, const char* meta, int opt) {
    HostCopy c;
    PD_TRY(fetch(h, c));
    if (opt & PD_CSV_WRITER) return write_csv(h, c, path);
    return write_vtp(h, c, path, meta, (opt & PD_FORMAT_BINARY) != 0);
}

}  // namespace pd

using namespace pd;

extern "C" {

int pd_save(pd_vd h, const char* path) {
    if (!h || !path) return PD_EINVAL;
    HostCopy c;
    PD_TRY(fetch(h, c));
    File f(path, "wb");
    if (!f.f) {
        set_error("save: cannot open %s", path);
        return PD_EIO;
    }
    const long long n = h->n_real;
    const unsigned int hdr[4] = {1u, 3u, (unsigned int)h->dtype, (unsigned int)h->props.size()};
    const int bc[4] = {h->bc[0], h->bc[1], h->bc[2], 0};
    bool ok = wr(f.f, MAGIC, 8) && wr(f.f, hdr, sizeof(hdr)) && wr(f.f, &n, 8) && wr(f.f, h->lo, 24) &&
              wr(f.f, h->hi, 24) && wr(f.f, h->g, 24) && wr(f.f, bc, sizeof(bc));
    for (auto& P : h->props) {
        const int d[2] = {P.type, P.ncomp};
        ok = ok && wr(f.f, d, 8);
    }
    Fnv sum;
    ok = ok && wr(f.f, c.pos.data(), c.pos.size(), &sum) && wr(f.f, c.gid.data(), c.gid.size() * 4, &sum);
    for (auto& col : c.prop) ok = ok && wr(f.f, col.data(), col.size(), &sum);
    ok = ok && wr(f.f, &sum.h, 8);
    if (!ok) {
        set_error("save: write to %s failed", path);
        return PD_EIO;
    }
    return PD_OK;
}

int pd_load(pd_vd h, const char* path) {
    if (!h || !path) return PD_EINVAL;
    File f(path, "rb");
    if (!f.f) {
        set_error("load: cannot open %s", path);
        return PD_EIO;
    }
    char magic[8];
    unsigned int hdr[4];
    long long n = 0;
    double lo[3], hi[3], g[3];
    int bc[4];
    if (!rd(f.f, magic, 8) || memcmp(magic, MAGIC, 8) != 0 || !rd(f.f, hdr, sizeof(hdr)) || hdr[0] != 1u ||
        hdr[1] != 3u || !rd(f.f, &n, 8) || n < 0 || n >= (1LL << 31) || !rd(f.f, lo, 24) || !rd(f.f, hi, 24) ||
        !rd(f.f, g, 24) || !rd(f.f, bc, sizeof(bc)) || hdr[3] > 16) {
        set_error("load: %s is not a checkpoint of this format", path);
        return PD_EIO;
    }
    if ((int)hdr[2] != h->dtype) {
        set_error("load: %s holds %s positions, the vector %s", path, hdr[2] == PD_F64 ? "FP64" : "FP32",
                  h->dtype == PD_F64 ? "FP64" : "FP32");
        return PD_EINVAL;
    }
    std::vector<int> pd_(2 * hdr[3]);
    if (!rd(f.f, pd_.data(), pd_.size() * 4)) {
        set_error("load: %s is truncated", path);
        return PD_EIO;
    }
    for (unsigned p = 0; p < hdr[3]; ++p)
        if (type_size(pd_[2 * p]) == 0 || pd_[2 * p + 1] < 1 || pd_[2 * p + 1] > 64) {
            set_error("load: %s has an invalid property table", path);
            return PD_EIO;
        }
    // the file must hold exactly the data its header announces (checked before any allocation)
    {
        size_t need = 8 + sizeof(hdr) + 8 + 72 + sizeof(bc) + pd_.size() * 4;
        const size_t esz = hdr[2] == PD_F64 ? 8 : 4;
        need += (size_t)n * (3 * esz + 4) + 8;
        for (unsigned p = 0; p < hdr[3]; ++p) need += (size_t)type_size(pd_[2 * p]) * pd_[2 * p + 1] * (size_t)n;
        const long here = ftell(f.f);
        if (here < 0 || fseek(f.f, 0, SEEK_END) != 0) {
            set_error("load: cannot size %s", path);
            return PD_EIO;
        }
        const long size = ftell(f.f);
        if (size < 0 || (size_t)size != need || fseek(f.f, here, SEEK_SET) != 0) {
            set_error("load: %s holds %ld bytes, its header announces %zu", path, size, need);
            return PD_EIO;
        }
    }
    const bool add = h->props.empty() && hdr[3] > 0;
    if (!add) {
        bool same = h->props.size() == hdr[3];
        for (unsigned p = 0; same && p < hdr[3]; ++p)
            same = h->props[p].type == pd_[2 * p] && h->props[p].ncomp == pd_[2 * p + 1];
        if (!same) {
            set_error("load: the properties of %s differ from the vector's", path);
            return PD_EINVAL;
        }
    }
    const size_t es = h->dtype == PD_F64 ? 8 : 4;
    HostCopy c;
    c.pos.resize(es * 3 * (size_t)n);
    c.gid.resize((size_t)n);
    c.prop.resize(hdr[3]);
    Fnv sum;
    bool ok = rd(f.f, c.pos.data(), c.pos.size(), &sum) && rd(f.f, c.gid.data(), c.gid.size() * 4, &sum);
    for (unsigned p = 0; ok && p < hdr[3]; ++p) {
        c.prop[p].resize((size_t)type_size(pd_[2 * p]) * pd_[2 * p + 1] * n);
        ok = rd(f.f, c.prop[p].data(), c.prop[p].size(), &sum);
    }
    unsigned long long stored = 0;
    ok = ok && rd(f.f, &stored, 8);
    if (!ok || stored != sum.h) {
        set_error("load: %s is truncated or corrupt (checksum)", path);
        return PD_EIO;
    }
    if (add)
        for (unsigned p = 0; p < hdr[3]; ++p) {
            int id = -1;
            PD_TRY(pd_add_prop(h, pd_[2 * p], pd_[2 * p + 1], &id));
        }
    PD_TRY(pd_resize(h, (long)n));
    if (n) {
        PD_TRY(pd_h2d_pos(h, c.pos.data(), 0, (long)n, nullptr));
        PD_CUDA(cudaMemcpy(h->gid, c.gid.data(), sizeof(int) * (size_t)n, cudaMemcpyHostToDevice));
        for (unsigned p = 0; p < hdr[3]; ++p) PD_TRY(pd_h2d_prop(h, (int)p, c.prop[p].data(), 0, (long)n, nullptr));
    }
    PD_CUDA(cudaDeviceSynchronize());
    return PD_OK;
}

int pd_write(pd_vd h, const char* out, const char* meta, int opt) {
    if (!h || !out) return PD_EINVAL;
    return write_any(h, std::string(out) + ((opt & PD_CSV_WRITER) ? "_0.csv" : "_0.vtp"), meta, opt);
}

int pd_write_frame(pd_vd h, const char* out, long iteration, const char* meta, int opt) {
    if (!h || !out || iteration < 0) return PD_EINVAL;
    return write_any(h, std::string(out) + "_0_" + std::to_string(iteration) + ((opt & PD_CSV_WRITER) ? ".csv" : ".vtp"),
                     meta, opt);
}

}  // extern "C"
