// kf_io.cpp -- reader and writer of the .kfh container (kf_io.hpp).
#include "kf_io.hpp"

#include <cstdio>
#include <cstring>

namespace kfio {

namespace {
Entry make(const std::string &name, uint8_t type, std::vector<uint64_t> dims, const void *p, size_t bytes) {
    Entry e;
    e.name = name;
    e.type = type;
    e.dims = std::move(dims);
    e.data.resize(bytes);
    if (bytes) std::memcpy(e.data.data(), p, bytes);
    return e;
}
size_t elem_size(uint8_t t) { return t == F64 || t == I64 ? 8 : t == I32 ? 4 : 1; }
}  // namespace

void File::f64(const std::string &name, double v) { entries.push_back(make(name, F64, {}, &v, 8)); }
void File::i32(const std::string &name, int32_t v) { entries.push_back(make(name, I32, {}, &v, 4)); }
void File::i64(const std::string &name, int64_t v) { entries.push_back(make(name, I64, {}, &v, 8)); }
void File::str(const std::string &name, const std::string &v) {
    entries.push_back(make(name, STR, {v.size()}, v.data(), v.size()));
}
void File::array(const std::string &name, const std::vector<uint64_t> &dims, const double *v) {
    size_t c = 1;
    for (auto d : dims) c *= d;
    entries.push_back(make(name, F64, dims, v, 8 * c));
}

bool File::write(const std::string &path, std::string &err) const {
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) {
        err = "cannot open " + path + " for writing";
        return false;
    }
    bool ok = std::fwrite("KFH1", 1, 4, f) == 4;
    const uint32_t n = (uint32_t)entries.size();
    ok = ok && std::fwrite(&n, 4, 1, f) == 1;
    for (const Entry &e : entries) {
        const uint16_t nl = (uint16_t)e.name.size();
        const uint8_t rank = (uint8_t)e.dims.size();
        ok = ok && std::fwrite(&nl, 2, 1, f) == 1 && std::fwrite(e.name.data(), 1, nl, f) == nl;
        ok = ok && std::fwrite(&e.type, 1, 1, f) == 1 && std::fwrite(&rank, 1, 1, f) == 1;
        if (rank) ok = ok && std::fwrite(e.dims.data(), 8, rank, f) == rank;
        if (!e.data.empty()) ok = ok && std::fwrite(e.data.data(), 1, e.data.size(), f) == e.data.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) err = "write error on " + path;
    return ok;
}

bool File::read(const std::string &path, std::string &err) {
    entries.clear();
    FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) {
        err = "cannot open " + path;
        return false;
    }
    char magic[4];
    uint32_t n = 0;
    bool ok = std::fread(magic, 1, 4, f) == 4 && std::memcmp(magic, "KFH1", 4) == 0 && std::fread(&n, 4, 1, f) == 1;
    for (uint32_t i = 0; ok && i < n; ++i) {
        Entry e;
        uint16_t nl = 0;
        uint8_t rank = 0;
        ok = std::fread(&nl, 2, 1, f) == 1;
        e.name.resize(nl);
        ok = ok && (nl == 0 || std::fread(&e.name[0], 1, nl, f) == nl);
        ok = ok && std::fread(&e.type, 1, 1, f) == 1 && std::fread(&rank, 1, 1, f) == 1;
        ok = ok && e.type >= F64 && e.type <= I64 && rank <= 8;
        if (!ok) break;
        e.dims.resize(rank);
        if (rank) ok = std::fread(e.dims.data(), 8, rank, f) == rank;
        if (!ok) break;
        const size_t bytes = e.count() * elem_size(e.type);
        if (bytes > (size_t)1 << 40) {
            ok = false;
            break;
        }
        e.data.resize(bytes);
        ok = bytes == 0 || std::fread(e.data.data(), 1, bytes, f) == bytes;
        if (ok) entries.push_back(std::move(e));
    }
    std::fclose(f);
    if (!ok) err = path + " is not a valid .kfh file";
    return ok;
}

const Entry *File::find(const std::string &name) const {
    for (const Entry &e : entries)
        if (e.name == name) return &e;
    return nullptr;
}

bool File::get_f64(const std::string &name, double &v) const {
    const Entry *e = find(name);
    if (!e || e->type != F64 || e->count() != 1) return false;
    std::memcpy(&v, e->data.data(), 8);
    return true;
}

bool File::get_i32(const std::string &name, int32_t &v) const {
    const Entry *e = find(name);
    if (!e || e->type != I32 || e->count() != 1) return false;
    std::memcpy(&v, e->data.data(), 4);
    return true;
}

}  // namespace kfio
