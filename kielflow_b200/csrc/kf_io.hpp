// kf_io.hpp -- the .kfh container: the reference's HDF5 file layout
// (IO.cpp:60-505, 1295-1340) written as a flat list of named datasets.
//
// File: "KFH1", u32 entry count, then per entry
//   u16 name length, name (the HDF5 path, e.g. "domain/N_x", "data/Ux"),
//   u8 type (1 f64, 2 i32, 3 string, 4 i64), u8 rank, u64 dims[rank],
//   payload (prod(dims) elements, little endian; a string's dims[0] bytes).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace kfio {

enum Type : uint8_t { F64 = 1, I32 = 2, STR = 3, I64 = 4 };

struct Entry {
    std::string name;
    uint8_t type = F64;
    std::vector<uint64_t> dims;
    std::vector<char> data;
    size_t count() const {
        size_t c = 1;
        for (auto d : dims) c *= d;
        return c;
    }
};

class File {
public:
    void f64(const std::string &name, double v);
    void i32(const std::string &name, int32_t v);
    void i64(const std::string &name, int64_t v);
    void str(const std::string &name, const std::string &v);
    void array(const std::string &name, const std::vector<uint64_t> &dims, const double *v);
    bool write(const std::string &path, std::string &err) const;
    bool read(const std::string &path, std::string &err);
    const Entry *find(const std::string &name) const;
    bool get_f64(const std::string &name, double &v) const;
    bool get_i32(const std::string &name, int32_t &v) const;
    std::vector<Entry> entries;
};

}  // namespace kfio
