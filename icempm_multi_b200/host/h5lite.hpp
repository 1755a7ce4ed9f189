// h5lite.hpp -- a small read-only HDF5 reader for the point-cloud files that
// SnapshotManager::LoadRawPoints opens (simulation/snapshotmanager.cpp:29-60):
// one root group holding 1-D datasets "x", "y" (float64) and "llGrainIDs"
// (integer) with a scalar attribute "volume".
//
// Written from the public HDF5 file-format specification.  It covers what
// such files use: superblock versions 0 and 1, version-1 object headers
// (with continuation blocks), old-style groups (symbol-table B-tree + local
// heap), dataspace / datatype / layout (compact, contiguous, chunked with a
// version-1 chunk B-tree) / filter-pipeline (deflate, shuffle, fletcher32)
// and attribute messages.  Anything else is reported as an error, never
// guessed.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace icy {
namespace h5 {

struct Datatype {
    int cls = -1;          // 0 fixed-point (integer), 1 floating point
    unsigned size = 0;     // bytes per element
    bool big_endian = false;
    bool is_signed = false;
};

class File {
public:
    explicit File(const std::string &path);   // throws std::runtime_error

    bool has(const std::string &name) const;
    std::vector<uint64_t> dims(const std::string &dataset) const;
    Datatype type(const std::string &dataset) const;
    // whole 1-D (or any-rank, row-major) dataset converted to double / uint64
    std::vector<double> read_double(const std::string &dataset) const;
    std::vector<uint64_t> read_uint64(const std::string &dataset) const;
    // scalar (or first element of an) attribute of a dataset, converted to double
    double attribute_double(const std::string &dataset, const std::string &attr) const;
    std::vector<std::string> names() const;

private:
    struct Message { uint16_t type; uint64_t pos; uint16_t size; };
    struct Object {
        std::vector<uint64_t> dims;
        Datatype dtype;
        int layout_class = -1;
        uint64_t data_addr = UINT64_MAX, data_size = 0;
        std::vector<uint32_t> chunk;            // chunk dims (last = element size)
        std::vector<uint8_t> compact;
        struct Filter { uint16_t id; uint16_t flags; std::vector<uint32_t> cd; };
        std::vector<Filter> filters;
        struct Attr { std::string name; Datatype dtype; std::vector<uint64_t> dims; uint64_t data_pos; };
        std::vector<Attr> attrs;
    };

    std::vector<uint8_t> buf_;
    unsigned so_ = 8, sl_ = 8;                 // size of offsets / lengths
    uint64_t base_ = 0;
    std::vector<std::pair<std::string, uint64_t>> entries_;   // root group: name -> object header

    uint64_t u(uint64_t pos, unsigned n) const;
    void need(uint64_t pos, uint64_t n) const;
    std::vector<Message> messages(uint64_t ohdr) const;
    void read_group(uint64_t btree, uint64_t heap);
    Object object(const std::string &name) const;
    Datatype parse_dtype(uint64_t pos) const;
    std::vector<uint64_t> parse_dataspace(uint64_t pos) const;
    std::vector<uint8_t> raw(const Object &o) const;
    std::vector<uint8_t> chunk_bytes(const Object &o, uint64_t addr, uint32_t size, uint32_t mask) const;
};

}  // namespace h5
}  // namespace icy
