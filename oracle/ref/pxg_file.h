// Binary CSR graph file shared by the reference drivers (test infrastructure).
//
// Layout (little endian):
//   char[8]  magic "PXCSR001"
//   u64      n            number of vertices
//   u64      m            number of undirected edges (the file holds 2m slots)
//   u64      offset_bytes 4 or 8
//   offsets  (n+1) * offset_bytes
//   columns  2m * u32
//
// The reference drivers only read 4-byte offsets, because the reference's
// Graph type stores ranges as unsigned int (lib/core/definitions.h:23-24).
#pragma once
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

struct PxgFile {
    uint64_t n = 0, m = 0;
    std::vector<uint32_t> offsets;
    std::vector<uint32_t> cols;
};

inline PxgFile pxg_read(const std::string& path) {
    PxgFile g;
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) { std::fprintf(stderr, "cannot open %s\n", path.c_str()); std::exit(2); }
    char magic[8];
    uint64_t hdr[3];
    if (std::fread(magic, 1, 8, f) != 8 || std::memcmp(magic, "PXCSR001", 8) != 0 ||
        std::fread(hdr, 8, 3, f) != 3) {
        std::fprintf(stderr, "bad graph file %s\n", path.c_str()); std::exit(2);
    }
    g.n = hdr[0]; g.m = hdr[1];
    if (hdr[2] != 4) { std::fprintf(stderr, "reference drivers need 4-byte offsets\n"); std::exit(2); }
    g.offsets.resize(g.n + 1);
    g.cols.resize(2 * g.m);
    if (std::fread(g.offsets.data(), 4, g.n + 1, f) != g.n + 1 ||
        std::fread(g.cols.data(), 4, 2 * g.m, f) != 2 * g.m) {
        std::fprintf(stderr, "short graph file %s\n", path.c_str()); std::exit(2);
    }
    std::fclose(f);
    return g;
}

template <typename T>
inline std::vector<T> raw_read(const std::string& path, size_t count) {
    std::vector<T> v(count);
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f || std::fread(v.data(), sizeof(T), count, f) != count) {
        std::fprintf(stderr, "cannot read %zu items from %s\n", count, path.c_str()); std::exit(2);
    }
    std::fclose(f);
    return v;
}

template <typename T>
inline void raw_write(const std::string& path, const T* data, size_t count) {
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f || std::fwrite(data, sizeof(T), count, f) != count) {
        std::fprintf(stderr, "cannot write %s\n", path.c_str()); std::exit(2);
    }
    std::fclose(f);
}
