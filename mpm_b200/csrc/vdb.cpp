// vdb.cpp -- OpenVDB file output of the density grid, without the OpenVDB
// library.
//
// The reference's MPMSolver3D::writeToOpenVDB (src/mpm_solver3d.cu:509-572)
// rasterises m_p w_ip / h^3 onto the grid nodes with an openvdb::FloatGrid
// accessor and writes one grid named "density" with OpenVDB's io::File.  The
// density itself comes from the GPU here (mpm_solver_download_density); this
// file writes it in the OpenVDB file format (file format version 224):
//
//   header     int64 magic 0x56444220, uint32 file version, uint32 library
//              major/minor, char has-grid-offsets (1), 36-char UUID text
//   file meta  uint32 count (0)
//   grids      int32 count (1), then per grid:
//     descriptor  string unique name, string type "Tree_float_5_4_3",
//                 string instance parent (""), int64 grid / block / end
//                 stream positions
//     grid        uint32 compression flags (2: active-mask compression, no
//                 zip or blosc), grid metadata (name, file bounding box and
//                 voxel count), transform ("UniformScaleMap", voxel size 1:
//                 the reference's default transform, voxel = node index),
//                 topology, buffers
//   topology   int32 buffer count (1); root: float background (0), uint32
//              tile count (0), uint32 child count, then per child (sorted by
//              origin) int32 origin[3] and the 32^3 internal node: child mask
//              (4096 bytes), value mask, one metadata byte (0: inactive
//              values are the background, only active values follow -- none
//              here), then its 16^3 children in mask order (child mask 512
//              bytes, value mask, metadata byte), then their 8^3 leaves in
//              mask order (value mask, 64 bytes)
//   buffers    per leaf in the same order: value mask, metadata byte (0), the
//              active voxels' floats in mask order
// Strings are a uint32 length and the bytes; everything is little endian.
// Node offsets put z fastest ((x << 2L) + (y << L) + z per level), mask bit i
// is bit i % 64 of 64-bit word i / 64, as OpenVDB does.
//
// Active voxels are the nodes with a non-zero density.  The reference also
// activates the zero-weight nodes at the exact edge of a stencil it visits;
// their value is the background 0 either way.
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <array>
#include <climits>
#include <map>
#include <random>
#include <string>
#include <vector>

#include "../../include/mpm_b200.h"

namespace mpm {

mpm_status recordError(mpm_status st, const char* msg);

namespace {

struct Out {
    std::vector<char> b;
    void raw(const void* p, size_t n) { b.insert(b.end(), (const char*)p, (const char*)p + n); }
    template <class T>
    void put(T v) {
        raw(&v, sizeof(T));
    }
    void str(const std::string& s) {
        put<uint32_t>((uint32_t)s.size());
        raw(s.data(), s.size());
    }
    template <class T>
    void patch(size_t at, T v) {
        memcpy(b.data() + at, &v, sizeof(T));
    }
};

using Coord = std::array<int32_t, 3>;

// A node of Log2 = L: child (or voxel) offset of a coordinate, and bit masks.
template <int L>
struct Mask {
    uint64_t w[(1u << (3 * L)) / 64] = {};
    void on(uint32_t i) { w[i >> 6] |= 1ull << (i & 63); }
    bool isOn(uint32_t i) const { return (w[i >> 6] >> (i & 63)) & 1ull; }
    void save(Out& o) const { o.raw(w, sizeof(w)); }
};

struct Leaf {  // 8^3
    Mask<3> mask;
    float v[512] = {};
};
struct Int1 {  // 16^3 children of 8^3 leaves: covers 128^3
    Mask<4> child;
    std::map<uint32_t, Leaf> leaves;  // by child offset (mask order)
};
struct Int2 {  // 32^3 children of Int1: covers 4096^3
    Mask<5> child;
    std::map<uint32_t, Int1> nodes;
};

template <int TOTAL_CHILD, int L>
uint32_t offsetOf(const Coord& c) {
    const int32_t dim = 1 << (TOTAL_CHILD + L);
    const uint32_t x = (uint32_t)(c[0] & (dim - 1)) >> TOTAL_CHILD, y = (uint32_t)(c[1] & (dim - 1)) >> TOTAL_CHILD,
                   z = (uint32_t)(c[2] & (dim - 1)) >> TOTAL_CHILD;
    return (x << (2 * L)) + (y << L) + z;
}

std::string uuidText() {
    std::random_device rd;
    std::mt19937_64 g(((uint64_t)rd() << 32) ^ rd());
    const char* hex = "0123456789abcdef";
    std::string s;
    for (int i = 0; i < 16; ++i) {
        if (i == 4 || i == 6 || i == 8 || i == 10) s += '-';
        const unsigned byte = (unsigned)(g() & 0xff);
        s += hex[byte >> 4];
        s += hex[byte & 15];
    }
    return s;  // 36 characters
}

}  // namespace

mpm_status writeDensityVdb(const float* density, const int32_t* res, const char* path) {
    if (!density || !res || !path) return recordError(MPM_ERR_INVALID_ARG, "write_vdb: null argument");
    for (int a = 0; a < 3; ++a)
        if (res[a] <= 0 || res[a] > (1 << 16)) return recordError(MPM_ERR_INVALID_ARG, "write_vdb: bad resolution");
    // Tree of the active voxels: root children (Int2) sorted by origin.
    std::map<Coord, Int2> root;
    int64_t voxels = 0;
    Coord lo = {INT32_MAX, INT32_MAX, INT32_MAX}, hi = {INT32_MIN, INT32_MIN, INT32_MIN};
    const size_t X = (size_t)res[0], Y = (size_t)res[1];
    for (int32_t z = 0; z < res[2]; ++z)
        for (int32_t y = 0; y < res[1]; ++y)
            for (int32_t x = 0; x < res[0]; ++x) {
                const float v = density[(size_t)x + X * ((size_t)y + Y * (size_t)z)];
                if (v == 0.0f) continue;
                const Coord c = {x, y, z};
                Int2& n2 = root[Coord{x & ~4095, y & ~4095, z & ~4095}];
                const uint32_t o2 = offsetOf<7, 5>(c);
                n2.child.on(o2);
                Int1& n1 = n2.nodes[o2];
                const uint32_t o1 = offsetOf<3, 4>(c);
                n1.child.on(o1);
                Leaf& lf = n1.leaves[o1];
                const uint32_t o0 = offsetOf<0, 3>(c);
                lf.mask.on(o0);
                lf.v[o0] = v;
                ++voxels;
                for (int a = 0; a < 3; ++a) {
                    lo[a] = std::min(lo[a], c[a]);
                    hi[a] = std::max(hi[a], c[a]);
                }
            }
    if (!voxels) lo = hi = Coord{0, 0, 0};

    Out o;
    // header
    o.put<int64_t>(0x56444220);
    o.put<uint32_t>(224);
    o.put<uint32_t>(10);
    o.put<uint32_t>(0);
    o.put<char>(1);
    const std::string uuid = uuidText();
    o.raw(uuid.data(), 36);
    o.put<uint32_t>(0);  // file-level metadata
    o.put<int32_t>(1);   // grids
    // grid descriptor
    o.str("density");
    o.str("Tree_float_5_4_3");
    o.str("");
    const size_t pos_at = o.b.size();
    o.put<int64_t>(0);
    o.put<int64_t>(0);
    o.put<int64_t>(0);
    const int64_t grid_pos = (int64_t)o.b.size();
    o.put<uint32_t>(2);  // COMPRESS_ACTIVE_MASK
    // grid metadata
    o.put<uint32_t>(4);
    o.str("file_bbox_max");
    o.str("vec3i");
    o.put<uint32_t>(12);
    o.raw(hi.data(), 12);
    o.str("file_bbox_min");
    o.str("vec3i");
    o.put<uint32_t>(12);
    o.raw(lo.data(), 12);
    o.str("file_voxel_count");
    o.str("int64");
    o.put<uint32_t>(8);
    o.put<int64_t>(voxels);
    o.str("name");
    o.str("string");
    o.str("density");
    // transform: uniform scale 1 (scale, voxel size, inverse scale, inverse
    // scale squared, inverse twice scale)
    o.str("UniformScaleMap");
    const double vec[5][3] = {{1, 1, 1}, {1, 1, 1}, {1, 1, 1}, {1, 1, 1}, {0.5, 0.5, 0.5}};
    o.raw(vec, sizeof(vec));
    // topology
    o.put<int32_t>(1);
    o.put<float>(0.0f);
    o.put<uint32_t>(0);
    o.put<uint32_t>((uint32_t)root.size());
    const Mask<5> none5;
    const Mask<4> none4;
    for (auto& [origin, n2] : root) {
        o.raw(origin.data(), 12);
        n2.child.save(o);
        none5.save(o);
        o.put<int8_t>(0);
        for (auto& [k1, n1] : n2.nodes) {
            n1.child.save(o);
            none4.save(o);
            o.put<int8_t>(0);
            for (auto& [k0, lf] : n1.leaves) lf.mask.save(o);
        }
    }
    const int64_t block_pos = (int64_t)o.b.size();
    // buffers
    for (auto& [origin, n2] : root)
        for (auto& [k1, n1] : n2.nodes)
            for (auto& [k0, lf] : n1.leaves) {
                lf.mask.save(o);
                o.put<int8_t>(0);
                for (uint32_t i = 0; i < 512; ++i)
                    if (lf.mask.isOn(i)) o.put<float>(lf.v[i]);
            }
    const int64_t end_pos = (int64_t)o.b.size();
    o.patch<int64_t>(pos_at, grid_pos);
    o.patch<int64_t>(pos_at + 8, block_pos);
    o.patch<int64_t>(pos_at + 16, end_pos);

    FILE* f = fopen(path, "wb");
    if (!f) return recordError(MPM_ERR_IO, (std::string("write_vdb: cannot open ") + path).c_str());
    const bool ok = fwrite(o.b.data(), 1, o.b.size(), f) == o.b.size();
    if (fclose(f) != 0 || !ok) return recordError(MPM_ERR_IO, (std::string("write_vdb: cannot write ") + path).c_str());
    return MPM_OK;
}

}  // namespace mpm

extern "C" mpm_status mpm_write_vdb_density(const float* density, const int32_t* resolution, const char* path) {
    return mpm::writeDensityVdb(density, resolution, path);
}
