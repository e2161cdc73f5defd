// Host side of the 2-D AMR path: the patch hierarchy, its validation,
// Berger-Rigoutsos clustering, the Berger-Oliger flag processing and the
// flat transfer plans uploaded to the device.  Restates the reference's
// src/geometry/amr/{grid,cluster,adapt,intergrid}.rs; the per-step work
// (ghost fill, restriction, tagging, stepping) runs on the device.
#pragma once

#include <array>
#include <cstdint>
#include <string>
#include <vector>

namespace lg {
namespace amr {

// Half-open box of cells at one level (amr/cluster.rs:27-113), 2-D.
struct Box {
    int64_t lo[2] = {0, 0}, hi[2] = {0, 0};
    int64_t extent(int d) const { return hi[d] - lo[d]; }
    uint64_t cells() const {
        return (extent(0) > 0 && extent(1) > 0) ? (uint64_t)extent(0) * (uint64_t)extent(1) : 0;
    }
    bool contains(int64_t x, int64_t y) const { return lo[0] <= x && x < hi[0] && lo[1] <= y && y < hi[1]; }
    bool intersects(const Box& o) const {
        return lo[0] < o.hi[0] && o.lo[0] < hi[0] && lo[1] < o.hi[1] && o.lo[1] < hi[1];
    }
    Box clipped(const Box& d) const;
    bool operator==(const Box& o) const {
        return lo[0] == o.lo[0] && lo[1] == o.lo[1] && hi[0] == o.hi[0] && hi[1] == o.hi[1];
    }
};

struct Patch {
    int level;
    Box bx;
};

struct Base {
    int64_t cells[2], block[2];
    double origin[2], spacing[2];
};

// The hierarchy: level 0 is the base tiling, finer levels are patches in
// their own index space; BlockId = patch index, level-major
// (amr/grid.rs:55-70).
struct Layout {
    Base base{};
    std::vector<uint32_t> ratios;
    std::vector<Patch> patches;
    std::vector<uint32_t> level_start;
    std::vector<std::array<double, 2>> level_spacing;
    // Per level, a bucket grid over the level's domain: bucket (bx, by) of
    // side `side` lists the patches of the level that intersect it (CSR).
    // Memory is proportional to the domain / side^2 plus the patch count,
    // not to the number of cells of a fine level's domain.
    struct Index {
        int64_t side = 32, nbx = 0, nby = 0;
        std::vector<uint32_t> start, items;
    };
    std::vector<Index> index;

    int num_levels() const { return (int)level_start.size() - 1; }
    int max_levels() const { return (int)ratios.size() + 1; }
    int num_blocks() const { return (int)patches.size(); }
    Box domain(int level) const;
    int find(int level, int64_t x, int64_t y) const;  // -1 if uncovered or outside
    // every cell of `need` lies in a patch of `level` (amr/grid.rs:293-322)
    bool covers(int level, const Box& need) const;
};

// AmrGrid::from_patches (amr/grid.rs:90-196); returns "" or the error text.
std::string build_layout(const Base& base, const std::vector<uint32_t>& ratios,
                         const std::vector<std::vector<Box>>& levels, Layout* out);

// Berger-Rigoutsos (amr/cluster.rs:144-290); `flags` is reordered.
std::vector<Box> cluster(std::vector<std::array<int64_t, 2>>& flags, double efficiency, int64_t min_width);

struct Policy {
    int64_t every = 4, buffer = 2, min_width = 4;
    double efficiency = 0.8, threshold = 0.1;
    int field = 0;
};

// BergerOliger::regrid's box construction (adapt.rs:164-226): `flags[l]`
// are the tags of level l; returns the proposed boxes per refined level.
std::vector<std::vector<Box>> propose(const Layout& g, std::vector<std::vector<std::array<int64_t, 2>>>& flags,
                                      const Policy& p);
// hierarchy_acceptable (adapt.rs:269-290)
bool acceptable(const Layout& g, const std::vector<std::vector<Box>>& proposed);

// ------------------------------------------------------------ plans ------
// Slab placement of one block in a state arena: field f of block b starts
// at off + f * stride; slabs are (nx+2)(ny+2), ghost 1.
struct BlockDesc {
    int level, nx, ny, pad;
    int64_t off, stride;
};

// One ghost entry to fill, every address resolved to an arena offset:
// field f of the target is dst + f * dst_stride; with n == 0 the value is a
// copy of src[0] + f * stride[0], else the bilinear fold acc + v w over the
// n <= 4 coarse corners src[k] + f * stride[k] with weights w[k], in corner
// order (intergrid.rs:183-223).  For the ops of a tile, dst is the window
// index instead.
struct GhostOp {
    int64_t dst;
    int32_t dst_stride, n;
    int64_t src[4];
    int32_t stride[4];
    double w[4];
};
// One covered coarse cell, arena offsets of field 0: coarse c <- mean of the
// r x r fine children starting at f (row pitch fsy).
struct RestrictOp {
    int64_t c, f;
    int32_t cstride, fstride, fsy, pad;
};
// A run of cells [start, start + count) of one block (row-major interior).
struct Unit {
    int block, start, count, pad;
};
// A rectangle of at most kTile x rows interior cells of one block (rows <=
// kTile, chosen per level), the work item of the fused fill + step
// kernels: [x0, x0 + w) x [y0, y0 + h) in block-interior coordinates of the
// block whose slab of field f starts at off + f * stride.  Its
// (w + 2) x (h + 2) window is staged in shared memory; the window entries
// that are ghosts of the block come from tile_fill[fill0, fill1), whose dst
// is the window index c + r (w + 2).
constexpr int kTile = 32;
struct Tile {
    int64_t off;
    int32_t stride, nx, ny, x0, y0, w, h, fill0, fill1, block;
};

struct Plans {
    std::string error;  // non-empty when the hierarchy is not properly nested
    std::vector<BlockDesc> blocks;
    int64_t arena_elems = 0;
    std::vector<GhostOp> fill;         // all levels, level-major
    std::vector<int64_t> fill_start;   // per level, + end
    std::vector<RestrictOp> restrict_ops;  // per fine level, level-major
    std::vector<int64_t> restrict_start;   // per fine level (index 0 unused), + end
    std::vector<Unit> units;
    std::vector<int64_t> unit_start;       // per level, + end
    std::vector<Tile> tiles;               // level-major
    std::vector<int64_t> tile_start;       // per level, + end
    std::vector<GhostOp> tile_fill;
};

// Ring, tile and unit lists are built for the levels >= first_level only
// (the others' ranges are empty).  Level-0 ghosts come from level 0 alone,
// so a caller may build level 0's lists once (first_level 0 on the base
// layout) and only the refined levels' at each regrid (first_level 1).
// `tile_rows[l]` (default kTile) is the tile height of level l.
Plans build_plans(const Layout& g, int nfields, int unit_cells, int first_level = 0,
                  const std::vector<int>& tile_rows = {});

}  // namespace amr
}  // namespace lg
