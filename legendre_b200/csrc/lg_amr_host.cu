// Host algorithms of the 2-D AMR path (see lg_amr_host.h).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <system_error>

#include "../../include/legendre_b200.h"
#include "lg_amr_host.h"

namespace lg {
namespace amr {

Box Box::clipped(const Box& d) const {
    Box r = *this;
    for (int k = 0; k < 2; ++k) {
        r.lo[k] = std::max(r.lo[k], d.lo[k]);
        r.hi[k] = std::max(std::min(r.hi[k], d.hi[k]), r.lo[k]);
    }
    return r;
}

namespace {

int64_t floor_div(int64_t a, int64_t b) {  // i64::div_euclid for b > 0
    int64_t q = a / b;
    return (a % b < 0) ? q - 1 : q;
}

// reflect_coord (boundary.rs:82-90)
int64_t reflect(int64_t c, int64_t lo, int64_t hi) {
    if (c < lo) return 2 * lo - 1 - c;
    if (c >= hi) return 2 * hi - 1 - c;
    return c;
}

// bucket index of the patches [p0, p1) of one level (see Layout::Index)
Layout::Index build_index(const std::vector<Patch>& patches, uint32_t p0, uint32_t p1, const Box& dom) {
    Layout::Index ix;
    ix.side = 32;
    while ((dom.hi[0] / ix.side + 1) * (dom.hi[1] / ix.side + 1) > (int64_t(1) << 22)) ix.side *= 2;
    ix.nbx = (dom.hi[0] + ix.side - 1) / ix.side;
    ix.nby = (dom.hi[1] + ix.side - 1) / ix.side;
    ix.start.assign((size_t)(ix.nbx * ix.nby + 1), 0);
    for (int pass = 0; pass < 2; ++pass) {
        std::vector<uint32_t> fillpos;
        if (pass == 1) {
            for (size_t k = 1; k < ix.start.size(); ++k) ix.start[k] += ix.start[k - 1];
            ix.items.assign(ix.start.back(), 0);
            fillpos.assign(ix.start.begin(), ix.start.end() - 1);
        }
        for (uint32_t p = p0; p < p1; ++p) {
            const Box& b = patches[p].bx;
            for (int64_t by = b.lo[1] / ix.side; by <= (b.hi[1] - 1) / ix.side; ++by)
                for (int64_t bx = b.lo[0] / ix.side; bx <= (b.hi[0] - 1) / ix.side; ++bx) {
                    const size_t k = (size_t)(bx + by * ix.nbx);
                    if (pass == 0)
                        ix.start[k + 1] += 1;
                    else
                        ix.items[fillpos[k]++] = p;
                }
        }
    }
    return ix;
}

}  // namespace

Box Layout::domain(int level) const {
    int64_t s = 1;
    for (int l = 0; l < level; ++l) s *= ratios[l];
    Box b;
    b.hi[0] = base.cells[0] * s;
    b.hi[1] = base.cells[1] * s;
    return b;
}

int Layout::find(int level, int64_t x, int64_t y) const {
    if (level < 0 || level >= (int)index.size()) return -1;
    const Box d = domain(level);
    if (!d.contains(x, y)) return -1;
    const Index& ix = index[level];
    const size_t k = (size_t)(x / ix.side + (y / ix.side) * ix.nbx);
    for (uint32_t q = ix.start[k]; q < ix.start[k + 1]; ++q)
        if (patches[ix.items[q]].bx.contains(x, y)) return (int)ix.items[q];
    return -1;
}

bool Layout::covers(int level, const Box& need) const {
    if (need.cells() == 0) return true;
    for (int64_t y = need.lo[1]; y < need.hi[1]; ++y) {
        int64_t x = need.lo[0];
        while (x < need.hi[0]) {
            const int p = find(level, x, y);
            if (p < 0) return false;
            x = patches[p].bx.hi[0];
        }
    }
    return true;
}

std::string build_layout(const Base& base, const std::vector<uint32_t>& ratios,
                         const std::vector<std::vector<Box>>& levels, Layout* out) {
    if (levels.size() > ratios.size()) return "more refined levels than refinement ratios";
    for (uint32_t r : ratios)
        if (r < 2) return "refinement ratios must be at least 2";
    for (int d = 0; d < 2; ++d)
        if (base.cells[d] <= 0 || base.block[d] <= 0 || base.cells[d] % base.block[d] != 0)
            return "base cells must be positive multiples of the block size";
    Layout g;
    g.base = base;
    g.ratios = ratios;
    const int64_t nbx = base.cells[0] / base.block[0], nby = base.cells[1] / base.block[1];
    for (int64_t b = 0; b < nbx * nby; ++b) {
        Patch p;
        p.level = 0;
        p.bx.lo[0] = (b % nbx) * base.block[0];
        p.bx.lo[1] = (b / nbx) * base.block[1];
        p.bx.hi[0] = p.bx.lo[0] + base.block[0];
        p.bx.hi[1] = p.bx.lo[1] + base.block[1];
        g.patches.push_back(p);
    }
    g.level_start = {0, (uint32_t)g.patches.size()};
    g.index.push_back(build_index(g.patches, 0, g.level_start[1], g.domain(0)));
    for (size_t l = 0; l < levels.size(); ++l) {
        const int level = (int)l + 1;
        const int64_t r = ratios[l];
        const Box dom = g.domain(level);
        const std::vector<Box>& boxes = levels[l];
        for (size_t i = 0; i < boxes.size(); ++i) {
            const Box& b = boxes[i];
            if (b.cells() == 0) return "empty patch at level " + std::to_string(level);
            if (!(b.clipped(dom) == b)) return "patch outside the domain at level " + std::to_string(level);
            for (int d = 0; d < 2; ++d)
                if (b.lo[d] % r != 0 || b.hi[d] % r != 0)
                    return "patch not aligned to the refinement ratio at level " + std::to_string(level);
            for (size_t k = 0; k < i; ++k)
                if (b.intersects(boxes[k])) return "overlapping patches at level " + std::to_string(level);
            Box need;
            for (int d = 0; d < 2; ++d) {
                need.lo[d] = floor_div(b.lo[d], r) - 1;
                need.hi[d] = floor_div(b.hi[d] + r - 1, r) + 1;
            }
            need = need.clipped(g.domain(level - 1));
            if (!g.covers(level - 1, need)) return "patch not properly nested at level " + std::to_string(level);
        }
        const uint32_t p0 = (uint32_t)g.patches.size();
        for (const Box& b : boxes) g.patches.push_back(Patch{level, b});
        g.level_start.push_back((uint32_t)g.patches.size());
        g.index.push_back(build_index(g.patches, p0, g.level_start.back(), dom));
    }
    g.level_spacing.push_back({base.spacing[0], base.spacing[1]});
    for (uint32_t r : g.ratios) {
        const auto prev = g.level_spacing.back();
        g.level_spacing.push_back({prev[0] / (double)r, prev[1] / (double)r});
    }
    *out = std::move(g);
    return "";
}

// ------------------------------------------------------------ cluster ----
namespace {

using Cell = std::array<int64_t, 2>;

Box bounding(const Cell* c, size_t n) {
    Box b;
    b.lo[0] = b.hi[0] = c[0][0];
    b.lo[1] = b.hi[1] = c[0][1];
    for (size_t i = 1; i < n; ++i)
        for (int d = 0; d < 2; ++d) {
            b.lo[d] = std::min(b.lo[d], c[i][d]);
            b.hi[d] = std::max(b.hi[d], c[i][d]);
        }
    b.hi[0] += 1;
    b.hi[1] += 1;
    return b;
}

// The split plane of one box, in the reference's order of preference:
// the most central interior hole of a signature, else the strongest
// second-difference zero crossing that leaves min_width on both sides,
// else a bisection of the longest axis (cluster.rs:205-268).
bool choose_split(const Box& bx, const std::vector<uint32_t> sig[2], int64_t min_width, int* axis, int64_t* plane) {
    bool hole = false;
    uint64_t best_c = 0;
    for (int d = 0; d < 2; ++d) {
        const size_t n = sig[d].size();
        for (size_t i = 1; i + 1 < n; ++i)
            if (sig[d][i] == 0) {
                const uint64_t c = std::min<uint64_t>(i, n - 1 - i);
                if (!hole || c > best_c) {
                    hole = true;
                    best_c = c;
                    *axis = d;
                    *plane = bx.lo[d] + (int64_t)i;
                }
            }
    }
    if (hole) return true;
    bool infl = false;
    int64_t best_s = 0;
    best_c = 0;
    for (int d = 0; d < 2; ++d) {
        const std::vector<uint32_t>& s = sig[d];
        const size_t n = s.size();
        if (n < 4) continue;
        for (size_t i = 1; i < n - 2; ++i) {
            const int64_t a = (int64_t)s[i + 1] - 2 * (int64_t)s[i] + (int64_t)s[i - 1];
            const int64_t b = (int64_t)s[i + 2] - 2 * (int64_t)s[i + 1] + (int64_t)s[i];
            if (a * b >= 0) continue;
            const size_t pl = i + 1;
            if ((int64_t)pl < min_width || (int64_t)(n - pl) < min_width) continue;
            const int64_t strength = std::llabs(b - a);
            const uint64_t c = std::min<uint64_t>(pl, n - pl);
            if (!infl || strength > best_s || (strength == best_s && c > best_c)) {
                infl = true;
                best_s = strength;
                best_c = c;
                *axis = d;
                *plane = bx.lo[d] + (int64_t)pl;
            }
        }
    }
    if (infl) return true;
    const int d = bx.extent(1) >= bx.extent(0) ? 1 : 0;  // longest axis, the later one on ties
    if (bx.extent(d) < 2 * min_width) return false;
    *axis = d;
    *plane = bx.lo[d] + bx.extent(d) / 2;
    return true;
}

void split(Cell* f, size_t n, double eff, int64_t min_width, std::vector<Box>& out) {
    const Box bx = bounding(f, n);
    if ((double)n / (double)bx.cells() >= eff) {
        out.push_back(bx);
        return;
    }
    std::vector<uint32_t> sig[2] = {std::vector<uint32_t>(bx.extent(0), 0), std::vector<uint32_t>(bx.extent(1), 0)};
    for (size_t i = 0; i < n; ++i) {
        sig[0][f[i][0] - bx.lo[0]] += 1;
        sig[1][f[i][1] - bx.lo[1]] += 1;
    }
    int axis = 0;
    int64_t plane = 0;
    if (!choose_split(bx, sig, min_width, &axis, &plane)) {
        out.push_back(bx);
        return;
    }
    size_t lt = 0;  // two-pointer partition (cluster.rs:272-281)
    for (size_t j = 0; j < n; ++j)
        if (f[j][axis] < plane) std::swap(f[lt++], f[j]);
    split(f, lt, eff, min_width, out);
    split(f + lt, n - lt, eff, min_width, out);
}

}  // namespace

std::vector<Box> cluster(std::vector<std::array<int64_t, 2>>& flags, double efficiency, int64_t min_width) {
    std::vector<Box> out;
    if (!flags.empty()) split(flags.data(), flags.size(), efficiency, min_width, out);
    return out;
}

// The cells of the union of `boxes` inside `dom`, sorted (x, then y) and
// without duplicates (adapt.rs:208-210): a bitmap over the boxes' bounding
// box, scanned x-major, or packed 64-bit keys sorted when that box is huge.
static std::vector<std::array<int64_t, 2>> union_cells(const std::vector<Box>& boxes, const Box& dom) {
    std::vector<std::array<int64_t, 2>> out;
    Box bb;
    bool any = false;
    for (const Box& b0 : boxes) {
        const Box b = b0.clipped(dom);
        if (b.cells() == 0) continue;
        if (!any) {
            bb = b;
            any = true;
            continue;
        }
        for (int d = 0; d < 2; ++d) {
            bb.lo[d] = std::min(bb.lo[d], b.lo[d]);
            bb.hi[d] = std::max(bb.hi[d], b.hi[d]);
        }
    }
    if (!any) return out;
    const int64_t w = bb.extent(0), h = bb.extent(1);
    if ((uint64_t)w * (uint64_t)h <= (uint64_t(1) << 27)) {
        std::vector<uint8_t> bits((size_t)(w * h), 0);  // x-major
        for (const Box& b0 : boxes) {
            const Box b = b0.clipped(dom);
            if (b.cells() == 0) continue;
            for (int64_t x = b.lo[0]; x < b.hi[0]; ++x)
                std::fill_n(bits.begin() + (size_t)((x - bb.lo[0]) * h + (b.lo[1] - bb.lo[1])), (size_t)b.extent(1),
                            uint8_t(1));
        }
        for (int64_t x = 0; x < w; ++x)
            for (int64_t y = 0; y < h; ++y)
                if (bits[(size_t)(x * h + y)]) out.push_back({bb.lo[0] + x, bb.lo[1] + y});
        return out;
    }
    std::vector<uint64_t> keys;  // cells of a level domain: non-negative, below 2^31
    for (const Box& b0 : boxes) {
        const Box b = b0.clipped(dom);
        for (int64_t x = b.lo[0]; x < b.hi[0]; ++x)
            for (int64_t y = b.lo[1]; y < b.hi[1]; ++y) keys.push_back(((uint64_t)x << 32) | (uint64_t)y);
    }
    std::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    out.resize(keys.size());
    for (size_t k = 0; k < keys.size(); ++k) out[k] = {(int64_t)(keys[k] >> 32), (int64_t)(keys[k] & 0xffffffffu)};
    return out;
}

std::vector<std::vector<Box>> propose(const Layout& g, std::vector<std::vector<std::array<int64_t, 2>>>& flags,
                                      const Policy& p) {
    const int capacity = g.max_levels() - 1;
    std::vector<std::vector<Box>> nl(capacity);
    for (int target = capacity; target >= 1; --target) {
        const int src = target - 1;
        std::vector<Box> parts;  // dilated tags and nesting boxes
        if (src < (int)flags.size()) {
            const int64_t bf = std::max<int64_t>(p.buffer, 0);
            for (const Cell& c : flags[src]) {
                Box b;
                b.lo[0] = c[0] - bf;
                b.lo[1] = c[1] - bf;
                b.hi[0] = c[0] + bf + 1;
                b.hi[1] = c[1] + bf + 1;
                parts.push_back(b);
            }
        }
        if (target < capacity && !nl[target].empty()) {  // nesting flags (adapt.rs:188-205)
            const int64_t rf = g.ratios[target], rs = g.ratios[target - 1];
            for (const Box& b : nl[target]) {
                Box n;
                n.lo[0] = floor_div(b.lo[0] / rf - 1, rs);
                n.lo[1] = floor_div(b.lo[1] / rf - 1, rs);
                n.hi[0] = floor_div(b.hi[0] / rf + 1 + rs - 1, rs);
                n.hi[1] = floor_div(b.hi[1] / rf + 1 + rs - 1, rs);
                parts.push_back(n);
            }
        }
        std::vector<Cell> f = union_cells(parts, g.domain(src));
        if (f.empty()) continue;
        const int64_t r = g.ratios[target - 1];
        for (Box b : cluster(f, p.efficiency, p.min_width)) {
            for (int d = 0; d < 2; ++d) {
                b.lo[d] *= r;
                b.hi[d] *= r;
            }
            nl[target - 1].push_back(b);
        }
    }
    while (!nl.empty() && nl.back().empty()) nl.pop_back();
    return nl;
}

bool acceptable(const Layout& g, const std::vector<std::vector<Box>>& proposed) {
    if ((int)proposed.size() != g.num_levels() - 1) return false;
    for (size_t l = 0; l < proposed.size(); ++l) {
        uint64_t pc = 0, cc = 0;
        for (const Box& b : proposed[l]) pc += b.cells();
        for (uint32_t b = g.level_start[l + 1]; b < g.level_start[l + 2]; ++b) cc += g.patches[b].bx.cells();
        if (cc > pc + pc / 2) return false;
        for (const Box& b : proposed[l])
            if (!g.covers((int)l + 1, b)) return false;
    }
    return true;
}

// ------------------------------------------------------------- plans -----
Plans build_plans(const Layout& g, int nfields, int unit_cells, int first_level, const std::vector<int>& tile_rows) {
    Plans P;
    int64_t off = 0;
    for (const Patch& p : g.patches) {
        BlockDesc d{};
        d.level = p.level;
        d.nx = (int)p.bx.extent(0);
        d.ny = (int)p.bx.extent(1);
        d.off = off;
        const int64_t len = (int64_t)(d.nx + 2) * (d.ny + 2);
        d.stride = (len + 31) / 32 * 32;
        off += d.stride * nfields;
        P.blocks.push_back(d);
    }
    P.arena_elems = off;
    auto slab_off = [&](int b, int64_t i, int64_t j) { return (int)((i + 1) + (j + 1) * (P.blocks[b].nx + 2)); };

    // ghost fill (intergrid.rs:267-351, ghost width 1), and the tiles of
    // every block with the ring entries their windows need
    for (int level = 0; level < g.num_levels(); ++level) {
        P.fill_start.push_back((int64_t)P.fill.size());
        P.tile_start.push_back((int64_t)P.tiles.size());
        if (level < first_level) continue;
        const Box dom = g.domain(level);
        for (uint32_t pb = g.level_start[level]; pb < g.level_start[level + 1]; ++pb) {
            const Box& bx = g.patches[pb].bx;
            const size_t ring0 = P.fill.size();
            auto visit = [&](int64_t x, int64_t y) {
                GhostOp op{};
                op.dst = P.blocks[pb].off + slab_off((int)pb, x - bx.lo[0], y - bx.lo[1]);
                op.dst_stride = (int32_t)P.blocks[pb].stride;
                const int64_t tx = reflect(x, dom.lo[0], dom.hi[0]), ty = reflect(y, dom.lo[1], dom.hi[1]);
                const int src = g.find(level, tx, ty);
                if (src >= 0) {
                    const Box& sb = g.patches[src].bx;
                    op.n = 0;
                    op.src[0] = P.blocks[src].off + slab_off(src, tx - sb.lo[0], ty - sb.lo[1]);
                    op.stride[0] = (int32_t)P.blocks[src].stride;
                } else {
                    const double r = (double)g.ratios[level - 1];
                    const Box cd = g.domain(level - 1);
                    const int64_t cell[2] = {tx, ty};
                    int64_t c0[2];
                    double w[2];
                    for (int d = 0; d < 2; ++d) {
                        const double pc = ((double)cell[d] + 0.5) / r - 0.5;
                        const double fl = std::floor(pc);
                        c0[d] = (int64_t)fl;
                        w[d] = pc - fl;
                    }
                    op.n = 0;
                    for (unsigned corner = 0; corner < 4; ++corner) {
                        int64_t cc[2] = {c0[0], c0[1]};
                        double weight = 1.0;
                        for (int d = 0; d < 2; ++d) {
                            if ((corner >> d) & 1) {
                                cc[d] += 1;
                                weight *= w[d];
                            } else {
                                weight *= 1.0 - w[d];
                            }
                        }
                        if (weight == 0.0) continue;
                        for (int d = 0; d < 2; ++d) cc[d] = reflect(cc[d], cd.lo[d], cd.hi[d]);
                        const int q = g.find(level - 1, cc[0], cc[1]);
                        if (q < 0) {  // the reference panics: proper nesting guarantees a donor
                            P.error = "no coarse donor for prolongation at level " + std::to_string(level);
                            continue;
                        }
                        const Box& qb = g.patches[q].bx;
                        op.src[op.n] = P.blocks[q].off + slab_off(q, cc[0] - qb.lo[0], cc[1] - qb.lo[1]);
                        op.stride[op.n] = (int32_t)P.blocks[q].stride;
                        op.w[op.n] = weight;
                        op.n += 1;
                    }
                }
                P.fill.push_back(op);
            };
            // ring of width 1 (intergrid.rs:73-86)
            for (int64_t y = bx.lo[1]; y < bx.hi[1]; ++y) visit(bx.lo[0] - 1, y);
            for (int64_t y = bx.lo[1]; y < bx.hi[1]; ++y) visit(bx.hi[0], y);
            for (int64_t x = bx.lo[0] - 1; x < bx.hi[0] + 1; ++x) visit(x, bx.lo[1] - 1);
            for (int64_t x = bx.lo[0] - 1; x < bx.hi[0] + 1; ++x) visit(x, bx.hi[1]);
            const int nx = (int)bx.extent(0), ny = (int)bx.extent(1);
            const int th = level < (int)tile_rows.size() ? std::max(1, std::min(kTile, tile_rows[level])) : kTile;
            for (int y0 = 0; y0 < ny; y0 += th)
                for (int x0 = 0; x0 < nx; x0 += kTile) {
                    Tile t{};
                    t.block = (int)pb;
                    t.off = P.blocks[pb].off;
                    t.stride = (int32_t)P.blocks[pb].stride;
                    t.nx = nx;
                    t.ny = ny;
                    t.x0 = x0;
                    t.y0 = y0;
                    t.w = std::min(kTile, nx - x0);
                    t.h = std::min(th, ny - y0);
                    t.fill0 = (int)P.tile_fill.size();
                    for (size_t k = ring0; k < P.fill.size(); ++k) {
                        const int toff = (int)(P.fill[k].dst - P.blocks[pb].off);
                        const int i = toff % (nx + 2) - 1, j = toff / (nx + 2) - 1;
                        const int c = i - (x0 - 1), r = j - (y0 - 1);
                        if (c < 0 || c > t.w + 1 || r < 0 || r > t.h + 1) continue;
                        GhostOp op = P.fill[k];
                        op.dst = c + r * (t.w + 2);
                        P.tile_fill.push_back(op);
                    }
                    t.fill1 = (int)P.tile_fill.size();
                    P.tiles.push_back(t);
                }
        }
    }
    P.fill_start.push_back((int64_t)P.fill.size());
    P.tile_start.push_back((int64_t)P.tiles.size());

    // restriction (intergrid.rs:110-150)
    P.restrict_start.push_back(0);
    for (int fine = 1; fine < g.num_levels(); ++fine) {
        P.restrict_start.push_back((int64_t)P.restrict_ops.size());
        const int64_t r = g.ratios[fine - 1];
        for (uint32_t fb = g.level_start[fine]; fb < g.level_start[fine + 1]; ++fb) {
            const Box& fp = g.patches[fb].bx;
            Box cov;
            for (int d = 0; d < 2; ++d) {
                cov.lo[d] = fp.lo[d] / r;
                cov.hi[d] = fp.hi[d] / r;
            }
            for (uint32_t cb = g.level_start[fine - 1]; cb < g.level_start[fine]; ++cb) {
                const Box& cp = g.patches[cb].bx;
                const Box ov = cov.clipped(cp);
                if (ov.cells() == 0) continue;
                for (int64_t y = ov.lo[1]; y < ov.hi[1]; ++y)
                    for (int64_t x = ov.lo[0]; x < ov.hi[0]; ++x)
                        P.restrict_ops.push_back(
                            RestrictOp{P.blocks[cb].off + slab_off((int)cb, x - cp.lo[0], y - cp.lo[1]),
                                       P.blocks[fb].off + slab_off((int)fb, x * r - fp.lo[0], y * r - fp.lo[1]),
                                       (int32_t)P.blocks[cb].stride, (int32_t)P.blocks[fb].stride,
                                       P.blocks[fb].nx + 2, 0});
            }
        }
    }
    P.restrict_start.push_back((int64_t)P.restrict_ops.size());

    // step work units
    for (int level = 0; level < g.num_levels(); ++level) {
        P.unit_start.push_back((int64_t)P.units.size());
        if (level < first_level) continue;
        for (uint32_t b = g.level_start[level]; b < g.level_start[level + 1]; ++b) {
            const int cells = P.blocks[b].nx * P.blocks[b].ny;
            for (int s = 0; s < cells; s += unit_cells) P.units.push_back(Unit{(int)b, s, std::min(unit_cells, cells - s), 0});
        }
    }
    P.unit_start.push_back((int64_t)P.units.size());
    return P;
}

}  // namespace amr
}  // namespace lg

extern "C" int lg_amr_cluster(const int64_t* flags, int64_t nflags, double efficiency, int64_t min_width,
                              int64_t* boxes, int64_t cap, int64_t* nboxes) {
    if (!nboxes || nflags < 0 || (nflags > 0 && !flags) || cap < 0 || (cap > 0 && !boxes) ||
        !(efficiency > 0.0 && efficiency <= 1.0) || min_width < 1)
        return LG_ERR_INVALID;  // the reference's debug_asserts (cluster.rs:145-149)
    try {
        std::vector<std::array<int64_t, 2>> f((size_t)nflags);
        for (int64_t i = 0; i < nflags; ++i) f[(size_t)i] = {flags[2 * i], flags[2 * i + 1]};
        const std::vector<lg::amr::Box> out = lg::amr::cluster(f, efficiency, min_width);
        *nboxes = (int64_t)out.size();
        for (int64_t k = 0; k < std::min<int64_t>(cap, (int64_t)out.size()); ++k) {
            const lg::amr::Box& b = out[(size_t)k];
            boxes[4 * k + 0] = b.lo[0];
            boxes[4 * k + 1] = b.lo[1];
            boxes[4 * k + 2] = b.hi[0];
            boxes[4 * k + 3] = b.hi[1];
        }
    } catch (const std::bad_alloc&) {
        return LG_ERR_NOMEM;
    }
    return LG_OK;
}

extern "C" int lg_amr_check_hierarchy(const int64_t* cells, const int64_t* block, const uint32_t* ratios, int nratios,
                                      const int64_t* patches, int64_t npatches, char* err, int64_t errlen) {
    auto put = [&](const std::string& m) {
        if (!err || errlen < 1) return;
        const size_t n = std::min<size_t>(m.size(), (size_t)(errlen - 1));
        std::copy(m.begin(), m.begin() + (std::ptrdiff_t)n, err);
        err[n] = '\0';
    };
    if (!cells || !block || nratios < 0 || (nratios > 0 && !ratios) || npatches < 0 || (npatches > 0 && !patches)) {
        put("null argument");
        return LG_ERR_INVALID;
    }
    try {
        lg::amr::Base base{};
        for (int d = 0; d < 2; ++d) {
            base.cells[d] = cells[d];
            base.block[d] = block[d];
            base.spacing[d] = 1.0;
        }
        const std::vector<uint32_t> r(ratios, ratios + nratios);
        std::vector<std::vector<lg::amr::Box>> levels;
        for (int64_t i = 0; i < npatches; ++i) {
            const int64_t lv = patches[5 * i];
            if (lv < 1 || lv > nratios) {
                put("patch level out of range");
                return LG_ERR_INVALID;
            }
            if ((int64_t)levels.size() < lv) levels.resize((size_t)lv);
            lg::amr::Box b;
            b.lo[0] = patches[5 * i + 1];
            b.lo[1] = patches[5 * i + 2];
            b.hi[0] = patches[5 * i + 3];
            b.hi[1] = patches[5 * i + 4];
            levels[(size_t)(lv - 1)].push_back(b);
        }
        lg::amr::Layout g;
        const std::string m = lg::amr::build_layout(base, r, levels, &g);
        put(m);
        return m.empty() ? LG_OK : LG_ERR_INVALID;
    } catch (const std::bad_alloc&) {
        put("out of memory");
        return LG_ERR_NOMEM;
    }
}
