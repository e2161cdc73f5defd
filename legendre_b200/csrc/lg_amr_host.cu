// Host algorithms of the 2-D AMR path (see lg_amr_host.h).
#include <algorithm>
#include <cmath>
#include <cstdlib>

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

// every cell of `need` lies in some box of `cover` (amr/grid.rs:293-322)
bool covered(const Box& need, const std::vector<Box>& cover) {
    if (need.cells() == 0) return true;
    for (int64_t y = need.lo[1]; y < need.hi[1]; ++y) {
        int64_t x = need.lo[0];
        while (x < need.hi[0]) {
            const Box* hit = nullptr;
            for (const Box& b : cover)
                if (b.contains(x, y)) {
                    hit = &b;
                    break;
                }
            if (!hit) return false;
            x = hit->hi[0];
        }
    }
    return true;
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
    if (level < 0 || level >= (int)owner.size()) return -1;
    const Box d = domain(level);
    if (!d.contains(x, y)) return -1;
    const uint32_t p = owner[level][(size_t)x + (size_t)y * (size_t)d.hi[0]];
    return p == UINT32_MAX ? -1 : (int)p;
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
    std::vector<Box> coarser;
    for (const Patch& p : g.patches) coarser.push_back(p.bx);
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
            if (!covered(need, coarser)) return "patch not properly nested at level " + std::to_string(level);
        }
        for (const Box& b : boxes) g.patches.push_back(Patch{level, b});
        g.level_start.push_back((uint32_t)g.patches.size());
        coarser = boxes;
    }
    g.level_spacing.push_back({base.spacing[0], base.spacing[1]});
    for (uint32_t r : g.ratios) {
        const auto prev = g.level_spacing.back();
        g.level_spacing.push_back({prev[0] / (double)r, prev[1] / (double)r});
    }
    for (int level = 0; level < g.num_levels(); ++level) {
        const Box d = g.domain(level);
        std::vector<uint32_t> map((size_t)d.hi[0] * (size_t)d.hi[1], UINT32_MAX);
        for (uint32_t p = g.level_start[level]; p < g.level_start[level + 1]; ++p) {
            const Box& b = g.patches[p].bx;
            for (int64_t y = b.lo[1]; y < b.hi[1]; ++y)
                std::fill(map.begin() + (size_t)(b.lo[0] + y * d.hi[0]), map.begin() + (size_t)(b.hi[0] + y * d.hi[0]),
                          p);
        }
        g.owner.push_back(std::move(map));
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

std::vector<std::vector<Box>> propose(const Layout& g, std::vector<std::vector<std::array<int64_t, 2>>>& flags,
                                      const Policy& p) {
    const int capacity = g.max_levels() - 1;
    std::vector<std::vector<Box>> nl(capacity);
    for (int target = capacity; target >= 1; --target) {
        const int src = target - 1;
        std::vector<Cell> f;
        if (src < (int)flags.size()) {
            if (p.buffer > 0) {
                for (const Cell& c : flags[src])
                    for (int64_t y = c[1] - p.buffer; y <= c[1] + p.buffer; ++y)
                        for (int64_t x = c[0] - p.buffer; x <= c[0] + p.buffer; ++x) f.push_back({x, y});
            } else {
                f = flags[src];
            }
        }
        if (target < capacity && !nl[target].empty()) {  // nesting flags (adapt.rs:188-205)
            const int64_t rf = g.ratios[target], rs = g.ratios[target - 1];
            for (const Box& b : nl[target]) {
                const int64_t lo0 = floor_div(b.lo[0] / rf - 1, rs), lo1 = floor_div(b.lo[1] / rf - 1, rs);
                const int64_t hi0 = floor_div(b.hi[0] / rf + 1 + rs - 1, rs), hi1 = floor_div(b.hi[1] / rf + 1 + rs - 1, rs);
                for (int64_t y = lo1; y < hi1; ++y)
                    for (int64_t x = lo0; x < hi0; ++x) f.push_back({x, y});
            }
        }
        const Box dom = g.domain(src);
        f.erase(std::remove_if(f.begin(), f.end(), [&](const Cell& c) { return !dom.contains(c[0], c[1]); }),
                f.end());
        std::sort(f.begin(), f.end());
        f.erase(std::unique(f.begin(), f.end()), f.end());
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
        std::vector<Box> cur;
        for (uint32_t b = g.level_start[l + 1]; b < g.level_start[l + 2]; ++b) cur.push_back(g.patches[b].bx);
        uint64_t pc = 0, cc = 0;
        for (const Box& b : proposed[l]) pc += b.cells();
        for (const Box& b : cur) cc += b.cells();
        if (cc > pc + pc / 2) return false;
        for (const Box& b : proposed[l])
            if (!covered(b, cur)) return false;
    }
    return true;
}

// ------------------------------------------------------------- plans -----
Plans build_plans(const Layout& g, int nfields, int unit_cells) {
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

    // ghost fill (intergrid.rs:267-351, ghost width 1)
    for (int level = 0; level < g.num_levels(); ++level) {
        P.fill_start.push_back((int64_t)P.fill.size());
        const Box dom = g.domain(level);
        for (uint32_t pb = g.level_start[level]; pb < g.level_start[level + 1]; ++pb) {
            const Box& bx = g.patches[pb].bx;
            auto visit = [&](int64_t x, int64_t y) {
                FillOp op{};
                op.tblock = (int)pb;
                op.toff = slab_off((int)pb, x - bx.lo[0], y - bx.lo[1]);
                const int64_t tx = reflect(x, dom.lo[0], dom.hi[0]), ty = reflect(y, dom.lo[1], dom.hi[1]);
                const int src = g.find(level, tx, ty);
                if (src >= 0) {
                    const Box& sb = g.patches[src].bx;
                    op.a = src;
                    op.b = slab_off(src, tx - sb.lo[0], ty - sb.lo[1]);
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
                    const int start = (int)P.corners.size();
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
                        P.corners.push_back(Corner{q, slab_off(q, cc[0] - qb.lo[0], cc[1] - qb.lo[1]), weight});
                    }
                    op.a = start;
                    op.b = -((int)P.corners.size() - start);
                }
                P.fill.push_back(op);
            };
            // ring of width 1 (intergrid.rs:73-86)
            for (int64_t y = bx.lo[1]; y < bx.hi[1]; ++y) visit(bx.lo[0] - 1, y);
            for (int64_t y = bx.lo[1]; y < bx.hi[1]; ++y) visit(bx.hi[0], y);
            for (int64_t x = bx.lo[0] - 1; x < bx.hi[0] + 1; ++x) visit(x, bx.lo[1] - 1);
            for (int64_t x = bx.lo[0] - 1; x < bx.hi[0] + 1; ++x) visit(x, bx.hi[1]);
        }
    }
    P.fill_start.push_back((int64_t)P.fill.size());

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
                        P.restrict_ops.push_back(RestrictOp{(int)cb, slab_off((int)cb, x - cp.lo[0], y - cp.lo[1]),
                                                            (int)fb,
                                                            slab_off((int)fb, x * r - fp.lo[0], y * r - fp.lo[1])});
            }
        }
    }
    P.restrict_start.push_back((int64_t)P.restrict_ops.size());

    // step work units
    for (int level = 0; level < g.num_levels(); ++level) {
        P.unit_start.push_back((int64_t)P.units.size());
        for (uint32_t b = g.level_start[level]; b < g.level_start[level + 1]; ++b) {
            const int cells = P.blocks[b].nx * P.blocks[b].ny;
            for (int s = 0; s < cells; s += unit_cells) P.units.push_back(Unit{(int)b, s, std::min(unit_cells, cells - s), 0});
        }
    }
    P.unit_start.push_back((int64_t)P.units.size());
    return P;
}

// ----------------------------------------------------------- migrate -----
namespace {

double sample(const Layout& g, const std::vector<std::vector<double>>& s, int level, int64_t x, int64_t y) {
    if (level < g.num_levels()) {
        const int b = g.find(level, x, y);
        if (b >= 0) {
            const Box& bx = g.patches[b].bx;
            return s[b][(size_t)((x - bx.lo[0] + 1) + (y - bx.lo[1] + 1) * (bx.extent(0) + 2))];
        }
    }
    const double r = (double)g.ratios[level - 1];
    const Box cd = g.domain(level - 1);
    const int64_t cell[2] = {x, y};
    int64_t c0[2];
    double w[2];
    for (int d = 0; d < 2; ++d) {
        const double pc = ((double)cell[d] + 0.5) / r - 0.5;
        const double fl = std::floor(pc);
        c0[d] = (int64_t)fl;
        w[d] = pc - fl;
    }
    double acc = 0.0;
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
        acc += sample(g, s, level - 1, cc[0], cc[1]) * weight;
    }
    return acc;
}

}  // namespace

void migrate_field(const Layout& og, const std::vector<std::vector<double>>& old, const Layout& ng,
                   std::vector<std::vector<double>>& out) {
    out.assign(ng.num_blocks(), {});
    for (int b = 0; b < ng.num_blocks(); ++b) {
        const Box& bx = ng.patches[b].bx;
        out[b].assign((size_t)(bx.extent(0) + 2) * (size_t)(bx.extent(1) + 2), 0.0);
    }
    for (uint32_t b = ng.level_start[0]; b < ng.level_start[1]; ++b) out[b] = old[b];  // the base tiling never changes
    for (int level = 1; level < ng.num_levels(); ++level)
        for (uint32_t b = ng.level_start[level]; b < ng.level_start[level + 1]; ++b) {
            const Box& bx = ng.patches[b].bx;
            for (int64_t j = 0; j < bx.extent(1); ++j)
                for (int64_t i = 0; i < bx.extent(0); ++i)
                    out[b][(size_t)((i + 1) + (j + 1) * (bx.extent(0) + 2))] =
                        sample(og, old, level, bx.lo[0] + i, bx.lo[1] + j);
        }
}

}  // namespace amr
}  // namespace lg
