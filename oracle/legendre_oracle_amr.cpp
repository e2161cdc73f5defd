// legendre oracle, AMR part -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
//
// CPU restatement of the reference's 2-D adaptive path: Berger-Rigoutsos
// clustering (src/geometry/amr/cluster.rs), the AmrGrid patch hierarchy
// (amr/grid.rs), intergrid transfers (amr/intergrid.rs), the Berger-Oliger
// regrid policy with migration (amr/adapt.rs) and the subcycling integrator
// (src/integrators/subcycling.rs), driving Model C (phasefield.rs) or the
// heat model of the reference's AMR tests (tests/amr.rs:297-345).  Same
// arithmetic rules as oracle_core.hpp.
#include <array>
#include <memory>
#include <string>

#include "oracle_core.hpp"

namespace {

using namespace orc;

// ---------------------------------------------------------- CellBox -------
// amr/cluster.rs:27-113 (D <= 3)
struct CellBox {
    int D = 2;
    int64_t lo[3] = {0, 0, 0}, hi[3] = {1, 1, 1};

    uint64_t extent(int d) const { return (uint64_t)(hi[d] - lo[d]); }
    uint64_t cells() const {
        uint64_t acc = 1;
        for (int d = 0; d < D; ++d) {
            uint64_t e = extent(d);
            acc = (e != 0 && acc > UINT64_MAX / e) ? UINT64_MAX : acc * e;
        }
        return acc;
    }
    bool contains(const int64_t* c) const {
        for (int d = 0; d < D; ++d)
            if (!(lo[d] <= c[d] && c[d] < hi[d])) return false;
        return true;
    }
    bool intersects(const CellBox& o) const {
        for (int d = 0; d < D; ++d)
            if (!(lo[d] < o.hi[d] && o.lo[d] < hi[d])) return false;
        return true;
    }
    CellBox grown(int64_t b) const {
        CellBox r = *this;
        for (int d = 0; d < D; ++d) {
            r.lo[d] -= b;
            r.hi[d] += b;
        }
        return r;
    }
    CellBox clipped(const CellBox& dom) const {
        CellBox r = *this;
        for (int d = 0; d < D; ++d) {
            r.lo[d] = std::max(r.lo[d], dom.lo[d]);
            r.hi[d] = std::max(std::min(r.hi[d], dom.hi[d]), r.lo[d]);
        }
        return r;
    }
    bool operator==(const CellBox& o) const {
        for (int d = 0; d < D; ++d)
            if (lo[d] != o.lo[d] || hi[d] != o.hi[d]) return false;
        return true;
    }
};

using Cell = std::array<int64_t, 3>;

CellBox bounding(int D, const Cell* c, size_t n) {
    CellBox b;
    b.D = D;
    for (int d = 0; d < D; ++d) b.lo[d] = b.hi[d] = c[0][d];
    for (size_t i = 0; i < n; ++i)
        for (int d = 0; d < D; ++d) {
            b.lo[d] = std::min(b.lo[d], c[i][d]);
            b.hi[d] = std::max(b.hi[d], c[i][d]);
        }
    for (int d = 0; d < D; ++d) b.hi[d] += 1;
    return b;
}

struct ClusterParams {
    double efficiency;
    int64_t min_width;
};

// cluster.rs:205-220
bool find_hole(const CellBox& bx, const std::vector<std::vector<uint32_t>>& sigs, int* axis, int64_t* plane) {
    bool found = false;
    uint64_t best_c = 0;
    for (int d = 0; d < bx.D; ++d) {
        const size_t n = sigs[d].size();
        for (size_t i = 1; i + 1 < n; ++i) {
            if (sigs[d][i] == 0) {
                uint64_t c = std::min<uint64_t>(i, n - 1 - i);
                if (!found || c > best_c) {
                    found = true;
                    best_c = c;
                    *axis = d;
                    *plane = bx.lo[d] + (int64_t)i;
                }
            }
        }
    }
    return found;
}

// cluster.rs:224-258
bool find_inflection(const CellBox& bx, const std::vector<std::vector<uint32_t>>& sigs, int64_t min_width, int* axis,
                     int64_t* plane) {
    bool found = false;
    int64_t best_s = 0;
    uint64_t best_c = 0;
    for (int d = 0; d < bx.D; ++d) {
        const auto& sig = sigs[d];
        const size_t n = sig.size();
        if (n < 4) continue;
        auto delta = [&](size_t i) -> int64_t {
            return (int64_t)sig[i + 1] - 2 * (int64_t)sig[i] + (int64_t)sig[i - 1];
        };
        for (size_t i = 1; i < n - 2; ++i) {
            int64_t a = delta(i), b = delta(i + 1);
            if (a * b < 0) {
                size_t pl = i + 1;
                if ((int64_t)pl < min_width || (int64_t)(n - pl) < min_width) continue;
                int64_t strength = std::llabs(b - a);
                uint64_t centrality = std::min<uint64_t>(pl, n - pl);
                bool better = !found || strength > best_s || (strength == best_s && centrality > best_c);
                if (better) {
                    found = true;
                    best_s = strength;
                    best_c = centrality;
                    *axis = d;
                    *plane = bx.lo[d] + (int64_t)pl;
                }
            }
        }
    }
    return found;
}

// cluster.rs:262-268 ; max_by_key returns the LAST maximum on ties
bool bisection(const CellBox& bx, int64_t min_width, int* axis, int64_t* plane) {
    int d = 0;
    for (int e = 1; e < bx.D; ++e)
        if (bx.extent(e) >= bx.extent(d)) d = e;
    if (bx.extent(d) < 2 * (uint64_t)min_width) return false;
    *axis = d;
    *plane = bx.lo[d] + (int64_t)(bx.extent(d) / 2);
    return true;
}

// cluster.rs:272-281
size_t partition_in_place(Cell* cells, size_t n, int axis, int64_t plane) {
    size_t lt = 0;
    for (size_t j = 0; j < n; ++j)
        if (cells[j][axis] < plane) {
            std::swap(cells[lt], cells[j]);
            ++lt;
        }
    return lt;
}

// cluster.rs:157-188
void split_or_accept(int D, Cell* flags, size_t n, const ClusterParams& p, std::vector<CellBox>& out) {
    CellBox bx = bounding(D, flags, n);
    double eff = (double)n / (double)bx.cells();
    if (eff >= p.efficiency) {
        out.push_back(bx);
        return;
    }
    std::vector<std::vector<uint32_t>> sigs(D);
    for (int d = 0; d < D; ++d) sigs[d].assign(bx.extent(d), 0);
    for (size_t i = 0; i < n; ++i)
        for (int d = 0; d < D; ++d) sigs[d][flags[i][d] - bx.lo[d]] += 1;
    int axis = 0;
    int64_t plane = 0;
    bool ok = find_hole(bx, sigs, &axis, &plane) || find_inflection(bx, sigs, p.min_width, &axis, &plane) ||
              bisection(bx, p.min_width, &axis, &plane);
    if (!ok) {
        out.push_back(bx);
        return;
    }
    size_t mid = partition_in_place(flags, n, axis, plane);
    split_or_accept(D, flags, mid, p, out);
    split_or_accept(D, flags + mid, n - mid, p, out);
}

std::vector<CellBox> cluster(int D, std::vector<Cell>& flags, const ClusterParams& p) {
    std::vector<CellBox> out;
    if (!flags.empty()) split_or_accept(D, flags.data(), flags.size(), p, out);
    return out;
}

// ---------------------------------------------------------- AmrGrid -------
struct Patch {
    int level;
    CellBox bx;
};

struct Base {
    int64_t cells[2], block[2], nb[2];
    double origin[2], spacing[2];
};

// amr/grid.rs:55-279 (2-D)
struct AmrGrid {
    Base base;
    std::vector<uint32_t> ratios;
    std::vector<Patch> patches;
    std::vector<std::array<double, 2>> level_spacing;
    std::vector<uint32_t> level_start;
    std::vector<std::vector<uint32_t>> lookup;

    int num_levels() const { return (int)level_start.size() - 1; }
    int max_levels() const { return (int)ratios.size() + 1; }
    int64_t num_blocks() const { return (int64_t)patches.size(); }
    CellBox level_domain(int level) const {
        int64_t scale = 1;
        for (int l = 0; l < level; ++l) scale *= ratios[l];
        CellBox b;
        b.D = 2;
        for (int d = 0; d < 2; ++d) {
            b.lo[d] = 0;
            b.hi[d] = base.cells[d] * scale;
        }
        return b;
    }
    std::pair<uint32_t, uint32_t> blocks_at(int level) const {
        if (level + 1 < (int)level_start.size()) return {level_start[level], level_start[level + 1]};
        return {0, 0};
    }
    int64_t find_patch(int level, const int64_t* c) const {
        if (level < 0 || level >= (int)lookup.size()) return -1;
        CellBox dom = level_domain(level);
        if (!dom.contains(c)) return -1;
        uint32_t pid = lookup[level][(size_t)c[0] + (size_t)c[1] * (size_t)dom.hi[0]];
        return pid == UINT32_MAX ? -1 : (int64_t)pid;
    }
    Ext ext(int64_t b) const {
        Ext e;
        e.D = 2;
        e.n[0] = (int64_t)patches[b].bx.extent(0);
        e.n[1] = (int64_t)patches[b].bx.extent(1);
        return e;
    }
    const double* spacing(int64_t b) const { return level_spacing[patches[b].level].data(); }
    void cell_center(int64_t b, const int64_t* idx, double* out) const {
        const Patch& p = patches[b];
        const double* h = level_spacing[p.level].data();
        for (int d = 0; d < 2; ++d) out[d] = std::fma((double)(p.bx.lo[d] + idx[d]) + 0.5, h[d], base.origin[d]);
    }
};

// amr/grid.rs:293-322
bool covered_by(const CellBox& need, const std::vector<CellBox>& cover) {
    if (need.cells() == 0) return true;
    int64_t idx[3] = {need.lo[0], need.lo[1], 0};
    for (;;) {
        const CellBox* hit = nullptr;
        for (const auto& b : cover)
            if (b.contains(idx)) {
                hit = &b;
                break;
            }
        if (!hit) return false;
        idx[0] = hit->hi[0] - 1;
        int d = 0;
        for (;;) {
            idx[d] += 1;
            if (idx[d] < need.hi[d]) break;
            idx[d] = need.lo[d];
            if (++d == 2) return true;
        }
    }
}

// i64::div_euclid for a positive divisor
inline int64_t div_euclid(int64_t a, int64_t b) {
    int64_t q = a / b;
    if (a % b < 0) q -= 1;
    return q;
}

enum AmrErr { AMR_OK = 0, AMR_RATIO = 1, AMR_EMPTY = 2, AMR_NOT_NESTED = 3, AMR_MISALIGNED = 4, AMR_OVERLAP = 5 };

// AmrGrid::from_patches (amr/grid.rs:90-196)
int from_patches(const Base& base, const std::vector<uint32_t>& ratios, const std::vector<std::vector<CellBox>>& levels,
                 AmrGrid* out) {
    if (levels.size() > ratios.size()) return AMR_RATIO;
    for (uint32_t r : ratios)
        if (r < 2) return AMR_RATIO;
    AmrGrid g;
    g.base = base;
    g.ratios = ratios;
    for (int64_t b = 0; b < base.nb[0] * base.nb[1]; ++b) {
        int64_t c0 = b % base.nb[0], c1 = b / base.nb[0];
        Patch p;
        p.level = 0;
        p.bx.D = 2;
        p.bx.lo[0] = c0 * base.block[0];
        p.bx.hi[0] = (c0 + 1) * base.block[0];
        p.bx.lo[1] = c1 * base.block[1];
        p.bx.hi[1] = (c1 + 1) * base.block[1];
        g.patches.push_back(p);
    }
    g.level_start = {0, (uint32_t)g.patches.size()};
    std::vector<CellBox> coarser;
    for (const auto& p : g.patches) coarser.push_back(p.bx);
    for (size_t l = 0; l < levels.size(); ++l) {
        const int level = (int)l + 1;
        const int64_t r = ratios[l];
        const CellBox domain = g.level_domain(level);
        const auto& boxes = levels[l];
        for (size_t i = 0; i < boxes.size(); ++i) {
            const CellBox& bx = boxes[i];
            if (bx.cells() == 0) return AMR_EMPTY;
            if (!(bx.clipped(domain) == bx)) return AMR_NOT_NESTED;
            for (int d = 0; d < 2; ++d)
                if (bx.lo[d] % r != 0 || bx.hi[d] % r != 0) return AMR_MISALIGNED;
            for (size_t k = 0; k < i; ++k)
                if (bx.intersects(boxes[k])) return AMR_OVERLAP;
            CellBox coarse;
            coarse.D = 2;
            for (int d = 0; d < 2; ++d) {
                coarse.lo[d] = div_euclid(bx.lo[d], r);
                coarse.hi[d] = div_euclid(bx.hi[d] + r - 1, r);
            }
            CellBox need = coarse.grown(1).clipped(g.level_domain(level - 1));
            if (!covered_by(need, coarser)) return AMR_NOT_NESTED;
        }
        for (const auto& bx : boxes) g.patches.push_back(Patch{level, bx});
        g.level_start.push_back((uint32_t)g.patches.size());
        coarser = boxes;
    }
    g.level_spacing.push_back({base.spacing[0], base.spacing[1]});
    for (uint32_t r : g.ratios) {
        auto prev = g.level_spacing.back();
        g.level_spacing.push_back({prev[0] / (double)r, prev[1] / (double)r});
    }
    for (int level = 0; level < g.num_levels(); ++level) {
        CellBox dom = g.level_domain(level);
        std::vector<uint32_t> map((size_t)dom.hi[0] * (size_t)dom.hi[1], UINT32_MAX);
        for (uint32_t pid = g.level_start[level]; pid < g.level_start[level + 1]; ++pid) {
            const CellBox& bx = g.patches[pid].bx;
            for (int64_t y = bx.lo[1]; y < bx.hi[1]; ++y)
                for (int64_t x = bx.lo[0]; x < bx.hi[0]; ++x) map[(size_t)x + (size_t)y * (size_t)dom.hi[0]] = pid;
        }
        g.lookup.push_back(std::move(map));
    }
    *out = std::move(g);
    return AMR_OK;
}

// --------------------------------------------------------- AMR state ------
struct AmrState {
    std::vector<int> ghost;
    std::vector<std::vector<std::vector<double>>> slab;  // [block][field]
};

AmrState make_amr_state(const AmrGrid& g, const std::vector<int>& ghosts) {
    AmrState s;
    s.ghost = ghosts;
    s.slab.resize(g.num_blocks());
    for (int64_t b = 0; b < g.num_blocks(); ++b) {
        s.slab[b].resize(ghosts.size());
        for (size_t f = 0; f < ghosts.size(); ++f) s.slab[b][f].assign(g.ext(b).len(ghosts[f]), 0.0);
    }
    return s;
}

// boundary.rs:82-90
inline int64_t reflect_coord(int64_t c, int64_t lo, int64_t hi) {
    if (c < lo) return 2 * lo - 1 - c;
    if (c >= hi) return 2 * hi - 1 - c;
    return c;
}

double get(const AmrGrid& g, const AmrState& s, int64_t b, int f, int64_t i, int64_t j) {
    const Ext e = g.ext(b);
    const int gh = s.ghost[f];
    int64_t idx[2] = {i, j};
    return s.slab[b][f][e.lin(idx, gh)];
}

// intergrid.rs:110-150
void restrict_level(const AmrGrid& g, AmrState& s, int f, int fine_level) {
    const int gh = s.ghost[f];
    const int64_t r = g.ratios[fine_level - 1];
    const double inv = 1.0 / ((double)r * (double)r);
    auto fr = g.blocks_at(fine_level);
    auto cr = g.blocks_at(fine_level - 1);
    for (uint32_t fb = fr.first; fb < fr.second; ++fb) {
        const Patch fp = g.patches[fb];
        CellBox covered;
        covered.D = 2;
        for (int d = 0; d < 2; ++d) {
            covered.lo[d] = fp.bx.lo[d] / r;
            covered.hi[d] = fp.bx.hi[d] / r;
        }
        for (uint32_t cb = cr.first; cb < cr.second; ++cb) {
            const Patch cp = g.patches[cb];
            CellBox ov = covered.clipped(cp.bx);
            if (ov.cells() == 0) continue;
            const Ext ce = g.ext(cb), fe = g.ext(fb);
            for (int64_t cy = ov.lo[1]; cy < ov.hi[1]; ++cy)
                for (int64_t cx = ov.lo[0]; cx < ov.hi[0]; ++cx) {
                    double sum = 0.0;
                    for (int64_t ky = cy * r - fp.bx.lo[1]; ky < (cy + 1) * r - fp.bx.lo[1]; ++ky)
                        for (int64_t kx = cx * r - fp.bx.lo[0]; kx < (cx + 1) * r - fp.bx.lo[0]; ++kx) {
                            int64_t ki[2] = {kx, ky};
                            sum += s.slab[fb][f][fe.lin(ki, gh)];
                        }
                    int64_t li[2] = {cx - cp.bx.lo[0], cy - cp.bx.lo[1]};
                    s.slab[cb][f][ce.lin(li, gh)] = sum * inv;
                }
        }
    }
}

// intergrid.rs:97-105
void restrict_all(const AmrGrid& g, AmrState& s, int f) {
    for (int fl = g.num_levels() - 1; fl >= 1; --fl) restrict_level(g, s, f, fl);
}

// intergrid.rs:414-459
double prolonged(const AmrGrid& g, const AmrState& s, int f, int level, const int64_t* cell) {
    const double r = (double)g.ratios[level - 1];
    const CellBox cd = g.level_domain(level - 1);
    int64_t c0[2];
    double w[2];
    for (int d = 0; d < 2; ++d) {
        double pc = ((double)cell[d] + 0.5) / r - 0.5;
        double fl = std::floor(pc);
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
        for (int d = 0; d < 2; ++d) cc[d] = reflect_coord(cc[d], cd.lo[d], cd.hi[d]);
        int64_t qb = g.find_patch(level - 1, cc);
        const Patch& q = g.patches[qb];
        acc += get(g, s, qb, f, cc[0] - q.bx.lo[0], cc[1] - q.bx.lo[1]) * weight;
    }
    return acc;
}

// intergrid.rs:73-86 + 358-408 ; old != nullptr is the subcycling time
// interpolation (fill_level, intergrid.rs:183-223)
void fill_one_level(const AmrGrid& g, AmrState& s, const AmrState* old, double alpha, int f, int level) {
    const int gh = s.ghost[f];
    if (gh == 0) return;
    const CellBox dom = g.level_domain(level);
    auto rng = g.blocks_at(level);
    for (uint32_t pb = rng.first; pb < rng.second; ++pb) {
        const Patch p = g.patches[pb];
        std::vector<std::pair<int64_t, double>> staged;
        auto visit = [&](const int64_t* cell) {
            int64_t target[2] = {reflect_coord(cell[0], dom.lo[0], dom.hi[0]),
                                 reflect_coord(cell[1], dom.lo[1], dom.hi[1])};
            int64_t src = g.find_patch(level, target);
            double value;
            if (src < 0) {
                double v_new = prolonged(g, s, f, level, target);
                if (old) {
                    double v_old = prolonged(g, *old, f, level, target);
                    value = v_old * (1.0 - alpha) + v_new * alpha;
                } else {
                    value = v_new;
                }
            } else {
                const Patch& sp = g.patches[src];
                value = get(g, s, src, f, target[0] - sp.bx.lo[0], target[1] - sp.bx.lo[1]);
            }
            int64_t li[2] = {cell[0] - p.bx.lo[0], cell[1] - p.bx.lo[1]};
            staged.push_back({g.ext(pb).lin(li, gh), value});
        };
        for (int d = 0; d < 2; ++d) {
            for (int side = 0; side < 2; ++side) {
                int64_t lo[2], hi[2];
                for (int e = 0; e < 2; ++e) {
                    if (e < d) {
                        lo[e] = p.bx.lo[e] - gh;
                        hi[e] = p.bx.hi[e] + gh;
                    } else {
                        lo[e] = p.bx.lo[e];
                        hi[e] = p.bx.hi[e];
                    }
                }
                if (side == 0) {
                    lo[d] = p.bx.lo[d] - gh;
                    hi[d] = p.bx.lo[d];
                } else {
                    lo[d] = p.bx.hi[d];
                    hi[d] = p.bx.hi[d] + gh;
                }
                for_each_box(2, lo, hi, visit);
            }
        }
        for (auto& sv : staged) s.slab[pb][f][sv.first] = sv.second;
    }
}

void fill_ghosts_all(const AmrGrid& g, AmrState& s, int f) {
    for (int level = 0; level < g.num_levels(); ++level) fill_one_level(g, s, nullptr, 0.0, f, level);
}

// adapt.rs:352-402
double sample(const AmrGrid& g, const AmrState& s, int f, int level, const int64_t* cell) {
    if (level < g.num_levels()) {
        int64_t b = g.find_patch(level, cell);
        if (b >= 0) {
            const Patch& p = g.patches[b];
            return get(g, s, b, f, cell[0] - p.bx.lo[0], cell[1] - p.bx.lo[1]);
        }
    }
    const double r = (double)g.ratios[level - 1];
    const CellBox cd = g.level_domain(level - 1);
    int64_t c0[2];
    double w[2];
    for (int d = 0; d < 2; ++d) {
        double pc = ((double)cell[d] + 0.5) / r - 0.5;
        double fl = std::floor(pc);
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
        for (int d = 0; d < 2; ++d) {
            if (cc[d] < cd.lo[d]) cc[d] = 2 * cd.lo[d] - 1 - cc[d];
            else if (cc[d] >= cd.hi[d]) cc[d] = 2 * cd.hi[d] - 1 - cc[d];
        }
        acc += sample(g, s, f, level - 1, cc) * weight;
    }
    return acc;
}

// adapt.rs:323-347
void migrate(const AmrGrid& og, const AmrState& os, const AmrGrid& ng, AmrState& ns) {
    for (size_t f = 0; f < os.ghost.size(); ++f) {
        auto r0 = ng.blocks_at(0);
        for (uint32_t b = r0.first; b < r0.second; ++b) ns.slab[b][f] = os.slab[b][f];
        for (int level = 1; level < ng.num_levels(); ++level) {
            auto rl = ng.blocks_at(level);
            for (uint32_t nb = rl.first; nb < rl.second; ++nb) {
                const Patch np = ng.patches[nb];
                const Ext e = ng.ext(nb);
                for_each_interior(e, [&](const int64_t* idx) {
                    int64_t cell[2] = {np.bx.lo[0] + idx[0], np.bx.lo[1] + idx[1]};
                    ns.slab[nb][f][e.lin(idx, ns.ghost[f])] = sample(og, os, (int)f, level, cell);
                });
            }
        }
    }
}

// adapt.rs:78-103 (GradientTagger::tag_level)
void tag_level(const AmrGrid& g, const AmrState& s, int f, double threshold, int level, std::vector<Cell>& flags) {
    auto rl = g.blocks_at(level);
    for (uint32_t pb = rl.first; pb < rl.second; ++pb) {
        const Patch p = g.patches[pb];
        const Ext e = g.ext(pb);
        for_each_interior(e, [&](const int64_t* idx) {
            double gmax = 0.0;
            for (int d = 0; d < 2; ++d) {
                int64_t hi[2] = {idx[0], idx[1]}, lo[2] = {idx[0], idx[1]};
                hi[d] += 1;
                lo[d] -= 1;
                double v = std::fabs((s.slab[pb][f][e.lin(hi, s.ghost[f])] - s.slab[pb][f][e.lin(lo, s.ghost[f])]) * 0.5);
                gmax = std::fmax(gmax, v);
            }
            if (gmax > threshold) flags.push_back({p.bx.lo[0] + idx[0], p.bx.lo[1] + idx[1], 0});
        });
    }
}

struct Policy {
    int64_t every, buffer;
    ClusterParams cluster;
    double threshold;
    int field;
};

// adapt.rs:269-317
bool box_covered(const CellBox& need, const std::vector<CellBox>& cover) { return covered_by(need, cover); }

bool hierarchy_acceptable(const AmrGrid& g, const std::vector<std::vector<CellBox>>& nl) {
    if ((int)nl.size() != g.num_levels() - 1) return false;
    for (size_t l = 0; l < nl.size(); ++l) {
        std::vector<CellBox> current;
        auto rl = g.blocks_at((int)l + 1);
        for (uint32_t b = rl.first; b < rl.second; ++b) current.push_back(g.patches[b].bx);
        uint64_t pc = 0, cc = 0;
        for (const auto& b : nl[l]) pc += b.cells();
        for (const auto& b : current) cc += b.cells();
        if (cc > pc + pc / 2) return false;
        for (const auto& b : nl[l])
            if (!box_covered(b, current)) return false;
    }
    return true;
}

// BergerOliger::regrid (adapt.rs:152-237); returns true with the new grid
// and migrated state when the hierarchy changes.  `forced`, when given,
// holds each source level's flags in place of the gradient tagger (a test's
// own TagCells, tests/amr.rs:800-823).
bool regrid(const AmrGrid& g, AmrState& s, const Policy& pol, const std::vector<int>& prepare_fields,
            int64_t step, AmrGrid* ng, AmrState* ns, const std::vector<std::vector<Cell>>* forced = nullptr) {
    if (step % pol.every != 0) return false;
    for (int f : prepare_fields) {
        restrict_all(g, s, f);
        fill_ghosts_all(g, s, f);
    }
    const int capacity = g.max_levels() - 1;
    std::vector<std::vector<CellBox>> new_levels(capacity);
    for (int target = capacity; target >= 1; --target) {
        const int src = target - 1;
        std::vector<Cell> flags;
        if (forced) {
            if (src < (int)forced->size()) flags = (*forced)[src];
        } else if (src < g.num_levels()) {
            tag_level(g, s, pol.field, pol.threshold, src, flags);
        }
        if (pol.buffer > 0) {
            std::vector<Cell> seeds;
            seeds.swap(flags);
            for (const auto& c : seeds)
                for (int64_t y = c[1] - pol.buffer; y < c[1] + pol.buffer + 1; ++y)
                    for (int64_t x = c[0] - pol.buffer; x < c[0] + pol.buffer + 1; ++x) flags.push_back({x, y, 0});
        }
        if (target < capacity && !new_levels[target].empty()) {
            const int64_t r_fine = g.ratios[target], r_src = g.ratios[target - 1];
            for (const auto& bx : new_levels[target]) {
                int64_t nlo[2], nhi[2], plo[2], phi[2];
                for (int d = 0; d < 2; ++d) {
                    nlo[d] = bx.lo[d] / r_fine - 1;
                    nhi[d] = bx.hi[d] / r_fine + 1;
                    plo[d] = div_euclid(nlo[d], r_src);
                    phi[d] = div_euclid(nhi[d] + r_src - 1, r_src);
                }
                for (int64_t y = plo[1]; y < phi[1]; ++y)
                    for (int64_t x = plo[0]; x < phi[0]; ++x) flags.push_back({x, y, 0});
            }
        }
        const CellBox dom = g.level_domain(src);
        std::vector<Cell> kept;
        for (const auto& c : flags)
            if (dom.contains(c.data())) kept.push_back(c);
        std::sort(kept.begin(), kept.end());
        kept.erase(std::unique(kept.begin(), kept.end()), kept.end());
        if (kept.empty()) continue;
        const int64_t r = g.ratios[target - 1];
        for (auto bx : cluster(2, kept, pol.cluster)) {
            for (int d = 0; d < 2; ++d) {
                bx.lo[d] *= r;
                bx.hi[d] *= r;
            }
            new_levels[target - 1].push_back(bx);
        }
    }
    while (!new_levels.empty() && new_levels.back().empty()) new_levels.pop_back();
    if (hierarchy_acceptable(g, new_levels)) return false;
    if (from_patches(g.base, g.ratios, new_levels, ng) != AMR_OK) return false;
    *ns = make_amr_state(*ng, s.ghost);
    migrate(g, s, *ng, *ns);
    return true;
}

// -------------------------------------------------------- simulation ------
enum ModelKind { MODEL_HEAT = 0, MODEL_C = 1 };
enum IntegratorKind { INT_SUBCYCLING = 0, INT_GLOBAL = 1 };

struct AmrSim {
    AmrGrid grid;
    AmrState state;
    int model;
    ModelC mc{};
    double kappa = 0.0;
    int integrator;
    uint64_t seed;
    bool wiener;
    bool has_policy = false;
    Policy policy{};
    double t = 0.0;
    int64_t step_index = 0;
    int64_t epoch = 0;
    int nthreads = 1;

    int nfields() const { return model == MODEL_C ? 2 : 1; }
    // phasefield.rs:446-449 (0.2 h^2 / D) ; tests/amr.rs:339-341 (0.25 h^2 / kappa)
    double stable_dt_at(int level) const {
        const auto& h = grid.level_spacing[level];
        double hm = std::min(h[0], h[1]);
        if (model == MODEL_C) return 0.2 * (hm * hm) / mc.d_thermal;
        return 0.25 * (hm * hm) / kappa;
    }
    double suggested_dt() const {
        return integrator == INT_SUBCYCLING ? stable_dt_at(0) : stable_dt_at(grid.max_levels() - 1);
    }

    // drift of one block into k (interior), the model's vector_field_block
    void drift_block(int64_t b, std::vector<std::vector<double>>& k) {
        const Ext e = grid.ext(b);
        const double* h = grid.spacing(b);
        if (model == MODEL_C)
            modelc_drift_block(e, h, mc, state.slab[b][0].data(), state.slab[b][1].data(), k[0].data(), k[1].data());
        else
            heat_drift_block(e, h, kappa, state.slab[b][0].data(), k[0].data());
    }

    // one Euler-Maruyama update of the blocks [b0, b1): drift, amplitude,
    // apply (state.rs:656-753), with the stage buffers of the reference
    // (zeroed once, interior-only writes)
    void em_blocks(uint32_t b0, uint32_t b1, double t_now, double dt) {
        const uint64_t salt = bits_of(t_now);
        std::vector<std::vector<std::vector<double>>> k(b1 - b0);
        parallel_blocks(b1 - b0, nthreads, [&](int64_t i) {
            const int64_t b = b0 + i;
            const Ext e = grid.ext(b);
            k[i].assign(nfields(), std::vector<double>(e.len(1), 0.0));
            drift_block(b, k[i]);
        });
        parallel_blocks(b1 - b0, nthreads, [&](int64_t i) {
            const int64_t b = b0 + i;
            const Ext e = grid.ext(b);
            for (int f = 0; f < nfields(); ++f) apply_time(state.slab[b][f], k[i][f], dt);
            if (wiener) {
                std::vector<double> amp(e.len(1), 0.0);
                for_each_interior(e, [&](const int64_t* idx) { amp[e.lin(idx, 1)] = mc.noise_amplitude; });
                apply_wiener(e, 1, state.slab[b][0], amp, dt, seed, salt, (uint64_t)b);
            }
        });
    }

    // Subcycle::advance (subcycling.rs:195-267)
    void advance(std::vector<AmrState>& snaps, int level, double t_now, double dt, double alpha) {
        snaps[level] = state;
        for (int f = 0; f < nfields(); ++f) {
            if (level > 0)
                fill_one_level(grid, state, &snaps[level - 1], alpha, f, level);
            else
                fill_one_level(grid, state, nullptr, 0.0, f, level);
        }
        auto rl = grid.blocks_at(level);
        em_blocks(rl.first, rl.second, t_now, dt);
        const int child = level + 1;
        if (child < grid.num_levels()) {
            double n_f = std::round(stable_dt_at(level) / stable_dt_at(child));
            uint64_t n = (uint64_t)std::max(n_f, 1.0);
            double dt_child = dt / (double)n;
            for (uint64_t s = 0; s < n; ++s)
                advance(snaps, child, std::fma((double)s, dt_child, t_now), dt_child, (double)s / (double)n);
            for (int f = 0; f < nfields(); ++f) restrict_level(grid, state, f, child);
        }
    }

    // Simulation::step (simulation.rs:255-290)
    void step(double dt) {
        if (has_policy) {
            AmrGrid ng;
            AmrState ns;
            std::vector<int> prep = {policy.field};
            if (regrid(grid, state, policy, prep, step_index, &ng, &ns)) {
                grid = std::move(ng);
                state = std::move(ns);
                epoch += 1;
            }
        }
        if (integrator == INT_SUBCYCLING) {
            std::vector<AmrState> snaps(grid.max_levels());
            advance(snaps, 0, t, dt, 0.0);
        } else {
            // eval_drift: the model's AMR fill_ghosts (phasefield.rs:454-467,
            // tests/amr.rs:314-322), then every block
            for (int f = 0; f < nfields(); ++f) restrict_all(grid, state, f);
            for (int f = 0; f < nfields(); ++f) fill_ghosts_all(grid, state, f);
            em_blocks(0, (uint32_t)grid.num_blocks(), t, dt);
        }
        t += dt;
        step_index += 1;
    }
};

}  // namespace

// ============================================================ C ABI =======
extern "C" {

int64_t orc_cluster(int D, const int64_t* flags, int64_t n, double efficiency, int64_t min_width, int64_t* out,
                    int64_t cap) {
    std::vector<Cell> f(n);
    for (int64_t i = 0; i < n; ++i) {
        f[i] = {0, 0, 0};
        for (int d = 0; d < D; ++d) f[i][d] = flags[i * D + d];
    }
    auto boxes = cluster(D, f, ClusterParams{efficiency, min_width});
    for (size_t i = 0; i < boxes.size() && (int64_t)i < cap; ++i)
        for (int d = 0; d < D; ++d) {
            out[i * 2 * D + d] = boxes[i].lo[d];
            out[i * 2 * D + D + d] = boxes[i].hi[d];
        }
    return (int64_t)boxes.size();
}

// patches: n x (level, lo0, lo1, hi0, hi1); returns NULL and *err on error
void* orc_amr_sim_create(const int64_t* cells, const int64_t* block, const double* origin, const double* spacing,
                         const uint32_t* ratios, int nratios, const int64_t* patches, int64_t npatches, int model,
                         const orc_modelc_params* p, double kappa, int integrator, uint64_t seed, int wiener,
                         const double* policy, int* err) {
    Base base;
    for (int d = 0; d < 2; ++d) {
        base.cells[d] = cells[d];
        base.block[d] = block[d];
        base.nb[d] = cells[d] / block[d];
        base.origin[d] = origin[d];
        base.spacing[d] = spacing[d];
    }
    std::vector<uint32_t> r(ratios, ratios + nratios);
    int maxl = 0;
    for (int64_t i = 0; i < npatches; ++i) maxl = std::max(maxl, (int)patches[5 * i]);
    std::vector<std::vector<CellBox>> levels(maxl);
    for (int64_t i = 0; i < npatches; ++i) {
        CellBox b;
        b.D = 2;
        b.lo[0] = patches[5 * i + 1];
        b.lo[1] = patches[5 * i + 2];
        b.hi[0] = patches[5 * i + 3];
        b.hi[1] = patches[5 * i + 4];
        levels[patches[5 * i] - 1].push_back(b);
    }
    auto sim = std::make_unique<AmrSim>();
    int rc = from_patches(base, r, levels, &sim->grid);
    if (err) *err = rc;
    if (rc != AMR_OK) return nullptr;
    sim->model = model;
    if (p) sim->mc = make_model(p);
    sim->kappa = kappa;
    sim->integrator = integrator;
    sim->seed = seed;
    sim->wiener = wiener != 0 && model == MODEL_C;
    std::vector<int> ghosts(sim->nfields(), 1);
    sim->state = make_amr_state(sim->grid, ghosts);
    if (policy) {
        // every, buffer, efficiency, min_width, threshold, field
        sim->has_policy = true;
        sim->policy.every = (int64_t)policy[0];
        sim->policy.buffer = (int64_t)policy[1];
        sim->policy.cluster = ClusterParams{policy[2], (int64_t)policy[3]};
        sim->policy.threshold = policy[4];
        sim->policy.field = (int)policy[5];
    }
    return sim.release();
}

void orc_amr_sim_destroy(void* s) { delete static_cast<AmrSim*>(s); }
void orc_amr_sim_set_threads(void* s, int n) { static_cast<AmrSim*>(s)->nthreads = n; }
int64_t orc_amr_sim_num_blocks(const void* s) { return static_cast<const AmrSim*>(s)->grid.num_blocks(); }
int orc_amr_sim_num_levels(const void* s) { return static_cast<const AmrSim*>(s)->grid.num_levels(); }
int64_t orc_amr_sim_epoch(const void* s) { return static_cast<const AmrSim*>(s)->epoch; }
void orc_amr_sim_patch(const void* s, int64_t b, int64_t* out) {
    const auto& p = static_cast<const AmrSim*>(s)->grid.patches[b];
    out[0] = p.level;
    out[1] = p.bx.lo[0];
    out[2] = p.bx.lo[1];
    out[3] = p.bx.hi[0];
    out[4] = p.bx.hi[1];
}
int64_t orc_amr_sim_field_len(const void* s) {
    const AmrSim* sim = static_cast<const AmrSim*>(s);
    int64_t n = 0;
    for (int64_t b = 0; b < sim->grid.num_blocks(); ++b) n += sim->grid.ext(b).len(1);
    return n;
}
void orc_amr_sim_get_field(const void* s, int f, double* out) {
    const AmrSim* sim = static_cast<const AmrSim*>(s);
    size_t off = 0;
    for (const auto& b : sim->state.slab) {
        std::memcpy(out + off, b[f].data(), b[f].size() * sizeof(double));
        off += b[f].size();
    }
}
void orc_amr_sim_set_field(void* s, int f, const double* in) {
    AmrSim* sim = static_cast<AmrSim*>(s);
    size_t off = 0;
    for (auto& b : sim->state.slab) {
        std::memcpy(b[f].data(), in + off, b[f].size() * sizeof(double));
        off += b[f].size();
    }
}
double orc_amr_sim_step(void* s, double dt, int64_t nsteps) {
    AmrSim* sim = static_cast<AmrSim*>(s);
    for (int64_t i = 0; i < nsteps; ++i) sim->step(dt);
    return sim->t;
}
double orc_amr_sim_suggested_dt(const void* s) { return static_cast<const AmrSim*>(s)->suggested_dt(); }
void orc_amr_sim_restrict(void* s, int f) {
    AmrSim* sim = static_cast<AmrSim*>(s);
    restrict_all(sim->grid, sim->state, f);
}
void orc_amr_sim_fill_ghosts(void* s, int f) {
    AmrSim* sim = static_cast<AmrSim*>(s);
    fill_ghosts_all(sim->grid, sim->state, f);
}
int64_t orc_amr_sim_tag(const void* s, int f, double threshold, int level, int64_t* out, int64_t cap) {
    const AmrSim* sim = static_cast<const AmrSim*>(s);
    std::vector<Cell> flags;
    tag_level(sim->grid, sim->state, f, threshold, level, flags);
    for (size_t i = 0; i < flags.size() && (int64_t)i < cap; ++i) {
        out[2 * i] = flags[i][0];
        out[2 * i + 1] = flags[i][1];
    }
    return (int64_t)flags.size();
}
// a regrid now, with the level-0 flags given (n (x, y) pairs) instead of the
// tagger, buffer and clustering as given, no field preparation; 1 when the
// hierarchy changed (its epoch advances), 0 when it was kept
int orc_amr_sim_regrid_flags(void* s, const int64_t* flags, int64_t n, int64_t buffer, double efficiency,
                             int64_t min_width) {
    AmrSim* sim = static_cast<AmrSim*>(s);
    Policy pol = sim->policy;
    pol.every = 1;
    pol.buffer = buffer;
    pol.cluster = ClusterParams{efficiency, min_width};
    std::vector<std::vector<Cell>> forced(1);
    for (int64_t i = 0; i < n; ++i) forced[0].push_back({flags[2 * i], flags[2 * i + 1], 0});
    AmrGrid ng;
    AmrState ns;
    if (!regrid(sim->grid, sim->state, pol, {}, 0, &ng, &ns, &forced)) return 0;
    sim->grid = std::move(ng);
    sim->state = std::move(ns);
    sim->epoch += 1;
    return 1;
}
void orc_amr_sim_cell_center(const void* s, int64_t b, const int64_t* idx, double* out) {
    static_cast<const AmrSim*>(s)->grid.cell_center(b, idx, out);
}

}  // extern "C"
