/*
 * Dynamic AMR, host half: the tag passes after the per-cell vote, 2:1
 * balance, refinement and coarsening of the block tree, and the rebuild of
 * the neighbour slots, with the reference's block order, slot order and
 * tolerances (src/prj_amr.c, src/prj_mesh.c).  The cell and face data are
 * moved by the device kernels of fx_amr.cu from the job lists built here.
 */
#include "fx_amr.h"
#include "fx_layout.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <unordered_map>

namespace {

constexpr int kBS = FX_BS;
constexpr int kNG = FX_NG; /* PRJ_NGHOST of the build: the slots' send / recv boxes depend on it */
constexpr double kTol = 1.0e-12;

enum { NB_NONE = 0, NB_FACE = 1, NB_EDGE = 2, NB_CORNER = 3 };

} /* namespace */

/* send/recv boxes of neighbour b as seen from a: prj_neighbor_compute_geometry
 * (src/prj_mesh.c:46-243) */
bool fx_neighbor_geometry(const fx_block_desc &a, const fx_block_desc &b, fx_slot &s)
{
    int axisrel[3] = {0, 0, 0};
    int touching = 0;
    for (int d = 0; d < 3; ++d) {
        const double tol = 1.0e-2 * std::fmin(a.dx[d], b.dx[d]);
        if (std::fabs(a.xmax[d] - b.xmin[d]) < tol) {
            axisrel[d] = 1;
            ++touching;
        } else if (std::fabs(b.xmax[d] - a.xmin[d]) < tol) {
            axisrel[d] = -1;
            ++touching;
        }
    }
    static const int kType[4] = {NB_NONE, NB_FACE, NB_EDGE, NB_CORNER};
    s.type = kType[touching];
    s.rel_level = b.level - a.level;
    for (int d = 0; d < 3; ++d) {
        int rs, re, ss, se;
        if (s.rel_level == 0) {
            if (axisrel[d] == 1) { rs = -kNG; re = 0; ss = kBS - kNG; se = kBS; }
            else if (axisrel[d] == -1) { rs = kBS; re = kBS + kNG; ss = 0; se = kNG; }
            else { rs = 0; re = kBS; ss = 0; se = kBS; }
        } else if (s.rel_level == -1) {
            if (axisrel[d] == 1) { rs = -kNG; re = 0; ss = kBS - 2 * kNG; se = kBS; }
            else if (axisrel[d] == -1) { rs = kBS; re = kBS + kNG; ss = 0; se = 2 * kNG; }
            else {
                if ((b.xmin[d] + b.xmax[d]) > (a.xmin[d] + a.xmax[d])) { rs = 0; re = kBS / 2; }
                else { rs = kBS / 2; re = kBS; }
                ss = 0;
                se = kBS;
            }
        } else if (s.rel_level == 1) {
            if (axisrel[d] == 1) { rs = -kNG; re = 0; ss = kBS - kNG / 2; se = kBS; }
            else if (axisrel[d] == -1) { rs = kBS; re = kBS + kNG; ss = 0; se = kNG / 2; }
            else {
                if ((b.xmin[d] + b.xmax[d]) > (a.xmin[d] + a.xmax[d])) {
                    rs = -kNG; re = kBS; ss = kBS / 2 - kNG / 2; se = kBS;
                } else {
                    rs = 0; re = kBS + kNG; ss = 0; se = kBS / 2 + kNG / 2;
                }
            }
        } else {
            return false; /* level jump larger than one */
        }
        s.recv_loc_start[d] = (int8_t)rs;
        s.recv_loc_end[d] = (int8_t)re;
        s.send_loc_start[d] = (int8_t)ss;
        s.send_loc_end[d] = (int8_t)se;
    }
    return true;
}

namespace {

bool is_active(const fx_block_desc &b) { return b.id >= 0 && b.active == 1; }

void clear_slots(fx_block_desc &b)
{
    for (int n = 0; n < 56; ++n) {
        fx_slot &s = b.slot[n];
        std::memset(&s, 0, sizeof(s));
        s.id = -1;
    }
}

void reset_children(fx_block_desc &b)
{
    for (int n = 0; n < 8; ++n) b.children[n] = -1;
}

/* prj_block_setup_geometry (src/prj_mesh.c:675-687) */
void setup_geometry(fx_block_desc &b)
{
    b.vol = b.dx[0] * b.dx[1] * b.dx[2];
    b.area[0] = b.dx[1] * b.dx[2];
    b.area[1] = b.dx[0] * b.dx[2];
    b.area[2] = b.dx[0] * b.dx[1];
}

/* prj_block_cell_size (src/prj_amr.c:42-57) */
double cell_size(const fx_block_desc &b)
{
    double c = b.dx[0];
    if (b.dx[1] > c) c = b.dx[1];
    if (b.dx[2] > c) c = b.dx[2];
    return c;
}

/* prj_boxes_touch_face_edge_corner (src/prj_amr.c:398-425) */
bool touch_face_edge_corner(const fx_block_desc &a, const fx_block_desc &b)
{
    int touches = 0;
    for (int ax = 0; ax < 3; ++ax) {
        if (!(std::fmin(a.xmax[ax], b.xmax[ax]) >= std::fmax(a.xmin[ax], b.xmin[ax]) - kTol)) return false;
        if (std::fabs(a.xmax[ax] - b.xmin[ax]) < kTol || std::fabs(b.xmax[ax] - a.xmin[ax]) < kTol) ++touches;
    }
    if (touches == 0) return false;
    bool same = true;
    for (int ax = 0; ax < 3; ++ax) {
        if (!(std::fabs(a.xmin[ax] - b.xmin[ax]) < kTol && std::fabs(a.xmax[ax] - b.xmax[ax]) < kTol)) {
            same = false;
        }
    }
    return !same;
}

/* prj_blocks_are_face_neighbors (src/prj_amr.c:511-538) */
bool face_neighbors(const fx_block_desc &a, const fx_block_desc &b)
{
    int touching = 0;
    for (int ax = 0; ax < 3; ++ax) {
        if (std::fabs(a.xmax[ax] - b.xmin[ax]) < kTol || std::fabs(b.xmax[ax] - a.xmin[ax]) < kTol) {
            ++touching;
        } else {
            const double overlap = std::fmin(a.xmax[ax], b.xmax[ax]) - std::fmax(a.xmin[ax], b.xmin[ax]);
            if (!(overlap > kTol)) return false;
        }
    }
    return touching == 1;
}

struct Mesh {
    const fx_config &cfg;
    const fx_amr_config &amr;
    std::vector<fx_block_desc> &b;
    int nmax;
    std::string *err;
    bool overflow = false;
    bool geom_error = false;

    int nblocks() const { return (int)b.size(); }

    /* prj_add_neighbor (src/prj_amr.c:540-573): first free slot */
    void add_neighbor(fx_block_desc &a, const fx_block_desc &nb)
    {
        for (int n = 0; n < 56; ++n) {
            if (a.slot[n].id == nb.id) return;
        }
        for (int n = 0; n < 56; ++n) {
            if (a.slot[n].id < 0) {
                a.slot[n].id = nb.id;
                if (!fx_neighbor_geometry(a, nb, a.slot[n])) geom_error = true;
                return;
            }
        }
        overflow = true;
    }

    /* prj_mesh_block_logical_coords (src/prj_mesh.c:1250-1288) */
    bool logical_coords(const fx_block_desc &blk, int out[3]) const
    {
        for (int ax = 0; ax < 3; ++ax) {
            const double lo = cfg.coord[2 * ax];
            const double hi = cfg.coord[2 * ax + 1];
            const double extent = hi - lo;
            const int count = amr.root_nx[ax] << blk.level;
            if (extent <= 0.0 || count <= 0) return false;
            const double scale = (double)count / extent;
            const double scaled = (blk.xmin[ax] - lo) * scale;
            if (!std::isfinite(scaled) || scaled < -0.5) return false;
            const int c = (int)(scaled + 0.5);
            if (c < 0 || c >= count) return false;
            out[ax] = c;
        }
        return true;
    }

    static uint64_t key(int level, int ix, int iy, int iz)
    {
        return ((uint64_t)(uint32_t)level << 57) | ((uint64_t)(uint32_t)ix << 38) |
            ((uint64_t)(uint32_t)iy << 19) | (uint64_t)(uint32_t)iz;
    }

    /* prj_amr_init_neighbors_with_mask, Morton path (src/prj_amr.c:1550-1579,
     * 575-711) */
    void init_neighbors(const std::vector<char> &dirty)
    {
        for (int i = 0; i < nblocks(); ++i) {
            if (b[i].id >= 0 && dirty[i]) clear_slots(b[i]);
        }
        std::unordered_map<uint64_t, int> lookup;
        lookup.reserve((size_t)nblocks() * 2);
        for (int i = 0; i < nblocks(); ++i) {
            int c[3];
            if (is_active(b[i]) && logical_coords(b[i], c)) {
                lookup.emplace(key(b[i].level, c[0], c[1], c[2]), i);
            }
        }
        for (int i = 0; i < nblocks(); ++i) {
            if (!is_active(b[i]) || !dirty[i]) continue;
            for (int level = b[i].level - 1; level <= b[i].level + 1; ++level) {
                if (level < 0) continue;
                int lo[3], hi[3];
                bool ok = true;
                for (int ax = 0; ax < 3; ++ax) {
                    const double cmin = cfg.coord[2 * ax];
                    const double extent = cfg.coord[2 * ax + 1] - cmin;
                    const double count = std::ldexp((double)amr.root_nx[ax], level);
                    if (!(extent > 0.0)) { ok = false; break; }
                    const double scale = count / extent;
                    const double l = (b[i].xmin[ax] - cmin) * scale;
                    const double h = (b[i].xmax[ax] - cmin) * scale;
                    lo[ax] = (int)std::floor(l) - 1;
                    hi[ax] = (int)std::ceil(h);
                }
                if (!ok) continue;
                for (int ix = lo[0]; ix <= hi[0]; ++ix) {
                    for (int iy = lo[1]; iy <= hi[1]; ++iy) {
                        for (int iz = lo[2]; iz <= hi[2]; ++iz) {
                            if (ix < 0 || iy < 0 || iz < 0) continue;
                            auto it = lookup.find(key(level, ix, iy, iz));
                            if (it == lookup.end()) continue;
                            const int nid = it->second;
                            if (nid == i || !is_active(b[nid])) continue;
                            if (touch_face_edge_corner(b[i], b[nid])) {
                                add_neighbor(b[i], b[nid]);
                                add_neighbor(b[nid], b[i]);
                            }
                        }
                    }
                }
            }
        }
    }

    /* prj_find_free_block_slot (src/prj_amr.c:369-391) */
    int free_slot()
    {
        for (int i = 0; i < nblocks(); ++i) {
            if (b[i].id < 0) return i;
        }
        if (nblocks() < nmax) {
            fx_block_desc blank;
            std::memset(&blank, 0, sizeof(blank));
            blank.id = -1;
            blank.parent = -1;
            reset_children(blank);
            clear_slots(blank);
            b.push_back(blank);
            return nblocks() - 1;
        }
        return -1;
    }

    void mark_dirty_and_neighbors(int id, std::vector<char> &dirty) const
    {
        if (id < 0 || id >= nblocks()) return;
        dirty[id] = 1;
        for (int n = 0; n < 56; ++n) {
            const int nid = b[id].slot[n].id;
            if (nid >= 0 && nid < nblocks()) dirty[nid] = 1;
        }
    }

    /* the face layers a new child copies from the parent's finer face
     * neighbours (src/prj_amr.c:2000-2083) */
    void copy_sources(const fx_block_desc &parent, const fx_block_desc &child, int copy_src[6]) const
    {
        for (int q = 0; q < 6; ++q) copy_src[q] = -1;
        for (int n = 0; n < 56; ++n) {
            const fx_slot &s = parent.slot[n];
            if (s.id < 0 || s.type != NB_FACE || s.rel_level < 1) continue;
            const fx_block_desc &nb = b[s.id];
            for (int dir = 0; dir < 3; ++dir) {
                const int t0 = (dir + 1) % 3;
                const int t1 = (dir + 2) % 3;
                if (!(std::fabs(child.xmin[t0] - nb.xmin[t0]) < 1.0e-12 * child.dx[t0])) continue;
                if (!(std::fabs(child.xmin[t1] - nb.xmin[t1]) < 1.0e-12 * child.dx[t1])) continue;
                if (std::fabs(child.xmax[dir] - nb.xmin[dir]) < 1.0e-12 * child.dx[dir]) {
                    copy_src[2 * dir + 1] = s.id;
                }
                if (std::fabs(child.xmin[dir] - nb.xmax[dir]) < 1.0e-12 * child.dx[dir]) {
                    copy_src[2 * dir + 0] = s.id;
                }
            }
        }
    }

    /* prj_amr_refine_block (src/prj_amr.c:2389-2504); false when the block
     * array is full */
    bool refine_block(int id, std::vector<FxAmrRefine> &jobs, std::vector<char> &dirty)
    {
        if (!is_active(b[id]) || (amr.max_level >= 0 && b[id].level >= amr.max_level)) return true;
        if (b[id].can_refine == 0) {
            flag[id] = 0;
            return true;
        }
        if (amr.min_dx > 0.0 && cell_size(b[id]) <= amr.min_dx) {
            flag[id] = 0;
            return true;
        }
        double xmid[3];
        for (int a = 0; a < 3; ++a) xmid[a] = 0.5 * (b[id].xmin[a] + b[id].xmax[a]);
        for (int oct = 0; oct < 8; ++oct) {
            const int cid = free_slot();
            if (cid < 0) return false;
            fx_block_desc &p = b[id]; /* free_slot may grow b */
            fx_block_desc &c = b[cid];
            std::memset(&c, 0, sizeof(c));
            c.id = cid;
            c.rank = p.rank;
            c.level = p.level + 1;
            c.active = 1;
            flag[cid] = 0;
            c.can_refine = 1;
            c.parent = p.id;
            reset_children(c);
            clear_slots(c);
            const int bit[3] = {oct & 1, (oct >> 1) & 1, (oct >> 2) & 1};
            for (int a = 0; a < 3; ++a) {
                c.xmin[a] = bit[a] == 0 ? p.xmin[a] : xmid[a];
                c.xmax[a] = bit[a] == 0 ? xmid[a] : p.xmax[a];
                c.dx[a] = p.dx[a] * 0.5;
            }
            setup_geometry(c);
            FxAmrRefine job;
            job.child = cid;
            job.parent = id;
            job.oct = oct;
            copy_sources(p, c, job.copy_src);
            jobs.push_back(job);
            p.children[oct] = cid;
        }
        b[id].active = 0;
        flag[id] = 0;
        (void)dirty;
        return true;
    }

    /* prj_can_coarsen_parent (src/prj_amr.c:1331-1370) */
    bool can_coarsen(int pid) const
    {
        if (pid < 0 || pid >= nblocks()) return false;
        const fx_block_desc &p = b[pid];
        if (p.id < 0 || p.active == 1) return false;
        for (int oct = 0; oct < 8; ++oct) {
            const int cid = p.children[oct];
            if (cid < 0 || cid >= nblocks() || !is_active(b[cid])) return false;
            if (flag[cid] >= 0) return false;
            for (int n = 0; n < 56; ++n) {
                const int nid = b[cid].slot[n].id;
                if (nid >= 0 && nid < nblocks() && is_active(b[nid]) && b[nid].parent != pid &&
                    b[nid].level > p.level + 1) {
                    return false;
                }
            }
        }
        return true;
    }

    /* prj_amr_coarsen_block (src/prj_amr.c:2506-2574), one rank */
    void coarsen_block(int pid, std::vector<FxAmrCoarsen> &jobs)
    {
        fx_block_desc &p = b[pid];
        FxAmrCoarsen job;
        job.parent = pid;
        for (int oct = 0; oct < 8; ++oct) job.children[oct] = p.children[oct];
        jobs.push_back(job);
        p.active = 1;
        flag[pid] = 0;
        for (int oct = 0; oct < 8; ++oct) {
            fx_block_desc &c = b[p.children[oct]];
            c.id = -1;
            c.active = 0;
            c.can_refine = 1;
            c.parent = -1;
            reset_children(c);
            clear_slots(c);
            p.children[oct] = -1;
        }
    }

    /* prj_has_face_neighbor_coarser_than (src/prj_amr.c:1254-1269) */
    bool face_neighbor_coarser_than(int i, int min_level) const
    {
        for (int n = 0; n < 56; ++n) {
            const int id = b[i].slot[n].id;
            if (id >= 0 && id < nblocks() && is_active(b[id]) && face_neighbors(b[i], b[id]) &&
                b[id].level < min_level) {
                return true;
            }
        }
        return false;
    }

    /* prj_block_neighbor_touch_offset (src/prj_amr.c:1271-1285) */
    static int touch_offset(const fx_block_desc &blk, const fx_block_desc &nb, int axis)
    {
        if (std::fabs(blk.xmin[axis] - nb.xmax[axis]) < kTol) return -1;
        if (std::fabs(blk.xmax[axis] - nb.xmin[axis]) < kTol) return 1;
        return 0;
    }

    /* prj_amr_boundary_mask_has_side (src/prj_amr.c:146-158) */
    static bool mask_has_side(unsigned mask, int axis, int sign)
    {
        if (sign == 0) return true;
        return (mask & (1u << (2 * axis + (sign < 0 ? 0 : 1)))) != 0u;
    }

    /* prj_amr_tag passes 2 and 4 (src/prj_amr.c:1707-1774) from pass-1 votes */
    void tag(const int32_t *votes)
    {
        const int nb = nblocks();
        std::vector<int32_t> pos(nb), neg(nb);
        for (int i = 0; i < nb; ++i) {
            pos[i] = votes[3 * i];
            neg[i] = votes[3 * i + 1];
        }
        for (int i = 0; i < nb; ++i) {
            const unsigned mask = (unsigned)votes[3 * i + 2];
            if (mask == 0u || !is_active(b[i])) continue;
            for (int n = 0; n < 56; ++n) {
                const int id = b[i].slot[n].id;
                if (id < 0 || id >= nb || !is_active(b[id]) || b[id].level > b[i].level) continue;
                bool matches = false;
                bool ok = true;
                for (int axis = 0; axis < 3; ++axis) {
                    const int off = touch_offset(b[i], b[id], axis);
                    if (off == 0) continue;
                    matches = true;
                    if (!mask_has_side(mask, axis, off)) {
                        ok = false;
                        break;
                    }
                }
                if (ok && matches) pos[id] = 1;
            }
        }
        for (int i = 0; i < nb; ++i) {
            if (!is_active(b[i])) {
                flag[i] = 0;
            } else if (pos[i] > 0) {
                const bool allowed = b[i].can_refine != 0 &&
                    (amr.max_level < 0 || b[i].level < amr.max_level) &&
                    (amr.min_dx <= 0.0 || cell_size(b[i]) > amr.min_dx) &&
                    !face_neighbor_coarser_than(i, b[i].level - 1);
                flag[i] = allowed ? 1 : 0;
            } else if (neg[i] < 0) {
                flag[i] = -1;
            } else {
                flag[i] = 0;
            }
        }
    }

    /* prj_amr_enforce_two_to_one (src/prj_amr.c:1471-1500) */
    void two_to_one()
    {
        bool changed;
        do {
            changed = false;
            for (int i = 0; i < nblocks(); ++i) {
                if (!is_active(b[i]) || flag[i] <= 0) continue;
                for (int n = 0; n < 56; ++n) {
                    const int id = b[i].slot[n].id;
                    if (id >= 0 && id < nblocks() && is_active(b[id]) && b[id].level < b[i].level &&
                        b[id].can_refine != 0 && flag[id] != 1) {
                        flag[id] = 1;
                        changed = true;
                    }
                }
            }
        } while (changed);
    }

    /* prj_amr_has_pending_change (src/prj_amr.c:1372-1397) */
    bool pending_change() const
    {
        for (int i = 0; i < nblocks(); ++i) {
            if (is_active(b[i]) && flag[i] > 0 && b[i].can_refine != 0) return true;
        }
        for (int i = 0; i < nblocks(); ++i) {
            if (b[i].id >= 0 && b[i].active != 1 && can_coarsen(i)) return true;
        }
        return false;
    }

    std::vector<int32_t> flag;
};

} /* namespace */

void fx_amr_flags(const fx_amr_config &amr, int nblocks, const fx_block_desc *blocks,
    const int32_t *votes, int32_t *flags)
{
    fx_config cfg;
    std::memset(&cfg, 0, sizeof(cfg));
    std::vector<fx_block_desc> b(blocks, blocks + nblocks);
    Mesh m{cfg, amr, b, nblocks, nullptr, false, false, {}};
    m.flag.assign(nblocks, 0);
    m.tag(votes);
    for (int i = 0; i < nblocks; ++i) flags[i] = m.flag[i];
}

int fx_amr_remesh(const fx_config &cfg, const fx_amr_config &amr, int nblocks,
    const fx_block_desc *blocks, const int32_t *votes, int capacity, FxAmrResult &res,
    std::string *err)
{
    res = FxAmrResult();
    res.blocks.assign(blocks, blocks + nblocks);
    const int nmax = std::min(capacity, amr.max_blocks > 0 ? amr.max_blocks : 65536);
    Mesh m{cfg, amr, res.blocks, nmax, err, false, false, {}};
    m.flag.assign(nblocks, 0);
    for (int i = 0; i < nblocks; ++i) {
        fx_block_desc &blk = res.blocks[i];
        if (blk.id >= 0 && blk.id != i) {
            if (err) *err = "block entry " + std::to_string(i) + " has id " + std::to_string(blk.id);
            return FX_EINVAL;
        }
    }

    m.tag(votes);
    res.flags.assign(m.flag.begin(), m.flag.end());
    m.two_to_one();
    if (!m.pending_change()) {
        return FX_SUCCESS;
    }

    /* refinement in block order; the children are appended or take freed
     * entries and are visited by the same loop (with flag 0) */
    std::vector<char> dirty((size_t)std::max(nmax, nblocks), 0);
    bool refined = false;
    m.flag.resize(dirty.size(), 0);
    for (int i = 0; i < m.nblocks(); ++i) {
        if (!(is_active(res.blocks[i]) && m.flag[i] > 0 && res.blocks[i].can_refine != 0)) continue;
        const int was_active = res.blocks[i].active;
        m.mark_dirty_and_neighbors(i, dirty);
        const size_t first = res.refine.size();
        if (!m.refine_block(i, res.refine, dirty)) {
            if (err) {
                *err = "block capacity exceeded (nblocks=" + std::to_string(m.nblocks()) +
                    " >= max_blocks=" + std::to_string(nmax) + ")";
            }
            return FX_ETOOBIG;
        }
        dirty[i] = 1;
        for (size_t j = first; j < res.refine.size(); ++j) dirty[res.refine[j].child] = 1;
        if (was_active != res.blocks[i].active) refined = true;
    }
    m.flag.resize((size_t)m.nblocks());
    if (refined) {
        m.init_neighbors(dirty);
        std::fill(dirty.begin(), dirty.end(), 0);
    }

    bool coarsened = false;
    for (int i = 0; i < m.nblocks(); ++i) {
        if (res.blocks[i].id < 0 || res.blocks[i].active == 1) continue;
        if (!m.can_coarsen(i)) continue;
        dirty[i] = 1;
        for (int oct = 0; oct < 8; ++oct) m.mark_dirty_and_neighbors(res.blocks[i].children[oct], dirty);
        m.coarsen_block(i, res.coarsen);
        dirty[i] = 1;
        coarsened = true;
    }
    if (coarsened) {
        m.init_neighbors(dirty);
    }
    if (m.overflow || m.geom_error) {
        if (err) *err = m.overflow ? "more than 56 neighbours" : "neighbour level jump larger than one";
        return FX_EINVAL;
    }
    if (!refined && !coarsened) {
        res.refine.clear();
        return FX_SUCCESS;
    }
    for (fx_block_desc &blk : res.blocks) {
        if (blk.id >= 0) setup_geometry(blk);
    }
    res.changed = true;
    return FX_SUCCESS;
}
