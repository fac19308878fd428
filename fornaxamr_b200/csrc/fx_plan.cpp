/*
 * Ghost-fill compiler.
 *
 * prj_boundary_fill_ghosts_and_bf (reference src/prj_boundary.c:1150-1241) is
 * a fixed sequence of element copies, averages and prolongations whose
 * pattern depends only on the mesh topology, never on the data: the face
 * "fidelity" bookkeeping that decides whether a Bf write lands
 * (src/prj_boundary.c:599-625) is itself data independent.  This file replays
 * that sequence once on the host, in the reference's exact loop order, and
 * records every write that lands as an element operation.  Then:
 *
 *  1. copy propagation: a single-source operation whose source currently
 *     holds a value produced by a plain copy (whose own source is unchanged
 *     since) reads that earlier source instead; chains collapse to their root;
 *  2. dead-write elimination: an operation whose result is overwritten
 *     before anything reads it is dropped;
 *  3. the closing prj_mhd_bf2bc_all_mesh pass (src/prj_boundary.c:1235-1239)
 *     becomes one operation per cell whose field may change (every ghost cell,
 *     and interior cells with a rewritten face), reading the final faces
 *     through the same copy chains;
 *  4. levelling: an operation is placed one wave after the latest earlier
 *     operation it conflicts with (read-after-write, write-after-read or
 *     write-after-write on any element), so each wave is free of conflicts and
 *     running the waves in order reproduces the sequential result, including
 *     which of several overlapping writers wins.
 *
 * Cell operations carry the primitive variables 0..5 only.  In an MHD run
 * the cell-centred field of every one of the 20^3 cells is rewritten from the
 * faces at the end of the fill and every ghost operation is variable-wise, so
 * the field components of the cell operations are dead; interior cells whose
 * faces the fill does not touch already hold the face average from the cell
 * update.  eosvar is not transferred: for the ideal gas it is a pointwise
 * function of W, and the reference's fill leaves eosvar == eos(W) in every
 * cell.
 */
#include "fx_plan.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

enum { KIND_SAME = 3, KIND_RESTRICT = 4, KIND_PROLONG = 5 };
enum { PHYS_FACE_ONLY = 0, PHYS_EDGE_CORNER = 2 };
enum { FID_NONE = 0, FID_COARSER = 1, FID_SAME = 2, FID_FINER = 3 };
enum { SPACE_CELL = 0, SPACE_FACE = 1 };

const int BS = FX_BS;
const int NG = FX_NG;

inline int lidx(int i, int j, int k) { return fx_lidx(i, j, k); }
inline int fidx(int dir, int i, int j, int k) { return fx_face_idx(dir, i, j, k); }

bool active_block(const fx_block_desc &b) { return b.id >= 0 && b.active == 1 && b.rank == 0; }

/* face storage bounds, src/prj_boundary.c:556-568 */
bool face_storage_ok(int dir, const int idx[3])
{
    for (int d = 0; d < 3; ++d) {
        const int hi = dir == d ? BS + NG : BS + NG - 1;
        if (idx[d] < -NG || idx[d] > hi) {
            return false;
        }
    }
    return true;
}

/* active faces, src/prj_boundary.c:575-590 */
bool face_active(int dir, int i, int j, int k)
{
    const int idx[3] = {i, j, k};
    for (int d = 0; d < 3; ++d) {
        const int hi = dir == d ? BS : BS - 1;
        if (idx[d] < 0 || idx[d] > hi) {
            return false;
        }
    }
    return true;
}

/* one landed write of the reference sequence */
struct SeqOp {
    FxGop op;
    int64_t w;         /* element written */
    int64_t src;       /* single source element, -1 for multi-source ops */
    int src_ver;       /* producer of the source value (op index, -1 initial) */
    int space;
    int prod_begin;    /* producers of the values read: [prod_begin, prod_end) */
    int prod_end;
};

class Compiler {
public:
    Compiler(const fx_config &cfg, int nblocks, const fx_block_desc *blocks)
        : cfg_(cfg), n_(nblocks), b_(blocks),
          ncell_((int64_t)nblocks * FX_NCELLS),
          nface_((int64_t)(cfg.mhd ? nblocks : 0) * 3 * FX_NFACES),
          fid_((size_t)nface_, 0),
          ver_((size_t)(2 * ncell_ + nface_), -1)
    {
    }

    bool run(FxPlan &plan, std::string *err)
    {
        err_ = err;
        for (int b = 0; b < n_; ++b) {
            if (active_block(b_[b])) {
                plan.active.push_back(b);
            }
        }
        if (!validate()) {
            return false;
        }
        /* the reference sequence */
        for (int b : plan.active) {
            physical(b, PHYS_FACE_ONLY);
        }
        if (cfg_.mhd) {
            for (int b : plan.active) {
                init_fidelity(b);
            }
            for (int b : plan.active) {
                if (!physical_bf(b)) return false;
            }
        }
        const int passes[3] = {KIND_SAME, KIND_RESTRICT, KIND_PROLONG};
        for (int kind : passes) {
            for (int b : plan.active) {
                if (!send_cells(b, kind)) return false;
            }
            if (cfg_.mhd) {
                for (int b : plan.active) {
                    if (!send_faces(b, kind)) return false;
                }
            }
        }
        for (int b : plan.active) {
            physical(b, PHYS_EDGE_CORNER);
        }
        if (cfg_.mhd) {
            for (int b : plan.active) {
                if (!physical_bf(b)) return false;
            }
        }
        finish(plan);
        return true;
    }

private:
    bool fail(const char *msg)
    {
        if (err_) *err_ = msg;
        return false;
    }

    bool validate()
    {
        for (int b = 0; b < n_; ++b) {
            if (!active_block(b_[b])) continue;
            for (int s = 0; s < FX_NSLOTS; ++s) {
                const fx_slot &sl = b_[b].slot[s];
                if (sl.id < 0 || sl.id >= n_ || !active_block(b_[sl.id])) continue;
                if (sl.rel_level < -1 || sl.rel_level > 1) {
                    return fail("slot rel_level outside [-1, 1] (the reference aborts: slot->rel_level unrecognized)");
                }
                if (sl.rel_level != 0) {
                    return fail("coarse/fine neighbours need the AMR transfer programs, not built in this version");
                }
            }
        }
        return true;
    }

    int64_t cell_elem(int b, int c) const { return (int64_t)b * FX_NCELLS + c; }
    int64_t cellb_elem(int b, int c) const { return ncell_ + (int64_t)b * FX_NCELLS + c; }
    int64_t face_elem(int b, int dir, int f) const { return 2 * ncell_ + ((int64_t)b * 3 + dir) * FX_NFACES + f; }

    /* ---- recording -------------------------------------------------------- */

    bool is_plain_copy(const SeqOp &o) const
    {
        return (o.space == SPACE_CELL && o.op.type == FX_GOP_COPY) ||
            (o.space == SPACE_FACE && o.op.type == FX_FOP_COPY);
    }

    /* follow plain-copy producers back to the oldest element that still
     * holds the same value; returns the element and its producer */
    void resolve(int64_t &e, int &v, long long *count) const
    {
        while (v >= 0) {
            const SeqOp &p = seq_[v];
            if (!is_plain_copy(p) || ver_[p.src] != p.src_ver) {
                break;
            }
            e = p.src;
            v = p.src_ver;
            if (count) ++*count;
        }
    }

    static int32_t cell_key(int64_t e) { return (int32_t)(((e / FX_NCELLS) << 13) | (e % FX_NCELLS)); }

    int32_t face_key(int64_t e) const
    {
        const int64_t r = e - 2 * ncell_;
        const int64_t bd = r / FX_NFACES;
        return (int32_t)(((bd / 3) << 15) | (r % FX_NFACES));
    }

    void add_single(FxGop op, int space, int64_t src, int64_t w)
    {
        SeqOp s;
        int v = ver_[src];
        resolve(src, v, &stats_.rewired);
        op.src = space == SPACE_CELL ? cell_key(src) : face_key(src);
        s.op = op;
        s.w = w;
        s.src = src;
        s.src_ver = v;
        s.space = space;
        s.prod_begin = (int)prod_.size();
        prod_.push_back(v);
        s.prod_end = (int)prod_.size();
        rd_.push_back(src);
        seq_.push_back(s);
        ver_[w] = (int)seq_.size() - 1;
    }

    void add_multi(FxGop op, int space, const int64_t *reads, int nr, int64_t w)
    {
        SeqOp s;
        s.op = op;
        s.w = w;
        s.src = -1;
        s.src_ver = -1;
        s.space = space;
        s.prod_begin = (int)prod_.size();
        for (int n = 0; n < nr; ++n) {
            prod_.push_back(ver_[reads[n]]);
            rd_.push_back(reads[n]);
        }
        s.prod_end = (int)prod_.size();
        seq_.push_back(s);
        ver_[w] = (int)seq_.size() - 1;
    }

    bool on_side(const fx_block_desc &blk, int axis, int side) const
    {
        const double tol = 1.0e-12;
        if (side == 0) {
            return std::fabs(blk.xmin[axis] - cfg_.coord[2 * axis]) < tol;
        }
        return std::fabs(blk.xmax[axis] - cfg_.coord[2 * axis + 1]) < tol;
    }

    /* prj_boundary_physical + prj_boundary_apply_axis_band
     * (src/prj_boundary.c:413-530) */
    void physical(int b, int mode)
    {
        const int npass = mode == PHYS_FACE_ONLY ? 1 : 3;
        for (int pass = 0; pass < npass; ++pass) {
            for (int axis = 0; axis < 3; ++axis) {
                for (int side = 0; side < 2; ++side) {
                    if (on_side(b_[b], axis, side)) {
                        band(b, axis, side, cfg_.bc[2 * axis + side], mode);
                    }
                }
            }
        }
    }

    void band(int b, int axis, int side, int bc, int region)
    {
        if (bc == FX_BC_PERIODIC) {
            return;
        }
        const int a1 = (axis + 1) % 3;
        const int a2 = (axis + 2) % 3;
        const int n_lo = side == 0 ? -NG : BS;
        const int n_hi = side == 0 ? 0 : BS + NG;
        const int t_lo = region == PHYS_FACE_ONLY ? 0 : -NG;
        const int t_hi = region == PHYS_FACE_ONLY ? BS : BS + NG;
        for (int a = n_lo; a < n_hi; ++a) {
            const int src_a = side == 0 ? -a - 1 : 2 * BS - 1 - a;
            for (int t1 = t_lo; t1 < t_hi; ++t1) {
                for (int t2 = t_lo; t2 < t_hi; ++t2) {
                    if (region == PHYS_EDGE_CORNER && t1 >= 0 && t1 < BS && t2 >= 0 && t2 < BS) {
                        continue;
                    }
                    int idx[3], src[3];
                    idx[axis] = a;
                    idx[a1] = t1;
                    idx[a2] = t2;
                    src[axis] = src_a;
                    src[a1] = t1;
                    src[a2] = t2;
                    const int dc = lidx(idx[0], idx[1], idx[2]);
                    const int sc = lidx(src[0], src[1], src[2]);
                    FxGop op;
                    op.dst = FX_CELL_KEY(b, dc);
                    if (bc == FX_BC_REFLECT) {
                        op.type = FX_GOP_COPY_NEG;
                        op.aux = FX_V1 + axis;
                    } else if (bc == FX_BC_USER) {
                        op.type = FX_GOP_COPY_USER;
                        op.aux = (axis == 0 && side == 0) ? 1 : 0;
                    } else {
                        op.type = FX_GOP_COPY;
                        op.aux = 0;
                    }
                    add_single(op, SPACE_CELL, cell_elem(b, sc), cell_elem(b, dc));
                }
            }
        }
    }

    /* prj_boundary_send (src/prj_boundary.c:190-399), cell part */
    bool send_cells(int b, int kind)
    {
        for (int n = 0; n < FX_NSLOTS; ++n) {
            const fx_slot &sl = b_[b].slot[n];
            const int id = sl.id;
            if (id < 0 || id >= n_ || !active_block(b_[id])) {
                continue;
            }
            const int sk = sl.rel_level == 0 ? KIND_SAME : sl.rel_level < 0 ? KIND_RESTRICT : KIND_PROLONG;
            if (sk != kind) {
                continue;
            }
            const int ni = sl.recv_loc_end[0] - sl.recv_loc_start[0];
            const int nj = sl.recv_loc_end[1] - sl.recv_loc_start[1];
            const int nk = sl.recv_loc_end[2] - sl.recv_loc_start[2];
            for (int i = 0; i < ni; ++i) {
                for (int j = 0; j < nj; ++j) {
                    for (int k = 0; k < nk; ++k) {
                        const int ai = i + sl.recv_loc_start[0];
                        const int aj = j + sl.recv_loc_start[1];
                        const int ak = k + sl.recv_loc_start[2];
                        const int dc = lidx(ai, aj, ak);
                        FxGop op;
                        op.dst = FX_CELL_KEY(id, dc);
                        op.aux = 0;
                        if (sl.rel_level == 0) {
                            const int sc = lidx(i + sl.send_loc_start[0], j + sl.send_loc_start[1],
                                k + sl.send_loc_start[2]);
                            op.type = FX_GOP_COPY;
                            add_single(op, SPACE_CELL, cell_elem(b, sc), cell_elem(id, dc));
                        } else if (sl.rel_level == -1) {
                            const int si = 2 * i + sl.send_loc_start[0];
                            const int sj = 2 * j + sl.send_loc_start[1];
                            const int sk2 = 2 * k + sl.send_loc_start[2];
                            op.src = FX_CELL_KEY(b, lidx(si, sj, sk2));
                            op.type = FX_GOP_RESTRICT;
                            int64_t r[8];
                            int q = 0;
                            for (int di = 0; di < 2; ++di)
                                for (int dj = 0; dj < 2; ++dj)
                                    for (int dk = 0; dk < 2; ++dk)
                                        r[q++] = cell_elem(b, lidx(si + di, sj + dj, sk2 + dk));
                            add_multi(op, SPACE_CELL, r, 8, cell_elem(id, dc));
                        } else {
                            const int ci = i / 2 + sl.send_loc_start[0];
                            const int cj = j / 2 + sl.send_loc_start[1];
                            const int ck = k / 2 + sl.send_loc_start[2];
                            op.src = FX_CELL_KEY(b, lidx(ci, cj, ck));
                            op.type = FX_GOP_PROLONG;
                            /* target offsets: (index % 2 == 0) ? -0.25 : +0.25 in C
                             * semantics (src/prj_boundary.c:318-320) */
                            op.aux = ((ai % 2 == 0) ? 0 : 4) | ((aj % 2 == 0) ? 0 : 2) | ((ak % 2 == 0) ? 0 : 1);
                            int64_t r[27];
                            int q = 0;
                            for (int di = -1; di <= 1; ++di)
                                for (int dj = -1; dj <= 1; ++dj)
                                    for (int dk = -1; dk <= 1; ++dk)
                                        r[q++] = cell_elem(b, lidx(ci + di, cj + dj, ck + dk));
                            add_multi(op, SPACE_CELL, r, 27, cell_elem(id, dc));
                        }
                    }
                }
            }
        }
        return true;
    }

    /* ---- face field ------------------------------------------------------ */

    int &fid(int b, int dir, int f) { return fid_[((int64_t)b * 3 + dir) * FX_NFACES + f]; }

    /* prj_boundary_init_face_fidelity, src/prj_boundary.c:840-873 */
    void init_fidelity(int b)
    {
        for (int dir = 0; dir < 3; ++dir) {
            for (int f = 0; f < FX_NFACES; ++f) {
                fid(b, dir, f) = FID_NONE;
            }
            for (int i = 0; i <= (dir == 0 ? BS : BS - 1); ++i)
                for (int j = 0; j <= (dir == 1 ? BS : BS - 1); ++j)
                    for (int k = 0; k <= (dir == 2 ? BS : BS - 1); ++k)
                        fid(b, dir, fidx(dir, i, j, k)) = FID_SAME;
        }
    }

    /* prj_boundary_write_bf_face, src/prj_boundary.c:599-625: a write lands
     * when its fidelity is at least the face's current fidelity. */
    bool lands(int db, int dir, int df, int fidelity)
    {
        int &cur = fid(db, dir, df);
        if (fidelity < cur) {
            return false;
        }
        if (fidelity > cur) {
            cur = fidelity;
        }
        return true;
    }

    /* prj_boundary_physical_bf + prj_boundary_apply_bf_axis
     * (src/prj_boundary.c:883-957) */
    bool physical_bf(int b)
    {
        for (int pass = 0; pass < 3; ++pass) {
            for (int axis = 0; axis < 3; ++axis) {
                for (int side = 0; side < 2; ++side) {
                    if (!on_side(b_[b], axis, side)) continue;
                    if (cfg_.bc[2 * axis + side] != FX_BC_OUTFLOW) {
                        return fail("prj_boundary_apply_bf_axis: only outflow magnetic-field boundary conditions are implemented");
                    }
                    bf_axis(b, axis, side);
                }
            }
        }
        return true;
    }

    void bf_axis(int b, int axis, int side)
    {
        for (int dir = 0; dir < 3; ++dir) {
            const int max_axis = dir == axis ? BS : BS - 1;
            for (int i = -NG; i < BS + NG; ++i) {
                for (int j = -NG; j < BS + NG; ++j) {
                    for (int k = -NG; k < BS + NG; ++k) {
                        const int idx[3] = {i, j, k};
                        int src[3] = {i, j, k};
                        if (side == 0) {
                            if (idx[axis] >= 0) continue;
                            src[axis] = 0;
                        } else {
                            if (idx[axis] <= max_axis) continue;
                            src[axis] = max_axis;
                        }
                        if (!face_storage_ok(dir, src)) continue;
                        const int sf = fidx(dir, src[0], src[1], src[2]);
                        const int fidelity = fid(b, dir, sf);
                        if (fidelity == FID_NONE) continue;
                        const int df = fidx(dir, i, j, k);
                        if (!lands(b, dir, df, fidelity)) continue;
                        FxGop op;
                        op.dst = (b << 15) | df;
                        op.aux = dir;
                        op.type = FX_FOP_COPY;
                        add_single(op, SPACE_FACE, face_elem(b, dir, sf), face_elem(b, dir, df));
                    }
                }
            }
        }
    }

    /* prj_boundary_send_bf (src/prj_boundary.c:997-1065) */
    bool send_faces(int b, int kind)
    {
        for (int n = 0; n < FX_NSLOTS; ++n) {
            const fx_slot &sl = b_[b].slot[n];
            const int id = sl.id;
            if (id < 0 || id >= n_ || !active_block(b_[id])) continue;
            if (kind == KIND_SAME && sl.rel_level == 0) {
                copy_same_level(b, id, sl);
            } else if (kind == KIND_RESTRICT && sl.rel_level < 0) {
                restrict_to_coarse(b, id, sl);
            } else if (kind == KIND_PROLONG && sl.rel_level > 0) {
                return fail("field prolongation to finer neighbours needs the AMR transfer programs");
            }
        }
        return true;
    }

    /* prj_boundary_copy_bf_same_level, src/prj_boundary.c:627-693.  The
     * reference buffers the source faces before writing; source and
     * destination are different blocks, so element operations are
     * equivalent. */
    void copy_same_level(int src_b, int dst_b, const fx_slot &sl)
    {
        for (int dir = 0; dir < 3; ++dir) {
            const int ni = sl.recv_loc_end[0] - sl.recv_loc_start[0] + (dir == 0 ? 1 : 0);
            const int nj = sl.recv_loc_end[1] - sl.recv_loc_start[1] + (dir == 1 ? 1 : 0);
            const int nk = sl.recv_loc_end[2] - sl.recv_loc_start[2] + (dir == 2 ? 1 : 0);
            for (int i = 0; i < ni; ++i) {
                for (int j = 0; j < nj; ++j) {
                    for (int k = 0; k < nk; ++k) {
                        const int ri = i + sl.recv_loc_start[0];
                        const int rj = j + sl.recv_loc_start[1];
                        const int rk = k + sl.recv_loc_start[2];
                        if (face_active(dir, ri, rj, rk)) continue;
                        const int sf = fidx(dir, i + sl.send_loc_start[0], j + sl.send_loc_start[1],
                            k + sl.send_loc_start[2]);
                        const int df = fidx(dir, ri, rj, rk);
                        if (!lands(dst_b, dir, df, FID_SAME)) continue;
                        FxGop op;
                        op.dst = (dst_b << 15) | df;
                        op.aux = dir;
                        op.type = FX_FOP_COPY;
                        add_single(op, SPACE_FACE, face_elem(src_b, dir, sf), face_elem(dst_b, dir, df));
                    }
                }
            }
        }
    }

    /* prj_boundary_restrict_bf_to_coarse, src/prj_boundary.c:695-773 */
    void restrict_to_coarse(int fine, int coarse, const fx_slot &sl)
    {
        for (int dir = 0; dir < 3; ++dir) {
            const int tan0 = (dir + 1) % 3;
            const int tan1 = (dir + 2) % 3;
            int e0[3] = {0, 0, 0};
            int e1[3] = {0, 0, 0};
            e0[tan0] = 1;
            e1[tan1] = 1;
            const int o0 = fidx(dir, e0[0], e0[1], e0[2]) - fidx(dir, 0, 0, 0);
            const int o1 = fidx(dir, e1[0], e1[1], e1[2]) - fidx(dir, 0, 0, 0);
            const int ni = sl.recv_loc_end[0] - sl.recv_loc_start[0] + (dir == 0 ? 1 : 0);
            const int nj = sl.recv_loc_end[1] - sl.recv_loc_start[1] + (dir == 1 ? 1 : 0);
            const int nk = sl.recv_loc_end[2] - sl.recv_loc_start[2] + (dir == 2 ? 1 : 0);
            for (int i = 0; i < ni; ++i) {
                for (int j = 0; j < nj; ++j) {
                    for (int k = 0; k < nk; ++k) {
                        const int s0 = fidx(dir, 2 * i + sl.send_loc_start[0], 2 * j + sl.send_loc_start[1],
                            2 * k + sl.send_loc_start[2]);
                        const int df = fidx(dir, i + sl.recv_loc_start[0], j + sl.recv_loc_start[1],
                            k + sl.recv_loc_start[2]);
                        if (!lands(coarse, dir, df, FID_FINER)) continue;
                        FxGop op;
                        op.dst = (coarse << 15) | df;
                        op.src = (fine << 15) | s0;
                        op.aux = dir | (o1 << 2) | (o0 << 12);
                        op.type = FX_FOP_RESTRICT;
                        const int64_t r[4] = {face_elem(fine, dir, s0), face_elem(fine, dir, s0 + o1),
                            face_elem(fine, dir, s0 + o0), face_elem(fine, dir, s0 + o0 + o1)};
                        add_multi(op, SPACE_FACE, r, 4, face_elem(coarse, dir, df));
                    }
                }
            }
        }
    }

    /* ---- optimisation and levelling -------------------------------------- */

    void finish(FxPlan &plan)
    {
        const int nseq = (int)seq_.size();
        /* 2. liveness in reverse order: final versions are live; an op is
         * live when a live op reads its value */
        std::vector<int> readers(nseq, 0);
        std::vector<char> live(nseq, 0);
        for (int x = nseq - 1; x >= 0; --x) {
            const SeqOp &o = seq_[x];
            if (seq_[x].space == SPACE_CELL) ++stats_.emitted_cell_ops;
            else ++stats_.emitted_face_ops;
            live[x] = (ver_[o.w] == x) || readers[x] > 0;
            if (!live[x]) {
                ++stats_.dead;
                continue;
            }
            for (int p = o.prod_begin; p < o.prod_end; ++p) {
                if (prod_[p] >= 0) ++readers[prod_[p]];
            }
        }
        /* 3. cell-field operations */
        std::vector<FxBop> bops;
        std::vector<std::array<int64_t, 6>> bop_reads;
        if (cfg_.mhd) {
            for (int b : plan.active) {
                for (int i = -NG; i < BS + NG; ++i) {
                    for (int j = -NG; j < BS + NG; ++j) {
                        for (int k = -NG; k < BS + NG; ++k) {
                            const bool ghost = i < 0 || i >= BS || j < 0 || j >= BS || k < 0 || k >= BS;
                            int64_t f[6] = {
                                face_elem(b, 0, fidx(0, i, j, k)), face_elem(b, 0, fidx(0, i + 1, j, k)),
                                face_elem(b, 1, fidx(1, i, j, k)), face_elem(b, 1, fidx(1, i, j + 1, k)),
                                face_elem(b, 2, fidx(2, i, j, k)), face_elem(b, 2, fidx(2, i, j, k + 1))};
                            bool touched = false;
                            for (int q = 0; q < 6; ++q) {
                                if (ver_[f[q]] >= 0) touched = true;
                            }
                            if (!ghost && !touched) continue;
                            FxBop bo;
                            bo.dst = FX_CELL_KEY(b, lidx(i, j, k));
                            bo.pad = 0;
                            std::array<int64_t, 6> rr;
                            for (int q = 0; q < 6; ++q) {
                                int v = ver_[f[q]];
                                int64_t e = f[q];
                                resolve(e, v, &stats_.rewired);
                                bo.f[q] = face_key(e);
                                rr[q] = e;
                            }
                            bops.push_back(bo);
                            bop_reads.push_back(rr);
                        }
                    }
                }
            }
        }
        /* 4. levelling over cell, cell-field and face elements */
        std::vector<int> lw((size_t)(2 * ncell_ + nface_), -1);
        std::vector<int> lr((size_t)(2 * ncell_ + nface_), -1);
        std::vector<std::vector<FxGop>> wc, wf;
        std::vector<std::vector<FxBop>> wb;
        auto place = [&](const int64_t *reads, int nr, int64_t w) {
            int wave = 0;
            for (int n = 0; n < nr; ++n) wave = std::max(wave, lw[reads[n]] + 1);
            wave = std::max(wave, lw[w] + 1);
            wave = std::max(wave, lr[w] + 1);
            for (int n = 0; n < nr; ++n) lr[reads[n]] = std::max(lr[reads[n]], wave);
            lw[w] = wave;
            if ((int)wc.size() <= wave) {
                wc.resize(wave + 1);
                wf.resize(wave + 1);
                wb.resize(wave + 1);
            }
            return wave;
        };
        for (int x = 0; x < nseq; ++x) {
            if (!live[x]) continue;
            const SeqOp &o = seq_[x];
            const int nr = o.prod_end - o.prod_begin;
            const int wave = place(&rd_[o.prod_begin], nr, o.w);
            (o.space == SPACE_CELL ? wc : wf)[wave].push_back(o.op);
        }
        for (size_t q = 0; q < bops.size(); ++q) {
            const int64_t w = cellb_elem(FX_CELL_BLOCK(bops[q].dst), FX_CELL_IDX(bops[q].dst));
            const int wave = place(bop_reads[q].data(), 6, w);
            wb[wave].push_back(bops[q]);
        }
        FxProgram &g = plan.ghost;
        auto by_type = [](const FxGop &a, const FxGop &b) {
            return a.type < b.type || (a.type == b.type && a.dst < b.dst);
        };
        for (size_t w = 0; w < wc.size(); ++w) {
            std::stable_sort(wc[w].begin(), wc[w].end(), by_type);
            std::stable_sort(wf[w].begin(), wf[w].end(), by_type);
            g.cell_begin.push_back((int)g.cell_ops.size());
            g.face_begin.push_back((int)g.face_ops.size());
            g.b_begin.push_back((int)g.b_ops.size());
            g.cell_ops.insert(g.cell_ops.end(), wc[w].begin(), wc[w].end());
            g.face_ops.insert(g.face_ops.end(), wf[w].begin(), wf[w].end());
            g.b_ops.insert(g.b_ops.end(), wb[w].begin(), wb[w].end());
        }
        g.cell_begin.push_back((int)g.cell_ops.size());
        g.face_begin.push_back((int)g.face_ops.size());
        g.b_begin.push_back((int)g.b_ops.size());
        plan.stats = stats_;
    }

    const fx_config &cfg_;
    int n_;
    const fx_block_desc *b_;
    int64_t ncell_;
    int64_t nface_;
    std::vector<int> fid_;
    std::vector<int> ver_;       /* element -> producer op (-1: initial value) */
    std::vector<SeqOp> seq_;
    std::vector<int> prod_;      /* producers of the values each op reads */
    std::vector<int64_t> rd_;    /* elements each op reads (parallel to prod_) */
    FxPlanStats stats_;
    std::string *err_ = nullptr;
};

} /* namespace */

bool fx_build_plan(const fx_config &cfg, int nblocks, const fx_block_desc *blocks,
    FxPlan &plan, std::string *err)
{
    plan = FxPlan();
    Compiler c(cfg, nblocks, blocks);
    return c.run(plan, err);
}
