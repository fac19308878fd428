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
#include <cstdlib>
#include <cstring>
#include <memory>
#include <thread>
#include <unordered_map>
#include <utility>

namespace {

/* worker threads for the data-parallel parts of the compiler */
int compile_threads()
{
    const unsigned n = std::thread::hardware_concurrency();
    return (int)std::max(1u, std::min(n, 32u));
}

/* runs fn(t) for t in [0, n) on n threads (the calling thread takes t = 0) */
template <typename F>
void parallel_for(int n, F fn);

/* stable sort of ops by destination key (keys are below 2^31; face keys
 * repeat across the three face directions): a parallel stable
 * most-significant pass on key >> 13 (the block, with two face bits), then
 * each bin stable-sorted on its own; tmp: room for n operations */
void sort_by_dst(FxGop *a, size_t n, int nt, FxGop *tmp)
{
    if (n < 2) return;
    uint32_t top = 0;
    for (size_t q = 0; q < n; ++q) top = std::max(top, (uint32_t)a[q].dst >> 13);
    const size_t nbins = (size_t)top + 1;
    nt = (int)std::max<size_t>(1, std::min<size_t>((size_t)nt, n / 65536 + 1));
    std::vector<size_t> cnt((size_t)nt * nbins, 0);
    auto chunk = [&](int t, size_t &lo, size_t &hi) {
        lo = n * (size_t)t / (size_t)nt;
        hi = n * (size_t)(t + 1) / (size_t)nt;
    };
    parallel_for(nt, [&](int t) {
        size_t lo, hi;
        chunk(t, lo, hi);
        size_t *c = cnt.data() + (size_t)t * nbins;
        for (size_t q = lo; q < hi; ++q) ++c[(uint32_t)a[q].dst >> 13];
    });
    /* exclusive offsets: bin-major, thread-minor (keeps the scatter stable) */
    std::vector<size_t> bin_begin(nbins + 1, 0);
    size_t run = 0;
    for (size_t bin = 0; bin < nbins; ++bin) {
        bin_begin[bin] = run;
        for (int t = 0; t < nt; ++t) {
            const size_t v = cnt[(size_t)t * nbins + bin];
            cnt[(size_t)t * nbins + bin] = run;
            run += v;
        }
    }
    bin_begin[nbins] = run;
    parallel_for(nt, [&](int t) {
        size_t lo, hi;
        chunk(t, lo, hi);
        size_t *c = cnt.data() + (size_t)t * nbins;
        for (size_t q = lo; q < hi; ++q) tmp[c[(uint32_t)a[q].dst >> 13]++] = a[q];
    });
    parallel_for(nt, [&](int t) {
        for (size_t bin = (size_t)t; bin < nbins; bin += (size_t)nt) {
            FxGop *x = tmp + bin_begin[bin];
            const size_t m = bin_begin[bin + 1] - bin_begin[bin];
            std::stable_sort(x, x + m, [](const FxGop &u, const FxGop &v) { return u.dst < v.dst; });
            std::memcpy(a + bin_begin[bin], x, m * sizeof(FxGop));
        }
    });
}

/* runs fn(t) for t in [0, n) on n threads (the calling thread takes t = 0) */
template <typename F>
void parallel_for(int n, F fn)
{
    std::vector<std::thread> th;
    for (int t = 1; t < n; ++t) th.emplace_back(fn, t);
    fn(0);
    for (auto &x : th) x.join();
}

enum { KIND_SAME = 3, KIND_RESTRICT = 4, KIND_PROLONG = 5 };
enum { PHYS_FACE_ONLY = 0, PHYS_EDGE_CORNER = 2 };
enum { FID_NONE = 0, FID_COARSER = 1, FID_SAME = 2, FID_FINER = 3 };
enum { SPACE_CELL = 0, SPACE_FACE = 1, SPACE_GROUP = 2 };

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

/* cell storage bounds, src/prj_boundary.c:62-64 */
bool cell_in_storage(int i, int j, int k)
{
    return i >= -NG && i < BS + NG && j >= -NG && j < BS + NG && k >= -NG && k < BS + NG;
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

/* one operation of the reference sequence: a landed write, or one
 * face-prolongation group (several writes) */
struct SeqOp {
    FxGop op;          /* SPACE_GROUP: op.dst indexes the group table */
    int32_t src_ver;   /* single-source ops: producer of the source value (op index, -1 initial) */
    int32_t prod_begin; /* producers of the values read: [prod_begin, next op's prod_begin) */
    int32_t w_begin;   /* elements written: [w_begin, next op's w_begin) of the write list */
    int32_t space;
};

/* element ids: cells, cell fields and faces of all blocks in one space */
using Elem = uint32_t;

/* an allocator whose resize leaves new elements uninitialised, so that the
 * threads which fill a grown buffer are the first to touch its pages */
template <class T>
struct UninitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <class U>
    UninitAlloc(const UninitAlloc<U> &) noexcept {}
    template <class U, class... A>
    void construct(U *p, A &&...a)
    {
        if constexpr (sizeof...(A) == 0) {
            ::new ((void *)p) U;
        } else {
            ::new ((void *)p) U(std::forward<A>(a)...);
        }
    }
};
template <class T>
using Buf = std::vector<T, UninitAlloc<T>>;

/* operations recorded by one worker thread of a parallel replay phase,
 * merged into the sequence afterwards (indices relative to these vectors) */
struct Rec {
    Buf<SeqOp> seq;
    Buf<int> prod;
    Buf<Elem> rd;
    Buf<Elem> wr;
    long long rewired = 0;
};

/* map from a face element (ids in [base, base + n)) to the signature of the
 * value a face-prolongation group stored there: a direct index per element
 * into the list of signatures.  The index array comes from calloc, so only
 * the pages of elements that groups write are ever touched (a 2864-block
 * mesh has 72 M face elements, of which about 1.5 M get a signature). */
template <typename V>
class FaceIndexMap {
public:
    void init(int64_t base, int64_t n)
    {
        base_ = base;
        n_ = n;
        idx_.reset(static_cast<int32_t *>(std::calloc((size_t)std::max<int64_t>(n, 1), sizeof(int32_t))));
        vals_.clear();
    }
    bool ok() const { return (bool)idx_; }
    V *find(int64_t key)
    {
        const int32_t q = idx_.get()[key - base_];
        return q ? &vals_[(size_t)q - 1] : nullptr;
    }
    void put(int64_t key, const V &v)
    {
        int32_t &q = idx_.get()[key - base_];
        if (q) {
            vals_[(size_t)q - 1] = v;
            return;
        }
        vals_.push_back(v);
        q = (int32_t)vals_.size();
    }

private:
    struct Free {
        void operator()(int32_t *p) const { std::free(p); }
    };
    int64_t base_ = 0;
    int64_t n_ = 0;
    std::unique_ptr<int32_t, Free> idx_;
    std::vector<V> vals_;
};

/* what a prolonged outer face was computed from: a recomputation with the
 * same coarse face, target and stencil versions stores the same value */
struct ProlongSig {
    int op;            /* the group that stored it */
    int64_t coarse_face;
    int target;
    int ver[9];        /* stencil versions: 5 (minmod cross) or 9 (Barth-Jespersen 3x3) */
};

} /* namespace */

struct FxPlanWorkspace {
    std::vector<int8_t> fid;
    std::vector<int> ver;
    Buf<SeqOp> seq;
    Buf<int> prod;
    Buf<Elem> rd, wr;
    std::vector<int16_t> lw, lr;
    std::vector<Rec> recs;                                   /* parallel replay passes */
    std::vector<Buf<std::pair<int16_t, FxBop>>> bparts;      /* cell-field operations per thread */
    Buf<FxGop> sort_tmp;                                     /* sort_by_dst scratch */
    FxProgram spare;                                         /* arrays of a retired plan */
};

namespace {

class Compiler {
public:
    Compiler(const fx_config &cfg, int nblocks, const fx_block_desc *blocks, FxPlanWorkspace *ws = nullptr)
        : cfg_(cfg), n_(nblocks), b_(blocks),
          ncell_((int64_t)nblocks * FX_NCELLS),
          nface_((int64_t)(cfg.mhd ? nblocks : 0) * 3 * FX_NFACES), ws_(ws)
    {
        if (ws_) {
            borrow();
            seq_.clear();
            prod_.clear();
            rd_.clear();
            wr_.clear();
        }
    }
    ~Compiler()
    {
        if (ws_) borrow();  /* the buffers go back, their memory kept */
    }
    Compiler(const Compiler &) = delete;
    Compiler &operator=(const Compiler &) = delete;

    /* the coarse/fine correction records only (no ghost-fill replay) */
    bool run_corrections(FxPlan &plan, std::string *err)
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
        flux_corrections(plan);
        if (cfg_.mhd) {
            emf_corrections(plan);
        } else {
            plan.emf_corr_begin.assign(1, 0);
        }
        return true;
    }

    /* sharded compile: owner[b] is the rank of block b; run() then keeps
     * rank `rank`'s part of the plan */
    void set_owners(const int *owner, int nranks, int rank)
    {
        owner_ = owner;
        nranks_ = nranks;
        rank_ = rank;
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
        fid_.assign((size_t)nface_, 0);
        if (cfg_.mhd) {
            psig_.init(2 * ncell_, nface_);
            if (!psig_.ok()) {
                return fail("ghost-fill compiler: no host memory for the face-prolongation signatures");
            }
        }
        ver_.assign((size_t)(2 * ncell_ + nface_), -1);
        /* the replay records about 36000 operations per block with a field
         * (ghost cells, ghost faces, groups, and the writes later found
         * dead), 4000 without */
        const size_t est = plan.active.size() * (size_t)(cfg_.mhd ? 40000 : 4000);
        seq_.reserve(est);
        prod_.reserve(est + est / 4);
        rd_.reserve(est + est / 4);
        wr_.reserve(est + est / 16);
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
            if (kind != KIND_SAME || !same_pass_parallel(plan, false)) {
                for (int b : plan.active) {
                    if (!send_cells(b, kind)) return false;
                }
            }
            if (cfg_.mhd && (kind != KIND_SAME || !same_pass_parallel(plan, true))) {
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
        if (overflow_) {
            return fail("ghost fill needs more than 32766 waves");
        }
        flux_corrections(plan);
        if (cfg_.mhd) {
            emf_corrections(plan);
        } else {
            plan.emf_corr_begin.assign(1, 0);
        }
        if (owner_) {
            shard_records(plan.flux_corr, plan.flux_corr_begin, 4, finit_);
            shard_records(plan.emf_corr, plan.emf_corr_begin, 2, einit_);
            localize(plan);
        }
        return true;
    }

private:
    void borrow()
    {
        fid_.swap(ws_->fid);
        ver_.swap(ws_->ver);
        seq_.swap(ws_->seq);
        prod_.swap(ws_->prod);
        rd_.swap(ws_->rd);
        wr_.swap(ws_->wr);
        lw_.swap(ws_->lw);
        lr_.swap(ws_->lr);
    }

    bool fail(const char *msg)
    {
        if (err_) *err_ = msg;
        return false;
    }

    bool validate()
    {
        /* packed keys hold a block index below 2^16 (faces: block << 15),
         * element ids fit 32 bits */
        if (n_ > 65535 || (uint64_t)(2 * ncell_ + nface_) >= (1ULL << 32)) {
            return fail("mesh too large for the ghost-fill compiler (at most 65535 blocks)");
        }
        for (int b = 0; b < n_; ++b) {
            if (!active_block(b_[b])) continue;
            for (int s = 0; s < FX_NSLOTS; ++s) {
                const fx_slot &sl = b_[b].slot[s];
                if (sl.id < 0 || sl.id >= n_ || !active_block(b_[sl.id])) continue;
                if (sl.rel_level < -1 || sl.rel_level > 1) {
                    return fail("slot rel_level outside [-1, 1] (the reference aborts: slot->rel_level unrecognized)");
                }
            }
        }
        return true;
    }

    int64_t cell_elem(int b, int c) const { return (int64_t)b * FX_NCELLS + c; }
    int64_t face_elem(int b, int dir, int f) const { return 2 * ncell_ + ((int64_t)b * 3 + dir) * FX_NFACES + f; }
    int block_of(int64_t e) const
    {
        if (e < ncell_) return (int)(e / FX_NCELLS);
        if (e < 2 * ncell_) return (int)((e - ncell_) / FX_NCELLS);
        return (int)((e - 2 * ncell_) / (3 * FX_NFACES));
    }

    /* ---- recording -------------------------------------------------------- */

    int prod_end(int x) const
    {
        return x + 1 < (int)seq_.size() ? seq_[x + 1].prod_begin : (int)prod_.size();
    }

    int w_end(int x) const
    {
        return x + 1 < (int)seq_.size() ? seq_[x + 1].w_begin : (int)wr_.size();
    }

    /* source element of a single-source operation (from its packed key) */
    int64_t src_elem(const SeqOp &o) const
    {
        if (o.space == SPACE_CELL) {
            return cell_elem(FX_CELL_BLOCK(o.op.src), FX_CELL_IDX(o.op.src));
        }
        return face_elem(o.op.src >> 15, o.op.aux & 3, o.op.src & 32767);
    }

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
            if (!is_plain_copy(p)) {
                break;
            }
            const int64_t ps = src_elem(p);
            if (ver_[ps] != p.src_ver) {
                break;
            }
            e = ps;
            v = p.src_ver;
            if (count) ++*count;
        }
    }

    static int32_t cell_key(int64_t e) { return (int32_t)FX_CELL_KEY(e / FX_NCELLS, e % FX_NCELLS); }

    int32_t face_key(int64_t e) const
    {
        const int64_t r = e - 2 * ncell_;
        const int64_t bd = r / FX_NFACES;
        return (int32_t)(((bd / 3) << 15) | (r % FX_NFACES));
    }

    /* r != nullptr: record into a worker's buffer; the element versions are
     * set when the buffers are merged (parallel phases never read an element
     * they write) */
    void add_single(FxGop op, int space, int64_t src, int64_t w, Rec *r = nullptr)
    {
        SeqOp s;
        int v = ver_[src];
        resolve(src, v, r ? &r->rewired : &stats_.rewired);
        op.src = space == SPACE_CELL ? cell_key(src) : face_key(src);
        s.op = op;
        s.src_ver = v;
        s.space = space;
        Buf<SeqOp> &seq = r ? r->seq : seq_;
        Buf<int> &prod = r ? r->prod : prod_;
        Buf<Elem> &rd = r ? r->rd : rd_;
        Buf<Elem> &wr = r ? r->wr : wr_;
        s.prod_begin = (int)prod.size();
        prod.push_back(v);
        rd.push_back((Elem)src);
        s.w_begin = (int)wr.size();
        wr.push_back((Elem)w);
        seq.push_back(s);
        if (!r) ver_[w] = (int)seq_.size() - 1;
    }

    /* appends the workers' buffers in worker order and sets the versions of
     * the elements they wrote; workers own disjoint destination blocks, so
     * each copies its part and sets its versions in parallel */
    void merge(std::vector<Rec> &recs)
    {
        const int nr = (int)recs.size();
        std::vector<size_t> sb(nr + 1), pb(nr + 1), wb(nr + 1);
        sb[0] = seq_.size();
        pb[0] = prod_.size();
        wb[0] = wr_.size();
        for (int t = 0; t < nr; ++t) {
            sb[t + 1] = sb[t] + recs[t].seq.size();
            pb[t + 1] = pb[t] + recs[t].prod.size();
            wb[t + 1] = wb[t] + recs[t].wr.size();
            stats_.rewired += recs[t].rewired;
        }
        seq_.resize(sb[nr]);
        prod_.resize(pb[nr]);
        rd_.resize(pb[nr]);
        wr_.resize(wb[nr]);
        parallel_for(nr, [&](int t) {
            Rec &r = recs[t];
            std::copy(r.prod.begin(), r.prod.end(), prod_.begin() + pb[t]);
            std::copy(r.rd.begin(), r.rd.end(), rd_.begin() + pb[t]);
            std::copy(r.wr.begin(), r.wr.end(), wr_.begin() + wb[t]);
            for (size_t q = 0; q < r.seq.size(); ++q) {
                SeqOp x = r.seq[q];
                x.prod_begin += (int)pb[t];
                x.w_begin += (int)wb[t];
                seq_[sb[t] + q] = x;
                ver_[wr_[x.w_begin]] = (int)(sb[t] + q);
            }
            if (ws_) {
                r.seq.clear();
                r.prod.clear();
                r.rd.clear();
                r.wr.clear();
                r.rewired = 0;
            } else {
                r = Rec();
            }
        });
    }

    /* The SAME pass of cell sends (faces = false) or field sends (true) with
     * the work split by destination block: every operation writes a ghost
     * element of its destination and reads active elements that no ghost
     * operation writes, so operations into different destinations commute
     * and each destination keeps the reference's (source block, slot)
     * order. */
    /* true when every element a same-level slot copies from is active:
     * a copy writes only ghost cells or inactive faces, so no copy of the
     * pass then reads what another one writes */
    static bool same_sources_active(const fx_slot &sl, bool faces)
    {
        for (int dir = 0; dir < (faces ? 3 : 1); ++dir) {
            const int ext = faces ? 1 : 0;
            const int ni = sl.recv_loc_end[0] - sl.recv_loc_start[0] + (ext && dir == 0 ? 1 : 0);
            const int nj = sl.recv_loc_end[1] - sl.recv_loc_start[1] + (ext && dir == 1 ? 1 : 0);
            const int nk = sl.recv_loc_end[2] - sl.recv_loc_start[2] + (ext && dir == 2 ? 1 : 0);
            for (int i = 0; i < ni; ++i) {
                for (int j = 0; j < nj; ++j) {
                    for (int k = 0; k < nk; ++k) {
                        const int si = i + sl.send_loc_start[0];
                        const int sj = j + sl.send_loc_start[1];
                        const int sk = k + sl.send_loc_start[2];
                        if (!faces) {
                            if (si < 0 || si >= BS || sj < 0 || sj >= BS || sk < 0 || sk >= BS) return false;
                        } else if (!face_active(dir, i + sl.recv_loc_start[0], j + sl.recv_loc_start[1],
                                       k + sl.recv_loc_start[2]) && !face_active(dir, si, sj, sk)) {
                            return false;
                        }
                    }
                }
            }
        }
        return true;
    }

    /* returns false (nothing recorded) when a source may be written in the
     * pass; the caller then replays it in the reference's order */
    bool same_pass_parallel(const FxPlan &plan, bool faces)
    {
        std::vector<std::vector<std::pair<int, int>>> in(n_);
        long long work = 0;
        for (int b : plan.active) {
            for (int n = 0; n < FX_NSLOTS; ++n) {
                const fx_slot &sl = b_[b].slot[n];
                if (sl.id < 0 || sl.id >= n_ || !active_block(b_[sl.id]) || sl.rel_level != 0) continue;
                in[sl.id].emplace_back(b, n);
                ++work;
            }
        }
        std::vector<int> dests;
        for (int d : plan.active) {
            if (!in[d].empty()) dests.push_back(d);
        }
        const int nt = std::max(1, std::min(compile_threads(), (int)dests.size()));
        std::vector<char> ok(nt, 1);
        parallel_for(nt, [&](int t) {
            for (size_t q = (size_t)t; q < dests.size() && ok[t]; q += nt) {
                for (const auto &e : in[dests[q]]) {
                    if (!same_sources_active(b_[e.first].slot[e.second], faces)) {
                        ok[t] = 0;
                        break;
                    }
                }
            }
        });
        for (char c : ok) {
            if (!c) return false;
        }
        /* contiguous destination ranges of about equal slot counts */
        std::vector<size_t> cut(nt + 1, dests.size());
        cut[0] = 0;
        {
            long long acc = 0;
            int t = 1;
            for (size_t q = 0; q < dests.size() && t < nt; ++q) {
                acc += (long long)in[dests[q]].size();
                if (acc * nt >= work * t) cut[t++] = q + 1;
            }
        }
        std::vector<Rec> own;
        std::vector<Rec> &recs = ws_ ? ws_->recs : own;
        if ((int)recs.size() < nt) recs.resize(nt);
        for (Rec &r : recs) {
            r.seq.clear();
            r.prod.clear();
            r.rd.clear();
            r.wr.clear();
            r.rewired = 0;
        }
        parallel_for(nt, [&](int t) {
            Rec &r = recs[t];
            for (size_t q = cut[t]; q < cut[t + 1]; ++q) {
                const int d = dests[q];
                for (const auto &e : in[d]) {
                    const fx_slot &sl = b_[e.first].slot[e.second];
                    if (faces) {
                        copy_same_level(e.first, d, sl, &r);
                    } else {
                        cells_same_level(e.first, sl, &r);
                    }
                }
            }
        });
        merge(recs);
        return true;
    }

    void add_multi(FxGop op, int space, const int64_t *reads, int nr, int64_t w)
    {
        SeqOp s;
        s.op = op;
        s.src_ver = -1;
        s.space = space;
        s.prod_begin = (int)prod_.size();
        for (int n = 0; n < nr; ++n) {
            prod_.push_back(ver_[reads[n]]);
            rd_.push_back((Elem)reads[n]);
        }
        s.w_begin = (int)wr_.size();
        wr_.push_back((Elem)w);
        seq_.push_back(s);
        ver_[w] = (int)seq_.size() - 1;
    }

    /* one face-prolongation group: reads, then writes several faces */
    void add_group(const FxPop &p, const std::vector<int64_t> &reads, const std::vector<int64_t> &writes)
    {
        SeqOp s;
        s.op.dst = (int32_t)groups_.size();
        s.op.src = 0;
        s.op.aux = 0;
        s.op.type = FX_FOP_PROLONG;
        groups_.push_back(p);
        s.src_ver = -1;
        s.space = SPACE_GROUP;
        s.prod_begin = (int)prod_.size();
        for (int64_t r : reads) {
            prod_.push_back(ver_[r]);
            rd_.push_back((Elem)r);
        }
        s.w_begin = (int)wr_.size();
        for (int64_t w : writes) {
            wr_.push_back((Elem)w);
        }
        seq_.push_back(s);
        for (int64_t w : writes) {
            ver_[w] = (int)seq_.size() - 1;
        }
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

    /* the copies of one same-level slot of prj_boundary_send
     * (src/prj_boundary.c:270-285) */
    void cells_same_level(int b, const fx_slot &sl, Rec *r)
    {
        const int id = sl.id;
        const int ni = sl.recv_loc_end[0] - sl.recv_loc_start[0];
        const int nj = sl.recv_loc_end[1] - sl.recv_loc_start[1];
        const int nk = sl.recv_loc_end[2] - sl.recv_loc_start[2];
        for (int i = 0; i < ni; ++i) {
            for (int j = 0; j < nj; ++j) {
                for (int k = 0; k < nk; ++k) {
                    const int si = i + sl.send_loc_start[0];
                    const int sj = j + sl.send_loc_start[1];
                    const int sk = k + sl.send_loc_start[2];
                    const int dc = lidx(i + sl.recv_loc_start[0], j + sl.recv_loc_start[1], k + sl.recv_loc_start[2]);
                    FxGop op;
                    op.dst = FX_CELL_KEY(id, dc);
                    op.aux = 0;
                    op.type = FX_GOP_COPY;
                    add_single(op, SPACE_CELL, cell_elem(b, lidx(si, sj, sk)), cell_elem(id, dc), r);
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
            if (sk == KIND_SAME) {
                cells_same_level(b, sl, nullptr);
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
                        if (sl.rel_level == -1) {
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
                            op.type = cfg_.use_bj ? FX_GOP_PROLONG_BJ : FX_GOP_PROLONG;
                            /* target offsets: (index % 2 == 0) ? -0.25 : +0.25 in C
                             * semantics (src/prj_boundary.c:318-320) */
                            op.aux = ((ai % 2 == 0) ? 0 : 4) | ((aj % 2 == 0) ? 0 : 2) | ((ak % 2 == 0) ? 0 : 1);
                            /* the 27-cell stencil is range checked
                             * (src/prj_boundary.c:60-72); the minmod limiter
                             * reads the centre and its six axis neighbours,
                             * Barth-Jespersen all 27 cells */
                            if (!cell_in_storage(ci - 1, cj - 1, ck - 1) || !cell_in_storage(ci + 1, cj + 1, ck + 1)) {
                                return fail("prj_boundary_read_value: out-of-range access");
                            }
                            if (cfg_.use_bj) {
                                int64_t r[27];
                                int q = 0;
                                for (int di = -1; di <= 1; ++di)
                                    for (int dj = -1; dj <= 1; ++dj)
                                        for (int dk = -1; dk <= 1; ++dk)
                                            r[q++] = cell_elem(b, lidx(ci + di, cj + dj, ck + dk));
                                add_multi(op, SPACE_CELL, r, 27, cell_elem(id, dc));
                                continue;
                            }
                            const int64_t r[7] = {cell_elem(b, lidx(ci, cj, ck)),
                                cell_elem(b, lidx(ci - 1, cj, ck)), cell_elem(b, lidx(ci + 1, cj, ck)),
                                cell_elem(b, lidx(ci, cj - 1, ck)), cell_elem(b, lidx(ci, cj + 1, ck)),
                                cell_elem(b, lidx(ci, cj, ck - 1)), cell_elem(b, lidx(ci, cj, ck + 1))};
                            add_multi(op, SPACE_CELL, r, 7, cell_elem(id, dc));
                        }
                    }
                }
            }
        }
        return true;
    }

    /* ---- face field ------------------------------------------------------ */

    int8_t &fid(int b, int dir, int f) { return fid_[((int64_t)b * 3 + dir) * FX_NFACES + f]; }

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
        int8_t &cur = fid(db, dir, df);
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
                if (!prolong_to_fine(b, id, sl)) return false;
            }
        }
        return true;
    }

    /* prj_boundary_copy_bf_same_level, src/prj_boundary.c:627-693.  The
     * reference buffers the source faces before writing; source and
     * destination are different blocks, so element operations are
     * equivalent. */
    void copy_same_level(int src_b, int dst_b, const fx_slot &sl, Rec *r = nullptr)
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
                        const int si = i + sl.send_loc_start[0];
                        const int sj = j + sl.send_loc_start[1];
                        const int sk = k + sl.send_loc_start[2];
                        const int sf = fidx(dir, si, sj, sk);
                        const int df = fidx(dir, ri, rj, rk);
                        if (!lands(dst_b, dir, df, FID_SAME)) continue;
                        FxGop op;
                        op.dst = (dst_b << 15) | df;
                        op.aux = dir;
                        op.type = FX_FOP_COPY;
                        add_single(op, SPACE_FACE, face_elem(src_b, dir, sf), face_elem(dst_b, dir, df), r);
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

    /* prj_boundary_prolong_bf_to_fine (src/prj_boundary.c:781-838): one
     * Toth-Roe group per 2x2x2 fine cells of the receive box.  The
     * reference buffers the coarse faces first; only the fine block is
     * written, so reading them at group time is equivalent. */
    bool prolong_to_fine(int coarse, int fine, const fx_slot &sl)
    {
        const int ni = sl.recv_loc_end[0] - sl.recv_loc_start[0];
        const int nj = sl.recv_loc_end[1] - sl.recv_loc_start[1];
        const int nk = sl.recv_loc_end[2] - sl.recv_loc_start[2];
        for (int i = 0; i < ni; i += 2) {
            for (int j = 0; j < nj; j += 2) {
                for (int k = 0; k < nk; k += 2) {
                    const int f[3] = {i + sl.recv_loc_start[0], j + sl.recv_loc_start[1], k + sl.recv_loc_start[2]};
                    const int c[3] = {i / 2 + sl.send_loc_start[0], j / 2 + sl.send_loc_start[1],
                        k / 2 + sl.send_loc_start[2]};
                    if (!prolong_group(coarse, fine, c, f)) return false;
                }
            }
        }
        return true;
    }

    /* prj_mhd_prolong_bf_from_buffer (src/prj_mhd.c:374-512) as one group
     * operation: 24 outer faces prolonged from the coarse faces (or kept when
     * their fidelity is above COARSER), 12 inner faces from
     * prj_mhd_compute_buffer_inner_fluxes (src/prj_mhd.c:309-372) */
    bool prolong_group(int coarse, int fine, const int c[3], const int f[3])
    {
        for (int d = 0; d < 3; ++d) {
            /* fine cells f, f + 1 and the coarse stencil c - 1 .. c + 1 lie
             * in storage (the outer face f + 2 along d is then at most 18) */
            if (f[d] < -NG || f[d] + 1 > BS + NG - 1 || c[d] - 1 < -NG || c[d] + 1 > BS + NG - 1) {
                return fail("prj_mhd_prolong_bf_from_buffer: group outside face storage");
            }
        }
        FxPop p;
        std::memset(&p, 0, sizeof(p));
        p.fine = fine;
        p.coarse = coarse;
        p.pos = (f[0] + FX_NG) | ((f[1] + FX_NG) << 5) | ((f[2] + FX_NG) << 10) | ((c[0] + FX_NG) << 15) |
            ((c[1] + FX_NG) << 20) | ((c[2] + FX_NG) << 25);
        p.flags = cfg_.use_bj ? 1 : 0;
        std::vector<int64_t> &reads = g_reads_;
        std::vector<int64_t> &writes = g_writes_;
        std::vector<std::pair<int64_t, ProlongSig>> &sigs = g_sigs_;
        reads.clear();
        writes.clear();
        sigs.clear();
        const int op_index = (int)seq_.size();
        for (int d = 0; d < 3; ++d) {
            const int t0 = d == 0 ? 1 : 0;
            const int t1 = d == 2 ? 1 : 2;
            for (int side = 0; side < 2; ++side) {
                /* the coarse face and its four tangential neighbours (minmod),
                 * or the 3x3 tangential block about it (Barth-Jespersen), are
                 * the stencil of all four outer faces of this side */
                int y[3] = {c[0], c[1], c[2]};
                y[d] += side;
                const int64_t cf = face_elem(coarse, d, fidx(d, y[0], y[1], y[2]));
                int64_t ze[9];
                int zv[9];
                bool stencil_read = false;
                static const int cross[5][2] = {{0, 0}, {-1, 0}, {1, 0}, {0, -1}, {0, 1}};
                static const int box[9][2] = {{-1, -1}, {-1, 0}, {-1, 1}, {0, -1}, {0, 0}, {0, 1},
                    {1, -1}, {1, 0}, {1, 1}};
                const int nst = cfg_.use_bj ? 9 : 5;
                const int (*off)[2] = cfg_.use_bj ? box : cross;
                for (int n = 0; n < nst; ++n) {
                    int z[3] = {y[0], y[1], y[2]};
                    z[t0] += off[n][0];
                    z[t1] += off[n][1];
                    ze[n] = face_elem(coarse, d, fidx(d, z[0], z[1], z[2]));
                    zv[n] = ver_[ze[n]];
                }
                for (int a = 0; a < 2; ++a) {
                    for (int bb = 0; bb < 2; ++bb) {
                        const int q = 8 * d + 4 * side + 2 * a + bb;
                        int x[3] = {f[0], f[1], f[2]};
                        x[d] += 2 * side;
                        x[t0] += a;
                        x[t1] += bb;
                        const int xf = fidx(d, x[0], x[1], x[2]);
                        const int64_t xe = face_elem(fine, d, xf);
                        if (fid(fine, d, xf) > FID_COARSER) {
                            p.keep |= 1 << q;
                            reads.push_back(xe);
                            continue;
                        }
                        if (!stencil_read) {
                            for (int n = 0; n < nst; ++n) reads.push_back(ze[n]);
                            stencil_read = true;
                        }
                        ProlongSig sg;
                        sg.op = op_index;
                        sg.coarse_face = cf;
                        sg.target = 2 * a + bb;
                        for (int n = 0; n < 9; ++n) sg.ver[n] = n < nst ? zv[n] : -2;
                        fid(fine, d, xf) = FID_COARSER;
                        const ProlongSig *prev = psig_.find(xe);
                        if (prev != nullptr && same_sig(*prev, sg) && ver_[xe] == prev->op) {
                            continue; /* recomputes the value the face already holds */
                        }
                        p.owrite |= 1 << q;
                        writes.push_back(xe);
                        sigs.emplace_back(xe, sg);
                    }
                }
            }
        }
        for (int d = 0; d < 3; ++d) {
            const int t0 = d == 0 ? 1 : 0;
            const int t1 = d == 2 ? 1 : 2;
            for (int a = 0; a < 2; ++a) {
                for (int bb = 0; bb < 2; ++bb) {
                    int x[3] = {f[0], f[1], f[2]};
                    x[d] += 1;
                    x[t0] += a;
                    x[t1] += bb;
                    const int xf = fidx(d, x[0], x[1], x[2]);
                    if (!lands(fine, d, xf, FID_COARSER)) continue;
                    p.iwrite |= 1 << (4 * d + 2 * a + bb);
                    writes.push_back(face_elem(fine, d, xf));
                }
            }
        }
        std::sort(reads.begin(), reads.end());
        reads.erase(std::unique(reads.begin(), reads.end()), reads.end());
        add_group(p, reads, writes);
        for (auto &e : sigs) {
            psig_.put(e.first, e.second);
        }
        return true;
    }

    static bool same_sig(const ProlongSig &a, const ProlongSig &b)
    {
        if (a.coarse_face != b.coarse_face || a.target != b.target) return false;
        for (int n = 0; n < 9; ++n) {
            if (a.ver[n] != b.ver[n]) return false;
        }
        return true;
    }

    /* ---- coarse/fine corrections ------------------------------------------ */

    /* prj_riemann_face_axis (src/prj_riemann.c:1666-1698) */
    static int face_axis(const fx_block_desc &blk, const double smin[3], const double smax[3], int *side)
    {
        int axis = -1;
        int sd = -1;
        for (int d = 0; d < 3; ++d) {
            if (std::fabs(blk.xmax[d] - smin[d]) < 1.0e-12 * blk.dx[d]) {
                if (axis >= 0) return -1;
                axis = d;
                sd = 1;
            } else if (std::fabs(smax[d] - blk.xmin[d]) < 1.0e-12 * blk.dx[d]) {
                if (axis >= 0) return -1;
                axis = d;
                sd = 0;
            }
        }
        if (axis < 0) return -1;
        for (int d = 0; d < 3; ++d) {
            if (d == axis) continue;
            const double hi = blk.xmax[d] < smax[d] ? blk.xmax[d] : smax[d];
            const double lo = blk.xmin[d] > smin[d] ? blk.xmin[d] : smin[d];
            if (!(hi - lo > 1.0e-12)) return -1;
        }
        *side = sd;
        return axis;
    }

    /* prj_riemann_flux_send (src/prj_riemann.c:1700-1768): coarse face flux
     * <- 0.25 (f0 + f_tan0 + f_tan1 + f_both) of the four fine faces */
    void flux_corrections(FxPlan &plan)
    {
        const int nv = cfg_.mhd ? 9 : 6;
        std::vector<FxCorr> seq;
        std::vector<std::array<int64_t, 5>> el;
        for (int b : plan.active) {
            for (int n = 0; n < FX_NSLOTS; ++n) {
                const fx_slot &sl = b_[b].slot[n];
                if (sl.type != 1 || sl.rel_level >= 0) continue;
                const int nid = sl.id;
                if (nid < 0 || nid >= n_) continue;
                int side = -1;
                const int axis = face_axis(b_[b], b_[nid].xmin, b_[nid].xmax, &side);
                if (axis < 0) continue;
                const int tan0 = (axis + 1) % 3;
                const int tan1 = (axis + 2) % 3;
                const int n0 = sl.recv_loc_end[tan0] - sl.recv_loc_start[tan0];
                const int n1 = sl.recv_loc_end[tan1] - sl.recv_loc_start[tan1];
                for (int it0 = 0; it0 < n0; ++it0) {
                    for (int it1 = 0; it1 < n1; ++it1) {
                        int r[3], s0[3];
                        r[axis] = side == 1 ? 0 : BS;
                        r[tan0] = it0 + sl.recv_loc_start[tan0];
                        r[tan1] = it1 + sl.recv_loc_start[tan1];
                        s0[axis] = side == 1 ? BS : 0;
                        s0[tan0] = 2 * it0 + sl.send_loc_start[tan0];
                        s0[tan1] = 2 * it1 + sl.send_loc_start[tan1];
                        const int add[4][2] = {{0, 0}, {1, 0}, {0, 1}, {1, 1}};
                        FxCorr rec;
                        std::memset(&rec, 0, sizeof(rec));
                        std::array<int64_t, 5> e;
                        const size_t dbase = (size_t)axis * nv * FX_NCELLS;
                        rec.dst_block = nid;
                        rec.dst = (int32_t)(dbase + fx_bidx(nv, 0, r[0], r[1], r[2]));
                        rec.src_block = b;
                        e[0] = ((int64_t)nid * 3 + axis) * FX_NCELLS + lidx(r[0], r[1], r[2]);
                        for (int q = 0; q < 4; ++q) {
                            int x[3] = {s0[0], s0[1], s0[2]};
                            x[tan0] += add[q][0];
                            x[tan1] += add[q][1];
                            rec.src[q] = (int32_t)(dbase + fx_bidx(nv, 0, x[0], x[1], x[2]));
                            e[1 + q] = ((int64_t)b * 3 + axis) * FX_NCELLS + lidx(x[0], x[1], x[2]);
                        }
                        seq.push_back(rec);
                        el.push_back(e);
                    }
                }
            }
        }
        level_records(seq, el, 4, plan.flux_corr, plan.flux_corr_begin);
    }

    /* prj_mhd_emf_send + prj_mhd_restrict_emf_to_coarse
     * (src/prj_mhd.c:1003-1029, 853-965): coarse edge EMF <- 0.5 (sum of the
     * two fine edges along it).  Every write carries fidelity FINER, the
     * highest, so every write lands; the last writer of an edge wins. */
    void emf_corrections(FxPlan &plan)
    {
        std::vector<FxCorr> seq;
        std::vector<std::array<int64_t, 5>> el;
        for (int b : plan.active) {
            for (int n = 0; n < FX_NSLOTS; ++n) {
                const fx_slot &sl = b_[b].slot[n];
                const int nid = sl.id;
                if (nid < 0 || nid >= n_ || sl.rel_level >= 0) continue;
                if (!active_block(b_[nid])) continue;
                restrict_emf(b, nid, seq, el);
            }
        }
        level_records(seq, el, 2, plan.emf_corr, plan.emf_corr_begin);
    }

    void restrict_emf(int fb, int cb, std::vector<FxCorr> &seq, std::vector<std::array<int64_t, 5>> &el)
    {
        const fx_block_desc &fine = b_[fb];
        const fx_block_desc &coarse = b_[cb];
        int axis[3];
        int touch = 0;
        for (int d = 0; d < 3; ++d) {
            if (std::fabs(fine.xmax[d] - coarse.xmin[d]) < 1.0e-12 * fine.dx[d]) {
                axis[d] = 1;
                ++touch;
            } else if (std::fabs(coarse.xmax[d] - fine.xmin[d]) < 1.0e-12 * fine.dx[d]) {
                axis[d] = -1;
                ++touch;
            } else {
                axis[d] = 0;
            }
        }
        if (touch == 0 || touch > 2) return;
        int it_send[3] = {-100, -100, -100};
        int it_recv[3] = {-100, -100, -100};
        for (int d = 0; d < 3; ++d) {
            if (axis[d] == 1) {
                it_send[d] = BS;
                it_recv[d] = 0;
            }
            if (axis[d] == -1) {
                it_send[d] = 0;
                it_recv[d] = BS;
            }
        }
        auto emit = [&](int dir, const int snd0[3], const int snd1[3], const int rcv[3]) {
            FxCorr rec;
            std::memset(&rec, 0, sizeof(rec));
            rec.dst_block = cb;
            rec.dst = dir * FX_NEDGES + fx_edge_idx(dir, rcv[0], rcv[1], rcv[2]);
            rec.src_block = fb;
            rec.src[0] = dir * FX_NEDGES + fx_edge_idx(dir, snd0[0], snd0[1], snd0[2]);
            rec.src[1] = dir * FX_NEDGES + fx_edge_idx(dir, snd1[0], snd1[1], snd1[2]);
            std::array<int64_t, 5> e;
            e[0] = (int64_t)cb * FX_EMF_COUNT + rec.dst;
            e[1] = (int64_t)fb * FX_EMF_COUNT + rec.src[0];
            e[2] = (int64_t)fb * FX_EMF_COUNT + rec.src[1];
            e[3] = e[4] = -1;
            seq.push_back(rec);
            el.push_back(e);
        };
        for (int dir = 0; dir < 3; ++dir) {
            if (axis[dir] != 0) continue;
            const int i_offset =
                (fine.xmin[dir] + fine.xmax[dir]) < (coarse.xmin[dir] + coarse.xmax[dir]) ? 0 : BS / 2;
            const int tan0 = (dir + 1) % 3;
            const int tan1 = (dir + 2) % 3;
            if (axis[tan0] != 0 && axis[tan1] != 0) {
                for (int i = 0; i < BS; i += 2) {
                    int s0[3] = {it_send[0], it_send[1], it_send[2]};
                    int s1[3] = {it_send[0], it_send[1], it_send[2]};
                    s0[dir] = i;
                    s1[dir] = i + 1;
                    it_recv[dir] = i / 2 + i_offset;
                    emit(dir, s0, s1, it_recv);
                }
            } else {
                const int free_ax = axis[tan0] != 0 ? tan1 : tan0;
                const int j_offset =
                    (fine.xmin[free_ax] + fine.xmax[free_ax]) < (coarse.xmin[free_ax] + coarse.xmax[free_ax]) ?
                    0 : BS / 2;
                for (int i = 0; i < BS; i += 2) {
                    for (int j = 0; j <= BS; j += 2) {
                        it_send[free_ax] = j;
                        it_recv[free_ax] = j / 2 + j_offset;
                        int s0[3] = {it_send[0], it_send[1], it_send[2]};
                        int s1[3] = {it_send[0], it_send[1], it_send[2]};
                        s0[dir] = i;
                        s1[dir] = i + 1;
                        it_recv[dir] = i / 2 + i_offset;
                        emit(dir, s0, s1, it_recv);
                    }
                }
            }
        }
    }

    /* sequential correction records -> waves: a record whose destination is
     * overwritten before anything reads it is dropped, the rest are levelled
     * like the ghost operations (read-after-write, write-after-read,
     * write-after-write) */
    static void level_records(const std::vector<FxCorr> &seq, const std::vector<std::array<int64_t, 5>> &el,
        int nsrc, std::vector<FxCorr> &out, std::vector<int> &begin)
    {
        const int n = (int)seq.size();
        const int stride = 1 + nsrc;
        /* dense element numbers */
        std::vector<int64_t> keys;
        keys.reserve((size_t)n * stride);
        for (int x = 0; x < n; ++x) {
            for (int q = 0; q < stride; ++q) keys.push_back(el[x][q]);
        }
        std::vector<int64_t> uniq(keys);
        std::sort(uniq.begin(), uniq.end());
        uniq.erase(std::unique(uniq.begin(), uniq.end()), uniq.end());
        std::vector<int32_t> ids(keys.size());
        for (size_t q = 0; q < keys.size(); ++q) {
            ids[q] = (int32_t)(std::lower_bound(uniq.begin(), uniq.end(), keys[q]) - uniq.begin());
        }
        std::vector<int64_t>().swap(keys);
        const size_t m = uniq.size();
        std::vector<char> live(n, 0);
        std::vector<char> needed(m, 2); /* 2: not yet seen from the end (a final value, needed) */
        for (int x = n - 1; x >= 0; --x) {
            const int32_t d = ids[(size_t)x * stride];
            live[x] = needed[d] != 0;
            needed[d] = 0;
            if (!live[x]) continue;
            for (int q = 1; q <= nsrc; ++q) needed[ids[(size_t)x * stride + q]] = 1;
        }
        std::vector<int> lw(m, -1), lr(m, -1);
        std::vector<std::vector<FxCorr>> waves;
        for (int x = 0; x < n; ++x) {
            if (!live[x]) continue;
            const int32_t *e = &ids[(size_t)x * stride];
            int wave = std::max(lw[e[0]], lr[e[0]]) + 1;
            for (int q = 1; q <= nsrc; ++q) wave = std::max(wave, lw[e[q]] + 1);
            for (int q = 1; q <= nsrc; ++q) lr[e[q]] = std::max(lr[e[q]], wave);
            lw[e[0]] = wave;
            if ((int)waves.size() <= wave) waves.resize(wave + 1);
            waves[wave].push_back(seq[x]);
        }
        out.clear();
        begin.clear();
        for (const auto &w : waves) {
            begin.push_back((int)out.size());
            out.insert(out.end(), w.begin(), w.end());
        }
        begin.push_back((int)out.size());
    }

    /* ---- optimisation and levelling -------------------------------------- */

    void finish(FxPlan &plan)
    {
        const int nseq = (int)seq_.size();
        /* 2. liveness in reverse order: final versions are live; an op is
         * live when a live op reads its value */
        /* live[x]: 1 once a live op reads op x's value */
        std::vector<char> live(nseq, 0);
        for (int x = nseq - 1; x >= 0; --x) {
            const SeqOp &o = seq_[x];
            if (seq_[x].space == SPACE_CELL) ++stats_.emitted_cell_ops;
            else ++stats_.emitted_face_ops;
            const int we = w_end(x);
            for (int q = o.w_begin; q < we && !live[x]; ++q) {
                live[x] = ver_[wr_[q]] == x;
            }
            if (!live[x]) {
                ++stats_.dead;
                continue;
            }
            const int pe = prod_end(x);
            for (int p = o.prod_begin; p < pe; ++p) {
                if (prod_[p] >= 0) live[prod_[p]] = 1;
            }
        }
        if (owner_) {
            /* a live op belongs to the ranks owning the blocks it writes */
            need_.assign(nseq, 0);
            ginit_.assign(nranks_, {});
            touched_.assign(n_, 0);
            for (int x = 0; x < nseq; ++x) {
                if (!live[x]) continue;
                for (int q = seq_[x].w_begin; q < w_end(x); ++q) {
                    need_[x] |= (uint16_t)(1u << owner_[block_of(wr_[q])]);
                }
            }
        }
        /* 3. levelling over cell, cell-field and face elements: latest wave
         * that wrote / read each element (a fill has a handful of waves, far
         * below the int16 range) */
        std::vector<int16_t> &lw = lw_;
        std::vector<int16_t> &lr = lr_;
        lw.assign((size_t)(2 * ncell_ + nface_), -1);
        lr.assign((size_t)(2 * ncell_ + nface_), -1);
        int nwaves = 0;
        auto place = [&](const Elem *reads, int nr, const Elem *writes, int nw) {
            int wave = 0;
            for (int n = 0; n < nr; ++n) wave = std::max(wave, lw[reads[n]] + 1);
            for (int n = 0; n < nw; ++n) {
                wave = std::max(wave, lw[writes[n]] + 1);
                wave = std::max(wave, lr[writes[n]] + 1);
            }
            if (wave >= 32767) {
                overflow_ = true;
                wave = 32766;
            }
            for (int n = 0; n < nr; ++n) lr[reads[n]] = (int16_t)std::max<int>(lr[reads[n]], wave);
            for (int n = 0; n < nw; ++n) lw[writes[n]] = (int16_t)wave;
            nwaves = std::max(nwaves, wave + 1);
            return wave;
        };
        std::vector<int16_t> opwave(nseq, -1);
        for (int x = 0; x < nseq; ++x) {
            if (!live[x]) continue;
            const SeqOp &o = seq_[x];
            const int nr = prod_end(x) - o.prod_begin;
            opwave[x] = (int16_t)place(rd_.data() + o.prod_begin, nr, wr_.data() + o.w_begin, w_end(x) - o.w_begin);
        }
        std::vector<char>().swap(live);
        /* 4. cell-field operations (bf2bc of every ghost cell and of interior
         * cells with a rewritten face), reading the final faces through the
         * copy chains, levelled after the operations they read.  Each writes
         * its own cell-field element, which nothing else touches, and reads
         * only final face versions, so its wave is max(lw[faces]) + 1 and
         * blocks are independent: they run on worker threads and are merged
         * in block order. */
        std::vector<FxBop> bops_all;
        if (ws_ && cfg_.mhd) bops_all.swap(ws_->spare.b_ops);   /* every entry is written below */
        std::vector<int> bops_begin;
        if (cfg_.mhd) {
            const int nt = compile_threads();
            const int na = (int)plan.active.size();
            std::vector<Buf<std::pair<int16_t, FxBop>>> own_parts;
            std::vector<Buf<std::pair<int16_t, FxBop>>> &part = ws_ ? ws_->bparts : own_parts;
            if ((int)part.size() < nt) part.resize(nt);
            for (auto &v : part) v.clear();
            std::vector<std::vector<int>> cnt(nt);
            std::vector<long long> rew(nt, 0);
            std::vector<std::vector<std::vector<Elem>>> tinit(nt, std::vector<std::vector<Elem>>(owner_ ? nranks_ : 0));
            parallel_for(nt, [&](int t) {
                Buf<std::pair<int16_t, FxBop>> &out = part[t];
                /* per block: every face resolved once through its copy chain */
                std::vector<int32_t> fkey(3 * FX_NFACES);
                std::vector<int16_t> fwave(3 * FX_NFACES);
                std::vector<char> ftouch(3 * FX_NFACES);
                /* sharded: the producer and element of each resolved face,
                 * and whether a cell-field op of the block read it yet */
                std::vector<int> fver(owner_ ? 3 * FX_NFACES : 0);
                std::vector<Elem> fel(owner_ ? 3 * FX_NFACES : 0);
                std::vector<char> fmark(owner_ ? 3 * FX_NFACES : 0);
                for (int ai = (int)((int64_t)na * t / nt); ai < (int)((int64_t)na * (t + 1) / nt); ++ai) {
                    const int b = plan.active[ai];
                    const int ob = owner_ ? owner_[b] : 0;
                    const bool emit = !owner_ || ob == rank_;
                    for (int d = 0; d < 3; ++d) {
                        for (int f = 0; f < FX_NFACES; ++f) {
                            int64_t e = face_elem(b, d, f);
                            int v = ver_[e];
                            ftouch[d * FX_NFACES + f] = v >= 0;
                            resolve(e, v, &rew[t]);
                            fkey[d * FX_NFACES + f] = face_key(e);
                            fwave[d * FX_NFACES + f] = (int16_t)(lw[(Elem)e] + 1);
                            if (owner_) {
                                fver[d * FX_NFACES + f] = v;
                                fel[d * FX_NFACES + f] = (Elem)e;
                                fmark[d * FX_NFACES + f] = 0;
                            }
                        }
                    }
                    for (int i = -NG; i < BS + NG; ++i) {
                        for (int j = -NG; j < BS + NG; ++j) {
                            for (int k = -NG; k < BS + NG; ++k) {
                                const bool ghost = i < 0 || i >= BS || j < 0 || j >= BS || k < 0 || k >= BS;
                                const int f[6] = {
                                    fidx(0, i, j, k), fidx(0, i + 1, j, k),
                                    FX_NFACES + fidx(1, i, j, k), FX_NFACES + fidx(1, i, j + 1, k),
                                    2 * FX_NFACES + fidx(2, i, j, k), 2 * FX_NFACES + fidx(2, i, j, k + 1)};
                                bool touched = false;
                                for (int q = 0; q < 6; ++q) {
                                    if (ftouch[f[q]]) touched = true;
                                }
                                if (!ghost && !touched) continue;
                                if (owner_) {
                                    /* the block's owner reads these faces:
                                     * their producers join its part, values
                                     * at fill start come from their owner */
                                    for (int q = 0; q < 6; ++q) {
                                        const int fq = f[q];
                                        if (fmark[fq]) continue;
                                        fmark[fq] = 1;
                                        if (fver[fq] >= 0) {
                                            __atomic_fetch_or(&need_[fver[fq]], (uint16_t)(1u << ob), __ATOMIC_RELAXED);
                                        } else if (owner_[block_of(fel[fq])] != ob) {
                                            tinit[t][ob].push_back(fel[fq]);
                                        }
                                    }
                                    if (!emit) continue;
                                }
                                FxBop bo;
                                bo.dst = FX_CELL_KEY(b, lidx(i, j, k));
                                bo.pad = 0;
                                int wave = 0;
                                for (int q = 0; q < 6; ++q) {
                                    bo.f[q] = fkey[f[q]];
                                    wave = std::max(wave, (int)fwave[f[q]]);
                                }
                                out.emplace_back((int16_t)wave, bo);
                                if ((int)cnt[t].size() <= wave) cnt[t].resize(wave + 1, 0);
                                ++cnt[t][wave];
                            }
                        }
                    }
                }
            });
            int nbw = 0;
            for (int t = 0; t < nt; ++t) {
                stats_.rewired += rew[t];
                nbw = std::max(nbw, (int)cnt[t].size());
                for (int r = 0; r < (int)tinit[t].size(); ++r) {
                    ginit_[r].insert(ginit_[r].end(), tinit[t][r].begin(), tinit[t][r].end());
                }
            }
            nwaves = std::max(nwaves, nbw);
            /* wave-major, thread-minor placement (block order within a wave) */
            std::vector<std::vector<size_t>> at(nt, std::vector<size_t>(nbw, 0));
            bops_begin.assign(nbw + 1, 0);
            size_t run = 0;
            for (int w = 0; w < nbw; ++w) {
                bops_begin[w] = (int)run;
                for (int t = 0; t < nt; ++t) {
                    at[t][w] = run;
                    run += w < (int)cnt[t].size() ? cnt[t][w] : 0;
                }
            }
            bops_begin[nbw] = (int)run;
            bops_all.resize(run);
            parallel_for(nt, [&](int t) {
                for (const auto &e : part[t]) bops_all[at[t][e.first]++] = e.second;
                if (ws_) {
                    part[t].clear();
                } else {
                    Buf<std::pair<int16_t, FxBop>>().swap(part[t]);
                }
            });
        }
        if (!ws_) {
            std::vector<int16_t>().swap(lw);
            std::vector<int16_t>().swap(lr);
        }
        if (owner_) {
            shard_closure();
        }
        const uint16_t rbit = (uint16_t)(1u << rank_);
        auto keep = [&](int x) { return opwave[x] >= 0 && (!owner_ || (need_[x] & rbit)); };
        /* 5. per-wave arrays: a counting sort of the operations by (wave,
         * type) -- faces by (wave, type, direction), so a warp's stores land
         * in one direction's array -- replay order kept within a bucket (the
         * replay visits each destination box in storage order).  Threads
         * count and place contiguous ranges of the sequence; bucket-major,
         * thread-minor offsets keep the serial order. */
        FxProgram &g = plan.ghost;
        constexpr int NT = 16;      /* op type values are below 16 */
        constexpr int NTF = 3 * NT; /* faces: (type, direction) */
        const size_t KC = (size_t)nwaves * NT, KF = (size_t)nwaves * NTF, KP = (size_t)nwaves;
        const int nts = compile_threads();
        auto seq_lo = [&](int t) { return (int)((int64_t)nseq * t / nts); };
        auto ckey = [&](const SeqOp &o, int x) { return (size_t)opwave[x] * NT + o.op.type; };
        auto fkey = [&](const SeqOp &o, int x) {
            return (size_t)opwave[x] * NTF + (size_t)o.op.type * 3 + (o.op.aux & 3);
        };
        std::vector<std::vector<int>> tcnt_c(nts, std::vector<int>(KC, 0));
        std::vector<std::vector<int>> tcnt_f(nts, std::vector<int>(KF, 0));
        std::vector<std::vector<int>> tcnt_p(nts, std::vector<int>(KP, 0));
        parallel_for(nts, [&](int t) {
            for (int x = seq_lo(t); x < seq_lo(t + 1); ++x) {
                if (!keep(x)) continue;
                const SeqOp &o = seq_[x];
                if (o.space == SPACE_CELL) ++tcnt_c[t][ckey(o, x)];
                else if (o.space == SPACE_FACE) ++tcnt_f[t][fkey(o, x)];
                else ++tcnt_p[t][opwave[x]];
            }
        });
        /* bucket starts; per-thread counts become per-thread write cursors */
        auto offsets = [&](std::vector<std::vector<int>> &tc, size_t K) {
            std::vector<int> start(K + 1);
            int run = 0;
            for (size_t k = 0; k < K; ++k) {
                start[k] = run;
                for (int t = 0; t < nts; ++t) {
                    const int n = tc[t][k];
                    tc[t][k] = run;
                    run += n;
                }
            }
            start[K] = run;
            return start;
        };
        const std::vector<int> bc = offsets(tcnt_c, KC);
        const std::vector<int> bf = offsets(tcnt_f, KF);
        const std::vector<int> bp = offsets(tcnt_p, KP);
        if (ws_) {
            /* every entry is written below: a retired plan's arrays serve
             * (resize keeps what they hold, so no new pages are touched) */
            g.cell_ops.swap(ws_->spare.cell_ops);
            g.face_ops.swap(ws_->spare.face_ops);
            g.p_ops.swap(ws_->spare.p_ops);
        }
        g.cell_ops.resize(bc[KC]);
        g.face_ops.resize(bf[KF]);
        g.p_ops.resize(bp[KP]);
        g.cell_begin.resize(nwaves + 1);
        g.face_begin.resize(nwaves + 1);
        g.p_begin.resize(nwaves + 1);
        for (int w = 0; w <= nwaves; ++w) {
            g.cell_begin[w] = bc[(size_t)w * NT];
            g.face_begin[w] = bf[(size_t)w * NTF];
            g.p_begin[w] = bp[(size_t)w];
        }
        parallel_for(nts, [&](int t) {
            for (int x = seq_lo(t); x < seq_lo(t + 1); ++x) {
                if (!keep(x)) continue;
                const SeqOp &o = seq_[x];
                if (o.space == SPACE_CELL) g.cell_ops[tcnt_c[t][ckey(o, x)]++] = o.op;
                else if (o.space == SPACE_FACE) g.face_ops[tcnt_f[t][fkey(o, x)]++] = o.op;
                else g.p_ops[tcnt_p[t][opwave[x]]++] = groups_[o.op.dst];
            }
        });
        /* within a bucket, destination order: neighbouring threads of the
         * fill kernel then store to neighbouring addresses */
        {
            std::vector<std::pair<FxGop *, size_t>> buckets;
            for (size_t k = 0; k < KC; ++k) {
                if (bc[k + 1] > bc[k]) buckets.emplace_back(g.cell_ops.data() + bc[k], (size_t)(bc[k + 1] - bc[k]));
            }
            for (size_t k = 0; k < KF; ++k) {
                if (bf[k + 1] > bf[k]) buckets.emplace_back(g.face_ops.data() + bf[k], (size_t)(bf[k + 1] - bf[k]));
            }
            size_t most = 0;
            for (const auto &bk : buckets) most = std::max(most, bk.second);
            Buf<FxGop> own_tmp;
            Buf<FxGop> &tmp = ws_ ? ws_->sort_tmp : own_tmp;
            if (tmp.size() < most) tmp.resize(most);
            for (const auto &bk : buckets) sort_by_dst(bk.first, bk.second, nts, tmp.data());
        }
        g.b_ops.swap(bops_all);
        g.b_begin.assign(1, 0);
        for (int w = 0; w < nwaves; ++w) {
            g.b_begin.push_back(w + 1 < (int)bops_begin.size() ? bops_begin[w + 1] : (int)g.b_ops.size());
        }
        plan.stats = stats_;
    }

    /* ---- sharding -------------------------------------------------------- */

    /* reverse pass: an op joins the parts of the ranks that read its value;
     * a read of a fill-start value from another rank's block is recorded
     * for the reading rank */
    void shard_closure()
    {
        const uint16_t rbit = (uint16_t)(1u << rank_);
        for (int x = (int)seq_.size() - 1; x >= 0; --x) {
            const uint16_t m = need_[x];
            if (!m) continue;
            const SeqOp &o = seq_[x];
            const int pe = prod_end(x);
            for (int p = o.prod_begin; p < pe; ++p) {
                const int pr = prod_[p];
                if (pr >= 0) {
                    need_[pr] |= m;
                } else {
                    unsigned rest = m & ~(1u << owner_[block_of(rd_[p])]);
                    while (rest) {
                        const int r = __builtin_ctz(rest);
                        rest &= rest - 1;
                        ginit_[r].push_back(rd_[p]);
                    }
                }
                if (m & rbit) touched_[block_of(rd_[p])] = 1;
            }
            if (m & rbit) {
                for (int q = o.w_begin; q < w_end(x); ++q) touched_[block_of(wr_[q])] = 1;
            }
        }
        for (auto &v : ginit_) {
            std::sort(v.begin(), v.end());
            v.erase(std::unique(v.begin(), v.end()), v.end());
        }
    }

    static int64_t rec_key(int b, int idx) { return ((int64_t)b << 32) | (uint32_t)idx; }

    /* the same for correction records (levelled, in wave order): a record
     * reads nsrc entries of src_block, as the face / edge kernel left them
     * or as an earlier record rewrote them; rank rank_ keeps the records
     * into its blocks and their producers */
    void shard_records(std::vector<FxCorr> &recs, std::vector<int> &begin, int nsrc,
        std::vector<std::vector<int64_t>> &init)
    {
        const int n = (int)recs.size();
        std::vector<int> prod((size_t)n * nsrc, -1);
        std::unordered_map<int64_t, int> last;
        last.reserve((size_t)n * 2 + 1);
        for (int r = 0; r < n; ++r) {
            for (int k = 0; k < nsrc; ++k) {
                auto it = last.find(rec_key(recs[r].src_block, recs[r].src[k]));
                if (it != last.end()) prod[(size_t)r * nsrc + k] = it->second;
            }
            last[rec_key(recs[r].dst_block, recs[r].dst)] = r;
        }
        std::vector<uint16_t> need(n);
        for (int r = 0; r < n; ++r) need[r] = (uint16_t)(1u << owner_[recs[r].dst_block]);
        init.assign(nranks_, {});
        for (int r = n - 1; r >= 0; --r) {
            for (int k = 0; k < nsrc; ++k) {
                const int p = prod[(size_t)r * nsrc + k];
                if (p >= 0) {
                    need[p] |= need[r];
                    continue;
                }
                unsigned rest = need[r] & ~(1u << owner_[recs[r].src_block]);
                while (rest) {
                    const int q = __builtin_ctz(rest);
                    rest &= rest - 1;
                    init[q].push_back(rec_key(recs[r].src_block, recs[r].src[k]));
                }
            }
        }
        std::vector<FxCorr> out;
        std::vector<int> ob(1, 0);
        for (size_t w = 0; w + 1 < begin.size(); ++w) {
            for (int r = begin[w]; r < begin[w + 1]; ++r) {
                if (!((need[r] >> rank_) & 1)) continue;
                out.push_back(recs[r]);
                touched_[recs[r].dst_block] = 1;
                touched_[recs[r].src_block] = 1;
            }
            ob.push_back((int)out.size());
        }
        recs.swap(out);
        begin.swap(ob);
        for (auto &v : init) {
            std::sort(v.begin(), v.end());
            v.erase(std::unique(v.begin(), v.end()), v.end());
        }
    }

    /* local numbering (owned active blocks, then the halo, each in mesh
     * order), the renumbered programs and records, and the exchange lists */
    void localize(FxPlan &plan)
    {
        FxShard &sh = plan.shard;
        sh.nranks = nranks_;
        sh.rank = rank_;
        for (Elem e : ginit_[rank_]) touched_[block_of(e)] = 1;
        for (int64_t k : finit_[rank_]) touched_[(int)(k >> 32)] = 1;
        for (int64_t k : einit_[rank_]) touched_[(int)(k >> 32)] = 1;
        std::vector<int> g2l(n_, -1);
        std::vector<int> &l2g = sh.local_to_global;
        for (int b : plan.active) {
            if (owner_[b] == rank_) l2g.push_back(b);
        }
        sh.nowned = (int)l2g.size();
        for (int b = 0; b < n_; ++b) {
            if (touched_[b] && owner_[b] != rank_) l2g.push_back(b);
        }
        for (int l = 0; l < (int)l2g.size(); ++l) g2l[l2g[l]] = l;
        auto ck = [&](int32_t key) { return FX_CELL_KEY(g2l[FX_CELL_BLOCK(key)], FX_CELL_IDX(key)); };
        auto fk = [&](int32_t key) { return (g2l[key >> 15] << 15) | (key & 32767); };
        FxProgram &g = plan.ghost;
        for (FxGop &o : g.cell_ops) {
            o.dst = ck(o.dst);
            o.src = ck(o.src);
        }
        for (FxGop &o : g.face_ops) {
            o.dst = fk(o.dst);
            o.src = fk(o.src);
        }
        for (FxPop &o : g.p_ops) {
            o.fine = g2l[o.fine];
            o.coarse = g2l[o.coarse];
        }
        for (FxBop &o : g.b_ops) {
            o.dst = ck(o.dst);
            for (int q = 0; q < 6; ++q) o.f[q] = fk(o.f[q]);
        }
        for (std::vector<FxCorr> *recs : {&plan.flux_corr, &plan.emf_corr}) {
            for (FxCorr &r : *recs) {
                r.dst_block = g2l[r.dst_block];
                r.src_block = g2l[r.src_block];
            }
        }
        plan.active.clear();
        for (int l = 0; l < sh.nowned; ++l) plan.active.push_back(l);
        /* exchange lists: rank r receives init[r] from the owners; this rank
         * sends the part of every init[r] it owns */
        auto add_ghost = [&](FxXlist *lists, Elem e) {
            const int b = block_of(e);
            if (e < (Elem)ncell_) {
                lists[FX_X_CELLS].el.push_back({g2l[b], (int32_t)(e % FX_NCELLS)});
            } else {
                lists[FX_X_FACES].el.push_back({g2l[b], (int32_t)((e - 2 * ncell_) % (3 * FX_NFACES))});
            }
        };
        auto add_rec = [&](FxXlist &list, int64_t k) {
            list.el.push_back({g2l[(int)(k >> 32)], (int32_t)(k & 0xffffffff)});
        };
        for (int k = 0; k < FX_X_KINDS; ++k) {
            sh.send[k].begin.assign(1, 0);
            sh.recv[k].begin.assign(1, 0);
        }
        for (int p = 0; p < nranks_; ++p) {
            if (p != rank_) {
                for (Elem e : ginit_[rank_]) {
                    if (owner_[block_of(e)] == p) add_ghost(sh.recv, e);
                }
                for (Elem e : ginit_[p]) {
                    if (owner_[block_of(e)] == rank_) add_ghost(sh.send, e);
                }
                for (int64_t k : finit_[rank_]) {
                    if (owner_[(int)(k >> 32)] == p) add_rec(sh.recv[FX_X_FLUX], k);
                }
                for (int64_t k : finit_[p]) {
                    if (owner_[(int)(k >> 32)] == rank_) add_rec(sh.send[FX_X_FLUX], k);
                }
                for (int64_t k : einit_[rank_]) {
                    if (owner_[(int)(k >> 32)] == p) add_rec(sh.recv[FX_X_EMF], k);
                }
                for (int64_t k : einit_[p]) {
                    if (owner_[(int)(k >> 32)] == rank_) add_rec(sh.send[FX_X_EMF], k);
                }
            }
            for (int k = 0; k < FX_X_KINDS; ++k) {
                sh.send[k].begin.push_back((int)sh.send[k].el.size());
                sh.recv[k].begin.push_back((int)sh.recv[k].el.size());
            }
        }
        for (int r = 0; r < nranks_; ++r) {
            for (Elem e : ginit_[r]) sh.any[e < (Elem)ncell_ ? FX_X_CELLS : FX_X_FACES] = true;
            sh.any[FX_X_FLUX] = sh.any[FX_X_FLUX] || !finit_[r].empty();
            sh.any[FX_X_EMF] = sh.any[FX_X_EMF] || !einit_[r].empty();
        }
    }

    const fx_config &cfg_;
    int n_;
    const fx_block_desc *b_;
    int64_t ncell_;
    int64_t nface_;
    std::vector<int8_t> fid_;
    std::vector<int> ver_;       /* element -> producer op (-1: initial value) */
    Buf<SeqOp> seq_;
    Buf<int> prod_;              /* producers of the values each op reads */
    Buf<Elem> rd_;               /* elements each op reads (parallel to prod_) */
    Buf<Elem> wr_;               /* elements each op writes */
    std::vector<int16_t> lw_, lr_; /* levelling: latest wave that wrote / read each element */
    FxPlanWorkspace *ws_ = nullptr;
    std::vector<FxPop> groups_;  /* face-prolongation groups (SPACE_GROUP ops) */
    FaceIndexMap<ProlongSig> psig_;
    std::vector<int64_t> g_reads_, g_writes_;             /* prolong_group scratch */
    std::vector<std::pair<int64_t, ProlongSig>> g_sigs_;
    FxPlanStats stats_;
    std::string *err_ = nullptr;
    bool overflow_ = false;
    /* sharding */
    const int *owner_ = nullptr;
    int nranks_ = 1;
    int rank_ = 0;
    std::vector<uint16_t> need_;               /* per op: ranks whose part holds it */
    std::vector<std::vector<Elem>> ginit_;     /* per rank: elements read at their
                                                  fill-start value from other ranks' blocks */
    std::vector<std::vector<int64_t>> finit_, einit_; /* same for the correction records */
    std::vector<char> touched_;                /* blocks this rank's part reads or writes */
};

} /* namespace */

FxPlanWorkspace *fx_plan_workspace_new()
{
    return new FxPlanWorkspace();
}

void fx_plan_workspace_free(FxPlanWorkspace *ws)
{
    delete ws;
}

void fx_plan_workspace_recycle(FxPlanWorkspace *ws, FxPlan &&old)
{
    if (!ws) return;
    ws->spare.cell_ops.swap(old.ghost.cell_ops);
    ws->spare.face_ops.swap(old.ghost.face_ops);
    ws->spare.p_ops.swap(old.ghost.p_ops);
    ws->spare.b_ops.swap(old.ghost.b_ops);
}

bool fx_build_plan(const fx_config &cfg, int nblocks, const fx_block_desc *blocks,
    FxPlan &plan, std::string *err, FxPlanWorkspace *ws)
{
    plan = FxPlan();
    Compiler c(cfg, nblocks, blocks, ws);
    return c.run(plan, err);
}

bool fx_build_shard_plan(const fx_config &cfg, int nblocks, const fx_block_desc *blocks,
    const int *owner, int nranks, int rank, FxPlan &plan, std::string *err)
{
    plan = FxPlan();
    if (nranks < 1 || nranks > FX_MAX_RANKS || rank < 0 || rank >= nranks || !owner) {
        if (err) *err = "sharding: nranks outside [1, 16] or rank outside [0, nranks)";
        return false;
    }
    /* the single-device sequence over all blocks: every block takes part */
    std::vector<fx_block_desc> all(blocks, blocks + nblocks);
    for (fx_block_desc &b : all) {
        if (b.id >= 0 && b.active == 1) b.rank = 0;
    }
    for (int b = 0; b < nblocks; ++b) {
        if (all[b].id >= 0 && all[b].active == 1 && (owner[b] < 0 || owner[b] >= nranks)) {
            if (err) *err = "sharding: an active block has no rank in [0, nranks)";
            return false;
        }
    }
    Compiler c(cfg, nblocks, all.data());
    c.set_owners(owner, nranks, rank);
    return c.run(plan, err);
}

bool fx_build_corrections(const fx_config &cfg, int nblocks, const fx_block_desc *blocks,
    FxPlan &plan, std::string *err)
{
    plan = FxPlan();
    Compiler c(cfg, nblocks, blocks);
    return c.run_corrections(plan, err);
}
