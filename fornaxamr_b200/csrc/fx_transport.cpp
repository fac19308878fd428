/*
 * Transports of a sharded mesh (see fx_transport.h).
 */
#include "fx_transport.h"

#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <vector>

#include "fx_plan.h"

/* ---- in-process group -------------------------------------------------- */

struct fx_shard_group {
    int n = 0;
    std::mutex m;
    std::condition_variable cv;
    int arrived = 0;
    long long gen = 0;
    bool broken = false; /* a rank gave up waiting: every later wait fails */
    struct Slot {
        const double *sbuf = nullptr;
        const size_t *soff = nullptr;
        unsigned long long red[2] = {0, 0};
    } slot[FX_MAX_RANKS];

    /* all ranks arrive, or false after the limit (a rank that failed before
     * reaching the exchange must not leave the others waiting for ever) */
    bool barrier()
    {
        std::unique_lock<std::mutex> l(m);
        if (broken) return false;
        const long long g = gen;
        if (++arrived == n) {
            arrived = 0;
            ++gen;
            cv.notify_all();
            return true;
        }
        const bool ok = cv.wait_for(l, std::chrono::seconds(120), [&] { return gen != g || broken; });
        if (!ok || broken) {
            broken = true;
            cv.notify_all();
            return false;
        }
        return true;
    }
};

fx_shard_group *fx_group_new(int nranks)
{
    if (nranks < 1 || nranks > FX_MAX_RANKS) return nullptr;
    fx_shard_group *g = new fx_shard_group;
    g->n = nranks;
    return g;
}

void fx_group_delete(fx_shard_group *g) { delete g; }

int fx_group_size(const fx_shard_group *g) { return g ? g->n : 0; }

namespace {

class GroupTransport : public FxTransport {
public:
    GroupTransport(fx_shard_group *g, int rank) : g_(g), rank_(rank) {}

    int exchange(int, const double *sbuf, const size_t *soff, double *rbuf, const size_t *roff,
        cudaStream_t s) override
    {
        if (cudaStreamSynchronize(s) != cudaSuccess) return fail("exchange: pack failed");
        g_->slot[rank_].sbuf = sbuf;
        g_->slot[rank_].soff = soff;
        if (!g_->barrier()) return fail("exchange: a rank did not arrive within 120 s");
        int rc = 0;
        for (int p = 0; p < g_->n && !rc; ++p) {
            const size_t n = roff[p + 1] - roff[p];
            if (p == rank_ || n == 0) continue;
            const fx_shard_group::Slot &q = g_->slot[p];
            if (q.soff[rank_ + 1] - q.soff[rank_] != n) {
                rc = fail("exchange: send and receive sizes differ");
                break;
            }
            if (cudaMemcpyAsync(rbuf + roff[p], q.sbuf + q.soff[rank_], n * sizeof(double),
                    cudaMemcpyDeviceToDevice, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                rc = fail("exchange: device copy failed");
            }
        }
        /* the senders keep their buffers until every receiver has copied */
        if (!g_->barrier()) return fail("exchange: a rank did not arrive within 120 s");
        return rc;
    }

    int min_u64(unsigned long long *d, int count, cudaStream_t s) override
    {
        if (count > 2) return fail("min_u64: at most two keys");
        if (cudaMemcpyAsync(h_, d, count * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            return fail("min_u64: device copy failed");
        }
        for (int q = 0; q < count; ++q) g_->slot[rank_].red[q] = h_[q];
        if (!g_->barrier()) return fail("min_u64: a rank did not arrive within 120 s");
        for (int q = 0; q < count; ++q) {
            for (int p = 0; p < g_->n; ++p) {
                if (g_->slot[p].red[q] < h_[q]) h_[q] = g_->slot[p].red[q];
            }
        }
        if (!g_->barrier()) return fail("min_u64: a rank did not arrive within 120 s");
        if (cudaMemcpyAsync(d, h_, count * sizeof(unsigned long long), cudaMemcpyHostToDevice, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            return fail("min_u64: device copy failed");
        }
        return 0;
    }

    bool capturable() const override { return false; }

private:
    int fail(const char *msg)
    {
        err = msg;
        return 1;
    }
    fx_shard_group *g_;
    int rank_;
    unsigned long long h_[2] = {0, 0};
};

/* ---- NCCL (resolved at run time: the library loads without it) ---------- */

struct NcclApi {
    bool ok = false;
    decltype(&ncclGetUniqueId) getUniqueId = nullptr;
    decltype(&ncclCommInitRank) commInitRank = nullptr;
    decltype(&ncclCommDestroy) commDestroy = nullptr;
    decltype(&ncclGroupStart) groupStart = nullptr;
    decltype(&ncclGroupEnd) groupEnd = nullptr;
    decltype(&ncclSend) send = nullptr;
    decltype(&ncclRecv) recv = nullptr;
    decltype(&ncclAllReduce) allReduce = nullptr;
    decltype(&ncclGetErrorString) errorString = nullptr;
};

const NcclApi &nccl_api()
{
    static NcclApi api;
    static std::once_flag once;
    std::call_once(once, [] {
        void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_GLOBAL);
        if (!h) return;
        api.getUniqueId = (decltype(api.getUniqueId))dlsym(h, "ncclGetUniqueId");
        api.commInitRank = (decltype(api.commInitRank))dlsym(h, "ncclCommInitRank");
        api.commDestroy = (decltype(api.commDestroy))dlsym(h, "ncclCommDestroy");
        api.groupStart = (decltype(api.groupStart))dlsym(h, "ncclGroupStart");
        api.groupEnd = (decltype(api.groupEnd))dlsym(h, "ncclGroupEnd");
        api.send = (decltype(api.send))dlsym(h, "ncclSend");
        api.recv = (decltype(api.recv))dlsym(h, "ncclRecv");
        api.allReduce = (decltype(api.allReduce))dlsym(h, "ncclAllReduce");
        api.errorString = (decltype(api.errorString))dlsym(h, "ncclGetErrorString");
        api.ok = api.getUniqueId && api.commInitRank && api.commDestroy && api.groupStart && api.groupEnd &&
            api.send && api.recv && api.allReduce && api.errorString;
    });
    return api;
}

class NcclTransport : public FxTransport {
public:
    NcclTransport(ncclComm_t comm, int nranks, int rank) : comm_(comm), n_(nranks), rank_(rank) {}
    ~NcclTransport() override
    {
        if (comm_) nccl_api().commDestroy(comm_);
    }

    int exchange(int, const double *sbuf, const size_t *soff, double *rbuf, const size_t *roff,
        cudaStream_t s) override
    {
        const NcclApi &a = nccl_api();
        ncclResult_t r = a.groupStart();
        for (int p = 0; p < n_ && r == ncclSuccess; ++p) {
            if (p == rank_) continue;
            const size_t sn = soff[p + 1] - soff[p];
            const size_t rn = roff[p + 1] - roff[p];
            if (sn) r = a.send(sbuf + soff[p], sn, ncclFloat64, p, comm_, s);
            if (rn && r == ncclSuccess) r = a.recv(rbuf + roff[p], rn, ncclFloat64, p, comm_, s);
        }
        const ncclResult_t e = a.groupEnd();
        if (r == ncclSuccess) r = e;
        return check(r, "exchange");
    }

    int min_u64(unsigned long long *d, int count, cudaStream_t s) override
    {
        return check(nccl_api().allReduce(d, d, count, ncclUint64, ncclMin, comm_, s), "min_u64");
    }

    bool capturable() const override { return true; }

private:
    int check(ncclResult_t r, const char *what)
    {
        if (r == ncclSuccess) return 0;
        err = std::string(what) + ": " + nccl_api().errorString(r);
        return 1;
    }
    ncclComm_t comm_;
    int n_;
    int rank_;
};

} /* namespace */

FxTransport *fx_transport_group(fx_shard_group *g, int rank)
{
    if (!g || rank < 0 || rank >= g->n) return nullptr;
    return new GroupTransport(g, rank);
}

int fx_transport_nccl_id(unsigned char id[128], std::string *err)
{
    const NcclApi &a = nccl_api();
    if (!a.ok) {
        if (err) *err = "libnccl.so.2 not found";
        return 1;
    }
    static_assert(sizeof(ncclUniqueId) == 128, "NCCL unique id size");
    ncclUniqueId u;
    const ncclResult_t r = a.getUniqueId(&u);
    if (r != ncclSuccess) {
        if (err) *err = std::string("ncclGetUniqueId: ") + a.errorString(r);
        return 1;
    }
    std::memcpy(id, &u, sizeof(u));
    return 0;
}

FxTransport *fx_transport_nccl(int nranks, int rank, const unsigned char id[128], int device, std::string *err)
{
    const NcclApi &a = nccl_api();
    if (!a.ok) {
        if (err) *err = "libnccl.so.2 not found";
        return nullptr;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        if (err) *err = "cudaSetDevice failed";
        return nullptr;
    }
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof(u));
    ncclComm_t comm = nullptr;
    const ncclResult_t r = a.commInitRank(&comm, nranks, u, rank);
    if (r != ncclSuccess) {
        if (err) *err = std::string("ncclCommInitRank: ") + a.errorString(r);
        return nullptr;
    }
    return new NcclTransport(comm, nranks, rank);
}
