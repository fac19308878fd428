/*
 * Transports of a sharded mesh: how the packed exchange buffers of one rank
 * reach the other ranks, and the minimum of the dt keys over ranks.
 *
 *   NCCL      one process per GPU; send/recv pairs in one group per exchange
 *             and an all-reduce (min) for the dt keys, all stream-ordered, so
 *             a whole step with its exchanges is captured as one CUDA graph.
 *   group     ranks emulated by contexts of one process (one host thread per
 *             rank, any number of contexts per GPU): device-to-device copies
 *             between the contexts' buffers with host barriers; no kernel
 *             ever waits on another rank.
 */
#ifndef FX_TRANSPORT_H
#define FX_TRANSPORT_H

#include <cuda_runtime.h>

#include <cstddef>
#include <string>

struct fx_shard_group;

class FxTransport {
public:
    virtual ~FxTransport() {}
    /* moves exchange `kind`: segment p of sbuf ([soff[p], soff[p + 1])
     * doubles) goes to rank p, segment p of rbuf is filled from rank p; the
     * packing was enqueued on s before the call, the unpacking follows it */
    virtual int exchange(int kind, const double *sbuf, const size_t *soff, double *rbuf,
        const size_t *roff, cudaStream_t s) = 0;
    /* d[0 .. count) <- element-wise minimum over the ranks (ordered keys) */
    virtual int min_u64(unsigned long long *d, int count, cudaStream_t s) = 0;
    /* whether exchange / min_u64 may be captured into a CUDA graph */
    virtual bool capturable() const = 0;
    std::string err;
};

/* rank `rank` of an in-process group (the group outlives the transport) */
FxTransport *fx_transport_group(fx_shard_group *g, int rank);
/* NCCL communicator of nranks ranks from a unique id made by
 * fx_transport_nccl_id; returns nullptr with *err set on failure */
FxTransport *fx_transport_nccl(int nranks, int rank, const unsigned char id[128], int device, std::string *err);
int fx_transport_nccl_id(unsigned char id[128], std::string *err);

fx_shard_group *fx_group_new(int nranks);
void fx_group_delete(fx_shard_group *g);
int fx_group_size(const fx_shard_group *g);

#endif
