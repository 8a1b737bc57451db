// Row-shard reducers (bb_comm): how the shards of one fit combine their
// integer partial sums so that every shard takes the same decisions.
//
// NCCL: one process per GPU, an in-place ncclAllReduce on the grower's
// stream (sums as uint64, maxima as uint32), so it orders with the kernels
// around it and is captured into the round's CUDA graph. libnccl.so.2 is
// opened at run time -- the copy the process already loaded (e.g.
// PyTorch's) when there is one -- so the library needs no NCCL at link time.
//
// Group: several shards in one process (one host thread per shard, each with
// its own stream). At each reduction every member records an event on its
// stream; the last to arrive makes its stream wait on all of them, sums the
// members' buffers with one kernel, and records a done event every member's
// stream waits on. Ordering is by stream events only: no kernel ever waits
// for another.
#include "bonsai_b200.h"
#include "shard.cuh"

#include <nccl.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace bb
{
namespace
{

// ---- NCCL, resolved at run time --------------------------------------------

struct NcclApi
{
    ncclResult_t (*get_unique_id)(ncclUniqueId *)                                   = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t *, int, ncclUniqueId, int)            = nullptr;
    ncclResult_t (*all_reduce)(void const *, void *, size_t, ncclDataType_t, ncclRedOp_t,
                               ncclComm_t, cudaStream_t)                           = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t)                                        = nullptr;
    char const *(*error_string)(ncclResult_t)                                       = nullptr;
};

NcclApi const &nccl()
{
    static NcclApi    api;
    static std::mutex m;
    std::lock_guard<std::mutex> lock(m);
    if (api.all_reduce != nullptr)
    {
        return api;
    }
    // the process's own NCCL when one is loaded (e.g. PyTorch's): loading a
    // second copy first would take the soname from the one it links against
    void *h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_NOLOAD);
    if (h == nullptr)
    {
        h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    }
    if (h == nullptr)
    {
        throw ConfigError(std::string("bb_comm: libnccl.so.2 not found: ") + dlerror());
    }
    auto sym = [&](char const *name)
    {
        void *p = dlsym(h, name);
        if (p == nullptr)
        {
            throw ConfigError(std::string("bb_comm: NCCL lacks ") + name);
        }
        return p;
    };
    api.get_unique_id  = reinterpret_cast<decltype(api.get_unique_id)>(sym("ncclGetUniqueId"));
    api.comm_init_rank = reinterpret_cast<decltype(api.comm_init_rank)>(sym("ncclCommInitRank"));
    api.comm_destroy   = reinterpret_cast<decltype(api.comm_destroy)>(sym("ncclCommDestroy"));
    api.error_string   = reinterpret_cast<decltype(api.error_string)>(sym("ncclGetErrorString"));
    api.all_reduce     = reinterpret_cast<decltype(api.all_reduce)>(sym("ncclAllReduce"));
    return api;
}

void nccl_check(ncclResult_t r, char const *what)
{
    if (r != ncclSuccess)
    {
        throw CudaError(std::string("nccl: ") + what + ": " + nccl().error_string(r));
    }
}

class NcclReducer final : public Reducer
{
  public:
    NcclReducer(ncclUniqueId const &id, int n_ranks, int rank)
    {
        nccl_check(nccl().comm_init_rank(&comm_, n_ranks, id, rank), "ncclCommInitRank");
    }
    ~NcclReducer() override
    {
        if (comm_ != nullptr)
        {
            nccl().comm_destroy(comm_);
        }
    }
    void sum_u64(void *buf, size_t n, cudaStream_t s) override
    {
        nccl_check(nccl().all_reduce(buf, buf, n, ncclUint64, ncclSum, comm_, s),
                   "ncclAllReduce");
    }
    void max_u32(void *buf, size_t n, cudaStream_t s) override
    {
        nccl_check(nccl().all_reduce(buf, buf, n, ncclUint32, ncclMax, comm_, s),
                   "ncclAllReduce");
    }

  private:
    ncclComm_t comm_ = nullptr;
};

// ---- in-process group ---------------------------------------------------------

constexpr uint32_t k_max_group = 16;

struct GroupPtrs
{
    void *p[k_max_group];
};

__global__ void group_sum_kernel(GroupPtrs b, uint32_t k, uint64_t n)
{
    for (uint64_t x = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x; x < n;
         x += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    {
        unsigned long long s = 0;
        for (uint32_t j = 0; j < k; ++j)
        {
            s += static_cast<unsigned long long const *>(b.p[j])[x];
        }
        for (uint32_t j = 0; j < k; ++j)
        {
            static_cast<unsigned long long *>(b.p[j])[x] = s;
        }
    }
}

__global__ void group_max_kernel(GroupPtrs b, uint32_t k, uint64_t n)
{
    for (uint64_t x = (static_cast<uint64_t>(blockIdx.x) * blockDim.x) + threadIdx.x; x < n;
         x += static_cast<uint64_t>(gridDim.x) * blockDim.x)
    {
        uint32_t m = 0;
        for (uint32_t j = 0; j < k; ++j)
        {
            m = max(m, static_cast<uint32_t const *>(b.p[j])[x]);
        }
        for (uint32_t j = 0; j < k; ++j)
        {
            static_cast<uint32_t *>(b.p[j])[x] = m;
        }
    }
}

class Group
{
  public:
    explicit Group(uint32_t k) : k_(k), bufs_(k, nullptr), ev_in_(k)
    {
        for (auto &e : ev_in_)
        {
            check(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
        }
        check(cudaEventCreateWithFlags(&ev_out_, cudaEventDisableTiming), "cudaEventCreate");
    }
    ~Group()
    {
        for (auto &e : ev_in_)
        {
            cudaEventDestroy(e);
        }
        cudaEventDestroy(ev_out_);
    }
    // Member m's buffer joins the reduction; returns once the reduction is
    // enqueued with m's stream ordered after it.
    void reduce(uint32_t m, void *buf, size_t n, cudaStream_t s, bool is_max)
    {
        check(cudaEventRecord(ev_in_[m], s), "cudaEventRecord");
        std::unique_lock<std::mutex> lock(mu_);
        uint64_t const               gen = gen_;
        if (arrived_ == 0)
        {
            n_ = n;
        }
        else if (n != n_)
        {
            throw std::invalid_argument("bb_comm group: members reduced different sizes");
        }
        bufs_[m] = buf;
        if (++arrived_ == k_)
        {
            for (uint32_t j = 0; j < k_; ++j)
            {
                check(cudaStreamWaitEvent(s, ev_in_[j], 0), "cudaStreamWaitEvent");
            }
            GroupPtrs ptrs{};
            for (uint32_t j = 0; j < k_; ++j)
            {
                ptrs.p[j] = bufs_[j];
            }
            uint32_t const grid = static_cast<uint32_t>(std::min<size_t>(
                std::max<size_t>(1, (n + 255) / 256), 148 * 8));
            if (is_max)
            {
                group_max_kernel<<<grid, 256, 0, s>>>(ptrs, k_, n);
            }
            else
            {
                group_sum_kernel<<<grid, 256, 0, s>>>(ptrs, k_, n);
            }
            check(cudaGetLastError(), "group reduce kernel");
            check(cudaEventRecord(ev_out_, s), "cudaEventRecord");
            arrived_ = 0;
            ++gen_;
            cv_.notify_all();
        }
        else if (!cv_.wait_for(lock, std::chrono::seconds(120), [&] { return gen_ != gen; }))
        {
            // a member never arrived (its thread failed or stopped calling):
            // give up rather than block its peers for good
            throw std::runtime_error("bb_comm group: a member missed a reduction");
        }
        check(cudaStreamWaitEvent(s, ev_out_, 0), "cudaStreamWaitEvent");
    }
    uint32_t size() const
    {
        return k_;
    }

  private:
    uint32_t                k_;
    std::vector<void *>     bufs_;
    std::vector<cudaEvent_t> ev_in_;
    cudaEvent_t             ev_out_{};
    std::mutex              mu_;
    std::condition_variable cv_;
    uint32_t                arrived_ = 0;
    uint64_t                gen_     = 0;
    size_t                  n_       = 0;
};

class GroupReducer final : public Reducer
{
  public:
    explicit GroupReducer(uint32_t k) : g_(std::make_shared<Group>(k)) {}
    std::shared_ptr<Group> g_;
    void                   sum_u64(void *, size_t, cudaStream_t) override
    {
        throw std::logic_error("bb_comm group: reduce through a member");
    }
    void max_u32(void *, size_t, cudaStream_t) override
    {
        throw std::logic_error("bb_comm group: reduce through a member");
    }
};

class GroupMember final : public Reducer
{
  public:
    GroupMember(std::shared_ptr<Group> g, uint32_t m) : g_(std::move(g)), m_(m) {}
    void sum_u64(void *buf, size_t n, cudaStream_t s) override
    {
        g_->reduce(m_, buf, n, s, false);
    }
    void max_u32(void *buf, size_t n, cudaStream_t s) override
    {
        g_->reduce(m_, buf, n, s, true);
    }

  private:
    std::shared_ptr<Group> g_;
    uint32_t               m_;
};

template <typename F> int comm_guard(F &&f)
{
    try
    {
        f();
        return BB_OK;
    }
    catch (ConfigError const &e)
    {
        set_last_error(e.what());
        return BB_ERR_CONFIG;
    }
    catch (std::invalid_argument const &e)
    {
        set_last_error(e.what());
        return BB_ERR_ARG;
    }
    catch (std::exception const &e)
    {
        set_last_error(e.what());
        return BB_ERR_CUDA;
    }
}

} // namespace
} // namespace bb

using namespace bb;

extern "C"
{
    int bb_comm_unique_id(uint8_t *out)
    {
        return comm_guard(
            [&]
            {
                if (out == nullptr)
                {
                    throw std::invalid_argument("bb_comm_unique_id: null argument");
                }
                ncclUniqueId id;
                nccl_check(nccl().get_unique_id(&id), "ncclGetUniqueId");
                static_assert(sizeof(id.internal) == BB_COMM_ID_BYTES, "NCCL id size");
                std::memcpy(out, id.internal, BB_COMM_ID_BYTES);
            });
    }

    int bb_comm_create(uint8_t const *id, uint32_t n_ranks, uint32_t rank, bb_comm **out)
    {
        return comm_guard(
            [&]
            {
                if (id == nullptr || out == nullptr || n_ranks == 0 || rank >= n_ranks)
                {
                    throw std::invalid_argument("bb_comm_create: bad arguments");
                }
                ncclUniqueId u;
                std::memcpy(u.internal, id, BB_COMM_ID_BYTES);
                auto c  = std::make_unique<bb_comm>();
                c->impl = std::make_shared<NcclReducer>(u, static_cast<int>(n_ranks),
                                                        static_cast<int>(rank));
                *out    = c.release();
            });
    }

    int bb_comm_group(uint32_t n_shards, bb_comm **members)
    {
        return comm_guard(
            [&]
            {
                if (members == nullptr || n_shards == 0 || n_shards > k_max_group)
                {
                    throw std::invalid_argument("bb_comm_group: 1 to 16 shards");
                }
                auto g = std::make_shared<GroupReducer>(n_shards);
                for (uint32_t m = 0; m < n_shards; ++m)
                {
                    auto c    = std::make_unique<bb_comm>();
                    c->impl   = g;
                    c->member = std::make_unique<GroupMember>(g->g_, m);
                    members[m] = c.release();
                }
            });
    }

    void bb_comm_destroy(bb_comm *c)
    {
        delete c;
    }
}
