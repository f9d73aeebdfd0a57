#include "shard.hpp"

#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <cstring>
#include <string>

namespace gtob {

namespace {
#define GTOB_CUDA_OK(x)                                                                             \
    do {                                                                                            \
        cudaError_t e_ = (x);                                                                       \
        if (e_ != cudaSuccess) throw Error(std::string("cuda: ") + cudaGetErrorString(e_) + " at " #x); \
    } while (0)

struct NcclApi {
    ncclResult_t (*get_unique_id)(ncclUniqueId*) = nullptr;
    ncclResult_t (*comm_init_rank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
    ncclResult_t (*all_reduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                               cudaStream_t) = nullptr;
    ncclResult_t (*comm_destroy)(ncclComm_t) = nullptr;
    const char* (*error_string)(ncclResult_t) = nullptr;
};
const NcclApi& nccl() {
    static std::once_flag once;
    static NcclApi api;
    static std::string err;
    std::call_once(once, [] {
        void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
        if (!h) {
            err = std::string("nccl: cannot load libnccl.so.2: ") + dlerror();
            return;
        }
        auto sym = [&](const char* n) { return dlsym(h, n); };
        api.get_unique_id = (decltype(api.get_unique_id))sym("ncclGetUniqueId");
        api.comm_init_rank = (decltype(api.comm_init_rank))sym("ncclCommInitRank");
        api.all_reduce = (decltype(api.all_reduce))sym("ncclAllReduce");
        api.comm_destroy = (decltype(api.comm_destroy))sym("ncclCommDestroy");
        api.error_string = (decltype(api.error_string))sym("ncclGetErrorString");
        if (!api.get_unique_id || !api.comm_init_rank || !api.all_reduce ||
            !api.comm_destroy || !api.error_string)
            err = "nccl: libnccl.so.2 lacks an entry point";
    });
    if (!err.empty()) throw Error(err);
    return api;
}
void nccl_check(ncclResult_t r, const char* what) {
    if (r != ncclSuccess) throw Error(std::string("nccl: ") + what + ": " + nccl().error_string(r));
}

class NcclReducer : public ShardReducer {
  public:
    NcclReducer(int rank, int world, const unsigned char* id) {
        ncclUniqueId uid;
        std::memcpy(uid.internal, id, kNcclIdBytes);
        nccl_check(nccl().comm_init_rank(&comm_, world, uid, rank), "ncclCommInitRank");
    }
    ~NcclReducer() override {
        if (comm_) nccl().comm_destroy(comm_);
    }
    void reduce(float* buf, size_t count, cudaStream_t stream) override {
        nccl_check(nccl().all_reduce(buf, buf, count, ncclFloat32, ncclSum, comm_, stream), "ncclAllReduce");
    }
    bool capturable() const override { return true; }

  private:
    ncclComm_t comm_ = nullptr;
};

class HostReducer : public ShardReducer {
  public:
    HostReducer(std::shared_ptr<HostExchange> x, int shard) : x_(std::move(x)), shard_(shard) {}
    void reduce(float* buf, size_t count, cudaStream_t stream) override { x_->exchange(shard_, buf, count, stream); }
    bool capturable() const override { return false; }

  private:
    std::shared_ptr<HostExchange> x_;
    int shard_;
};

class CallbackReducer : public ShardReducer {
  public:
    CallbackReducer(HostReduceFn fn, void* user) : fn_(fn), user_(user) {}
    void reduce(float* buf, size_t count, cudaStream_t stream) override {
        host_.resize(count);
        GTOB_CUDA_OK(cudaMemcpyAsync(host_.data(), buf, count * sizeof(float), cudaMemcpyDeviceToHost, stream));
        GTOB_CUDA_OK(cudaStreamSynchronize(stream));
        const int rc = fn_(user_, host_.data(), count);
        if (rc != 0) throw Error("shard reduce callback failed (status " + std::to_string(rc) + ")");
        GTOB_CUDA_OK(cudaMemcpyAsync(buf, host_.data(), count * sizeof(float), cudaMemcpyHostToDevice, stream));
        GTOB_CUDA_OK(cudaStreamSynchronize(stream));
    }
    bool capturable() const override { return false; }

  private:
    HostReduceFn fn_;
    void* user_;
    std::vector<float> host_;
};
}  // namespace

void nccl_unique_id(unsigned char* out) {
    ncclUniqueId uid;
    nccl_check(nccl().get_unique_id(&uid), "ncclGetUniqueId");
    std::memcpy(out, uid.internal, kNcclIdBytes);
}
std::shared_ptr<ShardReducer> make_nccl_reducer(int rank, int world, const unsigned char* id) {
    if (world < 1 || rank < 0 || rank >= world) throw Error("invalid argument: rank / world");
    return std::make_shared<NcclReducer>(rank, world, id);
}

HostExchange::HostExchange(int nshards) : n_(nshards), bufs_(nshards) {
    if (nshards < 1) throw Error("invalid argument: shard count");
}
// All shards arrive or, after 60 s, an error: a shard that stopped early
// ends the others' waits instead of hanging them.
void HostExchange::barrier() {
    std::unique_lock<std::mutex> lk(mu_);
    const unsigned g = gen_;
    if (++arrived_ == n_) {
        arrived_ = 0;
        gen_++;
        cv_.notify_all();
        return;
    }
    if (!cv_.wait_for(lk, std::chrono::seconds(60), [&] { return gen_ != g; }))
        throw Error("timeout: a shard did not reach the exchange");
}
void HostExchange::exchange(int shard, float* buf, size_t count, cudaStream_t stream) {
    std::vector<float>& mine = bufs_[shard];
    mine.resize(count);
    GTOB_CUDA_OK(cudaMemcpyAsync(mine.data(), buf, count * sizeof(float), cudaMemcpyDeviceToHost, stream));
    GTOB_CUDA_OK(cudaStreamSynchronize(stream));
    barrier();  // every shard's values are on the host
    std::vector<float> sum(count, 0.0f);
    for (int s = 0; s < n_; s++)
        for (size_t i = 0; i < count; i++) sum[i] += bufs_[s][i];
    barrier();  // every shard has read them: buffers may be refilled
    GTOB_CUDA_OK(cudaMemcpyAsync(buf, sum.data(), count * sizeof(float), cudaMemcpyHostToDevice, stream));
    GTOB_CUDA_OK(cudaStreamSynchronize(stream));
}
std::shared_ptr<ShardReducer> make_host_reducer(std::shared_ptr<HostExchange> x, int shard) {
    return std::make_shared<HostReducer>(std::move(x), shard);
}
std::shared_ptr<ShardReducer> make_callback_reducer(HostReduceFn fn, void* user) {
    if (!fn) throw Error("invalid argument: reduce callback");
    return std::make_shared<CallbackReducer>(fn, user);
}

}  // namespace gtob
