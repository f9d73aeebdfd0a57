// Sharding one spot over several engines (a flop split by turn card, so that
// a spot larger than one GPU's memory, or its iterations, spread over GPUs).  Every shard keeps the tree above the first
// chance nodes and every nshards-th representative subtree below them; the
// values of those subtrees' roots are summed over the shards (exactly: each
// is nonzero on one shard) before the chance nodes above add them up:
//   * over NCCL between processes, one GPU each (NcclReducer, captured in the
//     iteration's CUDA graph like every other launch);
//   * on the host between engines of one process (HostExchange), which lets
//     a single device run -- and a test check -- every shard of a spot.
#pragma once
#include <condition_variable>
#include <memory>
#include <mutex>
#include <vector>

#include "../kernels/engine.hpp"

namespace gtob {

constexpr int kNcclIdBytes = 128;
// ncclGetUniqueId through a lazily loaded libnccl.so.2 (the library links no
// NCCL: it is loaded only when a sharded engine is built).
void nccl_unique_id(unsigned char* out);
// The reducer of shard `rank` of `world` processes (ncclCommInitRank: every
// rank must make this call; it returns once all have joined).
std::shared_ptr<ShardReducer> make_nccl_reducer(int rank, int world, const unsigned char* id);

// Shards of one process: reduce() copies the shard's buffer to the host,
// waits (bounded) for every shard, adds them in shard order and copies the
// sums back -- the same bits on every shard.
class HostExchange {
  public:
    explicit HostExchange(int nshards);
    void exchange(int shard, float* buf, size_t count, cudaStream_t stream);

  private:
    void barrier();
    int n_;
    std::mutex mu_;
    std::condition_variable cv_;
    int arrived_ = 0;
    unsigned gen_ = 0;
    std::vector<std::vector<float>> bufs_;
};
std::shared_ptr<ShardReducer> make_host_reducer(std::shared_ptr<HostExchange> x, int shard);

// Shards in separate processes that sum over a channel of the caller's own
// (a torch.distributed group, MPI, sockets): reduce() copies the shard's
// values to a host buffer, calls fn(user, values, count), which must leave
// there the sum over every rank and return 0, and copies the sums back.  The
// engine runs plain launches (the call synchronises on the host), and no
// kernel ever waits on another rank.
using HostReduceFn = int (*)(void* user, float* values, size_t count);
std::shared_ptr<ShardReducer> make_callback_reducer(HostReduceFn fn, void* user);

}  // namespace gtob
