// GPU engine for one spot: the role of the reference's gpu::GpuSolver
// (crates/solver/src/gpu/mod.rs).  Owns every device buffer; copies arenas and
// locks out of a HostSolver and syncs results back into it.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "../host/plan.hpp"
#include "../host/solver.hpp"

namespace gtob {

// FP8: E4M3 with a per-node scale.  I16SR: the i16/u16 arenas, requantised
// after each update with stochastic rounding instead of store.rs's round to
// nearest (an engine option: the layout and every other rule are I16's).
enum ArenaFormat { kFmtF32 = 0, kFmtI16 = 1, kFmtFP8 = 2, kFmtI16SR = 3 };
constexpr size_t kNodeScratchElems = 16384;  // 64 KiB of f32: the read_node_static limit
enum EngineKind {
    kEngineFused = 0,
    kEnginePlain = 1,
    kEngineFused32 = 2,
    kEngineWarp = 3,
    kEngineStaged = 4,
    kEngineStagedRiver = 5
};

struct Profile {
    double ms[7];
    uint32_t launches[7];
};
extern const char* const kKernelNames[7];

struct EngineImpl;
class LeafNet;

// Sums one device buffer over the shards of one sharded spot (see
// build_plan): each shard calls reduce with its copy of the same count floats
// and returns (in stream order) with it holding the sum over the shards.
struct ShardReducer {
    virtual ~ShardReducer() = default;
    virtual void reduce(float* buf, size_t count, cudaStream_t stream) = 0;
    // false: the reduction synchronises on the host, so the engine runs its
    // sweeps as plain launches instead of captured graphs
    virtual bool capturable() const = 0;
};

class GpuEngine {
  public:
    // fmt < 0: follow the host storage (f32 -> f32 arenas, compressed -> i16/u16).
    // engine: kEngineFused (terminals evaluated inside their parents' kernels,
    // f64 terminal sums as the reference CPU engine), kEnginePlain (one launch
    // per terminal level, f64 sums), kEngineFused32 (fused, f32 sums as the
    // reference GPU kernels), kEngineWarp (one warp per action node, fold
    // children evaluated in place by the warp, showdowns one CTA each; f64),
    // kEngineStaged (one CTA per node staging its blocks and vectors in shared
    // memory with bulk copies; fold children in place; exact sums),
    // kEngineStagedRiver (the staged engine with river betting rounds solved
    // by river programs, cfr_river.cuh).
    GpuEngine(const HostSolver& host, int fmt, int engine = 0);
    // One shard of a sharded spot: the top of the tree and every nshards-th
    // representative subtree below its chance nodes; `reducer` adds the
    // shards' partial chance values after each such level of the up sweep.
    GpuEngine(const HostSolver& host, int fmt, int engine, int shard, int nshards, std::shared_ptr<ShardReducer> reducer,
              std::shared_ptr<LeafNet> leaf_net = nullptr);
    // A depth-limited solve of a flop spot: the tree is cut at the chance
    // nodes dealing the turn (where betting follows) and their values come
    // from leaf_net after every down sweep.  The net serves one engine at a
    // time (its activation buffers are its own).
    GpuEngine(const HostSolver& host, int fmt, int engine, std::shared_ptr<LeafNet> leaf_net)
        : GpuEngine(host, fmt, engine, 0, 1, nullptr, std::move(leaf_net)) {}
    bool fused() const;
    ~GpuEngine();
    void iterate(int n);
    // n iterations bracketed by CUDA events on the engine's stream; returns ms
    double time_iterations(int n);
    Profile iterate_profiled();
    double exploitability(const HostSolver& host);       // chips
    void root_cfv(int p, int mode, float* out);          // eval sweep root values (mode 0 BR, 1 average)
    void sync_to_cpu(HostSolver& host, bool strategy_only);
    void synchronize();
    void update_locks(const HostSolver& host);
    uint32_t iteration() const;
    int format() const;
    const Plan& plan() const;
    const Spot* plan_spot() const;  // the spot the engine was built for
    uint64_t device_bytes() const;
    // algorithmic bytes of one CFR iteration / one BR check (traffic model)
    double iter_bytes() const;
    uint64_t upload_bytes() const;  // host-to-device bytes the constructor copied
    uint32_t iteration_kernels();   // kernels one iteration launches (the captured graph's kernel nodes)
    uint32_t river_programs() const;  // river rounds the river kernel solves (0: level sweeps everywhere)
    // device arena exports for tests (reference layout, decoded f32)
    void export_arena(int which, int p, float* out);
    // One action node's block (reference layout, f32) through a static device
    // scratch of kNodeScratchElems floats: no allocation, host or device, on
    // success.  Returns the element count written to out.
    size_t read_node_static(int which, uint32_t node, float* out, size_t out_len);
    void fill_staging(int which, int p);
    // Average strategy of one action node the device holds (reference layout
    // [action * nh + hand]), by the rule the evaluation sweeps use.
    void node_average_strategy(uint32_t node, float* out);
    // One evaluation sweep for player p over the whole tree -- mode 0 best
    // response (best_response.rs br_into), 1 average strategies (avg_into) --
    // then the node's value for p, both players' reach at the node and, when
    // p acts there, each child's value (child_ok[a] = 0 for children
    // evaluated in place, which have no slot).
    void node_sweep_values(uint32_t node, int p, int mode, float* cfv, float* reach0, float* reach1, float* child_cfv,
                           uint8_t* child_ok);
    // One evaluation sweep as node_sweep_values, then the values for p of
    // n nodes (out[k * nh_p ...]; ok[k] = 0 for a node without a slot).
    void sweep_values(int p, int mode, const uint32_t* nodes, int n, float* out, uint8_t* ok);
    // time one kind of level launch set: used by bench for the roofline
    void discounts(float* out3);
    // .gto written from the device arenas through a pinned double buffer (no
    // host arena copy): the bytes sync_to_cpu into an f32 host solver,
    // ensure_symmetric and save would write.  Header (config, locks) from
    // `host`, iteration from this engine.
    void save(const HostSolver& host, const std::string& path);
    // The arena section of a .gto (`in` at its first arena) streamed into the
    // device arenas: the state an engine built from a host solver loaded from
    // that file starts with.  The blocks the engine does not hold (symmetric
    // branches, children of chance nodes for dealt cards) go to `host`'s
    // arenas, so that after sync_to_cpu it holds what a host load would.
    // PCFR+ predictions restart at zero.
    void load_arenas(std::istream& in, HostSolver& host);

  private:
    friend class BatchKernel;
    std::unique_ptr<EngineImpl> d_;
};

// Many spots' CFR iterations in ONE persistent kernel launch per iteration
// (cfr_batch.cuh: a (spot, step, node-tile) work queue).  The engines stay
// owned by the caller and must outlive their use here; all live on the
// current device with one arena format, each a staged engine without river
// programs, shards or a leaf network (unsupported() says why not).  An
// iteration through the batch leaves every engine bit for bit as its own
// iterate(1) would; the engines' other calls (exploitability, syncs,
// queries) work between batched iterations as usual.
struct BatchShape {
    int tile = 4;         // node records per ticket (down, up, edge and chance steps)
    int ctas_per_sm = 0;  // persistent CTAs per SM (0: as many as fit)
};
struct BatchImpl;
class BatchKernel {
  public:
    BatchKernel();
    ~BatchKernel();
    static std::string unsupported(const GpuEngine& e);  // empty when the engine can join a batch
    void configure(const std::vector<GpuEngine*>& engines, const BatchShape& s);
    void configure_shape(const BatchShape& s);  // same engines, another shape
    BatchShape shape() const;
    int max_ctas_per_sm() const;  // resident CTAs per SM for the current engines' shared memory
    int grid() const;
    size_t tickets() const;       // tickets of one iteration
    uint64_t records() const;     // node records of one iteration (independent of the shape)
    void iterate(int n);          // n CFR iterations of every engine
    double time_iterations(int n);  // ms (CUDA events on the batch stream)

  private:
    std::unique_ptr<BatchImpl> d_;
};

uint64_t estimate_vram(const Spot& spot);
bool vram_info_mb(uint64_t* free_mb, uint64_t* total_mb);

}  // namespace gtob
