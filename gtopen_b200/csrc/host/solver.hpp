// Host-side solver state: the arenas (f32, or i16 regrets / u16 strategy sums
// with one scale per node), locks, iteration counter and algorithm of one
// spot -- the state the reference's `Solver` holds (cfr.rs:66-88) and that
// its GpuSolver copies from and syncs back to.  The CFR iteration itself runs
// on the GPU (engine.cu); this object is the source of truth for queries,
// locks and .gto saves (save.rs).
#pragma once
#include <cstdio>
#include <functional>
#include <istream>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "core.hpp"

namespace gtob {

enum Storage { kStoreF32 = 0, kStoreCompressed = 1 };
enum Algo { kDcfr = 0, kCfrPlus = 1, kPcfrPlus = 2 };
enum ArenaWhich { kRegrets = 0, kStrategy = 1, kPreds = 2 };

// store.rs:153-215
float encode_i16(const float* src, size_t n, int16_t* dst);
float encode_u16(const float* src, size_t n, uint16_t* dst);
float quantize_i16(const float* src, size_t n, float max, int16_t* dst);
float quantize_u16(const float* src, size_t n, float max, uint16_t* dst);
void decode_i16(const int16_t* q, size_t n, float scale, float* out);
void decode_u16(const uint16_t* q, size_t n, float scale, float* out);

struct Arena {
    int kind = 0;  // 0 f32, 1 i16, 2 u16
    std::vector<float> f;
    std::vector<int16_t> qi;
    std::vector<uint16_t> qu;
    std::vector<float> scale;  // per tree node
    void init(int k, uint64_t len, size_t nodes);
    size_t bytes() const;
    void read(uint32_t node, uint64_t off, size_t n, float* out) const;
    void write(uint32_t node, uint64_t off, size_t n, const float* src);
};

struct HostSolver {
    std::shared_ptr<Spot> spot;
    int storage = kStoreF32;
    int algo = kDcfr;
    bool use_iso = true;
    uint32_t iteration = 0;
    Arena regrets[2], strat[2], preds[2];
    bool have_preds = false;
    std::map<uint32_t, std::vector<float>> locks;
    std::map<uint32_t, std::string> lock_labels;
    bool sym_dirty = false;
    // Every arena still holds its initial zeros (nothing has written one since
    // construction): GpuEngine then skips the upload, the device arenas start
    // zeroed as well.
    bool arenas_zero = true;

    // with_arenas = false: a solver that only describes the spot (algorithm,
    // locks, iteration) for a GPU engine whose arenas never come back to the
    // host -- nothing may read or sync its arenas.
    HostSolver(std::shared_ptr<Spot> s, int storage_mode, int algorithm, bool iso, bool with_arenas = true);
    void ensure_preds();
    uint64_t arena_bytes() const;
    // whole-arena f32 image in the reference layout (action-major per node at data_offset)
    void arena_f32(int which, int p, float* out) const;
    void set_arena_f32(int which, int p, const float* in);
    // average strategy of an action node (cfr.rs:668-726), action-major na*nh
    void solved_strategy(uint32_t node, float* sig) const;
    void average_strategy(uint32_t node, float* sig) const;
    // suit-isomorphism materialisation (cfr.rs:749-871)
    void ensure_symmetric();
    // lock creation (query.rs:656-773); steps >= 0 are action indices, < 0 encode (-1 - card)
    uint32_t lock_node(const std::vector<int>& steps, int mode, const std::vector<float>& freqs,
                       const std::vector<std::pair<std::string, std::vector<float>>>& edits, const std::string& label);
    void walk(const std::vector<int>& steps, uint32_t* node, std::vector<float> reach[2]) const;
    std::vector<int> canonical_steps(const std::vector<int>& steps, std::array<uint8_t, 4>* perm) const;
    // Action-node copies ensure_symmetric makes, in its order: dst's blocks
    // become src's under hand permutation `perm` (a locked src gives its lock
    // as the strategy sums).  Empty without suit isomorphism.
    struct SymCopy {
        uint32_t src, dst;
        int perm;
    };
    std::vector<SymCopy> symmetric_copies() const;
    // .gto (save.rs)
    void save(const std::string& path) const;
    static std::unique_ptr<HostSolver> load(const std::string& path, int storage_mode);
    // The save with its arena section written by the caller: header (config,
    // `iteration`, this solver's locks), then write_arena(k, f) for k = 0..3
    // (regrets of players 0, 1, strategy sums of players 0, 1), each writing
    // its little-endian u64 length and f32 data; staged in `path`.tmp and
    // renamed over `path` once durable (save.rs:92-143).
    void save_stream(const std::string& path, uint32_t iteration,
                     const std::function<bool(int, FILE*)>& write_arena) const;
    // The header half of load (save.rs:149-188): the spot rebuilt from the
    // saved config (lenient), locks validated, arenas still zero; `in` is left
    // at the first arena section.
    static std::unique_ptr<HostSolver> load_header(std::istream& in, int storage_mode);

  private:
    void sym_walk(uint32_t node, const uint8_t* dealt, int nd,
                  const std::function<void(uint32_t, uint32_t, int)>& on_branch) const;
    void branch_walk(uint32_t src, uint32_t dst, int k, const std::function<void(uint32_t, uint32_t)>& on_action) const;
    void copy_branch(uint32_t src, uint32_t dst, int k);
};

// One arena section's length field of a .gto: write it, or read it and check
// it against the tree's arena size.
bool write_arena_len(FILE* f, uint64_t len);
uint64_t read_arena_len(std::istream& in, uint64_t expected);

void validate_locks(const Spot& spot, const std::vector<std::pair<uint32_t, std::vector<float>>>& locks);
void rake_to_target(float* sigma, int na, int nh, const float* reach, const float* target);
std::vector<float> normalize_freqs(const std::vector<float>& f, int na);

}  // namespace gtob
