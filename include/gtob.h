/*
 * gtob -- C ABI of the B200 discounted-CFR engine for heads-up postflop spots.
 *
 * This is the drop-in boundary for the reference solver crate's GPU module
 * (MatthewPDingle/GTOpen, crates/solver/src/gpu/mod.rs) and the parts of the
 * crate that path needs (game.rs Spot, cfr.rs Solver state, save.rs).  Every
 * entry point below names the reference item it replaces.  Conventions:
 *   - every function returns an int status: GTOB_OK (0) or a negative error
 *     class; gtob_last_error() returns a thread-local message (the reference
 *     returns Result<_, String> with "cuda: ..." messages, gpu/mod.rs:56-58);
 *   - handles are opaque and owned by the library (free with gtob_*_free);
 *   - buffers are plain host pointers and sizes; no handle is thread-safe
 *     (the reference drives one GpuSolver from one worker thread).
 */
#ifndef GTOB_H
#define GTOB_H
#include <stddef.h>
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define GTOB_OK 0
#define GTOB_EINVAL (-1)          /* bad argument / config / file: the reference's Err(String) */
#define GTOB_ENOMEM_DEVICE (-2)   /* device allocation failed */
#define GTOB_ECUDA (-3)           /* any other CUDA error */
#define GTOB_ETIMEOUT_QUEUE (-4)  /* a bounded device wait gave up */
#define GTOB_EIO (-5)             /* save/load I/O */

#define GTOB_STORAGE_F32 0        /* store.rs Storage::F32 */
#define GTOB_STORAGE_COMPRESSED 1 /* store.rs Storage::Compressed (i16 regrets, u16 sums) */
#define GTOB_ALGO_DCFR 0          /* cfr.rs Algorithm::Dcfr (alpha 1.5, beta 0, gamma 2) */
#define GTOB_ALGO_CFRPLUS 1       /* cfr.rs Algorithm::CfrPlus */
#define GTOB_ALGO_PCFRPLUS 2      /* cfr.rs Algorithm::PcfrPlus */
#define GTOB_DEVICE_FOLLOW_HOST (-1) /* device arena format follows the host storage */
#define GTOB_DEVICE_F32 0
#define GTOB_DEVICE_I16 1
#define GTOB_DEVICE_FP8 2         /* FP8 E4M3 arenas with a per-node scale (precision study; staged engine) */
#define GTOB_DEVICE_I16_SR 3      /* i16/u16 arenas requantised with stochastic rounding after each update */
#define GTOB_ENGINE_FUSED 0     /* terminals in their parents' kernels, f64 terminal sums */
#define GTOB_ENGINE_PLAIN 1     /* one launch per node kind and level, f64 terminal sums */
#define GTOB_ENGINE_FUSED_F32 2 /* fused with f32 terminal sums (the reference GPU kernels'
                                   precision; exploitability matches, but near-tied
                                   regrets may round differently than the CPU engine) */
#define GTOB_ENGINE_WARP 3      /* one warp per action node with its fold child evaluated
                                   in the warp; showdowns one CTA each; f64 terminal sums */
#define GTOB_ENGINE_STAGED 4    /* one CTA per node staging its arena blocks and vectors in
                                   shared memory with bulk copies; fold children in place;
                                   exact terminal sums (nodes with more than 4 actions: the
                                   warp engine's kernels) */
#define GTOB_ENGINE_STAGED_RIVER 5 /* the staged engine with every river betting round solved by
                                   one CTA walking it depth first (river programs); the same
                                   results bit for bit, slower on this device (see DESIGN) */
#define GTOB_ARENA_REGRETS 0
#define GTOB_ARENA_STRATEGY 1
#define GTOB_ARENA_PREDICTIONS 2

typedef struct gtob_spot gtob_spot;
typedef struct gtob_solver gtob_solver;
typedef struct gtob_gpu gtob_gpu;

/* gpu/mod.rs:22-36 KERNEL_NAMES and Profile{ms:[f64;7], launches:[u32;7]} */
typedef struct {
    double ms[7];
    uint32_t launches[7];
} gtob_profile;

typedef struct {
    uint64_t num_nodes;
    uint64_t num_action_nodes;
    uint64_t num_children;
    uint64_t num_actions;
    uint64_t data_size[2];
    uint32_t num_hands[2];
    uint32_t root_street;
    uint32_t num_suit_perms;
} gtob_spot_info;

typedef struct {
    uint64_t device_bytes;
    uint64_t visited_nodes;
    uint64_t cfv_slots;
    uint64_t reach_slots[2];
    uint64_t device_action_nodes[2];
    uint64_t visited_terminals;
    uint32_t num_levels;
    uint32_t num_river_slots;
    int32_t arena_format;
    double iter_bytes; /* algorithmic bytes of one CFR iteration */
    uint64_t upload_bytes; /* host-to-device bytes copied by gtob_gpu_new (plan tables, arenas) */
    uint32_t iteration_kernels; /* kernel launches of one iteration (kernel nodes of its CUDA graph;
                                   reading it captures that graph if no iteration has run yet) */
    uint32_t river_programs;    /* river betting rounds solved by river programs (0: level sweeps) */
} gtob_gpu_info;

/* Thread-local message of the last failed call (Result::Err text). */
const char* gtob_last_error(void);
/* gpu/mod.rs:22-30 KERNEL_NAMES[k], k in 0..7 */
const char* gtob_kernel_name(int k);
const char* gtob_version(void);

/* ---- Spot (game.rs) ---------------------------------------------------- */
/* Spot::new / Spot::new_with_limit / Spot::new_lenient_with_limit (game.rs:103-133):
 * spot_config_json is the reference SpotConfig JSON (serde conventions:
 * {"PotPct":33}, {"PrevMult":2.5}, "AllIn"); max_nodes 0 = no budget. */
int gtob_spot_from_json(const char* spot_config_json, uint64_t max_nodes, int lenient, gtob_spot** out);
void gtob_spot_free(gtob_spot* spot);
int gtob_spot_info_get(const gtob_spot* spot, gtob_spot_info* out);
/* Tree arrays (tree.rs:178-211), each of num_nodes entries; NULL skips. */
int gtob_spot_tree(const gtob_spot* spot, uint8_t* kind, uint8_t* player, uint8_t* street, uint8_t* nchild,
                   uint32_t* child_start, uint32_t* action_start, uint64_t* data_offset, double* put0,
                   double* put1, double* t_win, double* t_lose, double* t_tie);
int gtob_spot_children(const gtob_spot* spot, uint32_t* out);
int gtob_spot_actions(const gtob_spot* spot, int32_t* kind, double* amount);
/* Spot::hands / weights / same_combo (game.rs:82-100) */
int gtob_spot_hands(const gtob_spot* spot, int player, uint8_t* c1, uint8_t* c2, float* weight, uint32_t* same_combo);
/* suit_perms (num_suit_perms x 4) and hand_perm[player] (num_suit_perms x num_hands) */
int gtob_spot_suit_perms(const gtob_spot* spot, uint8_t* perms4, uint16_t* hand_perm0, uint16_t* hand_perm1);
/* RiverTable::get for dealt cards (game.rs:36-62); returns the count of (strength, index) pairs */
int gtob_spot_river(const gtob_spot* spot, int player, const uint8_t* dealt, int ndealt, uint32_t* strength,
                    uint16_t* index);
double gtob_spot_pair_weight_sum(const gtob_spot* spot);
/* evaluator::evaluate7 (evaluator.rs:68) */
uint32_t gtob_evaluate7(const uint8_t* cards7);
/* range::Range::parse (range.rs:28) into 1326 weights indexed by combo_index */
int gtob_parse_range(const char* text, float* weights1326);
/* gpu::estimate_vram (gpu/mod.rs:946) and gpu::vram_info_mb (gpu/mod.rs:953) */
uint64_t gtob_estimate_vram(const gtob_spot* spot);
int gtob_vram_info_mb(uint64_t* free_mb, uint64_t* total_mb);

/* ---- host solver state (cfr.rs Solver, save.rs, query.rs locks) --------- */
/* Solver::with_storage (cfr.rs:122) + algo / use_isomorphism fields */
int gtob_solver_new(gtob_spot* spot, int storage, int algo, int use_iso, gtob_solver** out);
void gtob_solver_free(gtob_solver* solver);
uint32_t gtob_solver_iteration(const gtob_solver* solver);
int gtob_solver_set_iteration(gtob_solver* solver, uint32_t iteration);
uint64_t gtob_solver_arena_bytes(const gtob_solver* solver);
/* whole arena in the reference layout (save.rs:76-90): data_size[player] f32 */
int gtob_solver_get_arena(const gtob_solver* solver, int which, int player, float* out);
int gtob_solver_set_arena(gtob_solver* solver, int which, int player, const float* in);
/* Solver::average_strategy (cfr.rs:729) / solved_strategy_into (cfr.rs:679): na*nh, action-major */
int gtob_solver_average_strategy(const gtob_solver* solver, uint32_t node, float* out);
int gtob_solver_solved_strategy(const gtob_solver* solver, uint32_t node, float* out);
/* Solver::lock_node (query.rs:700-773).  steps: >= 0 action index, < 0 card (-1 - card).
 * mode 0 Freeze, 1 Range{freqs}, 2 Hands{edits}: edits_json = [["AcAd",[1,0]],...] */
int gtob_solver_lock_node(gtob_solver* solver, const int32_t* steps, int nsteps, int mode, const float* freqs,
                          int nfreqs, const char* edits_json, const char* label, uint32_t* node_out);
int gtob_solver_set_lock(gtob_solver* solver, uint32_t node, const float* sigma, uint64_t n, const char* label);
int gtob_solver_clear_locks(gtob_solver* solver);
int gtob_solver_num_locks(const gtob_solver* solver);
/* Solver::ensure_symmetric (cfr.rs:749) */
int gtob_solver_ensure_symmetric(gtob_solver* solver);
/* Solver::save (save.rs:92) / Solver::load_with_storage (save.rs:149) */
int gtob_save(const gtob_solver* solver, const char* path);
int gtob_load(const char* path, int storage, gtob_solver** out);

/* ---- GPU engine (gpu/mod.rs GpuSolver) ----------------------------------- */
/* Device for later gtob_gpu_new calls on this thread (the reference always
 * opens device 0, gpu/mod.rs:152; one process per GPU sets its own). */
int gtob_set_device(int device);
/* GpuSolver::new (gpu/mod.rs:146) with the staged engine; device_format GTOB_DEVICE_* */
int gtob_gpu_new(const gtob_solver* solver, int device_format, gtob_gpu** out);
/* GpuSolver::new with the engine choice: GTOB_ENGINE_STAGED (the default of
 * gtob_gpu_new), GTOB_ENGINE_FUSED (terminals evaluated inside their parents'
 * kernels), GTOB_ENGINE_PLAIN (one launch per node kind and level, the
 * reference's kernel split), GTOB_ENGINE_FUSED_F32 or GTOB_ENGINE_WARP. */
int gtob_gpu_new_ex(const gtob_solver* solver, int device_format, int engine, gtob_gpu** out);
void gtob_gpu_free(gtob_gpu* gpu);
/* GpuSolver::iterate (gpu/mod.rs:304), n times */
int gtob_gpu_iterate(gtob_gpu* gpu, int n);
/* GpuSolver::iterate_profiled (gpu/mod.rs:351) */
int gtob_gpu_iterate_profiled(gtob_gpu* gpu, gtob_profile* out);
/* GpuSolver::exploitability (gpu/mod.rs:367), chips */
int gtob_gpu_exploitability(gtob_gpu* gpu, const gtob_solver* solver, double* chips);
/* GpuSolver::sync_to_cpu (gpu/mod.rs:845) / sync_strategy (gpu/mod.rs:871) */
int gtob_gpu_sync_to_cpu(gtob_gpu* gpu, gtob_solver* solver);
int gtob_gpu_sync_strategy(gtob_gpu* gpu, gtob_solver* solver);
/* GpuSolver::synchronize (gpu/mod.rs:889) */
int gtob_gpu_synchronize(gtob_gpu* gpu);
/* GpuSolver::update_locks (gpu/mod.rs:894) */
int gtob_gpu_update_locks(gtob_gpu* gpu, const gtob_solver* solver);
/* GpuSolver::iteration (pub field) */
uint32_t gtob_gpu_iteration(const gtob_gpu* gpu);
int gtob_gpu_info_get(gtob_gpu* gpu, gtob_gpu_info* out);
/* root counterfactual values of one evaluation sweep (gpu/mod.rs:400-416; mode 0 BR, 1 average) */
int gtob_gpu_root_cfv(gtob_gpu* gpu, int player, int mode, float* out);
/* device arena decoded to the reference layout, without touching the host solver */
int gtob_gpu_export_arena(gtob_gpu* gpu, int which, int player, float* out);
/* n iterations bracketed by CUDA events on the engine's own stream (ms) */
int gtob_gpu_time_iterations(gtob_gpu* gpu, int n, double* ms);
/* the last discounts the device computed (pos, neg, strat) */
int gtob_gpu_discounts(gtob_gpu* gpu, float* out3);

/* Solver::save (save.rs:92-143) of the state GpuSolver::sync_to_cpu
 * (gpu/mod.rs:845) followed by Solver::ensure_symmetric (cfr.rs:749) leaves
 * in an f32 host solver, written from the device arenas: the arenas are
 * decoded on the device, symmetric branches gathered there, and the file is
 * streamed through two 32 MiB pinned buffers -- no host arena is touched.
 * Header (config, locks, labels) from `solver`, iteration from `gpu`; staged
 * in path.tmp and renamed once durable, as the reference's save. */
int gtob_gpu_save(gtob_gpu* gpu, const gtob_solver* solver, const char* path);
/* Solver::load_with_storage (save.rs:149-227) + GpuSolver::new
 * (gpu/mod.rs:146) with the arenas streamed from the file straight into
 * device memory.  *solver_out gets the spot (rebuilt leniently from the
 * saved config), locks, iteration and the blocks the device does not hold
 * (symmetric branches, children of chance nodes for dealt cards); the blocks
 * the device holds stay zero on the host until gtob_gpu_sync_to_cpu.
 * *gpu_out holds the loaded state (device_format GTOB_DEVICE_*, engine
 * GTOB_ENGINE_*).  PCFR+ predictions start at zero. */
int gtob_gpu_load(const char* path, int storage, int device_format, int engine, gtob_solver** solver_out,
                  gtob_gpu** gpu_out);

/* ---- node queries over the device arenas (query.rs:304-645) ------------ */
/* node_view's numbers (query.rs:490-600) at the node a path reaches, read
 * from device memory instead of a synced host solver: steps are action
 * indices (>= 0) and dealt cards (-1 - card) from the root, as
 * gtob_solver_lock_node takes them.  The strategies along the path come from
 * the device blocks (locks from `solver`), the values from one
 * average-strategy evaluation sweep per player (best_response.rs:128-223).
 * Through a suit-isomorphic branch the device holds the representative; its
 * values are returned under the hand permutation ensure_symmetric applies.
 * Outputs (NULL to skip): reach_p / valid_p / eq_p / ev_p per hand of player
 * p (eq: equity against the opponent's reach over the remaining runouts,
 * best_response.rs:292-386, NaN without compatible mass; ev in the pot-share
 * convention, NaN where valid <= 1e-9); at an action node,
 * strategy and action_ev (num_actions x hands of the actor, action-major).
 * Supported on the staged and plain engines (showdowns with slots).  The
 * sweeps reuse the engine's buffers: do not call it while another call on
 * the same gpu handle is running. */
typedef struct {
    uint32_t node;       /* tree index */
    int32_t kind;        /* 0 action, 1 chance, 2 fold, 3 showdown */
    int32_t player;      /* actor at an action node, else -1 */
    int32_t num_actions; /* at an action node, else 0 */
} gtob_node_info;
int gtob_gpu_node_values(gtob_gpu* gpu, const gtob_solver* solver, const int* steps, int nsteps, gtob_node_info* info,
                         float* reach0, float* reach1, float* valid0, float* valid1, float* eq0, float* eq1,
                         float* ev0, float* ev1, float* strategy, float* action_ev);
/* node_view's structure (query.rs:353-461, 490-640) at the node a path
 * reaches, without the per-hand numbers: a JSON object with the reference's
 * field names -- node, node_type, street, board, pot, put, player (null off
 * action nodes), actions [{label, kind, amount}] with tree.rs:139-169's
 * labels, available_cards (chance nodes, else null), locked (on the orbit
 * representative) and history (one step per path node, then the current
 * node: kind, player, stack, pot, street, actions, chosen, card).  Host only.
 * Writes at most cap bytes including the terminating NUL; *needed receives
 * the full size (call again with a larger buffer when it exceeds cap). */
int gtob_solver_path_view(const gtob_solver* solver, const int* steps, int nsteps, char* out, uint64_t cap,
                          uint64_t* needed);
/* runouts (query.rs:964-1106) at the chance node a path reaches: one row per
 * available card, descending -- the action frequencies at the following
 * action node (freqs[row * max_actions + a], reach-weighted), and per player
 * the reach x valid weighted equity (eq_p of node values; equity enumerates
 * the remaining runouts, best_response.rs:292-386) and average-strategy EV
 * (NaN when there is no mass).  *n_rows receives the row count (at most
 * max_rows), *player / *num_actions the actor at the runout nodes (-1 / 0 for
 * none), *pot the pot there. */
typedef struct {
    int32_t card;
    float eq[2];
    float ev[2];
} gtob_runout_row;
int gtob_gpu_runouts(gtob_gpu* gpu, const gtob_solver* solver, const int* steps, int nsteps, gtob_runout_row* rows,
                     float* freqs, int max_rows, int max_actions, int* n_rows, int* player, int* num_actions,
                     double* pot);

/* exploit_view's numbers (query.rs:808-930) for `exploiter` at the node a
 * path reaches, from device memory (one best-response and one
 * average-strategy evaluation sweep, strategies along the canonical path
 * from the device blocks): per hand of the exploiter in the browsed branch
 * reach, valid, br_ev, cur_ev and gain (NaN where valid <= 1e-9); where the
 * exploiter acts, br_strategy (one-hot, ties within 1e-5 split, the lock at a
 * locked node) and action_ev (num_actions x hands, action-major); averages =
 * {avg_br_ev, avg_cur_ev, avg_gain} weighted by reach x valid (NaN when
 * there is no mass).  info->node is the representative node read. */
int gtob_gpu_exploit_values(gtob_gpu* gpu, const gtob_solver* solver, const int* steps, int nsteps, int exploiter,
                            gtob_node_info* info, float* reach, float* valid, float* br_ev, float* cur_ev, float* gain,
                            float* br_strategy, float* action_ev, float* averages);

/* ---- one spot over several shards (a flop split by turn card) ---------- */
/* A spot split by its first chance card: every shard holds the tree above
 * the first chance nodes and every nshards-th representative subtree below
 * them; before the top chance nodes add up their children, the children's
 * values are summed over the shards (each is nonzero on the one shard that
 * holds it, so the sum is exact and every shard computes what one engine
 * would).  Each shard's arenas hold its own nodes and the top part. */
/* ncclGetUniqueId (libnccl.so.2 is loaded on first use) for rank 0 to share. */
int gtob_nccl_unique_id(unsigned char out[128]);
/* Shard `rank` of `world` processes, one GPU each (the current device),
 * reducing over NCCL inside the iteration's CUDA graph; every rank must call
 * it with the same id (ncclCommInitRank: it returns once all have joined). */
int gtob_gpu_new_sharded(const gtob_solver* solver, int device_format, int engine, int rank, int world,
                         const unsigned char id[128], gtob_gpu** out);
/* Shard `rank` of `world` processes that sum over a channel of the caller's
 * own instead of NCCL (a torch.distributed gloo group, MPI, sockets): after
 * each level whose chance nodes add up split subtrees, the shard's `count`
 * values are copied to a host buffer and fn(user, values, count) is called on
 * the calling thread; it must leave there the element-wise sum over every
 * rank and return 0 (non-zero fails the call with GTOB_EINVAL and that
 * status).  Every rank must make the same calls in the same order (iterate,
 * exploitability and the queries each reduce).  Plain launches, no graphs;
 * no kernel waits on another rank.  No reference counterpart (the reference
 * solves one spot on one GPU). */
typedef int (*gtob_reduce_fn)(void* user, float* values, size_t count);
int gtob_gpu_new_sharded_host(const gtob_solver* solver, int device_format, int engine, int rank, int world,
                              gtob_reduce_fn fn, void* user, gtob_gpu** out);
/* All nshards shards in this process on the current device, reducing on the
 * host (no graphs; each call below runs the shards on their own threads):
 * the whole sharded computation on one GPU, to check it against one engine. */
typedef struct gtob_shards gtob_shards;
int gtob_shards_new(const gtob_solver* solver, int device_format, int engine, int nshards, gtob_shards** out);
int gtob_shards_iterate(gtob_shards* shards, int n);
int gtob_shards_exploitability(gtob_shards* shards, const gtob_solver* solver, double* chips);
/* an arena of all shards merged in the reference layout (each node from a
 * shard that holds it) */
int gtob_shards_export_arena(gtob_shards* shards, int which, int player, float* out);
/* every shard's nodes (and the shared top part) into one host solver, as
 * gtob_gpu_sync_to_cpu of each shard in turn */
int gtob_shards_sync_to_cpu(gtob_shards* shards, gtob_solver* solver, int strategy_only);
void gtob_shards_free(gtob_shards* shards);
/* The persistent batch kernel's work queue for these spots, built on the host
 * with no GPU (the staged engine's plans): one segment per span of one step of
 * one spot, ordered by step then spot, with the ticket it starts at and the
 * tickets of its spot's earlier steps it waits for (need).  kind: 0 discounts,
 * 1 root reach, 2 down-sweep action nodes, 3 chance edges, 4 showdown
 * batches, 5 chance nodes, 6 / 7 up-sweep action nodes of the traverser / its
 * opponent; p: traverser (edges: mask of the players whose reach is
 * refreshed).  *nseg, *ntickets and *nrecords receive the totals; at most cap
 * segments are written.  It exists to check the queue's order on the CPU; no
 * reference counterpart. */
typedef struct {
    uint64_t first;
    uint32_t start, count, need, spot, step;
    int32_t kind, p, tile;
} gtob_batch_segment;
int gtob_spot_batch_queue(gtob_spot* const* spots, int n, int use_iso, int tile, gtob_batch_segment* out, int cap,
                          int* nseg, uint64_t* ntickets, uint64_t* nrecords);
/* The plan partition without a GPU: visited[node] = 1 for every node shard
 * `shard` of `nshards` visits (staged engine's plan). */
int gtob_spot_shard_visited(const gtob_spot* spot, int use_iso, int shard, int nshards, uint8_t* visited);

/* ---- batch of spots (solve_cli.rs:125-215 batch) ------------------------ */
/* The reference's batch report solves one board after another
 * (solve_quiet, solve_cli.rs:338-362).  A batch solves many spots on one GPU
 * at once: `workers` host threads each take the next spot, build its engine
 * (own streams and CUDA graphs), run solve_quiet's loop -- one iteration at a
 * time, exploitability when the iteration is a multiple of check_every (the
 * reference: 20) or reaches max_iterations, stop at target_pct or
 * max_iterations -- read the root EVs, sync the solver back and free the
 * engine.  Engines of different workers run concurrently on the device.
 * storage, algo, use_iso as gtob_solver_new; device_format / engine as
 * gtob_gpu_new_ex.  Call
 * gtob_batch_run with the device current; an error in one spot stays in its
 * row (status, gtob_batch_error) and the others go on. */
typedef struct gtob_batch gtob_batch;
typedef struct {
    int32_t status;      /* GTOB_OK, or the error class of this spot */
    uint32_t iterations; /* iterations run */
    double exploit_pct;  /* last exploitability check, % of the starting pot */
    double seconds;      /* wall time of this spot: engine build, solve, EVs, sync */
    double ev[2];        /* reach-weighted root EV per player, pot-share convention (solve_cli.rs:176-188) */
} gtob_batch_row;
/* keep = 1: one host solver per spot, synced after its solve and returned
 * by gtob_batch_solver; keep = 0: no solver is kept (each worker solves
 * against a host solver without arenas and drops it), so host memory stays
 * bounded by the spots in flight -- the report case. */
int gtob_batch_new(gtob_spot* const* spots, int n, int storage, int algo, int use_iso, int device_format, int engine,
                   int keep, gtob_batch** out);
int gtob_batch_run(gtob_batch* batch, uint32_t max_iterations, double target_pct, uint32_t check_every, int workers);
/* The same batch solved on ONE persistent kernel: every iteration of up to
 * `window` spots in flight is a single launch (a CUDA graph of one kernel)
 * whose CTAs take (spot, step, node tile) tickets from a device work queue;
 * a ticket waits (bounded) only for its own spot's earlier steps.  Spots
 * join as a builder thread readies their engines and leave at their checks
 * (the same rule as gtob_batch_run), so every row equals the spot solved
 * alone, bit for bit.  The kernel's shape -- node records per ticket, CTAs
 * per SM -- is tuned per size class on the batch's first iterations (each
 * trial is an ordinary iteration) and cached in GTOB_TUNE_CACHE or
 * ~/.cache/gtob/batch_shapes.txt.  Staged engines only: the batch's engine
 * argument is not used; a spot the kernel cannot take (nodes of more than 4
 * actions) fails in its row.  No reference counterpart (solve_cli.rs's
 * batch solves one spot at a time). */
int gtob_batch_run_persistent(gtob_batch* batch, uint32_t max_iterations, double target_pct, uint32_t check_every,
                              int window);
typedef struct {
    uint64_t launches;  /* batched iterations, one kernel launch each */
    double kernel_ms;   /* their device time (CUDA events) */
    int32_t tuned;      /* size classes tuned during the run */
    int32_t tile, ctas_per_sm, grid;  /* the last shape (ctas_per_sm 0: as many as fit) and its grid */
} gtob_batch_stats;
int gtob_batch_stats_get(const gtob_batch* batch, gtob_batch_stats* out);
int gtob_batch_size(const gtob_batch* batch);
int gtob_batch_row_get(const gtob_batch* batch, int i, gtob_batch_row* out);
/* spot i's root counterfactual values of the average strategies, per hand of
 * player p (*n = hand count; empty until the spot is solved) */
int gtob_batch_root_cfv(gtob_batch* batch, int i, int player, float* out, int cap, int* n);
/* the message of a failed row ("" when the row solved) */
const char* gtob_batch_error(const gtob_batch* batch, int i);
/* the i-th host solver, owned by the batch (valid until gtob_batch_free);
 * NULL when the batch keeps none */
gtob_solver* gtob_batch_solver(gtob_batch* batch, int i);
void gtob_batch_free(gtob_batch* batch);

/* No counterpart in the reference.  One action node's arena block (which:
 * GTOB_ARENA_*), decoded to f32 in the reference layout [action * nh + hand],
 * the same values gtob_gpu_export_arena gives for that node, read through a
 * static device scratch of GTOB_NODE_SCRATCH_ELEMS floats: on success the
 * call allocates no host or device memory.  It serves callers that must not
 * allocate while a solve holds the device -- a viewer polling one node
 * mid-solve, where the arenas were sized to fill HBM (a cudaMalloc there can
 * fail, and cudaMalloc/cudaFree synchronise the device) and where
 * gtob_gpu_export_arena would move a whole arena.
 *   - Blocks of more than GTOB_NODE_SCRATCH_ELEMS elements (nchild * hands)
 *     are refused with GTOB_EINVAL; so is out_len < the block size.
 *   - Call it with the solver's device current.  The first call on a device
 *     resolves the scratch address (cudaGetSymbolAddress) and loads the
 *     kernel, which may make the CUDA runtime allocate: make that first call
 *     before capturing any stream.
 *   - Nothing in the scratch has to start at zero: each call writes every
 *     element it copies out.
 *   - The scratch is one array per device: calls that overlap in time (two
 *     threads, or two solvers on one device) race on it.  The call returns
 *     after its copy is complete, so calls made one after another are safe.
 * *written (if not NULL) receives the element count. */
#define GTOB_NODE_SCRATCH_ELEMS 16384
int gtob_gpu_read_node_static(gtob_gpu* gpu, int which, uint32_t node, float* out, uint64_t out_len,
                              uint64_t* written);

/* ---- the turn-leaf value network (depth-limited solves) ----------------- */
/* No counterpart in the reference: a learned stand-in for the turn subtree
 * at the leaves of depth-limited solves.  A fully
 * connected net: din inputs, nhidden GELU layers of dh units, dout linear
 * outputs; BF16 weights and activations, FP32 accumulation and master
 * weights, every matrix product on a hand-written tcgen05 kernel.  Training
 * minimises the masked squared error mean(mask * (y - t)^2) over rows x dout
 * with Adam (0.9, 0.999, 1e-8). */
typedef struct gtob_net gtob_net;
int gtob_net_new(int din, int dh, int nhidden, int dout, uint64_t seed, gtob_net** out);
void gtob_net_free(gtob_net* net);
/* layer l in [0, nhidden]: weights [out x in] row-major and bias [out] (f32) */
int gtob_net_get_params(gtob_net* net, int layer, float* w, float* b);
int gtob_net_set_params(gtob_net* net, int layer, const float* w, const float* b);
/* the gradients of the last gtob_net_gradients call */
int gtob_net_get_grads(gtob_net* net, int layer, float* w, float* b);
/* rows x din inputs -> rows x dout outputs (host buffers) */
int gtob_net_forward(gtob_net* net, const float* x, int rows, float* y);
/* one forward + backward; *loss = the masked mean squared error */
int gtob_net_gradients(gtob_net* net, const float* x, const float* t, const float* mask, int rows, double* loss);
/* epochs of shuffled batches (batch a multiple of 128); losses[epoch] = the
 * epoch's mean batch loss (NULL: not reported) */
int gtob_net_train(gtob_net* net, const float* x, const float* t, const float* mask, int n, int epochs, int batch,
                   float lr, uint64_t seed, float* losses);
/* A depth-limited flop solve: the plan cuts the tree at the chance nodes
 * dealing the turn where betting follows (all-in runouts stay exact), and
 * after every down sweep the net evaluates each such leaf for every turn
 * card -- inputs: board + turn one-hot (52), pot / remaining stack, both
 * players' reach over the 1326 combos divided by its sum (hands holding the
 * card zeroed); outputs: both players' counterfactual values over the combos
 * divided by pot x the opponent's reach sum -- zero-sum corrected, scaled
 * back and averaged over the cards as the chance node would (x 1/45).  The
 * net must map 2705 inputs to 2652 outputs; it serves one solver at a time.
 * The other gtob_gpu_* calls work as on any solver (save and load refuse). */
int gtob_gpu_new_dl(const gtob_solver* solver, gtob_net* net, int device_format, int engine, gtob_gpu** out);
/* The depth-limited plan of a flop spot without a GPU: its leaves (tree
 * node, pot, remaining stack; *n = count) and, if visited is not NULL, one
 * byte per tree node, 1 for the nodes its sweeps visit. */
int gtob_spot_dl_plan(const gtob_spot* spot, uint32_t* nodes, float* pot, float* stack, int cap, int* n,
                      uint8_t* visited);
/* the depth-limited solver's leaves: tree node, pot, remaining stack; *n = count */
int gtob_gpu_leaves(gtob_gpu* gpu, uint32_t* nodes, float* pot, float* stack, int cap, int* n);
/* one evaluation sweep for player p (mode 0 best response, 1 average
 * strategies), then node's value for p and both players' reach there (any
 * output may be NULL) */
int gtob_gpu_node_sweep(gtob_gpu* gpu, uint32_t node, int p, int mode, float* cfv, float* reach0, float* reach1);
/* the average strategy [action * hands + hand] of an action node the GPU
 * solver holds */
int gtob_gpu_node_strategy(gtob_gpu* gpu, uint32_t node, float* out);
/* mean device time (CUDA events, after one untimed launch) of the
 * tensor-core product on m x k and n x k bf16 operands resident in HBM */
int gtob_gemm_time(int m, int n, int k, int reps, double* ms);
/* The tensor-core matrix product alone: C[M x N] = A[M x K] * B[N x K]^T,
 * A and B bf16 bit patterns (host), C f32; M, N multiples of 128, K of 64. */
int gtob_gemm_bf16(const uint16_t* a, const uint16_t* b, int m, int n, int k, float* c);

#ifdef __cplusplus
}
#endif
#endif
