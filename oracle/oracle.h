/*
 * CPU oracle for the GTOpen postflop DCFR hot path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library restates, in plain C++, the reference solver crate's CPU engine
 * (crates/solver/src/{cards,evaluator,range,tree,game,store,cfr,best_response,
 * query}.rs).  It exists so that tests, the smoke check and the CPU-baseline
 * leg of bench.py can check and time the product (libgtob) against the
 * reference's algorithm.  The product library never links or calls it.
 *
 * Pinning: tests/test_oracle_*.py check this library against the reference's
 * own known-answer tests (evaluator.rs, cards.rs, store.rs, range.rs,
 * convergence.rs) and against the reference's checked-in bench logs
 * (bench/new_f32_dcfr.log: the bench_spot.json trajectory).
 *
 * Two switches that the reference has no flag for:
 *   prune = 1  reproduces the reference CPU engine (zero-reach pruning,
 *              cfr.rs:424-430); prune = 0 traverses everything, which is the
 *              semantics of a level-synchronous GPU sweep (gpu/kernels.cu).
 *   orc_solver_exploitability_f64 is an all-double best-response oracle.
 */
#ifndef GTOB_ORACLE_H
#define GTOB_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct { int kind; double value; } orc_size; /* 0 PotPct, 1 PrevMult, 2 AllIn */

typedef struct {
    const char* board;
    const char* range_oop;
    const char* range_ip;
    double starting_pot, effective_stack, rake_pct, rake_cap, allin_threshold;
    int add_allin;
    int max_raises;
    int n[2][3][3];              /* [player][street][bet, raise, donk] */
    orc_size sizes[2][3][3][8];
} orc_config;

typedef struct orc_spot orc_spot;
typedef struct orc_solver orc_solver;

const char* orc_last_error(void);
void orc_set_threads(int n);
int orc_get_threads(void);

/* cards / evaluator / range */
uint32_t orc_evaluate7(const uint8_t* cards7);
void orc_ref_eval7(const uint8_t* cards7, uint32_t* cat, uint8_t* ranks, int* nranks);
int orc_straight_top(uint16_t mask);            /* -1 = none */
int orc_combo_index(int c1, int c2);
void orc_combo_from_index(int idx, int* hi, int* lo);
int orc_parse_range(const char* s, float* weights1326);   /* 0 ok */
int orc_parse_cards(const char* s, uint8_t* out, int cap); /* count or -1 */
int orc_canonical_flops(char* boards6, uint32_t* weights, int cap);
int orc_canonical_flops_subset(int n, char* boards6, uint32_t* weights, int cap);

/* store codecs (store.rs) */
float orc_encode_i16(const float* src, int n, int16_t* dst);
float orc_encode_u16(const float* src, int n, uint16_t* dst);
void orc_decode_i16(const int16_t* q, int n, float scale, float* out);
void orc_decode_u16(const uint16_t* q, int n, float scale, float* out);

/* spot / tree */
orc_spot* orc_spot_new(const orc_config* cfg, int lenient, uint64_t max_nodes);
void orc_spot_free(orc_spot* s);
int64_t orc_spot_num_nodes(const orc_spot* s);
int64_t orc_spot_num_children(const orc_spot* s);
int64_t orc_spot_num_actions(const orc_spot* s);
int orc_spot_num_hands(const orc_spot* s, int p);
uint64_t orc_spot_data_size(const orc_spot* s, int p);
int orc_spot_num_perms(const orc_spot* s);
/* node arrays, each of length num_nodes (NULL to skip) */
void orc_spot_nodes(const orc_spot* s, uint8_t* kind, uint8_t* player, uint8_t* street,
                    uint8_t* nchild, uint32_t* child_start, uint32_t* action_start,
                    uint64_t* data_off, double* put0, double* put1, double* twin,
                    double* tlose, double* ttie);
void orc_spot_children(const orc_spot* s, uint32_t* out);
void orc_spot_actions(const orc_spot* s, int* kind, double* amount); /* 0 fold 1 check 2 call 3 bet 4 raise */
void orc_spot_hands(const orc_spot* s, int p, uint8_t* c1, uint8_t* c2, float* w);
void orc_spot_same_combo(const orc_spot* s, int p, uint32_t* out);
void orc_spot_perms(const orc_spot* s, uint8_t* perms4, uint16_t* hand_perm0, uint16_t* hand_perm1);
/* river table entry for dealt cards (n extra = 0,1,2); returns count, fills (strength, idx) */
int orc_spot_river(const orc_spot* s, int p, const uint8_t* dealt, int ndealt, uint32_t* str, uint16_t* idx);
double orc_spot_pair_weight_sum(const orc_spot* s);

/* terminal evaluators (game.rs); exact = 0: the reference's f64 running sums,
   1: exact fixed-point sums (the GPU engine's order-independent arithmetic) */
void orc_fold_cfv(const orc_spot* s, int p, const float* reach_o, float amount, int exact, float* out);
void orc_showdown_cfv(const orc_spot* s, int p, const uint8_t* dealt, int ndealt, const float* reach_o,
                      float win, float lose, float tie, int exact, float* out);

/* solver (cfr.rs / best_response.rs) */
/* FP8 E4M3 codec of the precision-study arenas (round to nearest even, saturating to +-448) */
void orc_fp8_encode(const float* x, int n, uint8_t* out);
void orc_fp8_decode(const uint8_t* q, int n, float* out);
/* compressed: 0 f32 arenas, 1 i16 regrets / u16 strategy sums (store.rs), 2 FP8 E4M3 (precision study) */
orc_solver* orc_solver_new(orc_spot* s, int compressed, int algo, int use_iso, int prune);
void orc_solver_free(orc_solver* v);
/* terminal sums of the solver's sweeps: 0 the reference's f64 (default), 1 exact fixed point */
void orc_solver_set_sums(orc_solver* v, int exact);
/* 16-bit arenas' requantisation after an update: 0 round to nearest even (store.rs, default), 1 stochastic */
void orc_solver_set_rounding(orc_solver* v, int stochastic);
void orc_solver_iterate(orc_solver* v, int n);
uint32_t orc_solver_iteration(const orc_solver* v);
double orc_solver_exploitability(orc_solver* v);
double orc_solver_exploitability_f64(orc_solver* v);
/* which: 0 regrets, 1 strategy sums, 2 PCFR+ predictions. Decoded to f32, action-major */
int orc_solver_get_arena(const orc_solver* v, int which, int p, float* out);
int orc_solver_set_arena(orc_solver* v, int which, int p, const float* in);
void orc_solver_set_iteration(orc_solver* v, uint32_t it);
int orc_solver_set_lock(orc_solver* v, uint32_t node, const float* sigma, int n);
void orc_solver_clear_locks(orc_solver* v);
int orc_solver_avg_strategy(const orc_solver* v, uint32_t node, float* out);
int orc_solver_solved_strategy(const orc_solver* v, uint32_t node, float* out);
void orc_solver_ensure_symmetric(orc_solver* v);
void orc_solver_root_br_cfv(orc_solver* v, int p, float* out);
void orc_solver_discounts(int algo, uint32_t t, float* pos, float* neg, float* strat);
/* lock creation (query.rs): path steps >= 0 are action indices, < 0 encode card (-1 - card) */
/* node_view's traversals at the node a path reaches (query.rs:490-600):
 * cfv[nh_p] = traverse_avg (avg = 1) or traverse_br (avg = 0) of the node
 * for p, child_cfv[na*nh_p] (p acting) per child,
 * walk reach of both players; returns the node index or -1 */
int orc_solver_node_values(orc_solver* v, const int* steps, int nsteps, int p, int avg, float* cfv, float* child_cfv,
                           float* r0, float* r1);
int orc_solver_walk_path(orc_solver* v, const int* steps, int nsteps, uint32_t* node,
                         float* reach0, float* reach1);
void orc_rake_to_target(float* sigma, int na, int nh, const float* reach, const float* target);
int orc_normalize_freqs(const float* freqs, int n, float* out);
int orc_solver_lock_node(orc_solver* v, const int* steps, int nsteps, int mode,
                         const float* freqs, int nfreqs, const char* combo);

#ifdef __cplusplus
}
#endif
#endif
