// Host-side model of one postflop spot: cards, the 7-card evaluator, range
// parsing, the betting-tree builder and the Spot (hand lists, same-combo map,
// river strength tables, suit symmetries).  It restates the reference solver
// crate's semantics (crates/solver/src/{cards,evaluator,range,tree,game}.rs);
// node numbering, data offsets and river orderings are bit-exact with it.
// The tree is kept struct-of-arrays because the device plan is built from it.
#pragma once
#include <array>
#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "json.hpp"

namespace gtob {

constexpr uint32_t kSentinel = 0xFFFFFFFFu;
enum NodeKind : uint8_t { kAction = 0, kChance = 1, kFold = 2, kShowdown = 3 };
enum ActKind : uint8_t { kFoldA = 0, kCheck = 1, kCall = 2, kBet = 3, kRaise = 4 };
enum SizeKind : uint8_t { kPotPct = 0, kPrevMult = 1, kAllIn = 2 };

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

// --- cards (cards.rs) ---------------------------------------------------
inline int card_rank(uint8_t c) { return c >> 2; }
inline int card_suit(uint8_t c) { return c & 3; }
inline uint8_t card_make(int r, int s) { return (uint8_t)(r * 4 + s); }
inline uint8_t card_permute(uint8_t c, const std::array<uint8_t, 4>& pm) { return card_make(card_rank(c), pm[card_suit(c)]); }
inline int combo_id(uint8_t a, uint8_t b) {
    int h = a > b ? a : b, l = a > b ? b : a;
    return (h * (h - 1)) / 2 + l;
}
void combo_cards(int id, uint8_t* hi, uint8_t* lo);
uint8_t parse_card(const std::string& s);
std::vector<uint8_t> parse_board(const std::string& s);
std::string card_name(uint8_t c);

// --- evaluator (evaluator.rs) -------------------------------------------
uint32_t eval7(const uint8_t* cards);

// --- range (range.rs) ---------------------------------------------------
std::vector<float> parse_range_weights(const std::string& text);

// --- config (game.rs:22-27, tree.rs:14-95) --------------------------------
struct BetSize { uint8_t kind; double v; };
struct StreetSizing { std::vector<BetSize> bet, raise, donk; };
struct TreeConfig {
    double starting_pot = 60, effective_stack = 970, rake_pct = 0, rake_cap = 0, allin_threshold = 0.85;
    bool add_allin = false;
    int max_raises = 10;
    StreetSizing oop[3], ip[3];
    const StreetSizing& side(int player, int street) const { return player == 0 ? oop[street] : ip[street]; }
};
struct SpotConfig {
    std::string board, range_oop, range_ip;
    TreeConfig tree;
};
SpotConfig config_from_json(const json::Value& v);
json::Value config_to_json(const SpotConfig& c);

// --- tree (tree.rs), struct of arrays -----------------------------------
struct Tree {
    int root_street = 0;
    std::vector<uint8_t> kind, player, street, nchild;
    std::vector<uint32_t> child_start, action_start;
    std::vector<uint64_t> data_off;
    std::vector<double> put0, put1, twin, tlose, ttie;
    std::vector<uint32_t> children;
    std::vector<uint8_t> act_kind;
    std::vector<double> act_amount;
    uint64_t data_size[2] = {0, 0};
    size_t size() const { return kind.size(); }
    uint32_t child(uint32_t n, int a) const { return children[child_start[n] + a]; }
};
Tree build_tree(const TreeConfig& cfg, const std::vector<uint8_t>& board, uint64_t nh0, uint64_t nh1,
                uint64_t max_nodes, bool lenient);

// --- spot (game.rs) -----------------------------------------------------
struct Hands {
    std::vector<uint8_t> c1, c2;  // c1 = higher card index
    std::vector<float> w;
    std::vector<uint64_t> mask;
    size_t size() const { return c1.size(); }
};
// One completed 5-card board: each player's surviving hands sorted ascending
// by (strength, hand index), game.rs:29-34.
struct RiverBoard {
    std::vector<uint32_t> str[2];
    std::vector<uint16_t> idx[2];
};
struct Spot {
    SpotConfig config;
    std::vector<uint8_t> board;
    uint64_t board_mask = 0;
    Tree tree;
    Hands hands[2];
    std::vector<uint32_t> same[2];
    std::vector<std::unique_ptr<RiverBoard>> river;  // indexed by river_key
    std::vector<std::array<uint8_t, 4>> perms;        // entry 0 = identity
    std::vector<std::vector<uint16_t>> hand_perm[2];  // [k][i]
    size_t river_key(const uint8_t* dealt, int n) const;
    const RiverBoard& river_at(const uint8_t* dealt, int n) const;
    std::vector<int> perms_fixing(const uint8_t* dealt, int n) const;
    size_t num_action_nodes() const;
    double pair_weight_sum() const;
};
std::unique_ptr<Spot> build_spot(const SpotConfig& cfg, uint64_t max_nodes, bool lenient);

}  // namespace gtob
