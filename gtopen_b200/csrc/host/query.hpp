// Node queries over the device arenas (query.rs:304-645 node_view's
// numbers): the reach of both players at the node a path reaches, each
// player's compatible opponent mass and EV, and at an action node the
// actor's average strategy and per-action EVs -- without syncing the arenas
// to the host.  The strategies along the path come from the device blocks,
// the values from one average-strategy evaluation sweep per player.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "solver.hpp"

namespace gtob {

class GpuEngine;

struct NodeValues {
    uint32_t node = 0;  // tree index of the node the path reaches
    int kind = 0, player = -1, na = 0;
    std::vector<float> reach[2];  // walk reach (query.rs:304-340)
    std::vector<float> valid[2];  // compatible opponent reach mass (query.rs:463-488)
    std::vector<float> eq[2];     // equity over the remaining runouts (best_response.rs:292-386), NaN if none
    std::vector<float> ev[2];     // pot-share EV, NaN where valid <= 1e-9
    std::vector<float> strategy;  // the actor's average strategy, [action * nh + hand]
    std::vector<float> action_ev;  // the actor's EV per action, same layout, NaN where valid <= 1e-9
};

// exploit_view's numbers (query.rs:808-930) for exploiter p, per hand of the
// browsed branch: reach and compatible mass on the representative branch,
// best-response and current EVs and their difference (NaN where valid <=
// 1e-9); where p acts, the best response (one-hot, ties within 1e-5 split;
// the lock at a locked node) and the EV of each action under it; the
// reach x valid weighted averages of br_ev, cur_ev and gain.
struct ExploitValues {
    uint32_t node = 0;  // the representative node the values are read at
    int kind = 0, player = -1, na = 0;
    std::vector<float> reach, valid, br_ev, cur_ev, gain;
    std::vector<float> br_strategy, action_ev;  // [action * nh + hand]
    float avg[3];
};
ExploitValues exploit_values(GpuEngine& eng, const HostSolver& host, const std::vector<int>& steps, int p);

// runouts (query.rs:964-1106) at a chance node: per available card,
// descending, the action frequencies at the following action node, and per
// player the reach x valid weighted equity and average-strategy EV.
struct RunoutRow {
    int card = 0;
    std::vector<float> freqs;
    float eq[2], ev[2];  // NaN when no mass
};
struct Runouts {
    int player = -1, na = 0;  // actor and action count at the runout nodes (-1, 0: none)
    double pot = 0.0;
    std::vector<RunoutRow> rows;
};
Runouts runouts(GpuEngine& eng, const HostSolver& host, const std::vector<int>& steps);

// Equity of each of p's hands against the opponent reach, enumerating the
// remaining runouts of the board plus `dealt` (best_response.rs:292-386,
// game.rs:580-653 sweep_buckets); NaN where no compatible mass.
std::vector<float> equity(const Spot& sp, int p, const float* reach_o, const uint8_t* dealt, int nd);

// node_view's structure at the node a path reaches, without the per-hand
// numbers (query.rs:353-461, 490-640): node type, street, board (the spot's
// cards and the dealt ones), pot and puts, actor, the action views (label,
// kind, amount; tree.rs:139-169 labels), the cards a chance node can deal,
// whether the node -- on its orbit representative -- is locked, and the
// history bar (one step per node along the path, then the current node).  A
// JSON object with the reference's field names; Option fields are null.
std::string path_view_json(const HostSolver& host, const std::vector<int>& steps);

// steps: action indices (>= 0) and dealt cards (-1 - card), from the root.
// Through a suit-isomorphic branch the device holds the representative: its
// values are read under the hand permutation that ensure_symmetric applies.
NodeValues node_values(GpuEngine& eng, const HostSolver& host, const std::vector<int>& steps);

}  // namespace gtob
