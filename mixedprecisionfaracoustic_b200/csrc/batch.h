// batch.h - a set of resident shots advanced together: one launch per phase
// covers the tiles of every shot (tile table = per-shot prefix offsets).
#pragma once
#include <map>
#include <memory>
#include <tuple>
#include <vector>

#include "runner.h"

namespace bpk {

struct TuneKey {
    int dim, order, prec, cells_class, shots_class;   // log2 of the total cells and of the shot count
    bool operator<(const TuneKey& o) const {
        return std::tie(dim, order, prec, cells_class, shots_class) <
               std::tie(o.dim, o.order, o.prec, o.cells_class, o.shots_class);
    }
};
struct TuneVal {
    int ctas_per_sm, steps_per_sync;
    TileShape shape;
    int kernel;
};

// Process-wide cache of autotuning results keyed by (dim, order, precision
// and rounding, grid class: log2 of the batch's cells and of its shot count).
std::map<TuneKey, TuneVal>& tune_cache();

struct BatchCore {
    int dim = 0, order = 0, prec = 0;
    int rounding = BP_ROUND_FAST;
    int device = 0;
    cudaStream_t st = nullptr;
    std::vector<std::unique_ptr<Shot>> shots;   // resident shots
    ShotDesc* d_descs = nullptr;
    int d_cap = 0;
    size_t d_bytes = 0;                // block size of d_descs (from the arena cache)
    Runner run;
    int ctas_per_sm = 0, steps_per_sync = 0;    // 0 = autotune
    TileShape shape{0, 0, 0};                   // rows 0 = autotune (default shape until tuned)
    int kernel = BP_KERNEL_AUTO;                // family; AUTO = autotune (library default until tuned)
    bool tuned = false;
    long long cell_updates = 0;

    int init(int device_, cudaStream_t s);
    // Rebuilds the device descriptor table after shots were added or removed.
    int rebuild();
    // Advances every unfinished shot by up to n steps (asynchronous).
    int advance(int n);
    // Online autotuning: times real steps under candidate tile shapes, then
    // CTAs per SM, then steps per sync (each stage keeps the fastest so far)
    // within budget_steps steps, and caches the winner per grid class.
    int autotune(int budget_steps);
    TileShape effective_shape() const;
    long long total_cells() const;
    void release();
};

}  // namespace bpk
