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
    int dim, order, prec, cells_class;   // cells_class = log2 of total cells
    bool operator<(const TuneKey& o) const {
        return std::tie(dim, order, prec, cells_class) < std::tie(o.dim, o.order, o.prec, o.cells_class);
    }
};
struct TuneVal {
    int ctas_per_sm, steps_per_sync;
};

// Process-wide cache of autotuning results keyed by (dim, order, precision, size class).
std::map<TuneKey, TuneVal>& tune_cache();

struct BatchCore {
    int dim = 0, order = 0, prec = 0;
    int device = 0;
    cudaStream_t st = nullptr;
    std::vector<std::unique_ptr<Shot>> shots;   // resident shots
    ShotDesc* d_descs = nullptr;
    int d_cap = 0;
    size_t d_bytes = 0;                // block size of d_descs (from the arena cache)
    Runner run;
    int ctas_per_sm = 0, steps_per_sync = 0;    // 0 = autotune
    bool tuned = false;
    long long cell_updates = 0;

    int init(int device_, cudaStream_t s);
    // Rebuilds the device descriptor table after shots were added or removed.
    int rebuild();
    // Advances every unfinished shot by up to n steps (asynchronous).
    int advance(int n);
    // Online autotuning: the first calls time real steps under candidate
    // (CTAs per SM, steps per sync) settings and keep the fastest.
    int autotune(int budget_steps);
    long long total_cells() const;
    void release();
};

}  // namespace bpk
