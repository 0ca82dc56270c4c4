// Host build of the batched solver's table construction (batch_tables in
// csrc/fold3d_internal.h, the function the restage kernel runs on the device)
// for tests/test_batch_tables.py.  Test code only.
#include "fold3d_internal.h"

using namespace fold3d;

// order/steps/tiles: n entries (a direction's order); outputs sized n, n + 1,
// max_steps and max_steps + 1; returns the item count.
extern "C" unsigned host_batch_tables(const int *order, const int *steps, const long long *tiles, const int *active,
                                      int n, int max_steps, int *act, long long *tile_pre, int *step_k,
                                      long long *step_off)
{
    BatchDirTables t;
    t.order = order;
    t.steps = steps;
    t.tiles = tiles;
    t.act = act;
    t.tile_pre = tile_pre;
    t.step_k = step_k;
    t.step_off = step_off;
    return batch_tables(t, active, n, max_steps);
}
