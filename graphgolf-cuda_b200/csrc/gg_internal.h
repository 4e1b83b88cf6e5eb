// gg_internal.h -- declarations shared by the library's translation units (not
// part of the C ABI; hidden symbols).
#pragma once
#include <cstdint>
#include <string>
#include <vector>
#include <cuda_runtime.h>

#include "gg.h"

namespace gg {

// Options of an evaluation that only the library's own modules use.
struct EvalExtra {
    const int32_t *inv = nullptr;  // device [rows]: source index of each vertex (-1: none)
    int ns = 0;                    // sources in that list
    uint4 *planes = nullptr;       // distance bit-planes to write (every source, in order)
    int nplanes = 0;
    bool no_graph = false;         // launch directly, neither capture nor replay
};

__attribute__((visibility("hidden"))) void set_last_error(const char *msg);

// Autotuner cache (gg_tune.cpp): key = GPU name and SM count, evaluator, shape.
__attribute__((visibility("hidden"))) std::string tune_key(int device, const char *what,
                                                         const std::vector<long long> &dims);
__attribute__((visibility("hidden"))) bool tune_get(const std::string &key, std::vector<int> *vals);
__attribute__((visibility("hidden"))) void tune_put(const std::string &key, const std::vector<int> &vals);

// One evaluation of `e` on the device table `d_table` (on stream `st`, blocking),
// with the extra options `x` (nullptr: none).
__attribute__((visibility("hidden"))) gg_status engine_eval(gg_engine *e, const int32_t *d_table,
                                                          const gg_eval_opts *o, gg_result *r,
                                                          cudaStream_t st, const EvalExtra *x);

// Columns (chunks of 128 sources) of the distance planes an evaluation of every
// source writes, and the engine's rows.
__attribute__((visibility("hidden"))) int engine_plane_cols(const gg_engine *e);

}  // namespace gg
