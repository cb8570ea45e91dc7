// shard.cu -- communication-free partition of independent GEMM work across
// GPUs (one process per GPU): fg_shard_plan and fg_gemm_grouped_shard.
//
// ferray parallelises a stacked matmul only inside one process, splitting the
// batch over its rayon pool (products/mod.rs:625-638).  The B200 analogue is
// one process per GPU, each running a shard of the problems of a ragged batch
// or of the requests of a served stream.  Every rank computes the same
// assignment from the same list, so no rank has to tell another what it
// runs and no collective sits on the data path.
//
// Policies:
//   FG_SHARD_LPT     whole batch known up front: units sorted by cost,
//                    heaviest first (ties by index), each to the rank with the
//                    least cost so far (ties to the lower rank).  Shards are
//                    disjoint, cover every unit, and their costs differ by at
//                    most one unit's cost.
//   FG_SHARD_ONLINE  a stream: units taken in arrival order, each to the
//                    least-loaded rank so far (ties to the lower rank), so a
//                    rank can route request i as soon as it arrives.
// Cost of a unit: weight[i] when weights are given, else 2 m n k.
#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "runtime.h"

using namespace fgrt;

namespace {

fg_status plan(const int64_t* dims, const double* weight, size_t count, int world, int rank, int policy,
               std::vector<int64_t>& mine) {
    if (world < 1 || rank < 0 || rank >= world)
        return set_error(FG_ERR_INVALID, "shard: rank " + std::to_string(rank) + " outside a world of " +
                                             std::to_string(world));
    if (policy != FG_SHARD_LPT && policy != FG_SHARD_ONLINE)
        return set_error(FG_ERR_INVALID, "shard: unknown policy");
    if (count && !dims && !weight) return set_error(FG_ERR_INVALID, "shard: null dims and weights");
    std::vector<double> cost(count);
    for (size_t i = 0; i < count; ++i) {
        if (weight) {
            cost[i] = weight[i];
        } else {
            const int64_t m = dims[3 * i], n = dims[3 * i + 1], k = dims[3 * i + 2];
            if (m < 0 || n < 0 || k < 0) return set_error(FG_ERR_SHAPE, "shard: negative dimension");
            cost[i] = 2.0 * static_cast<double>(m) * static_cast<double>(n) * static_cast<double>(k);
        }
    }
    std::vector<size_t> order(count);
    std::iota(order.begin(), order.end(), size_t(0));
    if (policy == FG_SHARD_LPT)
        std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return cost[x] > cost[y]; });
    std::vector<double> load(world, 0.0);
    mine.clear();
    for (size_t i : order) {
        int r = 0;
        for (int q = 1; q < world; ++q)
            if (load[q] < load[r]) r = q;
        load[r] += cost[i];
        if (r == rank) mine.push_back(static_cast<int64_t>(i));
    }
    std::sort(mine.begin(), mine.end());
    return FG_OK;
}

}  // namespace

extern "C" {

fg_status fg_shard_plan(const int64_t* dims, const double* weight, size_t count, int world, int rank,
                        int policy, int64_t* out, size_t* out_count) {
    if (!out_count || (count && !out)) return set_error(FG_ERR_INVALID, "shard: null output");
    std::vector<int64_t> mine;
    FG_TRY(plan(dims, weight, count, world, rank, policy, mine));
    std::copy(mine.begin(), mine.end(), out);
    *out_count = mine.size();
    return FG_OK;
}

fg_status fg_gemm_grouped_shard(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const fg_problem* table,
                                size_t count, int world, int rank, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    if (count && !table) return set_error(FG_ERR_INVALID, "null problem table");
    std::vector<int64_t> dims(3 * count);
    for (size_t i = 0; i < count; ++i) {
        dims[3 * i] = table[i].m;
        dims[3 * i + 1] = table[i].n;
        dims[3 * i + 2] = table[i].k;
    }
    std::vector<int64_t> mine;
    FG_TRY(plan(dims.data(), nullptr, count, world, rank, FG_SHARD_LPT, mine));
    if (mine.empty()) return FG_OK;
    std::vector<fg_problem> sub(mine.size());
    for (size_t i = 0; i < mine.size(); ++i) sub[i] = table[mine[i]];
    return fg_gemm_grouped(ctx, dtype, mode, sub.data(), sub.size(), stream);
}

}  // extern "C"
