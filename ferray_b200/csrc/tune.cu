// tune.cu -- lookup in the compiled-in autotune table, forced choices and
// the C-ABI around them.
#include <algorithm>
#include <atomic>

#include "runtime.h"
#include "tune.h"

namespace fgrt {

namespace {

struct TuneEntry {
    uint8_t variant, splits;
};

// kTuneTable[op][bm][bn][bk]; generated by ferray_b200/autotune.py.
#include "tune_table.inc"

constexpr int kVariants[TUNE_OPS] = {4, 3, 6, 6};

std::atomic<int> g_force_variant[TUNE_OPS] = {{-1}, {-1}, {-1}, {-1}};
std::atomic<int> g_force_splits[TUNE_OPS] = {{1}, {1}, {1}, {1}};

}  // namespace

int tune_bucket(long long x) {
    int b = 0;
    long long lim = 16;
    while (b < TUNE_BUCKETS - 1 && x > lim) {
        ++b;
        lim *= 2;
    }
    return b;
}

int tune_variants(int op) { return (op >= 0 && op < TUNE_OPS) ? kVariants[op] : 0; }

TuneChoice tune_lookup(int op, long long m, long long n, long long k) {
    if (op < 0 || op >= TUNE_OPS) return {0, 1};
    const int fv = g_force_variant[op].load(std::memory_order_relaxed);
    if (fv >= 0) return {fv, g_force_splits[op].load(std::memory_order_relaxed)};
    const TuneEntry e = kTuneTable[op][tune_bucket(m)][tune_bucket(n)][tune_bucket(k)];
    TuneChoice c{e.variant, e.splits};
    if (c.variant >= kVariants[op]) c.variant = 0;
    if (c.splits < 1) c.splits = 1;
    return c;
}

int plan_splits(int want, int k_blocks, long long out_elems, long long esize, int* kb_per_split) {
    int s = std::max(1, std::min({want, k_blocks, TUNE_MAX_SPLITS}));
    while (s > 1 && static_cast<long long>(s) * out_elems * esize > (1LL << 30)) --s;
    int kps = (k_blocks + s - 1) / s;
    s = (k_blocks + kps - 1) / kps;  // no empty split
    *kb_per_split = kps;
    return s;
}

}  // namespace fgrt

using namespace fgrt;

extern "C" {

fg_status fg_tune_lookup(int op, size_t m, size_t n, size_t k, int* variant, int* splits) {
    if (op < 0 || op >= TUNE_OPS) return set_error(FG_ERR_INVALID, "fg_tune_lookup: unknown op");
    const TuneChoice c = tune_lookup(op, (long long)m, (long long)n, (long long)k);
    if (variant) *variant = c.variant;
    if (splits) *splits = c.splits;
    return FG_OK;
}

fg_status fg_tune_force(int op, int variant, int splits) {
    if (op < 0 || op >= TUNE_OPS) return set_error(FG_ERR_INVALID, "fg_tune_force: unknown op");
    if (variant >= kVariants[op]) return set_error(FG_ERR_INVALID, "fg_tune_force: no such variant");
    if (splits < 1 || splits > TUNE_MAX_SPLITS)
        return set_error(FG_ERR_INVALID, "fg_tune_force: splits outside 1..16");
    g_force_splits[op].store(splits);
    g_force_variant[op].store(variant < 0 ? -1 : variant);
    return FG_OK;
}

fg_status fg_tune_variants(int op, int* count) {
    if (op < 0 || op >= TUNE_OPS) return set_error(FG_ERR_INVALID, "fg_tune_variants: unknown op");
    if (count) *count = kVariants[op];
    return FG_OK;
}

}  // extern "C"
