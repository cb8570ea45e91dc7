// tune.h -- the autotuned dispatch table.
//
// Every tuned GEMM family ("op") picks a kernel variant (tile shape and
// pipeline depth) and a split-K count from a table indexed by the size
// buckets of M, N and K.  The table is written by ferray_b200/autotune.py
// from timings on the target GPU and compiled in (tune_table.inc); a forced
// choice (fg_tune_force) overrides it for every shape while the tuner runs.
#pragma once
#include <cstdint>

namespace fgrt {

enum TuneOp : int {
    TUNE_I8 = 0,         // i8 x i8 / u8 x i8 -> i32, tcgen05 kind::i8
    TUNE_SPLIT_F32 = 1,  // 3xBF16 split SGEMM, tcgen05 kind::f16
    TUNE_F64 = 2,        // plain DGEMM, DFMA
    TUNE_F32 = 3,        // plain SGEMM, FFMA
    TUNE_OPS = 4
};

// Bucket b covers (2^(b+3), 2^(b+4)]: <=16, <=32, ..., <=4096, >4096.
constexpr int TUNE_BUCKETS = 10;
constexpr int TUNE_MAX_SPLITS = 16;

struct TuneChoice {
    int variant;
    int splits;
};

int tune_bucket(long long x);
int tune_variants(int op);
TuneChoice tune_lookup(int op, long long m, long long n, long long k);

// Split count actually used: at most `want`, at most one split per K block,
// no empty split, and a workspace (splits x out_elems x esize bytes) of at
// most 1 GiB.  Writes the K blocks per split.
int plan_splits(int want, int k_blocks, long long out_elems, long long esize, int* kb_per_split);

}  // namespace fgrt
