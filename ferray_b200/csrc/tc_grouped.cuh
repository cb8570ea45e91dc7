// tc_grouped.cuh -- persistent grouped (ragged-batch) GEMM on tcgen05.
//
// One launch runs `count` independent problems of different M, N, K.  A
// device-side problem table holds, per problem, its shape, its tile range in
// a global tile numbering (prefix sums), its output, its operand pointers
// and the TMA descriptors of the operands TMA can read (written to global
// memory before the launch).  Tiles are numbered deepest problem first.  A
// device-side tile scheduler hands them out: each CTA's producer claims the
// next global tile with an atomic add on a counter (zeroed before every
// launch), so CTAs that drew short tiles come back for more and the heavy
// tiles go first (dynamic longest-processing-time order).  The producer
// passes each claimed tile to the MMA issuer and the four epilogue warps
// (as in tc_gemm.cuh) through a small ring of shared-memory slots guarded by
// mbarriers.  i8 operands TMA cannot read (rows that break its 16-byte
// rule) are staged by the producer warp's lanes (granule copies into raw
// slots) and two shift warps (shifted, swizzled shared stores), so they
// make no extra pass through HBM.  The split form's f32 operands are cut
// into bf16 hi/lo planes by split_prep_kernel (one pass; the planes are then
// read by TMA).  The producer claims tiles ahead of use.
#pragma once
#include "tc_gemm.cuh"

namespace fg {

struct GroupedProblem {
    int M, N, K;
    int k_blocks, tiles_m, tiles_n;
    long long tile_start;  // first global tile of this problem
    void* C;
    long long ldc;         // elements
    int tile;              // plain FP32 batches: square tile edge, 64 or 32
    const void* A;         // row-major M x K, leading dimension lda (elements)
    const void* B;         // row-major K x N, leading dimension ldb (elements)
    long long lda, ldb;
};

// Per global tile: problem index, tile row, tile column and the problem's K
// blocks, plus the operand fields the producer needs to stage the tile
// (written by the host with the problem table, so a tile costs one 64-byte
// record instead of a search and a second, dependent load).  The top bits
// of `kb` say which operands are staged (TILE_GEN_A, TILE_GEN_B); the rest
// is the K block count.  The MMA issuer and the epilogue get the first 16
// bytes through the tile ring.
struct alignas(16) TileRec {
    int problem, tm, tn, kb;
    const void* A;
    const void* B;
    long long lda, ldb;  // elements
    int M, N, K, pad;
};
static_assert(sizeof(TileRec) == 64, "tile records are copied as four 16-byte granules");
constexpr int TILE_GEN_SHIFT = 28;
constexpr int TILE_GEN_A = 1, TILE_GEN_B = 2;
constexpr int TILE_KB_MASK = (1 << TILE_GEN_SHIFT) - 1;

struct GroupedArgs {
    const GroupedProblem* problems;
    const TileRec* tiles;     // [total_tiles]
    unsigned long long* tile_counter;  // next unclaimed tile (zeroed before the launch)
    const CUtensorMap* maps;  // per problem: NA A maps then NB B maps
    int count;
    long long total_tiles;
    float alpha, beta;        // EPI_F32
    int accumulate;           // EPI_I32
    int kchunk;
    TcOp ops[TC_MAX_OPS];
    DevStatus* status;
    unsigned long long timeout_ns;
};

// ------------------------------------------------------------ loader warps
// i8 operands TMA cannot read are staged in "units" (the 128 rows of an
// operand tile).  The producer warp's lanes copy a unit's rows, as the
// aligned 16-byte granules that hold them, into a raw slot of shared memory
// with cp.async (a row per lane at a time, several units in flight, no
// registers held); the slot's raw_full barrier counts the copies'
// completion.  Two shift warps then move each row out of its raw granules
// into the stage buffer in TMA's 128-byte swizzle.  Units go through a ring
// of NRAW raw slots in stage order.  Granules are copied only when they
// hold a byte of the row, so every read stays on memory the row occupies.
// (Staging f32 rows for the split form in the same way was measured slower
// than a separate split pass: cutting every value into two bf16 halves in
// two warps costs more than the pass's one round trip through HBM.)
constexpr int GROUPED_LOADER_WARPS = 2;  // the shift warps (6 and 7)
constexpr int GROUPED_LOADER_THREADS = 32 * GROUPED_LOADER_WARPS;

// Each lane takes whole rows (row lane, lane + 32, ...), so a row's
// alignment offset is worked out once and its bytes are moved with selects
// and byte permutes, not per-chunk shifts.
template <class Cfg>
struct LoaderCfg {
    static constexpr bool STAGED = Cfg::KIND == KIND_I8;  // only the i8 kernel stages operands
    static constexpr int UNIT_ROWS = 128;              // a whole 128-row operand tile
    static constexpr int RPT = UNIT_ROWS / 32;         // rows per lane of the copying warp
    static constexpr int ROW_BYTES = 128;              // source bytes of a unit row
    static constexpr int GRAN = ROW_BYTES / 16 + 1;    // aligned granules that can hold them
    static constexpr int RAW_BYTES = STAGED ? UNIT_ROWS * GRAN * 16 : 0;
    static constexpr int NRAW = STAGED ? 6 : 1;        // raw slots
    static constexpr int FULL_ARRIVALS = STAGED ? 3 : 1;  // producer (+ both shift warps)
    static constexpr int THREADS = Cfg::THREADS + (STAGED ? 32 * GROUPED_LOADER_WARPS : 0);
};

// Raw-slot entry: one unit, a marker for a stage TMA loads entirely (the
// shift warps still arrive on it), or the end of the walk.
struct LoaderUnit {
    const uint8_t* src;  // first byte of the unit's first source row
    long long ld;        // source row pitch, bytes
    int nrows;           // source rows present (rows past it become 0)
    int valid;           // bytes of each row present (> 0)
    uint32_t dst0;       // shared address of the unit's first destination row
    int flags;           // LU_FIRST / LU_LAST of its stage, LU_MARKER: no data
    int stage;
    uint32_t par;        // the stage's phase parity
};
// LU_ZERO: rows past nrows are stored as zeros (otherwise they keep
// whatever is there).  LU_PROD: the stage has no TMA part, so the producer
// neither waits for it nor arrives on it; shift warp 6's arrival after the
// stage's last entry counts for the producer too.
constexpr int LU_FIRST = 1, LU_LAST = 2, LU_MARKER = 4, LU_END = 8, LU_ZERO = 16, LU_PROD = 32;

template <class Cfg>
constexpr size_t grouped_raw_offset() {
    return (sizeof(TcSmem<Cfg>) + 127) / 128 * 128;
}
template <class Cfg>
constexpr size_t grouped_smem_bytes() {
    return grouped_raw_offset<Cfg>() + static_cast<size_t>(LoaderCfg<Cfg>::NRAW) * LoaderCfg<Cfg>::RAW_BYTES + 1024;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, uintptr_t src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(dst), "l"(src) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ uint4 lds128(uint32_t addr) {
    uint4 v;
    asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "r"(addr));
    return v;
}
__device__ __forceinline__ void sts128(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
    asm volatile("st.shared.v4.u32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d)
                 : "memory");
}

// Copies of one unit: granule j of row r goes to raw + (r * GRAN + j) * 16,
// and only granules holding a byte of the row are read.
template <class LC>
__device__ __forceinline__ void loader_issue(const uint8_t* src, long long ld, int nrows, int valid,
                                             uint32_t raw, int lt) {
#pragma unroll
    for (int i = 0; i < LC::RPT; ++i) {
        const int r = lt + 32 * i;
        if (r >= nrows) continue;
        const uintptr_t a = reinterpret_cast<uintptr_t>(src + static_cast<long long>(r) * ld);
        const uintptr_t gbase = a & ~static_cast<uintptr_t>(15);
        const int end = static_cast<int>(a - gbase) + valid;  // granule j is needed when 16 j < end
        const uint32_t dst = raw + r * LC::GRAN * 16;
#pragma unroll
        for (int j = 0; j < LC::GRAN; ++j)
            if (16 * j < end) cp_async16(dst + 16 * j, gbase + 16 * j);
    }
}

// One row of an i8 unit: the row's 128 bytes start `sh` bytes into its first
// raw granule; its 36 raw words are rotated by sh / 4 words with two levels
// of selects (no divergent branch) and by sh % 4 bytes with byte permutes,
// then stored as 8 chunks at chunk c ^ (r & 7) of destination row r
// (128-byte swizzle).
template <class LC>
__device__ __forceinline__ void shift_row_u8(const LoaderUnit& u, uint32_t raw, int r) {
    const uint32_t d = u.dst0 + r * 128;
    const uint32_t sh = static_cast<uint32_t>(reinterpret_cast<uintptr_t>(u.src + static_cast<long long>(r) * u.ld) & 15);
    const uint32_t rr = raw + r * LC::GRAN * 16;
    uint32_t w[36];
#pragma unroll
    for (int g = 0; g < 9; ++g) {
        const uint4 v = lds128(rr + 16 * g);
        w[4 * g] = v.x;
        w[4 * g + 1] = v.y;
        w[4 * g + 2] = v.z;
        w[4 * g + 3] = v.w;
    }
#pragma unroll
    for (int k = 0; k < 35; ++k) w[k] = (sh & 4u) ? w[k + 1] : w[k];
#pragma unroll
    for (int k = 0; k < 33; ++k) w[k] = (sh & 8u) ? w[k + 2] : w[k];
    const uint32_t sel = 0x3210u + 0x1111u * (sh & 3u);
#pragma unroll
    for (int c = 0; c < 8; ++c)
        sts128(d + ((c ^ (r & 7)) << 4), __byte_perm(w[4 * c], w[4 * c + 1], sel),
               __byte_perm(w[4 * c + 1], w[4 * c + 2], sel), __byte_perm(w[4 * c + 2], w[4 * c + 3], sel),
               __byte_perm(w[4 * c + 3], w[4 * c + 4], sel));
}

// A shift warp's rows of an i8 unit: the 32-row blocks 2i + half (rows
// 32 (2i + half) + lane), so units shorter than 128 rows still split evenly
// between the two shift warps.  Rows past nrows are zero-filled for LU_ZERO
// units and skipped otherwise.
template <class LC>
__device__ __forceinline__ void shift_rows_u8(const LoaderUnit& u, uint32_t raw, int half, int lane) {
#pragma unroll
    for (int i = 0; i < LC::UNIT_ROWS / 64; ++i) {
        const int r = 32 * (2 * i + half) + lane;
        if (r < u.nrows) {
            shift_row_u8<LC>(u, raw, r);
        } else if (u.flags & LU_ZERO) {
            const uint32_t d = u.dst0 + r * 128;
#pragma unroll
            for (int c = 0; c < 8; ++c) sts128(d + (c << 4), 0u, 0u, 0u, 0u);
        }
    }
}

// Stores one warp's 32 rows x 32 columns: lane l holds row row0 + l.  The
// block goes through a padded shared-memory tile so that the global stores
// (and the reads of C for accumulate / beta) are 128-byte row segments.
template <class Cfg>
__device__ __forceinline__ void grouped_store(const GroupedArgs& g, const GroupedProblem& pr, int row0,
                                              int col0, const uint32_t (&v)[32], uint32_t (*stg)[33],
                                              int lane) {
#pragma unroll
    for (int j = 0; j < 32; ++j) stg[lane][j] = v[j];
    __syncwarp();
    const int col = col0 + lane;
    const int rows = min(32, pr.M - row0);
    if (col < pr.N) {
        // unrolled with predicates: all shared-memory reads (and the reads
        // of C for accumulate / beta) are issued before the first store, so
        // they overlap instead of costing one round trip per row
        uint32_t w[32];
#pragma unroll
        for (int r = 0; r < 32; ++r) w[r] = stg[r][lane];
        const long long ldc = pr.ldc;
        if constexpr (Cfg::EPI == EPI_I32) {
            int32_t* p = static_cast<int32_t*>(pr.C) + (long long)row0 * ldc + col;
            if (g.accumulate) {
#pragma unroll
                for (int r = 0; r < 32; ++r)
                    if (r < rows) w[r] += static_cast<uint32_t>(p[r * ldc]);
            }
#pragma unroll
            for (int r = 0; r < 32; ++r)
                if (r < rows) p[r * ldc] = static_cast<int32_t>(w[r]);
        } else {
            float* p = static_cast<float*>(pr.C) + (long long)row0 * ldc + col;
            float o[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) o[r] = g.alpha * __uint_as_float(w[r]);
            if (g.beta != 0.f) {
#pragma unroll
                for (int r = 0; r < 32; ++r)
                    if (r < rows) o[r] = fmaf(g.beta, p[r * ldc], o[r]);
            }
#pragma unroll
            for (int r = 0; r < 32; ++r)
                if (r < rows) p[r * ldc] = o[r];
        }
    }
    __syncwarp();
}

template <class Cfg>
__global__ void __launch_bounds__(LoaderCfg<Cfg>::THREADS, 1)
    tc_grouped_kernel(const __grid_constant__ GroupedArgs g) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* base = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    TcSmem<Cfg>& s = *reinterpret_cast<TcSmem<Cfg>*>(base);
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    volatile int* abort = &s.abort;
    constexpr int NMAPS = Cfg::NA + Cfg::NB;
    // tile-scheduler ring: the producer writes claimed tile records, the MMA
    // thread, the four epilogue warps and the loader warps read them in order
    constexpr int SLOTS = 16;
    __shared__ uint64_t sched_full[SLOTS], sched_empty[SLOTS];
    __shared__ int4 sched_rec[SLOTS];  // the tile's TileRec; problem < 0 ends the walk
    // staged operands: raw slot barriers (raw_full[0..NRAW), raw_empty
    // after them) and the unit records of the slots
    __shared__ uint64_t raw_full[2 * LoaderCfg<Cfg>::NRAW];
    __shared__ LoaderUnit lu[LoaderCfg<Cfg>::NRAW];

    if (threadIdx.x == 0) {
        for (int i = 0; i < SLOTS; ++i) {
            mbar_init(&sched_full[i], 1);
            mbar_init(&sched_empty[i], 5);  // MMA thread, four epilogue warps
        }
        for (int i = 0; i < Cfg::STAGES; ++i) {
            // the producer (with the TMA bytes) and, when staging, the two
            // shift warps
            mbar_init(&s.full[i], LoaderCfg<Cfg>::FULL_ARRIVALS);
            mbar_init(&s.empty[i], 1);
        }
        for (int i = 0; i < 4; ++i) {
            mbar_init(&s.acc_full[i], 1);
            mbar_init(&s.acc_empty[i], 4);
        }
        mbar_init(&s.drain, 1);
        for (int i = 0; i < LoaderCfg<Cfg>::NRAW; ++i) {
            mbar_init(&raw_full[i], 33);  // 32 copy completions (noinc) + the record's arrival
            mbar_init(&raw_full[LoaderCfg<Cfg>::NRAW + i], 2);  // raw_empty: both shift warps
        }
        s.abort = 0;
        fence_mbar_init();
    }
    if (warp == 1) {
        tmem_alloc(&s.tmem_base, Cfg::TMEM_COLS);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = s.tmem_base;

    using LC = LoaderCfg<Cfg>;
    const uint32_t raw0 = smem_u32(base + grouped_raw_offset<Cfg>());
    // a wait done by lane 0 whose outcome the whole warp takes
    auto wait0 = [&](uint64_t* bar, uint32_t par, int where) -> bool {
        int r = 1;
        if (lane == 0) r = mbar_wait(bar, par, g.timeout_ns, g.status, where, abort) ? 1 : 0;
        r = __shfl_sync(0xffffffffu, r, 0);
        __syncwarp();
        return r != 0;
    };

    if (warp == 0) {
        // Producer warp.  Lane 0 claims tiles, publishes them to the ring,
        // issues the TMA loads and arrives on the stage barriers; for the i8
        // kernel all 32 lanes also issue the granule copies of the units the
        // shift warps fill (a copy needs only a free raw slot, so the copies
        // of a stage go out before the stage itself is free).
        int stage = 0;
        uint32_t phase = 0;
        // lane 0, per stage: a TMA load was issued (bit) and its phase parity
        uint32_t issued_mask = 0, issued_par = 0;
        bool ok = true;
        int slot = 0;
        uint32_t sph = 0;
        int rs = 0;
        uint32_t rph = 0;
        // one unit record into the next raw slot, with its copies
        auto put = [&](const LoaderUnit& u) -> bool {
            if (!wait0(&raw_full[LC::NRAW + rs], rph ^ 1u, 0x66)) return false;  // raw_empty[rs]
            if (!(u.flags & (LU_MARKER | LU_END)))
                loader_issue<LC>(u.src, u.ld, u.nrows, u.valid, raw0 + rs * LC::RAW_BYTES, lane);
            if (lane == 0) lu[rs] = u;
            __syncwarp();
            // raw_full completes when every lane's copies have landed and
            // lane 0 has published the record
            asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(&raw_full[rs]))
                         : "memory");
            if (lane == 0) mbar_arrive(&raw_full[rs]);
            if (++rs == LC::NRAW) {
                rs = 0;
                rph ^= 1u;
            }
            return true;
        };
        // Claims run ahead of use: tiles are claimed TB at a time (one atomic
        // add on the tile counter) two batches ahead, and each batch's
        // records are copied into a ring of three batch slots in shared
        // memory (cp.async, lanes 0-15) while the batches before it are
        // loaded, so no global round trip sits between two tiles' loads.
        constexpr int TB = 4;
        __shared__ TileRec trec[3 * TB];
        const long long total = g.total_tiles;
        auto load_batch = [&](long long b, int sl) {
            if (lane < 4 * TB) {
                const long long t = b + (lane >> 2);
                if (t < total)
                    cp_async16(smem_u32(&trec[sl * TB + (lane >> 2)]) + 16 * (lane & 3),
                               reinterpret_cast<uintptr_t>(g.tiles + t) + 16 * (lane & 3));
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
        };
        long long b_cur = 0, b_nxt = 0, b_claim = 0;
        if (lane == 0) {
            b_cur = static_cast<long long>(atomicAdd(g.tile_counter, static_cast<unsigned long long>(TB)));
            b_nxt = static_cast<long long>(atomicAdd(g.tile_counter, static_cast<unsigned long long>(TB)));
            b_claim = static_cast<long long>(atomicAdd(g.tile_counter, static_cast<unsigned long long>(TB)));
        }
        b_cur = __shfl_sync(0xffffffffu, b_cur, 0);
        b_nxt = __shfl_sync(0xffffffffu, b_nxt, 0);
        load_batch(b_cur, 0);
        load_batch(b_nxt, 1);
        int sl_cur = 0, bi = 0;
        long long b_nn = 0;
        while (ok) {
            if (bi == 0) {
                // this batch's records have landed (the next batch's may not
                // have); start the batch after next and claim the one after it
                cp_async_wait<1>();
                __syncwarp();
                b_nn = __shfl_sync(0xffffffffu, b_claim, 0);
                if (lane == 0 && b_nn < total)
                    b_claim = static_cast<long long>(atomicAdd(g.tile_counter, static_cast<unsigned long long>(TB)));
                load_batch(b_nn, sl_cur == 0 ? 2 : sl_cur - 1);
            }
            const bool have = b_cur + bi < total;
            TileRec r0 = have ? trec[sl_cur * TB + bi] : TileRec{};
            if (!have) r0.problem = -1;
            // publish the tile (or the end marker) to the MMA and epilogue roles
            int okp = 1;
            if (lane == 0) {
                if (mbar_wait(&sched_empty[slot], sph ^ 1u, g.timeout_ns, g.status, 0x35, abort)) {
                    sched_rec[slot] = make_int4(r0.problem, r0.tm, r0.tn, r0.kb);
                    mbar_arrive(&sched_full[slot]);
                } else {
                    okp = 0;
                }
            }
            if (!__shfl_sync(0xffffffffu, okp, 0)) {
                ok = false;
                break;
            }
            if (++slot == SLOTS) {
                slot = 0;
                sph ^= 1u;
            }
            if (r0.problem < 0) break;
            const int pi = r0.problem, tm = r0.tm, tn = r0.tn;
            const int kbn = r0.kb & TILE_KB_MASK, gen = r0.kb >> TILE_GEN_SHIFT;
            // TMA bytes per stage: the operands the shift warps do not fill
            const uint32_t tx = ((gen & TILE_GEN_A) ? 0u : static_cast<uint32_t>(Cfg::NA * Cfg::A_TILE)) +
                                ((gen & TILE_GEN_B) ? 0u : static_cast<uint32_t>(Cfg::NB * Cfg::B_TILE));
            const CUtensorMap* mp = g.maps + (long long)pi * NMAPS;
            // A unit's source window: x = 0 is A (128 rows of the tile), x = 1
            // is B (128 K rows).  A rows past M and B columns past N only
            // reach outputs that are not stored, so they are left as they
            // are; K rows of B past K are stored as zeros (LU_ZERO), so the
            // unmasked K tail of A rows (and any stale bytes there) meets
            // only zero B rows.
            auto make_unit = [&](int x, int kb) -> LoaderUnit {
                LoaderUnit u{};
                if (x == 0) {
                    const int row0 = tm * Cfg::BM, col0 = kb * Cfg::BK;
                    u.src = static_cast<const uint8_t*>(r0.A) + static_cast<long long>(row0) * r0.lda + col0;
                    u.ld = r0.lda;
                    u.nrows = min(LC::UNIT_ROWS, r0.M - row0);
                    u.valid = min(Cfg::BK, r0.K - col0);
                    u.dst0 = smem_u32(s.a[stage][0]);
                } else {
                    const int row0 = kb * Cfg::BK, col0 = tn * Cfg::BN;
                    u.src = static_cast<const uint8_t*>(r0.B) + static_cast<long long>(row0) * r0.ldb + col0;
                    u.ld = r0.ldb;
                    u.nrows = min(Cfg::BK, r0.K - row0);
                    u.valid = min(Cfg::BN, r0.N - col0);
                    u.dst0 = smem_u32(s.b[stage][0]);
                    u.flags = LU_ZERO;
                }
                return u;
            };
            for (int kb = 0; kb < kbn && ok; ++kb) {
                if constexpr (LC::STAGED) {
                    // the shift warps' entries of this stage (a marker when TMA
                    // loads all of it: they arrive on every stage)
                    const int mask = gen & (TILE_GEN_A | TILE_GEN_B);
                    if (mask == 0) {
                        LoaderUnit u{};
                        u.flags = LU_MARKER | LU_FIRST | LU_LAST;
                        u.stage = stage;
                        u.par = phase;
                        ok = put(u);
                    } else {
#pragma unroll
                        for (int x = 0; x < 2; ++x) {
                            if (!((mask >> x) & 1) || !ok) continue;
                            LoaderUnit u = make_unit(x, kb);
                            u.flags |= (x == 0 || mask == TILE_GEN_B ? LU_FIRST : 0) |
                                       (x == 1 || mask == TILE_GEN_A ? LU_LAST : 0) | (tx == 0 ? LU_PROD : 0);
                            u.stage = stage;
                            u.par = phase;
                            ok = put(u);
                        }
                    }
                    if (!ok) break;
                }
                // the stage itself: TMA loads of the other operands, or the
                // producer's arrival alone -- except for a stage the shift
                // warps fill entirely (LU_PROD), which the producer leaves
                // to them, so its copies for later stages are not held up
                // by this stage's wait
                int oke = 1;
                if (lane == 0) {
                    if (LC::STAGED && tx == 0) {
                        issued_mask &= ~(1u << stage);
                    } else if (!mbar_wait(&s.empty[stage], phase ^ 1u, g.timeout_ns, g.status, 0x31, abort)) {
                        oke = 0;
                    } else if (tx == 0) {
                        mbar_arrive(&s.full[stage]);
                        issued_mask &= ~(1u << stage);
                    } else {
                        const int kx = kb * Cfg::BK;
                        mbar_arrive_expect_tx(&s.full[stage], tx);
                        if (!(gen & TILE_GEN_A))
                            for (int i2 = 0; i2 < Cfg::NA; ++i2)
                                tma_load_2d(s.a[stage][i2], mp + i2, kx, tm * Cfg::BM, &s.full[stage]);
                        if (!(gen & TILE_GEN_B))
                            for (int i2 = 0; i2 < Cfg::NB; ++i2) {
#pragma unroll
                                for (int c = 0; c < Cfg::B_CHUNKS; ++c)
                                    tma_load_2d(s.b[stage][i2] + c * Cfg::B_CHUNK_BYTES, mp + Cfg::NA + i2,
                                                tn * Cfg::BN + c * Cfg::B_CHUNK_ELEMS, kx, &s.full[stage]);
                            }
                        issued_mask |= 1u << stage;
                        issued_par = (issued_par & ~(1u << stage)) | (phase << stage);
                    }
                }
                if (!__shfl_sync(0xffffffffu, oke, 0)) {
                    ok = false;
                    break;
                }
                if (++stage == Cfg::STAGES) {
                    stage = 0;
                    phase ^= 1u;
                }
            }
            if (!ok) break;
            if (bi + 1 < TB && b_cur + bi + 1 < total) {
                // the next tile's descriptors, when TMA will read them
                const TileRec& r1 = trec[sl_cur * TB + bi + 1];
                if (lane == 0 && r1.problem != pi) {
                    const int gen1 = r1.kb >> TILE_GEN_SHIFT;
                    const CUtensorMap* mp1 = g.maps + (long long)r1.problem * NMAPS;
                    if (!(gen1 & TILE_GEN_A))
                        for (int i2 = 0; i2 < Cfg::NA; ++i2) tma_prefetch_desc(mp1 + i2);
                    if (!(gen1 & TILE_GEN_B))
                        for (int i2 = 0; i2 < Cfg::NB; ++i2) tma_prefetch_desc(mp1 + Cfg::NA + i2);
                }
            }
            if (++bi == TB) {
                bi = 0;
                b_cur = b_nxt;
                b_nxt = b_nn;
                sl_cur = sl_cur == 2 ? 0 : sl_cur + 1;
            }
        }
        if (LC::STAGED && ok) {
            LoaderUnit e{};
            e.flags = LU_END;  // tells the shift warps to stop
            ok = put(e);
        }
        cp_async_wait<0>();  // copies still in flight (error path) land before the block exits
        if (!ok && lane == 0) {
            // TMA copies still in flight must land before the CTA exits.  A
            // stage's phase also waits for the shift warps, which may have
            // given up, so each wait gets a share of the time limit.
            for (int i2 = 0; i2 < Cfg::STAGES; ++i2) {
                if (!((issued_mask >> i2) & 1u)) continue;
                volatile int never = 0;
                mbar_wait(&s.full[i2], (issued_par >> i2) & 1u, g.timeout_ns / Cfg::STAGES, nullptr, 0, &never);
            }
        }
    } else if (warp == 1) {
        if (elect_one()) {
            int stage = 0;
            uint32_t phase = 0;
            int it = 0;
            bool ok = true;
            int slot = 0;
            uint32_t sph = 0;
            while (ok) {
                if (!mbar_wait(&sched_full[slot], sph, g.timeout_ns, g.status, 0x45, abort)) {
                    ok = false;
                    break;
                }
                const int4 rec = sched_rec[slot];
                mbar_arrive(&sched_empty[slot]);
                if (++slot == SLOTS) {
                    slot = 0;
                    sph ^= 1u;
                }
                if (rec.x < 0) break;
                const int kblocks = rec.w & TILE_KB_MASK;
                const int kchunk = (Cfg::CHUNKED && g.kchunk > 0) ? g.kchunk : max(kblocks, 1);
                for (int kc0 = 0; kc0 < max(kblocks, 1) && ok; kc0 += kchunk, ++it) {
                    const int kc1 = min(kblocks, kc0 + kchunk);
                    const int buf = it % Cfg::ACC_BUFS;
                    const uint32_t acc_par = static_cast<uint32_t>((it / Cfg::ACC_BUFS) & 1);
                    if (!mbar_wait(&s.acc_empty[buf], acc_par ^ 1u, g.timeout_ns, g.status, 0x41, abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t acc_base = tmem + buf * Cfg::ACC_COLS;
                    for (int kb = kc0; kb < kc1; ++kb) {
                        if (!mbar_wait(&s.full[stage], phase, g.timeout_ns, g.status, 0x42, abort)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
#pragma unroll
                        for (int o = 0; o < Cfg::NOPS; ++o) {
                            const TcOp op = g.ops[o];
                            bool first_for_acc = true;
#pragma unroll
                            for (int q = 0; q < o; ++q)
                                if (g.ops[q].acc == op.acc) first_for_acc = false;
                            const uint32_t idesc = umma_idesc(Cfg::KIND == KIND_I8 ? 2u : 1u, op.a_fmt,
                                                              op.b_fmt, 0u, 1u, Cfg::BM, Cfg::BN);
                            const uint32_t a_addr = smem_u32(s.a[stage][op.a]);
                            const uint32_t b_addr = smem_u32(s.b[stage][op.b]);
#pragma unroll
                            for (int kk = 0; kk < Cfg::KSTEPS; ++kk) {
                                const uint64_t ad = umma_desc_sw128(a_addr + kk * Cfg::KSTEP_BYTES, 16, 1024);
                                const uint64_t bd = umma_desc_sw128(
                                    b_addr + kk * (Cfg::KSTEP_BYTES / Cfg::ESIZE) * 128, Cfg::B_CHUNK_BYTES, 1024);
                                const uint32_t acc = (kb > kc0 || kk > 0 || !first_for_acc) ? 1u : 0u;
                                if constexpr (Cfg::KIND == KIND_I8)
                                    tc_mma_i8(acc_base + op.acc * Cfg::BN, ad, bd, idesc, acc);
                                else
                                    tc_mma_f16(acc_base + op.acc * Cfg::BN, ad, bd, idesc, acc);
                            }
                        }
                        tc_commit(&s.empty[stage]);
                        if (++stage == Cfg::STAGES) {
                            stage = 0;
                            phase ^= 1u;
                        }
                    }
                    if (!ok) break;
                    tc_commit(&s.acc_full[buf]);
                }
            }
            tc_commit(&s.drain);
            volatile int never = 0;
            mbar_wait(&s.drain, 0, g.timeout_ns, ok ? g.status : nullptr, 0x43, &never);
        }
    } else if (warp < 6) {
        const int ew = warp & 3;
        __shared__ uint32_t epi_stage[4][32][33];
        uint32_t (*stg)[33] = epi_stage[ew];
        int it = 0;
        bool ok = true;
        int slot = 0;
        uint32_t sph = 0;
        while (ok) {
            if (!mbar_wait(&sched_full[slot], sph, g.timeout_ns, g.status, 0x55, abort)) {
                ok = false;
                break;
            }
            const int4 rec = sched_rec[slot];
            __syncwarp();
            if (lane == 0) mbar_arrive(&sched_empty[slot]);
            if (++slot == SLOTS) {
                slot = 0;
                sph ^= 1u;
            }
            if (rec.x < 0) break;
            const int tm = rec.y, tn = rec.z;
            const GroupedProblem pr = g.problems[rec.x];
            const int kblocks = max(rec.w & TILE_KB_MASK, 1);
            const int kchunk = (Cfg::CHUNKED && g.kchunk > 0) ? g.kchunk : kblocks;
            float run[Cfg::CHUNKED ? Cfg::BN : 1];
            if constexpr (Cfg::CHUNKED) {
#pragma unroll
                for (int j = 0; j < Cfg::BN; ++j) run[j] = 0.f;
            }
            const int row0 = tm * Cfg::BM + ew * 32;
            for (int kc0 = 0; kc0 < kblocks; kc0 += kchunk, ++it) {
                const int buf = it % Cfg::ACC_BUFS;
                const uint32_t acc_par = static_cast<uint32_t>((it / Cfg::ACC_BUFS) & 1);
                if (!mbar_wait(&s.acc_full[buf], acc_par, g.timeout_ns, g.status, 0x51, abort)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t row_addr = tmem + (static_cast<uint32_t>(ew * 32) << 16) + buf * Cfg::ACC_COLS;
                if constexpr (Cfg::CHUNKED) {
#pragma unroll
                    for (int c = 0; c < Cfg::BN / 32; ++c) {
                        uint32_t v[32];
                        tmem_ld_32x32b_x32(row_addr + c * 32, v);
                        tmem_wait_ld();
#pragma unroll
                        for (int j = 0; j < 32; ++j) run[c * 32 + j] = __fadd_rn(run[c * 32 + j], __uint_as_float(v[j]));
                    }
                } else {
                    // chunks past the problem's last row / column hold nothing
                    const int nch = row0 < pr.M ? min(Cfg::BN / 32, (pr.N - tn * Cfg::BN + 31) / 32) : 0;
#pragma unroll 1
                    for (int c = 0; c < nch; ++c) {
                        uint32_t v[32];
                        tmem_ld_32x32b_x32(row_addr + c * 32, v);
                        tmem_wait_ld();
                        grouped_store<Cfg>(g, pr, row0, tn * Cfg::BN + c * 32, v, stg, lane);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&s.acc_empty[buf]);
            }
            if (!ok) break;
            if constexpr (Cfg::CHUNKED) {
#pragma unroll
                for (int c = 0; c < Cfg::BN / 32; ++c) {
                    uint32_t v[32];
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[j] = __float_as_uint(run[c * 32 + j]);
                    grouped_store<Cfg>(g, pr, row0, tn * Cfg::BN + c * 32, v, stg, lane);
                }
            }
        }
    } else if constexpr (LC::STAGED) {
        // Shift warps 6 and 7: every entry in order, each warp half of every
        // unit's rows.  Per entry: wait for its copies and record (raw_full),
        // for the stage to be free (first entry of a stage), shift the rows
        // into the stage, fence the generic stores for the tensor cores, free
        // the raw slot and, after the last entry of a stage, arrive on its
        // full barrier.
        const int half = warp - 6;
        int rs = 0;
        uint32_t rph = 0;
        while (true) {
            if (!wait0(&raw_full[rs], rph, 0x67)) break;
            const LoaderUnit u = lu[rs];
            if (u.flags & LU_END) break;
            if ((u.flags & LU_FIRST) && !wait0(&s.empty[u.stage], u.par ^ 1u, 0x61)) break;
            if (!(u.flags & LU_MARKER)) {
                shift_rows_u8<LC>(u, raw0 + rs * LC::RAW_BYTES, half, lane);
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            }
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&raw_full[LC::NRAW + rs]);  // raw_empty[rs]
                if (u.flags & LU_LAST) {
                    mbar_arrive(&s.full[u.stage]);
                    if ((u.flags & LU_PROD) && half == 0) mbar_arrive(&s.full[u.stage]);
                }
            }
            if (++rs == LC::NRAW) {
                rs = 0;
                rph ^= 1u;
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, Cfg::TMEM_COLS);
    }
}

// ------------------------------------------------------------------ split prep
// The split form's pass over its f32 operands: each segment (one operand of
// one problem) is cut into bf16 hi = bf16(x) and lo = bf16(x - hi) planes
// (round to nearest even) with a 16-byte-multiple pitch that TMA reads.
// One block per segment (grid-stride over segments); the block's threads
// take the segment's 8-element destination chunks in row-major order, so
// rows shorter than a warp's reach still keep every lane busy.  Elements
// past a row's end become 0.
struct SplitSeg {
    const float* src;
    __nv_bfloat16* hi;
    __nv_bfloat16* lo;
    long long rows, cols, ld_src, ld_dst;  // elements
};

static __global__ void split_prep_kernel(const SplitSeg* __restrict__ segs, int nseg) {
    for (int si = blockIdx.x; si < nseg; si += gridDim.x) {
        const SplitSeg sg = segs[si];
        const long long cpr = sg.ld_dst / 8;  // chunks per row
        const long long total = sg.rows * cpr;
        for (long long idx = threadIdx.x; idx < total; idx += blockDim.x) {
            const long long r = idx / cpr, c = (idx - r * cpr) * 8;
            const float* src = sg.src + r * sg.ld_src;
            uint32_t h[4], l[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const float x0 = c + 2 * e < sg.cols ? __ldg(src + c + 2 * e) : 0.f;
                const float x1 = c + 2 * e + 1 < sg.cols ? __ldg(src + c + 2 * e + 1) : 0.f;
                const __nv_bfloat162 hv = __floats2bfloat162_rn(x0, x1);
                const __nv_bfloat162 lv = __floats2bfloat162_rn(x0 - __low2float(hv), x1 - __high2float(hv));
                h[e] = *reinterpret_cast<const uint32_t*>(&hv);
                l[e] = *reinterpret_cast<const uint32_t*>(&lv);
            }
            *reinterpret_cast<uint4*>(sg.hi + r * sg.ld_dst + c) = make_uint4(h[0], h[1], h[2], h[3]);
            *reinterpret_cast<uint4*>(sg.lo + r * sg.ld_dst + c) = make_uint4(l[0], l[1], l[2], l[3]);
        }
    }
}

// ------------------------------------------------------------------ SIMT
// Plain FP32 grouped GEMM (FFMA): 64x64 tiles, 128 threads, 4x8 outputs per
// thread, persistent over the global tile list.
struct SimtGroupedArgs {
    const GroupedProblem* problems;
    const TileRec* tiles;  // [total_tiles]
    unsigned long long* tile_counter;  // next unclaimed tile (zeroed before the launch)
    const void* const* a;  // per problem operand pointers and leading dims
    const void* const* b;
    const long long* lda;
    const long long* ldb;
    int count;
    long long total_tiles;
    float alpha, beta;
};

// A 32 x 32 tile of a small problem on the same 128 threads: 2 rows x 4
// columns a thread, the same double-buffered K blocks of 16 and the same
// per-output k order (one FMA per product, k ascending).  Uses the caller's
// shared tiles (the first 32 columns of each row).
__device__ __forceinline__ void grouped_tile32(const SimtGroupedArgs& g, const GroupedProblem& pr,
                                               const float* __restrict__ A, const float* __restrict__ B,
                                               long long lda, long long ldb, int m0, int n0,
                                               float (*As)[16][68], float (*Bs)[16][68]) {
    constexpr int BK = 16;
    const int tid = threadIdx.x, tx = tid % 8, ty = tid / 8;
    float ra[4], rb[4];
    auto load = [&](int k0) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = tid + q * 128;  // 512 elements of each 32 x 16 / 16 x 32 tile
            const int ar = e / BK, ac = e % BK;
            const int gr = m0 + ar, gk = k0 + ac;
            ra[q] = (gr < pr.M && gk < pr.K) ? A[(long long)gr * lda + gk] : 0.f;
            const int br = e / 32, bc = e % 32;
            const int gk2 = k0 + br, gn = n0 + bc;
            rb[q] = (gk2 < pr.K && gn < pr.N) ? B[(long long)gk2 * ldb + gn] : 0.f;
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int e = tid + q * 128;
            As[buf][e % BK][e / BK] = ra[q];
            Bs[buf][e / 32][e % 32] = rb[q];
        }
    };
    float acc[2][4] = {};
    const int kblocks = (pr.K + BK - 1) / BK;
    load(0);
    __syncthreads();  // the previous tile's readers are done with buffer 0
    store(0);
    __syncthreads();
    for (int kb = 0; kb < kblocks; ++kb) {
        const int cur = kb & 1;
        if (kb + 1 < kblocks) load((kb + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            const float2 a2 = *reinterpret_cast<const float2*>(&As[cur][kk][ty * 2]);
            const float4 b4 = *reinterpret_cast<const float4*>(&Bs[cur][kk][tx * 4]);
            const float af[2] = {a2.x, a2.y}, bf[4] = {b4.x, b4.y, b4.z, b4.w};
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = fmaf(af[i], bf[j], acc[i][j]);
        }
        if (kb + 1 < kblocks) store(cur ^ 1);
        __syncthreads();
    }
    float* C = static_cast<float*>(pr.C);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
        const int gr = m0 + ty * 2 + i;
        if (gr >= pr.M) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int gc = n0 + tx * 4 + j;
            if (gc >= pr.N) continue;
            float* p = C + (long long)gr * pr.ldc + gc;
            float o = g.alpha * acc[i][j];
            if (g.beta != 0.f) o = fmaf(g.beta, *p, o);
            *p = o;
        }
    }
}

static __global__ void __launch_bounds__(128) simt_grouped_sgemm(const SimtGroupedArgs g) {
    constexpr int BM = 64, BN = 64, BK = 16, NT = 128;
    constexpr int PER = BM * BK / NT;  // elements of each operand a thread loads per K block
    __shared__ __align__(16) float As[2][BK][BM + 4];
    __shared__ __align__(16) float Bs[2][BK][BN + 4];
    // 16 x 8 threads, 4 rows x 8 columns each (two 4-column groups 32 apart)
    const int tid = threadIdx.x, tx = tid % 8, ty = tid / 8;
    // device-side tile scheduler: thread 0 claims the next tile for the CTA;
    // two slots, so the claim for tile i + 1 cannot overwrite the index
    // others may still be reading for tile i
    __shared__ long long claim[2];
    for (int i = 0;; ++i) {
        if (tid == 0) claim[i & 1] = static_cast<long long>(atomicAdd(g.tile_counter, 1ull));
        __syncthreads();
        const long long t = claim[i & 1];
        if (t >= g.total_tiles) break;
        const TileRec tr = g.tiles[t];
        const int pi = tr.problem;
        const GroupedProblem pr = g.problems[pi];
        const float* A = static_cast<const float*>(g.a[pi]);
        const float* B = static_cast<const float*>(g.b[pi]);
        const long long lda = g.lda[pi], ldb = g.ldb[pi];
        if (pr.tile == 32) {
            grouped_tile32(g, pr, A, B, lda, ldb, tr.tm * 32, tr.tn * 32, As, Bs);
            continue;
        }
        const int m0 = tr.tm * BM, n0 = tr.tn * BN;
        // Next K block into registers while this one is computed; shared
        // tiles double-buffered, one barrier per K block.
        float ra[PER], rb[PER];
        auto load = [&](int k0) {
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const int e = tid + q * NT;
                const int ar = e / BK, ac = e % BK;
                const int gr = m0 + ar, gk = k0 + ac;
                ra[q] = (gr < pr.M && gk < pr.K) ? A[(long long)gr * lda + gk] : 0.f;
                const int br = e / BN, bc = e % BN;
                const int gk2 = k0 + br, gn = n0 + bc;
                rb[q] = (gk2 < pr.K && gn < pr.N) ? B[(long long)gk2 * ldb + gn] : 0.f;
            }
        };
        auto store = [&](int buf) {
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const int e = tid + q * NT;
                As[buf][e % BK][e / BK] = ra[q];
                Bs[buf][e / BN][e % BN] = rb[q];
            }
        };
        float acc[4][8] = {};
        const int kblocks = (pr.K + BK - 1) / BK;
        load(0);
        __syncthreads();  // the previous tile's readers are done with buffer 0
        store(0);
        __syncthreads();
        for (int kb = 0; kb < kblocks; ++kb) {
            const int cur = kb & 1;
            if (kb + 1 < kblocks) load((kb + 1) * BK);
#pragma unroll
            for (int kk = 0; kk < BK; ++kk) {
                const float4 a4 = *reinterpret_cast<const float4*>(&As[cur][kk][ty * 4]);
                const float4 b0 = *reinterpret_cast<const float4*>(&Bs[cur][kk][tx * 4]);
                const float4 b1 = *reinterpret_cast<const float4*>(&Bs[cur][kk][32 + tx * 4]);
                const float af[4] = {a4.x, a4.y, a4.z, a4.w};
                const float bf[8] = {b0.x, b0.y, b0.z, b0.w, b1.x, b1.y, b1.z, b1.w};
#pragma unroll
                for (int i = 0; i < 4; ++i)
#pragma unroll
                    for (int j = 0; j < 8; ++j) acc[i][j] = fmaf(af[i], bf[j], acc[i][j]);
            }
            if (kb + 1 < kblocks) store(cur ^ 1);
            __syncthreads();
        }
        float* C = static_cast<float*>(pr.C);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int gr = m0 + ty * 4 + i;
            if (gr >= pr.M) continue;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int gc = n0 + (j / 4) * 32 + tx * 4 + (j % 4);
                if (gc >= pr.N) continue;
                float* p = C + (long long)gr * pr.ldc + gc;
                float o = g.alpha * acc[i][j];
                if (g.beta != 0.f) o = fmaf(g.beta, *p, o);
                *p = o;
            }
        }
    }
}

}  // namespace fg
