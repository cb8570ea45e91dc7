// tc_grouped.cuh -- persistent grouped (ragged-batch) GEMM on tcgen05.
//
// One launch runs `count` independent problems of different M, N, K.  A
// device-side problem table holds, per problem, its shape, its tile range in
// a global tile numbering (prefix sums), its output and the TMA descriptors
// of its operands (written to global memory before the launch).  Tiles are
// numbered deepest problem first.  A device-side tile scheduler hands them
// out: each CTA's producer claims the next global tile with an atomic add
// on a counter (zeroed before every launch), so CTAs that drew short tiles
// come back for more and the heavy tiles go first (dynamic
// longest-processing-time order).  The producer passes each claimed tile
// record to the CTA's MMA and epilogue roles through a small ring of
// shared-memory slots guarded by mbarriers, so all three roles of
// tc_gemm.cuh (TMA producer, MMA issuer, epilogue) walk the same sequence;
// a record past the end tells them to stop.  The producer claims two tiles
// ahead and prefetches the next tile's tensor maps while the current one
// loads.  Operands TMA cannot read as they are (i8 rows that break its
// 16-byte rule, the split form's f32 operands) are rewritten once by
// grouped_prep_kernel into an arena before the launch.  A is loaded as
// 8-row boxes spread over the accumulator's lane quadrants (spread_row), so
// short tiles keep all four epilogue warps busy.
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
};

// Per global tile: problem index, tile row, tile column and the problem's K
// blocks (written by the host with the problem table, so a tile costs one
// 16-byte load instead of a search; the producer and the MMA issuer need
// nothing else).
struct TileRec {
    int problem, tm, tn, kb;
};

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


// Row spreading: the producer loads a tile's A rows as sixteen 8-row TMA
// boxes, source rows 8i .. 8i + 7 into shared-memory rows 32 (i % 4) +
// 8 (i / 4) (each box is one 1024-byte 128B-swizzle atom, so the layout is
// the canonical one with the rows permuted).  Accumulator row p -- TMEM lane
// p, read by epilogue warp p / 32 -- then holds tile row
// 32 ((p % 32) / 8) + 8 (p / 32) + p % 8, so a tile's first 32 rows are
// shared by all four epilogue warps instead of all landing on the first
// (ragged tiles are mostly short: M averages about 121).
__device__ __forceinline__ int spread_row(int ew, int lane) {
    return 32 * (lane >> 3) + 8 * ew + (lane & 7);
}

// Stores one warp's 32 rows x 32 columns: lane l holds tile row
// spread_row(ew, l) of the tile starting at row `base`.  The
// block goes through a padded shared-memory tile so that the global stores
// (and the reads of C for accumulate / beta) are 128-byte row segments.  The
// tile's rows are 36 words apart: each lane writes its row as eight 16-byte
// stores (banks 4l + 4q: no conflict within a quarter warp) and each lane
// then reads one column (banks 4r + l: no conflict).
constexpr int EPI_PITCH = 36;
template <class Cfg>
__device__ __forceinline__ void grouped_store(const GroupedArgs& g, const GroupedProblem& pr, int base, int ew,
                                              int col0, const uint32_t (&v)[32], uint32_t (*stg)[EPI_PITCH],
                                              int lane) {
#pragma unroll
    for (int q = 0; q < 8; ++q)
        *reinterpret_cast<uint4*>(&stg[lane][4 * q]) = make_uint4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
    __syncwarp();
    const int col = col0 + lane;
    // row r of the staged block is tile row spread_row(ew, r) = 8 ew + rel(r)
    const int lim = pr.M - base - 8 * ew;  // rel(r) < lim: the row exists
#define FG_REL(r) (32 * ((r) >> 3) + ((r) & 7))
    if (col < pr.N) {
        // unrolled with predicates: all shared-memory reads (and the reads
        // of C for accumulate / beta) are issued before the first store, so
        // they overlap instead of costing one round trip per row
        uint32_t w[32];
#pragma unroll
        for (int r = 0; r < 32; ++r) w[r] = stg[r][lane];
        const long long ldc = pr.ldc;
        if constexpr (Cfg::EPI == EPI_I32) {
            int32_t* p = static_cast<int32_t*>(pr.C) + (long long)(base + 8 * ew) * ldc + col;
            if (g.accumulate) {
#pragma unroll
                for (int r = 0; r < 32; ++r)
                    if (FG_REL(r) < lim) w[r] += static_cast<uint32_t>(p[FG_REL(r) * ldc]);
            }
#pragma unroll
            for (int r = 0; r < 32; ++r)
                if (FG_REL(r) < lim) p[FG_REL(r) * ldc] = static_cast<int32_t>(w[r]);
        } else {
            float* p = static_cast<float*>(pr.C) + (long long)(base + 8 * ew) * ldc + col;
            float o[32];
#pragma unroll
            for (int r = 0; r < 32; ++r) o[r] = g.alpha * __uint_as_float(w[r]);
            if (g.beta != 0.f) {
#pragma unroll
                for (int r = 0; r < 32; ++r)
                    if (FG_REL(r) < lim) o[r] = fmaf(g.beta, p[FG_REL(r) * ldc], o[r]);
            }
#pragma unroll
            for (int r = 0; r < 32; ++r)
                if (FG_REL(r) < lim) p[FG_REL(r) * ldc] = o[r];
        }
    }
#undef FG_REL
    __syncwarp();
}

template <class Cfg>
__global__ void __launch_bounds__(Cfg::THREADS, 1)
    tc_grouped_kernel(const __grid_constant__ GroupedArgs g) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* base = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    TcSmem<Cfg>& s = *reinterpret_cast<TcSmem<Cfg>*>(base);
    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    volatile int* abort = &s.abort;
    constexpr int NMAPS = Cfg::NA + Cfg::NB;
    // tile-scheduler ring: the producer writes claimed tile indices, the MMA
    // thread and the four epilogue warps read them in order
    constexpr int SLOTS = 16;
    __shared__ uint64_t sched_full[SLOTS], sched_empty[SLOTS];
    __shared__ int4 sched_rec[SLOTS];  // the tile's TileRec; problem < 0 ends the walk

    if (threadIdx.x == 0) {
        for (int i = 0; i < SLOTS; ++i) {
            mbar_init(&sched_full[i], 1);
            mbar_init(&sched_empty[i], 5);
        }
        for (int i = 0; i < Cfg::STAGES; ++i) {
            mbar_init(&s.full[i], 1);
            mbar_init(&s.empty[i], 1);
        }
        for (int i = 0; i < 4; ++i) {
            mbar_init(&s.acc_full[i], 1);
            mbar_init(&s.acc_empty[i], 4);
        }
        mbar_init(&s.drain, 1);
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

    if (warp == 0) {
        if (elect_one()) {
            int stage = 0;
            uint32_t phase = 0;
            // per stage: a load was issued (bit) and its phase parity (bit),
            // kept in registers
            uint32_t issued_mask = 0, issued_par = 0;
            bool ok = true;
            int slot = 0;
            uint32_t sph = 0;
            // Two claims ahead: while the loads of tile t0 are issued, the
            // record of t1 is already in flight and t2 is being claimed, so
            // no global round trip sits between two tiles' loads.
            const long long total = g.total_tiles;
            const TileRec none{-1, 0, 0, 0};
            long long t0 = static_cast<long long>(atomicAdd(g.tile_counter, 1ull));
            long long t1 = t0 < total ? static_cast<long long>(atomicAdd(g.tile_counter, 1ull)) : t0;
            TileRec r0 = t0 < total ? g.tiles[t0] : none;
            while (ok) {
                // publish the claimed tile (or the end marker) to the other roles
                if (!mbar_wait(&sched_empty[slot], sph ^ 1u, g.timeout_ns, g.status, 0x35, abort)) {
                    ok = false;
                    break;
                }
                sched_rec[slot] = make_int4(r0.problem, r0.tm, r0.tn, r0.kb);
                mbar_arrive(&sched_full[slot]);
                if (++slot == SLOTS) {
                    slot = 0;
                    sph ^= 1u;
                }
                if (t0 >= total) break;
                const long long t2 = t1 < total ? static_cast<long long>(atomicAdd(g.tile_counter, 1ull)) : t1;
                const TileRec r1 = t1 < total ? g.tiles[t1] : none;  // used after this tile's loads
                const int pi = r0.problem, tm = r0.tm, tn = r0.tn;
                const CUtensorMap* mp = g.maps + (long long)pi * NMAPS;
                for (int kb = 0; kb < r0.kb; ++kb) {
                    if (!mbar_wait(&s.empty[stage], phase ^ 1u, g.timeout_ns, g.status, 0x31, abort)) {
                        ok = false;
                        break;
                    }
                    mbar_arrive_expect_tx(&s.full[stage], Cfg::STAGE_BYTES);
                    const int kx = kb * Cfg::BK;
                    // A as sixteen 8-row boxes, spread over the accumulator's
                    // lane quadrants (spread_row)
                    for (int i = 0; i < Cfg::NA; ++i)
#pragma unroll
                        for (int bx = 0; bx < Cfg::BM / 8; ++bx)
                            tma_load_2d(s.a[stage][i] + (32 * (bx & 3) + 8 * (bx >> 2)) * Cfg::BK_BYTES, mp + i, kx,
                                        tm * Cfg::BM + 8 * bx, &s.full[stage]);
                    for (int i = 0; i < Cfg::NB; ++i) {
#pragma unroll
                        for (int c = 0; c < Cfg::B_CHUNKS; ++c)
                            tma_load_2d(s.b[stage][i] + c * Cfg::B_CHUNK_BYTES, mp + Cfg::NA + i,
                                        tn * Cfg::BN + c * Cfg::B_CHUNK_ELEMS, kx, &s.full[stage]);
                    }
                    issued_mask |= 1u << stage;
                    issued_par = (issued_par & ~(1u << stage)) | (phase << stage);
                    if (++stage == Cfg::STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                if (r1.problem >= 0 && r1.problem != pi)
                    for (int i = 0; i < NMAPS; ++i) tma_prefetch_desc(g.maps + (long long)r1.problem * NMAPS + i);
                t0 = t1;
                t1 = t2;
                r0 = r1;
            }
            if (!ok) {
                for (int i = 0; i < Cfg::STAGES; ++i) {
                    if (!((issued_mask >> i) & 1u)) continue;
                    volatile int never = 0;
                    mbar_wait(&s.full[i], (issued_par >> i) & 1u, g.timeout_ns, nullptr, 0, &never);
                }
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
                const int kblocks = rec.w;
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
    } else {
        const int ew = warp & 3;
        __shared__ __align__(16) uint32_t epi_stage[4][32][EPI_PITCH];
        uint32_t (*stg)[EPI_PITCH] = epi_stage[ew];
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
            const int kblocks = max(rec.w, 1);
            const int kchunk = (Cfg::CHUNKED && g.kchunk > 0) ? g.kchunk : kblocks;
            float run[Cfg::CHUNKED ? Cfg::BN : 1];
            if constexpr (Cfg::CHUNKED) {
#pragma unroll
                for (int j = 0; j < Cfg::BN; ++j) run[j] = 0.f;
            }
            const int base = tm * Cfg::BM;  // this warp's rows: base + spread_row(ew, lane)
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
                    const int nch = base + 8 * ew < pr.M ? min(Cfg::BN / 32, (pr.N - tn * Cfg::BN + 31) / 32) : 0;
                    // two chunks in flight: chunk c + 1 is read out of TMEM
                    // while chunk c goes to memory
                    uint32_t va[32], vb[32];
                    if (nch > 0) tmem_ld_32x32b_x32(row_addr, va);
#pragma unroll 1
                    for (int c = 0; c < nch; c += 2) {
                        tmem_wait_ld();
                        if (c + 1 < nch) tmem_ld_32x32b_x32(row_addr + (c + 1) * 32, vb);
                        grouped_store<Cfg>(g, pr, base, ew, tn * Cfg::BN + c * 32, va, stg, lane);
                        if (c + 1 < nch) {
                            tmem_wait_ld();
                            if (c + 2 < nch) tmem_ld_32x32b_x32(row_addr + (c + 2) * 32, va);
                            grouped_store<Cfg>(g, pr, base, ew, tn * Cfg::BN + (c + 1) * 32, vb, stg, lane);
                        }
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
                    if (base + 8 * ew < pr.M)
                        grouped_store<Cfg>(g, pr, base, ew, tn * Cfg::BN + c * 32, v, stg, lane);
                }
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

// ------------------------------------------------------------------ prep
// One launch over a list of segments, one per operand that TMA cannot read
// as it is: op 0 copies a byte matrix whose pointer or leading dimension
// breaks the TMA 16-byte rule into a 16-byte-pitched buffer (i8); op 1 cuts
// an f32 matrix into bf16 hi = bf16(x) and lo = bf16(x - hi) planes (round
// to nearest even; the split form).  Bytes / elements past a row's end
// become 0.  Source rows are read as the aligned 16-byte granules that hold
// them (a granule is read only when it holds a byte of the row, so every
// read stays on memory the row occupies) and shifted into place in
// registers, so each thread issues one to three 16-byte loads per 16-byte
// output chunk, PREP_ILP chunks per thread per pass with every load issued
// before the first store.
struct PrepSeg {
    const void* src;
    void* dst0;
    void* dst1;
    long long rows, cols, ld_src, ld_dst;  // elements
    int op;
};

// output chunks per thread per pass (loads issued first): one for both ops
// -- two halved the blocks per SM (registers) and were measured slower
constexpr int PREP_ILP = 1;

// op 0: 16 bytes of a row starting at byte address p, `valid` of them in
// the row (valid <= 0: none).
struct PrepBytes {
    ulonglong2 w0, w1;
    int sh;
    int valid;
};
__device__ __forceinline__ PrepBytes prep_load_bytes(const uint8_t* p, long long valid) {
    PrepBytes g;
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uintptr_t base = a & ~static_cast<uintptr_t>(15);
    g.sh = static_cast<int>(a - base);
    g.valid = static_cast<int>(valid < 0 ? 0 : valid > 16 ? 16 : valid);
    g.w0 = make_ulonglong2(0ull, 0ull);
    g.w1 = make_ulonglong2(0ull, 0ull);
    if (g.valid > 0) g.w0 = __ldg(reinterpret_cast<const ulonglong2*>(base));
    if (g.valid > 0 && g.sh + g.valid > 16) g.w1 = __ldg(reinterpret_cast<const ulonglong2*>(base + 16));
    return g;
}
__device__ __forceinline__ ulonglong2 prep_shift_bytes(const PrepBytes& g) {
    if (g.valid <= 0) return make_ulonglong2(0ull, 0ull);
    const bool hi = g.sh >= 8;
    const unsigned long long x0 = hi ? g.w0.y : g.w0.x, x1 = hi ? g.w1.x : g.w0.y, x2 = hi ? g.w1.y : g.w1.x;
    const int sb = (g.sh & 7) * 8;
    unsigned long long o0 = sb ? (x0 >> sb) | (x1 << (64 - sb)) : x0;
    unsigned long long o1 = sb ? (x1 >> sb) | (x2 << (64 - sb)) : x1;
    if (g.valid < 16) {
        o1 = g.valid <= 8 ? 0ull : (o1 & ((1ull << (8 * (g.valid - 8))) - 1));
        if (g.valid < 8) o0 &= (1ull << (8 * g.valid)) - 1;
    }
    return make_ulonglong2(o0, o1);
}

// op 1: 8 floats of a row starting at p (4-byte aligned), `valid` of them
// in the row, from the two or three aligned granules that hold them.
struct PrepFloats {
    float4 g0, g1, g2;
    int q;  // floats into the first granule
    int valid;
};
__device__ __forceinline__ PrepFloats prep_load_floats(const float* p, long long valid) {
    PrepFloats g;
    const uintptr_t a = reinterpret_cast<uintptr_t>(p);
    const uintptr_t base = a & ~static_cast<uintptr_t>(15);
    g.q = static_cast<int>(a - base) >> 2;
    g.valid = static_cast<int>(valid < 0 ? 0 : valid > 8 ? 8 : valid);
    const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
    const float4* gp = reinterpret_cast<const float4*>(base);
    g.g0 = g.valid > 0 ? __ldg(gp) : z;
    g.g1 = g.valid > 0 && g.q + g.valid > 4 ? __ldg(gp + 1) : z;
    g.g2 = g.valid > 0 && g.q > 0 && g.q + g.valid > 8 ? __ldg(gp + 2) : z;
    return g;
}
__device__ __forceinline__ void prep_split_floats(const PrepFloats& g, uint4& hi, uint4& lo) {
    const float w[12] = {g.g0.x, g.g0.y, g.g0.z, g.g0.w, g.g1.x, g.g1.y, g.g1.z, g.g1.w,
                         g.g2.x, g.g2.y, g.g2.z, g.g2.w};
    float v[11], f[8];
#pragma unroll
    for (int k = 0; k < 11; ++k) v[k] = (g.q & 1) ? w[k + 1] : w[k];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float x = (g.q & 2) ? v[k + 2] : v[k];
        f[k] = k < g.valid ? x : 0.f;
    }
    uint32_t h[4], l[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const __nv_bfloat162 hv = __floats2bfloat162_rn(f[2 * e], f[2 * e + 1]);
        const __nv_bfloat162 lv = __floats2bfloat162_rn(f[2 * e] - __low2float(hv), f[2 * e + 1] - __high2float(hv));
        h[e] = *reinterpret_cast<const uint32_t*>(&hv);
        l[e] = *reinterpret_cast<const uint32_t*>(&lv);
    }
    hi = make_uint4(h[0], h[1], h[2], h[3]);
    lo = make_uint4(l[0], l[1], l[2], l[3]);
}

// A block job: chunks [c0, c1) of one segment.  Segments longer than
// PREP_JOB_CHUNKS chunks are cut into several jobs (host-built table), so
// the largest operands do not leave one block working long after the rest.
struct PrepJob {
    int seg, pad;
    long long c0, c1;
};
constexpr long long PREP_JOB_CHUNKS = 4096;

// OP: every segment of a launch has the same op (a plan is all i8 or all
// split), so each op gets its own instantiation and register budget.
template <int OP>
static __global__ void __launch_bounds__(256) grouped_prep_kernel(const PrepSeg* __restrict__ segs,
                                                                  const PrepJob* __restrict__ jobs, int njobs) {
    // One block per job (grid-stride over jobs).  The block's threads take
    // the job's 16-byte destination chunks (destination pitch is a multiple
    // of 16 bytes) in row-major order, PREP_ILP per thread per pass with all
    // loads issued before the first store, so rows shorter than a warp's
    // reach still keep every lane busy and each thread keeps several loads in
    // flight; consecutive lanes write consecutive chunks.
    for (int ji = blockIdx.x; ji < njobs; ji += gridDim.x) {
        const PrepJob jb = jobs[ji];
        const PrepSeg sg = segs[jb.seg];
        const unsigned per = OP == 0 ? 16u : 8u;                      // elements per chunk
        const unsigned cpr = static_cast<unsigned>(sg.ld_dst / per);  // chunks per row
        const long long total = jb.c1;
        for (long long pass = jb.c0; pass < total; pass += static_cast<long long>(PREP_ILP) * blockDim.x) {
            long long r[PREP_ILP], c[PREP_ILP];
#pragma unroll
            for (int q = 0; q < PREP_ILP; ++q) {
                const long long idx = pass + threadIdx.x + static_cast<long long>(q) * blockDim.x;
                r[q] = -1;
                c[q] = 0;
                if (idx < total) {
                    if (total < (1LL << 31)) {  // 32-bit division where it fits
                        const unsigned u = static_cast<unsigned>(idx), ur = u / cpr;
                        r[q] = ur;
                        c[q] = static_cast<long long>(u - ur * cpr) * per;
                    } else {
                        r[q] = idx / cpr;
                        c[q] = (idx - r[q] * cpr) * per;
                    }
                }
            }
            if constexpr (OP == 0) {
                PrepBytes g[PREP_ILP];
#pragma unroll
                for (int q = 0; q < PREP_ILP; ++q)
                    g[q] = prep_load_bytes(static_cast<const uint8_t*>(sg.src) + (r[q] < 0 ? 0 : r[q] * sg.ld_src + c[q]),
                                           r[q] < 0 ? 0 : sg.cols - c[q]);
#pragma unroll
                for (int q = 0; q < PREP_ILP; ++q)
                    if (r[q] >= 0)
                        *reinterpret_cast<ulonglong2*>(static_cast<uint8_t*>(sg.dst0) + r[q] * sg.ld_dst + c[q]) =
                            prep_shift_bytes(g[q]);
            } else {
                PrepFloats g[PREP_ILP];
#pragma unroll
                for (int q = 0; q < PREP_ILP; ++q)
                    g[q] = prep_load_floats(static_cast<const float*>(sg.src) + (r[q] < 0 ? 0 : r[q] * sg.ld_src + c[q]),
                                            r[q] < 0 ? 0 : sg.cols - c[q]);
#pragma unroll
                for (int q = 0; q < PREP_ILP; ++q) {
                    if (r[q] < 0) continue;
                    uint4 hi, lo;
                    prep_split_floats(g[q], hi, lo);
                    *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(sg.dst0) + r[q] * sg.ld_dst + c[q]) = hi;
                    *reinterpret_cast<uint4*>(static_cast<__nv_bfloat16*>(sg.dst1) + r[q] * sg.ld_dst + c[q]) = lo;
                }
            }
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
