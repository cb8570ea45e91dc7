// tc_gemm2.cuh -- persistent tcgen05 GEMM on CTA pairs (cta_group::2).
//
// A cluster of two CTAs (one TPC) owns a 256 x BN output tile.  Each CTA
// stages its own 128 rows of A and BN/2 columns of B per K block, so per SM
// a K block moves (128 + BN/2) x 128 bytes through TMA and shared memory
// instead of (128 + BN) x 128 for the single-CTA 128 x BN tile -- the
// shared-memory / TMA request path, not the tensor pipe, bounds the
// single-CTA kernel.  The even CTA (cluster rank 0, the "leader") issues
// tcgen05.mma.cta_group::2 with M = 256: the hardware reads the peer's
// halves at the same shared-memory offsets and writes accumulator rows
// 128..255 into the peer's TMEM.
//
// Barriers (same offsets in both CTAs):
//   full[s]      leader only: the leader's producer arms it with both CTAs'
//                bytes; both CTAs' TMA loads complete on it (cta_group::2
//                form with the leader's cluster address);
//   empty[s]     each CTA: the leader's commit, multicast to the pair,
//                frees stage s in both;
//   acc_full[b]  each CTA: leader's commit (multicast) -> both epilogues;
//   acc_empty[b] leader only: 4 epilogue warps of each CTA arrive (the
//                peer's remotely) before accumulator b is reused
//                (up to 4 accumulator buffers when they fit in TMEM).
// Loads carry no cluster multicast: each CTA reads its own half from HBM.
// Every wait is bounded (timeout, abort flag) like the single-CTA kernel;
// both CTAs meet at a cluster barrier before TMEM is freed.
#pragma once
#include "tc_gemm.cuh"

namespace fg {

// COLSPLIT: the tile is NB x BN columns wide; B operand i holds columns
// [i BN, (i + 1) BN) of the tile and accumulator i receives them (product
// i = A x B_i), so one staged A tile feeds NB MMAs of N = BN -- less shared-
// memory traffic per MAC than NB separate tiles.  Otherwise all operands and
// accumulators cover the same BN columns (split / byte-slice schemes).
template <int KIND_, int BN_, int STAGES_, int NA_, int NB_, int NACC_, int NOPS_, int EPI_,
          int CHUNKED_ = 0, int COLSPLIT_ = 0>
struct Tc2Cfg {
    static constexpr int KIND = KIND_, BM = 256, BN = BN_, STAGES = STAGES_;
    static constexpr int NA = NA_, NB = NB_, NACC = NACC_, NOPS = NOPS_, EPI = EPI_;
    static constexpr int CHUNKED = CHUNKED_, COLSPLIT = COLSPLIT_;
    static constexpr int TILE_N = COLSPLIT ? NB * BN : BN;  // output columns per tile
    static constexpr int ESIZE = KIND == KIND_I8 ? 1 : 2;
    static constexpr int BK_BYTES = 128;
    static constexpr int BK = BK_BYTES / ESIZE;
    static constexpr int KSTEP_BYTES = 32;
    static constexpr int KSTEPS = BK_BYTES / KSTEP_BYTES;
    static constexpr int CTA_M = 128;       // A rows staged (and C rows stored) per CTA
    static constexpr int CTA_N = BN / 2;    // B columns staged per CTA
    static constexpr int A_TILE = CTA_M * BK_BYTES;
    static constexpr int B_TILE = CTA_N * BK_BYTES;
    static constexpr int B_CHUNK_ELEMS = 128 / ESIZE;
    static constexpr int B_CHUNKS = CTA_N / B_CHUNK_ELEMS;
    static constexpr int B_CHUNK_BYTES = BK * 128;
    static constexpr int STAGE_BYTES = NA * A_TILE + NB * B_TILE;  // per CTA
    static constexpr int ACC_COLS = NACC * BN;                     // per CTA
    static constexpr int ACC_BUFS = (4 * ACC_COLS <= 512) ? 4 : (2 * ACC_COLS <= 512) ? 2 : 1;
    static constexpr int TMEM_COLS = 512;
    static constexpr int THREADS = 192;
    static_assert(ACC_COLS <= 512, "accumulators exceed TMEM");
    static_assert(BN % 32 == 0 && BN <= 256, "UMMA N (pair)");
    static_assert(CTA_N % B_CHUNK_ELEMS == 0, "B half must be whole 128-byte chunks");
    static_assert(!COLSPLIT || (NACC == NB && NOPS == NB && !CHUNKED), "column split: one acc per B");
};

// Single-accumulator view of a config for epilogue_store (column-split
// accumulators are stored one at a time).
template <class Cfg>
struct Tc2EpiView {
    static constexpr int NACC = 1, EPI = Cfg::EPI;
};

template <class Cfg>
struct Tc2Smem {
    alignas(1024) uint8_t a[Cfg::STAGES][Cfg::NA][Cfg::A_TILE];
    alignas(1024) uint8_t b[Cfg::STAGES][Cfg::NB][Cfg::B_TILE];
    uint64_t full[Cfg::STAGES];
    uint64_t empty[Cfg::STAGES];
    uint64_t acc_full[4];
    uint64_t acc_empty[4];
    uint64_t drain;
    uint32_t tmem_base;
    int abort;
};

template <class Cfg>
constexpr size_t tc2_smem_bytes() {
    return sizeof(Tc2Smem<Cfg>) + 1024;
}

// Spins for `ns` of global time (bounded): lets loads this thread issued
// land before the CTA leaves after an abort (their barrier may be the
// peer's, which this CTA cannot wait on).
__device__ __forceinline__ void settle_ns(uint64_t ns) {
    const uint64_t t0 = global_timer_ns();
    while (global_timer_ns() - t0 < ns) {
    }
}

template <class Cfg>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(Cfg::THREADS, 1)
    tc_gemm2_kernel(const __grid_constant__ TcMaps maps, const __grid_constant__ TcArgs p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t* base = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    Tc2Smem<Cfg>& s = *reinterpret_cast<Tc2Smem<Cfg>*>(base);

    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    const uint32_t rank = cluster_ctarank();  // 0: leader (issues the MMAs)
    const bool leader = rank == 0;
    const int pair = blockIdx.x / 2, npairs = gridDim.x / 2;
    const int total = max(p.splits, 1) * p.batch * p.tiles_m * p.tiles_n;  // pair tiles
    volatile int* abort = &s.abort;

    if (threadIdx.x == 0) {
        for (int i = 0; i < Cfg::STAGES; ++i) {
            mbar_init(&s.full[i], 1);
            mbar_init(&s.empty[i], 1);
        }
        for (int i = 0; i < 4; ++i) {
            mbar_init(&s.acc_full[i], 1);
            mbar_init(&s.acc_empty[i], 8);  // 4 epilogue warps x 2 CTAs
        }
        mbar_init(&s.drain, 1);
        s.abort = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        for (int i = 0; i < Cfg::NA; ++i) tma_prefetch_desc(&maps.a[i]);
        for (int i = 0; i < (Cfg::COLSPLIT ? 1 : Cfg::NB); ++i) tma_prefetch_desc(&maps.b[i]);
    }
    if (warp == 1) {
        tmem_alloc_pair(&s.tmem_base, Cfg::TMEM_COLS);
        tmem_relinquish_pair();
    }
    tc_fence_before();
    __syncthreads();
    // Both CTAs' barriers are initialised and the pair's TMEM allocated
    // before either CTA touches the other's.
    cluster_sync();
    tc_fence_after();
    const uint32_t tmem = s.tmem_base;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer (both CTAs)
        if (elect_one()) {
            int stage = 0;
            uint32_t phase = 0;
            bool ok = true;
            const int groups = max(p.oz_groups, 1);  // fused Ozaki slice groups per tile
            for (int t = pair; t < total && ok; t += npairs) {
                int zo, bz, tm, tn, za, zb, kb0, kb1;
                unit_coords(p, t, zo, bz, tm, tn, kb0, kb1);
                batch_operands(p, bz, za, zb);
                const int row0 = tm * Cfg::BM + static_cast<int>(rank) * Cfg::CTA_M;
                const int col0 = tn * Cfg::TILE_N + static_cast<int>(rank) * Cfg::CTA_N;
                for (int gi = 0; gi < groups && ok; ++gi) {
                int g0, g1, b_koff;
                group_range(p, gi, kb0, kb1, g0, g1, b_koff);
                for (int kb = g0; kb < g1; ++kb) {
                    if (!mbar_wait(&s.empty[stage], phase ^ 1u, p.timeout_ns, p.status, 0x01, abort)) {
                        ok = false;
                        break;
                    }
                    if (leader) mbar_arrive_expect_tx(&s.full[stage], 2 * Cfg::STAGE_BYTES);
                    const uint32_t fb = mapa_shared(smem_u32(&s.full[stage]), 0);
                    const int kx = kb * Cfg::BK;
                    const int kbx = (kb + b_koff) * Cfg::BK;
                    for (int i = 0; i < Cfg::NA; ++i) {
                        if (p.a_rank3)
                            tma_load_3d_pair(s.a[stage][i], &maps.a[i], kx, row0, za, fb);
                        else
                            tma_load_2d_pair(s.a[stage][i], &maps.a[i], kx, row0, fb);
                    }
                    for (int i = 0; i < Cfg::NB; ++i) {
#pragma unroll
                        for (int c = 0; c < Cfg::B_CHUNKS; ++c) {
                            uint8_t* dst = s.b[stage][i] + c * Cfg::B_CHUNK_BYTES;
                            // column split: every B operand is a column range of map 0
                            const int nx = col0 + (Cfg::COLSPLIT ? i * Cfg::BN : 0) + c * Cfg::B_CHUNK_ELEMS;
                            const CUtensorMap* mb = &maps.b[Cfg::COLSPLIT ? 0 : i];
                            if (p.b_rank3)
                                tma_load_3d_pair(dst, mb, nx, kbx, zb, fb);
                            else
                                tma_load_2d_pair(dst, mb, nx, kbx, fb);
                        }
                    }
                    if (++stage == Cfg::STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                }
            }
            if (ok) {
                // Wait until the leader's MMAs released every stage, so no
                // commit still targets this CTA's barriers when it exits.
                for (int i = 0; i < Cfg::STAGES && ok; ++i) {
                    ok = mbar_wait(&s.empty[stage], phase ^ 1u, p.timeout_ns, p.status, 0x02, abort);
                    if (++stage == Cfg::STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
            }
            if (!ok) settle_ns(2000000);  // 2 ms: in-flight loads land
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer (leader)
        if (leader && elect_one()) {
            int stage = 0;
            uint32_t phase = 0;
            int it = 0;
            bool ok = true;
            const int groups = max(p.oz_groups, 1);
            for (int t = pair; t < total && ok; t += npairs) {
                int zo, bz, tm, tn, kb0, kb1;
                unit_coords(p, t, zo, bz, tm, tn, kb0, kb1);
                for (int gi = 0; gi < groups && ok; ++gi) {
                int g0, g1, b_koff;
                group_range(p, gi, kb0, kb1, g0, g1, b_koff);
                const int kchunk = (Cfg::CHUNKED && p.kchunk > 0) ? p.kchunk : g1 - g0;
                for (int kc0 = g0; kc0 < g1 && ok; kc0 += kchunk, ++it) {
                    const int kc1 = min(g1, kc0 + kchunk);
                    const int buf = it % Cfg::ACC_BUFS;
                    const uint32_t acc_par = static_cast<uint32_t>((it / Cfg::ACC_BUFS) & 1);
                    if (!mbar_wait(&s.acc_empty[buf], acc_par ^ 1u, p.timeout_ns, p.status, 0x11, abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t acc_base = tmem + buf * Cfg::ACC_COLS;
                    for (int kb = kc0; kb < kc1; ++kb) {
                        if (!mbar_wait(&s.full[stage], phase, p.timeout_ns, p.status, 0x12, abort)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
#pragma unroll
                        for (int o = 0; o < Cfg::NOPS; ++o) {
                            const TcOp op = p.ops[o];
                            bool first_for_acc = true;
#pragma unroll
                            for (int q = 0; q < o; ++q)
                                if (p.ops[q].acc == op.acc) first_for_acc = false;
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
                                    tc_mma_pair_i8(acc_base + op.acc * Cfg::BN, ad, bd, idesc, acc);
                                else
                                    tc_mma_pair_f16(acc_base + op.acc * Cfg::BN, ad, bd, idesc, acc);
                            }
                        }
                        tc_commit_pair_mc(&s.empty[stage], 0x3);
                        if (++stage == Cfg::STAGES) {
                            stage = 0;
                            phase ^= 1u;
                        }
                    }
                    if (!ok) break;
                    tc_commit_pair_mc(&s.acc_full[buf], 0x3);
                }
                }
            }
            tc_commit_pair(&s.drain);
            volatile int never = 0;
            mbar_wait(&s.drain, 0, p.timeout_ns, ok ? p.status : nullptr, 0x13, &never);
        }
    } else {
        // ------------------------------------------------ epilogue (both CTAs)
        const int ew = warp & 3;
        int it = 0;
        bool ok = true;
        for (int t = pair; t < total && ok; t += npairs) {
            int zo, bz, tm, tn, kb0, kb1;
            unit_coords(p, t, zo, bz, tm, tn, kb0, kb1);
            const int grow = tm * Cfg::BM + static_cast<int>(rank) * Cfg::CTA_M + ew * 32 + lane;
            if constexpr (Cfg::CHUNKED) {
                const int kchunk = p.kchunk > 0 ? p.kchunk : kb1 - kb0;
                float run[Cfg::BN];
#pragma unroll
                for (int j = 0; j < Cfg::BN; ++j) run[j] = 0.f;
                for (int kc0 = kb0; kc0 < kb1; kc0 += kchunk, ++it) {
                    const int buf = it % Cfg::ACC_BUFS;
                    const uint32_t acc_par = static_cast<uint32_t>((it / Cfg::ACC_BUFS) & 1);
                    if (!mbar_wait(&s.acc_full[buf], acc_par, p.timeout_ns, p.status, 0x21, abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t row_addr =
                        tmem + (static_cast<uint32_t>(ew * 32) << 16) + buf * Cfg::ACC_COLS;
#pragma unroll
                    for (int c = 0; c < Cfg::BN / 32; ++c) {
#pragma unroll
                        for (int q = Cfg::NACC - 1; q >= 0; --q) {
                            uint32_t v[32];
                            tmem_ld_32x32b_x32(row_addr + q * Cfg::BN + c * 32, v);
                            tmem_wait_ld();
#pragma unroll
                            for (int j = 0; j < 32; ++j)
                                run[c * 32 + j] = __fadd_rn(run[c * 32 + j], __uint_as_float(v[j]));
                        }
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive_cluster(mapa_shared(smem_u32(&s.acc_empty[buf]), 0));
                }
                if (!ok) break;
#pragma unroll
                for (int c = 0; c < Cfg::BN / 32; ++c) {
                    uint32_t v[Cfg::NACC][32];
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[0][j] = __float_as_uint(run[c * 32 + j]);
                    epilogue_store<Cfg>(p, zo, grow, tn * Cfg::BN + c * 32, v);
                }
            } else {
                for (int gi = 0; gi < max(p.oz_groups, 1); ++gi) {
                const int buf = it % Cfg::ACC_BUFS;
                const uint32_t acc_par = static_cast<uint32_t>((it / Cfg::ACC_BUFS) & 1);
                ++it;
                if (!mbar_wait(&s.acc_full[buf], acc_par, p.timeout_ns, p.status, 0x21, abort)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t row_addr =
                    tmem + (static_cast<uint32_t>(ew * 32) << 16) + buf * Cfg::ACC_COLS;
                if constexpr (Cfg::COLSPLIT) {
                    // accumulator a holds tile columns [a BN, (a + 1) BN)
                    for (int a = 0; a < Cfg::NACC; ++a) {
#pragma unroll 1
                        for (int c = 0; c < Cfg::BN / 32; ++c) {
                            uint32_t v[1][32];
                            tmem_ld_32x32b_x32(row_addr + a * Cfg::BN + c * 32, v[0]);
                            tmem_wait_ld();
                            epilogue_store<Tc2EpiView<Cfg>>(p, zo, grow, tn * Cfg::TILE_N + a * Cfg::BN + c * 32, v);
                        }
                    }
                } else {
#pragma unroll 1
                    for (int c = 0; c < Cfg::BN / 32; ++c) {
                        uint32_t v[Cfg::NACC][32];
#pragma unroll
                        for (int a = 0; a < Cfg::NACC; ++a) tmem_ld_32x32b_x32(row_addr + a * Cfg::BN + c * 32, v[a]);
                        tmem_wait_ld();
                        epilogue_store<Cfg>(p, zo, grow, tn * Cfg::BN + c * 32, v, gi);
                    }
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive_cluster(mapa_shared(smem_u32(&s.acc_empty[buf]), 0));
                }
            }
        }
    }

    tc_fence_before();
    __syncthreads();
    cluster_sync();  // neither CTA frees TMEM or exits while the pair still works
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc_pair(tmem, Cfg::TMEM_COLS);
    }
}

}  // namespace fg
