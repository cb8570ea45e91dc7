// tc_gemm.cuh -- persistent, warp-specialised tcgen05 GEMM for sm_100a.
//
// One CTA per SM walks a strided list of output tiles (BM=128 rows x BN
// columns).  Warp roles:
//   warp 0      TMA producer: loads the operand tiles of one K block
//               (128 bytes of K) into a ring of shared-memory stages;
//   warp 1      TMEM owner + MMA issuer: one elected thread issues
//               tcgen05.mma for every (A tile, B tile, accumulator) product
//               of the stage, then tcgen05.commit frees the stage;
//   warps 2-5   epilogue: tcgen05.ld the accumulators of a finished tile
//               (one TMEM lane = one output row per thread), combine them
//               (wrapping i32, i16 byte-slice recombination, alpha/beta,
//               quantized zero-point correction, complex interleave) and
//               store to global memory.
// Accumulators live in TMEM and are double-buffered when they fit in the 512
// columns, so the epilogue of tile t overlaps the MMAs of tile t+1.
//
// A is K-major (row-major M x K in global memory), B is MN-major (row-major
// K x N): both are read straight from the user's layout, 128-byte swizzled by
// TMA, with no transpose pass.
//
// A "scheme" describes which operand tiles a K block loads and which
// products accumulate where:
//   plain i8/u8   1 A x 1 B -> 1 accumulator;
//   i16           A = hi(s8)*256 + lo(u8), B likewise: 4 products into
//                 3 accumulators (hh, hl+lh, ll), recombined mod 2^32;
//   split bf16    A = hi + lo, B = hi + lo (bf16): lo*hi + hi*lo + hi*hi
//                 into one f32 accumulator (the 3xBF16 SGEMM).
#pragma once
#include "fg_device.cuh"

namespace fg {

enum : int { KIND_I8 = 0, KIND_BF16 = 1 };
enum : int { EPI_I32 = 0, EPI_I16 = 1, EPI_F32 = 2, EPI_QMM = 3, EPI_OZAKI = 4, EPI_CRT = 5 };

constexpr int TC_MAX_OPS = 8;
constexpr int TC_MAX_OPERANDS = 4;

struct TcOp {
    int a, b, acc;
    int a_fmt, b_fmt;  // kind::i8: 0 = u8, 1 = s8; kind::f16: 1 = bf16
};

template <int KIND_, int BN_, int STAGES_, int NA_, int NB_, int NACC_, int NOPS_, int EPI_,
          int CHUNKED_ = 0>
struct TcCfg {
    static constexpr int KIND = KIND_, BM = 128, BN = BN_, STAGES = STAGES_;
    // CHUNKED: K is accumulated in TMEM in chunks of p.kchunk blocks that the
    // epilogue sums in FP32 registers (EPI_F32 only), adding all NACC
    // accumulators of the chunk (the MMA unit rounds its FP32 accumulator
    // toward zero at every instruction, so short chunks and a separate
    // accumulator for the small correction products keep that error below
    // FFMA's).
    static constexpr int CHUNKED = CHUNKED_;
    static constexpr int NA = NA_, NB = NB_, NACC = NACC_, NOPS = NOPS_, EPI = EPI_;
    static constexpr int ESIZE = KIND == KIND_I8 ? 1 : 2;  // operand bytes
    static constexpr int BK_BYTES = 128;
    static constexpr int BK = BK_BYTES / ESIZE;             // K elements per block
    static constexpr int KSTEP_BYTES = 32;                  // one MMA: 256 bits of K
    static constexpr int KSTEPS = BK_BYTES / KSTEP_BYTES;   // MMAs per tile product
    static constexpr int A_TILE = BM * BK_BYTES;            // bytes
    static constexpr int B_TILE = BN * BK_BYTES;
    static constexpr int B_CHUNK_ELEMS = 128 / ESIZE;       // N elements per TMA box
    static constexpr int B_CHUNKS = BN / B_CHUNK_ELEMS;
    static constexpr int B_CHUNK_BYTES = BK * 128;
    static constexpr int STAGE_BYTES = NA * A_TILE + NB * B_TILE;
    static constexpr int ACC_COLS = NACC * BN;
    static constexpr int ACC_BUFS = (4 * ACC_COLS <= 512) ? 4 : (2 * ACC_COLS <= 512) ? 2 : 1;
    static constexpr int TMEM_COLS = 512;
    static constexpr int THREADS = 192;
    static_assert(ACC_COLS <= 512, "accumulators exceed TMEM");
    static_assert(BN % 16 == 0 && BN <= 256, "UMMA N");
    static_assert(BN % B_CHUNK_ELEMS == 0, "B tile must be whole 128-byte chunks");
};

struct TcMaps {
    CUtensorMap a[TC_MAX_OPERANDS];
    CUtensorMap b[TC_MAX_OPERANDS];
};

struct TcArgs {
    int M, N, K;
    int tiles_m, tiles_n, k_blocks;
    int batch;                 // number of output matrices
    int a_rank3, b_rank3;      // 1 when the operand map is 3-D (batched)
    // NumPy-style broadcast: output batch index -> operand matrix index.
    int bdims;                 // number of batch dims (<= 4)
    int bshape[4];             // output batch shape
    long long a_bstride[4];    // operand matrix index strides (0 = broadcast)
    long long b_bstride[4];
    void* C;
    long long ldc, strideC;    // elements
    int accumulate;            // integer epilogues: add into C
    float alpha, beta;         // EPI_F32 (beta == 0: C is not read)
    // EPI_F32, FP16 split: max |A| and max |B| as float bits; the products
    // were formed from A 2^sA and B 2^sB (f16_scale_exp), so the epilogue
    // multiplies by 2^-sA 2^-sB.  Null: no scaling.
    const unsigned* f16_amax;
    int cplx_half;             // EPI_F32: >0 writes column j<h as Re, j>=h as Im
    // EPI_QMM
    const int* row_sum;
    const int* col_sum;
    int a_zp, b_zp;
    float scale;
    int kchunk;                // CHUNKED configs: K blocks per TMEM chunk
    // split-K: work unit t covers K blocks [s*kb_per_split, (s+1)*kb_per_split)
    // of one tile, s = t / (batch*tiles); its partial result goes to output
    // matrix s*batch + bz.  splits <= 1: no split (zero-initialised args).
    int splits, kb_per_split;
    int raster;                // row tiles per raster group (0: 8)
    // EPI_OZAKI: C (f64) (+)= oz_w * 2^(e_i + f_j) * acc; the first group of a
    // call applies C = oz_beta * C first.  cplx_half > 0 interleaves complex.
    const double* row_scale;
    const double* col_scale;
    double oz_w, oz_beta;
    int oz_first;
    // EPI_OZAKI, all slice groups in one launch (oz_groups > 0): every tile
    // runs groups d = oz_d0, oz_d0 - 1, ... (oz_groups of them) back to back
    // in this CTA, group d reading K blocks [0, (d-1) oz_kc_blocks) of A and
    // B from K block (oz_S - d + 1) oz_kc_blocks on, with weight
    // oz_w 2^(-7d); only the first group applies oz_beta.  The tile's C block
    // stays in L2 between its groups.
    int oz_groups, oz_d0, oz_kc_blocks, oz_S;
    // EPI_CRT (Ozaki scheme II): group gi is the product of residue planes gi
    // (A K blocks [gi oz_kc_blocks, (gi + 1) oz_kc_blocks), B rows the same),
    // written as the byte ((acc mod m) y) mod m, m = crt_m[gi], y = crt_y[gi],
    // into plane gi of C (planes crt_plane bytes apart, row pitch ldc).
    int oz_crt;
    int crt_m[24], crt_y[24];
    long long crt_plane;
    TcOp ops[TC_MAX_OPS];
    DevStatus* status;
    unsigned long long timeout_ns;
};

__device__ __forceinline__ void tile_coords(const TcArgs& p, int t, int& bz, int& tm, int& tn) {
    const int per_batch = p.tiles_m * p.tiles_n;
    bz = t / per_batch;
    int r = t - bz * per_batch;
    // Grouped raster: `raster` (default 8) row-tiles share each sweep over
    // the column tiles so the A rows and B columns of concurrently running
    // tiles stay in L2.
    const int GROUP = p.raster > 0 ? p.raster : 8;
    int per_group = GROUP * p.tiles_n;
    int g = r / per_group;
    int first_m = g * GROUP;
    int gm = min(p.tiles_m - first_m, GROUP);
    int q = r - g * per_group;
    tm = first_m + q % gm;
    tn = q / gm;
}

// Work unit t -> output matrix index, batch index, tile and K-block range.
__device__ __forceinline__ void unit_coords(const TcArgs& p, int t, int& zo, int& bz, int& tm,
                                            int& tn, int& kb0, int& kb1) {
    if (p.splits > 1) {
        const int per_split = p.batch * p.tiles_m * p.tiles_n;
        const int s = t / per_split;
        tile_coords(p, t - s * per_split, bz, tm, tn);
        zo = s * p.batch + bz;
        kb0 = s * p.kb_per_split;
        kb1 = min(p.k_blocks, kb0 + p.kb_per_split);
    } else {
        tile_coords(p, t, bz, tm, tn);
        zo = bz;
        kb0 = 0;
        kb1 = p.k_blocks;
    }
}

// Sub-unit `gi` of a tile: its K-block range and the K offset of its B rows.
// Without fused Ozaki groups a tile has one sub-unit, the given range.
__device__ __forceinline__ void group_range(const TcArgs& p, int gi, int kb0, int kb1, int& g0, int& g1,
                                            int& b_koff) {
    if (p.oz_crt) {
        g0 = gi * p.oz_kc_blocks;
        g1 = g0 + p.oz_kc_blocks;
        b_koff = 0;
    } else if (p.oz_groups > 0) {
        const int d = p.oz_d0 - gi;
        g0 = 0;
        g1 = (d - 1) * p.oz_kc_blocks;
        b_koff = (p.oz_S - d + 1) * p.oz_kc_blocks;
    } else {
        g0 = kb0;
        g1 = kb1;
        b_koff = 0;
    }
}

__device__ __forceinline__ void batch_operands(const TcArgs& p, int bz, int& za, int& zb) {
    long long ia = 0, ib = 0;
    int rem = bz;
    for (int d = p.bdims - 1; d >= 0; --d) {
        int idx = rem % p.bshape[d];
        rem /= p.bshape[d];
        ia += idx * p.a_bstride[d];
        ib += idx * p.b_bstride[d];
    }
    za = static_cast<int>(ia);
    zb = static_cast<int>(ib);
}

template <class Cfg>
struct TcSmem {
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
__device__ __forceinline__ void epilogue_store(const TcArgs& p, int bz, int grow, int gcol0,
                                               const uint32_t (&v)[Cfg::NACC][32], int oz_grp = 0) {
    const uint32_t (&v_)[Cfg::NACC][32] = v;
    if (grow >= p.M) return;
    const int ncols = min(32, p.N - gcol0);
    if (ncols <= 0) return;
    if constexpr (Cfg::EPI == EPI_I32 || Cfg::EPI == EPI_I16) {
        int32_t* crow = static_cast<int32_t*>(p.C) + bz * p.strideC + (long long)grow * p.ldc + gcol0;
        uint32_t out[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            if constexpr (Cfg::EPI == EPI_I32) {
                out[j] = v[0][j];
            } else {
                out[j] = (v[0][j] << 16) + (v[1][j] << 8) + v[2][j];
            }
        }
        const bool vec = ncols == 32 && (reinterpret_cast<uintptr_t>(crow) & 15) == 0;
        if (vec) {
            if (p.accumulate) {
                // all loads before the first store: they overlap instead of
                // waiting behind stores that might alias them
                uint4 o[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) o[q] = *reinterpret_cast<const uint4*>(crow + 4 * q);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    out[4 * q] += o[q].x; out[4 * q + 1] += o[q].y;
                    out[4 * q + 2] += o[q].z; out[4 * q + 3] += o[q].w;
                }
            }
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                *reinterpret_cast<uint4*>(crow + j) = make_uint4(out[j], out[j + 1], out[j + 2], out[j + 3]);
        } else {
            // fully unrolled with a predicate: a runtime trip count would
            // index `out` dynamically and move it to local memory
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                if (j < ncols) {
                    uint32_t w = out[j];
                    if (p.accumulate) w += static_cast<uint32_t>(crow[j]);
                    crow[j] = static_cast<int32_t>(w);
                }
            }
        }
    } else if constexpr (Cfg::EPI == EPI_QMM) {
        float* crow = static_cast<float*>(p.C) + bz * p.strideC + (long long)grow * p.ldc + gcol0;
        const uint32_t rs = static_cast<uint32_t>(p.row_sum[grow]);
        const uint32_t azp = static_cast<uint32_t>(p.a_zp), bzp = static_cast<uint32_t>(p.b_zp);
        const uint32_t kab = static_cast<uint32_t>(p.K) * azp * bzp;
        // every load of the chunk is issued before the first store (stores
        // to C could alias the sums, which would serialise load -> store)
        uint32_t cs[32];
        float old[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            cs[j] = j < ncols ? static_cast<uint32_t>(p.col_sum[gcol0 + j]) : 0u;
            old[j] = (p.accumulate && j < ncols) ? crow[j] : 0.f;
        }
        float out[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            const uint32_t corr = v[0][j] - azp * cs[j] - bzp * rs + kab;
            // Separate roundings, as gemm/mod.rs:566-571 computes them (no FMA).
            float o = __fmul_rn(p.scale, static_cast<float>(static_cast<int32_t>(corr)));
            if (p.accumulate) o = __fadd_rn(old[j], o);
            out[j] = o;
        }
        if (ncols == 32 && (reinterpret_cast<uintptr_t>(crow) & 15) == 0) {
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                *reinterpret_cast<float4*>(crow + j) = make_float4(out[j], out[j + 1], out[j + 2], out[j + 3]);
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (j < ncols) crow[j] = out[j];
        }
    } else if constexpr (Cfg::EPI == EPI_CRT) {
        // exact int32 product of two residue planes -> its CRT residue byte
        const int m = p.crt_m[oz_grp], y = p.crt_y[oz_grp];
        uint8_t* crow = static_cast<uint8_t*>(p.C) + oz_grp * p.crt_plane + (long long)grow * p.ldc + gcol0;
        uint32_t pk[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) pk[q] = 0;
#pragma unroll
        for (int j = 0; j < 32; ++j) {
            int r = static_cast<int32_t>(v[0][j]) % m;
            r += r < 0 ? m : 0;
            r = (r * y) % m;
            pk[j / 4] |= static_cast<uint32_t>(r) << (8 * (j % 4));
        }
        if (ncols == 32 && (reinterpret_cast<uintptr_t>(crow) & 15) == 0) {
            *reinterpret_cast<uint4*>(crow) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
            *reinterpret_cast<uint4*>(crow + 16) = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j)
                if (j < ncols) crow[j] = static_cast<uint8_t>(pk[j / 4] >> (8 * (j % 4)));
        }
    } else if constexpr (Cfg::EPI == EPI_OZAKI) {
        double* cbase = static_cast<double*>(p.C) + bz * p.strideC;
        // fused groups: weight oz_w 2^(-7d) of group d = oz_d0 - oz_grp (exact)
        const double w = p.oz_groups > 0 ? ldexp(p.oz_w, -7 * (p.oz_d0 - oz_grp)) : p.oz_w;
        const bool first = p.oz_first && oz_grp == 0;
        const double rs = p.row_scale[grow] * w;
        const int h = p.cplx_half;
        const bool need_old = !first || p.oz_beta != 0.0;
        double* crow = cbase + (long long)grow * p.ldc;
        const bool vec = h == 0 && ncols == 32 && ((reinterpret_cast<uintptr_t>(crow + gcol0) & 15) == 0);
        // Two halves of 16 columns; in each, all loads (scales, old C) are
        // issued before the stores so they overlap instead of serialising.
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int j0 = half * 16;
            double cs[16], old[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                const int j = j0 + u;
                const int col = gcol0 + j;
                const int cc = (h > 0 && col >= h) ? col - h : col;
                cs[u] = j < ncols ? p.col_scale[cc] : 0.0;
            }
            if (vec) {
                if (need_old) {
#pragma unroll
                    for (int u = 0; u < 16; u += 2) {
                        const double2 w = *reinterpret_cast<const double2*>(crow + gcol0 + j0 + u);
                        old[u] = w.x;
                        old[u + 1] = w.y;
                    }
                } else {
#pragma unroll
                    for (int u = 0; u < 16; ++u) old[u] = 0.0;
                }
            } else {
#pragma unroll
                for (int u = 0; u < 16; ++u) {
                    const int j = j0 + u;
                    const int col = gcol0 + j;
                    const int cc = (h > 0 && col >= h) ? col - h : col;
                    const double* src = h > 0 ? crow + 2 * cc + (col < h ? 0 : 1) : crow + col;
                    old[u] = (need_old && j < ncols) ? *src : 0.0;
                }
            }
            double out[16];
#pragma unroll
            for (int u = 0; u < 16; ++u) {
                // exact int32 -> f64, then power-of-two scalings (exact) and alpha
                const double t = static_cast<double>(static_cast<int32_t>(v_[0][j0 + u])) * cs[u] * rs;
                out[u] = first ? (p.oz_beta != 0.0 ? fma(p.oz_beta, old[u], t) : t) : old[u] + t;
            }
            if (vec) {
#pragma unroll
                for (int u = 0; u < 16; u += 2)
                    *reinterpret_cast<double2*>(crow + gcol0 + j0 + u) = make_double2(out[u], out[u + 1]);
            } else {
#pragma unroll
                for (int u = 0; u < 16; ++u) {
                    const int j = j0 + u;
                    if (j < ncols) {
                        const int col = gcol0 + j;
                        const int cc = (h > 0 && col >= h) ? col - h : col;
                        double* dst = h > 0 ? crow + 2 * cc + (col < h ? 0 : 1) : crow + col;
                        *dst = out[u];
                    }
                }
            }
        }
    } else {  // EPI_F32
        float* cbase = static_cast<float*>(p.C) + bz * p.strideC;
        // the FP16 split's operand scaling, undone (exact powers of two)
        const int unscale = p.f16_amax ? -(f16_scale_exp(p.f16_amax[0]) + f16_scale_exp(p.f16_amax[1])) : 0;
        if (p.cplx_half > 0) {
            // Column j of the real-embedded product is Re (j < h) or Im (j >= h)
            // of complex column j mod h; C is interleaved (re, im).
            const int h = p.cplx_half;
            float* crow = cbase + (long long)grow * p.ldc;
            float old[32];
#pragma unroll
            for (int j = 0; j < 32; ++j) {  // loads first, then stores
                const int col = gcol0 + j;
                const int cc = col < h ? col : col - h;
                old[j] = (p.beta != 0.f && j < ncols) ? crow[2 * cc + (col < h ? 0 : 1)] : 0.f;
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                if (j < ncols) {
                    const int col = gcol0 + j;
                    const int cc = col < h ? col : col - h;
                    float acc = __uint_as_float(v[0][j]);
                    if (unscale) acc = mul_pow2(acc, unscale);
                    float o = p.alpha * acc;
                    if (p.beta != 0.f) o = fmaf(p.beta, old[j], o);
                    crow[2 * cc + (col < h ? 0 : 1)] = o;
                }
            }
            return;
        }
        float* crow = cbase + (long long)grow * p.ldc + gcol0;
        float out[32];
#pragma unroll
        for (int j = 0; j < 32; ++j) out[j] = p.alpha * __uint_as_float(v[0][j]);
        if (unscale) {
#pragma unroll
            for (int j = 0; j < 32; ++j) out[j] = p.alpha * mul_pow2(__uint_as_float(v[0][j]), unscale);
        }
        const bool vec = ncols == 32 && (reinterpret_cast<uintptr_t>(crow) & 15) == 0;
        if (vec) {
            if (p.beta != 0.f) {
                float4 o[8];
#pragma unroll
                for (int q = 0; q < 8; ++q) o[q] = *reinterpret_cast<const float4*>(crow + 4 * q);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    out[4 * q] = fmaf(p.beta, o[q].x, out[4 * q]);
                    out[4 * q + 1] = fmaf(p.beta, o[q].y, out[4 * q + 1]);
                    out[4 * q + 2] = fmaf(p.beta, o[q].z, out[4 * q + 2]);
                    out[4 * q + 3] = fmaf(p.beta, o[q].w, out[4 * q + 3]);
                }
            }
#pragma unroll
            for (int j = 0; j < 32; j += 4)
                *reinterpret_cast<float4*>(crow + j) = make_float4(out[j], out[j + 1], out[j + 2], out[j + 3]);
        } else {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                if (j < ncols) {
                    float o = out[j];
                    if (p.beta != 0.f) o = fmaf(p.beta, crow[j], o);
                    crow[j] = o;
                }
            }
        }
    }
}

template <class Cfg>
__global__ void __launch_bounds__(Cfg::THREADS, 1)
    tc_gemm_kernel(const __grid_constant__ TcMaps maps, const __grid_constant__ TcArgs p) {
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    // The dynamic shared window is only guaranteed 16-byte aligned: round up
    // to the 1024-byte alignment the 128-byte swizzle atoms need (the launch
    // reserves the extra kilobyte).
    uint8_t* base = reinterpret_cast<uint8_t*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~static_cast<uintptr_t>(1023));
    TcSmem<Cfg>& s = *reinterpret_cast<TcSmem<Cfg>*>(base);

    const int warp = threadIdx.x / 32;
    const int lane = threadIdx.x % 32;
    const int total_tiles = max(p.splits, 1) * p.batch * p.tiles_m * p.tiles_n;
    volatile int* abort = &s.abort;

    if (threadIdx.x == 0) {
        for (int i = 0; i < Cfg::STAGES; ++i) {
            mbar_init(&s.full[i], 1);
            mbar_init(&s.empty[i], 1);
        }
        for (int i = 0; i < 4; ++i) {
            mbar_init(&s.acc_full[i], 1);
            mbar_init(&s.acc_empty[i], 4);  // one arrive per epilogue warp
        }
        mbar_init(&s.drain, 1);
        s.abort = 0;
        fence_mbar_init();
    }
    if (warp == 0 && lane == 0) {
        for (int i = 0; i < Cfg::NA; ++i) tma_prefetch_desc(&maps.a[i]);
        for (int i = 0; i < Cfg::NB; ++i) tma_prefetch_desc(&maps.b[i]);
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
        // ------------------------------------------------ TMA producer
        if (elect_one()) {
            int stage = 0;
            uint32_t phase = 0;
            // per stage: bit = a load was issued, bit = its phase parity
            // (register bitmasks; an indexed array would live in local memory)
            uint32_t issued_mask = 0, issued_par = 0;
            bool ok = true;
            const int groups = max(p.oz_groups, 1);
            for (int t = blockIdx.x; t < total_tiles && ok; t += gridDim.x) {
                int zo, bz, tm, tn, za, zb, kb0, kb1;
                unit_coords(p, t, zo, bz, tm, tn, kb0, kb1);
                batch_operands(p, bz, za, zb);
                for (int gi = 0; gi < groups && ok; ++gi) {
                int g0, g1, b_koff;
                group_range(p, gi, kb0, kb1, g0, g1, b_koff);
                for (int kb = g0; kb < g1; ++kb) {
                    if (!mbar_wait(&s.empty[stage], phase ^ 1u, p.timeout_ns, p.status, 0x01,
                                   abort)) {
                        ok = false;
                        break;
                    }
                    mbar_arrive_expect_tx(&s.full[stage], Cfg::STAGE_BYTES);
                    const int kx = kb * Cfg::BK;
                    const int kbx = (kb + b_koff) * Cfg::BK;
                    for (int i = 0; i < Cfg::NA; ++i) {
                        if (p.a_rank3)
                            tma_load_3d(s.a[stage][i], &maps.a[i], kx, tm * Cfg::BM, za, &s.full[stage]);
                        else
                            tma_load_2d(s.a[stage][i], &maps.a[i], kx, tm * Cfg::BM, &s.full[stage]);
                    }
                    for (int i = 0; i < Cfg::NB; ++i) {
#pragma unroll
                        for (int c = 0; c < Cfg::B_CHUNKS; ++c) {
                            uint8_t* dst = s.b[stage][i] + c * Cfg::B_CHUNK_BYTES;
                            const int nx = tn * Cfg::BN + c * Cfg::B_CHUNK_ELEMS;
                            if (p.b_rank3)
                                tma_load_3d(dst, &maps.b[i], nx, kbx, zb, &s.full[stage]);
                            else
                                tma_load_2d(dst, &maps.b[i], nx, kbx, &s.full[stage]);
                        }
                    }
                    issued_mask |= 1u << stage;
                    issued_par = (issued_par & ~(1u << stage)) | (phase << stage);
                    if (++stage == Cfg::STAGES) {
                        stage = 0;
                        phase ^= 1u;
                    }
                }
                }
            }
            if (!ok) {
                // Let every load this thread issued land before the CTA exits.
                for (int i = 0; i < Cfg::STAGES; ++i) {
                    if (!((issued_mask >> i) & 1u)) continue;
                    volatile int never = 0;
                    mbar_wait(&s.full[i], (issued_par >> i) & 1u, p.timeout_ns, nullptr, 0, &never);
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer
        if (elect_one()) {
            int stage = 0;
            uint32_t phase = 0;
            int it = 0;  // accumulator units (tile x K chunk) issued so far
            bool ok = true;
            const int groups = max(p.oz_groups, 1);
            for (int t = blockIdx.x; t < total_tiles && ok; t += gridDim.x) {
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
                            // first product into this accumulator in the unit?
                            bool first_for_acc = true;
#pragma unroll
                            for (int q = 0; q < o; ++q)
                                if (p.ops[q].acc == op.acc) first_for_acc = false;
                            const uint32_t idesc = umma_idesc(Cfg::KIND == KIND_I8 ? 2u : 1u,
                                                              op.a_fmt, op.b_fmt, 0u, 1u, Cfg::BM, Cfg::BN);
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
            }
            // Every MMA issued above has completed once `drain` flips.
            tc_commit(&s.drain);
            volatile int never = 0;
            mbar_wait(&s.drain, 0, p.timeout_ns, ok ? p.status : nullptr, 0x13, &never);
        }
    } else {
        // ------------------------------------------------ epilogue
        const int ew = warp & 3;  // TMEM lane quarter this warp may access
        int it = 0;
        if constexpr (Cfg::CHUNKED) {
            // Tensor-core FP32 accumulation truncates at every MMA, so long K
            // runs drift.  Each K chunk is accumulated in TMEM from zero and
            // the chunk sums are added here in FP32 registers with
            // round-to-nearest.
            bool ok = true;
            for (int t = blockIdx.x; t < total_tiles && ok; t += gridDim.x) {
                int zo, bz, tm, tn, kb0, kb1;
                unit_coords(p, t, zo, bz, tm, tn, kb0, kb1);
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
                        // accumulators are summed smallest first: the last
                        // (correction products) before acc 0 (hi * hi)
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
                    if (lane == 0) mbar_arrive(&s.acc_empty[buf]);
                }
                if (!ok) break;
                const int grow = tm * Cfg::BM + ew * 32 + lane;
#pragma unroll
                for (int c = 0; c < Cfg::BN / 32; ++c) {
                    uint32_t v[Cfg::NACC][32];
#pragma unroll
                    for (int j = 0; j < 32; ++j) v[0][j] = __float_as_uint(run[c * 32 + j]);
                    epilogue_store<Cfg>(p, zo, grow, tn * Cfg::BN + c * 32, v);
                }
            }
        } else {
            const int groups = max(p.oz_groups, 1);
            bool ok = true;
            for (int t = blockIdx.x; t < total_tiles && ok; t += gridDim.x) {
                for (int gi = 0; gi < groups; ++gi, ++it) {
                const int buf = it % Cfg::ACC_BUFS;
                const uint32_t acc_par = static_cast<uint32_t>((it / Cfg::ACC_BUFS) & 1);
                if (!mbar_wait(&s.acc_full[buf], acc_par, p.timeout_ns, p.status, 0x21, abort)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                int zo, bz, tm, tn, kb0, kb1;
                unit_coords(p, t, zo, bz, tm, tn, kb0, kb1);
                const int grow = tm * Cfg::BM + ew * 32 + lane;
                const uint32_t row_addr = tmem + (static_cast<uint32_t>(ew * 32) << 16) + buf * Cfg::ACC_COLS;
#pragma unroll 1
                for (int c = 0; c < Cfg::BN / 32; ++c) {
                    uint32_t v[Cfg::NACC][32];
#pragma unroll
                    for (int a = 0; a < Cfg::NACC; ++a) tmem_ld_32x32b_x32(row_addr + a * Cfg::BN + c * 32, v[a]);
                    tmem_wait_ld();
                    epilogue_store<Cfg>(p, zo, grow, tn * Cfg::BN + c * 32, v, gi);
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&s.acc_empty[buf]);
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

template <class Cfg>
constexpr size_t tc_smem_bytes() {
    return sizeof(TcSmem<Cfg>) + 1024;
}

}  // namespace fg
