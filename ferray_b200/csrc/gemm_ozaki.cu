// gemm_ozaki.cu -- split-mode DGEMM / ZGEMM: INT8 Ozaki slicing on the
// integer tensor cores (method and layouts in ozaki_kernels.cuh).
//
// Per call: row/column exponent scan (FP64), slice extraction into int8
// digit planes (FP64 -> int8), then for each K chunk and each slice group
// d = S+1 .. 2 (smallest weight first) ONE tcgen05 kind::i8 GEMM over the
// concatenated K of that group, whose epilogue adds 2^-7d * 2^(e_i+f_j) * G_d
// into C in FP64.  Every group sum G_d = sum_{s+t=d} A_s B_t is exact in
// int32: at most S products of K_chunk * 127^2, with K_chunk chosen so that
// S * K_chunk * 127^2 < 2^31.
#include <algorithm>
#include <cstdlib>
#include <mutex>
#include <vector>

#include "ozaki_kernels.cuh"
#include "runtime.h"
#include "tc_gemm.cuh"
#include "tc_gemm2.cuh"
#include "tune.h"

namespace fgrt {

using namespace fg;

using CfgOzaki = TcCfg<KIND_I8, 256, 4, 1, 1, 1, 1, EPI_OZAKI>;
// CTA-pair form (256 x 256 tiles), used where the tuned i8 table picks the
// pair kernel for the group's (M, N, K).
using CfgOzakiPair = Tc2Cfg<KIND_I8, 256, 6, 1, 1, 1, 1, EPI_OZAKI>;

static int grid_for(long long total) {
    return static_cast<int>(std::min<long long>(std::max<long long>((total + 255) / 256, 1), 8192));
}

static long long round_up(long long x, long long a) { return (x + a - 1) / a * a; }

// One launch for all slice groups (default); FG_OZAKI_FUSED=0 restores one
// launch per group.
static bool fused_groups() {
    static const bool v = [] {
        const char* e = getenv("FG_OZAKI_FUSED");
        return !(e && e[0] == '0');
    }();
    return v;
}

template <class Cfg>
static fg_status launch_group(fg_ctx* ctx, const TcMaps& maps, TcArgs& args, cudaStream_t st) {
    constexpr bool pair = Cfg::BM == 256;
    static std::once_flag once;
    static cudaError_t attr_err = cudaSuccess;
    static int max_units = 0;
    std::call_once(once, [ctx] {
        if constexpr (pair) {
            attr_err = cudaFuncSetAttribute(tc_gemm2_kernel<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(tc2_smem_bytes<Cfg>()));
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(static_cast<unsigned>(ctx->sm_count & ~1), 1, 1);
            cfg.blockDim = dim3(Cfg::THREADS, 1, 1);
            cfg.dynamicSmemBytes = tc2_smem_bytes<Cfg>();
            int n = 0;
            if (attr_err == cudaSuccess &&
                cudaOccupancyMaxActiveClusters(&n, tc_gemm2_kernel<Cfg>, &cfg) == cudaSuccess && n > 0)
                max_units = n;
            else
                cudaGetLastError();
            if (max_units <= 0) max_units = ctx->sm_count / 2;
        } else {
            attr_err = cudaFuncSetAttribute(tc_gemm_kernel<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            static_cast<int>(tc_smem_bytes<Cfg>()));
            max_units = ctx->sm_count;
        }
    });
    FG_CUDA(attr_err);
    args.status = ctx->d_status;
    args.timeout_ns = 4000000000ull;
    const long long tiles = (long long)args.tiles_m * args.tiles_n;
    const int units = static_cast<int>(std::min<long long>(tiles, max_units));
    ProfScope prof(pair ? "tc_gemm2_ozaki_i8" : "tc_gemm_ozaki_i8", st);
    if constexpr (pair)
        tc_gemm2_kernel<Cfg><<<2 * units, Cfg::THREADS, tc2_smem_bytes<Cfg>(), st>>>(maps, args);
    else
        tc_gemm_kernel<Cfg><<<units, Cfg::THREADS, tc_smem_bytes<Cfg>(), st>>>(maps, args);
    prof.stop();
    count_launch();
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// Balancing exponents of the inner dimension, then the row scales of A D
// and the column scales of D^-1 B (powers of two), shared by both schemes.
static fg_status scale_operands(const Gemm& g, bool cplx, double* rsc, double* csc,
                                unsigned long long* cmax, unsigned long long* kmax_a,
                                unsigned long long* kmax_b, int* shift, cudaStream_t st) {
    const double* A = static_cast<const double*>(g.A);
    const double* B = static_cast<const double*>(g.B);
    const long long M = g.M, K = g.K, N = g.N;
    const int cx = cplx ? 1 : 0;
    // column-max passes: rows per thread, 32 (more blocks in flight) unless
    // the grid's y extent (65535) needs more
    const long long rows_a = std::max<long long>(32, (M + 65534) / 65535);
    const long long rows_b = std::max<long long>(32, (K + 65534) / 65535);
    // balancing exponents of the inner dimension
    FG_CUDA(cudaMemsetAsync(kmax_a, 0, K * sizeof(unsigned long long), st));
    dim3 agrid(static_cast<unsigned>((K + 255) / 256), static_cast<unsigned>((M + rows_a - 1) / rows_a));
    ozaki_a_colmax_kernel<<<agrid, 256, 0, st>>>(A, M, K, g.lda, cx, rows_a, kmax_a);
    ozaki_b_rowmax_kernel<<<static_cast<unsigned>(std::min<long long>(K, 65535)), 256, 0, st>>>(B, K, N, g.ldb, cx, kmax_b);
    ozaki_shift_kernel<<<grid_for(K), 256, 0, st>>>(kmax_a, kmax_b, K, shift);
    // row / column scales of the balanced operands
    ozaki_row_scale_kernel<<<static_cast<unsigned>(std::min<long long>(M, 65535)), 256, 0, st>>>(A, M, K, g.lda, cx, shift, rsc);
    FG_CUDA(cudaMemsetAsync(cmax, 0, N * sizeof(unsigned long long), st));
    dim3 cgrid(static_cast<unsigned>((N + 255) / 256), static_cast<unsigned>((K + rows_b - 1) / rows_b));
    ozaki_col_max_kernel<<<cgrid, 256, 0, st>>>(B, K, N, g.ldb, cx, rows_b, shift, cmax);
    ozaki_col_scale_kernel<<<grid_for(N), 256, 0, st>>>(cmax, N, csc);
    count_launch(6);
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

template <int S>
static fg_status slice_operands(const Gemm& g, bool cplx, long long Kc, long long nchunks,
                                long long Np, int8_t* a_all, int8_t* b_all, double* rsc,
                                double* csc, unsigned long long* cmax, unsigned long long* kmax_a,
                                unsigned long long* kmax_b, int* shift, cudaStream_t st) {
    const double* A = static_cast<const double*>(g.A);
    const double* B = static_cast<const double*>(g.B);
    const long long M = g.M, K = g.K, N = g.N;
    const int cx = cplx ? 1 : 0;
    FG_TRY(scale_operands(g, cplx, rsc, csc, cmax, kmax_a, kmax_b, shift, st));
    // Slice chunk by chunk so each chunk's digit planes are contiguous.
    for (long long c = 0; c < nchunks; ++c) {
        ozaki_slice_a_kernel<S><<<grid_for(M * Kc), 256, 0, st>>>(
            A, M, K, g.lda, cx, shift, rsc, a_all + c * M * S * Kc, Kc, c * Kc);
        ozaki_slice_b_kernel<S><<<grid_for(Kc * Np), 256, 0, st>>>(
            B, K, N, g.ldb, cx, shift, csc, b_all + c * S * Kc * Np, Kc, Np, c * Kc);
        count_launch(2);
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// ------------------------------------------------------------ scheme II
// Pairwise coprime moduli, largest first, each <= 256 so that a symmetric
// residue fits int8; a call uses the first n (12..20).
static const int kOz2Moduli[20] = {256, 255, 253, 251, 247, 241, 239, 233, 229, 227,
                                   223, 217, 211, 199, 197, 193, 191, 181, 179, 173};

// Unsigned big integer, base 2^32 limbs, least significant first: just the
// operations the CRT constants need.
struct BigU {
    std::vector<uint32_t> w{1u};
    void mul(uint32_t f) {
        uint64_t carry = 0;
        for (auto& x : w) {
            const uint64_t t = static_cast<uint64_t>(x) * f + carry;
            x = static_cast<uint32_t>(t);
            carry = t >> 32;
        }
        if (carry) w.push_back(static_cast<uint32_t>(carry));
    }
    uint32_t divmod(uint32_t d) {  // *this /= d, returns the remainder
        uint64_t rem = 0;
        for (size_t i = w.size(); i-- > 0;) {
            const uint64_t cur = (rem << 32) | w[i];
            w[i] = static_cast<uint32_t>(cur / d);
            rem = cur % d;
        }
        while (w.size() > 1 && w.back() == 0) w.pop_back();
        return static_cast<uint32_t>(rem);
    }
    int bits() const {
        int b = 32 * static_cast<int>(w.size() - 1);
        for (uint32_t t = w.back(); t; t >>= 1) ++b;
        return b;
    }
    uint64_t bits_at(int lo, int n) const {  // n <= 40 bits starting at bit lo
        uint64_t v = 0;
        for (int b = 0; b < n; ++b) {
            const int q = lo + b;
            if (q / 32 < static_cast<int>(w.size()) && ((w[q / 32] >> (q % 32)) & 1u)) v |= 1ull << b;
        }
        return v;
    }
    double to_double() const {
        double v = 0;
        for (size_t i = w.size(); i-- > 0;) v = v * 4294967296.0 + w[i];
        return v;
    }
};

static int inverse_mod(int a, int m) {  // a^-1 mod m (gcd(a, m) = 1)
    int t = 0, nt = 1, r = m, nr = a % m;
    while (nr) {
        const int q = r / nr;
        std::swap(t, nt);
        nt -= q * t;
        std::swap(r, nr);
        nr -= q * r;
    }
    return t < 0 ? t + m : t;
}

// Constants of an n-moduli call with inner dimension K: P is the largest
// integer precision (at most 59, so rint(x / m) in oz2_residue is off by at
// most one) with K 2^(2P) < Mp / 4, i.e. every |C'| far from Mp / 2.
static Oz2Consts oz2_consts(int n, long long K) {
    Oz2Consts c{};
    c.n = n;
    BigU Mp;
    for (int l = 0; l < n; ++l) Mp.mul(static_cast<uint32_t>(kOz2Moduli[l]));
    int logk = 0;
    while ((1ll << logk) < K) ++logk;
    c.P = std::min(59, (Mp.bits() - 1 - logk - 2) / 2);
    for (int l = 0; l < n; ++l) {
        const int m = kOz2Moduli[l];
        BigU W = Mp;
        W.divmod(static_cast<uint32_t>(m));  // exact: Mp / m_l
        c.m[l] = m;
        c.inv_m[l] = 1.0 / m;
        c.magic[l] = static_cast<uint32_t>(((1ull << 32) + m - 1) / m);
        c.c20[l] = static_cast<uint32_t>((1ull << 20) % m);
        c.c40[l] = static_cast<uint32_t>((1ull << 40) % m);
        for (int d = 0; d < 4; ++d) c.W[l][d] = static_cast<double>(W.bits_at(40 * d, 40));
    }
    for (int d = 0; d < 4; ++d) c.Mc[d] = static_cast<double>(Mp.bits_at(40 * d, 40));
    c.M_d = Mp.to_double();
    c.inv_M = 1.0 / c.M_d;
    return c;
}

static int oz2_y(int n, int l) {  // ((Mp / m_l) mod m_l)^-1 mod m_l
    BigU Mp;
    for (int q = 0; q < n; ++q) Mp.mul(static_cast<uint32_t>(kOz2Moduli[q]));
    Mp.divmod(static_cast<uint32_t>(kOz2Moduli[l]));
    const int w_mod = static_cast<int>(Mp.divmod(static_cast<uint32_t>(kOz2Moduli[l])));
    return inverse_mod(w_mod, kOz2Moduli[l]);
}

using CfgCrt = TcCfg<KIND_I8, 256, 4, 1, 1, 1, 1, EPI_CRT>;
using CfgCrtPair = Tc2Cfg<KIND_I8, 256, 7, 1, 1, 1, 1, EPI_CRT>;

// Scheme II DGEMM / ZGEMM with n moduli (real GEMM, or the complex real
// embedding (M x 2K)(2K x 2N) like scheme I).
static fg_status launch_ozaki2(fg_ctx* ctx, const Gemm& g, int n, cudaStream_t st) {
    const bool cplx = g.dtype == FG_C64;
    const long long M = g.M, Kw = cplx ? 2 * g.K : g.K, Nw = cplx ? 2 * g.N : g.N;
    const long long Kp = round_up(std::max<long long>(Kw, 1), 128), Np = round_up(Nw, 16);
    const Oz2Consts c = oz2_consts(n, Kw);
    const size_t a_bytes = static_cast<size_t>(M * n * Kp), b_bytes = static_cast<size_t>(n * Kp * Np);
    const size_t r_bytes = static_cast<size_t>(n * M * Nw);
    const size_t n_sc = static_cast<size_t>(g.N);
    const size_t meta = (M + n_sc) * sizeof(double) + n_sc * sizeof(unsigned long long) +
                        2 * g.K * sizeof(unsigned long long) + g.K * sizeof(int);
    Scratch sc;
    FG_TRY(sc.alloc(round_up(a_bytes, 256) + round_up(b_bytes, 256) + round_up(r_bytes, 256) + meta, st));
    int8_t* a_all = static_cast<int8_t*>(sc.p);
    int8_t* b_all = a_all + round_up(a_bytes, 256);
    uint8_t* res = reinterpret_cast<uint8_t*>(b_all + round_up(b_bytes, 256));
    double* rsc = reinterpret_cast<double*>(res + round_up(r_bytes, 256));
    double* csc = rsc + M;
    unsigned long long* cmax = reinterpret_cast<unsigned long long*>(csc + n_sc);
    unsigned long long* kmax_a = cmax + n_sc;
    unsigned long long* kmax_b = kmax_a + g.K;
    int* shift = reinterpret_cast<int*>(kmax_b + g.K);
    FG_TRY(scale_operands(g, cplx, rsc, csc, cmax, kmax_a, kmax_b, shift, st));
    const double* A = static_cast<const double*>(g.A);
    const double* B = static_cast<const double*>(g.B);
    oz2_residue_a_kernel<<<grid_for(M * Kp / 8), 256, 0, st>>>(A, M, g.K, g.lda, cplx ? 1 : 0, shift, rsc, a_all, Kp, c);
    oz2_residue_b_kernel<<<grid_for(Kp * Np / 8), 256, 0, st>>>(B, g.K, g.N, g.ldb, cplx ? 1 : 0, shift, csc, b_all, Kp, Np, c);
    count_launch(2);
    FG_CUDA(cudaGetLastError());

    const bool pair = tune_lookup(TUNE_I8, M, Nw, Kp).variant == 2;
    // one launch for all moduli up to about 24 M outputs; beyond, one launch
    // per modulus keeps the CTAs' K positions in step for L2 reuse
    // (DGEMM 8192: 9.9 ms against 11.2 ms fused)
    const bool fused = fused_groups() && M * Nw <= (24ll << 20);
    const int launches = fused ? 1 : n;
    for (int L = 0; L < launches; ++L) {
        TcMaps maps;
        TcArgs args{};
        const long long kw = fused ? n * Kp : Kp;
        {
            uint64_t dims[2] = {static_cast<uint64_t>(kw), static_cast<uint64_t>(M)};
            uint64_t strides[1] = {static_cast<uint64_t>(n * Kp)};
            uint32_t box[2] = {128, 128};
            FG_TRY(encode_map(&maps.a[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, a_all + (fused ? 0 : L * Kp), dims,
                              strides, box));
        }
        {
            uint64_t dims[2] = {static_cast<uint64_t>(Nw), static_cast<uint64_t>(kw)};
            uint64_t strides[1] = {static_cast<uint64_t>(Np)};
            uint32_t box[2] = {128, 128};
            FG_TRY(encode_map(&maps.b[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, b_all + (fused ? 0 : L * Kp * Np), dims,
                              strides, box));
        }
        args.M = static_cast<int>(M);
        args.N = static_cast<int>(Nw);
        args.K = static_cast<int>(kw);
        args.tiles_m = static_cast<int>((M + (pair ? 255 : 127)) / (pair ? 256 : 128));
        args.tiles_n = static_cast<int>((Nw + CfgCrt::BN - 1) / CfgCrt::BN);
        args.k_blocks = static_cast<int>(kw / CfgCrt::BK);
        args.batch = 1;
        args.bdims = 1;
        args.bshape[0] = 1;
        args.C = res + (fused ? 0 : L * M * Nw);
        args.ldc = Nw;
        args.oz_crt = 1;
        args.oz_groups = fused ? n : 1;
        args.oz_kc_blocks = static_cast<int>(Kp / CfgCrt::BK);
        args.crt_plane = M * Nw;
        for (int q = 0; q < (fused ? n : 1); ++q) {
            const int l = fused ? q : L;
            args.crt_m[q] = kOz2Moduli[l];
            args.crt_y[q] = oz2_y(n, l);
        }
        args.ops[0] = TcOp{0, 0, 0, 1, 1};
        if (pair)
            FG_TRY(launch_group<CfgCrtPair>(ctx, maps, args, st));
        else
            FG_TRY(launch_group<CfgCrt>(ctx, maps, args, st));
    }
    {
        ProfScope prof("oz2_reconstruct", st);
        oz2_reconstruct_kernel<<<grid_for(M * Nw), 256, 0, st>>>(
            res, M, Nw, M * Nw, rsc, csc, static_cast<double*>(g.C), g.ldc, cplx ? static_cast<int>(g.N) : 0,
            g.alpha_re, g.beta_re, c);
        prof.stop();
        count_launch();
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

fg_status launch_ozaki(fg_ctx* ctx, const Gemm& g0, cudaStream_t st) {
    if (g0.batch > 1) {
        for (int i = 0; i < g0.batch; ++i) {
            Gemm s = g0;
            long long ia = 0, ib = 0;
            int rem = i;
            for (int d = g0.bdims - 1; d >= 0; --d) {
                int idx = rem % g0.bshape[d];
                rem /= g0.bshape[d];
                ia += idx * g0.a_istride[d];
                ib += idx * g0.b_istride[d];
            }
            const size_t es = g0.dtype == FG_C64 ? 2 : 1;  // doubles per element
            s.batch = 1;
            s.bdims = 0;
            s.a_count = s.b_count = 1;
            s.A = static_cast<const double*>(g0.A) + es * ia * g0.a_mstride;
            s.B = static_cast<const double*>(g0.B) + es * ib * g0.b_mstride;
            s.C = static_cast<double*>(g0.C) + es * i * g0.c_stride;
            FG_TRY(launch_ozaki(ctx, s, st));
        }
        return FG_OK;
    }
    const Gemm& g = g0;
    const bool cplx = g.dtype == FG_C64;
    // Default: scheme II with 16 moduli (DGEMM 8192: 3.3-3.5x plain FP64 at
    // 0.01-0.03x its normwise error for exponent spreads up to 10^8).
    // Scheme I: 9 slices keep the error well below plain FP64's (8 are about
    // equal).
    int S = g.slices > 0 ? g.slices : 16;
    if (S < 3 || (S > 10 && S < 12) || S > 20)
        return set_error(FG_ERR_INVALID, "ozaki_slices must be in 3..10 (scheme I slices) or 12..20 (scheme II moduli)");
    if (g.alpha_im != 0.0 || g.beta_im != 0.0)
        return set_error(FG_ERR_UNSUPPORTED, "split ZGEMM: complex alpha/beta must be real");
    if (S >= 12) {
        // scheme II: one int8 GEMM per modulus, while each product's exact
        // int32 sum holds (K 128^2 < 2^31); longer K (and empty problems)
        // run as scheme I with 9 slices
        if (round_up(cplx ? 2 * g.K : g.K, 128) <= 130944 && g.K > 0 && g.M > 0 && g.N > 0)
            return launch_ozaki2(ctx, g, S, st);
        S = 9;
    }
    const long long M = g.M, Kw = cplx ? 2 * g.K : g.K, Nw = cplx ? 2 * g.N : g.N;
    // The operands are sliced once over the whole (padded) K; int32
    // exactness is kept per launch instead: a launch accumulates at most
    // kpiece digit products (each |.| <= 127^2) in one int32, so a group
    // whose concatenated K ((d-1) Kp) is longer runs as several launches.
    const long long kpiece = ((2147483647ll / 16129ll) / 128) * 128;
    const long long Kp = round_up(Kw, 128);
    const long long nchunks = 1;
    const long long Kc = Kp;
    const long long Np = round_up(Nw, 16);
    const size_t a_bytes = static_cast<size_t>(nchunks * M * S * Kc);
    const size_t b_bytes = static_cast<size_t>(nchunks * S * Kc * Np);
    const size_t n_sc = static_cast<size_t>(cplx ? g.N : g.N);
    Scratch sc;
    const size_t meta = (M + n_sc) * sizeof(double) + n_sc * sizeof(unsigned long long) +
                        2 * g.K * sizeof(unsigned long long) + g.K * sizeof(int);
    FG_TRY(sc.alloc(round_up((long long)a_bytes, 256) + round_up((long long)b_bytes, 256) + meta, st));
    int8_t* a_all = static_cast<int8_t*>(sc.p);
    int8_t* b_all = a_all + round_up((long long)a_bytes, 256);
    double* rsc = reinterpret_cast<double*>(b_all + round_up((long long)b_bytes, 256));
    double* csc = rsc + M;
    unsigned long long* cmax = reinterpret_cast<unsigned long long*>(csc + n_sc);
    unsigned long long* kmax_a = cmax + n_sc;
    unsigned long long* kmax_b = kmax_a + g.K;
    int* shift = reinterpret_cast<int*>(kmax_b + g.K);
    fg_status sst;
    switch (S) {
        case 3: sst = slice_operands<3>(g, cplx, Kc, nchunks, Np, a_all, b_all, rsc, csc, cmax, kmax_a, kmax_b, shift, st); break;
        case 4: sst = slice_operands<4>(g, cplx, Kc, nchunks, Np, a_all, b_all, rsc, csc, cmax, kmax_a, kmax_b, shift, st); break;
        case 5: sst = slice_operands<5>(g, cplx, Kc, nchunks, Np, a_all, b_all, rsc, csc, cmax, kmax_a, kmax_b, shift, st); break;
        case 6: sst = slice_operands<6>(g, cplx, Kc, nchunks, Np, a_all, b_all, rsc, csc, cmax, kmax_a, kmax_b, shift, st); break;
        case 9: sst = slice_operands<9>(g, cplx, Kc, nchunks, Np, a_all, b_all, rsc, csc, cmax, kmax_a, kmax_b, shift, st); break;
        case 10: sst = slice_operands<10>(g, cplx, Kc, nchunks, Np, a_all, b_all, rsc, csc, cmax, kmax_a, kmax_b, shift, st); break;
        case 7: sst = slice_operands<7>(g, cplx, Kc, nchunks, Np, a_all, b_all, rsc, csc, cmax, kmax_a, kmax_b, shift, st); break;
        default: sst = slice_operands<8>(g, cplx, Kc, nchunks, Np, a_all, b_all, rsc, csc, cmax, kmax_a, kmax_b, shift, st); break;
    }
    FG_TRY(sst);

    // All S slice groups in one launch when the longest group's K (S Kc)
    // keeps its int32 accumulation exact: each tile runs its groups back to
    // back, so C is read and written from L2 between groups, the epilogue
    // of one group overlaps the products of the next, and there is one
    // launch instead of S.  Longer K: one launch per group (and K piece).
    // Measured on B200: one launch wins up to about 24 M outputs (DGEMM
    // 4096: 1.4-1.65x plain against 1.3x); beyond, the per-group launches
    // keep the CTAs' K positions in step and reuse operand panels in L2
    // better (DGEMM 8192: 1.8-2.05x against 1.5-1.8x).
    if (fused_groups() && S * Kc <= kpiece && Kc % CfgOzaki::BK == 0 && M * Nw <= (24ll << 20)) {
        TcMaps maps;
        TcArgs args{};
        {
            uint64_t dims[2] = {static_cast<uint64_t>(S * Kc), static_cast<uint64_t>(M)};
            uint64_t strides[1] = {static_cast<uint64_t>(S * Kc)};
            uint32_t box[2] = {128, 128};
            FG_TRY(encode_map(&maps.a[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, a_all, dims, strides, box));
        }
        {
            uint64_t dims[2] = {static_cast<uint64_t>(Nw), static_cast<uint64_t>(S * Kc)};
            uint64_t strides[1] = {static_cast<uint64_t>(Np)};
            uint32_t box[2] = {128, 128};
            FG_TRY(encode_map(&maps.b[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, b_all, dims, strides, box));
        }
        args.M = static_cast<int>(M);
        args.N = static_cast<int>(Nw);
        args.K = static_cast<int>(S * Kc);
        args.tiles_m = static_cast<int>((M + 127) / 128);
        args.tiles_n = static_cast<int>((Nw + CfgOzaki::BN - 1) / CfgOzaki::BN);
        args.k_blocks = static_cast<int>(S * Kc / CfgOzaki::BK);
        args.batch = 1;
        args.bdims = 1;
        args.bshape[0] = 1;
        args.C = g.C;
        args.ldc = cplx ? 2 * g.ldc : g.ldc;
        args.cplx_half = cplx ? static_cast<int>(g.N) : 0;
        args.row_scale = rsc;
        args.col_scale = csc;
        args.oz_w = g.alpha_re;
        args.oz_beta = g.beta_re;
        args.oz_first = 1;
        args.oz_groups = S;
        args.oz_d0 = S + 1;
        args.oz_kc_blocks = static_cast<int>(Kc / CfgOzaki::BK);
        args.oz_S = S;
        args.ops[0] = TcOp{0, 0, 0, 1, 1};
        // CTA pairs (256 x 256 tiles) where the tuned i8 table picks them for
        // the group products' shape
        if (tune_lookup(TUNE_I8, M, Nw, Kc).variant == 2) {
            args.tiles_m = static_cast<int>((M + 255) / 256);
            return launch_group<CfgOzakiPair>(ctx, maps, args, st);
        }
        return launch_group<CfgOzaki>(ctx, maps, args, st);
    }

    bool first = true;
    for (int d = S + 1; d >= 2; --d) {
        const long long Kd_all = (d - 1) * Kc;
        for (long long k0 = 0; k0 < Kd_all; k0 += kpiece) {
            const long long Kd = std::min(kpiece, Kd_all - k0);
            TcMaps maps;
            TcArgs args{};
            {
                uint64_t dims[2] = {static_cast<uint64_t>(Kd), static_cast<uint64_t>(M)};
                uint64_t strides[1] = {static_cast<uint64_t>(S * Kc)};
                uint32_t box[2] = {128, 128};
                FG_TRY(encode_map(&maps.a[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, a_all + k0, dims, strides, box));
            }
            {
                uint64_t dims[2] = {static_cast<uint64_t>(Nw), static_cast<uint64_t>(Kd)};
                uint64_t strides[1] = {static_cast<uint64_t>(Np)};
                uint32_t box[2] = {128, 128};
                FG_TRY(encode_map(&maps.b[0], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2,
                                  b_all + ((S - d + 1) * Kc + k0) * Np, dims, strides, box));
            }
            const bool pair = tune_lookup(TUNE_I8, M, Nw, Kd).variant == 2;
            args.M = static_cast<int>(M);
            args.N = static_cast<int>(Nw);
            args.K = static_cast<int>(Kd);
            args.tiles_m = static_cast<int>((M + (pair ? 255 : 127)) / (pair ? 256 : 128));
            args.tiles_n = static_cast<int>((Nw + CfgOzaki::BN - 1) / CfgOzaki::BN);
            args.k_blocks = static_cast<int>((Kd + CfgOzaki::BK - 1) / CfgOzaki::BK);
            args.batch = 1;
            args.bdims = 1;
            args.bshape[0] = 1;
            args.C = g.C;
            args.ldc = cplx ? 2 * g.ldc : g.ldc;
            args.cplx_half = cplx ? static_cast<int>(g.N) : 0;
            args.row_scale = rsc;
            args.col_scale = csc;
            args.oz_w = g.alpha_re * std::ldexp(1.0, -7 * d);
            args.oz_beta = g.beta_re;
            args.oz_first = first ? 1 : 0;
            args.ops[0] = TcOp{0, 0, 0, 1, 1};
            if (pair)
                FG_TRY(launch_group<CfgOzakiPair>(ctx, maps, args, st));
            else
                FG_TRY(launch_group<CfgOzaki>(ctx, maps, args, st));
            first = false;
        }
    }
    return FG_OK;
}

}  // namespace fgrt
