// grouped.cu -- fg_gemm_grouped and prepared grouped plans (CUDA graphs).
//
// Lowering of a host problem table:
//  * dtype FG_I8 / FG_U8I8: tcgen05 kind::i8 grouped kernel; operands whose
//    pointer or leading dimension breaks the TMA 16-byte rule are copied into
//    a 16-byte-pitched arena by the prep launch, the rest are read in place;
//  * dtype FG_F32, mode SPLIT: the prep launch splits every operand into bf16
//    hi/lo planes in the arena; tcgen05 kind::f16 grouped kernel, three
//    products, K-chunked FP32 accumulation;
//  * dtype FG_F32, mode PLAIN: persistent FFMA grouped kernel.
// Tiles are numbered deepest problem first and handed out by the kernels'
// device-side scheduler (an atomic tile counter, zeroed before every launch).
// A plan keeps the tables and arena resident and replays the counter reset,
// prep and grouped launches from a CUDA graph.
#include <cuda_bf16.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <numeric>
#include <vector>

#include "prep_kernels.cuh"
#include "runtime.h"
#include "tc_grouped.cuh"

using namespace fg;

namespace {

using CfgGroupedI8 = TcCfg<KIND_I8, 128, 6, 1, 1, 1, 1, EPI_I32>;
using CfgGroupedBf16 = TcCfg<KIND_BF16, 128, 3, 2, 2, 1, 3, EPI_F32, 1>;

long long rup(long long x, long long a) { return (x + a - 1) / a * a; }

template <class Cfg>
fg_status set_smem_attr() {
    static std::once_flag once;
    static cudaError_t err = cudaSuccess;
    std::call_once(once, [] {
        err = cudaFuncSetAttribute(tc_grouped_kernel<Cfg>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(tc_smem_bytes<Cfg>()));
    });
    if (err != cudaSuccess) return fgrt::cuda_error(err, "cudaFuncSetAttribute(grouped)");
    return FG_OK;
}

}  // namespace

// A grouped batch lowered to device form.  build() is host-only (ordering,
// tiling, layout sizes); bind() fixes the device base address, encodes the
// TMA descriptors and writes the tables into a host image laid out exactly
// like the front of the device region; launch() copies that image with one
// async memcpy and issues the prep and grouped kernels on a stream.
struct fgrt::GroupedJob {
    fg_ctx* ctx = nullptr;
    fg_dtype dtype = FG_F32;
    fg_mode mode = FG_MODE_PLAIN;
    int kind = 0;  // 0 = FFMA, 1 = i8 tensor, 2 = bf16x3 tensor
    struct Opnd {
        const void* src = nullptr;
        long long off0 = -1, off1 = -1, ld = 0;
    };
    struct Zero {
        void* c;
        long long m, n, ldc;
    };
    std::vector<fg_problem> probs_in;  // ordered, K > 0
    std::vector<GroupedProblem> probs;
    std::vector<Opnd> oa, ob;
    std::vector<Zero> zeros;
    long long total_tiles = 0;
    long long arena = 0;
    int nseg = 0;
    int njobs = 0;  // prep launch blocks: segments cut at PREP_JOB_CHUNKS chunks
    size_t sz_probs = 0, sz_maps = 0, sz_ptrs = 0, sz_segs = 0, sz_jobs = 0, sz_tiles = 0;
    static constexpr size_t sz_sched = 256;  // the tile scheduler's counter
    // bound state
    void* dev = nullptr;
    const void* host = nullptr;
    GroupedArgs targs{};
    SimtGroupedArgs sargs{};
    PrepSeg* d_segs = nullptr;
    PrepJob* d_jobs = nullptr;
    unsigned long long* d_counter = nullptr;
    size_t host_bytes() const { return sz_probs + sz_maps + sz_ptrs + sz_segs + sz_jobs + sz_tiles + sz_sched; }
    size_t dev_bytes() const { return host_bytes() + static_cast<size_t>(arena); }
};

struct fg_grouped_plan {
    fgrt::GroupedJob job;
    void* mem = nullptr;
    void* host = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
};

namespace fgrt {

GroupedJob* grouped_job_new() { return new GroupedJob(); }
void grouped_job_free(GroupedJob* j) { delete j; }
size_t grouped_job_dev_bytes(const GroupedJob* j) { return j->dev_bytes(); }
size_t grouped_job_host_bytes(const GroupedJob* j) { return j->host_bytes(); }

fg_status grouped_job_build(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const fg_problem* table,
                            size_t count, GroupedJob* j) {
    if (!ctx || (!table && count)) return set_error(FG_ERR_INVALID, "null argument");
    if (dtype != FG_F32 && dtype != FG_I8 && dtype != FG_U8I8)
        return set_error(FG_ERR_DTYPE, "grouped GEMM: dtype must be FG_F32, FG_I8 or FG_U8I8");
    if (count > (1u << 30)) return set_error(FG_ERR_UNSUPPORTED, "too many problems");
    *j = GroupedJob();
    j->ctx = ctx;
    j->dtype = dtype;
    j->mode = mode;
    j->kind = dtype == FG_F32 ? (mode != FG_MODE_PLAIN ? 2 : 0) : 1;
    std::vector<int> order;
    for (size_t i = 0; i < count; ++i) {
        const fg_problem& q = table[i];
        if (q.m < 0 || q.n < 0 || q.k < 0)
            return set_error(FG_ERR_SHAPE, "grouped GEMM: negative dimension in problem " + std::to_string(i));
        if (q.m == 0 || q.n == 0) continue;
        if (!q.c || (q.k > 0 && (!q.a || !q.b)) || q.ldc < q.n || (q.k > 0 && (q.lda < q.k || q.ldb < q.n)))
            return set_error(FG_ERR_INVALID, "grouped GEMM: bad pointer or leading dimension in problem " + std::to_string(i));
        if (q.m > (1 << 30) || q.n > (1 << 30) || q.k > (1 << 30) ||
            (j->kind == 1 && q.k > (dtype == FG_I8 ? 131072 : 65536)))
            return set_error(FG_ERR_UNSUPPORTED, "grouped GEMM: problem " + std::to_string(i) + " too large");
        if (q.k == 0) {
            j->zeros.push_back({q.c, q.m, q.n, q.ldc});
            continue;
        }
        order.push_back(static_cast<int>(i));
    }
    // longest K first: the static strided tile walk then balances SMs
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return table[x].k > table[y].k; });
    const int np = static_cast<int>(order.size());
    const int bm = j->kind == 0 ? 64 : 128;
    j->probs_in.resize(np);
    j->probs.resize(np);
    j->oa.resize(np);
    j->ob.resize(np);
    int nseg = 0;
    for (int x = 0; x < np; ++x) {
        const fg_problem& q = table[order[x]];
        j->probs_in[x] = q;
        GroupedProblem& g = j->probs[x];
        g.M = static_cast<int>(q.m);
        g.N = static_cast<int>(q.n);
        g.K = static_cast<int>(q.k);
        // plain FP32: a 32 x 32 tile where it pads at most 0.7x the area a
        // 64 x 64 one does (small problems; its FMAs cost more each)
        int tb = bm;
        if (j->kind == 0) {
            const long long a64 = (q.m + 63) / 64 * 64 * ((q.n + 63) / 64 * 64);
            const long long a32 = (q.m + 31) / 32 * 32 * ((q.n + 31) / 32 * 32);
            if (10 * a32 <= 7 * a64) tb = 32;
        }
        g.tile = tb;
        g.tiles_m = static_cast<int>((q.m + tb - 1) / tb);
        g.tiles_n = static_cast<int>((q.n + tb - 1) / tb);
        g.tile_start = j->total_tiles;
        j->total_tiles += (long long)g.tiles_m * g.tiles_n;
        g.C = q.c;
        g.ldc = q.ldc;
        auto& oa = j->oa[x];
        auto& ob = j->ob[x];
        oa.src = q.a;
        ob.src = q.b;
        if (j->kind == 1) {
            g.k_blocks = static_cast<int>((q.k + 127) / 128);
            if ((reinterpret_cast<uintptr_t>(q.a) & 15) || (q.lda % 16)) {
                oa.ld = rup(q.k, 16);
                oa.off0 = j->arena;
                j->arena = rup(j->arena + oa.ld * q.m, 256);
                ++nseg;
                j->njobs += static_cast<int>((q.m * (oa.ld / 16) + PREP_JOB_CHUNKS - 1) / PREP_JOB_CHUNKS);
            } else {
                oa.ld = q.lda;
            }
            if ((reinterpret_cast<uintptr_t>(q.b) & 15) || (q.ldb % 16)) {
                ob.ld = rup(q.n, 16);
                ob.off0 = j->arena;
                j->arena = rup(j->arena + ob.ld * q.k, 256);
                ++nseg;
                j->njobs += static_cast<int>((q.k * (ob.ld / 16) + PREP_JOB_CHUNKS - 1) / PREP_JOB_CHUNKS);
            } else {
                ob.ld = q.ldb;
            }
        } else if (j->kind == 2) {
            g.k_blocks = static_cast<int>((q.k + 63) / 64);
            oa.ld = rup(q.k, 8);
            oa.off0 = j->arena;
            j->arena = rup(j->arena + 2 * oa.ld * q.m, 256);
            oa.off1 = j->arena;
            j->arena = rup(j->arena + 2 * oa.ld * q.m, 256);
            ob.ld = rup(q.n, 8);
            ob.off0 = j->arena;
            j->arena = rup(j->arena + 2 * ob.ld * q.k, 256);
            ob.off1 = j->arena;
            j->arena = rup(j->arena + 2 * ob.ld * q.k, 256);
            nseg += 2;
            j->njobs += static_cast<int>((q.m * (oa.ld / 8) + PREP_JOB_CHUNKS - 1) / PREP_JOB_CHUNKS +
                                         (q.k * (ob.ld / 8) + PREP_JOB_CHUNKS - 1) / PREP_JOB_CHUNKS);
        } else {
            g.k_blocks = static_cast<int>((q.k + 15) / 16);
            oa.ld = q.lda;
            ob.ld = q.ldb;
        }
    }
    j->nseg = nseg;
    const int nmaps = j->kind == 2 ? 4 : 2;
    const size_t npp = static_cast<size_t>(std::max(np, 1));
    j->sz_probs = rup(sizeof(GroupedProblem) * npp, 256);
    j->sz_maps = j->kind == 0 ? 0 : rup(sizeof(CUtensorMap) * nmaps * npp, 256);
    j->sz_ptrs = j->kind == 0 ? rup((2 * sizeof(void*) + 2 * sizeof(long long)) * npp, 256) : 0;
    j->sz_segs = rup(sizeof(PrepSeg) * std::max(nseg, 1), 256);
    j->sz_jobs = rup(sizeof(PrepJob) * static_cast<size_t>(std::max(j->njobs, 1)), 256);
    j->sz_tiles = rup(sizeof(TileRec) * static_cast<size_t>(std::max<long long>(j->total_tiles, 1)), 256);
    return FG_OK;
}

fg_status grouped_job_bind(GroupedJob* j, void* dev_base, void* host_stage) {
    const int np = static_cast<int>(j->probs.size());
    const size_t npp = static_cast<size_t>(std::max(np, 1));
    char* dbase = static_cast<char*>(dev_base);
    char* hbase = static_cast<char*>(host_stage);
    const size_t o_maps = j->sz_probs, o_ptrs = o_maps + j->sz_maps, o_segs = o_ptrs + j->sz_ptrs;
    const size_t o_jobs = o_segs + j->sz_segs, o_tiles = o_jobs + j->sz_jobs, o_sched = o_tiles + j->sz_tiles;
    char* d_arena = dbase + j->host_bytes();
    std::memset(hbase + o_sched, 0, j->sz_sched);
    j->d_counter = reinterpret_cast<unsigned long long*>(dbase + o_sched);
    std::memcpy(hbase, j->probs.data(), sizeof(GroupedProblem) * np);
    TileRec* htiles = reinterpret_cast<TileRec*>(hbase + o_tiles);
    // Tiles of the deepest problems first: the scheduler hands them out in
    // this order, so the long tiles start first and the short ones fill in
    // behind them (longest-first balance).
    std::vector<int> order(static_cast<size_t>(np));
    for (int x = 0; x < np; ++x) order[x] = x;
    std::stable_sort(order.begin(), order.end(),
                     [&](int u, int v) { return j->probs[u].k_blocks > j->probs[v].k_blocks; });
    long long t = 0;
    for (int x : order) {
        const GroupedProblem& g = j->probs[x];
        for (int tm = 0; tm < g.tiles_m; ++tm)
            for (int tn = 0; tn < g.tiles_n; ++tn) htiles[t++] = TileRec{x, tm, tn, g.k_blocks};
    }
    const TileRec* dtiles = reinterpret_cast<const TileRec*>(dbase + o_tiles);
    CUtensorMap* hmaps = reinterpret_cast<CUtensorMap*>(hbase + o_maps);
    PrepSeg* hsegs = reinterpret_cast<PrepSeg*>(hbase + o_segs);
    int si = 0;
    for (int x = 0; x < np; ++x) {
        const fg_problem& q = j->probs_in[x];
        const auto& oa = j->oa[x];
        const auto& ob = j->ob[x];
        if (j->kind == 1) {
            const void* pa = q.a;
            const void* pb = q.b;
            if (oa.off0 >= 0) {
                pa = d_arena + oa.off0;
                hsegs[si++] = PrepSeg{q.a, const_cast<void*>(pa), nullptr, q.m, q.k, q.lda, oa.ld, 0};
            }
            if (ob.off0 >= 0) {
                pb = d_arena + ob.off0;
                hsegs[si++] = PrepSeg{q.b, const_cast<void*>(pb), nullptr, q.k, q.n, q.ldb, ob.ld, 0};
            }
            uint64_t da[2] = {(uint64_t)q.k, (uint64_t)q.m}, sa[1] = {(uint64_t)oa.ld};
            uint64_t db[2] = {(uint64_t)q.n, (uint64_t)q.k}, sb[1] = {(uint64_t)ob.ld};
            // A in 8-row boxes (the kernel spreads them over the accumulator's
            // lane quadrants), B in 128 x 128 boxes
            uint32_t boxa[2] = {128, 8}, box[2] = {128, 128};
            FG_TRY(encode_map(&hmaps[2 * x], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, pa, da, sa, boxa));
            FG_TRY(encode_map(&hmaps[2 * x + 1], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, pb, db, sb, box));
        } else if (j->kind == 2) {
            void* ah = d_arena + oa.off0;
            void* al = d_arena + oa.off1;
            void* bh = d_arena + ob.off0;
            void* bl = d_arena + ob.off1;
            hsegs[si++] = PrepSeg{q.a, ah, al, q.m, q.k, q.lda, oa.ld, 1};
            hsegs[si++] = PrepSeg{q.b, bh, bl, q.k, q.n, q.ldb, ob.ld, 1};
            uint64_t da[2] = {(uint64_t)q.k, (uint64_t)q.m}, sa[1] = {(uint64_t)(2 * oa.ld)};
            uint64_t db[2] = {(uint64_t)q.n, (uint64_t)q.k}, sb[1] = {(uint64_t)(2 * ob.ld)};
            uint32_t boxa[2] = {64, 8}, boxb[2] = {64, 64};  // A in 8-row boxes (row spreading)
            FG_TRY(encode_map(&hmaps[4 * x + 0], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ah, da, sa, boxa));
            FG_TRY(encode_map(&hmaps[4 * x + 1], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, al, da, sa, boxa));
            FG_TRY(encode_map(&hmaps[4 * x + 2], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, bh, db, sb, boxb));
            FG_TRY(encode_map(&hmaps[4 * x + 3], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, bl, db, sb, boxb));
        }
    }
    {
        // block jobs: each segment cut into runs of at most PREP_JOB_CHUNKS chunks
        PrepJob* hjobs = reinterpret_cast<PrepJob*>(hbase + o_jobs);
        int ji = 0;
        for (int k = 0; k < si; ++k) {
            const PrepSeg& sg = hsegs[k];
            const long long n = sg.rows * (sg.ld_dst / (sg.op == 0 ? 16 : 8));
            for (long long c0 = 0; c0 < n && ji < j->njobs; c0 += PREP_JOB_CHUNKS)
                hjobs[ji++] = PrepJob{k, 0, c0, std::min(n, c0 + PREP_JOB_CHUNKS)};
        }
        if (ji != j->njobs || si != j->nseg) return set_error(FG_ERR_INVALID, "grouped plan: prep table mismatch");
    }
    j->d_jobs = reinterpret_cast<PrepJob*>(dbase + o_jobs);
    if (j->kind == 0) {
        const void** pa = reinterpret_cast<const void**>(hbase + o_ptrs);
        const void** pb = pa + npp;
        long long* la = reinterpret_cast<long long*>(pb + npp);
        long long* lb = la + npp;
        for (int x = 0; x < np; ++x) {
            pa[x] = j->oa[x].src;
            pb[x] = j->ob[x].src;
            la[x] = j->oa[x].ld;
            lb[x] = j->ob[x].ld;
        }
        const void** dpa = reinterpret_cast<const void**>(dbase + o_ptrs);
        j->sargs.problems = reinterpret_cast<const GroupedProblem*>(dbase);
        j->sargs.tiles = dtiles;
        j->sargs.tile_counter = j->d_counter;
        j->sargs.a = dpa;
        j->sargs.b = dpa + npp;
        j->sargs.lda = reinterpret_cast<const long long*>(dpa + 2 * npp);
        j->sargs.ldb = reinterpret_cast<const long long*>(dpa + 2 * npp) + npp;
        j->sargs.count = np;
        j->sargs.total_tiles = j->total_tiles;
        j->sargs.alpha = 1.f;
        j->sargs.beta = 0.f;
    }
    j->d_segs = reinterpret_cast<PrepSeg*>(dbase + o_segs);
    j->targs = GroupedArgs{};
    j->targs.problems = reinterpret_cast<const GroupedProblem*>(dbase);
    j->targs.tiles = dtiles;
    j->targs.tile_counter = j->d_counter;
    j->targs.maps = reinterpret_cast<const CUtensorMap*>(dbase + o_maps);
    j->targs.count = np;
    j->targs.total_tiles = j->total_tiles;
    j->targs.alpha = 1.f;
    j->targs.beta = 0.f;
    j->targs.status = j->ctx->d_status;
    j->targs.timeout_ns = 4000000000ull;
    // split form: K blocks (64 values each) per TMEM accumulation chunk, as
    // in the single-problem split GEMM
    j->targs.kchunk = 4;
    if (j->kind == 1) {
        j->targs.ops[0] = TcOp{0, 0, 0, j->dtype == FG_I8 ? 1 : 0, 1};
        FG_TRY(set_smem_attr<CfgGroupedI8>());
    } else if (j->kind == 2) {
        j->targs.ops[0] = TcOp{1, 0, 0, 1, 1};
        j->targs.ops[1] = TcOp{0, 1, 0, 1, 1};
        j->targs.ops[2] = TcOp{0, 0, 0, 1, 1};
        FG_TRY(set_smem_attr<CfgGroupedBf16>());
    }
    j->dev = dev_base;
    j->host = host_stage;
    return FG_OK;
}

// Kernels only (tables already on the device).
static fg_status grouped_job_kernels(GroupedJob* j, cudaStream_t st) {
    fg_ctx* ctx = j->ctx;
    for (auto& z : j->zeros) {
        const long long blocks = std::min<long long>((z.m * z.n + 255) / 256 + 1, 1024);
        if (j->dtype == FG_F32)
            scale_kernel<float><<<blocks, 256, 0, st>>>(static_cast<float*>(z.c), z.m, z.n, z.ldc, 0.f);
        else
            scale_kernel<int><<<blocks, 256, 0, st>>>(static_cast<int*>(z.c), z.m, z.n, z.ldc, 0);
        count_launch();
    }
    if (j->nseg > 0) {
        ProfScope prof("grouped_prep", st);
        const int blocks = std::min(j->njobs, 1 << 20);
        if (j->kind == 1)
            grouped_prep_kernel<0><<<blocks, 256, 0, st>>>(j->d_segs, j->d_jobs, j->njobs);
        else
            grouped_prep_kernel<1><<<blocks, 256, 0, st>>>(j->d_segs, j->d_jobs, j->njobs);
        prof.stop();
        count_launch();
    }
    if (j->total_tiles == 0) {
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }
    const int grid = static_cast<int>(std::min<long long>(j->total_tiles, ctx->sm_count));
    FG_CUDA(cudaMemsetAsync(j->d_counter, 0, sizeof(unsigned long long), st));
    if (j->kind == 0) {
        ProfScope prof("simt_grouped_sgemm", st);
        simt_grouped_sgemm<<<std::min<long long>(j->total_tiles, ctx->sm_count * 8), 128, 0, st>>>(j->sargs);
        prof.stop();
    } else if (j->kind == 1) {
        ProfScope prof("tc_grouped_i8", st);
        tc_grouped_kernel<CfgGroupedI8><<<grid, CfgGroupedI8::THREADS, tc_smem_bytes<CfgGroupedI8>(), st>>>(j->targs);
        prof.stop();
    } else {
        ProfScope prof("tc_grouped_3xbf16", st);
        tc_grouped_kernel<CfgGroupedBf16><<<grid, CfgGroupedBf16::THREADS, tc_smem_bytes<CfgGroupedBf16>(), st>>>(j->targs);
        prof.stop();
    }
    count_launch();
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

fg_status grouped_job_launch(GroupedJob* j, cudaStream_t st) {
    if (j->host_bytes() && !j->probs.empty())
        FG_CUDA(cudaMemcpyAsync(j->dev, j->host, j->host_bytes(), cudaMemcpyHostToDevice, st));
    return grouped_job_kernels(j, st);
}

static void free_plan(fg_grouped_plan* p) {
    if (!p) return;
    if (p->job.ctx) cudaSetDevice(p->job.ctx->device);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->mem) cudaFree(p->mem);
    if (p->host) cudaFreeHost(p->host);
    delete p;
}

// Plan: build + device/pinned memory + synchronous table upload.
static fg_status make_plan(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const fg_problem* table,
                           size_t count, cudaStream_t st, fg_grouped_plan** out) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    FG_CUDA(cudaSetDevice(ctx->device));
    auto* p = new fg_grouped_plan();
    fg_status s = grouped_job_build(ctx, dtype, mode, table, count, &p->job);
    if (s != FG_OK) {
        delete p;
        return s;
    }
    cudaError_t e = cudaMalloc(&p->mem, std::max<size_t>(p->job.dev_bytes(), 256));
    if (e == cudaSuccess) e = cudaMallocHost(&p->host, std::max<size_t>(p->job.host_bytes(), 256));
    if (e != cudaSuccess) {
        cudaGetLastError();
        free_plan(p);
        return set_error(FG_ERR_OOM, "grouped plan: allocation failed");
    }
    s = grouped_job_bind(&p->job, p->mem, p->host);
    if (s == FG_OK && !p->job.probs.empty()) {
        e = cudaMemcpyAsync(p->mem, p->host, p->job.host_bytes(), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) s = cuda_error(e, "grouped plan upload");
    }
    if (s != FG_OK) {
        free_plan(p);
        return s;
    }
    *out = p;
    return FG_OK;
}

}  // namespace fgrt

using namespace fgrt;

extern "C" {

fg_status fg_gemm_grouped(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const fg_problem* table,
                          size_t count, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    cudaStream_t st = stream_of(ctx, stream);
    fg_grouped_plan* p = nullptr;
    FG_TRY(make_plan(ctx, dtype, mode, table, count, st, &p));
    fg_status s = grouped_job_kernels(&p->job, st);
    cudaError_t e = cudaStreamSynchronize(st);  // the plan's memory is freed next
    free_plan(p);
    if (s != FG_OK) return s;
    if (e != cudaSuccess) return cuda_error(e, "grouped GEMM");
    return FG_OK;
}

fg_status fg_grouped_plan_create(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const fg_problem* table,
                                 size_t count, fg_stream stream, fg_grouped_plan** out) {
    if (!out) return set_error(FG_ERR_INVALID, "null out");
    *out = nullptr;
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    cudaStream_t st = stream_of(ctx, stream);
    fg_grouped_plan* p = nullptr;
    FG_TRY(make_plan(ctx, dtype, mode, table, count, st, &p));
    // Capture the launch sequence once; runs replay it.
    cudaStream_t cap;
    cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    fg_status s = FG_OK;
    if (e == cudaSuccess) {
        e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            const int prof = g_prof_on.exchange(0);  // no event records inside the graph
            s = grouped_job_kernels(&p->job, cap);
            g_prof_on.store(prof);
            cudaGraph_t graph = nullptr;
            cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
            if (e2 == cudaSuccess) {
                p->graph = graph;
                e2 = cudaGraphInstantiate(&p->exec, graph, 0);
            }
            e = e2;
        }
        cudaStreamDestroy(cap);
    }
    if (s != FG_OK || e != cudaSuccess) {
        free_plan(p);
        return s != FG_OK ? s : cuda_error(e, "grouped plan capture");
    }
    *out = p;
    return FG_OK;
}

fg_status fg_grouped_plan_run(fg_grouped_plan* p, fg_stream stream) {
    if (!p) return set_error(FG_ERR_INVALID, "null plan");
    FG_CUDA(cudaSetDevice(p->job.ctx->device));
    cudaStream_t st = stream_of(p->job.ctx, stream);
    ProfScope prof(p->job.kind == 0 ? "grouped_plan_ffma" : p->job.kind == 1 ? "grouped_plan_i8" : "grouped_plan_3xbf16", st);
    FG_CUDA(cudaGraphLaunch(p->exec, st));
    prof.stop();
    count_launch(1 + (p->job.nseg > 0 ? 1 : 0) + p->job.zeros.size());
    return FG_OK;
}

fg_status fg_grouped_plan_destroy(fg_grouped_plan* p) {
    free_plan(p);
    return FG_OK;
}

}  // extern "C"
