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
// Problems are ordered by decreasing K (longest first) so the static strided
// tile walk balances SMs.  A plan keeps the tables and arena resident and
// replays the prep + grouped launches from a CUDA graph.
#include <cuda_bf16.h>

#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "prep_kernels.cuh"
#include "runtime.h"
#include "tc_grouped.cuh"

using namespace fg;

namespace {

using CfgGroupedI8 = TcCfg<KIND_I8, 128, 4, 1, 1, 1, 1, EPI_I32>;
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

struct fg_grouped_plan {
    fg_ctx* ctx = nullptr;
    fg_dtype dtype = FG_F32;
    fg_mode mode = FG_MODE_PLAIN;
    int kind = 0;  // 0 = FFMA, 1 = i8 tensor, 2 = bf16x3 tensor
    void* mem = nullptr;  // one device allocation: tables, maps, segments, arena
    GroupedArgs targs{};
    SimtGroupedArgs sargs{};
    PrepSeg* d_segs = nullptr;
    int nseg = 0;
    long long prep_total = 0;
    struct Zero {
        void* c;
        long long m, n, ldc;
        int accumulate;
    };
    std::vector<Zero> zeros;  // K == 0 problems
    long long total_tiles = 0;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
};

namespace fgrt {

static fg_status launch_plan(fg_grouped_plan* p, cudaStream_t st) {
    fg_ctx* ctx = p->ctx;
    for (auto& z : p->zeros) {
        if (z.accumulate) continue;
        if (p->dtype == FG_F32) {
            scale_kernel<float><<<std::min<long long>((z.m * z.n + 255) / 256 + 1, 1024), 256, 0, st>>>(
                static_cast<float*>(z.c), z.m, z.n, z.ldc, p->targs.beta);
        } else {
            scale_kernel<int><<<std::min<long long>((z.m * z.n + 255) / 256 + 1, 1024), 256, 0, st>>>(
                static_cast<int*>(z.c), z.m, z.n, z.ldc, 0);
        }
        count_launch();
    }
    if (p->nseg > 0) {
        const int grid = static_cast<int>(std::min<long long>((p->prep_total + 255) / 256, 8 * 148 * 4));
        grouped_prep_kernel<<<grid, 256, 0, st>>>(p->d_segs, p->nseg, p->prep_total);
        count_launch();
    }
    if (p->total_tiles == 0) {
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }
    const int grid = static_cast<int>(std::min<long long>(p->total_tiles, ctx->sm_count));
    if (p->kind == 0) {
        ProfScope prof("simt_grouped_sgemm", st);
        simt_grouped_sgemm<<<std::min<long long>(p->total_tiles, ctx->sm_count * 4), 256, 0, st>>>(p->sargs);
        prof.stop();
    } else if (p->kind == 1) {
        ProfScope prof("tc_grouped_i8", st);
        tc_grouped_kernel<CfgGroupedI8><<<grid, CfgGroupedI8::THREADS, tc_smem_bytes<CfgGroupedI8>(), st>>>(p->targs);
        prof.stop();
    } else {
        ProfScope prof("tc_grouped_3xbf16", st);
        tc_grouped_kernel<CfgGroupedBf16><<<grid, CfgGroupedBf16::THREADS, tc_smem_bytes<CfgGroupedBf16>(), st>>>(p->targs);
        prof.stop();
    }
    count_launch();
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

static fg_status build_plan(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const fg_problem* table,
                            size_t count, cudaStream_t st, fg_grouped_plan** out) {
    if (!ctx || !out || (!table && count)) return set_error(FG_ERR_INVALID, "null argument");
    if (dtype != FG_F32 && dtype != FG_I8 && dtype != FG_U8I8)
        return set_error(FG_ERR_DTYPE, "grouped GEMM: dtype must be FG_F32, FG_I8 or FG_U8I8");
    if (count > (1u << 30)) return set_error(FG_ERR_UNSUPPORTED, "too many problems");
    FG_CUDA(cudaSetDevice(ctx->device));
    auto* p = new fg_grouped_plan();
    p->ctx = ctx;
    p->dtype = dtype;
    p->mode = mode;
    p->kind = dtype == FG_F32 ? (mode == FG_MODE_SPLIT ? 2 : 0) : 1;
    p->targs.alpha = 1.f;
    p->targs.beta = 0.f;
    p->sargs.alpha = 1.f;
    p->sargs.beta = 0.f;

    // validate, drop empty problems, order by decreasing K
    std::vector<int> order;
    for (size_t i = 0; i < count; ++i) {
        const fg_problem& q = table[i];
        if (q.m < 0 || q.n < 0 || q.k < 0) {
            delete p;
            return set_error(FG_ERR_SHAPE, "grouped GEMM: negative dimension in problem " + std::to_string(i));
        }
        if (q.m == 0 || q.n == 0) continue;
        if (!q.c || (q.k > 0 && (!q.a || !q.b)) || q.ldc < q.n || (q.k > 0 && (q.lda < q.k || q.ldb < q.n))) {
            delete p;
            return set_error(FG_ERR_INVALID, "grouped GEMM: bad pointer or leading dimension in problem " + std::to_string(i));
        }
        if (q.m > (1 << 30) || q.n > (1 << 30) || q.k > (1 << 30) ||
            (p->kind == 1 && q.k > (dtype == FG_I8 ? 131072 : 65536))) {
            delete p;
            return set_error(FG_ERR_UNSUPPORTED, "grouped GEMM: problem " + std::to_string(i) + " too large");
        }
        if (q.k == 0) {
            p->zeros.push_back({q.c, q.m, q.n, q.ldc, 0});
            continue;
        }
        order.push_back(static_cast<int>(i));
    }
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return table[x].k > table[y].k; });
    const int np = static_cast<int>(order.size());

    // layout of the single device allocation
    const int nmaps = p->kind == 2 ? 4 : 2;
    const int bm = p->kind == 0 ? 64 : 128, bn = p->kind == 0 ? 64 : 128;
    std::vector<GroupedProblem> probs(np);
    std::vector<PrepSeg> segs;
    long long arena = 0;
    struct Opnd {
        const void* src;
        long long off0 = -1, off1 = -1, ld;
    };
    std::vector<Opnd> oa(np), ob(np);
    long long tiles = 0;
    for (int j = 0; j < np; ++j) {
        const fg_problem& q = table[order[j]];
        GroupedProblem& g = probs[j];
        g.M = static_cast<int>(q.m);
        g.N = static_cast<int>(q.n);
        g.K = static_cast<int>(q.k);
        g.tiles_m = static_cast<int>((q.m + bm - 1) / bm);
        g.tiles_n = static_cast<int>((q.n + bn - 1) / bn);
        g.tile_start = tiles;
        tiles += (long long)g.tiles_m * g.tiles_n;
        g.C = q.c;
        g.ldc = q.ldc;
        oa[j].src = q.a;
        ob[j].src = q.b;
        if (p->kind == 1) {
            g.k_blocks = static_cast<int>((q.k + 127) / 128);
            if ((reinterpret_cast<uintptr_t>(q.a) & 15) || (q.lda % 16)) {
                oa[j].ld = rup(q.k, 16);
                oa[j].off0 = arena;
                arena = rup(arena + oa[j].ld * q.m, 256);
            } else {
                oa[j].ld = q.lda;
            }
            if ((reinterpret_cast<uintptr_t>(q.b) & 15) || (q.ldb % 16)) {
                ob[j].ld = rup(q.n, 16);
                ob[j].off0 = arena;
                arena = rup(arena + ob[j].ld * q.k, 256);
            } else {
                ob[j].ld = q.ldb;
            }
        } else if (p->kind == 2) {
            g.k_blocks = static_cast<int>((q.k + 63) / 64);
            oa[j].ld = rup(q.k, 8);
            oa[j].off0 = arena;
            arena = rup(arena + 2 * oa[j].ld * q.m, 256);
            oa[j].off1 = arena;
            arena = rup(arena + 2 * oa[j].ld * q.m, 256);
            ob[j].ld = rup(q.n, 8);
            ob[j].off0 = arena;
            arena = rup(arena + 2 * ob[j].ld * q.k, 256);
            ob[j].off1 = arena;
            arena = rup(arena + 2 * ob[j].ld * q.k, 256);
        } else {
            g.k_blocks = static_cast<int>((q.k + 15) / 16);
            oa[j].ld = q.lda;
            ob[j].ld = q.ldb;
        }
    }
    p->total_tiles = tiles;
    const size_t sz_probs = rup(sizeof(GroupedProblem) * std::max(np, 1), 256);
    const size_t sz_maps = rup(sizeof(CUtensorMap) * nmaps * std::max(np, 1), 256);
    const size_t sz_ptrs = rup((2 * sizeof(void*) + 2 * sizeof(long long)) * std::max(np, 1), 256);
    // segments are built after the arena base is known
    const size_t max_segs = static_cast<size_t>(2 * np);
    const size_t sz_segs = rup(sizeof(PrepSeg) * std::max<size_t>(max_segs, 1), 256);
    const size_t total = sz_probs + sz_maps + sz_ptrs + sz_segs + arena;
    cudaError_t e = cudaMalloc(&p->mem, total);
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete p;
        return set_error(FG_ERR_OOM, "grouped plan: allocation of " + std::to_string(total) + " bytes failed");
    }
    char* base = static_cast<char*>(p->mem);
    GroupedProblem* d_probs = reinterpret_cast<GroupedProblem*>(base);
    CUtensorMap* d_maps = reinterpret_cast<CUtensorMap*>(base + sz_probs);
    char* d_ptrs = base + sz_probs + sz_maps;
    p->d_segs = reinterpret_cast<PrepSeg*>(d_ptrs + sz_ptrs);
    char* d_arena = d_ptrs + sz_ptrs + sz_segs;

    std::vector<CUtensorMap> maps(static_cast<size_t>(nmaps) * np);
    long long seg_total = 0;
    auto add_seg = [&](const void* src, void* d0, void* d1, long long rows, long long cols,
                       long long lds, long long ldd, int op) {
        PrepSeg sgm{src, d0, d1, rows, cols, lds, ldd, seg_total, op};
        segs.push_back(sgm);
        seg_total += rows * ldd;
    };
    fg_status fs = FG_OK;
    for (int j = 0; j < np && fs == FG_OK; ++j) {
        const fg_problem& q = table[order[j]];
        if (p->kind == 1) {
            const void* pa = q.a;
            const void* pb = q.b;
            if (oa[j].off0 >= 0) {
                pa = d_arena + oa[j].off0;
                add_seg(q.a, const_cast<void*>(pa), nullptr, q.m, q.k, q.lda, oa[j].ld, 0);
            }
            if (ob[j].off0 >= 0) {
                pb = d_arena + ob[j].off0;
                add_seg(q.b, const_cast<void*>(pb), nullptr, q.k, q.n, q.ldb, ob[j].ld, 0);
            }
            uint64_t da[2] = {(uint64_t)q.k, (uint64_t)q.m}, sa[1] = {(uint64_t)oa[j].ld};
            uint64_t db[2] = {(uint64_t)q.n, (uint64_t)q.k}, sb[1] = {(uint64_t)ob[j].ld};
            uint32_t box[2] = {128, 128};
            fs = encode_map(&maps[2 * j], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, pa, da, sa, box);
            if (fs == FG_OK) fs = encode_map(&maps[2 * j + 1], CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, pb, db, sb, box);
        } else if (p->kind == 2) {
            void* ah = d_arena + oa[j].off0;
            void* al = d_arena + oa[j].off1;
            void* bh = d_arena + ob[j].off0;
            void* bl = d_arena + ob[j].off1;
            add_seg(q.a, ah, al, q.m, q.k, q.lda, oa[j].ld, 1);
            add_seg(q.b, bh, bl, q.k, q.n, q.ldb, ob[j].ld, 1);
            uint64_t da[2] = {(uint64_t)q.k, (uint64_t)q.m}, sa[1] = {(uint64_t)(2 * oa[j].ld)};
            uint64_t db[2] = {(uint64_t)q.n, (uint64_t)q.k}, sb[1] = {(uint64_t)(2 * ob[j].ld)};
            uint32_t boxa[2] = {64, 128}, boxb[2] = {64, 64};
            fs = encode_map(&maps[4 * j + 0], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, ah, da, sa, boxa);
            if (fs == FG_OK) fs = encode_map(&maps[4 * j + 1], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, al, da, sa, boxa);
            if (fs == FG_OK) fs = encode_map(&maps[4 * j + 2], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, bh, db, sb, boxb);
            if (fs == FG_OK) fs = encode_map(&maps[4 * j + 3], CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, bl, db, sb, boxb);
        }
    }
    if (fs != FG_OK) {
        cudaFree(p->mem);
        delete p;
        return fs;
    }
    p->nseg = static_cast<int>(segs.size());
    p->prep_total = seg_total;
    // tables -> device (synchronous: the host vectors go away)
    cudaError_t ce = cudaSuccess;
    if (np) ce = cudaMemcpyAsync(d_probs, probs.data(), sizeof(GroupedProblem) * np, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && !maps.empty())
        ce = cudaMemcpyAsync(d_maps, maps.data(), sizeof(CUtensorMap) * maps.size(), cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && !segs.empty())
        ce = cudaMemcpyAsync(p->d_segs, segs.data(), sizeof(PrepSeg) * segs.size(), cudaMemcpyHostToDevice, st);
    std::vector<const void*> pa(np), pb(np);
    std::vector<long long> la(np), lb(np);
    for (int j = 0; j < np; ++j) {
        pa[j] = oa[j].src;
        pb[j] = ob[j].src;
        la[j] = oa[j].ld;
        lb[j] = ob[j].ld;
    }
    const void** d_pa = reinterpret_cast<const void**>(d_ptrs);
    const void** d_pb = d_pa + std::max(np, 1);
    long long* d_la = reinterpret_cast<long long*>(d_pb + std::max(np, 1));
    long long* d_lb = d_la + std::max(np, 1);
    if (ce == cudaSuccess && np) ce = cudaMemcpyAsync(d_pa, pa.data(), sizeof(void*) * np, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && np) ce = cudaMemcpyAsync(d_pb, pb.data(), sizeof(void*) * np, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && np) ce = cudaMemcpyAsync(d_la, la.data(), sizeof(long long) * np, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess && np) ce = cudaMemcpyAsync(d_lb, lb.data(), sizeof(long long) * np, cudaMemcpyHostToDevice, st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) {
        cudaFree(p->mem);
        delete p;
        return cuda_error(ce, "grouped plan upload");
    }
    p->targs.problems = d_probs;
    p->targs.maps = d_maps;
    p->targs.count = np;
    p->targs.total_tiles = tiles;
    p->targs.status = ctx->d_status;
    p->targs.timeout_ns = 4000000000ull;
    p->targs.kchunk = 2;
    if (p->kind == 1) {
        p->targs.ops[0] = TcOp{0, 0, 0, dtype == FG_I8 ? 1 : 0, 1};
        fs = set_smem_attr<CfgGroupedI8>();
    } else if (p->kind == 2) {
        p->targs.ops[0] = TcOp{1, 0, 0, 1, 1};
        p->targs.ops[1] = TcOp{0, 1, 0, 1, 1};
        p->targs.ops[2] = TcOp{0, 0, 0, 1, 1};
        fs = set_smem_attr<CfgGroupedBf16>();
    }
    p->sargs.problems = d_probs;
    p->sargs.a = d_pa;
    p->sargs.b = d_pb;
    p->sargs.lda = d_la;
    p->sargs.ldb = d_lb;
    p->sargs.count = np;
    p->sargs.total_tiles = tiles;
    if (fs != FG_OK) {
        cudaFree(p->mem);
        delete p;
        return fs;
    }
    *out = p;
    return FG_OK;
}

static void free_plan(fg_grouped_plan* p) {
    if (!p) return;
    cudaSetDevice(p->ctx->device);
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->mem) cudaFree(p->mem);
    delete p;
}

}  // namespace fgrt

using namespace fgrt;

extern "C" {

fg_status fg_gemm_grouped(fg_ctx* ctx, fg_dtype dtype, fg_mode mode, const fg_problem* table,
                          size_t count, fg_stream stream) {
    if (!ctx) return set_error(FG_ERR_INVALID, "null context");
    cudaStream_t st = stream_of(ctx, stream);
    fg_grouped_plan* p = nullptr;
    FG_TRY(build_plan(ctx, dtype, mode, table, count, st, &p));
    fg_status s = launch_plan(p, st);
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
    cudaStream_t st = stream_of(ctx, stream);
    fg_grouped_plan* p = nullptr;
    FG_TRY(build_plan(ctx, dtype, mode, table, count, st, &p));
    // Capture the launch sequence once; runs replay it.
    cudaStream_t cap;
    cudaError_t e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    fg_status s = FG_OK;
    if (e == cudaSuccess) {
        const int prof = g_prof_on.exchange(0);  // no event records inside the graph
        s = launch_plan(p, cap);
        g_prof_on.store(prof);
        cudaGraph_t graph = nullptr;
        cudaError_t e2 = cudaStreamEndCapture(cap, &graph);
        if (e2 == cudaSuccess) {
            p->graph = graph;
            e2 = cudaGraphInstantiate(&p->exec, graph, 0);
        }
        if (e == cudaSuccess) e = e2;
    }
    cudaStreamDestroy(cap);
    if (s != FG_OK || e != cudaSuccess) {
        free_plan(p);
        return s != FG_OK ? s : cuda_error(e, "grouped plan capture");
    }
    *out = p;
    return FG_OK;
}

fg_status fg_grouped_plan_run(fg_grouped_plan* p, fg_stream stream) {
    if (!p) return set_error(FG_ERR_INVALID, "null plan");
    FG_CUDA(cudaSetDevice(p->ctx->device));
    cudaStream_t st = stream_of(p->ctx, stream);
    ProfScope prof(p->kind == 0 ? "grouped_plan_ffma" : p->kind == 1 ? "grouped_plan_i8" : "grouped_plan_3xbf16", st);
    FG_CUDA(cudaGraphLaunch(p->exec, st));
    prof.stop();
    count_launch(1 + (p->nseg > 0 ? 1 : 0) + p->zeros.size());
    return FG_OK;
}

fg_status fg_grouped_plan_destroy(fg_grouped_plan* p) {
    free_plan(p);
    return FG_OK;
}

}  // extern "C"
