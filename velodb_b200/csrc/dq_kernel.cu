// Device consumer of the persistent command queue (job format: dq.cuh).
//
// One CTA of 256 threads per SM slot (two per SM) loops: thread 0 decides
// what the CTA does next, the CTA does it.
//   WORK    thread 0 holds a claimed item of the global item sequence that
//           lies inside a published job: it finds the job (a short forward
//           walk over the device job table) and the step (binary search over
//           the job's steps), claims the following item ahead, and waits --
//           bounded on %globaltimer -- until the job has completed every item
//           of the earlier steps (and, for the first step, until every job
//           the job was ordered after is complete).  The CTA stages the
//           step's argument block in shared memory and runs the tile.
//   INGEST  the CTA whose claim is the first unpublished item copies the
//           next job from the host-mapped ring into the device job table and
//           publishes its items.
//   WAIT    nothing to run yet: back off with __nanosleep.
//   EXIT    every published job is done and either the host asked the
//           queue to stop or nothing arrived for the idle time.
// Every wait is bounded: a dependency wait that runs out records
// VELO_ETIMEDOUT in the job's status and the item runs anyway, so the
// launch always terminates; the host reads the status with the job.
#include "dq.cuh"
#include "net_host.cuh"

namespace velo {

using DqLI2 = LiTypes<2>::Rec;
using DqLI3 = LiTypes<3>::Rec;
using NetKP = Net<RowKP, 8, 4>;
using NetKPM = Net<RowKPM, 8, 4>;
using NetLI2 = Net<DqLI2, 8, 4>;
using NetLI3 = Net<DqLI3, 8, 3>;
using NetJ = Net<JRec, 8, 4>;
using NetR3 = Net<Rec3, 8, 3>;
using NetR3K2 = Net<Rec3K2, 8, 3>;

constexpr size_t dq_max(size_t a, size_t b) { return a > b ? a : b; }
// dynamic shared memory of the consumer: the largest step
constexpr size_t DQ_SMEM = dq_max(
    dq_max(dq_max(NetKP::smem_bytes_sort(), NetKPM::smem_bytes_compact()),
           dq_max(NetLI2::smem_bytes_compact(), NetLI3::smem_bytes_compact())),
    dq_max(dq_max(NetJ::smem_bytes_compact(), dq_max(NetR3::smem_bytes_sort(), NetR3K2::smem_bytes_compact())),
           dq_max(dq_max(LiTypes<3>::Seg::SMEM, JSEG_TOPK_SMEM),
                  dq_max((size_t)2 * TK_RED_ROWS * 8, (size_t)FILL_TS * 8))));
static_assert(DQ_SMEM <= 110 * 1024, "two consumer CTAs fit on an SM");
static_assert(TK_RED_ROWS / 2 % DQ_THREADS == 0, "top-k rounds: whole compare-exchanges a thread");

enum : int { DQ_A_WORK = 0, DQ_A_INGEST = 1, DQ_A_WAIT = 2, DQ_A_EXIT = 3 };

__device__ __forceinline__ uint64_t dq_now()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned long long dq_acq_sys(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long dq_acq(const unsigned long long* p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned int dq_acq32(const unsigned int* p)
{
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template <class T>
__device__ __forceinline__ T dq_vol(const T& x)
{
    return *const_cast<const volatile T*>(&x);
}

// ---- one work item -------------------------------------------------------------

template <class A>
__device__ __forceinline__ const A& dq_arg(const unsigned char* s_args)
{
    return *reinterpret_cast<const A*>(s_args);
}

// shared-memory scratch of the small block-wide scans (carved per step)
struct DqSmall {
    alignas(16) unsigned char b[1024];
};

__device__ void dq_run(const DqStep& step, const unsigned char* s_args, uint32_t tile, char* sm, DqSmall& sx)
{
    uint32_t* tmp = reinterpret_cast<uint32_t*>(sx.b);
    const size_t nt = step.ntiles;
    switch (step.kind) {
    case DQ_K_NOP:
        break;
    // ---- networks
    case DQ_K_SORT_KP: {
        const auto& A = dq_arg<DqNetArgs<RowKP>>(s_args);
        NetKP::run<true>(A.c, A.g, step.pass, nullptr, (int)tile, sm);
        break;
    }
    case DQ_K_COMPACT_KPM: {
        const auto& A = dq_arg<DqNetArgs<RowKPM>>(s_args);
        NetKPM::run<false>(A.c, A.g, step.pass, A.prefix, (int)tile, sm);
        break;
    }
    case DQ_K_SORT_LI2: {
        const auto& A = dq_arg<DqNetArgs<DqLI2>>(s_args);
        NetLI2::run<true>(A.c, A.g, step.pass, nullptr, (int)tile, sm);
        break;
    }
    case DQ_K_COMPACT_LI2: {
        const auto& A = dq_arg<DqNetArgs<DqLI2>>(s_args);
        NetLI2::run<false>(A.c, A.g, step.pass, A.prefix, (int)tile, sm);
        break;
    }
    case DQ_K_SORT_LI3: {
        const auto& A = dq_arg<DqNetArgs<DqLI3>>(s_args);
        NetLI3::run<true>(A.c, A.g, step.pass, nullptr, (int)tile, sm);
        break;
    }
    case DQ_K_COMPACT_LI3: {
        const auto& A = dq_arg<DqNetArgs<DqLI3>>(s_args);
        NetLI3::run<false>(A.c, A.g, step.pass, A.prefix, (int)tile, sm);
        break;
    }
    case DQ_K_SORT_JREC: {
        const auto& A = dq_arg<DqNetArgs<JRec>>(s_args);
        NetJ::run<true>(A.c, A.g, step.pass, nullptr, (int)tile, sm);
        break;
    }
    case DQ_K_COMPACT_JREC: {
        const auto& A = dq_arg<DqNetArgs<JRec>>(s_args);
        NetJ::run<false>(A.c, A.g, step.pass, A.prefix, (int)tile, sm);
        break;
    }
    case DQ_K_SORT_REC3: {
        const auto& A = dq_arg<DqNetArgs<Rec3>>(s_args);
        NetR3::run<true>(A.c, A.g, step.pass, nullptr, (int)tile, sm);
        break;
    }
    case DQ_K_SORT_REC3K2: {
        const auto& A = dq_arg<DqNetArgs<Rec3K2>>(s_args);
        NetR3K2::run<true>(A.c, A.g, step.pass, nullptr, (int)tile, sm);
        break;
    }
    case DQ_K_COMPACT_REC3K2: {
        const auto& A = dq_arg<DqNetArgs<Rec3K2>>(s_args);
        NetR3K2::run<false>(A.c, A.g, step.pass, A.prefix, (int)tile, sm);
        break;
    }
    // ---- mark counts and their scan
    case DQ_K_COUNT_KPM: {
        const auto& A = dq_arg<DqCountArgs<RowKPM>>(s_args);
        count_tile<RowKPM>(A.c, A.n, A.lt, (int)tile, A.counts, tmp);
        break;
    }
    case DQ_K_COUNT_JREC: {
        const auto& A = dq_arg<DqCountArgs<JRec>>(s_args);
        count_tile<JRec>(A.c, A.n, A.lt, (int)tile, A.counts, tmp);
        break;
    }
    case DQ_K_COUNT_REC3K2: {
        const auto& A = dq_arg<DqCountArgs<Rec3K2>>(s_args);
        count_tile<Rec3K2>(A.c, A.n, A.lt, (int)tile, A.counts, tmp);
        break;
    }
    case DQ_K_SCAN_TILES: {
        const auto& A = dq_arg<DqScanArgs>(s_args);
        scan_tiles(A.counts, A.ntiles, A.prefix, A.d_count, tmp);
        break;
    }
    // ---- filter + group-by
    case DQ_K_LI_PACK2:
    case DQ_K_LI_PACK3: {
        const auto& A = dq_arg<DqLiPackArgs>(s_args);
        if (step.kind == DQ_K_LI_PACK2)
            li_pack_tile<2>(A.c, A.p, A.prm, A.n, A.n_rec, A.lt, A.w[0], A.w[1], A.w[2], A.counts, tile, tmp);
        else
            li_pack_tile<3>(A.c, A.p, A.prm, A.n, A.n_rec, A.lt, A.w[0], A.w[1], A.w[2], A.counts, tile, tmp);
        break;
    }
    case DQ_K_SEG_SUMMARY2: {
        const auto& A = dq_arg<DqSegArgs>(s_args);
        LiTypes<2>::Seg::tile_summary(A.w, (int)tile, A.aggs, A.runs, A.prm, sm);
        break;
    }
    case DQ_K_SEG_SUMMARY3: {
        const auto& A = dq_arg<DqSegArgs>(s_args);
        LiTypes<3>::Seg::tile_summary(A.w, (int)tile, A.aggs, A.runs, A.prm, sm);
        break;
    }
    case DQ_K_SEG_CARRIES2: {
        const auto& A = dq_arg<DqSegArgs>(s_args);
        LiTypes<2>::Seg::carries(A.aggs, A.runs, A.ntiles, A.carry, A.tail_prefix, A.n_groups, sm);
        break;
    }
    case DQ_K_SEG_CARRIES3: {
        const auto& A = dq_arg<DqSegArgs>(s_args);
        LiTypes<3>::Seg::carries(A.aggs, A.runs, A.ntiles, A.carry, A.tail_prefix, A.n_groups, sm);
        break;
    }
    case DQ_K_SEG_EMIT2: {
        const auto& A = dq_arg<DqSegArgs>(s_args);
        LiTypes<2>::Seg::emit(A.w, (int)tile, A.ntiles, A.aggs, A.carry, A.tail_prefix, A.G, A.tile_out, A.prm, sm);
        break;
    }
    case DQ_K_SEG_EMIT3: {
        const auto& A = dq_arg<DqSegArgs>(s_args);
        LiTypes<3>::Seg::emit(A.w, (int)tile, A.ntiles, A.aggs, A.carry, A.tail_prefix, A.G, A.tile_out, A.prm, sm);
        break;
    }
    case DQ_K_SEG_FINISH: {
        const auto& A = dq_arg<DqSegArgs>(s_args);
        LiTypes<3>::Seg::finish(A.tile_out, A.ntiles, A.G, A.out, (int)tile);
        if (tile == 0 && threadIdx.x == 0) {
            A.d_counts[0] = *A.d_rows;
            A.d_counts[1] = *A.n_groups;
        }
        break;
    }
    // ---- join + group-by + top-k
    case DQ_K_JOIN_PACK: {
        const auto& A = dq_arg<DqJoinPackArgs>(s_args);
        join_pack_body(A.dk, A.dd, A.nd, A.ff, A.fp, A.nf, A.date_hi, A.price_hi, A.n_rec, A.w0, A.w1, tile, nt);
        break;
    }
    case DQ_K_JFILL_SUMMARY: {
        const auto& A = dq_arg<DqJFillArgs>(s_args);
        DimCarry* s8 = reinterpret_cast<DimCarry*>(sx.b);
        fill_summary_tile(A.w0, A.tile_last, tile, s8, reinterpret_cast<int*>(s8 + FILL_THREADS / 32));
        break;
    }
    case DQ_K_JFILL_CARRIES: {
        const auto& A = dq_arg<DqJFillArgs>(s_args);
        fill_carries_body(A.tile_last, A.ntiles, A.carry, reinterpret_cast<DimCarry*>(sx.b));
        break;
    }
    case DQ_K_JFILL_APPLY: {
        const auto& A = dq_arg<DqJFillArgs>(s_args);
        fill_apply_tile(A.w0, A.carry, tile, reinterpret_cast<uint64_t*>(sm), reinterpret_cast<DimCarry*>(sx.b));
        break;
    }
    case DQ_K_JSEG_SUMMARY: {
        const auto& A = dq_arg<DqJSegArgs>(s_args);
        JSeg::tile_summary(A.c.w, (int)tile, A.aggs, A.runs, JoinAgg::Params {}, sm);
        break;
    }
    case DQ_K_JSEG_CARRIES: {
        const auto& A = dq_arg<DqJSegArgs>(s_args);
        JSeg::carries(A.aggs, A.runs, A.ntiles, A.carry, A.tail_prefix, A.n_groups, sm);
        break;
    }
    case DQ_K_JSEG_EMIT_TOPK: {
        const auto& A = dq_arg<DqJSegArgs>(s_args);
        jseg_emit_topk_tile(A.c, A.ntiles, A.aggs, A.carry, A.cand, A.out0, A.out1, tile, sm);
        break;
    }
    case DQ_K_TOPK_REDUCE: {
        const auto& A = dq_arg<DqTopkArgs>(s_args);
        topk_reduce_tile<TK_RED_ROWS / 2 / DQ_THREADS>(A.in0, A.in1, A.rn, A.c, A.out0, A.out1, tile, sm);
        break;
    }
    case DQ_K_TOPK_OUT: {
        const auto& A = dq_arg<DqTopkArgs>(s_args);
        topk_out_body(A.in0, A.in1, A.k, A.out, A.n_groups, A.n_joined, A.d_counts);
        break;
    }
    // ---- union-sort operators
    case DQ_K_UFILL_SUM_JOIN:
    case DQ_K_UFILL_SUM_GATHER: {
        const auto& A = dq_arg<DqUFillArgs>(s_args);
        FillCarry* s8 = reinterpret_cast<FillCarry*>(sx.b);
        int* i8 = reinterpret_cast<int*>(s8 + FL_THREADS / 32);
        if (step.kind == DQ_K_UFILL_SUM_JOIN)
            fill_sum_tile<JoinFill>(A.w0, A.w1, A.w2, A.tl, tile, s8, i8);
        else
            fill_sum_tile<GatherFill>(A.w0, A.w1, A.w2, A.tl, tile, s8, i8);
        break;
    }
    case DQ_K_UFILL_SCAN: {
        const auto& A = dq_arg<DqUFillArgs>(s_args);
        fill_scan_body(A.tl, A.ntiles, A.carry, reinterpret_cast<FillCarry*>(sx.b));
        break;
    }
    case DQ_K_UFILL_APPLY_JOIN:
    case DQ_K_UFILL_APPLY_GATHER: {
        const auto& A = dq_arg<DqUFillArgs>(s_args);
        FillCarry* w33 = reinterpret_cast<FillCarry*>(sx.b);
        uint32_t* t33 = reinterpret_cast<uint32_t*>(w33 + 33);
        if (step.kind == DQ_K_UFILL_APPLY_JOIN)
            fill_apply_tile<JoinFill>(A.w0, A.w1, A.w2, A.carry, A.d_stat, tile, w33, t33);
        else
            fill_apply_tile<GatherFill>(A.w0, A.w1, A.w2, A.carry, A.d_stat, tile, w33, t33);
        break;
    }
    case DQ_K_OJOIN_PACK: {
        const auto& A = dq_arg<DqOJoinArgs>(s_args);
        ojoin_pack_body(A.bk, A.bm, A.bn, A.pk, A.pm, A.pn, A.key64, A.rows, A.w0, A.w1, A.w2, tile, nt);
        break;
    }
    case DQ_K_OJOIN_OUT: {
        const auto& A = dq_arg<DqOJoinArgs>(s_args);
        ojoin_out_body(A.w1, A.w2, A.pn, A.ob, A.op, tile, nt);
        break;
    }
    case DQ_K_JOIN_COUNTS: {
        const auto& A = dq_arg<DqOJoinArgs>(s_args);
        if (threadIdx.x == 0)
            join_counts_body(A.n_joined, A.dups, A.d_counts);
        break;
    }
    case DQ_K_OGATHER_PACK: {
        const auto& A = dq_arg<DqOGatherArgs>(s_args);
        ogather_pack_body(A.table, A.tn, A.rids, A.rn, A.rows, A.w0, A.w1, A.w2, tile, nt);
        break;
    }
    case DQ_K_OGATHER_OUT: {
        const auto& A = dq_arg<DqOGatherArgs>(s_args);
        ogather_out_body(A.w1, A.rn, A.out, tile, nt);
        break;
    }
    // ---- element-wise operators
    case DQ_K_PERMUTE: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        const int64_t* idx = static_cast<const int64_t*>(A.idx);
        switch (A.bytes) {
        case 1: permute_body((uint8_t*)A.out, (const uint8_t*)A.in, idx, A.n, tile, nt); break;
        case 2: permute_body((uint16_t*)A.out, (const uint16_t*)A.in, idx, A.n, tile, nt); break;
        case 4: permute_body((uint32_t*)A.out, (const uint32_t*)A.in, idx, A.n, tile, nt); break;
        default: permute_body((uint64_t*)A.out, (const uint64_t*)A.in, idx, A.n, tile, nt); break;
        }
        break;
    }
    case DQ_K_GATHER: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        const int32_t* idx = static_cast<const int32_t*>(A.idx);
        switch (A.bytes) {
        case 1: gather_body((uint8_t*)A.out, (const uint8_t*)A.in, idx, A.mask, A.n, tile, nt); break;
        case 2: gather_body((uint16_t*)A.out, (const uint16_t*)A.in, idx, A.mask, A.n, tile, nt); break;
        case 4: gather_body((uint32_t*)A.out, (const uint32_t*)A.in, idx, A.mask, A.n, tile, nt); break;
        default: gather_body((uint64_t*)A.out, (const uint64_t*)A.in, idx, A.mask, A.n, tile, nt); break;
        }
        break;
    }
    case DQ_K_COMPARE_EQ: {
        // element type: value = velo_type
        const auto& A = dq_arg<DqElemArgs>(s_args);
        uint8_t* o = static_cast<uint8_t*>(A.out);
        switch (A.value) {
        case VELO_TINYINT: compare_eq_body((const int8_t*)A.in, (const int8_t*)A.in2, o, A.n, tile, nt); break;
        case VELO_SMALLINT: compare_eq_body((const int16_t*)A.in, (const int16_t*)A.in2, o, A.n, tile, nt); break;
        case VELO_INTEGER:
        case VELO_DATE: compare_eq_body((const int32_t*)A.in, (const int32_t*)A.in2, o, A.n, tile, nt); break;
        case VELO_BIGINT: compare_eq_body((const int64_t*)A.in, (const int64_t*)A.in2, o, A.n, tile, nt); break;
        case VELO_FLOAT: compare_eq_body((const float*)A.in, (const float*)A.in2, o, A.n, tile, nt); break;
        case VELO_DOUBLE: compare_eq_body((const double*)A.in, (const double*)A.in2, o, A.n, tile, nt); break;
        default: fill_u8_body(o, 0, A.n, tile, nt); break;
        }
        break;
    }
    case DQ_K_COMPOSE: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        compose_body((const uint32_t*)A.in, (const uint32_t*)A.idx, (uint32_t*)A.out, A.n, tile, nt);
        break;
    }
    case DQ_K_FILL_U8: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        fill_u8_body((uint8_t*)A.out, (uint8_t)A.value, A.n, tile, nt);
        break;
    }
    case DQ_K_SCATTER_COUNT: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        scatter_count_tile(A.mask, A.n, (uint32_t*)A.out, tile, tmp);
        break;
    }
    case DQ_K_SCATTER_WRITE: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        scatter_write_tile(A.mask, A.n, (const uint32_t*)A.in, (int32_t*)A.out, tile, tmp);
        break;
    }
    case DQ_K_SHUFFLE_PACK: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        shuffle_pack_body((const uint32_t*)A.in, A.n, A.np, A.counter, A.key, (uint64_t*)A.out, (uint32_t*)A.idx, tile,
                          nt);
        break;
    }
    case DQ_K_COPY_U32: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        copy_u32_body((uint32_t*)A.out, (const uint32_t*)A.in, A.n, tile, nt);
        break;
    }
    // ---- served three-way join chain, result delivery
    case DQ_K_RANGE_MASK_I32: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        range_mask_body((const int32_t*)A.in, A.n, (int32_t)A.lo, (int32_t)A.hi, (uint8_t*)A.out, tile, nt);
        break;
    }
    case DQ_K_RANGE_MASK_I64: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        range_mask_body((const int64_t*)A.in, A.n, (int64_t)A.lo, (int64_t)A.hi, (uint8_t*)A.out, tile, nt);
        break;
    }
    case DQ_K_ROWID_KEYS: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        rowid_keys_body((const int64_t*)A.in, A.n, A.lo, (int64_t*)A.out, (uint8_t*)A.idx, tile, nt);
        break;
    }
    case DQ_K_ROWID_RIDS: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        rowid_rids_body((const int64_t*)A.in, A.n, A.value, (uint32_t*)A.out, tile, nt);
        break;
    }
    case DQ_K_SUM_U64: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        sum_u64_body((const uint64_t*)A.in, A.n, (unsigned long long*)A.out, tile, nt,
                     reinterpret_cast<unsigned long long*>(sx.b));
        break;
    }
    case DQ_K_SET_WORDS: {
        const auto& A = dq_arg<DqElemArgs>(s_args);
        for (size_t i = (size_t)tile * DQ_THREADS + threadIdx.x; i < A.n; i += nt * DQ_THREADS)
            static_cast<uint64_t*>(A.out)[i] = A.key;
        break;
    }
    case DQ_K_COPY_WORDS: {
        const auto& A = dq_arg<DqCopyArgs>(s_args);
        for (uint32_t i = threadIdx.x; i < A.words; i += DQ_THREADS)
            A.dst[i] = __ldcg(A.src + i);
        // the destination may be host memory: make the words visible there
        // before the job's completion is
        __threadfence_system();
        break;
    }
    default:
        break;
    }
}

// ---- thread 0: the next action ---------------------------------------------------

struct DqLocal {
    unsigned long long cursor; // lowest job that can hold this CTA's next item
    uint64_t idle_since;
    uint32_t backoff;
};

struct alignas(16) DqShared {
    unsigned long long next;  // the claim this CTA holds
    unsigned long long seq;   // job to ingest
    DqJobHdr hdr;             // header of the job being ingested
    DqStep step;
    uint32_t ds;              // device slot of the item's job
    uint32_t tile;            // item index within the step
    uint32_t rel;             // item index within the job
    int action;
};

__device__ __forceinline__ void dq_backoff(DqLocal& L)
{
    __nanosleep(L.backoff);
    L.backoff = L.backoff < 4096 ? L.backoff * 2 : 4096;
}

// job holding claimed item x (x < published); false if none is found
__device__ __forceinline__ bool dq_find_job(const DqParams& a, unsigned long long x, DqLocal& L, uint32_t& ds,
                                            unsigned long long& begin, uint32_t& nsteps, uint64_t& after)
{
    DqState* st = a.st;
    const unsigned long long ing = dq_vol(st->ingested);
    // jobs more than a host ring behind the newest are complete (the host
    // reuses a ring slot only after its job completed), so they cannot
    // hold an unfinished item
    const unsigned long long lo = ing > (unsigned long long)DQ_HOST_RING ? ing - DQ_HOST_RING + 1 : 1;
    if (L.cursor < lo)
        L.cursor = lo;
    for (; L.cursor <= ing; L.cursor++) {
        const uint32_t d = (uint32_t)((L.cursor - 1) % DQ_DEV_RING);
        const DqSlot& sl = st->slot[d];
        if (dq_acq(&sl.seq) != L.cursor)
            continue;
        const unsigned long long b = dq_vol(sl.begin);
        const unsigned int n = dq_vol(sl.nitems);
        if (x >= b && x < b + n) {
            ds = d;
            begin = b;
            const DqJob& J = a.table[d];
            nsteps = __ldcg(&J.h.nsteps);
            after = __ldcg(&J.h.after);
            return true;
        }
    }
    return false;
}

__device__ int dq_decide(const DqParams& a, DqLocal& L, DqShared& S)
{
    DqState* st = a.st;
    const unsigned long long x = S.next;
    const unsigned long long pub = dq_acq(&st->published);
    if (x < pub) {
        uint32_t ds = 0, nsteps = 0;
        unsigned long long begin = 0;
        uint64_t after = 0;
        if (!dq_find_job(a, x, L, ds, begin, nsteps, after)) {
            // the job table lost the item's job: stop the grid rather than
            // run unknown work (never expected); the host fails every
            // pending job when it sees the fault word
            atomicExch(&st->exiting, 1);
            *const_cast<volatile int*>(&a.ctl->fault) = 1;
            __threadfence_system();
            return DQ_A_EXIT;
        }
        const DqJob& J = a.table[ds];
        const uint32_t rel = (uint32_t)(x - begin);
        uint32_t lo = 0, hi = nsteps - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (__ldcg(&J.steps[mid].begin) <= rel)
                lo = mid;
            else
                hi = mid - 1;
        }
        DqStep step;
        {
            const uint4* src = reinterpret_cast<const uint4*>(&J.steps[lo]);
            uint4* dst = reinterpret_cast<uint4*>(&step);
            dst[0] = __ldcg(src);
            dst[1] = __ldcg(src + 1);
        }
        S.step = step;
        S.ds = ds;
        S.rel = rel;
        S.tile = rel - step.begin;
        // claim the following item now, so the claim overlaps this item
        S.next = atomicAdd(&st->next_item, 1ull);
        const uint64_t t0 = dq_now();
        bool late = false;
        if (lo == 0 && after != 0) {
            uint32_t spins = 0;
            while (dq_acq(&st->complete_below) <= after) {
                if (dq_now() - t0 > a.wait_ns) {
                    late = true;
                    break;
                }
                __nanosleep(spins++ < 64 ? 64 : 512);
            }
        }
        if (step.begin != 0) {
            uint32_t spins = 0;
            while (dq_acq32(&st->slot[ds].done) < step.begin) {
                if (dq_now() - t0 > a.wait_ns) {
                    late = true;
                    break;
                }
                __nanosleep(spins++ < 64 ? 32 : 256);
            }
        }
        if (late)
            atomicCAS(&st->slot[ds].status, (int)VELO_OK, (int)VELO_ETIMEDOUT);
        L.idle_since = 0;
        L.backoff = 32;
        return DQ_A_WORK;
    }
    if (dq_vol(st->exiting))
        return DQ_A_EXIT;
    if (x != pub) {
        // another CTA holds the first unpublished item and polls the host
        dq_backoff(L);
        return DQ_A_WAIT;
    }
    const unsigned long long head = dq_acq_sys(&a.ctl->head);
    if (head > dq_vol(st->ingested)) {
        if (atomicCAS(&st->lock, 0, 1) == 0) {
            if (dq_vol(st->exiting)) {
                atomicExch(&st->lock, 0);
                return DQ_A_EXIT;
            }
            S.seq = dq_vol(st->ingested) + 1;
            return DQ_A_INGEST;
        }
        dq_backoff(L);
        return DQ_A_WAIT;
    }
    const uint64_t now = dq_now();
    if (L.idle_since == 0)
        L.idle_since = now;
    if (now - L.idle_since > a.wait_ns) {
        // published items neither finished nor claimable for a whole wait
        // limit: the job table is inconsistent (never expected); stop
        atomicExch(&st->exiting, 1);
        *const_cast<volatile int*>(&a.ctl->fault) = 1;
        __threadfence_system();
        return DQ_A_EXIT;
    }
    if (dq_vol(a.ctl->stop) != 0 || now - L.idle_since > a.idle_ns) {
        if (atomicCAS(&st->lock, 0, 1) == 0) {
            const bool drained = dq_acq_sys(&a.ctl->head) == dq_vol(st->ingested)
                && dq_acq(&st->completed_items) == dq_acq(&st->published);
            if (drained) {
                st->exiting = 1;
                __threadfence();
            }
            atomicExch(&st->lock, 0);
            if (drained)
                return DQ_A_EXIT;
        }
    }
    dq_backoff(L);
    return DQ_A_WAIT;
}

// ---- the CTA: ingest a job ------------------------------------------------------

__device__ void dq_ingest(const DqParams& a, DqShared& S)
{
    DqState* st = a.st;
    const unsigned long long seq = S.seq;
    const DqJob* src = a.ring + (seq - 1) % DQ_HOST_RING;
    DqJob* dst = a.table + (seq - 1) % DQ_DEV_RING;
    if (threadIdx.x < 4) {
        // the header, uncached: the host rewrites this ring slot for later jobs
        reinterpret_cast<uint4*>(&S.hdr)[threadIdx.x] = __ldcv(reinterpret_cast<const uint4*>(&src->h) + threadIdx.x);
    }
    __syncthreads();
    const DqJobHdr h = S.hdr;
    const bool ok = h.seq == seq && h.nsteps >= 1 && h.nsteps <= (uint32_t)DQ_MAX_STEPS && h.nitems >= 1
        && h.arg_bytes <= (uint32_t)DQ_ARG_BYTES;
    if (ok) {
        const uint4* ss = reinterpret_cast<const uint4*>(src->steps);
        uint4* sd = reinterpret_cast<uint4*>(dst->steps);
        for (uint32_t i = threadIdx.x; i < h.nsteps * 2; i += DQ_THREADS)
            __stcg(sd + i, __ldcv(ss + i));
        const uint4* as = reinterpret_cast<const uint4*>(src->args);
        uint4* ad = reinterpret_cast<uint4*>(dst->args);
        for (uint32_t i = threadIdx.x; i < (h.arg_bytes + 15) / 16; i += DQ_THREADS)
            __stcg(ad + i, __ldcv(as + i));
        if (threadIdx.x < 4)
            __stcg(reinterpret_cast<uint4*>(&dst->h) + threadIdx.x, reinterpret_cast<const uint4*>(&h)[threadIdx.x]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t ds = (uint32_t)((seq - 1) % DQ_DEV_RING);
        DqSlot& sl = st->slot[ds];
        if (!ok) {
            // a malformed job (never written by this library's planner): a
            // one-item job that reports VELO_EINVAL
            __stcg(&dst->h.nsteps, 1u);
            __stcg(&dst->h.after, (uint64_t)0);
            DqStep nop {};
            nop.kind = DQ_K_NOP;
            nop.ntiles = 1;
            const uint4* np = reinterpret_cast<const uint4*>(&nop);
            __stcg(reinterpret_cast<uint4*>(&dst->steps[0]), np[0]);
            __stcg(reinterpret_cast<uint4*>(&dst->steps[0]) + 1, np[1]);
        }
        const unsigned int nitems = ok ? h.nitems : 1u;
        sl.complete = 0;
        sl.done = 0;
        sl.status = ok ? (int)VELO_OK : (int)VELO_EINVAL;
        sl.nitems = nitems;
        sl.begin = dq_vol(st->published);
        __threadfence();
        sl.seq = seq;
        __threadfence();
        st->ingested = seq;
        __threadfence();
        atomicAdd(&st->published, (unsigned long long)nitems);
        __threadfence();
        atomicExch(&st->lock, 0);
    }
}

// ---- thread 0: count an item done ----------------------------------------------

__device__ void dq_complete(const DqParams& a, uint32_t ds)
{
    DqState* st = a.st;
    DqSlot& sl = st->slot[ds];
    __threadfence();
    const unsigned int old = atomicAdd(&sl.done, 1u);
    if (old + 1 == dq_vol(sl.nitems)) {
        const unsigned long long seq = dq_vol(sl.seq);
        const int hs = (int)((seq - 1) % DQ_HOST_RING);
        a.ctl->status[hs] = dq_vol(sl.status);
        __threadfence_system();
        *const_cast<volatile unsigned long long*>(&a.ctl->done_seq[hs]) = seq;
        __threadfence_system();
        sl.complete = 1;
        __threadfence();
        // advance the "every job below is complete" mark over finished jobs
        for (int it = 0; it < DQ_DEV_RING; it++) {
            const unsigned long long c = dq_acq(&st->complete_below);
            const DqSlot& cs = st->slot[(c - 1) % DQ_DEV_RING];
            if (dq_acq(&cs.seq) != c || dq_acq32(&cs.complete) == 0)
                break;
            atomicCAS(&st->complete_below, c, c + 1);
        }
    }
    atomicAdd(&st->completed_items, 1ull);
}

__global__ void __launch_bounds__(DQ_THREADS, 2) k_dq(DqParams a)
{
    extern __shared__ __align__(16) char sm[];
    __shared__ __align__(16) unsigned char s_args[DQ_STEP_ARG_MAX];
    __shared__ DqSmall s_small;
    __shared__ __align__(16) DqShared S;
    VELO_TRACE_KERNEL(TS_K_DQ);
    DqLocal L { 1, 0, 32 };
    if (threadIdx.x == 0)
        S.next = atomicAdd(&a.st->next_item, 1ull);
    for (;;) {
        if (threadIdx.x == 0)
            S.action = dq_decide(a, L, S);
        __syncthreads();
        const int act = S.action;
        if (act == DQ_A_EXIT)
            return;
        if (act == DQ_A_WAIT) {
            __syncthreads();
            continue;
        }
        if (act == DQ_A_INGEST) {
            dq_ingest(a, S);
            __syncthreads();
            continue;
        }
        const DqStep step = S.step;
        const uint32_t ds = S.ds;
        {
            const uint4* src = reinterpret_cast<const uint4*>(a.table[ds].args + step.arg);
            for (int i = threadIdx.x; i < DQ_STEP_ARG_MAX / 16; i += DQ_THREADS)
                reinterpret_cast<uint4*>(s_args)[i] = __ldcg(src + i);
        }
        VELO_TRACE_WORK(S.rel);
        __syncthreads();
        dq_run(step, s_args, S.tile, sm, s_small);
        __syncthreads();
        if (threadIdx.x == 0)
            dq_complete(a, ds);
    }
}

// state before a launch: a fresh queue (first launch) or a resumed one
// (claims of the previous grid are void; nothing is in flight)
__global__ void k_dq_reset(DqState* st, int fresh)
{
    if (threadIdx.x != 0)
        return;
    if (fresh) {
        st->published = 0;
        st->ingested = 0;
        st->completed_items = 0;
        st->complete_below = 1;
        st->launches = 0;
        for (int i = 0; i < DQ_DEV_RING; i++) {
            st->slot[i].seq = 0;
            st->slot[i].complete = 0;
        }
    }
    st->next_item = st->published;
    st->lock = 0;
    st->exiting = 0;
    st->launches++;
    __threadfence();
}

velo_status dq_launch(const DqParams& a, bool fresh, cudaStream_t stream, int* grid_out)
{
    static int done[64] = {};
    static int grid_of[64] = {};
    int dev = 0;
    VELO_CUDA_TRY(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= 64)
        return einval("device ordinal out of range");
    velo_status rc = ensure_smem(k_dq, DQ_SMEM, done);
    if (rc != VELO_OK)
        return rc;
    if (grid_of[dev] == 0) {
        int per = 0, sms = 0;
        VELO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_dq, DQ_THREADS, DQ_SMEM),
                      "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        VELO_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "cudaDeviceGetAttribute");
        if (per < 1)
            return einval("persistent command queue: the consumer kernel does not fit on an SM");
        grid_of[dev] = per * sms;
    }
    k_dq_reset<<<1, 32, 0, stream>>>(a.st, fresh ? 1 : 0);
    k_dq<<<grid_of[dev], DQ_THREADS, DQ_SMEM, stream>>>(a);
    VELO_CUDA_TRY(cudaGetLastError(), "persistent command queue launch");
    if (grid_out)
        *grid_out = grid_of[dev];
    return VELO_OK;
}

} // namespace velo
