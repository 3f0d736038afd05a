// Device consumer of the persistent command queue (job format: dq.cuh).
//
// One CTA of 256 threads per SM slot (two per SM) loops: warp 0 decides what
// the CTA does next, the CTA does it.
//   WORK    warp 0 took an item of a job's open step: its lanes read the
//           claim words of up to 32 open jobs at once (oldest first) and the
//           oldest job with an unclaimed item wins a compare-and-swap.  The
//           CTA stages the step's argument block in shared memory, runs the
//           tile and counts it done; the step's last item opens the job's
//           next step, or completes the job and reports it to the host.  An
//           item is only ever taken when its step is open, so no CTA waits
//           on another item.
//   INGEST  a new job is in the host-mapped ring: copy it into the device
//           job table and open its first step.
//   WAIT    nothing to take: back off with __nanosleep.
//   EXIT    no open job, and the host asked the queue to stop or nothing
//           arrived for the idle time.
// A job ordered after others opens its first step only once they are all
// complete.  If open jobs offer nothing to take for a whole wait limit the
// grid stops and reports a fault word to the host, so the launch always
// terminates.
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
                  dq_max((size_t)2 * TK_RED_ROWS * 8, (size_t)FILL_TS_PAD * 8))));
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

// claim: the item's inputs (what the earlier steps wrote) become visible
__device__ __forceinline__ unsigned long long dq_add_acquire(unsigned long long* p, unsigned long long v)
{
    unsigned long long old;
    asm volatile("atom.acquire.gpu.global.add.u64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    return old;
}

// item done: the CTA's writes are released with the count, and the step's
// last item acquires every other item's
__device__ __forceinline__ unsigned int dq_add_acq_rel(unsigned int* p, unsigned int v)
{
    unsigned int old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

// opening a step releases everything the step's items wrote
__device__ __forceinline__ void dq_exch_release(unsigned long long* p, unsigned long long v)
{
    unsigned long long old;
    asm volatile("atom.release.gpu.global.exch.b64 %0, [%1], %2;" : "=l"(old) : "l"(p), "l"(v) : "memory");
    (void)old;
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

// ---- warp 0: the next action ------------------------------------------------------

struct DqLocal {
    uint64_t idle_since;
    uint32_t backoff;
};

struct alignas(16) DqShared {
    DqJobHdr hdr;       // header of the job being ingested
    DqStep step;        // step of the claimed item
    unsigned long long seq; // job to ingest
    uint32_t ds;        // device slot of the item's job
    uint32_t sidx;      // index of the step in its job
    uint32_t tile;      // item index within the step
    uint32_t nsteps;    // steps of the item's job
    int action;
    int cont;           // 1: the CTA keeps the next step's first item (set after an item)
};

// Idle CTAs back off exponentially (a sleep lasts up to twice the request):
// to 1 us while jobs are open, so that the items of a newly opened step are
// taken quickly, and to 4 us when nothing is open.  A CTA that finishes a
// step's last item takes the next step's first item itself.
__device__ __forceinline__ void dq_backoff(DqLocal& L, bool open_jobs)
{
    const uint32_t cap = open_jobs ? 1024u : 4096u;
    __nanosleep(L.backoff < cap ? L.backoff : cap);
    L.backoff = L.backoff < cap ? L.backoff * 2 : cap;
}

__device__ __forceinline__ bool dq_claimable(unsigned long long claim)
{
    const unsigned long long step = claim >> 48, nt = (claim >> 24) & 0xFFFFFFull, k = claim & 0xFFFFFFull;
    return step != DQ_STEP_DONE && k < nt;
}

// Warp 0: takes a ready item of the oldest open job.  The lanes read the
// claim words of 32 consecutive jobs at once; the oldest claimable job's lane
// adds one to its claim word and owns item k if the word it replaced still
// had k below the step's item count (a lost race leaves the count past the
// end, which nothing reads, and the warp looks again).  Claims only follow a
// read that saw an unclaimed item, so the count exceeds the step's items by
// at most one per CTA.
__device__ bool dq_claim(const DqParams& a, DqShared& S)
{
    DqState* st = a.st;
    const int lane = threadIdx.x & 31;
    unsigned long long lo = 0, hi = 0;
    if (lane == 0) {
        lo = dq_vol(st->complete_below);
        hi = dq_vol(st->ingested);
    }
    lo = __shfl_sync(0xFFFFFFFFu, lo, 0);
    hi = __shfl_sync(0xFFFFFFFFu, hi, 0);
    for (unsigned long long base = lo; base <= hi; base += 32) {
        const unsigned long long j = base + (unsigned long long)lane;
        const uint32_t ds = (uint32_t)((j - 1) % DQ_DEV_RING);
        DqSlot* sl = &st->slot[ds];
        unsigned long long claim = 0;
        bool ok = false;
        if (j <= hi) {
            const ulonglong2 v = __ldcg(reinterpret_cast<const ulonglong2*>(sl)); // { claim, seq }
            claim = v.x;
            ok = v.y == j && dq_claimable(claim);
            if (ok && (claim >> 48) == 0 && (claim & 0xFFFFFFull) == 0) {
                // the job's first item waits for the jobs it is ordered after
                const uint64_t after = __ldcg(&a.table[ds].h.after);
                ok = after == 0 || after < lo;
            }
        }
        unsigned mask = __ballot_sync(0xFFFFFFFFu, ok);
        for (int tries = 0; mask != 0 && tries < 64; tries++) {
            const int leader = __ffs(mask) - 1;
            bool got = false;
            if (lane == leader) {
                const unsigned long long old = dq_add_acquire(&sl->claim, 1ull);
                got = dq_claimable(old);
                claim = old;
                ok = false;
            }
            got = __shfl_sync(0xFFFFFFFFu, got ? 1 : 0, leader) != 0;
            if (got) {
                if (lane == leader) {
                    const uint32_t sidx = (uint32_t)(claim >> 48);
                    S.ds = ds;
                    S.sidx = sidx;
                    S.tile = (uint32_t)(claim & 0xFFFFFFull);
                    S.nsteps = __ldcg(&a.table[ds].h.nsteps);
                    const uint4* src = reinterpret_cast<const uint4*>(&a.table[ds].steps[sidx]);
                    reinterpret_cast<uint4*>(&S.step)[0] = __ldcg(src);
                    reinterpret_cast<uint4*>(&S.step)[1] = __ldcg(src + 1);
                }
                __syncwarp();
                return true;
            }
            mask = __ballot_sync(0xFFFFFFFFu, ok);
        }
    }
    return false;
}

// lane 0 of warp 0, nothing claimable: ingest, exit or back off
__device__ int dq_idle(const DqParams& a, DqLocal& L, DqShared& S)
{
    DqState* st = a.st;
    if (dq_vol(st->exiting))
        return DQ_A_EXIT;
    const uint64_t now = dq_now();
    // host memory is read over the bus: the ring head and the stop word at
    // most once every two microseconds for the whole grid, by whichever idle
    // CTA wins the poll, with plain (relaxed) loads; the others read the
    // device copy of the stop word.  Polling loads are relaxed throughout:
    // ordering comes from the claim and done atomics and the ingest's fence.
    const unsigned long long last = dq_vol(st->last_poll);
    if (now - last > 2000 && atomicCAS(&st->last_poll, last, (unsigned long long)now) == last) {
        st->host_stop = dq_vol(a.ctl->stop);
        const unsigned long long head = dq_vol(a.ctl->head);
        if (head > dq_vol(st->ingested) && atomicCAS(&st->lock, 0, 1) == 0) {
            if (dq_vol(st->exiting)) {
                atomicExch(&st->lock, 0);
                return DQ_A_EXIT;
            }
            // another CTA may have ingested since `head` was compared: the
            // next job must still be published
            const unsigned long long ing = dq_vol(st->ingested);
            if (head > ing) {
                S.seq = ing + 1;
                L.idle_since = 0;
                return DQ_A_INGEST;
            }
            atomicExch(&st->lock, 0);
        }
    }
    if (L.idle_since == 0)
        L.idle_since = now;
    const bool open_jobs = dq_vol(st->complete_below) <= dq_vol(st->ingested);
    if (open_jobs) {
        if (now - L.idle_since > a.wait_ns) {
            // open jobs, yet nothing to take for a whole wait limit: the job
            // table is inconsistent (never expected); stop, and let the host
            // fail the pending jobs
            atomicExch(&st->exiting, 1);
            *const_cast<volatile int*>(&a.ctl->fault) = 1;
            __threadfence_system();
            return DQ_A_EXIT;
        }
    } else if (dq_vol(st->host_stop) != 0 || now - L.idle_since > a.idle_ns) {
        if (atomicCAS(&st->lock, 0, 1) == 0) {
            const bool drained = dq_acq_sys(&a.ctl->head) == dq_vol(st->ingested)
                && dq_acq(&st->complete_below) > dq_vol(st->ingested);
            if (drained) {
                st->exiting = 1;
                __threadfence();
                // tell the host this launch is leaving: a job it publishes
                // from now on needs a new launch
                *const_cast<volatile unsigned long long*>(&a.ctl->exited_launch) = dq_vol(st->launches);
                __threadfence_system();
            }
            atomicExch(&st->lock, 0);
            if (drained)
                return DQ_A_EXIT;
        }
    }
    dq_backoff(L, open_jobs);
    return DQ_A_WAIT;
}

// warp 0
__device__ int dq_decide(const DqParams& a, DqLocal& L, DqShared& S)
{
    if (dq_claim(a, S)) {
        L.idle_since = 0;
        L.backoff = 32;
        return DQ_A_WORK;
    }
    int act = DQ_A_WAIT;
    if ((threadIdx.x & 31) == 0)
        act = dq_idle(a, L, S);
    return __shfl_sync(0xFFFFFFFFu, act, 0);
}

// ---- the CTA: ingest a job ------------------------------------------------------

__device__ void dq_ingest(const DqParams& a, DqShared& S)
{
    DqState* st = a.st;
    const unsigned long long seq = S.seq;
    const DqJob* src = a.ring + (seq - 1) % DQ_HOST_RING;
    DqJob* dst = a.table + (seq - 1) % DQ_DEV_RING;
    // the job was written before the head that announced it
    asm volatile("fence.acq_rel.sys;" ::: "memory");
    if (threadIdx.x < 4) {
        // the header, uncached: the host rewrites this ring slot for later jobs
        reinterpret_cast<uint4*>(&S.hdr)[threadIdx.x] = __ldcv(reinterpret_cast<const uint4*>(&src->h) + threadIdx.x);
    }
    __syncthreads();
    const DqJobHdr h = S.hdr;
    const bool ok = h.seq == seq && h.nsteps >= 1 && h.nsteps <= (uint32_t)DQ_MAX_STEPS
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
            DqJobHdr bad {};
            bad.seq = seq;
            bad.nsteps = 1;
            bad.nitems = 1;
            DqStep nop {};
            nop.kind = DQ_K_NOP;
            nop.ntiles = 1;
            for (int i = 0; i < 4; i++)
                __stcg(reinterpret_cast<uint4*>(&dst->h) + i, reinterpret_cast<const uint4*>(&bad)[i]);
            __stcg(reinterpret_cast<uint4*>(&dst->steps[0]), reinterpret_cast<const uint4*>(&nop)[0]);
            __stcg(reinterpret_cast<uint4*>(&dst->steps[0]) + 1, reinterpret_cast<const uint4*>(&nop)[1]);
        }
        __threadfence();
        sl.done = 0;
        sl.status = ok ? (int)VELO_OK : (int)VELO_EINVAL;
        sl.nsteps = ok ? h.nsteps : 1u;
        sl.claim = dq_claim_word(0, __ldcg(&dst->steps[0].ntiles));
        __threadfence();
        sl.seq = seq;
        __threadfence();
        st->ingested = seq;
        __threadfence();
        atomicExch(&st->lock, 0);
    }
}

// ---- thread 0: count an item done ----------------------------------------------

// Returns true when this CTA keeps the next step's first item: the CTA that
// completes a step opens the next one with item 0 already taken, and S
// describes that item.
__device__ bool dq_complete(const DqParams& a, DqShared& S)
{
    DqState* st = a.st;
    DqSlot& sl = st->slot[S.ds];
    const unsigned int old = dq_add_acq_rel(&sl.done, 1u);
    if (old + 1 != S.step.ntiles)
        return false;
    // the step's last item: open the next step, or complete the job
    sl.done = 0;
    const uint32_t next = S.sidx + 1;
    if (next < S.nsteps) {
        const uint4* src = reinterpret_cast<const uint4*>(&a.table[S.ds].steps[next]);
        reinterpret_cast<uint4*>(&S.step)[0] = __ldcg(src);
        reinterpret_cast<uint4*>(&S.step)[1] = __ldcg(src + 1);
        dq_exch_release(&sl.claim, dq_claim_word(next, S.step.ntiles) + 1);
        S.sidx = next;
        S.tile = 0;
        return true;
    }
    const unsigned long long seq = dq_vol(sl.seq);
    const int hs = (int)((seq - 1) % DQ_HOST_RING);
    a.ctl->status[hs] = dq_vol(sl.status);
    __threadfence_system();
    *const_cast<volatile unsigned long long*>(&a.ctl->done_seq[hs]) = seq;
    __threadfence_system();
    atomicExch(&sl.claim, dq_claim_word(DQ_STEP_DONE, 0));
    __threadfence();
    // advance the "every job below is complete" mark over finished jobs
    for (int it = 0; it < DQ_DEV_RING; it++) {
        const unsigned long long c = dq_acq(&st->complete_below);
        const DqSlot& cs = st->slot[(c - 1) % DQ_DEV_RING];
        if (dq_acq(&cs.seq) != c || (dq_acq(&cs.claim) >> 48) != DQ_STEP_DONE)
            break;
        atomicCAS(&st->complete_below, c, c + 1);
    }
    return false;
}

__global__ void __launch_bounds__(DQ_THREADS, 2) k_dq(DqParams a)
{
    extern __shared__ __align__(16) char sm[];
    __shared__ __align__(16) unsigned char s_args[DQ_STEP_ARG_MAX];
    __shared__ DqSmall s_small;
    __shared__ __align__(16) DqShared S;
    VELO_TRACE_KERNEL(TS_K_DQ);
    DqLocal L { 0, 32 };
    bool have = false; // S already holds this CTA's next item
    for (;;) {
        if (!have) {
            if (threadIdx.x < 32) {
                const int act = dq_decide(a, L, S);
                if (threadIdx.x == 0)
                    S.action = act;
            }
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
        }
        const DqStep step = S.step;
        {
            const uint4* src = reinterpret_cast<const uint4*>(a.table[S.ds].args + step.arg);
            for (int i = threadIdx.x; i < DQ_STEP_ARG_MAX / 16; i += DQ_THREADS)
                reinterpret_cast<uint4*>(s_args)[i] = __ldcg(src + i);
        }
        VELO_TRACE_WORK(step.begin + S.tile);
        __syncthreads();
        dq_run(step, s_args, S.tile, sm, s_small);
        __syncthreads();
        if (threadIdx.x == 0)
            S.cont = dq_complete(a, S) ? 1 : 0;
        __syncthreads();
        have = S.cont != 0;
    }
}

// state before a launch: a fresh queue (first launch) or a resumed one
__global__ void k_dq_reset(DqState* st, int fresh)
{
    if (threadIdx.x != 0)
        return;
    if (fresh) {
        st->ingested = 0;
        st->complete_below = 1;
        st->host_stop = 0;
        st->last_poll = 0;
        st->launches = 0;
        for (int i = 0; i < DQ_DEV_RING; i++) {
            st->slot[i].seq = 0;
            st->slot[i].claim = dq_claim_word(DQ_STEP_DONE, 0);
        }
    }
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
