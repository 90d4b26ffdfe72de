// numeric_rows.cu - step 3 (values) of the tiled SpGEMM, one CTA per C tile row.
//
// Work unit: C tile row I (16 scalar rows).  Gustavson over tiles (reference
// step4, src/spgemm-cpu.h:284-367, reorganised row-wise as the reference's
// Super16 path does for its candidate step, src/super16_symbolic.cuh:973-1073):
//   C(I, :) = sum over K in A.row(I) of A(I,K) * B(K, :)
//
// Warp-specialised pipeline.  A producer warp streams the 16 scalar rows of
// B tile row K - the row-k segments of every tile of B.row(K) in column
// order, i.e. B's CSR rows 16K..16K+15, contiguous in HBM - into a ring of
// shared-memory stages with TMA bulk copies (cp.async.bulk, completion on the
// stage's "full" mbarrier); eight consumer warps wait on "full", compute and
// release the stage on its "empty" mbarrier.  Every wait is bounded.  The
// plans of the K steps are computed up front in one parallel round, so the
// producer issues copies back to back.
//
// Consumers own output rows: warp w owns rows 2w and 2w+1 of the tile row, so
// no two warps touch the same accumulator entry and the K loop needs no CTA
// barrier.  The warp walks its A entries (r, k, a) of A(I,K) in order; for
// each, the lanes take consecutive entries of B row k (one product per lane,
// distinct columns, so no conflicts) and add a*b into the accumulator.  Every
// output is summed in the fixed order K ascending, k ascending (the
// reference's order) without atomics: results are bitwise reproducible.
//
// Accumulator: one FP64 slot per structural entry of the C tile row, laid out
// in CSR order (row, tile, column).  The position of (tile s, row r, col c) is
// base[s][r] + popc(mask[s][r] >> (16 - c)), with base and mask packed in one
// word and tile column -> slot read from a byte table.  The fused tile2csr
// write-out is a contiguous copy per row.
//
// Dense pairs (nnz(A tile) * nnz(B tile) >= cutoff) are flagged per (K step,
// C slot), skipped by the scalar loop and computed afterwards on the FP64
// tensor cores: a warp expands both tiles in shared memory and runs 16
// mma.sync.m8n8k4.f64 over the 8x4 (A) / 4x8 (B) sub-tiles; warp w takes the
// C tiles with slot % 8 == w, pairs in K order.
//
// Tile rows whose accumulator or C tile count exceeds the shared budget are
// processed in windows of C tiles, long A tile rows in chunks of K steps; B
// row groups larger than a stage are read from global memory directly.
#include "rtt_internal.cuh"

namespace rtt
{
namespace
{

constexpr int NW = 8;                 // consumer warps
constexpr int NR_THREADS = NW * 32 + 32;
constexpr int NSTAGE = 5;             // ring depth
constexpr int ACC_CAP = 2304;         // FP64 accumulator slots per window
constexpr int SLOT_CAP = 128;         // C tiles per window
constexpr int BE_CAP = 448;           // B row entries per stage
constexpr int KCH = 64;               // K steps per chunk
constexpr int AV_CAP = 640;           // staged A entries of a chunk
constexpr int SPAN_CAP = 4096;        // tile-column span covered by the slot table
constexpr long long WAIT_LIMIT = 1ll << 22;

struct Stage
{
    double val[BE_CAP + 2];
    int col[BE_CAP + 8];
    int rp[TD + 8];
    // header written by the producer before it arrives on "full"
    int off_val, off_col, off_rp, pad;
};

struct RowSmem
{
    double acc[ACC_CAP];
    Stage st[NSTAGE];
    double aval[AV_CAP];
    uint8_t acol[AV_CAP];
    uint8_t aptr[KCH * TD];
    int atnnz[KCH + 1];
    // per K step of the chunk
    int p_K[KCH], p_e0[KCH], p_e1[KCH], p_staged[KCH];
    uint32_t dense[KCH][SLOT_CAP / 32]; // (K step, C slot) pairs for the tensor cores
    // C structure of the window
    uint32_t cm[SLOT_CAP * TD];          // (acc base << 16) | row mask
    int cJ[SLOT_CAP];
    uint8_t slot8[SPAN_CAP];             // tile column - Jlo -> slot (255 = none)
    int rowacc0[TD + 1];
    int rowcsr0[TD];
    int rowrun[TD];
    int win_nnz;
    unsigned long long full[NSTAGE];
    unsigned long long empty[NSTAGE];
};

struct DenseSmem
{
    double da[NW][TD * TD];
    double db[NW][TD * TD];
};

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(unsigned long long *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// 1-D bulk copy, no multicast.  dst, src and bytes are multiples of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes,
                                         unsigned long long *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Bounded wait on an mbarrier phase; records an error and returns false when
// the poll limit is reached.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t parity, int *err)
{
    const uint32_t addr = smem_u32(bar);
    for (long long it = 0; it < WAIT_LIMIT; ++it)
    {
        uint32_t done;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(done)
                     : "r"(addr), "r"(parity)
                     : "memory");
        if (done)
            return true;
    }
    set_error(err, DERR_WINDOW);
    return false;
}

__device__ __forceinline__ uintptr_t down16(uintptr_t p) { return p & ~(uintptr_t)15; }
__device__ __forceinline__ uintptr_t up16(uintptr_t p) { return (p + 15) & ~(uintptr_t)15; }

__device__ __forceinline__ void dmma_m8n8k4(double &d0, double &d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// Producer: fill stage st with B's scalar rows 16K..16K+nr-1 (one thread).
__device__ __forceinline__ void produce(const DevTiles &B, const RowSmem &S, int ai, Stage &st,
                                       unsigned long long *full)
{
    if (!S.p_staged[ai])
    {
        mbar_arrive(full); // consumers read this K step from global memory
        return;
    }
    const int r0 = S.p_K[ai] * TD, r1 = min(r0 + TD, B.m);
    const int e0 = S.p_e0[ai], e1 = S.p_e1[ai];
    const uintptr_t v_lo = down16((uintptr_t)(B.csr_val + e0)), v_hi = up16((uintptr_t)(B.csr_val + e1));
    const uintptr_t c_lo = down16((uintptr_t)(B.csr_col + e0)), c_hi = up16((uintptr_t)(B.csr_col + e1));
    const uintptr_t r_lo = down16((uintptr_t)(B.csr_rowptr + r0));
    const uintptr_t r_hi = up16((uintptr_t)(B.csr_rowptr + r1 + 1));
    st.off_val = (int)(((uintptr_t)(B.csr_val + e0) - v_lo) / 8);
    st.off_col = (int)(((uintptr_t)(B.csr_col + e0) - c_lo) / 4);
    st.off_rp = (int)(((uintptr_t)(B.csr_rowptr + r0) - r_lo) / 4);
    const uint32_t bytes = (uint32_t)((v_hi - v_lo) + (c_hi - c_lo) + (r_hi - r_lo));
    mbar_expect_tx(full, bytes);
    bulk_g2s(st.val, (const void *)v_lo, (uint32_t)(v_hi - v_lo), full);
    bulk_g2s(st.col, (const void *)c_lo, (uint32_t)(c_hi - c_lo), full);
    bulk_g2s(st.rp, (const void *)r_lo, (uint32_t)(r_hi - r_lo), full);
}

// C slot of tile column J in the current window, -1 if absent.
__device__ __forceinline__ int slot_of(const RowSmem &S, int J, int Jlo, int Jhi, int nW,
                                       bool table)
{
    if (J < Jlo || J > Jhi)
        return -1;
    if (table)
    {
        const int s = S.slot8[J - Jlo];
        return s == 255 ? -1 : s;
    }
    const int s = lower_bound(S.cJ, 0, nW, J);
    return (s < nW && S.cJ[s] == J) ? s : -1;
}

// 3 CTAs per SM fit the shared budget without the dense buffers, 2 with them.
template <bool DMMA>
__global__ void __launch_bounds__(NR_THREADS, DMMA ? 2 : 3)
    k_numeric_rows(DevTiles A, DevTiles B, int tilem, long long nnzC,
                   const int *__restrict__ c_tile_ptr, const int *__restrict__ c_tile_col,
                   const uint16_t *__restrict__ c_mask, const int *__restrict__ c_tile_nnz,
                   uint8_t *__restrict__ c_ptr, uint8_t *__restrict__ c_colb,
                   double *__restrict__ c_val, const int *__restrict__ csr_rowptr,
                   int *__restrict__ csr_col, double *__restrict__ csr_val, int cutoff, int stage_b,
                   int safe, long long *counters, int *err)
{
    extern __shared__ __align__(128) unsigned char dyn[];
    RowSmem &S = *reinterpret_cast<RowSmem *>(dyn);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool producer = warp == NW;
    const int I = blockIdx.x;
    if (I >= tilem)
        return;
    const int a0 = __ldg(A.tile_ptr + I), a1 = __ldg(A.tile_ptr + I + 1);
    const int nA = a1 - a0;
    const int cs0 = __ldg(c_tile_ptr + I), cs1 = __ldg(c_tile_ptr + I + 1);
    if (cs0 == cs1 || nA == 0)
        return; // no C tiles in this tile row (uniform)
    if (tid < TD)
        S.rowrun[tid] = 0;
    if (tid == 0)
    {
        for (int s = 0; s < NSTAGE; ++s)
        {
            mbar_init(&S.full[s], 1);
            mbar_init(&S.empty[s], NW);
        }
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    __syncthreads();
    const int nrows = min(TD, A.m - I * TD);
    long long n_dense = 0, n_fma = 0;
    int gk = 0; // K steps through the stage ring so far (ring position)
    bool failed = false;

    for (int w0 = cs0; w0 < cs1;)
    {
        // ---- window of C tiles [w0, w1): the longest run with <= SLOT_CAP
        // tiles and <= ACC_CAP entries (scanned per-tile offsets make the
        // admissible tiles a prefix; a barrier count finds its length)
        const int base_nnz = __ldg(c_tile_nnz + w0);
        bool ok = false;
        if (tid < SLOT_CAP && w0 + tid < cs1)
            ok = __ldg(c_tile_nnz + w0 + tid + 1) - base_nnz <= ACC_CAP;
        const int nW = __syncthreads_count(ok);
        if (nW == 0)
        {
            if (tid == 0)
                set_error(err, DERR_NUM_BOUNDS); // a C tile holds at most 256 entries
            return;
        }
        const int w1 = w0 + nW;
        if (tid == 0)
            S.win_nnz = __ldg(c_tile_nnz + w1) - base_nnz;
        for (int i = tid; i < nW * TD; i += NR_THREADS)
            S.cm[i] = __ldg(c_mask + (size_t)w0 * TD + i);
        for (int i = tid; i < nW; i += NR_THREADS)
            S.cJ[i] = __ldg(c_tile_col + w0 + i);
        for (int i = tid; i < SPAN_CAP / 4; i += NR_THREADS)
            reinterpret_cast<uint32_t *>(S.slot8)[i] = 0xFFFFFFFFu;
        __syncthreads();
        const int Jlo = S.cJ[0], Jhi = S.cJ[nW - 1];
        const bool table = Jhi - Jlo < SPAN_CAP;
        if (table)
            for (int i = tid; i < nW; i += NR_THREADS)
                S.slot8[S.cJ[i] - Jlo] = (uint8_t)i;
        // per-row prefix over the window's tiles (warp w: rows 2w, 2w+1)
        if (!producer)
        {
            for (int rr = 0; rr < 2; ++rr)
            {
                const int r = warp * 2 + rr;
                int run = 0;
                for (int s0 = 0; s0 < nW; s0 += 32)
                {
                    const int s = s0 + lane;
                    const uint32_t m = s < nW ? S.cm[s * TD + r] : 0u;
                    const int v = __popc(m);
                    const int incl = warp_incl_scan(v);
                    if (s < nW)
                        S.cm[s * TD + r] = ((uint32_t)(run + incl - v) << 16) | m;
                    run += __shfl_sync(FULL, incl, 31);
                }
                if (lane == 0)
                    S.rowacc0[r + 1] = run;
            }
        }
        __syncthreads();
        if (tid == 0)
        {
            S.rowacc0[0] = 0;
            for (int r = 0; r < TD; ++r)
                S.rowacc0[r + 1] += S.rowacc0[r];
        }
        __syncthreads();
        if (tid < nrows && csr_rowptr != nullptr)
            S.rowcsr0[tid] = __ldg(csr_rowptr + I * TD + tid) + S.rowrun[tid];
        for (int i = tid; i < nW * TD; i += NR_THREADS)
            S.cm[i] += (uint32_t)S.rowacc0[i & 15] << 16;
        for (int i = tid; i < S.win_nnz; i += NR_THREADS)
            S.acc[i] = 0.0;

        for (int c0 = 0; c0 < nA; c0 += KCH)
        {
            const int nK = min(KCH, nA - c0);
            const int ab = a0 + c0;
            // ---- chunk set-up: A tiles and K-step plans (one parallel round)
            const int av0 = __ldg(A.tile_nnz + ab), av1 = __ldg(A.tile_nnz + ab + nK);
            const bool a_staged = (av1 - av0) <= AV_CAP;
            if (a_staged)
                for (int i = tid; i < av1 - av0; i += NR_THREADS)
                {
                    S.aval[i] = __ldg(A.val + av0 + i);
                    S.acol[i] = A.col[av0 + i];
                }
            for (int i = tid; i < nK * TD; i += NR_THREADS)
                S.aptr[i] = A.ptr[(size_t)ab * TD + i];
            for (int i = tid; i <= nK; i += NR_THREADS)
                S.atnnz[i] = __ldg(A.tile_nnz + ab + i) - av0;
            for (int ai = tid; ai < nK; ai += NR_THREADS)
            {
                const int K = __ldg(A.tile_col + ab + ai);
                const int r0 = K * TD, r1 = min(r0 + TD, B.m);
                const int e0 = __ldg(B.csr_rowptr + r0), e1 = __ldg(B.csr_rowptr + r1);
                // a bulk copy moves whole 16-byte granules: stage only when the
                // rounded ranges stay inside B's arrays (caller-owned memory)
                const bool inside =
                    down16((uintptr_t)(B.csr_val + e0)) >= (uintptr_t)B.csr_val &&
                    up16((uintptr_t)(B.csr_val + e1)) <= (uintptr_t)(B.csr_val + B.nnz) &&
                    down16((uintptr_t)(B.csr_col + e0)) >= (uintptr_t)B.csr_col &&
                    up16((uintptr_t)(B.csr_col + e1)) <= (uintptr_t)(B.csr_col + B.nnz) &&
                    down16((uintptr_t)(B.csr_rowptr + r0)) >= (uintptr_t)B.csr_rowptr &&
                    up16((uintptr_t)(B.csr_rowptr + r1 + 1)) <= (uintptr_t)(B.csr_rowptr + B.m + 1);
                S.p_K[ai] = K;
                S.p_e0[ai] = e0;
                S.p_e1[ai] = e1;
                S.p_staged[ai] = stage_b && inside && e1 > e0 && (e1 - e0) <= BE_CAP;
            }
            if constexpr (DMMA)
                for (int i = tid; i < nK * (SLOT_CAP / 32); i += NR_THREADS)
                    (&S.dense[0][0])[i] = 0u;
            __syncthreads();
            if constexpr (DMMA)
            {
                // classify tile pairs: nnz(A(I,K)) * nnz(B(K,J)) >= cutoff
                for (int ai = warp; ai < nK; ai += NW + 1)
                {
                    const int K = S.p_K[ai];
                    const int acnt = S.atnnz[ai + 1] - S.atnnz[ai];
                    const int tb0 = __ldg(B.tile_ptr + K), tb1 = __ldg(B.tile_ptr + K + 1);
                    for (int j = tb0 + lane; j < tb1; j += 32)
                    {
                        const int tb = B.row_data ? __ldg(B.row_data + j) : j;
                        const int bcnt = __ldg(B.tile_nnz + tb + 1) - __ldg(B.tile_nnz + tb);
                        if ((long long)acnt * bcnt < (long long)cutoff)
                            continue;
                        const int slot = slot_of(S, __ldg(B.tile_col + j), Jlo, Jhi, nW, table);
                        if (slot >= 0)
                            atomicOr(&S.dense[ai][slot >> 5], 1u << (slot & 31));
                    }
                }
                __syncthreads();
            }

            // ---- K loop: producer warp streams B row groups, consumers compute
            if (producer)
            {
                if (lane == 0)
                {
                    for (int ai = 0; ai < nK; ++ai)
                    {
                        const int g = gk + ai, s = g % NSTAGE;
                        if (g >= NSTAGE && !mbar_wait(&S.empty[s], ((g / NSTAGE) - 1) & 1, err))
                        {
                            failed = true;
                            break;
                        }
                        produce(B, S, ai, S.st[s], &S.full[s]);
                    }
                }
                __syncwarp(); // lanes 1-31 wait here so the warp meets the barrier converged
            }
            else
            {
                const int r_lo = warp * 2;
                for (int ai = 0; ai < nK; ++ai)
                {
                    const int g = gk + ai, s = g % NSTAGE;
                    if (!__all_sync(FULL, mbar_wait(&S.full[s], (g / NSTAGE) & 1, err)))
                    {
                        failed = true; // warp-uniform
                        break;
                    }
                    const uint8_t *aptr_t = &S.aptr[ai * TD];
                    const int acnt = S.atnnz[ai + 1] - S.atnnz[ai];
                    const int e0 = aptr_t[r_lo], e1 = aptr_t[r_lo + 1];
                    const int e2 = r_lo + 1 == TD - 1 ? acnt : aptr_t[r_lo + 2];
                    if (e0 < e2)
                    {
                        const Stage &st = S.st[s];
                        const bool staged = S.p_staged[ai] != 0;
                        const int rb = S.p_K[ai] * TD;
                        const int ebase = S.p_e0[ai];
                        const int *bcol;
                        const double *bval;
                        const int *brp;
                        int eoff; // subtract from a global entry index to index bcol/bval
                        if (staged)
                        {
                            bcol = &st.col[st.off_col];
                            bval = &st.val[st.off_val];
                            brp = &st.rp[st.off_rp];
                            eoff = ebase;
                        }
                        else
                        {
                            bcol = B.csr_col;
                            bval = B.csr_val;
                            brp = B.csr_rowptr + rb;
                            eoff = 0;
                        }
                        const int aoff = S.atnnz[ai];
                        for (int e = e0; e < e2; ++e)
                        {
                            const int ae = aoff + e;
                            const int k = (a_staged ? S.acol[ae] : A.col[av0 + ae]) & 15;
                            const double a = a_staged ? S.aval[ae] : __ldg(A.val + av0 + ae);
                            const int r = e < e1 ? r_lo : r_lo + 1;
                            // row bounds clamped into the K step's entry range, so
                            // inconsistent operands cannot steer an access outside B
                            const int lo_e = staged ? 0 : ebase, hi_e = S.p_e1[ai] - (staged ? ebase : 0);
                            const int fs = max(brp[k] - eoff, lo_e);
                            const int fe = min(max(brp[k + 1] - eoff, fs), hi_e);
                            if (w0 == cs0) // count each pair once, in the first window
                                n_fma += fe - fs;
                            for (int f = fs + lane; f < fe; f += 32)
                            {
                                const int col = bcol[f];
                                const int slot = slot_of(S, col >> 4, Jlo, Jhi, nW, table);
                                if (slot < 0)
                                    continue;
                                if (DMMA && ((S.dense[ai][slot >> 5] >> (slot & 31)) & 1u))
                                    continue;
                                const uint32_t w = S.cm[slot * TD + r];
                                const int pos = (int)(w >> 16) + __popc((w & 0xFFFFu) >> (16 - (col & 15)));
                                if (safe)
                                    atomicAdd(&S.acc[pos], a * bval[f]); // B row repeats a column
                                else
                                    S.acc[pos] = fma(a, bval[f], S.acc[pos]);
                            }
                        }
                    }
                    __syncwarp();
                    if (lane == 0)
                        mbar_arrive(&S.empty[s]);
                }
                __syncwarp();
            }
            gk += nK;
            if (__syncthreads_or(failed))
            {
                // a stage never filled or drained within the poll limit (error
                // recorded): give copies still in flight a bounded chance to land
                if (tid == 0)
                    for (int q = 0; q < NSTAGE; ++q)
                    {
                        const int g = gk - 1 - q;
                        if (g >= 0)
                            mbar_wait(&S.full[g % NSTAGE], (g / NSTAGE) & 1, err);
                    }
                __syncwarp();
                __syncthreads();
                return;
            }

            // ---- dense pairs of this chunk on the tensor cores
            if constexpr (DMMA)
            {
                if (!producer)
                {
                    DenseSmem &D = *reinterpret_cast<DenseSmem *>(dyn + sizeof(RowSmem));
                    double *da = D.da[warp];
                    double *db = D.db[warp];
                    const int g = lane >> 2, t4 = lane & 3;
                    for (int ai = 0; ai < nK; ++ai)
                    {
                        const int ta = ab + ai, an = __ldg(A.tile_nnz + ta);
                        const int acnt = __ldg(A.tile_nnz + ta + 1) - an;
                        const int K = S.p_K[ai];
                        const int tb0 = __ldg(B.tile_ptr + K), tb1 = __ldg(B.tile_ptr + K + 1);
                        for (int sw = 0; sw < SLOT_CAP / 32; ++sw)
                        {
                            uint32_t bits = S.dense[ai][sw];
                            while (bits)
                            {
                                const int slot = sw * 32 + __ffs(bits) - 1;
                                bits &= bits - 1;
                                if ((slot % NW) != warp)
                                    continue;
                                const int jp = lower_bound(B.tile_col, tb0, tb1, S.cJ[slot]);
                                if (jp >= tb1 || __ldg(B.tile_col + jp) != S.cJ[slot])
                                    continue; // cannot happen: the pair was classified from this list
                                ++n_dense;
                                const int tb = B.row_data ? __ldg(B.row_data + jp) : jp;
                                const int bn = __ldg(B.tile_nnz + tb), bcnt = __ldg(B.tile_nnz + tb + 1) - bn;
                                for (int i = lane; i < TD * TD; i += 32)
                                {
                                    da[i] = 0.0;
                                    db[i] = 0.0;
                                }
                                __syncwarp();
                                {
                                    const int r = lane & 15;
                                    if (lane < TD)
                                    {
                                        const int i0 = A.ptr[(size_t)ta * TD + r];
                                        const int i1 = r == TD - 1 ? acnt : A.ptr[(size_t)ta * TD + r + 1];
                                        for (int i = i0; i < i1; ++i)
                                            da[r * TD + (A.col[an + i] & 15)] += __ldg(A.val + an + i);
                                    }
                                    else
                                    {
                                        const int f0 = B.ptr[(size_t)tb * TD + r];
                                        const int f1 = r == TD - 1 ? bcnt : B.ptr[(size_t)tb * TD + r + 1];
                                        for (int f = f0; f < f1; ++f)
                                            db[r * TD + (B.col[bn + f] & 15)] += __ldg(B.val + bn + f);
                                    }
                                }
                                __syncwarp();
                                double d[8];
#pragma unroll
                                for (int q = 0; q < 8; ++q)
                                    d[q] = 0.0;
#pragma unroll
                                for (int qr = 0; qr < 2; ++qr)
#pragma unroll
                                    for (int qc = 0; qc < 2; ++qc)
#pragma unroll
                                        for (int kb = 0; kb < 4; ++kb)
                                            dmma_m8n8k4(d[(qr * 2 + qc) * 2], d[(qr * 2 + qc) * 2 + 1],
                                                        da[(qr * 8 + g) * TD + kb * 4 + t4],
                                                        db[(kb * 4 + t4) * TD + qc * 8 + g]);
#pragma unroll
                                for (int qr = 0; qr < 2; ++qr)
#pragma unroll
                                    for (int qc = 0; qc < 2; ++qc)
#pragma unroll
                                        for (int q = 0; q < 2; ++q)
                                        {
                                            const int r = qr * 8 + g, c = qc * 8 + t4 * 2 + q;
                                            const uint32_t w = S.cm[slot * TD + r];
                                            if (w & (0x8000u >> c))
                                                S.acc[(int)(w >> 16) + __popc((w & 0xFFFFu) >> (16 - c))] +=
                                                    d[(qr * 2 + qc) * 2 + q];
                                        }
                                __syncwarp();
                            }
                        }
                    }
                }
            }
            __syncthreads(); // chunk arrays are rewritten by the next chunk
        }

        // ---- write-out of the window (consecutive threads: same row, next tile)
        for (int it = tid; it < nW * TD; it += NR_THREADS)
        {
            const int r = it / nW, s = it - r * nW;
            const uint32_t w = S.cm[s * TD + r];
            const uint32_t m = w & 0xFFFFu;
            const int abase = (int)(w >> 16);
            const int J = S.cJ[s];
            if (csr_col != nullptr && m)
            {
                const long long pos = (long long)S.rowcsr0[r] + (abase - S.rowacc0[r]);
                uint32_t mm = m;
                int k = 0;
                while (mm)
                {
                    const int c = __clz(mm) - 16;
                    mm &= ~(0x8000u >> c);
                    if (pos + k >= nnzC)
                    {
                        set_error(err, DERR_NUM_BOUNDS);
                        break;
                    }
                    csr_col[pos + k] = J * TD + c;
                    csr_val[pos + k] = S.acc[abase + k];
                    ++k;
                }
            }
            if (c_val != nullptr)
            {
                const int t = w0 + s;
                int pre = 0;
                for (int rr = 0; rr < r; ++rr)
                    pre += __popc(S.cm[s * TD + rr] & 0xFFFFu);
                c_ptr[(size_t)t * TD + r] = (uint8_t)pre;
                const long long tpos = (long long)__ldg(c_tile_nnz + t) + pre;
                uint32_t mm = m;
                int k = 0;
                while (mm)
                {
                    const int c = __clz(mm) - 16;
                    mm &= ~(0x8000u >> c);
                    if (tpos + k >= nnzC)
                    {
                        set_error(err, DERR_NUM_BOUNDS);
                        break;
                    }
                    c_colb[tpos + k] = (uint8_t)c;
                    c_val[tpos + k] = S.acc[abase + k];
                    ++k;
                }
            }
        }
        __syncthreads();
        if (tid < TD)
            S.rowrun[tid] += S.rowacc0[tid + 1] - S.rowacc0[tid];
        __syncthreads();
        w0 = w1;
    }
    if (counters != nullptr)
    {
        // n_dense is counted by all 32 lanes of the warp that ran the pair;
        // n_fma is counted once per A entry by every lane of the warp
        const long long nd = warp_sum(n_dense) / 32, nf = warp_sum(n_fma) / 32;
        if (lane == 0)
        {
            if (nd)
                atomicAdd((unsigned long long *)&counters[0], (unsigned long long)nd);
            if (nf)
                atomicAdd((unsigned long long *)&counters[1], (unsigned long long)nf);
        }
    }
}

__global__ void k_max_tile_nnz(const int *__restrict__ tnnz, int nt, int *out)
{
    int m = 0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x)
        m = max(m, tnnz[t + 1] - tnnz[t]);
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0)
        atomicMax(out, m);
}

} // namespace

int max_tile_nnz_device(Workspace &ws, const int *tile_nnz, int numtile, int *out)
{
    RTT_CUDA(cudaMemsetAsync(out, 0, sizeof(int), ws.stream));
    if (numtile > 0)
    {
        k_max_tile_nnz<<<std::min(1184, (numtile + 255) / 256), 256, 0, ws.stream>>>(tile_nnz,
                                                                                 numtile, out);
        ws.launches++;
    }
    return RTT_OK;
}

int numeric_rows_device(Workspace &ws, const DevTiles &A, const DevTiles &B, SymbolicOut &S,
                        const NumericConfig &cfg)
{
    cudaStream_t s = ws.stream;
    const size_t nnz = (size_t)S.nnz;
    if (cfg.write_tiles)
    {
        RTT_CHECK(S.c_col.ensure(nnz + 16, s));
        RTT_CHECK(S.c_val.ensure(sizeof(double) * nnz + 16, s));
    }
    if (cfg.csr_col != nullptr)
        RTT_CHECK(csr_rowptr_device(ws, S, cfg.csr_rowptr));
    if (S.numtile == 0 || S.tilem == 0)
        return RTT_OK;
    if (cfg.ev_begin != nullptr)
        RTT_CUDA(cudaEventRecord(cfg.ev_begin, s));
    const bool dmma = cfg.dmma_pair_cutoff > 0;
    const size_t smem = sizeof(RowSmem) + (dmma ? sizeof(DenseSmem) : 0);
    auto launch = [&](auto kern) -> int {
        RTT_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        kern<<<S.tilem, NR_THREADS, smem, s>>>(
            A, B, S.tilem, S.nnz, S.c_tile_ptr.as<int>(), S.c_tile_col.as<int>(),
            S.c_mask.as<uint16_t>(), S.c_tile_nnz.as<int>(), S.c_ptr.as<uint8_t>(),
            cfg.write_tiles ? S.c_col.as<uint8_t>() : nullptr,
            cfg.write_tiles ? S.c_val.as<double>() : nullptr, cfg.csr_col ? cfg.csr_rowptr : nullptr,
            cfg.csr_col, cfg.csr_val, cfg.dmma_pair_cutoff, cfg.b_staging ? 1 : 0,
            cfg.conflict_safe ? 1 : 0, cfg.counters, ws.err.as<int>());
        return RTT_OK;
    };
    if (dmma)
        RTT_CHECK(launch(k_numeric_rows<true>));
    else
        RTT_CHECK(launch(k_numeric_rows<false>));
    ws.launches++;
    if (cfg.ev_end != nullptr)
        RTT_CUDA(cudaEventRecord(cfg.ev_end, s));
    return RTT_OK;
}

} // namespace rtt
