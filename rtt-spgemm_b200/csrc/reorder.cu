// reorder.cu - row / inner (K) reordering of A for the tiled SpGEMM.
//
// The reference's BGRF reorder (src/dmma_reorder.h:37-47, :2651-3085) is a
// bipartite Cuthill-McKee traversal of A's row/column graph on the GPU whose
// joint row/K proposal is committed only if it cuts the number of 8x4 A
// tiles (the exact commit rule, :1671-1727), followed by fine passes that
// pack 8x4 tensor-core groups inside fixed windows.  Here:
//
//  * proposal: a level-synchronous breadth-first traversal that alternates
//    rows and columns.  Each level's new vertices are ordered by the position
//    of their earliest-placed neighbour in the level before (the Cuthill-McKee
//    rule), then by degree, then by index.  A component starts at its
//    unplaced row of least (degree, index); rows and columns without entries
//    go last, in index order.
//  * commit: the distinct 8x4 tiles of A under the proposal are counted
//    exactly (sort + unique of tile keys) against the current order; the
//    proposal is taken only if it has fewer tiles.
//  * fine passes (rows in windows of 32 and groups of 8, then inner indices
//    in windows of 16 and groups of 4, :2865-2990): every index gets a
//    profile under the other axis's current order - entry count, a soft
//    degree bucket (log2 / 2), the range of 4-column (8-row) panels it
//    touches and a 128-bit fingerprint of those panels; one warp per window
//    (a lane per index) packs the window greedily: an anchor, the least
//    unused index in the coarse profile order (:1287-1311), then the index
//    that adds the fewest new fingerprint bits to the group (ties: the
//    larger overlap share, the smaller panel-span growth, the closer degree,
//    :1386-1416), until the group is full.  A window's packing is committed
//    only if it has fewer 8x4 tiles than the window as it stands, or as many
//    and a smaller fan-out (sum over its groups of the span of the opposite
//    tiles they touch), counted exactly per window (:1730-1887).
//
// Each committed step keeps or cuts the tile count, so a plan never has more
// 8x4 tiles than A (except in the unguarded ablation).  With C = A*B,
// A' = P A Q^T and B' = Q B give A' B' = P C: C's rows come back with
// rtt_tile2csr_restore_rows or rtt_csr_permute(row_new_to_old = P^T).
#include "rtt_internal.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_segmented_sort.cuh>
#include <algorithm>
#include <climits>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace rtt
{
namespace
{

constexpr int RO_UNSEEN = -1;  // vertex not reached
constexpr int RO_PENDING = -2; // reached in the current level, position pending
// Components traversed one by one (each costs host round trips); the
// vertices of any further components keep their index order, after the
// traversed ones.
constexpr int RO_MAX_COMPONENTS = 256;

inline int grid_of(long long n, int b) { return (int)((n + b - 1) / b); }

__global__ void k_ro_degrees(int n, const int *__restrict__ ptr, int *__restrict__ deg)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n)
        deg[v] = ptr[v + 1] - ptr[v];
}

__global__ void k_ro_fill(int n, int *a, int v)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        a[i] = v;
}

// Start of a component: the unplaced vertex of least (degree, index) among
// those with entries; *best = (degree << 32) | index, or all ones if none.
__global__ void k_ro_start(int n, const int *__restrict__ pos, const int *__restrict__ deg,
                           unsigned long long *best)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n && pos[v] == RO_UNSEEN && deg[v] > 0)
        atomicMin(best, ((unsigned long long)deg[v] << 32) | (unsigned)v);
}

// One level: a warp per frontier vertex v (position pos_x[v]) visits its
// neighbours u on the other side; an unreached u records the least position
// of a neighbour that reached it and joins the next frontier once.
__global__ void k_ro_expand(int nf, const int *__restrict__ frontier, const int *__restrict__ pos_x,
                            const int *__restrict__ adj_ptr, const int *__restrict__ adj,
                            int *__restrict__ pos_y, int *__restrict__ claim_y,
                            int *__restrict__ next, int *__restrict__ next_count)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= nf)
        return;
    const int v = frontier[w];
    const int o = pos_x[v];
    for (int j = adj_ptr[v] + lane; j < adj_ptr[v + 1]; j += 32)
    {
        const int u = adj[j];
        if (pos_y[u] == RO_UNSEEN || pos_y[u] == RO_PENDING)
        {
            atomicMin(&claim_y[u], o);
            if (atomicCAS(&pos_y[u], RO_UNSEEN, RO_PENDING) == RO_UNSEEN)
                next[atomicAdd(next_count, 1)] = u;
        }
    }
}

// Sort keys of the next frontier: (earliest neighbour position, degree).
__global__ void k_ro_keys(int n, const int *__restrict__ ids, const int *__restrict__ claim,
                          const int *__restrict__ deg, unsigned long long *__restrict__ keys)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
    {
        const int u = ids[i];
        keys[i] = ((unsigned long long)(unsigned)claim[u] << 32) | (unsigned)deg[u];
    }
}

__global__ void k_ro_place(int n, const int *__restrict__ ids, int base, int *__restrict__ pos)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        pos[ids[i]] = base + i;
}

// Vertices never reached go last, in index order: flag + scan + place.
__global__ void k_ro_unplaced_flags(int n, const int *__restrict__ pos, int *__restrict__ flag)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n)
        flag[v] = pos[v] < 0;
}

__global__ void k_ro_unplaced_place(int n, const int *__restrict__ scan, int base,
                                    int *__restrict__ pos)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n && pos[v] < 0)
        pos[v] = base + scan[v];
}

__global__ void k_ro_inverse(int n, const int *__restrict__ old_to_new, int *__restrict__ new_to_old)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v < n)
        new_to_old[old_to_new[v]] = v;
}

// Tile keys of A's entries under row / column maps (nullptr = identity):
// (row / 8) * tile columns + column / 4, the 8x4 A tiles of the reference.
__global__ void k_ro_tile_keys(int m, const int *__restrict__ rp, const int *__restrict__ col,
                               const int *__restrict__ row_map, const int *__restrict__ col_map,
                               long long tile_cols, unsigned long long *__restrict__ keys)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= m)
        return;
    const int r = (int)w;
    const long long R = (row_map ? row_map[r] : r) / 8;
    for (int j = rp[r] + lane; j < rp[r + 1]; j += 32)
    {
        const int c = col[j];
        keys[j] = (unsigned long long)(R * tile_cols + (col_map ? col_map[c] : c) / 4);
    }
}

__global__ void k_ro_count_distinct(long long n, const unsigned long long *__restrict__ sorted,
                                    unsigned long long *count)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const bool head = i < n && (i == 0 || sorted[i] != sorted[i - 1]);
    const unsigned b = __ballot_sync(0xFFFFFFFFu, head);
    if ((threadIdx.x & 31) == 0 && b)
        atomicAdd(count, (unsigned long long)__popc(b));
}

// ---- fine passes

// Two fingerprint bits per panel, one in each 64-bit word: MurmurHash3's
// 64-bit finaliser as the mixer.
__device__ __forceinline__ unsigned long long ro_mix(unsigned long long k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdull;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ull;
    k ^= k >> 33;
    return k;
}

struct AxisProfile
{
    int id, degree, bucket, occupancy, pmin, pmax, span, pad;
    unsigned long long fp[2];
};

// Profile of the index at position i of an axis (old id n2o[i]): its entries
// adj[ptr[id] .. ptr[id + 1]) are indices of the other axis, placed by
// other_o2n and cut into panels of `panel` (4 columns for a row, 8 rows for
// an inner index).  One warp per position.
__global__ void k_ro_profiles(int count, const int *__restrict__ n2o, const int *__restrict__ ptr,
                              const int *__restrict__ adj, const int *__restrict__ other_o2n,
                              int panel, AxisProfile *__restrict__ prof)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= count)
        return;
    const int id = n2o[(int)w];
    const int b = ptr[id], e = ptr[id + 1];
    int lo = INT_MAX, hi = -1;
    unsigned long long f0 = 0ull, f1 = 0ull;
    for (int j = b + lane; j < e; j += 32)
    {
        const int p = other_o2n[adj[j]] / panel;
        lo = min(lo, p);
        hi = max(hi, p);
        f0 |= 1ull << (ro_mix(2ull * (unsigned)p + 1ull) & 63);
        f1 |= 1ull << (ro_mix(2ull * (unsigned)p + 2ull) & 63);
    }
    lo = warp_min(lo);
    hi = warp_max(hi);
    for (int o = 16; o > 0; o >>= 1)
    {
        f0 |= __shfl_xor_sync(FULL, f0, o);
        f1 |= __shfl_xor_sync(FULL, f1, o);
    }
    if (lane == 0)
    {
        AxisProfile q;
        q.id = id;
        q.degree = e - b;
        q.bucket = q.degree > 0 ? (31 - __clz(q.degree)) / 2 : -1;
        q.occupancy = __popcll(f0) + __popcll(f1);
        q.pmin = q.degree > 0 ? lo : -1;
        q.pmax = q.degree > 0 ? hi : -1;
        q.span = q.degree > 0 ? hi - lo + 1 : 0;
        q.pad = 0;
        q.fp[0] = f0;
        q.fp[1] = f1;
        prof[w] = q;
    }
}

// The lane holding the lexicographically least key tuple (every lane gets
// the same lane; ties on every key go to the lower lane).
template <int N>
__device__ __forceinline__ int ro_warp_argmin(unsigned long long (&k)[N])
{
    int best = threadIdx.x & 31;
    for (int o = 16; o > 0; o >>= 1)
    {
        unsigned long long a[N];
#pragma unroll
        for (int i = 0; i < N; ++i)
            a[i] = __shfl_xor_sync(FULL, k[i], o);
        const int ab = __shfl_xor_sync(FULL, best, o);
        int cmp = 0; // -1: a is less, 1: k is less
#pragma unroll
        for (int i = 0; i < N; ++i)
            if (cmp == 0 && a[i] != k[i])
                cmp = a[i] < k[i] ? -1 : 1;
        if (cmp < 0 || (cmp == 0 && ab < best))
        {
#pragma unroll
            for (int i = 0; i < N; ++i)
                k[i] = a[i];
            best = ab;
        }
    }
    return best;
}

// Greedy packing of one window of W consecutive positions into groups of G
// (one warp per window, a lane per position): an anchor - the least unused
// profile in the coarse order (indices with entries first, then the larger
// soft bucket, the larger fingerprint occupancy, the lower first panel, the
// narrower panel span, more entries, the fingerprint words, the id) - then,
// until the group is full, the unused profile with the best score against
// the group (the nearer soft bucket to the anchor's, the fewest fingerprint
// bits new to the group, the larger overlap / union share of bits, the
// larger overlap, the least growth of the group's panel span, the nearer
// entry count to the anchor's, the lower id).  out_n2o[position] = old id.
template <int W, int G>
__global__ void k_ro_pack(int count, const AxisProfile *__restrict__ prof, int *__restrict__ out_n2o)
{
    static_assert(W <= 32 && W % G == 0, "one warp per window");
    const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long begin = wid * W;
    if (begin >= count)
        return;
    const int n = (int)min((long long)W, (long long)count - begin);
    const bool mine = lane < n;
    AxisProfile q{};
    if (mine)
        q = prof[begin + lane];
    bool used = !mine;
    const unsigned long long NONE = ~0ull;
    // the coarse order as five keys, least first
    unsigned long long ck[5];
    ck[0] = ((unsigned long long)(q.degree == 0) << 63) |
            ((unsigned long long)(31 - (q.bucket + 1)) << 58) |
            ((unsigned long long)(255 - q.occupancy) << 50) | (unsigned long long)(q.pmin + 1);
    ck[1] = ((unsigned long long)(unsigned)q.span << 32) |
            (unsigned long long)(0xFFFFFFFFu - (unsigned)q.degree);
    ck[2] = q.fp[0];
    ck[3] = q.fp[1];
    ck[4] = (unsigned long long)(unsigned)q.id;
    int written = 0;
    while (written < n)
    {
        unsigned long long k[5];
#pragma unroll
        for (int i = 0; i < 5; ++i)
            k[i] = used ? NONE : ck[i];
        const int a = ro_warp_argmin<5>(k);
        const int a_bucket = __shfl_sync(FULL, q.bucket, a);
        const int a_degree = __shfl_sync(FULL, q.degree, a);
        const int a_id = __shfl_sync(FULL, q.id, a);
        unsigned long long g0 = __shfl_sync(FULL, q.fp[0], a), g1 = __shfl_sync(FULL, q.fp[1], a);
        int gmin = __shfl_sync(FULL, q.pmin, a), gmax = __shfl_sync(FULL, q.pmax, a);
        if (lane == a)
            used = true;
        if (lane == 0)
            out_n2o[begin + written] = a_id;
        ++written;
        for (int slot = 1; slot < G && written < n; ++slot)
        {
            unsigned long long sk[3] = {NONE, NONE, NONE};
            if (!used)
            {
                const int overlap = __popcll(g0 & q.fp[0]) + __popcll(g1 & q.fp[1]);
                const int adds = __popcll(~g0 & q.fp[0]) + __popcll(~g1 & q.fp[1]);
                const int uni = max(__popcll(g0 | q.fp[0]) + __popcll(g1 | q.fp[1]), 1);
                int nmin = gmin, nmax = gmax;
                if (q.pmin >= 0)
                {
                    nmin = gmin < 0 ? q.pmin : min(gmin, q.pmin);
                    nmax = max(gmax, q.pmax);
                }
                const int cur_span = gmin < 0 ? 0 : gmax - gmin + 1;
                const int next_span = nmin < 0 ? 0 : nmax - nmin + 1;
                // overlap / union as an exact fixed-point rank: distinct
                // fractions with denominators <= 128 differ by more than 2^-20
                const unsigned ratio = ((unsigned)overlap << 20) / (unsigned)uni;
                sk[0] = ((unsigned long long)abs(a_bucket - q.bucket) << 58) |
                        ((unsigned long long)adds << 50) |
                        ((unsigned long long)((1u << 21) - ratio) << 8) |
                        (unsigned long long)(255 - overlap);
                sk[1] = ((unsigned long long)(unsigned)(next_span - cur_span) << 32) |
                        (unsigned long long)(unsigned)abs(a_degree - q.degree);
                sk[2] = (unsigned long long)(unsigned)q.id;
            }
            const int b = ro_warp_argmin<3>(sk);
            const int b_id = __shfl_sync(FULL, q.id, b);
            const unsigned long long b0 = __shfl_sync(FULL, q.fp[0], b);
            const unsigned long long b1 = __shfl_sync(FULL, q.fp[1], b);
            const int bmin = __shfl_sync(FULL, q.pmin, b), bmax = __shfl_sync(FULL, q.pmax, b);
            if (lane == b)
                used = true;
            if (lane == 0)
                out_n2o[begin + written] = b_id;
            ++written;
            if (bmin >= 0)
            {
                gmin = gmin < 0 ? bmin : min(gmin, bmin);
                gmax = max(gmax, bmax);
            }
            g0 |= b0;
            g1 |= b1;
        }
    }
}

// Keys of the 8x4 tiles inside the fine pass's windows, for the current
// order and for the proposal: ((window * opposite tiles + opposite tile) *
// groups per window + group).  ROWS: windows of W rows in groups of 8
// against 4-column tiles; else windows of W inner indices in groups of 4
// against 8-row tiles.  One warp per row of A.
template <bool ROWS, int W>
__global__ void k_ro_window_keys(int m, const int *__restrict__ rp, const int *__restrict__ col,
                                 const int *__restrict__ cur_r, const int *__restrict__ cur_c,
                                 const int *__restrict__ prop_o2n, long long opp_tiles,
                                 unsigned long long *__restrict__ keys_cur,
                                 unsigned long long *__restrict__ keys_prop)
{
    constexpr int GSZ = ROWS ? 8 : 4, GPW = W / GSZ;
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= m)
        return;
    const int r = (int)w;
    const int R = cur_r[r];
    const int PR = ROWS ? prop_o2n[r] : R;
    for (int j = rp[r] + lane; j < rp[r + 1]; j += 32)
    {
        const int c = col[j];
        const int Cc = cur_c[c];
        const int PC = ROWS ? Cc : prop_o2n[c];
        const int pos = ROWS ? R : Cc, ppos = ROWS ? PR : PC;
        const long long opp = ROWS ? Cc / 4 : R / 8;
        const unsigned long long pair = (unsigned long long)(pos / W) * opp_tiles + opp;
        keys_cur[j] = pair * GPW + (pos % W) / GSZ;
        keys_prop[j] = pair * GPW + (ppos % W) / GSZ;
    }
}

// Distinct tiles per window and the span of opposite tiles per group, from
// sorted keys (a run head is a distinct tile).
template <int GPW>
__global__ void k_ro_window_count(long long n, const unsigned long long *__restrict__ sorted,
                                  long long opp_tiles, int *__restrict__ counts,
                                  int *__restrict__ smin, int *__restrict__ smax)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || (i > 0 && sorted[i] == sorted[i - 1]))
        return;
    const unsigned long long key = sorted[i];
    const int g = (int)(key % GPW);
    const unsigned long long pair = key / GPW;
    const int opp = (int)(pair % (unsigned long long)opp_tiles);
    const int win = (int)(pair / (unsigned long long)opp_tiles);
    atomicAdd(&counts[win], 1);
    atomicMin(&smin[win * GPW + g], opp);
    atomicMax(&smax[win * GPW + g], opp);
}

// One thread per window: the proposal's packing replaces the window's order
// when it has fewer tiles, or as many and a smaller fan-out (the sum over
// the groups of the span of opposite tiles); always when !guarded.
// stats: accepted windows, tiles removed, fan-out before, fan-out after.
template <int W, int GPW>
__global__ void k_ro_window_commit(int count, int windows, const int *__restrict__ cnt,
                                   const int *__restrict__ smin, const int *__restrict__ smax,
                                   bool guarded, const int *__restrict__ prop_n2o,
                                   int *__restrict__ cur_n2o, unsigned long long *stats)
{
    const int w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= windows)
        return;
    // [0, windows): current order; [windows, 2 windows): proposal
    const int cc = cnt[w], cp = cnt[windows + w];
    int fc = 0, fp = 0;
    for (int g = 0; g < GPW; ++g)
    {
        const int ic = w * GPW + g, ip = (windows + w) * GPW + g;
        if (smax[ic] >= 0)
            fc += smax[ic] - smin[ic] + 1;
        if (smax[ip] >= 0)
            fp += smax[ip] - smin[ip] + 1;
    }
    const bool accept = !guarded || cp < cc || (cp == cc && fp < fc);
    atomicAdd(&stats[2], (unsigned long long)fc);
    atomicAdd(&stats[3], (unsigned long long)(accept ? fp : fc));
    if (!accept)
        return;
    const int b = w * W, e = min(count, b + W);
    for (int i = b; i < e; ++i)
        cur_n2o[i] = prop_n2o[i];
    atomicAdd(&stats[0], 1ull);
    if (cc > cp)
        atomicAdd(&stats[1], (unsigned long long)(cc - cp));
}

__global__ void k_ro_iota(int n, int *__restrict__ a, int *__restrict__ b)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        a[i] = b[i] = i;
}

// ---- CSR permutation: out row i = A row new_to_old[i], columns mapped
__global__ void k_perm_lengths(int m, const int *__restrict__ rp, const int *__restrict__ n2o,
                               int *__restrict__ len)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < m)
    {
        const int r = n2o ? n2o[i] : i;
        len[i] = rp[r + 1] - rp[r];
    }
}

__global__ void k_perm_copy(int m, const int *__restrict__ rp, const int *__restrict__ col,
                            const double *__restrict__ val, const int *__restrict__ n2o,
                            const int *__restrict__ col_map, const int *__restrict__ out_rp,
                            int *__restrict__ out_col, double *__restrict__ out_val)
{
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= m)
        return;
    const int i = (int)w, r = n2o ? n2o[i] : i;
    const int b = rp[r], d = out_rp[i];
    for (int j = lane; j < rp[r + 1] - b; j += 32)
    {
        const int c = col[b + j];
        out_col[d + j] = col_map ? col_map[c] : c;
        out_val[d + j] = val[b + j];
    }
}

// Checks that a device int array of n entries is a permutation of [0, n).
__global__ void k_perm_check(int n, const int *__restrict__ p, int *__restrict__ seen, int *err)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int v = p[i];
    if (v < 0 || v >= n || atomicExch(&seen[v], 1) != 0)
        set_error(err, DERR_CSR_COL);
}

struct Bufs
{
    DevBuf b[12];
    void release()
    {
        for (DevBuf &x : b)
            x.release();
    }
};

int radix_sort_keys_u64(Workspace &ws, unsigned long long *in, unsigned long long *out,
                        long long n)
{
    if (n <= 0)
        return RTT_OK;
    size_t bytes = 0;
    RTT_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, bytes, in, out, (int)n, 0, 64, ws.stream));
    RTT_CHECK(ws.scan_tmp.ensure(bytes, ws.stream));
    RTT_CUDA(cub::DeviceRadixSort::SortKeys(ws.scan_tmp.p, bytes, in, out, (int)n, 0, 64,
                                            ws.stream));
    ws.launches += 3;
    return RTT_OK;
}

// Distinct 8x4 tiles of A under the maps.
int count_tiles(Workspace &ws, const rtt_csr_view &A, const int *row_map, const int *col_map,
                DevBuf &k0, DevBuf &k1, long long *tiles)
{
    cudaStream_t s = ws.stream;
    const long long nnz = A.nnz;
    *tiles = 0;
    if (nnz == 0)
        return RTT_OK;
    RTT_CHECK(k0.ensure(sizeof(unsigned long long) * (size_t)nnz, s));
    RTT_CHECK(k1.ensure(sizeof(unsigned long long) * (size_t)nnz + 16, s));
    const long long tile_cols = (A.cols + 3) / 4;
    k_ro_tile_keys<<<grid_of((long long)A.rows * 32, 256), 256, 0, s>>>(
        A.rows, A.row_ptr, A.col_idx, row_map, col_map, tile_cols,
        k0.as<unsigned long long>());
    ws.launches++;
    RTT_CHECK(radix_sort_keys_u64(ws, k0.as<unsigned long long>(), k1.as<unsigned long long>() + 1,
                                  nnz));
    unsigned long long *cnt = k1.as<unsigned long long>(); // slot 0 holds the count
    RTT_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
    k_ro_count_distinct<<<grid_of(nnz, 256), 256, 0, s>>>(nnz, cnt + 1, cnt);
    ws.launches++;
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars64, cnt, sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, s));
    RTT_CUDA(cudaStreamSynchronize(s));
    ws.syncs++;
    *tiles = ws.h_scalars64[0];
    return RTT_OK;
}

// Bipartite Cuthill-McKee positions of A's rows (pos_r) and columns (pos_c).
int bipartite_cm(Workspace &ws, const rtt_csr_view &A, const int *at_ptr, const int *at_idx,
                 int *pos_r, int *pos_c, Bufs &B, int *components, int *levels, int *active_r,
                 int *active_c)
{
    cudaStream_t s = ws.stream;
    const int m = A.rows, n = A.cols;
    const int big = std::max(m, n) + 16;
    RTT_CHECK(B.b[0].ensure(sizeof(int) * (size_t)m + 16, s)); // deg_r
    RTT_CHECK(B.b[1].ensure(sizeof(int) * (size_t)n + 16, s)); // deg_c
    RTT_CHECK(B.b[2].ensure(sizeof(int) * (size_t)m + 16, s)); // claim_r
    RTT_CHECK(B.b[3].ensure(sizeof(int) * (size_t)n + 16, s)); // claim_c
    RTT_CHECK(B.b[4].ensure(sizeof(int) * (size_t)big, s));   // frontier
    RTT_CHECK(B.b[5].ensure(sizeof(int) * (size_t)big, s));   // next (unsorted)
    RTT_CHECK(B.b[6].ensure(sizeof(int) * (size_t)big, s));   // next sorted by index
    RTT_CHECK(B.b[7].ensure(sizeof(unsigned long long) * (size_t)big, s)); // keys
    RTT_CHECK(B.b[8].ensure(sizeof(unsigned long long) * (size_t)big, s)); // keys sorted
    RTT_CHECK(B.b[9].ensure(sizeof(unsigned long long) * 2, s)); // start / counter
    int *deg_r = B.b[0].as<int>(), *deg_c = B.b[1].as<int>();
    int *claim_r = B.b[2].as<int>(), *claim_c = B.b[3].as<int>();
    int *front = B.b[4].as<int>(), *next = B.b[5].as<int>(), *next_s = B.b[6].as<int>();
    unsigned long long *keys = B.b[7].as<unsigned long long>();
    unsigned long long *keys_s = B.b[8].as<unsigned long long>();
    unsigned long long *start = B.b[9].as<unsigned long long>();
    int *counter = reinterpret_cast<int *>(start + 1);
    if (m > 0)
    {
        k_ro_degrees<<<grid_of(m, 256), 256, 0, s>>>(m, A.row_ptr, deg_r);
        k_ro_fill<<<grid_of(m, 256), 256, 0, s>>>(m, pos_r, RO_UNSEEN);
        k_ro_fill<<<grid_of(m, 256), 256, 0, s>>>(m, claim_r, INT_MAX);
        ws.launches += 3;
    }
    if (n > 0)
    {
        k_ro_degrees<<<grid_of(n, 256), 256, 0, s>>>(n, at_ptr, deg_c);
        k_ro_fill<<<grid_of(n, 256), 256, 0, s>>>(n, pos_c, RO_UNSEEN);
        k_ro_fill<<<grid_of(n, 256), 256, 0, s>>>(n, claim_c, INT_MAX);
        ws.launches += 3;
    }
    int placed_r = 0, placed_c = 0;
    *components = 0;
    *levels = 0;
    // sorts the next frontier by (claim, degree, index) and places it
    auto place = [&](int nn, const int *claim, const int *deg, int *pos, int base) -> int {
        size_t bytes = 0;
        // by index first (the compaction order is arbitrary), then stable by key
        RTT_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, bytes, next, next_s, nn, 0, 32, s));
        size_t b2 = 0;
        RTT_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, b2, keys, keys_s, next_s, next, nn, 0,
                                                 64, s));
        RTT_CHECK(ws.scan_tmp.ensure(std::max(bytes, b2), s));
        RTT_CUDA(cub::DeviceRadixSort::SortKeys(ws.scan_tmp.p, bytes, next, next_s, nn, 0, 32, s));
        k_ro_keys<<<grid_of(nn, 256), 256, 0, s>>>(nn, next_s, claim, deg, keys);
        bytes = std::max(bytes, b2);
        RTT_CUDA(cub::DeviceRadixSort::SortPairs(ws.scan_tmp.p, bytes, keys, keys_s, next_s, next,
                                                 nn, 0, 64, s));
        k_ro_place<<<grid_of(nn, 256), 256, 0, s>>>(nn, next, base, pos);
        ws.launches += 8;
        return RTT_OK;
    };
    for (int comp = 0; comp < RO_MAX_COMPONENTS; ++comp)
    {
        // next component: its row of least (degree, index)
        RTT_CUDA(cudaMemsetAsync(start, 0xFF, sizeof(unsigned long long), s));
        if (m > 0)
        {
            k_ro_start<<<grid_of(m, 256), 256, 0, s>>>(m, pos_r, deg_r, start);
            ws.launches++;
        }
        RTT_CUDA(cudaMemcpyAsync(ws.h_scalars64, start, sizeof(unsigned long long),
                                 cudaMemcpyDeviceToHost, s));
        RTT_CUDA(cudaStreamSynchronize(s));
        ws.syncs++;
        if (ws.h_scalars64[0] == -1ll)
            break;
        const int r0 = (int)(ws.h_scalars64[0] & 0xFFFFFFFFull);
        ++*components;
        RTT_CUDA(cudaMemcpyAsync(front, &r0, sizeof(int), cudaMemcpyHostToDevice, s));
        RTT_CUDA(cudaMemcpyAsync(pos_r + r0, &placed_r, sizeof(int), cudaMemcpyHostToDevice, s));
        RTT_CUDA(cudaStreamSynchronize(s)); // the host values above are stack copies
        ++placed_r;
        int nf = 1;
        bool rows_side = true; // the frontier holds rows
        while (nf > 0)
        {
            RTT_CUDA(cudaMemsetAsync(counter, 0, sizeof(int), s));
            if (rows_side)
                k_ro_expand<<<grid_of((long long)nf * 32, 256), 256, 0, s>>>(
                    nf, front, pos_r, A.row_ptr, A.col_idx, pos_c, claim_c, next, counter);
            else
                k_ro_expand<<<grid_of((long long)nf * 32, 256), 256, 0, s>>>(
                    nf, front, pos_c, at_ptr, at_idx, pos_r, claim_r, next, counter);
            ws.launches++;
            RTT_CUDA(cudaMemcpyAsync(ws.h_scalars + 14, counter, sizeof(int),
                                     cudaMemcpyDeviceToHost, s));
            RTT_CUDA(cudaStreamSynchronize(s));
            ws.syncs++;
            const int nn = ws.h_scalars[14];
            if (nn > 0)
            {
                if (rows_side)
                {
                    RTT_CHECK(place(nn, claim_c, deg_c, pos_c, placed_c));
                    placed_c += nn;
                }
                else
                {
                    RTT_CHECK(place(nn, claim_r, deg_r, pos_r, placed_r));
                    placed_r += nn;
                }
                ++*levels;
                std::swap(front, next); // the placed order is the next frontier
            }
            nf = nn;
            rows_side = !rows_side;
        }
    }
    *active_r = placed_r;
    *active_c = placed_c;
    // rows and columns never reached: last, in index order
    RTT_CHECK(B.b[10].ensure(sizeof(int) * ((size_t)big + 1), s));
    RTT_CHECK(B.b[11].ensure(sizeof(int) * ((size_t)big + 1), s));
    int *flag = B.b[10].as<int>(), *scn = B.b[11].as<int>();
    const int sizes[2] = {m, n};
    int *poss[2] = {pos_r, pos_c};
    const int bases[2] = {placed_r, placed_c};
    for (int side = 0; side < 2; ++side)
    {
        const int nv = sizes[side];
        if (nv == 0)
            continue;
        k_ro_unplaced_flags<<<grid_of(nv, 256), 256, 0, s>>>(nv, poss[side], flag);
        ws.launches++;
        RTT_CHECK(scan_exclusive_int(ws, flag, scn, nv));
        k_ro_unplaced_place<<<grid_of(nv, 256), 256, 0, s>>>(nv, scn, bases[side], poss[side]);
        ws.launches++;
    }
    return RTT_OK;
}

} // namespace

namespace
{

// Maps of the two axes as the plan stands: old_to_new and new_to_old.
struct AxisMaps
{
    DevBuf o2n, n2o;
};

// One fine pass over an axis (ROWS: A's rows, windows of 32 in groups of 8;
// else A's columns, windows of 16 in groups of 4), on top of the current
// maps; updates the axis's maps and the plan's counters.
template <bool ROWS>
int fine_pass(Workspace &ws, const rtt_csr_view &A, const int *at_ptr, const int *at_idx,
              AxisMaps &rows, AxisMaps &cols, bool guarded, DevBuf &prof, DevBuf &prop_n2o,
              DevBuf &prop_o2n, DevBuf &keys, DevBuf &sorted, DevBuf &counts, DevBuf &stats,
              rtt_reorder_plan &P)
{
    constexpr int W = ROWS ? 32 : 16, G = ROWS ? 8 : 4, GPW = W / G;
    cudaStream_t s = ws.stream;
    const int count = ROWS ? A.rows : A.cols;
    if (count == 0)
        return RTT_OK;
    AxisMaps &mine = ROWS ? rows : cols;
    const AxisMaps &other = ROWS ? cols : rows;
    const int windows = (count + W - 1) / W;
    RTT_CHECK(prof.ensure(sizeof(AxisProfile) * (size_t)count, s));
    RTT_CHECK(prop_n2o.ensure(sizeof(int) * (size_t)count, s));
    RTT_CHECK(prop_o2n.ensure(sizeof(int) * (size_t)count, s));
    // profiles in current position order, then the windows' packings
    k_ro_profiles<<<grid_of((long long)count * 32, 256), 256, 0, s>>>(
        count, mine.n2o.as<int>(), ROWS ? A.row_ptr : at_ptr, ROWS ? A.col_idx : at_idx,
        other.o2n.as<int>(), ROWS ? 4 : 8, prof.as<AxisProfile>());
    k_ro_pack<W, G><<<grid_of((long long)windows * 32, 256), 256, 0, s>>>(
        count, prof.as<AxisProfile>(), prop_n2o.as<int>());
    k_ro_inverse<<<grid_of(count, 256), 256, 0, s>>>(count, prop_n2o.as<int>(), prop_o2n.as<int>());
    ws.launches += 3;
    // exact tiles and fan-out per window, current order against the proposal
    const size_t slots = (size_t)2 * windows * (1 + 2 * GPW);
    RTT_CHECK(counts.ensure(sizeof(int) * slots, s));
    int *cnt = counts.as<int>();
    int *smin = cnt + 2 * windows, *smax = smin + 2 * (size_t)windows * GPW;
    RTT_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * 2 * (size_t)windows, s));
    RTT_CUDA(cudaMemsetAsync(smin, 0x7F, sizeof(int) * 2 * (size_t)windows * GPW, s));
    RTT_CUDA(cudaMemsetAsync(smax, 0xFF, sizeof(int) * 2 * (size_t)windows * GPW, s));
    const long long nnz = A.nnz;
    const long long opp_tiles = ROWS ? (A.cols + 3) / 4 : (A.rows + 7) / 8;
    if (nnz > 0)
    {
        RTT_CHECK(keys.ensure(sizeof(unsigned long long) * 2 * (size_t)nnz, s));
        RTT_CHECK(sorted.ensure(sizeof(unsigned long long) * 2 * (size_t)nnz, s));
        unsigned long long *kc = keys.as<unsigned long long>(), *kp = kc + nnz;
        unsigned long long *sc = sorted.as<unsigned long long>(), *sp = sc + nnz;
        k_ro_window_keys<ROWS, W><<<grid_of((long long)A.rows * 32, 256), 256, 0, s>>>(
            A.rows, A.row_ptr, A.col_idx, rows.o2n.as<int>(), cols.o2n.as<int>(),
            prop_o2n.as<int>(), opp_tiles, kc, kp);
        ws.launches++;
        RTT_CHECK(radix_sort_keys_u64(ws, kc, sc, nnz));
        RTT_CHECK(radix_sort_keys_u64(ws, kp, sp, nnz));
        k_ro_window_count<GPW><<<grid_of(nnz, 256), 256, 0, s>>>(nnz, sc, opp_tiles, cnt, smin, smax);
        k_ro_window_count<GPW><<<grid_of(nnz, 256), 256, 0, s>>>(
            nnz, sp, opp_tiles, cnt + windows, smin + (size_t)windows * GPW,
            smax + (size_t)windows * GPW);
        ws.launches += 2;
    }
    RTT_CHECK(stats.ensure(sizeof(unsigned long long) * 4, s));
    RTT_CUDA(cudaMemsetAsync(stats.p, 0, sizeof(unsigned long long) * 4, s));
    k_ro_window_commit<W, GPW><<<grid_of(windows, 256), 256, 0, s>>>(
        count, windows, cnt, smin, smax, guarded, prop_n2o.as<int>(), mine.n2o.as<int>(),
        stats.as<unsigned long long>());
    k_ro_inverse<<<grid_of(count, 256), 256, 0, s>>>(count, mine.n2o.as<int>(), mine.o2n.as<int>());
    ws.launches += 2;
    RTT_CUDA(cudaMemcpyAsync(ws.h_scalars64, stats.p, sizeof(unsigned long long) * 4,
                             cudaMemcpyDeviceToHost, s));
    RTT_CUDA(cudaStreamSynchronize(s));
    ws.syncs++;
    const long long *h = ws.h_scalars64;
    if (ROWS)
    {
        P.row_windows = windows;
        P.accepted_row_windows = (int)h[0];
        P.row_tile_reduction = h[1];
        P.row_fanout_before = h[2];
        P.row_fanout_after = h[3];
    }
    else
    {
        P.inner_windows = windows;
        P.accepted_inner_windows = (int)h[0];
        P.inner_tile_reduction = h[1];
        P.inner_fanout_before = h[2];
        P.inner_fanout_after = h[3];
    }
    return RTT_OK;
}

} // namespace

int reorder_plan_device(Workspace &ws, const rtt_csr_view &A, int variant, rtt_reorder_plan *plan)
{
    if (variant < RTT_REORDER_FULL || variant > RTT_REORDER_UNGUARDED)
        return fail(RTT_ERR_INVALID_ARGUMENT, "reorder plan: unknown variant");
    // the stages of the variant (the reference's resolve_dmma_reorder_variant)
    const bool coarse = variant != RTT_REORDER_FINE;
    const bool row_fine = variant != RTT_REORDER_COARSE && variant != RTT_REORDER_COARSE_INNER;
    const bool inner_fine = variant != RTT_REORDER_COARSE && variant != RTT_REORDER_COARSE_ROW;
    const bool guarded = variant != RTT_REORDER_UNGUARDED;
    cudaStream_t s = ws.stream;
    const int m = A.rows, n = A.cols;
    Bufs B;
    DevBuf at_ptr, at_idx, at_val, pos_r, pos_c, k0, k1, prof, prop_n2o, prop_o2n, cnts, stats;
    AxisMaps rows, cols;
    int st = RTT_OK;
    rtt_reorder_plan P;
    std::memset(&P, 0, sizeof(P));
    P.rows = m;
    P.cols = n;
    P.nnz = (int)A.nnz;
    P.variant = variant;
    do
    {
        // column adjacency: A^T
        if ((st = at_ptr.ensure(sizeof(int) * ((size_t)n + 1), s)) != RTT_OK ||
            (st = at_idx.ensure(sizeof(int) * (size_t)A.nnz + 16, s)) != RTT_OK ||
            (st = at_val.ensure(sizeof(double) * (size_t)A.nnz + 16, s)) != RTT_OK ||
            (st = pos_r.ensure(sizeof(int) * (size_t)m + 16, s)) != RTT_OK ||
            (st = pos_c.ensure(sizeof(int) * (size_t)n + 16, s)) != RTT_OK ||
            (st = rows.o2n.ensure(sizeof(int) * (size_t)m + 16, s)) != RTT_OK ||
            (st = rows.n2o.ensure(sizeof(int) * (size_t)m + 16, s)) != RTT_OK ||
            (st = cols.o2n.ensure(sizeof(int) * (size_t)n + 16, s)) != RTT_OK ||
            (st = cols.n2o.ensure(sizeof(int) * (size_t)n + 16, s)) != RTT_OK)
            break;
        if ((st = csr_transpose_device(ws, m, n, (int)A.nnz, A.row_ptr, A.col_idx, A.values,
                                       at_ptr.as<int>(), at_idx.as<int>(),
                                       at_val.as<double>())) != RTT_OK)
            break;
        // the plan starts as A's own order
        if (m > 0)
            k_ro_iota<<<grid_of(m, 256), 256, 0, s>>>(m, rows.o2n.as<int>(), rows.n2o.as<int>());
        if (n > 0)
            k_ro_iota<<<grid_of(n, 256), 256, 0, s>>>(n, cols.o2n.as<int>(), cols.n2o.as<int>());
        ws.launches += 2;
        long long t_id = 0;
        if ((st = count_tiles(ws, A, nullptr, nullptr, k0, k1, &t_id)) != RTT_OK)
            break;
        P.tiles_before = t_id;
        P.proposal_tiles = t_id;
        if (coarse)
        {
            if ((st = bipartite_cm(ws, A, at_ptr.as<int>(), at_idx.as<int>(), pos_r.as<int>(),
                                   pos_c.as<int>(), B, &P.components, &P.levels, &P.active_rows,
                                   &P.active_inner)) != RTT_OK)
                break;
            // the exact commit rule: fewer 8x4 A tiles, or A's order stays
            long long t_new = 0;
            if ((st = count_tiles(ws, A, pos_r.as<int>(), pos_c.as<int>(), k0, k1, &t_new)) !=
                RTT_OK)
                break;
            P.proposal_tiles = t_new;
            P.accepted = !guarded || t_new < t_id;
            if (P.accepted)
            {
                const int sizes[2] = {m, n};
                const int *maps[2] = {pos_r.as<int>(), pos_c.as<int>()};
                AxisMaps *ax[2] = {&rows, &cols};
                for (int side = 0; side < 2 && st == RTT_OK; ++side)
                {
                    const int nv = sizes[side];
                    if (nv == 0)
                        continue;
                    cudaError_t e = cudaMemcpyAsync(ax[side]->o2n.p, maps[side],
                                                    sizeof(int) * (size_t)nv,
                                                    cudaMemcpyDeviceToDevice, s);
                    if (e != cudaSuccess)
                        st = cuda_fail(e, "reorder plan: coarse maps");
                    k_ro_inverse<<<grid_of(nv, 256), 256, 0, s>>>(nv, maps[side],
                                                                  ax[side]->n2o.as<int>());
                    ws.launches++;
                }
                if (st != RTT_OK)
                    break;
            }
        }
        if (row_fine && (st = fine_pass<true>(ws, A, at_ptr.as<int>(), at_idx.as<int>(), rows,
                                              cols, guarded, prof, prop_n2o, prop_o2n, k0, k1,
                                              cnts, stats, P)) != RTT_OK)
            break;
        if (inner_fine && (st = fine_pass<false>(ws, A, at_ptr.as<int>(), at_idx.as<int>(), rows,
                                                 cols, guarded, prof, prop_n2o, prop_o2n, k0, k1,
                                                 cnts, stats, P)) != RTT_OK)
            break;
        long long t_final = 0;
        if ((st = count_tiles(ws, A, rows.o2n.as<int>(), cols.o2n.as<int>(), k0, k1, &t_final)) !=
            RTT_OK)
            break;
        P.tiles_after = t_final;
        // host maps
        const size_t bm = sizeof(int) * (size_t)std::max(m, 1), bn = sizeof(int) * (size_t)std::max(n, 1);
        P.row_old_to_new = static_cast<int *>(std::malloc(bm));
        P.row_new_to_old = static_cast<int *>(std::malloc(bm));
        P.inner_old_to_new = static_cast<int *>(std::malloc(bn));
        P.inner_new_to_old = static_cast<int *>(std::malloc(bn));
        if (!P.row_old_to_new || !P.row_new_to_old || !P.inner_old_to_new || !P.inner_new_to_old)
        {
            st = fail(RTT_ERR_OUT_OF_MEMORY, "reorder plan: host maps");
            break;
        }
        const int sizes[2] = {m, n};
        const AxisMaps *ax[2] = {&rows, &cols};
        int *o2n[2] = {P.row_old_to_new, P.inner_old_to_new};
        int *n2o[2] = {P.row_new_to_old, P.inner_new_to_old};
        for (int side = 0; side < 2 && st == RTT_OK; ++side)
        {
            const int nv = sizes[side];
            if (nv == 0)
                continue;
            cudaError_t e = cudaMemcpyAsync(o2n[side], ax[side]->o2n.p, sizeof(int) * (size_t)nv,
                                            cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(n2o[side], ax[side]->n2o.p, sizeof(int) * (size_t)nv,
                                    cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess)
                e = cudaStreamSynchronize(s);
            if (e != cudaSuccess)
                st = cuda_fail(e, "reorder plan maps");
        }
        if (st != RTT_OK)
            break;
        for (int v = 0; v < m; ++v)
            P.moved_rows += P.row_old_to_new[v] != v;
        for (int v = 0; v < n; ++v)
            P.moved_inner += P.inner_old_to_new[v] != v;
    } while (0);
    cudaStreamSynchronize(s);
    B.release();
    DevBuf *tmp[] = {&at_ptr, &at_idx, &at_val, &pos_r, &pos_c, &k0, &k1, &prof, &prop_n2o,
                     &prop_o2n, &cnts, &stats, &rows.o2n, &rows.n2o, &cols.o2n, &cols.n2o};
    for (DevBuf *b : tmp)
        b->release();
    if (st != RTT_OK)
    {
        std::free(P.row_old_to_new);
        std::free(P.row_new_to_old);
        std::free(P.inner_old_to_new);
        std::free(P.inner_new_to_old);
        return st;
    }
    *plan = P;
    return RTT_OK;
}

int csr_permute_device(Workspace &ws, const rtt_csr_view &A, const int *row_new_to_old,
                       const int *col_old_to_new, int *out_rp, int *out_col, double *out_val)
{
    cudaStream_t s = ws.stream;
    const int m = A.rows;
    const long long nnz = A.nnz;
    // the maps must be permutations (no entry may land outside the output)
    RTT_CHECK(ws.tmp[0].ensure(sizeof(int) * ((size_t)std::max(m, A.cols) + 16), s));
    int *seen = ws.tmp[0].as<int>();
    if (row_new_to_old != nullptr && m > 0)
    {
        RTT_CUDA(cudaMemsetAsync(seen, 0, sizeof(int) * (size_t)m, s));
        k_perm_check<<<grid_of(m, 256), 256, 0, s>>>(m, row_new_to_old, seen, ws.err.as<int>());
        ws.launches++;
    }
    if (col_old_to_new != nullptr && A.cols > 0)
    {
        RTT_CUDA(cudaMemsetAsync(seen, 0, sizeof(int) * (size_t)A.cols, s));
        k_perm_check<<<grid_of(A.cols, 256), 256, 0, s>>>(A.cols, col_old_to_new, seen,
                                                          ws.err.as<int>());
        ws.launches++;
    }
    RTT_CHECK(check_device_error(ws, "csr_permute: maps"));
    RTT_CHECK(ws.tmp[1].ensure(sizeof(int) * ((size_t)m + 16), s));
    int *len = ws.tmp[1].as<int>();
    if (m > 0)
    {
        k_perm_lengths<<<grid_of(m, 256), 256, 0, s>>>(m, A.row_ptr, row_new_to_old, len);
        ws.launches++;
    }
    RTT_CHECK(scan_exclusive_int(ws, len, out_rp, m));
    if (nnz == 0)
        return RTT_OK;
    if (col_old_to_new == nullptr)
    {
        k_perm_copy<<<grid_of((long long)m * 32, 256), 256, 0, s>>>(
            m, A.row_ptr, A.col_idx, A.values, row_new_to_old, nullptr, out_rp, out_col, out_val);
        ws.launches++;
        return RTT_OK;
    }
    // mapped columns, then each row sorted by its new columns
    RTT_CHECK(ws.tmp[2].ensure(sizeof(int) * (size_t)nnz + 16, s));
    RTT_CHECK(ws.tmp[3].ensure(sizeof(double) * (size_t)nnz + 16, s));
    int *kc = ws.tmp[2].as<int>();
    double *kv = reinterpret_cast<double *>(ws.tmp[3].p);
    k_perm_copy<<<grid_of((long long)m * 32, 256), 256, 0, s>>>(
        m, A.row_ptr, A.col_idx, A.values, row_new_to_old, col_old_to_new, out_rp, kc, kv);
    ws.launches++;
    size_t bytes = 0;
    RTT_CUDA(cub::DeviceSegmentedSort::StableSortPairs(nullptr, bytes, kc, out_col, kv, out_val,
                                                       (int)nnz, m, out_rp, out_rp + 1, s));
    RTT_CHECK(ws.scan_tmp.ensure(bytes, s));
    RTT_CUDA(cub::DeviceSegmentedSort::StableSortPairs(ws.scan_tmp.p, bytes, kc, out_col, kv,
                                                       out_val, (int)nnz, m, out_rp, out_rp + 1,
                                                       s));
    ws.launches += 2;
    return RTT_OK;
}

} // namespace rtt
