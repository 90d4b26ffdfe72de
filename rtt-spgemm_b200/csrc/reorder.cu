// reorder.cu - row / inner (K) reordering of A for the tiled SpGEMM.
//
// The reference's BGRF reorder (src/dmma_reorder.h:37-47, :2651-3085) is a
// bipartite Cuthill-McKee traversal of A's row/column graph on the GPU whose
// joint row/K proposal is committed only if it cuts the number of 8x4 A
// tiles (the exact commit rule, :1671-1727), followed by fine passes that
// pack 8x4 tensor-core groups.  This build keeps the traversal and the commit
// rule and leaves out the fine passes:
//
//  * proposal: a level-synchronous breadth-first traversal that alternates
//    rows and columns.  Each level's new vertices are ordered by the position
//    of their earliest-placed neighbour in the level before (the Cuthill-McKee
//    rule), then by degree, then by index.  A component starts at its
//    unplaced row of least (degree, index); rows and columns without entries
//    go last, in index order.
//  * commit: the distinct 8x4 tiles of A under the proposal are counted
//    exactly (sort + unique of tile keys) against the identity; the proposal
//    becomes the plan only if it has fewer tiles, so a plan never increases
//    A's tile count.
//
// With C = A*B, A' = P A Q^T and B' = Q B give A' B' = P C: C's rows come back
// with rtt_tile2csr_restore_rows or rtt_csr_permute(row_new_to_old = P^T).
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

int reorder_plan_device(Workspace &ws, const rtt_csr_view &A, rtt_reorder_plan *plan)
{
    cudaStream_t s = ws.stream;
    const int m = A.rows, n = A.cols;
    Bufs B;
    DevBuf at_ptr, at_idx, at_val, pos_r, pos_c, k0, k1, inv;
    int st = RTT_OK;
    rtt_reorder_plan P;
    std::memset(&P, 0, sizeof(P));
    P.rows = m;
    P.cols = n;
    P.nnz = (int)A.nnz;
    do
    {
        // column adjacency: A^T
        if ((st = at_ptr.ensure(sizeof(int) * ((size_t)n + 1), s)) != RTT_OK ||
            (st = at_idx.ensure(sizeof(int) * (size_t)A.nnz + 16, s)) != RTT_OK ||
            (st = at_val.ensure(sizeof(double) * (size_t)A.nnz + 16, s)) != RTT_OK ||
            (st = pos_r.ensure(sizeof(int) * (size_t)m + 16, s)) != RTT_OK ||
            (st = pos_c.ensure(sizeof(int) * (size_t)n + 16, s)) != RTT_OK)
            break;
        if ((st = csr_transpose_device(ws, m, n, (int)A.nnz, A.row_ptr, A.col_idx, A.values,
                                       at_ptr.as<int>(), at_idx.as<int>(),
                                       at_val.as<double>())) != RTT_OK)
            break;
        if ((st = bipartite_cm(ws, A, at_ptr.as<int>(), at_idx.as<int>(), pos_r.as<int>(),
                               pos_c.as<int>(), B, &P.components, &P.levels, &P.active_rows,
                               &P.active_inner)) != RTT_OK)
            break;
        // the exact commit rule: fewer 8x4 A tiles, or the identity
        long long t_id = 0, t_new = 0;
        if ((st = count_tiles(ws, A, nullptr, nullptr, k0, k1, &t_id)) != RTT_OK ||
            (st = count_tiles(ws, A, pos_r.as<int>(), pos_c.as<int>(), k0, k1, &t_new)) != RTT_OK)
            break;
        P.tiles_before = t_id;
        P.accepted = t_new < t_id;
        P.tiles_after = P.accepted ? t_new : t_id;
        P.proposal_tiles = t_new;
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
        if ((st = inv.ensure(sizeof(int) * ((size_t)std::max(m, n) + 16), s)) != RTT_OK)
            break;
        const int sizes[2] = {m, n};
        const int *maps[2] = {pos_r.as<int>(), pos_c.as<int>()};
        int *o2n[2] = {P.row_old_to_new, P.inner_old_to_new};
        int *n2o[2] = {P.row_new_to_old, P.inner_new_to_old};
        for (int side = 0; side < 2 && st == RTT_OK; ++side)
        {
            const int nv = sizes[side];
            if (nv == 0)
                continue;
            if (!P.accepted)
            {
                for (int v = 0; v < nv; ++v)
                    o2n[side][v] = n2o[side][v] = v;
                continue;
            }
            k_ro_inverse<<<grid_of(nv, 256), 256, 0, s>>>(nv, maps[side], inv.as<int>());
            ws.launches++;
            cudaError_t e = cudaMemcpyAsync(o2n[side], maps[side], sizeof(int) * (size_t)nv,
                                            cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(n2o[side], inv.as<int>(), sizeof(int) * (size_t)nv,
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
    DevBuf *tmp[] = {&at_ptr, &at_idx, &at_val, &pos_r, &pos_c, &k0, &k1, &inv};
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
