// tile8.cu - legacy 16x16 C tiles -> the reference's native 8x8 output tiles.
//
// The reference's GPU path exports C as 8x8 tiles (dmma_copy_output_to_host,
// src/dmma_spgemm.h:6399-6488; per-tile row offsets as in dmma_numeric_kernel,
// :4266-4283; empty quadrants dropped, src/super16_symbolic.cuh:1740-1963).
// Each 16x16 tile splits into its four 8x8 quadrants; quadrants with no entry
// are dropped; tiles are ordered by 8-row tile row, then 8-column tile column.
// A warp owns one 16-row tile row: lanes take 16x16 tiles 32 at a time and a
// warp scan places the emitted quadrants (tile index and value offset).
#include "rtt_internal.cuh"

#include <cstdlib>
#include <cstring>

namespace rtt
{
namespace
{

// quadrant entry counts of 16x16 tile t for half h (rows 8h..8h+7)
__device__ __forceinline__ void quad_counts(const int *tnnz, const uint8_t *ptr, const uint8_t *col,
                                            int t, int h, int &n0, int &n1)
{
    const int b = tnnz[t], cnt = tnnz[t + 1] - b;
    n0 = 0;
    n1 = 0;
    for (int r = 8 * h; r < 8 * h + 8; ++r)
    {
        int s = ptr[(size_t)t * TD + r];
        int e = r == TD - 1 ? cnt : ptr[(size_t)t * TD + r + 1];
        s = min(s, cnt);
        e = min(max(e, s), cnt);
        for (int i = s; i < e; ++i)
        {
            if (col[b + i] < 8)
                ++n0;
            else if (col[b + i] < 16)
                ++n1;
        }
    }
}

__global__ void k_t8_count(int tilem, int tm8, const int *__restrict__ tile_ptr,
                           const int *__restrict__ tnnz, const uint8_t *__restrict__ ptr,
                           const uint8_t *__restrict__ col, int *__restrict__ cnt8,
                           int *__restrict__ nnz8)
{
    const int lane = threadIdx.x & 31;
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (I >= tilem)
        return;
    for (int h = 0; h < 2; ++h)
    {
        const int R8 = 2 * I + h;
        int tiles = 0, ent = 0;
        for (int t = tile_ptr[I] + lane; t < tile_ptr[I + 1]; t += 32)
        {
            int n0, n1;
            quad_counts(tnnz, ptr, col, t, h, n0, n1);
            tiles += (n0 > 0) + (n1 > 0);
            ent += n0 + n1;
        }
        tiles = warp_sum(tiles);
        ent = warp_sum(ent);
        if (lane == 0 && R8 < tm8)
        {
            cnt8[R8] = tiles;
            nnz8[R8] = ent;
        }
    }
}

__global__ void k_t8_fill(int tilem, int tm8, const int *__restrict__ tile_ptr,
                          const int *__restrict__ tile_col, const int *__restrict__ tnnz,
                          const uint8_t *__restrict__ ptr, const uint8_t *__restrict__ col,
                          const double *__restrict__ val, const int *__restrict__ tp8,
                          const int *__restrict__ base8, int *__restrict__ o_col,
                          int *__restrict__ o_row, int *__restrict__ o_nnz,
                          uint8_t *__restrict__ o_ptr, uint8_t *__restrict__ o_colb,
                          double *__restrict__ o_val)
{
    const int lane = threadIdx.x & 31;
    const int I = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (I >= tilem)
        return;
    for (int h = 0; h < 2; ++h)
    {
        const int R8 = 2 * I + h;
        if (R8 >= tm8)
            break;
        int t8 = tp8[R8], v8 = base8[R8];
        for (int t0 = tile_ptr[I]; t0 < tile_ptr[I + 1]; t0 += 32)
        {
            const int t = t0 + lane;
            int n0 = 0, n1 = 0;
            if (t < tile_ptr[I + 1])
                quad_counts(tnnz, ptr, col, t, h, n0, n1);
            const int nt = (n0 > 0) + (n1 > 0), ne = n0 + n1;
            const int it = warp_incl_scan(nt), ie = warp_incl_scan(ne);
            int my_t = t8 + it - nt, my_v = v8 + ie - ne;
            if (t < tile_ptr[I + 1])
            {
                const int J = tile_col[t];
                const int b = tnnz[t], cnt = tnnz[t + 1] - b;
                for (int qc = 0; qc < 2; ++qc)
                {
                    if ((qc == 0 ? n0 : n1) == 0)
                        continue;
                    o_col[my_t] = 2 * J + qc;
                    o_row[my_t] = R8;
                    o_nnz[my_t] = my_v;
                    int k = 0;
                    for (int rr = 0; rr < 8; ++rr)
                    {
                        const int r = 8 * h + rr;
                        o_ptr[(size_t)my_t * 8 + rr] = (uint8_t)k;
                        int s = ptr[(size_t)t * TD + r];
                        int e = r == TD - 1 ? cnt : ptr[(size_t)t * TD + r + 1];
                        s = min(s, cnt);
                        e = min(max(e, s), cnt);
                        for (int i = s; i < e; ++i)
                        {
                            const int c = col[b + i];
                            if (c >= 8 * qc && c < 8 * qc + 8)
                            {
                                o_colb[my_v + k] = (uint8_t)(c - 8 * qc);
                                o_val[my_v + k] = val[b + i];
                                ++k;
                            }
                        }
                    }
                    my_v += k;
                    ++my_t;
                }
            }
            t8 += __shfl_sync(FULL, it, 31);
            v8 += __shfl_sync(FULL, ie, 31);
        }
    }
}

__global__ void k_put_int(int *p, const int *src) { *p = *src; }

inline int grid_for(long long threads, int block) { return (int)((threads + block - 1) / block); }

} // namespace
} // namespace rtt

extern "C" int rtt_tile16_to_tile8(const SMatrix *C, SMatrix *O)
{
    using namespace rtt;
    if (C == nullptr || O == nullptr || C->m < 0 || C->n < 0 || C->numtile < 0 ||
        C->tile_ptr == nullptr || C->tile_nnz == nullptr ||
        (C->numtile > 0 && (C->tile_columnidx == nullptr || C->tile_csr_Ptr == nullptr)))
        return fail(RTT_ERR_INVALID_ARGUMENT, "tile16_to_tile8: malformed tile matrix");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
    {
        cudaGetLastError();
        return fail(RTT_ERR_NO_DEVICE, "no CUDA device available");
    }
    Workspace ws;
    RTT_CHECK(ws.init(dev));
    struct WsGuard
    {
        Workspace &w;
        ~WsGuard() { w.destroy(); }
    } wsg{ws};
    cudaStream_t s = ws.stream;
    const int tilem = ceil_div(C->m, TD), nt = C->numtile;
    const int tm8 = ceil_div(C->m, 8), tn8 = ceil_div(C->n, 8);
    const int nent = C->tile_nnz[nt];
    DevBuf tp, tc, tn, P, Cb, V, cnt8, nnz8, tp8, base8;
    DevBuf *all[] = {&tp, &tc, &tn, &P, &Cb, &V, &cnt8, &nnz8, &tp8, &base8};
    struct BufGuard
    {
        DevBuf **b;
        int n;
        ~BufGuard()
        {
            for (int i = 0; i < n; ++i)
                b[i]->release();
        }
    } bg{all, 10};
    auto up = [&](DevBuf &b, const void *h, size_t bytes) -> int {
        RTT_CHECK(b.ensure(bytes + 16, s));
        if (bytes > 0)
            RTT_CUDA(cudaMemcpyAsync(b.p, h, bytes, cudaMemcpyHostToDevice, s));
        return RTT_OK;
    };
    RTT_CHECK(up(tp, C->tile_ptr, sizeof(int) * ((size_t)tilem + 1)));
    RTT_CHECK(up(tc, C->tile_columnidx, sizeof(int) * (size_t)nt));
    RTT_CHECK(up(tn, C->tile_nnz, sizeof(int) * ((size_t)nt + 1)));
    RTT_CHECK(up(P, C->tile_csr_Ptr, (size_t)nt * TD));
    RTT_CHECK(up(Cb, C->tile_csr_Col, (size_t)nent));
    RTT_CHECK(up(V, C->tile_csr_Value, sizeof(double) * (size_t)nent));
    RTT_CHECK(cnt8.ensure(sizeof(int) * ((size_t)tm8 + 1), s));
    RTT_CHECK(nnz8.ensure(sizeof(int) * ((size_t)tm8 + 1), s));
    RTT_CHECK(tp8.ensure(sizeof(int) * ((size_t)tm8 + 1), s));
    RTT_CHECK(base8.ensure(sizeof(int) * ((size_t)tm8 + 1), s));
    RTT_CUDA(cudaMemsetAsync(cnt8.p, 0, sizeof(int) * ((size_t)tm8 + 1), s));
    RTT_CUDA(cudaMemsetAsync(nnz8.p, 0, sizeof(int) * ((size_t)tm8 + 1), s));
    if (tilem > 0)
        k_t8_count<<<grid_for((long long)tilem * 32, 256), 256, 0, s>>>(
            tilem, tm8, tp.as<int>(), tn.as<int>(), P.as<uint8_t>(), Cb.as<uint8_t>(),
            cnt8.as<int>(), nnz8.as<int>());
    RTT_CHECK(scan_exclusive_int(ws, cnt8.as<int>(), tp8.as<int>(), tm8));
    RTT_CHECK(scan_exclusive_int(ws, nnz8.as<int>(), base8.as<int>(), tm8));
    int nt8 = 0, ne8 = 0;
    RTT_CHECK(read_int(ws, tp8.as<int>() + tm8, &nt8));
    RTT_CHECK(read_int(ws, base8.as<int>() + tm8, &ne8));
    DevBuf oc, orow, on, op, ocb, ov;
    DevBuf *outs[] = {&oc, &orow, &on, &op, &ocb, &ov};
    BufGuard og{outs, 6};
    RTT_CHECK(oc.ensure(sizeof(int) * (size_t)nt8 + 16, s));
    RTT_CHECK(orow.ensure(sizeof(int) * (size_t)nt8 + 16, s));
    RTT_CHECK(on.ensure(sizeof(int) * ((size_t)nt8 + 1) + 16, s));
    RTT_CHECK(op.ensure((size_t)nt8 * 8 + 16, s));
    RTT_CHECK(ocb.ensure((size_t)ne8 + 16, s));
    RTT_CHECK(ov.ensure(sizeof(double) * (size_t)ne8 + 16, s));
    if (tilem > 0)
        k_t8_fill<<<grid_for((long long)tilem * 32, 256), 256, 0, s>>>(
            tilem, tm8, tp.as<int>(), tc.as<int>(), tn.as<int>(), P.as<uint8_t>(), Cb.as<uint8_t>(),
            V.as<double>(), tp8.as<int>(), base8.as<int>(), oc.as<int>(), orow.as<int>(),
            on.as<int>(), op.as<uint8_t>(), ocb.as<uint8_t>(), ov.as<double>());
    k_put_int<<<1, 1, 0, s>>>(on.as<int>() + nt8, base8.as<int>() + tm8);
    RTT_CHECK(check_device_error(ws, "tile16_to_tile8"));
    int *h_tp = (int *)std::malloc(sizeof(int) * ((size_t)tm8 + 1));
    int *h_tc = (int *)std::malloc(sizeof(int) * ((size_t)nt8 + 1));
    int *h_tr = (int *)std::malloc(sizeof(int) * ((size_t)nt8 + 1));
    int *h_tn = (int *)std::malloc(sizeof(int) * ((size_t)nt8 + 1));
    unsigned char *h_p = (unsigned char *)std::malloc((size_t)nt8 * 8 + 1);
    unsigned char *h_c = (unsigned char *)std::malloc((size_t)ne8 + 1);
    double *h_v = (double *)std::malloc(sizeof(double) * ((size_t)ne8 + 1));
    if (!h_tp || !h_tc || !h_tr || !h_tn || !h_p || !h_c || !h_v)
    {
        std::free(h_tp);
        std::free(h_tc);
        std::free(h_tr);
        std::free(h_tn);
        std::free(h_p);
        std::free(h_c);
        std::free(h_v);
        return fail(RTT_ERR_OUT_OF_MEMORY, "host malloc failed");
    }
    cudaError_t e = cudaMemcpyAsync(h_tp, tp8.p, sizeof(int) * ((size_t)tm8 + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_tc, oc.p, sizeof(int) * (size_t)nt8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_tr, orow.p, sizeof(int) * (size_t)nt8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_tn, on.p, sizeof(int) * ((size_t)nt8 + 1), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_p, op.p, (size_t)nt8 * 8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_c, ocb.p, (size_t)ne8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h_v, ov.p, sizeof(double) * (size_t)ne8, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess)
        e = cudaStreamSynchronize(s);
    if (e != cudaSuccess)
    {
        std::free(h_tp);
        std::free(h_tc);
        std::free(h_tr);
        std::free(h_tn);
        std::free(h_p);
        std::free(h_c);
        std::free(h_v);
        return cuda_fail(e, "tile16_to_tile8 copy back");
    }
    std::memset(O, 0, sizeof(*O));
    O->m = C->m;
    O->n = C->n;
    O->nnz = ne8;
    O->tilem = tm8;
    O->tilen = tn8;
    O->numtile = nt8;
    O->tile_ptr = h_tp;
    O->tile_columnidx = h_tc;
    O->tile_rowidx = h_tr;
    O->tile_nnz = h_tn;
    O->tile_csr_Ptr = h_p;
    O->tile_csr_Col = h_c;
    O->tile_csr_Value = h_v;
    return RTT_OK;
}
