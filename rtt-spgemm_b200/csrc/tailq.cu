// tailq.cu - the tail-queue admission planner on the device.
//
// Semantics of dmma_plan_tile_tail_queue (reference
// src/dmma_tile_tail_queue.h:190-291, with the chunk rule of :148-176): a
// task (one output tile of the numeric step, described by its K-list merge
// scans, matched pairs and output entries) stays an ordinary one-warp task
// unless its FP32 work scan * scans + match * matches exceeds the admission
// threshold and it has more than one scan; an admitted (heavy) task is split
// into ceil(work / chunk_target) chunks, clamped to [2, max_chunks] and to its
// scan count.  Tasks are checked in order: the first invalid task, or the
// first heavy task past the record capacity, voids the plan.  Otherwise the
// plan is gated on zero heavy tasks, the heavy fraction and the partial
// workspace (one 8x8 FP64 accumulator, 512 bytes, per chunk).
//
// One thread per task computes validity and chunks with the same
// round-to-nearest FP32 operations (no contraction); the first-failure
// indices and the totals come from device reductions.
#include "rtt_internal.cuh"

#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>

#include <climits>
#include <cmath>
#include <cstring>

namespace rtt
{
namespace
{

enum TailReason
{
    TQ_DEFAULT_OFF = 0,
    TQ_ENABLED = 1,
    TQ_INVALID_POLICY = 2,
    TQ_INVALID_TASK = 3,
    TQ_ZERO_HEAVY = 4,
    TQ_RECORD_CAPACITY = 5,
    TQ_HEAVY_FRACTION = 6,
    TQ_WORKSPACE_CAPACITY = 7,
};

struct TqParams
{
    float scan, match, threshold, target, max_chunks_f;
    int max_chunks;
};

// chunks of one task (0 = ordinary), the reference's FP32 rule
__device__ __forceinline__ int tq_chunks(int scans, int matches, const TqParams &p)
{
    const float work = __fadd_rn(__fmul_rn(p.scan, (float)scans), __fmul_rn(p.match, (float)matches));
    if (!(work > p.threshold) || scans <= 1)
        return 0;
    const float requested = ceilf(__fdiv_rn(work, p.target));
    int chunks = requested >= p.max_chunks_f ? p.max_chunks : (int)requested;
    if (chunks < 2)
        chunks = 2;
    if (chunks > scans)
        chunks = scans;
    return chunks >= 2 ? chunks : 0;
}

// per task: chunks, heavy flag; first invalid task index (atomicMin)
__global__ void k_tq_tasks(int n, const int *__restrict__ scans, const int *__restrict__ matches,
                           const int *__restrict__ out_nnz, TqParams p, int *__restrict__ chunks,
                           int *__restrict__ heavy, int *__restrict__ first_invalid)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const int s = scans[i], mt = matches[i], o = out_nnz[i];
    if (s < 0 || mt < 0 || mt > s || o < 0 || o > 64)
    {
        atomicMin(first_invalid, i);
        chunks[i] = 0;
        heavy[i] = 0;
        return;
    }
    const int c = tq_chunks(s, mt, p);
    chunks[i] = c;
    heavy[i] = c > 0 ? 1 : 0;
}

// first task whose inclusive heavy count exceeds the record capacity
__global__ void k_tq_capacity(int n, const int *__restrict__ heavy_incl, int capacity,
                              int *__restrict__ first_over)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && heavy_incl[i] > capacity)
        atomicMin(first_over, i);
}

inline int nblocks(long long n) { return (int)((n + 255) / 256); }

} // namespace

int plan_tail_queue_device(Workspace &ws, int n, const int *d_scans, const int *d_matches,
                           const int *d_out, const rtt_tail_policy &pol,
                           const rtt_tail_cost_model &model, int *d_chunks, rtt_tail_plan *plan)
{
    cudaStream_t s = ws.stream;
    std::memset(plan, 0, sizeof(*plan));
    plan->output_tasks = n;
    plan->ordinary_tasks = n;
    if (!pol.enabled)
    {
        plan->reason = TQ_DEFAULT_OFF;
        RTT_CUDA(cudaMemsetAsync(d_chunks, 0, sizeof(int) * (size_t)(n > 0 ? n : 1), s));
        return RTT_OK;
    }
    const bool valid = std::isfinite(pol.admission_threshold) && pol.admission_threshold > 0.0 &&
                       std::isfinite(pol.chunk_target) && pol.chunk_target > 0.0 &&
                       pol.max_chunks >= 2 && pol.max_chunks <= 32 &&
                       std::isfinite(pol.max_heavy_fraction) && pol.max_heavy_fraction >= 0.0 &&
                       pol.max_heavy_fraction <= 1.0 && pol.record_capacity > 0 &&
                       std::isfinite(model.intercept) && model.intercept >= 0.0 &&
                       std::isfinite(model.scan) && model.scan >= 0.0 &&
                       std::isfinite(model.match) && model.match >= 0.0 &&
                       std::isfinite(model.output) && model.output >= 0.0;
    if (!valid)
    {
        plan->reason = TQ_INVALID_POLICY;
        RTT_CUDA(cudaMemsetAsync(d_chunks, 0, sizeof(int) * (size_t)(n > 0 ? n : 1), s));
        return RTT_OK;
    }
    TqParams p;
    p.scan = (float)model.scan;
    p.match = (float)model.match;
    p.threshold = (float)pol.admission_threshold;
    p.target = (float)pol.chunk_target;
    p.max_chunks = pol.max_chunks;
    p.max_chunks_f = (float)pol.max_chunks;

    long long heavy = 0, chunks = 0;
    int first_invalid = INT_MAX, first_over = INT_MAX;
    if (n > 0)
    {
        DevBuf heavy_b, incl_b, cnt_b, small_b, sum_b;
        RTT_CHECK(heavy_b.ensure(sizeof(int) * (size_t)n, s));
        RTT_CHECK(incl_b.ensure(sizeof(int) * ((size_t)n + 1), s));
        RTT_CHECK(small_b.ensure(sizeof(int) * 4, s));
        RTT_CHECK(sum_b.ensure(sizeof(long long) * 2, s));
        int *flags = small_b.as<int>();
        const int init[2] = {INT_MAX, INT_MAX};
        RTT_CUDA(cudaMemcpyAsync(flags, init, sizeof(init), cudaMemcpyHostToDevice, s));
        k_tq_tasks<<<nblocks(n), 256, 0, s>>>(n, d_scans, d_matches, d_out, p, d_chunks,
                                              heavy_b.as<int>(), flags);
        // inclusive heavy counts (exclusive scan shifted by one)
        RTT_CHECK(scan_exclusive_int(ws, heavy_b.as<int>(), incl_b.as<int>(), n));
        k_tq_capacity<<<nblocks(n), 256, 0, s>>>(n, incl_b.as<int>() + 1, pol.record_capacity,
                                                 flags + 1);
        long long *sums = sum_b.as<long long>();
        size_t bytes = 0;
        RTT_CUDA(cub::DeviceReduce::Sum(nullptr, bytes, d_chunks, sums, n, s));
        RTT_CHECK(ws.scan_tmp.ensure(bytes, s));
        RTT_CUDA(cub::DeviceReduce::Sum(ws.scan_tmp.p, bytes, d_chunks, sums, n, s));
        int hflags[2];
        RTT_CUDA(cudaMemcpyAsync(hflags, flags, sizeof(hflags), cudaMemcpyDeviceToHost, s));
        int h_heavy = 0;
        RTT_CUDA(cudaMemcpyAsync(&h_heavy, incl_b.as<int>() + n, sizeof(int), cudaMemcpyDeviceToHost, s));
        RTT_CUDA(cudaMemcpyAsync(&chunks, sums, sizeof(long long), cudaMemcpyDeviceToHost, s));
        RTT_CUDA(cudaStreamSynchronize(s));
        heavy_b.release();
        incl_b.release();
        small_b.release();
        sum_b.release();
        first_invalid = hflags[0];
        first_over = hflags[1];
        heavy = h_heavy;
    }
    // the first failure in task order voids the plan (the reference returns
    // at the first invalid task or the first heavy task past the capacity)
    if (first_invalid != INT_MAX || first_over != INT_MAX)
    {
        plan->reason = first_invalid <= first_over ? TQ_INVALID_TASK : TQ_RECORD_CAPACITY;
        RTT_CUDA(cudaMemsetAsync(d_chunks, 0, sizeof(int) * (size_t)n, s));
        return RTT_OK;
    }
    plan->heavy_tasks = heavy;
    plan->ordinary_tasks = n - heavy;
    plan->chunks = chunks;
    plan->heavy_fraction = n == 0 ? 0.0 : (double)heavy / (double)n;
    plan->average_chunks = heavy == 0 ? 0.0 : (double)chunks / (double)heavy;
    plan->heavy_flag_bytes = (((long long)n + 31) / 32) * 4;
    plan->descriptor_bytes = chunks * 16;
    plan->partial_workspace_bytes = chunks * 64 * (long long)sizeof(double);
    if (heavy == 0)
        plan->reason = TQ_ZERO_HEAVY;
    else if (plan->heavy_fraction > pol.max_heavy_fraction)
        plan->reason = TQ_HEAVY_FRACTION;
    else if (pol.workspace_reduction && plan->partial_workspace_bytes > pol.workspace_limit_bytes)
        plan->reason = TQ_WORKSPACE_CAPACITY;
    else
        plan->reason = TQ_ENABLED;
    return RTT_OK;
}

} // namespace rtt
