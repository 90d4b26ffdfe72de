// diagnostics.cu - observability of the tile layout: the reorder plan dump
// and tile-count heatmaps of the last product's 16x16 tile grids.
//
// rtt_reorder_plan_dump writes the three files of the reference's
// dump_dmma_reorder_plan (src/dmma_reorder.h:3087-3209): <stem>_permutations.csv
// (axis,old_id,new_id,new_to_old_at_new_id), <stem>_unified_stats.csv
// (key,value) and <stem>_A_reordered.mtx (A's pattern under the plan, entries
// in A's original order).  The stats hold the counters this build's plan
// carries.  rtt_tile_heatmap bins the tiles of A, B or C of the last
// symbolic phase on a bins x bins grid over the tile grid, the role of the
// reference's export_diagnostic_heatmaps (src/super16_symbolic.cuh:2034) for
// this build's 16x16 tiles.
#include "rtt_internal.cuh"

#include <cstdio>
#include <string>
#include <vector>

namespace rtt
{
namespace
{

// one thread per tile row: every tile (I, J) adds one to bin (I * bins /
// tilem, J * bins / tilen)
__global__ void k_tile_heatmap(int tilem, int tilen, int bins, const int *__restrict__ tile_ptr,
                               const int *__restrict__ tile_col,
                               unsigned long long *__restrict__ hist, int *err)
{
    const int I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= tilem)
        return;
    const long long bi = (long long)I * bins / tilem;
    for (int t = tile_ptr[I]; t < tile_ptr[I + 1]; ++t)
    {
        const int J = tile_col[t];
        if (J < 0 || J >= tilen)
        {
            set_error(err, DERR_NUM_BOUNDS);
            continue;
        }
        const long long bj = (long long)J * bins / tilen;
        atomicAdd(&hist[bi * bins + bj], 1ull);
    }
}

} // namespace

int tile_heatmap_device(Workspace &ws, int tilem, int tilen, const int *tile_ptr,
                        const int *tile_col, int bins, unsigned long long *d_hist)
{
    RTT_CUDA(cudaMemsetAsync(d_hist, 0, sizeof(unsigned long long) * (size_t)bins * bins,
                             ws.stream));
    if (tilem > 0 && tilen > 0)
    {
        k_tile_heatmap<<<(tilem + 255) / 256, 256, 0, ws.stream>>>(tilem, tilen, bins, tile_ptr,
                                                                    tile_col, d_hist,
                                                                    ws.err.as<int>());
        ws.launches++;
    }
    return RTT_OK;
}

} // namespace rtt

extern "C" {

int rtt_reorder_plan_dump(const rtt_reorder_plan *plan, const char *stem, const int *d_row_ptr,
                          const int *d_col_idx, int dump_matrix)
{
    using rtt::fail;
    if (plan == nullptr || stem == nullptr || *stem == '\0' ||
        (plan->rows > 0 && (plan->row_old_to_new == nullptr || plan->row_new_to_old == nullptr)) ||
        (plan->cols > 0 && (plan->inner_old_to_new == nullptr || plan->inner_new_to_old == nullptr)))
        return fail(RTT_ERR_INVALID_ARGUMENT, "reorder_plan_dump: bad arguments");
    const std::string prefix(stem);
    FILE *f = std::fopen((prefix + "_permutations.csv").c_str(), "w");
    if (f == nullptr)
        return fail(RTT_ERR_INVALID_ARGUMENT, "reorder_plan_dump: cannot write " + prefix);
    std::fprintf(f, "axis,old_id,new_id,new_to_old_at_new_id\n");
    for (int o = 0; o < plan->rows; ++o)
    {
        const int nw = plan->row_old_to_new[o];
        std::fprintf(f, "row,%d,%d,%d\n", o, nw, plan->row_new_to_old[nw]);
    }
    for (int o = 0; o < plan->cols; ++o)
    {
        const int nw = plan->inner_old_to_new[o];
        std::fprintf(f, "inner,%d,%d,%d\n", o, nw, plan->inner_new_to_old[nw]);
    }
    if (std::fclose(f) != 0)
        return fail(RTT_ERR_INVALID_ARGUMENT, "reorder_plan_dump: write failed");
    f = std::fopen((prefix + "_unified_stats.csv").c_str(), "w");
    if (f == nullptr)
        return fail(RTT_ERR_INVALID_ARGUMENT, "reorder_plan_dump: cannot write stats");
    static const char *const variants[] = {"full", "coarse", "fine", "coarse-row",
                                           "coarse-inner", "unguarded"};
    const int vi = plan->variant >= 0 && plan->variant <= 5 ? plan->variant : 0;
    std::fprintf(f, "key,value\nalgorithm,bipartite_cm+fine\nvariant,%s\n", variants[vi]);
    std::fprintf(f,
                 "rows,%d\ncols,%d\nnnz,%d\nactive_rows,%d\nactive_inner,%d\n"
                 "moved_rows,%lld\nmoved_inner,%lld\ncoarse_components,%d\ncoarse_levels,%d\n"
                 "coarse_candidate_accepted,%d\ntiles_before,%lld\ntiles_after,%lld\n"
                 "proposal_tiles,%lld\ncoarse_tile_reduction,%lld\n",
                 plan->rows, plan->cols, plan->nnz, plan->active_rows, plan->active_inner,
                 plan->moved_rows, plan->moved_inner, plan->components, plan->levels,
                 plan->accepted, plan->tiles_before, plan->tiles_after, plan->proposal_tiles,
                 plan->accepted ? plan->tiles_before - plan->proposal_tiles : 0ll);
    std::fprintf(f,
                 "row_windows,%d\naccepted_row_windows,%d\nrow_tile_reduction,%lld\n"
                 "row_fanout_before,%lld\nrow_fanout_after,%lld\n"
                 "inner_windows,%d\naccepted_inner_windows,%d\ninner_tile_reduction,%lld\n"
                 "inner_fanout_before,%lld\ninner_fanout_after,%lld\n",
                 plan->row_windows, plan->accepted_row_windows, plan->row_tile_reduction,
                 plan->row_fanout_before, plan->row_fanout_after, plan->inner_windows,
                 plan->accepted_inner_windows, plan->inner_tile_reduction,
                 plan->inner_fanout_before, plan->inner_fanout_after);
    if (std::fclose(f) != 0)
        return fail(RTT_ERR_INVALID_ARGUMENT, "reorder_plan_dump: write failed");
    if (!dump_matrix)
        return RTT_OK;
    if ((plan->rows > 0 && d_row_ptr == nullptr) || (plan->nnz > 0 && d_col_idx == nullptr))
        return fail(RTT_ERR_INVALID_ARGUMENT, "reorder_plan_dump: A's structure is needed");
    std::vector<int> rp((size_t)plan->rows + 1, 0), ci((size_t)plan->nnz);
    if (plan->rows >= 0)
        RTT_CUDA(cudaMemcpy(rp.data(), d_row_ptr, sizeof(int) * rp.size(), cudaMemcpyDeviceToHost));
    if (plan->nnz > 0)
        RTT_CUDA(cudaMemcpy(ci.data(), d_col_idx, sizeof(int) * ci.size(), cudaMemcpyDeviceToHost));
    if (rp[0] != 0 || rp[(size_t)plan->rows] != plan->nnz)
        return fail(RTT_ERR_INVALID_CSR, "reorder_plan_dump: row pointer disagrees with the plan");
    f = std::fopen((prefix + "_A_reordered.mtx").c_str(), "w");
    if (f == nullptr)
        return fail(RTT_ERR_INVALID_ARGUMENT, "reorder_plan_dump: cannot write the matrix");
    std::fprintf(f, "%%%%MatrixMarket matrix coordinate pattern general\n");
    std::fprintf(f, "%% A under the row / inner reorder plan\n");
    std::fprintf(f, "%d %d %d\n", plan->rows, plan->cols, plan->nnz);
    for (int o = 0; o < plan->rows; ++o)
        for (int e = rp[(size_t)o]; e < rp[(size_t)o + 1]; ++e)
        {
            const int c = ci[(size_t)e];
            if (c < 0 || c >= plan->cols)
            {
                std::fclose(f);
                return fail(RTT_ERR_INVALID_CSR, "reorder_plan_dump: column out of range");
            }
            std::fprintf(f, "%d %d\n", plan->row_old_to_new[o] + 1, plan->inner_old_to_new[c] + 1);
        }
    if (std::fclose(f) != 0)
        return fail(RTT_ERR_INVALID_ARGUMENT, "reorder_plan_dump: write failed");
    return RTT_OK;
}

} // extern "C"
