// Multi-network batch kernel: one persistent launch over many (network,
// query) jobs, each run simulated by one thread with the step of
// sim_run.cuh.
//
// Work queue.  The runs of all jobs are numbered in one index space (job j
// owns [run_begin_j, run_begin_j + n_runs_j)); a lane whose run ends takes
// the next index from the shared device counter (warp-aggregated atomic),
// finds its job by binary search in the job table (staged in shared memory)
// and starts that run, so uneven run lengths and uneven job sizes leave no
// lane idle until the whole batch is drained.  Lanes of one warp are on the
// same job except at the few indices where one job ends and the next begins.
//
// Memory.  Networks stay in global memory (read-only, L1/L2-resident while
// in use); each CTA's run state is a global slab laid out for the largest
// job of the batch (interleaved by thread, so warp accesses coalesce).
// Results depend only on the job and the run index.
#pragma once
#include "sim_run.cuh"

namespace csmc {
namespace detail {

#ifndef CSMC_BATCH_MIN_CTAS_PER_SM
#define CSMC_BATCH_MIN_CTAS_PER_SM 4
#endif

// Index of the job owning run index r: the last job with run_begin <= r.
static __device__ __forceinline__ uint32_t find_job(const BatchJob *jobs, uint32_t n_jobs, unsigned long long r) {
    uint32_t lo = 0, hi = n_jobs;  // invariant: jobs[lo].run_begin <= r < jobs[hi].run_begin
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (jobs[mid].run_begin <= r) lo = mid;
        else hi = mid;
    }
    return lo;
}

static __device__ __forceinline__ void flush_counters(const BatchJob &J, unsigned long long &hits,
                                                      unsigned long long &steps, unsigned long long &capped) {
    if (hits) atomicAdd(J.counters + 0, hits);
    if (steps) atomicAdd(J.counters + 1, steps);
    if (capped) atomicAdd(J.counters + 2, capped);
    hits = steps = capped = 0;
}

template <bool VERIFY>
__global__ void __launch_bounds__(128, CSMC_BATCH_MIN_CTAS_PER_SM) batch_kernel(const BatchParams p) {
    extern __shared__ __align__(16) uint8_t smem[];
    {  // stage the job table
        const uint4 *src = reinterpret_cast<const uint4 *>(p.jobs);
        uint4 *dst = reinterpret_cast<uint4 *>(smem);
        const uint32_t words = p.n_jobs * static_cast<uint32_t>(sizeof(BatchJob) / 16);
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    const BatchJob *jobs = reinterpret_cast<const BatchJob *>(smem);

    const uint32_t T = blockDim.x, t = threadIdx.x;
    uint8_t *st = p.state + static_cast<size_t>(blockIdx.x) * p.state_stride;
    const RunView<false> rv = carve_run_view<false>(st, p.max_vars, p.max_rate_prog, p.max_comps, T, t);

    const uint32_t lane = threadIdx.x & 31u;
    unsigned long long acc_hits = 0, acc_steps = 0, acc_capped = 0;
    uint32_t jb = 0;  // job of this lane's current run
    bool have = false;
    unsigned long long local = 0;  // run index within the job
    uint64_t run = 0;
    float time = 0.0f;
    uint32_t step = 0;
    RunScalars sc{0.0, 0.0, 0, 0, -1, 0, 0};

    for (;;) {
        // ---- refill finished lanes from the shared run counter
        const bool need = !have;
        const unsigned act = __activemask();
        const unsigned want = __ballot_sync(act, need);
        if (want) {
            const int leader = __ffs(want) - 1;
            unsigned long long base = 0;
            if (static_cast<int>(lane) == leader) base = atomicAdd(p.queue, static_cast<unsigned long long>(__popc(want)));
            base = __shfl_sync(act, base, leader);
            if (need) {
                const unsigned long long r = base + __popc(want & ((1u << lane) - 1u));
                if (r >= p.total_runs) break;
                const uint32_t j = find_job(jobs, p.n_jobs, r);
                if (j != jb) {
                    flush_counters(jobs[jb], acc_hits, acc_steps, acc_capped);
                    jb = j;
                }
                const BatchJob &J = jobs[jb];
                have = true;
                local = r - J.run_begin;
                run = J.first_run + local;
                const Net n = net_view(J.blob, J.net);
                run_init<true>(n, J.net.n_comps, J.net.n_vars, rv, sc, J.var_id);
                time = 0.0f;
                step = 0;
            }
        }

        const BatchJob &J = jobs[jb];
        const Net n = net_view(J.blob, J.net);
        const uint32_t C = J.net.n_comps, V = J.net.n_vars;

        // ---- end of run (simulation.cu:835-849, 887-893)
        const RunEnd e = run_end(sc, time, J.horizon, step, J.max_steps, J.loc_mode, J.is_max, J.threshold);
        if (e.done) {
            if (J.flags) J.flags[local] = static_cast<uint8_t>(e.flag);
            if (J.values) J.values[local] = e.value;
            if (J.steps) J.steps[local] = step;
            if (VERIFY) {
                if (J.digests) J.digests[local] = sc.digest;
                if (J.final_state) run_final_state(n, C, V, rv, J.final_state + local * (C + V));
            }
            acc_hits += e.flag;
            acc_steps += step;
            acc_capped += e.capped;
            have = false;
            continue;
        }

        const uint32_t P = J.net.n_rate_prog;
        const bool rate_table = (J.net.flags & CSMC_NET_RATE_TABLE) && P > 0;
        run_step<VERIFY, true, false>(n, C, V, P, J.net.n_clocks, rate_table, rv, sc, J.seed, J.var_id, run, step,
                                      time);
    }
    flush_counters(jobs[jb], acc_hits, acc_steps, acc_capped);
}

}  // namespace detail

template <bool VERIFY>
int batch_launch_one(const BatchParams &p, int grid, int block, void *stream) {
    auto fn = detail::batch_kernel<VERIFY>;
    const size_t smem = batch_smem_bytes(p.n_jobs);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <bool VERIFY>
int batch_occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = detail::batch_kernel<VERIFY>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

}  // namespace csmc
