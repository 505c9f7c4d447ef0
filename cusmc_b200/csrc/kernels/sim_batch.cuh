// Multi-network batch kernel: one persistent launch over many (network,
// query) jobs.  Runs of small networks are simulated by one thread each
// with the step of sim_run.cuh; runs of large networks (the jobs the host
// marks, at most CSMC_BATCH_GROUP_MAX_COMPS components) by one warp each,
// 32 lanes x K components, with the lane-group run of sim_impl.cuh, so that
// the long runs of a large network do not leave one thread working alone
// at the end of the batch.
//
// Work queue.  The runs of all jobs are numbered in one index space (job j
// owns [run_begin_j, run_begin_j + n_runs_j)); a lane whose run ends takes
// the next index from the shared device counter (warp-aggregated atomic),
// finds its job by binary search in the job table (staged in shared memory)
// and starts that run, so uneven run lengths and uneven job sizes leave no
// lane idle until the whole batch is drained.  Lanes of one warp are on the
// same job except at the few indices where one job ends and the next begins.
//
// Warp-per-run jobs have their own run space and counter.  Every warp first
// takes runs of those (the long ones) until their counter is drained, then
// joins the thread-per-run queue, so the short runs fill in behind the long
// ones.
//
// Memory.  Networks stay in global memory (read-only, L1/L2-resident while
// in use); each CTA's thread-per-run state is a global slab laid out for the
// largest thread-per-run job (interleaved by thread, so warp accesses
// coalesce); a warp-per-run run keeps its scalars, variables and rate table
// in shared memory after the job table.  Results depend only on the job and
// the run index, never on which mode ran it.
#pragma once
#include "sim_impl.cuh"
#include "sim_run.cuh"

namespace csmc {
namespace detail {

#ifndef CSMC_BATCH_MIN_CTAS_PER_SM
#define CSMC_BATCH_MIN_CTAS_PER_SM 4
#endif
#ifndef CSMC_BATCH_GROUP_MIN_CTAS_PER_SM
#define CSMC_BATCH_GROUP_MIN_CTAS_PER_SM 3
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

// Warp-per-run jobs (K components per lane): whole warps take runs from
// p.group_queue until it passes p.group_runs.  Not inlined, so that its
// registers are allocated apart from the thread-per-run phase's.
template <int K, bool VERIFY>
static __device__ __forceinline__ void batch_group_phase(const BatchParams &p, const BatchJob *jobs, uint8_t *smem) {
    const uint32_t lane = threadIdx.x & 31u;
    RunState *s = reinterpret_cast<RunState *>(smem + p.n_jobs * sizeof(BatchJob) + (threadIdx.x >> 5) * p.group_stride);
    unsigned long long acc_hits = 0, acc_steps = 0, acc_capped = 0;
    uint32_t jb = 0;
    for (;;) {
        unsigned long long r = 0;
        if (lane == 0) r = atomicAdd(p.group_queue, 1ull);
        r = __shfl_sync(0xffffffffu, r, 0);
        if (r >= p.group_runs) break;
        const uint32_t j = find_job(jobs, p.n_group_jobs, r);
        if (j != jb) {
            if (lane == 0) flush_counters(jobs[jb], acc_hits, acc_steps, acc_capped);
            jb = j;
        }
        const BatchJob &J = jobs[jb];
        const Net n = net_view(J.blob, J.net);
        const unsigned long long local = r - J.run_begin;
        group_run<32, K, VERIFY>(n, s, J, J.first_run + local, local, lane, 0u, 0xffffffffu, acc_hits, acc_steps,
                                 acc_capped);
    }
    if (lane == 0) flush_counters(jobs[jb], acc_hits, acc_steps, acc_capped);
}

template <bool VERIFY, int K>
__global__ void __launch_bounds__(128, K > 0 ? CSMC_BATCH_GROUP_MIN_CTAS_PER_SM : CSMC_BATCH_MIN_CTAS_PER_SM) batch_kernel(const __grid_constant__ BatchParams p) {
    extern __shared__ __align__(16) uint8_t smem[];
    {  // stage the job table
        const uint4 *src = reinterpret_cast<const uint4 *>(p.jobs);
        uint4 *dst = reinterpret_cast<uint4 *>(smem);
        const uint32_t words = p.n_jobs * static_cast<uint32_t>(sizeof(BatchJob) / 16);
        for (uint32_t i = threadIdx.x; i < words; i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    if constexpr (K > 0) {
        if (p.n_group_jobs > 0) batch_group_phase<K, VERIFY>(p, reinterpret_cast<const BatchJob *>(smem), smem);
    }
    if (p.n_jobs == p.n_group_jobs) return;
    const BatchJob *jobs = reinterpret_cast<const BatchJob *>(smem) + p.n_group_jobs;
    const uint32_t n_jobs = p.n_jobs - p.n_group_jobs;

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
                const uint32_t j = find_job(jobs, n_jobs, r);
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

template <bool VERIFY, int K>
int batch_launch_one(const BatchParams &p, int grid, int block, void *stream) {
    auto fn = detail::batch_kernel<VERIFY, K>;
    const size_t smem = batch_smem_bytes(p.n_jobs, p.n_group_jobs ? p.group_stride : 0u, block);
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    fn<<<grid, block, smem, static_cast<cudaStream_t>(stream)>>>(p);
    return static_cast<int>(cudaGetLastError());
}

template <bool VERIFY, int K>
int batch_occupancy_one(int block, size_t smem, int *ctas) {
    auto fn = detail::batch_kernel<VERIFY, K>;
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
    if (e != cudaSuccess) return static_cast<int>(e);
    return static_cast<int>(cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas, fn, block, smem));
}

}  // namespace csmc
