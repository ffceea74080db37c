// pool.cuh -- the batch kernels: many matrices in one launch, several thread
// groups per CTA, the biggest matrices on thread-block-cluster teams.
//
// A "pool" shape is <B, EMAX, GB, GE, MINB>: CTAs of B threads (a cluster
// team of whole CTAs chunks EMAX edges per CTA) split into B / GB thread
// groups of GB threads that reorder one matrix each (GE edges per chunk),
// compiled for MINB CTAs per SM.  Each shape is
// instantiated in its own translation unit (pool_p<N>.cu) through
// PBRCM_DEFINE_POOL, which exports its entry points as a PoolFns table.
#pragma once

#include <algorithm>

#include "engine.cuh"
#include "kernels.h"
#include "solo.cuh"

namespace pbrcm {

// Whether CTAs of B threads can give each of their groups of GB threads the
// solo engine's shared memory (its visited bitmap is 32 KB per group).
template <int B, int GB, int GE>
__host__ __device__ constexpr bool solo_fits()
{
    return (size_t)(B / GB) * ((sizeof(SoloSmem<GB, GE>) + 127) & ~(size_t)127) <= (size_t)226 * 1024;
}

// Bytes of one group's shared memory: the engine's chunk buffers or, where
// it fits, the solo engine's (the two are never live at once).
template <int B, int GB, int GE>
__host__ __device__ constexpr size_t group_stride()
{
    constexpr size_t a = sizeof(Smem<GB, GE>);
    constexpr size_t b = solo_fits<B, GB, GE>() ? sizeof(SoloSmem<GB, GE>) : 0;
    return ((a > b ? a : b) + 127) & ~(size_t)127;
}

// Shared memory of thread group g when a CTA of B threads runs groups of GB
// threads.
template <int B, int GB, int GE>
__device__ __forceinline__ unsigned char* group_smem(unsigned char* raw)
{
    return raw + (threadIdx.x / GB) * group_stride<B, GB, GE>();
}

// Before a group reorders a matrix of the batch: waits (bounded) for its CSR
// to arrive when the batch is still being copied in, then checks the CSR and
// builds the solo engine's edge records where the job has room for them.
// Every group of a team does the same and reaches the same verdict.  Returns
// false if the matrix must not be reordered.
template <int B, int E>
__device__ bool prepare_job(Smem<B, E>& s, const BatchJob& job, const Options& opt)
{
    if (job.ready != nullptr) {
        wait_ready<B>(job.ready, opt.data_wait_ns, job.M.res, s.gsh);
        const bool arrived = s.gsh[0] != 0;
        gsync<B>();  // everyone has read gsh[0] before it is written again
        if (!arrived)
            return false;
    }
    validate_group<B>(job.M, s.tmp32);
    if (job.e2 != nullptr) {
        solo_build_edges<B>(job.M, job.e2);
        gsync<B>();
    }
    return true;
}

// One thread group's share of a batch: it takes the next slot of the work
// list until none is left; a slot names a job and the group's rank in the
// job's team (teams: consecutive slots, biggest jobs first).  Every group
// runs the whole reorder of its slot's matrix.
template <int B, int GB, int GE>
__device__ void group_take_slots(unsigned char* raw, const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots,
                                 uint32_t* counter, const Options& opt)
{
    auto& s = *reinterpret_cast<Smem<GB, GE>*>(raw);
    while (true) {
        if (gtid<GB>() == 0)
            s.bcast[7] = atomicAdd(counter, 1u);
        gsync<GB>();
        const uint32_t slot = s.bcast[7];
        gsync<GB>();
        if (slot >= nslots)
            break;
        const BatchSlot sl = slots[slot];
        const BatchJob job = jobs[sl.job];
        if (!prepare_job<GB>(s, job, opt))
            continue;
        if constexpr (solo_fits<B, GB, GE>()) {
            // one group alone on a matrix whose rows fit a chunk: the solo
            // engine (visited bitmap in shared memory, or in global memory
            // for a matrix over kSoloMaxN nodes)
            if (job.e2 != nullptr && job.team == 1 && job.M.n <= kSoloMaxNodes &&
                (job.M.n <= kSoloMaxN || job.gvis != nullptr) &&
                read_status(job.M.res) == 0 && __ldcg(&job.M.res->maxdeg) <= (uint32_t)GE) {
                solo_reorder<GB, GE>(*reinterpret_cast<SoloSmem<GB, GE>*>(raw), job.M, job.e2, job.inv,
                                     job.M.n > kSoloMaxN ? job.gvis : nullptr, opt);
                gsync<GB>();
                continue;
            }
        }
        if (skip_matrix<GE>(job.M, sl.rank == 0 && gtid<GB>() == 0))
            continue;
        Team team;
        team.gs = job.team > 1 ? job.gs : nullptr;
        team.flags = job.team > 1 ? reinterpret_cast<unsigned int*>(job.words + 2 * job.team) : nullptr;
        team.size = job.team;
        team.rank = sl.rank;
        team.expected = job.team;
        team.mode = 0;
        team.target = 0;
        team.epoch = 0;
        team.wait_ns = opt.wait_ns;
        team.res = job.M.res;
        bind_group<GB>(team, s);
        reorder_matrix<GB, GE>(s, job.M, team, job.words, opt);
        gsync<GB>();
    }
}

// Bytes of one group's shared memory in the solo batch kernel.
template <int GB, int GE>
__host__ __device__ constexpr size_t solo_stride()
{
    return (sizeof(SoloSmem<GB, GE>) + 127) & ~(size_t)127;
}

// One thread group's share of a batch in which every job is a one-group job
// with edge records (no teams, no clusters): the solo engine alone, so the
// kernel carries none of the team engine's registers.  A matrix with a row
// longer than a chunk is left to the host's rerun on the team path
// (kNeedHub), as the general kernel does.
template <int GB, int GE>
__device__ void group_take_solo(unsigned char* raw, const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots,
                                uint32_t* counter, const Options& opt)
{
    auto& s = *reinterpret_cast<SoloSmem<GB, GE>*>(raw);
    const uint32_t t = gtid<GB>();
    while (true) {
        if (t == 0)
            s.bcast[0] = atomicAdd(counter, 1u);
        gsync<GB>();
        const uint32_t slot = s.bcast[0];
        gsync<GB>();
        if (slot >= nslots)
            break;
        const BatchJob job = jobs[slots[slot].job];
        if (job.ready != nullptr) {
            wait_ready<GB>(job.ready, opt.data_wait_ns, job.M.res, reinterpret_cast<int*>(&s.bcast[1]));
            const bool arrived = s.bcast[1] != 0;
            gsync<GB>();  // everyone has read bcast[1] before it is written again
            if (!arrived)
                continue;
        }
        validate_rows<GB>(job.M, s.tmp32);
        if (read_status(job.M.res) != 0)
            continue;
        // rows longer than a chunk, or no room for edge records (the host
        // gives a matrix of more than kSoloMaxNodes nodes none): the host
        // reruns the matrix on the team path
        if (__ldcg(&job.M.res->maxdeg) > (uint32_t)GE || (job.e2 == nullptr && job.M.nnz > 0) ||
            (job.M.n > kSoloMaxN && job.gvis == nullptr)) {
            if (t == 0)
                set_status(job.M.res, kNeedHub, 0);
            continue;
        }
        solo_build_edges<GB>(job.M, job.e2);  // tests the columns too
        gsync<GB>();
        if (read_status(job.M.res) != 0)
            continue;
        solo_reorder<GB, GE>(s, job.M, job.e2, job.inv, job.M.n > kSoloMaxN ? job.gvis : nullptr, opt);
        gsync<GB>();
    }
}

// The solo batch kernel: CTAs of B threads split into B / GB groups, each
// reordering one matrix at a time with the solo engine (compiled for MINB
// CTAs per SM).
template <int B, int GB, int GE, int MINB>
__global__ void __launch_bounds__(B, MINB) k_solo_batch(const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots,
                                                        uint32_t* counter, Options opt)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    group_take_solo<GB, GE>(smem_raw + (threadIdx.x / GB) * solo_stride<GB, GE>(), jobs, slots, nslots, counter,
                            opt);
}

// Many matrices in one launch.  A CTA of B threads runs B / GB independent
// thread groups, each taking slots of the work list (group_take_slots), so
// that several matrices are in flight per SM.  The launch is cooperative
// when some job has a team of several groups (every member resident).
template <int B, int GB, int GE, int MINB>
__global__ void __launch_bounds__(B, MINB) k_reorder_batch(const BatchJob* jobs, const BatchSlot* slots,
                                                           uint32_t nslots, uint32_t* counter, Options opt)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    group_take_slots<B, GB, GE>(group_smem<B, GB, GE>(smem_raw), jobs, slots, nslots, counter, opt);
}

// A batch launched in thread-block clusters.  First the big matrices,
// jobs[0..nbig), one per cluster at a time: the cluster's CTA 0 takes the next
// index from counters[0], the others read it from CTA 0's shared memory, and
// the cluster reorders the matrix as one ClusterTeam of whole CTAs (copt,
// B threads and EMAX edges per CTA).  Every CTA passes every cluster barrier:
// the job index and the skip test are the same in all of them, and
// reorder_matrix stops only through cluster-wide decisions.  When no big
// matrix is left, each CTA splits into B / GB thread groups that take the
// remaining one-group slots from counters[1] on their own, as
// k_reorder_batch does (no cluster barrier and no shared-memory access
// across CTAs from then on).
template <int B, int EMAX, int GB, int GE, int MINB>
__global__ void __launch_bounds__(B, MINB) k_reorder_cluster(const BatchJob* jobs, uint32_t nbig, const BatchSlot* slots,
                                                          uint32_t nslots, uint32_t* counters, Options copt,
                                                          Options opt)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ ClusterShared cs;
    __shared__ uint32_t s_job;
    cooperative_groups::cluster_group cl = cooperative_groups::this_cluster();
    const uint32_t csize = cl.num_blocks(), crank = cl.block_rank();
    if (nbig > 0) {
        auto& s = *reinterpret_cast<Smem<B, EMAX>*>(smem_raw);
        while (true) {
            if (crank == 0 && threadIdx.x == 0)
                cs.job = atomicAdd(counters, 1u);
            cluster_arrive();
            cluster_wait();
            if (threadIdx.x == 0)
                s_job = cl.map_shared_rank(&cs, 0)->job;
            __syncthreads();
            const uint32_t j = s_job;
            // nobody goes on while a peer still reads its shared memory
            cluster_arrive();
            cluster_wait();
            if (j >= nbig)
                break;
            const BatchJob job = jobs[j];
            // every CTA checks the CSR; the cluster goes on only if all of
            // them do (a wait for the data that ran out on one CTA must not
            // leave the others alone at a cluster barrier)
            const bool mine = prepare_job<B>(s, job, copt) && !skip_matrix<EMAX>(job.M, crank == 0 && threadIdx.x == 0);
            if (threadIdx.x == 0)
                cs.job_ok = mine ? 1u : 0u;
            cluster_arrive();
            cluster_wait();
            if (threadIdx.x == 0) {
                uint32_t all = 1;
                for (uint32_t r = 0; r < csize; ++r)
                    all &= cl.map_shared_rank(&cs, r)->job_ok;
                s_job = all;
            }
            __syncthreads();
            const bool go = s_job != 0;
            cluster_arrive();  // every peer has read job_ok before it is written again
            cluster_wait();
            if (go) {
                ClusterTeam team{&cs, csize, crank, 0u, job.M.res};
                bind_group<B>(team, s);
                reorder_matrix<B, EMAX>(s, job.M, team, nullptr, copt);
            }
            cluster_arrive();
            cluster_wait();
        }
    }
    // the CTA's shared memory now belongs to its groups
    group_take_slots<B, GB, GE>(group_smem<B, GB, GE>(smem_raw), jobs, slots, nslots, counters + 1, opt);
}

namespace {

// The batch kernels of one pool shape: CTAs of B threads (cluster teams of
// whole CTAs, EMAX edges per chunk), split into groups of GB threads (GE
// edges per chunk) for the one-group slots; MINB CTAs per SM (the register
// bound the kernels are compiled for); the solo batch kernel of the same
// groups for SMINB CTAs per SM (0: none for this shape).
template <int B, int EMAX, int GB, int GE, int MINB, int SMINB>
struct Pool {
    static_assert(B % GB == 0 && B / GB <= 15, "at most 15 groups (named barriers 1..15) per CTA");
    static size_t batch_smem() { return (size_t)(B / GB) * group_stride<B, GB, GE>(); }
    static size_t cluster_smem() { return std::max(sizeof(Smem<B, EMAX>), batch_smem()); }
    static cudaError_t prepare()
    {
        static cudaError_t once = [] {
            cudaError_t e = cudaFuncSetAttribute(k_reorder_batch<B, GB, GE, MINB>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)batch_smem());
            if (e != cudaSuccess)
                return e;
            e = cudaFuncSetAttribute(k_reorder_cluster<B, EMAX, GB, GE, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)cluster_smem());
            if (e != cudaSuccess)
                return e;
            return cudaFuncSetAttribute(k_reorder_cluster<B, EMAX, GB, GE, MINB>,
                                        cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        }();
        return once;
    }
    static cudaLaunchConfig_t cluster_config(int csize, int nclusters, cudaStream_t st, cudaLaunchAttribute* at)
    {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(csize * nclusters));
        cfg.blockDim = dim3(B);
        cfg.dynamicSmemBytes = cluster_smem();
        cfg.stream = st;
        at[0].id = cudaLaunchAttributeClusterDimension;
        at[0].val.clusterDim.x = (unsigned)csize;
        at[0].val.clusterDim.y = 1;
        at[0].val.clusterDim.z = 1;
        cfg.attrs = at;
        cfg.numAttrs = 1;
        return cfg;
    }
    static int cluster_max_active(int csize)
    {
        if (prepare() != cudaSuccess)
            return 0;
        cudaLaunchAttribute at[1];
        cudaLaunchConfig_t cfg = cluster_config(csize, 1, nullptr, at);
        int n = 0;
        if (cudaOccupancyMaxActiveClusters(&n, (void*)k_reorder_cluster<B, EMAX, GB, GE, MINB>, &cfg) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        return n;
    }
    static cudaError_t cluster(const BatchJob* jobs, uint32_t nbig, const BatchSlot* slots, uint32_t nslots,
                               uint32_t* counters, const Options& copt, const Options& opt, int csize, int nclusters,
                               cudaStream_t st)
    {
        cudaError_t e = prepare();
        if (e != cudaSuccess)
            return e;
        cudaLaunchAttribute at[1];
        cudaLaunchConfig_t cfg = cluster_config(csize, nclusters, st, at);
        return cudaLaunchKernelEx(&cfg, k_reorder_cluster<B, EMAX, GB, GE, MINB>, jobs, nbig, slots, nslots, counters, copt,
                                  opt);
    }
    static constexpr bool kSolo = SMINB > 0 && (size_t)(B / GB) * solo_stride<GB, GE>() <= (size_t)226 * 1024;
    static size_t solo_smem() { return (size_t)(B / GB) * solo_stride<GB, GE>(); }
    static const void* solo_fn()
    {
        if constexpr (kSolo)
            return (const void*)k_solo_batch<B, GB, GE, (SMINB > 0 ? SMINB : 1)>;
        return nullptr;
    }
    static cudaError_t solo_prepare()
    {
        static cudaError_t once = [] {
            if (!kSolo)
                return cudaErrorInvalidValue;
            return cudaFuncSetAttribute(solo_fn(), cudaFuncAttributeMaxDynamicSharedMemorySize, (int)solo_smem());
        }();
        return once;
    }
    static int solo_max_ctas(int sms)
    {
        if (solo_prepare() != cudaSuccess)
            return 0;
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, solo_fn(), B, solo_smem()) != cudaSuccess) {
            cudaGetLastError();
            return 0;
        }
        return nb * sms;
    }
    static cudaError_t solo(const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots, uint32_t* counter,
                            const Options& opt, int ctas, cudaStream_t st)
    {
        if constexpr (kSolo) {
            cudaError_t e = solo_prepare();
            if (e != cudaSuccess)
                return e;
            k_solo_batch<B, GB, GE, (SMINB > 0 ? SMINB : 1)><<<ctas, B, solo_smem(), st>>>(jobs, slots, nslots,
                                                                                           counter, opt);
            return cudaGetLastError();
        }
        return cudaErrorInvalidValue;
    }
    static int batch_max_ctas(int sms)
    {
        if (prepare() != cudaSuccess)
            return 0;
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_reorder_batch<B, GB, GE, MINB>, B, batch_smem()) !=
            cudaSuccess)
            return 0;
        return nb * sms;
    }
    static cudaError_t batch(const BatchJob* jobs, const BatchSlot* slots, uint32_t nslots, uint32_t* counter,
                             const Options& opt, int ctas, bool cooperative, cudaStream_t st)
    {
        cudaError_t e = prepare();
        if (e != cudaSuccess)
            return e;
        if (!cooperative) {
            // no team: groups never wait for each other, a plain launch will do
            k_reorder_batch<B, GB, GE, MINB><<<ctas, B, batch_smem(), st>>>(jobs, slots, nslots, counter, opt);
            return cudaGetLastError();
        }
        const BatchJob* j = jobs;
        const BatchSlot* sl = slots;
        uint32_t ns = nslots;
        uint32_t* c = counter;
        Options o = opt;
        void* args[] = {&j, &sl, &ns, &c, &o};
        return cudaLaunchCooperativeKernel((const void*)k_reorder_batch<B, GB, GE, MINB>, dim3(ctas), dim3(B), args,
                                           batch_smem(), st);
    }
};

}  // namespace

}  // namespace pbrcm

#define PBRCM_DEFINE_POOL(IDX, B, EMAX, GB, GE, MINB, SMINB)                                                \
    namespace pbrcm {                                                                                       \
    extern const PoolFns kPoolFns##IDX = {                                                                  \
        &Pool<B, EMAX, GB, GE, MINB, SMINB>::batch_max_ctas, &Pool<B, EMAX, GB, GE, MINB, SMINB>::cluster_max_active, \
        &Pool<B, EMAX, GB, GE, MINB, SMINB>::batch, &Pool<B, EMAX, GB, GE, MINB, SMINB>::cluster,                    \
        &Pool<B, EMAX, GB, GE, MINB, SMINB>::solo_max_ctas, &Pool<B, EMAX, GB, GE, MINB, SMINB>::solo};             \
    }
