// Host-side helpers shared by the batch entry point (anneal_host.cu) and the
// serving runtime (serve_host.cu).
#pragma once
#include <string>
#include <vector>

#include "anneal.cuh"
#include "common.cuh"

namespace sqs {
namespace ann {

struct Plan {
    int cs, Rl, Gmax;
    int64_t rb;   // shared-memory bytes of one replica
    float cell;   // minimum cell side
};

// A launch shape chosen by the autotuner (cs = 0: none, use the default plan).
struct Shape {
    int cs = 0;
    float cell = kCellSide;
};

int prime_anneal();
int launch_trace(cudaStream_t stream, int items, const int2* list, const JobDev* jdev, const JobMut* jmut,
                 const float4* pos, TraceRec* out, size_t smem);
size_t energy_smem_bytes(int n);
int launch_energy_states(cudaStream_t stream, int count, const int32_t* n_of, const int64_t* row0, const double* side,
                         const double* xya, double* energy_out, double* grad, size_t smem);

// One launch of the anneal kernel: the jobs job_list[0 .. njobs) sharing a
// cluster shape, with the shared memory of the largest.
struct Group {
    int njobs, cs, Rl;
    size_t smem;
    const int32_t* list;
    bool moves;  // the jobs use move-set options (the kernel instance with them)
};
// Launch every group for one slice.  Several groups run concurrently on the
// context's side streams, forked from and joined back to its main stream
// (under stream capture they become parallel branches of the graph).
int launch_groups(sqs_ctx* ctx, const std::vector<Group>& groups, const JobDev* jdev, JobMut* jmut, float4* pos,
                  double* best, int slice);
int anneal_max_clusters(int cs, int Rl, size_t smem, bool moves, int* out);
// Shared memory to launch with: the replicas, and the quench scratch when it fits
// without lowering the resident clusters.
size_t anneal_smem(int cs, int Rl, int64_t rb, int n_max, bool moves, int need = 1 << 30);
int launch_anneal(cudaStream_t stream, int njobs, int cs, int Rl, size_t smem, bool moves, const int32_t* job_list,
                  const JobDev* jdev, JobMut* jmut, float4* pos, double* best, int slice);
int launch_polish(cudaStream_t stream, int njobs, const int32_t* job_list, const JobDev* jdev, JobMut* jmut,
                  double* best, size_t smem);
size_t polish_smem_bytes(int n);
int launch_polish_states(cudaStream_t stream, int count, const int32_t* n_of, const int64_t* row0, int iters,
                         double* xya, double* res, size_t smem);

void put(char* dst, size_t cap, const std::string& s);
// Validate one job and fill its device records (offsets left to the caller).
// `shape` (optional) fixes the cluster size and cell side instead of the
// default (smallest cluster that fits, cells of side kCellSide).
int prepare_job(const sqs_job& J, int j, JobDev& d, JobMut& m, Plan& p, const Shape* shape = nullptr);
// Resolve SQS_JOB_AUTOTUNE: the tuned shape of the job's class (tuning it on
// first sight) and, when the job leaves exchange_every at 0, the tuned
// interval written into `eff` (a copy of the job).  No flag: eff = job.
int resolve_job(sqs_ctx* ctx, const sqs_job& job, int mode, sqs_job& eff, Shape& shape);
// float4 elements of a job's state region: R*n replica squares + 2n quench scratch.
int64_t job_pos_elems(const sqs_job& J);
// Proposals per replica in a job's budget (sweeps * n, or -sweeps), and that
// budget in whole sweeps, rounded up.
int64_t job_props(const sqs_job& J);
int64_t job_sweeps(const sqs_job& J);
// Every replica starts from the job's initial state (angles wrapped to [0, pi/2)).
void init_replicas(const sqs_job& J, float4* dst);
void fill_result(const sqs_job& J, const JobDev& d, const JobMut& m, float dev_ms, sqs_job_result& o);
// A finished job that certified no state during its anneal would return
// nothing: its coldest replica's final state is polished from scratch
// instead (the sqs_polish_batch path: overlaps resolved in a spread box,
// then the compress-and-descend attempts, `iters` gradient steps), and a
// certified side found that way becomes the job's best (*m, best[3n]).
struct Rescue {
    int n, iters;
    const float4* d_state;  // the replica's final (x, y, angle, -) on the device
    double* best;           // host, n x 3
    JobMut* m;              // host copy of the job's record
};
int rescue_uncertified(sqs_ctx* ctx, const std::vector<Rescue>& items);
// The rescue candidates among finished jobs: annealed (sweeps > 0), best
// side still unset, polish requested.
void add_rescue(std::vector<Rescue>& out, const sqs_job& J, const JobDev& d, JobMut& m, const float4* d_pos,
                double* best);
int certify_states(sqs_ctx* ctx, const std::vector<int>& ns, const std::vector<const double*>& best,
                   const std::vector<sqs_job_result*>& out, const std::vector<double*>& xya_out);

}  // namespace ann
}  // namespace sqs
