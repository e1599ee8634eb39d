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
    int64_t rb;  // shared-memory bytes of one replica
};

int launch_anneal(cudaStream_t stream, int njobs, int cs, int Rl, size_t smem, const int32_t* job_list,
                  const JobDev* jdev, JobMut* jmut, float4* pos, double* best, int slice);
int launch_polish(cudaStream_t stream, int njobs, const int32_t* job_list, const JobDev* jdev, JobMut* jmut,
                  double* best, size_t smem);
size_t polish_smem_bytes(int n);

void put(char* dst, size_t cap, const std::string& s);
// Validate one job and fill its device records (offsets left to the caller).
int prepare_job(const sqs_job& J, int j, JobDev& d, JobMut& m, Plan& p);
// float4 elements of a job's state region: R*n replica squares + 2n quench scratch.
int64_t job_pos_elems(const sqs_job& J);
// Every replica starts from the job's initial state (angles wrapped to [0, pi/2)).
void init_replicas(const sqs_job& J, float4* dst);
void fill_result(const sqs_job& J, const JobMut& m, float dev_ms, sqs_job_result& o);
int certify_states(sqs_ctx* ctx, const std::vector<int>& ns, const std::vector<const double*>& best,
                   const std::vector<sqs_job_result*>& out, const std::vector<double*>& xya_out);

}  // namespace ann
}  // namespace sqs
