// batch.cu -- many solves on several lattices at once (no reference
// counterpart: the reference solves one system per MPI job).
//
// Each job is a batch of right-hand sides on some context; a context is one
// lattice with its own links, parameters and CUDA stream.  For the even-odd
// mixed solver with graphs on, the jobs of a context are merged into one batch
// (each right-hand side with its own twisted mass) and every context's whole
// solve is one branch of a single CUDA graph: one launch for all lattices
// (invert_batch_graph, mixed.cu).  Otherwise the jobs of a context run in order
// on one host thread and different contexts run on different threads, so their
// kernels overlap on the GPU through their streams.  Either way contexts start
// in order of decreasing volume (longest first), which bounds the makespan
// when lattices are uneven.
#include <stdio.h>

#include <algorithm>
#include <chrono>
#include <thread>
#include <vector>

#include "qkx_ctx.cuh"

using namespace qkx;

extern "C" {

int qkx_invert_batch(qkx_batch_job* jobs, int njobs, const qkx_solver_params* sp) {
  if (!jobs || !sp || njobs < 1) {
    set_error("invalid argument: jobs, njobs or params");
    return QKX_ERR_INVALID;
  }
  for (int i = 0; i < njobs; i++)
    if (!jobs[i].ctx || jobs[i].nrhs < 1 || !jobs[i].b_dev || !jobs[i].x_dev) {
      set_error("invalid argument: job %d", i);
      return QKX_ERR_INVALID;
    }
  // group the jobs by context, contexts by decreasing volume
  std::vector<qkx_ctx*> ctxs;
  for (int i = 0; i < njobs; i++)
    if (std::find(ctxs.begin(), ctxs.end(), jobs[i].ctx) == ctxs.end()) ctxs.push_back(jobs[i].ctx);
  std::stable_sort(ctxs.begin(), ctxs.end(), [](qkx_ctx* a, qkx_ctx* b) { return a->V > b->V; });
  const auto t0 = std::chrono::steady_clock::now();
  const int g = invert_batch_graph(jobs, njobs, sp,
                                   std::chrono::duration<double>(t0.time_since_epoch()).count());
  if (g < 0) return g;
  if (g == 0) {
    for (int i = 0; i < njobs; i++)
      if (jobs[i].status != QKX_OK) {
        set_error("job %d failed with status %d: %s", i, jobs[i].status, jobs[i].message);
        return jobs[i].status;
      }
    return QKX_OK;
  }
  std::vector<std::thread> threads;
  for (qkx_ctx* c : ctxs) {
    threads.emplace_back([=]() {
      for (int i = 0; i < njobs; i++) {
        if (jobs[i].ctx != c) continue;
        qkx_solver_params p = *sp;
        p.mu = jobs[i].mu;
        jobs[i].status = qkx_invert_dev(c, &p, jobs[i].nrhs, jobs[i].b_dev, jobs[i].x_dev, &jobs[i].info);
        jobs[i].message[0] = 0;
        if (jobs[i].status != QKX_OK) {  // the message is per thread: keep it in the job
          snprintf(jobs[i].message, sizeof jobs[i].message, "%s", qkx_last_error());
        }
        cudaStreamSynchronize(c->st);
        jobs[i].latency = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      }
    });
  }
  for (std::thread& t : threads) t.join();
  for (int i = 0; i < njobs; i++)
    if (jobs[i].status != QKX_OK) {
      set_error("job %d failed with status %d: %s", i, jobs[i].status, jobs[i].message);
      return jobs[i].status;
    }
  return QKX_OK;
}

}  // extern "C"
