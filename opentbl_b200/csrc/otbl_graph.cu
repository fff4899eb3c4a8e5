// CUDA graphs of whole RK3 steps for one or many contexts (an ensemble of
// independent boxes), and a non-blocking completion query. No counterpart in
// the reference, which advances one box per MPI job.
//
// A substep needs no host synchronisation (dt, the genflu integrals and the
// implzy factors are produced and consumed on the device), so otbl_advance
// can be captured as it is. The capture forks from the graph's own stream to
// every member context's stream and joins back, so the members' kernels are
// independent branches of one graph and run concurrently on the GPU; one
// cudaGraphLaunch then advances every box by nsteps RK3 steps.
#include <string>
#include <vector>

#include "otbl_internal.cuh"
#include "tma.cuh"

using namespace otbl;

// Self-test of the bounded mbarrier wait that every TMA-fed kernel uses:
// the barrier is armed for 16 bytes that no copy ever delivers (nothing is
// issued, so nothing is in flight), every thread waits with a limit of
// limit_ns and, as the product kernels do on a timeout, the CTA agrees on
// the failure, records OTBL_ERR_TIMEOUT and returns.
__global__ void k_wait_selftest(int *status, unsigned long long limit_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16);
  __syncthreads();
  const bool ok = mbar_wait_bounded(&bar, 0, limit_ns);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) atomicExch(status, OTBL_ERR_TIMEOUT);
    return;
  }
  if (threadIdx.x == 0) atomicExch(status, OTBL_OK);
}

struct otbl_graph {
  int device;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  std::vector<otbl_ctx *> members;
  std::vector<long long> kernels;  // kernel launches per member per graph launch
  std::vector<cudaEvent_t> events;
  long long total_kernels = 0;
};

static void graph_free(otbl_graph *g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  for (cudaEvent_t e : g->events) cudaEventDestroy(e);
  if (g->stream) cudaStreamDestroy(g->stream);
  delete g;
}

extern "C" int otbl_graph_create(otbl_ctx *const *ctxs, int n, int nsteps, otbl_graph **out) {
  if (!ctxs || n < 1 || nsteps < 1 || !out) return OTBL_ERR_ARG;
  *out = nullptr;
  const int dev = ctxs[0] ? ctxs[0]->device : -1;
  for (int k = 0; k < n; ++k) {
    if (!ctxs[k] || ctxs[k]->device != dev) return OTBL_ERR_ARG;
    if (ctxs[k]->prof_on) return OTBL_ERR_ARG;  // per-launch events cannot be captured
    for (int q = 0; q < k; ++q)
      if (ctxs[q] == ctxs[k]) return OTBL_ERR_ARG;
  }
  if (cudaSetDevice(dev) != cudaSuccess) return OTBL_ERR_CUDA;
  otbl_graph *g = new otbl_graph();
  g->device = dev;
  g->members.assign(ctxs, ctxs + n);
  // finish outstanding work of the members before capturing
  for (otbl_ctx *c : g->members)
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
      graph_free(g);
      return OTBL_ERR_CUDA;
    }
  if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess) {
    graph_free(g);
    return OTBL_ERR_CUDA;
  }
  g->events.resize(n + 1, nullptr);
  for (auto &e : g->events)
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
      graph_free(g);
      return OTBL_ERR_CUDA;
    }
  int st = OTBL_OK;
  if (cudaStreamBeginCapture(g->stream, cudaStreamCaptureModeRelaxed) != cudaSuccess) {
    graph_free(g);
    return OTBL_ERR_CUDA;
  }
  cudaEventRecord(g->events[n], g->stream);
  g->kernels.assign(n, 0);
  for (int k = 0; k < n && st == OTBL_OK; ++k) {
    otbl_ctx *c = g->members[k];
    cudaStreamWaitEvent(c->stream, g->events[n], 0);  // fork
    const long long l0 = c->launches;
    st = otbl_advance(c, nsteps);
    g->kernels[k] = c->launches - l0;
    c->launches = l0;  // counted again at every launch of the graph
    cudaEventRecord(g->events[k], c->stream);
    cudaStreamWaitEvent(g->stream, g->events[k], 0);  // join
  }
  cudaGraph_t graph = nullptr;
  const cudaError_t ec = cudaStreamEndCapture(g->stream, &graph);
  g->graph = graph;
  if (st != OTBL_OK || ec != cudaSuccess) {
    cudaGetLastError();
    graph_free(g);
    return st != OTBL_OK ? st : OTBL_ERR_CUDA;
  }
  // keep the priorities of the streams the kernels were captured from
  if (cudaGraphInstantiate(&g->exec, g->graph, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess) {
    cudaGetLastError();
    graph_free(g);
    return OTBL_ERR_CUDA;
  }
  for (long long k : g->kernels) g->total_kernels += k;
  *out = g;
  return OTBL_OK;
}

extern "C" int otbl_graph_launch(otbl_graph *g) {
  if (!g) return OTBL_ERR_ARG;
  cudaSetDevice(g->device);
  if (cudaGraphLaunch(g->exec, g->stream) != cudaSuccess) return OTBL_ERR_CUDA;
  for (size_t k = 0; k < g->members.size(); ++k) g->members[k]->launches += g->kernels[k];
  return OTBL_OK;
}

extern "C" int otbl_graph_sync(otbl_graph *g) {
  if (!g) return OTBL_ERR_ARG;
  cudaSetDevice(g->device);
  if (cudaStreamSynchronize(g->stream) != cudaSuccess) return OTBL_ERR_CUDA;
  for (otbl_ctx *c : g->members) {
    const int s = otbl_sync(c);
    if (s != OTBL_OK) return s;
  }
  return OTBL_OK;
}

extern "C" int otbl_graph_query(otbl_graph *g) {
  if (!g) return OTBL_ERR_ARG;
  cudaSetDevice(g->device);
  const cudaError_t e = cudaStreamQuery(g->stream);
  if (e == cudaSuccess) return OTBL_OK;
  if (e == cudaErrorNotReady) return OTBL_BUSY;
  return OTBL_ERR_CUDA;
}

extern "C" int otbl_graph_stream(otbl_graph *g, void **stream) {
  if (!g || !stream) return OTBL_ERR_ARG;
  *stream = (void *)g->stream;
  return OTBL_OK;
}

extern "C" long long otbl_graph_kernels(const otbl_graph *g) { return g ? g->total_kernels : 0; }

extern "C" void otbl_graph_destroy(otbl_graph *g) {
  if (!g) return;
  cudaSetDevice(g->device);
  cudaStreamSynchronize(g->stream);
  graph_free(g);
}

extern "C" int otbl_query(otbl_ctx *c) {
  if (!c) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  const cudaError_t e = cudaStreamQuery(c->stream);
  if (e == cudaSuccess) return OTBL_OK;
  if (e == cudaErrorNotReady) return OTBL_BUSY;
  return OTBL_ERR_CUDA;
}

// Autotuner: for each line kernel whose outputs are only work arrays (they
// are pure functions of the state, so repeating them changes nothing), time
// each CTA size with CUDA events after one warm-up launch and keep the
// fastest. The choice is per context, i.e. per box size and precision.
extern "C" int otbl_autotune(otbl_ctx *c, int *choice) {
  if (!c) return OTBL_ERR_ARG;
  if (c->prof_on) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  static const int cand[] = {32, 64, 128};
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return OTBL_ERR_CUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return OTBL_ERR_CUDA;
  }
  const long long l0 = c->launches;
  int st = OTBL_OK;
  for (int k = 0; k < 3 && st == OTBL_OK; ++k) {
    float best = 1e30f;
    int bbs = c->tune_bs[k];
    for (int bs : cand) {
      c->tune_bs[k] = bs;
      auto run = [&]() {
        return k == 0 ? launch_interpx(c) : (k == 1 ? launch_difvisx(c) : launch_interpy(c));
      };
      if (run() != cudaSuccess) {
        st = OTBL_ERR_CUDA;
        break;
      }
      cudaEventRecord(e0, c->stream);
      for (int r = 0; r < 3; ++r) run();
      cudaEventRecord(e1, c->stream);
      if (cudaEventSynchronize(e1) != cudaSuccess) {
        st = OTBL_ERR_CUDA;
        break;
      }
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      if (ms < best) {
        best = ms;
        bbs = bs;
      }
    }
    c->tune_bs[k] = bbs;
  }
  c->launches = l0;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != OTBL_OK) {
    cudaGetLastError();
    c->err = "autotune launch failed";
    return st;
  }
  if (choice)
    for (int k = 0; k < 3; ++k) choice[k] = c->tune_bs[k];
  return OTBL_OK;
}

extern "C" int otbl_set_tuning(otbl_ctx *c, const int *bs) {
  if (!c || !bs) return OTBL_ERR_ARG;
  for (int k = 0; k < 3; ++k)
    if (bs[k] != 32 && bs[k] != 64 && bs[k] != 128) return OTBL_ERR_ARG;
  for (int k = 0; k < 3; ++k) c->tune_bs[k] = bs[k];
  return OTBL_OK;
}

extern "C" int otbl_selftest_wait(otbl_ctx *c, int *status) {
  if (!c || !status) return OTBL_ERR_ARG;
  cudaSetDevice(c->device);
  int *d = nullptr;
  if (cudaMalloc(&d, sizeof(int)) != cudaSuccess) return OTBL_ERR_OOM;
  const int init = -1;
  cudaMemcpyAsync(d, &init, sizeof(int), cudaMemcpyHostToDevice, c->stream);
  k_wait_selftest<<<1, 64, 0, c->stream>>>(d, 1000000ull);  // 1 ms
  int st = OTBL_OK;
  if (cudaGetLastError() != cudaSuccess) st = OTBL_ERR_CUDA;
  if (st == OTBL_OK && cudaMemcpyAsync(status, d, sizeof(int), cudaMemcpyDeviceToHost, c->stream) != cudaSuccess)
    st = OTBL_ERR_CUDA;
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) st = OTBL_ERR_CUDA;
  cudaFree(d);
  return st;
}
