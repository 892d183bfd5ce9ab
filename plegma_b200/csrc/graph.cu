// CUDA-graph form of p2_contract_project (p2_graph_*).
//
// A graph owns a private workspace context with the same geometry as its
// parent: the launch sequence of the requests is run once eagerly (it sizes
// every workspace, builds the phase tiles, settles the autotuner's choices
// and raises the kernels' shared-memory limits) and then recorded by stream
// capture, so the recorded sequence contains no allocation and no host
// synchronisation.  Replays read the propagator buffers given at creation
// and overwrite the results given at creation.
#include <vector>

#include "ctx.h"

struct p2_graph {
  p2_ctx* parent = nullptr;
  p2_ctx* priv = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t last = nullptr;  // stream of the last launch
};

namespace {

void destroy_graph(p2_graph* g) {
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->priv) p2_ctx_destroy(g->priv);
  delete g;
}

}  // namespace

extern "C" {

p2_status p2_graph_create(p2_ctx* c, const p2_prop* props, int nprops, const p2_request* reqs, int nreq,
                          p2_graph** out) {
  if (!c || !out) return c ? c->fail(P2_ERR_INVALID_ARG, "p2_graph_create: null output") : P2_ERR_INVALID_ARG;
  *out = nullptr;
  if (c->host_only) return c->fail(P2_ERR_UNSUPPORTED, "host-only context");
  if (!props || nprops < 1 || !reqs || nreq < 1) return c->fail(P2_ERR_INVALID_ARG, "empty props or requests");
  for (int i = 0; i < nprops; i++)
    if (props[i].location != P2_DEVICE) return c->fail(P2_ERR_UNSUPPORTED, "graphs need device-resident propagators");
  for (int i = 0; i < nreq; i++)
    if (reqs[i].out_location != P2_DEVICE) return c->fail(P2_ERR_UNSUPPORTED, "graphs need device-resident results");

  p2_graph* g = new p2_graph();
  g->parent = c;
  p2_status st = p2_ctx_create(&c->g, &g->priv);
  if (st != P2_OK) {
    delete g;
    return c->fail(st, "p2_graph_create: workspace context");
  }
  p2_ctx* p = g->priv;
  p->ws_budget = c->ws_budget;
  p->tuner = c->tuner;  // the parent's tuning cache and settings
  // eager run: sizes, tables, tuning
  st = p2_contract_project(p, props, nprops, reqs, nreq);
  if (st == P2_OK) st = p2_sync(p);
  if (st != P2_OK) {
    c->fail(st, std::string("p2_graph_create: eager run: ") + p->err);
    destroy_graph(g);
    return st;
  }
  cudaError_t e = cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    p->capturing = true;
    st = p2_contract_project(p, props, nprops, reqs, nreq);
    p->capturing = false;
    cudaGraph_t graph = nullptr;
    const cudaError_t e2 = cudaStreamEndCapture(p->stream, &graph);
    g->graph = graph;
    if (st == P2_OK && e2 != cudaSuccess) e = e2;
  }
  if (st != P2_OK || e != cudaSuccess) {
    if (st == P2_OK) st = c->cuda(e, "p2_graph_create: capture");
    else c->fail(st, std::string("p2_graph_create: capture: ") + p->err);
    cudaGetLastError();
    destroy_graph(g);
    return st;
  }
  e = cudaGraphInstantiate(&g->exec, g->graph, 0);
  if (e != cudaSuccess) {
    st = c->cuda(e, "p2_graph_create: instantiate");
    destroy_graph(g);
    return st;
  }
  *out = g;
  return P2_OK;
}

p2_status p2_graph_launch(p2_graph* g, void* stream) {
  if (!g) return P2_ERR_INVALID_ARG;
  g->last = stream ? (cudaStream_t)stream : g->parent->stream;
  return g->parent->cuda(cudaGraphLaunch(g->exec, g->last), "p2_graph_launch");
}

p2_status p2_graph_sync(p2_graph* g) {
  if (!g) return P2_ERR_INVALID_ARG;
  p2_ctx* c = g->parent;
  if (g->last) P2_TRY(c, cudaStreamSynchronize(g->last), "p2_graph_sync");
  p2_ctx* p = g->priv;
  if (p->errflag.p) {
    int e = 0;
    P2_TRY(c, cudaMemcpy(&e, p->errflag.p, sizeof(int), cudaMemcpyDeviceToHost), "error flag read");
    if (e) {
      P2_TRY(c, cudaMemset(p->errflag.p, 0, sizeof(int)), "error flag reset");
      return c->fail(P2_ERR_DEVICE_TIMEOUT, "a tensor-core pipeline wait gave up; results of the launch are invalid");
    }
  }
  return P2_OK;
}

p2_status p2_graph_destroy(p2_graph* g) {
  if (!g) return P2_ERR_INVALID_ARG;
  if (g->last) cudaStreamSynchronize(g->last);
  destroy_graph(g);
  return P2_OK;
}

}  // extern "C"
