// Batch engine: many slices of uneven size in one captured CUDA graph (no
// counterpart in the reference, which runs one slice per process).
//
// Per run of an MBFPA batch the graph holds one launch per stage, each over
// the blocks of every job:
//   - the packing of every job's maps into its padded layout;
//   - ONE persistent forward launch over the ray tiles of all jobs
//     (forward_batch_kernel), which writes every job's un-normalised sinogram
//     and statistics;
//   - the max-normalisation and noise of vct_mbfpa;
//   - the FBP's weight, filter and backprojection (quarter-turn and general
//     backprojector jobs in one launch each), for the jobs that ask for an
//     image.
// A batch of jobs that ask for a gradient runs the adjoint (loss and dl/drho)
// the same way: map packing, a reset of the exact-walk accumulators, ONE
// persistent adjoint forward over the 128-ray tiles of all jobs, the loss
// sums, the exact-walk scatter, the pixel-driven gather over the tiles of
// all jobs and the fold, one launch each.
// The ray-tile size of the persistent launch and the view split of the
// backprojector are chosen by timing candidates on (a sample of) the batch
// itself when it is created.
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "vct_ctx.h"

using namespace vct;

struct vct_batch {
  int device = 0;
  int n = 0, M = 0, ne_max = 0;
  int adjoint = 0;  // 1: jobs compute loss and gradient instead of MBFPA (+FBP)
  std::vector<vct_job> jobs;
  std::vector<vct_ctx*> ctx;
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;                           // the adjoint's exact-walk scatter
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // persistent forward
  DBuf<FwdJob> d_jobs;
  DBuf<unsigned int> d_counter;
  DBuf<unsigned int> d_xfirst;  // prefix sums of the jobs' exact-walk ray counts
  unsigned int nexact_total = 0;
  // the batched stages around it: map packing, normalisation + noise, FBP
  DBuf<PackJob> d_pack;
  DBuf<PostJob> d_post;
  DBuf<unsigned int> d_first;  // [pack n+1][post kPostStages][n+1]
  // the adjoint's batched stages
  DBuf<AdjJob> d_adj;
  DBuf<unsigned int> d_adj_first;  // [kAdjStages][n+1]
  unsigned int adj_blocks[kAdjStages] = {}, adj_ray_tiles = 0;
  unsigned int pack_blocks = 0, post_blocks[kPostStages] = {};
  int cmax = 0, winmax = 0;
  unsigned int ntiles = 0;
  int tile_rays = 64, blocks_per_sm = 0, grid = 0, view_groups = 4;
  double tuned_ms = 0.0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

int sm_count(int device) {
  int n = 0;
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, device);
  return n > 0 ? n : 1;
}

// The job table for a tile size: tile0 of every job, total tiles.
int upload_jobs(vct_batch* b, int tile_rays) {
  std::vector<FwdJob> h(b->n);
  std::vector<unsigned int> xfirst((size_t)b->n + 1, 0u);
  unsigned long long tiles = 0;
  for (int i = 0; i < b->n; i++) {
    const vct_ctx* c = b->ctx[i];
    FwdJob& J = h[i];
    J.g = c->dg;
    J.maps = c->maps.p;
    J.mu = c->mu_log2.p;
    J.pdf = c->pdf.p;
    J.cos_t = c->cos_t.p;
    J.sin_t = c->sin_t.p;
    J.px0 = c->det_px0.p;
    J.py0 = c->det_py0.p;
    J.out = b->jobs[i].d_sino;
    J.stats = c->stats.p;
    J.NE = c->NE;
    J.fast = !c->dg.rmax_active;
    J.exact = J.fast && c->fwd_nexact > 0 ? c->fwd_exact.p + 1 : nullptr;
    J.nexact = J.exact ? c->fwd_nexact : 0;
    xfirst[i + 1] = xfirst[i] + (unsigned int)J.nexact;
    J.tile0 = (unsigned int)tiles;
    const long long nrays = (long long)c->dg.views_used * c->dg.C;
    tiles += (unsigned long long)((nrays + tile_rays - 1) / tile_rays);
  }
  if (tiles >= 0xffffffffull) return fail(VCT_E_ARG, "batch: too many ray tiles");
  b->ntiles = (unsigned int)tiles;
  VCT_CUDA(cudaMemcpy(b->d_jobs.p, h.data(), h.size() * sizeof(FwdJob), cudaMemcpyHostToDevice));
  int rc;
  if ((rc = b->d_xfirst.ensure(xfirst.size()))) return rc;
  VCT_CUDA(cudaMemcpy(b->d_xfirst.p, xfirst.data(), xfirst.size() * sizeof(unsigned int), cudaMemcpyHostToDevice));
  b->nexact_total = xfirst[b->n];
  return VCT_OK;
}

int enqueue_forward(vct_batch* b, cudaStream_t st) {
  return launch_forward_batch(b->d_jobs.p, b->n, b->M, b->tile_rays, b->ntiles, b->ne_max, b->grid,
                              b->d_counter.p, b->d_xfirst.p, b->nexact_total, st);
}

// The job tables of the batched stages (after every context exists and its
// filter is built): per job its arguments and, per stage, its first block.
int upload_stage_tables(vct_batch* b) {
  const int n = b->n;
  std::vector<PackJob> pk(n);
  std::vector<PostJob> post(n);
  std::vector<unsigned int> first((size_t)(1 + kPostStages) * (n + 1), 0u);
  unsigned int* fp = first.data();
  unsigned int* fs = first.data() + (n + 1);
  unsigned int acc_pack = 0, acc[kPostStages] = {};
  b->cmax = b->winmax = 0;
  for (int i = 0; i < n; i++) {
    vct_ctx* c = b->ctx[i];
    const vct_job& j = b->jobs[i];
    pk[i] = PackJob{j.d_maps, c->maps.p, c->dg.N};
    fp[i] = acc_pack;
    acc_pack += pack_maps_blocks(c->dg.N);
    PostJob& p = post[i];
    p = PostJob{};
    const vct_geometry& g = c->geo;
    fbp_bp_params(g.views, g.width, g.start_channel, c->dg.C, c->dg.N, g.pixel_cm, g.sid_cm, g.max_beta, g.xfactor,
                  &p);
    p.sino = j.d_sino;
    p.stats = c->stats.p;
    p.pad_zero = ctx_pad_zero(c);
    p.sigma = j.sigma;
    p.key0 = (unsigned int)j.seed;
    p.key1 = (unsigned int)(j.seed >> 32);
    if (j.d_img) {
      p.img = j.d_img;
      p.coeff = c->fbp_coeff.p;
      p.h0 = c->fbp_h[j.filter].p;
      p.cs = reinterpret_cast<const float2*>(c->cs_f.p);
      p.q = c->fbp_q.p;
      p.q2 = p.sym ? c->fbp_q2.p : nullptr;
      b->cmax = std::max(b->cmax, p.C);
      if (!p.sym) b->winmax = std::max(b->winmax, p.win);
    }
    unsigned int blk[kPostStages];
    post_job_blocks(p, blk);
    for (int k = 0; k < kPostStages; k++) {
      fs[k * (n + 1) + i] = acc[k];
      acc[k] += blk[k];
    }
  }
  fp[n] = acc_pack;
  for (int k = 0; k < kPostStages; k++) fs[k * (n + 1) + n] = acc[k];
  b->pack_blocks = acc_pack;
  for (int k = 0; k < kPostStages; k++) b->post_blocks[k] = acc[k];
  int rc;
  if ((rc = b->d_pack.ensure(n)) || (rc = b->d_post.ensure(n)) || (rc = b->d_first.ensure(first.size()))) return rc;
  VCT_CUDA(cudaMemcpy(b->d_pack.p, pk.data(), n * sizeof(PackJob), cudaMemcpyHostToDevice));
  VCT_CUDA(cudaMemcpy(b->d_post.p, post.data(), n * sizeof(PostJob), cudaMemcpyHostToDevice));
  VCT_CUDA(cudaMemcpy(b->d_first.p, first.data(), first.size() * sizeof(unsigned int), cudaMemcpyHostToDevice));
  return VCT_OK;
}

// The adjoint job table: every job's loss-and-gradient arguments (each job
// gathers in its own tile shape), 128-ray tiles for the persistent forward,
// and per stage each job's first block.
int upload_adjoint_tables(vct_batch* b) {
  const int n = b->n;
  int rc;
  std::vector<AdjJob> h(n);
  std::vector<unsigned int> first((size_t)kAdjStages * (n + 1), 0u);
  unsigned int acc[kAdjStages] = {}, tiles = 0;
  for (int i = 0; i < n; i++) {
    vct_ctx* c = b->ctx[i];
    const vct_job& j = b->jobs[i];
    AdjJob& J = h[i];
    J = AdjJob{};
    J.g = c->dg;
    J.a = c->ag;
    J.maps = c->maps.p;
    J.mu = c->mu_log2.p;
    J.pdf = c->pdf.p;
    J.NE = c->NE;
    J.ynorm = c->ynorm;
    J.cos_t = c->cos_t.p;
    J.sin_t = c->sin_t.p;
    J.px0 = c->det_px0.p;
    J.py0 = c->det_py0.p;
    J.dir = c->adj_dir.p;
    J.rec = c->adj_rec.p;
    J.tv = c->adj_tv.p;
    J.meas = j.d_meas;
    J.wts = j.d_weights;
    J.gr = c->adj_g.p;
    J.part = c->adj_part.p;
    J.loss = j.d_loss ? j.d_loss : c->adj_loss.p;
    J.gmax = c->adj_gmax.p;
    J.special = c->adj_special.p;
    J.nspecial = c->adj_nspecial;
    J.lsp = c->adj_lsp.p;
    J.sacc = c->adj_nspecial > 0 ? c->adj_sacc.p : nullptr;
    J.lmax = c->ag.lmax;
    J.log2_terms = c->ag.log2_terms;
    J.ext = c->adj_ext.p;
    J.grad = j.d_grad;
    J.tile0 = tiles;
    tiles += adj_job_ray_tiles(c->dg);
    unsigned int blk[kAdjStages];
    adj_job_blocks(J, b->M, c->adj_tile, blk);
    for (int k = 0; k < kAdjStages; k++) {
      first[(size_t)k * (n + 1) + i] = acc[k];
      acc[k] += blk[k];
    }
  }
  for (int k = 0; k < kAdjStages; k++) {
    first[(size_t)k * (n + 1) + n] = acc[k];
    b->adj_blocks[k] = acc[k];
  }
  b->adj_ray_tiles = tiles;
  if ((rc = b->d_adj.ensure(n)) || (rc = b->d_adj_first.ensure(first.size()))) return rc;
  VCT_CUDA(cudaMemcpy(b->d_adj.p, h.data(), n * sizeof(AdjJob), cudaMemcpyHostToDevice));
  VCT_CUDA(cudaMemcpy(b->d_adj_first.p, first.data(), first.size() * sizeof(unsigned int), cudaMemcpyHostToDevice));
  return VCT_OK;
}

int enqueue_all(vct_batch* b) {
  int rc;
  const int n = b->n;
  if ((rc = launch_pack_maps_batch(b->d_pack.p, b->d_first.p, n, b->M, b->pack_blocks, b->stream))) return rc;
  if (b->adjoint)
    return launch_adj_batch(b->d_adj.p, b->d_adj_first.p, n, b->M, b->ne_max, b->adj_ray_tiles, b->adj_blocks,
                            b->d_counter.p, b->stream, b->side, b->ev_fork, b->ev_join);
  if ((rc = enqueue_forward(b, b->stream))) return rc;
  const unsigned int* fs = b->d_first.p + (n + 1);
  if ((rc = launch_normalize_noise_batch(b->d_post.p, fs + kPostNorm * (n + 1), n, b->post_blocks[kPostNorm],
                                         b->stream)))
    return rc;
  return launch_fbp_batch(b->d_post.p, fs, n, b->post_blocks, b->cmax, b->winmax, b->view_groups, b->stream);
}

// Milliseconds of fn() on the batch stream: best of `reps` after one warm-up.
template <class F>
int time_ms(vct_batch* b, int reps, F fn, double* best) {
  cudaEvent_t e0, e1;
  VCT_CUDA(cudaEventCreate(&e0));
  VCT_CUDA(cudaEventCreate(&e1));
  int rc = fn();
  *best = 1e30;
  for (int r = 0; r < reps && !rc; r++) {
    cudaEventRecord(e0, b->stream);
    rc = fn();
    cudaEventRecord(e1, b->stream);
    if (!rc && cudaEventSynchronize(e1) == cudaSuccess) {
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      *best = std::min(*best, (double)ms);
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!rc) VCT_CUDA(cudaStreamSynchronize(b->stream));
  return rc;
}

// The tuner: ray-tile size of the persistent forward, then the view split of
// the quarter-turn backprojector on the batch's largest image.
int autotune(vct_batch* b) {
  int rc;
  double best_total = 0.0;
  if (!b->adjoint) {
    const int cand[] = {32, 64, 128, 256};
    double best = 1e30;
    int best_t = b->tile_rays;
    for (int t : cand) {
      if ((rc = upload_jobs(b, t))) return rc;
      b->tile_rays = t;
      double ms;
      if ((rc = time_ms(b, 2, [&] { return enqueue_forward(b, b->stream); }, &ms))) return rc;
      if (ms < best) {
        best = ms;
        best_t = t;
      }
    }
    b->tile_rays = best_t;
    if ((rc = upload_jobs(b, best_t))) return rc;
    best_total += best;
  }
  // backprojector view split on the largest FBP job
  int big = -1;
  long long big_px = -1;
  for (int i = 0; i < b->n; i++)
    if (!b->adjoint && b->jobs[i].d_img && (long long)b->ctx[i]->dg.N * b->ctx[i]->dg.N > big_px) {
      big = i;
      big_px = (long long)b->ctx[i]->dg.N * b->ctx[i]->dg.N;
    }
  if (big >= 0) {
    vct_ctx* c = b->ctx[big];
    const vct_job& j = b->jobs[big];
    double best = 1e30;
    int best_vs = 4;
    cudaStream_t saved = c->stream;
    c->stream = b->stream;
    for (int vs : {2, 4, 8}) {
      double ms;
      rc = time_ms(b, 3, [&] { return ctx_fbp(c, j.d_sino, j.filter, j.d_img, vs); }, &ms);
      if (rc) break;
      if (ms < best) {
        best = ms;
        best_vs = vs;
      }
    }
    c->stream = saved;
    if (rc) return rc;
    b->view_groups = best_vs;
  }
  b->tuned_ms = best_total;
  return VCT_OK;
}

void release(vct_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->ev_fork) cudaEventDestroy(b->ev_fork);
  if (b->ev_join) cudaEventDestroy(b->ev_join);
  if (b->side) cudaStreamDestroy(b->side);
  if (b->stream) cudaStreamDestroy(b->stream);
  for (auto c : b->ctx) vct_destroy(c);
  b->d_jobs.release();
  b->d_counter.release();
  b->d_xfirst.release();
  b->d_pack.release();
  b->d_post.release();
  b->d_first.release();
  b->d_adj.release();
  b->d_adj_first.release();
}

}  // namespace

extern "C" {

int vct_batch_create(const vct_job* jobs, int n, int M, int device, int tune, vct_batch** out) {
  if (!jobs || n < 1 || !out || M < 1 || M > VCT_MAX_MATERIALS) return fail(VCT_E_ARG, "vct_batch_create: bad argument");
  *out = nullptr;
  int adj = jobs[0].d_grad != nullptr;
  for (int i = 0; i < n; i++) {
    const vct_job& j = jobs[i];
    if ((j.d_grad != nullptr) != adj) return fail(VCT_E_ARG, "vct_batch_create: mixed gradient and MBFPA jobs");
    if (!j.d_maps || !j.mu || !j.pdf || j.NE < 1) return fail(VCT_E_ARG, "vct_batch_create: job without maps or spectrum");
    if (adj ? !j.d_meas : !j.d_sino) return fail(VCT_E_ARG, "vct_batch_create: job without its output/input sinogram");
    if (!adj && j.d_img && j.filter != 1 && j.filter != 2) return fail(VCT_E_ARG, "vct_batch_create: bad filter");
  }
  VCT_CUDA(cudaSetDevice(device));
  vct_batch* b = new vct_batch();
  b->device = device;
  b->n = n;
  b->M = M;
  b->adjoint = adj;
  b->jobs.assign(jobs, jobs + n);
  int rc = VCT_OK;
  auto bail = [&](int code) {
    release(b);
    delete b;
    return code;
  };
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&b->ev_join, cudaEventDisableTiming) != cudaSuccess)
    return bail(fail(VCT_E_CUDA, "vct_batch_create: stream"));
  // One context per job: geometry tables, packed maps, spectrum, scratch.
  for (int i = 0; i < n; i++) {
    const vct_job& j = jobs[i];
    vct_ctx* c = nullptr;
    if ((rc = vct_create(&j.geo, device, &c))) return bail(rc);
    b->ctx.push_back(c);
    if (j.density_units > 0 && (rc = vct_set_density_scale(c, j.density_units))) return bail(rc);
    if ((rc = vct_set_spectrum(c, j.mu, j.pdf, M, j.NE)) || (rc = vct_set_maps_dev(c, j.d_maps, M))) return bail(rc);
    b->ne_max = std::max(b->ne_max, j.NE);
    if (adj) {
      if ((rc = ctx_adj_prepare(c))) return bail(rc);
      // allocates the adjoint's scratch (and checks the call) before capture
      if ((rc = ctx_adj_run(c, 0, j.d_meas, j.d_weights, nullptr, j.d_grad, j.d_loss))) return bail(rc);
    } else if (j.d_img) {
      if ((rc = ctx_build_filter(c, j.filter))) return bail(rc);
      const size_t vc = (size_t)j.geo.views * (j.geo.end_channel - j.geo.start_channel);
      if ((rc = c->fbp_q.ensure(vc)) || (rc = c->fbp_q2.ensure(vc))) return bail(rc);
    }
    if (cudaStreamSynchronize(c->stream) != cudaSuccess) return bail(fail(VCT_E_CUDA, "vct_batch_create: job set-up"));
  }
  if ((rc = b->d_jobs.ensure(n)) || (rc = b->d_counter.ensure(1))) return bail(rc);
  if (!adj) {
    int occ = 0;
    if ((rc = forward_batch_occupancy(M, b->ne_max, &occ))) return bail(rc);
    b->blocks_per_sm = std::max(occ, 1);
    b->grid = b->blocks_per_sm * sm_count(device);
    if ((rc = upload_jobs(b, b->tile_rays))) return bail(rc);
  }
  if ((rc = upload_stage_tables(b))) return bail(rc);
  if (adj && (rc = upload_adjoint_tables(b))) return bail(rc);
  if (tune && (rc = autotune(b))) return bail(rc);
  // Capture one run.
  cudaError_t e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return bail(cuda_fail(e, "vct_batch_create: begin capture"));
  rc = enqueue_all(b);
  cudaGraph_t g = nullptr;
  e = cudaStreamEndCapture(b->stream, &g);
  if (rc) {
    if (g) cudaGraphDestroy(g);
    return bail(rc);
  }
  if (e != cudaSuccess) return bail(cuda_fail(e, "vct_batch_create: end capture"));
  b->graph = g;
  if ((e = cudaGraphInstantiate(&b->exec, g, 0)) != cudaSuccess) return bail(cuda_fail(e, "vct_batch_create: instantiate"));
  *out = b;
  return VCT_OK;
}

int vct_batch_run(vct_batch* b, void* stream) {
  if (!b) return fail(VCT_E_ARG, "vct_batch_run: null batch");
  nvtxRangePushA("vct_batch_run");
  struct Pop {
    ~Pop() { nvtxRangePop(); }
  } pop;
  VCT_CUDA(cudaSetDevice(b->device));
  VCT_CUDA(cudaGraphLaunch(b->exec, stream ? (cudaStream_t)stream : b->stream));
  return VCT_OK;
}

int vct_batch_synchronize(vct_batch* b) {
  if (!b) return fail(VCT_E_ARG, "vct_batch_synchronize: null batch");
  VCT_CUDA(cudaSetDevice(b->device));
  VCT_CUDA(cudaStreamSynchronize(b->stream));
  return VCT_OK;
}

int vct_batch_config(const vct_batch* b, int* tile_rays, int* blocks_per_sm, int* view_groups, int* kernels) {
  if (!b) return fail(VCT_E_ARG, "vct_batch_config: null batch");
  if (tile_rays) *tile_rays = b->adjoint ? 128 : b->tile_rays;
  if (blocks_per_sm) *blocks_per_sm = b->blocks_per_sm;
  if (view_groups) *view_groups = b->view_groups;
  if (kernels) {
    size_t nodes = 0;
    int k = 0;
    if (b->graph && cudaGraphGetNodes(b->graph, nullptr, &nodes) == cudaSuccess) {
      std::vector<cudaGraphNode_t> v(nodes);
      cudaGraphGetNodes(b->graph, v.data(), &nodes);
      for (auto nd : v) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) k++;
      }
    }
    *kernels = k;
  }
  return VCT_OK;
}

void vct_batch_destroy(vct_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  release(b);
  delete b;
}

int vct_forward_batched(const vct_job* jobs, int n, int M, int device) {
  vct_batch* b = nullptr;
  int rc = vct_batch_create(jobs, n, M, device, 0, &b);
  if (rc) return rc;
  rc = vct_batch_run(b, nullptr);
  if (!rc) rc = vct_batch_synchronize(b);
  vct_batch_destroy(b);
  return rc;
}

}  // extern "C"
