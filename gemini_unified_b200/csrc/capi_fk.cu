// C ABI of the FK hot path (include/gemini_fk.h): context, model, nodes,
// frequency grid and the batched FK run.
//
// The reference's driver loops (computeGreenFKSpectraForSynthetics.f90:361-501)
// become one launch: all (omega, l) items of a frequency slab are queued,
// most expensive frequencies first, and drained by a persistent grid.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/gemini_fk.h"
#include "fk_kernel.h"
#include "fk_types.cuh"
#include "proposer.h"
#include "synth.h"

using namespace gem;

struct gem_ctx {
  int device = 0;
  int backend = GEM_BACKEND_GPU_FP64;
  int nsm = 148;
  std::string err;
  // model (1-based host copies)
  bool have_model = false;
  double fref = 1, rearth = 0, ric = 0, roc = 0;
  int aniflag = 0, fsflag = 0, equidis = 0, nlay = 0, nk = 0, nic = 0, noc = 0;
  std::vector<int> iflso, iktop, ikbot;
  std::vector<double> rb, drk, rk, ro, vpv, vph, vsv, vsh, eta, qkinv, qminv;
  // device copies of the knot arrays (1-based)
  double* d_knots = nullptr;   // 11 arrays of nk+1
  int* d_lay = nullptr;        // iktop, ikbot
  // nodes
  bool have_nodes = false;
  int nnod = 0;
  std::vector<double> rnod;
  std::vector<int> state, layer;
  // buffers grown on demand
  double* d_spl = nullptr; size_t spl_cap = 0;
  double* d_poly = nullptr; size_t poly_cap = 0;
  double2* d_scratch = nullptr; size_t scratch_cap = 0;
  int2* d_items = nullptr; size_t items_cap = 0;
  int* d_order = nullptr; size_t order_cap = 0;
  int32_t* d_status = nullptr; size_t status_cap = 0;
  double* d_rstart = nullptr; size_t rstart_cap = 0;
  double2* d_um = nullptr; size_t um_cap = 0;
  double2* d_dm = nullptr; size_t dm_cap = 0;
  double2* d_dets = nullptr; size_t dets_cap = 0;
  cudaEvent_t ev_ph[3] = {nullptr, nullptr, nullptr};
  float phase_ms[3] = {0, 0, 0};
  int* d_slots = nullptr; size_t slots_cap = 0;   // jf + koff
  unsigned int* d_queue = nullptr;
  unsigned long long* d_stats = nullptr;
  int* d_err = nullptr;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  // optional instrumentation (enabled by gem_instrument)
  unsigned long long* d_prof = nullptr;
  unsigned long long* d_warp_ns = nullptr;
  int last_grid = 0;
  gem_stats stats{};
  // device buffers of the other entry points, grown on demand
  void* d_aux[16] = {};
  size_t aux_cap[16] = {};
  int kopt = 6;   // order target of the step-size control (gem_order_target; fast backend)
  unsigned long long tc_wait_ns = 0;   // pipeline wait limit of the tensor-core sums (gem_tc_wait_limit; 0: 1 s)
  int dsv = 0;    // set by gem_fk_run_dsv* for the length of one run: DSV spectra with derivatives
  int jsl = 0, jsr = 0;   // set by gem_fk_run_aski* for one run: node range of the minors (0: the receiver)
  // schedule of each solver phase (index into FK_SCHED_*), per build: [0] plain, [1] fast
  int sched[2][3] = {{FK_SCHED_DEFAULT[0], FK_SCHED_DEFAULT[1], FK_SCHED_DEFAULT[2]},
                     {FK_SCHED_DEFAULT[0], FK_SCHED_DEFAULT[1], FK_SCHED_DEFAULT[2]}};
  int last_block = 0;   // threads per block of the last spheroidal launch (instrumentation)
  // bookkeeping deferral of each phase (index into FK_DEFER_*), per build
  int defer[2][3] = {{FK_DEFER_DEFAULT, FK_DEFER_DEFAULT, FK_DEFER_DEFAULT},
                     {FK_DEFER_DEFAULT, FK_DEFER_DEFAULT, FK_DEFER_DEFAULT}};
  // queue granularity of each phase (index into FK_GRAN), per build
  int qgran[2][3] = {{FK_GRAN_DEFAULT, FK_GRAN_DEFAULT, FK_GRAN_DEFAULT},
                     {FK_GRAN_DEFAULT, FK_GRAN_DEFAULT, FK_GRAN_DEFAULT}};
  // captured launch sequence of one slab (gem_fk_graph_build)
  cudaGraphExec_t graph_exec = nullptr;
  cudaStream_t graph_stream = nullptr;
  bool graph_valid = false;
  long long graph_items = 0;
  // learned proposer (fast backend): FP16 weights, feature normalisation, proposals per (phase, item)
  __half* d_propw = nullptr;
  float* d_propnorm = nullptr;
  int prop_use = 0;
  float prop_margin = 0.1f;
  signed char* d_prop_kopt = nullptr; size_t prop_kopt_cap = 0;
  float* d_prop_hs = nullptr; size_t prop_hs_cap = 0;
  float* d_feat = nullptr; size_t feat_cap = 0;
  bool dump_feat = false;
  long long feat_n = 0;
  // optional step log (gem_steplog)
  StepRec* d_steplog = nullptr;
  unsigned long long steplog_cap = 0;
  unsigned long long* d_steplog_n = nullptr;
};

namespace {

int fail(gem_ctx* c, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (c) c->err = buf;
  return GEM_ERROR;
}

#define CK(call)                                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess) return fail(ctx, "%s: %s", #call, cudaGetErrorString(e_));   \
  } while (0)

template <class T>
int grow(gem_ctx* ctx, T*& p, size_t& cap, size_t n) {
  if (n <= cap && p) return GEM_OK;
  if (p) cudaFree(p);
  p = nullptr; cap = 0;
  size_t want = std::max(n, (size_t)1);
  CK(cudaMalloc((void**)&p, want * sizeof(T)));
  cap = want;
  return GEM_OK;
}

int nint_(double x) { return x >= 0 ? (int)std::floor(x + 0.5) : -(int)std::floor(-x + 0.5); }

struct Grid {
  double df, sigma, dwn;
  int nf1, nf2, nwnmax;
  std::vector<int> nwn;   // [nf2+1], 1-based jf
};

// computeGreenFKSpectraForSynthetics.f90:186-236
void make_grid(const gem_fk_params* p, double rearth, Grid& g) {
  const double PIF = PI_F, TWOPIF = TWO_PI_F;
  g.df = 1.0 / p->tlen;
  g.nf2 = nint_(p->fmax / g.df) + 1;
  g.nf1 = std::max(nint_(p->fmin / g.df), 2);
  double ommax = TWOPIF * (double)(g.nf2 - 1) * g.df;
  g.sigma = 5.0 * g.df;
  g.dwn = TWOPIF / p->xlen;
  double wnmax = 0.5 * ommax * (p->p1lim + p->p2lim) / (1.0 - p->frac);
  g.nwnmax = (int)(wnmax / g.dwn) + 1;
  if (p->global_ == 1) g.nwnmax = nint_(wnmax * rearth - 0.5) + 1;
  g.nwn.assign(g.nf2 + 1, 0);
  for (int jf = g.nf1; jf <= g.nf2; ++jf) {
    double f = (double)(jf - 1) * g.df;
    double omre = 2.0 * PIF * f;
    double wn2;
    if (f <= 0.5 * (double)(g.nf2 - 1) * g.df) wn2 = omre * p->p1lim + p->frac * wnmax;
    else wn2 = 0.5 * ommax * (p->p1lim + p->p2lim) + (omre - ommax) * p->p2lim + p->frac * wnmax;
    if (p->global_ == 1) g.nwn[jf] = nint_(wn2 * rearth - 0.5) + 1;
    else g.nwn[jf] = (int)(wn2 / g.dwn) + 1;
  }
}

int nsp_of(const gem_fk_params* p) {
  int njsph = p->istyp == 0 ? 2 : 4, njtor = p->istyp == 0 ? 1 : 2;
  return p->stressflag ? 4 * njsph + 2 * njtor : 2 * njsph + njtor;
}

// spectra per node of a run: U, V, dU/dr, dV/dr and W, dW/dr in DSV mode
// (computeGreenFKSpectraForASKI.f90:231-233,328)
int nsp_run(const gem_ctx* ctx, const gem_fk_params* p) {
  int njsph = p->istyp == 0 ? 2 : 4, njtor = p->istyp == 0 ? 1 : 2;
  return ctx->dsv ? 4 * njsph + 2 * njtor : nsp_of(p);
}

int check_params(gem_ctx* ctx, const gem_fk_params* p) {
  if (!ctx->have_model) return fail(ctx, "no earth model loaded");
  if (!ctx->have_nodes) return fail(ctx, "no external nodes set");
  if (!p) return fail(ctx, "null parameters");
  if (!(p->tlen > 0) || !(p->fmax > 0) || !(p->eps > 0)) return fail(ctx, "invalid TLEN/FMAX/ACCURACY");
  if (p->attmode < 0 || p->attmode > 3) return fail(ctx, "Invalid attenuation mode");
  if (p->istyp != 0 && p->istyp != 1) return fail(ctx, "Invalid source type");
  if (p->jre < 1 || p->jre > ctx->nnod) return fail(ctx, "Invalid index for receiver node");
  if (p->global_ == 0 && !(p->xlen > 0)) return fail(ctx, "invalid XLEN");
  if (ctx->state[p->jre] == 1) return fail(ctx, "receiver in an ocean layer is not supported");
  if (ctx->dsv)
    for (int n = 1; n <= ctx->nnod; ++n)
      if (ctx->state[n] != 0) return fail(ctx, "DSV spectra: node %d lies in a fluid layer (not supported)", n);
  if (ctx->rnod[1] < ctx->rb[1])
    return fail(ctx, "External nodes within inner homogeneous sphere (halfspace) are not allowed.");
  return GEM_OK;
}

}  // namespace

int gem_set_error(gem_ctx* ctx, const char* msg) { return fail(ctx, "%s", msg); }
void gem_note_synth_ms(gem_ctx* ctx, float ms) { if (ctx) ctx->stats.synth_ms = ms; }
int gem_ctx_device(const gem_ctx* ctx) { return ctx->device; }
int gem_ctx_backend(const gem_ctx* ctx) { return ctx->backend; }
unsigned long long gem_ctx_tc_wait_ns(const gem_ctx* ctx) { return ctx->tc_wait_ns; }
void* gem_ctx_aux(gem_ctx* ctx, int slot, size_t bytes) {
  if (slot < 0 || slot >= 16) return nullptr;
  if (ctx->d_aux[slot] && ctx->aux_cap[slot] >= bytes) return ctx->d_aux[slot];
  cudaFree(ctx->d_aux[slot]);
  ctx->d_aux[slot] = nullptr; ctx->aux_cap[slot] = 0;
  if (cudaMalloc(&ctx->d_aux[slot], std::max(bytes, (size_t)256)) != cudaSuccess) {
    ctx->d_aux[slot] = nullptr;
    fail(ctx, "device allocation of %zu bytes failed", bytes);
    return nullptr;
  }
  ctx->aux_cap[slot] = std::max(bytes, (size_t)256);
  return ctx->d_aux[slot];
}

extern "C" {

int gem_ctx_create(int device, int backend, gem_ctx** out) {
  if (!out) return GEM_ERROR;
  *out = nullptr;
  if (backend != GEM_BACKEND_GPU_FP64 && backend != GEM_BACKEND_GPU_FAST) return GEM_ERROR;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= device || device < 0) return GEM_ERROR;
  gem_ctx* ctx = new gem_ctx();
  ctx->device = device;
  ctx->backend = backend;
  if (cudaSetDevice(device) != cudaSuccess) { delete ctx; return GEM_ERROR; }
  cudaDeviceGetAttribute(&ctx->nsm, cudaDevAttrMultiProcessorCount, device);
  if (cudaMalloc(&ctx->d_queue, 4 * sizeof(unsigned int)) != cudaSuccess ||
      cudaMalloc(&ctx->d_stats, 32 * sizeof(unsigned long long)) != cudaSuccess ||
      cudaMalloc(&ctx->d_err, sizeof(int)) != cudaSuccess) {
    gem_ctx_destroy(ctx);
    return GEM_ERROR;
  }
  for (auto& e : ctx->ev) cudaEventCreate(&e);
  for (auto& e : ctx->ev_ph) cudaEventCreate(&e);
  *out = ctx;
  return GEM_OK;
}

void gem_ctx_destroy(gem_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaFree(ctx->d_knots); cudaFree(ctx->d_lay); cudaFree(ctx->d_spl); cudaFree(ctx->d_scratch); cudaFree(ctx->d_poly);
  cudaFree(ctx->d_items); cudaFree(ctx->d_slots); cudaFree(ctx->d_queue); cudaFree(ctx->d_stats);
  cudaFree(ctx->d_err); cudaFree(ctx->d_prof); cudaFree(ctx->d_warp_ns);
  cudaFree(ctx->d_order); cudaFree(ctx->d_status); cudaFree(ctx->d_rstart); cudaFree(ctx->d_um);
  cudaFree(ctx->d_dm); cudaFree(ctx->d_dets);
  for (auto* a : ctx->d_aux) cudaFree(a);
  cudaFree(ctx->d_steplog); cudaFree(ctx->d_steplog_n);
  cudaFree(ctx->d_propw); cudaFree(ctx->d_propnorm); cudaFree(ctx->d_prop_kopt); cudaFree(ctx->d_prop_hs);
  cudaFree(ctx->d_feat);
  if (ctx->graph_exec) cudaGraphExecDestroy(ctx->graph_exec);
  if (ctx->graph_stream) cudaStreamDestroy(ctx->graph_stream);
  for (auto& e : ctx->ev) if (e) cudaEventDestroy(e);
  for (auto& e : ctx->ev_ph) if (e) cudaEventDestroy(e);
  delete ctx;
}

const char* gem_last_error(const gem_ctx* ctx) { return ctx ? ctx->err.c_str() : "null context"; }

int gem_model_load(gem_ctx* ctx, const gem_model_desc* m) {
  if (!ctx || !m) return GEM_ERROR;
  ctx->graph_valid = false;
  CK(cudaSetDevice(ctx->device));
  if (m->nlay < 2 || m->nlay > MAXLAY) return fail(ctx, "number of layers %d outside 2..%d", m->nlay, MAXLAY);
  if (m->nk < 2 || m->nk > MAXKNOT - 1) return fail(ctx, "number of knots %d outside 2..%d", m->nk, MAXKNOT - 1);
  if (m->iflso[m->nlay - 1] == 1 && m->fsflag == 1) return fail(ctx, "Full space and ocean is not allowed!!");
  int L = m->nlay, K = m->nk;
  ctx->fref = m->fref; ctx->rearth = m->rearth; ctx->ric = m->ric; ctx->roc = m->roc;
  ctx->aniflag = m->aniflag; ctx->fsflag = m->fsflag; ctx->equidis = m->equidis;
  ctx->nlay = L; ctx->nk = K; ctx->nic = m->nic; ctx->noc = m->noc;
  ctx->iflso.assign(L + 1, 0); ctx->iktop.assign(L + 1, 0); ctx->ikbot.assign(L + 1, 0);
  ctx->rb.assign(L + 1, 0.0); ctx->drk.assign(L + 1, -1.0);
  for (int i = 1; i <= L; ++i) { ctx->iflso[i] = m->iflso[i - 1]; ctx->iktop[i] = m->iktop[i - 1]; ctx->rb[i] = m->rb[i - 1]; }
  for (int i = 2; i <= L; ++i) ctx->ikbot[i] = ctx->iktop[i - 1] + 1;
  for (int i = 1; i <= L; ++i)
    if (ctx->iktop[i] < 1 || ctx->iktop[i] > K || (i > 1 && ctx->iktop[i] - ctx->ikbot[i] + 1 > MAX_LAYER_KNOTS))
      return fail(ctx, "invalid layer knot indices");
  auto cp = [&](std::vector<double>& v, const double* s) { v.assign(K + 1, 0.0); for (int i = 1; i <= K; ++i) v[i] = s[i - 1]; };
  ctx->rk.assign(K + 1, 0.0);
  for (int i = 1; i <= K; ++i) ctx->rk[i] = m->rearth - m->depth[i - 1];             // nodeEarthmodel.f90:175
  for (int i = 2; i < K + 1; ++i)
    if (!(ctx->rk[i] >= ctx->rk[i - 1])) return fail(ctx, "knot radii must not decrease");
  if (m->equidis == 1)
    for (int nl = 2; nl <= L; ++nl)
      ctx->drk[nl] = (ctx->rk[ctx->iktop[nl]] - ctx->rk[ctx->ikbot[nl]]) / (double)(ctx->iktop[nl] - ctx->ikbot[nl]);
  cp(ctx->ro, m->ro);
  ctx->qkinv.assign(K + 1, 0.0); ctx->qminv.assign(K + 1, 0.0);
  for (int i = 1; i <= K; ++i) {
    ctx->qkinv[i] = 1.0 / m->qk[i - 1];
    ctx->qminv[i] = 1.0 / m->qm[i - 1];
    if (ctx->qminv[i] < 0.0) ctx->qminv[i] = 0.0;
  }
  if (m->aniflag == 0) {
    cp(ctx->vpv, m->vpv); cp(ctx->vph, m->vpv); cp(ctx->vsv, m->vsv); cp(ctx->vsh, m->vsv);
    ctx->eta.assign(K + 1, 1.0);
  } else {
    cp(ctx->vpv, m->vpv); cp(ctx->vph, m->vph); cp(ctx->vsv, m->vsv); cp(ctx->vsh, m->vsh); cp(ctx->eta, m->eta);
  }
  for (int i = 1; i <= K; ++i)
    if (!std::isfinite(ctx->ro[i]) || !std::isfinite(ctx->vpv[i]) || !std::isfinite(ctx->vsv[i]) ||
        !std::isfinite(ctx->rk[i]))
      return fail(ctx, "non-finite model value at knot %d", i);
  // device knot arrays: ro vpv vph vsv vsh eta qkinv qminv rk
  cudaFree(ctx->d_knots); ctx->d_knots = nullptr;
  cudaFree(ctx->d_lay); ctx->d_lay = nullptr;
  CK(cudaMalloc(&ctx->d_knots, 9 * (K + 1) * sizeof(double)));
  CK(cudaMalloc(&ctx->d_lay, 2 * (L + 1) * sizeof(int)));
  const std::vector<double>* arr[9] = {&ctx->ro, &ctx->vpv, &ctx->vph, &ctx->vsv, &ctx->vsh,
                                       &ctx->eta, &ctx->qkinv, &ctx->qminv, &ctx->rk};
  for (int a = 0; a < 9; ++a)
    CK(cudaMemcpy(ctx->d_knots + a * (K + 1), arr[a]->data(), (K + 1) * sizeof(double), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_lay, ctx->iktop.data(), (L + 1) * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_lay + (L + 1), ctx->ikbot.data(), (L + 1) * sizeof(int), cudaMemcpyHostToDevice));
  ctx->have_model = true;
  ctx->have_nodes = false;
  return GEM_OK;
}

int gem_nodes_set(gem_ctx* ctx, int nnod, const double* r, const int* state, const int* layer) {
  if (ctx) ctx->graph_valid = false;
  if (!ctx) return GEM_ERROR;
  if (!ctx->have_model) return fail(ctx, "load the earth model before the nodes");
  if (nnod < 1 || nnod > MAXNOD) return fail(ctx, "number of nodes %d outside 1..%d", nnod, MAXNOD);
  ctx->nnod = nnod;
  ctx->rnod.assign(nnod + 1, 0.0); ctx->state.assign(nnod + 1, 0); ctx->layer.assign(nnod + 1, 0);
  for (int i = 1; i <= nnod; ++i) {
    ctx->rnod[i] = r[i - 1]; ctx->state[i] = state[i - 1]; ctx->layer[i] = layer[i - 1];
    if (ctx->layer[i] < 1 || ctx->layer[i] > ctx->nlay) return fail(ctx, "node %d: layer out of range", i);
    if (!(ctx->rnod[i] > 0) || (i > 1 && !(ctx->rnod[i] > ctx->rnod[i - 1])))
      return fail(ctx, "node radii must be positive and ascending");
  }
  ctx->have_nodes = true;
  return GEM_OK;
}

int gem_fk_grid(gem_ctx* ctx, const gem_fk_params* p, int* nf1, int* nf2, int* nwnmax, int* nsp, int* nwn, int cap) {
  if (!ctx || !p) return GEM_ERROR;
  if (!ctx->have_model) return fail(ctx, "no earth model loaded");
  Grid g;
  make_grid(p, ctx->rearth, g);
  if (nf1) *nf1 = g.nf1;
  if (nf2) *nf2 = g.nf2;
  if (nwnmax) *nwnmax = g.nwnmax;
  if (nsp) *nsp = nsp_of(p);
  if (nwn) {
    if (cap < g.nf2) return fail(ctx, "nwn capacity %d < nf2 %d", cap, g.nf2);
    for (int jf = 1; jf <= g.nf2; ++jf) nwn[jf - 1] = g.nwn[jf];
  }
  return GEM_OK;
}

}  // extern "C"

namespace {

// Everything one FK slab run needs on the device, prepared on the host: the
// parameter block, the item and queue tables (uploaded), the kernel arguments
// and the grids.  fk_enqueue then issues only device work, so that the same
// sequence can be run directly or captured into a CUDA graph.
struct SlabPlan {
  FKStatic P;
  PrepArgs A;
  PropArgs PA;
  FKLaunch L;
  int grid[3];
  int nslot, nitems, nsp;
  long long nkf;
  size_t spl_n, nout, nu, nd, ndet;
  bool fast, propose;
  int sched[3], defer[3], qgran[3];
  float* gfre;
  float* gfim;
  double* gf64;
  int32_t* status;
};

int fk_prepare(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* d_gfre, float* d_gfim,
               double* d_gf64, int32_t* d_status, SlabPlan& S) {
  int rc = check_params(ctx, p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  ctx->graph_valid = false;   // the tables below are rewritten: a captured graph no longer matches them
  Grid g;
  make_grid(p, ctx->rearth, g);
  if (jf_first < g.nf1 || jf_last > g.nf2 || jf_first > jf_last)
    return fail(ctx, "frequency range %d..%d outside %d..%d", jf_first, jf_last, g.nf1, g.nf2);
  const int nslot = jf_last - jf_first + 1;
  const int nsp = nsp_run(ctx, p);
  S.nslot = nslot; S.nsp = nsp;
  // ---- parameter block
  FKStatic& P = S.P;
  memset(&P, 0, sizeof P);
  P.nlay = ctx->nlay; P.nk = ctx->nk; P.noc = ctx->noc; P.nic = ctx->nic; P.equidis = ctx->equidis;
  P.fsflag = ctx->fsflag; P.nnod = ctx->nnod; P.jre = p->jre;
  P.hascore = (ctx->noc > 0 && ctx->iflso[ctx->noc] == 1) ? 1 : 0;
  P.hasocean = ctx->iflso[ctx->nlay] == 1 ? 1 : 0;
  P.istyp = p->istyp; P.stressflag = p->stressflag; P.global_ = p->global_; P.nsp = nsp;
  P.ncsph = 4; P.nctor = 2;
  P.njsph = p->istyp == 0 ? 2 : 4; P.njtor = p->istyp == 0 ? 1 : 2;
  P.dsvstep = p->stressflag ? 1 : 2;
  P.dsv = ctx->dsv;
  P.jsl = ctx->jsl ? ctx->jsl : p->jre;
  P.jsr = ctx->jsr ? ctx->jsr : p->jre;
  P.rearth = ctx->rearth; P.ric = ctx->ric; P.roc = ctx->roc; P.rhs = ctx->rb[1];
  P.ruc = P.hasocean ? ctx->rb[ctx->nlay - 1] : ctx->rearth;
  P.eps = p->eps; P.sigma = g.sigma; P.df = g.df; P.dwn = g.dwn;
  P.kopt = ctx->backend == GEM_BACKEND_GPU_FAST ? ctx->kopt : 6;
  for (int i = 1; i <= ctx->nlay; ++i) {
    P.rb[i] = ctx->rb[i]; P.drk[i] = ctx->drk[i]; P.iflso[i] = ctx->iflso[i]; P.iktop[i] = ctx->iktop[i];
  }
  for (int i = 1; i <= ctx->nk; ++i) P.rk[i] = ctx->rk[i];
  for (int i = 1; i <= ctx->nnod; ++i) { P.rnod[i] = ctx->rnod[i]; P.state[i] = ctx->state[i]; P.layer[i] = ctx->layer[i]; }
  // ---- frequency slots; output index k = koff[slot] + iwn - 1
  std::vector<int> slots(2 * nslot);
  long long nkf = 0;
  for (int s = 0; s < nslot; ++s) {
    slots[s] = jf_first + s;
    slots[nslot + s] = (int)nkf;
    nkf += g.nwn[jf_first + s];
  }
  std::vector<int2> items((size_t)nkf);
  for (int s = 0; s < nslot; ++s)
    for (int iwn = 1; iwn <= g.nwn[jf_first + s]; ++iwn) items[slots[nslot + s] + iwn - 1] = make_int2(s, iwn);
  // work queue: high frequencies first, low degrees (long paths) first within a frequency
  std::vector<int> order;
  order.reserve((size_t)nkf);
  for (int s = nslot - 1; s >= 0; --s)
    for (int iwn = 1; iwn <= g.nwn[jf_first + s]; ++iwn) order.push_back(slots[nslot + s] + iwn - 1);
  const int nitems = (int)nkf;
  S.nkf = nkf; S.nitems = nitems;
  if (grow(ctx, ctx->d_items, ctx->items_cap, items.size())) return GEM_ERROR;
  if (grow(ctx, ctx->d_order, ctx->order_cap, order.size())) return GEM_ERROR;
  if (grow(ctx, ctx->d_slots, ctx->slots_cap, slots.size())) return GEM_ERROR;
  CK(cudaMemcpy(ctx->d_items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_order, order.data(), order.size() * sizeof(int), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_slots, slots.data(), slots.size() * sizeof(int), cudaMemcpyHostToDevice));
  // ---- model preparation for all slots
  S.spl_n = (size_t)nslot * (ctx->nk + 1) * SPL_STRIDE;
  if (grow(ctx, ctx->d_spl, ctx->spl_cap, S.spl_n)) return GEM_ERROR;
  PrepArgs& A = S.A;
  const int K1 = ctx->nk + 1;
  A.nslot = nslot; A.nk = ctx->nk; A.nlay = ctx->nlay; A.attmode = p->attmode; A.df = g.df; A.fref = ctx->fref;
  A.jf = ctx->d_slots;
  A.ro = ctx->d_knots; A.vpv = ctx->d_knots + K1; A.vph = ctx->d_knots + 2 * K1; A.vsv = ctx->d_knots + 3 * K1;
  A.vsh = ctx->d_knots + 4 * K1; A.eta = ctx->d_knots + 5 * K1; A.qkinv = ctx->d_knots + 6 * K1;
  A.qminv = ctx->d_knots + 7 * K1; A.rk = ctx->d_knots + 8 * K1;
  A.iktop = ctx->d_lay; A.ikbot = ctx->d_lay + (ctx->nlay + 1);
  A.spl = ctx->d_spl;
  const bool fast = ctx->backend == GEM_BACKEND_GPU_FAST;
  S.fast = fast;
  if (fast) {
    size_t poly_n = (size_t)nslot * (ctx->nk + 1) * POLY_STRIDE;
    if (grow(ctx, ctx->d_poly, ctx->poly_cap, poly_n)) return GEM_ERROR;
  }
  // ---- outputs and per-item storage (zeroed by fk_enqueue)
  S.nout = (size_t)nkf * nsp * ctx->nnod;
  S.gfre = d_gfre; S.gfim = d_gfim; S.gf64 = d_gf64;
  int32_t* status = d_status;
  if (!status) {
    if (grow(ctx, ctx->d_status, ctx->status_cap, (size_t)nkf)) return GEM_ERROR;
    status = ctx->d_status;
  }
  S.status = status;
  // minors at nodes 1..jsr (up) and jsl..nnod (down), determinants at jsl..jsr
  S.nu = (size_t)P.jsr * 6 * nkf;
  S.nd = (size_t)(ctx->nnod - P.jsl + 1) * 6 * nkf;
  S.ndet = (size_t)(P.jsr - P.jsl + 1) * nkf;
  if (grow(ctx, ctx->d_um, ctx->um_cap, S.nu)) return GEM_ERROR;
  if (grow(ctx, ctx->d_dm, ctx->dm_cap, S.nd)) return GEM_ERROR;
  if (grow(ctx, ctx->d_rstart, ctx->rstart_cap, 2 * (size_t)nkf)) return GEM_ERROR;
  if (grow(ctx, ctx->d_dets, ctx->dets_cap, S.ndet)) return GEM_ERROR;
  // ---- grid: the largest of the three phases sets the per-lane scratch
  long long nthreads = 0;
  for (int ph = 0; ph < 3; ++ph) {
    const int sc = ctx->sched[fast ? 1 : 0][ph];
    S.sched[ph] = sc;
    S.defer[ph] = ctx->defer[fast ? 1 : 0][ph];
    S.qgran[ph] = ctx->qgran[fast ? 1 : 0][ph];
    S.grid[ph] = ctx->nsm * (fast ? gem_fast::fk_phase_blocks_per_sm(ph, sc) : gem_plain::fk_phase_blocks_per_sm(ph, sc));
    nthreads = std::max(nthreads, (long long)S.grid[ph] * FK_SCHED_BLOCK[sc]);
  }
  size_t scratch_n = (size_t)nthreads * ((ctx->nnod + 1) * gem_plain::fk_lane_slot_per_node() + FK_LANE_STEP_SLOTS);
  if (grow(ctx, ctx->d_scratch, ctx->scratch_cap, scratch_n)) return GEM_ERROR;
  FKLaunch& L = S.L;
  L.spl = ctx->d_spl; L.poly = fast ? ctx->d_poly : nullptr; L.jf = ctx->d_slots; L.koff = ctx->d_slots + nslot; L.items = ctx->d_items;
  L.order = ctx->d_order;
  L.nitems = nitems; L.nkf = nkf; L.gf64 = (double2*)d_gf64; L.gfre = d_gfre; L.gfim = d_gfim;
  L.status = status; L.scratch = ctx->d_scratch; L.nthreads = nthreads; L.queue = ctx->d_queue;
  L.stats = ctx->d_stats;
  L.rstart = ctx->d_rstart; L.um = (double2*)ctx->d_um; L.dm = (double2*)ctx->d_dm; L.dets = (double2*)ctx->d_dets;
  L.prof = nullptr;
  L.warp_ns = nullptr;
  L.steplog = ctx->d_steplog; L.steplog_cap = ctx->steplog_cap; L.steplog_n = ctx->d_steplog_n;
  L.prop_kopt = nullptr; L.prop_hs = nullptr;
  L.adv_min = 1; L.adv_wait = 0; L.qgran = 1; L.qchunk = 0;
  L.nsrc = 0; L.src_blk = 0;
  ctx->last_grid = S.grid[1];
  ctx->last_block = FK_SCHED_BLOCK[S.sched[1]];
  // ---- learned proposer: features / proposals per (phase, item) from the start radii
  S.propose = fast && ctx->prop_use != 0 && ctx->d_propw;
  if (ctx->dump_feat || S.propose) {
    PropArgs& PA = S.PA;
    PA = PropArgs{};
    PA.items = ctx->d_items; PA.jf = ctx->d_slots; PA.rstart = ctx->d_rstart; PA.nkf = nkf; PA.nitems = nitems;
    PA.nk = ctx->nk; PA.nlay = ctx->nlay; PA.use = ctx->prop_use; PA.margin = ctx->prop_margin;
    PA.df = P.df; PA.rearth = ctx->rearth;
    for (int i = 0; i <= ctx->nk; ++i) {
      PA.rk[i] = ctx->rk[i];
      PA.knot_feat[3 * i + 0] = (float)(ctx->vpv[i] / 1e4);
      PA.knot_feat[3 * i + 1] = (float)(ctx->vsv[i] / 1e4);
      PA.knot_feat[3 * i + 2] = (float)(ctx->ro[i] / 1e4);
    }
    for (int i = 0; i <= ctx->nlay; ++i) PA.rb[i] = ctx->rb[i];
    if (ctx->dump_feat && grow(ctx, ctx->d_feat, ctx->feat_cap, (size_t)3 * nitems * PROP_NF)) return GEM_ERROR;
    if (S.propose) {
      if (grow(ctx, ctx->d_prop_kopt, ctx->prop_kopt_cap, (size_t)3 * nkf)) return GEM_ERROR;
      if (grow(ctx, ctx->d_prop_hs, ctx->prop_hs_cap, (size_t)3 * nkf)) return GEM_ERROR;
      L.prop_kopt = ctx->d_prop_kopt;
      L.prop_hs = ctx->d_prop_hs;
    }
  }
  return GEM_OK;
}

// The device work of one slab on stream st: zeroing, model preparation, start
// radii, proposals, the three phases and the per-phase counter snapshots.
// timed: record the context's events (not inside a graph capture).
int fk_enqueue(gem_ctx* ctx, SlabPlan& S, cudaStream_t st, bool timed) {
  const FKStatic& P = S.P;
  CK(cudaMemsetAsync(ctx->d_spl, 0, S.spl_n * sizeof(double), st));
  CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st));
  if (timed) CK(cudaEventRecord(ctx->ev[0], st));
  CK(launch_prep(S.A, ctx->d_err, st));
  if (S.fast) CK(launch_poly(S.A, ctx->d_poly, st));
  if (timed) CK(cudaEventRecord(ctx->ev[1], st));
  if (S.gf64) CK(cudaMemsetAsync(S.gf64, 0, S.nout * 2 * sizeof(double), st));
  if (S.gfre) CK(cudaMemsetAsync(S.gfre, 0, S.nout * sizeof(float), st));
  if (S.gfim) CK(cudaMemsetAsync(S.gfim, 0, S.nout * sizeof(float), st));
  CK(cudaMemsetAsync(S.status, 0, (size_t)S.nkf * sizeof(int32_t), st));
  CK(cudaMemsetAsync(ctx->d_um, 0, S.nu * sizeof(double2), st));
  CK(cudaMemsetAsync(ctx->d_dm, 0, S.nd * sizeof(double2), st));
  CK(cudaMemsetAsync(ctx->d_dets, 0, S.ndet * sizeof(double2), st));
  CK(cudaMemsetAsync(ctx->d_queue, 0, 4 * sizeof(unsigned int), st));
  CK(cudaMemsetAsync(ctx->d_stats, 0, 8 * sizeof(unsigned long long), st));
  if (ctx->d_steplog_n) CK(cudaMemsetAsync(ctx->d_steplog_n, 0, sizeof(unsigned long long), st));
  if (ctx->d_prof) CK(cudaMemsetAsync(ctx->d_prof, 0, 32 * sizeof(unsigned long long), st));
  if (timed) CK(cudaEventRecord(ctx->ev[2], st));
  auto launch = [&](int ph, const FKLaunch& LX, int g) {
    const int sc = ph >= 0 ? S.sched[ph] : 0;
    return S.fast ? gem_fast::launch_fk_phase(ph, sc, P, LX, g, st) : gem_plain::launch_fk_phase(ph, sc, P, LX, g, st);
  };
  CK(launch(-1, S.L, ctx->nsm * 8));
  if (ctx->dump_feat) {
    CK(prop_features_launch(S.PA, ctx->d_feat, st));
    ctx->feat_n = 3LL * S.nitems * PROP_NF;
  }
  if (S.propose) CK(prop_infer_launch(S.PA, ctx->d_propw, ctx->d_propnorm, ctx->d_prop_kopt, ctx->d_prop_hs, st));
  static const char* const phase_name[3] = {"gem_fk: toroidal phase", "gem_fk: spheroidal phase",
                                            "gem_fk: adjoint phase"};
  for (int ph = 0; ph < 3; ++ph) {
    nvtxRangePushA(phase_name[ph]);   // profiler range per phase launch (no cost without a tool)
    FKLaunch Lp = S.L;
    Lp.adv_min = FK_DEFER_MIN[S.defer[ph]];
    Lp.adv_wait = FK_DEFER_WAIT[S.defer[ph]];
    Lp.qgran = FK_GRAN[S.qgran[ph]];
    Lp.qchunk = FK_QCHUNK[S.qgran[ph]];
    if (ctx->d_prof) Lp.prof = ctx->d_prof + 8 * ph;
    if (ctx->d_warp_ns && ph == 1) Lp.warp_ns = ctx->d_warp_ns;
    const cudaError_t le = launch(ph, Lp, S.grid[ph]);
    nvtxRangePop();
    CK(le);
    if (timed) CK(cudaEventRecord(ctx->ev_ph[ph], st));
    // running counters after this phase (stream-ordered snapshot)
    CK(cudaMemcpyAsync(ctx->d_stats + 8 * (ph + 1), ctx->d_stats, 8 * sizeof(unsigned long long),
                       cudaMemcpyDeviceToDevice, st));
  }
  if (timed) CK(cudaEventRecord(ctx->ev[3], st));
  return GEM_OK;
}

// The device work of the ASKI program's FK spectra for a set of source nodes
// (computeGreenFKSpectraForASKI.f90:439-560): start radii; the toroidal phase
// once, with the minors over the node range jsl..jsr of the plan and the
// toroidal spectra of every source; the spheroidal minors once over the range;
// then per source node (the moment or force sources jsnod[b], then the force at
// jre) the adjoint phase with that node as the source.  Each source writes its
// own output block (block b at b * blk_m; the force block is blk_f long).
int fk_enqueue_aski(gem_ctx* ctx, SlabPlan& S, int nsnod, const int* jsnod, int jre, int istyp, float* gre,
                    float* gim, double* g64, size_t blk_m, size_t blk_f, cudaStream_t st) {
  CK(cudaMemsetAsync(ctx->d_spl, 0, S.spl_n * sizeof(double), st));
  CK(cudaMemsetAsync(ctx->d_err, 0, sizeof(int), st));
  CK(launch_prep(S.A, ctx->d_err, st));
  if (S.fast) CK(launch_poly(S.A, ctx->d_poly, st));
  const size_t ntot = blk_m * nsnod + blk_f;
  if (g64) CK(cudaMemsetAsync(g64, 0, ntot * 2 * sizeof(double), st));
  if (gre) CK(cudaMemsetAsync(gre, 0, ntot * sizeof(float), st));
  if (gim) CK(cudaMemsetAsync(gim, 0, ntot * sizeof(float), st));
  CK(cudaMemsetAsync(S.status, 0, (size_t)S.nkf * sizeof(int32_t), st));
  CK(cudaMemsetAsync(ctx->d_um, 0, S.nu * sizeof(double2), st));
  CK(cudaMemsetAsync(ctx->d_dm, 0, S.nd * sizeof(double2), st));
  CK(cudaMemsetAsync(ctx->d_dets, 0, S.ndet * sizeof(double2), st));
  CK(cudaMemsetAsync(ctx->d_queue, 0, 4 * sizeof(unsigned int), st));
  CK(cudaMemsetAsync(ctx->d_stats, 0, 32 * sizeof(unsigned long long), st));
  if (ctx->d_steplog_n) CK(cudaMemsetAsync(ctx->d_steplog_n, 0, sizeof(unsigned long long), st));
  if (ctx->d_prof) CK(cudaMemsetAsync(ctx->d_prof, 0, 32 * sizeof(unsigned long long), st));
  auto launch = [&](int ph, const FKStatic& PX, FKLaunch LX) {
    const int sc = ph >= 0 ? S.sched[ph] : 0;
    if (ph >= 0) {
      LX.adv_min = FK_DEFER_MIN[S.defer[ph]]; LX.adv_wait = FK_DEFER_WAIT[S.defer[ph]];
      LX.qgran = FK_GRAN[S.qgran[ph]];
      LX.qchunk = FK_QCHUNK[S.qgran[ph]];
    }
    const int g = ph >= 0 ? S.grid[ph] : ctx->nsm * 8;
    return S.fast ? gem_fast::launch_fk_phase(ph, sc, PX, LX, g, st) : gem_plain::launch_fk_phase(ph, sc, PX, LX, g, st);
  };
  FKLaunch L0 = S.L;
  L0.prop_kopt = nullptr; L0.prop_hs = nullptr;
  CK(launch(-1, S.P, L0));
  // source table of the toroidal phase, passed by value: nodes and types; block b
  // starts at b * blk_m
  const int nsrc = nsnod + 1;
  if (nsrc > MAXNOD + 2) return fail(ctx, "gem_fk_run_aski: %d source nodes, above the %d supported", nsnod, MAXNOD + 1);
  FKLaunch Lt = L0;
  Lt.gf64 = reinterpret_cast<double2*>(g64); Lt.gfre = gre; Lt.gfim = gim;
  Lt.nsrc = nsrc;
  Lt.src_blk = (long long)blk_m;
  for (int b = 0; b < nsrc; ++b) {
    Lt.src_node[b] = (unsigned char)(b == nsnod ? jre : jsnod[b]);
    Lt.src_type[b] = (unsigned char)(b == nsnod ? 0 : istyp);
  }
  nvtxRangePushA("gem_fk: toroidal phase over the source-node range");
  cudaError_t le = launch(0, S.P, Lt);
  nvtxRangePop();
  CK(le);
  nvtxRangePushA("gem_fk: spheroidal phase over the source-node range");
  le = launch(1, S.P, L0);
  nvtxRangePop();
  CK(le);
  for (int b = 0; b <= nsnod; ++b) {
    const bool force = b == nsnod;
    const int js = force ? jre : jsnod[b], ty = force ? 0 : istyp;
    FKStatic Pb = S.P;
    Pb.jre = js; Pb.istyp = ty;
    Pb.njsph = ty == 0 ? 2 : 4; Pb.njtor = ty == 0 ? 1 : 2;
    Pb.nsp = 4 * Pb.njsph + 2 * Pb.njtor;
    FKLaunch Lb = L0;
    const size_t off = (size_t)b * blk_m;
    Lb.gf64 = g64 ? reinterpret_cast<double2*>(g64) + off : nullptr;
    Lb.gfre = gre ? gre + off : nullptr;
    Lb.gfim = gim ? gim + off : nullptr;
    Lb.dets = reinterpret_cast<double2*>(ctx->d_dets) + (size_t)(js - S.P.jsl) * S.nkf;
    CK(cudaMemsetAsync(ctx->d_queue, 0, 4 * sizeof(unsigned int), st));
    CK(launch(2, Pb, Lb));
  }
  // totals only: the per-phase split is not recorded for a set of sources
  for (int ph = 0; ph < 3; ++ph)
    CK(cudaMemcpyAsync(ctx->d_stats + 8 * (ph + 1), ctx->d_stats, 8 * sizeof(unsigned long long),
                       cudaMemcpyDeviceToDevice, st));
  return GEM_OK;
}

// counters and times of the last slab (synchronises the stream)
int fk_finish(gem_ctx* ctx, const SlabPlan& S, cudaStream_t st, bool timed) {
  unsigned long long hs[32];
  int herr = 0;
  CK(cudaMemcpyAsync(hs, ctx->d_stats, 32 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(&herr, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if (herr) return fail(ctx, "Cubic spline interpolation not successful (code %d)", herr);
  float t_prep = 0, t_solve = 0, t0 = 0;
  if (timed) {
    cudaEventElapsedTime(&t_prep, ctx->ev[0], ctx->ev[1]);
    cudaEventElapsedTime(&t_solve, ctx->ev[2], ctx->ev[3]);
  }
  for (int ph = 0; ph < 3; ++ph) {
    float t = 0;
    if (timed) cudaEventElapsedTime(&t, ctx->ev[2], ctx->ev_ph[ph]);
    ctx->phase_ms[ph] = t - t0;
    ctx->stats.phase_ms[ph] = t - t0;
    ctx->stats.phase_flops[ph] = (int64_t)(hs[8 * (ph + 1) + 5] - (ph ? hs[8 * ph + 5] : 0ULL));
    t0 = t;
  }
  ctx->stats.steps_ok = hs[0]; ctx->stats.steps_rej = hs[1]; ctx->stats.attempts = hs[2];
  ctx->stats.sysmats = hs[3]; ctx->stats.matvecs = hs[4]; ctx->stats.flops = hs[5];
  ctx->stats.items = S.nitems; ctx->stats.failed = 0;
  ctx->stats.prep_ms = t_prep; ctx->stats.solve_ms = t_solve;
  return GEM_OK;
}

}  // namespace

extern "C" {

int gem_fk_run_device(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* d_gfre, float* d_gfim,
                      double* d_gf64, int32_t* d_status, void* stream) {
  if (!ctx) return GEM_ERROR;
  SlabPlan S;
  int rc = fk_prepare(ctx, p, jf_first, jf_last, d_gfre, d_gfim, d_gf64, d_status, S);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  rc = fk_enqueue(ctx, S, st, true);
  if (rc) return rc;
  return fk_finish(ctx, S, st, true);
}

// CUDA-graph form of gem_fk_run_device (no counterpart in the reference): the
// host-side preparation runs once here, the device work of the slab is captured
// into a graph that gem_fk_graph_launch replays.  The graph reads and writes
// the same device buffers as a direct run; any later run, graph build, model or
// node change on this context invalidates it.
int gem_fk_graph_build(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* d_gfre,
                       float* d_gfim, double* d_gf64, int32_t* d_status) {
  if (!ctx) return GEM_ERROR;
  if (ctx->graph_exec) { cudaGraphExecDestroy(ctx->graph_exec); ctx->graph_exec = nullptr; }
  SlabPlan S;
  int rc = fk_prepare(ctx, p, jf_first, jf_last, d_gfre, d_gfim, d_gf64, d_status, S);
  if (rc) return rc;
  if (!ctx->graph_stream) CK(cudaStreamCreateWithFlags(&ctx->graph_stream, cudaStreamNonBlocking));
  // run once directly: kernel attributes and lazily loaded modules are set up outside the capture
  rc = fk_enqueue(ctx, S, ctx->graph_stream, false);
  if (rc) return rc;
  CK(cudaStreamSynchronize(ctx->graph_stream));
  cudaGraph_t graph = nullptr;
  CK(cudaStreamBeginCapture(ctx->graph_stream, cudaStreamCaptureModeThreadLocal));
  rc = fk_enqueue(ctx, S, ctx->graph_stream, false);
  cudaError_t e = cudaStreamEndCapture(ctx->graph_stream, &graph);
  if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
  if (e != cudaSuccess) return fail(ctx, "graph capture: %s", cudaGetErrorString(e));
  e = cudaGraphInstantiate(&ctx->graph_exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) { ctx->graph_exec = nullptr; return fail(ctx, "graph instantiate: %s", cudaGetErrorString(e)); }
  ctx->graph_items = S.nitems;
  ctx->graph_valid = true;
  return GEM_OK;
}

// Replays the graph of gem_fk_graph_build on stream (asynchronous); the outputs
// and per-item status are complete when the stream reaches this point.
int gem_fk_graph_launch(gem_ctx* ctx, void* stream) {
  if (!ctx) return GEM_ERROR;
  if (!ctx->graph_exec || !ctx->graph_valid) return fail(ctx, "no valid FK graph (build it again)");
  CK(cudaSetDevice(ctx->device));
  CK(cudaGraphLaunch(ctx->graph_exec, (cudaStream_t)stream));
  return GEM_OK;
}

int gem_fk_run(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* gfre, float* gfim,
               double* gf64, int32_t* status) {
  if (!ctx) return GEM_ERROR;
  int rc = check_params(ctx, p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  Grid g;
  make_grid(p, ctx->rearth, g);
  if (jf_first < g.nf1 || jf_last > g.nf2 || jf_first > jf_last)
    return fail(ctx, "frequency range %d..%d outside %d..%d", jf_first, jf_last, g.nf1, g.nf2);
  long long nkf = 0;
  for (int jf = jf_first; jf <= jf_last; ++jf) nkf += g.nwn[jf];
  size_t nout = (size_t)nkf * nsp_run(ctx, p) * ctx->nnod;
  // device outputs: context-owned buffers (slots 8..11), grown on demand and
  // kept for the next call; the host buffers are the caller's (pinned ones copy
  // at full DMA rate)
  float* dre = gfre ? (float*)gem_ctx_aux(ctx, 8, nout * sizeof(float)) : nullptr;
  float* dim = gfim ? (float*)gem_ctx_aux(ctx, 9, nout * sizeof(float)) : nullptr;
  double* d64 = gf64 ? (double*)gem_ctx_aux(ctx, 10, nout * 2 * sizeof(double)) : nullptr;
  int32_t* dst = (int32_t*)gem_ctx_aux(ctx, 11, (size_t)nkf * sizeof(int32_t));
  if ((gfre && !dre) || (gfim && !dim) || (gf64 && !d64) || !dst) return GEM_ERROR;
  int ret = GEM_OK;
  cudaStream_t st = nullptr;
  ret = gem_fk_run_device(ctx, p, jf_first, jf_last, dre, dim, d64, dst, st);
  if (ret == GEM_OK) {
    std::vector<int32_t> hst((size_t)nkf);
    if ((gfre && cudaMemcpy(gfre, dre, nout * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (gfim && cudaMemcpy(gfim, dim, nout * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (gf64 && cudaMemcpy(gf64, d64, nout * 2 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        cudaMemcpy(hst.data(), dst, (size_t)nkf * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
      ret = fail(ctx, "copy of FK spectra to the host failed");
    } else {
      long long nfail = 0;
      for (auto v : hst) nfail += v != 0;
      ctx->stats.failed = nfail;
      if (status) memcpy(status, hst.data(), hst.size() * sizeof(int32_t));
      if (nfail) ret = fail(ctx, "%lld (omega,l) items failed; see the per-item status", nfail);
    }
  }
  return ret;
}

// DSV spectra with radial derivatives of one source node (the body of the
// source-node loop of computeGreenFKSpectraForASKI.f90:451-541): the same
// phase kernels as gem_fk_run with the source at node p->jre and output mode
// dsv, for the length of this call.
namespace {
struct DsvScope {
  gem_ctx* c;
  explicit DsvScope(gem_ctx* ctx) : c(ctx) { c->dsv = 1; }
  ~DsvScope() { c->dsv = 0; }
};
}  // namespace

int gem_fk_run_dsv(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* gfre, float* gfim,
                   double* gf64, int32_t* status) {
  if (!ctx) return GEM_ERROR;
  DsvScope scope(ctx);
  return gem_fk_run(ctx, p, jf_first, jf_last, gfre, gfim, gf64, status);
}

int gem_fk_run_dsv_device(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* d_gfre,
                          float* d_gfim, double* d_gf64, int32_t* d_status, void* stream) {
  if (!ctx) return GEM_ERROR;
  DsvScope scope(ctx);
  return gem_fk_run_device(ctx, p, jf_first, jf_last, d_gfre, d_gfim, d_gf64, d_status, stream);
}

// FK spectra of computeGreenFKSpectraForASKI for a set of source nodes: the
// minors once over the node range, then per source node the unit-jump Green
// functions and the DSV spectra with derivatives (see fk_enqueue_aski).
namespace {
struct AskiScope {
  gem_ctx* c;
  AskiScope(gem_ctx* ctx, int lo, int hi) : c(ctx) { c->dsv = 1; c->jsl = lo; c->jsr = hi; }
  ~AskiScope() { c->dsv = 0; c->jsl = 0; c->jsr = 0; }
};
}  // namespace

int gem_fk_aski_nsp(int istyp) { return istyp == 0 ? 10 : 20; }

int gem_fk_run_aski_device(gem_ctx* ctx, const gem_fk_params* p, int nsnod, const int* jsnod, int jf_first,
                           int jf_last, float* d_gfre, float* d_gfim, double* d_gf64, int32_t* d_status,
                           void* stream) {
  if (!ctx) return GEM_ERROR;
  if (!p) return fail(ctx, "null parameters");
  if (nsnod < 1 || !jsnod) return fail(ctx, "ASKI spectra: no source nodes");
  if (!ctx->have_nodes) return fail(ctx, "no external nodes set");
  int lo = ctx->nnod + 1, hi = 0;
  bool has_re = false;
  for (int i = 0; i < nsnod; ++i) {
    if (jsnod[i] < 1 || jsnod[i] > ctx->nnod) return fail(ctx, "ASKI spectra: source node %d out of range", jsnod[i]);
    lo = std::min(lo, jsnod[i]); hi = std::max(hi, jsnod[i]);
    has_re = has_re || jsnod[i] == p->jre;
  }
  if (!has_re) return fail(ctx, "receiver node must also be a source node");
  AskiScope scope(ctx, lo, hi);
  SlabPlan S;
  int rc = fk_prepare(ctx, p, jf_first, jf_last, nullptr, nullptr, nullptr, d_status, S);
  if (rc) return rc;
  const size_t blk_m = (size_t)S.nkf * gem_fk_aski_nsp(p->istyp) * ctx->nnod;
  const size_t blk_f = (size_t)S.nkf * gem_fk_aski_nsp(0) * ctx->nnod;
  cudaStream_t st = (cudaStream_t)stream;
  rc = fk_enqueue_aski(ctx, S, nsnod, jsnod, p->jre, p->istyp, d_gfre, d_gfim, d_gf64, blk_m, blk_f, st);
  if (rc) return rc;
  return fk_finish(ctx, S, st, false);
}

int gem_fk_run_aski(gem_ctx* ctx, const gem_fk_params* p, int nsnod, const int* jsnod, int jf_first, int jf_last,
                    float* gfre, float* gfim, double* gf64, int32_t* status) {
  if (!ctx) return GEM_ERROR;
  if (!p) return fail(ctx, "null parameters");
  if (!ctx->have_model) return fail(ctx, "no earth model loaded");
  if (!ctx->have_nodes) return fail(ctx, "no external nodes set");
  CK(cudaSetDevice(ctx->device));
  Grid g;
  make_grid(p, ctx->rearth, g);
  if (jf_first < g.nf1 || jf_last > g.nf2 || jf_first > jf_last)
    return fail(ctx, "frequency range %d..%d outside %d..%d", jf_first, jf_last, g.nf1, g.nf2);
  long long nkf = 0;
  for (int jf = jf_first; jf <= jf_last; ++jf) nkf += g.nwn[jf];
  if (nsnod < 1) return fail(ctx, "ASKI spectra: no source nodes");
  const size_t nout = (size_t)nkf * ctx->nnod * ((size_t)nsnod * gem_fk_aski_nsp(p->istyp) + gem_fk_aski_nsp(0));
  float* dre = gfre ? (float*)gem_ctx_aux(ctx, 8, nout * sizeof(float)) : nullptr;
  float* dim = gfim ? (float*)gem_ctx_aux(ctx, 9, nout * sizeof(float)) : nullptr;
  double* d64 = gf64 ? (double*)gem_ctx_aux(ctx, 10, nout * 2 * sizeof(double)) : nullptr;
  int32_t* dst = (int32_t*)gem_ctx_aux(ctx, 11, (size_t)nkf * sizeof(int32_t));
  if ((gfre && !dre) || (gfim && !dim) || (gf64 && !d64) || !dst) return GEM_ERROR;
  int ret = gem_fk_run_aski_device(ctx, p, nsnod, jsnod, jf_first, jf_last, dre, dim, d64, dst, nullptr);
  if (ret == GEM_OK) {
    std::vector<int32_t> hst((size_t)nkf);
    if ((gfre && cudaMemcpy(gfre, dre, nout * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (gfim && cudaMemcpy(gfim, dim, nout * sizeof(float), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        (gf64 && cudaMemcpy(gf64, d64, nout * 2 * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) ||
        cudaMemcpy(hst.data(), dst, (size_t)nkf * sizeof(int32_t), cudaMemcpyDeviceToHost) != cudaSuccess) {
      ret = fail(ctx, "copy of FK spectra to the host failed");
    } else {
      long long nfail = 0;
      for (auto v : hst) nfail += v != 0;
      ctx->stats.failed = nfail;
      if (status) memcpy(status, hst.data(), hst.size() * sizeof(int32_t));
      if (nfail) ret = fail(ctx, "%lld (omega,l) items failed; see the per-item status", nfail);
    }
  }
  return ret;
}

// Instrumentation of the solver (not part of the reference interface):
// enable = 1 allocates lockstep counters and per-warp timestamps for the
// following runs; gem_instrument_read copies them out.
int gem_instrument(gem_ctx* ctx, int enable) {
  if (!ctx) return GEM_ERROR;
  CK(cudaSetDevice(ctx->device));
  cudaFree(ctx->d_prof); cudaFree(ctx->d_warp_ns);
  ctx->d_prof = nullptr; ctx->d_warp_ns = nullptr;
  if (enable) {
    CK(cudaMalloc(&ctx->d_prof, 32 * sizeof(unsigned long long)));
    CK(cudaMalloc(&ctx->d_warp_ns, (size_t)2 * ctx->nsm * 64 * sizeof(unsigned long long)));
  }
  return GEM_OK;
}

int gem_instrument_read(gem_ctx* ctx, unsigned long long* prof8, unsigned long long* warp_ns, int* nwarps) {
  if (!ctx || !ctx->d_prof) return fail(ctx, "instrumentation not enabled");
  CK(cudaMemcpy(prof8, ctx->d_prof, 24 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  for (int ph = 0; ph < 3; ++ph) prof8[24 + ph] = (unsigned long long)(ctx->phase_ms[ph] * 1000.0);
  int nw = ctx->last_grid * (ctx->last_block / 32);   // the spheroidal phase's warps
  if (nwarps) *nwarps = nw;
  if (warp_ns) CK(cudaMemcpy(warp_ns, ctx->d_warp_ns, (size_t)2 * nw * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  return GEM_OK;
}

// Step log (instrumentation, no counterpart in the reference): capacity > 0
// makes the following runs record every Bulirsch-Stoer step attempt of every
// lane (StepRec, 32 bytes) up to capacity records; 0 switches it off.
int gem_steplog(gem_ctx* ctx, long long capacity) {
  if (!ctx) return GEM_ERROR;
  CK(cudaSetDevice(ctx->device));
  cudaFree(ctx->d_steplog); cudaFree(ctx->d_steplog_n);
  ctx->d_steplog = nullptr; ctx->d_steplog_n = nullptr; ctx->steplog_cap = 0;
  if (capacity > 0) {
    CK(cudaMalloc(&ctx->d_steplog, (size_t)capacity * sizeof(StepRec)));
    CK(cudaMalloc(&ctx->d_steplog_n, sizeof(unsigned long long)));
    CK(cudaMemset(ctx->d_steplog_n, 0, sizeof(unsigned long long)));
    ctx->steplog_cap = (unsigned long long)capacity;
  }
  return GEM_OK;
}

// Copies up to cap records of the last run into out (32 bytes each); *n = records
// the run produced (may exceed the capacity, then only the first were kept).
int gem_steplog_read(gem_ctx* ctx, void* out, long long cap, long long* n) {
  if (!ctx || !ctx->d_steplog) return fail(ctx, "step log not enabled");
  unsigned long long hn = 0;
  CK(cudaMemcpy(&hn, ctx->d_steplog_n, sizeof hn, cudaMemcpyDeviceToHost));
  if (n) *n = (long long)hn;
  unsigned long long m = std::min<unsigned long long>(hn, std::min<unsigned long long>(ctx->steplog_cap, (unsigned long long)cap));
  if (out && m) CK(cudaMemcpy(out, ctx->d_steplog, m * sizeof(StepRec), cudaMemcpyDeviceToHost));
  return GEM_OK;
}

// Learned proposer (no counterpart in the reference): w = PROP_NPARAM FP32
// weights (kept as FP16 on the device), norm = feature mean and deviation
// (2 * PROP_NF), use = PROP_USE_ORDER | PROP_USE_STEP, margin = least predicted
// log work saving that moves the order target off 6.  use = 0 or w = NULL
// switches it off.  Fast backend only.
int gem_proposer_set(gem_ctx* ctx, const float* w, const float* norm, int use, float margin) {
  if (!ctx) return GEM_ERROR;
  CK(cudaSetDevice(ctx->device));
  ctx->prop_use = 0;
  if (!w || use == 0) return GEM_OK;
  if (!norm) return fail(ctx, "proposer: feature normalisation missing");
  if (use & ~(PROP_USE_ORDER | PROP_USE_STEP)) return fail(ctx, "proposer: unknown use flags %d", use);
  if (!(margin >= 0.f)) return fail(ctx, "proposer: margin must be >= 0");
  for (int i = 0; i < PROP_NF; ++i)
    if (!(norm[PROP_NF + i] > 0.f)) return fail(ctx, "proposer: feature deviation must be positive");
  std::vector<__half> hw(PROP_NPARAM);
  for (int i = 0; i < PROP_NPARAM; ++i) {
    if (!std::isfinite(w[i])) return fail(ctx, "proposer: non-finite weight %d", i);
    hw[i] = __float2half_rn(w[i]);
  }
  if (!ctx->d_propw) CK(cudaMalloc(&ctx->d_propw, PROP_NPARAM * sizeof(__half)));
  if (!ctx->d_propnorm) CK(cudaMalloc(&ctx->d_propnorm, PROP_NNORM * sizeof(float)));
  CK(cudaMemcpy(ctx->d_propw, hw.data(), PROP_NPARAM * sizeof(__half), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(ctx->d_propnorm, norm, PROP_NNORM * sizeof(float), cudaMemcpyHostToDevice));
  ctx->prop_use = use;
  ctx->prop_margin = margin;
  return GEM_OK;
}

// Training data of the proposer: enable = 1 makes the following runs keep the
// raw features of every (phase, item), [3][nitems][PROP_NF].
int gem_proposer_dump(gem_ctx* ctx, int enable) {
  if (!ctx) return GEM_ERROR;
  ctx->dump_feat = enable != 0;
  ctx->feat_n = 0;
  return GEM_OK;
}

int gem_proposer_dump_read(gem_ctx* ctx, float* out, long long cap, long long* n) {
  if (!ctx || !ctx->d_feat) return fail(ctx, "proposer feature dump not enabled");
  if (n) *n = ctx->feat_n;
  const long long m = std::min(cap, ctx->feat_n);
  if (out && m > 0) CK(cudaMemcpy(out, ctx->d_feat, (size_t)m * sizeof(float), cudaMemcpyDeviceToHost));
  return GEM_OK;
}

// Solver schedules (no counterpart in the reference): per phase (toroidal,
// spheroidal, adjoint) an index into FK_SCHED_BLOCK / FK_SCHED_BIGCACHE, kept
// per backend.  Every schedule gives bit-identical spectra; only the time differs.
int gem_fk_schedule_set(gem_ctx* ctx, const int* sched3) {
  if (!ctx || !sched3) return GEM_ERROR;
  for (int ph = 0; ph < 3; ++ph)
    if (sched3[ph] < 0 || sched3[ph] >= FK_NSCHED) return fail(ctx, "schedule index must be 0..%d", FK_NSCHED - 1);
  const int b = ctx->backend == GEM_BACKEND_GPU_FAST ? 1 : 0;
  for (int ph = 0; ph < 3; ++ph) ctx->sched[b][ph] = sched3[ph];
  ctx->graph_valid = false;
  return GEM_OK;
}

int gem_fk_schedule_get(const gem_ctx* ctx, int* sched3) {
  if (!ctx || !sched3) return GEM_ERROR;
  const int b = ctx->backend == GEM_BACKEND_GPU_FAST ? 1 : 0;
  for (int ph = 0; ph < 3; ++ph) sched3[ph] = ctx->sched[b][ph];
  return GEM_OK;
}

// Bookkeeping deferral per phase (no counterpart in the reference): an index
// into FK_DEFER_MIN / FK_DEFER_WAIT, kept per backend; bit-identical spectra.
int gem_fk_defer_set(gem_ctx* ctx, const int* defer3) {
  if (!ctx || !defer3) return GEM_ERROR;
  for (int ph = 0; ph < 3; ++ph)
    if (defer3[ph] < 0 || defer3[ph] >= FK_NDEFER) return fail(ctx, "deferral index must be 0..%d", FK_NDEFER - 1);
  const int b = ctx->backend == GEM_BACKEND_GPU_FAST ? 1 : 0;
  for (int ph = 0; ph < 3; ++ph) ctx->defer[b][ph] = defer3[ph];
  ctx->graph_valid = false;
  return GEM_OK;
}

int gem_fk_defer_get(const gem_ctx* ctx, int* defer3) {
  if (!ctx || !defer3) return GEM_ERROR;
  const int b = ctx->backend == GEM_BACKEND_GPU_FAST ? 1 : 0;
  for (int ph = 0; ph < 3; ++ph) defer3[ph] = ctx->defer[b][ph];
  return GEM_OK;
}

// Queue granularity (no counterpart in the reference): per phase an index into
// FK_GRAN / FK_QCHUNK, the queue positions a lane or a block reserves per
// fetch, kept per backend.
int gem_fk_queue_set(gem_ctx* ctx, const int* gran3) {
  if (!ctx || !gran3) return GEM_ERROR;
  for (int ph = 0; ph < 3; ++ph)
    if (gran3[ph] < 0 || gran3[ph] >= FK_NGRAN) return fail(ctx, "queue granularity index must be 0..%d", FK_NGRAN - 1);
  const int b = ctx->backend == GEM_BACKEND_GPU_FAST ? 1 : 0;
  for (int ph = 0; ph < 3; ++ph) ctx->qgran[b][ph] = gran3[ph];
  ctx->graph_valid = false;
  return GEM_OK;
}

int gem_fk_queue_get(const gem_ctx* ctx, int* gran3) {
  if (!ctx || !gran3) return GEM_ERROR;
  const int b = ctx->backend == GEM_BACKEND_GPU_FAST ? 1 : 0;
  for (int ph = 0; ph < 3; ++ph) gran3[ph] = ctx->qgran[b][ph];
  return GEM_OK;
}

// Autotuner: runs frequencies jf_first..jf_last once per candidate (all three
// phases at once, repeats times, the minimum kept) and keeps per phase the
// fastest.  Stage 1 tries the schedules (block size, matrix caching) under the
// current deferral and queue granularity, stage 2 the deferrals under the
// chosen schedules, stage 3 the queue granularities under both.
// ms[c*3 + ph]: stage-1 times for c < GEM_FK_NSCHED, then the stage-2 and the
// stage-3 times; -1 for candidates not run (the plain build has no
// matrix-caching variants).
int gem_fk_autotune(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, int repeats, float* ms,
                    int* sched3, int* defer3) {
  if (!ctx) return GEM_ERROR;
  int rc = check_params(ctx, p);
  if (rc) return rc;
  CK(cudaSetDevice(ctx->device));
  Grid g;
  make_grid(p, ctx->rearth, g);
  if (jf_first < g.nf1 || jf_last > g.nf2 || jf_first > jf_last)
    return fail(ctx, "frequency range %d..%d outside %d..%d", jf_first, jf_last, g.nf1, g.nf2);
  long long nkf = 0;
  for (int jf = jf_first; jf <= jf_last; ++jf) nkf += g.nwn[jf];
  const size_t nout = (size_t)nkf * nsp_of(p) * ctx->nnod;
  float* dre = (float*)gem_ctx_aux(ctx, 8, nout * sizeof(float));
  float* dim = dre ? (float*)gem_ctx_aux(ctx, 9, nout * sizeof(float)) : nullptr;
  int32_t* dst = dim ? (int32_t*)gem_ctx_aux(ctx, 11, (size_t)nkf * sizeof(int32_t)) : nullptr;
  if (!dst) return GEM_ERROR;
  const int b = ctx->backend == GEM_BACKEND_GPU_FAST ? 1 : 0;
  const int saved_s[3] = {ctx->sched[b][0], ctx->sched[b][1], ctx->sched[b][2]};
  const int saved_d[3] = {ctx->defer[b][0], ctx->defer[b][1], ctx->defer[b][2]};
  const int saved_q[3] = {ctx->qgran[b][0], ctx->qgran[b][1], ctx->qgran[b][2]};
  float t[FK_NSCHED + FK_NDEFER + FK_NGRAN][3];
  for (auto& row : t)
    for (float& v : row) v = -1.0f;
  auto run = [&](float* tc) -> int {
    for (int r = 0; r < std::max(1, repeats); ++r) {
      SlabPlan S;
      int e = fk_prepare(ctx, p, jf_first, jf_last, dre, dim, nullptr, dst, S);
      if (!e) e = fk_enqueue(ctx, S, nullptr, true);
      if (!e) e = fk_finish(ctx, S, nullptr, true);
      if (e) return e;
      for (int ph = 0; ph < 3; ++ph)
        if (tc[ph] < 0.0f || ctx->phase_ms[ph] < tc[ph]) tc[ph] = ctx->phase_ms[ph];
    }
    return GEM_OK;
  };
  auto restore = [&]() {
    for (int ph = 0; ph < 3; ++ph) {
      ctx->sched[b][ph] = saved_s[ph]; ctx->defer[b][ph] = saved_d[ph]; ctx->qgran[b][ph] = saved_q[ph];
    }
  };
  auto argmin = [&](int c0, int n, int ph) {
    int best = c0;
    for (int c = c0 + 1; c < c0 + n; ++c)
      if (t[c][ph] < t[best][ph]) best = c;
    return best - c0;
  };
  // stage 1: schedules
  const int ncand = b ? FK_NSCHED : 3;
  for (int c = 0; c < ncand; ++c) {
    for (int ph = 0; ph < 3; ++ph) ctx->sched[b][ph] = c;
    if ((rc = run(t[c]))) { restore(); return rc; }
  }
  for (int ph = 0; ph < 3; ++ph) ctx->sched[b][ph] = argmin(0, ncand, ph);
  // stage 2: deferrals under the chosen schedules
  for (int c = 0; c < FK_NDEFER; ++c) {
    for (int ph = 0; ph < 3; ++ph) ctx->defer[b][ph] = c;
    if ((rc = run(t[FK_NSCHED + c]))) { restore(); return rc; }
  }
  for (int ph = 0; ph < 3; ++ph) ctx->defer[b][ph] = argmin(FK_NSCHED, FK_NDEFER, ph);
  // stage 3: queue granularities under the chosen schedules and deferrals
  for (int c = 0; c < FK_NGRAN; ++c) {
    for (int ph = 0; ph < 3; ++ph) ctx->qgran[b][ph] = c;
    if ((rc = run(t[FK_NSCHED + FK_NDEFER + c]))) { restore(); return rc; }
  }
  for (int ph = 0; ph < 3; ++ph) ctx->qgran[b][ph] = argmin(FK_NSCHED + FK_NDEFER, FK_NGRAN, ph);
  for (int ph = 0; ph < 3; ++ph) {
    if (sched3) sched3[ph] = ctx->sched[b][ph];
    if (defer3) defer3[ph] = ctx->defer[b][ph];
  }
  if (ms)
    for (int c = 0; c < FK_NSCHED + FK_NDEFER + FK_NGRAN; ++c)
      for (int ph = 0; ph < 3; ++ph) ms[c * 3 + ph] = t[c][ph];
  ctx->graph_valid = false;
  return GEM_OK;
}

// Travel-time table by ray tracing (computeTravelTimeTable.f90:160-226) on the
// context's model and nodes: model at the reference frequency, one GPU thread per
// turning radius.  Host outputs sized by ntp_cap; *ntp receives the count.
int gem_ray_table(gem_ctx* ctx, int stype, int attmode, double eps, double drtp, double rtmax, int ntp_cap,
                  int* ntp, double* rtp, double* slowness, float* table, int32_t* status) {
  if (!ctx) return GEM_ERROR;
  if (!ctx->have_model || !ctx->have_nodes) return fail(ctx, "travel times: load the model and the nodes first");
  if (stype != 0 && stype != 1) return fail(ctx, "travel times: ray type must be 0 (P) or 1 (S)");
  if (attmode < 0 || attmode > 3 || !(eps > 0) || !(drtp > 0)) return fail(ctx, "travel times: invalid parameters");
  if (!ntp || !rtp || !slowness || !table || !status) return fail(ctx, "travel times: null output");
  const int n = (int)((double)(int)(rtmax - ctx->roc) / drtp + 1.0);   // computeTravelTimeTable.f90:163
  *ntp = n;
  if (n < 1) return fail(ctx, "travel times: TURNING_NODES_RMAX below the core-mantle boundary");
  if (n > ntp_cap) return fail(ctx, "travel times: %d turning radii do not fit %d", n, ntp_cap);
  CK(cudaSetDevice(ctx->device));
  FKStatic P;
  memset(&P, 0, sizeof P);
  P.nlay = ctx->nlay; P.nk = ctx->nk; P.noc = ctx->noc; P.nic = ctx->nic; P.equidis = ctx->equidis;
  P.fsflag = ctx->fsflag; P.nnod = ctx->nnod;
  P.rearth = ctx->rearth; P.ric = ctx->ric; P.roc = ctx->roc; P.rhs = ctx->rb[1];
  for (int i = 1; i <= ctx->nlay; ++i) {
    P.rb[i] = ctx->rb[i]; P.drk[i] = ctx->drk[i]; P.iflso[i] = ctx->iflso[i]; P.iktop[i] = ctx->iktop[i];
  }
  for (int i = 1; i <= ctx->nk; ++i) P.rk[i] = ctx->rk[i];
  for (int i = 1; i <= ctx->nnod; ++i) { P.rnod[i] = ctx->rnod[i]; P.state[i] = ctx->state[i]; P.layer[i] = ctx->layer[i]; }
  // the model at the reference frequency: one slot with f = (2 - 1) * fref
  const int K1 = ctx->nk + 1;
  if (grow(ctx, ctx->d_spl, ctx->spl_cap, (size_t)K1 * SPL_STRIDE)) return GEM_ERROR;
  if (grow(ctx, ctx->d_slots, ctx->slots_cap, (size_t)2)) return GEM_ERROR;
  const int slots[2] = {2, 0};
  CK(cudaMemcpy(ctx->d_slots, slots, sizeof slots, cudaMemcpyHostToDevice));
  PrepArgs A;
  A.nslot = 1; A.nk = ctx->nk; A.nlay = ctx->nlay; A.attmode = attmode; A.df = ctx->fref; A.fref = ctx->fref;
  A.jf = ctx->d_slots;
  A.ro = ctx->d_knots; A.vpv = ctx->d_knots + K1; A.vph = ctx->d_knots + 2 * K1; A.vsv = ctx->d_knots + 3 * K1;
  A.vsh = ctx->d_knots + 4 * K1; A.eta = ctx->d_knots + 5 * K1; A.qkinv = ctx->d_knots + 6 * K1;
  A.qminv = ctx->d_knots + 7 * K1; A.rk = ctx->d_knots + 8 * K1;
  A.iktop = ctx->d_lay; A.ikbot = ctx->d_lay + (ctx->nlay + 1);
  A.spl = ctx->d_spl;
  CK(cudaMemset(ctx->d_err, 0, sizeof(int)));
  CK(launch_prep(A, ctx->d_err, nullptr));
  // outputs
  const size_t tb = (size_t)n * ctx->nnod * 2 * sizeof(float);
  char* d = nullptr;
  CK(cudaMalloc(&d, tb + (size_t)n * (2 * sizeof(double) + sizeof(int)) + 64));
  double* d_rtp = (double*)d;
  double* d_slow = d_rtp + n;
  int* d_st = (int*)(d_slow + n);
  float* d_tab = (float*)(((uintptr_t)(d_st + n) + 15) / 16 * 16);
  const double a0 = std::atan(std::sqrt(2.0 * eps));   // the start values of the ray (:204)
  cudaError_t e = gem_ray::launch_ray_table(P, ctx->d_spl, n, stype, eps, drtp, a0, d_rtp, d_slow, d_tab, d_st, nullptr);
  int herr = 0;
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = cudaMemcpy(&herr, ctx->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(rtp, d_rtp, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(slowness, d_slow, n * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(status, d_st, n * sizeof(int), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(table, d_tab, tb, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(ctx, "travel times: %s", cudaGetErrorString(e));
  if (herr) return fail(ctx, "Cubic spline interpolation not successful (code %d)", herr);
  for (int i = 0; i < n; ++i)
    if (status[i]) return fail(ctx, "travel times: the ray of turning radius %g failed (status %d)", rtp[i], status[i]);
  return GEM_OK;
}

// Order target of the step-size control (fast backend; no counterpart in the
// reference, which fixes it at 6, parametersBulirschStep.f90:28-48): k in 3..7;
// 0 restores 6.
int gem_order_target(gem_ctx* ctx, int k) {
  if (!ctx) return GEM_ERROR;
  if (k == 0) k = 6;
  if (k < 3 || k > 7) return fail(ctx, "order target must be 3..7");
  ctx->kopt = k;
  return GEM_OK;
}

int gem_tc_wait_limit(gem_ctx* ctx, long long ns) {
  if (!ctx) return GEM_ERROR;
  if (ns < 0) return fail(ctx, "wait limit must be >= 0");
  ctx->tc_wait_ns = (unsigned long long)ns;
  return GEM_OK;
}

int gem_stats_get(const gem_ctx* ctx, gem_stats* out) {
  if (!ctx || !out) return GEM_ERROR;
  *out = ctx->stats;
  return GEM_OK;
}

}  // extern "C"
