/*
 * gemini_fk.h -- C ABI of the B200 GEMINI frequency-wavenumber hot path.
 *
 * Plain C types only; every array is caller-owned.  FK spectra use the
 * reference's Fortran layout gf(iwn, isp, node), iwn fastest, i.e. element
 * (k, isp, n) of a slab of frequencies is at  k + nkf*(isp + nsp*n)  where k
 * runs over the wavenumbers of all frequencies of the slab
 * (computeGreenFKSpectraForSynthetics.f90:508-519, HDF5 dataset
 * (nkfmax, nsp, nnod)).
 *
 * Return codes follow the reference's error levels (errorMessage.f90:47):
 * 0 ok, 1 warning, 2 error.  The library never exits or aborts; the text of
 * the last error is available from gem_last_error.
 *
 * Per-item status codes (int32, one per wavenumber-frequency index k):
 *   0 ok, 1 step size below minimum (integrationStep.f90:176-180),
 *   2 maximum number of steps (integrationStep.f90:186),
 *   3 continued fraction did not converge (initialValues.f90:490-574),
 *   4 node/discontinuity bookkeeping (propagateOde.f90:177-186,319-324),
 *   5 non-finite value, 7 receiver or source in an ocean layer (unsupported).
 */
#ifndef GEMINI_FK_H
#define GEMINI_FK_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GEM_OK 0
#define GEM_WARNING 1
#define GEM_ERROR 2

#define GEM_BACKEND_GPU_FP64 1 /* FP64 solver in the reference's operation order (parity path) */
#define GEM_BACKEND_GPU_FAST 2 /* FP64 solver with FMA, division-free spline, reciprocal inverses */

typedef struct gem_ctx gem_ctx;

/* Node earth model: replaces createNodeEarthmodel (nodeEarthmodel.f90:98-257).
 * Arrays are the JSON file's columns: 1-based semantics, 0-based storage. */
typedef struct gem_model_desc {
  double fref, rearth, ric, roc;
  int aniflag, fsflag, equidis, nlay, nk, nic, noc;
  const int* iflso;    /* [nlay] 1 fluid, 0 solid */
  const int* iktop;    /* [nlay] 1-based knot index of each layer's top */
  const double* rb;    /* [nlay] radius of each layer's top (m) */
  const double* depth; /* [nk] knot depth (m) */
  const double* ro;    /* [nk] density */
  const double* vpv;
  const double* vph;
  const double* vsv;
  const double* vsh;
  const double* eta;
  const double* qk;    /* Q kappa */
  const double* qm;    /* Q mu */
} gem_model_desc;

/* Parfile keys of computeGreenFKSpectraForSynthetics on the hot path
 * (computeGreenFKSpectraForSynthetics.f90:89-94,186-236). */
typedef struct gem_fk_params {
  double tlen, fmax, fmin, p1lim, p2lim, frac, xlen, eps;
  int global_;     /* GLOBAL: 1 spherical harmonics, 0 wavenumbers */
  int attmode;     /* 0 ELASTIC 1 ATTENUATION_ONLY 2 DISPERSION_ONLY 3 ATTENUATION_AND_DISPERSION */
  int istyp;       /* 0 FORCE, 1 MOMENT */
  int stressflag;  /* STRESSFLAG */
  int jre;         /* receiver node, 1-based */
} gem_fk_params;

typedef struct gem_stats {
  int64_t steps_ok, steps_rej, attempts, sysmats, matvecs, flops;
  int64_t items, failed;
  double solve_ms; /* device time of the last solver launch */
  double prep_ms;  /* device time of the last model preparation */
  double synth_ms; /* device time of the last synthetics run */
  int64_t phase_flops[3]; /* FP64 flops of the toroidal, spheroidal and adjoint phase kernels */
  double phase_ms[3];     /* device time of each phase (the first includes the start-radius kernel) */
} gem_stats;

/* Synthetics parameters (computeSyntheticSeismograms.f90:136-240); df and
 * sigma are the values stored with the FK spectra (float32 in the reference's
 * file), the filter is EVENT_FILTER_TYPE = BUTTERWORTH_BANDPASS. */
typedef struct gem_synth_params {
  int nf1, nf2, nwnmax;   /* frequency range and largest number of degrees */
  long long nkfmax;       /* wavenumber-frequency extent of the FK spectra */
  int nsp;                /* spectra per node (10: U, V x 4 jumps, W x 2 jumps) */
  int istyp;              /* 1 MOMENT (sources: moment tensors [6]), 0 FORCE (forces [3]: Fr, Ft, Ff) */
  int global_;            /* 1: spherical harmonics (Legendre), 0: wavenumber integrals (Bessel) */
  double df, sigma;
  int nsamp;              /* power of two */
  double dt;              /* nsamp * dt * df = 1 */
  int velocity;           /* SEISMO_TYPE velocity (1) or displacement (0) */
  double tred;            /* reduction time */
  int order_highpass;
  double fc_highpass;
  int order_lowpass;
  double fc_lowpass;
  double dwn;             /* wavenumber spacing (regional mode; float32 in the reference's FK file) */
  double rearth;          /* earth radius of the FK file (regional mode; float32 there) */
} gem_synth_params;

/* Parameters of the synthetics for SPECFEM coupling
 * (computeSyntheticsForSpecfemCoupling.f90:136-250,376-453): the FK slab's
 * frequency range and extent as stored with the DSV spectra, the radius of the
 * boundary points' node, the event filter (BUTTERWORTH_BANDPASS specs), the
 * reduction time, the source's and the box centre's colatitude and longitude
 * (rad), and COMPUTE_SPECTRA. */
typedef struct gem_coupling_params {
  int nf1, nf2, nwnmax;
  long long nkfmax;
  int nsp;               /* >= 20: U, V, dU/dr, dV/dr x 4 jumps, W, dW/dr x 2 jumps */
  double df, sigma;
  double re;             /* radius of the node of the boundary points (m) */
  int nsamp;
  double dt, tred;
  int order_highpass;
  double fc_highpass;
  int order_lowpass;
  double fc_lowpass;
  double thetas, phis, thetac, phic;
  int spectra;           /* 1: unfiltered displacement and traction spectra instead of time series */
  int istyp;             /* 1 MOMENT (mt[6], nsp >= 20, 42 sums), 0 FORCE (mt[3] = Fr, Ft, Ff; nsp >= 10, 21 sums) */
} gem_coupling_params;

/* Context holding the model, nodes and device buffers of one GPU.
 * Replaces the module globals sec_* (splineEarthmodelCoefficients.f90:28-41);
 * one host thread per context. */
int gem_ctx_create(int device, int backend, gem_ctx** out);
void gem_ctx_destroy(gem_ctx* ctx);
const char* gem_last_error(const gem_ctx* ctx);

/* Earth model (createNodeEarthmodel, nodeEarthmodel.f90:98). */
int gem_model_load(gem_ctx* ctx, const gem_model_desc* model);

/* External radial nodes after splitting at discontinuities
 * (createExternalRadialNodes, externalRadialNodes.f90:82); radii ascending. */
int gem_nodes_set(gem_ctx* ctx, int nnod, const double* rnod, const int* state, const int* layer);

/* Frequency grid (computeGreenFKSpectraForSynthetics.f90:186-236): nf1, nf2,
 * nwnmax and nwn[jf-1] for jf = 1..nf2 (nwn_cap >= nf2); *nsp = spectra per node. */
int gem_fk_grid(gem_ctx* ctx, const gem_fk_params* p, int* nf1, int* nf2, int* nwnmax, int* nsp, int* nwn,
                int nwn_cap);

/* FK spectra of frequencies jf_first..jf_last (the wavenumber loop body
 * computeGreenFKSpectraForSynthetics.f90:410-501 for all l, all frequencies in
 * one launch).  Host buffers; any output pointer may be NULL.  Blocking.
 * gfre/gfim: float32, gf64: interleaved complex128, status: int32 per k. */
int gem_fk_run(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* gfre, float* gfim,
               double* gf64, int32_t* status);

/* Same with device buffers, ordered on `stream` (a cudaStream_t, may be NULL). */
int gem_fk_run_device(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* d_gfre,
                      float* d_gfim, double* d_gf64, int32_t* d_status, void* stream);

/* DSV spectra with radial derivatives for a source at node p->jre (type
 * p->istyp): replaces the body of the source-node loop of
 * computeGreenFKSpectraForASKI.f90:451-541 -- unit-jump Green functions of the
 * source node (unitJumpGreenFunctions.f90:62-380), gfsph = ujgf * zsph and
 * gftor = ujgf * ztor at every node (no reciprocity), and their radial
 * derivatives A(r) * gf (dsvDerivatives.f90:39-72, solidOdeSystem.f90:77-114,
 * toroidalOdeSystem.f90:81-102).  Spectra per node: U, V for each spheroidal
 * jump, then dU/dr, dV/dr, then W, dW/dr for each toroidal jump, i.e.
 * nsp = 4*njsph + 2*njtor (20 for a moment, 10 for a force); p->stressflag is
 * ignored.  Every node must be solid.  The ASKI program's set of source nodes
 * (SOURCE_NODE_RADII) plus the force at the receiver is one call per source
 * node.  Layout, buffers and return codes as gem_fk_run / gem_fk_run_device. */
int gem_fk_run_dsv(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* gfre, float* gfim,
                   double* gf64, int32_t* status);
int gem_fk_run_dsv_device(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* d_gfre,
                          float* d_gfim, double* d_gf64, int32_t* d_status, void* stream);

/* All FK spectra of computeGreenFKSpectraForASKI for frequencies
 * jf_first..jf_last in one call (the wavenumber loop :439-560 for the whole
 * slab): minors once over the node range min(jsnod)..max(jsnod)
 * (toroidalMinors.f90:71-268, spheroidalMinors.f90:72-585, as the program
 * calls them at :444-447), then for each source node jsnod[0..nsnod-1] (type
 * p->istyp) and for a force at the receiver node p->jre, which must be among
 * jsnod (:206-209), the DSV spectra of gem_fk_run_dsv.  The outputs hold
 * nsnod + 1 blocks, block b at offset b * nkf * gem_fk_aski_nsp(p->istyp) *
 * nnod (the force block last, gem_fk_aski_nsp(0) spectra per node), each in
 * the (nkf, nsp, nnod) layout of the program's file <DSVBASENAME>.<type>.<b+1>.
 * Every node must be solid. */
int gem_fk_aski_nsp(int istyp);
int gem_fk_run_aski(gem_ctx* ctx, const gem_fk_params* p, int nsnod, const int* jsnod, int jf_first, int jf_last,
                    float* gfre, float* gfim, double* gf64, int32_t* status);
int gem_fk_run_aski_device(gem_ctx* ctx, const gem_fk_params* p, int nsnod, const int* jsnod, int jf_first,
                           int jf_last, float* d_gfre, float* d_gfim, double* d_gf64, int32_t* d_status,
                           void* stream);

/* Synthetics for SPECFEM coupling of a moment or force source at npts boundary
 * points of one node: replaces computeSynthetics and computeTension of
 * computeSyntheticsForSpecfemCoupling.f90:677-793 in the loops :509-549 and
 * :571-590.  Per point and frequency: the 42 (moment) or 21 (force) degree sums
 * of the DSV spectra with derivatives (harmonicDegreeSums.f90:95-369),
 * displacement and its r, theta
 * and phi derivatives, strain and stress (singleFrequencyDisplacement.f90:
 * 108-262), rotation to the box frame (axesRotation.f90), traction = stress *
 * nrm, then either the unfiltered spectra (p->spectra) or velocity and traction
 * through the event filter and the time shift, inverse-transformed
 * (frequencyTime.f90:55-113).  gr/gi: float32 spectra (nkfmax, nsp) of the
 * points' node; nwn[nf2]; zelcon[nf2*7] the node's complex elastic constants per
 * frequency (interleaved, getComplexConstantsSelectedExternalRadialNodes);
 * mt[6]; delta, xi[npts] epicentral distance and azimuth (rad); nrm[npts*3] box
 * normals.  Output per point: velocity x, y, z then traction x, y, z, as
 * spec[(p*6 + c)*nf2 + jf-1] (complex) or traces[(p*6 + c)*nsamp + i]. */
int gem_coupling_run(gem_ctx* ctx, const gem_coupling_params* p, const int* nwn, const float* gr, const float* gi,
                     const double* zelcon, const double* mt, int npts, const double* delta, const double* xi,
                     const double* nrm, double* spec, float* traces);
/* Same with the spectra and the outputs on the device, ordered on `stream`;
 * nwn, zelcon, mt and the point arrays are host arrays. */
int gem_coupling_run_device(gem_ctx* ctx, const gem_coupling_params* p, const int* nwn, const float* d_gr,
                            const float* d_gi, const double* zelcon, const double* mt, int npts, const double* delta,
                            const double* xi, const double* nrm, double* d_spec, float* d_traces, void* stream);

/* CUDA-graph form of gem_fk_run_device (no counterpart in the reference).
 * gem_fk_graph_build does the host-side preparation of the slab once (item and
 * queue tables, buffers) and captures its device work (zeroing, model
 * preparation, start radii, phase kernels) into a graph on the context;
 * gem_fk_graph_launch replays it on a stream, asynchronously, writing the
 * device outputs given at build time.  Any later run, graph build, model or
 * node change on the context invalidates the graph (launch then fails). */
int gem_fk_graph_build(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, float* d_gfre,
                       float* d_gfim, double* d_gf64, int32_t* d_status);
int gem_fk_graph_launch(gem_ctx* ctx, void* stream);

/* Solver schedules and their autotuner (no counterpart in the reference; the
 * reference runs one solve at a time).  Each phase kernel (toroidal,
 * spheroidal, adjoint) runs one block per SM under one of GEM_FK_NSCHED
 * schedules: threads per block (384, 512, 256, 384, 512, 256) and, for
 * schedules 3..5, the 4- and 5-variable systems of the fast backend keep their
 * half- and end-step matrices across the attempts of a Bulirsch-Stoer step.
 * Every schedule gives bit-identical spectra.  sched3[ph] is kept per context
 * and backend; the default is {1, 0, 1}. */
#define GEM_FK_NSCHED 6
int gem_fk_schedule_set(gem_ctx* ctx, const int* sched3);
int gem_fk_schedule_get(const gem_ctx* ctx, int* sched3);
/* Deferral of the bookkeeping between integrations, per phase: a lane that
 * ends an integration sub-interval waits until (1, 8, 16, 32, 32, 32) lanes of
 * its warp wait, it has waited (0, 6, 10, 24, 48, 1000000) steps, or no lane of
 * the warp integrates, so that the divergent bookkeeping runs for many lanes at
 * once.  Index 0..GEM_FK_NDEFER-1, kept per context and backend, default 4;
 * bit-identical spectra. */
#define GEM_FK_NDEFER 6
int gem_fk_defer_set(gem_ctx* ctx, const int* defer3);
int gem_fk_defer_get(const gem_ctx* ctx, int* defer3);
/* Queue granularity of each phase (no counterpart in the reference): a lane
 * that fetches work reserves (1, 2, 4) consecutive positions of the phase's
 * work queue and takes the next of them without the queue until they are used
 * up (indices 0..2), or the warps of a block share runs of 1024 consecutive
 * positions (index 3).  Index 0..GEM_FK_NGRAN-1, kept per context and backend,
 * default 0; bit-identical spectra. */
#define GEM_FK_NGRAN 4
int gem_fk_queue_set(gem_ctx* ctx, const int* gran3);
int gem_fk_queue_get(const gem_ctx* ctx, int* gran3);
/* Autotuner: runs frequencies jf_first..jf_last once per candidate (repeats
 * times, minimum kept), first the schedules, then the deferrals under the
 * chosen schedules, then the queue granularities under both, and keeps per
 * phase the fastest of each.  ms (may be NULL,
 * (GEM_FK_NSCHED + GEM_FK_NDEFER + GEM_FK_NGRAN) * 3 floats) receives the phase
 * times in ms of every candidate, -1 for candidates not run (the plain backend
 * tries schedules 0..2 only); sched3 and defer3 (may be NULL) the choice, and
 * gem_fk_queue_get the chosen granularities. */
int gem_fk_autotune(gem_ctx* ctx, const gem_fk_params* p, int jf_first, int jf_last, int repeats, float* ms,
                    int* sched3, int* defer3);

/* Synthetic seismograms of all stations and moment tensors of one source
 * node: replaces, for every station, computeLegendreFunctions +
 * sphericalHarmonicsDisplacementSpectra (displacementSpectra.f90:49) + event
 * filter + ZNE rotation + transformFrequencyTime (frequencyTime.f90:55)
 * (computeSyntheticSeismograms.f90:311-388).  gfkr/gfki: float32 FK spectra
 * of the node in the file layout (nkfmax, nsp); nwn[jf-1] for jf = 1..nf2;
 * theta = epicentral distance (rad), phi = azimuth at the source, propdir =
 * propagation direction at the receiver (rad); for p->istyp 1 mt[nmt][6] =
 * (Mrr, Mtt, Mff, Mrt, Mrf, Mtf) and the 10 moment spectra (nsp >= 10), for
 * p->istyp 0 mt[nmt][3] = (Fr, Ft, Ff) and the 5 force spectra (nsp >= 5;
 * forceHarmonicDegreeSums, forceSingleFrequencyDisplacement).
 * traces[((sta*nmt + imt)*3 + comp)*nsamp + i], comp Z, N, E.
 * Host buffers, blocking. */
int gem_synth_run(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* gfkr, const float* gfki,
                  int nsta, const double* theta, const double* phi, const double* propdir, int nmt,
                  const double* mt, float* traces);

/* Same with the FK spectra and the traces in device memory. */
int gem_synth_run_device(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* d_gfkr,
                         const float* d_gfki, int nsta, const double* theta, const double* phi,
                         const double* propdir, int nmt, const double* mt, float* d_traces, void* stream);

/* Per-station options of the reference's station loop
 * (computeSyntheticSeismograms.f90:344-397); host arrays, any member may be NULL / 0:
 *   tred        [nsta] reduction time of each station (s), as getTravelTimes - TIME_SHIFT_BUFFER
 *               gives it with AUTOMATIC_TIMESHIFT; NULL: p->tred for all stations;
 *   nsamp_true  [nsta] samples kept per station (1..nsamp, the reference's nstrue); the
 *               samples after them are written as 0; NULL: all nsamp;
 *   stafilter   [nsta][3][nf2] complex interleaved station filter (the reference's
 *               stafilter(nf2, 3, nstat)), applied per component before the ZNE rotation;
 *               NULL: the unit filter;
 *   nstf, tanf_stf, stf  source wavelet of nstf <= 8192 float32 samples, the first at time
 *               tanf_stf (s); convolveWithSourceWavelet (:463-484) after the inverse FFT.
 * The options need nsamp <= 8192. */
typedef struct gem_synth_station_opts {
  const double* tred;
  const int* nsamp_true;
  const double* stafilter;
  int nstf;
  double tanf_stf;
  const float* stf;
} gem_synth_station_opts;
int gem_synth_run_opts(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* gfkr, const float* gfki,
                       int nsta, const double* theta, const double* phi, const double* propdir, int nmt,
                       const double* mt, const gem_synth_station_opts* opts, float* traces);
int gem_synth_run_device_opts(gem_ctx* ctx, const gem_synth_params* p, const int* nwn, const float* d_gfkr,
                              const float* d_gfki, int nsta, const double* theta, const double* phi,
                              const double* propdir, int nmt, const double* mt,
                              const gem_synth_station_opts* opts, float* d_traces, void* stream);

/* Travel-time table by ray tracing: replaces computeTravelTimeTable
 * (computeTravelTimeTable.f90:160-226) on the context's model and nodes.  stype 0
 * P, 1 S; the model at its reference frequency under attmode; eps the accuracy
 * (ACCURACY), drtp and rtmax the spacing and the largest turning radius
 * (TURNING_NODES_DR, TURNING_NODES_RMAX, m).  ntp = int(rtmax - roc)/drtp + 1 turning
 * radii rtp[i] = roc + i*drtp with slowness[i] = rtp/v(rtp) (s/rad), and
 * table[(i*nnod + j)*2 + {0,1}] = (Delta (rad), T (s)) of ray i at node j (0 where
 * the ray does not reach): the reference's rayTable(2, nnod, ntp).  One GPU thread
 * per ray; *ntp is set before the size check against ntp_cap. */
int gem_ray_table(gem_ctx* ctx, int stype, int attmode, double eps, double drtp, double rtmax, int ntp_cap,
                  int* ntp, double* rtp, double* slowness, float* table, int32_t* status);

/* Travel times from such a table as the reference reads it back (float32 radii,
 * slownesses and table; getTravelTimes, travelTimes.f90:105-260): source radius rs,
 * receivers at radii re[s] and epicentral distances delta[s] (rad) -> tt[s] (s).
 * istele 1 for a TELE table (turning points in the lower mantle), 0 LOCAL.  The
 * reduction time of AUTOMATIC_TIMESHIFT is tt - TIME_SHIFT_BUFFER
 * (computeSyntheticSeismograms.f90:344-350); pass it in gem_synth_station_opts. */
int gem_travel_times(gem_ctx* ctx, int nnod, int ntp, const float* rnod, const float* rtp, const float* slowness,
                     const float* table, int istele, double rs, int n, const double* re, const double* delta,
                     double* tt);

/* Batched transformFrequencyTime (frequencyTime.f90:55-113): ntr complex
 * spectra to ntr float32 time series.  Spectrum t is interleaved complex128
 * at sp + 2*t*ldsp; element j (0-based) is frequency j*df; elements
 * nf1-1..nf2-1 are read (ldsp >= nf2), the others are taken as zero.  Series t
 * is written to ts + t*nsamp.  The FFT length is the reference's (nsamp, or
 * the next power of two above 2*nf2 followed by decimation to dt, which
 * returns GEM_WARNING as the reference does); at most 8192.
 * ts(i) = Re(FFT(+1) of the Hermitian-completed spectrum)(ndec*(i-1)+1)
 *         * df * exp(sigma*dts)^(i-1).
 * Host buffers, blocking. */
int gem_ifft_run(gem_ctx* ctx, int nf1, int nf2, double df, double sigma, int ntr, const double* sp,
                 long long ldsp, int nsamp, double dt, float* ts);

/* Same with sp and ts in device memory, ordered on stream. */
int gem_ifft_run_device(gem_ctx* ctx, int nf1, int nf2, double df, double sigma, int ntr, const double* d_sp,
                        long long ldsp, int nsamp, double dt, float* d_ts, void* stream);

/* gem_ifft_run_noalloc -- no counterpart in the reference.  The transform of
 * gem_ifft_run_device for callers that cannot allocate device memory when they
 * call it: codes whose device memory is already handed out by their own pool
 * allocator, or that must not let cudaMalloc/cudaFree synchronise the device
 * while other streams run.  It takes no context and allocates nothing (no
 * cudaMalloc, no cudaFree, no host heap); its tables live in one static 256 KiB
 * device array that every GPU loading this library holds until exit.  Same
 * arguments and limits as gem_ifft_run_device (FFT length <= 8192; larger sizes
 * are rejected with GEM_ERROR and a message); the device is the caller's
 * current one; errors and the decimation warning are written to errbuf
 * (errlen bytes, may be NULL).  Returns after queuing its kernels on stream.
 * All calls on a device share the array: calls that overlap on the GPU race and
 * must be ordered on one stream.  Every call looks up the array's address in
 * the current context (cudaGetSymbolAddress, no allocation), so it stays valid
 * after cudaDeviceReset; the first call on each device may load the library's
 * device code and should come before any stream capture. */
int gem_ifft_run_noalloc(int nf1, int nf2, double df, double sigma, int ntr, const double* d_sp, long long ldsp,
                         int nsamp, double dt, float* d_ts, void* stream, char* errbuf, int errlen);

/* Failure-detection knob (no counterpart in the reference): the time limit, in
 * ns, of each pipeline wait of the tensor-core degree sums of this context
 * (fast backend); 0 restores the default of 1 s.  A wait that runs out makes
 * the kernel stop issuing work, drain its own copies and products (bounded by
 * 1 s whatever the limit), free its tensor memory and return; the synthetics
 * call then returns GEM_ERROR with "a pipeline wait timed out".  A limit far
 * below the pipeline's latency (a few ns) makes every call fail that way. */
int gem_tc_wait_limit(gem_ctx* ctx, long long ns);

/* Counters of the last run (accepted/rejected steps, attempts, flops, ...). */
int gem_stats_get(const gem_ctx* ctx, gem_stats* out);

/* Instrumentation (no counterpart in the reference): enable = 1 makes the
 * following runs record, per phase ph = 0 toroidal, 1 spheroidal, 2 adjoint,
 * lockstep counters prof[8*ph + 0..3] = {warp trips, integrating lanes summed
 * over trips, attempt iterations, lanes computing an attempt summed over
 * iterations}, phase times prof[24 + ph] in microseconds (prof holds 32
 * entries), and per-warp (start, end) timestamps in ns of the spheroidal phase. */
int gem_instrument(gem_ctx* ctx, int enable);
int gem_instrument_read(gem_ctx* ctx, unsigned long long* prof8, unsigned long long* warp_ns, int* nwarps);

/* Step log (instrumentation, no counterpart in the reference): capacity > 0
 * makes the following FK runs record every Bulirsch-Stoer step attempt (32-byte
 * records: double x, double h, int32 item, float log10|y|, int16 layer, int8
 * system, int8 converged attempt or 0 when rejected, int16 phase, int16 step
 * number) up to capacity records; 0 switches it off.  gem_steplog_read copies
 * up to cap records of the last run and returns the number produced in *n. */
int gem_steplog(gem_ctx* ctx, long long capacity);
int gem_steplog_read(gem_ctx* ctx, void* out, long long cap, long long* n);

/* Order target of the step-size control (fast backend; no counterpart in the
 * reference, which fixes it at 6, parametersBulirschStep.f90:28-48): the step
 * grows when a step converges before attempt k and shrinks when after; k in
 * 3..7, 0 restores 6.  Acceptance and rejection are unchanged. */
int gem_order_target(gem_ctx* ctx, int k);

/* Learned step/order proposer (no counterpart in the reference).  A 3-layer
 * MLP of width 64 maps 11 features of each (item, phase) to the predicted work
 * with the step-size control aiming at attempt 5 and 7 (relative to 6) and to
 * a factor for the initial steps of the initial-value formulas; the fast
 * backend sets each lane's order target (use & GEM_PROP_USE_ORDER; 5 or 7
 * only when the predicted log saving exceeds margin) and initial steps (use &
 * GEM_PROP_USE_STEP) from it.  The error control still accepts or rejects
 * every step.  w: GEM_PROP_NPARAM FP32 weights (W1 [64][11], b1, W2 [64][64],
 * b2, W3 [3][64], b3), used as FP16; norm: feature mean [11] then deviation
 * [11].  use = 0 or w = NULL switches it off. */
#define GEM_PROP_NF 11
#define GEM_PROP_NPARAM 5123
#define GEM_PROP_USE_ORDER 1
#define GEM_PROP_USE_STEP 2
int gem_proposer_set(gem_ctx* ctx, const float* w, const float* norm, int use, float margin);
/* Training data: enable = 1 makes the following runs keep the raw features of
 * every (phase, item), [3][nitems][11]; read them with gem_proposer_dump_read. */
int gem_proposer_dump(gem_ctx* ctx, int enable);
int gem_proposer_dump_read(gem_ctx* ctx, float* out, long long cap, long long* n);
/* Training kernels of the proposer: gradient of the masked mean-squared error
 * on n standardised samples (x [n][11], y and mask [n][3], host buffers), and
 * Adam training in place of the FP32 weights (epochs over n samples in batches,
 * order from seed; loss_hist[epochs] may be NULL).  They allocate their own
 * device buffers on the current device. */
int gem_prop_grad(const float* w, const float* x, const float* y, const float* mask, int n, float* grad, float* loss);
int gem_prop_train(float* w, const float* x, const float* y, const float* mask, int n, int epochs, int batch,
                   float lr, unsigned seed, float* loss_hist);

#ifdef __cplusplus
}
#endif
#endif /* GEMINI_FK_H */
