/*
 * plegma2pt — C ABI of the B200 hadron two-point contraction + momentum
 * projection library.
 *
 * One call replaces the reference's contraction path
 *   PLEGMA_Correlator<Float>::contract{Baryons,MesonsAll,MesonsNew,Mesons}
 *     -> contract_{baryons,mesons_all,mesons_new,mesons}        (lib/kernels)
 *     -> fourier_transform_3D inside the kernel, host block sum,
 *        MPI_Allreduce over the spatial communicator
 * and the generic projection PLEGMA_FT<Float>::apply.  Plain pointers and
 * sizes only; every entry point returns a p2_status and never exits.
 *
 * Data formats
 *  - Propagator (PLEGMA_Propagator storage, lib/PLEGMA_Propagator.cu:33-49,
 *    lib/kernels/PLEGMA_kernel_getSet.cuh:791-851): structure of arrays,
 *    component i = ((mu*4 + nu)*3 + c1)*3 + c2 (144 components) major, the
 *    site index x + Lx*(y + Ly*(z + Lz*j)) fastest, each element a complex
 *    (re, im) pair of double (P2_FP64) or float (P2_FP32).  j counts the
 *    stored time slices: slice j holds global time (t_first + j) mod Lt.
 *  - Momenta: integer triples n, p = 2*pi*n/L; the list of
 *    PLEGMA_FT::createMom (lib/PLEGMA_FT.cu:50-72) when built from Q^2_max.
 *  - Result of a request: for every contraction block in bit order below,
 *    [group][dataset][tau][mom][component] complex double, tau = 0..totalT-1
 *    the time measured from the source (the order in which the reference's
 *    HDF5 writer stores it, lib/PLEGMA_Correlator.cu:810-950).
 *    p2_block_info() gives each block's shape and offset.
 */
#ifndef PLEGMA2PT_H
#define PLEGMA2PT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define P2_ABI_VERSION 1

typedef enum {
  P2_OK = 0,
  P2_ERR_INVALID_ARG = 1,
  P2_ERR_OOM = 2,
  P2_ERR_CUDA = 3,
  P2_ERR_DEVICE_TIMEOUT = 4,
  P2_ERR_UNSUPPORTED = 5
} p2_status;

typedef enum { P2_FP64 = 0, P2_FP32 = 1 } p2_precision;

/* Arithmetic of a request.
 * P2_PLAIN_FP64: FP64 site contraction, FP64 direct phase sum.
 * P2_SPLIT_FP16: FP32 site contraction with power-of-two scaling per time
 *   slice; projection on the tensor cores as hi+lo FP16 products with FP32
 *   accumulation; FP64 cross-block sums and normalisation. */
typedef enum { P2_PLAIN_FP64 = 0, P2_SPLIT_FP16 = 1 } p2_mode;

typedef enum { P2_DEVICE = 0, P2_HOST = 1 } p2_location;

/* Contraction blocks, in their order in the result.
 *   groups x datasets x components per site                     reference
 *   NUCLEON_CG5   1 x 2 x 16  nucl_nucl: proton (u,u,d), neutron   PLEGMA_baryons_NtoN.cu:6-46
 *                 16 = (mu, mu') open spin, mu*4 + mu'
 *   NUCLEON_NTOR  1 x 2 x 16  nucl_nucl2: N = eps (u C g5 d) u at  PLEGMA_baryons_NtoR.cu:6-52
 *                 the sink, R = eps (u C d) g5 u at the source
 *   NUCLEON_RTON  1 x 2 x 16  nucl2_nucl                           PLEGMA_baryons_RtoN.cu:6-52
 *   NUCLEON_RTOR  1 x 2 x 16  nucl2_nucl2                          PLEGMA_baryons_RtoR.cu:6-46
 *   DELTA_ISO12   3 x 2 x 16  deltap_deltaz_kk, k = 1..3          PLEGMA_baryons_deltas.cu:7-59
 *   DELTA_ISO32   3 x 2 x 16  deltapp_deltamm_kk, k = 1..3        PLEGMA_baryons_deltas.cu:62-110
 *   MESON_G16     1 x 1 x 256 all (G_sink, G_src) pairs of the 16 PLEGMA_mesonsAll.cuh:52-76
 *                 structures, component g_sink*16 + g_src, G_sink u G_src d^dagger
 *   MESON_ALL34   1 x 1 x 34  contractMesonsAll subset              PLEGMA_mesonsAll.cuh:8-95
 *   MESON_NEW10   1 x 1 x 10  contractMesonsNew (u . d^dagger)      PLEGMA_mesonsNew.cuh:5-56
 *   MESON_DIAG10  1 x 2 x 10  contractMesons (u u^dag, d d^dag)     PLEGMA_mesons.cuh:10-65
 */
enum {
  P2_NUCLEON_CG5 = 1u << 0,
  P2_DELTA_ISO12 = 1u << 1,
  P2_DELTA_ISO32 = 1u << 2,
  P2_MESON_G16 = 1u << 3,
  P2_MESON_ALL34 = 1u << 4,
  P2_MESON_NEW10 = 1u << 5,
  P2_MESON_DIAG10 = 1u << 6,
  P2_NUCLEON_NTOR = 1u << 7,
  P2_NUCLEON_RTON = 1u << 8,
  P2_NUCLEON_RTOR = 1u << 9
};

typedef struct p2_ctx p2_ctx;

/* Lattice and process geometry; replaces PLEGMA_init's globals
 * (lib/PLEGMA.cu:19-212, include/global/PLEGMA_global_constants.h:64-110).
 * L is the global extent; procs/coords the process grid and this rank's
 * position in it (all 1 / 0 for one GPU).  device < 0 creates a host-only
 * context: argument checks, shapes and the host generator work, every
 * device entry point returns P2_ERR_UNSUPPORTED. */
typedef struct {
  int L[4];
  int procs[4];
  int coords[4];
  int device;
} p2_geom;

/* Pre-processing a contraction applies to a propagator while loading it, in
 * this order (the production driver applies the first and the last in place
 * before contracting, plegma/Calc_2pt.cpp:112-113):
 *   ROTATE_PLUS / ROTATE_MINUS  twisted-mass rotation to the physical basis,
 *     P'[mu][nu] = (P[mu][nu] - P[mu+2][nu+2] + s i (P[mu][nu+2] + P[mu+2][nu])) / 2
 *     with s = +1 / -1, indices mod 4 (PLEGMA_propagator_utils.cuh:97-126);
 *   GAMMA5    g5 P, P'[mu][nu] = P[mu+2][nu] (PLEGMA_propagator_utils.cuh:31-53);
 *   BOUNDARY  antiperiodic sign: P' = -P on global times t < boundary_t0
 *     (PLEGMA_propagator_utils.cuh:64-80). */
enum {
  P2_PROP_ROTATE_PLUS = 1u << 0,
  P2_PROP_ROTATE_MINUS = 1u << 1,
  P2_PROP_GAMMA5 = 1u << 2,
  P2_PROP_BOUNDARY = 1u << 3
};

/* Non-owning view of one propagator (PLEGMA_Propagator<Float>::D_elem()/H_elem()). */
typedef struct {
  const void* data;
  int precision; /* p2_precision */
  int location;  /* p2_location; host views are streamed through the device */
  int t_first;   /* global time of stored slice 0 */
  int nt;        /* stored slices (the local time extent for a full field) */
  unsigned transform; /* P2_PROP_* applied on load (0 = none) */
  int boundary_t0;    /* for P2_PROP_BOUNDARY */
} p2_prop;

/* One two-point request: one source, one time window, one contraction set. */
typedef struct {
  int source[4];       /* x, y, z, t (PLEGMA's `site`) */
  int totalT;          /* window from the source (PLEGMA_Correlator totalT) */
  const int* moms;     /* int[nmom][3]; NULL: build from q2max */
  int nmom;
  int q2max;
  unsigned contractions;
  int mode;            /* p2_mode */
  int prop_u, prop_d;  /* indices into the props array of the call */
  double* out;         /* result, layout in the file header */
  int out_location;    /* p2_location */
} p2_request;

/* Shape of one block of a request's result. */
typedef struct {
  unsigned bit;
  int groups, datasets, comps;
  size_t offset; /* in complex elements from the start of the result */
} p2_block;

/* ---- context ---------------------------------------------------------- */
/* Replaces PLEGMA_init's geometry setup for this path; the context owns the
 * stream-ordered workspaces, momentum tables and tuned launch shapes. */
p2_status p2_ctx_create(const p2_geom* geom, p2_ctx** ctx);
p2_status p2_ctx_destroy(p2_ctx* ctx);
/* Text of the last error on this context (never NULL). */
const char* p2_last_error(const p2_ctx* ctx);
/* Block until all work issued on the context's stream is done. */
p2_status p2_sync(p2_ctx* ctx);
/* Work is issued on `stream` (a cudaStream_t; NULL = the context's own). */
p2_status p2_set_stream(p2_ctx* ctx, void* stream);
/* Upper bound on the context's per-chunk position-space buffer (time slices
 * are contracted and projected in chunks that fit it; default min(8 GiB,
 * free/4)).  Smaller values cut memory and make more, shorter launches; the
 * result does not depend on it beyond rounding.  No counterpart in the
 * reference (it allocates per call, lib/kernels/PLEGMA_baryons.cuh:122). */
p2_status p2_set_workspace(p2_ctx* ctx, size_t bytes);

/* ---- shapes ----------------------------------------------------------- */
/* Components per site of a contraction set (sum over blocks of groups*datasets*comps). */
int p2_components(unsigned contractions);
/* Number of momenta with |n|^2 <= q2max; fills moms[n][3] in createMom order
 * when moms is not NULL (PLEGMA_FT::createMom, lib/PLEGMA_FT.cu:50-72). */
int p2_mom_list(int q2max, int* moms);
/* Block layout of a result: writes up to max_blocks entries, returns count;
 * *total gets the result size in complex elements for (totalT, nmom). */
int p2_block_info(unsigned contractions, int totalT, int nmom, p2_block* blocks, int max_blocks, size_t* total);

/* ---- the hot path ------------------------------------------------------ */
/* Contraction + projection of nreq requests over the given propagators.
 * Replaces contract_baryons / contract_mesons_all / contract_mesons_new /
 * contract_mesons (lib/kernels/PLEGMA_baryons.cuh:99-206,
 * PLEGMA_mesonsAll.cuh:98-192, PLEGMA_mesonsNew.cuh:63-157,
 * PLEGMA_mesons.cuh:68-165) including their host block sums and spatial
 * all-reduce (one GPU holds the full spatial volume).  Asynchronous on the
 * context's stream when all outputs are on the device; synchronous when a
 * result or a propagator lives on the host. */
p2_status p2_contract_project(p2_ctx* ctx, const p2_prop* props, int nprops, const p2_request* reqs, int nreq);

/* Position-space contraction (the reference's POSITION_SPACE correlator):
 * out[tau][k][x3] complex double, k over p2_components(contractions),
 * x3 the spatial site index; the request's moms/mode are ignored (FP64). */
p2_status p2_contract_position(p2_ctx* ctx, const p2_prop* props, int nprops, const p2_request* req);

/* Generic momentum projection of a field, PLEGMA_FT<Float>::apply with
 * FT_NAIVE/FT_GEMV (lib/PLEGMA_FT.cu:122-162): field SoA [dof][V3*nt]
 * complex double on the device, out [nt][dof][nmom] complex double
 * (host or device per out_location), phase exp(sign * i p.x) with the
 * origin at x = 0. */
p2_status p2_ft_apply(p2_ctx* ctx, const double* field, int dof, int nt, const int* moms, int nmom, int sign,
                      double* out, int out_location);

/* The same transform on the tensor cores (the split projection of the
 * contractions): each time slice of the field is scaled by 2^-e (e the binary
 * exponent of its largest entry, exact), converted to FP32 and projected with
 * hi+lo FP16 operands and FP32 accumulation; per (t, component, momentum) the
 * error is <= 1e-6 of sum_x |field(x, t)| of that component. */
p2_status p2_ft_apply_split(p2_ctx* ctx, const double* field, int dof, int nt, const int* moms, int nmom, int sign,
                            double* out, int out_location);

/* Allocation-free variant of p2_ft_apply (no counterpart in the reference).
 * For callers that cannot allocate device memory at call time, e.g. a host
 * framework that reserves all device memory for its own pool up front, or a
 * caller with a fixed device-memory budget: its scratch (momenta, phase
 * tables, partial sums) lives in a 32 MiB file-scope device array that every
 * GPU loading the library holds until exit; no cudaMalloc/cudaFree or other
 * allocating routine is called.  `out` is a device pointer ([nt][dof][nmom]
 * complex double).  Requests needing more than the scratch
 * (3*nmom*4 + 3*nmom*L*16 + nt*nmom*dof*16 bytes, each part rounded up to
 * 256) are rejected with P2_ERR_INVALID_ARG.  The first call on a device
 * looks up the array's address with that device current; make it before any
 * stream capture.  All calls share the array: calls that overlap on the GPU
 * race. */
p2_status p2_ft_apply_noalloc(p2_ctx* ctx, const double* field, int dof, int nt, const int* moms, int nmom,
                              int sign, double* out);

/* Copy a spinor field (12 complex components per site, SoA [mu][c1][site]
 * with mu 3 + c1 major, as the reference's PLEGMA_Vector / PLEGMA_Vector3D)
 * into column (nu, c2) of a device propagator field (layout as p2_prop, nt
 * slices from global time t_first), asynchronously on the context's stream:
 * PLEGMA_Propagator::absorb (lib/PLEGMA_Propagator.cu:33-95).
 * global_t < 0: the 4-D vector (same nt slices) is copied whole.
 * global_t >= 0: the column is zeroed and only global slice global_t, when it
 * lies in the view, is filled: from the same slice of a 4-D vector
 * (vec_3d = 0) or from a 3-D vector of V3 sites (vec_3d = 1).
 * global_t >= T is P2_ERR_INVALID_ARG (the reference aborts). */
p2_status p2_prop_absorb(p2_ctx* ctx, void* prop, const void* vec, int precision, int t_first, int nt, int nu, int c2,
                         int vec_3d, int global_t);

/* Apply P2_PROP_* transforms in place to a device propagator field (layout as
 * p2_prop, nt slices from global time t_first), asynchronously on the
 * context's stream: rotateToPhysicalBase_device / apply_gamma5 /
 * applyBoundaries_device of PLEGMA_Propagator (lib/PLEGMA_Propagator.cu,
 * lib/kernels/PLEGMA_propagator_utils.cuh:31-134).  Setting p2_prop::transform
 * instead applies them while contracting, without touching the field. */
p2_status p2_prop_transform(p2_ctx* ctx, void* data, int precision, int t_first, int nt, unsigned transform,
                            int boundary_t0);

/* Source-relative times tau of a request that this rank computes: the slices
 * of the window inside its time slab (p2_geom coords[3]) that both
 * propagator views hold.  Writes up to max of them into taus (may be NULL)
 * and returns their count, or -1 for an invalid request; works on host-only
 * contexts.  The reference's counterpart is the window bookkeeping of
 * PLEGMA_Correlator (startT/endT/localT, include/PLEGMA_Correlator.h:53-79). */
int p2_local_taus(p2_ctx* ctx, const p2_prop* props, int nprops, const p2_request* req, int* taus, int max);

/* ---- table-driven baryons (the reference's UDSC set) --------------------- */
/* contractBaryonsUDSC(propUP, propDN, propST, propCH, only_st, only_ch)
 * (lib/PLEGMA_Correlator.cu:137-189, lib/kernels/PLEGMA_baryons_udsc.cu:
 * 85-309): the octet and decuplet baryons of u, d, s, c quarks with the
 * projected interpolators of the reference's generated spin tables (e.g.
 * proton/Pp_Cg5_Cg5, DeltaPl/Pp_Cgi_Cgi, DeltaPlPl/Ppgigj_Cgi_Cgj).  The
 * flavour products run in the reference's order, skipping those that need a
 * propagator that is not given (index -1); only_st / only_ch keep only the
 * products containing s / c.  Result: [dataset][tau][mom] complex double,
 * datasets in the order of p2_udsc_datasets.  Device-resident propagators:
 * mode P2_PLAIN_FP64 (FP64 arithmetic, FP64 propagators) or P2_SPLIT_FP16
 * (FP32 contraction of power-of-two scaled inputs and the hi+lo FP16
 * tensor-core projection, FP64 or FP32 propagators, per-time-slice error
 * <= 1e-6 of sum_x |c_d(x,t)|). */
typedef struct {
  int source[4];
  int totalT;
  const int* moms; /* explicit momenta [nmom][3], or NULL for q2max */
  int nmom;
  int q2max;
  int prop_u, prop_d, prop_s, prop_c; /* indices into props, -1 = not given */
  int only_st, only_ch;
  double* out;
  int out_location;
  int mode; /* P2_PLAIN_FP64 or P2_SPLIT_FP16 */
} p2_udsc_request;

/* Dataset names ("proton/Pp_Cg5_Cg5", ...) a request produces, one per line,
 * into names (capacity cap, NUL-terminated; may be NULL); returns their count. */
int p2_udsc_datasets(const p2_udsc_request* req, char* names, size_t cap);
p2_status p2_contract_udsc(p2_ctx* ctx, const p2_prop* props, int nprops, const p2_udsc_request* req);

/* ---- CUDA graphs -------------------------------------------------------- */
/* The whole launch sequence of p2_contract_project(props, reqs) recorded once
 * and replayed with one cudaGraphLaunch: batched sources in one submission,
 * no per-call host work.  Creation runs the requests once eagerly (results
 * are written), then records them; the graph keeps its own workspaces, so
 * other calls on the context may run between replays.  Propagator and result
 * pointers are those given at creation: refill the propagator buffers in place
 * between launches.  Device-resident propagators and results only.  The
 * requests must form one batch (same form, contraction set, momentum list and
 * propagator precisions; any sources and windows): P2_ERR_UNSUPPORTED
 * otherwise, make one graph per batch.  Errors are reported on the parent
 * context.  No counterpart in the reference (it
 * launches each kernel from the host and synchronises after each,
 * lib/kernels/PLEGMA_baryons.cuh:134-164). */
typedef struct p2_graph p2_graph;
p2_status p2_graph_create(p2_ctx* ctx, const p2_prop* props, int nprops, const p2_request* reqs, int nreq,
                          p2_graph** graph);
/* Enqueue one replay on `stream` (a cudaStream_t; NULL = the context's stream). */
p2_status p2_graph_launch(p2_graph* graph, void* stream);
/* Wait for the last replay and check its device-side error flag. */
p2_status p2_graph_sync(p2_graph* graph);
p2_status p2_graph_destroy(p2_graph* graph);

/* ---- autotuning -------------------------------------------------------- */
/* With tuning on, the first call with a new shape times the candidate launch
 * shapes of the tunable kernels (tensor-core projection: N-tile width and
 * site splits; FP64 projection: component tile and site splits) and keeps the
 * fastest.  Choices are cached per (kernel, shape) for the context and its
 * graphs, and, when cache_path is not NULL, in that tab-separated file (read
 * now, rewritten after each new entry; "key<TAB>params<TAB>ms" per line).
 * Cached choices are used even with tuning off.  The reference's counterpart
 * is tuneAndRun with QUDA's tune cache (lib/kernels/PLEGMA_kernel_tuner.cuh). */
p2_status p2_tune_enable(p2_ctx* ctx, int on, const char* cache_path);
/* Entries in the context's tuning cache. */
int p2_tune_count(p2_ctx* ctx);

/* ---- memory ------------------------------------------------------------ */
/* Field storage for callers that do not link the CUDA runtime themselves
 * (PLEGMA_Field::create_device / create_host, lib/PLEGMA_Field.cu:226-235):
 * P2_DEVICE allocates device memory on the context's device, P2_HOST pinned
 * host memory.  p2_copy copies between any two of them and waits for it. */
p2_status p2_alloc(p2_ctx* ctx, size_t bytes, int location, void** ptr);
p2_status p2_free(p2_ctx* ctx, void* ptr, int location);
p2_status p2_copy(p2_ctx* ctx, void* dst, const void* src, size_t bytes);

/* ---- kernel timing ----------------------------------------------------- */
/* When enabled, every kernel the library launches is bracketed by CUDA
 * events on the launching stream; p2_profile_read() returns per-kernel
 * launch counts and summed device time (it synchronises the events). */
typedef struct {
  char name[48];
  long long launches;
  double ms;
} p2_kernel_time;
p2_status p2_profile_enable(p2_ctx* ctx, int on);
/* Fills up to max entries, returns the number of kernels seen; reset != 0 clears. */
int p2_profile_read(p2_ctx* ctx, p2_kernel_time* out, int max, int reset);

/* Test hook for the device-side failure path: the next tensor-core
 * projection launched on this context (split form, p2_ft_apply_split)
 * withholds its converters' operand-ready signals and gives every mbarrier
 * wait a short limit, so its waits run out; the kernel records the timeout,
 * waits for its own bulk copies, frees its TMEM and returns, and the next
 * p2_sync (or the synchronising call itself) reports P2_ERR_DEVICE_TIMEOUT.
 * The context stays usable.  Cleared by that launch.  Nothing faults or hangs:
 * every wait is bounded.  No counterpart in the reference (it aborts through
 * PLEGMA_error, include/global/PLEGMA_prints.hpp:49-81). */
p2_status p2_debug_wait_timeout(p2_ctx* ctx);

/* FP64 FMA rate of the context's device, the roofline denominator of the
 * plain form's FP64 kernels: an FMA loop (8 independent chains per thread,
 * 8 CTAs of 256 threads per SM) timed with CUDA events on the context's
 * stream, best of five launches after one warm-up.  *tflops = 2 x FMAs /
 * time; *ms (may be NULL) the launch time.  Synchronises the stream.  No
 * counterpart in the reference. */
p2_status p2_measure_fp64_rate(p2_ctx* ctx, double* tflops, double* ms);

/* ---- synthetic inputs (benchmarks and tests) --------------------------- */
/* Fill a propagator with entries Re, Im ~ N(0,1) scaled by exp(-a*|t - t0|),
 * drawn from a counter-based SplitMix64 + Box-Muller stream keyed by
 * (seed, flavour, global site, component).  `dst` is a device pointer
 * (on_device = 1, fast, device libm) or a host pointer (on_device = 0,
 * host libm, OpenMP).  Layout as p2_prop with the given t_first/nt. */
p2_status p2_synth_propagator(p2_ctx* ctx, void* dst, int on_device, int precision, uint64_t seed, int flavour,
                              int t0, double decay, int t_first, int nt);

#ifdef __cplusplus
}
#endif
#endif /* PLEGMA2PT_H */
