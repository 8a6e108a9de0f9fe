/*
 * fr_b200.h - C ABI of the B200 Flux Reconstruction residual / RK-update path.
 *
 * The library (flurrypp_b200/libfr_b200.so) replaces the explicit FR residual
 * and Runge-Kutta update of FlurryPP's `solver` class with CUDA kernels for
 * sm_100a.  One `fr_case` is one reference `solver` (one mesh, one order)
 * together with the `input` options that drive it.  State arrays keep the
 * reference layout [point][element][field] (last index fastest,
 * include/matrix.hpp:52-116), so a host buffer filled for the reference's
 * U_spts can be passed here unchanged.
 *
 * Conventions
 *   - every entry point returns an int status (FR_OK == 0); none calls exit();
 *     fr_last_error() gives the message of the last failure on a case;
 *   - host pointers are plain C arrays of the stated size; the library copies
 *     them to and from device memory it owns;
 *   - one case is used by one host thread at a time; kernels run on the
 *     case's CUDA stream (fr_set_stream), the host calls that return results
 *     synchronise that stream.
 */
#ifndef FR_B200_H
#define FR_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  FR_OK = 0,
  FR_ERR_ARG = 1,         /* bad argument or size */
  FR_ERR_SETUP = 2,       /* mesh / connectivity / metric failure (reference: FatalError) */
  FR_ERR_CUDA = 3,        /* CUDA runtime error */
  FR_ERR_NONFINITE = 4,   /* NaN/Inf or non-positive density in the state */
  FR_ERR_BUDGET = 5,      /* device-memory budget exceeded (server admission) */
  FR_ERR_TIMEOUT = 6,     /* a bounded wait ran out */
  FR_ERR_UNSUPPORTED = 7, /* option outside the B200 path */
  FR_ERR_STATE = 8        /* call out of order (e.g. no state set) */
};

/* Arithmetic of the path. */
enum {
  FR_PREC_FP64 = 0,        /* plain form: everything in FP64 (the correctness oracle) */
  FR_PREC_MIXED = 1,       /* precision form: FP32 state/fluxes, split-precision operators */
  FR_PREC_MIXED_REFINE = 2 /* solve server only: a request runs in the precision form until its
                              residual stops falling (the FP32 floor), then goes on in FP64 from
                              that state to the residual-drop target */
};

typedef struct fr_case fr_case;

/* Options of a case beyond the reference deck. */
typedef struct fr_setup_opts {
  int precision;               /* FR_PREC_* */
  int perturb;                 /* 1: perturb interior vertices before setup */
  unsigned long long seed;     /* std::mt19937_64 seed for the perturbation */
  double perturb_frac;         /* amplitude as a fraction of the cell size */
  int mu_override;             /* 1: use mu_inf below instead of the deck's */
  double mu_inf;
  int visc_flux_quirk;         /* 1 (default): reference 3-D viscous-flux formulas */
  int debug_arrays;            /* 1: keep F_spts / disFn_fpts of residual calls */
  int device;                  /* CUDA device ordinal; -1: host-side setup only */
  int generic_kernels;         /* 1: use the general sparse-operator element kernel */
  int no_tma;                  /* 1: tensor-product element kernel without TMA tiles */
  int tile_variant;            /* precision form: element tile shape, -1 (default) = autotuned at setup;
                                  the last variant of 2-D orders 1..4 is the tensor-core (tcgen05) kernel */
  int no_tensor_cores;         /* 1: leave the tensor-core variant out of the autotuner's choice */
  int no_pdl;                  /* 1: no programmatic dependent launch (used for small cases by default) */
} fr_setup_opts;

/* Mesh supplied by the caller (linear quads or hexes, reference node order).
 * Boundary faces are listed by their vertices (2 per quad edge, 4 per hex
 * face) with a BC code of include/global.hpp:116-132 (0 = periodic, 1 = char,
 * 8 = slip_wall, ...).  Replaces geo::readGmsh + processConnectivity
 * (src/geo.cpp:1021-1475, 150-219) for callers that own their mesh. */
typedef struct fr_mesh {
  int nDims;
  int nVerts;
  const double *xv;       /* [nVerts][nDims] */
  int nEles;
  int nNodes;             /* quads: 4, 9, 16, ... (n+1)^2; hexes: 8, 20, 27, ... (n+1)^3 */
  const int *c2v;         /* [nEles][nNodes], Gmsh node order (corners first) */
  int nBndFaces;
  const int *bndFaceVerts; /* [nBndFaces][4] (2-D: last two entries ignored) */
  const int *bndFaceBc;    /* [nBndFaces] */
  double period[3];        /* periodic translation per axis (>= 1e299: none) */
} fr_mesh;

typedef struct fr_info {
  int nDims, nFields, order, nEles, nSpts, nFpts, nFaces, nFacePts, nRKSteps;
  int precision, dtType, timeType;
  long long iter;
  double time, dt;
  long long launches; /* kernels this case has launched (graph replays counted per kernel) */
  int tensor_kernels; /* 0 general, 1 tensor-product, 2 tensor-product with TMA tiles */
  int tile_variant;   /* precision form: element tile shape in use (-1: none) */
  int elems_per_block;
} fr_info;

/* Default fr_setup_opts (FP64, no perturbation, reference quirks on). */
void fr_setup_opts_default(fr_setup_opts *o);

/* Reads a reference input deck and sets up the case: mesh (meshType 1:
 * Cartesian generator), connectivity, operators, metrics, device buffers.
 * Replaces input::readInputFile (src/input.cpp:257-523) followed by
 * solver::setup(input*, order, geo* = NULL) (src/solver.cpp:60-115). */
int fr_create_from_deck(const char *deck_path, const fr_setup_opts *opts, fr_case **out);

/* As fr_create_from_deck, with the mesh given by the caller instead of the
 * deck's meshType (solver::setup with a prepared geo*, solver.cpp:60-75). */
int fr_create_with_mesh(const char *deck_path, const fr_mesh *mesh, const fr_setup_opts *opts,
                        fr_case **out);

void fr_destroy(fr_case *c);
const char *fr_last_error(const fr_case *c);
int fr_get_info(fr_case *c, fr_info *info);

/* Kernels of the case run on this stream (a cudaStream_t; NULL = default). */
int fr_set_stream(fr_case *c, void *stream);

/* Initial condition on the device.  kind 0: the deck's icType
 * (solver::initializeSolution, src/solver.cpp:1892-1943, ele.cpp:733-832);
 * 1: isentropic vortex (prm: eps, xc, yc, Mach); 2: Taylor-Green vortex
 * (prm: Mach); 3: uniform boundary state. */
int fr_init_solution(fr_case *c, int kind, const double *prm, int nprm);

/* Host <-> device state, [nSpts][nEles][nFields] doubles (solver::U_spts,
 * include/solver.hpp:94). */
int fr_set_state(fr_case *c, const double *U, size_t count);
int fr_get_state(fr_case *c, double *U, size_t count);
/* fr_get_state without the wait: the copy is queued on the case's stream
 * behind the work already queued there, and U holds the state once that
 * stream (fr_synchronize, or an event the caller records) has reached it.
 * Overlaps with other work only when U is page-locked host memory. */
int fr_get_state_async(fr_case *c, double *U, size_t count);

/* One residual evaluation into divF_spts[step] (solver::calcResidual,
 * include/solver.hpp:175, src/solver.cpp:366-445). */
int fr_calc_residual(fr_case *c, int step);
/* divF_spts[step] to the host, [nSpts][nEles][nFields]. */
int fr_get_residual(fr_case *c, int step, double *divF, size_t count);

/* One time step, all RK stages (solver::update, include/solver.hpp:172,
 * src/solver.cpp:319-363); advances time by dt. */
int fr_update(fr_case *c, int pmg_source);
/* One P-multigrid V-cycle on the case's coarse levels (multiGrid::cycle,
 * src/multigrid.cpp:169-313); the deck must have PMG 1.  The levels
 * (orders lowOrder .. order-1, same mesh) are built by fr_create_*. */
int fr_pmg_cycle(fr_case *c);

/* n steps of the reference's driver loop: update(), then, with PMG 1, the
 * V-cycle (src/flurry.cpp:162-170).  The steady-state step is captured once
 * as a CUDA graph and replayed. */
int fr_run(fr_case *c, int nsteps);

/* CFL time step (solver::calcDt, src/solver.cpp:447-468); *dt = global dt. */
int fr_calc_dt(fr_case *c, double *dt);
/* Fixed dt for dtType 0 ("dt" in the deck). */
int fr_set_dt(fr_case *c, double dt);

/* Residual norm per field of divF_spts[0] as writeResidual computes it
 * (src/output.cpp:1011-1090, ele.cpp:1922-1944); resType 1, 2 or 3. */
int fr_residual_norm(fr_case *c, int resType, double *out, int nFields);

/* Checks the device state for NaN/Inf or non-positive density
 * (FR_ERR_NONFINITE), the fail-stop checks of writeResidual. */
int fr_check_state(fr_case *c);

/* Copies a named array to the host (tests and tools): device arrays
 * "U_spts", "U0", "U_fpts", "Fn_fpts", "divF_<s>", "waveSp_fpts",
 * "F_spts", "disFn_fpts" (debug_arrays), "ele_dt"; setup arrays "pos_spts",
 * "detJac_spts", "JGinv_spts", "norm_fpts", "dA_fpts", "xv",
 * "opp_spts_to_fpts", "opp_grad_spts_<d>", "opp_extrapolateFn_<d>",
 * "opp_correction", "opp_correctU_<d>", "opp_prolong", "opp_restrict"
 * (doubles); "face_eL", "face_locL", "face_eR", "face_locR", "face_bc",
 * "face_fptR" (ints).  *count on input: capacity in elements; on output: size. */
int fr_get_array(fr_case *c, const char *name, void *host, size_t *count);

/* ---- Solution files --------------------------------------------------------
 * fr_checkpoint takes a snapshot of the current state for output: one kernel
 * on the case's stream forms the primitive variables at the plot points, and
 * their copy to pinned host memory runs on a side stream, so the caller can
 * keep stepping while it is in flight.  A later checkpoint replaces one that
 * was not written yet.
 * fr_write_data writes the latest checkpoint (taking one first if none is
 * pending) as the reference's writeData does (src/output.cpp:43-58): with
 * the deck's plotType 1 a ParaView file <dataFileName>_<iter, 9 digits>.vtu
 * in the reference's layout (src/output.cpp:137-512); with plotType 0 the CSV
 * <dataFileName>.csv.<iter> of primitives at the solution and flux points
 * (output.cpp:60-135, synchronous).  `path` NULL: that name, else `path`.
 * fr_read_restart sets the state and time from a ParaView file as
 * solver::readRestartFile does (src/solver.cpp:1789-1890, ele.cpp:1497-1921),
 * interpolating when the file's order differs from the case's; `path` NULL:
 * <dataFileName>_<restartIter>.vtu of the deck, and the iteration count
 * becomes restartIter.  fr_init_solution with kind 0 on a deck with
 * "restart 1" reads that file instead of the initial condition. */
/* solver::integrateError (src/solver.cpp:1945-2028) as writeError reports
 * it for testCase 1: per field, errorNorm 0 the integral of the exact
 * solution (|int(U - exact) - int U|, solution-point quadrature), 1 the
 * integral of |U - exact| and 2 the square root of the integral of
 * (U - exact)^2 on (quadOrder+1)^d Gauss points; exact = the deck's icType
 * field at the current time (src/funcs.cpp:1318-1476).  errorNorm < 0: the
 * deck's.  No reference counterpart for other testCase values. */
int fr_integrate_error(fr_case *c, int errorNorm, double *out, int nFields);

/* Boundary monitors on the face data of the last residual evaluation (call
 * fr_calc_residual first to evaluate them on the current state).
 * fr_wall_force: the force coefficients writeResidual prints
 * (src/output.cpp:1048-1066, boundFace::computeWallForce,
 * src/boundFace.cpp:412-458): out[0..2] pressure force, out[3..5] viscous
 * force, summed over slip, adiabatic and isothermal walls, divided by
 * 0.5 rhoBound Uinf^2 and turned to the free-stream direction (x, y).
 * fr_mass_flux: boundFace::computeMassFlux (src/boundFace.cpp:460-496), the
 * testCase 2 monitor: per field, the common flux through characteristic and
 * sub/supersonic boundaries, integrated (errorNorm 0), |.| n_x (1) or
 * (.)^2 n_x (2); errorNorm < 0: the deck's. */
int fr_wall_force(fr_case *c, double *out);
int fr_mass_flux(fr_case *c, int errorNorm, double *out, int nFields);

/* Sharding plan for running the case on nparts GPUs (host only; works on a
 * case created without a device).  The elements are split by recursive
 * coordinate bisection of their centroids, where the reference uses METIS
 * (geo::partitionMesh, src/geo.cpp:2380-2470).  For part `rank`: part[nEles]
 * (may be NULL) receives every element's part, *n_owned its element count
 * (local element ids follow ascending global ids), and *n_halo the number of
 * points on faces cut by the partition that it shares with other parts; with
 * cap >= *n_halo, halo_peer[k] and halo_slot[k] receive each point's peer
 * part and its slot fpt * n_owned + local element.  Both sides of a cut list
 * their shared points in the same order (by face, then by point in the
 * face's left order), so traces packed in list order are what the peer
 * expects, as mpiFace::communicate / getRightState exchange them
 * (src/mpiFace.cpp:122-175). */
int fr_shard_plan(fr_case *c, int nparts, int rank, int *part, int *n_owned, long long *n_halo, int *halo_peer,
                  long long *halo_slot, long long cap);

int fr_checkpoint(fr_case *c);
int fr_write_data(fr_case *c, const char *path);
int fr_read_restart(fr_case *c, const char *path);

/* Device pointer of a state array ("U_spts", "U_fpts", "divF_0", ...) for
 * callers that keep data resident (no copy).  Valid until fr_destroy.  For a
 * case created with FR_PREC_MIXED these are the precision form's FP32 working
 * arrays (4 bytes per value; *bytes says so), not FP64. */
int fr_device_ptr(fr_case *c, const char *name, void **ptr, size_t *bytes);

/* Instrumentation: launches one kernel of the steady-state RK stage `reps`
 * times on the case's stream ("element_stage": the fused element kernel of
 * an intermediate stage; "faces": the face kernel).  Mutates the state; for
 * timing only.  No reference counterpart. */
int fr_bench_kernel(fr_case *c, const char *kernel, int reps);

/* ---- Batching: many independent cases advanced together ----------------
 * Same-order cases are merged along the element axis into one group, so each
 * RK stage is one face launch and one element launch per order present and a
 * group's whole step replays as one CUDA graph; groups of different orders run
 * concurrently on their own streams.  Members must be inviscid, fixed-dt
 * (dtType 0, per-case dt kept), one RK scheme, state set.  No reference
 * counterpart (the reference runs one case per process). */
typedef struct fr_batch fr_batch;
int fr_batch_create(fr_case *const *cases, int n, fr_batch **out);
/* nsteps of every member (each with its own dt), then a device sync. */
int fr_batch_run(fr_batch *b, int nsteps);
/* Copies each member's state and last stage-0 residual back into its case. */
int fr_batch_gather(fr_batch *b);
/* writeResidual norms of every member: out[n][nFields]. */
int fr_batch_residual_norms(fr_batch *b, int resType, double *out, int nFields);
int fr_batch_info(fr_batch *b, int *nGroups, long long *launches);
/* Forms of a batch's step.  FR_BATCH_GROUPS: each order group's step graph
 * (one face and one element launch per stage) on the group's own stream.
 * FR_BATCH_MANY_ORDER: one face launch and one persistent element launch per
 * RK stage for all groups: CTAs take element blocks of every order from a
 * device work counter and run the tensor-product stage of each block's order
 * (inviscid groups of one precision, at most 6 orders).  fr_batch_create
 * times both on the batch's own state (3 steps each, state restored) and
 * keeps the faster; fr_batch_form reports the choice and the measured ms per
 * step of each (-1: not timed), fr_batch_set_form forces one. */
enum { FR_BATCH_GROUPS = 0, FR_BATCH_MANY_ORDER = 1 };
int fr_batch_form(fr_batch *b, int *form, float *ms_groups, float *ms_many_order);
int fr_batch_set_form(fr_batch *b, int form);
const char *fr_batch_last_error(const fr_batch *b);
void fr_batch_destroy(fr_batch *b);

/* ---- One case split into parts (sharding) ---------------------------------
 * The reference runs one case on several MPI ranks: geo::partitionMesh splits
 * the elements (METIS, src/geo.cpp:2380-2470), every face the split cuts
 * becomes an mpiFace whose right trace comes from the rank across it at every
 * stage (mpiFace::communicate / getRightState, src/mpiFace.cpp:122-175), each
 * side forming the common flux as its own left side, and calcDt takes the
 * minimum over ranks (src/solver.cpp:462-465).  A shard is that run with its
 * parts on one device: the partition of fr_shard_plan, one fr_case per part
 * (its elements, faces, metrics sliced from the whole case's), the cut traces
 * packed by a kernel and exchanged by device copies at every stage, the cut
 * faces formed by their own kernel, dt reduced over the parts on the device,
 * and a whole step of all parts replayed as one CUDA graph.  Its residual and
 * steps equal the unsplit case's to round-off (each side of a cut uses its
 * own normal), also for CFL time steps: a cut face writes its wave speed only
 * to the side that was the face's left side (face.cpp:372), where the
 * reference's mpiFace writes it to both sides.  Plain form (FP64), inviscid,
 * static mesh, no P-multigrid; nparts <= 64. */
typedef struct fr_shard fr_shard;
int fr_shard_create(const char *deck_path, const fr_setup_opts *opts, int nparts, fr_shard **out);
/* Parts, elements owned by each (owned[nparts]) and cut face points of each
 * (cut_points[nparts]); arrays may be null. */
int fr_shard_info(fr_shard *s, int *nparts, int *owned, long long *cut_points);
/* State and residual in the whole case's layout [nSpts][nEles][nFields]. */
int fr_shard_set_state(fr_shard *s, const double *U, size_t count);
int fr_shard_get_state(fr_shard *s, double *U, size_t count);
int fr_shard_set_dt(fr_shard *s, double dt);
int fr_shard_calc_residual(fr_shard *s, int step);
int fr_shard_get_residual(fr_shard *s, int step, double *divF, size_t count);
/* nsteps of solver::update over all parts (a CUDA graph after the first). */
int fr_shard_run(fr_shard *s, int nsteps);
/* Simulation time and the last dt (equal on every part). */
int fr_shard_time(fr_shard *s, double *time, double *dt);
const char *fr_shard_last_error(const fr_shard *s);
void fr_shard_destroy(fr_shard *s);

/* A part of a split case on its own rank: one process and one GPU per rank,
 * as the reference's MPI ranks.  Part `rank` of the partition of fr_shard_plan
 * (its elements in ascending global order; local state [nSpts][nOwned][nFields]
 * through fr_set_state / fr_get_state), stepped by fr_update / fr_run /
 * fr_calc_residual like any case: every face pass packs the part's cut traces
 * and exchanges them with each peer by grouped ncclSend/ncclRecv on the case's
 * stream, and dt (dtType 1, 2) is an ncclAllReduce(min).  nccl_comm is an
 * ncclComm_t of the nparts ranks (fr_nccl_comm_init makes one; it may be null
 * for nparts 1).  NCCL is resolved at run time (the process's libnccl.so.2).
 * Plain form, inviscid, static mesh, no P-multigrid.  The in-process shard
 * (fr_shard_*) runs the same parts, kernels and exchange order on one device. */
int fr_part_create(const char *deck_path, const fr_setup_opts *opts, int nparts, int rank, void *nccl_comm,
                   fr_case **out);
/* FR_ERR_CUDA if an NCCL call of the part's exchange reported an error. */
int fr_part_nccl_ok(fr_case *c);
/* NCCL communicator set-up for callers without NCCL bindings: rank 0 makes
 * the 128-byte id, every rank receives it (any transport) and calls
 * fr_nccl_comm_init with its device. */
int fr_nccl_unique_id(void *id128);
int fr_nccl_comm_init(int nranks, const void *id128, int rank, int device, void **comm);
int fr_nccl_comm_destroy(void *comm);

/* ---- Serving: a request loop with continuous batching --------------------
 * Requests (deck, optional mesh, initial condition, residual-drop target)
 * are admitted while the device-memory budget and the slot count allow; all
 * admitted cases stay on the device and advance together (own streams, graph
 * replays, overlapping on the GPU); a case retires when max over fields of
 * res/res0 (writeResidual norm, resType 2) <= tol or after max_steps, and
 * waiting requests take its place.  No reference counterpart. */
typedef struct fr_server fr_server;
int fr_server_create(size_t budget_bytes, int max_inflight, int check_every, int device, fr_server **out);
/* Form (FR_PREC_FP64, FR_PREC_MIXED or FR_PREC_MIXED_REFINE) of the requests the server admits
 * from now on (default FP64).  No reference counterpart. */
int fr_server_set_precision(fr_server *s, int precision);
int fr_server_submit(fr_server *s, const char *deck, const fr_mesh *mesh, int ic_kind, const double *ic_prm,
                     int n_prm, double tol, int max_steps, long long *id);
/* status: 0 queued, 1 running, 2 done, 3 failed, 4 cancelled; latency from submission. */
int fr_server_poll(fr_server *s, long long id, int *status, double *latency_s, int *steps, double *res_ratio);
/* Form a request runs (or finished) in, and the steps it ran in the
 * precision form (FR_PREC_MIXED_REFINE: before it went on in FP64). */
int fr_server_poll_form(fr_server *s, long long id, int *precision, int *steps_fp32);
/* Waits (bounded) for a request to finish; FR_ERR_TIMEOUT if it has not. */
int fr_server_wait(fr_server *s, long long id, double timeout_s);
/* Final state of a finished request, [nSpts][nEles][nFields]. */
int fr_server_result(fr_server *s, long long id, double *U, size_t count);
int fr_server_cancel(fr_server *s, long long id);
int fr_server_stats(fr_server *s, int *queued, int *inflight, size_t *inflight_bytes);
void fr_server_destroy(fr_server *s);

/* Blocks until the case's stream is idle; returns FR_ERR_CUDA on a sticky error. */
int fr_synchronize(fr_case *c);
/* 1 when all work issued on the case's stream has completed, 0 while some is
 * running, -FR_ERR_CUDA on an error (cudaStreamQuery); no reference
 * counterpart (used by the solve server to advance cases independently). */
int fr_stream_idle(fr_case *c);

/* Residual norm that allocates no device memory.  No counterpart in the
 * reference; it computes what fr_residual_norm computes (writeResidual,
 * src/output.cpp:1011-1090, ele.cpp:1922-1944), for callers that may not
 * allocate device memory: applications that hand out every device byte from
 * their own pool, and loops that may not take the synchronisation a
 * cudaMalloc/cudaFree brings.  divF and detJ are device arrays in the
 * library's layout ([nSpts][nEles][nFields] and [nSpts][nEles]), nFields =
 * nDims + 2, order <= 5, nEles <= FR_NOALLOC_MAX_ELES; out is a host array of
 * nFields.  divF and detJ must hold FP64 values: the FP32 working arrays of a
 * precision-form case (what fr_device_ptr returns for FR_PREC_MIXED) are
 * refused with FR_ERR_ARG.  Partial sums live in one fixed static device
 * array of FR_NOALLOC_SCRATCH_BYTES per GPU, so:
 *   - the first call on a device (with that device current) looks up the
 *     array's address and keeps it; after a cudaDeviceReset of that device
 *     the kept address is stale: do not call it on that device again;
 *   - no call may be made while its stream is being captured into a CUDA
 *     graph (each call copies from host memory and synchronises the stream);
 *   - calls that overlap in time (other streams, other host threads) race
 *     on the array: issue them one after another;
 *   - nothing needs zeroing: each call writes every partial it reads.
 * Returns when the result is in out (the stream is synchronised);
 * FR_ERR_ARG for sizes beyond the limits or FP32 arrays, FR_ERR_NONFINITE
 * when a norm is NaN (a NaN anywhere in divF, for every resType). */
#define FR_NOALLOC_MAX_SPTS 216
#define FR_NOALLOC_MAX_ELES 2147483647
#define FR_NOALLOC_SCRATCH_BYTES ((1024 * 5 + 5 + FR_NOALLOC_MAX_SPTS) * 8)
int fr_residual_norm_noalloc(const double *divF, const double *detJ, int nDims, int order, int nEles, int nFields,
                             int resType, double *out, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FR_B200_H */
