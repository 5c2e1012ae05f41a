/*
 * topx.h -- C ABI of the B200-native TOP3D_XL engine (libtopx.so).
 *
 * The MATLAB reference (TOP3D_XL.m) has no foreign-function interface; this
 * header is the boundary a MATLAB/Octave MEX gateway (or ctypes, or any C
 * caller) binds.  Each entry point names the reference function it replaces
 * ("TX:<line>" = line in TOP3D_XL.m).
 *
 * Conventions
 *  - Every call returns a topx_status; TOPX_OK is 0.  No C++ exception crosses
 *    this boundary; topx_last_error() gives the message of the last failure.
 *  - The caller owns every host buffer.  Arrays follow the reference's layouts:
 *    voxel volumes are column-major (nely, nelx, nelz) like MATLAB logical
 *    arrays; DOF vectors are interleaved (3k-2, 3k-1, 3k in MATLAB numbering,
 *    i.e. 3k+c 0-based) over the compact node numbering of meshHierarchy_(1);
 *    element vectors follow the compact element numbering (eleMapBack order).
 *  - Integer index arrays returned by topx_get_index_array are 1-based, as in
 *    the reference.
 *  - A context is not thread-safe: use one host thread per context.  Device
 *    memory is allocated at the first GPU call and freed by topx_destroy.
 *  - There is no CPU fallback: GPU calls return TOPX_ERR_CUDA when no usable
 *    sm_100 device is present.
 */
#ifndef TOPX_H_
#define TOPX_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int topx_status;
enum {
  TOPX_OK = 0,
  TOPX_STOP = 1,          /* topx_step: the loop condition ended the run (TX:111 / TX:311) */
  TOPX_ERR_ARG = -1,      /* bad argument (the reference's error('Wrong Input!') etc.) */
  TOPX_ERR_STATE = -2,    /* call out of order (no model loaded, no run begun) */
  TOPX_ERR_CUDA = -3,     /* CUDA runtime error or no usable device */
  TOPX_ERR_MODEL = -4,    /* model/BC error (format, no loads, no fixations, unsupported BCs) */
  TOPX_ERR_NUMERIC = -5,  /* solver failure (MMA dual solve did not finish, non-finite values) */
  TOPX_ERR_INTERNAL = -6,
  TOPX_ERR_TIMEOUT = -7   /* a bounded wait inside a kernel gave up (its poll limit, about a second,
                             ran out); the error word was cleared and the context stays usable */
};

enum { TOPX_GLOBAL = 0, TOPX_LOCAL = 1 };        /* consType (TX:12-18) */
/* arithmetic of the solver: TOPX_FP64 everything in FP64 (the reference's precision);
   TOPX_MIXED the multigrid preconditioner in FP32 inside the FP64 Krylov iteration (operator,
   residual, dots, compliance, optimiser and PDE filter in FP64); TOPX_MIXED_F32_FILTER the PDE
   filter's CG in FP32 as well */
enum { TOPX_FP64 = 0, TOPX_MIXED = 1, TOPX_MIXED_F32_FILTER = 2 };
enum { TOPX_VCYCLE_ADAPTED = 0, TOPX_VCYCLE_STANDARD = 1 };  /* typeVcycle_ (TX:34, 747-781) */

typedef struct topx_ctx topx_ctx;

/* InitialSettings (TX:21-38) plus engine options */
typedef struct topx_params {
  double modulus;          /* E0, 1.0 */
  double poissonRatio;     /* 0.3 */
  double modulusMin;       /* Emin, 1e-6 */
  double SIMPpenalty;      /* 3 */
  double cellSize;         /* 1 */
  double tol;              /* PCG relative tolerance, 1e-3 */
  int maxIT;               /* PCG iteration cap, 800 */
  double weightFactorJacobi; /* 0.6 */
  int64_t coarsestResolutionControl; /* 50000 */
  int precision;           /* TOPX_FP64, TOPX_MIXED or TOPX_MIXED_F32_FILTER */
  int device;              /* CUDA device ordinal */
  int coarse_coop;         /* 1: coarsest solve as one cooperative launch when available (default);
                              0: one launch per chain step (for engines sharing the GPU) */
  int typeVcycle;          /* TOPX_VCYCLE_ADAPTED (default, the reference's setting) or
                              TOPX_VCYCLE_STANDARD (smoothing against K x on every level; FP64 only,
                              otherwise topx_create returns TOPX_ERR_ARG) */
  int specifyPassiveRegions[3]; /* specifyPassiveRegions_ (TX:37): layers of passive elements on the
                              boundary, near loads, near fixations; {0, 0, 0} (default) adds none.
                              Applied when a model is loaded (TopOpti_SetPassiveElements, TX:1511) */
} topx_params;

/* sizes of the loaded model */
typedef struct topx_info {
  int numLevels;
  int nelx, nely, nelz;             /* input resolution */
  int64_t numElements, numNodes, numDOFs;  /* level 1 */
  int resX[8], resY[8], resZ[8];    /* padded resolution per level */
  int64_t levelElements[8], levelNodes[8];
  int numLoadCases;
  int64_t numFixedDOFs;
  int64_t numPassive;
} topx_info;

/* Load cases a model may have.  The reference allows any number (TX:483-493); a model with more
   is refused by topx_load_topvoxel / topx_set_bc with TOPX_ERR_MODEL, so that no history row
   (topx_iter.its) is ever truncated. */
#define TOPX_MAX_LOAD_CASES 8

/* one optimisation iteration (history row of TX:186-191 / TX:393-399) */
typedef struct topx_iter {
  int loop;
  double c;        /* cDesign: objective (compliance) */
  double vol;      /* V: mean density before the update */
  double sharp;    /* sharpness after the update */
  double cons;     /* fval: constraint value */
  double change;   /* max density change */
  int its[TOPX_MAX_LOAD_CASES]; /* PCG iterations per load case (iters_Target.dat) */
  int filter_its;  /* PDE-filter PCG iterations summed over the filters of this iteration */
  double t_assemble, t_cg, t_opt, t_filter, t_total;  /* seconds */
} topx_iter;

/* which index array topx_get_index_array returns */
enum {
  TOPX_ARR_ENODMAT = 0,            /* numElements x 8, row-major [e][j] (meshHierarchy_(l).eNodMat) */
  TOPX_ARR_ELEMAPBACK = 1,         /* numElements */
  TOPX_ARR_NODMAPBACK = 2,         /* numNodes (grid ids of the level's own grid) */
  TOPX_ARR_NODESONBOUNDARY = 3,
  TOPX_ARR_ELEMENTSONBOUNDARY = 4, /* level 1 only */
  TOPX_ARR_ELEMENTUPWARDMAP = 5,   /* numElements x span^3 (levels >= 2) */
  TOPX_ARR_TRANSFERMAT = 6,        /* numElements x (span+1)^3 (levels >= 2), [e][k] */
  TOPX_ARR_SOLIDNODEMAP = 7,       /* solidNodeMapCoarser2Finer (levels >= 2) */
  TOPX_ARR_FIXEDDOFS = 8,          /* numDOFs 0/1 (level 1) */
  TOPX_ARR_MAPUNIQUEKES = 9,       /* numElements (level 1) */
  TOPX_ARR_ISTHISELE2NDLEVEL = 10, /* level-2 elements holding fixed DOFs (level 2) */
  TOPX_ARR_PASSIVEELEMENTS = 11    /* passiveElements_, sorted compact ids (level 1) */
};

/* ---- lifecycle ------------------------------------------------------------ */
topx_status topx_default_params(topx_params* p);
topx_status topx_create(topx_ctx** ctx, const topx_params* p);
topx_status topx_destroy(topx_ctx* ctx);
const char* topx_last_error(const topx_ctx* ctx);
const char* topx_version(void);

/* ---- model (host only; no GPU needed) ------------------------------------- */
/* CreateVoxelFEAmodel, logical input with built-in cuboid BCs (TX:529-560) +
 * FEA_ApplyBoundaryCondition (TX:1294) + FEA_SetupVoxelBased (TX:1238) */
topx_status topx_load_voxels(topx_ctx* ctx, const uint8_t* vox, int nely, int nelx, int nelz);
/* CreateVoxelFEAmodel, .TopVoxel v1.0 input (TX:448-528) */
topx_status topx_load_topvoxel(topx_ctx* ctx, const char* path);
/* Boundary conditions of the loaded model as a .TopVoxel file gives them (TX:480-497,
   AdaptBCExternalMdl TX:1439-1490, then FEA_ApplyBoundaryCondition TX:1294-1336), replacing the
   built-in ones of topx_load_voxels or the file's.  Node ids are 1-based in the input model's own
   (nely+1) x (nelx+1) x (nelz+1) node grid, y fastest.  fixing: nfix rows (node, fixX, fixY,
   fixZ), a direction fixed where its value is 1; loads: nload rows (node, Fx, Fy, Fz, loadCase),
   load cases numbered from 1 (the reference's additional load cases).  Repeated nodes: the first
   row counts.  A node outside the grid returns TOPX_ERR_ARG, one outside the solid model
   TOPX_ERR_MODEL, no loads TOPX_ERR_MODEL ('No Loads!'). */
topx_status topx_set_bc(topx_ctx* ctx, const double* fixing, int64_t nfix, const double* loads, int64_t nload);
topx_status topx_get_info(const topx_ctx* ctx, topx_info* out);
/* element stiffness matrix (TX:1254-1292), 24x24 row-major */
topx_status topx_get_ke(const topx_ctx* ctx, double* out576);
/* integer arrays of meshHierarchy_(level) / BC set-up for bit-exact comparison */
topx_status topx_get_index_array(const topx_ctx* ctx, int level, int which, int32_t* out, size_t n, size_t* n_needed);
/* transferMatCoeffi of a level >= 2 */
topx_status topx_get_transfer_coeffi(const topx_ctx* ctx, int level, double* out, size_t n, size_t* n_needed);
/* load vector F_(:,lc), interleaved DOFs (TX:1316-1322) */
topx_status topx_get_load(const topx_ctx* ctx, int lc, double* out, size_t n);

/* ---- solver building blocks (GPU; host buffers) --------------------------- */
/* element moduli E (numElements) for the calls below; SIMP is applied by the caller */
topx_status topx_set_moduli(topx_ctx* ctx, const double* E, size_t n);
/* Solving_KbyU_MatrixFree, level 1 (TX:641-725): y = K(E) u, FP64 */
topx_status topx_ku(topx_ctx* ctx, const double* u, double* y, size_t ndof);
/* No counterpart in the reference.  y = K(E) u exactly like topx_ku, but u and y are device
   pointers (ndof doubles each, on the context's GPU) and the call allocates no device memory:
   topx_ku allocates temporary device buffers on every call, which callers whose device memory
   is owned by another allocator (MATLAB gpuArray, a framework's caching pool) or whose loop may
   not call cudaMalloc/cudaFree cannot accept.  Its scratch is one fixed 32 MiB static device
   array, enough for level-1 grids of up to 699,040 padded nodes; larger models get
   TOPX_ERR_ARG.  The context's device state must exist already (e.g. after topx_set_moduli).
   The first call on each GPU looks up the array's address; make it before any stream capture.
   All calls share the array: calls that overlap on the GPU race.  The call runs after the work
   already queued on the legacy default stream (stream 0), so u may be written there
   asynchronously just before; work pending on the caller's other streams (non-blocking or
   per-thread default streams) is not waited for and must be synchronised by the caller.
   Returns after y is written. */
topx_status topx_ku_noalloc(topx_ctx* ctx, const double* u_dev, double* y_dev, size_t ndof);
/* Solving_AssembleFEAstencil (TX:919-1066) for the current moduli */
topx_status topx_assemble(topx_ctx* ctx);
/* Solving_Vcycle (TX:747-781): z = M r in the context's precision */
topx_status topx_vcycle(topx_ctx* ctx, const double* r, double* z, size_t ndof);

/* Design output files (host only, no context).  vol is the padded density volume V(y, x, z),
   column-major ny x nx x nz as the reference forms it (TX:206-208, 565-568; void = 0).
   topx_write_design_nii: IO_ExportDesignInVolume_nii (TX:564-570), NIfTI-1 FLOAT64.
   topx_write_design_stl: the 'Vis.' block and IO_ExportDesignInTriSurface_stl (TX:206-222,
   572-577): V flipped along y, its isosurface at `iso` (the reference uses 0.5) closed by caps on
   the volume boundary, in MATLAB's vertex coordinates (x = column, y = row, z = page, from 1),
   as binary STL with outward normals; *ntriangles (may be NULL) gets the triangle count. */
topx_status topx_write_design_nii(const double* vol, int ny, int nx, int nz, const char* path);
topx_status topx_write_design_stl(const double* vol, int ny, int nx, int nz, double iso, const char* path,
                                  int64_t* ntriangles);
/* Jacobi diagonal meshHierarchy_(level).diagK (level < numLevels), interleaved */
topx_status topx_get_diag(topx_ctx* ctx, int level, double* out, size_t n);
/* Solving_PCG with K*u and the V-cycle (TX:600-639), warm start from u; its = iterations */
topx_status topx_pcg(topx_ctx* ctx, int lc, double* u, size_t ndof, int* its);
/* TopOpti_ConductPDEFiltering_matrixFree (TX:870-902) with radius rmin */
topx_status topx_filter(topx_ctx* ctx, double rmin, const double* src, double* out, size_t ne, int* its);
/* TopOpti_ComputeUnitCompliance (TX:579-598) of displacement fields U (numDOFs x numLoadCases, column-major) */
topx_status topx_unit_compliance(topx_ctx* ctx, const double* U, double* ce, size_t ne);

/* ---- optimisation (TOP3D_XL_TO TX:40-223, TOP3D_XL_PIO TX:225-440) -------- */
/* set-up + compliance of the fully solid domain (iteration 0) */
topx_status topx_begin(topx_ctx* ctx, int consType, double V0, int nLoop, double rMin, double rHat,
                       double* cSolid);
/* one iteration of the while loop; TOPX_STOP when the loop condition fails */
topx_status topx_step(topx_ctx* ctx, topx_iter* out);
/* full run: begin + steps; hist may be NULL, else an array of at least nLoop rows */
topx_status topx_run(topx_ctx* ctx, int consType, double V0, int nLoop, double rMin, double rHat,
                     topx_iter* hist, int* loops, double* cSolid);
/* densityLayout_ = xPhys (numElements) */
topx_status topx_get_density(topx_ctx* ctx, double* out, size_t ne);
topx_status topx_set_density(topx_ctx* ctx, const double* xPhys, size_t ne);
/* displacement U(:,lc), interleaved DOFs */
topx_status topx_get_displacement(topx_ctx* ctx, int lc, double* out, size_t ndof);

/* ---- failure handling (no reference counterpart) ----------------------------- */
/* Test of the give-up path of the one bounded wait in the library's kernels: in the persistent
   coarsest-level solve (contexts with topx_params.coarse_coop = 1) a task waits for the tasks of
   the fronts it reads.  which must be 0: one CTA waits for a counter that nothing raises, so its
   wait exhausts its poll limit (about a second) and sets the solve's error word.  Returns
   TOPX_ERR_TIMEOUT with a message naming the wait, as a real give-up inside a solve would; the
   context stays usable. */
topx_status topx_selftest_wait(topx_ctx* ctx, int which);

/* ---- measurement (no reference counterpart) --------------------------------- */
#define TOPX_PROFILE_SECTIONS 14
typedef struct topx_profile {
  double ku_ms;             /* summed device time of the level-1 K*u launches inside PCG solves */
  int64_t ku_launches;      /* launches that ran a PCG iteration */
  int64_t pcg_iterations;   /* PCG iterations since profiling was switched on */
  double section_ms[TOPX_PROFILE_SECTIONS];     /* device time per section (see topx_profile_section_name) */
  int64_t section_count[TOPX_PROFILE_SECTIONS]; /* timed launch groups per section */
} topx_profile;
const char* topx_profile_section_name(int section);
/* CUDA-event timer on the engine's stream */
topx_status topx_timer_start(topx_ctx* ctx);
topx_status topx_timer_stop(topx_ctx* ctx, double* ms);
/* per-launch timing of the K*u kernel (events around each launch); on != 0 resets the counters */
topx_status topx_set_profiling(topx_ctx* ctx, int on);
topx_status topx_get_profile(topx_ctx* ctx, topx_profile* out);
/* kernels this library has launched in this process so far (graph replays count their kernels) */
int64_t topx_launch_count(void);

/* ---- serving: continuous batching of design jobs (no reference counterpart) -------
   A server runs design jobs (each one TOP3D_XL call) on one GPU for many clients.  Up to
   `slots` jobs are on the device at once, each with its own engine and stream, so their work
   overlaps.  A queued job is admitted as soon as a slot is free and its device-memory
   footprint fits the HBM budget; jobs are taken in arrival order, skipping one that does not
   fit yet.  The result of a job does not depend on what runs beside it. */
typedef struct topx_server topx_server;
typedef struct topx_server_params {
  int slots;                /* jobs on the device at once (worker threads), default 6 */
  double hbm_budget_bytes;  /* device memory admitted jobs may hold; <= 0: 85% of free memory */
  int precision;            /* TOPX_FP64, TOPX_MIXED or TOPX_MIXED_F32_FILTER */
  int device;               /* CUDA device ordinal */
} topx_server_params;
typedef struct topx_job {
  int nely, nelx, nelz;     /* voxel grid; with voxels == NULL a solid cuboid (built-in BCs) */
  const uint8_t* voxels;    /* optional column-major nely x nelx x nelz mask, copied at submit */
  int consType;             /* TOPX_GLOBAL or TOPX_LOCAL */
  double V0;
  int nLoop;
  double rMin, rHat;
  int keep_density;         /* 1: keep the final density for topx_server_get_density */
} topx_job;
typedef struct topx_job_result {
  int status;               /* TOPX_OK, or the status the job failed with */
  int loops;                /* optimisation iterations run */
  double cSolid;            /* compliance of the fully solid domain */
  double c_last;            /* compliance of the last iteration */
  int64_t pcg_its;          /* elasticity PCG iterations over the whole job */
  int64_t numElements;
  int64_t footprint_estimate; /* bytes used for admission */
  int64_t footprint_bytes;    /* device bytes its engine held */
  double t_submit, t_admit, t_end; /* seconds on the server's clock */
} topx_job_result;
typedef struct topx_server_stats {
  int64_t submitted, done, failed, running, queued;
  int max_running;          /* most jobs on the device at once so far */
  double budget_bytes, peak_bytes; /* admission budget and peak admitted footprint */
} topx_server_stats;
topx_status topx_server_default_params(topx_server_params* p);
topx_status topx_server_create(topx_server** srv, const topx_server_params* p);
/* waits for the running jobs; queued jobs end with TOPX_ERR_STATE */
topx_status topx_server_destroy(topx_server* srv);
/* enqueue a job; never blocks on the device */
topx_status topx_server_submit(topx_server* srv, const topx_job* job, int64_t* job_id);
/* TOPX_OK and the result once the job has ended, TOPX_STOP while it is queued or running */
topx_status topx_server_poll(topx_server* srv, int64_t job_id, topx_job_result* out);
/* blocks until the job has ended */
topx_status topx_server_wait(topx_server* srv, int64_t job_id, topx_job_result* out);
/* per-iteration history of an ended job (n entries at most) */
topx_status topx_server_get_history(topx_server* srv, int64_t job_id, topx_iter* hist, int n, int* loops);
/* final density (numElements) of an ended job submitted with keep_density */
topx_status topx_server_get_density(topx_server* srv, int64_t job_id, double* out, size_t n);
topx_status topx_server_get_stats(topx_server* srv, topx_server_stats* out);
const char* topx_server_last_error(topx_server* srv);

#ifdef __cplusplus
}
#endif

#endif /* TOPX_H_ */
