/*
 * pcc_gpu.h -- C ABI of the B200 (sm_100a) collision hot path of the
 * ProliferatingCellCollectives simulator.
 *
 * One context (pcc_ctx) holds one colony resident on one GPU.  Every entry
 * point returns a pcc_status (0 = PCC_OK); pcc_last_error() gives the message
 * of the last failure on a context.  Calls on one context are not
 * thread-safe: use one host thread per context.  All state arrays that cross
 * this boundary are caller-owned host buffers in structure-of-arrays form;
 * they are copied, never retained.
 *
 * Reference interfaces replaced (paths are inside the reference project,
 * under code/cpp/src/):
 *   pcc_solve            ParticleManager::step (simulation/ParticleManager.cpp:150-166)
 *                        -> solveHardModel (dynamics/models/Hard.h:9, Hard.cpp:91-192)
 *                        -> solveSoftPotential (dynamics/models/Soft.h:8, Soft.cpp:21-114)
 *   pcc_step             one iteration of Domain::run at one rank
 *                        (spatial/Domain.cpp:120-153): divideParticles + commit,
 *                        assignGlobalIDs (492-508), step, adaptDt (69-118), radius
 *   pcc_detect_contacts  CollisionDetector::detectCollisions (spatial/CollisionDetector.cpp:84-111)
 *   pcc_get_constraints  SolverSolution::constraints (simulation/ParticleManager.h:33-39)
 *   pcc_bbpgd_frozen     BBPGD (solver/BBPGD.h:26-31) on a frozen constraint set
 *   pcc_soft_forces_frozen  the Hertz force loop of solveSoftPotential (Soft.cpp:46-83)
 * Errors that the reference raises as std::runtime_error come back as
 * PCC_ERR_NOCONV_BBPGD ("BBPGD did not converge", solver/BBPGD.cpp:118-121) and
 * PCC_ERR_NOCONV_RELCP ("Maximum number of constraint iterations reached",
 * dynamics/models/Hard.cpp:187-190).
 */
#ifndef PCC_GPU_H
#define PCC_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int pcc_status;
#define PCC_OK 0
#define PCC_ERR_INVALID 1       /* bad argument or call order */
#define PCC_ERR_NOCONV_BBPGD 2  /* BBPGD hit max_bbpgd_iterations */
#define PCC_ERR_NOCONV_RELCP 3  /* ReLCP hit max_recursive_iterations */
#define PCC_ERR_CAPACITY 4      /* caller buffer too small; *n holds the size needed */
#define PCC_ERR_TIMEOUT 5       /* a bounded device-side wait gave up */
#define PCC_ERR_BOUNDS 6        /* a device-side bounds check failed */
#define PCC_ERR_CUDA 7          /* CUDA runtime error */
#define PCC_ERR_NAN 8           /* non-finite state detected */
#define PCC_ERR_NOMEM 9         /* device allocation failed */

#define PCC_MODE_HARD 0
#define PCC_MODE_SOFT 1

/* What the per-phase ghost exchange of the reference driver supplies at one
 * rank (Domain::exchangeGhostParticles, spatial/Domain.cpp:339-403): at world
 * size 1 the angular-neighbour test picks the rank itself, so every cell with
 * |(x,y)| >= 8 whose distance to the 0/360-degree sector edge is below 2.5
 * becomes a ghost copy of itself.  The ownership rule of
 * CollisionDetector::tryCreateConstraint (spatial/CollisionDetector.cpp:261-275)
 * then emits a second, identical constraint for every contact whose
 * larger-id cell has such a copy.  PCC_GHOSTS_SINGLE_RANK reproduces that;
 * PCC_GHOSTS_NONE is the same solver with no ghost copies. */
#define PCC_GHOSTS_NONE 0
#define PCC_GHOSTS_SINGLE_RANK 1

#define PCC_PRECISION_FP64 0
/* Mixed precision (planar colonies): the BBPGD operands D, L, M and U and the
 * D / M products in FP32; gamma, the gradient, Phi, the stress sums, the BB dot
 * products, the residual, positions and orientations in FP64.  Contact
 * geometry stays FP64, so the contact set is the FP64 one.  Non-planar
 * colonies run the FP64 solver. */
#define PCC_PRECISION_MIXED 1

/* Mirrors SimulationParameters (util/Config.h:27-56, defaults in
 * util/CLIParser.h:296-365) plus the run-time switches of this library. */
typedef struct pcc_params {
  /* SimulationConfig */
  double dt;          /* -dt: first (or fixed) time step */
  double end_radius;  /* -end_radius: pcc_run stops once the colony radius reaches it */
  /* PhysicsConfig */
  double xi;          /* -xi: drag per unit length */
  double tau;         /* -tau: growth time constant */
  double l0;          /* -l0: birth length; cells divide at 2*l0 */
  double lambda;      /* -lambda: stress sensitivity of growth */
  double temperature; /* -temperature: Brownian rotational kicks (Physics.cpp:59-81); 0 turns them off */
  double kcc;         /* -kcc: Hertz constant of the soft model */
  int monolayer;      /* -monolayer (only affects Brownian kicks) */
  /* SolverConfig */
  double tolerance;                    /* -tolerance: BBPGD residual, ReLCP overlap, CFL */
  long long max_bbpgd_iterations;      /* -max_bbpgd_iterations */
  long long max_recursive_iterations;  /* -max_recursive_iterations */
  double linked_cell_size;             /* -linked_cell_size (2.2*l0 when unset) */
  double cfl_factor;                   /* -cfl_factor */
  /* -mode */
  int mode;                            /* PCC_MODE_HARD or PCC_MODE_SOFT */
  /* additions (default off) */
  int fixed_dt;                        /* 1: skip adaptDt, keep dt */
  double dt_cap;                       /* > 0: adapted dt never exceeds this */
  int ghost_mode;                      /* PCC_GHOSTS_* */
  unsigned long long seed;             /* seeds the division length draws */
  int precision;                       /* PCC_PRECISION_FP64 or PCC_PRECISION_MIXED */
  long long capacity_hint;             /* expected peak cell count (0: grow on demand) */
  int solver_variant;                  /* PCC_SOLVER_AUTO or PCC_SOLVER_GENERAL */
  double log_every_colony_radius_delta;  /* VTK output cadence of the driver (CLI default 0.5) */
  double log_every_sim_time_delta;       /* ... and by simulated time (CLI default 100000) */
  int log_bbpgd_trace;                   /* 1: -log_bbgd_trace, trace BBPGD on every 10th step;
                                            2: record every solve without changing the solver
                                            (residual still tested every 10th iteration) */
} pcc_params;

/* BBPGD kernel choice.  A planar colony (every z = 0, rotation about z only)
 * keeps those zeros exactly through a step, so the planar form -- which skips
 * the terms that are exact zeros -- gives bit-identical results with half the
 * memory traffic.  AUTO picks it whenever the colony is planar. */
#define PCC_SOLVER_AUTO 0
#define PCC_SOLVER_GENERAL 1

/* Host SoA view of n cells (index = global id after the x-sort).  Optional
 * arrays may be NULL.  force/velocity hold 6 values per cell (linear, angular). */
typedef struct pcc_cells {
  double *x, *y, *z;           /* centre */
  double *q0, *q1, *q2, *q3;   /* unit quaternion (w, x, y, z) */
  double *length, *l0, *diameter;
  double *ldot, *impedance, *stress;  /* optional */
  int *age;                           /* optional */
  double *force, *velocity;           /* optional, 6 per cell */
  int *num_constraints;               /* optional, download only: contacts counted during the last solve */
} pcc_cells;

/* Host SoA view of constraints (Constraint, dynamics/Constraint.h:6-49). */
typedef struct pcc_contacts {
  int *gid_i, *gid_j;
  double *sd;            /* signed distance (phi) */
  double *normal;        /* 3 per contact: normI, unit, from j towards i */
  double *r_i, *r_j;     /* 3 each: contact point minus centre */
  double *contact_point; /* 3 */
  double *stress_i, *stress_j;
  double *gamma;
  int *phase;            /* ReLCP iteration that detected it */
} pcc_contacts;

/* SolverSolution scalars (simulation/ParticleManager.h:33-39) plus driver data. */
typedef struct pcc_step_stats {
  int relcp_iterations;         /* constraint_iterations */
  long long bbpgd_iterations;   /* summed over ReLCP phases */
  double residual;
  double max_overlap;
  long long n_constraints;      /* size of the returned constraint set */
  long long n_cells;            /* cells during the solve */
  long long n_divided;          /* divisions committed at the start of the step */
  double dt_used;               /* dt of this step */
  double dt_next;               /* dt after adaptDt */
  double colony_radius;         /* after the step */
  double sim_time;              /* after the step */
} pcc_step_stats;

/* Device-time accounting of the last pcc_reset_profile .. now window
 * (CUDA events on the context's stream; only while profiling is on). */
typedef struct pcc_profile {
  long long bbpgd_launches;     /* persistent BBPGD kernel launches */
  long long bbpgd_iterations;   /* iterations they ran */
  double bbpgd_ms;              /* device time of those launches */
  double bbpgd_algo_bytes;      /* sum over launches of iterations * (312 C + 288 N); (192 C + 144 N) mixed */
  double detect_ms;             /* contact detection + incidence lists */
  double solve_ms;              /* whole pcc_solve calls */
  long long solves;
  double cell_solves;           /* sum of cell counts over solves */
  long long detect_full_passes; /* detections that rebinned the colony (counted with profiling off too) */
  long long detect_list_passes; /* later ReLCP phases served from the candidate lists */
  long long bbpgd_grid_launches;  /* BBPGD launches of the multi-block (grid-synchronised) kernel
                                     (counted with profiling off too) */
  long long bbpgd_cta_launches;   /* BBPGD launches of the one-block kernels (small colonies) */
} pcc_profile;

typedef struct pcc_ctx pcc_ctx;

/* Reference defaults (CLIParser.h:296-365), except temperature 0 (the
 * reference's 1e-28 moves no quaternion at FP64 resolution and would cost a
 * host draw per step): hard mode, ghost
 * copies as the reference driver makes them at one rank (PCC_GHOSTS_SINGLE_RANK). */
void pcc_default_params(pcc_params* p);

pcc_status pcc_create(const pcc_params* params, int device, pcc_ctx** out);
pcc_status pcc_destroy(pcc_ctx* ctx);
const char* pcc_last_error(const pcc_ctx* ctx);

/* Runtime parameters that the driver may change between steps. */
pcc_status pcc_set_dt(pcc_ctx* ctx, double dt);
pcc_status pcc_get_dt(const pcc_ctx* ctx, double* dt);

/* Replace the colony with n cells (copied).  Any order; pcc_step sorts. */
pcc_status pcc_upload_cells(pcc_ctx* ctx, const pcc_cells* cells, size_t n);
/* Copy the colony out in global-id order.  PCC_ERR_CAPACITY if cap < n. */
pcc_status pcc_download_cells(pcc_ctx* ctx, pcc_cells* cells, size_t cap, size_t* n);
pcc_status pcc_cell_count(const pcc_ctx* ctx, size_t* n);

/* One solver call on the resident cells, which must already be in global-id
 * order (ParticleManager::step): ReLCP/BBPGD (hard) or Hertz forces (soft),
 * then move, set growth parameters and grow with time step dt. */
pcc_status pcc_solve(pcc_ctx* ctx, double dt, int iter, pcc_step_stats* out);

/* One Domain::run iteration: divide, append daughters, sort by x and
 * renumber, pcc_solve, advance time, adapt dt (unless fixed), colony radius. */
pcc_status pcc_step(pcc_ctx* ctx, pcc_step_stats* out);

/* Repeat pcc_step until the colony radius reaches end_radius or max_steps
 * steps ran.  Sums cells over steps into *cell_steps when non-NULL. */
pcc_status pcc_run(pcc_ctx* ctx, double end_radius, long long max_steps, long long* steps_done,
                   double* cell_steps, pcc_step_stats* last);

/* Contact detection on the resident state with tolerance tol (phase is
 * recorded in the output).  Order: grouped by the smaller global id. */
pcc_status pcc_detect_contacts(pcc_ctx* ctx, double tol, int phase, pcc_contacts* out, size_t cap, size_t* n);

/* The constraint set returned by the last pcc_solve (after write-back). */
pcc_status pcc_get_constraints(pcc_ctx* ctx, pcc_contacts* out, size_t cap, size_t* n);

/* Microbench / parity entry points on a frozen state. */
pcc_status pcc_bbpgd_frozen(pcc_ctx* ctx, double dt, int repeats, long long* iterations, double* residual,
                            float* ms_per_solve);
pcc_status pcc_soft_forces_frozen(pcc_ctx* ctx, int repeats, float* ms_per_assembly);

/* Soft-model force assembly that allocates no device memory.  It has no
 * counterpart in the reference: it exists for hosts that must not let this
 * library allocate -- a host that accounts its HBM through its own fixed pool
 * (such as a serving loop admitting colonies against a byte budget), or a
 * stepping loop sharing the GPU with other colonies' streams, where
 * cudaFree's device-wide wait would stall them.  Every pointer is a device
 * pointer the caller owns: contacts in the pcc_contacts layout (normal, r_i,
 * r_j hold 3 values per contact) and the cell diameters are inputs; force
 * (6 per cell: force, torque) and stress (1 per cell) are outputs, equal to
 * the force assembly of pcc_soft_forces_frozen / solveSoftPotential
 * (Soft.cpp:46-83).  Limit: 65536 cells and 393216 contacts per call
 * (PCC_ERR_CAPACITY beyond, before any GPU work).  Every gid_i / gid_j must be
 * a cell index in [0, n); a contact outside that range is skipped on the
 * device and the call returns PCC_ERR_BOUNDS (the call waits for its own work
 * on `stream` to read that flag back).  An error already pending from earlier
 * work in the process makes the call return PCC_ERR_CUDA without launching.
 * Intermediates live in one fixed 6.75 MiB device array that every call on a
 * GPU shares, so calls must not overlap on one device; the first call on a
 * device looks the array up and should come before any stream capture, and
 * with lazy module loading it may make the driver load this code into device
 * memory of its own (later calls allocate nothing).  stream is a cudaStream_t
 * (NULL: the default stream). */
pcc_status pcc_soft_forces_noalloc(const int* gid_i, const int* gid_j, const double* sd, const double* normal,
                                   const double* r_i, const double* r_j, const double* stress_i,
                                   const double* stress_j, size_t m, const double* diameter, size_t n, double kcc,
                                   double* force, double* stress, void* stream);

/* One colony job of a batch sweep or a serving stream: grow one colony from a
 * single cell (orientation theta ~ U[0, pi) drawn from params.seed) until its
 * radius reaches end_radius. */
typedef struct pcc_job {
  pcc_params params;   /* per job: mode, seed, tau (= 1 / growth rate), tolerances, ... */
  double end_radius;
  double arrival_s;    /* arrival time after the start of pcc_serve (0: immediately) */
  long long max_steps; /* 0: no cap */
} pcc_job;

typedef struct pcc_job_result {
  int status;                  /* pcc_status of the job */
  long long steps;
  long long cells;             /* final cell count */
  double cell_steps;           /* sum over steps of the cell count */
  long long bbpgd_iterations;
  double arrival_s, start_s, finish_s;  /* seconds after the start of pcc_serve */
  double footprint_bytes;      /* projected device footprint used for admission */
  double checksum;             /* sum over final cells of x+y+z+q0+q1+q2+q3+length */
  long long max_step_bbpgd;    /* most BBPGD iterations in one step */
  double radius;               /* colony radius after the last step */
  double dt;                   /* time step of the last step */
} pcc_job_result;

/* Continuous batching of independent colonies (no counterpart in the
 * reference, which runs one colony per MPI job): runs the jobs with at most
 * `slots` in flight, each on its own context, CUDA stream and host thread so
 * their kernels overlap on the device.  A job is admitted, in arrival order,
 * once it has arrived, a slot is free and its projected device footprint at
 * end_radius fits in hbm_budget_bytes beside the jobs in flight; a finishing
 * job frees its slot and budget.  Results are bit-identical alone and in any
 * mix.  Returns the first failing job's status (all results are filled). */
pcc_status pcc_serve(const pcc_job* jobs, size_t n_jobs, int slots, double hbm_budget_bytes, int device,
                     pcc_job_result* results, double* wall_s);

/* ---- VTK output and restart (the reference's file formats, one rank) ---- */

/* The per-log record of vtk::SimulationStep (logger/SimulationLogger.h:7-30);
 * field names and order as the reference writes them. */
typedef struct pcc_sim_record {
  double simulation_time_s;
  double time_since_last_log_s;
  unsigned long long step;
  int num_particles;
  unsigned long long num_constraints;
  double colony_radius;
  int recursive_iterations;
  unsigned long long bbpgd_iterations;
  double max_overlap;
  double residual;
  double dt_s;
  double memory_usage_mb;
  double peak_memory_mb;
  double cpu_time_s;
  double mpi_comm_time_s;
  double load_imbalance;
} pcc_sim_record;

/* Writes one particle file pair, <outdir>/data/<prefix>_<index, 7 digits>_rank_0000.vtu
 * and <outdir>/<prefix>_<index>.pvtu, byte-identical to vtk::ParticleLogger::log
 * (logger/ParticleLogger.cpp:13-76, logger/VTK.h) at one rank for the same
 * cells.  With ghost_copies, writes the self-ghost copies of the single-rank
 * decomposition instead (Domain::exchangeGhostParticles, spatial/Domain.cpp:339-403),
 * as copies carry them: no force, velocity, impedance, stress or contact count. */
pcc_status pcc_vtk_write_particles(const char* outdir, const char* prefix, unsigned long long index,
                                   const pcc_cells* cells, size_t n, int ghost_copies);
/* simulation_<index> files of vtk::SimulationLogger::log (logger/SimulationLogger.cpp:9-36). */
pcc_status pcc_vtk_write_simulation(const char* outdir, unsigned long long index, const pcc_sim_record* rec);
/* parameters_<index> files of vtk::ParameterLogger::log (logger/ParameterLogger.cpp:11-40). */
pcc_status pcc_vtk_write_parameters(const char* outdir, unsigned long long index, const pcc_params* params);

/* Asynchronous log point of Domain::run (spatial/Domain.cpp:188-200): snapshots
 * the resident cells on the device, in stream order after the last step, and
 * returns; a background thread copies the snapshot to the host and writes the
 * particles_, ghost_particles_ and (rec != NULL) simulation_ files of `index`
 * while the colony keeps stepping.  pcc_log_vtk_wait blocks until every
 * pending write is on disk and reports a failed write. */
pcc_status pcc_log_vtk(pcc_ctx* ctx, const char* outdir, unsigned long long index, const pcc_sim_record* rec);
pcc_status pcc_log_vtk_wait(pcc_ctx* ctx);

/* Restart (-starter_vtk): vtk::VTKStateLoader::loadLatestState
 * (loader/VTKStateLoader.cpp:24-162) on a VTK output directory (or a file in
 * it): the latest simulation_ record and the particles of the same index.
 * Cells come back as the loader builds them (l0 = 1, diameter 0.5, age 1,
 * no torque; force and velocities from the file, positions at the file's
 * float precision).  With out = NULL only *n (and the clock) are returned;
 * PCC_ERR_CAPACITY if cap < *n.  dt is the file's dt_s field, which the
 * reference reads but does not use. */
pcc_status pcc_vtk_load(const char* vtk_path, pcc_cells* out, size_t cap, size_t* n, double* sim_time,
                        long long* step, double* dt);
/* BBPGD trace (-log_bbgd_trace; solver/BBPGD.cpp:55-81, logger/BBPGDLogger.cpp,
 * HardModelGradient::energy, HardModelGradient.cpp:160-203).  On a hard-model
 * solve whose step counter is a multiple of 10, with params.log_bbpgd_trace
 * set, the solver evaluates and tests the residual at every iteration (as the
 * reference does while tracing) and records, per iteration, the residual, the
 * step size and the energy terms; after the ReLCP loop the records are written
 * as bbpgdtrace_<index> files (index from 1; earlier bbpgdtrace files in the
 * directory are removed first, as the reference's logger does) into the
 * trace directory, "logs" by default. */
typedef struct pcc_bbpgd_trace_step {
  unsigned long long step;                /* BBPGD iteration */
  unsigned long long recursive_iteration; /* ReLCP phase */
  unsigned long long total_constraints;
  double residual;
  double step_size;
  double linear;     /* gamma . Phi */
  double quadratic;  /* dt/2 gamma^T D^T M D gamma */
  double growth;     /* dt/(lambda tau) sum l exp(-lambda L^T gamma) */
  double total;
} pcc_bbpgd_trace_step;
pcc_status pcc_set_trace_dir(pcc_ctx* ctx, const char* dir);
/* Writes trace records as bbpgdtrace_<first_index + k> files (host only). */
pcc_status pcc_vtk_write_trace(const char* outdir, unsigned long long first_index, const pcc_bbpgd_trace_step* steps,
                               size_t n);
/* Records of the last traced solve (n = 0 if none); out = NULL returns n. */
pcc_status pcc_get_bbpgd_trace(const pcc_ctx* ctx, pcc_bbpgd_trace_step* out, size_t cap, size_t* n);

/* Sets the simulated time and the step counter of a context (after a restart). */
pcc_status pcc_set_clock(pcc_ctx* ctx, double sim_time, long long iteration);

/* Request loop (no counterpart in the reference): the admission and
 * execution of pcc_serve as a long-lived server that accepts jobs while it
 * runs.  submit queues a job (arrival = submit time; PCC_ERR_CAPACITY if its
 * projected footprint alone exceeds the budget); a scheduler thread admits
 * queued jobs in submit order as slots and budget free up; poll returns up to
 * cap finished results with their ids, waiting up to wait_s seconds for the
 * first; destroy finishes every queued and running job, then frees the
 * server (results not polled by then are dropped). */
typedef struct pcc_server pcc_server;
pcc_status pcc_server_create(int slots, double hbm_budget_bytes, int device, pcc_server** out);
pcc_status pcc_server_submit(pcc_server* server, const pcc_job* job, unsigned long long* id);
pcc_status pcc_server_poll(pcc_server* server, pcc_job_result* out, unsigned long long* ids, size_t cap, size_t* n,
                           double wait_s);
pcc_status pcc_server_pending(pcc_server* server, size_t* queued, size_t* running);
pcc_status pcc_server_destroy(pcc_server* server);

/* Lockstep batch of colonies (no counterpart in the reference): one context
 * per colony, made from per_colony[k]; pcc_batch_step advances every colony
 * by one pcc_step, spread over a pool of host threads so their kernels overlap
 * on the device, and returns when all are done (out, if given, receives n
 * stats; the first failing colony's status is returned).  pcc_batch_context
 * gives colony k's context for upload, download and queries.  Each colony
 * follows the trajectory it has alone. */
typedef struct pcc_batch pcc_batch;
pcc_status pcc_batch_create(const pcc_params* per_colony, int n, int device, pcc_batch** out);
pcc_status pcc_batch_context(pcc_batch* batch, int k, pcc_ctx** ctx);
pcc_status pcc_batch_step(pcc_batch* batch, pcc_step_stats* out);
pcc_status pcc_batch_destroy(pcc_batch* batch);

/* The CUDA stream all work of the context is queued on (a cudaStream_t). */
void* pcc_get_stream(const pcc_ctx* ctx);

/* Stage timing with CUDA events (off by default; adds no host syncs). */
pcc_status pcc_set_profiling(pcc_ctx* ctx, int on);
pcc_status pcc_reset_profile(pcc_ctx* ctx);
pcc_status pcc_get_profile(const pcc_ctx* ctx, pcc_profile* out);

/* Kernel launches issued by this context so far (for launch accounting). */
long long pcc_launch_count(const pcc_ctx* ctx);

/* Division length draw used by the device (exposed for tests): the length of
 * the left daughter of a cell of length len, for the k-th division of a
 * colony seeded with seed -- std::mt19937 seeded with pcc_division_seed(seed, k),
 * then std::uniform_real_distribution<double>(0.98*len/2, 1.02*len/2). */
unsigned int pcc_division_seed(unsigned long long seed, unsigned long long k);
double pcc_division_length_host(unsigned long long seed, unsigned long long k, double len);

#ifdef __cplusplus
}
#endif

#endif /* PCC_GPU_H */
