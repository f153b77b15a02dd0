/*
 * pot_gpu.h -- C ABI of the B200 (sm_100a) implementation of pot's
 * per-timestep particle loop.
 *
 * The reference (drewthomas/pot, pot.c) runs one time step as two C calls
 * inside run()'s loop:
 *     build_tree(Proc*, Run)                          pot.c:4308 -> 1457-1643
 *     move_particles(Proc*, Run, Tree*, ..., t)       pot.c:4386 -> 2330-2934
 * on a host array of `Particle` records (pot.c:295-303) replicated on every
 * MPI rank.  This library replaces both calls, and the MPI decomposition
 * around them, with one GPU: particles live in HBM in Morton order, and a
 * step is a fixed sequence of CUDA kernels (Morton keys, radix sort, octree
 * build, upward moments, Barnes-Hut walk fused with the Boris push,
 * grain absorption with an integer tally, boundary reinjection, grain
 * update).  The host keeps ownership of its arrays; every pointer in this
 * header is a plain host pointer.
 *
 * Every function returns POT_OK (0) or a negative POT_E_* status and never
 * aborts; the reference's fatal paths (abort() at pot.c:1651 and 1802,
 * NULL from build_tree at pot.c:1498 and 1583) map to status codes, with
 * pot_gpu_strerror() giving a message.  A context is used by one host
 * thread at a time.
 */
#ifndef POT_GPU_H
#define POT_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define POT_OK 0
#define POT_E_ARG (-1)          /* invalid argument or configuration */
#define POT_E_CUDA (-2)         /* CUDA runtime error (no device, launch failure) */
#define POT_E_NOMEM (-3)        /* device allocation failed */
#define POT_E_DOMAIN (-4)       /* particle outside the root cell: build_tree's NULL, pot.c:1491-1500 */
#define POT_E_COINCIDENT (-5)   /* two particles at one position, pot.c:1578-1586 / 1800-1802 */
#define POT_E_WALK (-6)         /* walk stack overflow, pot.c:1647-1652 */
#define POT_E_NONFINITE (-7)    /* NaN position, pot.c:1434-1446 */
#define POT_E_ITER (-8)         /* an iteration cap in a sampler was reached */
#define POT_E_CAPACITY (-9)     /* tree larger than the node arrays */
#define POT_E_STATE (-10)       /* call out of order (e.g. step before upload) */
#define POT_E_LIMIT (-11)       /* request larger than a non-allocating entry point's fixed scratch */

/* ---- records shared with the reference --------------------------------- */

/* Byte-compatible with pot.c:295-303 on x86-64 (56 bytes). */
typedef struct pot_particle {
	double x, y, z;
	double vx, vy, vz;
	int32_t species; /* 0 dust grain, 1 ion, 2 electron (pot.c:286-290) */
	int32_t pad;
} pot_particle;

/* Run settings: the reference's `Run` (pot.c:335-358, spherical domain)
   plus the compile-time switches of pot.c:25-196 that the hot path reads. */
typedef struct pot_run_cfg {
	uint64_t N;       /* particles incl. the grain at index 0 (-N) */
	uint32_t r;       /* domain radius in pixels (-r) */
	uint32_t flags;   /* POT_CFG_* */
	double dt;        /* time step, s (-d) */
	double mpp;       /* metres per pixel (-m) */
	double soft;      /* softening length, m (-s) */
	double Te, Ti;    /* injection temperatures, K (-E, -I) */
	double x_drift;   /* drift velocity along x, m/s (-x) */
	double a;         /* grain radius, m (-a) */
	double settle;    /* settling time before absorption starts, s (-e) */
	double theta;     /* opening angle OAP (pot.c:97) */
	double B[3];      /* EXTERNAL_B_X/Y/Z, tesla (pot.c:55-57) */
	double A;         /* spheroid aspect ratio (-A of pot-spheroid.c): 0 = the sphere of
	                     pot.c; > 1 prolate, in (0, 1) oblate (PROLATE / OBLATE programs,
	                     whose grain stays out of the tree and whose m_i/m_e is 1836.153) */
	double axis[3];   /* spheroid symmetry axis; zero = x, the reference's.  Any other
	                     direction tilts the grain (no counterpart in the reference) */
	double bounce;    /* OUT_BOUNCE (pot.c:113-119, 2036-2069): the domain wall's coefficient of
	                     restitution, in (0, 1]; 0 = particles that leave are reinjected (the
	                     default program) */
	uint32_t integrator;  /* POT_INT_*: the particle integrator (pot.c:121-133) */
	uint32_t pad;
} pot_run_cfg;

#define POT_CFG_SCEPTIC 0x1u        /* SCEPTIC_REINJECTION (pot.c:181): flux-weighted reinjection */
#define POT_CFG_DISABLE_GRAIN 0x2u  /* DISABLE_GRAIN (pot.c:30): no absorption */
#define POT_CFG_DIPOLES 0x4u        /* DIPOLES (pot.c:99-104): cells carry dipole moments about their
                                       centre of charge, used in fields and potentials; in the fast
                                       form with groups of at most 32 (one target per lane) */
#define POT_CFG_POIS_IONS 0x8u      /* POIS_POS_COLLECTION (pot.c:165-173, 2837-2854): absorbed ions
                                       add no charge; each step after the settling time the grain
                                       gains a Poisson number of elementary charges at the OML ion
                                       flux of the cached ion temperature (pot_gpu_set_ion_temp) */

#define POT_INT_BORIS 0u             /* BORIS (pot.c:132, 2472-2532), the default program */
#define POT_INT_VERLET 1u            /* BORIS off: velocity Verlet, two field evaluations per step
                                        (pot.c:2533-2639) */
#define POT_INT_EULER_RICHARDSON 2u  /* EULER_RICHARDSON (pot.c:127): midpoint (RK2) form */

/* Execution options (no counterpart in the reference). */
typedef struct pot_gpu_opts {
	uint32_t form;        /* POT_FORM_PLAIN or POT_FORM_FAST */
	uint32_t leaf_size;   /* particles per leaf; 1 in POT_FORM_PLAIN (the reference's tree) */
	uint32_t group_size;  /* POT_FORM_FAST: largest target group per warp: 8, 16, 32 (default) or 64;
	                         groups of at most 16 (8) share each warp between 2 (4) lanes per
	                         target, 64 puts two targets on each lane */
	uint32_t flags;       /* POT_OPT_* */
	int32_t device;       /* CUDA device ordinal */
	uint32_t chi_b_ranks; /* SCEPTIC edge potential: the mean over this many equally spaced
	                         azimuths, as a run of that many MPI ranks measures it
	                         (pot.c:2251-2279, 2409-2418); 0 or 1 = one rank, at most 64 */
	uint64_t seed;        /* key of the Philox streams used for (re)injection */
	void* stream;         /* cudaStream_t to launch on; NULL = a private stream */
} pot_gpu_opts;

#define POT_FORM_PLAIN 0u  /* FP64 walk per target, leaf size 1: the reference's arithmetic */
#define POT_FORM_FAST 1u   /* FP32 leaf-grouped warp walk, FP64 positions and push */

#define POT_OPT_TIMING 0x1u  /* record CUDA events around each kernel (pot_gpu_kernel_times) */
/* SCEPTIC reinjection with the edge potential capped (no counterpart in the
   reference): the speed sampler is given min(chi, 0.95 chi*) for each
   species, chi* = U^2 + 1/2 + U exp(-U^2) / (sqrt(pi) erf(U)) (1 as U -> 0),
   U its drift in units of its normalisation speed.  Above chi* the
   reference's inverse CDF is NaN for every draw (its normaliser vanishes
   there, prng.c:171-214) and sceptically_reinject retries without end
   (pot.c:582-599); a noisy single-point edge potential of a small grain in
   cold ions can read that high.  Off, such a run stops with POT_E_ITER and
   warn bit 64 (the reference's behaviour made finite); on, it goes on and
   sets warn bit 512 (kept, like the other warn bits) once the cap has
   applied.  A run whose edge potential stays below the cap gives the same
   results either way. */
#define POT_OPT_CHI_CAP 0x2u

/* Grain state: the reference keeps it in Proc (pot.c:370-371, 397) and in
   parts[0] (pot.c:890-899). */
typedef struct pot_grain_state {
	int64_t q;            /* net charge, elementary charges (Proc.dust_grain_q) */
	double m;             /* mass, kg (Proc.dust_grain_m) */
	double x, y, z;       /* position, m */
	double vx, vy, vz;    /* velocity, m/s */
	uint64_t tot_absor_e; /* electrons absorbed so far (Proc.tot_absor_e) */
	uint64_t t_steps;     /* steps taken so far (Proc.t_steps) */
	double chi_b;         /* normalised edge potential (Proc.chi_b, SCEPTIC) */
} pot_grain_state;

/* Per-step results, written by pot_gpu_step for the last step it ran. */
typedef struct pot_step_stats {
	uint64_t t_steps;      /* step index after the step */
	int64_t grain_q;       /* grain charge after the step */
	int64_t dq;            /* charge absorbed this step (pot.c:2663) */
	uint64_t de;           /* electrons absorbed this step */
	uint64_t n_absorbed;   /* particles absorbed this step */
	uint64_t n_reinjected; /* reinjections this step (absorption + boundary) */
	uint64_t n_pushed;     /* particles advanced this step */
	uint64_t interactions; /* cell + pair terms evaluated for each target this step */
	uint64_t n_nodes;      /* internal tree nodes this step */
	double chi_b;          /* edge potential in force after the step */
	int32_t status;        /* POT_OK or the first device-side error */
	uint32_t stack_max;    /* fast form: deepest per-warp walk stack this step
	                          (POT_WALK_STACK entries at most; 0 in the plain form) */
	double epe[3];         /* POT_STEP_EPE: electrostatic potential energy (J) of the
	                          grain, the ions, the electrons (Proc.epe, pot.c:2771-2864) */
	int64_t q_sum;         /* sum of the grain charge after each step since upload / init
	                          (moving means of the charge; no counterpart in the reference) */
	uint32_t warn;         /* non-fatal conditions and causes: bit 0 a leaf-size-1 key
	                          collision at 21 levels (an overflow bucket); with POT_E_ITER,
	                          the sampler cap reached: 2 inverse-CDF Newton, 4 the u^2 <
	                          chi_b rejection, 8 NaN-alpha retries, 16 orbit-integral
	                          halvings, 32 the initial shell radius, 64 no speed
	                          distribution for the edge potential (the reference's inverse
	                          CDF is NaN there and it retries without end); 128 a particle in
	                          the domain wall moving inwards (OUT_BOUNCE, the reference's
	                          warning at pot.c:2719-2722); 256 the Poisson variate's cap;
	                          512 POT_OPT_CHI_CAP capped the edge potential for the sampler */
	uint32_t n_collected;  /* POT_CFG_POIS_IONS: charges the Poisson ion collection added */
	uint32_t n_wall;       /* OUT_BOUNCE: particles found outside moving inwards, left in place */
	uint32_t n_bounced;    /* OUT_BOUNCE: particles bounced off the wall */
	uint32_t n_groups;     /* fast form: target groups the walk ran this step, one warp each
	                          (n_pushed / n_groups targets per group on average); 0 in the plain form */
	uint32_t pad;
	uint64_t far_cells;    /* fast form: accepted cells far from their group that were expanded
	                          once about the group's centre instead of evaluated for each target
	                          (not counted in interactions); 0 in the plain form */
} pot_step_stats;

/* capacity of the fast form's per-warp stack of cells awaiting a test;
   a walk that needs more fails with POT_E_WALK */
#define POT_WALK_STACK 1536

/* pot_gpu_step flags */
#define POT_STEP_EPE 0x1u  /* compute the potential energies (pot.c:2771-2804) */

typedef struct pot_gpu_ctx pot_gpu_ctx;

/* ---- life cycle -------------------------------------------------------- */

/* Allocate device state for one run of cfg->N particles.  Replaces the
   allocations of main() and run() (pot.c:5117-5130, 4115-4146). */
int pot_gpu_create(const pot_run_cfg* cfg, const pot_gpu_opts* opts, pot_gpu_ctx** out);
void pot_gpu_destroy(pot_gpu_ctx* ctx);
const char* pot_gpu_strerror(int status);

/* Copy a host particle array (reference order: grain, ions, electrons) and
   the grain state to the device.  Replaces the per-step MPI_Bcast of all
   particles (pot.c:4299).  grain may be NULL (charge 0, mass 1.67e-12 kg,
   t_steps 0, as main() starts a run, pot.c:5184-5190). */
int pot_gpu_upload(pot_gpu_ctx* ctx, const pot_particle* parts, uint64_t N,
                   const pot_grain_state* grain);

/* init_particles (pot.c:887-996) on the device: grain at the centre,
   (N-1)/2 ions then electrons, positions uniform in the shell a < r < R,
   Maxwellian velocities, each particle drawing from its own Philox stream. */
int pot_gpu_init_particles(pot_gpu_ctx* ctx);

/* Run nsteps steps (each: t_steps++, build_tree, move_particles).  `flags`:
   POT_STEP_EPE also evaluates every particle's potential energy over the
   step's tree (compute_epe of move_particles, pot.c:2771-2804, with each
   particle at its step-start position).  `out` (may be NULL) receives the
   last step's stats. */
int pot_gpu_step(pot_gpu_ctx* ctx, uint32_t nsteps, uint32_t flags, pot_step_stats* out);

/* Enqueue nsteps steps on the context's stream and return without waiting.
   Device-side errors surface at the next pot_gpu_sync / pot_gpu_step /
   pot_gpu_download, which return the first status recorded. */
int pot_gpu_step_async(pot_gpu_ctx* ctx, uint32_t nsteps, uint32_t flags);

/* Copy particles back in reference order (index = original position), and
   the grain state.  Either pointer may be NULL. */
int pot_gpu_download(pot_gpu_ctx* ctx, pot_particle* parts, pot_grain_state* grain);

/* Drop-in for one iteration of run()'s hot path (pot.c:4299-4386): upload
   `parts` (N records, reference order) and `grain`, t_steps++, build the
   tree, move the particles, download both back into the same arrays.  The
   transfers run in chunks that overlap the conversions (page-locked host
   memory lets them overlap the most).  Only the records the step can have
   changed are copied back: the grain's and the contiguous range of
   reference indices holding every particle due this step (species s is due
   when t_steps % tss[s] == 0); the records outside it are neither pushed
   nor reinjected and keep their values.  On an error status the particles
   in that range hold the device's state at the failure (kernels skip their
   work once a status is set) and `grain` is left as passed. */
int pot_gpu_move_particles(pot_gpu_ctx* ctx, pot_particle* parts, uint64_t N,
                           pot_grain_state* grain, pot_step_stats* out);

/* ---- inspection (parity tests) ----------------------------------------- */

/* Build the tree from the current device particles without stepping
   (build_tree, pot.c:1457-1643).  Returns the number of internal nodes in
   *n_nodes. */
int pot_gpu_build_tree(pot_gpu_ctx* ctx, uint64_t* n_nodes);

/* Canonical dump of the last tree built: internal nodes and leaves, each
   labelled by (level, octal-digit path from the root); the same format as
   the oracle's dump of the reference's pointer tree.  Leaves report the
   original particle index of each occupant (leaf_size 1). */
int pot_gpu_tree_dump(pot_gpu_ctx* ctx, uint64_t max_nodes,
                      uint64_t* n_int, int32_t* int_level, uint64_t* int_path, int32_t* int_q,
                      uint32_t* int_aq, double* int_c, double* int_w,
                      uint64_t* n_leaf, uint32_t* leaf_part, int32_t* leaf_level,
                      uint64_t* leaf_path);

/* E field (V/m) at n points xyz[3k..3k+2], each for the target particle
   with original index idx[k] (excluded from its own field), over the last
   tree built: field_particle_feels_at (pot.c:1696-1808) for many targets. */
int pot_gpu_field_at(pot_gpu_ctx* ctx, uint64_t n, const uint32_t* idx, const double* xyz,
                     double* E);

/* pot_gpu_field_at without allocation (no counterpart in the reference,
   which has no device memory).  For callers that must not allocate device
   memory while they run, e.g. a host program that owns the device heap
   through its own pool, or a step loop in which cudaMalloc is not allowed.
   The staging buffers live in one fixed array of about 3.5 MiB that every
   device which loads the library holds until the process exits; hence at
   most POT_NOALLOC_MAX_POINTS points per call, larger n returns
   POT_E_LIMIT.  The first call on each device looks the array's device
   address up and keeps it (make that call before any stream capture); the
   kept address is valid while the device's primary context lives, so a
   program that calls cudaDeviceReset must not call this function again.
   All calls on a device share the array: calls whose work overlaps on the
   GPU race. */
#define POT_NOALLOC_MAX_POINTS 65536u
int pot_gpu_field_at_noalloc(pot_gpu_ctx* ctx, uint64_t n, const uint32_t* idx, const double* xyz,
                             double* E);

/* Potential (V) at n points over the last tree built, every particle
   included: phi_at (pot.c:1818-1901). */
int pot_gpu_phi_at(pot_gpu_ctx* ctx, uint64_t n, const double* xyz, double* phi);

/* Accumulated per-kernel device time since creation or the last reset
   (requires POT_OPT_TIMING).  Writes up to `max` entries; returns the count
   of kernels known (names are static strings). */
int pot_gpu_kernel_times(pot_gpu_ctx* ctx, int max, const char** names, double* ms,
                         uint64_t* launches);
int pot_gpu_reset_kernel_times(pot_gpu_ctx* ctx);

/* Number of CUDA kernels this context has enqueued since creation. */
int pot_gpu_launch_count(pot_gpu_ctx* ctx, uint64_t* n);

/* Block the calling thread until all work queued on the context's stream
   has finished; returns the first device-side status seen. */
int pot_gpu_sync(pot_gpu_ctx* ctx);

/* Sums behind the macroscopic summary (write_macroscopic_data_to_file,
   pot.c:3261-3508) over the plasma particles of the current state, in two
   passes like the reference's, without downloading the particles.  FP64
   with a fixed summation order (the reference uses long double). */
typedef struct pot_macro_sums {
	/* pass 1 */
	double n_e, n_i;          /* electrons, ions */
	double K_e;               /* sum 0.5 m_e |v|^2, electrons */
	double s_e, s_i;          /* sum |v| */
	double v_e[3], v_i[3];    /* sum v */
	double am_e[3], am_i[3];  /* sum (r - c) x v, c the domain centre (times the mass gives the
	                             angular momentum) */
	double pad1[3];
	/* pass 2, about the pass-1 means */
	double sumsq_K_e, sum_x_e, sumsq_x_e;
	double K_e_c[3];          /* sum (K - <K>)^k, k = 2, 3, 4, electrons */
	double s_e_c[3];          /* sum (|v| - <|v|>)^k, k = 2, 3, 4, electrons */
	double T_e;               /* sum |v - <v>|^2, electrons */
	double sum_K_i, sumsq_K_i;
	double s_i_c[3];          /* sum (|v| - <|v|>)^k, k = 2, 3, 4, ions */
	double T_i;               /* sum |v - <v>|^2, ions */
	double pad2[2];
} pot_macro_sums;

int pot_gpu_macro(pot_gpu_ctx* ctx, pot_macro_sums* out);

/* The grain's state alone (pot_gpu_download without the particles). */
int pot_gpu_grain(pot_gpu_ctx* ctx, pot_grain_state* grain);

/* POT_CFG_POIS_IONS: the cached ion temperature (Proc.Ti, K) that sets the
   collection rate.  It starts at cfg->Ti (pot.c:4252); pot_gpu_macro
   replaces it with the ions' measured temperature, as the reference's
   macroscopic summary does (pot.c:3442-3448); a caller that computes the
   summary itself sets it here. */
int pot_gpu_set_ion_temp(pot_gpu_ctx* ctx, double Ti);
int pot_gpu_ion_temp(pot_gpu_ctx* ctx, double* Ti);

/* Device bytes a context with these settings allocates (no device work). */
int pot_gpu_bytes_needed(const pot_run_cfg* cfg, const pot_gpu_opts* opts, uint64_t* bytes);

/* ---- batches of independent runs ---------------------------------------
   No counterpart in the reference, which runs one grain per MPI job.  A
   batch holds many runs (each its own context) and advances all of them
   with one CUDA-graph launch per `steps_per_launch` steps; runs are admitted
   while free HBM allows and evicted when done.  Fast-form Boris runs with
   the same group size and key depth are packed: each kernel of their step
   is one launch over all of them (a grid shared out by run size, the walk
   one persistent launch over every run's target groups).  Other runs step
   as their own kernel sequences in the same graph.  Runs share no state:
   each result is bit-identical to the same run stepped alone. */
typedef struct pot_batch pot_batch;

#define POT_BATCH_NO_PACK 0x1u  /* step every run as its own kernel sequence */

typedef struct pot_batch_opts {
	int32_t device;
	uint32_t steps_per_launch;  /* steps per graph launch, even; 0 = 2 */
	uint64_t reserve_bytes;     /* HBM left free when admitting */
	uint32_t flags;             /* POT_BATCH_* */
	uint32_t pad;
} pot_batch_opts;

/* One member's state, gathered on the device for the whole batch. */
typedef struct pot_batch_row {
	int32_t slot;
	int32_t status;
	uint64_t t_steps;
	int64_t grain_q;
	int64_t q_sum;        /* sum of the grain charge after each step since upload/init */
	uint64_t tot_absor_e;
	uint64_t particles;
	uint32_t warn;        /* as pot_step_stats.warn */
	uint32_t pad;
} pot_batch_row;

int pot_batch_create(const pot_batch_opts* opts, pot_batch** out);
void pot_batch_destroy(pot_batch* b);
/* Admit a run: POT_E_NOMEM (nothing allocated) when its device state would
   leave less than reserve_bytes of HBM free.  parts == NULL initialises
   the particles as pot_gpu_init_particles does; else they are uploaded
   with `grain`.  Writes the run's slot id. */
int pot_batch_admit(pot_batch* b, const pot_run_cfg* cfg, const pot_gpu_opts* opts, const pot_particle* parts,
                    const pot_grain_state* grain, int32_t* slot);
int pot_batch_evict(pot_batch* b, int32_t slot);
/* Enqueue nsteps (a multiple of steps_per_launch) for every member. */
int pot_batch_step(pot_batch* b, uint32_t nsteps);
int pot_batch_sync(pot_batch* b);
/* Members' current state (synchronises). */
int pot_batch_summary(pot_batch* b, uint32_t max, pot_batch_row* rows, uint32_t* n_rows);
int pot_batch_count(pot_batch* b, uint32_t* runs, uint64_t* particles, uint64_t* bytes);
/* A member's own context (after the batch's queued work), for downloads
   and queries; stepping it directly is allowed (the batch re-captures). */
int pot_batch_ctx(pot_batch* b, int32_t slot, pot_gpu_ctx** ctx);

/* Autotuner: time `steps` steps of each candidate (leaf size, group size)
   of the fast form -- (8, 32), (16, 32), (32, 32), (16, 64), (32, 64) -- on
   one run of cfg (created once, its particles initialised again for each
   candidate) and write the fastest into opts (its ms per step into
   *ms_per_step). */
int pot_gpu_tune(const pot_run_cfg* cfg, pot_gpu_opts* opts, uint32_t steps, double* ms_per_step);

#ifdef __cplusplus
}
#endif

#endif
