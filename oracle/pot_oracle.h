/*
 * CPU oracle for pot's per-timestep particle loop -- TEST INFRASTRUCTURE.
 *
 * A plain-C restatement of the reference's algorithm (pot.c, prng.c,
 * coord.c of drewthomas/pot), used only by tests/, __graft_entry__.smoke()
 * and the CPU-baseline leg of bench.py as the checker.  The GPU product path
 * never links, loads or calls it.
 *
 * Parity pin: the restatement is checked against the reference program
 * itself (compiled by oracle/build.py into oracle/_ref/) and against the
 * golden vectors that tests/golden/make_golden.py wrote from it.
 *
 * Two modes per run:
 *   reference mode  (quirk = 1, rng = WELL512): the reference's own loop
 *                   order, including its in-place half-drift (pot.c:2478-2485)
 *                   that lets later targets see earlier targets at their
 *                   half-drifted positions, and its single sequential WELL512
 *                   stream (prng.c:11-28);
 *   GPU semantics   (quirk = 0, rng = PHILOX): every target sees the tree's
 *                   pre-step sources, and every reinjection draws from a
 *                   Philox4x32-10 counter stream keyed by (seed, particle id,
 *                   step, attempt), as the CUDA kernels do.
 */
#ifndef POT_ORACLE_H
#define POT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Particle record, byte-compatible with pot.c:295-303 on x86-64 (56 B). */
typedef struct pto_particle {
	double x, y, z, vx, vy, vz;
	int32_t species; /* 0 dust, 1 ion, 2 electron */
	int32_t pad;
} pto_particle;

/* WELL512 state, byte-compatible with prng.h:17-24 (84 B). */
typedef struct pto_well {
	uint32_t a, b, c, d, index;
	uint32_t state[16];
} pto_well;

typedef struct pto_cfg {
	uint64_t N;       /* particles incl. the grain at index 0 */
	uint32_t r;       /* domain radius, pixels */
	double dt;        /* base time step, s */
	double mpp;       /* metres per pixel */
	double soft;      /* softening length, m */
	double Te, Ti;    /* injection temperatures, K */
	double x_drift;   /* drift velocity along x, m/s */
	double a;         /* grain radius, m */
	double settle;    /* settling time before absorption, s */
	double theta;     /* opening angle (OAP) */
	double B[3];      /* external magnetic field, T */
	int32_t sceptic;  /* 1: flux-weighted (SCEPTIC) reinjection */
	int32_t quirk;    /* 1: reference in-place half-drift ordering */
	int32_t rng;      /* 0: WELL512 stream, 1: Philox counter stream */
	int32_t pad;
	uint64_t seed;    /* Philox key (rng = 1) */
	/* grain shape: 0 the sphere of pot.c; 1 prolate, 2 oblate spheroid of
	   pot-spheroid.c (PROLATE / OBLATE), which also bring that program's
	   constants (m_i/m_e = 1836.153, SCEPTIC max_lin_dev = 0.1) and keep the
	   grain out of the tree */
	int32_t shape;
	int32_t chi_ranks; /* chi_b as the mean over this many ranks' azimuths (0/1 = one) */
	double A;         /* aspect ratio (pot-spheroid.c -A) */
	double axis[3];   /* symmetry axis, unit vector; (1, 0, 0) in the reference,
	                     anything else is an extension (unpinned) */
	/* the reference's other compile-time variants (pot.c:99-196), off = 0 */
	double bounce;      /* OUT_BOUNCE (pot.c:113-119): the domain wall's coefficient of
	                       restitution; 0 = reinject particles that leave */
	int32_t integrator; /* 0 Boris (BORIS), 1 velocity Verlet (BORIS off), 2 Euler-Richardson
	                       (EULER_RICHARDSON), pot.c:121-133 */
	int32_t dipoles;    /* DIPOLES (pot.c:99-104): cell dipole moments in fields and potentials */
	int32_t pois_ions;  /* POIS_POS_COLLECTION (pot.c:165-173): absorbed ions add no charge; the
	                       grain gains a Poisson number of elementary charges each step */
	int32_t pad2;
} pto_cfg;

typedef struct pto_ctx pto_ctx;

pto_ctx* pto_create(const pto_cfg* cfg);
void pto_destroy(pto_ctx* c);
int pto_sizeof_particle(void);
void pto_get_tss(const pto_ctx* c, uint32_t* out3);

void pto_set_particles(pto_ctx* c, const pto_particle* in);
void pto_get_particles(const pto_ctx* c, pto_particle* out);
void pto_set_well(pto_ctx* c, const pto_well* w);
void pto_get_well(const pto_ctx* c, pto_well* w);
void pto_seed_well(pto_ctx* c, const uint32_t* seed16);
void pto_set_grain(pto_ctx* c, int32_t q, double m, uint32_t tot_absor_e, uint64_t t_steps, double chi_b);
void pto_get_grain(const pto_ctx* c, int32_t* q, double* m, uint32_t* tot_absor_e, uint64_t* t_steps,
                   double* chi_b, double* grain_v3);

int pto_init_particles(pto_ctx* c);
int pto_build_tree(pto_ctx* c);
int pto_tree_dump(const pto_ctx* c, uint64_t max_nodes,
                  uint64_t* n_int, int32_t* int_level, uint64_t* int_path, int32_t* int_q,
                  uint32_t* int_aq, double* int_c, double* int_w,
                  uint64_t* n_leaf, uint32_t* leaf_part, int32_t* leaf_level, uint64_t* leaf_path);
/* DIPOLES: the internal nodes' dipole moments (3 per node) in pto_tree_dump's order */
int64_t pto_tree_dipoles(const pto_ctx* c, uint64_t max_nodes, double* int_p);
void pto_field_many(const pto_ctx* c, uint64_t n, const uint32_t* idx, const double* xyz,
                    double* hi, double* lo);
void pto_field_direct_many(const pto_ctx* c, uint64_t n, const uint32_t* idx, const double* xyz,
                           int32_t soften_all, double* hi, double* lo);
double pto_phi_at(const pto_ctx* c, double x, double y, double z);
double pto_phi_particle_feels(const pto_ctx* c, uint32_t part);
int pto_cross_grain(const pto_particle* p, const double* d_pos, const pto_particle* gr, double a);
/* the run's absorption test (sphere, or the spheroid of its shape) */
int pto_cross_grain_run(const pto_ctx* c, const pto_particle* p, const double* d_pos, const pto_particle* gr);
/* the spheroid's own field and potential at a point (grain charge and
   position of the run), pot-spheroid.c:1689-1779 and 2037-2085 */
void pto_grain_field(const pto_ctx* c, double x, double y, double z, double* E3);
double pto_grain_phi(const pto_ctx* c, double x, double y, double z);
double pto_measure_chi_b(const pto_ctx* c);
/* the mean of measure_chi_b over P ranks' azimuths 2 pi k / P (pot.c:2268, 2409-2418) */
double pto_measure_chi_b_ranks(const pto_ctx* c, int32_t P);
/* POIS_POS_COLLECTION: the cached ion temperature (Proc.Ti) that sets the
   collection rate; the run's Ti at set-up (pot.c:4252), then whatever the
   macroscopic summary last measured (pot.c:3444-3448) */
void pto_set_ion_temp(pto_ctx* c, double Ti);
double pto_ion_temp(const pto_ctx* c);
/* Poisson variate of prng.c:50-70 on the context's stream, for tests */
uint32_t pto_poisson(pto_ctx* c, double lambda);

/* One step: t_steps++, build the tree, move the particles (pot.c:4261-4386).
   Returns 0, or a negative status (tree build failure). */
int pto_step(pto_ctx* c, int32_t compute_epe);
int pto_run_steps(pto_ctx* c, uint64_t n, int32_t compute_epe);
void pto_last_step_stats(const pto_ctx* c, int64_t* dq, uint32_t* de, uint32_t* n_absorbed,
                         uint32_t* n_reinjected, uint64_t* n_pushed, double* epe3);
/* charges added by the Poisson ion collection, and particles found in the
   wall moving inwards (OUT_BOUNCE), in the last step */
void pto_last_step_variant_stats(const pto_ctx* c, uint32_t* n_pois, uint32_t* n_wall);

/* Reinjection sampler, for distribution tests: n draws of `species` through
   inject(reinjection = 1) on the context's RNG; out holds n particles. */
void pto_sample_reinject(pto_ctx* c, uint64_t n, int32_t species, pto_particle* out);
double pto_u_icdf(double U, double chi, double q);
double pto_u_no_flow_icdf(double chi, double q);
double pto_integrate_for_alpha(double s, double chi_b, double u2, double Rol);
double pto_integrate_for_alpha_dev(double s, double chi_b, double u2, double Rol, double max_lin_dev);

/* Philox4x32-10 block function (Salmon et al., SC'11), for RNG tests. */
void pto_philox4x32(const uint32_t* ctr4, const uint32_t* key2, uint32_t* out4);

#ifdef __cplusplus
}
#endif

#endif
