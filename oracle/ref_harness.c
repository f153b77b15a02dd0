/*
 * Test-infrastructure harness around the reference program (never part of
 * the GPU product path).  It #includes a flag-patched copy of the reference
 * pot.c (written by oracle/build.py into oracle/_ref/src_<variant>/) with
 * `main` renamed, and exports plain C entry points so that the tests and the
 * CPU-baseline leg of bench.py can call the reference's own functions on a
 * chosen particle snapshot:
 *   build_tree            pot.c:1457-1643
 *   field_particle_feels_at pot.c:1696-1808
 *   phi_at                pot.c:1818-1901
 *   phi_particle_feels    pot.c:1934-2018
 *   does_particle_cross_grain pot.c:2287-2325
 *   move_particles        pot.c:2330-2934
 *   inject / init_particles pot.c:658-846 / 887-996
 *   measure_chi_b         pot.c:2251-2279 (SCEPTIC variant)
 * The spheroid variants include pot-spheroid.c instead (same entry points;
 * grain field pot-spheroid.c:1689-1779, absorption 2448-2537).
 * Process set-up mirrors what main() and run() do for a single rank
 * (pot.c:4998-5190 and pot.c:4115-4159), without the output writers.
 */
#include "pot.c"

double pot_ref_oap = 0.5;
double pot_ref_bx = 0.0;
double pot_ref_by = 0.0;
double pot_ref_bz = 0.0;
static double pot_ref_aspect = 3.0;  /* Run.A of pot-spheroid.c (pot-spheroid.c:376-378) */

#if defined(PROLATE) || defined(OBLATE)
#define H_SPHEROID 1
#else
#define H_SPHEROID 0
#endif

/* 0 sphere (pot.c), 1 prolate, 2 oblate (pot-spheroid.c) */
int potref_shape(void)
{
#if defined(PROLATE)
	return 1;
#elif defined(OBLATE)
	return 2;
#else
	return 0;
#endif
}

/* the other variant switches compiled in: 1 DIPOLES, 2 OUT_BOUNCE,
   4 POIS_POS_COLLECTION, 8 BORIS off (velocity Verlet), 16 EULER_RICHARDSON */
int potref_variant_flags(void)
{
	int f = 0;
#ifdef DIPOLES
	f |= 1;
#endif
#ifdef OUT_BOUNCE
	f |= 2;
#endif
#ifdef POIS_POS_COLLECTION
	f |= 4;
#endif
#ifndef BORIS
	f |= 8;
#endif
#ifdef EULER_RICHARDSON
	f |= 16;
#endif
	return f;
}

#ifdef OUT_BOUNCE
double potref_bounce(void) { return OUT_BOUNCE; }
#else
double potref_bounce(void) { return 0.0; }
#endif

/* 1 when the grain absorbs (DISABLE_GRAIN off), 0 otherwise */
int potref_grain_enabled(void)
{
#ifdef DISABLE_GRAIN
	return 0;
#else
	return 1;
#endif
}

/* aspect ratio for the next potref_setup (spheroid variants) */
void potref_set_aspect(double A) { pot_ref_aspect = A; }

static Proc H;
static Run R;
static int H_ready = 0;
static MPI_Datatype H_mpi_particle = 56;

int potref_sizeof_particle(void) { return (int) sizeof(Particle); }
int potref_sizeof_prng(void) { return (int) sizeof(PRNG); }
int potref_has_sceptic(void)
{
#ifdef SCEPTIC_REINJECTION
	return 1;
#else
	return 0;
#endif
}

static void h_free(void)
{
	if (!H_ready) return;
	free(H.parts);
	free(H.new_parts);
	free(H.a_x1);
	free(H.prev_x);
	free(H.root);
	free(H.starts);
	free(H.pits[0]);
	free(H.pits);
	memset(&H, 0, sizeof(H));
	H_ready = 0;
}

/* Set up one rank's Proc/Run exactly as main() + run() do for a new run.
   `init` != 0 also calls init_particles (pot.c:5211). Returns 0 on success. */
int potref_setup(unsigned long N, unsigned int r, double dt, double mpp, double soft,
                 double Te, double Ti, double x_drift, double a, double settle,
                 double oap, double bx, double by, double bz,
                 const uint32_t* seed16, int init, int nprocs, int rank)
{
	h_free();
	memset(&R, 0, sizeof(R));
	R.N = N;
	R.r = r;
	R.dt = dt;
	R.mpp = mpp;
	R.run_for = 0;
	R.soft = soft;
	R.x_drift = x_drift;
	R.a = a;
	R.settle = settle;
	R.sw_path = NULL;
	R.sr_path = NULL;
	R.tim_lim = 0.0;
	R.Te = Te;
	R.Ti = Ti;
#if H_SPHEROID
	R.A = pot_ref_aspect;
#else
	R.read_out = false;
#endif
	pot_ref_oap = oap;
	pot_ref_bx = bx;
	pot_ref_by = by;
	pot_ref_bz = bz;

	memset(&H, 0, sizeof(H));
	/* One rank of an nprocs-rank run: the block decomposition of
	   set_up_workers_for_assignments (pot.c:2936-2998) and the per-block
	   species layout of init_particles (pot.c:908-930) are the reference's;
	   MPI traffic is absent, so this rank steps only its own block. */
	H.rank = rank;
	H.num_procs = nprocs > 0 ? nprocs : 1;
	if (set_up_workers_for_assignments(&H, R)) return -1;
	H.parts = malloc(sizeof(Particle) * N);
	H.new_parts = malloc(sizeof(Particle) * N);
	H.a_x1 = malloc(3 * sizeof(long double) * N);
	H.prev_x = malloc(3 * sizeof(double) * N);
	H.tr_alloc = 9 * N;
	H.root = malloc(sizeof(Tree) * H.tr_alloc);
	H.starts = malloc(sizeof(unsigned int) * (H.num_procs > 0 ? H.num_procs : 1));
	if (!H.parts || !H.new_parts || !H.a_x1 || !H.prev_x || !H.root || !H.starts) return -2;
	H.a_y1 = &(H.a_x1[N]);
	H.a_z1 = &(H.a_x1[2 * N]);
	H.prev_y = &(H.prev_x[N]);
	H.prev_z = &(H.prev_x[2 * N]);
	memset(H.parts, 0, sizeof(Particle) * N);
	memset(H.new_parts, 0, sizeof(Particle) * N);
	init_prng(&(H.ps), (uint32_t*) seed16);
	H.t_steps = 0;
	H.tot_absor_e = 0;
	H.dust_grain_q = CHARGE[DUST];
	H.dust_grain_m = MASS[DUST];
#ifdef SCEPTIC_REINJECTION
	H.chi_b = 0.0;
#endif
	/* time-step multiples per species, pot.c:4157-4159 */
	H.tss[ELECTRON] = 1;
	H.tss[ION] = (int) sqrt(R.Te * MASS[ION] / (R.Ti * MASS[ELECTRON]));
	H.tss[DUST] = H.tss[ION] * (int) sqrt(0.1 * MASS[DUST] / MASS[ION]);
#ifdef POIS_POS_COLLECTION
	/* run()'s set-up of the Poisson collection (pot.c:4251-4255) */
	H.Ti = R.Ti;
	H.pos_rate_const = 4.0 * PI * R.a * R.a * CHARGE[ION];
	H.pos_rate_const /= sqrt(2.0 * PI * MASS[ION]);
	H.pos_rate_const *= R.dt * total_number_density(R) / 2.0;
#endif
	H_ready = 1;
	if (init) init_particles(&H, R);
	return 0;
}

void potref_free(void) { h_free(); }

#ifdef POIS_POS_COLLECTION
/* Proc.Ti, the cached ion temperature of the Poisson collection rate */
void potref_set_ion_temp(double Ti) { H.Ti = Ti; }
double potref_ion_temp(void) { return H.Ti; }
double potref_pos_rate_const(void) { return H.pos_rate_const; }
#endif

void potref_get_tss(unsigned int* out3) { out3[0] = H.tss[0]; out3[1] = H.tss[1]; out3[2] = H.tss[2]; }

void potref_get_particles(Particle* out) { memcpy(out, H.parts, sizeof(Particle) * R.N); }
void potref_set_particles(const Particle* in) { memcpy(H.parts, in, sizeof(Particle) * R.N); }
void potref_get_prng(PRNG* out) { *out = H.ps; }
void potref_set_prng(const PRNG* in) { H.ps = *in; }

void potref_get_grain(int* q, double* m, unsigned int* tot_absor_e, unsigned long* t_steps, double* chi_b)
{
	*q = H.dust_grain_q;
	*m = (double) H.dust_grain_m;
	*tot_absor_e = H.tot_absor_e;
	*t_steps = H.t_steps;
#ifdef SCEPTIC_REINJECTION
	*chi_b = H.chi_b;
#else
	*chi_b = 0.0;
#endif
}

void potref_set_grain(int q, double m, unsigned int tot_absor_e, unsigned long t_steps, double chi_b)
{
	H.dust_grain_q = q;
	H.dust_grain_m = m;
	H.tot_absor_e = tot_absor_e;
	H.t_steps = t_steps;
#ifdef SCEPTIC_REINJECTION
	H.chi_b = chi_b;
#else
	(void) chi_b;
#endif
}

/* Returns 0, or -1 when the reference's build_tree returned NULL. */
int potref_build_tree(void) { return build_tree(&H, R) == NULL ? -1 : 0; }

/* Child slot order of the reference's Tree record, mapped to the octal digit
   (bx << 2) | (by << 1) | bz, bit = 1 for the "greater" half. */
static const int SLOT_DIGIT[8] = { 4, 5, 0, 1, 2, 3, 6, 7 };

static unsigned int slot_child(const Tree* t, int s)
{
	switch (s) {
	case 0: return t->gxlylz;
	case 1: return t->gxlygz;
	case 2: return t->lxlylz;
	case 3: return t->lxlygz;
	case 4: return t->lxgylz;
	case 5: return t->lxgygz;
	case 6: return t->gxgylz;
	default: return t->gxgygz;
	}
}

/* Canonical dump of the tree just built: internal nodes (those with
   children) and occupied leaves, each labelled by (level, octal-digit path).
   Arrays are sized by the caller (at most tr_alloc entries each).
   Returns 0 or -1 when an array would overflow or the tree is too deep. */
int potref_tree_dump(unsigned long max_nodes,
                     unsigned long* n_int, int* int_level, unsigned long long* int_path,
                     int* int_q, unsigned int* int_aq, double* int_c /* 3 per node */,
                     double* int_w /* x2-x1 */,
                     unsigned long* n_leaf, unsigned int* leaf_part, int* leaf_level,
                     unsigned long long* leaf_path)
{
	unsigned int stack_node[1024];
	int stack_level[1024];
	unsigned long long stack_path[1024];
	int sp = 0;
	unsigned long ni = 0, nl = 0;
	stack_node[0] = 0; stack_level[0] = 0; stack_path[0] = 0ULL; sp = 1;
	while (sp) {
		sp--;
		unsigned int nd = stack_node[sp];
		int lev = stack_level[sp];
		unsigned long long path = stack_path[sp];
		const Tree* t = &(H.root[nd]);
		if (t->part != UINT_MAX) {
			if (nl >= max_nodes) return -1;
			leaf_part[nl] = t->part; leaf_level[nl] = lev; leaf_path[nl] = path; nl++;
		} else if (t->gxlylz) {
			if (ni >= max_nodes || lev >= 21 || sp + 8 > 1024) return -1;
			int_level[ni] = lev; int_path[ni] = path; int_q[ni] = t->q; int_aq[ni] = t->aq;
			int_c[3 * ni] = t->cx; int_c[3 * ni + 1] = t->cy; int_c[3 * ni + 2] = t->cz;
			int_w[ni] = t->x2 - t->x1;
			ni++;
			for (int s = 0; s < 8; s++) {
				stack_node[sp] = slot_child(t, s);
				stack_level[sp] = lev + 1;
				stack_path[sp] = (path << 3) | (unsigned long long) SLOT_DIGIT[s];
				sp++;
			}
		}
	}
	*n_int = ni;
	*n_leaf = nl;
	return 0;
}

#ifdef DIPOLES
/* Dipole moments (px, py, pz) of the internal nodes, in the order of
   potref_tree_dump.  Returns the node count or -1. */
long potref_tree_dipoles(unsigned long max_nodes, double* int_p)
{
	unsigned int stack_node[1024];
	int stack_level[1024];
	int sp = 1;
	unsigned long ni = 0;
	stack_node[0] = 0;
	stack_level[0] = 0;
	while (sp) {
		sp--;
		const Tree* t = &(H.root[stack_node[sp]]);
		const int lev = stack_level[sp];
		if (t->part == UINT_MAX && t->gxlylz) {
			if (ni >= max_nodes || lev >= 21 || sp + 8 > 1024) return -1;
			int_p[3 * ni] = t->px;
			int_p[3 * ni + 1] = t->py;
			int_p[3 * ni + 2] = t->pz;
			ni++;
			for (int s = 0; s < 8; s++) {
				stack_node[sp] = slot_child(t, s);
				stack_level[sp] = lev + 1;
				sp++;
			}
		}
	}
	return (long) ni;
}
#endif

static void split_ld(long double v, double* hi, double* lo)
{
	*hi = (double) v;
	*lo = (double) (v - (long double) *hi);
}

/* E field (V/m) at (x, y, z) for target `part`, pot.c:1696-1808, returned
   as a double-double split of the reference's long double accumulators. */
void potref_field_at(unsigned int part, double x, double y, double z, double* hi3, double* lo3)
{
	long double E[3];
	field_particle_feels_at(part, &H, &R, x, y, z, E, H.root);
	for (int k = 0; k < 3; k++) split_ld(E[k], &hi3[k], &lo3[k]);
}

/* Many targets at once: E for part idx[k] at xyz[3k..3k+2]. */
void potref_field_many(unsigned long n, const unsigned int* idx, const double* xyz, double* hi, double* lo)
{
	for (unsigned long k = 0; k < n; k++)
		potref_field_at(idx[k], xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2], &hi[3 * k], &lo[3 * k]);
}

#ifdef USING_PHI_AT
double potref_phi_at(double x, double y, double z) { return phi_at(x, y, z, &H, &R, H.root); }
int potref_has_phi_at(void) { return 1; }
#else
int potref_has_phi_at(void) { return 0; }
#endif

void potref_phi_particle_feels(unsigned int part, double* hi, double* lo)
{
	split_ld(phi_particle_feels(part, &H, &R, H.root), hi, lo);
}

int potref_cross_grain(const Particle* p, const double* d_pos, const Particle* gr, double a)
{
#if H_SPHEROID
	return does_particle_cross_grain(p, d_pos, gr, a, R.A) ? 1 : 0;
#else
	return does_particle_cross_grain(p, d_pos, gr, a) ? 1 : 0;
#endif
}

/* inject() on a caller-supplied particle with the harness PRNG (pot.c:658). */
void potref_inject(Particle* p, int reinjection) { inject(p, R, reinjection != 0, &H); }

#ifdef SCEPTIC_REINJECTION
double potref_measure_chi_b(void) { return measure_chi_b(&H, R, H.root); }
double potref_u_icdf(double U, double chi, double q) { return u_icdf(U, chi, q); }
double potref_u_no_flow_icdf(double chi, double q) { return u_no_flow_icdf(chi, q); }
double potref_integrate_for_alpha(double s, double chi_b, double u2, double Rol)
{
	return integrate_for_alpha(s, chi_b, u2, Rol);
}
#endif

/* The reference's own state-file writer and reader (pot.c:3816-3901,
   3904-4019), on the harness's run: format C, one worker record.  read
   returns 0 on success, as read_sim_state_from_file does. */
void potref_write_state(const char* path)
{
	/* run() writes at the top of an iteration, after its t_steps++
	   (pot.c:4261, 4353-4356), and the file holds t_steps - 1: the steps
	   completed, which is what H.t_steps counts here */
	H.t_steps++;
	write_sim_state_to_file((unsigned int) R.N, &H, path);
	H.t_steps--;
}
int potref_read_state(const char* path) { return read_sim_state_from_file((unsigned int) R.N, &H, path) ? -1 : 0; }

#ifdef RECORD_PHI_DATA
/* write_phi_data_to_file (pot.c:3001-3042) for the tree last built, the
   rows appended to `path` with time time_step * dt. */
void potref_write_phi(const char* path, unsigned long time_step)
{
	write_phi_data_to_file(path, &H, R, time_step, H.root);
}
int potref_has_write_phi(void) { return 1; }
#else
int potref_has_write_phi(void) { return 0; }
#endif

/* One iteration of run()'s loop body for the hot path (pot.c:4261 t_steps++,
   4308 build_tree, 4386 move_particles), without the writers.
   Returns 0, or -1 if build_tree failed. */
int potref_step(int compute_epe)
{
	H.t_steps++;
	if (build_tree(&H, R) == NULL) return -1;
	move_particles(&H, R, H.root, H_mpi_particle, compute_epe != 0, H.t_steps);
	if (H.rank) {
		/* A worker rank of a multi-rank run: its stepped block reaches its
		   own particle array only through the master's broadcast at the
		   next step (pot.c:4299), which the single-rank stand-in does not
		   carry, so copy the block back here.  Without it the in-place
		   half drifts (pot.c:2478-2485) accumulate and the block leaves the
		   domain unreinjected. */
		const unsigned int a = H.pits[H.rank][0], b = H.pits[H.rank][1];
		memcpy(&H.parts[a], &H.new_parts[a], sizeof(Particle) * (b - a + 1));
	}
	return 0;
}

int potref_run_steps(unsigned long n, int compute_epe)
{
	for (unsigned long k = 0; k < n; k++)
		if (potref_step(compute_epe)) return -1;
	return 0;
}

/* move_particles only (the caller has already called potref_build_tree),
   with an explicit step index; pot.c:2330. */
void potref_move(unsigned long time_steps, int compute_epe)
{
	move_particles(&H, R, H.root, H_mpi_particle, compute_epe != 0, time_steps);
}

void potref_get_epe(double* out3)
{
	for (int k = 0; k < 3; k++) out3[k] = (double) H.epe[k];
}
