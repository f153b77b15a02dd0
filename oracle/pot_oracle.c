/*
 * CPU oracle for pot's per-timestep particle loop -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain-C restatement of drewthomas/pot's hot path, written for this
 * project; each function names the reference lines it follows.  It is the
 * checker for the CUDA kernels and never part of the product: only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
 *
 * Parity pin: in reference mode (quirk = 1, WELL512) a run of this file is
 * compared against the reference program compiled from its own sources
 * (oracle/_ref, built by oracle/build.py) and against the golden vectors in
 * tests/golden/ written from that program.
 *
 * Arithmetic types follow the reference call by call: x87 `long double`
 * where pot.c declares it (field accumulators, qom, accelerations, masses,
 * the PRNG's return value), `double` elsewhere, so that reference mode is
 * bit-identical to the reference on x86-64 with gcc.
 */
#include "pot_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* Physical constants of pot.c:278-282 (SI).  PI and SQRT_PI are the values
   prng.h:10-15 defines (pot.c includes prng.h before its own long-double PI
   definition, so the 15-digit double is the one in force everywhere). */
#define O_KB 1.38065e-23
#define O_EPSILON0 8.85419e-12
#define O_QE 1.6021766e-19
#define O_ME 9.109383e-31
#define O_MIME 1836.15
#define O_MIME_SPHEROID 1836.153  /* pot-spheroid.c:61 */
#define O_PI 3.14159265358979
#define O_SQRT_PI 1.77245385090552
#define O_MAX_PATH 400   /* pot.c:196 */
#define O_NONE UINT_MAX  /* empty-leaf marker, pot.c:1251 */

enum { O_DUST = 0, O_ION = 1, O_ELECTRON = 2 };
static const int O_CHARGE[3] = { 0, 1, -1 };                               /* pot.c:291 */
/* MASS of pot.c:292 is { 1.67e-12, MIME * 9.109383e-31, 9.109383e-31 };
   per run here, since pot-spheroid.c's MIME differs */

/* Octree node.  Child slots are kept in the reference's member order
   (pot.c:323-330): gxlylz, gxlygz, lxlylz, lxlygz, lxgylz, lxgygz, gxgylz,
   gxgygz; index 0 doubles as "no child" exactly as in the reference. */
typedef struct onode {
	double x1, y1, z1, x2, y2, z2;
	uint32_t part;
	double cx, cy, cz;
	int32_t q;
	uint32_t aq;
	uint32_t ch[8];
	double px, py, pz;  /* dipole moment about (cx, cy, cz), DIPOLES (pot.c:319-323) */
} onode;

/* slot of the child containing a point, by octal digit (gx<<2 | gy<<1 | gz) */
static const int DIGIT_SLOT[8] = { 2, 3, 4, 5, 0, 1, 6, 7 };
/* octal digit of each slot */
static const int SLOT_DIGIT[8] = { 4, 5, 0, 1, 2, 3, 6, 7 };

struct pto_ctx {
	pto_cfg cfg;
	long double dt;          /* Run.dt is long double (pot.c:341) */
	pto_particle* parts;
	pto_particle* new_parts;
	double* prev;            /* 3 per particle */
	onode* nodes;
	uint64_t n_alloc;
	uint64_t n_used;
	pto_well well;
	int32_t grain_q;
	long double grain_m;
	uint32_t tot_absor_e;
	uint64_t t_steps;
	double chi_b;
	uint32_t tss[3];
	long double mass[3];     /* MASS, pot.c:292 / pot-spheroid.c:61 */
	double max_lin_dev;      /* integrate_for_alpha tolerance, pot.c:436 / pot-spheroid.c:457 */
	int tilted;              /* spheroid axis other than x */
	double ax[3], e1[3], e2[3];  /* spheroid frame */
	/* Philox stream currently feeding rnd() (rng = 1) */
	uint32_t ph_ctr[4];
	uint32_t ph_buf[4];
	int ph_left;
	/* last-step statistics */
	int64_t st_dq;
	uint32_t st_de, st_nabs, st_nrein;
	uint64_t st_npush;
	long double epe[3];
	/* variants */
	long double* acc;        /* first-half accelerations (Proc.a_x1..a_z1), non-Boris integrators */
	double ion_temp;         /* Proc.Ti, POIS_POS_COLLECTION (pot.c:390) */
	double pos_rate_const;   /* Proc.pos_rate_const (pot.c:391) */
	uint32_t st_pois;        /* charges added by the Poisson collection this step */
	uint32_t st_wall;        /* OUT_BOUNCE: particles found in the wall moving inwards */
};

/* ------------------------------------------------------------------------ */
/* Random numbers                                                           */
/* ------------------------------------------------------------------------ */

/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
   easy as 1, 2, 3", SC'11): ten rounds of two 32x32->64 multiplies with the
   published multipliers and Weyl key increments. */
void pto_philox4x32(const uint32_t* ctr4, const uint32_t* key2, uint32_t* out4)
{
	uint32_t c0 = ctr4[0], c1 = ctr4[1], c2 = ctr4[2], c3 = ctr4[3];
	uint32_t k0 = key2[0], k1 = key2[1];
	for (int round = 0; round < 10; round++) {
		uint64_t p0 = (uint64_t) 0xD2511F53u * c0;
		uint64_t p1 = (uint64_t) 0xCD9E8D57u * c2;
		uint32_t n0 = (uint32_t) (p1 >> 32) ^ c1 ^ k0;
		uint32_t n2 = (uint32_t) (p0 >> 32) ^ c3 ^ k1;
		c0 = n0;
		c1 = (uint32_t) p1;
		c2 = n2;
		c3 = (uint32_t) p0;
		k0 += 0x9E3779B9u;
		k1 += 0xBB67AE85u;
	}
	out4[0] = c0; out4[1] = c1; out4[2] = c2; out4[3] = c3;
}

/* Select the Philox stream for particle `id` at step `t`; `tag` separates
   initial injection (0x20000) from the k-th reinjection within a step
   (0x10000 | k).  The same layout is used by the CUDA kernels. */
static void ph_stream(pto_ctx* c, uint32_t id, uint64_t t, uint32_t tag)
{
	c->ph_ctr[0] = id;
	c->ph_ctr[1] = (uint32_t) t;
	c->ph_ctr[2] = tag;
	c->ph_ctr[3] = 0;
	c->ph_left = 0;
}

static uint32_t ph_next(pto_ctx* c)
{
	if (c->ph_left == 0) {
		uint32_t key[2] = { (uint32_t) c->cfg.seed, (uint32_t) (c->cfg.seed >> 32) };
		pto_philox4x32(c->ph_ctr, key, c->ph_buf);
		c->ph_ctr[3]++;
		c->ph_left = 4;
	}
	return c->ph_buf[4 - c->ph_left--];
}

/* WELL512 step (Panneton, L'Ecuyer & Matsumoto 2006), in the form of
   prng.c:11-28, returning maximum * u / UINT32_MAX as a long double
   in [0, maximum] inclusive. */
static uint32_t well_next(pto_well* s)
{
	uint32_t i = s->index;
	uint32_t a = s->state[i];
	uint32_t c = s->state[(i + 13) & 15];
	uint32_t b = a ^ c ^ (a << 16) ^ (c << 15);
	c = s->state[(i + 9) & 15];
	c ^= (c >> 11);
	s->state[i] = b ^ c;
	uint32_t d = a ^ ((a << 5) & 0xda442d24UL);
	i = (i + 15) & 15;
	a = s->state[i];
	s->state[i] = a ^ b ^ d ^ (a << 2) ^ (b << 18) ^ (c << 28);
	s->index = i;
	s->a = a; s->b = b; s->c = c; s->d = d;
	return s->state[i];
}

static long double o_rnd(pto_ctx* c, long double maximum)
{
	uint32_t u = c->cfg.rng ? ph_next(c) : well_next(&c->well);
	return maximum * (u / (long double) UINT32_MAX);
}

/* Polar... in fact trigonometric Box-Muller pair, prng.c:32-47. */
static void o_nrv_pair(pto_ctx* c, double sd, double* nrv1, double* nrv2)
{
	double r;
	double theta;
	long double urv1;
	long double urv2 = o_rnd(c, 1.0L);
	do {
		urv1 = o_rnd(c, 1.0L);
	} while (urv1 == 0.0);
	r = sqrt(-2.0 * (double) logl(urv1));
	theta = 2.0 * O_PI * urv2;
	*nrv1 = sd * r * cos(theta);
	*nrv2 = sd * r * sin(theta);
}

/* Poisson variate by inversion, prng.c:50-70: walk the CDF from k = 0
   until the uniform draw is used up.  The reference loops until the
   term underflows; the cap only guards against a non-terminating loop
   (a rate of NaN or infinity) and returns 0 as the reference's exit does. */
static uint32_t o_prv(pto_ctx* c, double lambda)
{
	double exp_lambda = exp(-lambda);
	uint32_t k = 0;
	double ratio_term = 1.0;
	double uni = o_rnd(c, 1.0L);
	while (ratio_term) {
		uni -= ratio_term * exp_lambda;
		if (uni < 0.0) break;
		k++;
		ratio_term *= lambda / k;
		if (k >= (1u << 20)) return 0;
	}
	return ratio_term ? k : 0;
}

uint32_t pto_poisson(pto_ctx* c, double lambda) { return o_prv(c, lambda); }

/* Inverse CDF of |u| at infinity without flow (Hutchinson 2003, eqs 18-19),
   Newton iteration as prng.c:138-156.  The iteration cap only guards
   against a non-terminating loop; converged calls never reach it. */
double pto_u_no_flow_icdf(double chi, double q)
{
	double omc = 1.0 - chi;
	double p;
	double u = 1.29951;
	double usq;
	int it = 0;
	do {
		usq = u * u;
		p = 1.0 - ((usq + omc) * exp(-usq) / omc) - q;
		u -= p / (2.0 * u * exp(-usq) * (chi - usq) / -omc);
	} while ((p * p) > 1e-16 && ++it < 10000);
	return u;
}

/* Inverse CDF of |u| at infinity with drift U > 0 (Hutchinson 2003 eq 19),
   Newton iteration as prng.c:171-214. */
double pto_u_icdf(double U, double chi, double q)
{
	const double Usq = U * U;
	const double psi = O_SQRT_PI * (1.0 + (2.0 * (Usq - chi))) / 2.0;
	const double p_den = 2.0 * ((U * exp(-Usq)) + (psi * erf(U)));
	double dp_den, dp_num, p, p_num, temp, u, usq;
	int it = 0;

	if (U > 2.1) {
		u = U + (1.0 / U);
	} else {
		u = 1.2586147 + (0.221 * U) + (0.1903312 * U * U);
	}
	dp_den = 2.0 * O_SQRT_PI * (U + (psi * exp(Usq) * erf(U)));
	do {
		usq = u * u;
		temp = -(U + u) * (U + u);
		p_num = (U - u) * exp(temp);
		p_num += (U + u) * exp((4.0 * U * u) + temp);
		p_num += psi * (erf(U - u) + erf(U + u));
		p = 1.0 - (p_num / p_den) - q;
		dp_num = (O_SQRT_PI * (1.0 + (2.0 * (Usq - usq)))) - (2.0 * psi);
		dp_num *= exp(-u * ((2.0 * U) + u)) - exp((2.0 * U * u) - usq);
		u -= p / (dp_num / dp_den);
	} while ((p * p) > 1e-16 && ++it < 10000);
	return u;
}

/* ------------------------------------------------------------------------ */
/* Rotations (coord.c:6-59)                                                 */
/* ------------------------------------------------------------------------ */

/* spherical (v_r, v_phi, v_theta) at angles (phi, theta) -> Cartesian,
   coord.c:6-14 */
static void o_vel_cart(const double* v, double phi, double theta, double* vx, double* vy, double* vz)
{
	*vx = (v[0] * cos(phi) * sin(theta)) - (v[1] * sin(phi)) + (v[2] * cos(phi) * cos(theta));
	*vy = (v[0] * sin(phi) * sin(theta)) + (v[1] * cos(phi)) + (v[2] * sin(phi) * cos(theta));
	*vz = (v[0] * cos(theta)) - (v[2] * sin(theta));
}

/* rotation about a unit axis d = (d0, d1, 0) by the angle with sine s and
   cosine cs, then translation by `offset`; coord.c:22-37 */
static void o_rot_xy(const double* d, double s, double cs, double* x, double* y, double* z, double offset)
{
	const double omc = 1.0 - cs;
	double t0, t1, t2;
	t0 = d[0] * ((d[0] * *x) + (d[1] * *y)) * omc;
	t0 += (*x * cs) + (d[1] * *z * s);
	t1 = d[1] * ((d[0] * *x) + (d[1] * *y)) * omc;
	t1 += (*y * cs) - (d[0] * *z * s);
	t2 = *z * cs;
	t2 += ((d[0] * *y) - (d[1] * *x)) * s;
	*x = offset + t0;
	*y = offset + t1;
	*z = offset + t2;
}

/* rotation about an arbitrary unit axis d (Rodrigues), coord.c:45-59 */
static void o_rot(const double* d, double s, double cs, double* x, double* y, double* z)
{
	const double omc = 1.0 - cs;
	const double dot = (d[0] * *x) + (d[1] * *y) + (d[2] * *z);
	double t0, t1, t2;
	t0 = d[0] * dot * omc;
	t0 += (*x * cs) + (((d[1] * *z) - (d[2] * *y)) * s);
	t1 = d[1] * dot * omc;
	t1 += (*y * cs) + (((d[2] * *x) - (d[0] * *z)) * s);
	t2 = d[2] * dot * omc;
	t2 += (*z * cs) + (((d[0] * *y) - (d[1] * *x)) * s);
	*x = t0;
	*y = t1;
	*z = t2;
}

/* ------------------------------------------------------------------------ */
/* (Re)injection                                                            */
/* ------------------------------------------------------------------------ */

/* Orbit-angle integral of Hutchinson's SCEPTIC by crude adaptive Simpson,
   pot.c:433-492.  A cap on the interval halvings keeps the loop finite. */
double pto_integrate_for_alpha_dev(double s, double chi_b, double u2, double Rol, double max_lin_dev)
{
	const double chu2 = chi_b / u2;
	const double s2 = s * s;
	const double y_one = s / sqrt(1.0 - chu2 - s2);
	double alpha = 0.0;
	double xi[3] = { 0.0, 0.5, 1.0 };
	double y[3] = { s, -9.9, y_one };
	int guard = 0;

	if (s == 0.0) return 0.0;
	do {
		xi[2] = 1.0;
		y[2] = y_one;
		xi[1] = (xi[0] + xi[2]) / 2.0;
		y[1] = 1.0 - (chu2 * xi[1] * exp(Rol * (1.0 - (1.0 / xi[1]))));
		y[1] = 1.0 / sqrt((y[1] / s2) - (xi[1] * xi[1]));
		while (fabs(y[2] - y[1] - (y[1] - y[0])) > max_lin_dev) {
			xi[2] = xi[1];
			y[2] = y[1];
			xi[1] = (xi[0] + xi[2]) / 2.0;
			y[1] = 1.0 - (chu2 * xi[1] * exp(Rol * (1.0 - (1.0 / xi[1]))));
			y[1] = 1.0 / sqrt((y[1] / s2) - (xi[1] * xi[1]));
			if (++guard > 1000000) return NAN;
		}
		alpha += (xi[2] - xi[0]) * (y[0] + (4.0 * y[1]) + y[2]) / 6.0;
		xi[0] = xi[2];
		y[0] = y[2];
		if (++guard > 1000000) return NAN;
	} while (xi[2] < 1.0);
	return alpha;
}

double pto_integrate_for_alpha(double s, double chi_b, double u2, double Rol)
{
	return pto_integrate_for_alpha_dev(s, chi_b, u2, Rol, 0.01);
}

/* SCEPTIC-like reinjection at the domain edge, pot.c:496-652.  The
   reference retries by recursion when alpha is NaN; this is the same retry
   as a loop, including the reference's undo of the electron rescaling of
   chi_b (pot.c:591-596). */
static void o_sceptic(pto_ctx* c, pto_particle* part, double chi_b)
{
	const pto_cfg* ru = &c->cfg;
	double a[2], alpha, b, cz, co_z, phi, psi, q, Rol, U, u_mag, u2, u[3], v[3], v_n;
	int tries = 0;

	for (;;) {
		v_n = 2.0 * O_KB / c->mass[part->species];
		if (part->species == O_ELECTRON) {
			v_n *= ru->Te;
			chi_b *= -ru->Ti / ru->Te;
		} else {
			v_n *= ru->Ti;
		}
		v_n = sqrt(v_n);

		if (ru->x_drift) {
			U = ru->x_drift / v_n;
			do {
				u_mag = pto_u_icdf(U, chi_b, o_rnd(c, 1.0));
				u2 = u_mag * u_mag;
			} while (u2 < chi_b);
			q = o_rnd(c, 1.0);
			cz = log(q + (1.0 - q) * exp(-4.0 * u_mag * U)) / (2.0 * u_mag * U);
			cz += 1.0;
		} else {
			do {
				u_mag = pto_u_no_flow_icdf(chi_b, o_rnd(c, 1.0));
				u2 = u_mag * u_mag;
			} while (u2 < chi_b);
			cz = o_rnd(c, 2.0) - 1.0;
		}

		u[0] = 0.0;
		u[1] = 0.0;
		u[2] = u_mag;
		a[0] = 0.0;
		a[1] = 1.0;
		o_rot_xy(a, cz, sqrt(1.0 - (cz * cz)), &u[0], &u[1], &u[2], 0.0);
		a[0] = 1.0;
		a[1] = 0.0;
		psi = o_rnd(c, 2.0 * O_PI);
		o_rot_xy(a, sin(psi), cos(psi), &u[0], &u[1], &u[2], 0.0);

		b = sqrt(o_rnd(c, 1.0 - (chi_b / u2)));

		Rol = O_QE * O_QE * (ru->N - 1) / 2.0;
		Rol /= (4.0 * O_PI / 3.0) * ru->mpp * ru->r * O_EPSILON0 * O_KB * ru->Te;
		Rol = sqrt(Rol);
		alpha = pto_integrate_for_alpha_dev(b, chi_b, u2, Rol, c->max_lin_dev);
		if (isnan(alpha) && ++tries < 100000) {
			if (part->species == O_ELECTRON) {
				chi_b /= -ru->Ti / ru->Te;
			}
			continue;
		}
		break;
	}

	phi = o_rnd(c, 2.0 * O_PI);
	part->x = ru->mpp * ru->r * sin(alpha) * cos(phi);
	part->y = ru->mpp * ru->r * sin(alpha) * sin(phi);
	part->z = ru->mpp * ru->r * cos(alpha);

	a[0] = u[1];
	a[1] = -u[0];
	a[0] /= sqrt((u[0] * u[0]) + (u[1] * u[1]));
	a[1] /= sqrt((u[0] * u[0]) + (u[1] * u[1]));

	co_z = u[2] / u_mag;
	o_rot_xy(a, sin(acos(co_z)), co_z, &part->x, &part->y, &part->z, ru->mpp * ru->r);

	v[1] = 0.0;
	v[2] = u_mag * b;
	v[0] = -sqrt(u2 - chi_b - (v[2] * v[2]));
	o_vel_cart(v, phi, alpha, &part->vx, &part->vy, &part->vz);
	o_rot_xy(a, sin(acos(co_z)), co_z, &part->vx, &part->vy, &part->vz, 0.0);

	part->vx *= v_n;
	part->vy *= v_n;
	part->vz *= v_n;
}

/* (Re)inject one particle in the spherical domain with the grain enabled,
   pot.c:658-765 (SPHERICAL branch). */
static void o_inject(pto_ctx* c, pto_particle* part, int reinjection)
{
	const pto_cfg* ru = &c->cfg;
	double sigma, phi, r, theta, v[3];

	if (part->species == O_ION) {
		sigma = sqrt(O_KB * ru->Ti / c->mass[O_ION]);
	} else {
		sigma = sqrt(O_KB * ru->Te / c->mass[O_ELECTRON]);
	}
	if (!ru->sceptic && !reinjection) {
		sigma *= 0.85;  /* pot.c:684-690 */
	}

	if (!reinjection) {
		r = ru->mpp * cbrt(o_rnd(c, ru->r * ru->r * ru->r));
		while (r <= ru->a) {
			r = ru->mpp * cbrt(o_rnd(c, ru->r * ru->r * ru->r));
		}
	} else {
		r = ru->mpp * ru->r;
	}

	if (ru->sceptic && reinjection) {
		o_sceptic(c, part, c->chi_b);
		return;
	}
	phi = o_rnd(c, 2.0 * O_PI);
	theta = acos(o_rnd(c, 2.0) - 1.0);
	part->x = (ru->mpp * ru->r) + (r * sin(theta) * cos(phi));
	part->y = (ru->mpp * ru->r) + (r * sin(theta) * sin(phi));
	part->z = (ru->mpp * ru->r) + (r * cos(theta));

	if (!reinjection) {
		o_nrv_pair(c, sigma, &part->vx, &part->vy);
		o_nrv_pair(c, sigma, &part->vz, &part->vz);
	} else {
		o_nrv_pair(c, sigma, &v[0], &v[1]);
		o_nrv_pair(c, sigma, &v[2], &v[2]);
		if (v[0] > 0.0) v[0] = -v[0];
		o_vel_cart(v, phi, theta, &part->vx, &part->vy, &part->vz);
	}
	part->vx += ru->x_drift;
}

/* ------------------------------------------------------------------------ */
/* Context                                                                  */
/* ------------------------------------------------------------------------ */

int pto_sizeof_particle(void) { return (int) sizeof(pto_particle); }

pto_ctx* pto_create(const pto_cfg* cfg)
{
	pto_ctx* c = calloc(1, sizeof(pto_ctx));
	if (!c) return NULL;
	c->cfg = *cfg;
	c->dt = (long double) cfg->dt;
	c->parts = calloc(cfg->N, sizeof(pto_particle));
	c->new_parts = calloc(cfg->N, sizeof(pto_particle));
	c->prev = calloc(3 * cfg->N, sizeof(double));
	c->acc = calloc(3 * cfg->N, sizeof(long double));
	c->n_alloc = 9 * cfg->N + 9;   /* pot.c:4143 */
	c->nodes = malloc(sizeof(onode) * c->n_alloc);
	if (!c->parts || !c->new_parts || !c->prev || !c->acc || !c->nodes) {
		pto_destroy(c);
		return NULL;
	}
	{
		const double mime = cfg->shape ? O_MIME_SPHEROID : O_MIME;
		c->mass[O_DUST] = 1.67e-12;
		c->mass[O_ION] = mime * O_ME;
		c->mass[O_ELECTRON] = O_ME;
		c->max_lin_dev = cfg->shape ? 0.1 : 0.01;
	}
	if (cfg->shape) {
		/* spheroid frame: axis, then e1 = y (or z) made orthogonal, e2 = axis x e1 */
		double n = sqrt(cfg->axis[0] * cfg->axis[0] + cfg->axis[1] * cfg->axis[1] + cfg->axis[2] * cfg->axis[2]);
		if (!(n > 0.0)) {
			c->ax[0] = 1.0;
			c->ax[1] = c->ax[2] = 0.0;
		} else {
			for (int k = 0; k < 3; k++) c->ax[k] = cfg->axis[k] / n;
		}
		c->tilted = !(c->ax[0] == 1.0 && c->ax[1] == 0.0 && c->ax[2] == 0.0);
		double ref[3] = { 0.0, 1.0, 0.0 };
		if (fabs(c->ax[1]) > 0.9) {
			ref[1] = 0.0;
			ref[2] = 1.0;
		}
		double d = ref[0] * c->ax[0] + ref[1] * c->ax[1] + ref[2] * c->ax[2];
		for (int k = 0; k < 3; k++) c->e1[k] = ref[k] - d * c->ax[k];
		n = sqrt(c->e1[0] * c->e1[0] + c->e1[1] * c->e1[1] + c->e1[2] * c->e1[2]);
		for (int k = 0; k < 3; k++) c->e1[k] /= n;
		c->e2[0] = c->ax[1] * c->e1[2] - c->ax[2] * c->e1[1];
		c->e2[1] = c->ax[2] * c->e1[0] - c->ax[0] * c->e1[2];
		c->e2[2] = c->ax[0] * c->e1[1] - c->ax[1] * c->e1[0];
	}
	c->grain_q = O_CHARGE[O_DUST];
	c->grain_m = c->mass[O_DUST];
	/* species time-step multiples, pot.c:4157-4159 */
	c->tss[O_ELECTRON] = 1;
	c->tss[O_ION] = (int) sqrt(cfg->Te * c->mass[O_ION] / (cfg->Ti * c->mass[O_ELECTRON]));
	c->tss[O_DUST] = c->tss[O_ION] * (int) sqrt(0.1 * c->mass[O_DUST] / c->mass[O_ION]);
	/* POIS_POS_COLLECTION set-up, pot.c:4251-4255: the cached ion temperature
	   starts at the injection temperature; the constant part of the rate */
	c->ion_temp = cfg->Ti;
	{
		const long double n = (cfg->N - 1) / ((4.0 / 3.0) * O_PI * powl(cfg->r * cfg->mpp, 3.0));
		double k = 4.0 * O_PI * cfg->a * cfg->a * O_CHARGE[O_ION];
		k /= sqrt(2.0 * O_PI * c->mass[O_ION]);
		k *= c->dt * n / 2.0;
		c->pos_rate_const = k;
	}
	return c;
}

void pto_set_ion_temp(pto_ctx* c, double Ti) { c->ion_temp = Ti; }
double pto_ion_temp(const pto_ctx* c) { return c->ion_temp; }

void pto_destroy(pto_ctx* c)
{
	if (!c) return;
	free(c->parts);
	free(c->new_parts);
	free(c->prev);
	free(c->acc);
	free(c->nodes);
	free(c);
}

void pto_get_tss(const pto_ctx* c, uint32_t* out3) { memcpy(out3, c->tss, sizeof(c->tss)); }
void pto_set_particles(pto_ctx* c, const pto_particle* in) { memcpy(c->parts, in, sizeof(pto_particle) * c->cfg.N); }
void pto_get_particles(const pto_ctx* c, pto_particle* out) { memcpy(out, c->parts, sizeof(pto_particle) * c->cfg.N); }
void pto_set_well(pto_ctx* c, const pto_well* w) { c->well = *w; }
void pto_get_well(const pto_ctx* c, pto_well* w) { *w = c->well; }

/* init_prng, prng.c:4-8 */
void pto_seed_well(pto_ctx* c, const uint32_t* seed16)
{
	memcpy(c->well.state, seed16, 16 * sizeof(uint32_t));
	c->well.index = 0;
}

void pto_set_grain(pto_ctx* c, int32_t q, double m, uint32_t tot_absor_e, uint64_t t_steps, double chi_b)
{
	c->grain_q = q;
	c->grain_m = m;
	c->tot_absor_e = tot_absor_e;
	c->t_steps = t_steps;
	c->chi_b = chi_b;
}

void pto_get_grain(const pto_ctx* c, int32_t* q, double* m, uint32_t* tot_absor_e, uint64_t* t_steps,
                   double* chi_b, double* grain_v3)
{
	*q = c->grain_q;
	*m = (double) c->grain_m;
	*tot_absor_e = c->tot_absor_e;
	*t_steps = c->t_steps;
	*chi_b = c->chi_b;
	grain_v3[0] = c->parts[0].vx;
	grain_v3[1] = c->parts[0].vy;
	grain_v3[2] = c->parts[0].vz;
}

/* init_particles for one rank, pot.c:887-935: grain at the centre, then
   (N-1)/2 ions at indices 1..N_i and electrons after them, each injected in
   index order. */
int pto_init_particles(pto_ctx* c)
{
	const pto_cfg* ru = &c->cfg;
	pto_particle* p = c->parts;
	uint64_t n_i = (ru->N - 1) / 2;
	p[0].x = ru->r * ru->mpp;
	p[0].y = p[0].x;
	p[0].z = p[0].x;
	p[0].vx = p[0].vy = p[0].vz = 0.0;
	p[0].species = O_DUST;
	for (uint64_t i = 1; i < ru->N; i++) p[i].species = (i <= n_i) ? O_ION : O_ELECTRON;
	for (uint64_t i = 1; i < ru->N; i++) {
		if (ru->rng) ph_stream(c, (uint32_t) i, 0, 0x20000u);
		o_inject(c, &p[i], 0);
	}
	return 0;
}

/* ------------------------------------------------------------------------ */
/* Tree                                                                     */
/* ------------------------------------------------------------------------ */

/* child boxes by halving, pot.c:1225-1288 */
static void o_init_children(onode* nl, uint64_t k)
{
	onode* t = &nl[k];
	double mx = (t->x1 + t->x2) / 2;
	double my = (t->y1 + t->y2) / 2;
	double mz = (t->z1 + t->z2) / 2;
	for (int s = 0; s < 8; s++) {
		onode* ch = &nl[t->ch[s]];
		int d = SLOT_DIGIT[s];
		ch->x1 = t->x1; ch->x2 = t->x2;
		ch->y1 = t->y1; ch->y2 = t->y2;
		ch->z1 = t->z1; ch->z2 = t->z2;
		ch->part = O_NONE;
		memset(ch->ch, 0, sizeof(ch->ch));
		if (d & 4) ch->x1 = mx; else ch->x2 = mx;
		if (d & 2) ch->y1 = my; else ch->y2 = my;
		if (d & 1) ch->z1 = mz; else ch->z2 = mz;
	}
}

/* running |q|-weighted centre, pot.c:1290-1310; with dipoles the node's
   moment is first moved to the new centre, then the child's, moved there
   too, is added */
static void o_update_moments(onode* node, const onode* chi, int dipoles)
{
	const double ocx = node->cx, ocy = node->cy, ocz = node->cz;
	node->cx = (node->aq * node->cx + chi->aq * chi->cx) / (node->aq + chi->aq);
	node->cy = (node->aq * node->cy + chi->aq * chi->cy) / (node->aq + chi->aq);
	node->cz = (node->aq * node->cz + chi->aq * chi->cz) / (node->aq + chi->aq);
	if (dipoles) {
		node->px -= (node->cx - ocx) * node->q;
		node->py -= (node->cy - ocy) * node->q;
		node->pz -= (node->cz - ocz) * node->q;
		node->px += chi->px - (node->cx - chi->cx) * chi->q;
		node->py += chi->py - (node->cy - chi->cy) * chi->q;
		node->pz += chi->pz - (node->cz - chi->cz) * chi->q;
	}
	node->q += chi->q;
	node->aq += chi->aq;
}

/* recursive upward pass, pot.c:1312-1402 */
static void o_node_values(pto_ctx* c, uint64_t k)
{
	onode* node = &c->nodes[k];
	if (node->part != O_NONE) {
		const pto_particle* p = &c->parts[node->part];
		node->q = (p->species == O_DUST) ? c->grain_q : O_CHARGE[p->species];
		node->aq = (uint32_t) abs(node->q);
		node->cx = p->x;
		node->cy = p->y;
		node->cz = p->z;
		node->px = node->py = node->pz = 0.0;
		return;
	}
	node->q = 0;
	node->aq = 0;
	node->cx = node->cy = node->cz = 0.0;
	node->px = node->py = node->pz = 0.0;
	for (int s = 0; s < 8; s++) {
		uint32_t ck = c->nodes[k].ch[s];
		if (ck) {
			o_node_values(c, ck);
			node = &c->nodes[k];
			if (c->nodes[ck].aq) o_update_moments(node, &c->nodes[ck], c->cfg.dipoles);
		}
	}
}

/* Serial insertion octree with one particle per leaf, pot.c:1457-1643.
   Returns 0; -1 for a particle outside the root box; -2 for two particles
   at one position (the reference loops forever on those unless a
   reallocation happens to catch them, pot.c:1578-1586); -3 out of memory. */
int pto_build_tree(pto_ctx* c)
{
	const pto_cfg* ru = &c->cfg;
	onode* root = &c->nodes[0];
	uint64_t used = 0;
	memset(root, 0, sizeof(*root));
	root->x2 = 2.0 * ru->r * ru->mpp;
	root->y2 = root->x2;
	root->z2 = root->y2;
	root->part = O_NONE;

	/* pot-spheroid.c:1516-1518: the spheroidal grain is not in the tree */
	uint64_t pn = ru->shape ? 1 : 0;
	while (pn < ru->N) {
		const pto_particle* part = &c->parts[pn];
		if ((part->x < 0.0) || (part->x > root->x2) || (part->y < 0.0) || (part->y > root->y2)
		    || (part->z < 0.0) || (part->z > root->z2) || isnan(part->x) || isnan(part->y)
		    || isnan(part->z)) {
			return -1;
		}
		uint64_t cur, next = 0;
		onode* t;
		double mx, my, mz;
		int depth = 0;
		do {
			cur = next;
			t = &c->nodes[cur];
			mx = (t->x1 + t->x2) / 2.0;
			my = (t->y1 + t->y2) / 2.0;
			mz = (t->z1 + t->z2) / 2.0;
			int d = ((part->x < mx) ? 0 : 4) | ((part->y < my) ? 0 : 2) | ((part->z < mz) ? 0 : 1);
			next = t->ch[DIGIT_SLOT[d]];
		} while (next && ++depth < 4096);

		if (t->part == O_NONE) {
			t->part = (uint32_t) pn;
			pn++;
			continue;
		}
		const pto_particle* occ = &c->parts[t->part];
		if (occ->x == part->x && occ->y == part->y && occ->z == part->z) return -2;
		if (c->n_alloc < used + 9) {
			/* growth rule of pot.c:1406-1432 */
			uint64_t na = (uint64_t) (c->n_alloc * 1.1) + 9;
			onode* nn = realloc(c->nodes, sizeof(onode) * na);
			if (!nn) return -3;
			c->nodes = nn;
			c->n_alloc = na;
			root = &c->nodes[0];
			t = &c->nodes[cur];
		}
		for (int s = 0; s < 8; s++) t->ch[s] = (uint32_t) ++used;
		o_init_children(c->nodes, cur);
		t = &c->nodes[cur];
		int d = ((occ->x < mx) ? 0 : 4) | ((occ->y < my) ? 0 : 2) | ((occ->z < mz) ? 0 : 1);
		c->nodes[t->ch[DIGIT_SLOT[d]]].part = t->part;
		t->part = O_NONE;
	}
	c->n_used = used + 1;
	o_node_values(c, 0);
	return 0;
}

/* Same canonical dump as oracle/ref_harness.c: internal nodes and occupied
   leaves labelled by (level, octal-digit path), depth-first. */
int pto_tree_dump(const pto_ctx* c, uint64_t max_nodes,
                  uint64_t* n_int, int32_t* int_level, uint64_t* int_path, int32_t* int_q,
                  uint32_t* int_aq, double* int_c, double* int_w,
                  uint64_t* n_leaf, uint32_t* leaf_part, int32_t* leaf_level, uint64_t* leaf_path)
{
	uint32_t sn[1024];
	int sl[1024];
	uint64_t spath[1024];
	int sp = 1;
	uint64_t ni = 0, nl = 0;
	sn[0] = 0; sl[0] = 0; spath[0] = 0;
	while (sp) {
		sp--;
		const onode* t = &c->nodes[sn[sp]];
		int lev = sl[sp];
		uint64_t path = spath[sp];
		if (t->part != O_NONE) {
			if (nl >= max_nodes) return -1;
			leaf_part[nl] = t->part; leaf_level[nl] = lev; leaf_path[nl] = path; nl++;
		} else if (t->ch[0]) {
			if (ni >= max_nodes || lev >= 21 || sp + 8 > 1024) return -1;
			int_level[ni] = lev; int_path[ni] = path; int_q[ni] = t->q; int_aq[ni] = t->aq;
			int_c[3 * ni] = t->cx; int_c[3 * ni + 1] = t->cy; int_c[3 * ni + 2] = t->cz;
			int_w[ni] = t->x2 - t->x1;
			ni++;
			for (int s = 0; s < 8; s++) {
				sn[sp] = t->ch[s];
				sl[sp] = lev + 1;
				spath[sp] = (path << 3) | (uint64_t) SLOT_DIGIT[s];
				sp++;
			}
		}
	}
	*n_int = ni;
	*n_leaf = nl;
	return 0;
}

/* Dipole moments of the internal nodes in pto_tree_dump's order; returns the
   node count or -1. */
int64_t pto_tree_dipoles(const pto_ctx* c, uint64_t max_nodes, double* int_p)
{
	uint32_t sn[1024];
	int sl[1024];
	int sp = 1;
	uint64_t ni = 0;
	sn[0] = 0; sl[0] = 0;
	while (sp) {
		sp--;
		const onode* t = &c->nodes[sn[sp]];
		const int lev = sl[sp];
		if (t->part == O_NONE && t->ch[0]) {
			if (ni >= max_nodes || lev >= 21 || sp + 8 > 1024) return -1;
			int_p[3 * ni] = t->px; int_p[3 * ni + 1] = t->py; int_p[3 * ni + 2] = t->pz;
			ni++;
			for (int s = 0; s < 8; s++) {
				sn[sp] = t->ch[s];
				sl[sp] = lev + 1;
				sp++;
			}
		}
	}
	return (int64_t) ni;
}

/* ------------------------------------------------------------------------ */
/* Field and potential walks                                                */
/* ------------------------------------------------------------------------ */

/* ------------------------------------------------------------------------ */
/* Spheroidal grain (pot-spheroid.c, PROLATE / OBLATE)                      */
/* ------------------------------------------------------------------------ */

/* Components of a grain-relative vector along the spheroid's axis and two
   perpendicular directions; the identity (bit for bit) for the reference's
   x axis. */
static void o_to_frame(const pto_ctx* c, double dx, double dy, double dz, double* u, double* v, double* w)
{
	if (!c->tilted) {
		*u = dx;
		*v = dy;
		*w = dz;
		return;
	}
	*u = dx * c->ax[0] + dy * c->ax[1] + dz * c->ax[2];
	*v = dx * c->e1[0] + dy * c->e1[1] + dz * c->e1[2];
	*w = dx * c->e2[0] + dy * c->e2[1] + dz * c->e2[2];
}

static void o_from_frame(const pto_ctx* c, double u, double v, double w, double* out)
{
	if (!c->tilted) {
		out[0] = u;
		out[1] = v;
		out[2] = w;
		return;
	}
	for (int k = 0; k < 3; k++) out[k] = u * c->ax[k] + v * c->e1[k] + w * c->e2[k];
}

/* field_particle_feels_from_grain, pot-spheroid.c:1689-1779: the analytic
   field of the charged conducting spheroid at (x, y, z); zero for the grain
   itself.  Expressions in the reference's order (double arithmetic). */
static void o_spheroid_field(const pto_ctx* c, uint32_t part, double x, double y, double z, double* Eo)
{
	const double A = c->cfg.A;
	const double a = c->cfg.a;
	double fc, phi_const, rho2, rt, e2, E_n, beta, theta, dx, dy, dz;
	if (c->cfg.shape == 1) {
		fc = (a * sqrt(A * A - 1.0)) * pow(A, -1.0 / 3.0);
		phi_const = (O_QE * c->grain_q * acosh(A)) / (4.0 * O_PI * O_EPSILON0 * fc * log(A - sqrt(A * A - 1.0)));
	} else {
		fc = (a * sqrt(1.0 - A * A)) * pow(A, -1.0 / 3.0);
		phi_const = (O_QE * c->grain_q * acos(A))
		            / (8.0 * O_PI * O_EPSILON0 * fc * (atan((1.0 - sqrt(1.0 - A * A)) / A) - 0.25 * O_PI));
	}
	if (!part) {
		Eo[0] = Eo[1] = Eo[2] = 0.0;
		return;
	}
	const pto_particle* g = &c->parts[0];
	o_to_frame(c, x - g->x, y - g->y, z - g->z, &dx, &dy, &dz);
	rho2 = (dy * dy) + (dz * dz);
	if (c->cfg.shape == 1) {
		rt = sqrt(rho2 * rho2 + dx * dx * dx * dx + fc * fc * fc * fc + 2.0 * rho2 * dx * dx
		          + 2.0 * rho2 * fc * fc - 2.0 * dx * dx * fc * fc);
		e2 = (rho2 + dx * dx - fc * fc + rt) / (2.0 * fc * fc);   /* sinh^2 */
		E_n = -phi_const / sqrt(e2 * rt);
		beta = atan((-e2 * dx) / ((e2 + 1.0) * sqrt(rho2)));
	} else {
		rt = sqrt(rho2 * rho2 + dx * dx * dx * dx + fc * fc * fc * fc + 2.0 * rho2 * dx * dx
		          - 2.0 * rho2 * fc * fc + 2.0 * dx * dx * fc * fc);
		e2 = (rho2 + dx * dx + fc * fc + rt) / (2.0 * fc * fc);   /* cosh^2 */
		E_n = -phi_const / sqrt(e2 * rt);
		beta = atan((-e2 * dx) / ((e2 - 1.0) * sqrt(rho2)));
	}
	theta = atan(fabs(dz) / fabs(dy));
	o_from_frame(c, -E_n * sin(beta), E_n * cos(beta) * cos(theta) * fabs(dy) / dy,
	             E_n * cos(beta) * sin(theta) * fabs(dz) / dz, Eo);
}

/* the spheroid's potential at grain-relative (dx, dy, dz) in its frame:
   phi_particle_feels_from_grain, pot-spheroid.c:2054-2078 */
static double o_spheroid_phi_rel(const pto_ctx* c, double dx, double dy, double dz)
{
	const double A = c->cfg.A;
	const double a = c->cfg.a;
	const double rho2 = (dy * dy) + (dz * dz);
	if (c->cfg.shape == 1) {
		const double fc = a * sqrt(A * A - 1.0) / pow(A, 1.0 / 3.0);
		const double phi_const = (O_QE * c->grain_q * acosh(A))
		                         / (4.0 * O_PI * O_EPSILON0 * fc * log(A - sqrt(A * A - 1.0)));
		const double rt = sqrt(rho2 * rho2 + dx * dx * dx * dx + fc * fc * fc * fc + 2.0 * rho2 * dx * dx
		                       + 2.0 * rho2 * fc * fc - 2.0 * dx * dx * fc * fc);
		return phi_const * log((sqrt(rho2 + dx * dx + fc * fc + rt) - fc * sqrt(2.0))
		                       / sqrt(rho2 + dx * dx - fc * fc + rt));
	}
	const double fc = (a * sqrt(1.0 - A * A)) * pow(A, -1.0 / 3.0);
	const double phi_const = (O_QE * c->grain_q * acos(A))
	                         / (4.0 * O_PI * O_EPSILON0 * fc * (atan((1.0 - sqrt(1.0 - A * A)) / A) - 0.25 * O_PI));
	const double rt = sqrt(rho2 * rho2 + dx * dx * dx * dx + fc * fc * fc * fc + 2.0 * rho2 * dx * dx
	                       - 2.0 * rho2 * fc * fc + 2.0 * dx * dx * fc * fc);
	return phi_const * (atan((sqrt(rho2 + dx * dx + fc * fc + rt) - fc * sqrt(2.0))
	                         / sqrt(rho2 + dx * dx - fc * fc + rt)) - 0.25 * O_PI);
}

/* potential of the spheroid felt by particle `part` at its stored position
   (pot-spheroid.c:2037-2085); zero for the grain */
static double o_spheroid_phi_particle(const pto_ctx* c, uint32_t part)
{
	double u, v, w;
	if (!part) return 0.0;
	const pto_particle* g = &c->parts[0];
	const pto_particle* p = &c->parts[part];
	o_to_frame(c, p->x - g->x, p->y - g->y, p->z - g->z, &u, &v, &w);
	return o_spheroid_phi_rel(c, u, v, w);
}

void pto_grain_field(const pto_ctx* c, double x, double y, double z, double* E3)
{
	if (!c->cfg.shape) {
		E3[0] = E3[1] = E3[2] = 0.0;
		return;
	}
	o_spheroid_field(c, 1, x, y, z, E3);
}

double pto_grain_phi(const pto_ctx* c, double x, double y, double z)
{
	double u, v, w;
	if (!c->cfg.shape) return 0.0;
	const pto_particle* g = &c->parts[0];
	o_to_frame(c, x - g->x, y - g->y, z - g->z, &u, &v, &w);
	return o_spheroid_phi_rel(c, u, v, w);
}

/* Barnes-Hut E at (x, y, z) for target `part`, pot.c:1696-1808 (monopole):
   accepted cells add an unsoftened monopole, leaves add a Plummer-softened
   pair term, the target itself is skipped by index.  Returns -1 when the
   explicit stack would overflow (the reference aborts, pot.c:1755-1757). */
static int o_field(const pto_ctx* c, uint32_t part, double x, double y, double z, long double* E)
{
	const double oap = c->cfg.theta;
	const double soft = c->cfg.soft;
	const onode* nodes = c->nodes;
	uint32_t path[O_MAX_PATH];
	unsigned int len = 1;
	double dist, dist2, dx, dy, dz;
	long double E_scale;
	E[0] = E[1] = E[2] = 0.0;
	if (c->cfg.shape) {
		/* pot-spheroid.c:1815-1819: E starts as the spheroid's own field */
		double Eg[3];
		o_spheroid_field(c, part, x, y, z, Eg);
		E[0] = Eg[0];
		E[1] = Eg[1];
		E[2] = Eg[2];
	}
	path[0] = 0;
	do {
		const onode* node = &nodes[path[len - 1]];
		len--;
		if (node->part == O_NONE) {
			dx = x - node->cx;
			dy = y - node->cy;
			dz = z - node->cz;
			dist2 = (dx * dx) + (dy * dy) + (dz * dz);
			if (((node->x2 - node->x1) * (node->x2 - node->x1)) < (oap * oap * dist2)) {
				if (c->cfg.dipoles ? node->aq != 0 : node->q != 0) {
					dist = sqrt(dist2);
					E_scale = O_QE / (4 * O_PI * O_EPSILON0 * dist2 * dist);
					if (c->cfg.dipoles) {
						/* pot.c:1739-1745 */
						double r_dot_p_d2 = (dx * node->px) + (dy * node->py) + (dz * node->pz);
						r_dot_p_d2 /= dist2;
						E[0] += E_scale * ((node->q * dx) - node->px + (3 * dx * r_dot_p_d2));
						E[1] += E_scale * ((node->q * dy) - node->py + (3 * dy * r_dot_p_d2));
						E[2] += E_scale * ((node->q * dz) - node->pz + (3 * dz * r_dot_p_d2));
					} else {
						E_scale *= node->q;
						E[0] += E_scale * dx;
						E[1] += E_scale * dy;
						E[2] += E_scale * dz;
					}
				}
			} else {
				if ((len + 8) > O_MAX_PATH) return -1;
				if (node->ch[0]) {
					for (int s = 0; s < 8; s++) path[len++] = node->ch[s];
				}
			}
		} else if (node->part != part) {
			const pto_particle* p = &c->parts[node->part];
			dx = x - p->x;
			dy = y - p->y;
			dz = z - p->z;
			dist2 = (dx * dx) + (dy * dy) + (dz * dz);
			if (dist2 != 0.0) {
				dist2 += soft * soft;
				dist = sqrt(dist2);
				if (p->species == O_DUST) {
					E_scale = O_QE * c->grain_q / ((4 * O_PI * O_EPSILON0) * dist2 * dist);
				} else {
					E_scale = O_QE * O_CHARGE[p->species] / ((4 * O_PI * O_EPSILON0) * dist2 * dist);
				}
				E[0] += E_scale * dx;
				E[1] += E_scale * dy;
				E[2] += E_scale * dz;
			} else {
				return -2;  /* coincident particles, pot.c:1800-1802 */
			}
		}
	} while (len);
	return 0;
}

static void split_ld(long double v, double* hi, double* lo)
{
	*hi = (double) v;
	*lo = (double) (v - (long double) *hi);
}

void pto_field_many(const pto_ctx* c, uint64_t n, const uint32_t* idx, const double* xyz, double* hi, double* lo)
{
	for (uint64_t k = 0; k < n; k++) {
		long double E[3];
		if (o_field(c, idx[k], xyz[3 * k], xyz[3 * k + 1], xyz[3 * k + 2], E) != 0) {
			E[0] = E[1] = E[2] = NAN;
		}
		for (int d = 0; d < 3; d++) split_ld(E[d], &hi[3 * k + d], &lo[3 * k + d]);
	}
}

/* Direct O(N) sum in long double, after the reference's own accuracy check
   (pot.c:2197-2238) but with the grain's true charge.  soften_all = 1
   softens every pair (as the check does); 0 softens none. */
void pto_field_direct_many(const pto_ctx* c, uint64_t n, const uint32_t* idx, const double* xyz,
                           int32_t soften_all, double* hi, double* lo)
{
	const long double k4 = 4.0L * O_PI * O_EPSILON0;
	for (uint64_t k = 0; k < n; k++) {
		long double E[3] = { 0, 0, 0 };
		long double x = xyz[3 * k], y = xyz[3 * k + 1], z = xyz[3 * k + 2];
		for (uint64_t j = 0; j < c->cfg.N; j++) {
			if (j == idx[k]) continue;
			const pto_particle* p = &c->parts[j];
			long double dx = x - p->x, dy = y - p->y, dz = z - p->z;
			long double d2 = dx * dx + dy * dy + dz * dz;
			if (soften_all) d2 += (long double) c->cfg.soft * c->cfg.soft;
			if (d2 == 0.0L) continue;
			int q = (p->species == O_DUST) ? c->grain_q : O_CHARGE[p->species];
			long double s = O_QE * (long double) q / (k4 * d2 * sqrtl(d2));
			E[0] += s * dx;
			E[1] += s * dy;
			E[2] += s * dz;
		}
		for (int d = 0; d < 3; d++) split_ld(E[d], &hi[3 * k + d], &lo[3 * k + d]);
	}
}

/* potential at a point, every particle included, pot.c:1818-1901 */
double pto_phi_at(const pto_ctx* c, double x, double y, double z)
{
	const double oap = c->cfg.theta;
	const double soft = c->cfg.soft;
	uint32_t path[O_MAX_PATH];
	unsigned int len = 1;
	double phi = 0.0, dist, dist2, dx, dy, dz;
	if (c->cfg.shape) {
		/* pot-spheroid.c:1924-1953 evaluates the spheroid's potential at the
		   point's coordinates themselves, not relative to the grain */
		double u, v, w;
		o_to_frame(c, x, y, z, &u, &v, &w);
		phi = o_spheroid_phi_rel(c, u, v, w);
	}
	path[0] = 0;
	do {
		const onode* node = &c->nodes[path[len - 1]];
		if (node->part != O_NONE) {
			const pto_particle* p = &c->parts[node->part];
			dist2 = ((x - p->x) * (x - p->x)) + ((y - p->y) * (y - p->y)) + ((z - p->z) * (z - p->z));
			dist = sqrt(dist2 + (soft * soft));
			if (p->species == O_DUST) {
				phi += O_QE * c->grain_q / (4 * O_PI * O_EPSILON0 * dist);
			} else {
				phi += O_QE * O_CHARGE[p->species] / (4 * O_PI * O_EPSILON0 * dist);
			}
			len--;
		} else {
			dx = x - node->cx;
			dy = y - node->cy;
			dz = z - node->cz;
			dist2 = (dx * dx) + (dy * dy) + (dz * dz);
			if (((node->x2 - node->x1) * (node->x2 - node->x1)) < (oap * oap * dist2)) {
				if (c->cfg.dipoles) {
					if (node->aq) {  /* pot.c:1860-1868 */
						dist = sqrt(dist2);
						double r_dot_p = (dx * node->px) + (dy * node->py) + (dz * node->pz);
						phi += (O_QE / (4 * O_PI * O_EPSILON0)) * ((node->q / dist) + (r_dot_p / (dist * dist2)));
					}
				} else if (node->q) {
					phi += O_QE * node->q / (4 * O_PI * O_EPSILON0 * sqrt(dist2));
				}
				len--;
			} else {
				len--;
				if ((len + 8) > O_MAX_PATH) return NAN;
				if (node->ch[0]) {
					for (int s = 0; s < 8; s++) path[len++] = node->ch[s];
				}
			}
		}
	} while (len);
	return phi;
}

/* potential felt by particle `part` at its stored position, target
   excluded, pot.c:1934-2018 */
static long double o_phi_particle(const pto_ctx* c, uint32_t part)
{
	const double oap = c->cfg.theta;
	const double soft = c->cfg.soft;
	const pto_particle* t = &c->parts[part];
	uint32_t path[O_MAX_PATH];
	unsigned int len = 1;
	long double phi = 0.0;
	double dist, dist2, dx, dy, dz;
	if (c->cfg.shape) phi = o_spheroid_phi_particle(c, part);  /* pot-spheroid.c:2107-2109 */
	path[0] = 0;
	do {
		const onode* node = &c->nodes[path[len - 1]];
		len--;
		if (node->part == O_NONE) {
			dx = t->x - node->cx;
			dy = t->y - node->cy;
			dz = t->z - node->cz;
			dist2 = (dx * dx) + (dy * dy) + (dz * dz);
			if (((node->x2 - node->x1) * (node->x2 - node->x1)) < (oap * oap * dist2)) {
				if (c->cfg.dipoles) {
					if (node->aq) {  /* pot.c:1966-1974 */
						dist = sqrt(dist2);
						double r_dot_p = (dx * node->px) + (dy * node->py) + (dz * node->pz);
						phi += O_QE * ((node->q / dist) + (r_dot_p / (dist * dist2))) / (4 * O_PI * O_EPSILON0);
					}
				} else if (node->q) {
					phi += O_QE * node->q / (4 * O_PI * O_EPSILON0 * sqrt(dist2));
				}
			} else {
				if ((len + 8) > O_MAX_PATH) return NAN;
				if (node->ch[0]) {
					for (int s = 0; s < 8; s++) path[len++] = node->ch[s];
				}
			}
		} else if (node->part != part) {
			const pto_particle* p = &c->parts[node->part];
			dx = t->x - p->x;
			dy = t->y - p->y;
			dz = t->z - p->z;
			dist2 = (dx * dx) + (dy * dy) + (dz * dz);
			dist = sqrt(dist2 + (soft * soft));
			if (p->species == O_DUST) {
				phi += O_QE * c->grain_q / (4 * O_PI * O_EPSILON0 * dist);
			} else {
				phi += O_QE * O_CHARGE[p->species] / (4 * O_PI * O_EPSILON0 * dist);
			}
		}
	} while (len);
	return phi;
}

double pto_phi_particle_feels(const pto_ctx* c, uint32_t part) { return (double) o_phi_particle(c, part); }

/* normalised edge potential seen by rank k of P, pot.c:2251-2279 */
static double o_chi_b_rank(const pto_ctx* c, int32_t k, int32_t P)
{
	const double azi = 2.0 * O_PI * k / P;
	const double zen = O_PI / 2.0;
	const double r = c->cfg.r * c->cfg.mpp;
	const pto_particle* g = &c->parts[0];
	double phi = pto_phi_at(c, g->x + (r * cos(azi) * sin(zen)), g->y + (r * sin(azi) * sin(zen)),
	                        g->z + (r * cos(zen)));
	return phi / (O_KB * c->cfg.Ti / (O_CHARGE[O_ION] * O_QE));
}

/* MPI_Allreduce(SUM) of the ranks' samples, then / num_workers (pot.c:2409-2418) */
double pto_measure_chi_b_ranks(const pto_ctx* c, int32_t P)
{
	if (P < 1) P = 1;
	double sum = 0.0;
	for (int32_t k = 0; k < P; k++) sum += o_chi_b_rank(c, k, P);
	return sum / P;
}

/* normalised edge potential at azimuth 0 (one rank), pot.c:2251-2279 */
double pto_measure_chi_b(const pto_ctx* c)
{
	const double azi = 0.0;
	const double zen = O_PI / 2.0;
	const double r = c->cfg.r * c->cfg.mpp;
	const pto_particle* g = &c->parts[0];
	double phi = pto_phi_at(c, g->x + (r * cos(azi) * sin(zen)), g->y + (r * sin(azi) * sin(zen)),
	                        g->z + (r * cos(zen)));
	return phi / (O_KB * c->cfg.Ti / (O_CHARGE[O_ION] * O_QE));
}

/* ------------------------------------------------------------------------ */
/* Absorption and the step                                                  */
/* ------------------------------------------------------------------------ */

/* point-in-sphere or segment closest approach, pot.c:2287-2325 */
int pto_cross_grain(const pto_particle* p, const double* d_pos, const pto_particle* gr, double a)
{
	double alpha, d_dot_s, d_pos2, dist2, s[3], s2;
	s[0] = gr->x - p->x;
	s[1] = gr->y - p->y;
	s[2] = gr->z - p->z;
	s2 = (s[0] * s[0]) + (s[1] * s[1]) + (s[2] * s[2]);
	if (s2 <= (a * a)) return 1;
	d_pos2 = (d_pos[0] * d_pos[0]) + (d_pos[1] * d_pos[1]) + (d_pos[2] * d_pos[2]);
	d_dot_s = (d_pos[0] * s[0]) + (d_pos[1] * s[1]) + (d_pos[2] * s[2]);
	alpha = d_dot_s / d_pos2;
	if ((alpha < -1.0) || (alpha > 0.0)) return 0;
	dist2 = s2 - (alpha * d_dot_s);
	return dist2 <= (a * a);
}

/* spheroid absorption test, pot-spheroid.c:2448-2537: (1) the new position
   inside x^2 + A^2 rho^2 <= a^2 A^(4/3); (2) the closest approach of the
   step's line, found in the x-rho plane, between the old and new x and
   inside the surface.  s and d_pos are taken into the spheroid's frame
   first (the identity for the reference's x axis). */
static int o_cross_spheroid(const pto_ctx* c, const pto_particle* p, const double* d_pos, const pto_particle* gr)
{
	const double a = c->cfg.a, A = c->cfg.A;
	double s[3], d[3], x_min, x_prev, y_min, z_min;
	o_to_frame(c, gr->x - p->x, gr->y - p->y, gr->z - p->z, &s[0], &s[1], &s[2]);
	o_to_frame(c, d_pos[0], d_pos[1], d_pos[2], &d[0], &d[1], &d[2]);
	if ((s[0] * s[0] + (s[1] * s[1] + s[2] * s[2]) * A * A) <= (a * a * pow(A, 4.0 / 3.0))) return 1;
	x_min = (d[1] * (d[1] * s[0] - d[0] * s[1]) + d[2] * (d[2] * s[0] - d[0] * s[2]))
	        / ((d[0] * d[0] / (A * A)) + d[1] * d[1] + d[2] * d[2]);
	x_prev = s[0] - d[0];
	if (((x_min > s[0]) && (x_min > x_prev)) || ((x_min < s[0]) && (x_min < x_prev))) return 0;
	y_min = d[1] * (x_min - s[0]) / d[0] + s[1];
	z_min = d[2] * (x_min - s[0]) / d[0] + s[2];
	return ((x_min * x_min) + (y_min * y_min + z_min * z_min) * A * A) <= (a * a * pow(A, 4.0 / 3.0));
}

int pto_cross_grain_run(const pto_ctx* c, const pto_particle* p, const double* d_pos, const pto_particle* gr)
{
	if (c->cfg.shape) return o_cross_spheroid(c, p, d_pos, gr);
	return pto_cross_grain(p, d_pos, gr, c->cfg.a);
}

/* One rank's move_particles with the Boris integrator, pot.c:2330-2934,
   without MPI: memcpy, chi_b refresh, due range, half-drift, field, kick,
   rotate, kick, half-drift, absorption + reinjection, boundary reinjection,
   optional potential energies, grain update. */
static int o_move(pto_ctx* c, int compute_epe, uint64_t time_steps)
{
	const pto_cfg* ru = &c->cfg;
	const uint64_t N = ru->N;
	const double B[3] = { ru->B[0], ru->B[1], ru->B[2] };
	const double B_mag = sqrt(B[0] * B[0] + B[1] * B[1] + B[2] * B[2]);
	const double bh[3] = { B[0] / B_mag, B[1] / B_mag, B[2] / B_mag };
	pto_particle* parts = c->parts;
	pto_particle* np = c->new_parts;
	uint32_t absorbed_e = 0, n_abs = 0, n_rein = 0;
	long double absorbed_m = 0.0;
	int absorbed_q = 0;
	long double dpx = 0.0, dpy = 0.0, dpz = 0.0;
	uint64_t start, i;

	memcpy(np, parts, sizeof(pto_particle) * N);

	if (ru->sceptic && !(c->t_steps % 20)) {
		if (ru->chi_ranks > 1) {
			c->chi_b = pto_measure_chi_b_ranks(c, ru->chi_ranks);
		} else {
			c->chi_b = pto_measure_chi_b(c);
			c->chi_b /= 1;  /* averaged over one rank */
		}
	}

	for (start = 0; start < N; start++) {
		if (!(time_steps % c->tss[parts[start].species])) break;
	}
	for (i = start; i < N; i++) {
		c->prev[3 * (i - start)] = parts[i].x;
		c->prev[3 * (i - start) + 1] = parts[i].y;
		c->prev[3 * (i - start) + 2] = parts[i].z;
	}

	for (i = start; i < N; i++) {
		pto_particle* p = &parts[i];
		long double dt = c->dt * c->tss[p->species];
		double hx, hy, hz;
		long double E[3], qom, ax, ay, az;
		if (ru->integrator) {
			/* velocity Verlet / Euler-Richardson, first half (pot.c:2533-2552):
			   the field at the old position, no half drift */
			int rc = o_field(c, (uint32_t) i, p->x, p->y, p->z, E);
			if (rc) return rc == -1 ? -4 : -2;
			if (p->species == O_DUST) {
				qom = O_QE * c->grain_q;
			} else {
				qom = O_QE * O_CHARGE[p->species];
			}
			qom /= c->mass[p->species];
			long double* a1 = &c->acc[3 * (i - start)];
			a1[0] = qom * (E[0] + p->vy * B[2] - p->vz * B[1]);
			a1[1] = qom * (E[1] + p->vz * B[0] - p->vx * B[2]);
			a1[2] = qom * (E[2] + p->vx * B[1] - p->vy * B[0]);
			np[i].vx += 0.5 * dt * a1[0];
			np[i].vy += 0.5 * dt * a1[1];
			np[i].vz += 0.5 * dt * a1[2];
			if (ru->integrator == 2) {
				np[i].x += 0.5 * dt * p->vx;
				np[i].y += 0.5 * dt * p->vy;
				np[i].z += 0.5 * dt * p->vz;
			} else {
				np[i].x += dt * (p->vx + (0.5 * dt * a1[0]));
				np[i].y += dt * (p->vy + (0.5 * dt * a1[1]));
				np[i].z += dt * (p->vz + (0.5 * dt * a1[2]));
			}
			continue;
		}
		if (ru->quirk) {
			p->x += 0.5 * dt * p->vx;
			p->y += 0.5 * dt * p->vy;
			p->z += 0.5 * dt * p->vz;
			hx = p->x; hy = p->y; hz = p->z;
		} else {
			hx = p->x + 0.5 * dt * p->vx;
			hy = p->y + 0.5 * dt * p->vy;
			hz = p->z + 0.5 * dt * p->vz;
		}
		int rc = o_field(c, (uint32_t) i, hx, hy, hz, E);
		if (rc) return rc == -1 ? -4 : -2;
		if (p->species == O_DUST) {
			qom = O_QE * c->grain_q;
		} else {
			qom = O_QE * O_CHARGE[p->species];
		}
		qom /= c->mass[p->species];
		ax = 0.5 * qom * E[0];
		ay = 0.5 * qom * E[1];
		az = 0.5 * qom * E[2];
		np[i].vx += dt * ax;
		np[i].vy += dt * ay;
		np[i].vz += dt * az;
		if (B_mag) {
			double dephi = 2.0 * atanl(0.5 * dt * qom * B_mag);
			o_rot(bh, sin(dephi), cos(dephi), &np[i].vx, &np[i].vy, &np[i].vz);
		}
		np[i].vx += dt * ax;
		np[i].vy += dt * ay;
		np[i].vz += dt * az;
		np[i].x = hx + (0.5 * dt * np[i].vx);
		np[i].y = hy + (0.5 * dt * np[i].vy);
		np[i].z = hz + (0.5 * dt * np[i].vz);
	}

	/* the non-Boris integrators' mid-step exchange (pot.c:2556-2597): every
	   particle's intermediate state replaces the old one, so the second
	   field evaluation sees leaf particles there while the cells keep the
	   moments of the tree built at the start of the step */
	if (ru->integrator) memcpy(parts, np, sizeof(pto_particle) * N);

	const double rad = ru->r * ru->mpp;
	uint32_t n_wall = 0;
	for (i = start; i < N; i++) {
		pto_particle* pn = &np[i];
		uint64_t ims = i - start;
		uint32_t attempt = 0;
		if (ru->integrator) {
			/* second half (pot.c:2605-2638) */
			const pto_particle* p = &parts[i];
			long double E[3], qom, a_x2, a_y2, a_z2;
			int rc = o_field(c, (uint32_t) i, p->x, p->y, p->z, E);
			if (rc) return rc == -1 ? -4 : -2;
			if (p->species == O_DUST) {
				qom = O_QE * c->grain_q;
			} else {
				qom = O_QE * O_CHARGE[p->species];
			}
			qom /= c->mass[p->species];
			a_x2 = qom * (E[0] + p->vy * B[2] - p->vz * B[1]);
			a_y2 = qom * (E[1] + p->vz * B[0] - p->vx * B[2]);
			a_z2 = qom * (E[2] + p->vx * B[1] - p->vy * B[0]);
			long double dt = c->dt * c->tss[p->species];
			const long double* a1 = &c->acc[3 * ims];
			if (ru->integrator == 2) {
				pn->x = (p->x - 0.5 * dt * (p->vx - 0.5 * dt * a1[0])) + dt * p->vx;
				pn->y = (p->y - 0.5 * dt * (p->vy - 0.5 * dt * a1[1])) + dt * p->vy;
				pn->z = (p->z - 0.5 * dt * (p->vz - 0.5 * dt * a1[2])) + dt * p->vz;
				pn->vx = (p->vx - 0.5 * dt * a1[0]) + dt * a_x2;
				pn->vy = (p->vy - 0.5 * dt * a1[1]) + dt * a_y2;
				pn->vz = (p->vz - 0.5 * dt * a1[2]) + dt * a_z2;
			} else {
				pn->vx += 0.5 * dt * a_x2;
				pn->vy += 0.5 * dt * a_y2;
				pn->vz += 0.5 * dt * a_z2;
			}
		}
		if ((i > 0) && ((time_steps * c->dt) > ru->settle)) {
			double d[3] = { pn->x - c->prev[3 * ims], pn->y - c->prev[3 * ims + 1], pn->z - c->prev[3 * ims + 2] };
			if (pto_cross_grain_run(c, pn, d, &np[0])) {
				if (pn->species == O_ELECTRON) absorbed_e++;
				absorbed_m += c->mass[pn->species];
				absorbed_q += O_CHARGE[pn->species];
				/* POIS_POS_COLLECTION: a positive particle's charge is undone
				   (pot.c:2664-2670) */
				if (ru->pois_ions && O_CHARGE[pn->species] > 0) absorbed_q -= O_CHARGE[pn->species];
				dpx += c->mass[pn->species] * pn->vx;
				dpy += c->mass[pn->species] * pn->vy;
				dpz += c->mass[pn->species] * pn->vz;
				if (ru->rng) ph_stream(c, (uint32_t) i, time_steps, 0x10000u | attempt);
				attempt++;
				o_inject(c, pn, 1);
				n_abs++;
				n_rein++;
			}
		}
		if (ru->bounce > 0.0) {
			/* check_particle_in_sim_area with OUT_BOUNCE, pot.c:2036-2069: a
			   particle outside the sphere moving outwards has its radial
			   velocity reversed, every component scaled by the coefficient
			   of restitution, and goes back to its position at the start of
			   the step; one moving inwards is left where it is (the
			   reference's warning, pot.c:2719-2722) */
			const double bounce = ru->bounce;
			double r[3], v[3];
			r[0] = sqrt((pn->x - rad) * (pn->x - rad) + (pn->y - rad) * (pn->y - rad) + (pn->z - rad) * (pn->z - rad));
			if (r[0] > rad) {
				r[1] = atan2l(pn->y - rad, pn->x - rad);
				r[2] = acosl((pn->z - rad) / r[0]);
				v[0] = pn->vx * cos(r[1]) * sin(r[2]) + pn->vy * sin(r[1]) * sin(r[2]) + pn->vz * cos(r[2]);
				v[1] = -pn->vx * sin(r[1]) + pn->vy * cos(r[1]);
				v[2] = pn->vx * cos(r[1]) * cos(r[2]) + pn->vy * sin(r[1]) * cos(r[2]) - pn->vz * sin(r[2]);
				if (v[0] > 0.0) {
					v[0] *= -bounce;
					v[1] *= bounce;
					v[2] *= bounce;
					o_vel_cart(v, r[1], r[2], &pn->vx, &pn->vy, &pn->vz);
					pn->x = c->prev[3 * ims];
					pn->y = c->prev[3 * ims + 1];
					pn->z = c->prev[3 * ims + 2];
				} else {
					n_wall++;
				}
			}
			continue;
		}
		/* check_particle_in_sim_area, pot.c:2025-2076 (spherical, no bounce) */
		{
			double ddx = pn->x - rad, ddy = pn->y - rad, ddz = pn->z - rad;
			if (sqrt((ddx * ddx) + (ddy * ddy) + (ddz * ddz)) > rad) {
				if (ru->rng) ph_stream(c, (uint32_t) i, time_steps, 0x10000u | attempt);
				attempt++;
				o_inject(c, pn, 1);
				n_rein++;
			}
		}
	}

	if (compute_epe) {
		c->epe[O_ELECTRON] = 0.0;
		c->epe[O_ION] = 0.0;
		for (i = 1; i < N; i++) {
			pto_particle* pn = &np[i];
			c->epe[pn->species] += O_QE * O_CHARGE[pn->species] * o_phi_particle(c, (uint32_t) i);
		}
	}

	c->grain_m += absorbed_m;
	np[0].vx += dpx / c->grain_m;
	np[0].vy += dpy / c->grain_m;
	np[0].vz += dpz / c->grain_m;
	c->grain_q += absorbed_q;
	c->tot_absor_e += absorbed_e;
	c->st_pois = 0;
	if (ru->pois_ions && ((time_steps * c->dt) > ru->settle)) {
		/* POIS_POS_COLLECTION, pot.c:2837-2854: an OML ion flux at the cached
		   ion temperature, Poisson-sampled once per step */
		double kb_ti = O_KB * c->ion_temp;
		double phi_normed = O_CHARGE[O_ION] * O_QE * O_QE * c->grain_q;
		phi_normed /= 4.0 * O_PI * O_EPSILON0 * ru->a * kb_ti;
		double lambda = c->pos_rate_const * sqrt(kb_ti) * (1.0 - phi_normed);
		if (ru->rng) ph_stream(c, 0, time_steps, 0x30000u);
		c->st_pois = o_prv(c, lambda);
		c->grain_q += c->st_pois;
	}
	c->st_wall = n_wall;
	if (compute_epe) {
		c->epe[O_DUST] = c->grain_q ? c->grain_q * O_QE * o_phi_particle(c, 0) : 0.0;
	}
	memcpy(parts, np, sizeof(pto_particle) * N);

	c->st_dq = absorbed_q;
	c->st_de = absorbed_e;
	c->st_nabs = n_abs;
	c->st_nrein = n_rein;
	c->st_npush = N - start;
	return 0;
}

int pto_step(pto_ctx* c, int32_t compute_epe)
{
	c->t_steps++;
	int rc = pto_build_tree(c);
	if (rc) return rc;
	return o_move(c, compute_epe, c->t_steps);
}

int pto_run_steps(pto_ctx* c, uint64_t n, int32_t compute_epe)
{
	for (uint64_t k = 0; k < n; k++) {
		int rc = pto_step(c, compute_epe);
		if (rc) return rc;
	}
	return 0;
}

void pto_last_step_stats(const pto_ctx* c, int64_t* dq, uint32_t* de, uint32_t* n_absorbed,
                         uint32_t* n_reinjected, uint64_t* n_pushed, double* epe3)
{
	*dq = c->st_dq;
	*de = c->st_de;
	*n_absorbed = c->st_nabs;
	*n_reinjected = c->st_nrein;
	*n_pushed = c->st_npush;
	for (int k = 0; k < 3; k++) epe3[k] = (double) c->epe[k];
}

void pto_last_step_variant_stats(const pto_ctx* c, uint32_t* n_pois, uint32_t* n_wall)
{
	*n_pois = c->st_pois;
	*n_wall = c->st_wall;
}

void pto_sample_reinject(pto_ctx* c, uint64_t n, int32_t species, pto_particle* out)
{
	for (uint64_t k = 0; k < n; k++) {
		pto_particle p;
		memset(&p, 0, sizeof(p));
		p.species = species;
		if (c->cfg.rng) ph_stream(c, (uint32_t) k, c->t_steps, 0x10000u);
		o_inject(c, &p, 1);
		out[k] = p;
	}
}
