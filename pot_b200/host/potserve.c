/*
 * potserve -- many grain-charging runs on one B200: a batched sweep and a
 * serving loop with continuous batching (no counterpart in the reference,
 * which runs one grain per MPI job).
 *
 * Jobs.  Each job is one run of the reference's physics (spherical domain of
 * radius 8 Debye lengths, theta 0.5, SCEPTIC reinjection, Boris push) with
 *   N        log-uniform in [--nmin, --nmax] particles (odd: grain + pairs),
 *   a        log-uniform in [0.01, 1] Debye lengths,
 *   Te/Ti    uniform in {1, 3, 10, 30} (Te = 11,600 K),
 *   Mach     uniform in [0, 2] of the ion sound speed sqrt(k Te / m_i),
 *   B        (serve mode) uniform in [0, --bmax] tesla along z,
 * a Debye length fixed by N and the domain, lambda = 3 (N - 1) e^2 /
 * (4096 pi eps0 k Te), softening 0.01 lambda, dt = 0.005 / omega_pe, and
 * Philox seed --seed + i.
 *
 * Convergence.  A run is done when the 500-step moving mean of its grain
 * charge changes by less than 0.5 % between consecutive 500-step windows
 * (checked every --epoch steps from the device-side charge sums), or at
 * --max-steps.
 *
 * sweep: all --runs jobs are queued at t = 0.
 * serve: jobs arrive as a Poisson stream of --rate per second for
 *        --duration seconds; a job is admitted as soon as the batch has room
 *        (free HBM above --reserve-gb and fewer than --max-runs members) and
 *        joins the next graph launch; a finished run is evicted at once.
 * Both print one JSON object: p50 / p99 time from arrival to converged
 * charge, aggregate particle-steps/s, queue depth, and (with
 * --plain-sample K) the first K jobs run one at a time in the plain FP64
 * form for comparison.  --tune picks leaf and group sizes per size class
 * with the library's autotuner.  The batch packs its fast-form runs (one
 * launch per kernel of the step over all of them); --no-pack steps each run
 * as its own kernel sequence instead, for comparison.  --wall-limit S stops
 * after S seconds and reports the jobs finished inside that window, and the
 * jobs running and waiting at the stop.  Jobs run with
 * POT_OPT_CHI_CAP (the sampler's edge potential capped where the
 * reference's inverse CDF is undefined, so a cold-ion job with a noisy edge
 * potential goes on instead of stopping with POT_E_ITER); --strict-sampler
 * runs them as the reference would, stopping such jobs.
 */
#define _POSIX_C_SOURCE 200809L
#include <math.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "pot_gpu.h"

#define KB 1.38065e-23
#define EPSILON0 8.85419e-12
#define QE 1.6021766e-19
#define ME 9.109383e-31
#define MI (1836.15 * ME)
#define PI 3.14159265358979

typedef struct {
	pot_run_cfg cfg;
	uint64_t seed;
	double arrival, admitted, done;
	uint64_t steps;
	int slot;
	int state;  /* 0 waiting, 1 running, 2 finished */
	bool converged;
	int64_t* qs;      /* q_sum checkpoints, one per epoch */
	uint32_t n_qs, cap_qs;
	uint64_t t0;      /* t_steps at admission */
	uint32_t leaf, group;
} Job;

static uint64_t sm_state;
static double urand(void)
{
	uint64_t z = (sm_state += 0x9E3779B97F4A7C15ull);
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	z ^= z >> 31;
	return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

static double now_s(void)
{
	struct timespec t;
	clock_gettime(CLOCK_MONOTONIC, &t);
	return (double)t.tv_sec + 1e-9 * (double)t.tv_nsec;
}

static void make_job(Job* j, uint64_t id, double nmin, double nmax, double bmax, uint64_t seed0)
{
	memset(j, 0, sizeof(*j));
	uint64_t N = (uint64_t)exp(log(nmin) + urand() * (log(nmax) - log(nmin)));
	N |= 1u;
	const double Te = 11600.0;
	const double ratios[4] = { 1.0, 3.0, 10.0, 30.0 };
	const double Ti = Te / ratios[(int)(urand() * 4.0) & 3];
	const double mach = 2.0 * urand();
	const double a_rel = exp(log(0.01) + urand() * (log(1.0) - log(0.01)));
	const double lambda = 3.0 * (double)(N - 1) * QE * QE / (4096.0 * PI * EPSILON0 * KB * Te);
	const double R = 8.0 * lambda;
	const double n_tot = (double)(N - 1) / ((4.0 / 3.0) * PI * R * R * R);
	const double w_pe = sqrt((n_tot / 2.0) * QE * QE / (EPSILON0 * ME));
	pot_run_cfg* c = &j->cfg;
	c->N = N;
	c->r = 1000;
	c->flags = POT_CFG_SCEPTIC;
	c->mpp = R / 1000.0;
	c->a = a_rel * lambda;
	c->soft = 0.01 * lambda;
	c->dt = 0.005 / w_pe;
	c->Te = Te;
	c->Ti = Ti;
	c->x_drift = mach * sqrt(KB * Te / MI);
	c->settle = 0.0;
	c->theta = 0.5;
	c->B[2] = bmax > 0.0 ? bmax * urand() : 0.0;
	j->seed = seed0 + id;
	j->slot = -1;
}

static int cmp_double(const void* a, const void* b)
{
	const double x = *(const double*)a, y = *(const double*)b;
	return (x > y) - (x < y);
}

static double pct(double* v, int n, double p)
{
	if (n <= 0) return NAN;
	qsort(v, (size_t)n, sizeof(double), cmp_double);
	int k = (int)ceil(p * n) - 1;
	if (k < 0) k = 0;
	if (k >= n) k = n - 1;
	return v[k];
}

/* moving-mean test on the checkpoints (spaced `epoch` steps) */
static bool converged(const Job* j, uint32_t epoch)
{
	const uint32_t w = 500 / epoch;
	if (j->n_qs < 2 * w + 1) return false;
	const int64_t* q = j->qs;
	const uint32_t e = j->n_qs - 1;
	const double m1 = (double)(q[e] - q[e - w]) / 500.0;
	const double m0 = (double)(q[e - w] - q[e - 2 * w]) / 500.0;
	if (m1 == 0.0) return false;
	return fabs(m1 - m0) <= 0.005 * fabs(m1);
}

/* the grain charge averaged over the run's last 500 steps (NaN if shorter) */
static double final_mean(const Job* j, uint32_t epoch)
{
	const uint32_t w = 500 / epoch;
	if (j->n_qs < w + 1) return NAN;
	const uint32_t e = j->n_qs - 1;
	return (double)(j->qs[e] - j->qs[e - w]) / 500.0;
}

static void push_q(Job* j, int64_t q)
{
	if (j->n_qs == j->cap_qs) {
		j->cap_qs = j->cap_qs ? 2 * j->cap_qs : 64;
		j->qs = realloc(j->qs, sizeof(int64_t) * j->cap_qs);
	}
	j->qs[j->n_qs++] = q;
}

typedef struct {
	double n;
	uint32_t leaf, group;
} TuneEntry;

/* a JSON number, or null for NaN / infinity */
static const char* jnum(char* buf, double v)
{
	if (!isfinite(v)) return "null";
	snprintf(buf, 32, "%.4f", v);
	return buf;
}

int main(int argc, char** argv)
{
	const char* mode = "sweep";
	int runs = 256, plain_sample = 0, max_runs = 4096, device = 0;
	double nmin = 16000, nmax = 256000, rate = 20.0, duration = 600.0, bmax = 0.0, reserve_gb = 8.0;
	uint64_t max_steps = 20000, seed0 = 1000, gen_seed = 12345;
	uint32_t epoch = 50;
	bool tune = false, pack = true, chi_cap = true;
	double wall_limit = 0.0;  /* stop after this many seconds (0: when every job is done) */
	for (int k = 1; k < argc; k++) {
		const char* f = argv[k];
		const char* v = k + 1 < argc ? argv[k + 1] : "";
		if (!strcmp(f, "--mode")) { mode = v; k++; }
		else if (!strcmp(f, "--runs")) { runs = atoi(v); k++; }
		else if (!strcmp(f, "--nmin")) { nmin = atof(v); k++; }
		else if (!strcmp(f, "--nmax")) { nmax = atof(v); k++; }
		else if (!strcmp(f, "--rate")) { rate = atof(v); k++; }
		else if (!strcmp(f, "--duration")) { duration = atof(v); k++; }
		else if (!strcmp(f, "--bmax")) { bmax = atof(v); k++; }
		else if (!strcmp(f, "--max-steps")) { max_steps = strtoull(v, NULL, 10); k++; }
		else if (!strcmp(f, "--max-runs")) { max_runs = atoi(v); k++; }
		else if (!strcmp(f, "--epoch")) { epoch = (uint32_t)atoi(v); k++; }
		else if (!strcmp(f, "--seed")) { seed0 = strtoull(v, NULL, 10); k++; }
		else if (!strcmp(f, "--gen-seed")) { gen_seed = strtoull(v, NULL, 10); k++; }
		else if (!strcmp(f, "--reserve-gb")) { reserve_gb = atof(v); k++; }
		else if (!strcmp(f, "--plain-sample")) { plain_sample = atoi(v); k++; }
		else if (!strcmp(f, "--device")) { device = atoi(v); k++; }
		else if (!strcmp(f, "--tune")) { tune = true; }
		else if (!strcmp(f, "--no-pack")) { pack = false; }
		else if (!strcmp(f, "--strict-sampler")) { chi_cap = false; }
		else if (!strcmp(f, "--wall-limit")) { wall_limit = atof(v); k++; }
		else {
			fprintf(stderr, "usage: %s [--mode sweep|serve] [--runs N] [--nmin N] [--nmax N] [--rate R] "
			                "[--duration S] [--bmax T] [--max-steps N] [--max-runs N] [--epoch N] [--seed S] "
			                "[--gen-seed S] [--reserve-gb G] [--plain-sample K] [--tune] [--no-pack] [--strict-sampler] "
			        "[--wall-limit S] [--device D]\n",
			        argv[0]);
			return 2;
		}
	}
	const bool serve = !strcmp(mode, "serve");
	if (epoch == 0 || epoch % 2 || 500 % epoch) {
		fprintf(stderr, "--epoch must be even and divide 500\n");
		return 2;
	}
	sm_state = gen_seed;
	/* the job list: arrival times and parameters */
	int n_jobs = serve ? 0 : runs;
	Job* jobs = NULL;
	if (serve) {
		int cap = 1024;
		jobs = calloc((size_t)cap, sizeof(Job));
		double t = 0.0;
		for (;;) {
			t += -log(1.0 - urand()) / rate;
			if (t > duration) break;
			if (n_jobs == cap) {
				cap *= 2;
				jobs = realloc(jobs, sizeof(Job) * (size_t)cap);
			}
			make_job(&jobs[n_jobs], (uint64_t)n_jobs, nmin, nmax, bmax, seed0);
			jobs[n_jobs].arrival = t;
			n_jobs++;
		}
	} else {
		jobs = calloc((size_t)(n_jobs > 0 ? n_jobs : 1), sizeof(Job));
		for (int i = 0; i < n_jobs; i++) make_job(&jobs[i], (uint64_t)i, nmin, nmax, bmax, seed0);
	}
	pot_batch* b = NULL;
	pot_batch_opts bo;
	memset(&bo, 0, sizeof(bo));
	bo.device = device;
	bo.steps_per_launch = 2;
	bo.reserve_bytes = (uint64_t)(reserve_gb * 1073741824.0);
	bo.flags = pack ? 0u : POT_BATCH_NO_PACK;
	int rc = pot_batch_create(&bo, &b);
	if (rc != POT_OK) {
		fprintf(stderr, "pot_batch_create: %s\n", pot_gpu_strerror(rc));
		return 1;
	}
	/* autotuner cache per size class (N rounded to a power of two) */
	TuneEntry tcache[64];
	int n_tc = 0;
	double tune_s = 0.0;
	pot_batch_row* rows = calloc((size_t)(n_jobs > 0 ? n_jobs : 1), sizeof(pot_batch_row));
	int* slot_job = calloc((size_t)(n_jobs + 4096), sizeof(int));
	int next = 0, active = 0, finished = 0, max_active = 0, converged_n = 0, failed_n = 0, capped_n = 0;
	double ps = 0.0, queue_sum = 0.0, queue_max = 0.0;
	uint64_t n_epochs = 0;
	const double t_start = now_s();
	bool stopped = false;
	while (finished < n_jobs) {
		const double t = now_s() - t_start;
		if (wall_limit > 0.0 && t >= wall_limit) {
			stopped = true;  /* the window is over: report what finished inside it */
			break;
		}
		/* admission (FIFO) */
		while (next < n_jobs && (!serve || jobs[next].arrival <= t) && active < max_runs) {
			Job* j = &jobs[next];
			pot_gpu_opts o;
			memset(&o, 0, sizeof(o));
			o.form = POT_FORM_FAST;
			o.device = device;
			o.seed = j->seed;
			o.flags = chi_cap ? POT_OPT_CHI_CAP : 0u;
			if (tune) {
				const double cls = pow(2.0, floor(log2((double)j->cfg.N) + 0.5));
				int e = 0;
				while (e < n_tc && tcache[e].n != cls) e++;
				if (e == n_tc && n_tc < 64) {
					const double t0 = now_s();
					pot_gpu_opts to = o;
					double ms = 0.0;
					if (pot_gpu_tune(&j->cfg, &to, 6, &ms) != POT_OK) {
						to.leaf_size = 16;
						to.group_size = 32;
					}
					tcache[n_tc].n = cls;
					tcache[n_tc].leaf = to.leaf_size;
					tcache[n_tc].group = to.group_size;
					n_tc++;
					tune_s += now_s() - t0;
				}
				if (e < n_tc) {
					o.leaf_size = tcache[e].leaf;
					o.group_size = tcache[e].group;
				}
			}
			int32_t slot = -1;
			rc = pot_batch_admit(b, &j->cfg, &o, NULL, NULL, &slot);
			if (rc == POT_E_NOMEM) break;  /* HBM full: wait for evictions */
			if (rc != POT_OK) {
				fprintf(stderr, "admit job %d (N=%lu): %s\n", next, (unsigned long)j->cfg.N, pot_gpu_strerror(rc));
				j->state = 2;
				j->done = now_s() - t_start;
				finished++;
				next++;
				continue;
			}
			j->slot = slot;
			j->state = 1;
			j->admitted = now_s() - t_start;
			j->leaf = o.leaf_size;
			j->group = o.group_size;
			slot_job[slot] = next;
			push_q(j, 0);
			active++;
			next++;
		}
		if (active > max_active) max_active = active;
		/* queue depth: arrived but not admitted */
		int queued = 0;
		for (int i = next; i < n_jobs && (!serve || jobs[i].arrival <= t); i++) queued++;
		queue_sum += queued;
		if (queued > queue_max) queue_max = queued;
		n_epochs++;
		if (active == 0) {
			if (next < n_jobs) {
				/* idle until the next arrival */
				const double wait = jobs[next].arrival - (now_s() - t_start);
				if (wait > 0) {
					struct timespec ts = { (time_t)wait, (long)((wait - floor(wait)) * 1e9) };
					nanosleep(&ts, NULL);
				}
				continue;
			}
			break;
		}
		if ((rc = pot_batch_step(b, epoch)) != POT_OK) {
			fprintf(stderr, "pot_batch_step: %s\n", pot_gpu_strerror(rc));
			break;
		}
		uint32_t nr = 0;
		if ((rc = pot_batch_summary(b, (uint32_t)n_jobs, rows, &nr)) != POT_OK) {
			fprintf(stderr, "pot_batch_summary: %s\n", pot_gpu_strerror(rc));
			break;
		}
		const double tnow = now_s() - t_start;
		for (uint32_t r = 0; r < nr; r++) {
			Job* j = &jobs[slot_job[rows[r].slot]];
			if (rows[r].status != POT_OK) {
				const pot_run_cfg* c = &j->cfg;
				fprintf(stderr, "run %d failed at step %lu: %s (warn %u; N %lu, a %g m, Te/Ti %g, drift %g m/s, q %ld)\n",
				        slot_job[rows[r].slot], (unsigned long)rows[r].t_steps, pot_gpu_strerror(rows[r].status),
				        rows[r].warn, (unsigned long)c->N, c->a, c->Te / c->Ti, c->x_drift, (long)rows[r].grain_q);
				failed_n++;
			}
			const uint64_t st = rows[r].t_steps;
			ps += (double)(st - j->steps) * (double)(j->cfg.N - 1);
			j->steps = st;
			push_q(j, rows[r].q_sum);
			const bool conv = converged(j, epoch);
			if (conv || st >= max_steps || rows[r].status != POT_OK) {
				j->converged = conv;
				converged_n += conv;
				capped_n += (rows[r].warn & 512u) != 0;
				j->done = tnow;
				j->state = 2;
				pot_batch_evict(b, rows[r].slot);
				active--;
				finished++;
			}
		}
	}
	const double wall = now_s() - t_start;
	/* latencies */
	double* lat = calloc((size_t)(n_jobs > 0 ? n_jobs : 1), sizeof(double));
	double* lat_c = calloc((size_t)(n_jobs > 0 ? n_jobs : 1), sizeof(double));
	int nl = 0, nlc = 0;
	double steps_sum = 0.0;
	for (int i = 0; i < n_jobs; i++) {
		if (jobs[i].state != 2) continue;
		lat[nl++] = jobs[i].done - jobs[i].arrival;
		if (jobs[i].converged) lat_c[nlc++] = jobs[i].done - jobs[i].arrival;
		steps_sum += (double)jobs[i].steps;
	}
	char b1[32], b2[32], b3[32], b4[32], b5[32];
	printf("{\"mode\": \"%s\", \"jobs\": %d, \"finished\": %d, \"failed\": %d, \"converged\": %d, \"capped_at_max_steps\": %d, "
	       "\"max_steps\": %lu, \"wall_s\": %.3f, \"particle_steps\": %.6e, \"particle_steps_per_s\": %.6e, "
	       "\"latency_s\": {\"p50\": %s, \"p99\": %s, \"max\": %s}, "
	       "\"latency_converged_s\": {\"p50\": %s, \"p99\": %s}, \"mean_steps\": %.1f, "
	       "\"max_concurrent_runs\": %d, \"queue_depth\": {\"mean\": %.2f, \"max\": %.0f}, \"epochs\": %lu, "
	       "\"epoch_steps\": %u, \"tuned_classes\": %d, \"tune_s\": %.3f, \"packed\": %s, \"chi_cap\": %s, "
	       "\"runs_chi_capped\": %d",
	       mode, n_jobs, finished, failed_n, converged_n, finished - converged_n - failed_n, (unsigned long)max_steps, wall, ps,
	       wall > 0 ? ps / wall : 0.0, jnum(b1, pct(lat, nl, 0.5)), jnum(b2, pct(lat, nl, 0.99)),
	       jnum(b3, pct(lat, nl, 1.0)), jnum(b4, pct(lat_c, nlc, 0.5)), jnum(b5, pct(lat_c, nlc, 0.99)),
	       nl ? steps_sum / nl : 0.0, max_active,
	       n_epochs ? queue_sum / (double)n_epochs : 0.0, queue_max, (unsigned long)n_epochs, epoch, n_tc, tune_s,
	       pack ? "true" : "false", chi_cap ? "true" : "false", capped_n);
	if (serve) printf(", \"rate_per_s\": %g, \"duration_s\": %g", rate, duration);
	if (wall_limit > 0.0) {
		int arrived = 0;
		for (int i = 0; i < n_jobs; i++) arrived += !serve || jobs[i].arrival <= wall;
		printf(", \"wall_limit_s\": %g, \"stopped_at_wall_limit\": %s, \"arrived\": %d, \"running_at_stop\": %d, "
		       "\"waiting_at_stop\": %d", wall_limit, stopped ? "true" : "false", arrived, active, arrived - next);
	}
	printf(", \"n_range\": [%g, %g]", nmin, nmax);
	if (tune && n_tc) {
		printf(", \"tuned\": [");
		for (int e = 0; e < n_tc; e++)
			printf("%s{\"n_class\": %.0f, \"leaf\": %u, \"group\": %u}", e ? ", " : "", tcache[e].n, tcache[e].leaf,
			       tcache[e].group);
		printf("]");
	}
	pot_batch_destroy(b);
	/* one at a time, plain FP64 form, for the first K jobs */
	if (plain_sample > 0) {
		const int K = plain_sample < n_jobs ? plain_sample : n_jobs;
		double t_sum = 0.0, ps_p = 0.0;
		int conv_p = 0;
		double* q_fast = calloc((size_t)K, sizeof(double));
		double* q_plain = calloc((size_t)K, sizeof(double));
		for (int i = 0; i < K; i++) {
			q_fast[i] = q_plain[i] = NAN;
			Job* j = &jobs[i];
			pot_gpu_opts o;
			memset(&o, 0, sizeof(o));
			o.form = POT_FORM_PLAIN;
			o.device = device;
			o.seed = j->seed;
			o.flags = chi_cap ? POT_OPT_CHI_CAP : 0u;
			pot_gpu_ctx* c = NULL;
			const double t0 = now_s();
			if (pot_gpu_create(&j->cfg, &o, &c) != POT_OK || pot_gpu_init_particles(c) != POT_OK) {
				if (c) pot_gpu_destroy(c);
				continue;
			}
			Job jj = *j;
			jj.qs = NULL;
			jj.n_qs = jj.cap_qs = 0;
			push_q(&jj, 0);
			uint64_t st = 0;
			bool cv = false;
			while (st < max_steps) {
				pot_step_stats s;
				if (pot_gpu_step(c, epoch, 0, &s) != POT_OK) break;
				st = s.t_steps;
				push_q(&jj, s.q_sum);
				if ((cv = converged(&jj, epoch))) break;
			}
			const double dt = now_s() - t0;
			pot_gpu_destroy(c);
			q_fast[i] = final_mean(j, epoch);
			q_plain[i] = final_mean(&jj, epoch);
			free(jj.qs);
			t_sum += dt;
			ps_p += (double)st * (double)(j->cfg.N - 1);
			conv_p += cv;
		}
		printf(", \"plain_one_at_a_time\": {\"jobs\": %d, \"converged\": %d, \"wall_s\": %.3f, "
		       "\"mean_s_per_job\": %.4f, \"particle_steps_per_s\": %.6e, \"note\": \"the first %d jobs, each alone in "
		       "the plain FP64 form from creation to convergence or --max-steps\"}",
		       K, conv_p, t_sum, K ? t_sum / K : 0.0, t_sum > 0 ? ps_p / t_sum : 0.0, K);
		/* the same jobs' charge in both forms: the mean over each run's last
		   500 steps (fast in the batch, plain alone) */
		printf(", \"final_charge_fast_vs_plain\": [");
		for (int i = 0; i < K; i++) {
			char f1[32], f2[32];
			printf("%s{\"job\": %d, \"N\": %lu, \"fast\": %s, \"plain\": %s}", i ? ", " : "", i,
			       (unsigned long)jobs[i].cfg.N, jnum(f1, q_fast[i]), jnum(f2, q_plain[i]));
		}
		printf("]");
		free(q_fast);
		free(q_plain);
	}
	printf("}\n");
	for (int i = 0; i < n_jobs; i++) free(jobs[i].qs);
	free(jobs);
	free(rows);
	free(slot_job);
	free(lat);
	free(lat_c);
	return 0;
}
