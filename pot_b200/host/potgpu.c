/*
 * potgpu -- pot's command line and output files, stepping on one B200.
 *
 * The host program of the reference (pot.c main() and run(), pot.c:4998-5311
 * and 4066-4555; pot-spheroid.c the same) with its MPI ranks replaced by one
 * GPU through the C ABI of include/pot_gpu.h.  Kept from the reference:
 *   - the flags of set_run_params_from_args (pot.c:4557-4850): -a -d -E -e -f
 *     -g -I -i -l -m -N -R -r -s -t -w -x, and -A of pot-spheroid.c, with the
 *     same defaults (pot.c:199-217, pot-spheroid.c:205-228) and messages;
 *   - the output files under ./output/: pot-run-init-info.txt and
 *     pot-run-descrip.txt at start (pot.c:3512-3812), pot-macroscopic.dat on
 *     the reference's record steps (pot.c:4364-4373, 3261-3508),
 *     pot-phi.dat every 20,000 steps (pot.c:3001-3042, 4397-4403), and the
 *     format C state file of -f every 50,000 steps and at the end
 *     (pot.c:3816-3900), read back by -g / -R (pot.c:3903-4019, 4948-4961);
 *   - the stopping rules: -i steps, -w minutes of wall time.
 * The reference selects its physics with compile-time switches; here they
 * are options (defaults = the configuration its benchmarks use):
 *   --oap X (OAP, pot.c:97), --bx/--by/--bz T (EXTERNAL_B_*, pot.c:55-57),
 *   --no-sceptic (SCEPTIC_REINJECTION, pot.c:181), --disable-grain
 *   (DISABLE_GRAIN, pot.c:30), --prolate / --oblate (pot-spheroid.c's
 *   PROLATE / OBLATE programs, with that program's defaults), --dipoles
 *   (DIPOLES, pot.c:99-104), --bounce C (OUT_BOUNCE C,
 *   pot.c:113-119), --integrator boris|verlet|euler-richardson (BORIS,
 *   EULER_RICHARDSON, pot.c:121-133), --pois-ions (POIS_POS_COLLECTION,
 *   pot.c:165-173; the macroscopic summary refreshes the cached ion
 *   temperature as pot.c:3444-3448 does), and for the
 *   GPU: --form fast|plain, --leaf N, --group 32|64, --seed S, --axis x,y,z
 *   (spheroid axis; x in the reference), --output-dir DIR.
 * Random numbers: the device draws from Philox4x32-10 streams keyed by a
 * 64-bit seed (--seed, else 8 bytes of /dev/urandom), not from the
 * reference's WELL512 state.  State files carry the seed in the WELL512
 * slot (see prng_block_from_seed); a reference-written state seeds Philox
 * from a hash of its WELL512 words.
 */
#define _POSIX_C_SOURCE 200809L
#include <errno.h>
#include <inttypes.h>
#include <math.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

#include "pot_gpu.h"

/* Physical constants of pot.c:278-282 and PI of prng.h. */
#define KB (1.38065e-23)
#define EPSILON0 (8.85419e-12)
#define QE (1.6021766e-19)
#define ME (9.109383e-31)
#define PI 3.14159265358979
#define MAX_PATH_LEN 400
#define CELLS_R 50
#define CELLS_AZI 4
#define CELLS_ZEN 10

enum { DUST = 0, ION = 1, ELECTRON = 2 };
static const int CHARGE[3] = { 0, 1, -1 };

typedef struct {
	unsigned long N;
	unsigned int r;
	long double dt;
	double mpp;
	unsigned long run_for;
	double soft, Te, Ti, x_drift, a, settle;
	double tim_lim;
	unsigned short track;
	char* sw_path;
	const char* sr_path;
	bool read_out;
	/* compile-time switches of the reference, as options */
	double oap;
	double B[3];
	bool sceptic, disable_grain;
	bool dipoles, pois_ions;
	double bounce;             /* 0: reinjection at the wall */
	unsigned int integrator;   /* POT_INT_* */
	int shape; /* 0 sphere, 1 prolate, 2 oblate */
	double A;
	double axis[3];
	/* GPU execution */
	unsigned int form, leaf, group;
	uint64_t seed;
	bool have_seed;
	bool host_macro;  /* summary sums from downloaded particles instead of on the device */
	bool phi_start;   /* pot-phi.dat rows for the starting state as well */
	char out_dir[4096];
} Run;

typedef struct {
	unsigned long N, r, run_for;
	double dt, mpp, soft, Te, Ti, x_drift, a, settle, tim_lim, A;
} Defaults;

/* pot.c:199-217 */
static const Defaults SPHERE_DEFAULTS = { 150001, 1000, 0, 1e-12, 4e-7, 2e-8, 220, 220, 0.0, 2.5e-6, 5e-7, 0.0, 0.0 };
/* pot-spheroid.c:203-228 */
static const Defaults PROLATE_DEFAULTS = { 150001, 654, 0, 1e-12, 4e-7, 4e-10, 11600, 11600, 0.0, 2.5e-6, 0.0, 0.0, 5.0 };
static const Defaults OBLATE_DEFAULTS = { 150001, 654, 0, 1e-12, 4e-7, 4e-10, 11600, 11600, 0.0, 2.5e-6, 0.0, 0.0, 0.5 };

static double mime_of(const Run* ru) { return ru->shape ? 1836.153 : 1836.15; }
static long double mass_of(const Run* ru, int sp)
{
	if (sp == DUST) return 1.67e-12;
	if (sp == ION) return (long double)(mime_of(ru) * ME);
	return ME;
}

static void e_puts(const char* s) { fprintf(stderr, "%s\n", s); }

static const Defaults* defaults_of(const Run* ru)
{
	return ru->shape == 1 ? &PROLATE_DEFAULTS : (ru->shape == 2 ? &OBLATE_DEFAULTS : &SPHERE_DEFAULTS);
}

static void set_defaults(Run* ru)
{
	const Defaults* d = defaults_of(ru);
	ru->N = d->N;
	ru->r = (unsigned int)d->r;
	ru->dt = d->dt;
	ru->mpp = d->mpp;
	ru->run_for = d->run_for;
	ru->soft = d->soft;
	ru->Te = d->Te;
	ru->Ti = d->Ti;
	ru->x_drift = d->x_drift;
	ru->a = d->a;
	ru->settle = d->settle;
	ru->tim_lim = d->tim_lim;
	ru->A = d->A;
	ru->track = 0;
}

static void usage(const char* prog)
{
	fprintf(stderr, "Usage: %s [OPTIONS]\n", prog);
	e_puts("  -a [SIZE]     grain radius in metres");
	e_puts("  -A [NUMBER]   aspect ratio of a spheroidal grain (with --prolate / --oblate)");
	e_puts("  -d [NUMBER]   time step in seconds");
	e_puts("  -E [NUMBER]   initial electron temperature in Kelvin");
	e_puts("  -e [NUMBER]   initial settling/equilibration time");
	e_puts("  -f [PATH]     write final simulation state to [PATH]");
	e_puts("  -g [PATH]     read initial simulation state from [PATH]");
	e_puts("  -I [NUMBER]   initial ion temperature in Kelvin");
	e_puts("  -i [INTEGER]  number of time steps to run for");
	e_puts("  -l            show runtime settings as command-line arguments");
	e_puts("  -m [SIZE]     pixel length in metres");
	e_puts("  -N [INTEGER]  number of particles to simulate");
	e_puts("  -R [PATH]     read out the simulation state at [PATH]");
	e_puts("  -r [INTEGER]  simulation radius in pixels");
	e_puts("  -s [NUMBER]   softening parameter in metres");
	e_puts("  -t [NUMBER]   number of particle trajectories to display (no display here)");
	e_puts("  -w [NUMBER]   limit on wall-time spent running in minutes");
	e_puts("  -x [NUMBER]   drift velocity in x-direction");
	e_puts("The reference's compile-time switches:");
	e_puts("  --oap X  --bx T --by T --bz T  --no-sceptic  --disable-grain  --prolate  --oblate");
	e_puts("  --dipoles  --bounce C  --integrator boris|verlet|euler-richardson  --pois-ions");
	e_puts("GPU execution:");
	e_puts("  --form fast|plain  --leaf N  --group 8|16|32|64  --seed S  --axis X,Y,Z  --output-dir DIR");
	e_puts("  --host-macro  compute the summary from downloaded particles (default: on the device)");
	e_puts("  --phi-start   also write pot-phi.dat rows for the starting (or resumed) state");
}

static int want(int* n, int argc) { return ++(*n) < argc; }

/* 0 OK, 1 usage, 2 message shown, 3 list settings (pot.c:4557-4850) */
static int parse_args(int argc, char** argv, Run* ru)
{
	bool just_output_args = false;
	/* the program variant first: it sets the defaults */
	for (int n = 1; n < argc; n++) {
		if (!strcmp(argv[n], "--prolate")) ru->shape = 1;
		if (!strcmp(argv[n], "--oblate")) ru->shape = 2;
	}
	set_defaults(ru);
	for (int n = 1; n < argc; n++) {
		const char* f = argv[n];
		if (f[0] != '-') return 1;
		if (f[1] == '-') {
			if (!strcmp(f, "--prolate") || !strcmp(f, "--oblate")) continue;
			if (!strcmp(f, "--no-sceptic")) { ru->sceptic = false; continue; }
			if (!strcmp(f, "--disable-grain")) { ru->disable_grain = true; continue; }
			if (!strcmp(f, "--host-macro")) { ru->host_macro = true; continue; }
			if (!strcmp(f, "--phi-start")) { ru->phi_start = true; continue; }
			if (!strcmp(f, "--dipoles")) { ru->dipoles = true; continue; }
			if (!strcmp(f, "--pois-ions")) { ru->pois_ions = true; continue; }
			if (!want(&n, argc)) return 1;
			const char* v = argv[n];
			if (!strcmp(f, "--oap")) ru->oap = strtod(v, NULL);
			else if (!strcmp(f, "--bx")) ru->B[0] = strtod(v, NULL);
			else if (!strcmp(f, "--by")) ru->B[1] = strtod(v, NULL);
			else if (!strcmp(f, "--bz")) ru->B[2] = strtod(v, NULL);
			else if (!strcmp(f, "--bounce")) {
				ru->bounce = strtod(v, NULL);
				if (!(ru->bounce >= 0.0)) {
					e_puts("Coefficient of restitution must be non-negative.");
					return 2;
				}
			} else if (!strcmp(f, "--integrator")) {
				if (!strcmp(v, "boris")) ru->integrator = POT_INT_BORIS;
				else if (!strcmp(v, "verlet")) ru->integrator = POT_INT_VERLET;
				else if (!strcmp(v, "euler-richardson")) ru->integrator = POT_INT_EULER_RICHARDSON;
				else return 1;
			}
			else if (!strcmp(f, "--form")) {
				if (!strcmp(v, "fast")) ru->form = POT_FORM_FAST;
				else if (!strcmp(v, "plain")) ru->form = POT_FORM_PLAIN;
				else return 1;
			} else if (!strcmp(f, "--leaf")) ru->leaf = (unsigned int)strtoul(v, NULL, 10);
			else if (!strcmp(f, "--group")) ru->group = (unsigned int)strtoul(v, NULL, 10);
			else if (!strcmp(f, "--seed")) {
				ru->seed = strtoull(v, NULL, 10);
				ru->have_seed = true;
			} else if (!strcmp(f, "--axis")) {
				if (sscanf(v, "%lf,%lf,%lf", &ru->axis[0], &ru->axis[1], &ru->axis[2]) != 3) return 1;
			} else if (!strcmp(f, "--output-dir")) {
				snprintf(ru->out_dir, sizeof(ru->out_dir), "%s/", v);
			} else return 1;
			continue;
		}
		switch (f[1]) {
		case 'a':
			if (!want(&n, argc)) return 1;
			ru->a = strtod(argv[n], NULL);
			if (ru->a <= 0.0) { e_puts("Grain radius must be positive."); return 2; }
			if (ru->a == HUGE_VAL) { e_puts("Given grain radius is too huge!"); return 2; }
			break;
		case 'A':
			if (!want(&n, argc)) return 1;
			ru->A = strtod(argv[n], NULL);
			if (ru->shape == 1 && ru->A <= 1.0) { e_puts("Prolate aspect ratio must be greater than 1."); return 2; }
			if (ru->shape == 2 && ru->A >= 1.0) { e_puts("Oblate aspect ratio must be less than 1."); return 2; }
			if (ru->shape == 0) { e_puts("Aspect ratio is not a parameter for a sphere."); return 2; }
			break;
		case 'd':
			if (!want(&n, argc)) return 1;
			ru->dt = strtold(argv[n], NULL);
			if (ru->dt <= 0.0) { e_puts("Time step must be positive."); return 2; }
			if (ru->dt == HUGE_VALL) { e_puts("Given time step is too huge!"); return 2; }
			break;
		case 'E':
			if (!want(&n, argc)) return 1;
			ru->Te = (double)strtold(argv[n], NULL);
			if (ru->Te < 0.0) { e_puts("Electron temperature must be non-negative."); return 2; }
			break;
		case 'e':
			if (!want(&n, argc)) return 1;
			ru->settle = (double)strtold(argv[n], NULL);
			if (ru->settle < 0.0) { e_puts("Settling time must be non-negative."); return 2; }
			break;
		case 'f':
			if (!want(&n, argc)) return 1;
			free(ru->sw_path);
			ru->sw_path = strdup(argv[n]);
			if (!ru->sw_path) { e_puts("Can't allocate memory for -f's argument."); return 2; }
			break;
		case 'g':
			if (!want(&n, argc)) return 1;
			ru->sr_path = argv[n];
			break;
		case 'I':
			if (!want(&n, argc)) return 1;
			ru->Ti = (double)strtold(argv[n], NULL);
			if (ru->Ti < 0.0) { e_puts("Ion temperature must be non-negative."); return 2; }
			break;
		case 'i':
			if (!want(&n, argc)) return 1;
			if ((ru->run_for = strtoul(argv[n], NULL, 10)) == 0) {
				e_puts("Number of time steps to run for must be a valid nonzero integer.");
				return 2;
			}
			break;
		case 'l':
			just_output_args = true;
			break;
		case 'm':
			if (!want(&n, argc)) return 1;
			ru->mpp = strtod(argv[n], NULL);
			if (ru->mpp <= 0.0) { e_puts("Pixel size must be positive."); return 2; }
			break;
		case 'N':
			if (!want(&n, argc)) return 1;
			if ((ru->N = strtoul(argv[n], NULL, 10)) == 0) {
				e_puts("Number of particles must be a valid nonzero integer.");
				return 2;
			}
			break;
		case 'R':
			if (!want(&n, argc)) return 1;
			ru->read_out = true;
			ru->sr_path = argv[n];
			break;
		case 'r':
			if (!want(&n, argc)) return 1;
			if ((ru->r = (unsigned int)strtoul(argv[n], NULL, 10)) == 0) {
				e_puts("Simulation radius in pixels must be a valid nonzero integer.");
				return 2;
			}
			break;
		case 's':
			if (!want(&n, argc)) return 1;
			ru->soft = strtod(argv[n], NULL);
			if (ru->soft < 0.0) { e_puts("Softening parameter must be non-negative."); return 2; }
			break;
		case 't':
			if (!want(&n, argc)) return 1;
			ru->track = (unsigned short)strtoul(argv[n], NULL, 10);
			break;
		case 'w':
			if (!want(&n, argc)) return 1;
			ru->tim_lim = strtod(argv[n], NULL);
			if (ru->tim_lim < 0.0) { e_puts("Wall-time limit must be non-negative."); return 2; }
			break;
		case 'x':
			if (!want(&n, argc)) return 1;
			ru->x_drift = strtod(argv[n], NULL);
			break;
		default:
			return 1;
		}
	}
	return just_output_args ? 3 : 0;
}

/* output_args_for_run, pot.c:4879-4917 */
static void output_args_for_run(const char* prog, const Run* ru)
{
	printf("Settings: %s -N %lu -r %u", prog, ru->N, ru->r);
	printf(" -d %Lg -m %g -s %g -E %g -I %g -x %g -a %g -e %g", ru->dt, ru->mpp, ru->soft, ru->Te, ru->Ti,
	       ru->x_drift, ru->a, ru->settle);
	if (ru->shape) printf(" -A %g", ru->A);
	if (ru->run_for) printf(" -i %lu", ru->run_for);
	if (ru->tim_lim > 0.0) printf(" -w %g", ru->tim_lim);
	if (ru->sw_path) printf(" -f %s", ru->sw_path);
	if (ru->sr_path) printf(ru->read_out ? " -R %s" : " -g %s", ru->sr_path);
	printf(" --oap %g", ru->oap);
	if (ru->B[0] != 0.0 || ru->B[1] != 0.0 || ru->B[2] != 0.0) printf(" --bx %g --by %g --bz %g", ru->B[0], ru->B[1], ru->B[2]);
	if (!ru->sceptic) printf(" --no-sceptic");
	if (ru->disable_grain) printf(" --disable-grain");
	if (ru->dipoles) printf(" --dipoles");
	if (ru->bounce > 0.0) printf(" --bounce %g", ru->bounce);
	if (ru->integrator == POT_INT_VERLET) printf(" --integrator verlet");
	if (ru->integrator == POT_INT_EULER_RICHARDSON) printf(" --integrator euler-richardson");
	if (ru->pois_ions) printf(" --pois-ions");
	if (ru->shape == 1) printf(" --prolate");
	if (ru->shape == 2) printf(" --oblate");
	printf(" --form %s", ru->form == POT_FORM_PLAIN ? "plain" : "fast");
	putchar('\n');
}

static FILE* open_out(const Run* ru, const char* name, const char* mode)
{
	char path[4200];
	snprintf(path, sizeof(path), "%s%s", ru->out_dir, name);
	return fopen(path, mode);
}

/* ---- run descriptions (pot.c:3512-3812) --------------------------------- */

static long double total_number_density(const Run* ru)
{
	return (ru->N - 1) / ((4.0 / 3.0) * PI * powl(ru->r * ru->mpp, 3.0));
}

static double early_oml_charge_time(const Run* ru, double n_total)
{
	const double mi = (double)mass_of(ru, ION), me = (double)mass_of(ru, ELECTRON);
	const double nu = sqrt(mi * ru->Te / (me * ru->Ti));
	double tim = EPSILON0 * sqrt(2.0 * PI * mi * KB * ru->Te * ru->Te / ru->Ti);
	tim /= (QE * QE * ru->a * n_total / 2.0);
	tim *= log((1.0 - nu) / (pow(nu, 1.0 - exp(-1.0)) - nu));
	return tim;
}

static void write_run_info(const Run* ru)
{
	FILE* fp = open_out(ru, "pot-run-init-info.txt", "ab");
	char date_time[50];
	time_t t = time(NULL);
	struct tm* tm = localtime(&t);
	if (!fp) {
		fprintf(stderr, "Can't open %spot-run-init-info.txt to write information about this run.\n", ru->out_dir);
		return;
	}
	if (!tm || !strftime(date_time, sizeof(date_time), "%Y-%m-%d %H:%M:%S", tm)) snprintf(date_time, sizeof(date_time), "?");
	fprintf(fp, "%s\t%lu\t%Lg\t%g\t%g\t%g\t%g\t%g\t%s\t%s\t%u\t%g\t%u\t%g\n", date_time, ru->N, ru->dt, ru->soft,
	        ru->mpp, ru->Ti, ru->Te, ru->x_drift, __DATE__, __TIME__, ru->r, ru->a, 1u, ru->oap);
	fclose(fp);
}

static void write_run_description(const Run* ru)
{
	const Defaults* d = defaults_of(ru);
	FILE* fp = open_out(ru, "pot-run-descrip.txt", "ab");
	if (!fp) {
		fprintf(stderr, "Can't open %spot-run-descrip.txt to write this run's initial description.\n", ru->out_dir);
		return;
	}
	fprintf(fp,
	        "%c total particle count:          %lu\n"
	        "%c time step (s):                 %Lg\n"
	        "%c nominal elec. temperature (K): %g\n"
	        "%c nominal ion temperature (K):   %g\n"
	        "%c softening parameter (m):       %g\n"
	        "%c drift velocity (m*s^-1):       %g\n"
	        "%c pixel size (m):                %g\n"
	        "%c simulation radius (px.):       %u\n"
	        "%c tracked particles:             %hu\n"
	        "%c number of time steps:          %lu\n"
	        "%c grain radius (m):              %g\n"
	        "%c settling time (s):             %g\n",
	        (ru->N != d->N) ? '*' : ' ', ru->N, (ru->dt != d->dt) ? '*' : ' ', ru->dt,
	        (ru->Te != d->Te) ? '*' : ' ', ru->Te, (ru->Ti != d->Ti) ? '*' : ' ', ru->Ti,
	        (ru->soft != d->soft) ? '*' : ' ', ru->soft, (ru->x_drift != d->x_drift) ? '*' : ' ', ru->x_drift,
	        (ru->mpp != d->mpp) ? '*' : ' ', ru->mpp, (ru->r != d->r) ? '*' : ' ', ru->r, ' ', (unsigned short)0,
	        (ru->run_for != d->run_for) ? '*' : ' ', ru->run_for, (ru->a != d->a) ? '*' : ' ', ru->a,
	        (ru->settle != d->settle) ? '*' : ' ', ru->settle);
	if (ru->shape) fprintf(fp, "%c aspect ratio:                  %g\n", (ru->A != d->A) ? '*' : ' ', ru->A);
	fputc('\n', fp);

	const long double n = total_number_density(ru);
	const long double size = 2.0 * ru->r * ru->mpp;
	const long double mi = mass_of(ru, ION), me = mass_of(ru, ELECTRON);
	const long double debye_len = sqrtl(EPSILON0 * KB * ru->Te / ((n / 2.0) * QE * QE));
	const double debye_number = (4.0 / 3.0) * PI * powl(debye_len, 3.0) * n / 2.0;
	const long double wsr = powl(4.0 * PI * n / 3.0, -1.0 / 3.0);
	double ccp = QE * CHARGE[ION] * QE * CHARGE[ION];
	ccp /= (4.0 * PI * EPSILON0 * wsr * KB * ru->Te);
	const double coulomb_log = log(9.0 * debye_number);
	const long double e_colll = 16.0 * PI * (n / 2.0) * powl(debye_len, 4.0) / coulomb_log;
	const long double edct = ru->a / sqrtl(3.0 * KB * ru->Te / me);
	const long double eop = 2.0 * PI * sqrtl(ME * EPSILON0 / (n * QE * QE / 2.0));
	const double charge_osc_rat = early_oml_charge_time(ru, (double)n) / eop;
	long double htcd = QE * QE / (12 * PI * EPSILON0 * KB);
	htcd /= (ru->Te > ru->Ti) ? ru->Te : ru->Ti;
	fprintf(fp,
	        "  particle density (m^-3):    %Lg\n"
	        "  Debye length (m):           %Lg\n"
	        "  grain radius/DL:            %Lg\n"
	        "  elec. oscil. period (s):    %Lg\n"
	        "  early OML chg. time (s):    %g\n"
	        "  Wigner-Seitz radius (m):    %Lg\n"
	        "  normalized drift speed:     %Lg\n"
	        "  ion traversal time (s):     %Lg\n"
	        "  Coulomb logarithm:          %g\n"
	        "  electron coll. len. (m):    %Lg\n"
	        "%c electron Knudsen number:    %Lg\n"
	        "%c Debye number:               %g\n"
	        "%c Coulomb coupling param.:    %g\n"
	        "%c softening parameter/WSR:    %Lg\n"
	        "%c t. step/elec. cross time:   %Lg\n"
	        "%c DL/characteristic size:     %Lg\n"
	        "%c OML time/elec. osc. period: %g\n"
	        "%c soft. par./head coll. dist: %Lg\n"
	        "%c soft. par./grain radius:    %g\n\n",
	        n, debye_len, ru->a / debye_len, eop, early_oml_charge_time(ru, (double)n), wsr,
	        ru->x_drift / sqrtl(KB * ru->Ti / mi), size / sqrtl(3.0 * KB * ru->Ti / mi), coulomb_log, e_colll,
	        ((e_colll / size) > 0.5) ? '!' : ' ', e_colll / size, (debye_number < 2.0) ? '!' : ' ', debye_number,
	        (ccp > 1.0) ? '!' : ' ', ccp, ((ru->soft / wsr) > 1.0) ? '!' : ' ', ru->soft / wsr,
	        ((ru->dt / edct) > 0.5) ? '!' : ' ', ru->dt / edct, ((debye_len / size) > 0.1) ? '!' : ' ',
	        debye_len / size, (charge_osc_rat < 100.0) ? '!' : ' ', charge_osc_rat,
	        ((ru->soft / htcd) > 0.5) ? '!' : ' ', ru->soft / htcd, ((ru->soft / ru->a) > 0.1) ? '!' : ' ',
	        ru->soft / ru->a);
	fprintf(fp,
	        "opening angle parameter: %g\n"
	        "ion/electron mass ratio: %Lg\n"
	        "external B field (T):    (%g, %g, %g)\n"
	        "spatial bin counts:      (%i, %i, %i)\n"
	        "max. tree walk length:   %i\n"
	        "grain mass (kg):         %Lg\n\n",
	        ru->oap, mi / me, ru->B[0], ru->B[1], ru->B[2], CELLS_R, CELLS_AZI, CELLS_ZEN, MAX_PATH_LEN,
	        mass_of(ru, DUST));
	fputs(ru->disable_grain ? "grain:                disabled\n" : "grain:                enabled\n", fp);
	fputs("OpenGL interface:     no\n", fp);
	fputs("trajectory length:    N/A\n", fp);
	if (ru->bounce > 0.0) {
		fprintf(fp, "containment:          bouncing (c.o.e. %g)\n", ru->bounce);
	} else {
		fputs(ru->sceptic ? "containment:          reinjection (SCEPTIC-style)\n"
		                  : "containment:          reinjection (old-style)\n", fp);
	}
	fputs("FP exceptions:        no\n", fp);
	fputs(ru->dipoles ? "multipole expansion:  dipole\n" : "multipole expansion:  monopole\n", fp);
	fputs("simulation shape:     spherical\n", fp);
	fputs(ru->integrator == POT_INT_EULER_RICHARDSON ? "numerical integrator: Euler-Richardson\n"
	      : ru->integrator == POT_INT_VERLET ? "numerical integrator: velocity Verlet\n"
	                                         : "numerical integrator: Boris\n", fp);
	fputs(ru->pois_ions ? "pos. Pois. collec'n:  yes\n" : "pos. Pois. collec'n:  no\n", fp);
	fputs("Langmuir test wave:   no\n", fp);
	fputs("P-P interactions:     yes\n", fp);
	fputs(ru->shape == 1 ? "Grain shape:          prolate spheroid\n\n"
	      : ru->shape == 2 ? "Grain shape:          oblate spheroid\n\n" : "Grain shape:          sphere\n\n", fp);
	fprintf(fp, "output file dir.:     %s\ncompiled on:          %s %s\n",
	        ru->out_dir[0] ? ru->out_dir : "./output/", __DATE__, __TIME__);
	fprintf(fp, "stepped on:           one GPU (%s form)\n",
	        ru->form == POT_FORM_PLAIN ? "plain FP64" : "fast FP32-walk");
	fclose(fp);
}

/* ---- macroscopic summary (pot.c:3249-3508) ------------------------------ */

#define isnt_weird(x) (isnormal(x) || (fpclassify(x) == FP_ZERO))
#define pythag(x, y, z) sqrt((x) * (x) + (y) * (y) + (z) * (z))

static void central_moments(long double* cms, unsigned int N)
{
	cms[1] /= N;
	cms[2] /= N * powl(cms[1], 1.5);
	cms[3] /= N * cms[1] * cms[1];
	cms[3] -= 3.0;
}

/* The sums of both passes from downloaded particles, accumulated in long
   double as pot.c:3354-3461 does (the --host-macro path). */
static void host_macro_sums(const Run* ru, const pot_particle* P, pot_macro_sums* m)
{
	long double a1[20] = { 0 }, a2[18] = { 0 };
	const double cent = ru->r * ru->mpp;
	const long double me = mass_of(ru, ELECTRON), mi = mass_of(ru, ION);
	for (unsigned long k = 1; k < ru->N; k++) {
		const pot_particle* p = &P[k];
		const long double v = pythag(p->vx, p->vy, p->vz);
		const int e = p->species == ELECTRON;
		const long double amx = ((p->y - cent) * p->vz) - ((p->z - cent) * p->vy);
		const long double amy = -(((p->x - cent) * p->vz) - ((p->z - cent) * p->vx));
		const long double amz = ((p->x - cent) * p->vy) - ((p->y - cent) * p->vx);
		if (e) {
			a1[0] += 1;
			a1[2] += 0.5 * me * v * v;
			a1[3] += v;
			a1[5] += p->vx; a1[6] += p->vy; a1[7] += p->vz;
			a1[11] += amx; a1[12] += amy; a1[13] += amz;
		} else {
			a1[1] += 1;
			a1[4] += v;
			a1[8] += p->vx; a1[9] += p->vy; a1[10] += p->vz;
			a1[14] += amx; a1[15] += amy; a1[16] += amz;
		}
	}
	const long double Km = a1[2] / a1[0], sme = a1[3] / a1[0], smi = a1[4] / a1[1];
	const long double ve[3] = { a1[5] / a1[0], a1[6] / a1[0], a1[7] / a1[0] };
	const long double vi[3] = { a1[8] / a1[1], a1[9] / a1[1], a1[10] / a1[1] };
	for (unsigned long k = 1; k < ru->N; k++) {
		const pot_particle* p = &P[k];
		const long double v = pythag(p->vx, p->vy, p->vz);
		if (p->species == ELECTRON) {
			const long double K = 0.5 * me * v * v, Ks = K - Km, vs = v - sme;
			a2[0] += K * K;
			a2[1] += p->x;
			a2[2] += p->x * p->x;
			a2[3] += Ks * Ks; a2[4] += Ks * Ks * Ks; a2[5] += Ks * Ks * Ks * Ks;
			a2[6] += vs * vs; a2[7] += vs * vs * vs; a2[8] += vs * vs * vs * vs;
			a2[9] += (p->vx - ve[0]) * (p->vx - ve[0]) + (p->vy - ve[1]) * (p->vy - ve[1]) +
			         (p->vz - ve[2]) * (p->vz - ve[2]);
		} else {
			const long double K = 0.5 * mi * v * v, vs = v - smi;
			a2[10] += K;
			a2[11] += K * K;
			a2[12] += vs * vs; a2[13] += vs * vs * vs; a2[14] += vs * vs * vs * vs;
			a2[15] += (p->vx - vi[0]) * (p->vx - vi[0]) + (p->vy - vi[1]) * (p->vy - vi[1]) +
			          (p->vz - vi[2]) * (p->vz - vi[2]);
		}
	}
	double* out = (double*)m;
	for (int k = 0; k < 20; k++) out[k] = (double)a1[k];
	for (int k = 0; k < 18; k++) out[20 + k] = (double)a2[k];
}

/* One row of pot-macroscopic.dat from the sums (pot.c:3398-3508). */
static void write_macro(FILE* fp, const Run* ru, const pot_macro_sums* m, const pot_grain_state* g,
                        const long double epe[3], unsigned long step)
{
	if (ru->N < 6 || !fp) return;
	const long double me = mass_of(ru, ELECTRON), mi = mass_of(ru, ION);
	const unsigned int N_e = (unsigned int)m->n_e, N_i = (unsigned int)m->n_i;
	const long double volume = (4.0 / 3.0) * PI * powl(ru->r * ru->mpp, 3.0);
	long double K_e[4] = { m->K_e, m->K_e_c[0], m->K_e_c[1], m->K_e_c[2] };
	long double s_e[4] = { m->s_e, m->s_e_c[0], m->s_e_c[1], m->s_e_c[2] };
	long double s_i[4] = { m->s_i, m->s_i_c[0], m->s_i_c[1], m->s_i_c[2] };
	long double lm_e[3], lm_i[3], am_e[3], am_i[3];
	K_e[0] /= N_e;
	s_e[0] /= N_e;
	s_i[0] /= N_i;
	for (int k = 0; k < 3; k++) {
		lm_e[k] = me * ((long double)m->v_e[k] / N_e);
		lm_i[k] = mi * ((long double)m->v_i[k] / N_i);
		am_e[k] = (long double)m->am_e[k] * me;
		am_i[k] = (long double)m->am_i[k] * mi;
	}
	central_moments(K_e, N_e);
	central_moments(s_e, N_e);
	central_moments(s_i, N_i);
	const double temp_e = m->T_e * (me / (3.0 * KB)) / N_e;
	const double temp_i = m->T_i * (mi / (3.0 * KB)) / N_i;
	const long double sum_x_elec = m->sum_x_e, sum_sq_x_elec = m->sumsq_x_e;
	const long double debye = sqrtl(EPSILON0 * KB * temp_e / ((N_e / volume) * QE * QE));
	fprintf(fp, "%.7Lg %Lg ", step * ru->dt, K_e[0]);
	if (isnt_weird(epe[ELECTRON])) fprintf(fp, "%Lg ", epe[ELECTRON] / N_e); else fputs("NA ", fp);
	fprintf(fp, "%Lg ", (long double)m->sum_K_i / N_i);
	if (isnt_weird(epe[ION])) fprintf(fp, "%Lg ", epe[ION] / N_i); else fputs("NA ", fp);
	fprintf(fp, "%Lg ", 0.5 * (long double)g->m * hypot(g->vx, hypot(g->vy, g->vz)));
	if (isnt_weird(epe[DUST])) fprintf(fp, "%Lg ", epe[DUST]); else fputs("NA ", fp);
	fprintf(fp,
	        "%.7Lg %.7Lg %i %Lg %Lg"
	        " %Lg %Lg %Lg %Lg %Lg %Lg %Lg %Lg %g %g %Lg %Lg %Lg"
	        " %Lg %Lg %Lg %Lg %Lg %Lg %Lg %Lg %Lg %u\n",
	        sum_x_elec / N_e, sqrtl(sum_sq_x_elec / N_e - (sum_x_elec / N_e) * sum_x_elec / N_e), (int)g->q, debye,
	        (4.0 * PI / 3.0) * debye * debye * debye * N_e / volume, s_e[0], s_e[1], s_e[2], s_e[3], s_i[0], s_i[1],
	        s_i[2], s_i[3], temp_e, temp_i, lm_e[0], lm_e[1], lm_e[2], lm_i[0], lm_i[1], lm_i[2], am_e[0], am_e[1],
	        am_e[2], am_i[0], am_i[1], am_i[2], (unsigned int)g->tot_absor_e);
	if (fflush(fp)) e_puts("Can't force write of macroscopic summary data to disk.");
}

/* a record step's row: on-device sums (default) or from downloaded particles */
static int record_row(FILE* fp, const Run* ru, pot_gpu_ctx* ctx, pot_particle* P, pot_grain_state* g,
                      const long double epe[3], unsigned long step)
{
	pot_macro_sums m;
	int rc;
	if (ru->host_macro) {
		if ((rc = pot_gpu_download(ctx, P, g)) != POT_OK) return rc;
		host_macro_sums(ru, P, &m);
		if (ru->pois_ions && m.n_i > 0.0) {
			/* the measured ion temperature becomes the cached one, pot.c:3442-3448
			   (pot_gpu_macro does this on the device) */
			double Ti = m.T_i;
			Ti *= (mass_of(ru, ION) / (3.0 * KB)) / m.n_i;
			if ((rc = pot_gpu_set_ion_temp(ctx, Ti)) != POT_OK) return rc;
		}
	} else {
		if ((rc = pot_gpu_macro(ctx, &m)) != POT_OK) return rc;
		if ((rc = pot_gpu_grain(ctx, g)) != POT_OK) return rc;
	}
	write_macro(fp, ru, &m, g, epe, step);
	return POT_OK;
}

/* ---- pot-phi.dat (pot.c:3001-3042) -------------------------------------- */

static int write_phi(const Run* ru, pot_gpu_ctx* ctx, const pot_grain_state* g, unsigned long step)
{
	enum { NP = CELLS_R * CELLS_AZI * (CELLS_ZEN + 1) };
	static double xyz[3 * NP], phi[NP], rr[NP], az[NP], ze[NP];
	const double r_step = ru->r * ru->mpp / CELLS_R;
	int k = 0;
	for (unsigned int ri = 1; ri <= CELLS_R; ri++) {
		for (unsigned int ai = 0; ai < CELLS_AZI; ai++) {
			for (unsigned int zi = 0; zi <= CELLS_ZEN; zi++) {
				const double r = r_step * ri, azi = 2.0 * PI * ai / CELLS_AZI, zen = PI * zi / CELLS_ZEN;
				rr[k] = r;
				az[k] = azi;
				ze[k] = zen;
				xyz[3 * k] = g->x + (r * cos(azi) * sin(zen));
				xyz[3 * k + 1] = g->y + (r * sin(azi) * sin(zen));
				xyz[3 * k + 2] = g->z + (r * cos(zen));
				k++;
			}
		}
	}
	const int rc = pot_gpu_phi_at(ctx, NP, xyz, phi);
	if (rc != POT_OK) return rc;
	FILE* fp = open_out(ru, "pot-phi.dat", "ab");
	if (!fp) {
		fprintf(stderr, "Can't open %spot-phi.dat to write electric potential data.\n", ru->out_dir);
		return POT_OK;
	}
	for (int j = 0; j < NP; j++) fprintf(fp, "%Lg %g %g %g %g\n", step * ru->dt, rr[j], az[j], ze[j], phi[j]);
	fclose(fp);
	return POT_OK;
}

/* ---- state files (pot.c:3816-4019) -------------------------------------- */

/* WELL512 record of prng.h:17-24 (84 bytes) */
typedef struct {
	uint32_t a, b, c, d, index;
	uint32_t state[16];
} PrngBlock;

static uint64_t splitmix64(uint64_t* x)
{
	uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
	z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
	z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
	return z ^ (z >> 31);
}

#define SEED_MARK 0x506F7447u /* "GtoP" */

/* The Philox seed in the WELL512 slot: words 0-1 the seed, word 2 a mark,
   words 3-15 a splitmix64 stream of the seed (a valid WELL512 state should
   the reference read it). */
static void prng_block_from_seed(uint64_t seed, PrngBlock* b)
{
	memset(b, 0, sizeof(*b));
	b->state[0] = (uint32_t)seed;
	b->state[1] = (uint32_t)(seed >> 32);
	b->state[2] = SEED_MARK;
	uint64_t x = seed;
	for (int k = 3; k < 16; k++) b->state[k] = (uint32_t)splitmix64(&x);
}

static uint64_t seed_from_prng_block(const PrngBlock* b)
{
	PrngBlock mine;
	const uint64_t s = (uint64_t)b->state[0] | ((uint64_t)b->state[1] << 32);
	prng_block_from_seed(s, &mine);
	if (!memcmp(mine.state, b->state, sizeof(mine.state))) return s;
	uint64_t h = 0x243F6A8885A308D3ull;
	for (int k = 0; k < 16; k++) {
		h ^= b->state[k];
		h = splitmix64(&h);
	}
	return h;
}

static int write_state(const Run* ru, const char* path, const pot_particle* P, const pot_grain_state* g,
                       const long double epe[3], uint64_t seed)
{
	FILE* fp = fopen(path, "wb");
	PrngBlock b;
	if (!fp) {
		fprintf(stderr, "Failed to open simulation state file %s for writing.\n", path);
		return -1;
	}
	fprintf(fp, "C %u %i %Lg %lu %Lg %Lg %Lg %u %g\n", 1u, (int)g->q, (long double)g->m,
	        (unsigned long)g->t_steps, epe[0], epe[1], epe[2], (unsigned int)g->tot_absor_e,
	        ru->sceptic ? g->chi_b : 9999.99);
	prng_block_from_seed(seed, &b);
	if (fwrite(&b, sizeof(b), 1, fp) != 1) fprintf(stderr, "Failed to write proc. 0's PRNG state to %s.\n", path);
	if (fwrite(P, sizeof(pot_particle), ru->N, fp) != ru->N) fprintf(stderr, "Failed to write particle states to %s.\n", path);
	if (fclose(fp)) fprintf(stderr, "Failed to close simulation state output file %s.\n", path);
	return 0;
}

/* formats A, B and C; any worker count (one GPU replaces them all; the
   first rank's PRNG record seeds the run) */
static int read_state(const Run* ru, const char* path, pot_particle* P, pot_grain_state* g, long double epe[3],
                      uint64_t* seed)
{
	FILE* fp = fopen(path, "rb");
	unsigned int workers = 0, tae = 0;
	int q = 0;
	unsigned long t = 0;
	long double m = 1.67e-12;
	double chi_b = 0.0;
	if (!fp) {
		fprintf(stderr, "0: failed to open simulation state file %s to read.\n", path);
		return -1;
	}
	const int c = getc(fp);
	int ok;
	if (c == 'C') {
		ok = fscanf(fp, " %u %i %Lg %lu %Lg %Lg %Lg %u %lg\n", &workers, &q, &m, &t, &epe[0], &epe[1], &epe[2], &tae,
		            &chi_b) == 9;
	} else if (c == 'B') {
		ok = fscanf(fp, " %u %i %lu %Lg %Lg %Lg %u\n", &workers, &q, &t, &epe[0], &epe[1], &epe[2], &tae) == 7;
	} else if (c >= '0' && c <= '9') {
		rewind(fp);
		ok = fscanf(fp, "%u %i %lu %Lg %Lg %Lg\n", &workers, &q, &t, &epe[0], &epe[1], &epe[2]) == 6;
	} else {
		fprintf(stderr, "0: alleged state file %s isn't.\n", path);
		fclose(fp);
		return -1;
	}
	if (!ok || workers == 0) {
		fprintf(stderr, "0: failed to read the assorted data values from %s.\n", path);
		fclose(fp);
		return -1;
	}
	for (unsigned int w = 0; w < workers; w++) {
		PrngBlock b;
		if (fread(&b, sizeof(b), 1, fp) != 1) {
			fprintf(stderr, "0: failed to read proc. %u's PRNG state from %s.\n", w, path);
			fclose(fp);
			return -1;
		}
		if (w == 0) *seed = seed_from_prng_block(&b);
	}
	if (fread(P, sizeof(pot_particle), ru->N, fp) != ru->N) {
		fprintf(stderr, "0: failed to read particle states from %s.\n", path);
		fclose(fp);
		return -1;
	}
	fclose(fp);
	memset(g, 0, sizeof(*g));
	g->q = q;
	g->m = (double)m;
	g->x = P[0].x;
	g->y = P[0].y;
	g->z = P[0].z;
	g->vx = P[0].vx;
	g->vy = P[0].vy;
	g->vz = P[0].vz;
	g->tot_absor_e = tae;
	g->t_steps = t;
	g->chi_b = chi_b;
	return 0;
}

static void read_out_state(const Run* ru, const pot_particle* P)
{
	const char letters[] = "die";
	puts("NO S X Y Z VX VY VZ");
	for (unsigned long k = 0; k < ru->N; k++) {
		const pot_particle* p = &P[k];
		printf("%lu \"%c\" %g %g %g %g %g %g\n", k, letters[p->species], p->x, p->y, p->z, p->vx, p->vy, p->vz);
	}
}

/* ---- main (pot.c:4998-5311, run() 4066-4555) ---------------------------- */

static bool record_macro(const Run* ru, unsigned long t)
{
	bool rec = t <= 200;
	if ((t * ru->dt) > (2.0 * ru->settle)) rec |= !(t % 2000);
	else rec |= !(t % 200);
	return rec;
}

static int fail(pot_gpu_ctx* ctx, unsigned long t, int rc)
{
	fprintf(stderr, "0:%lu: %s\n", t, pot_gpu_strerror(rc));
	(void)ctx;
	return rc;
}

int main(int argc, char** argv)
{
	Run ru;
	memset(&ru, 0, sizeof(ru));
	ru.oap = 0.5;
	ru.sceptic = true;
	ru.form = POT_FORM_FAST;
	snprintf(ru.out_dir, sizeof(ru.out_dir), "./output/");
	if (argc < 2) e_puts("Run without arguments; attempting to use default settings.");
	switch (parse_args(argc, argv, &ru)) {
	case 1:
		usage(argv[0]);
		free(ru.sw_path);
		return EXIT_FAILURE;
	case 2:
		free(ru.sw_path);
		return EXIT_FAILURE;
	case 3:
		output_args_for_run(argv[0], &ru);
		free(ru.sw_path);
		return EXIT_SUCCESS;
	default:
		break;
	}
	if (ru.a >= (ru.r * ru.mpp)) {
		fprintf(stderr, "Grain radius (%g m) must be less than simulation region radius (%g m).\n", ru.a,
		        ru.r * ru.mpp);
		free(ru.sw_path);
		return EXIT_FAILURE;
	}
	pot_particle* P = malloc(sizeof(pot_particle) * ru.N);
	if (!P) {
		fprintf(stderr, "0: can't allocate %.1f MiB for %lu particles' data.\n",
		        sizeof(pot_particle) * ru.N / 1048576.0, ru.N);
		free(ru.sw_path);
		return EXIT_FAILURE;
	}
	pot_grain_state g;
	long double epe[3] = { 0.0L, 0.0L, 0.0L };
	memset(&g, 0, sizeof(g));
	uint64_t seed = ru.seed;
	if (ru.sr_path) {
		uint64_t file_seed = 0;
		if (read_state(&ru, ru.sr_path, P, &g, epe, &file_seed)) {
			free(P);
			free(ru.sw_path);
			return EXIT_FAILURE;
		}
		if (ru.read_out) {
			read_out_state(&ru, P);
			free(P);
			free(ru.sw_path);
			return EXIT_SUCCESS;
		}
		if (!ru.have_seed) seed = file_seed;
		if (ru.run_for && g.t_steps >= ru.run_for) {
			printf("0: simulation's already run for %lu steps, exiting.\n", ru.run_for);
			free(P);
			free(ru.sw_path);
			return EXIT_SUCCESS;
		}
	} else if (!ru.have_seed) {
		FILE* ur = fopen("/dev/urandom", "rb");
		if (!ur || fread(&seed, sizeof(seed), 1, ur) != 1) {
			fprintf(stderr, "0: can't read PRNG seed from /dev/urandom, PRNG may behave inadequately.\n");
			seed = 0;
		}
		if (ur) fclose(ur);
	}

	pot_run_cfg cfg;
	pot_gpu_opts opt;
	memset(&cfg, 0, sizeof(cfg));
	memset(&opt, 0, sizeof(opt));
	cfg.N = ru.N;
	cfg.r = ru.r;
	cfg.flags = (ru.sceptic ? POT_CFG_SCEPTIC : 0u) | (ru.disable_grain ? POT_CFG_DISABLE_GRAIN : 0u) |
	            (ru.dipoles ? POT_CFG_DIPOLES : 0u) | (ru.pois_ions ? POT_CFG_POIS_IONS : 0u);
	cfg.bounce = ru.bounce;
	cfg.integrator = ru.integrator;
	cfg.dt = (double)ru.dt;
	cfg.mpp = ru.mpp;
	cfg.soft = ru.soft;
	cfg.Te = ru.Te;
	cfg.Ti = ru.Ti;
	cfg.x_drift = ru.x_drift;
	cfg.a = ru.a;
	cfg.settle = ru.settle;
	cfg.theta = ru.oap;
	for (int k = 0; k < 3; k++) {
		cfg.B[k] = ru.B[k];
		cfg.axis[k] = ru.axis[k];
	}
	cfg.A = ru.shape ? ru.A : 0.0;
	opt.form = ru.form;
	opt.leaf_size = ru.leaf;
	opt.group_size = ru.group;
	opt.seed = seed;
	pot_gpu_ctx* ctx = NULL;
	int rc = pot_gpu_create(&cfg, &opt, &ctx);
	if (rc != POT_OK) {
		fprintf(stderr, "0: can't set up the GPU run: %s\n", pot_gpu_strerror(rc));
		free(P);
		free(ru.sw_path);
		return EXIT_FAILURE;
	}
	rc = ru.sr_path ? pot_gpu_upload(ctx, P, ru.N, &g) : pot_gpu_init_particles(ctx);
	if (rc != POT_OK) {
		fail(ctx, 0, rc);
		pot_gpu_destroy(ctx);
		free(P);
		free(ru.sw_path);
		return EXIT_FAILURE;
	}
	if (ru.phi_start) {
		/* the potential profile of the starting state (write_phi_data_to_file
		   as pot.c:4397-4403 calls it, at the resumed step) over its own tree */
		if ((rc = pot_gpu_build_tree(ctx, NULL)) != POT_OK || (rc = pot_gpu_download(ctx, P, &g)) != POT_OK ||
		    (rc = write_phi(&ru, ctx, &g, g.t_steps)) != POT_OK) {
			fail(ctx, g.t_steps, rc);
			pot_gpu_destroy(ctx);
			free(P);
			free(ru.sw_path);
			return EXIT_FAILURE;
		}
	}
	FILE* fp_macro = NULL;
	if (ru.N >= 6) {
		if (!(fp_macro = open_out(&ru, "pot-macroscopic.dat", "ab"))) {
			fprintf(stderr, "Can't open %spot-macroscopic.dat to write macroscopic data.\n", ru.out_dir);
		} else if (!ftell(fp_macro)) {
			fputs("TIME KE PE KI PI KG PG XE XESD DGQ DL DN "
			      "SE1 SE2 SE3 SE4 SI1 SI2 SI3 SI4 TE TI LMEX LMEY LMEZ "
			      "LMIX LMIY LMIZ AMEX AMEY AMEZ AMIX AMIY AMIZ TOTE\n", fp_macro);
		}
	}
	write_run_info(&ru);
	write_run_description(&ru);

	const time_t start = time(NULL);
	unsigned long t = g.t_steps;  /* steps completed */
	bool recorded_last = false;
	int status = EXIT_SUCCESS;
	pot_step_stats st;
	for (;;) {
		const unsigned long next = t + 1;
		if (ru.run_for && next > ru.run_for) break;
		if (ru.tim_lim > 0.0 && (time(NULL) - start) > (60 * ru.tim_lim)) break;
		/* state file every 50,000 steps, before the step (pot.c:4353-4356) */
		if (ru.sw_path && !(next % 50000)) {
			if ((rc = pot_gpu_download(ctx, P, &g)) != POT_OK) { status = fail(ctx, t, rc); break; }
			write_state(&ru, ru.sw_path, P, &g, epe, seed);
		}
		/* steps that record nothing run straight through, up to the next
		   event (at most 1,000 per call, so the wall-time limit is seen) */
		if (!record_macro(&ru, next) && (next % 20000)) {
			unsigned long run_to = next;
			while (true) {
				const unsigned long u = run_to + 1;
				if ((ru.run_for && u > ru.run_for) || record_macro(&ru, u) || !(u % 20000) ||
				    (ru.sw_path && !(u % 50000)) || u - next >= 1000)
					break;
				run_to = u;
			}
			if ((rc = pot_gpu_step(ctx, (uint32_t)(run_to - next + 1), 0, &st)) != POT_OK) {
				status = fail(ctx, t, rc);
				break;
			}
			t = run_to;
			recorded_last = false;
			continue;
		}
		const bool rec = record_macro(&ru, next);
		if ((rc = pot_gpu_step(ctx, 1, rec ? POT_STEP_EPE : 0u, &st)) != POT_OK) { status = fail(ctx, next, rc); break; }
		t = next;
		if (rec)
			for (int k = 0; k < 3; k++) epe[k] = st.epe[k];
		if (!(t % 20000)) {
			if ((rc = pot_gpu_download(ctx, P, &g)) != POT_OK) { status = fail(ctx, t, rc); break; }
			if ((rc = write_phi(&ru, ctx, &g, t)) != POT_OK) { status = fail(ctx, t, rc); break; }
		}
		if (rec && (rc = record_row(fp_macro, &ru, ctx, P, &g, epe, t)) != POT_OK) {
			status = fail(ctx, t, rc);
			break;
		}
		recorded_last = rec;
		if (ru.tim_lim > 0.0 && (time(NULL) - start) > (60 * ru.tim_lim)) break;
	}
	if (status == EXIT_SUCCESS) {
		if (ru.sw_path && pot_gpu_download(ctx, P, &g) == POT_OK) write_state(&ru, ru.sw_path, P, &g, epe, seed);
		if (!recorded_last) record_row(fp_macro, &ru, ctx, P, &g, epe, t);
	}
	if (fp_macro) fclose(fp_macro);
	pot_gpu_destroy(ctx);
	free(P);
	free(ru.sw_path);
	return status == EXIT_SUCCESS ? EXIT_SUCCESS : EXIT_FAILURE;
}
