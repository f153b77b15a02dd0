// Initial injection and boundary reinjection on the device.
//
// Each (re)injected particle draws from its own Philox4x32-10 stream keyed
// by (run seed, original particle index, step, attempt), so the result does
// not depend on thread scheduling or on which other particles are reinjected
// in the same step.  The samplers are the reference's:
//   * inject (pot.c:658-765, spherical domain): uniform in the shell
//     a < r < R at start (cube-root transform), on the sphere r = R at
//     reinjection with the inward radial velocity component, Maxwellian
//     components, drift added along x;
//   * sceptically_reinject (pot.c:496-652): flux-weighted drifting
//     Maxwellian at infinity through the inverse CDFs of Hutchinson 2003
//     (prng.c:138-214, Newton), entry point on the sphere from the OML orbit
//     angle alpha (integrate_for_alpha, pot.c:433-492).
// Every loop that the reference leaves unbounded (Newton iterations, the
// u^2 < chi_b rejection, the retry on NaN alpha) has a cap here; reaching one
// sets POT_E_ITER and leaves the particle at a valid boundary state.
#include "pot_push.cuh"

namespace pot {

// Which cap stopped a sampler: bits recorded in RunRec::warn beside POT_E_ITER.
constexpr uint32_t FAIL_NEWTON = 2u;   // inverse-CDF Newton iteration (prng.c:138-214)
constexpr uint32_t FAIL_REJECT = 4u;   // u^2 < chi_b rejection (pot.c:530-546)
constexpr uint32_t FAIL_RETRY = 8u;    // NaN alpha retries (pot.c:584-598)
constexpr uint32_t FAIL_SIMPSON = 16u; // orbit-integral halvings (pot.c:433-492)
constexpr uint32_t FAIL_SHELL = 32u;   // initial radius outside the grain (pot.c:703-708)
constexpr uint32_t FAIL_SPEED = 64u;   // no speed distribution for this chi_b: the inverse CDF is NaN
                                       // (u_icdf for chi_b above about U^2 + 1/2, prng.c:171-214)
// Not a failure: POT_OPT_CHI_CAP capped the edge potential (warn bit 512,
// no status).
constexpr uint32_t FAIL_CAPPED = WARN_CHI_CAP;
constexpr int NEWTON_CAP = 200;
constexpr int REJECT_CAP = 10000;
// NaN alpha means the sampled orbit meets a potential barrier; with cold ions
// (Te/Ti >> 1) and a noisy single-point edge potential, most samples can be
// rejected for a while, so this cap is generous (the reference recurses
// without bound).
constexpr int RETRY_CAP = 100000;
constexpr int SIMPSON_CAP = 100000;
constexpr int NAN_SPEED_CAP = 64;  // NaN speeds in a row taken as "every draw is NaN"

__device__ double d_u_no_flow_icdf(double chi, double q, uint32_t& fail)
{
	const double omc = 1.0 - chi;
	double u = 1.29951, p;
	int it = 0;
	do {
		const double usq = u * u;
		p = 1.0 - ((usq + omc) * exp(-usq) / omc) - q;
		u -= p / (2.0 * u * exp(-usq) * (chi - usq) / -omc);
	} while ((p * p) > 1e-16 && ++it < NEWTON_CAP);
	if (it >= NEWTON_CAP) fail |= FAIL_NEWTON;
	return u;
}

__device__ double d_u_icdf(double U, double chi, double q, uint32_t& fail)
{
	const double Usq = U * U;
	const double psi = SQRT_PI_REF * (1.0 + (2.0 * (Usq - chi))) / 2.0;
	const double p_den = 2.0 * ((U * exp(-Usq)) + (psi * erf(U)));
	const double dp_den = 2.0 * SQRT_PI_REF * (U + (psi * exp(Usq) * erf(U)));
	double u = (U > 2.1) ? U + (1.0 / U) : 1.2586147 + (0.221 * U) + (0.1903312 * U * U);
	double p;
	int it = 0;
	do {
		const double usq = u * u;
		const double temp = -(U + u) * (U + u);
		double p_num = (U - u) * exp(temp);
		p_num += (U + u) * exp((4.0 * U * u) + temp);
		p_num += psi * (erf(U - u) + erf(U + u));
		p = 1.0 - (p_num / p_den) - q;
		double dp_num = (SQRT_PI_REF * (1.0 + (2.0 * (Usq - usq)))) - (2.0 * psi);
		dp_num *= exp(-u * ((2.0 * U) + u)) - exp((2.0 * U * u) - usq);
		u -= p / (dp_num / dp_den);
	} while ((p * p) > 1e-16 && ++it < NEWTON_CAP);
	if (it >= NEWTON_CAP) fail |= FAIL_NEWTON;
	return u;
}

// mld: max_lin_dev, 0.01 in pot.c:436 and 0.1 in pot-spheroid.c:457
__device__ double d_integrate_for_alpha(double s, double chi_b, double u2, double Rol, double mld, uint32_t& fail)
{
	const double chu2 = chi_b / u2;
	const double s2 = s * s;
	const double y_one = s / sqrt(1.0 - chu2 - s2);
	double alpha = 0.0;
	double xi0 = 0.0, xi1, xi2, y0 = s, y1, y2;
	int guard = 0;
	if (s == 0.0) return 0.0;
	do {
		xi2 = 1.0;
		y2 = y_one;
		xi1 = (xi0 + xi2) / 2.0;
		y1 = 1.0 - (chu2 * xi1 * exp(Rol * (1.0 - (1.0 / xi1))));
		y1 = 1.0 / sqrt((y1 / s2) - (xi1 * xi1));
		while (fabs(y2 - y1 - (y1 - y0)) > mld) {
			xi2 = xi1;
			y2 = y1;
			xi1 = (xi0 + xi2) / 2.0;
			y1 = 1.0 - (chu2 * xi1 * exp(Rol * (1.0 - (1.0 / xi1))));
			y1 = 1.0 / sqrt((y1 / s2) - (xi1 * xi1));
			if (++guard > SIMPSON_CAP) { fail |= FAIL_SIMPSON; return 0.0; }
		}
		alpha += (xi2 - xi0) * (y0 + (4.0 * y1) + y2) / 6.0;
		xi0 = xi2;
		y0 = y2;
		if (++guard > SIMPSON_CAP) { fail |= FAIL_SIMPSON; return 0.0; }
	} while (xi2 < 1.0);
	return alpha;
}

// The same integral with a warp: for the interval starting at xi0 the
// reference halves [xi0, 1] until the integrand looks linear, re-evaluating
// one point per halving.  Here lane k evaluates the k-th halving's end point
// e_k (e_0 = 1, e_{k+1} = (xi0 + e_k) / 2, the reference's recursion) at
// once, and a ballot picks the first k that passes the linearity test -- the
// interval the sequential loop stops at, with the same values.  All lanes
// return the same alpha.
__device__ double d_integrate_for_alpha_warp(double s, double chi_b, double u2, double Rol, double mld, uint32_t& fail)
{
	const uint32_t lane = threadIdx.x & 31u;
	const double chu2 = chi_b / u2;
	const double s2 = s * s;
	const double y_one = s / sqrt(1.0 - chu2 - s2);
	if (s == 0.0) return 0.0;
	double alpha = 0.0, xi0 = 0.0, y0 = s;
	int intervals = 0;
	for (;;) {
		// Most intervals pass within the first few halvings, so halvings 1-8
		// are tried first (lanes 0-7): their end points need a recursion 8
		// deep, not 32.  The full 32-lane batch below runs only when none of
		// them passes, so the interval chosen is the same either way.
		// Lanes 8-31 meanwhile try the next interval, in groups of 8, for
		// the three likeliest outcomes (the interval ends at e_2, e_3 or e_4,
		// together about 70 % of intervals): group g = lane / 8 starts its
		// halvings at e_{g+1}, computed by the same recursion, with y(e_{g+1})
		// from lane g.  When the outcome was guessed, one round takes two
		// intervals, with the values the sequential loop would compute.
		{
			const uint32_t grp = lane >> 3, j = lane & 7u;
			double x_lo = xi0;  // start of this group's interval
			if (grp) {
				x_lo = 1.0;
				for (uint32_t k = 0; k <= grp; k++) x_lo = (xi0 + x_lo) / 2.0;  // e_{grp+1}
			}
			double ep = 1.0;
			for (uint32_t k = 0; k <= j; k++) ep = (x_lo + ep) / 2.0;  // this group's e_{j+1}
			double y = 1.0 - (chu2 * ep * exp(Rol * (1.0 - (1.0 / ep))));
			y = 1.0 / sqrt((y / s2) - (ep * ep));
			const double y_lo_g = __shfl_sync(0xffffffffu, y, grp);  // y(e_{grp+1}) from lane grp
			const double y_lo = grp ? y_lo_g : y0;
			const double y_up = __shfl_up_sync(0xffffffffu, y, 1);
			const double e_up = __shfl_up_sync(0xffffffffu, ep, 1);
			const double y_ek = j == 0 ? y_one : y_up;
			const double e_k = j == 0 ? 1.0 : e_up;
			const bool linear = !(fabs(y_ek - y - (y - y_lo)) > mld);
			const uint32_t pass_all = __ballot_sync(0xffffffffu, linear);
			const uint32_t pass = pass_all & 0xFFu;
			if (pass) {
				const int k = __ffs(pass) - 1;
				const double xk = __shfl_sync(0xffffffffu, e_k, k);
				const double yk = __shfl_sync(0xffffffffu, y_ek, k);
				const double ym = __shfl_sync(0xffffffffu, y, k);
				alpha += (xk - xi0) * (y0 + (4.0 * ym) + yk) / 6.0;
				xi0 = xk;
				y0 = yk;
				if (!(xi0 < 1.0)) break;
				if (++intervals > SIMPSON_CAP) {
					fail |= FAIL_SIMPSON;
					return 0.0;
				}
				// the interval ended at e_k: group k - 1 started there
				const uint32_t pass2 = (k >= 2 && k <= 4) ? (pass_all >> (8 * (k - 1))) & 0xFFu : 0u;
				if (pass2) {
					const int k2 = 8 * (k - 1) + __ffs(pass2) - 1;
					const double xk2 = __shfl_sync(0xffffffffu, e_k, k2);
					const double yk2 = __shfl_sync(0xffffffffu, y_ek, k2);
					const double ym2 = __shfl_sync(0xffffffffu, y, k2);
					alpha += (xk2 - xi0) * (y0 + (4.0 * ym2) + yk2) / 6.0;
					xi0 = xk2;
					y0 = yk2;
					if (!(xi0 < 1.0)) break;
					if (++intervals > SIMPSON_CAP) {
						fail |= FAIL_SIMPSON;
						return 0.0;
					}
				}
				continue;
			}
		}
		// end points e_0 .. e_32 (lane k holds e_{k+1} and its integrand)
		double e = 1.0, ek1 = 0.0;
		for (uint32_t k = 0; k <= lane; k++) e = (xi0 + e) / 2.0;  // e_{lane+1}
		ek1 = e;
		double y = 1.0 - (chu2 * ek1 * exp(Rol * (1.0 - (1.0 / ek1))));
		y = 1.0 / sqrt((y / s2) - (ek1 * ek1));
		// interval k: [xi0, e_k] with midpoint e_{k+1}; y(e_k) is y_one for k = 0
		// and the lower lane's value otherwise
		// every lane takes part in each shuffle; lane 0 then substitutes e_0, y_one
		const double y_up = __shfl_up_sync(0xffffffffu, y, 1);
		const double e_up = __shfl_up_sync(0xffffffffu, ek1, 1);
		const double y_ek = lane == 0 ? y_one : y_up;
		const double e_k = lane == 0 ? 1.0 : e_up;
		const bool linear = !(fabs(y_ek - y - (y - y0)) > mld);
		const uint32_t pass = __ballot_sync(0xffffffffu, linear);
		if (pass == 0) {
			// more than 32 halvings needed at this xi0: continue from e_32
			const double e32 = __shfl_sync(0xffffffffu, ek1, 31);
			if (e32 <= xi0 || ++intervals > SIMPSON_CAP) {
				fail |= FAIL_SIMPSON;
				return 0.0;
			}
			// the sequential loop would keep halving towards xi0 from e_32;
			// restart the batch with e_32 playing the role of 1
			double e2 = e32, y2 = __shfl_sync(0xffffffffu, y, 31);
			bool done = false;
			for (int guard = 0; guard < SIMPSON_CAP && !done; guard++) {
				double xe = e2;
				for (uint32_t k = 0; k <= lane; k++) xe = (xi0 + xe) / 2.0;
				double yy = 1.0 - (chu2 * xe * exp(Rol * (1.0 - (1.0 / xe))));
				yy = 1.0 / sqrt((yy / s2) - (xe * xe));
				const double yy_up = __shfl_up_sync(0xffffffffu, yy, 1);
				const double xe_up = __shfl_up_sync(0xffffffffu, xe, 1);
				const double y_hi = lane == 0 ? y2 : yy_up;
				const double x_hi = lane == 0 ? e2 : xe_up;
				const bool lin = !(fabs(y_hi - yy - (yy - y0)) > mld);
				const uint32_t pb = __ballot_sync(0xffffffffu, lin);
				if (pb) {
					const int k = __ffs(pb) - 1;
					const double xk = __shfl_sync(0xffffffffu, x_hi, k);
					const double yk = __shfl_sync(0xffffffffu, y_hi, k);
					const double ym = __shfl_sync(0xffffffffu, yy, k);
					alpha += (xk - xi0) * (y0 + (4.0 * ym) + yk) / 6.0;
					xi0 = xk;
					y0 = yk;
					done = true;
				} else {
					e2 = __shfl_sync(0xffffffffu, xe, 31);
					y2 = __shfl_sync(0xffffffffu, yy, 31);
				}
			}
			if (!done) {
				fail |= FAIL_SIMPSON;
				return 0.0;
			}
		} else {
			const int k = __ffs(pass) - 1;
			const double xk = __shfl_sync(0xffffffffu, e_k, k);
			const double yk = __shfl_sync(0xffffffffu, y_ek, k);
			const double ym = __shfl_sync(0xffffffffu, y, k);
			alpha += (xk - xi0) * (y0 + (4.0 * ym) + yk) / 6.0;
			xi0 = xk;
			y0 = yk;
		}
		if (!(xi0 < 1.0)) break;
		if (++intervals > SIMPSON_CAP) {
			fail |= FAIL_SIMPSON;
			return 0.0;
		}
	}
	return alpha;
}

// rotate_vec_about_xy_dir, coord.c:22-37
__device__ __forceinline__ void rot_xy(double d0, double d1, double s, double c, double& x, double& y, double& z,
                                       double offset)
{
	const double omc = 1.0 - c;
	double t0 = d0 * ((d0 * x) + (d1 * y)) * omc;
	t0 += (x * c) + (d1 * z * s);
	double t1 = d1 * ((d0 * x) + (d1 * y)) * omc;
	t1 += (y * c) - (d0 * z * s);
	double t2 = z * c;
	t2 += ((d0 * y) - (d1 * x)) * s;
	x = offset + t0;
	y = offset + t1;
	z = offset + t2;
}

// velocity_in_cartesian_coords, coord.c:6-14
__device__ __forceinline__ void vel_cart(double v0, double v1, double v2, double phi, double theta, double& vx,
                                         double& vy, double& vz)
{
	double sp, cp, st, ct;
	sincos(phi, &sp, &cp);
	sincos(theta, &st, &ct);
	vx = (v0 * cp * st) - (v1 * sp) + (v2 * cp * ct);
	vy = (v0 * sp * st) + (v1 * cp) + (v2 * sp * ct);
	vz = (v0 * ct) - (v2 * st);
}

// nrv_pair, prng.c:32-47
__device__ __forceinline__ void nrv_pair(Stream& st, double sd, double& a, double& b)
{
	const double urv2 = st.rnd(1.0);
	double urv1;
	int guard = 0;
	do {
		urv1 = st.rnd(1.0);
	} while (urv1 == 0.0 && ++guard < 64);
	const double r = sqrt(-2.0 * log(urv1));
	const double theta = 2.0 * PI_REF * urv2;
	double s, c;
	sincos(theta, &s, &c);
	a = sd * r * c;
	b = sd * r * s;
}

// sceptically_reinject, pot.c:496-652.  WARP: every lane of a warp runs
// this for the same particle with identical streams (identical results) and
// the orbit integral is evaluated cooperatively.
template <bool WARP>
__device__ void sceptic_reinject(Stream& st, int sp, double chi_b_in, const Params& P, double4& p, double4& v,
                                 uint32_t& fail)
{
	const double v_n = sp == SP_E ? P.vn_e : P.vn_i;
	double chi_b = chi_b_in;
	double u_mag = 0.0, u2 = 0.0, cz = 0.0, b = 0.0, alpha = 0.0, u[3];
	int nan_speeds = 0;
	for (int attempt = 0;; attempt++) {
		chi_b = chi_b_in;
		if (sp == SP_E) chi_b *= -P.Ti / P.Te;
		if (P.flags & FLAG_CHI_CAP) {
			// POT_OPT_CHI_CAP: keep the speed distribution defined.  The inverse
			// CDF's normaliser 2 (U exp(-U^2) + psi erf(U)), psi = sqrt(pi)
			// (1 + 2 (U^2 - chi)) / 2, vanishes at chi* = U^2 + 1/2 +
			// U exp(-U^2) / (sqrt(pi) erf(U)) (1 in the limit U -> 0, the no-flow
			// form's 1 - chi > 0); above it every draw is NaN.  The cap is 0.95 chi*.
			const double U = P.x_drift / v_n;
			const double cap = 0.95 * ((U * U) + 0.5 + (U > 1e-8 ? U * exp(-U * U) / (SQRT_PI_REF * erf(U)) : 0.5));
			if (chi_b > cap) {
				chi_b = cap;
				fail |= FAIL_CAPPED;
			}
		}
		if (P.x_drift != 0.0) {
			const double U = P.x_drift / v_n;
			int k = 0;
			do {
				u_mag = d_u_icdf(U, chi_b, st.rnd(1.0), fail);
				u2 = u_mag * u_mag;
			} while (u2 < chi_b && ++k < REJECT_CAP);
			if (k >= REJECT_CAP) fail |= FAIL_REJECT;
			const double q = st.rnd(1.0);
			cz = log(q + (1.0 - q) * exp(-4.0 * u_mag * U)) / (2.0 * u_mag * U);
			cz += 1.0;
		} else {
			int k = 0;
			do {
				u_mag = d_u_no_flow_icdf(chi_b, st.rnd(1.0), fail);
				u2 = u_mag * u_mag;
			} while (u2 < chi_b && ++k < REJECT_CAP);
			if (k >= REJECT_CAP) fail |= FAIL_REJECT;
			cz = st.rnd(2.0) - 1.0;
		}
		if (isnan(u2)) {
			// A NaN speed makes alpha NaN in the reference, which retries
			// (pot.c:582-599): the same here.  When every speed it can draw is
			// NaN (chi above about U^2 + 1/2) it would retry without end: a run
			// of NAN_SPEED_CAP NaN speeds in a row stops the sampler instead.
			if (++nan_speeds >= NAN_SPEED_CAP) {
				fail |= FAIL_SPEED;
				alpha = 0.0;
				break;
			}
			alpha = NAN;
			if (attempt + 1 >= RETRY_CAP) break;
			continue;
		}
		nan_speeds = 0;
		u[0] = 0.0;
		u[1] = 0.0;
		u[2] = u_mag;
		rot_xy(0.0, 1.0, cz, sqrt(1.0 - (cz * cz)), u[0], u[1], u[2], 0.0);
		const double psi = st.rnd(2.0 * PI_REF);
		double sps, cps;
		sincos(psi, &sps, &cps);
		rot_xy(1.0, 0.0, sps, cps, u[0], u[1], u[2], 0.0);
		b = sqrt(st.rnd(1.0 - (chi_b / u2)));
		alpha = WARP ? d_integrate_for_alpha_warp(b, chi_b, u2, P.Rol, P.max_lin_dev, fail)
		             : d_integrate_for_alpha(b, chi_b, u2, P.Rol, P.max_lin_dev, fail);
		if (!isnan(alpha) || attempt + 1 >= RETRY_CAP) break;
	}
	if (isnan(alpha)) {
		fail |= FAIL_RETRY;
		alpha = 0.0;
	}
	const double phi = st.rnd(2.0 * PI_REF);
	double sa, ca, sph, cph;
	sincos(alpha, &sa, &ca);
	sincos(phi, &sph, &cph);
	double x = P.mpp * P.r_pix * sa * cph;
	double y = P.mpp * P.r_pix * sa * sph;
	double z = P.mpp * P.r_pix * ca;
	const double nrm = sqrt((u[0] * u[0]) + (u[1] * u[1]));
	const double a0 = u[1] / nrm, a1 = -u[0] / nrm;
	const double co_z = u[2] / u_mag;
	const double si_z = sin(acos(co_z));
	rot_xy(a0, a1, si_z, co_z, x, y, z, P.mpp * P.r_pix);
	const double vz_ = u_mag * b;
	const double vr = -sqrt(u2 - chi_b - (vz_ * vz_));
	double vx, vy, vz;
	vel_cart(vr, 0.0, vz_, phi, alpha, vx, vy, vz);
	rot_xy(a0, a1, si_z, co_z, vx, vy, vz, 0.0);
	p = make_double4(x, y, z, p.w);
	v = make_double4(vx * v_n, vy * v_n, vz * v_n, 0.0);
}

// inject, pot.c:658-765 (spherical domain, grain enabled)
template <bool WARP>
__device__ void inject(Stream& st, int sp, bool reinjection, double chi_b, const Params& P, double4& p, double4& v,
                       uint32_t& fail)
{
	double sigma = sp == SP_ION ? P.sigma_i : P.sigma_e;
	const bool sceptic = (P.flags & FLAG_SCEPTIC) != 0;
	if (!sceptic && !reinjection) sigma *= 0.85;
	double r;
	if (!reinjection) {
		const double rmax3 = (double)(P.r_pix * P.r_pix * P.r_pix);
		r = P.mpp * cbrt(st.rnd(rmax3));
		int guard = 0;
		while (r <= P.a && ++guard < REJECT_CAP) r = P.mpp * cbrt(st.rnd(rmax3));
		if (guard >= REJECT_CAP) fail |= FAIL_SHELL;
	} else {
		r = P.mpp * P.r_pix;
	}
	if (sceptic && reinjection) {
		sceptic_reinject<WARP>(st, sp, chi_b, P, p, v, fail);
		return;
	}
	const double phi = st.rnd(2.0 * PI_REF);
	const double theta = acos(st.rnd(2.0) - 1.0);
	double sth, cth, sph, cph;
	sincos(theta, &sth, &cth);
	sincos(phi, &sph, &cph);
	const double c = P.mpp * P.r_pix;
	p = make_double4(c + (r * sth * cph), c + (r * sth * sph), c + (r * cth), p.w);
	double vx, vy, vz;
	if (!reinjection) {
		nrv_pair(st, sigma, vx, vy);
		double d;
		nrv_pair(st, sigma, d, vz);
	} else {
		double v0, v1, v2, d;
		nrv_pair(st, sigma, v0, v1);
		nrv_pair(st, sigma, d, v2);
		if (v0 > 0.0) v0 = -v0;
		vel_cart(v0, v1, v2, phi, theta, vx, vy, vz);
	}
	v = make_double4(vx + P.x_drift, vy, vz, 0.0);
}

__device__ __forceinline__ bool outside_sphere(const double4& p, const Params& P)
{
	return sqrt(dsq3(dsub(p.x, P.rad), dsub(p.y, P.rad), dsub(p.z, P.rad))) > P.rad;
}

// Reinjection list entries: slot | reason << 30, reason 1 = absorbed by
// the grain (reinjected, then tested against the boundary once more, as
// pot.c:2676 followed by pot.c:2691 -- with OUT_BOUNCE that test is the
// wall's, against the start-of-step position in src64), 2 = left the domain.
template <class G>
__device__ __forceinline__ void reinject_body(G grd, double4* __restrict__ pos, double4* __restrict__ vel,
                                              const uint32_t* __restrict__ pid, const uint32_t* __restrict__ list,
                                              const double4* __restrict__ src64, const Params& P, RunRec* rec)
{
	if (rec->status != POT_OK) return;
	const uint32_t n = rec->n_rein;
	const uint32_t t = (uint32_t)rec->t_steps;
	const double chi_b = rec->chi_b;
	const uint32_t lane = threadIdx.x & 31u;
	const uint32_t warps = grd.n() * (blockDim.x >> 5);
	// one warp per reinjected particle
	for (uint32_t e = grd.id() * (blockDim.x >> 5) + (threadIdx.x >> 5); e < n; e += warps) {
		const uint32_t w = list[e];
		const uint32_t s = w & 0x3FFFFFFFu;
		const uint32_t reason = w >> 30;
		const uint32_t id = pid[s];
		double4 p = pos[s];
		double4 v = vel[s];
		const int sp = (int)p.w;
		uint32_t fail = 0;
		uint32_t attempt = 0;
		Stream st;
		st.init(P.seed, id, t, 0x10000u | attempt++);
		inject<true>(st, sp, true, chi_b, P, p, v, fail);
		int wall = 0;
		if ((reason & 1u) && P.bounce > 0.0) {
			double3 x = make_double3(p.x, p.y, p.z);
			wall = bounce_wall(src64[s], x, v, P);
			p = make_double4(x.x, x.y, x.z, p.w);
		} else if ((reason & 1u) && outside_sphere(p, P)) {
			st.init(P.seed, id, t, 0x10000u | attempt++);
			inject<true>(st, sp, true, chi_b, P, p, v, fail);
		}
		if (lane == 0) {
			count_wall(rec, wall);
			if (fail) {
				atomicOr(&rec->warn, fail);
				if (fail & ~FAIL_CAPPED) set_status(rec, POT_E_ITER);
			}
			pos[s] = p;
			vel[s] = v;
		}
	}
}

__global__ void k_reinject(double4* __restrict__ pos, double4* __restrict__ vel, const uint32_t* __restrict__ pid,
                           const uint32_t* __restrict__ list, const double4* __restrict__ src64, Params P, RunRec* rec)
{
	reinject_body(GridSelf {}, pos, vel, pid, list, src64, P, rec);
}

// init_particles for one rank (pot.c:887-935), reference order: slot i holds
// particle i.
__global__ void k_init(double4* __restrict__ pos, double4* __restrict__ vel, uint32_t* __restrict__ pid, Params P,
                       RunRec* rec)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= P.n_total) return;
	pid[i] = i;
	if (i == 0) {
		pos[0] = make_double4(P.rad, P.rad, P.rad, (double)SP_DUST);
		vel[0] = make_double4(0.0, 0.0, 0.0, 0.0);
		return;
	}
	const int sp = species_of_id(i, P.n_ions);
	double4 p = make_double4(0.0, 0.0, 0.0, (double)sp), v;
	uint32_t fail = 0;
	Stream st;
	st.init(P.seed, i, 0u, 0x20000u);
	inject<false>(st, sp, false, 0.0, P, p, v, fail);
	if (fail) {
		atomicOr(&rec->warn, fail);
		if (fail & ~FAIL_CAPPED) set_status(rec, POT_E_ITER);
	}
	pos[i] = p;
	vel[i] = v;
}

void launch_reinject(double4* pos, double4* vel, const uint32_t* pid, const uint32_t* rein_list,
                     const double4* src64, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm)
{
	ScopedKernel k(tm, "reinject");
	k_reinject<<<148, 128, 0, s>>>(pos, vel, pid, rein_list, src64, P, rec);
}

void launch_init(double4* pos, double4* vel, uint32_t* pid, const Params& P, RunRec* rec, cudaStream_t s,
                 Timer& tm)
{
	ScopedKernel k(tm, "init");
	k_init<<<(P.n_total + 127) / 128, 128, 0, s>>>(pos, vel, pid, P, rec);
}

}  // namespace pot

// ---------------------------------------------------------------------------
// packed batch: the reinjection of every member in one launch
// ---------------------------------------------------------------------------
namespace pot {

__global__ void kp_reinject(PackDev B, int k)
{
	const SegBlock sb = seg_block(B.pre[PS_SMALL], B.M);
	const MemberView& v = B.mv[sb.m];
	const uint32_t b = pack_out(v, k);
	reinject_body(GridSeg { sb.id, sb.n }, v.pos[b], v.vel[b], v.pid[b], v.rein_list, v.src64, v.P, v.rec);
}

void pack_reinject(const PackDev& B, int k, cudaStream_t s)
{
	kp_reinject<<<B.blocks[PS_SMALL], 128, 0, s>>>(B, k);
}

}  // namespace pot
