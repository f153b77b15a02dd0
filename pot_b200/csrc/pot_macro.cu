// Macroscopic summary sums on the device (write_macroscopic_data_to_file,
// pot.c:3261-3508), so that a record step needs no download of the
// particles: the same two passes over the plasma particles as the reference
// -- counts, kinetic energies, speeds, mean velocities and angular momenta
// about the domain centre; then, about those means, the central moments of
// the electron kinetic energy and of both species' speeds, the velocity
// dispersions and the electron x moments -- as per-block partial sums in
// FP64 (the reference accumulates in x87 long double), added in block order
// so the result does not depend on scheduling.
#include "pot_tree.cuh"

namespace pot {

constexpr int MACRO_BLOCKS = 296;  // 2 x 148
constexpr int MACRO_THREADS = 256;
// pass-1 sums (the first 20 doubles of pot_macro_sums): 0 n_e, 1 n_i, 2 K_e,
// 3 s_e, 4 s_i, 5-7 v_e, 8-10 v_i, 11-13 am_e, 14-16 am_i, 17-19 unused
constexpr int M2 = 18;  // pass-2 sums (the next 18 doubles)

struct MacroMeans {
	double n_e, n_i, K_e, s_e, s_i;
	double v_e[3], v_i[3];
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
	for (int o = 16; o; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
	return v;
}

template <int K>
__device__ void block_reduce(double (&acc)[K], double* __restrict__ out)
{
	__shared__ double part[MACRO_THREADS / 32][K];
	const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
	for (int k = 0; k < K; k++) {
		const double s = warp_sum(acc[k]);
		if (lane == 0) part[w][k] = s;
	}
	__syncthreads();
	if (threadIdx.x < K) {
		double t = 0.0;
		for (int j = 0; j < MACRO_THREADS / 32; j++) t += part[j][threadIdx.x];
		out[threadIdx.x] = t;
	}
}

// pass 1 (pot.c:3354-3394)
__global__ void __launch_bounds__(MACRO_THREADS) k_macro1(const double4* __restrict__ pos,
                                                          const double4* __restrict__ vel, Params P,
                                                          double* __restrict__ partial)
{
	double a[20];
#pragma unroll
	for (int k = 0; k < 20; k++) a[k] = 0.0;
	const double cent = P.rad;
	for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < P.n; s += gridDim.x * blockDim.x) {
		const double4 p = pos[s];
		const int sp = (int)p.w;
		if (sp == SP_DUST) continue;
		const double4 v = vel[s];
		const double sp2 = v.x * v.x + v.y * v.y + v.z * v.z;
		const double vm = sqrt(sp2);
		const double rx = p.x - cent, ry = p.y - cent, rz = p.z - cent;
		const double amx = (ry * v.z) - (rz * v.y);
		const double amy = -((rx * v.z) - (rz * v.x));
		const double amz = (rx * v.y) - (ry * v.x);
		if (sp == SP_E) {
			a[0] += 1.0;
			a[2] += 0.5 * MASS_E * vm * vm;
			a[3] += vm;
			a[5] += v.x;
			a[6] += v.y;
			a[7] += v.z;
			a[11] += amx;
			a[12] += amy;
			a[13] += amz;
		} else {
			a[1] += 1.0;
			a[4] += vm;
			a[8] += v.x;
			a[9] += v.y;
			a[10] += v.z;
			a[14] += amx;
			a[15] += amy;
			a[16] += amz;
		}
	}
	block_reduce<20>(a, &partial[20 * blockIdx.x]);
}

// sum the pass-1 partials in block order; means for pass 2
__global__ void k_macro1_final(const double* __restrict__ partial, double* __restrict__ sums1, MacroMeans* means)
{
	__shared__ double t[20];
	if (threadIdx.x < 20) {
		double s = 0.0;
		for (int b = 0; b < MACRO_BLOCKS; b++) s += partial[20 * b + threadIdx.x];
		t[threadIdx.x] = s;
		sums1[threadIdx.x] = s;
	}
	__syncthreads();
	if (threadIdx.x == 0) {
		MacroMeans m;
		m.n_e = t[0];
		m.n_i = t[1];
		m.K_e = t[2] / t[0];
		m.s_e = t[3] / t[0];
		m.s_i = t[4] / t[1];
		for (int k = 0; k < 3; k++) {
			m.v_e[k] = t[5 + k] / t[0];
			m.v_i[k] = t[8 + k] / t[1];
		}
		*means = m;
	}
}

// pass 2 (pot.c:3427-3461): 0 sum K_e^2, 1-2 sum x, x^2 (electrons), 3-5 central
// moments 2-4 of K_e, 6-8 of |v_e|, 9 sum |v_e - <v_e>|^2, 10-11 sum K_i, K_i^2,
// 12-14 central moments 2-4 of |v_i|, 15 sum |v_i - <v_i>|^2, 16-17 unused
__global__ void __launch_bounds__(MACRO_THREADS) k_macro2(const double4* __restrict__ pos,
                                                          const double4* __restrict__ vel, Params P,
                                                          const MacroMeans* __restrict__ means,
                                                          double* __restrict__ partial)
{
	double a[M2];
#pragma unroll
	for (int k = 0; k < M2; k++) a[k] = 0.0;
	const MacroMeans m = *means;
	for (uint32_t s = blockIdx.x * blockDim.x + threadIdx.x; s < P.n; s += gridDim.x * blockDim.x) {
		const double4 p = pos[s];
		const int sp = (int)p.w;
		if (sp == SP_DUST) continue;
		const double4 v = vel[s];
		const double vm = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
		if (sp == SP_E) {
			const double K = 0.5 * MASS_E * vm * vm;
			a[0] += K * K;
			a[1] += p.x;
			a[2] += p.x * p.x;
			const double Ks = K - m.K_e;
			a[3] += Ks * Ks;
			a[4] += Ks * Ks * Ks;
			a[5] += Ks * Ks * Ks * Ks;
			const double vs = vm - m.s_e;
			a[6] += vs * vs;
			a[7] += vs * vs * vs;
			a[8] += vs * vs * vs * vs;
			const double dx = v.x - m.v_e[0], dy = v.y - m.v_e[1], dz = v.z - m.v_e[2];
			a[9] += dx * dx + dy * dy + dz * dz;
		} else {
			const double K = 0.5 * P.m_ion * vm * vm;
			a[10] += K;
			a[11] += K * K;
			const double vs = vm - m.s_i;
			a[12] += vs * vs;
			a[13] += vs * vs * vs;
			a[14] += vs * vs * vs * vs;
			const double dx = v.x - m.v_i[0], dy = v.y - m.v_i[1], dz = v.z - m.v_i[2];
			a[15] += dx * dx + dy * dy + dz * dz;
		}
	}
	block_reduce<M2>(a, &partial[M2 * blockIdx.x]);
}

// With the Poisson ion collection the ions' temperature from the velocity
// dispersion becomes the cached Proc.Ti, as pot.c:3442-3448 does.
__global__ void k_macro2_final(const double* __restrict__ partial, const double* __restrict__ sums1,
                               double* __restrict__ sums2, Params P, RunRec* rec)
{
	if (threadIdx.x < M2) {
		double s = 0.0;
		for (int b = 0; b < MACRO_BLOCKS; b++) s += partial[M2 * b + threadIdx.x];
		sums2[threadIdx.x] = s;
		if (rec && threadIdx.x == 15 && sums1[1] > 0.0) rec->ion_temp = s * ((P.m_ion / (3.0 * KB)) / sums1[1]);
	}
}

size_t macro_scratch_doubles() { return (size_t)MACRO_BLOCKS * 20 + 64 + 16; }

// scratch: partials (MACRO_BLOCKS x 20), then sums1[20], sums2[M2], means
void launch_macro(const double4* pos, const double4* vel, const Params& P, double* scratch, RunRec* rec,
                  cudaStream_t s, Timer& tm)
{
	double* partial = scratch;
	double* sums1 = scratch + (size_t)MACRO_BLOCKS * 20;
	double* sums2 = sums1 + 20;
	MacroMeans* means = reinterpret_cast<MacroMeans*>(sums2 + 24);
	ScopedKernel k(tm, "macro", 4);
	k_macro1<<<MACRO_BLOCKS, MACRO_THREADS, 0, s>>>(pos, vel, P, partial);
	k_macro1_final<<<1, 32, 0, s>>>(partial, sums1, means);
	k_macro2<<<MACRO_BLOCKS, MACRO_THREADS, 0, s>>>(pos, vel, P, means, partial);
	k_macro2_final<<<1, 32, 0, s>>>(partial, sums1, sums2, P, (P.flags & FLAG_POIS) ? rec : nullptr);
}

}  // namespace pot
