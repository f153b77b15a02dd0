// C ABI (include/pot_gpu.h): run context, host <-> device transfers, the
// per-step launch sequence, inspection queries and the kernel timer.
#include <cmath>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>

#include "pot_tree.cuh"

using namespace pot;

struct pot_gpu_ctx {
	pot_run_cfg cfg;
	pot_gpu_opts opts;
	Params P;
	cudaStream_t stream = nullptr;
	bool own_stream = false;
	int device = 0;
	uint32_t n = 0;
	double4* pos[2] = { nullptr, nullptr };
	double4* vel[2] = { nullptr, nullptr };
	uint32_t* pid[2] = { nullptr, nullptr };
	int cur = 0;
	double4* src64 = nullptr;
	float4* src32 = nullptr;
	// non-Boris integrators: first-half accelerations and intermediate sources
	double4* acc = nullptr;
	double4* src64b = nullptr;
	float4* src32b = nullptr;
	uint64_t* keys[2] = { nullptr, nullptr };
	uint32_t* vals[2] = { nullptr, nullptr };
	int kb = 0;  // which key buffer holds the sorted keys
	uint32_t* counts = nullptr;
	uint32_t* block_sums = nullptr;
	uint8_t* due = nullptr;
	uint32_t* due_tiles = nullptr;   // due flags per scan tile (counted by the reorder)
	uint32_t* due_list = nullptr;
	uint32_t* due_prefix = nullptr;  // n + 1
	uint2* groups = nullptr;
	uint2* groups_all = nullptr;     // fast form, potential energies
	uint8_t* gcell = nullptr;        // fast form: groups per tree cell (pre-order group build)
	uint32_t* gblk = nullptr;        // fast form: groups per build block, then their prefix
	double* epe_partial = nullptr;   // per-block / per-group partial sums
	double* macro = nullptr;         // macroscopic-summary partials and sums
	uint32_t* rein_list = nullptr;
	uint32_t* inv = nullptr;
	pot_particle* aos = nullptr;
	TreeDev T {};
	RunRec* rec = nullptr;
	StepHist* hist = nullptr;
	// query scratch
	double* q_xyz = nullptr;
	double* q_out = nullptr;
	uint32_t* q_idx = nullptr;
	uint32_t* q_slot = nullptr;
	size_t q_cap = 0;
	bool uploaded = false;
	bool tree_valid = false;
	int sticky = POT_OK;
	bool dry = false;       // count bytes, allocate nothing (pot_gpu_bytes_needed)
	uint64_t bytes = 0;     // device bytes held (or needed, when dry)
	Timer timer;
	std::vector<void*> allocs;
	// one step as a CUDA graph, per buffer parity before the step and per
	// POT_STEP_EPE (captured on first use; not with event timing)
	cudaGraphExec_t step_exec[2][2] = { { nullptr, nullptr }, { nullptr, nullptr } };
	uint64_t step_launches[2][2] = { { 0, 0 }, { 0, 0 } };
	bool graphs_off = false;  // a capture failed once: enqueue kernel by kernel
	// the drop-in call's copy stream, chunk events and pinned records
	cudaStream_t xfer = nullptr;
	cudaEvent_t xev[2 * 4 + 1] = {};
	RunRec* h_rec = nullptr;
	StepHist* h_hist = nullptr;
	// reference-index range [lo, hi] of the particles due in the drop-in
	// call's step (device and pinned host copies) and the event after which
	// the host reads it
	uint32_t* due_rng = nullptr;
	uint32_t* h_due_rng = nullptr;
	cudaEvent_t rng_ev = nullptr;
};

// ---------------------------------------------------------------------------
// Timer
// ---------------------------------------------------------------------------
namespace pot {

cudaEvent_t Timer::take()
{
	if (!pool_.empty()) {
		cudaEvent_t e = pool_.back();
		pool_.pop_back();
		return e;
	}
	cudaEvent_t e = nullptr;
	cudaEventCreate(&e);
	return e;
}

int Timer::kind_of(const char* name)
{
	for (size_t i = 0; i < names_.size(); i++)
		if (std::strcmp(names_[i], name) == 0) return (int)i;
	names_.push_back(name);
	ms_.push_back(0.0);
	count_.push_back(0);
	return (int)names_.size() - 1;
}

void Timer::begin(const char* name)
{
	if (!enabled || open_kind_ >= 0) return;  // nested scopes: the outer one times
	open_kind_ = kind_of(name);
	open_a_ = take();
	cudaEventRecord(open_a_, stream);
}

void Timer::end()
{
	if (!enabled || open_kind_ < 0) return;
	cudaEvent_t b = take();
	cudaEventRecord(b, stream);
	pending_.push_back({ open_kind_, open_a_, b });
	open_kind_ = -1;
	open_a_ = nullptr;
}

void Timer::resolve()
{
	for (auto& p : pending_) {
		float ms = 0.f;
		if (cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
			ms_[p.kind] += ms;
			count_[p.kind] += 1;
		}
		pool_.push_back(p.a);
		pool_.push_back(p.b);
	}
	pending_.clear();
}

void Timer::reset()
{
	resolve();
	for (auto& m : ms_) m = 0.0;
	for (auto& c : count_) c = 0;
}

int Timer::report(int max, const char** names, double* ms, uint64_t* launches) const
{
	const int n = (int)names_.size();
	for (int i = 0; i < n && i < max; i++) {
		if (names) names[i] = names_[i];
		if (ms) ms[i] = ms_[i];
		if (launches) launches[i] = count_[i];
	}
	return n;
}

Timer::~Timer()
{
	for (auto& p : pending_) {
		cudaEventDestroy(p.a);
		cudaEventDestroy(p.b);
	}
	for (auto e : pool_) cudaEventDestroy(e);
}

}  // namespace pot

// ---------------------------------------------------------------------------
// small kernels: layout conversion, inverse permutation
// ---------------------------------------------------------------------------
__global__ void k_from_aos(const pot_particle* __restrict__ aos, uint32_t n, double4* __restrict__ pos,
                           double4* __restrict__ vel, uint32_t* __restrict__ pid, RunRec* rec)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const pot_particle p = aos[i];
	int sp = p.species;
	if (sp < 0 || sp > 2) {
		set_status(rec, POT_E_ARG);
		sp = SP_E;
	}
	pos[i] = make_double4(p.x, p.y, p.z, (double)sp);
	vel[i] = make_double4(p.vx, p.vy, p.vz, 0.0);
	pid[i] = i;
}

__global__ void k_to_aos(const double4* __restrict__ pos, const double4* __restrict__ vel,
                         const uint32_t* __restrict__ pid, uint32_t n, pot_particle* __restrict__ aos)
{
	const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s >= n) return;
	const double4 p = pos[s];
	const double4 v = vel[s];
	pot_particle o;
	o.x = p.x; o.y = p.y; o.z = p.z;
	o.vx = v.x; o.vy = v.y; o.vz = v.z;
	o.species = (int32_t)p.w;
	o.pad = 0;
	aos[pid[s]] = o;
}

// The drop-in call's chunked forms: particles [i0, i0 + cnt) from the host
// record array, and (gathered through the inverse permutation) back into it
// with coalesced writes.
__global__ void k_from_aos_range(const pot_particle* __restrict__ aos, uint32_t i0, uint32_t cnt,
                                 double4* __restrict__ pos, double4* __restrict__ vel, uint32_t* __restrict__ pid,
                                 RunRec* rec)
{
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= cnt) return;
	const uint32_t i = i0 + k;
	const pot_particle p = aos[i];
	int sp = p.species;
	if (sp < 0 || sp > 2) {
		set_status(rec, POT_E_ARG);
		sp = SP_E;
	}
	pos[i] = make_double4(p.x, p.y, p.z, (double)sp);
	vel[i] = make_double4(p.vx, p.vy, p.vz, 0.0);
	pid[i] = i;
}

// k_from_aos_range that also records the smallest and largest reference
// index of the particles due at step t (t % tss[species] == 0, as the
// reorder's due flags have it) in rng[0] (atomicMin) and rng[1] (atomicMax).
__global__ void k_from_aos_range_due(const pot_particle* __restrict__ aos, uint32_t i0, uint32_t cnt,
                                     double4* __restrict__ pos, double4* __restrict__ vel,
                                     uint32_t* __restrict__ pid, RunRec* rec, unsigned long long t, uint3 tss,
                                     uint32_t* __restrict__ rng)
{
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	bool due = false;
	uint32_t i = 0;
	if (k < cnt) {
		i = i0 + k;
		const pot_particle p = aos[i];
		int sp = p.species;
		if (sp < 0 || sp > 2) {
			set_status(rec, POT_E_ARG);
			sp = SP_E;
		}
		pos[i] = make_double4(p.x, p.y, p.z, (double)sp);
		vel[i] = make_double4(p.vx, p.vy, p.vz, 0.0);
		pid[i] = i;
		const uint32_t m = sp == SP_DUST ? tss.x : (sp == SP_ION ? tss.y : tss.z);
		due = (t % m) == 0;
	}
	// one atomic pair per warp
	const unsigned int b = __ballot_sync(0xffffffffu, due);
	if (b && (threadIdx.x & 31u) == 0) {
		const uint32_t w0 = i0 + (blockIdx.x * blockDim.x + (threadIdx.x & ~31u));
		atomicMin(&rng[0], w0 + (uint32_t)(__ffs(b) - 1));
		atomicMax(&rng[1], w0 + (uint32_t)(31 - __clz(b)));
	}
}

__global__ void k_to_aos_gather(const double4* __restrict__ pos, const double4* __restrict__ vel,
                                const uint32_t* __restrict__ inv, uint32_t i0, uint32_t cnt,
                                pot_particle* __restrict__ aos)
{
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k >= cnt) return;
	const uint32_t i = i0 + k;
	const uint32_t s = inv[i];
	const double4 p = pos[s];
	const double4 v = vel[s];
	pot_particle o;
	o.x = p.x; o.y = p.y; o.z = p.z;
	o.vx = v.x; o.vy = v.y; o.vz = v.z;
	o.species = (int32_t)p.w;
	o.pad = 0;
	aos[i] = o;
}

__global__ void k_inverse(const uint32_t* __restrict__ pid, uint32_t n, uint32_t* __restrict__ inv)
{
	const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
	if (s < n) inv[pid[s]] = s;
}

__global__ void k_map_slots(const uint32_t* __restrict__ inv, const uint32_t* __restrict__ idx, uint32_t nq,
                            uint32_t n, uint32_t* __restrict__ slot)
{
	const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
	if (k < nq) slot[k] = idx[k] < n ? inv[idx[k]] : 0xFFFFFFFFu;
}

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
#define CK(call)                                                        \
	do {                                                                \
		cudaError_t e_ = (call);                                        \
		if (e_ != cudaSuccess) {                                        \
			fprintf(stderr, "pot_gpu: %s: %s\n", #call, cudaGetErrorString(e_)); \
			return e_ == cudaErrorMemoryAllocation ? POT_E_NOMEM : POT_E_CUDA; \
		}                                                               \
	} while (0)

template <typename T>
static int dalloc(pot_gpu_ctx* c, T** p, size_t count)
{
	*p = nullptr;
	if (count == 0) count = 1;
	c->bytes += (sizeof(T) * count + 255) & ~(size_t)255;
	if (c->dry) return POT_OK;
	cudaError_t e = cudaMalloc((void**)p, sizeof(T) * count);
	if (e != cudaSuccess) {
		*p = nullptr;
		return e == cudaErrorMemoryAllocation ? POT_E_NOMEM : POT_E_CUDA;
	}
	c->allocs.push_back((void*)*p);
	return POT_OK;
}

static inline uint32_t nblk(size_t n, int t) { return (uint32_t)((n + t - 1) / t); }

// From this many particles on, a single run builds its target groups in tree
// pre-order (two more launches).  The walk's warps then share the tree nodes
// they read in L2: on the 4,000,001-particle plasma the walk's L2 hit rate
// went from 79 % to 92 %, its DRAM traffic from 1.28 GB to 0.48 GB a launch
// and the step from 4.80 to 4.66 ms.  On the 1,000,001-particle plasma, whose
// tree and sources (about 30 MB) stay in L2 in any order, the two launches
// only cost time (1.188 against 1.204 ms).
constexpr uint32_t ORDERED_GROUPS_MIN_N = 2000000u;

static int fill_params(pot_gpu_ctx* c)
{
	const pot_run_cfg& r = c->cfg;
	Params& P = c->P;
	std::memset(&P, 0, sizeof(P));
	P.n = (uint32_t)r.N;
	P.n_total = (uint32_t)r.N;
	P.n_ions = (uint32_t)((r.N - 1) / 2);
	P.r_pix = r.r;
	P.leaf_size = c->opts.leaf_size;
	P.flags = r.flags | ((c->opts.flags & POT_OPT_CHI_CAP) ? FLAG_CHI_CAP : 0u);
	P.form = c->opts.form;
	// Fast form: bucket leaves of 8 or more need few levels (a level-10 cell holds on
	// average N / 5.6e8 particles, 0.03 at the largest N), and 30 key bits sort in
	// four passes; smaller leaves keep 16 levels.  A cell at the deepest level is a
	// leaf whatever its count.
	P.max_level = c->opts.form == POT_FORM_FAST ? (c->opts.leaf_size >= 8 ? 10u : 16u) : (uint32_t)MAX_LEVELS;
	P.key_bits = c->opts.form == POT_FORM_FAST ? 63u - 3u * P.max_level : 0u;
	P.group_max = c->opts.group_size ? c->opts.group_size : 32u;
	P.chi_ranks = c->opts.chi_b_ranks ? c->opts.chi_b_ranks : 1u;
	if (P.chi_ranks > 64) return POT_E_ARG;
	P.seed = c->opts.seed;
	// grain shape: 0 sphere, A > 1 prolate, 0 < A < 1 oblate (pot-spheroid.c:4797-4827)
	if (r.A == 0.0) {
		P.shape = 0;
	} else if (r.A > 1.0) {
		P.shape = 1;
	} else if (r.A > 0.0 && r.A < 1.0) {
		P.shape = 2;
	} else {
		return POT_E_ARG;
	}
	P.n_tree = P.shape ? P.n - 1 : P.n;
	P.m_ion = (P.shape ? 1836.153 : MIME) * ME;
	P.max_lin_dev = P.shape ? 0.1 : 0.01;
	if (P.shape) {
		const double A = r.A, a = r.a;
		P.s_A = A;
		P.s_thr = a * a * std::pow(A, 4.0 / 3.0);
		if (P.shape == 1) {
			P.s_fc_f = (a * std::sqrt(A * A - 1.0)) * std::pow(A, -1.0 / 3.0);
			P.s_fc_p = a * std::sqrt(A * A - 1.0) / std::pow(A, 1.0 / 3.0);
			P.s_num = std::acosh(A);
			P.s_den_f = 4.0 * PI_REF * EPSILON0 * P.s_fc_f * std::log(A - std::sqrt(A * A - 1.0));
			P.s_den_p = 4.0 * PI_REF * EPSILON0 * P.s_fc_p * std::log(A - std::sqrt(A * A - 1.0));
		} else {
			P.s_fc_f = (a * std::sqrt(1.0 - A * A)) * std::pow(A, -1.0 / 3.0);
			P.s_fc_p = P.s_fc_f;
			P.s_num = std::acos(A);
			const double at = std::atan((1.0 - std::sqrt(1.0 - A * A)) / A) - 0.25 * PI_REF;
			P.s_den_f = 8.0 * PI_REF * EPSILON0 * P.s_fc_f * at;
			P.s_den_p = 4.0 * PI_REF * EPSILON0 * P.s_fc_p * at;
		}
		double ax[3] = { r.axis[0], r.axis[1], r.axis[2] };
		double nrm = std::sqrt(ax[0] * ax[0] + ax[1] * ax[1] + ax[2] * ax[2]);
		if (!(nrm > 0.0)) {
			ax[0] = 1.0;
			ax[1] = ax[2] = 0.0;
		} else {
			for (int k = 0; k < 3; k++) ax[k] /= nrm;
		}
		P.s_tilted = !(ax[0] == 1.0 && ax[1] == 0.0 && ax[2] == 0.0);
		double ref[3] = { 0.0, 1.0, 0.0 };
		if (std::fabs(ax[1]) > 0.9) {
			ref[1] = 0.0;
			ref[2] = 1.0;
		}
		const double d = ref[0] * ax[0] + ref[1] * ax[1] + ref[2] * ax[2];
		double e1[3];
		for (int k = 0; k < 3; k++) e1[k] = ref[k] - d * ax[k];
		nrm = std::sqrt(e1[0] * e1[0] + e1[1] * e1[1] + e1[2] * e1[2]);
		for (int k = 0; k < 3; k++) e1[k] /= nrm;
		const double e2[3] = { ax[1] * e1[2] - ax[2] * e1[1], ax[2] * e1[0] - ax[0] * e1[2],
		                       ax[0] * e1[1] - ax[1] * e1[0] };
		for (int k = 0; k < 3; k++) {
			P.s_ax[k] = ax[k];
			P.s_e1[k] = e1[k];
			P.s_e2[k] = e2[k];
		}
	}
	const long double m_ion = (long double)P.m_ion, m_e = (long double)MASS_E, m_d = (long double)MASS_DUST;
	// species time-step multiples, pot.c:4157-4159
	P.tss[SP_E] = 1;
	P.tss[SP_ION] = (uint32_t)(int)std::sqrt((double)(r.Te * m_ion / (r.Ti * m_e)));
	P.tss[SP_DUST] = P.tss[SP_ION] * (uint32_t)(int)std::sqrt((double)(0.1 * m_d / m_ion));
	if (P.tss[SP_ION] == 0 || P.tss[SP_DUST] == 0) return POT_E_ARG;
	P.dt = r.dt;
	P.mpp = r.mpp;
	P.rad = r.r * r.mpp;           // pot.c:2032
	P.root_w = 2.0 * r.r * r.mpp;  // pot.c:1476
	P.inv_rad = 1.0 / P.rad;
	P.soft = r.soft;
	P.soft2 = r.soft * r.soft;
	P.a = r.a;
	P.Te = r.Te;
	P.Ti = r.Ti;
	P.x_drift = r.x_drift;
	P.oap2 = r.theta * r.theta;
	P.k4 = 4 * PI_REF * EPSILON0;
	P.Bmag = std::sqrt(r.B[0] * r.B[0] + r.B[1] * r.B[1] + r.B[2] * r.B[2]);
	for (int k = 0; k < 3; k++) P.bhat[k] = P.Bmag != 0.0 ? r.B[k] / P.Bmag : 0.0;
	P.oap2_f = (float)P.oap2;
	P.soft2_f = (float)((r.soft * P.inv_rad) * (r.soft * P.inv_rad));
	// sigma = sqrt(KB T / MASS) with the division in long double, pot.c:675-681
	P.sigma_i = std::sqrt((double)((long double)(KB * r.Ti) / m_ion));
	P.sigma_e = std::sqrt((double)((long double)(KB * r.Te) / m_e));
	// v_n of pot.c:517-524: (2 KB / MASS) rounded to double, times T
	{
		double vi = (double)((long double)(2.0 * KB) / m_ion);
		double ve = (double)((long double)(2.0 * KB) / m_e);
		P.vn_i = std::sqrt(vi * r.Ti);
		P.vn_e = std::sqrt(ve * r.Te);
	}
	// Rol of pot.c:577-579
	{
		double Rol = QE * QE * (r.N - 1) / 2.0;
		Rol /= (4.0 * PI_REF / 3.0) * r.mpp * r.r * EPSILON0 * KB * r.Te;
		P.Rol = std::sqrt(Rol);
	}
	// absorption starts at the first step with t * dt > settle (long double, pot.c:2644)
	{
		const long double dtl = (long double)r.dt, st = (long double)r.settle;
		unsigned long long t0 = 1;
		if (st > 0.0L) {
			const long double g = st / dtl;
			t0 = g > 2.0L ? (unsigned long long)(g - 2.0L) : 1ull;
			if (t0 < 1) t0 = 1;
			while ((long double)t0 * dtl <= st) t0++;
		} else {
			while ((long double)t0 * dtl <= st) t0++;
		}
		P.t_settle = t0;
	}
	// the reference's other compile-time variants (pot.c:99-133, 165-173)
	if (r.flags & ~(POT_CFG_SCEPTIC | POT_CFG_DISABLE_GRAIN | POT_CFG_DIPOLES | POT_CFG_POIS_IONS))
		return POT_E_ARG;
	if (!(r.bounce >= 0.0) || !std::isfinite(r.bounce)) return POT_E_ARG;
	if (r.integrator > POT_INT_EULER_RICHARDSON) return POT_E_ARG;
	// the fast form's dipole cells are evaluated with one target per lane
	if ((r.flags & POT_CFG_DIPOLES) && c->opts.form == POT_FORM_FAST && c->opts.group_size > 32) return POT_E_ARG;
	P.bounce = r.bounce;
	P.integrator = r.integrator;
	for (int k = 0; k < 3; k++) P.B[k] = r.B[k];
	// POIS_POS_COLLECTION's constant rate factor, pot.c:4253-4255, with the
	// density of pot.c:3581-3588; MASS[ION], Run.dt and the density are long
	// double there
	{
		const long double n = (r.N - 1) / ((4.0 / 3.0) * PI_REF * powl((long double)(r.r * r.mpp), 3.0L));
		double k = 4.0 * PI_REF * r.a * r.a * 1;
		k /= std::sqrt((double)(2.0 * PI_REF * m_ion));
		k *= (long double)r.dt * n / 2.0;
		P.pos_rate_const = k;
	}
	return POT_OK;
}

static void tree_ptrs_fast(pot_gpu_ctx* c, bool fast)
{
	if (!fast) {
		c->T.f = nullptr;
		c->T.r2 = nullptr;
		c->T.lf = nullptr;
		c->T.lr2 = nullptr;
	}
}

static int sync_status(pot_gpu_ctx* c)
{
	cudaError_t e = cudaStreamSynchronize(c->stream);
	if (e != cudaSuccess) {
		fprintf(stderr, "pot_gpu: %s\n", cudaGetErrorString(e));
		return POT_E_CUDA;
	}
	c->timer.resolve();
	int st = 0;
	e = cudaMemcpy(&st, &c->rec->status, sizeof(int), cudaMemcpyDeviceToHost);
	if (e != cudaSuccess) return POT_E_CUDA;
	if (st != POT_OK && c->sticky == POT_OK) c->sticky = st;
	return st;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
template <typename T>
static int fetch(std::vector<T>& v, const T* d, size_t n)
{
	v.resize(n);
	if (n == 0) return POT_OK;
	CK(cudaMemcpy(v.data(), d, sizeof(T) * n, cudaMemcpyDeviceToHost));
	return POT_OK;
}

extern "C" {
static void enqueue_step(pot_gpu_ctx* c, uint32_t flags);
}

// ---- internal interface of the batch runtime (pot_batch.cu) --------------
namespace pot {
cudaStream_t ctx_stream(pot_gpu_ctx* c) { return c->stream; }
int ctx_parity(const pot_gpu_ctx* c) { return c->cur; }
RunRec* ctx_rec(pot_gpu_ctx* c) { return c->rec; }
uint64_t ctx_bytes(const pot_gpu_ctx* c) { return c->bytes; }
uint64_t ctx_particles(const pot_gpu_ctx* c) { return c->n; }
int ctx_ready(const pot_gpu_ctx* c) { return !c->uploaded ? POT_E_STATE : c->sticky; }
// Enqueue steps without synchronising (stream capture safe: no host sync,
// no allocation; the timer must be off).
int ctx_enqueue(pot_gpu_ctx* c, uint32_t nsteps)
{
	const int rc = ctx_ready(c);
	if (rc != POT_OK) return rc;
	for (uint32_t k = 0; k < nsteps; k++) enqueue_step(c, 0);
	c->tree_valid = true;
	return POT_OK;
}
void ctx_mark_error(pot_gpu_ctx* c, int rc) { if (c->sticky == POT_OK) c->sticky = rc; }
void ctx_set_tree_valid(pot_gpu_ctx* c) { c->tree_valid = true; }
// The autotuner's candidates on one context: a fast-form context created
// with leaf size 8 (the largest tree capacity of the sizes that key ten
// levels) takes any leaf size of 8 or more and any group size; its step
// graphs are dropped and its particles initialised again.
int ctx_retune(pot_gpu_ctx* c, uint32_t leaf, uint32_t group)
{
	if (c->P.form != POT_FORM_FAST || c->opts.leaf_size != 8 || leaf < 8 || leaf > 64 ||
	    (group != 32 && group != 64) || (c->cfg.flags & POT_CFG_DIPOLES))
		return POT_E_ARG;
	if (c->cfg.N <= (uint64_t)leaf + (c->cfg.A != 0.0 ? 1u : 0u)) return POT_E_ARG;
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	for (auto& row : c->step_exec)
		for (auto& g : row)
			if (g) {
				cudaGraphExecDestroy(g);
				g = nullptr;
			}
	c->graphs_off = false;
	pot_gpu_opts o = c->opts;
	o.leaf_size = leaf;
	o.group_size = group;
	c->opts = o;
	int rc = fill_params(c);
	if (rc != POT_OK) return rc;
	c->opts.leaf_size = 8;  // the allocation's leaf size: the next retune checks it
	c->P.leaf_size = leaf;
	return pot_gpu_init_particles(c);
}
// The packed-batch view of a run (pot_batch.cu); false when the run cannot
// join a packed launch: the plain form, dipoles or a non-Boris integrator
// (their steps have other kernels), or a query-only context.
bool ctx_member_view(pot_gpu_ctx* c, MemberView* v)
{
	if (c->P.form != POT_FORM_FAST || c->P.integrator != POT_INT_BORIS || (c->cfg.flags & POT_CFG_DIPOLES) ||
	    !c->T.mom_pre || !c->src32)
		return false;
	std::memset(v, 0, sizeof(*v));
	v->P = c->P;
	v->T = c->T;
	v->rec = c->rec;
	v->hist = c->hist;
	for (int b = 0; b < 2; b++) {
		v->pos[b] = c->pos[b];
		v->vel[b] = c->vel[b];
		v->pid[b] = c->pid[b];
		v->keys[b] = c->keys[b];
		v->vals[b] = c->vals[b];
	}
	v->src64 = c->src64;
	v->src32 = c->src32;
	v->counts = c->counts;
	v->block_sums = c->block_sums;
	v->due = c->due;
	v->due_tiles = c->due_tiles;
	v->due_list = c->due_list;
	v->due_prefix = c->due_prefix;
	v->groups = c->groups;
	v->rein_list = c->rein_list;
	v->cur = (uint32_t)c->cur;
	v->kb = (uint32_t)(radix_passes((int)c->P.key_bits) & 1);
	v->tiles = radix_tiles(c->n);
	return true;
}
}  // namespace pot

extern "C" {

const char* pot_gpu_strerror(int s)
{
	switch (s) {
	case POT_OK: return "ok";
	case POT_E_ARG: return "invalid argument";
	case POT_E_CUDA: return "CUDA error";
	case POT_E_NOMEM: return "out of device memory";
	case POT_E_DOMAIN: return "particle not in simulation area (tree building failed)";
	case POT_E_COINCIDENT: return "multiple particles at one location";
	case POT_E_WALK: return "particle tree path length exceeded";
	case POT_E_NONFINITE: return "particle has a NaN position";
	case POT_E_ITER: return "sampler iteration cap reached";
	case POT_E_CAPACITY: return "tree larger than its node arrays";
	case POT_E_STATE: return "call out of order";
	case POT_E_LIMIT: return "request larger than the fixed scratch of a non-allocating entry point";
	default: return "unknown status";
	}
}

void pot_gpu_destroy(pot_gpu_ctx* c)
{
	if (!c) return;
	cudaSetDevice(c->device);
	if (c->stream) cudaStreamSynchronize(c->stream);
	for (auto& row : c->step_exec)
		for (auto& g : row)
			if (g) cudaGraphExecDestroy(g);
	if (c->xfer) cudaStreamSynchronize(c->xfer);
	for (auto& e : c->xev)
		if (e) cudaEventDestroy(e);
	if (c->xfer) cudaStreamDestroy(c->xfer);
	if (c->rng_ev) cudaEventDestroy(c->rng_ev);
	if (c->h_rec) cudaFreeHost(c->h_rec);
	if (c->h_hist) cudaFreeHost(c->h_hist);
	if (c->h_due_rng) cudaFreeHost(c->h_due_rng);
	for (void* p : c->allocs) cudaFree(p);
	if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
	delete c;
}

static int create_impl(const pot_run_cfg* cfg, const pot_gpu_opts* opts, pot_gpu_ctx** out, bool dry,
                       uint64_t* bytes);

int pot_gpu_create(const pot_run_cfg* cfg, const pot_gpu_opts* opts, pot_gpu_ctx** out)
{
	return create_impl(cfg, opts, out, false, nullptr);
}

int pot_gpu_bytes_needed(const pot_run_cfg* cfg, const pot_gpu_opts* opts, uint64_t* bytes)
{
	pot_gpu_ctx* c = nullptr;
	if (!bytes) return POT_E_ARG;
	return create_impl(cfg, opts, &c, true, bytes);
}

static int create_impl(const pot_run_cfg* cfg, const pot_gpu_opts* opts, pot_gpu_ctx** out, bool dry,
                       uint64_t* bytes)
{
	if (!cfg || !out) return POT_E_ARG;
	*out = nullptr;
	pot_gpu_opts o {};
	if (opts) o = *opts;
	if (o.form != POT_FORM_PLAIN && o.form != POT_FORM_FAST) return POT_E_ARG;
	if (o.leaf_size == 0) o.leaf_size = o.form == POT_FORM_PLAIN ? 1 : 16;
	if (o.form == POT_FORM_PLAIN && o.leaf_size != 1) return POT_E_ARG;
	if (o.leaf_size > 64) return POT_E_ARG;
	if (o.group_size != 0 && o.group_size != 8 && o.group_size != 16 && o.group_size != 32 && o.group_size != 64)
		return POT_E_ARG;
	// aspect ratio: 0 (sphere), > 1 (prolate) or in (0, 1) (oblate)
	if (!(cfg->A == 0.0 || cfg->A > 1.0 || (cfg->A > 0.0 && cfg->A < 1.0))) return POT_E_ARG;
	// scans cover 2^24; the tree needs more sources than a leaf holds
	if (cfg->N < 2 || cfg->N > (1ull << 24) || cfg->N <= o.leaf_size + (cfg->A != 0.0 ? 1u : 0u)) return POT_E_ARG;
	if (cfg->r == 0 || !(cfg->mpp > 0.0) || !(cfg->dt > 0.0) || !(cfg->a > 0.0) || cfg->soft < 0.0 ||
	    !(cfg->theta > 0.0) || cfg->Te < 0.0 || cfg->Ti <= 0.0)
		return POT_E_ARG;
	if (!dry) {
		int ndev = 0;
		if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return POT_E_CUDA;
		if (o.device < 0 || o.device >= ndev) return POT_E_ARG;
	}
	pot_gpu_ctx* c = new (std::nothrow) pot_gpu_ctx();
	if (!c) return POT_E_NOMEM;
	c->cfg = *cfg;
	c->opts = o;
	c->device = o.device;
	c->dry = dry;
	if (!dry && cudaSetDevice(c->device) != cudaSuccess) {
		delete c;
		return POT_E_CUDA;
	}
	int rc = fill_params(c);
	if (rc) {
		delete c;
		return rc;
	}
	if (dry) {
		// the allocation plan below only counts
	} else if (o.stream) {
		c->stream = (cudaStream_t)o.stream;
	} else {
		if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
			delete c;
			return POT_E_CUDA;
		}
		c->own_stream = true;
	}
	c->timer.enabled = (o.flags & POT_OPT_TIMING) != 0;
	c->timer.stream = c->stream;
	const uint32_t n = (uint32_t)cfg->N;
	c->n = n;
	const bool fast = o.form == POT_FORM_FAST;
	const uint32_t L = o.leaf_size;
	const uint32_t cap = (L == 1 ? 4u * n : (4u * n) / L + 8u * n / 64u) + 4096u;
	const size_t nsum = std::max(scan_blocks(radix_counts_words(n)), scan_blocks(n)) + 16;
#define AL(ptr, count)                         \
	do {                                       \
		if ((rc = dalloc(c, &(ptr), (count)))) { \
			pot_gpu_destroy(c);                \
			return rc;                         \
		}                                      \
	} while (0)
	for (int b = 0; b < 2; b++) {
		AL(c->pos[b], n);
		AL(c->vel[b], n);
		AL(c->pid[b], n);
		AL(c->keys[b], n);
		AL(c->vals[b], n);
	}
	AL(c->src64, n);
	if (fast) AL(c->src32, n);
	AL(c->counts, radix_counts_words(n));
	AL(c->block_sums, nsum);
	AL(c->due, n);
	AL(c->due_tiles, scan_blocks(n) + 1);
	AL(c->due_list, n);
	AL(c->due_prefix, (size_t)n + 1);
	if (fast) AL(c->groups, n);
	if (fast) AL(c->groups_all, n);
	if (fast && n >= ORDERED_GROUPS_MIN_N) {
		AL(c->gcell, cap);
		AL(c->gblk, (size_t)group_blocks() + 1);
	}
	AL(c->epe_partial, 3 * (size_t)(n > (uint32_t)EPE_BLOCKS ? n : (uint32_t)EPE_BLOCKS));
	AL(c->rein_list, 2 * (size_t)n);
	AL(c->macro, macro_scratch_doubles());
	AL(c->inv, n);
	AL(c->rec, 1);
	AL(c->hist, HIST);
	TreeDev& T = c->T;
	T.cap = cap;
	AL(T.lvl8, n);
	AL(T.cnt, n);
	AL(T.base, n);
	AL(T.first, cap);
	AL(T.last, cap);
	AL(T.level, cap);
	AL(T.child, 8ull * cap);
	AL(T.parent, cap);
	AL(T.nint, cap);
	AL(T.ctr, cap);
	AL(T.q, cap);
	AL(T.aq, cap);
	AL(T.cq, cap);
	AL(T.w2, cap);
	if (cfg->flags & POT_CFG_DIPOLES) AL(T.dip, cap);
	if (cfg->integrator != POT_INT_BORIS) {
		AL(c->acc, n);
		AL(c->src64b, n);
		if (fast) AL(c->src32b, n);
	}
	AL(T.ovf, OVF_CAP);
	if (fast) {
		AL(T.f, cap);
		AL(T.r2, cap);
		AL(T.mom_pre, 5 * mom_prefix_entries(n));
		AL(T.mom_blk, 5 * mom_block_entries(n));
		if (cfg->flags & POT_CFG_DIPOLES) {
			AL(T.mom_pre_d, 5 * mom_prefix_entries(n));
			AL(T.mom_blk_d, 5 * mom_block_entries(n));
			AL(T.fd, cap);
			if (L > 1) AL(T.lfd, 8ull * cap);
		}
		if (L > 1) {
			AL(T.lf, 8ull * cap);
			AL(T.lr2, 8ull * cap);
			AL(T.lrange, 8ull * cap);
		}
	}
	if (!fast || L == 1) {
		T.lf = nullptr;
		T.lr2 = nullptr;
		if (!T.lrange) T.lrange = nullptr;
	}
	tree_ptrs_fast(c, fast);
#undef AL
	if (dry) {
		*bytes = c->bytes;
		delete c;
		return POT_OK;
	}
	RunRec r0;
	std::memset(&r0, 0, sizeof(r0));
	r0.grain_m = MASS_DUST;
	r0.grain_slot = 0xFFFFFFFFu;
	r0.ion_temp = cfg->Ti;  // Proc.Ti starts at the injection temperature, pot.c:4252
	if (cudaMemcpy(c->rec, &r0, sizeof(r0), cudaMemcpyHostToDevice) != cudaSuccess) {
		pot_gpu_destroy(c);
		return POT_E_CUDA;
	}
	*out = c;
	return POT_OK;
}

static int set_rec_from_grain(pot_gpu_ctx* c, const pot_grain_state* g, const double4& g_pos, const double4& g_vel)
{
	RunRec r;
	std::memset(&r, 0, sizeof(r));
	if (g) {
		r.grain_q = g->q;
		r.grain_m = g->m;
		r.grain_pos[0] = g->x; r.grain_pos[1] = g->y; r.grain_pos[2] = g->z;
		r.grain_vel[0] = g->vx; r.grain_vel[1] = g->vy; r.grain_vel[2] = g->vz;
		r.tot_absor_e = g->tot_absor_e;
		r.t_steps = g->t_steps;
		r.chi_b = g->chi_b;
	} else {
		r.grain_q = 0;
		r.grain_m = MASS_DUST;
		r.grain_pos[0] = g_pos.x; r.grain_pos[1] = g_pos.y; r.grain_pos[2] = g_pos.z;
		r.grain_vel[0] = g_vel.x; r.grain_vel[1] = g_vel.y; r.grain_vel[2] = g_vel.z;
	}
	r.grain_slot = 0xFFFFFFFFu;
	// the record up to the per-step variant counters: the cached ion
	// temperature after them survives uploads
	CK(cudaMemcpyAsync(c->rec, &r, offsetof(RunRec, n_collected), cudaMemcpyHostToDevice, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	c->sticky = POT_OK;
	return POT_OK;
}

int pot_gpu_upload(pot_gpu_ctx* c, const pot_particle* parts, uint64_t N, const pot_grain_state* grain)
{
	if (!c || !parts || N != c->cfg.N) return POT_E_ARG;
	if (parts[0].species != SP_DUST) return POT_E_ARG;
	CK(cudaSetDevice(c->device));
	if (!c->aos) {
		const int ra = dalloc(c, &c->aos, c->n);
		if (ra) return ra;
	}
	CK(cudaMemcpyAsync(c->aos, parts, sizeof(pot_particle) * c->n, cudaMemcpyHostToDevice, c->stream));
	c->cur = 0;
	// the record first, so a bad species found by the conversion is kept
	const double4 gp = make_double4(parts[0].x, parts[0].y, parts[0].z, 0.0);
	const double4 gv = make_double4(parts[0].vx, parts[0].vy, parts[0].vz, 0.0);
	int rc = set_rec_from_grain(c, grain, gp, gv);
	if (rc) return rc;
	k_from_aos<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->aos, c->n, c->pos[0], c->vel[0], c->pid[0], c->rec);
	CK(cudaGetLastError());
	c->uploaded = true;
	c->tree_valid = false;
	return POT_OK;
}

int pot_gpu_init_particles(pot_gpu_ctx* c)
{
	if (!c) return POT_E_ARG;
	CK(cudaSetDevice(c->device));
	RunRec r;
	std::memset(&r, 0, sizeof(r));
	r.grain_m = MASS_DUST;
	r.grain_pos[0] = r.grain_pos[1] = r.grain_pos[2] = c->P.rad;
	r.grain_slot = 0xFFFFFFFFu;
	CK(cudaMemcpyAsync(c->rec, &r, offsetof(RunRec, n_collected), cudaMemcpyHostToDevice, c->stream));
	c->cur = 0;
	launch_init(c->pos[0], c->vel[0], c->pid[0], c->P, c->rec, c->stream, c->timer);
	CK(cudaGetLastError());
	c->sticky = POT_OK;
	int st = sync_status(c);
	if (st != POT_OK) return st;
	c->uploaded = true;
	c->tree_valid = false;
	return POT_OK;
}

// Keys, sort, reorder (+ due flags) and tree for the current state.
static void enqueue_tree(pot_gpu_ctx* c, int begin_step)
{
	Params& P = c->P;
	cudaStream_t s = c->stream;
	uint32_t* hist = radix_sort_begin(c->counts, c->n, (int)P.key_bits, s);
	launch_keys(c->pos[c->cur], c->keys[0], c->vals[0], P, c->rec, begin_step, hist, s, c->timer);
	const int kb = radix_sort_pairs(c->keys, c->vals, c->n, c->counts, c->block_sums, (int)P.key_bits, s, c->timer,
	                                &c->rec->status);
	c->kb = kb;
	const int nx = c->cur ^ 1;
	cudaMemsetAsync(c->due_tiles, 0, sizeof(uint32_t) * scan_blocks(c->n), s);
	launch_reorder(c->vals[kb], c->pos[c->cur], c->vel[c->cur], c->pid[c->cur], c->pos[nx], c->vel[nx], c->pid[nx],
	               c->src64, c->src32, c->due, P, c->rec, c->due_tiles, s, c->timer);
	c->cur = nx;
	launch_build(c->keys[kb], c->T, c->src64, P, c->rec, c->block_sums, s, c->timer);
}

static void enqueue_step(pot_gpu_ctx* c, uint32_t flags)
{
	const int epe = (flags & POT_STEP_EPE) ? 1 : 0;
	Params& P = c->P;
	cudaStream_t s = c->stream;
	enqueue_tree(c, 1);
	compact_flags(c->due, c->n, c->due_list, c->due_tiles, &c->rec->n_due, s, c->timer, c->due_prefix, true);
	if (P.form == POT_FORM_FAST)
		launch_groups(c->T, c->due_prefix, c->groups, c->gcell, c->gblk, P, c->rec, s, c->timer);
	launch_chi_b(c->T, c->src64, P, c->rec, 0, s, c->timer);
	if (P.integrator == POT_INT_BORIS) {
		launch_push(c->pos[c->cur], c->vel[c->cur], c->T, c->src64, c->src32, c->due_list, c->groups, c->rein_list,
		            P, c->rec, StageBufs { 0, nullptr, nullptr, nullptr }, s, c->timer);
	} else {
		// two field evaluations (pot.c:2533-2639): the second sees every
		// particle that moved at its intermediate position
		StageBufs sb { 1, c->acc, c->src64b, c->src32b };
		cudaMemcpyAsync(c->src64b, c->src64, sizeof(double4) * c->n, cudaMemcpyDeviceToDevice, s);
		if (c->src32b) cudaMemcpyAsync(c->src32b, c->src32, sizeof(float4) * c->n, cudaMemcpyDeviceToDevice, s);
		launch_push(c->pos[c->cur], c->vel[c->cur], c->T, c->src64, c->src32, c->due_list, c->groups, c->rein_list,
		            P, c->rec, sb, s, c->timer);
		cudaMemsetAsync(&c->rec->work_ctr, 0, sizeof(unsigned int), s);
		sb.stage = 2;
		launch_push(c->pos[c->cur], c->vel[c->cur], c->T, c->src64, c->src32, c->due_list, c->groups, c->rein_list,
		            P, c->rec, sb, s, c->timer);
	}
	launch_absorb_late(c->pos[c->cur], c->vel[c->cur], c->src64, c->due_list, c->rein_list, P, c->rec, s, c->timer);
	if (epe) {
		// with two field evaluations the energies are those of the
		// intermediate state, whose sources the second evaluation used
		const bool two = P.integrator != POT_INT_BORIS;
		launch_epe(c->pos[c->cur], c->T, two ? c->src64b : c->src64, two ? c->src32b : c->src32, c->groups_all,
		           c->epe_partial, P, c->rec, s, c->timer);
	}
	launch_reinject(c->pos[c->cur], c->vel[c->cur], c->pid[c->cur], c->rein_list, c->src64, P, c->rec, s, c->timer);
	launch_grain_end(c->pos[c->cur], c->vel[c->cur], c->hist, P, c->rec, epe, s, c->timer);
}


// One step: replay of the step's CUDA graph for the current parity (the
// step's ~25 launches become one), captured the first time; kernel by kernel
// when timing events are on, when the caller's stream is itself being
// captured, or after a failed capture.
static int step_once(pot_gpu_ctx* c, uint32_t flags)
{
	cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
	if (c->graphs_off || c->timer.enabled || cudaStreamIsCapturing(c->stream, &cs) != cudaSuccess ||
	    cs != cudaStreamCaptureStatusNone) {
		enqueue_step(c, flags);
		return POT_OK;
	}
	const int e = (flags & POT_STEP_EPE) ? 1 : 0;
	const int p = c->cur;
	if (!c->step_exec[p][e]) {
		const uint64_t l0 = c->timer.launches;
		cudaGraph_t g = nullptr;
		if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
			c->graphs_off = true;
			enqueue_step(c, flags);
			return POT_OK;
		}
		enqueue_step(c, flags);  // records the launches; flips c->cur
		const cudaError_t ec = cudaStreamEndCapture(c->stream, &g);
		const uint64_t per_step = c->timer.launches - l0;
		c->cur = p;
		c->timer.launches = l0;
		cudaGraphExec_t x = nullptr;
		if (ec == cudaSuccess && g && cudaGraphInstantiate(&x, g, 0) == cudaSuccess) {
			c->step_exec[p][e] = x;
		}
		if (g) cudaGraphDestroy(g);
		if (!c->step_exec[p][e]) {
			cudaGetLastError();
			c->graphs_off = true;
			enqueue_step(c, flags);
			return POT_OK;
		}
		c->step_launches[p][e] = per_step;
	}
	CK(cudaGraphLaunch(c->step_exec[p][e], c->stream));
	c->timer.launches += c->step_launches[p][e];
	c->cur = p ^ 1;
	return POT_OK;
}

int pot_gpu_step(pot_gpu_ctx* c, uint32_t nsteps, uint32_t flags, pot_step_stats* out)
{
	if (!c) return POT_E_ARG;
	if (flags & ~POT_STEP_EPE) return POT_E_ARG;
	if (!c->uploaded) return POT_E_STATE;
	if (c->sticky != POT_OK) return c->sticky;
	CK(cudaSetDevice(c->device));
	for (uint32_t k = 0; k < nsteps; k++) {
		const int rc = step_once(c, flags);
		if (rc != POT_OK) return rc;
	}
	CK(cudaGetLastError());
	c->tree_valid = true;
	const int st = sync_status(c);
	if (out) {
		RunRec r;
		CK(cudaMemcpy(&r, c->rec, sizeof(r), cudaMemcpyDeviceToHost));
		StepHist h;
		CK(cudaMemcpy(&h, &c->hist[r.t_steps % HIST], sizeof(h), cudaMemcpyDeviceToHost));
		std::memset(out, 0, sizeof(*out));
		out->t_steps = r.t_steps;
		out->grain_q = r.grain_q;
		out->dq = h.dq;
		out->de = h.de;
		out->n_absorbed = h.n_absorbed;
		out->n_reinjected = h.n_reinjected;
		out->n_pushed = h.n_pushed;
		out->interactions = h.interactions;
		out->far_cells = h.far_cells;
		out->n_nodes = h.n_nodes;
		out->chi_b = r.chi_b;
		out->status = r.status;
		out->stack_max = r.stack_max;
		for (int k = 0; k < 3; k++) out->epe[k] = h.epe[k];
		out->q_sum = r.q_sum;
		out->warn = r.warn;
		out->n_collected = r.n_collected;
		out->n_wall = r.n_wall;
		out->n_bounced = r.n_bounced;
		out->n_groups = c->P.form == POT_FORM_FAST ? r.n_groups : 0u;
	}
	return st;
}

int pot_gpu_step_async(pot_gpu_ctx* c, uint32_t nsteps, uint32_t flags)
{
	if (!c) return POT_E_ARG;
	if (flags & ~POT_STEP_EPE) return POT_E_ARG;
	if (!c->uploaded) return POT_E_STATE;
	if (c->sticky != POT_OK) return c->sticky;
	CK(cudaSetDevice(c->device));
	for (uint32_t k = 0; k < nsteps; k++) {
		const int rc = step_once(c, flags);
		if (rc != POT_OK) return rc;
	}
	CK(cudaGetLastError());
	c->tree_valid = true;
	return POT_OK;
}

int pot_gpu_download(pot_gpu_ctx* c, pot_particle* parts, pot_grain_state* grain)
{
	if (!c) return POT_E_ARG;
	if (!c->uploaded) return POT_E_STATE;
	CK(cudaSetDevice(c->device));
	if (parts) {
		if (!c->aos) {
			const int ra = dalloc(c, &c->aos, c->n);
			if (ra) return ra;
		}
		k_to_aos<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->pos[c->cur], c->vel[c->cur], c->pid[c->cur], c->n,
		                                                   c->aos);
		CK(cudaGetLastError());
		CK(cudaMemcpyAsync(parts, c->aos, sizeof(pot_particle) * c->n, cudaMemcpyDeviceToHost, c->stream));
	}
	RunRec r;
	CK(cudaMemcpyAsync(&r, c->rec, sizeof(r), cudaMemcpyDeviceToHost, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	if (grain) {
		grain->q = r.grain_q;
		grain->m = r.grain_m;
		grain->x = r.grain_pos[0]; grain->y = r.grain_pos[1]; grain->z = r.grain_pos[2];
		grain->vx = r.grain_vel[0]; grain->vy = r.grain_vel[1]; grain->vz = r.grain_vel[2];
		grain->tot_absor_e = r.tot_absor_e;
		grain->t_steps = r.t_steps;
		grain->chi_b = r.chi_b;
	}
	return r.status;
}

// The drop-in call as one pipeline: the upload in chunks on a copy stream,
// each chunk converted as soon as it has arrived; the step; the download of
// the records the step can have changed (the grain's and the range of the
// particles due), gathered in chunks in reference order, each chunk copied
// back while the next is gathered; the run record and step history copied
// with it.  The host waits twice: for the upload (to learn the due range,
// while the step runs) and at the end.  Same results as pot_gpu_upload,
// pot_gpu_step and pot_gpu_download in turn.
constexpr int XFER_CHUNKS = 4;

static int xfer_setup(pot_gpu_ctx* c)
{
	if (c->xfer) return POT_OK;
	CK(cudaStreamCreateWithFlags(&c->xfer, cudaStreamNonBlocking));
	for (auto& e : c->xev) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
	CK(cudaEventCreateWithFlags(&c->rng_ev, cudaEventDisableTiming));
	CK(cudaMallocHost((void**)&c->h_rec, sizeof(RunRec)));
	CK(cudaMallocHost((void**)&c->h_hist, sizeof(StepHist) * HIST));
	CK(cudaMallocHost((void**)&c->h_due_rng, 2 * sizeof(uint32_t)));
	const int ra = dalloc(c, &c->due_rng, 2);
	if (ra) return ra;
	return POT_OK;
}

// The drop-in call's first half: the run record, the upload in chunks on the
// copy stream with each chunk converted on the context's stream as soon as
// it has landed (recording the reference-index range of the particles due
// this step), that range copied to pinned memory behind rng_ev, and the
// step.  The caller waits for both streams whatever this returns, so no copy
// outlives the call.
static int move_enqueue_in(pot_gpu_ctx* c, pot_particle* parts, const pot_grain_state* grain)
{
	int rc = POT_OK;
	const uint32_t n = c->n;
	const int K = n >= 4u * 65536u ? XFER_CHUNKS : 1;
	// the run record first (as set_rec_from_grain writes it, from pinned
	// memory), so a bad species found by the conversion below is not overwritten
	unsigned long long t_prev = 0;
	{
		RunRec& r = *c->h_rec;
		std::memset(&r, 0, sizeof(r));
		if (grain) {
			r.grain_q = grain->q;
			r.grain_m = grain->m;
			r.grain_pos[0] = grain->x; r.grain_pos[1] = grain->y; r.grain_pos[2] = grain->z;
			r.grain_vel[0] = grain->vx; r.grain_vel[1] = grain->vy; r.grain_vel[2] = grain->vz;
			r.tot_absor_e = grain->tot_absor_e;
			r.t_steps = grain->t_steps;
			r.chi_b = grain->chi_b;
		} else {
			r.grain_m = MASS_DUST;
			r.grain_pos[0] = parts[0].x; r.grain_pos[1] = parts[0].y; r.grain_pos[2] = parts[0].z;
			r.grain_vel[0] = parts[0].vx; r.grain_vel[1] = parts[0].vy; r.grain_vel[2] = parts[0].vz;
		}
		r.grain_slot = 0xFFFFFFFFu;
		t_prev = r.t_steps;
		CK(cudaMemcpyAsync(c->rec, &r, offsetof(RunRec, n_collected), cudaMemcpyHostToDevice, c->stream));
	}
	// due range: lo starts at ~0 (every byte 0xFF), hi at 0
	CK(cudaMemsetAsync(&c->due_rng[0], 0xFF, sizeof(uint32_t), c->stream));
	CK(cudaMemsetAsync(&c->due_rng[1], 0, sizeof(uint32_t), c->stream));
	const uint3 tss = make_uint3(c->P.tss[SP_DUST], c->P.tss[SP_ION], c->P.tss[SP_E]);
	// upload: chunk k lands on the copy stream, then is converted on the
	// context's stream (after whatever that stream already holds)
	c->cur = 0;
	CK(cudaEventRecord(c->xev[2 * XFER_CHUNKS], c->stream));  // the copies follow the stream's earlier work
	CK(cudaStreamWaitEvent(c->xfer, c->xev[2 * XFER_CHUNKS], 0));
	for (int k = 0; k < K; k++) {
		const uint32_t i0 = (uint32_t)((uint64_t)n * k / K), i1 = (uint32_t)((uint64_t)n * (k + 1) / K);
		CK(cudaMemcpyAsync(c->aos + i0, parts + i0, sizeof(pot_particle) * (i1 - i0), cudaMemcpyHostToDevice,
		                   c->xfer));
		CK(cudaEventRecord(c->xev[k], c->xfer));
		CK(cudaStreamWaitEvent(c->stream, c->xev[k], 0));
		k_from_aos_range_due<<<nblk(i1 - i0, 256), 256, 0, c->stream>>>(c->aos, i0, i1 - i0, c->pos[0], c->vel[0],
		                                                                  c->pid[0], c->rec, t_prev + 1ull, tss,
		                                                                  c->due_rng);
	}
	CK(cudaMemcpyAsync(c->h_due_rng, c->due_rng, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, c->stream));
	CK(cudaEventRecord(c->rng_ev, c->stream));
	c->sticky = POT_OK;  // as pot_gpu_upload: a new state clears the run's status
	c->uploaded = true;
	c->tree_valid = false;
	// the step
	rc = step_once(c, 0);
	if (rc != POT_OK) return rc;
	c->tree_valid = true;
	CK(cudaGetLastError());
	return POT_OK;
}

// The second half, once the host has the due range [lo, hi]: only those
// records and the grain's (index 0) can have changed in the step (a particle
// not due is neither pushed nor reinjected), so only they are gathered in
// reference order and copied back, in chunks, each copied while the next is
// gathered; the caller's other records already hold the same values.  Then
// the run record and step history.
static int move_enqueue_out(pot_gpu_ctx* c, pot_particle* parts, uint32_t lo, uint32_t hi, bool want_hist)
{
	const uint32_t n = c->n;
	k_inverse<<<nblk(n, 256), 256, 0, c->stream>>>(c->pid[c->cur], n, c->inv);
	if (lo > 0 || hi < lo) {  // the grain's record on its own
		k_to_aos_gather<<<1, 32, 0, c->stream>>>(c->pos[c->cur], c->vel[c->cur], c->inv, 0u, 1u, c->aos);
		CK(cudaEventRecord(c->xev[2 * XFER_CHUNKS], c->stream));
		CK(cudaStreamWaitEvent(c->xfer, c->xev[2 * XFER_CHUNKS], 0));
		CK(cudaMemcpyAsync(parts, c->aos, sizeof(pot_particle), cudaMemcpyDeviceToHost, c->xfer));
	}
	if (hi >= lo && hi < n) {
		const uint32_t m = hi - lo + 1u;
		const int K = m >= 4u * 65536u ? XFER_CHUNKS : 1;
		for (int k = 0; k < K; k++) {
			const uint32_t i0 = lo + (uint32_t)((uint64_t)m * k / K), i1 = lo + (uint32_t)((uint64_t)m * (k + 1) / K);
			k_to_aos_gather<<<nblk(i1 - i0, 256), 256, 0, c->stream>>>(c->pos[c->cur], c->vel[c->cur], c->inv, i0,
			                                                             i1 - i0, c->aos);
			CK(cudaEventRecord(c->xev[XFER_CHUNKS + k], c->stream));
			CK(cudaStreamWaitEvent(c->xfer, c->xev[XFER_CHUNKS + k], 0));
			CK(cudaMemcpyAsync(parts + i0, c->aos + i0, sizeof(pot_particle) * (i1 - i0), cudaMemcpyDeviceToHost,
			                   c->xfer));
		}
	}
	CK(cudaMemcpyAsync(c->h_rec, c->rec, sizeof(RunRec), cudaMemcpyDeviceToHost, c->stream));
	if (want_hist) CK(cudaMemcpyAsync(c->h_hist, c->hist, sizeof(StepHist) * HIST, cudaMemcpyDeviceToHost, c->stream));
	CK(cudaGetLastError());
	return POT_OK;
}

int pot_gpu_move_particles(pot_gpu_ctx* c, pot_particle* parts, uint64_t N, pot_grain_state* grain,
                           pot_step_stats* out)
{
	if (!c || !parts || N != c->cfg.N) return POT_E_ARG;
	if (parts[0].species != SP_DUST) return POT_E_ARG;
	CK(cudaSetDevice(c->device));
	if (!c->aos) {
		const int ra = dalloc(c, &c->aos, c->n);
		if (ra) return ra;
	}
	int rc = xfer_setup(c);
	if (rc) return rc;
	rc = move_enqueue_in(c, parts, grain);
	if (rc == POT_OK) {
		// the host waits for the upload and the due range only; the step is
		// already queued behind them, so the GPU does not wait for the host
		if (cudaEventSynchronize(c->rng_ev) != cudaSuccess) {
			rc = POT_E_CUDA;
		} else {
			rc = move_enqueue_out(c, parts, c->h_due_rng[0], c->h_due_rng[1], out != nullptr);
		}
	}
	const cudaError_t e1 = cudaStreamSynchronize(c->xfer);
	const cudaError_t e2 = cudaStreamSynchronize(c->stream);
	if (rc != POT_OK) return rc;
	if (e1 != cudaSuccess || e2 != cudaSuccess) return POT_E_CUDA;
	c->timer.resolve();
	const RunRec& r = *c->h_rec;
	if (r.status != POT_OK && c->sticky == POT_OK) c->sticky = r.status;
	if (out) {
		const StepHist& h = c->h_hist[r.t_steps % HIST];
		std::memset(out, 0, sizeof(*out));
		out->t_steps = r.t_steps;
		out->grain_q = r.grain_q;
		out->dq = h.dq;
		out->de = h.de;
		out->n_absorbed = h.n_absorbed;
		out->n_reinjected = h.n_reinjected;
		out->n_pushed = h.n_pushed;
		out->interactions = h.interactions;
		out->far_cells = h.far_cells;
		out->n_nodes = h.n_nodes;
		out->chi_b = r.chi_b;
		out->status = r.status;
		out->stack_max = r.stack_max;
		for (int k = 0; k < 3; k++) out->epe[k] = h.epe[k];
		out->q_sum = r.q_sum;
		out->warn = r.warn;
		out->n_collected = r.n_collected;
		out->n_wall = r.n_wall;
		out->n_bounced = r.n_bounced;
		out->n_groups = c->P.form == POT_FORM_FAST ? r.n_groups : 0u;
	}
	if (r.status != POT_OK) return r.status;
	if (grain) {
		grain->q = r.grain_q;
		grain->m = r.grain_m;
		grain->x = r.grain_pos[0]; grain->y = r.grain_pos[1]; grain->z = r.grain_pos[2];
		grain->vx = r.grain_vel[0]; grain->vy = r.grain_vel[1]; grain->vz = r.grain_vel[2];
		grain->tot_absor_e = r.tot_absor_e;
		grain->t_steps = r.t_steps;
		grain->chi_b = r.chi_b;
	}
	return POT_OK;
}

int pot_gpu_build_tree(pot_gpu_ctx* c, uint64_t* n_nodes)
{
	if (!c) return POT_E_ARG;
	if (!c->uploaded) return POT_E_STATE;
	CK(cudaSetDevice(c->device));
	enqueue_tree(c, 0);
	CK(cudaGetLastError());
	const int st = sync_status(c);
	if (n_nodes) {
		unsigned int m = 0;
		CK(cudaMemcpy(&m, &c->rec->n_nodes, sizeof(m), cudaMemcpyDeviceToHost));
		*n_nodes = m;
	}
	c->tree_valid = st == POT_OK;
	return st;
}

int pot_gpu_tree_dump(pot_gpu_ctx* c, uint64_t max_nodes, uint64_t* n_int, int32_t* int_level, uint64_t* int_path,
                      int32_t* int_q, uint32_t* int_aq, double* int_c, double* int_w, uint64_t* n_leaf,
                      uint32_t* leaf_part, int32_t* leaf_level, uint64_t* leaf_path)
{
	if (!c || !n_int || !n_leaf) return POT_E_ARG;
	if (!c->tree_valid) return POT_E_STATE;
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	unsigned int M = 0;
	CK(cudaMemcpy(&M, &c->rec->n_nodes, sizeof(M), cudaMemcpyDeviceToHost));
	std::vector<uint64_t> keys;
	std::vector<uint32_t> first, pid;
	std::vector<uint8_t> level;
	std::vector<int32_t> child, q;
	std::vector<uint32_t> aq;
	std::vector<double4> cq;
	std::vector<double> w2;
	std::vector<uint2> lrange;
	int rc;
	if ((rc = fetch(keys, c->keys[c->kb], c->n)) || (rc = fetch(first, c->T.first, M)) ||
	    (rc = fetch(pid, c->pid[c->cur], c->n)) || (rc = fetch(level, c->T.level, M)) ||
	    (rc = fetch(child, c->T.child, 8ull * M)) || (rc = fetch(q, c->T.q, M)) || (rc = fetch(aq, c->T.aq, M)) ||
	    (rc = fetch(cq, c->T.cq, M)) || (rc = fetch(w2, c->T.w2, M)))
		return rc;
	if (c->P.leaf_size > 1 && (rc = fetch(lrange, c->T.lrange, 8ull * M))) return rc;
	std::vector<uint2> ovf;
	if (c->P.leaf_size == 1 && (rc = fetch(ovf, c->T.ovf, (size_t)OVF_CAP))) return rc;
	uint64_t ni = 0, nl = 0;
	for (uint32_t k = 0; k < M; k++) {
		const int l = level[k];
		const uint64_t pfx = l == 0 ? 0ull : keys[first[k]] >> (63 - 3 * l);
		if (ni >= max_nodes) return POT_E_ARG;
		if (int_level) int_level[ni] = l;
		if (int_path) int_path[ni] = pfx;
		if (int_q) int_q[ni] = q[k];
		if (int_aq) int_aq[ni] = aq[k];
		if (int_c) {
			int_c[3 * ni] = cq[k].x;
			int_c[3 * ni + 1] = cq[k].y;
			int_c[3 * ni + 2] = cq[k].z;
		}
		if (int_w) int_w[ni] = std::sqrt(w2[k]);
		ni++;
		for (int d = 0; d < 8; d++) {
			const int32_t code = child[8ull * k + d];
			if (code >= CH_EMPTY) continue;
			const uint32_t e = leaf_payload(code);
			uint32_t s0 = e, cnt = 1;
			if (c->P.leaf_size > 1) {
				s0 = lrange[e].x;
				cnt = lrange[e].y;
			} else if (e >= c->P.n_tree) {
				s0 = ovf[e - c->P.n_tree].x;
				cnt = ovf[e - c->P.n_tree].y;
			}
			for (uint32_t j = 0; j < cnt; j++) {
				if (nl >= max_nodes) return POT_E_ARG;
				if (leaf_part) leaf_part[nl] = pid[s0 + j];
				if (leaf_level) leaf_level[nl] = l + 1;
				if (leaf_path) leaf_path[nl] = (pfx << 3) | (uint64_t)d;
				nl++;
			}
		}
	}
	*n_int = ni;
	*n_leaf = nl;
	return POT_OK;
}

static int ensure_query(pot_gpu_ctx* c, size_t n)
{
	if (n <= c->q_cap) return POT_OK;
	for (void* p : { (void*)c->q_xyz, (void*)c->q_out, (void*)c->q_idx, (void*)c->q_slot }) {
		if (!p) continue;
		for (auto& a : c->allocs)
			if (a == p) a = nullptr;
		cudaFree(p);
	}
	int rc;
	if ((rc = dalloc(c, &c->q_xyz, 3 * n)) || (rc = dalloc(c, &c->q_out, 3 * n)) || (rc = dalloc(c, &c->q_idx, n)) ||
	    (rc = dalloc(c, &c->q_slot, n)))
		return rc;
	c->q_cap = n;
	return POT_OK;
}

int pot_gpu_field_at(pot_gpu_ctx* c, uint64_t n, const uint32_t* idx, const double* xyz, double* E)
{
	if (!c || !idx || !xyz || !E) return POT_E_ARG;
	if (!c->tree_valid) return POT_E_STATE;
	if (n == 0) return POT_OK;
	CK(cudaSetDevice(c->device));
	int rc = ensure_query(c, n);
	if (rc) return rc;
	CK(cudaMemcpyAsync(c->q_xyz, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
	CK(cudaMemcpyAsync(c->q_idx, idx, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, c->stream));
	k_inverse<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->pid[c->cur], c->n, c->inv);
	k_map_slots<<<nblk(n, 256), 256, 0, c->stream>>>(c->inv, c->q_idx, (uint32_t)n, c->n, c->q_slot);
	launch_field_query(c->T, c->src64, c->src32, c->q_xyz, c->q_slot, (uint32_t)n, c->q_out, c->P, c->rec,
	                   c->stream, c->timer);
	CK(cudaGetLastError());
	CK(cudaMemcpyAsync(E, c->q_out, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->stream));
	return sync_status(c);
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Field query without allocation.
//
// pot_gpu_field_at stages its points, target slots and results in device
// buffers that it allocates on first use (and grows).  Callers that may not
// allocate device memory while they run -- a host program that owns the
// device heap through its own pool, a step loop that must not call
// cudaMalloc between its iterations -- use pot_gpu_field_at_noalloc, which
// stages everything in this fixed array instead: at most
// POT_NOALLOC_MAX_POINTS points per call, about 3.5 MiB held on every device
// that loads the library until the process exits.  Every call on a device
// shares the array and overwrites all of it that it reads (nothing needs to
// start at zero); calls whose work overlaps on the GPU, from any context on
// that device, race on it.
// ---------------------------------------------------------------------------
struct NoAllocScratch {
	double xyz[3 * POT_NOALLOC_MAX_POINTS];
	double E[3 * POT_NOALLOC_MAX_POINTS];
	uint32_t idx[POT_NOALLOC_MAX_POINTS];
	uint32_t slot[POT_NOALLOC_MAX_POINTS];
};
static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

// Device address of g_noalloc_scratch on `device` (the current device),
// looked up once per device and kept for the life of the process: valid
// while that device's primary context lives (cudaDeviceReset would leave it
// stale).  In host code the symbol names a host-side stand-in, never device
// memory, so kernels only ever get this address.
static int noalloc_scratch(int device, NoAllocScratch** out)
{
	static std::mutex mu;
	static void* addr[256] = { nullptr };
	if (device < 0 || device >= 256) return POT_E_ARG;
	std::lock_guard<std::mutex> lock(mu);
	if (!addr[device]) {
		void* p = nullptr;
		const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
		if (e != cudaSuccess || !p) {
			fprintf(stderr, "pot_gpu: cudaGetSymbolAddress: %s\n", cudaGetErrorString(e));
			return POT_E_CUDA;
		}
		addr[device] = p;
	}
	*out = static_cast<NoAllocScratch*>(addr[device]);
	return POT_OK;
}

extern "C" {

int pot_gpu_field_at_noalloc(pot_gpu_ctx* c, uint64_t n, const uint32_t* idx, const double* xyz, double* E)
{
	if (!c || !idx || !xyz || !E) return POT_E_ARG;
	if (n > POT_NOALLOC_MAX_POINTS) {
		fprintf(stderr, "pot_gpu_field_at_noalloc: %llu points requested, at most %u per call\n",
		        (unsigned long long)n, (unsigned)POT_NOALLOC_MAX_POINTS);
		return POT_E_LIMIT;
	}
	if (!c->tree_valid) return POT_E_STATE;
	if (n == 0) return POT_OK;
	CK(cudaSetDevice(c->device));
	NoAllocScratch* sc = nullptr;
	int rc = noalloc_scratch(c->device, &sc);
	if (rc) return rc;
	CK(cudaMemcpyAsync(sc->xyz, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
	CK(cudaMemcpyAsync(sc->idx, idx, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, c->stream));
	k_inverse<<<nblk(c->n, 256), 256, 0, c->stream>>>(c->pid[c->cur], c->n, c->inv);
	k_map_slots<<<nblk(n, 256), 256, 0, c->stream>>>(c->inv, sc->idx, (uint32_t)n, c->n, sc->slot);
	launch_field_query(c->T, c->src64, c->src32, sc->xyz, sc->slot, (uint32_t)n, sc->E, c->P, c->rec, c->stream,
	                   c->timer);
	CK(cudaGetLastError());
	CK(cudaMemcpyAsync(E, sc->E, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c->stream));
	return sync_status(c);
}

int pot_gpu_phi_at(pot_gpu_ctx* c, uint64_t n, const double* xyz, double* phi)
{
	if (!c || !xyz || !phi) return POT_E_ARG;
	if (!c->tree_valid) return POT_E_STATE;
	if (n == 0) return POT_OK;
	CK(cudaSetDevice(c->device));
	int rc = ensure_query(c, n);
	if (rc) return rc;
	CK(cudaMemcpyAsync(c->q_xyz, xyz, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c->stream));
	launch_phi_query(c->T, c->src64, c->q_xyz, (uint32_t)n, c->q_out, c->P, c->rec, c->stream, c->timer);
	CK(cudaGetLastError());
	CK(cudaMemcpyAsync(phi, c->q_out, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
	return sync_status(c);
}

int pot_gpu_macro(pot_gpu_ctx* c, pot_macro_sums* out)
{
	static_assert(sizeof(pot_macro_sums) == 38 * sizeof(double), "two passes of 20 and 18 sums");
	if (!c || !out) return POT_E_ARG;
	if (!c->uploaded) return POT_E_STATE;
	CK(cudaSetDevice(c->device));
	launch_macro(c->pos[c->cur], c->vel[c->cur], c->P, c->macro, c->rec, c->stream, c->timer);
	CK(cudaGetLastError());
	CK(cudaMemcpyAsync(out, c->macro + (macro_scratch_doubles() - 80), sizeof(pot_macro_sums),
	                   cudaMemcpyDeviceToHost, c->stream));
	return sync_status(c);
}

int pot_gpu_grain(pot_gpu_ctx* c, pot_grain_state* g)
{
	if (!c || !g) return POT_E_ARG;
	if (!c->uploaded) return POT_E_STATE;
	CK(cudaSetDevice(c->device));
	const int st = sync_status(c);
	RunRec r;
	CK(cudaMemcpy(&r, c->rec, sizeof(r), cudaMemcpyDeviceToHost));
	std::memset(g, 0, sizeof(*g));
	g->q = r.grain_q;
	g->m = r.grain_m;
	g->x = r.grain_pos[0]; g->y = r.grain_pos[1]; g->z = r.grain_pos[2];
	g->vx = r.grain_vel[0]; g->vy = r.grain_vel[1]; g->vz = r.grain_vel[2];
	g->tot_absor_e = r.tot_absor_e;
	g->t_steps = r.t_steps;
	g->chi_b = r.chi_b;
	return st;
}

int pot_gpu_set_ion_temp(pot_gpu_ctx* c, double Ti)
{
	if (!c || !(Ti >= 0.0) || !std::isfinite(Ti)) return POT_E_ARG;
	CK(cudaSetDevice(c->device));
	CK(cudaMemcpyAsync(&c->rec->ion_temp, &Ti, sizeof(double), cudaMemcpyHostToDevice, c->stream));
	CK(cudaStreamSynchronize(c->stream));
	return POT_OK;
}

int pot_gpu_ion_temp(pot_gpu_ctx* c, double* Ti)
{
	if (!c || !Ti) return POT_E_ARG;
	CK(cudaSetDevice(c->device));
	CK(cudaStreamSynchronize(c->stream));
	CK(cudaMemcpy(Ti, &c->rec->ion_temp, sizeof(double), cudaMemcpyDeviceToHost));
	return POT_OK;
}

int pot_gpu_kernel_times(pot_gpu_ctx* c, int max, const char** names, double* ms, uint64_t* launches)
{
	if (!c) return POT_E_ARG;
	c->timer.resolve();
	return c->timer.report(max, names, ms, launches);
}

int pot_gpu_reset_kernel_times(pot_gpu_ctx* c)
{
	if (!c) return POT_E_ARG;
	CK(cudaStreamSynchronize(c->stream));
	c->timer.reset();
	return POT_OK;
}

int pot_gpu_launch_count(pot_gpu_ctx* c, uint64_t* n)
{
	if (!c || !n) return POT_E_ARG;
	*n = c->timer.launches;
	return POT_OK;
}

int pot_gpu_sync(pot_gpu_ctx* c)
{
	if (!c) return POT_E_ARG;
	CK(cudaSetDevice(c->device));
	return sync_status(c);
}

}  // extern "C"
