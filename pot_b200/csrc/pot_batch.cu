// Batches of independent runs (no counterpart in the reference, which runs
// one grain per MPI job): admission by free HBM, eviction, and stepping every
// member with one CUDA-graph launch, plus the autotuner that picks leaf and
// group sizes.
//
// Each run keeps its own context (device state sized for its N, its own
// stream).  A batch step captures every member's step sequence into one
// graph: the origin stream forks to each member's stream, each member
// enqueues `steps_per_launch` steps (an even count, so the double-buffered
// state returns to the captured parity), every member joins back, and a
// gather kernel copies each member's step count, grain charge, charge sum and
// status into one summary array.  Independent runs share nothing, so the
// graph's branches run concurrently and a small run never waits for a large
// one inside a launch.  The graph is re-captured only when membership (or a
// member's buffer parity) changed since the last capture.
#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "pot_tree.cuh"

namespace pot {
cudaStream_t ctx_stream(pot_gpu_ctx* c);
int ctx_parity(const pot_gpu_ctx* c);
RunRec* ctx_rec(pot_gpu_ctx* c);
uint64_t ctx_bytes(const pot_gpu_ctx* c);
uint64_t ctx_particles(const pot_gpu_ctx* c);
int ctx_ready(const pot_gpu_ctx* c);
int ctx_enqueue(pot_gpu_ctx* c, uint32_t nsteps);
void ctx_mark_error(pot_gpu_ctx* c, int rc);
bool ctx_member_view(pot_gpu_ctx* c, MemberView* v);
void ctx_set_tree_valid(pot_gpu_ctx* c);
int ctx_retune(pot_gpu_ctx* c, uint32_t leaf, uint32_t group);

// one member's summary row
struct BatchRow {
	unsigned long long t_steps;
	long long grain_q;
	long long q_sum;
	unsigned long long tot_absor_e;
	int status;
	unsigned int warn;
};

__global__ void k_batch_gather(RunRec* const* __restrict__ recs, uint32_t n, BatchRow* __restrict__ rows)
{
	const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
	if (i >= n) return;
	const RunRec* r = recs[i];
	BatchRow b;
	b.t_steps = r->t_steps;
	b.grain_q = r->grain_q;
	b.q_sum = r->q_sum;
	b.tot_absor_e = r->tot_absor_e;
	b.status = r->status;
	b.warn = r->warn;
	rows[i] = b;
}
}  // namespace pot

using namespace pot;

struct BatchSlot {
	pot_gpu_ctx* ctx = nullptr;
	int parity = -1;       // buffer parity at the last capture
	cudaEvent_t join = nullptr;
};

// Members that share one packed launch per kernel: fast-form Boris runs
// with the same group size and the same radix passes.  Its device block
// holds the members' views, each stage's block prefix, the walk's group
// prefix and work counter.
struct PackClass {
	uint32_t group_max = 0, npass = 0;
	std::vector<int> slots;
	void* mem = nullptr;
	PackDev B {};
	cudaStream_t st = nullptr;
	cudaEvent_t join = nullptr;
};

struct pot_batch {
	int device = 0;
	uint32_t spl = 2;            // steps per graph launch (even)
	uint64_t reserve = 0;        // HBM bytes kept free
	cudaStream_t origin = nullptr;
	cudaEvent_t fork = nullptr;
	std::vector<BatchSlot> slots;  // index = slot id; ctx == nullptr when free
	cudaGraphExec_t exec = nullptr;
	bool dirty = true;
	// summary
	RunRec** d_recs = nullptr;
	BatchRow* d_rows = nullptr;
	BatchRow* h_rows = nullptr;  // pinned
	uint32_t cap_rows = 0;
	std::vector<int> order;      // slot of each summary row
	std::vector<PackClass> packs;  // packed launches of the last capture
	bool pack = true;            // pack the members that can be packed
	int sticky = POT_OK;
};

static void free_packs(pot_batch* b)
{
	for (auto& pc : b->packs) {
		if (pc.mem) cudaFree(pc.mem);
		if (pc.join) cudaEventDestroy(pc.join);
		if (pc.st) cudaStreamDestroy(pc.st);
	}
	b->packs.clear();
}

#define BCK(x)                                                        \
	do {                                                              \
		cudaError_t e_ = (x);                                         \
		if (e_ != cudaSuccess) return e_ == cudaErrorMemoryAllocation \
		                                  ? POT_E_NOMEM               \
		                                  : POT_E_CUDA;               \
	} while (0)

extern "C" {

int pot_batch_create(const pot_batch_opts* opts, pot_batch** out)
{
	if (!out) return POT_E_ARG;
	*out = nullptr;
	pot_batch_opts o {};
	if (opts) o = *opts;
	if (o.steps_per_launch == 0) o.steps_per_launch = 2;
	if (o.steps_per_launch % 2) return POT_E_ARG;
	int ndev = 0;
	if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return POT_E_CUDA;
	if (o.device < 0 || o.device >= ndev) return POT_E_ARG;
	pot_batch* b = new (std::nothrow) pot_batch();
	if (!b) return POT_E_NOMEM;
	b->device = o.device;
	b->spl = o.steps_per_launch;
	b->reserve = o.reserve_bytes;
	b->pack = (o.flags & POT_BATCH_NO_PACK) == 0;
	if (cudaSetDevice(b->device) != cudaSuccess ||
	    cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking) != cudaSuccess ||
	    cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) {
		pot_batch_destroy(b);
		return POT_E_CUDA;
	}
	*out = b;
	return POT_OK;
}

void pot_batch_destroy(pot_batch* b)
{
	if (!b) return;
	cudaSetDevice(b->device);
	if (b->origin) cudaStreamSynchronize(b->origin);
	if (b->exec) cudaGraphExecDestroy(b->exec);
	free_packs(b);
	for (auto& s : b->slots) {
		if (s.ctx) pot_gpu_destroy(s.ctx);
		if (s.join) cudaEventDestroy(s.join);
	}
	if (b->d_recs) cudaFree(b->d_recs);
	if (b->d_rows) cudaFree(b->d_rows);
	if (b->h_rows) cudaFreeHost(b->h_rows);
	if (b->fork) cudaEventDestroy(b->fork);
	if (b->origin) cudaStreamDestroy(b->origin);
	delete b;
}

int pot_batch_admit(pot_batch* b, const pot_run_cfg* cfg, const pot_gpu_opts* opts, const pot_particle* parts,
                    const pot_grain_state* grain, int32_t* slot)
{
	if (!b || !cfg || !slot) return POT_E_ARG;
	*slot = -1;
	pot_gpu_opts o {};
	if (opts) o = *opts;
	o.device = b->device;
	o.stream = nullptr;            // each member has its own stream
	o.flags &= ~POT_OPT_TIMING;    // event timing cannot be captured
	uint64_t need = 0;
	int rc = pot_gpu_bytes_needed(cfg, &o, &need);
	if (rc != POT_OK) return rc;
	if (cudaSetDevice(b->device) != cudaSuccess) return POT_E_CUDA;
	size_t free_b = 0, total_b = 0;
	if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return POT_E_CUDA;
	if ((uint64_t)free_b < need + b->reserve) return POT_E_NOMEM;
	// the batch must not be running while a member is set up
	if (cudaStreamSynchronize(b->origin) != cudaSuccess) return POT_E_CUDA;
	pot_gpu_ctx* c = nullptr;
	if ((rc = pot_gpu_create(cfg, &o, &c)) != POT_OK) return rc;
	rc = parts ? pot_gpu_upload(c, parts, cfg->N, grain) : pot_gpu_init_particles(c);
	if (rc != POT_OK) {
		pot_gpu_destroy(c);
		return rc;
	}
	size_t k = 0;
	while (k < b->slots.size() && b->slots[k].ctx) k++;
	if (k == b->slots.size()) b->slots.emplace_back();
	BatchSlot& s = b->slots[k];
	if (!s.join && cudaEventCreateWithFlags(&s.join, cudaEventDisableTiming) != cudaSuccess) {
		pot_gpu_destroy(c);
		return POT_E_CUDA;
	}
	s.ctx = c;
	s.parity = -1;
	b->dirty = true;
	*slot = (int32_t)k;
	return POT_OK;
}

int pot_batch_evict(pot_batch* b, int32_t slot)
{
	if (!b || slot < 0 || (size_t)slot >= b->slots.size() || !b->slots[slot].ctx) return POT_E_ARG;
	if (cudaSetDevice(b->device) != cudaSuccess) return POT_E_CUDA;
	if (cudaStreamSynchronize(b->origin) != cudaSuccess) return POT_E_CUDA;
	pot_gpu_destroy(b->slots[slot].ctx);
	b->slots[slot].ctx = nullptr;
	b->dirty = true;
	return POT_OK;
}

int pot_batch_ctx(pot_batch* b, int32_t slot, pot_gpu_ctx** ctx)
{
	if (!b || !ctx || slot < 0 || (size_t)slot >= b->slots.size() || !b->slots[slot].ctx) return POT_E_ARG;
	if (cudaSetDevice(b->device) != cudaSuccess) return POT_E_CUDA;
	if (cudaStreamSynchronize(b->origin) != cudaSuccess) return POT_E_CUDA;
	*ctx = b->slots[slot].ctx;
	return POT_OK;
}

static int ensure_rows(pot_batch* b, uint32_t n)
{
	if (n <= b->cap_rows) return POT_OK;
	const uint32_t cap = std::max<uint32_t>(n, 2 * b->cap_rows);
	if (b->d_recs) cudaFree(b->d_recs);
	if (b->d_rows) cudaFree(b->d_rows);
	if (b->h_rows) cudaFreeHost(b->h_rows);
	b->d_recs = nullptr;
	b->d_rows = nullptr;
	b->h_rows = nullptr;
	b->cap_rows = 0;
	BCK(cudaMalloc((void**)&b->d_recs, sizeof(RunRec*) * cap));
	BCK(cudaMalloc((void**)&b->d_rows, sizeof(BatchRow) * cap));
	BCK(cudaMallocHost((void**)&b->h_rows, sizeof(BatchRow) * cap));
	b->cap_rows = cap;
	return POT_OK;
}

static inline uint32_t div_up(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Blocks of each packed stage for one member (the single run's grids,
// except where a kernel strides over a device-side count: there a share
// proportional to the member's size).
static void member_blocks(const MemberView& v, uint32_t out[PS_COUNT])
{
	const uint32_t n = v.P.n, nt = v.P.n_tree, L = v.P.leaf_size;
	out[PS_KEYS] = keys_blocks(n);
	out[PS_N256] = div_up(n, 256);
	out[PS_TILES] = v.tiles;
	out[PS_CMP] = pack_scan_blocks(n);
	out[PS_PAIRS] = div_up(nt - 1, 256);
	out[PS_NODES] = pack_scan_blocks(nt - L);
	out[PS_FILL] = div_up(nt - L, 256);
	out[PS_FINISH] = div_up(nt, 256);
	out[PS_MOM] = div_up(nt, PACK_MOM_TILE);
	out[PS_MOMPRE] = div_up(nt / 4 + 1, 256);
	out[PS_GROUPS] = std::min<uint32_t>(592u, std::max<uint32_t>(1u, div_up(nt, 2048)));
	out[PS_ONE] = 1;
	out[PS_SMALL] = std::max<uint32_t>(4u, std::min<uint32_t>(148u, n / 8192u));
}

// Sort the batch's live members into packed classes (left in b->packs,
// with their device blocks filled) and the rest (`chains`), which step as
// their own kernel sequences.
static int plan_packs(pot_batch* b, std::vector<int>& chains)
{
	free_packs(b);
	chains.clear();
	std::vector<std::vector<MemberView>> views;
	for (int k : b->order) {
		MemberView v;
		if (!b->pack || !ctx_member_view(b->slots[k].ctx, &v)) {
			chains.push_back(k);
			continue;
		}
		const uint32_t npass = (uint32_t)radix_passes((int)v.P.key_bits);
		size_t c = 0;
		while (c < b->packs.size() && (b->packs[c].group_max != v.P.group_max || b->packs[c].npass != npass)) c++;
		if (c == b->packs.size()) {
			b->packs.emplace_back();
			b->packs.back().group_max = v.P.group_max;
			b->packs.back().npass = npass;
			views.emplace_back();
		}
		b->packs[c].slots.push_back(k);
		views[c].push_back(v);
	}
	for (size_t c = 0; c < b->packs.size(); c++) {
		PackClass& pc = b->packs[c];
		const uint32_t M = (uint32_t)views[c].size();
		// device block: views, then per stage M + 1 prefix words, the group prefix, the counter
		const size_t views_b = (sizeof(MemberView) * M + 255) / 256 * 256;
		const size_t words = (size_t)PS_COUNT * (M + 1) + (M + 1) + 1;
		std::vector<uint32_t> h(words, 0u);
		for (uint32_t m = 0; m < M; m++) {
			uint32_t nb[PS_COUNT];
			member_blocks(views[c][m], nb);
			for (int st = 0; st < PS_COUNT; st++) h[(size_t)st * (M + 1) + m + 1] = h[(size_t)st * (M + 1) + m] + nb[st];
		}
		BCK(cudaMalloc(&pc.mem, views_b + words * sizeof(uint32_t)));
		char* base = static_cast<char*>(pc.mem);
		uint32_t* w = reinterpret_cast<uint32_t*>(base + views_b);
		BCK(cudaMemcpy(base, views[c].data(), sizeof(MemberView) * M, cudaMemcpyHostToDevice));
		BCK(cudaMemcpy(w, h.data(), words * sizeof(uint32_t), cudaMemcpyHostToDevice));
		pc.B.mv = reinterpret_cast<const MemberView*>(base);
		pc.B.M = M;
		pc.B.npass = pc.npass;
		for (int st = 0; st < PS_COUNT; st++) {
			pc.B.pre[st] = w + (size_t)st * (M + 1);
			pc.B.blocks[st] = h[(size_t)st * (M + 1) + M];
		}
		pc.B.gpre = w + (size_t)PS_COUNT * (M + 1);
		pc.B.ctr = w + (size_t)PS_COUNT * (M + 1) + (M + 1);
		BCK(cudaStreamCreateWithFlags(&pc.st, cudaStreamNonBlocking));
		BCK(cudaEventCreateWithFlags(&pc.join, cudaEventDisableTiming));
	}
	return POT_OK;
}

// One packed class's `spl` steps: every kernel of the fast Boris step once
// for all its members (enqueue_step's sequence).
static void enqueue_pack(const PackClass& pc, uint32_t spl)
{
	const PackDev& B = pc.B;
	cudaStream_t s = pc.st;
	for (uint32_t k = 0; k < spl; k++) {
		pack_sort_begin(B, s);
		pack_keys(B, (int)k, s);
		pack_sort(B, s);
		pack_reorder(B, (int)k, s);
		pack_build(B, s);
		pack_compact(B, s);
		pack_groups(B, s);
		pack_chi_b(B, s);
		pack_push(B, (int)k, pc.group_max > 32 ? 2u : 1u, s);
		pack_absorb_late(B, (int)k, s);
		pack_reinject(B, (int)k, s);
		pack_grain_end(B, (int)k, s);
	}
}

// Capture every member's `spl` steps and the summary gather into one graph.
static int capture(pot_batch* b)
{
	if (b->exec) {
		cudaGraphExecDestroy(b->exec);
		b->exec = nullptr;
	}
	b->order.clear();
	for (size_t k = 0; k < b->slots.size(); k++)
		if (b->slots[k].ctx) b->order.push_back((int)k);
	const uint32_t n = (uint32_t)b->order.size();
	if (n == 0) {
		b->dirty = false;
		return POT_OK;
	}
	int rc = ensure_rows(b, n);
	if (rc != POT_OK) return rc;
	std::vector<RunRec*> recs(n);
	for (uint32_t i = 0; i < n; i++) recs[i] = ctx_rec(b->slots[b->order[i]].ctx);
	BCK(cudaMemcpyAsync(b->d_recs, recs.data(), sizeof(RunRec*) * n, cudaMemcpyHostToDevice, b->origin));
	BCK(cudaStreamSynchronize(b->origin));
	// every member's own queue must be idle before it joins the capture
	for (int k : b->order) BCK(cudaStreamSynchronize(ctx_stream(b->slots[k].ctx)));
	std::vector<int> chains;
	rc = plan_packs(b, chains);
	if (rc != POT_OK) return rc;
	BCK(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
	cudaError_t ce = cudaEventRecord(b->fork, b->origin);
	int first_err = ce == cudaSuccess ? POT_OK : POT_E_CUDA;
	for (auto& pc : b->packs) {
		if (first_err != POT_OK) break;
		if (cudaStreamWaitEvent(pc.st, b->fork, 0) != cudaSuccess) {
			first_err = POT_E_CUDA;
			break;
		}
		enqueue_pack(pc, b->spl);
		if (cudaGetLastError() != cudaSuccess) first_err = POT_E_CUDA;
		if (cudaEventRecord(pc.join, pc.st) != cudaSuccess || cudaStreamWaitEvent(b->origin, pc.join, 0) != cudaSuccess) {
			if (first_err == POT_OK) first_err = POT_E_CUDA;
		}
		for (int k : pc.slots) {
			b->slots[k].parity = ctx_parity(b->slots[k].ctx);
			ctx_set_tree_valid(b->slots[k].ctx);
		}
	}
	for (int k : chains) {
		if (first_err != POT_OK) break;
		BatchSlot& s = b->slots[k];
		cudaStream_t st = ctx_stream(s.ctx);
		if (cudaStreamWaitEvent(st, b->fork, 0) != cudaSuccess) {
			first_err = POT_E_CUDA;
			break;
		}
		const int erc = ctx_enqueue(s.ctx, b->spl);
		if (erc != POT_OK) first_err = erc;
		if (cudaEventRecord(s.join, st) != cudaSuccess || cudaStreamWaitEvent(b->origin, s.join, 0) != cudaSuccess) {
			if (first_err == POT_OK) first_err = POT_E_CUDA;
		}
		s.parity = ctx_parity(s.ctx);
	}
	if (first_err == POT_OK) {
		k_batch_gather<<<(n + 127) / 128, 128, 0, b->origin>>>(b->d_recs, n, b->d_rows);
		if (cudaGetLastError() != cudaSuccess) first_err = POT_E_CUDA;
	}
	cudaGraph_t g = nullptr;
	const cudaError_t ee = cudaStreamEndCapture(b->origin, &g);
	if (first_err == POT_OK && ee != cudaSuccess) first_err = POT_E_CUDA;
	if (first_err == POT_OK && cudaGraphInstantiate(&b->exec, g, 0) != cudaSuccess) {
		b->exec = nullptr;
		first_err = POT_E_CUDA;
	}
	if (g) cudaGraphDestroy(g);
	if (first_err != POT_OK) return first_err;
	b->dirty = false;
	return POT_OK;
}

static bool stale(const pot_batch* b)
{
	if (b->dirty) return true;
	for (int k : b->order) {
		const BatchSlot& s = b->slots[k];
		if (!s.ctx || ctx_parity(s.ctx) != s.parity) return true;
	}
	return false;
}

int pot_batch_step(pot_batch* b, uint32_t nsteps)
{
	if (!b) return POT_E_ARG;
	if (b->sticky != POT_OK) return b->sticky;
	if (nsteps % b->spl) return POT_E_ARG;
	if (cudaSetDevice(b->device) != cudaSuccess) return POT_E_CUDA;
	for (auto& s : b->slots)
		if (s.ctx && ctx_ready(s.ctx) != POT_OK) return ctx_ready(s.ctx);
	if (stale(b)) {
		const int rc = capture(b);
		if (rc != POT_OK) {
			b->sticky = rc;
			return rc;
		}
	}
	if (!b->exec) return POT_OK;  // no members
	for (uint32_t k = 0; k < nsteps; k += b->spl) {
		if (cudaGraphLaunch(b->exec, b->origin) != cudaSuccess) {
			b->sticky = POT_E_CUDA;
			return POT_E_CUDA;
		}
	}
	return POT_OK;
}

int pot_batch_sync(pot_batch* b)
{
	if (!b) return POT_E_ARG;
	if (cudaSetDevice(b->device) != cudaSuccess) return POT_E_CUDA;
	if (cudaStreamSynchronize(b->origin) != cudaSuccess) return POT_E_CUDA;
	return b->sticky;
}

int pot_batch_summary(pot_batch* b, uint32_t max, pot_batch_row* rows, uint32_t* n_rows)
{
	if (!b || !n_rows) return POT_E_ARG;
	*n_rows = 0;
	if (cudaSetDevice(b->device) != cudaSuccess) return POT_E_CUDA;
	if (stale(b)) {
		// membership changed since the last launch: refresh by capture
		int rc = capture(b);
		if (rc != POT_OK) return rc;
	}
	const uint32_t n = (uint32_t)b->order.size();
	if (n == 0) return POT_OK;
	// rows of the current state (the gather alone, outside the graph)
	k_batch_gather<<<(n + 127) / 128, 128, 0, b->origin>>>(b->d_recs, n, b->d_rows);
	BCK(cudaGetLastError());
	BCK(cudaMemcpyAsync(b->h_rows, b->d_rows, sizeof(BatchRow) * n, cudaMemcpyDeviceToHost, b->origin));
	BCK(cudaStreamSynchronize(b->origin));
	const uint32_t m = std::min(n, max);
	for (uint32_t i = 0; i < m; i++) {
		const BatchRow& r = b->h_rows[i];
		rows[i].slot = b->order[i];
		rows[i].status = r.status;
		rows[i].t_steps = r.t_steps;
		rows[i].grain_q = r.grain_q;
		rows[i].q_sum = r.q_sum;
		rows[i].tot_absor_e = r.tot_absor_e;
		rows[i].particles = ctx_particles(b->slots[b->order[i]].ctx);
		rows[i].warn = r.warn;
		rows[i].pad = 0;
		if (r.status != POT_OK) ctx_mark_error(b->slots[b->order[i]].ctx, r.status);
	}
	*n_rows = m;
	return POT_OK;
}

int pot_batch_count(pot_batch* b, uint32_t* runs, uint64_t* particles, uint64_t* bytes)
{
	if (!b) return POT_E_ARG;
	uint32_t nr = 0;
	uint64_t np = 0, nb = 0;
	for (auto& s : b->slots) {
		if (!s.ctx) continue;
		nr++;
		np += ctx_particles(s.ctx);
		nb += ctx_bytes(s.ctx);
	}
	if (runs) *runs = nr;
	if (particles) *particles = np;
	if (bytes) *bytes = nb;
	return POT_OK;
}

// ---------------------------------------------------------------------------
// autotuner
// ---------------------------------------------------------------------------
int pot_gpu_tune(const pot_run_cfg* cfg, pot_gpu_opts* opts, uint32_t steps, double* ms_per_step)
{
	if (!cfg || !opts) return POT_E_ARG;
	if (opts->form != POT_FORM_FAST) {  // the plain form has no sizes to choose
		if (ms_per_step) *ms_per_step = 0.0;
		return POT_OK;
	}
	if (steps < 2) steps = 2;
	steps += steps % 2;
	static const uint32_t cand[][2] = { { 8, 32 }, { 16, 32 }, { 32, 32 }, { 16, 64 }, { 32, 64 } };
	double best = -1.0;
	uint32_t best_l = 0, best_g = 0;
	if (cudaSetDevice(opts->device) != cudaSuccess) return POT_E_CUDA;
	// one context for every candidate: created with leaf size 8, the largest
	// tree of the candidates, and switched between them (ctx_retune)
	pot_gpu_opts o = *opts;
	o.leaf_size = 8;
	o.group_size = 32;
	o.flags &= ~POT_OPT_TIMING;
	o.stream = nullptr;
	pot_gpu_ctx* c = nullptr;
	int rc = pot_gpu_create(cfg, &o, &c);
	if (rc != POT_OK) return rc;
	cudaEvent_t e0 = nullptr, e1 = nullptr;
	if (cudaEventCreate(&e0) != cudaSuccess || cudaEventCreate(&e1) != cudaSuccess) {
		if (e0) cudaEventDestroy(e0);
		pot_gpu_destroy(c);
		return POT_E_CUDA;
	}
	int last_rc = POT_OK;
	for (const auto& c2 : cand) {
		rc = ctx_retune(c, c2[0], c2[1]);
		if (rc == POT_OK) rc = ctx_enqueue(c, 2);  // warm-up, kernel by kernel as the batch enqueues them
		if (rc == POT_OK) rc = pot_gpu_sync(c);
		float ms = 0.f;
		if (rc == POT_OK) {
			cudaStream_t s = ctx_stream(c);
			cudaEventRecord(e0, s);
			rc = ctx_enqueue(c, steps);
			cudaEventRecord(e1, s);
			if (cudaEventSynchronize(e1) != cudaSuccess) rc = POT_E_CUDA;
			if (rc == POT_OK) cudaEventElapsedTime(&ms, e0, e1);
			if (rc == POT_OK) rc = pot_gpu_sync(c);
		}
		if (rc != POT_OK) {
			last_rc = rc;
			if (rc == POT_E_CUDA) break;
			continue;
		}
		const double per = ms / steps;
		if (best < 0.0 || per < best) {
			best = per;
			best_l = c2[0];
			best_g = c2[1];
		}
	}
	cudaEventDestroy(e0);
	cudaEventDestroy(e1);
	pot_gpu_destroy(c);
	if (best < 0.0) return last_rc != POT_OK ? last_rc : POT_E_CUDA;
	opts->leaf_size = best_l;
	opts->group_size = best_g;
	if (ms_per_step) *ms_per_step = best;
	return POT_OK;
}

}  // extern "C"
