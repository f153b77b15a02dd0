// Tree storage and launchers shared by the tree and walk translation units.
#pragma once

#include "pot_host.h"

namespace pot {

// Internal nodes in pre-order, structure of arrays; `cap` entries each
// (the leaf table of bucket leaves has 8 * cap entries).
struct TreeDev {
	uint32_t cap;
	int8_t* lvl8;      // [n] common levels of pair (i, i + L), capped at 20
	uint32_t* cnt;     // [n] cells owned by pair i
	uint32_t* base;    // [n] exclusive scan of cnt: index of pair i's first cell
	uint32_t* first;   // first particle (Morton slot)
	uint32_t* last;    // last particle
	uint8_t* level;    // depth (root 0)
	int32_t* child;    // [8 * cap] child codes by octal digit
	int32_t* parent;
	uint8_t* nint;     // internal children
	uint32_t* ctr;     // arrivals in the upward pass
	int32_t* q;        // net charge (Tree.q)
	uint32_t* aq;      // absolute charge (Tree.aq)
	double4* cq;       // centre of |q| and q
	double* w2;        // (x2 - x1)^2
	double4* dip;      // DIPOLES: dipole moment about cq (FP64, both forms); null otherwise
	// FP32 walk (fast form only; null otherwise)
	float4* f;         // centre relative to the domain centre, q
	float* r2;         // w2 / OAP^2: accepted when d^2 > r2
	float4* lf;        // [8 * cap] bucket-leaf moments
	float* lr2;        // [8 * cap] bucket-leaf critical radius^2
	uint2* lrange;     // [8 * cap] bucket-leaf (first slot, count)
	uint2* ovf;        // [OVF_CAP] leaf-size-1 overflow buckets (first slot, count)
	// fast form: exclusive prefix sums of (q, |q|, |q| x, |q| y, |q| z), 5 doubles each
	double* mom_pre;   // [n + 1]
	double* mom_blk;   // [blocks + 1]
	// fast form with DIPOLES: prefix sums of (q x, q y, q z) in the same layout,
	// and the cells' and bucket leaves' dipoles in FP32 units of q R
	double* mom_pre_d;
	double* mom_blk_d;
	float4* fd;        // [cap]
	float4* lfd;       // [8 * cap]
};

// One member run of a packed batch as the batched kernels see it: the
// run's parameters, tree, record and device arrays (those of its context).
// Buffer parity: at step k of a graph launch a member's state is in
// pos[cur ^ (k & 1)]; kb is the key buffer holding the sorted keys (the
// number of radix passes is the same for every member of a batch).
struct MemberView {
	Params P;
	TreeDev T;
	RunRec* rec;
	StepHist* hist;
	double4* pos[2];
	double4* vel[2];
	uint32_t* pid[2];
	double4* src64;
	float4* src32;
	uint64_t* keys[2];
	uint32_t* vals[2];
	uint32_t* counts;      // radix-sort status words, histograms and tile counters
	uint32_t* block_sums;  // scan block sums
	uint8_t* due;
	uint32_t* due_tiles;   // due flags per scan tile, counted by the reorder
	uint32_t* due_list;
	uint32_t* due_prefix;
	uint2* groups;
	uint32_t* rein_list;
	uint32_t cur;
	uint32_t kb;
	uint32_t tiles;        // radix-sort tiles
	uint32_t pad;
};

// A packed batch's step: each kernel of the step is one launch over every
// member (pot_batch.cu builds this).  pre[stage] is the exclusive prefix of
// the members' block counts for that stage's kernels (device, M + 1
// entries), blocks[stage] its total.  Stages:
//   PS_KEYS    keys_blocks(n): keys and the sort's digit counts
//   PS_N256    blocks_for(n, 256): reorder
//   PS_TILES   the sort's tiles: clearing the status words, each pass
//   PS_CMP     scan tiles over n: the due list
//   PS_PAIRS   blocks_for(n_tree - 1, 256)
//   PS_NODES   scan tiles over the n_tree - L key pairs: cell numbering
//   PS_FILL    blocks_for(n_tree - L, 256)
//   PS_FINISH  blocks_for(n_tree, 256)
//   PS_MOM     moment tiles over n_tree: prefix sums
//   PS_MOMPRE  blocks_for(n_tree / 4 + 1, 256): cell moments from the sums
//   PS_GROUPS  target groups
//   PS_ONE     one block per member: digit offsets, scan tops, chi_b, grain
//   PS_SMALL   4-148 blocks per member (one per 8,192 particles): late
//              absorption, reinjection (one warp per reinjected particle)
enum PackStage : int {
	PS_KEYS, PS_N256, PS_TILES, PS_CMP, PS_PAIRS, PS_NODES, PS_FILL, PS_FINISH, PS_MOM, PS_MOMPRE, PS_GROUPS,
	PS_ONE, PS_SMALL, PS_COUNT
};
struct PackDev {
	const MemberView* mv;           // [M], device
	uint32_t M;
	uint32_t npass;                 // radix passes, the same for every member
	const uint32_t* pre[PS_COUNT];
	uint32_t blocks[PS_COUNT];
	uint32_t* gpre;                 // [M + 1] prefix of the members' target groups this step (device)
	unsigned int* ctr;              // the batch walk's work counter (device)
};
// The member's state at step k of a graph launch is in buffer cur ^ (k & 1)
// until the reorder, which writes the other buffer.
__device__ __forceinline__ uint32_t pack_in(const MemberView& v, int k) { return v.cur ^ (uint32_t)(k & 1); }
__device__ __forceinline__ uint32_t pack_out(const MemberView& v, int k) { return v.cur ^ (uint32_t)(k & 1) ^ 1u; }

// the packed step's launches, in stream order (tree.cu, sort.cu, walk.cu,
// walk_fast.cu, inject.cu)
void pack_sort_begin(const PackDev& B, cudaStream_t s);
void pack_keys(const PackDev& B, int k, cudaStream_t s);
void pack_sort(const PackDev& B, cudaStream_t s);
void pack_reorder(const PackDev& B, int k, cudaStream_t s);
void pack_build(const PackDev& B, cudaStream_t s);
void pack_compact(const PackDev& B, cudaStream_t s);
void pack_node_scan(const PackDev& B, cudaStream_t s);
void pack_groups(const PackDev& B, cudaStream_t s);
void pack_chi_b(const PackDev& B, cudaStream_t s);
void pack_push(const PackDev& B, int k, uint32_t tpl, cudaStream_t s);
void pack_absorb_late(const PackDev& B, int k, cudaStream_t s);
void pack_reinject(const PackDev& B, int k, cudaStream_t s);
void pack_grain_end(const PackDev& B, int k, cudaStream_t s);
constexpr uint32_t PACK_MOM_TILE = 256 * 16;  // moment prefix-sum tile (tree.cu MOM_TILE)
uint32_t pack_scan_blocks(uint32_t n);        // scan tiles over n items

size_t mom_prefix_entries(size_t n);
size_t mom_block_entries(size_t n);
void launch_keys(const double4* pos, uint64_t* keys, uint32_t* vals, const Params& P, RunRec* rec,
                 int begin_step, uint32_t* hist, cudaStream_t s, Timer& tm);
uint32_t keys_blocks(size_t n);
void launch_reorder(const uint32_t* perm, const double4* pos_in, const double4* vel_in, const uint32_t* pid_in,
                    double4* pos_out, double4* vel_out, uint32_t* pid_out, double4* src64, float4* src32,
                    uint8_t* due, const Params& P, RunRec* rec, uint32_t* due_tiles, cudaStream_t s, Timer& tm);
void launch_build(const uint64_t* keys, TreeDev& T, const double4* src64, const Params& P, RunRec* rec,
                  uint32_t* block_sums, cudaStream_t s, Timer& tm);

// walk.cu
size_t macro_scratch_doubles();
void launch_macro(const double4* pos, const double4* vel, const Params& P, double* scratch, RunRec* rec,
                  cudaStream_t s, Timer& tm);
void launch_chi_b(const TreeDev& T, const double4* src64, const Params& P, RunRec* rec, int force,
                  cudaStream_t s, Timer& tm);
// Buffers of the non-Boris integrators' two-launch step: stage 0 is the
// one-launch Boris step; stage 1 writes each due particle's first-half
// acceleration (acc) and its intermediate source entry (src64b, and src32b in
// the fast form); stage 2 reads them.
struct StageBufs {
	int stage;
	double4* acc;
	double4* src64b;
	float4* src32b;
};
void launch_push(double4* pos, double4* vel, const TreeDev& T, const double4* src64, const float4* src32,
                 const uint32_t* due_list, const uint2* groups, uint32_t* rein_list, const Params& P, RunRec* rec,
                 const StageBufs& sb, cudaStream_t s, Timer& tm);
// Target groups of at most P.group_max due particles, each inside one tree
// cell.  With gcell (a byte per tree cell) and gblk (group_blocks() + 1
// words) the groups are laid out in tree pre-order, so that the walk's
// concurrent warps work on neighbouring groups; with gcell == nullptr they
// are built by one launch, in the order their cells finish.
uint32_t group_blocks();
void launch_groups(const TreeDev& T, const uint32_t* dpre, uint2* groups, uint8_t* gcell, uint32_t* gblk,
                   const Params& P, RunRec* rec, cudaStream_t s, Timer& tm);
void launch_absorb_late(double4* pos, double4* vel, const double4* src64, const uint32_t* due_list,
                        uint32_t* rein_list, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm);
void launch_grain_end(double4* pos, double4* vel, StepHist* hist, const Params& P, RunRec* rec, int epe,
                      cudaStream_t s, Timer& tm);
void launch_epe(const double4* pos, const TreeDev& T, const double4* src64, const float4* src32, uint2* groups_all,
                double* partial, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm);
void launch_field_query(const TreeDev& T, const double4* src64, const float4* src32, const double* xyz,
                        const uint32_t* self_slot, uint32_t nq, double* E, const Params& P, RunRec* rec,
                        cudaStream_t s, Timer& tm);
void launch_phi_query(const TreeDev& T, const double4* src64, const double* xyz, uint32_t nq, double* phi,
                      const Params& P, RunRec* rec, cudaStream_t s, Timer& tm);

// inject.cu
void launch_reinject(double4* pos, double4* vel, const uint32_t* pid, const uint32_t* rein_list,
                     const double4* src64, const Params& P, RunRec* rec, cudaStream_t s, Timer& tm);
void launch_init(double4* pos, double4* vel, uint32_t* pid, const Params& P, RunRec* rec, cudaStream_t s,
                 Timer& tm);

}  // namespace pot
