/*
 * Single-rank MPI stand-in used only to compile the reference program as a
 * CPU oracle (test infrastructure, never part of the GPU product path).
 *
 * The reference (pot.c, prng.c) is an MPI-1 program.  No MPI implementation
 * is installed on these machines, so this header supplies every MPI symbol the
 * reference names, with the semantics of a communicator of exactly one rank:
 *   - Bcast/Send/Recv are no-ops (rank 0 already owns every byte);
 *   - Gather/Reduce/Allreduce copy the send buffer into the receive buffer
 *     (a one-element reduction is the identity), or do nothing for
 *     MPI_IN_PLACE;
 *   - derived datatypes are opaque handles whose byte size is remembered so
 *     that the copies above move the right number of bytes.
 * With one rank, pot.c's loops over workers (pot.c:2570, pot.c:2884) never
 * execute a Send/Recv pair, so no message ever needs to be queued.
 */
#ifndef POT_ORACLE_MPI_STUB_H
#define POT_ORACLE_MPI_STUB_H

#include <stddef.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Group;
typedef long MPI_Datatype;   /* encodes the element size in bytes */
typedef long MPI_Aint;
typedef int MPI_Op;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_WORLD 0
#define MPI_SUM 1
#define MPI_LOR 2
#define MPI_IN_PLACE ((void*) 1)
#define MPI_STATUS_IGNORE ((MPI_Status*) 0)

#define MPI_BYTE ((MPI_Datatype) 1)
#define MPI_UNSIGNED_CHAR ((MPI_Datatype) 1)
#define MPI_C_BOOL ((MPI_Datatype) sizeof(_Bool))
#define MPI_INT ((MPI_Datatype) sizeof(int))
#define MPI_UNSIGNED ((MPI_Datatype) sizeof(unsigned int))
#define MPI_UINT32_T ((MPI_Datatype) 4)
#define MPI_DOUBLE ((MPI_Datatype) sizeof(double))
#define MPI_LONG_DOUBLE ((MPI_Datatype) sizeof(long double))

static inline int MPI_Init(int* argc, char*** argv) { (void) argc; (void) argv; return MPI_SUCCESS; }
static inline int MPI_Initialized(int* flag) { *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int* r) { (void) c; *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int* s) { (void) c; *s = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_group(MPI_Comm c, MPI_Group* g) { (void) c; *g = 0; return MPI_SUCCESS; }
static inline int MPI_Group_range_incl(MPI_Group g, int n, int r[][3], MPI_Group* out)
{ (void) g; (void) n; (void) r; *out = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_create(MPI_Comm c, MPI_Group g, MPI_Comm* out)
{ (void) c; (void) g; *out = 0; return MPI_SUCCESS; }

static inline int MPI_Get_address(const void* p, MPI_Aint* a) { *a = (MPI_Aint) p; return MPI_SUCCESS; }
static inline int MPI_Type_create_struct(int n, const int* lens, const MPI_Aint* disps,
                                         const MPI_Datatype* types, MPI_Datatype* out)
{
	/* Size = end of the last field; the only struct type pot.c builds is
	   its Particle record (pot.c:4119-4133), whose padding is irrelevant
	   because single-rank transfers never happen. */
	MPI_Aint end = 0;
	int i;
	for (i = 0; i < n; i++) {
		MPI_Aint e = disps[i] + (MPI_Aint) lens[i] * (MPI_Aint) types[i];
		if (e > end) end = e;
	}
	*out = (MPI_Datatype) end;
	return MPI_SUCCESS;
}
static inline int MPI_Type_contiguous(int n, MPI_Datatype t, MPI_Datatype* out)
{ *out = (MPI_Datatype) n * t; return MPI_SUCCESS; }
static inline int MPI_Type_commit(MPI_Datatype* t) { (void) t; return MPI_SUCCESS; }
static inline int MPI_Type_free(MPI_Datatype* t) { (void) t; return MPI_SUCCESS; }

static inline int MPI_Bcast(void* b, int n, MPI_Datatype t, int root, MPI_Comm c)
{ (void) b; (void) n; (void) t; (void) root; (void) c; return MPI_SUCCESS; }
static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int d, int tag, MPI_Comm c)
{ (void) b; (void) n; (void) t; (void) d; (void) tag; (void) c; return MPI_SUCCESS; }
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int s, int tag, MPI_Comm c, MPI_Status* st)
{ (void) b; (void) n; (void) t; (void) s; (void) tag; (void) c; (void) st; return MPI_SUCCESS; }

static inline int MPI_Gather(const void* sb, int sn, MPI_Datatype st, void* rb, int rn,
                             MPI_Datatype rt, int root, MPI_Comm c)
{
	(void) rn; (void) rt; (void) root; (void) c;
	if (sb != MPI_IN_PLACE && rb != NULL) memmove(rb, sb, (size_t) sn * (size_t) st);
	return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op op,
                             int root, MPI_Comm c)
{
	(void) op; (void) root; (void) c;
	if (sb != MPI_IN_PLACE && rb != NULL) memmove(rb, sb, (size_t) n * (size_t) t);
	return MPI_SUCCESS;
}
static inline int MPI_Allreduce(const void* sb, void* rb, int n, MPI_Datatype t, MPI_Op op,
                                MPI_Comm c)
{
	(void) op; (void) c;
	if (sb != MPI_IN_PLACE) memmove(rb, sb, (size_t) n * (size_t) t);
	return MPI_SUCCESS;
}

#endif
