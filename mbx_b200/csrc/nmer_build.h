// Shared declarations for the n-mer builder (nmer_build.cu) and its host
// driver (mbx_capi.cu).  Internal to the library.
#pragma once
#include <cuda_runtime.h>

#include "holder_common.cuh"

#define MBX_MAX_TYPES 8     // monomer types of one topology
#define MBX_MAX_BUCKETS 16  // evaluators (buckets) of one term

// device status word bits (status[0]); status[1] holds the largest
// neighbour count seen when MBX_STATUS_NB_OVERFLOW is set
#define MBX_STATUS_NB_OVERFLOW 1
#define MBX_STATUS_BUCKET_OVERFLOW 2
#define MBX_STATUS_LIST_OVERFLOW 4
// a kernel's bounded barrier wait ran out (results discarded; an error, not a retry)
#define MBX_STATUS_WAIT_TIMEOUT 8

// shared-memory bytes per staged match of k_trimers (3 + 1 doubles, 4 ints)
#define MBX_TRIMATCH_BYTES 48

struct CellGrid {
    int n[3];
    int one_copy;          // PBC, n >= 3 on every axis and cells wider than the cutoff (with a margin):
                           // of a member's eight cloud points only the one its cell's wrap implies can match
    double lo[3];          // unused
    double inv_extent[3];  // no PBC: 1 / cell edge of the hashed grid
};

struct NbEntry {
    int member;  // index into the search's member list
    int copy;    // cloud copy 0..7
    double d2;   // squared distance to the query, reference arithmetic
};

struct DimerRules {
    int bucket[MBX_MAX_TYPES * MBX_MAX_TYPES];  // type pair (in n-mer order) -> bucket or -1
    int swap[MBX_MAX_TYPES * MBX_MAX_TYPES];    // 1: evaluator order is (j, i)
    double pre2[MBX_MAX_BUCKETS];               // (evaluator cutoff + margin)^2
    int cap[MBX_MAX_BUCKETS];
    long offset[MBX_MAX_BUCKETS];
    int near[MBX_MAX_BUCKETS];                  // bucket for dimers with d^2 < split2 (-1: none)
    double split2[MBX_MAX_BUCKETS];             // 0: no split
};

struct TrimerRules {
    int bucket[MBX_MAX_TYPES * MBX_MAX_TYPES * MBX_MAX_TYPES];
    int perm[MBX_MAX_TYPES * MBX_MAX_TYPES * MBX_MAX_TYPES];  // evaluator slot s <- original slot (perm >> 2s) & 3
    int skip[MBX_MAX_BUCKETS];                                // 1 two_of_three_gt, 2 all_three_gt
    double pre2[MBX_MAX_BUCKETS];
    int cap[MBX_MAX_BUCKETS];
    long offset[MBX_MAX_BUCKETS];
};

// One configuration of a batched search (all configurations of a batch in
// one set of launches): its box, its cell grid, and the index of its first
// cell in the batch's concatenated cell array.
struct BatchGrid {
    BoxParams bp;
    CellGrid cg;
    int cell_off;
};

__global__ void k_fix_monomers(double* xyz, const int* first_index, const int* nat, int nmon, BoxParams bp);
__global__ void k_cloud(const double* xyz, const int* first_index, const int* members, int nmem, BoxParams bp,
                        CellGrid cg, double* cloud, int* cell_of, int* copy_dir);
// The same for a batch: members are the batch's monomers in order (member
// position = monomer), each with the grid of its configuration conf_of[q].
__global__ void k_cloud_batch(const double* xyz, const int* first_index, int nmem, const int* conf_of,
                              const BatchGrid* grids, double* cloud, int* cell_of, int* copy_dir);
__global__ void k_cell_count(const int* cell_of, int nmem, int* cell_count);
__global__ void k_cell_scan(const int* cell_count, int ncell, int* cell_start, int* cell_fill);
__global__ void k_cell_fill(const int* cell_of, int nmem, int* cell_fill, int* cell_items);
__global__ void k_cell_sort(const int* cell_start, int ncell, const int* items, int* sorted);
// Matches of every query monomer (k_neighbors): `warps` warps per query (1 or
// 4), `unroll` independent 32-point blocks per iteration (1, 2 or 4).
int launch_neighbors(int warps, int unroll, const double* cloud, const int* copy_dir, const int* cell_of,
                     const int* cell_start, const int* cell_items, const int* query, int nquery, CellGrid cg,
                     int use_pbc, double rc2,
                     int cap, int* nb_count, NbEntry* nb, int* status, cudaStream_t s);
// The same over a batch (queries are member positions, conf_of and grids as
// for k_cloud_batch).
int launch_neighbors_batch(int warps, int unroll, const double* cloud, const int* copy_dir, const int* cell_of,
                           const int* cell_start,
                           const int* cell_items, const int* query, int nquery, const int* conf_of,
                           const BatchGrid* grids, double rc2, int cap, int* nb_count, NbEntry* nb, int* status,
                           cudaStream_t s);
__global__ void k_dimers(const int* query, int nquery, const int* members, const int* tag, const int* type,
                         const int* nb_count, const NbEntry* nb, int cap, double rc2, DimerRules R,
                         unsigned long long* listed, int4* list, long list_cap, int4* bucket_data,
                         int* bucket_count, int* status);
__global__ void k_trimers(const int* query, int nquery, const int* members, const int* tag, const int* type,
                          const double* cloud, const int* nb_count, const NbEntry* nb, int cap, double rc2,
                          TrimerRules R, unsigned long long* listed, int4* list, long list_cap, int4* bucket_data,
                          int* bucket_count, int* status);
