/* mbx_b200: B200-native many-body 2-body/3-body engine -- C ABI.
 *
 * The drop-in boundary is the reference's bblock::System 2-body/3-body path:
 *   double System::Get2B(bool do_grads, bool use_ghost)
 *   double System::Get3B(bool do_grads, bool use_ghost)
 * (bblock/system.h:1268,1279; bblock/system.cpp:2425-2725, 2769-3073), reached
 * from TwoBodyEnergy/ThreeBodyEnergy (system.h:1088,1100, system.cpp:2403-2423,
 * 2727-2745), plus the evaluator and generated-polynomial calling conventions
 * below them.  Plain pointers and sizes only; every call returns 0 on success
 * or an MBX_E* code, with a message in mbx_last_error().
 *
 * Coordinates follow the reference's internal layout: one array of 3 doubles
 * per site (real atoms and electrostatic virtual sites), monomers in internal
 * order, monomer m starting at site first_index[m].  Gradients are dE/dx
 * (kcal/mol/A), energies kcal/mol, virial -sum r (x) dE/dr (9, row-major,
 * symmetric).
 */
#ifndef MBX_B200_H
#define MBX_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct mbx_ctx mbx_ctx;

enum {
    MBX_OK = 0,
    MBX_EINVAL = 22,    /* bad argument, size or box */
    MBX_ENOMEM = 12,    /* device allocation failed */
    MBX_EDOM = 33,      /* cutoff too large for the periodic box */
    MBX_ENOTSUP = 95,   /* unknown evaluator or monomer type */
    MBX_ECUDA = 1000,   /* CUDA runtime error (message has details) */
    MBX_ENODEV = 1001   /* no CUDA device */
};

/* flags */
#define MBX_DEVICE_PTRS 1   /* array arguments are device pointers (else host) */
#define MBX_MIXED 2         /* FP32 monomials, FP64 accumulation (else FP64) */
#define MBX_NO_GRADS 4      /* energy only */
#define MBX_GRAPH 8         /* mbx_batch_energy: capture the sequence in a CUDA graph, replay it */

/* Context on one device with its own stream.  Replaces the state a
 * bblock::System keeps for the 2b/3b path (system.h:1175ff).  One context per
 * host thread; calls on a context are serialised on its stream.  stream may be
 * NULL (the context creates one) or a cudaStream_t to run on. */
int mbx_create(mbx_ctx** ctx, int device, void* stream);
int mbx_destroy(mbx_ctx* ctx);
const char* mbx_last_error(const mbx_ctx* ctx);
const char* mbx_version(void);

/* Monomers in internal order (System::AddMonomerInfo, system.cpp:1794-1969):
 * ids[m] (the reference's monomer ids of this path: "h2o", "ch4", "li+",
 * "na+", "k+", "rb+", "cs+", "f-", "cl-", "br-", "i-", "ar", "h2", "nh3",
 * "nh3pbe0d3bj", "co2", "co2_archive", "co2cm5100", "co2cm595", "co2cm590",
 * "co2cm585", "co2cm5875", "co2cm580", "mbpbe", "he", "n2o5"),
 * first_index[m] (first site), tag[m] (tag of the
 * monomer's first atom; n-mers are owned by the lowest tag,
 * sys_tools.cpp:562,585), is_local[m] (NULL = all local), numsites. */
int mbx_set_topology(mbx_ctx* ctx, int nmon, const char* const* ids, const int* first_index, const int* tag,
                     const int* is_local, int numsites);

/* cutoff2b/cutoff3b (System::Set2bCutoff/Set3bCutoff), box (9 doubles,
 * row vectors, NULL for no periodic boundaries; System::SetPBC), and the
 * ignored type tuples (ignore_2b_poly / ignore_3b_poly: n2 pairs in
 * ignore2b[2*i..], n3 triples in ignore3b[3*i..]). */
int mbx_set_config(mbx_ctx* ctx, double cutoff2b, double cutoff3b, const double* box, int n2,
                   const char* const* ignore2b, int n3, const char* const* ignore3b);

/* Get1B (nbody 1, bblock/system.cpp:2269) / Get2B (nbody 2,
 * system.cpp:2425) / Get3B (nbody 3, system.cpp:2769).  xyz: 3*numsites
 * doubles, wrapped in place as System::SetPBC does (FixMonomerCoordinates,
 * sys_tools.cpp:257).  *energy receives the term; grad (3*numsites, may be
 * NULL) and virial (9, may be NULL) are ACCUMULATED (+=) like grad_/virial_
 * in the reference.  flags: MBX_DEVICE_PTRS, MBX_MIXED, MBX_NO_GRADS.
 * use_ghost as in TwoBodyEnergy(do_grads, use_ghost) (ignored by nbody 1).
 * The 1-body term covers the local waters (MB-pol: the Partridge-Schwenke
 * surface, ps::pot_nasa, potential/1b/ps.cpp:346); a topology with a
 * monomer type whose 1-body term the reference computes on the CPU only
 * here (ch4, co2*, nh3*, h2, n2o5, mbpbe) returns MBX_ENOTSUP for nbody 1
 * unless that type is in the 1-body ignore list. */
int mbx_energy(mbx_ctx* ctx, int nbody, double* xyz, int use_ghost, double* energy, double* grad, double* virial,
               int flags);

/* GPU-resident callers (i-PI, LAMMPS: coordinates kept in the caller's
 * own atom order on the device).  mbx_set_real_order gives the site of
 * every real atom of the input order (the inverse of the topology's
 * OrderMonomers, numat entries); mbx_energy_real then takes the real
 * coordinates in input order (3*numat, not modified: the context wraps its
 * own site copy, as System::SetRealXyz + SetPBC do, system.cpp:830-846) and
 * accumulates the gradient in input order (+=, GetRealGrads), for nbody 1, 2
 * or 3 with the flags of mbx_energy. */
int mbx_set_real_order(mbx_ctx* ctx, int numat, const int* site_of_atom);
int mbx_energy_real(mbx_ctx* ctx, int nbody, const double* xyz_real, int use_ghost, double* energy,
                    double* grad_real, double* virial, int flags);

/* Monomer types skipped by the 1-body term (System ignore_1b_poly_,
 * system.cpp:2293-2296); replaces the previous list. */
int mbx_set_ignore_1b(mbx_ctx* ctx, int n, const char* const* ids);

/* Listed n-mers of the last mbx_energy call for nbody (dimers within
 * cutoff2b, trimers by the AddClusters rule within cutoff3b) and the number
 * that reached an evaluator. */
int mbx_last_counts(const mbx_ctx* ctx, int nbody, long* listed, long* evaluated);

/* The n-mer list itself (System::GetPairList / AddClustersParallel,
 * system.cpp:313, 1971): internal monomer indices, nbody per n-mer, order
 * unspecified (canonicalise before comparing).  xyz on the host.  Writes at
 * most cap n-mers, *count gets the total. */
int mbx_nmers(mbx_ctx* ctx, int nbody, double cutoff, const double* xyz, int use_ghost, long* out, long cap,
              long* count);

/* Evaluator calling convention (x2b_v9x::eval(w1, w2, g1, g2, nd, virial),
 * 2b/x2b-v9x.h:83; x3b_v2x::eval, 3b/x3b-v2x.h:85; the MB-nrg classes):
 * n n-mers of one evaluator ("mbpol2b", "mbpol3b", "ch4h2o2b", "ch4ch42b",
 * "ch4h2o3b", the ion types "h2o<ion>2b" / "h2o<ion>3b" / "<halide>h2o2b" /
 * "<halide>h2o3b", "n2o5h2o2b", "n2o5h2o3b", ...; mbx_evaluator_info
 * answers for any name), coordinates
 * xyz[n][nreal*3] with the monomers in evaluator
 * order and already imaged.  grad (same layout, +=), virial (9, +=), e_per
 * (n switched energies) may be NULL.  *energy gets the sum. */
int mbx_evaluate(mbx_ctx* ctx, const char* evaluator, long n, const double* xyz, double* grad, double* virial,
                 double* e_per, double* energy, int flags);

/* Adjoint with respect to the linear coefficients: out[k] += sum_n w[n] *
 * dE_n/da_k (w may be NULL for all ones), monomials recomputed from xyz. */
int mbx_evaluate_dcoef(mbx_ctx* ctx, const char* evaluator, long n, const double* xyz, const double* w,
                       double* out, int flags);

/* Generated-polynomial calling convention (poly_2b_v6x::eval(nd, a, x, t, g),
 * 2b/poly-2b-v6x.h:95): nd configurations, x and g variable-major
 * (x[v*nd + i]), energies in e.  The coefficients in use are the evaluator's
 * current ones (mbx_set_coefficients). */
int mbx_poly(mbx_ctx* ctx, const char* evaluator, long nd, const double* x, double* g, double* e, int flags);

/* Operands of the tensor-core kernel of the mixed mode (MBX_MIXED) for the
 * evaluators that have one ("mbpol3b"): the polynomial in the FP32 basis as a
 * quadratic form m^T C m over a basis of monomials of degree <= 2, C scaled
 * by powers of two and split into FP16 parts in the kernel's shared-memory
 * layout.  Host only (no device needed): *image_bytes and *nb get the image
 * size and the padded basis size; with image, colf and b0 non-NULL the image,
 * the nb per-column factors and the constant term are written for the
 * coefficients coef (ncoef doubles; NULL: the fitted ones), exactly as
 * mbx_set_coefficients uploads them.  MBX_ENOTSUP for other evaluators. */
int mbx_qf_image(const char* evaluator, const double* coef, long* image_bytes, int* nb, unsigned char* image,
                 float* colf, double* b0);

/* Replace the linear coefficients of an evaluator (ncoef doubles; NULL
 * restores the fitted ones).  Coefficients are per device, not per context:
 * they live in the kernels' constant memory and in one global-memory copy
 * for the table-driven kernels, shared by every context on the device, and
 * an alias evaluator shares its target's.  The call takes a process-wide
 * lock and waits until the device is idle before writing, so work in flight
 * on other streams finishes with the old coefficients and later work uses
 * the new ones; two models that need different coefficients for the same
 * evaluator at the same time need two devices (or must take turns).  The
 * first context created on a device loads the fitted coefficients; later
 * contexts keep whatever is set. */
int mbx_set_coefficients(mbx_ctx* ctx, const char* evaluator, const double* a, int flags);
int mbx_evaluator_info(const char* evaluator, int* nbody, int* nreal, int* nvars, int* ncoef);

/* Device-side timing of the last mbx_energy call (ms) split into n-mer build
 * and evaluation, and the number of kernels it launched. */
int mbx_last_timing(const mbx_ctx* ctx, double* ms_build, double* ms_eval, int* kernels);

/* Both terms in one call (no counterpart in the reference, whose
 * System::Energy calls Get2B and Get3B one after the other): the coordinates
 * are wrapped once, then the 2b and the 3b term run side by side on two
 * streams (the 2b term on a child context with its own buffers), so that
 * each fills the SMs the other leaves idle.  Arguments as for mbx_energy;
 * *e2 and *e3 receive the term energies, grad and virial the sum of both
 * terms (+=).  mbx_last_counts gives both terms' counts afterwards;
 * mbx_last_timing the 3b term's. */
int mbx_energy_2b3b(mbx_ctx* ctx, double* xyz, int use_ghost, double* e2, double* e3, double* grad, double* virial,
                    int flags);

/* Batched configurations.  No counterpart in the reference (MBX evaluates
 * one bblock::System per call); for path-integral beads, cluster sets and
 * other independent configurations evaluated together.  The topology given
 * to mbx_set_topology is the concatenation of nconf configurations, all
 * monomers local: configuration k owns monomers conf_mon[k] .. conf_mon[k+1]-1
 * (conf_mon[0] = 0, conf_mon[nconf] = nmon) and has the box boxes[9k..9k+8]
 * when has_box[k] (boxes NULL: no configuration has one; has_box NULL: all
 * have).  Each box must satisfy the cutoff rule of mbx_set_config. */
int mbx_set_batch(mbx_ctx* ctx, int nconf, const int* conf_mon, const double* boxes, const int* has_box);

/* One term (nbody 2 or 3) of every configuration of the batch: the n-mers of
 * each configuration are built inside it (its box, its monomers only), then
 * every evaluator runs once over all configurations' n-mers.  xyz: device
 * site array of the whole batch (wrapped in place per box like mbx_energy);
 * grad: device, += (NULL: energy only); energies[nconf] (host) receive each
 * configuration's term energy, virials[9 nconf] (host, may be NULL) are +=.
 * flags: MBX_DEVICE_PTRS (required), MBX_MIXED, MBX_NO_GRADS, MBX_GRAPH: the
 * device sequence is captured into a CUDA graph after the call and replayed
 * by later calls with the same xyz, grad and flags (re-captured whenever a
 * buffer has to grow). */
int mbx_batch_energy(mbx_ctx* ctx, int nbody, double* xyz, double* grad, double* energies, double* virials,
                     int flags);

/* Both terms of every configuration of the batch in one call, side by side
 * on two streams (the 2b term on a child context mirroring the batch);
 * arguments as for mbx_batch_energy, e2[nconf] and e3[nconf] the term
 * energies, virials the sum of both (+=).  MBX_GRAPH captures both streams'
 * work into one graph. */
int mbx_batch_energy_2b3b(mbx_ctx* ctx, double* xyz, double* grad, double* e2, double* e3, double* virials,
                          int flags);

/* Autotuner of the n-mer builder's launch shapes for one term (no
 * counterpart in the reference): times the term on the current batch (or the
 * whole system when no batch is set) with device arrays xyz/grad and flags as
 * in mbx_batch_energy / mbx_energy, and keeps, axis by axis, the fastest
 * warps per neighbour query (1, 4), unroll depth of the neighbour loop
 * (1, 2, 4) and threads per trimer block (64, 128, 256) or per dimer block.
 * out[4] (may be NULL): nb_warps, nb_unroll, tri_threads, dim_threads;
 * best_ms (may be NULL): the time of the chosen shape. */
int mbx_tune(mbx_ctx* ctx, int nbody, double* xyz, double* grad, int flags, int* out, double* best_ms);
/* The launch shapes in use for a term (out[4] as for mbx_tune), and setting
 * them (e.g. a shape tuned in an earlier run; MBX_EINVAL out of range). */
int mbx_get_knobs(const mbx_ctx* ctx, int nbody, int* out);
int mbx_set_knobs(mbx_ctx* ctx, int nbody, const int* in);

/* No counterpart in the reference.  Evaluator entry point that allocates no
 * device memory, for callers that must not call cudaMalloc (allocator-free
 * real-time loops, fixed memory pools, plugins that may not grow the
 * process's device memory).  Same evaluator calling convention as
 * mbx_evaluate, straight-line evaluators only ("mbpol2b", "mbpol3b",
 * "ch4h2o2b", "ch4h2o3b"), with the coefficients last set on the device by
 * mbx_set_coefficients -- or, where no context and no mbx_set_coefficients
 * call has set them on this device yet, the models' fitted coefficients,
 * which the first call copies into the kernels' constant memory itself (a
 * copy, no allocation); every pointer is device memory owned by the caller;
 * runs on `stream` on the current device:
 *   xyz[n][nreal*3] in, grad (+=, NULL for energy only) and e_per (n
 *   switched energies, may be NULL) out, result[7] out (overwritten):
 *   energy, then virial xx xy xz yy yz zz.
 * The energy is summed over the n-mers in a fixed order (reproducible from
 * call to call).  Scratch lives in one static device array shared by all
 * calls: n must not exceed MBX_NOALLOC_MAX_NMERS (MBX_EINVAL otherwise);
 * calls that overlap on the GPU race on it.  The first call on a device
 * looks up the array's device address (and may load the fitted
 * coefficients, waiting for the device); make that call before any stream
 * capture. */
#define MBX_NOALLOC_MAX_NMERS 262144
int mbx_evaluate_noalloc(const char* evaluator, long n, const double* xyz, double* grad, double* e_per,
                         double* result, void* stream);

/* Measured FMA-pipe throughput of the device (results[0] FP64, results[1]
 * FP32, results[2] FP32 issued as paired fma.rn.f32x2; TFLOP/s): the
 * roofline denominators for the polynomial kernels.  results has 3 slots. */
int mbx_fma_peaks(int device, double* results);

#ifdef __cplusplus
}
#endif
#endif
