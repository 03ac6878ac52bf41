// Host runtime and C ABI of mbx_b200 (declared in include/mbx_b200.h).
//
// A context owns one CUDA stream and the device state the reference keeps in
// bblock::System for the 2-body/3-body path: the topology (first_index_,
// atom tags, local flags, monomer types), the configuration (cutoff2b_,
// cutoff3b_, box_, box_inverse_, ignore_2b_poly_, ignore_3b_poly_) and the
// work buffers.  mbx_energy() is System::Get2B/Get3B: FixMonomerCoordinates,
// the n-mer enumeration, the type dispatch of e2b::get_2b_energy /
// e3b::get_3b_energy and the evaluators, with energy, gradients and virial
// accumulated like grad_ and virial_.
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mbx_b200.h"
#include "holder_kernel.cuh"
#include "nmer_build.h"

// The 1-body term of water (onebody.cu).
struct OneBodyArgs {
    const double* xyz;
    const int* first;
    long n;
    double* grad;
    double* out;
};
int mbx_launch_ps1b(const OneBodyArgs& A, int sms, cudaStream_t s);

// Generic table-driven polynomial over caller-supplied variables
// (table_kernels.cu).
int mbx_launch_poly_table(long nd, int nvars, const double* x, double* g, double* e, const int4* terms,
                          const double* tcoef, long nterms, const double* coef, int pairs, int sms, cudaStream_t s);

typedef int (*launch_fn)(const HolderArgs&, int, int, cudaStream_t);
typedef int (*dcoef_fn)(const HolderArgs&, const double*, double*, int, int, cudaStream_t);
typedef int (*prime_fn)(cudaStream_t);
typedef int (*warp_fn)(const HolderArgs&, int, int, cudaStream_t);
typedef int (*setcoef_fn)(const double*, int, cudaStream_t);

struct EvaluatorInfo {
    const char* name;
    int nbody;
    const char* ids[3];
    double rf;
    int skip;
    int ncoef, nreal, nvars;
    const double* fit;
    launch_fn g, e;   // straight-line FP64 kernels (energy + gradient, energy only), or null
    dcoef_fn c;       // coefficient adjoint (table-driven)
    warp_fn w;        // table-driven evaluation of the types without straight-line kernels, or null
    launch_fn s;      // FP32 kernel of the mixed mode (FP32 basis), or null
    double split_r;   // mixed mode: n-mers with first-atom distance below this run in FP64 (0: none)
    prime_fn pg, pe, ps;   // code prefetch of the g, e and s kernels (holder_prime_kernel), or null
    setcoef_fn set[7];     // constant-memory coefficient setters of the straight-line kernels
    int table;        // term table (mbx_term_tables)
    int kern;         // evaluator whose kernels and coefficients this one runs (itself or an alias target)
};

#include "gen/registry.inc"
#include "gen/terms_index.inc"
#include "device_state.h"

#define MBX_VERSION_STRING "mbx_b200 0.1 (sm_100a)"

namespace {

// Incremented whenever a device buffer is reallocated: a captured graph holds
// the old addresses and is re-captured when this has moved on.
std::atomic<unsigned long> g_realloc_gen{0};

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t ensure(size_t want) {
        if (want <= n && p) return cudaSuccess;
        size_t m = std::max(want, n + n / 2);
        if (m == 0) m = 1;
        g_realloc_gen.fetch_add(1);
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, m * sizeof(T));
        if (e == cudaSuccess) n = m;
        return e;
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

const EvaluatorInfo* find_evaluator(const char* name) {
    for (int i = 0; i < mbx_num_evaluators; ++i)
        if (!strcmp(mbx_evaluators[i].name, name)) return &mbx_evaluators[i];
    return nullptr;
}

constexpr int kMaxDevices = 64;
std::mutex g_dev_mu;
bool g_dev_constants[kMaxDevices] = {false};
DeviceTables g_dev_tables[kMaxDevices];
long g_coef_off[256];
long g_coef_off_1b[16];
long g_coef_total = -1;

void coef_layout() {
    if (g_coef_total >= 0) return;
    long off = 0;
    for (int i = 0; i < mbx_num_evaluators; ++i) {
        g_coef_off[i] = off;
        off += mbx_evaluators[i].ncoef;
    }
    for (int i = 0; i < mbx_num_onebody; ++i) {
        g_coef_off_1b[i] = off;
        off += mbx_onebody[i].ncoef;
    }
    g_coef_total = off;
}

}  // namespace

// The embedded term tables (gen/terms_blob.cpp).
extern "C" const unsigned char mbx_terms_blob[];

std::mutex& mbx_device_mutex() { return g_dev_mu; }

long mbx_coef_offset(int evaluator) {
    coef_layout();
    return g_coef_off[evaluator];
}

// Caller holds g_dev_mu.
static int device_constants_locked(int dev) {
    if (dev < 0 || dev >= kMaxDevices) return MBX_EINVAL;
    if (g_dev_constants[dev]) return MBX_OK;
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) return MBX_ENODEV;
    if (cur != dev && cudaSetDevice(dev) != cudaSuccess) return MBX_ECUDA;
    int rc = MBX_OK;
    for (int i = 0; i < mbx_num_evaluators && rc == MBX_OK; ++i) {
        const EvaluatorInfo& E = mbx_evaluators[i];
        if (E.kern != i) continue;   // an alias shares its target's kernels and coefficients
        for (int v = 0; v < 7; ++v)
            if (E.set[v] && E.set[v](E.fit, 0, nullptr) != 0) rc = MBX_ECUDA;
    }
    if (rc == MBX_OK && cudaDeviceSynchronize() != cudaSuccess) rc = MBX_ECUDA;
    if (rc == MBX_OK) g_dev_constants[dev] = true;
    if (cur != dev) cudaSetDevice(cur);
    return rc;
}

int mbx_device_constants(int dev) {
    std::lock_guard<std::mutex> lock(g_dev_mu);
    return device_constants_locked(dev);
}

int mbx_device_tables(int dev, DeviceTables* out) {
    std::lock_guard<std::mutex> lock(g_dev_mu);
    int rc = device_constants_locked(dev);
    if (rc) return rc;
    DeviceTables& T = g_dev_tables[dev];
    if (!T.blob) {
        coef_layout();
        int cur = 0;
        if (cudaGetDevice(&cur) != cudaSuccess) return MBX_ENODEV;
        if (cur != dev && cudaSetDevice(dev) != cudaSuccess) return MBX_ECUDA;
        void* blob = nullptr;
        void* coef = nullptr;
        cudaError_t e = cudaMalloc(&blob, (size_t)mbx_terms_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&coef, (size_t)g_coef_total * sizeof(double));
        if (e == cudaSuccess) e = cudaMemcpy(blob, mbx_terms_blob, (size_t)mbx_terms_bytes, cudaMemcpyHostToDevice);
        for (int i = 0; i < mbx_num_evaluators && e == cudaSuccess; ++i)
            e = cudaMemcpy(static_cast<double*>(coef) + g_coef_off[i], mbx_evaluators[i].fit,
                           mbx_evaluators[i].ncoef * sizeof(double), cudaMemcpyHostToDevice);
        for (int i = 0; i < mbx_num_onebody && e == cudaSuccess; ++i)
            e = cudaMemcpy(static_cast<double*>(coef) + g_coef_off_1b[i], mbx_onebody[i].fit,
                           mbx_onebody[i].ncoef * sizeof(double), cudaMemcpyHostToDevice);
        if (cur != dev) cudaSetDevice(cur);
        if (e != cudaSuccess) {
            if (blob) cudaFree(blob);
            if (coef) cudaFree(coef);
            return MBX_ECUDA;
        }
        T.blob = static_cast<const unsigned char*>(blob);
        T.coef = static_cast<double*>(coef);
    }
    *out = T;
    return MBX_OK;
}

namespace {

// Slot order the reference's dispatch sorts the monomer ids into
// (e2b::get_2b_energy, potential/2b/energy2b.cpp:240-254;
//  e3b::get_3b_energy, potential/3b/energy3b.cpp:185-216).
void sorted_slots(int nb, const std::string* ids, int* idx) {
    if (nb == 2) {
        if (ids[1] < ids[0]) { idx[0] = 1; idx[1] = 0; } else { idx[0] = 0; idx[1] = 1; }
        return;
    }
    std::string m[3] = {ids[0], ids[1], ids[2]};
    int k[3] = {0, 1, 2};
    if (m[2] < m[0] && m[2] < m[1]) { std::swap(m[0], m[2]); std::swap(k[0], k[2]); }
    if (m[0] > m[1] && m[0] > m[2]) {
        std::swap(m[0], m[2]); std::swap(k[0], k[2]);
    } else if (m[1] > m[0] && m[1] > m[2]) {
        std::swap(m[1], m[2]); std::swap(k[1], k[2]);
    }
    if (m[0] > m[1]) { std::swap(m[0], m[1]); std::swap(k[0], k[1]); }
    for (int i = 0; i < 3; ++i) idx[i] = k[i];
}

}  // namespace

// Scratch of one n-mer search (cloud, cell list, matches).  A context owns
// several, so that the searches of a batch's configurations can run side by
// side on their own streams.
struct BuildScratch {
    DevBuf<double> cloud;
    DevBuf<int> cell_of, cell_count, cell_start, cell_fill, cell_items, cell_sorted, nb_count, copy_dir;
    DevBuf<NbEntry> nb;
    void release() {
        cloud.release();
        copy_dir.release();
        cell_of.release();
        cell_count.release();
        cell_start.release();
        cell_fill.release();
        cell_items.release();
        cell_sorted.release();
        nb_count.release();
        nb.release();
    }
};
// pinned result block (h_out, 64 doubles): [0..7) term energy + virial, [8]
// listed n-mers, then the bucket counts (ints) and the status words (2 ints)
#define MBX_H_COUNTS 9
#define MBX_H_STATUS (MBX_H_COUNTS + (MBX_MAX_BUCKETS + 1) / 2)
static_assert(MBX_H_STATUS + 1 <= 64, "pinned result block too small");

struct mbx_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int sm_count = 148;
    std::string err;

    // topology
    int nmon = 0, numsites = 0, ntypes = 0;
    std::string type_names[MBX_MAX_TYPES];
    std::vector<int> h_first, h_nat, h_tag, h_type, h_local;
    DevBuf<int> d_first, d_nat, d_tag, d_type;
    DevBuf<int> d_members[2], d_query[2];
    int nmem[2] = {0, 0}, nquery[2] = {0, 0};

    // configuration
    double cutoff[4] = {0, 0, 9.0, 7.0};  // indexed by nbody
    BoxParams bp{};
    std::vector<std::vector<std::string>> ignore[4];
    std::vector<std::string> ignore1b;   // monomer types without a 1-body term (ignore_1b_poly_)
    // input (real-atom) order of the caller: site of every real atom (mbx_set_real_order)
    int numat = 0;
    DevBuf<int> d_real2site;
    DevBuf<double> xreal, greal, gsite;
    // 1-body term: first sites of the local waters, then of the local
    // monomers of each table-driven 1-body evaluator (n1b[i] of them), built
    // for topology generation w1b_gen
    DevBuf<int> d_w1b;
    long n_w1b = 0;
    long n1b[16] = {0};
    unsigned long w1b_gen = ~0ul;

    // per-term dispatch
    int nbucket[4] = {0, 0, 0, 0};
    const EvaluatorInfo* bucket_eval[4][MBX_MAX_BUCKETS];
    bool bucket_near[4][MBX_MAX_BUCKETS];   // the FP64 short-range share of a split evaluator
    DimerRules drules{};
    TrimerRules trules{};
    long bucket_cap[4][MBX_MAX_BUCKETS];

    // work buffers
    DevBuf<double> xyz, grad, out, coef_ws;
    DevBuf<int> bucket_count, status, counters;
    BuildScratch scratch;   // of every search (a batch searches all its configurations at once)
    // code prefetch of a term's evaluation kernels, beside its n-mer search
    cudaStream_t prime_stream = nullptr;
    cudaEvent_t prime_fork = nullptr, prime_join = nullptr;
    // mbx_energy_2b3b: the 2b term on a child context, kept in step with this
    // one (gen counts topology/configuration changes)
    mbx_ctx* child = nullptr;
    unsigned long gen = 0, child_gen = ~0ul;
    cudaEvent_t ev_fork = nullptr;
    DevBuf<int4> buckets, list;
    DevBuf<unsigned long long> listed;
    DeviceTables tables;   // per-device term tables and coefficients (shared, not owned)
    DevBuf<unsigned char> pair_scratch;   // between the three mixed-precision kernels
    int nb_cap = 192;
    // runtime launch shapes of the builder (set by mbx_tune)
    struct Knobs {
        int nb_warps = 4, nb_unroll = 2, tri_threads = 128, dim_threads = 128;
    } knobs[4];         // per term (indexed by nbody)
    double* h_out = nullptr;  // pinned: [0..7] term outputs, [8..15] counters
    double* h_grad = nullptr;  // pinned staging of the gradient of a call with host arrays
    size_t h_grad_n = 0;
    cudaEvent_t ev[3];


    // batched configurations: configuration k owns monomers conf_mon[k] ..
    // conf_mon[k+1]-1 and has box conf_bp[k]
    int nconf = 0;
    std::vector<int> conf_mon;
    std::vector<BoxParams> conf_bp;
    DevBuf<BoxParams> d_conf_bp;
    // batched search: every configuration's grid for the term's cutoff, its
    // cells concatenated (ncell in all), built for context generation gen
    DevBuf<BatchGrid> d_bgrid[4];
    int bgrid_ncell[4] = {0, 0, 0, 0};
    unsigned long bgrid_gen[4] = {0, 0, 0, 0};
    double bgrid_cut[4] = {0, 0, 0, 0};
    DevBuf<int> d_mon_conf;
    DevBuf<double> conf_out;
    double* h_conf = nullptr;   // pinned, 8 per configuration
    // captured batch sequences (per term), replayed while the key matches
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        const double* xyz = nullptr;
        const double* grad = nullptr;
        int flags = 0;
        unsigned long gen = 0;
    } graph[4];

    // results of the last call
    long last_listed[4] = {0, 0, 0, 0};
    long last_evaluated[4] = {0, 0, 0, 0};
    float last_ms_build = 0, last_ms_eval = 0;
    int last_kernels = 0;
};

static int fail(mbx_ctx* c, int code, const std::string& msg) {
    if (c) c->err = msg;
    return code;
}

#define CUCHK(c, expr)                                                                        \
    do {                                                                                      \
        cudaError_t _e = (expr);                                                              \
        if (_e != cudaSuccess)                                                                \
            return fail(c, MBX_ECUDA, std::string(#expr) + ": " + cudaGetErrorString(_e));    \
    } while (0)

#define RCHK(c, expr)                                                                         \
    do {                                                                                      \
        int _r = (expr);                                                                      \
        if (_r != 0)                                                                          \
            return fail(c, MBX_ECUDA, std::string(#expr) + ": " + cudaGetErrorString((cudaError_t)_r)); \
    } while (0)

extern "C" {

const char* mbx_version(void) { return MBX_VERSION_STRING; }

const char* mbx_last_error(const mbx_ctx* c) { return c ? c->err.c_str() : "null context"; }

int mbx_create(mbx_ctx** out, int device, void* stream) {
    if (!out) return MBX_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MBX_ENODEV;
    if (device < 0 || device >= ndev) return MBX_EINVAL;
    mbx_ctx* c = new mbx_ctx();
    c->device = device;
    CUCHK(c, cudaSetDevice(device));
    CUCHK(c, cudaDeviceGetAttribute(&c->sm_count, cudaDevAttrMultiProcessorCount, device));
    if (stream) {
        c->stream = (cudaStream_t)stream;
    } else {
        CUCHK(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    CUCHK(c, cudaMallocHost(&c->h_out, 64 * sizeof(double)));
    for (int i = 0; i < 3; ++i) CUCHK(c, cudaEventCreate(&c->ev[i]));
    CUCHK(c, cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
    CUCHK(c, cudaStreamCreateWithFlags(&c->prime_stream, cudaStreamNonBlocking));
    CUCHK(c, cudaEventCreateWithFlags(&c->prime_fork, cudaEventDisableTiming));
    CUCHK(c, cudaEventCreateWithFlags(&c->prime_join, cudaEventDisableTiming));

    CUCHK(c, c->out.ensure(64));
    CUCHK(c, c->status.ensure(4));
    CUCHK(c, c->counters.ensure(MBX_MAX_BUCKETS));
    CUCHK(c, c->listed.ensure(4));
    for (int nb = 0; nb < 4; ++nb)
        for (int b = 0; b < MBX_MAX_BUCKETS; ++b) c->bucket_cap[nb][b] = 0;
    // the fitted coefficients (constant banks, per device: loaded by the
    // first context on a device, kept by later ones) and the term tables
    {
        const int r = mbx_device_tables(device, &c->tables);
        if (r) {
            mbx_destroy(c);
            return r;
        }
    }
    CUCHK(c, cudaStreamSynchronize(c->stream));
    *out = c;
    return MBX_OK;
}

int mbx_destroy(mbx_ctx* c) {
    if (!c) return MBX_OK;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    DevBuf<int>* ib[] = {&c->d_first, &c->d_nat, &c->d_tag, &c->d_type, &c->d_members[0], &c->d_members[1],
                         &c->d_query[0], &c->d_query[1], &c->bucket_count, &c->status, &c->counters};
    for (auto* b : ib) b->release();
    DevBuf<double>* db[] = {&c->xyz, &c->grad, &c->out, &c->coef_ws};
    for (auto* b : db) b->release();
    c->scratch.release();
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->prime_stream) {
        cudaStreamSynchronize(c->prime_stream);
        cudaStreamDestroy(c->prime_stream);
    }
    if (c->prime_fork) cudaEventDestroy(c->prime_fork);
    if (c->prime_join) cudaEventDestroy(c->prime_join);
    if (c->child) mbx_destroy(c->child);
    c->pair_scratch.release();
    c->buckets.release();
    c->list.release();
    c->listed.release();
    c->d_conf_bp.release();
    c->d_mon_conf.release();
    for (auto& g : c->d_bgrid) g.release();
    c->conf_out.release();
    if (c->h_out) cudaFreeHost(c->h_out);
    if (c->h_grad) cudaFreeHost(c->h_grad);
    for (int i = 0; i < 3; ++i) cudaEventDestroy(c->ev[i]);
    for (auto& gr : c->graph)
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
    if (c->h_conf) cudaFreeHost(c->h_conf);
    if (c->own_stream) cudaStreamDestroy(c->stream);
    delete c;
    return MBX_OK;
}

int mbx_evaluator_info(const char* name, int* nbody, int* nreal, int* nvars, int* ncoef) {
    const EvaluatorInfo* E = name ? find_evaluator(name) : nullptr;
    if (!E) return MBX_ENOTSUP;
    if (nbody) *nbody = E->nbody;
    if (nreal) *nreal = E->nreal;
    if (nvars) *nvars = E->nvars;
    if (ncoef) *ncoef = E->ncoef;
    return MBX_OK;
}

}  // extern "C"

// Dispatch tables for the current topology and ignore lists.
static int build_rules(mbx_ctx* c) {
    for (int nb = 2; nb <= 3; ++nb) {
        c->nbucket[nb] = 0;
        for (int b = 0; b < MBX_MAX_BUCKETS; ++b) c->bucket_near[nb][b] = false;
        const int T = c->ntypes;
        const int ncode = nb == 2 ? T * T : T * T * T;
        for (int code = 0; code < (nb == 2 ? MBX_MAX_TYPES * MBX_MAX_TYPES : MBX_MAX_TYPES * MBX_MAX_TYPES * MBX_MAX_TYPES);
             ++code) {
            if (nb == 2) { c->drules.bucket[code] = -1; c->drules.swap[code] = 0; }
            else { c->trules.bucket[code] = -1; c->trules.perm[code] = 0; }
        }
        for (int code = 0; code < ncode; ++code) {
            std::string ids[3];
            // code enumerates (slot0 slowest): reconstruct the original order
            if (nb == 2) { ids[0] = c->type_names[code / T]; ids[1] = c->type_names[code % T]; }
            else {
                ids[0] = c->type_names[code / (T * T)];
                ids[1] = c->type_names[(code / T) % T];
                ids[2] = c->type_names[code % T];
            }
            int so[3];
            sorted_slots(nb, ids, so);
            std::vector<std::string> sorted_ids;
            for (int s = 0; s < nb; ++s) sorted_ids.push_back(ids[so[s]]);
            // ignored tuples are skipped after the search (system.cpp:2606-2618,2940-2952)
            bool ignored = false;
            for (auto& ig : c->ignore[nb]) {
                std::vector<std::string> a = ig, b = sorted_ids;
                std::sort(a.begin(), a.end());
                std::sort(b.begin(), b.end());
                if (a == b) ignored = true;
            }
            const EvaluatorInfo* E = nullptr;
            for (int i = 0; i < mbx_num_evaluators && !ignored; ++i) {
                const EvaluatorInfo& X = mbx_evaluators[i];
                if (X.nbody != nb) continue;
                std::vector<std::string> a(X.ids, X.ids + nb), b = sorted_ids;
                std::sort(a.begin(), a.end());
                if (a == b) E = &X;
            }
            if (!E) continue;  // unknown tuples evaluate to 0 (energy2b.cpp:370, energy3b.cpp:258)
            // evaluator slot h <- sorted slot: first unused sorted slot with the same id
            int holder_from_orig[3];
            bool used[3] = {false, false, false};
            for (int h = 0; h < nb; ++h) {
                for (int s = 0; s < nb; ++s) {
                    if (!used[s] && sorted_ids[s] == E->ids[h]) {
                        used[s] = true;
                        holder_from_orig[h] = so[s];
                        break;
                    }
                }
            }
            int b = -1;
            for (int k = 0; k < c->nbucket[nb]; ++k)
                if (c->bucket_eval[nb][k] == E) b = k;
            if (b < 0) {
                if (c->nbucket[nb] == MBX_MAX_BUCKETS) return fail(c, MBX_ENOTSUP, "too many evaluator buckets");
                b = c->nbucket[nb]++;
                c->bucket_eval[nb][b] = E;
            }
            const int dcode = nb == 2 ? (code / T) * MBX_MAX_TYPES + code % T
                                      : ((code / (T * T)) * MBX_MAX_TYPES + (code / T) % T) * MBX_MAX_TYPES + code % T;
            if (nb == 2) {
                c->drules.bucket[dcode] = b;
                c->drules.swap[dcode] = holder_from_orig[0] == 1;
            } else {
                c->trules.bucket[dcode] = b;
                c->trules.perm[dcode] = holder_from_orig[0] | (holder_from_orig[1] << 2) | (holder_from_orig[2] << 4);
            }
        }
        for (int b = 0; b < c->nbucket[nb]; ++b) {
            const EvaluatorInfo* E = c->bucket_eval[nb][b];
            const double pre = E->rf + 1e-6;
            if (nb == 2) c->drules.pre2[b] = pre * pre;
            else {
                c->trules.pre2[b] = pre * pre;
                c->trules.skip[b] = E->skip;
            }
        }
        if (nb == 2) {
            // mixed mode: a second bucket per split evaluator takes the dimers
            // closer than split_r (evaluated in FP64); unused otherwise
            const int nmain = c->nbucket[2];
            for (int b = 0; b < MBX_MAX_BUCKETS; ++b) {
                c->drules.near[b] = -1;
                c->drules.split2[b] = 0.0;
            }
            for (int b = 0; b < nmain; ++b) {
                const EvaluatorInfo* E = c->bucket_eval[2][b];
                if (!(E->split_r > 0) || !E->s) continue;
                if (c->nbucket[2] == MBX_MAX_BUCKETS) return fail(c, MBX_ENOTSUP, "too many evaluator buckets");
                const int nbk = c->nbucket[2]++;
                c->bucket_eval[2][nbk] = E;
                c->bucket_near[2][nbk] = true;
                c->drules.pre2[nbk] = c->drules.pre2[b];
                c->drules.near[b] = nbk;
                c->drules.split2[b] = E->split_r * E->split_r;
            }
        }
    }
    return MBX_OK;
}

extern "C" int mbx_set_topology(mbx_ctx* c, int nmon, const char* const* ids, const int* first_index, const int* tag,
                                const int* is_local, int numsites) {
    if (!c || nmon <= 0 || !ids || !first_index || !tag || numsites <= 0) return fail(c, MBX_EINVAL, "bad topology");
    CUCHK(c, cudaSetDevice(c->device));
    c->nmon = nmon;
    c->numsites = numsites;
    c->ntypes = 0;
    c->h_first.assign(first_index, first_index + nmon);
    c->h_tag.assign(tag, tag + nmon);
    c->h_local.assign(nmon, 1);
    if (is_local) c->h_local.assign(is_local, is_local + nmon);
    c->h_type.resize(nmon);
    c->h_nat.resize(nmon);
    for (int m = 0; m < nmon; ++m) {
        std::string id = ids[m];
        int nat = 0;
        for (int k = 0; k < mbx_num_monomers; ++k)
            if (id == mbx_monomers[k].id) nat = mbx_monomers[k].nat;
        if (!nat) return fail(c, MBX_ENOTSUP, "unknown monomer id " + id);
        c->h_nat[m] = nat;
        int t = -1;
        for (int k = 0; k < c->ntypes; ++k)
            if (c->type_names[k] == id) t = k;
        if (t < 0) {
            if (c->ntypes == MBX_MAX_TYPES) return fail(c, MBX_ENOTSUP, "too many monomer types");
            t = c->ntypes;
            c->type_names[c->ntypes++] = id;
        }
        c->h_type[m] = t;
        if (first_index[m] < 0 || first_index[m] + nat > numsites) return fail(c, MBX_EINVAL, "first_index out of range");
    }
    CUCHK(c, c->d_first.ensure(nmon));
    CUCHK(c, c->d_nat.ensure(nmon));
    CUCHK(c, c->d_tag.ensure(nmon));
    CUCHK(c, c->d_type.ensure(nmon));
    CUCHK(c, cudaMemcpyAsync(c->d_first.p, c->h_first.data(), nmon * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUCHK(c, cudaMemcpyAsync(c->d_nat.p, c->h_nat.data(), nmon * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUCHK(c, cudaMemcpyAsync(c->d_tag.p, c->h_tag.data(), nmon * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUCHK(c, cudaMemcpyAsync(c->d_type.p, c->h_type.data(), nmon * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    // search members and queries (AddClusters, sys_tools.cpp:502-517,535-537):
    // use_ghost = 0: members and queries are the local monomers;
    // use_ghost = 1: all monomers are members, the local ones query.
    for (int g = 0; g < 2; ++g) {
        std::vector<int> mem, qry;
        for (int m = 0; m < nmon; ++m)
            if (g || c->h_local[m]) mem.push_back(m);
        for (int q = 0; q < (int)mem.size(); ++q)
            if (c->h_local[mem[q]]) qry.push_back(q);
        c->nmem[g] = (int)mem.size();
        c->nquery[g] = (int)qry.size();
        CUCHK(c, c->d_members[g].ensure(mem.size() + 1));
        CUCHK(c, c->d_query[g].ensure(qry.size() + 1));
        if (!mem.empty())
            CUCHK(c, cudaMemcpyAsync(c->d_members[g].p, mem.data(), mem.size() * sizeof(int), cudaMemcpyHostToDevice,
                                     c->stream));
        if (!qry.empty())
            CUCHK(c, cudaMemcpyAsync(c->d_query[g].p, qry.data(), qry.size() * sizeof(int), cudaMemcpyHostToDevice,
                                     c->stream));
    }
    CUCHK(c, cudaStreamSynchronize(c->stream));
    for (int nb = 0; nb < 4; ++nb)
        for (int b = 0; b < MBX_MAX_BUCKETS; ++b) c->bucket_cap[nb][b] = 0;
    ++c->gen;
    return build_rules(c);
}

static int invert_box(const double* b, double* inv) {
    // InvertUnitCell (tools/math_tools.cpp:37-64), same operation order
    volatile double det = b[0] * (b[4] * b[8] - b[7] * b[5]) - b[1] * (b[3] * b[8] - b[5] * b[6]) +
                          b[2] * (b[3] * b[7] - b[4] * b[6]);
    if (std::fabs(det) < 1e-36) return 1;
    const double di = 1 / det;
    inv[0] = (b[4] * b[8] - b[7] * b[5]) * di;
    inv[1] = (b[2] * b[7] - b[1] * b[8]) * di;
    inv[2] = (b[1] * b[5] - b[2] * b[4]) * di;
    inv[3] = (b[5] * b[6] - b[3] * b[8]) * di;
    inv[4] = (b[0] * b[8] - b[2] * b[6]) * di;
    inv[5] = (b[3] * b[2] - b[0] * b[5]) * di;
    inv[6] = (b[3] * b[7] - b[6] * b[4]) * di;
    inv[7] = (b[6] * b[1] - b[0] * b[7]) * di;
    inv[8] = (b[0] * b[4] - b[3] * b[1]) * di;
    return 0;
}

// BoxParams of a box (NULL: no periodic boundaries).  The search finds at
// most one image of each monomer only while the cutoff rc is below half of
// every box height (sys_tools.cpp:553-555): MBX_EDOM otherwise.
static int make_box(mbx_ctx* c, const double* box, double rc, BoxParams* out) {
    memset(out, 0, sizeof(*out));
    out->use_pbc = box ? 1 : 0;
    if (!box) return MBX_OK;
    for (int i = 0; i < 9; ++i) out->box[i] = box[i];
    if (invert_box(box, out->inv)) return fail(c, MBX_EINVAL, "Matrix has no inverse. Determinant is 0");
    const double* a = box;
    const double* bb = box + 3;
    const double* cc = box + 6;
    auto cross = [](const double* u, const double* v, double* w) {
        w[0] = u[1] * v[2] - u[2] * v[1];
        w[1] = u[2] * v[0] - u[0] * v[2];
        w[2] = u[0] * v[1] - u[1] * v[0];
    };
    double bc[3], ca[3], ab[3];
    cross(bb, cc, bc);
    cross(cc, a, ca);
    cross(a, bb, ab);
    const double vol = std::fabs(a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2]);
    const double h[3] = {vol / std::sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]),
                         vol / std::sqrt(ca[0] * ca[0] + ca[1] * ca[1] + ca[2] * ca[2]),
                         vol / std::sqrt(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2])};
    for (int k = 0; k < 3; ++k)
        if (2.0 * rc >= h[k])
            return fail(c, MBX_EDOM, "cutoff " + std::to_string(rc) + " is not below half the box height " +
                                         std::to_string(h[k]));
    return MBX_OK;
}

static void drop_graphs(mbx_ctx* c);

extern "C" int mbx_set_config(mbx_ctx* c, double cutoff2b, double cutoff3b, const double* box, int n2,
                              const char* const* ignore2b, int n3, const char* const* ignore3b) {
    if (!c || !(cutoff2b >= 0) || !(cutoff3b >= 0)) return fail(c, MBX_EINVAL, "bad cutoffs");
    c->cutoff[2] = cutoff2b;
    c->cutoff[3] = cutoff3b;
    int r = make_box(c, box, std::max(cutoff2b, cutoff3b), &c->bp);
    if (r) return r;
    ++c->gen;
    // captured batch graphs hold the old cutoffs, rules and search grids
    drop_graphs(c);
    c->ignore[2].clear();
    c->ignore[3].clear();
    for (int i = 0; i < n2; ++i) c->ignore[2].push_back({ignore2b[2 * i], ignore2b[2 * i + 1]});
    for (int i = 0; i < n3; ++i) c->ignore[3].push_back({ignore3b[3 * i], ignore3b[3 * i + 1], ignore3b[3 * i + 2]});
    if (c->nmon) return build_rules(c);
    return MBX_OK;
}

// Cell grid for a search of radius rc in box bp.
static CellGrid make_grid(const BoxParams& bp, double rc, int nmem) {
    CellGrid g{};
    if (bp.use_pbc) {
        const double* a = bp.box;
        const double* b = bp.box + 3;
        const double* cc = bp.box + 6;
        auto cross = [](const double* u, const double* v, double* w) {
            w[0] = u[1] * v[2] - u[2] * v[1];
            w[1] = u[2] * v[0] - u[0] * v[2];
            w[2] = u[0] * v[1] - u[1] * v[0];
        };
        double bc[3], ca[3], ab[3];
        cross(b, cc, bc);
        cross(cc, a, ca);
        cross(a, b, ab);
        const double vol = std::fabs(a[0] * bc[0] + a[1] * bc[1] + a[2] * bc[2]);
        const double h[3] = {vol / std::sqrt(bc[0] * bc[0] + bc[1] * bc[1] + bc[2] * bc[2]),
                             vol / std::sqrt(ca[0] * ca[0] + ca[1] * ca[1] + ca[2] * ca[2]),
                             vol / std::sqrt(ab[0] * ab[0] + ab[1] * ab[1] + ab[2] * ab[2])};
        for (int k = 0; k < 3; ++k) g.n[k] = std::max(1, std::min(64, (int)std::floor(h[k] / rc)));
        // one cloud point per candidate when every axis has 3 or more cells,
        // each wider than the cutoff by a margin far above rounding (the
        // search then tests only the copy the cell's wrap implies)
        g.one_copy = 1;
        for (int k = 0; k < 3; ++k)
            if (g.n[k] < 3 || h[k] / g.n[k] < rc * (1.0 + 1e-9)) g.one_copy = 0;
    } else {
        // hashed grid: cell = floor(x / rc) mod n on every axis
        const int n = std::max(3, std::min(32, (int)std::ceil(std::cbrt((double)nmem / 2.0))));
        for (int k = 0; k < 3; ++k) {
            g.n[k] = n;
            g.lo[k] = rc;
            g.inv_extent[k] = 1.0 / rc;
        }
    }
    return g;
}

// Bucket capacities (grown on overflow; first guess from the query count)
// and offsets of one term; zeroes the bucket counters and the status word.
static int prepare_buckets(mbx_ctx* c, int nbody, long nq_guess, long list_cap) {
    CUCHK(c, c->bucket_count.ensure(MBX_MAX_BUCKETS));
    long total = 0;
    for (int b = 0; b < c->nbucket[nbody]; ++b) {
        if (c->bucket_cap[nbody][b] == 0) c->bucket_cap[nbody][b] = std::max(nq_guess, 1L) * (nbody == 2 ? 40 : 80);
        total += c->bucket_cap[nbody][b];
    }
    CUCHK(c, c->buckets.ensure(std::max(total, 1L)));
    long off = 0;
    for (int b = 0; b < c->nbucket[nbody]; ++b) {
        if (nbody == 2) { c->drules.offset[b] = off; c->drules.cap[b] = (int)c->bucket_cap[2][b]; }
        else { c->trules.offset[b] = off; c->trules.cap[b] = (int)c->bucket_cap[3][b]; }
        off += c->bucket_cap[nbody][b];
    }
    if (list_cap > 0) CUCHK(c, c->list.ensure(list_cap));
    CUCHK(c, cudaMemsetAsync(c->bucket_count.p, 0, MBX_MAX_BUCKETS * sizeof(int), c->stream));
    CUCHK(c, cudaMemsetAsync(c->listed.p, 0, 4 * sizeof(unsigned long long), c->stream));
    CUCHK(c, cudaMemsetAsync(c->status.p, 0, 4 * sizeof(int), c->stream));
    return MBX_OK;
}

// One search: the monomers members[0..nmem) (global ids) searched around
// the queries query[0..nq) (positions in members), in box bp.
struct BuildScope {
    const int* members;
    int nmem;
    const int* query;
    int nq;
    BoxParams bp;
};

// Enumerates the n-mers of one scope into the evaluator buckets (appending:
// the counters are zeroed by prepare_buckets) and, when list_cap > 0, into
// c->list.  Asynchronous; status and counts on device.
static int launch_build_scope(mbx_ctx* c, int nbody, const BuildScope& S, const double* xyz, long list_cap,
                              int* kernels, bool mixed) {
    BuildScratch& B = c->scratch;
    cudaStream_t st = c->stream;
    const int nmem = S.nmem, nq = S.nq;
    if (nmem < 2 || (nbody == 3 && nmem < 3) || nq == 0) return MBX_OK;
    const double rc = c->cutoff[nbody];
    const double rc2 = rc * rc;
    CellGrid cg = make_grid(S.bp, rc, nmem);
    const int ncell = cg.n[0] * cg.n[1] * cg.n[2];
    CUCHK(c, B.cloud.ensure((size_t)std::max(nmem, 1) * 24));
    CUCHK(c, B.copy_dir.ensure(std::max(nmem, 1)));
    CUCHK(c, B.cell_of.ensure(std::max(nmem, 1)));
    CUCHK(c, B.cell_items.ensure(std::max(nmem, 1)));
    CUCHK(c, B.cell_sorted.ensure(std::max(nmem, 1)));
    CUCHK(c, B.cell_count.ensure(ncell + 1));
    CUCHK(c, B.cell_start.ensure(ncell + 1));
    CUCHK(c, B.cell_fill.ensure(ncell + 1));
    CUCHK(c, B.nb_count.ensure(std::max(nq, 1)));
    CUCHK(c, B.nb.ensure((size_t)std::max(nq, 1) * c->nb_cap));
    CUCHK(c, cudaMemsetAsync(B.cell_count.p, 0, (ncell + 1) * sizeof(int), st));
    const int T = 128;
    k_cloud<<<(nmem + T - 1) / T, T, 0, st>>>(xyz, c->d_first.p, S.members, nmem, S.bp, cg, B.cloud.p,
                                                     B.cell_of.p, B.copy_dir.p);
    k_cell_count<<<(nmem + T - 1) / T, T, 0, st>>>(B.cell_of.p, nmem, B.cell_count.p);
    k_cell_scan<<<1, 1024, 0, st>>>(B.cell_count.p, ncell, B.cell_start.p, B.cell_fill.p);
    k_cell_fill<<<(nmem + T - 1) / T, T, 0, st>>>(B.cell_of.p, nmem, B.cell_fill.p, B.cell_items.p);
    k_cell_sort<<<(ncell * 32 + T - 1) / T, T, 0, st>>>(B.cell_start.p, ncell, B.cell_items.p,
                                                                B.cell_sorted.p);
    // neighbour search: warps per query and unroll depth are tunable; one
    // warp when four staging areas would not fit in shared memory
    const auto& K = c->knobs[nbody];
    const int nbw = (size_t)4 * c->nb_cap * sizeof(NbEntry) <= 160 * 1024 ? K.nb_warps : 1;
    if ((size_t)c->nb_cap * sizeof(NbEntry) > 227 * 1024) return fail(c, MBX_ENOMEM, "neighbour staging");
    RCHK(c, launch_neighbors(nbw, K.nb_unroll, B.cloud.p, B.copy_dir.p, B.cell_of.p, B.cell_start.p, B.cell_sorted.p,
                             S.query, nq, cg, S.bp.use_pbc, rc2, c->nb_cap, B.nb_count.p, B.nb.p, c->status.p,
                             st));
    if (nbody == 2) {
        DimerRules R = c->drules;
        if (!mixed)
            for (int b = 0; b < MBX_MAX_BUCKETS; ++b) R.split2[b] = 0.0;   // no short-range split
        const int DT = K.dim_threads;
        k_dimers<<<(int)(((long)nq * 32 + DT - 1) / DT), DT, 0, st>>>(
            S.query, nq, S.members, c->d_tag.p, c->d_type.p, B.nb_count.p, B.nb.p, c->nb_cap, rc2, R, c->listed.p,
            list_cap > 0 ? c->list.p : nullptr, list_cap, c->buckets.p, c->bucket_count.p, c->status.p);
    } else {
        // a block per query (tunable threads); its matches staged in shared memory
        const size_t smem = (size_t)c->nb_cap * MBX_TRIMATCH_BYTES;
        if (smem > 227 * 1024) return fail(c, MBX_ENOMEM, "trimer staging exceeds shared memory");
        if (smem > 48 * 1024)
            CUCHK(c, cudaFuncSetAttribute(k_trimers, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_trimers<<<nq, K.tri_threads, smem, st>>>(
            S.query, nq, S.members, c->d_tag.p, c->d_type.p, B.cloud.p, B.nb_count.p, B.nb.p, c->nb_cap, rc2,
            c->trules, c->listed.p, list_cap > 0 ? c->list.p : nullptr, list_cap, c->buckets.p, c->bucket_count.p,
            c->status.p);
    }
    CUCHK(c, cudaGetLastError());
    *kernels += 8;
    return MBX_OK;
}

// The whole system as one search (members/queries of the ghost mode).
static int launch_build(mbx_ctx* c, int nbody, int use_ghost, const double* xyz, long list_cap, int* kernels,
                        bool mixed = false) {
    const int g = use_ghost ? 1 : 0;
    int r = prepare_buckets(c, nbody, c->nquery[g], list_cap);
    if (r) return r;
    BuildScope S{c->d_members[g].p, c->nmem[g], c->d_query[g].p, c->nquery[g], c->bp};
    return launch_build_scope(c, nbody, S, xyz, list_cap, kernels, mixed);
}

// The grids of a batched search for term nbody (BatchGrid per configuration,
// cells concatenated), uploaded when the batch or the cutoff changed.  The
// upload is synchronous, so it must not happen inside a graph capture; every
// capture follows a plain run of the same sequence, which leaves them fresh.
static int ensure_batch_grids(mbx_ctx* c, int nbody) {
    const double rc = c->cutoff[nbody];
    if (c->d_bgrid[nbody].p && c->bgrid_gen[nbody] == c->gen && c->bgrid_cut[nbody] == rc) return MBX_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    CUCHK(c, cudaStreamIsCapturing(c->stream, &cs));
    if (cs != cudaStreamCaptureStatusNone) return fail(c, MBX_EINVAL, "batch grids changed inside a graph capture");
    std::vector<BatchGrid> g(c->nconf);
    long ncell = 0;
    for (int k = 0; k < c->nconf; ++k) {
        g[k].bp = c->conf_bp[k];
        g[k].cg = make_grid(c->conf_bp[k], rc, std::max(c->conf_mon[k + 1] - c->conf_mon[k], 1));
        g[k].cell_off = (int)ncell;
        ncell += (long)g[k].cg.n[0] * g[k].cg.n[1] * g[k].cg.n[2];
    }
    if (ncell >= (1L << 30)) return fail(c, MBX_ENOMEM, "batched cell grid too large");
    CUCHK(c, c->d_bgrid[nbody].ensure(c->nconf));
    CUCHK(c, cudaMemcpy(c->d_bgrid[nbody].p, g.data(), c->nconf * sizeof(BatchGrid), cudaMemcpyHostToDevice));
    c->bgrid_ncell[nbody] = (int)ncell;
    c->bgrid_gen[nbody] = c->gen;
    c->bgrid_cut[nbody] = rc;
    return MBX_OK;
}

// A whole batch as one search: members and queries are the batch's monomers
// (the identity list of its all-local topology), each searching the cells of
// its own configuration (k_cloud_batch, k_neighbors_batch); the cell kernels
// run once over every configuration's cells, the dimer and trimer rules once
// over every query.  One launch per kernel for the batch, where a search per
// configuration took ~8 small launches each.
static int launch_build_batch(mbx_ctx* c, int nbody, const double* xyz, int* kernels, bool mixed) {
    int r = ensure_batch_grids(c, nbody);
    if (r) return r;
    BuildScratch& B = c->scratch;
    cudaStream_t st = c->stream;
    const int nmem = c->nmon, nq = c->nmon;
    if (nmem < 2 || (nbody == 3 && nmem < 3)) return MBX_OK;
    const double rc = c->cutoff[nbody];
    const double rc2 = rc * rc;
    const int ncell = c->bgrid_ncell[nbody];
    const int* ids = c->d_members[0].p;   // identity: member position = monomer = query
    CUCHK(c, B.cloud.ensure((size_t)nmem * 24));
    CUCHK(c, B.copy_dir.ensure(nmem));
    CUCHK(c, B.cell_of.ensure(nmem));
    CUCHK(c, B.cell_items.ensure(nmem));
    CUCHK(c, B.cell_sorted.ensure(nmem));
    CUCHK(c, B.cell_count.ensure(ncell + 1));
    CUCHK(c, B.cell_start.ensure(ncell + 1));
    CUCHK(c, B.cell_fill.ensure(ncell + 1));
    CUCHK(c, B.nb_count.ensure(nq));
    CUCHK(c, B.nb.ensure((size_t)nq * c->nb_cap));
    CUCHK(c, cudaMemsetAsync(B.cell_count.p, 0, (ncell + 1) * sizeof(int), st));
    const int T = 128;
    k_cloud_batch<<<(nmem + T - 1) / T, T, 0, st>>>(xyz, c->d_first.p, nmem, c->d_mon_conf.p, c->d_bgrid[nbody].p,
                                                    B.cloud.p, B.cell_of.p, B.copy_dir.p);
    k_cell_count<<<(nmem + T - 1) / T, T, 0, st>>>(B.cell_of.p, nmem, B.cell_count.p);
    k_cell_scan<<<1, 1024, 0, st>>>(B.cell_count.p, ncell, B.cell_start.p, B.cell_fill.p);
    k_cell_fill<<<(nmem + T - 1) / T, T, 0, st>>>(B.cell_of.p, nmem, B.cell_fill.p, B.cell_items.p);
    k_cell_sort<<<(int)(((long)ncell * 32 + T - 1) / T), T, 0, st>>>(B.cell_start.p, ncell, B.cell_items.p,
                                                                      B.cell_sorted.p);
    const auto& K = c->knobs[nbody];
    const int nbw = (size_t)4 * c->nb_cap * sizeof(NbEntry) <= 160 * 1024 ? K.nb_warps : 1;
    if ((size_t)c->nb_cap * sizeof(NbEntry) > 227 * 1024) return fail(c, MBX_ENOMEM, "neighbour staging");
    RCHK(c, launch_neighbors_batch(nbw, K.nb_unroll, B.cloud.p, B.copy_dir.p, B.cell_of.p, B.cell_start.p,
                                   B.cell_sorted.p, ids, nq,
                                   c->d_mon_conf.p, c->d_bgrid[nbody].p, rc2, c->nb_cap, B.nb_count.p, B.nb.p,
                                   c->status.p, st));
    if (nbody == 2) {
        DimerRules R = c->drules;
        if (!mixed)
            for (int b = 0; b < MBX_MAX_BUCKETS; ++b) R.split2[b] = 0.0;   // no short-range split
        const int DT = K.dim_threads;
        k_dimers<<<(int)(((long)nq * 32 + DT - 1) / DT), DT, 0, st>>>(
            ids, nq, ids, c->d_tag.p, c->d_type.p, B.nb_count.p, B.nb.p, c->nb_cap, rc2, R, c->listed.p, nullptr, 0,
            c->buckets.p, c->bucket_count.p, c->status.p);
    } else {
        const size_t smem = (size_t)c->nb_cap * MBX_TRIMATCH_BYTES;
        if (smem > 227 * 1024) return fail(c, MBX_ENOMEM, "trimer staging exceeds shared memory");
        if (smem > 48 * 1024)
            CUCHK(c, cudaFuncSetAttribute(k_trimers, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        k_trimers<<<nq, K.tri_threads, smem, st>>>(ids, nq, ids, c->d_tag.p, c->d_type.p, B.cloud.p, B.nb_count.p,
                                                    B.nb.p, c->nb_cap, rc2, c->trules, c->listed.p, nullptr, 0,
                                                    c->buckets.p, c->bucket_count.p, c->status.p);
    }
    CUCHK(c, cudaGetLastError());
    *kernels += 8;
    return MBX_OK;
}

static HolderArgs base_args(mbx_ctx* c) {
    HolderArgs A;
    memset(&A, 0, sizeof(A));
    A.bp = c->bp;
    return A;
}

// Term table and global-memory coefficients of evaluator E on the context's
// device, for the table-driven kernels.
static void table_args(mbx_ctx* c, const EvaluatorInfo* E, HolderArgs& A) {
    const TermTableInfo& T = mbx_term_tables[E->table];
    A.terms = reinterpret_cast<const int4*>(c->tables.blob + T.off_terms);
    A.tcoef = reinterpret_cast<const double*>(c->tables.blob + T.off_tcoef);
    A.nterms = T.nterms;
    if (!A.coef) A.coef = c->tables.coef + mbx_coef_offset(E->kern);
}

static int launch_eval(mbx_ctx* c, const EvaluatorInfo* E, HolderArgs A, int flags, int* kernels,
                       bool near = false) {
    const bool grads = !(flags & MBX_NO_GRADS);
    const bool mixed = (flags & MBX_MIXED) != 0;
    const int block = 128;
    if (E->w) {
        table_args(c, E, A);
        long nw = A.n;
        int grid = (int)std::min<long>((nw + 3) / 4, (long)c->sm_count * 8);
        RCHK(c, E->w(A, grads ? 1 : 0, std::max(grid, 1), c->stream));
        ++*kernels;
        return MBX_OK;
    }
    // mixed mode: the FP32-basis kernel where the type has one; FP64 for the
    // short-range bucket of a split type, for a split type's AoS input (no
    // builder to separate the short-range n-mers) and for types without one
    const bool fp32 = mixed && !near && E->s && !(A.aos && E->split_r > 0);
    launch_fn fn = !grads ? E->e : fp32 ? E->s : E->g;
    if (!fn) return fail(c, MBX_ENOTSUP, std::string("no kernel for ") + E->name);
    if (fn == E->s) {
        // scratch of the three mixed-precision kernels for up to A.n n-mers
        auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
        const long cap = std::max<long>(A.n, 1);
        const size_t vb = up((size_t)E->nvars * cap * sizeof(float));
        const size_t qb = 2 * vb;   // FP64 radial factors
        const size_t eb = up((size_t)cap * sizeof(double));
        CUCHK(c, c->pair_scratch.ensure(qb + 2 * vb + eb + up((size_t)cap)));
        unsigned char* base = c->pair_scratch.p;
        A.ps.q = reinterpret_cast<double*>(base);
        A.ps.dx = reinterpret_cast<float*>(base + qb);
        A.ps.g = reinterpret_cast<float*>(base + qb + vb);
        A.ps.ep = reinterpret_cast<double*>(base + qb + 2 * vb);
        A.ps.live = base + qb + 2 * vb + eb;
        A.ps.cap = cap;
        A.ps.err = c->status.p;   // status word: MBX_STATUS_WAIT_TIMEOUT
    }
    // persistent grid: a few resident blocks per SM, grid-stride over n-mers
    const long want = (A.n + block - 1) / block;
    const int grid = (int)std::max<long>(1, std::min<long>(want, (long)c->sm_count * 4));
    RCHK(c, fn(A, grid, block, c->stream));
    *kernels += fn == E->s ? 3 : 1;   // the mixed path is three kernels
    return MBX_OK;
}

// Code prefetch (holder_prime_kernel) of the evaluation kernels that a term's
// buckets will launch, forked from the context stream onto the prime stream
// so that it runs beside the n-mer search; prime_join marks its end and the
// first evaluation waits for it.  Same kernel choice as launch_eval.
static int launch_prime(mbx_ctx* c, int nbody, int flags, int* kernels) {
    const bool grads = !(flags & MBX_NO_GRADS);
    const bool mixed = (flags & MBX_MIXED) != 0;
    prime_fn done[MBX_MAX_BUCKETS];
    int ndone = 0;
    CUCHK(c, cudaEventRecord(c->prime_fork, c->stream));
    CUCHK(c, cudaStreamWaitEvent(c->prime_stream, c->prime_fork, 0));
    for (int b = 0; b < c->nbucket[nbody]; ++b) {
        const bool near = c->bucket_near[nbody][b];
        if (near && !mixed) continue;
        const EvaluatorInfo* E = c->bucket_eval[nbody][b];
        if (E->w) continue;
        const bool fp32 = mixed && !near && E->s;
        const prime_fn fn = !grads ? E->pe : fp32 ? E->ps : E->pg;
        if (!fn || std::find(done, done + ndone, fn) != done + ndone) continue;
        done[ndone++] = fn;
        RCHK(c, fn(c->prime_stream));
        ++*kernels;
    }
    CUCHK(c, cudaEventRecord(c->prime_join, c->prime_stream));
    return MBX_OK;
}

// Enqueues one term on the context's stream (n-mer build, evaluation, the
// results copied to pinned memory), on device coordinates X (already
// wrapped) accumulating into the device gradient G (NULL: energy only).
static int term_enqueue(mbx_ctx* c, int nbody, int use_ghost, double* X, double* G, int flags, int* kernels) {
    const bool grads = !(flags & MBX_NO_GRADS);
    const bool mixed = (flags & MBX_MIXED) && grads;
    CUCHK(c, cudaEventRecord(c->ev[0], c->stream));
    int r = launch_prime(c, nbody, flags, kernels);
    if (r) return r;
    r = launch_build(c, nbody, use_ghost, X, 0, kernels, mixed);
    if (r) return r;
    CUCHK(c, cudaStreamWaitEvent(c->stream, c->prime_join, 0));
    CUCHK(c, cudaEventRecord(c->ev[1], c->stream));
    CUCHK(c, cudaMemsetAsync(c->out.p, 0, 16 * sizeof(double), c->stream));
    CUCHK(c, cudaMemsetAsync(c->counters.p, 0, MBX_MAX_BUCKETS * sizeof(int), c->stream));
    long off = 0;
    for (int b = 0; b < c->nbucket[nbody]; ++b) {
        HolderArgs A = base_args(c);
        A.counter = c->counters.p + b;
        A.n = c->bucket_cap[nbody][b];
        A.n_dev = c->bucket_count.p + b;
        A.status = c->status.p;
        A.nmers = c->buckets.p + off;
        A.xyz = X;
        A.first_index = c->d_first.p;
        A.grad = grads ? G : nullptr;
        A.out = c->out.p;
        off += c->bucket_cap[nbody][b];
        if (c->bucket_near[nbody][b] && !mixed) continue;   // empty without the split
        r = launch_eval(c, c->bucket_eval[nbody][b], A, flags, kernels, c->bucket_near[nbody][b]);
        if (r) return r;
    }
    CUCHK(c, cudaEventRecord(c->ev[2], c->stream));
    // results: energy + virial, counters, status
    CUCHK(c, cudaMemcpyAsync(c->h_out, c->out.p, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUCHK(c, cudaMemcpyAsync(c->h_out + 8, c->listed.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             c->stream));
    CUCHK(c, cudaMemcpyAsync(c->h_out + MBX_H_COUNTS, c->bucket_count.p, MBX_MAX_BUCKETS * sizeof(int), cudaMemcpyDeviceToHost,
                             c->stream));
    CUCHK(c, cudaMemcpyAsync(c->h_out + MBX_H_STATUS, c->status.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    return MBX_OK;
}

// After the stream of a term_enqueue has completed: 1 when the build did not
// fit its buffers (capacities grown; the evaluators saw the status word and
// added nothing: enqueue again), a negative value when a kernel reported a
// timeout (error set), else 0 with the energy, the virial (+=), the counts
// and the timing recorded.
static int term_finish(mbx_ctx* c, int nbody, double* energy, double* virial, int kernels) {
    int status[2];
    memcpy(status, c->h_out + MBX_H_STATUS, sizeof(status));
    int counts[MBX_MAX_BUCKETS];
    memcpy(counts, c->h_out + MBX_H_COUNTS, sizeof(counts));
    if (status[0] & MBX_STATUS_WAIT_TIMEOUT)
        return -fail(c, MBX_ECUDA, "an evaluation kernel's barrier wait timed out (results discarded)");
    if (status[0]) {
        if (status[0] & MBX_STATUS_NB_OVERFLOW) c->nb_cap = std::max(c->nb_cap * 2, status[1] + 32);
        for (int b = 0; b < c->nbucket[nbody]; ++b)
            if (counts[b] > c->bucket_cap[nbody][b]) c->bucket_cap[nbody][b] = (long)(counts[b] * 1.25) + 1024;
        if ((status[0] & MBX_STATUS_BUCKET_OVERFLOW) && !(status[0] & MBX_STATUS_NB_OVERFLOW)) {
            for (int b = 0; b < c->nbucket[nbody]; ++b)
                if (counts[b] >= c->bucket_cap[nbody][b]) c->bucket_cap[nbody][b] *= 2;
        }
        return 1;
    }
    unsigned long long listed;
    memcpy(&listed, c->h_out + 8, sizeof(listed));
    c->last_listed[nbody] = (long)listed;
    long ev = 0;
    for (int b = 0; b < c->nbucket[nbody]; ++b) ev += counts[b];
    c->last_evaluated[nbody] = ev;
    cudaEventElapsedTime(&c->last_ms_build, c->ev[0], c->ev[1]);
    cudaEventElapsedTime(&c->last_ms_eval, c->ev[1], c->ev[2]);
    c->last_kernels = kernels;
    *energy = c->h_out[0];
    if (virial) {
        virial[0] += c->h_out[1];
        virial[1] += c->h_out[2];
        virial[2] += c->h_out[3];
        virial[4] += c->h_out[4];
        virial[5] += c->h_out[5];
        virial[8] += c->h_out[6];
        virial[3] = virial[1];
        virial[6] = virial[2];
        virial[7] = virial[5];
    }
    return 0;
}

// Coordinates on the device (staged from the host when needed) and wrapped
// (SetPBC: FixMonomerCoordinates on every call, system.cpp:741-744); the
// gradient accumulator on the device (the caller's when it is device memory).
static int stage_term_io(mbx_ctx* c, double* xyz, double* grad, int flags, double** X, double** G, int* kernels) {
    const bool dev = (flags & MBX_DEVICE_PTRS) != 0;
    const bool grads = !(flags & MBX_NO_GRADS);
    const size_t nx = 3 * (size_t)c->numsites;
    *X = xyz;
    if (!dev) {
        CUCHK(c, c->xyz.ensure(nx));
        CUCHK(c, cudaMemcpyAsync(c->xyz.p, xyz, nx * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        *X = c->xyz.p;
    }
    if (c->bp.use_pbc) {
        k_fix_monomers<<<(c->nmon + 127) / 128, 128, 0, c->stream>>>(*X, c->d_first.p, c->d_nat.p, c->nmon, c->bp);
        ++*kernels;
    }
    *G = nullptr;
    if (grads) {
        if (dev && grad) {
            *G = grad;  // accumulate straight into the caller's array
        } else {
            CUCHK(c, c->grad.ensure(nx));
            CUCHK(c, cudaMemsetAsync(c->grad.p, 0, nx * sizeof(double), c->stream));
            *G = c->grad.p;
        }
    }
    return MBX_OK;
}

// The device-to-host copies of a call with host arrays, enqueued on the
// context stream: the wrapped coordinates into the caller's array, the
// gradient into a pinned staging buffer of the context (a DMA copy, no
// allocation per call).
static int copy_term_outputs(mbx_ctx* c, double* xyz, double* grad, int flags, double* X, double* G) {
    const bool grads = !(flags & MBX_NO_GRADS);
    const size_t nx = 3 * (size_t)c->numsites;
    if (c->bp.use_pbc) CUCHK(c, cudaMemcpyAsync(xyz, X, nx * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (grads && grad) {
        if (c->h_grad_n < nx) {
            if (c->h_grad) CUCHK(c, cudaFreeHost(c->h_grad));
            c->h_grad = nullptr;
            c->h_grad_n = 0;
            CUCHK(c, cudaMallocHost(&c->h_grad, nx * sizeof(double)));
            c->h_grad_n = nx;
        }
        CUCHK(c, cudaMemcpyAsync(c->h_grad, G, nx * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    return MBX_OK;
}

// Host outputs of a call with host arrays: the wrapped coordinates and the
// gradient (+=) back into the caller's arrays.  copied: copy_term_outputs
// already ran behind the call's last kernels (and the stream was waited for).
static int unstage_term_io(mbx_ctx* c, double* xyz, double* grad, int flags, double* X, double* G,
                           bool copied = false) {
    const bool dev = (flags & MBX_DEVICE_PTRS) != 0;
    const bool grads = !(flags & MBX_NO_GRADS);
    const size_t nx = 3 * (size_t)c->numsites;
    if (dev) return MBX_OK;
    if (!copied) {
        int r = copy_term_outputs(c, xyz, grad, flags, X, G);
        if (r) return r;
        CUCHK(c, cudaStreamSynchronize(c->stream));
    }
    if (grads && grad) {
        const double* tmp = c->h_grad;
        for (size_t i = 0; i < nx; ++i) grad[i] += tmp[i];
    }
    return MBX_OK;
}

// Monomer types whose 1-body term the reference computes
// (e1b::get_1b_energy, potential/1b/energy1b.cpp:53-86) but that have no
// GPU evaluator here (water and CH4 have), and a topology holding them (and not
// ignoring them) gets MBX_ENOTSUP for the 1-body term rather than a silent
// zero.  Every other type has no 1-body term (0, as in the reference).
static const char* const k1bCpuOnly[] = {"co2_archive", "nh3", "nh3pbe0d3bj", "co2", "co2cm5100", "co2cm595",
                                         "co2cm590", "co2cm5875", "co2cm585", "co2cm580", "h2", "n2o5", "mbpbe"};

// System::Get1B (bblock/system.cpp:2269-2401) on device coordinates X
// (wrapped): the local waters through the Partridge-Schwenke kernel.
static int onebody_term(mbx_ctx* c, double* X, double* G, double* energy, double* virial, int* kernels) {
    auto ignored = [&](const std::string& t) {
        return std::find(c->ignore1b.begin(), c->ignore1b.end(), t) != c->ignore1b.end();
    };
    for (int t = 0; t < c->ntypes; ++t)
        for (const char* id : k1bCpuOnly)
            if (c->type_names[t] == id && !ignored(id))
                return fail(c, MBX_ENOTSUP, std::string("no GPU 1-body term for monomer type ") + id);
    if (c->w1b_gen != c->gen) {
        std::vector<int> first;
        for (int m = 0; m < c->nmon; ++m)
            if (c->type_names[c->h_type[m]] == "h2o" && c->h_local[m] && !ignored("h2o")) first.push_back(c->h_first[m]);
        c->n_w1b = (long)first.size();
        for (int i = 0; i < mbx_num_onebody; ++i) {
            const std::string id = mbx_onebody[i].mon;
            const size_t before = first.size();
            for (int m = 0; m < c->nmon; ++m)
                if (c->type_names[c->h_type[m]] == id && c->h_local[m] && !ignored(id)) first.push_back(c->h_first[m]);
            c->n1b[i] = (long)(first.size() - before);
        }
        CUCHK(c, c->d_w1b.ensure(std::max<size_t>(first.size(), 1)));
        if (!first.empty())
            CUCHK(c, cudaMemcpyAsync(c->d_w1b.p, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice,
                                     c->stream));
        CUCHK(c, cudaStreamSynchronize(c->stream));
        c->w1b_gen = c->gen;
    }
    CUCHK(c, cudaEventRecord(c->ev[1], c->stream));
    CUCHK(c, cudaMemsetAsync(c->out.p, 0, 8 * sizeof(double), c->stream));
    OneBodyArgs A{X, c->d_w1b.p, c->n_w1b, G, c->out.p};
    RCHK(c, mbx_launch_ps1b(A, c->sm_count, c->stream));
    if (c->n_w1b > 0) ++*kernels;
    long off = c->n_w1b, n1 = c->n_w1b;
    for (int i = 0; i < mbx_num_onebody; ++i) {
        if (c->n1b[i] > 0) {
            const TermTableInfo& T = mbx_term_tables[mbx_onebody[i].table];
            HolderArgs H = base_args(c);
            H.n = c->n1b[i];
            H.first_index = c->d_w1b.p + off;
            H.xyz = X;
            H.grad = G;
            H.out = c->out.p;
            H.terms = reinterpret_cast<const int4*>(c->tables.blob + T.off_terms);
            H.tcoef = reinterpret_cast<const double*>(c->tables.blob + T.off_tcoef);
            H.nterms = T.nterms;
            H.coef = c->tables.coef + g_coef_off_1b[i];
            RCHK(c, mbx_onebody[i].launch(H, 0, 128, c->stream));
            ++*kernels;
        }
        off += c->n1b[i];
        n1 += c->n1b[i];
    }
    CUCHK(c, cudaEventRecord(c->ev[2], c->stream));
    CUCHK(c, cudaMemcpyAsync(c->h_out, c->out.p, 7 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUCHK(c, cudaStreamSynchronize(c->stream));
    *energy = c->h_out[0];
    if (virial) {
        virial[0] += c->h_out[1];
        virial[1] += c->h_out[2];
        virial[2] += c->h_out[3];
        virial[4] += c->h_out[4];
        virial[5] += c->h_out[5];
        virial[8] += c->h_out[6];
        virial[3] = virial[1];
        virial[6] = virial[2];
        virial[7] = virial[5];
    }
    c->last_ms_build = 0;
    cudaEventElapsedTime(&c->last_ms_eval, c->ev[1], c->ev[2]);
    c->last_kernels = *kernels;
    c->last_listed[1] = c->last_evaluated[1] = n1;
    return MBX_OK;
}

// Input order <-> site order (System::SetRealXyz, bblock/system.cpp:830-846,
// and GetRealGrads): site of real atom i = real2site[i].
__global__ void k_gather_real(const double* __restrict__ xr, const int* __restrict__ real2site, int numat,
                              double* __restrict__ sites) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < numat; i += gridDim.x * blockDim.x) {
        const int s = real2site[i];
        sites[3 * s] = xr[3 * i];
        sites[3 * s + 1] = xr[3 * i + 1];
        sites[3 * s + 2] = xr[3 * i + 2];
    }
}

__global__ void k_scatter_real(const double* __restrict__ gsite, const int* __restrict__ real2site, int numat,
                               double* __restrict__ greal) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < numat; i += gridDim.x * blockDim.x) {
        const int s = real2site[i];
        greal[3 * i] += gsite[3 * s];
        greal[3 * i + 1] += gsite[3 * s + 1];
        greal[3 * i + 2] += gsite[3 * s + 2];
    }
}

extern "C" int mbx_set_real_order(mbx_ctx* c, int numat, const int* real2site) {
    if (!c || numat <= 0 || !real2site) return fail(c, MBX_EINVAL, "bad arguments");
    if (!c->nmon) return fail(c, MBX_EINVAL, "set the topology first");
    for (int i = 0; i < numat; ++i)
        if (real2site[i] < 0 || real2site[i] >= c->numsites) return fail(c, MBX_EINVAL, "site index out of range");
    CUCHK(c, cudaSetDevice(c->device));
    CUCHK(c, c->d_real2site.ensure(numat));
    CUCHK(c, cudaMemcpyAsync(c->d_real2site.p, real2site, numat * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    CUCHK(c, cudaStreamSynchronize(c->stream));
    c->numat = numat;
    return MBX_OK;
}

extern "C" int mbx_energy_real(mbx_ctx* c, int nbody, const double* xyz_real, int use_ghost, double* energy,
                               double* grad_real, double* virial, int flags) {
    if (!c || nbody < 1 || nbody > 3 || !xyz_real || !energy) return fail(c, MBX_EINVAL, "bad arguments");
    if (!c->numat) return fail(c, MBX_EINVAL, "no input order (mbx_set_real_order)");
    CUCHK(c, cudaSetDevice(c->device));
    const bool dev = (flags & MBX_DEVICE_PTRS) != 0;
    const bool grads = !(flags & MBX_NO_GRADS) && grad_real;
    const size_t na3 = 3 * (size_t)c->numat, ns3 = 3 * (size_t)c->numsites;
    const double* XR = xyz_real;
    if (!dev) {
        CUCHK(c, c->xreal.ensure(na3));
        CUCHK(c, cudaMemcpyAsync(c->xreal.p, xyz_real, na3 * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        XR = c->xreal.p;
    }
    CUCHK(c, c->xyz.ensure(ns3));
    const int grid = std::max(1, std::min((c->numat + 255) / 256, c->sm_count * 4));
    k_gather_real<<<grid, 256, 0, c->stream>>>(XR, c->d_real2site.p, c->numat, c->xyz.p);
    CUCHK(c, cudaGetLastError());
    if (grads) {
        CUCHK(c, c->gsite.ensure(ns3));
        CUCHK(c, cudaMemsetAsync(c->gsite.p, 0, ns3 * sizeof(double), c->stream));
    }
    // the term on the internal (device) site array; mbx_energy wraps it in place
    int r = mbx_energy(c, nbody, c->xyz.p, use_ghost, energy, grads ? c->gsite.p : nullptr, virial,
                       flags | MBX_DEVICE_PTRS | (grads ? 0 : MBX_NO_GRADS));
    if (r) return r;
    if (!grads) return MBX_OK;
    double* GR = grad_real;
    if (!dev) {
        CUCHK(c, c->greal.ensure(na3));
        CUCHK(c, cudaMemsetAsync(c->greal.p, 0, na3 * sizeof(double), c->stream));
        GR = c->greal.p;
    }
    k_scatter_real<<<grid, 256, 0, c->stream>>>(c->gsite.p, c->d_real2site.p, c->numat, GR);
    CUCHK(c, cudaGetLastError());
    if (!dev) {
        std::vector<double> h(na3);
        CUCHK(c, cudaMemcpyAsync(h.data(), GR, na3 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CUCHK(c, cudaStreamSynchronize(c->stream));
        for (size_t i = 0; i < na3; ++i) grad_real[i] += h[i];
    } else {
        CUCHK(c, cudaStreamSynchronize(c->stream));
    }
    return MBX_OK;
}

extern "C" int mbx_set_ignore_1b(mbx_ctx* c, int n, const char* const* ids) {
    if (!c || n < 0 || (n > 0 && !ids)) return fail(c, MBX_EINVAL, "bad arguments");
    c->ignore1b.clear();
    for (int i = 0; i < n; ++i) c->ignore1b.push_back(ids[i]);
    ++c->gen;
    return MBX_OK;
}

extern "C" int mbx_energy(mbx_ctx* c, int nbody, double* xyz, int use_ghost, double* energy, double* grad,
                          double* virial, int flags) {
    if (!c || nbody < 1 || nbody > 3 || !xyz || !energy) return fail(c, MBX_EINVAL, "bad arguments");
    if (!c->nmon) return fail(c, MBX_EINVAL, "System has not been initialized (no topology)");
    CUCHK(c, cudaSetDevice(c->device));
    int kernels = 0;
    double *X, *G;
    int r = stage_term_io(c, xyz, grad, flags, &X, &G, &kernels);
    if (r) return r;
    if (nbody == 1) {
        r = onebody_term(c, X, G, energy, virial, &kernels);
        if (r) return r;
        return unstage_term_io(c, xyz, grad, flags, X, G);
    }
    for (int attempt = 0; attempt < 4; ++attempt) {
        r = term_enqueue(c, nbody, use_ghost, X, G, flags, &kernels);
        if (r) return r;
        CUCHK(c, cudaStreamSynchronize(c->stream));
        const int f = term_finish(c, nbody, energy, virial, kernels);
        if (f < 0) return MBX_ECUDA;
        if (f == 0) return unstage_term_io(c, xyz, grad, flags, X, G);
        kernels = 0;
    }
    return fail(c, MBX_ECUDA, "n-mer buffers did not converge");
}

// The child context of mbx_energy_2b3b: the 2b term on its own stream and
// buffers, same topology, configuration and launch shapes as the parent
// (coefficients are per device, so shared already).
static int sync_child(mbx_ctx* c) {
    if (c->child && c->child_gen == c->gen) return MBX_OK;
    if (!c->child) {
        int r = mbx_create(&c->child, c->device, nullptr);
        if (r) return fail(c, r, "child context");
        // the 2b term's stream at the device's highest priority: the 3b
        // term is enqueued first and its tensor-core kernel takes whole SMs,
        // so at equal priority the 2b evaluation waits for SMs behind the
        // 3b kernels and ends the step; first pick of the SMs that free up
        // lets the two terms end closer together
        int lo = 0, hi = 0;
        cudaStream_t hs = nullptr;
        CUCHK(c, cudaDeviceGetStreamPriorityRange(&lo, &hi));
        CUCHK(c, cudaStreamCreateWithPriority(&hs, cudaStreamNonBlocking, hi));
        CUCHK(c, cudaStreamDestroy(c->child->stream));
        c->child->stream = hs;
    }
    mbx_ctx* k = c->child;
    std::vector<const char*> ids(c->nmon);
    for (int m = 0; m < c->nmon; ++m) ids[m] = c->type_names[c->h_type[m]].c_str();
    int r = mbx_set_topology(k, c->nmon, ids.data(), c->h_first.data(), c->h_tag.data(), c->h_local.data(),
                             c->numsites);
    if (r) return fail(c, r, std::string("child topology: ") + k->err);
    std::vector<const char*> i2, i3;
    for (auto& t : c->ignore[2]) for (auto& x : t) i2.push_back(x.c_str());
    for (auto& t : c->ignore[3]) for (auto& x : t) i3.push_back(x.c_str());
    r = mbx_set_config(k, c->cutoff[2], c->cutoff[3], c->bp.use_pbc ? c->bp.box : nullptr, (int)c->ignore[2].size(),
                       i2.data(), (int)c->ignore[3].size(), i3.data());
    if (r) return fail(c, r, std::string("child configuration: ") + k->err);
    for (int nb = 0; nb < 4; ++nb) k->knobs[nb] = c->knobs[nb];
    if (c->nconf) {
        std::vector<double> boxes(9 * (size_t)c->nconf);
        std::vector<int> has(c->nconf);
        for (int q = 0; q < c->nconf; ++q) {
            for (int i = 0; i < 9; ++i) boxes[9 * q + i] = c->conf_bp[q].box[i];
            has[q] = c->conf_bp[q].use_pbc;
        }
        r = mbx_set_batch(k, c->nconf, c->conf_mon.data(), boxes.data(), has.data());
        if (r) return fail(c, r, std::string("child batch: ") + k->err);
    }
    c->child_gen = c->gen;
    return MBX_OK;
}

extern "C" int mbx_energy_2b3b(mbx_ctx* c, double* xyz, int use_ghost, double* e2, double* e3, double* grad,
                               double* virial, int flags) {
    if (!c || !xyz || !e2 || !e3) return fail(c, MBX_EINVAL, "bad arguments");
    if (!c->nmon) return fail(c, MBX_EINVAL, "System has not been initialized (no topology)");
    CUCHK(c, cudaSetDevice(c->device));
    int r = sync_child(c);
    if (r) return r;
    mbx_ctx* k = c->child;
    int kernels = 0, kk = 0;
    double *X, *G;
    r = stage_term_io(c, xyz, grad, flags, &X, &G, &kernels);
    if (r) return r;
    // the 2b term on the child's stream once the coordinates are wrapped
    CUCHK(c, cudaEventRecord(c->ev_fork, c->stream));
    CUCHK(c, cudaStreamWaitEvent(k->stream, c->ev_fork, 0));
    r = term_enqueue(c, 3, use_ghost, X, G, flags, &kernels);
    if (r) return r;
    r = term_enqueue(k, 2, use_ghost, X, G, flags, &kk);
    if (r) return fail(c, r, std::string("2b term: ") + k->err);
    // host arrays: the output copies behind both terms, before the host
    // waits (redone below if a term has to run again)
    bool copied = false;
    if (!(flags & MBX_DEVICE_PTRS)) {
        CUCHK(c, cudaEventRecord(k->ev[2], k->stream));
        CUCHK(c, cudaStreamWaitEvent(c->stream, k->ev[2], 0));
        r = copy_term_outputs(c, xyz, grad, flags, X, G);
        if (r) return r;
        copied = true;
    }
    CUCHK(c, cudaStreamSynchronize(k->stream));
    CUCHK(c, cudaStreamSynchronize(c->stream));
    int again3 = term_finish(c, 3, e3, virial, kernels);
    int again2 = term_finish(k, 2, e2, virial, kk);
    if (again3 < 0) return MBX_ECUDA;
    if (again2 < 0) return fail(c, MBX_ECUDA, std::string("2b term: ") + k->err);
    // a term whose n-mers did not fit its buffers added nothing: run it again
    for (int attempt = 0; (again2 || again3) && attempt < 4; ++attempt) {
        copied = false;
        if (again3) {
            kernels = 0;
            r = term_enqueue(c, 3, use_ghost, X, G, flags, &kernels);
            if (r) return r;
        }
        if (again2) {
            CUCHK(c, cudaEventRecord(c->ev_fork, c->stream));
            CUCHK(c, cudaStreamWaitEvent(k->stream, c->ev_fork, 0));
            kk = 0;
            r = term_enqueue(k, 2, use_ghost, X, G, flags, &kk);
            if (r) return fail(c, r, std::string("2b term: ") + k->err);
        }
        CUCHK(c, cudaStreamSynchronize(k->stream));
        CUCHK(c, cudaStreamSynchronize(c->stream));
        if (again3) again3 = term_finish(c, 3, e3, virial, kernels);
        if (again2) again2 = term_finish(k, 2, e2, virial, kk);
        if (again3 < 0) return MBX_ECUDA;
        if (again2 < 0) return fail(c, MBX_ECUDA, std::string("2b term: ") + k->err);
    }
    if (again2 || again3) return fail(c, MBX_ECUDA, "n-mer buffers did not converge");
    c->last_listed[2] = k->last_listed[2];
    c->last_evaluated[2] = k->last_evaluated[2];
    c->last_kernels = kernels + kk;
    // the 2b term also waited for the wrap: make the caller's stream see its work
    CUCHK(c, cudaEventRecord(k->ev[2], k->stream));
    CUCHK(c, cudaStreamWaitEvent(c->stream, k->ev[2], 0));
    return unstage_term_io(c, xyz, grad, flags, X, G, copied);
}

extern "C" int mbx_last_counts(const mbx_ctx* c, int nbody, long* listed, long* evaluated) {
    if (!c || nbody < 1 || nbody > 3) return MBX_EINVAL;
    if (listed) *listed = c->last_listed[nbody];
    if (evaluated) *evaluated = c->last_evaluated[nbody];
    return MBX_OK;
}

extern "C" int mbx_last_timing(const mbx_ctx* c, double* ms_build, double* ms_eval, int* kernels) {
    if (!c) return MBX_EINVAL;
    if (ms_build) *ms_build = c->last_ms_build;
    if (ms_eval) *ms_eval = c->last_ms_eval;
    if (kernels) *kernels = c->last_kernels;
    return MBX_OK;
}

extern "C" int mbx_nmers(mbx_ctx* c, int nbody, double cutoff, const double* xyz, int use_ghost, long* out, long cap,
                         long* count) {
    if (!c || (nbody != 2 && nbody != 3) || !xyz || !count) return fail(c, MBX_EINVAL, "bad arguments");
    if (!c->nmon) return fail(c, MBX_EINVAL, "no topology");
    CUCHK(c, cudaSetDevice(c->device));
    const double saved = c->cutoff[nbody];
    c->cutoff[nbody] = cutoff;
    const size_t nx = 3 * (size_t)c->numsites;
    long list_cap = std::max<long>(1024, (long)c->nquery[use_ghost ? 1 : 0] * (nbody == 2 ? 64 : 1024));
    int rc = MBX_OK;
    for (int attempt = 0; attempt < 6; ++attempt) {
        int kernels = 0;
        CUCHK(c, c->xyz.ensure(nx));
        CUCHK(c, cudaMemcpyAsync(c->xyz.p, xyz, nx * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        rc = launch_build(c, nbody, use_ghost, c->xyz.p, list_cap, &kernels);
        if (rc) break;
        unsigned long long listed[2];
        int status[2];
        CUCHK(c, cudaMemcpyAsync(listed, c->listed.p, sizeof(listed), cudaMemcpyDeviceToHost, c->stream));
        CUCHK(c, cudaMemcpyAsync(status, c->status.p, sizeof(status), cudaMemcpyDeviceToHost, c->stream));
        CUCHK(c, cudaStreamSynchronize(c->stream));
        if (status[0] & MBX_STATUS_NB_OVERFLOW) {
            c->nb_cap = std::max(c->nb_cap * 2, status[1] + 32);
            continue;
        }
        if (status[0] & MBX_STATUS_BUCKET_OVERFLOW) {
            for (int b = 0; b < c->nbucket[nbody]; ++b) c->bucket_cap[nbody][b] *= 2;
            continue;
        }
        if ((long)listed[1] > list_cap) {
            list_cap = (long)listed[1] + 16;
            continue;
        }
        *count = (long)listed[0];
        const long n = std::min<long>(cap, (long)listed[0]);
        if (n > 0 && out) {
            std::vector<int4> tmp(n);
            CUCHK(c, cudaMemcpy(tmp.data(), c->list.p, n * sizeof(int4), cudaMemcpyDeviceToHost));
            for (long i = 0; i < n; ++i) {
                out[nbody * i] = tmp[i].x;
                out[nbody * i + 1] = tmp[i].y;
                if (nbody == 3) out[nbody * i + 2] = tmp[i].z;
            }
        }
        c->cutoff[nbody] = saved;
        return MBX_OK;
    }
    c->cutoff[nbody] = saved;
    return rc ? rc : fail(c, MBX_ECUDA, "n-mer list buffers did not converge");
}

// Copies an input array to the device when needed; returns the device pointer.
static int stage_in(mbx_ctx* c, DevBuf<double>& buf, const double* src, size_t n, bool dev, const double** dst) {
    if (dev || !src) {
        *dst = src;
        return MBX_OK;
    }
    CUCHK(c, buf.ensure(n));
    CUCHK(c, cudaMemcpyAsync(buf.p, src, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    *dst = buf.p;
    return MBX_OK;
}

extern "C" int mbx_evaluate(mbx_ctx* c, const char* name, long n, const double* xyz, double* grad, double* virial,
                            double* e_per, double* energy, int flags) {
    if (!c || !name || n < 0 || (n > 0 && !xyz)) return fail(c, MBX_EINVAL, "bad arguments");
    const EvaluatorInfo* E = find_evaluator(name);
    if (!E) return fail(c, MBX_ENOTSUP, std::string("unknown evaluator ") + name);
    CUCHK(c, cudaSetDevice(c->device));
    const bool dev = (flags & MBX_DEVICE_PTRS) != 0;
    const size_t nx = (size_t)n * E->nreal * 3;
    static thread_local DevBuf<double> in_buf, g_buf, e_buf;
    const double* X;
    int r = stage_in(c, in_buf, xyz, nx, dev, &X);
    if (r) return r;
    const bool grads = !(flags & MBX_NO_GRADS) && grad;
    double* G = nullptr;
    if (grads) {
        if (dev) G = grad;
        else {
            CUCHK(c, g_buf.ensure(nx));
            CUCHK(c, cudaMemsetAsync(g_buf.p, 0, nx * sizeof(double), c->stream));
            G = g_buf.p;
        }
    }
    double* EP = nullptr;
    if (e_per) {
        if (dev) EP = e_per;
        else {
            CUCHK(c, e_buf.ensure(std::max<long>(n, 1)));
            EP = e_buf.p;
        }
    }
    CUCHK(c, cudaMemsetAsync(c->out.p, 0, 16 * sizeof(double), c->stream));
    CUCHK(c, cudaMemsetAsync(c->counters.p, 0, sizeof(int), c->stream));
    HolderArgs A = base_args(c);
    A.counter = c->counters.p;
    A.bp.use_pbc = 0;
    A.n = n;
    A.aos = 1;
    A.xyz = X;
    A.grad = G;
    A.out = c->out.p;
    A.e_per = EP;
    int kernels = 0;
    CUCHK(c, cudaMemsetAsync(c->status.p, 0, sizeof(int), c->stream));
    CUCHK(c, cudaEventRecord(c->ev[1], c->stream));
    if (n > 0) {
        r = launch_eval(c, E, A, grads ? (flags & MBX_MIXED) : (flags | MBX_NO_GRADS), &kernels);
        if (r) return r;
    }
    CUCHK(c, cudaEventRecord(c->ev[2], c->stream));
    CUCHK(c, cudaMemcpyAsync(c->h_out, c->out.p, 8 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUCHK(c, cudaMemcpyAsync(c->h_out + MBX_H_STATUS, c->status.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    std::vector<double> gt, et;
    if (grads && !dev) {
        gt.resize(nx);
        CUCHK(c, cudaMemcpyAsync(gt.data(), G, nx * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    if (e_per && !dev && n > 0) CUCHK(c, cudaMemcpyAsync(e_per, EP, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CUCHK(c, cudaStreamSynchronize(c->stream));
    int status0;
    memcpy(&status0, c->h_out + MBX_H_STATUS, sizeof(int));
    if (status0 & MBX_STATUS_WAIT_TIMEOUT)
        return fail(c, MBX_ECUDA, "an evaluation kernel's barrier wait timed out (results discarded)");
    if (grads && !dev)
        for (size_t i = 0; i < nx; ++i) grad[i] += gt[i];
    c->last_ms_build = 0;
    cudaEventElapsedTime(&c->last_ms_eval, c->ev[1], c->ev[2]);
    c->last_kernels = kernels;
    if (energy) *energy = c->h_out[0];
    if (virial) {
        virial[0] += c->h_out[1];
        virial[1] += c->h_out[2];
        virial[2] += c->h_out[3];
        virial[4] += c->h_out[4];
        virial[5] += c->h_out[5];
        virial[8] += c->h_out[6];
        virial[3] = virial[1];
        virial[6] = virial[2];
        virial[7] = virial[5];
    }
    return MBX_OK;
}

extern "C" int mbx_evaluate_dcoef(mbx_ctx* c, const char* name, long n, const double* xyz, const double* w,
                                  double* out, int flags) {
    if (!c || !name || n < 0 || !out) return fail(c, MBX_EINVAL, "bad arguments");
    const EvaluatorInfo* E = find_evaluator(name);
    if (!E) return fail(c, MBX_ENOTSUP, std::string("unknown evaluator ") + name);
    if (!E->c) return fail(c, MBX_ENOTSUP, std::string("no coefficient adjoint for ") + name);
    CUCHK(c, cudaSetDevice(c->device));
    const bool dev = (flags & MBX_DEVICE_PTRS) != 0;
    const size_t nx = (size_t)n * E->nreal * 3;
    static thread_local DevBuf<double> in_buf, w_buf, o_buf;
    const double *X, *W;
    int r = stage_in(c, in_buf, xyz, nx, dev, &X);
    if (r) return r;
    r = stage_in(c, w_buf, w, (size_t)n, dev, &W);
    if (r) return r;
    double* O = out;
    if (!dev) {
        CUCHK(c, o_buf.ensure(E->ncoef));
        CUCHK(c, cudaMemsetAsync(o_buf.p, 0, E->ncoef * sizeof(double), c->stream));
        O = o_buf.p;
    }
    HolderArgs A = base_args(c);
    A.bp.use_pbc = 0;
    A.n = n;
    A.aos = 1;
    A.xyz = X;
    table_args(c, E, A);
    if (n > 0) {
        const int grid = (int)std::max<long>(1, std::min<long>((n + 127) / 128, (long)c->sm_count * 2));
        RCHK(c, E->c(A, W, O, grid, 128, c->stream));
    }
    if (!dev) {
        std::vector<double> tmp(E->ncoef);
        CUCHK(c, cudaMemcpyAsync(tmp.data(), O, E->ncoef * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        CUCHK(c, cudaStreamSynchronize(c->stream));
        for (int k = 0; k < E->ncoef; ++k) out[k] += tmp[k];
    }
    return MBX_OK;
}

extern "C" int mbx_qf_image(const char* name, const double* coef, long* image_bytes, int* nb, unsigned char* image,
                            float* colf, double* b0) {
    if (!name) return MBX_EINVAL;
    const EvaluatorInfo* E = find_evaluator(name);
    if (!E) return MBX_ENOTSUP;
    const char* kern = mbx_evaluators[E->kern].name;
    for (int i = 0; i < mbx_num_qf_types; ++i) {
        const QfInfo& Q = mbx_qf_types[i];
        if (strcmp(Q.name, kern) != 0) continue;
        if (image_bytes) *image_bytes = Q.image_bytes;
        if (nb) *nb = Q.nb;
        if (image && colf && b0) return Q.build(coef ? coef : E->fit, image, colf, b0);
        return MBX_OK;
    }
    return MBX_ENOTSUP;
}

extern "C" int mbx_poly(mbx_ctx* c, const char* name, long nd, const double* x, double* g, double* e, int flags) {
    if (!c || !name || nd < 0 || (nd > 0 && (!x || !e))) return fail(c, MBX_EINVAL, "bad arguments");
    const EvaluatorInfo* E = find_evaluator(name);
    if (!E) return fail(c, MBX_ENOTSUP, std::string("unknown evaluator ") + name);
    CUCHK(c, cudaSetDevice(c->device));
    const bool dev = (flags & MBX_DEVICE_PTRS) != 0;
    const size_t nv = (size_t)nd * E->nvars;
    static thread_local DevBuf<double> xb, gb, eb;
    const double* X;
    int r = stage_in(c, xb, x, nv, dev, &X);
    if (r) return r;
    double *G = g, *Ev = e;
    if (!dev) {
        CUCHK(c, gb.ensure(std::max<size_t>(nv, 1)));
        CUCHK(c, eb.ensure(std::max<long>(nd, 1)));
        G = g ? gb.p : nullptr;
        Ev = eb.p;
    }
    if (nd > 0) {
        HolderArgs A = base_args(c);
        table_args(c, E, A);
        RCHK(c, mbx_launch_poly_table(nd, E->nvars, X, G, Ev, A.terms, A.tcoef, A.nterms, A.coef,
                                      mbx_term_tables[E->table].pairs, c->sm_count, c->stream));
    }
    if (!dev && nd > 0) {
        CUCHK(c, cudaMemcpyAsync(e, Ev, nd * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        if (g) CUCHK(c, cudaMemcpyAsync(g, G, nv * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    }
    CUCHK(c, cudaStreamSynchronize(c->stream));
    return MBX_OK;
}

extern "C" int mbx_set_coefficients(mbx_ctx* c, const char* name, const double* a, int flags) {
    if (!c || !name) return fail(c, MBX_EINVAL, "bad arguments");
    const EvaluatorInfo* E = find_evaluator(name);
    if (!E) return fail(c, MBX_ENOTSUP, std::string("unknown evaluator ") + name);
    CUCHK(c, cudaSetDevice(c->device));
    const bool dev = a && (flags & MBX_DEVICE_PTRS);
    const EvaluatorInfo* K = &mbx_evaluators[E->kern];
    const double* src = a ? a : K->fit;
    // coefficients are per device: wait for all work on the device (any
    // context's) before changing them, under the device-state lock
    std::lock_guard<std::mutex> lock(mbx_device_mutex());
    CUCHK(c, cudaDeviceSynchronize());
    for (int v = 0; v < 7; ++v)
        if (K->set[v]) RCHK(c, K->set[v](src, dev ? 1 : 0, c->stream));
    CUCHK(c, cudaMemcpyAsync(c->tables.coef + mbx_coef_offset(E->kern), src, E->ncoef * sizeof(double),
                             dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, c->stream));
    CUCHK(c, cudaStreamSynchronize(c->stream));
    return MBX_OK;
}

// ---------------------------------------------------------------------------
// Batched configurations (no counterpart in the reference, which evaluates
// one System per call): the topology is the concatenation of nconf
// configurations, each with its own box; one n-mer build per configuration
// into shared buckets, then one evaluation launch per evaluator over all of
// them, energies and virials summed per configuration.

static void drop_graphs(mbx_ctx* c) {
    for (auto& gr : c->graph) {
        if (gr.exec) cudaGraphExecDestroy(gr.exec);
        gr = mbx_ctx::Graph{};
    }
}

extern "C" int mbx_set_batch(mbx_ctx* c, int nconf, const int* conf_mon, const double* boxes, const int* has_box) {
    if (!c || nconf <= 0 || !conf_mon) return fail(c, MBX_EINVAL, "bad batch");
    if (!c->nmon) return fail(c, MBX_EINVAL, "no topology");
    if (conf_mon[0] != 0 || conf_mon[nconf] != c->nmon) return fail(c, MBX_EINVAL, "batch does not cover the topology");
    for (int k = 0; k < nconf; ++k)
        if (conf_mon[k + 1] < conf_mon[k]) return fail(c, MBX_EINVAL, "configuration ranges out of order");
    for (int m = 0; m < c->nmon; ++m)
        if (!c->h_local[m]) return fail(c, MBX_EINVAL, "batches take local monomers only");
    CUCHK(c, cudaSetDevice(c->device));
    const double rc = std::max(c->cutoff[2], c->cutoff[3]);
    std::vector<BoxParams> bp(nconf);
    for (int k = 0; k < nconf; ++k) {
        const bool pbc = boxes && (!has_box || has_box[k]);
        int r = make_box(c, pbc ? boxes + 9 * k : nullptr, rc, &bp[k]);
        if (r) return r;
    }
    std::vector<int> mon_conf(c->nmon);
    for (int k = 0; k < nconf; ++k)
        for (int m = conf_mon[k]; m < conf_mon[k + 1]; ++m) mon_conf[m] = k;
    drop_graphs(c);
    ++c->gen;
    c->nconf = nconf;
    c->conf_mon.assign(conf_mon, conf_mon + nconf + 1);
    c->conf_bp = bp;
    CUCHK(c, c->d_conf_bp.ensure(nconf));
    CUCHK(c, c->d_mon_conf.ensure(c->nmon));
    CUCHK(c, c->conf_out.ensure(8 * (size_t)nconf));
    if (c->h_conf) CUCHK(c, cudaFreeHost(c->h_conf));
    c->h_conf = nullptr;
    CUCHK(c, cudaMallocHost(&c->h_conf, 8 * (size_t)nconf * sizeof(double)));
    CUCHK(c, cudaMemcpyAsync(c->d_conf_bp.p, bp.data(), nconf * sizeof(BoxParams), cudaMemcpyHostToDevice, c->stream));
    CUCHK(c, cudaMemcpyAsync(c->d_mon_conf.p, mon_conf.data(), c->nmon * sizeof(int), cudaMemcpyHostToDevice,
                             c->stream));
    CUCHK(c, cudaStreamSynchronize(c->stream));
    return MBX_OK;
}

// Everything one batched term does on the device, without a host
// synchronisation (so that it can be captured into a graph): wrap every
// configuration, build every configuration's n-mers, evaluate every bucket
// once, copy the per-configuration sums and the status back to pinned memory.
static int batch_wrap(mbx_ctx* c, double* X, int* kernels) {
    for (int k = 0; k < c->nconf; ++k) {
        const int b = c->conf_mon[k], n = c->conf_mon[k + 1] - b;
        if (n > 0 && c->conf_bp[k].use_pbc) {
            k_fix_monomers<<<(n + 127) / 128, 128, 0, c->stream>>>(X, c->d_first.p + b, c->d_nat.p + b, n,
                                                                   c->conf_bp[k]);
            ++*kernels;
        }
    }
    CUCHK(c, cudaGetLastError());
    return MBX_OK;
}

static int batch_sequence(mbx_ctx* c, int nbody, double* X, double* G, bool grads, bool mixed, int* kernels,
                          bool wrap = true) {
    if (wrap) {
        int rw = batch_wrap(c, X, kernels);
        if (rw) return rw;
    }
    int r = prepare_buckets(c, nbody, c->nmon, 0);
    if (r) return r;
    r = launch_prime(c, nbody, (mixed ? MBX_MIXED : 0) | (grads ? 0 : MBX_NO_GRADS), kernels);
    if (r) return r;
    // every configuration's search in one set of launches
    r = launch_build_batch(c, nbody, X, kernels, mixed);
    if (r) return r;
    CUCHK(c, cudaStreamWaitEvent(c->stream, c->prime_join, 0));
    CUCHK(c, cudaMemsetAsync(c->conf_out.p, 0, 8 * (size_t)c->nconf * sizeof(double), c->stream));
    CUCHK(c, cudaMemsetAsync(c->out.p, 0, 16 * sizeof(double), c->stream));
    CUCHK(c, cudaMemsetAsync(c->counters.p, 0, MBX_MAX_BUCKETS * sizeof(int), c->stream));
    long off = 0;
    for (int b = 0; b < c->nbucket[nbody]; ++b) {
        HolderArgs A = base_args(c);
        A.counter = c->counters.p + b;
        A.n = c->bucket_cap[nbody][b];
        A.n_dev = c->bucket_count.p + b;
        A.status = c->status.p;
        A.nmers = c->buckets.p + off;
        A.xyz = X;
        A.first_index = c->d_first.p;
        A.grad = G;
        A.out = c->out.p;
        A.conf_bp = c->d_conf_bp.p;
        A.mon_conf = c->d_mon_conf.p;
        A.conf_out = c->conf_out.p;
        off += c->bucket_cap[nbody][b];
        if (c->bucket_near[nbody][b] && !mixed) continue;
        r = launch_eval(c, c->bucket_eval[nbody][b], A, (mixed ? MBX_MIXED : 0) | (grads ? 0 : MBX_NO_GRADS),
                        kernels, c->bucket_near[nbody][b]);
        if (r) return r;
    }
    CUCHK(c, cudaMemcpyAsync(c->h_conf, c->conf_out.p, 8 * (size_t)c->nconf * sizeof(double), cudaMemcpyDeviceToHost,
                             c->stream));
    CUCHK(c, cudaMemcpyAsync(c->h_out + 8, c->listed.p, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             c->stream));
    CUCHK(c, cudaMemcpyAsync(c->h_out + MBX_H_COUNTS, c->bucket_count.p, MBX_MAX_BUCKETS * sizeof(int), cudaMemcpyDeviceToHost,
                             c->stream));
    CUCHK(c, cudaMemcpyAsync(c->h_out + MBX_H_STATUS, c->status.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    return MBX_OK;
}

// After a sequence: 0 when the build fit its buffers (counts recorded), a
// negative value when a kernel reported a timeout (error set), else the
// capacities are grown and 1 is returned (run it again).
static int batch_check(mbx_ctx* c, int nbody) {
    int status[2];
    memcpy(status, c->h_out + MBX_H_STATUS, sizeof(status));
    int counts[MBX_MAX_BUCKETS];
    memcpy(counts, c->h_out + MBX_H_COUNTS, sizeof(counts));
    if (status[0] & MBX_STATUS_WAIT_TIMEOUT)
        return -fail(c, MBX_ECUDA, "an evaluation kernel's barrier wait timed out (results discarded)");
    if (status[0]) {
        if (status[0] & MBX_STATUS_NB_OVERFLOW) c->nb_cap = std::max(c->nb_cap * 2, status[1] + 32);
        for (int b = 0; b < c->nbucket[nbody]; ++b) {
            if (counts[b] > c->bucket_cap[nbody][b]) c->bucket_cap[nbody][b] = (long)(counts[b] * 1.25) + 1024;
            else if ((status[0] & MBX_STATUS_BUCKET_OVERFLOW) && counts[b] >= c->bucket_cap[nbody][b])
                c->bucket_cap[nbody][b] *= 2;
        }
        return 1;
    }
    unsigned long long listed;
    memcpy(&listed, c->h_out + 8, sizeof(listed));
    c->last_listed[nbody] = (long)listed;
    long ev = 0;
    for (int b = 0; b < c->nbucket[nbody]; ++b) ev += counts[b];
    c->last_evaluated[nbody] = ev;
    return 0;
}

extern "C" int mbx_batch_energy(mbx_ctx* c, int nbody, double* xyz, double* grad, double* energies, double* virials,
                                int flags) {
    if (!c || (nbody != 2 && nbody != 3) || !xyz || !energies) return fail(c, MBX_EINVAL, "bad arguments");
    if (!c->nconf) return fail(c, MBX_EINVAL, "no batch (mbx_set_batch)");
    if (!(flags & MBX_DEVICE_PTRS)) return fail(c, MBX_EINVAL, "batches take device arrays (MBX_DEVICE_PTRS)");
    CUCHK(c, cudaSetDevice(c->device));
    const bool grads = !(flags & MBX_NO_GRADS) && grad;
    const bool mixed = (flags & MBX_MIXED) && grads;
    const int key = flags & (MBX_MIXED | MBX_NO_GRADS);
    auto& gr = c->graph[nbody];
    int kernels = 0;
    bool done = false;
    CUCHK(c, cudaEventRecord(c->ev[0], c->stream));
    if ((flags & MBX_GRAPH) && gr.exec && gr.xyz == xyz && gr.grad == grad && gr.flags == key &&
        gr.gen == g_realloc_gen.load()) {
        CUCHK(c, cudaGraphLaunch(gr.exec, c->stream));
        CUCHK(c, cudaEventRecord(c->ev[2], c->stream));
        CUCHK(c, cudaStreamSynchronize(c->stream));
        const int f = batch_check(c, nbody);
        if (f < 0) return MBX_ECUDA;
        if (f == 0) {
            done = true;
            kernels = 1;
        } else {
            drop_graphs(c);   // buffers grow: capture again after a plain run
        }
    }
    if (!done) {
        for (int attempt = 0;; ++attempt) {
            if (attempt == 4) return fail(c, MBX_ENOMEM, "batch buffers kept overflowing");
            kernels = 0;
            CUCHK(c, cudaEventRecord(c->ev[0], c->stream));
            int r = batch_sequence(c, nbody, xyz, grads ? grad : nullptr, grads, mixed, &kernels);
            if (r) return r;
            CUCHK(c, cudaEventRecord(c->ev[2], c->stream));
            CUCHK(c, cudaStreamSynchronize(c->stream));
            const int f = batch_check(c, nbody);
            if (f < 0) return MBX_ECUDA;
            if (f == 0) break;
            // the failed pass added nothing (the evaluators saw the status
            // word), so it can simply run again with the larger buffers
        }
        if (flags & MBX_GRAPH) {
            // capture the same sequence for the next calls
            if (gr.exec) cudaGraphExecDestroy(gr.exec);
            gr = mbx_ctx::Graph{};
            cudaGraph_t g = nullptr;
            int dummy = 0;
            CUCHK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
            const unsigned long gen = g_realloc_gen.load();
            int r = batch_sequence(c, nbody, xyz, grads ? grad : nullptr, grads, mixed, &dummy);
            cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            if (r) {
                if (g) cudaGraphDestroy(g);
                return r;
            }
            if (e != cudaSuccess) return fail(c, MBX_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            if (gen != g_realloc_gen.load()) {
                cudaGraphDestroy(g);   // a buffer moved while capturing: next call captures again
            } else {
                e = cudaGraphInstantiate(&gr.exec, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return fail(c, MBX_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
                gr.xyz = xyz;
                gr.grad = grad;
                gr.flags = key;
                gr.gen = gen;
            }
        }
    }
    for (int k = 0; k < c->nconf; ++k) {
        const double* o = c->h_conf + 8 * k;
        energies[k] = o[0];
        if (virials) {
            double* v = virials + 9 * k;
            v[0] += o[1]; v[1] += o[2]; v[2] += o[3];
            v[3] += o[2]; v[4] += o[4]; v[5] += o[5];
            v[6] += o[3]; v[7] += o[5]; v[8] += o[6];
        }
    }
    c->last_ms_build = 0;
    cudaEventElapsedTime(&c->last_ms_eval, c->ev[0], c->ev[2]);
    c->last_kernels = kernels;
    return MBX_OK;
}

// Launch shapes of the builder for one term, chosen by timing the term on the
// caller's batch (or the whole system when no batch is set): coordinate
// descent over the warps per neighbour query and its unroll depth, the
// threads of the trimer pair loop ("trimers per block") and of the dimer
// rules.  out[4] (optional) receives the choice: nb_warps, nb_unroll,
// tri_threads, dim_threads; *best_ms the time.
extern "C" int mbx_tune(mbx_ctx* c, int nbody, double* xyz, double* grad, int flags, int* out, double* best_ms) {
    if (!c || (nbody != 2 && nbody != 3) || !xyz) return fail(c, MBX_EINVAL, "bad arguments");
    if (!(flags & MBX_DEVICE_PTRS)) return fail(c, MBX_EINVAL, "tuning takes device arrays (MBX_DEVICE_PTRS)");
    const int reps = 3;
    auto time_once = [&](double* ms) -> int {
        double e0 = 0.0;
        std::vector<double> e(std::max(c->nconf, 1));
        float best = 1e30f;
        for (int r = 0; r <= reps; ++r) {   // first pass untimed (sizes buffers, loads code)
            int rc = c->nconf ? mbx_batch_energy(c, nbody, xyz, grad, e.data(), nullptr, flags & ~MBX_GRAPH)
                              : mbx_energy(c, nbody, xyz, 0, &e0, grad, nullptr, flags);
            if (rc) return rc;
            const float t = c->nconf ? c->last_ms_eval : c->last_ms_build + c->last_ms_eval;
            if (r > 0) best = std::min(best, t);
        }
        *ms = best;
        return MBX_OK;
    };
    auto& K = c->knobs[nbody];
    double cur;
    int rc = time_once(&cur);
    if (rc) return rc;
    struct Axis { int* field; std::vector<int> values; };
    std::vector<Axis> axes = {{&K.nb_warps, {4, 1}}, {&K.nb_unroll, {1, 2, 4}}};
    if (nbody == 3) axes.push_back({&K.tri_threads, {64, 128, 256}});
    else axes.push_back({&K.dim_threads, {64, 128, 256}});
    for (auto& ax : axes) {
        const int keep = *ax.field;
        int best_v = keep;
        for (int v : ax.values) {
            if (v == keep) continue;
            *ax.field = v;
            double t;
            rc = time_once(&t);
            if (rc) {
                *ax.field = keep;
                return rc;
            }
            if (t < cur * 0.98) {   // a clear gain only
                cur = t;
                best_v = v;
            }
        }
        *ax.field = best_v;
    }
    drop_graphs(c);
    ++c->gen;
    if (out) {
        out[0] = K.nb_warps;
        out[1] = K.nb_unroll;
        out[2] = K.tri_threads;
        out[3] = K.dim_threads;
    }
    if (best_ms) *best_ms = cur;
    return MBX_OK;
}

extern "C" int mbx_get_knobs(const mbx_ctx* c, int nbody, int* out) {
    if (!c || (nbody != 2 && nbody != 3) || !out) return MBX_EINVAL;
    const auto& K = c->knobs[nbody];
    out[0] = K.nb_warps;
    out[1] = K.nb_unroll;
    out[2] = K.tri_threads;
    out[3] = K.dim_threads;
    return MBX_OK;
}

extern "C" int mbx_set_knobs(mbx_ctx* c, int nbody, const int* in) {
    if (!c || (nbody != 2 && nbody != 3) || !in) return fail(c, MBX_EINVAL, "bad arguments");
    const bool ok = (in[0] == 1 || in[0] == 4) && (in[1] == 1 || in[1] == 2 || in[1] == 4) &&
                    (in[2] == 64 || in[2] == 128 || in[2] == 256) && (in[3] == 64 || in[3] == 128 || in[3] == 256);
    if (!ok) return fail(c, MBX_EINVAL, "launch shape out of range");
    auto& K = c->knobs[nbody];
    K.nb_warps = in[0];
    K.nb_unroll = in[1];
    K.tri_threads = in[2];
    K.dim_threads = in[3];
    drop_graphs(c);
    ++c->gen;
    return MBX_OK;
}

// Both terms of every configuration of the batch, side by side: the 3b term
// on this context's stream, the 2b term on the child's (a mirror of the
// batch), the coordinates wrapped once before they fork.  With MBX_GRAPH the
// two streams' work is captured into one graph.
static int batch_enqueue_2b3b(mbx_ctx* c, double* X, double* G, bool grads, bool mixed, bool run3, bool run2,
                              int* kernels) {
    mbx_ctx* k = c->child;
    int r = batch_wrap(c, X, kernels);
    if (r) return r;
    if (run2) {
        CUCHK(c, cudaEventRecord(c->ev_fork, c->stream));
        CUCHK(c, cudaStreamWaitEvent(k->stream, c->ev_fork, 0));
    }
    if (run3) {
        r = batch_sequence(c, 3, X, G, grads, mixed, kernels, false);
        if (r) return r;
    }
    if (run2) {
        r = batch_sequence(k, 2, X, G, grads, mixed, kernels, false);
        if (r) return fail(c, r, std::string("2b term: ") + k->err);
        CUCHK(c, cudaEventRecord(k->ev_fork, k->stream));
        CUCHK(c, cudaStreamWaitEvent(c->stream, k->ev_fork, 0));
    }
    return MBX_OK;
}

extern "C" int mbx_batch_energy_2b3b(mbx_ctx* c, double* xyz, double* grad, double* e2, double* e3,
                                     double* virials, int flags) {
    if (!c || !xyz || !e2 || !e3) return fail(c, MBX_EINVAL, "bad arguments");
    if (!c->nconf) return fail(c, MBX_EINVAL, "no batch (mbx_set_batch)");
    if (!(flags & MBX_DEVICE_PTRS)) return fail(c, MBX_EINVAL, "batches take device arrays (MBX_DEVICE_PTRS)");
    CUCHK(c, cudaSetDevice(c->device));
    int r = sync_child(c);
    if (r) return r;
    mbx_ctx* k = c->child;
    const bool grads = !(flags & MBX_NO_GRADS) && grad;
    const bool mixed = (flags & MBX_MIXED) && grads;
    double* G = grads ? grad : nullptr;
    const int key = (flags & (MBX_MIXED | MBX_NO_GRADS)) | 0x100;
    auto& gr = c->graph[0];
    int kernels = 0;
    bool need3 = true, need2 = true;
    CUCHK(c, cudaEventRecord(c->ev[0], c->stream));
    if ((flags & MBX_GRAPH) && gr.exec && gr.xyz == xyz && gr.grad == grad && gr.flags == key &&
        gr.gen == g_realloc_gen.load()) {
        CUCHK(c, cudaGraphLaunch(gr.exec, c->stream));
        CUCHK(c, cudaEventRecord(c->ev[2], c->stream));
        CUCHK(c, cudaStreamSynchronize(c->stream));
        kernels = 1;
        const int f3 = batch_check(c, 3), f2 = batch_check(k, 2);
        if (f3 < 0) return MBX_ECUDA;
        if (f2 < 0) return fail(c, MBX_ECUDA, std::string("2b term: ") + k->err);
        need3 = f3 != 0;
        need2 = f2 != 0;
        if (need3 || need2) drop_graphs(c);   // buffers grow: capture again after a plain run
    }
    if (need3 || need2) {
        // a term whose n-mers did not fit added nothing: (re)run only such terms
        for (int attempt = 0; need3 || need2; ++attempt) {
            if (attempt == 4) return fail(c, MBX_ENOMEM, "batch buffers kept overflowing");
            CUCHK(c, cudaEventRecord(c->ev[0], c->stream));
            r = batch_enqueue_2b3b(c, xyz, G, grads, mixed, need3, need2, &kernels);
            if (r) return r;
            CUCHK(c, cudaEventRecord(c->ev[2], c->stream));
            CUCHK(c, cudaStreamSynchronize(c->stream));
            const int f3 = need3 ? batch_check(c, 3) : 0, f2 = need2 ? batch_check(k, 2) : 0;
            if (f3 < 0) return MBX_ECUDA;
            if (f2 < 0) return fail(c, MBX_ECUDA, std::string("2b term: ") + k->err);
            need3 = f3 != 0;
            need2 = f2 != 0;
        }
        if (flags & MBX_GRAPH) {
            if (gr.exec) cudaGraphExecDestroy(gr.exec);
            gr = mbx_ctx::Graph{};
            cudaGraph_t g = nullptr;
            int dummy = 0;
            CUCHK(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
            const unsigned long gen = g_realloc_gen.load();
            r = batch_enqueue_2b3b(c, xyz, G, grads, mixed, true, true, &dummy);
            cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            if (r) {
                if (g) cudaGraphDestroy(g);
                return r;
            }
            if (e != cudaSuccess) return fail(c, MBX_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
            if (gen != g_realloc_gen.load()) {
                cudaGraphDestroy(g);
            } else {
                e = cudaGraphInstantiate(&gr.exec, g, 0);
                cudaGraphDestroy(g);
                if (e != cudaSuccess) return fail(c, MBX_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
                gr.xyz = xyz;
                gr.grad = grad;
                gr.flags = key;
                gr.gen = gen;
            }
        }
    }
    for (int q = 0; q < c->nconf; ++q) {
        const double* o3 = c->h_conf + 8 * q;
        const double* o2 = k->h_conf + 8 * q;
        e3[q] = o3[0];
        e2[q] = o2[0];
        if (virials) {
            double* v = virials + 9 * q;
            const double s1 = o2[1] + o3[1], s2 = o2[2] + o3[2], s3 = o2[3] + o3[3];
            const double s4 = o2[4] + o3[4], s5 = o2[5] + o3[5], s6 = o2[6] + o3[6];
            v[0] += s1; v[1] += s2; v[2] += s3;
            v[3] += s2; v[4] += s4; v[5] += s5;
            v[6] += s3; v[7] += s5; v[8] += s6;
        }
    }
    c->last_listed[2] = k->last_listed[2];
    c->last_evaluated[2] = k->last_evaluated[2];
    c->last_ms_build = 0;
    cudaEventElapsedTime(&c->last_ms_eval, c->ev[0], c->ev[2]);
    c->last_kernels = kernels;
    return MBX_OK;
}
